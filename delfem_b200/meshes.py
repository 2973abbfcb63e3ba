"""Deterministic structured meshes for the solver configurations.

Every generator returns a :class:`Mesh` with 0-based node numbers.  The node
numbering is the "natural" ordering the reference's ILU(0) sees: the reference
applies no reordering unless ``CPreconditioner_ILU::SetOrdering`` is called
(include/delfem/ls/preconditioner.h:62-64), so the level sets of the triangular
solves follow directly from these numbers.

* :func:`unit_square_tri` - the (n+1)^2 grid, each cell split along its
  (i,j)->(i+1,j+1) diagonal: node p gets triangles {p, p+1, p+n+2} and
  {p, p+n+2, p+n+1}.
* :func:`box_tet` - an nx*ny*nz hexahedral grid, each hex split into 6 Kuhn
  tetrahedra around its v0-v6 diagonal, all positively oriented.
* :func:`unit_disk_tri` - concentric rings (ring k has 6k nodes) triangulated
  ring to ring, with the circle as boundary bars.
"""
from __future__ import annotations

import dataclasses

import numpy as np


@dataclasses.dataclass
class Mesh:
    coord: np.ndarray          # float64 [nnode, ndim]
    elem: np.ndarray           # int32 [nelem, nnoel]  (3 = TRI, 4 = TET)
    bnd: np.ndarray            # int32 [nbnd, bnd_nnoel] (2 = BAR, 3 = TRI); Dirichlet / absorbing
    extra: dict = dataclasses.field(default_factory=dict)

    @property
    def ndim(self) -> int:
        return int(self.coord.shape[1])

    @property
    def nnode(self) -> int:
        return int(self.coord.shape[0])

    @property
    def nnoel(self) -> int:
        return int(self.elem.shape[1])


def unit_square_tri(n: int, bnd: str = "all") -> Mesh:
    """(n+1)^2 nodes on [0,1]^2, 2 n^2 P1 triangles.

    ``bnd`` selects the boundary bars: "all" (4 sides), "left" (x = 0),
    "right" (x = 1) or "none".  Bars on the right edge are also returned in
    ``extra["right"]`` for traction loads.
    """
    m = n + 1
    ii, jj = np.meshgrid(np.arange(m), np.arange(m), indexing="xy")
    coord = np.stack([ii.ravel() / n, jj.ravel() / n], axis=1).astype(np.float64)
    ci, cj = np.meshgrid(np.arange(n), np.arange(n), indexing="xy")
    p = (ci + cj * m).ravel()
    t0 = np.stack([p, p + 1, p + m + 1], axis=1)
    t1 = np.stack([p, p + m + 1, p + m], axis=1)
    elem = np.empty((2 * n * n, 3), dtype=np.int32)
    elem[0::2] = t0
    elem[1::2] = t1
    k = np.arange(n)
    bottom = np.stack([k, k + 1], axis=1)
    right = np.stack([n + k * m, n + (k + 1) * m], axis=1)
    top = np.stack([n * m + n - k, n * m + n - k - 1], axis=1)
    left = np.stack([(n - k) * m, (n - k - 1) * m], axis=1)
    sides = {"bottom": bottom, "right": right, "top": top, "left": left}
    if bnd == "all":
        b = np.concatenate([bottom, right, top, left])
    elif bnd == "none":
        b = np.zeros((0, 2), dtype=np.int32)
    else:
        b = sides[bnd]
    return Mesh(coord, elem, b.astype(np.int32), {"right": right.astype(np.int32), "sides": sides})


# Kuhn subdivision of the unit cube around the v0-v6 diagonal.  Hex corners:
# v0=(0,0,0) v1=(1,0,0) v2=(1,1,0) v3=(0,1,0) v4=(0,0,1) v5=(1,0,1) v6=(1,1,1) v7=(0,1,1).
_KUHN = [(0, 1, 2, 6), (0, 2, 3, 6), (0, 3, 7, 6), (0, 7, 4, 6), (0, 4, 5, 6), (0, 5, 1, 6)]
_HEX = [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)]


def box_tet(nx: int, ny: int, nz: int, lx: float = 1.0, ly: float = 0.2, lz: float = 0.2) -> Mesh:
    """(nx+1)(ny+1)(nz+1) nodes (x fastest), 6 nx ny nz tetrahedra; the x = 0
    face (2 ny nz triangles) is the boundary array (clamped)."""
    mx, my, mz = nx + 1, ny + 1, nz + 1
    i, j, k = np.meshgrid(np.arange(mx), np.arange(my), np.arange(mz), indexing="ij")
    idx = lambda a, b, c: a + mx * (b + my * c)  # noqa: E731
    coord = np.zeros((mx * my * mz, 3))
    n = idx(i, j, k).ravel()
    coord[n, 0] = (i.ravel() / nx) * lx
    coord[n, 1] = (j.ravel() / ny) * ly
    coord[n, 2] = (k.ravel() / nz) * lz
    ci, cj, ck = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    # element order: cells in node order of their v0 (x fastest), 6 tets per cell
    order = np.argsort(idx(ci, cj, ck).ravel(), kind="stable")
    ci, cj, ck = ci.ravel()[order], cj.ravel()[order], ck.ravel()[order]
    corners = [idx(ci + dx, cj + dy, ck + dz) for (dx, dy, dz) in _HEX]
    tets = []
    for t in _KUHN:
        tet = np.stack([corners[v] for v in t], axis=1)
        tets.append(tet)
    elem = np.stack(tets, axis=1).reshape(-1, 4).astype(np.int32)
    # orient positively
    p = coord[elem]
    vol = np.einsum("ij,ij->i", p[:, 1] - p[:, 0], np.cross(p[:, 2] - p[:, 0], p[:, 3] - p[:, 0]))
    neg = vol < 0
    elem[neg, 1], elem[neg, 2] = elem[neg, 2].copy(), elem[neg, 1].copy()
    # x = 0 face
    fj, fk = np.meshgrid(np.arange(ny), np.arange(nz), indexing="ij")
    fj, fk = fj.ravel(), fk.ravel()
    a, b_, c, d = idx(0, fj, fk), idx(0, fj + 1, fk), idx(0, fj + 1, fk + 1), idx(0, fj, fk + 1)
    bnd = np.concatenate([np.stack([a, d, c], 1), np.stack([a, c, b_], 1)]).astype(np.int32)
    return Mesh(coord, elem, bnd)


def unit_disk_tri(nring: int, numbering: str = "rings") -> Mesh:
    """Unit disk: centre node plus rings k = 1..nring of 6k nodes at radius
    k/nring; 6 nring^2 triangles; the outer circle as 6 nring bars.

    numbering "rings": centre, then ring by ring in angle order.  Every node of
    a ring is adjacent to the one before it and a ring's first node to the
    previous ring's last, so the lower triangle of the natural ordering is one
    chain: ILU(0) level depth = nnode (fully sequential sweeps).
    numbering "bands": the same nodes and triangles renumbered row-major in
    horizontal bands one ring spacing high (by band, then x), like a
    structured grid: level depth O(nring)."""
    starts = [0, 1]
    for k in range(1, nring + 1):
        starts.append(starts[-1] + 6 * k)
    nnode = starts[-1]
    coord = np.zeros((nnode, 2))
    for k in range(1, nring + 1):
        m = 6 * k
        th = 2.0 * np.pi * np.arange(m) / m
        coord[starts[k]:starts[k] + m, 0] = (k / nring) * np.cos(th)
        coord[starts[k]:starts[k] + m, 1] = (k / nring) * np.sin(th)
    tris = []
    for k in range(1, nring + 1):
        m1 = 6 * k
        o1 = starts[k]
        if k == 1:
            for j in range(m1):
                tris.append((0, o1 + j, o1 + (j + 1) % m1))
            continue
        m0 = 6 * (k - 1)
        o0 = starts[k - 1]
        a0, a1 = 0, 0
        while a0 < m0 or a1 < m1:
            # advance the ring whose next node has the smaller angle
            t0 = (a0 + 1) / m0 if a0 < m0 else 2.0
            t1 = (a1 + 1) / m1 if a1 < m1 else 2.0
            if t1 <= t0:
                tris.append((o0 + a0 % m0, o1 + a1 % m1, o1 + (a1 + 1) % m1))
                a1 += 1
            else:
                tris.append((o0 + a0 % m0, o1 + a1 % m1, o0 + (a0 + 1) % m0))
                a0 += 1
    elem = np.asarray(tris, dtype=np.int32)
    p = coord[elem]
    area = (p[:, 1, 0] - p[:, 0, 0]) * (p[:, 2, 1] - p[:, 0, 1]) - (p[:, 2, 0] - p[:, 0, 0]) * (p[:, 1, 1] - p[:, 0, 1])
    neg = area < 0
    elem[neg, 1], elem[neg, 2] = elem[neg, 2].copy(), elem[neg, 1].copy()
    o = starts[nring]
    m = 6 * nring
    bnd = np.stack([o + np.arange(m), o + (np.arange(m) + 1) % m], axis=1).astype(np.int32)
    if numbering == "bands":
        band = np.floor((coord[:, 1] + 1.0) * nring + 0.5).astype(np.int64)
        old = np.lexsort((coord[:, 0], band))  # new -> old
        new = np.empty(nnode, np.int64)
        new[old] = np.arange(nnode)
        coord, elem, bnd = coord[old], new[elem].astype(np.int32), new[bnd].astype(np.int32)
    elif numbering != "rings":
        raise ValueError(f"unknown numbering {numbering!r}")
    return Mesh(coord, elem, bnd)


def right_edge_traction(mesh: Mesh, n: int, t=(0.0, -1.0)) -> np.ndarray:
    """Lumped nodal load of a uniform traction on the right edge bars: each bar
    of length l adds t*l/2 to both of its nodes (the rule of the commented-out
    edge-load code in src/femeqn/eqnsys_solid.cpp:509-572)."""
    load = np.zeros((mesh.nnode, 2))
    for a, b in mesh.extra["right"]:
        ell = float(np.hypot(*(mesh.coord[a] - mesh.coord[b])))
        for v in (a, b):
            load[v, 0] += t[0] * ell * 0.5
            load[v, 1] += t[1] * ell * 0.5
    return load


def gaussian_source_load(mesh: Mesh, center=(0.3, 0.1), sigma=0.05) -> np.ndarray:
    """Nodal load of f(x) = exp(-|x-c|^2 / (2 sigma^2)) with the one-point rule
    area/3 * f(centroid) per triangle node (the rule of
    src/femeqn/eqn_poisson.cpp:108-110).  Complex interleaved (re, im)."""
    p = mesh.coord[mesh.elem]
    area = 0.5 * ((p[:, 1, 0] - p[:, 0, 0]) * (p[:, 2, 1] - p[:, 0, 1]) - (p[:, 2, 0] - p[:, 0, 0]) * (p[:, 1, 1] - p[:, 0, 1]))
    cen = p.mean(axis=1)
    f = np.exp(-((cen[:, 0] - center[0]) ** 2 + (cen[:, 1] - center[1]) ** 2) / (2 * sigma * sigma))
    load = np.zeros((mesh.nnode, 2))
    w = area * f / 3.0
    for k in range(3):
        np.add.at(load[:, 0], mesh.elem[:, k], w)
    return load


def concat(meshes: list) -> tuple:
    """Disjoint union of meshes of one element kind, for a batch: node numbers of
    mesh k are shifted by the nodes of meshes 0..k-1, so the union's pattern is
    block-diagonal with mesh k's rows in [node_off[k], node_off[k+1]).  Returns
    (Mesh, node_off, elem_off)."""
    node_off = np.zeros(len(meshes) + 1, np.int64)
    elem_off = np.zeros(len(meshes) + 1, np.int64)
    for k, m in enumerate(meshes):
        node_off[k + 1] = node_off[k] + m.nnode
        elem_off[k + 1] = elem_off[k] + m.elem.shape[0]
    coord = np.concatenate([m.coord for m in meshes])
    elem = np.concatenate([m.elem + node_off[k] for k, m in enumerate(meshes)]).astype(np.int32)
    bnd = np.concatenate([m.bnd + node_off[k] for k, m in enumerate(meshes) if m.bnd.size]).astype(np.int32) \
        if any(m.bnd.size for m in meshes) else np.zeros((0, 2), np.int32)
    return Mesh(coord, elem, bnd, {}), node_off, elem_off


def batch_sizes(count: int, lo: int, hi: int, seed: int) -> np.ndarray:
    """Grid sides n drawn log-uniformly in [lo, hi] (integers) from the seed."""
    rng = np.random.default_rng(seed)
    return np.rint(np.exp(rng.uniform(np.log(lo), np.log(hi), count))).astype(np.int64)
