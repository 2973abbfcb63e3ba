"""Seeded problem builders shared by the tests: each returns the mesh and the
oracle system (oracle/dfm_oracle.c) assembled with the reference's kernels,
Dirichlet elimination applied."""
from __future__ import annotations

import numpy as np

from delfem_b200 import meshes
from oracle import port as P

NU = 0.3
LAM3 = 1.0 * NU / ((1 + NU) * (1 - 2 * NU))
MYU3 = 1.0 / (2 * (1 + NU))
LAM2_PS = NU / (1 - NU * NU)        # plane-stress lambda* at E = 1
MYU2 = 1.0 / (2 * (1 + NU))
WAVE_LENGTH = 2 * 3.1416 / 20       # k = 20 with the reference's truncated pi


def poisson(n, coef=None):
    m = meshes.unit_square_tri(n)
    rp, ci = P.pattern(m.nnode, m.elem)
    S = P.System(rp, ci, 1)
    S.asm_poisson(m, 1.0, 1.0, coef)
    S.apply_bc(P.bc_flags_from_bnd(m.nnode, 1, m.bnd))
    return m, S


def solid2d(n, theta=None):
    m = meshes.unit_square_tri(n, bnd="left")
    rp, ci = P.pattern(m.nnode, m.elem)
    S = P.System(rp, ci, 2)
    S.asm_solid2d(m, LAM2_PS, MYU2, 0.0, 0.0, 0.0, theta)
    S.rhs += meshes.right_edge_traction(m, n).ravel()
    S.apply_bc(P.bc_flags_from_bnd(m.nnode, 2, m.bnd))
    return m, S


def solid3d(nx, ny, nz):
    m = meshes.box_tet(nx, ny, nz)
    rp, ci = P.pattern(m.nnode, m.elem)
    S = P.System(rp, ci, 3)
    S.asm_solid3d(m, LAM3, MYU3, 1.0, 0.0, 0.0, -1.0)
    S.apply_bc(P.bc_flags_from_bnd(m.nnode, 3, m.bnd))
    return m, S


def helmholtz(nring, numbering="rings"):
    m = meshes.unit_disk_tri(nring, numbering=numbering)
    rp, ci = P.pattern(m.nnode, m.elem)
    S = P.System(rp, ci, 1, cplx=True)
    S.asm_helmholtz(m, WAVE_LENGTH)
    S.rhs += meshes.gaussian_source_load(m).ravel()
    return m, S


def random_spd_like(N, b, seed=0, density=6):
    """A random block pattern (symmetric) with diagonally dominant values."""
    rng = np.random.default_rng(seed)
    rows = [set() for _ in range(N)]
    for i in range(N):
        for j in rng.integers(0, N, size=rng.integers(0, density + 1)):
            if j != i:
                rows[i].add(int(j))
                rows[int(j)].add(i)
    rp = np.zeros(N + 1, np.uint32)
    for i in range(N):
        rp[i + 1] = rp[i] + len(rows[i])
    ci = np.concatenate([np.array(sorted(r), np.uint32) for r in rows]) if rp[-1] else np.zeros(0, np.uint32)
    S = P.System(rp, ci, b)
    bb = b * b
    S.off[:] = rng.standard_normal(S.off.size) * 0.1
    d = np.zeros((N, b, b))
    for i in range(N):
        d[i] = np.eye(b) * (2.0 + rng.random()) + rng.standard_normal((b, b)) * 0.05
    S.diag[:] = d.reshape(-1)
    S.rhs[:] = rng.standard_normal(N * b)
    return S


def adjoint_case(n, seed=0, nobs=256):
    """Plane-stress cantilever on the unit square (n x n grid of P1 triangles,
    nu = 0.3): per-element Young's modulus theta ~ lognormal(0, 0.5), left edge
    clamped, traction (0, -1) on the right edge; u_target from a second seeded
    theta field, observed at nobs random nodes (both components)."""
    m = meshes.unit_square_tri(n, bnd="left")
    rng = np.random.default_rng(seed)
    theta = rng.lognormal(0.0, 0.5, m.elem.shape[0])
    theta_t = rng.lognormal(0.0, 0.5, m.elem.shape[0])
    obs = rng.choice(m.nnode, size=min(nobs, m.nnode), replace=False)
    fixed = np.unique(m.bnd.ravel())
    load = meshes.right_edge_traction(m, n)
    return m, theta, theta_t, obs, fixed, load


def write_zmat_text(path, rowptr, colind, diag, off, shuffle_rows=None, skip_diag=()):
    """Writes a complex matrix in the reference's text format (read by
    CZMatDia_BlkCrs(file_path)): "nblk nnz", then "icol irow re im" per entry,
    rows ascending, the diagonal among the row's entries in column order.
    shuffle_rows: a numpy Generator to shuffle the columns inside each row;
    skip_diag: rows written without a diagonal entry."""
    N = rowptr.size - 1
    lines = []
    for i in range(N):
        ent = [(int(colind[s]), off[2 * s], off[2 * s + 1]) for s in range(rowptr[i], rowptr[i + 1])]
        if i not in skip_diag:
            ent.append((i, diag[2 * i], diag[2 * i + 1]))
        ent.sort()
        if shuffle_rows is not None:
            shuffle_rows.shuffle(ent)
        lines += [f"{i} {j} {float(re)!r} {float(im)!r}" for j, re, im in ent]
    with open(path, "w") as f:
        f.write(f"{N} {len(lines)}\n" + "\n".join(lines) + "\n")


def write_gid_mesh(path, coord, elem, elem_type, ndim=3):
    """Writes a GiD ASCII mesh (the format Msh::CMesh3D / CMesher2D
    ReadFromFile_GiDMsh read): coordinates padded to `ndim` columns, 1-based
    nodes, a material column on every element line."""
    coord = np.asarray(coord, np.float64)
    elem = np.asarray(elem)
    if coord.shape[1] < ndim:
        coord = np.hstack([coord, np.zeros((coord.shape[0], ndim - coord.shape[1]))])
    lines = [f"MESH dimension {ndim} ElemType {elem_type} Nnode {elem.shape[1]}", "Coordinates"]
    lines += [f"{i + 1} " + " ".join(repr(float(v)) for v in c[:ndim]) for i, c in enumerate(coord)]
    lines += ["end coordinates", "", "Elements"]
    lines += [f"{e + 1} " + " ".join(str(int(v) + 1) for v in row) + " 1" for e, row in enumerate(elem)]
    lines += ["end elements"]
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def poisson_raw(n):
    """As poisson(), before the Dirichlet elimination."""
    m = meshes.unit_square_tri(n)
    S = P.System(*P.pattern(m.nnode, m.elem), 1)
    S.asm_poisson(m, 1.0, 1.0)
    return m, S


def solid2d_raw(n):
    """As solid2d() with unit modulus, before the Dirichlet elimination."""
    m = meshes.unit_square_tri(n, bnd="left")
    S = P.System(*P.pattern(m.nnode, m.elem), 2)
    S.asm_solid2d(m, LAM2_PS, MYU2, 0.0, 0.0, 0.0)
    return m, S


def solid3d_raw(nx, ny, nz):
    """As solid3d(), before the Dirichlet elimination."""
    m = meshes.box_tet(nx, ny, nz)
    S = P.System(*P.pattern(m.nnode, m.elem), 3)
    S.asm_solid3d(m, LAM3, MYU3, 1.0, 0.0, 0.0, -1.0)
    return m, S
