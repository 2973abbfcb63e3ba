"""Generate the golden fixtures tests/golden/*.npz from the reference itself.

Each fixture is one small seeded problem run through the reference's own CPU
code (DelFEM sources compiled by oracle/Makefile, driven through
oracle/ref_shim.cpp): the block-CRS pattern of CMatDia_BlkCrs, the assembled
matrix and residual after Dirichlet elimination (CLinearSystem_Field), the
ILU(0) factor (CPreconditioner_ILU), the reference's solve (Solve_PCG /
Solve_PBiCGSTAB / Solve_PCOCG: x, iterations, convergence ratio) and one
matrix-level SpMV and preconditioner application on a seeded vector.

Run where the reference tree and its build are available:
    make -C oracle REF=<reference tree> ref
    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from delfem_b200 import meshes  # noqa: E402
from oracle import refshim as R  # noqa: E402
from tests import cases  # noqa: E402


def case_list():
    rng = np.random.default_rng(2024)
    out = []
    m = meshes.unit_square_tri(6)
    out.append(("poisson_n6", R.POISSON2D, m, [1.0, 1.0], None, None, R.PCG))
    m = meshes.unit_square_tri(6)
    out.append(("poisson_coef_n6", R.POISSON2D, m, [1.0, 1.0], rng.lognormal(0, 1.0, m.elem.shape[0]), None, R.PCG))
    m = meshes.unit_square_tri(5, bnd="left")
    out.append(("solid2d_n5", R.SOLID2D, m, [cases.LAM2_PS, cases.MYU2, 0.0, 0.0, 0.0],
                rng.lognormal(0, 0.5, m.elem.shape[0]), meshes.right_edge_traction(m, 5), R.PCG))
    m = meshes.box_tet(4, 2, 2)
    out.append(("solid3d_4x2x2", R.SOLID3D, m, [cases.LAM3, cases.MYU3, 1.0, 0.0, 0.0, -1.0], None, None, R.PCG))
    m = meshes.box_tet(4, 2, 2)
    out.append(("solid3d_bicgstab", R.SOLID3D, m, [cases.LAM3, cases.MYU3, 1.0, 0.0, 0.0, -1.0], None, None,
                R.PBICGSTAB))
    m = meshes.unit_disk_tri(8)
    out.append(("helmholtz_r8_k4", R.HELMHOLTZ2D, m, [2 * 3.1416 / 4], None, meshes.gaussian_source_load(m),
                R.PCOCG))
    # under-resolved (k h = 2.5): stops at max_iter, the reference's exit values
    out.append(("helmholtz_r8_maxit", R.HELMHOLTZ2D, m, [cases.WAVE_LENGTH], None, meshes.gaussian_source_load(m),
                R.PCOCG))
    return out


def generate(path=HERE):
    rng = np.random.default_rng(7)
    for name, kind, m, params, coef, load, method in case_list():
        S = R.RefSystem(kind, m)
        rp, ci = S.pattern()
        S.assemble(params, coef, load)
        diag, off, rhs = S.system()
        flags = S.bcflag()
        S.ilu()
        _, fd, fo = S.ilu_factor()
        tol = 1e-10
        maxit = 60 if name.endswith("maxit") else 2000
        rc, x, it, conv, _ = S.solve(method, tol, maxit)
        ok = rc == 0  # the shim returns 0 when the reference's solver returned true
        v = rng.standard_normal(S.N * S.xw)
        if S.cplx:
            y = R.zmat_spmv(S.N, rp, ci, diag, off, 1.0, v, 0.0, np.zeros_like(v))
            z = np.zeros(0)
        else:
            y = R.mat_spmv(S.N, S.b, rp, ci, diag, off, 1.0, v, 0.0, np.zeros_like(v))
            z = R.mat_precond(S.N, S.b, rp, ci, fd, fo, v)
        np.savez_compressed(
            os.path.join(path, f"{name}.npz"),
            kind=kind, method=method, params=np.asarray(params, np.float64),
            coord=m.coord, elem=m.elem, bnd=m.bnd,
            coef=np.zeros(0) if coef is None else coef,
            load=np.zeros(0) if load is None else np.asarray(load, np.float64).ravel(),
            rowptr=rp, colind=ci, diag=diag, off=off, rhs=rhs, bcflag=flags,
            ilu_diag=fd, ilu_off=fo, x=x, iters=it, conv=conv, ok=int(bool(ok)), tol=tol, maxit=maxit,
            vec=v, spmv=y, precond=z)
        print(f"{name}: N={S.N} b={S.b} ncrs={S.ncrs} iters={it} conv={conv:.3e}")


def generate_iluk(path=HERE):
    """ILU(k) fixtures: a seeded system, the reference's fill pattern and
    factor (CMatDiaFrac_BlkCrs(lev, A) + SetValue_Initialize + DoILUDecomp)
    and its Solve_PCG with CPreconditioner_ILU::SetFillInLevel(lev)."""
    for name, S, lev in [("iluk1_solid3d_4x2x2", cases.solid3d(4, 2, 2)[1], 1),
                         ("iluk2_poisson_n8", cases.poisson(8)[1], 2),
                         ("iluk3_solid2d_n5", cases.solid2d(5, np.random.default_rng(5).lognormal(0, 0.5, 50))[1],
                          3)]:
        rc, fr, fc, fd, fo = R.mat_iluk(S.N, S.b, S.rowptr, S.colind, S.diag, S.off, lev)
        assert rc == 0
        rc, x, it, conv, _, _ = R.mat_solve(S.N, S.b, S.rowptr, S.colind, S.diag, S.off, S.rhs, tol=1e-10,
                                            maxit=2000, lev=lev)
        assert rc == 0
        np.savez_compressed(os.path.join(path, f"{name}.npz"), lev=lev, b=S.b, rowptr=S.rowptr, colind=S.colind,
                            diag=S.diag, off=S.off, rhs=S.rhs, frowptr=fr, fcolind=fc, ilu_diag=fd, ilu_off=fo, x=x,
                            iters=it, conv=conv, tol=1e-10)
        print(f"{name}: N={S.N} b={S.b} ncrs={S.colind.size} -> {fc.size} iters={it} conv={conv:.3e}")


def generate_zmat_text(path=HERE):
    """A complex matrix in the reference's text format (a Helmholtz disk
    system with two rows lacking their diagonal entry and shuffled columns) and
    the pattern and values the reference's CZMatDia_BlkCrs(file_path) reads
    from it."""
    m, S = cases.helmholtz(4)
    txt = os.path.join(path, "zmat_helmholtz_r4.txt")
    cases.write_zmat_text(txt, S.rowptr, S.colind, S.diag, S.off, shuffle_rows=None, skip_diag=(2, 5))
    N, rp, ci, d, o = R.zmat_read(txt)
    np.savez_compressed(os.path.join(path, "zmatref_helmholtz_r4.npz"), N=N, rowptr=rp, colind=ci, diag=d, off=o)
    print(f"zmat_helmholtz_r4: N={N} ncrs={ci.size}")


def generate_gid(path=HERE):
    """Two GiD ASCII meshes (a tetrahedral box, scaled by pi so that the
    coordinates use every digit; a triangulated square on the plane x = 0.25
    in 3-D) and what the reference's readers (Msh::CMesh3D and
    Msh::CMesher2D ReadFromFile_GiDMsh) build from them: nodes, elements and
    the boundary facets they derive."""
    m = meshes.box_tet(3, 2, 2)
    f3 = os.path.join(path, "gid_box_tet.msh")
    cases.write_gid_mesh(f3, m.coord * np.pi, m.elem, "Tetrahedra")
    rc, c3, e3 = R.gid_read(f3, want2d=False)
    assert rc == 0
    t = meshes.unit_square_tri(3)
    p3 = np.zeros((t.nnode, 3))
    p3[:, 0], p3[:, 1], p3[:, 2] = 0.25, t.coord[:, 0] * 1.3, t.coord[:, 1] * 0.7
    f2 = os.path.join(path, "gid_square_tri.msh")
    cases.write_gid_mesh(f2, p3, t.elem, "Triangle")
    rc, c2, e2 = R.gid_read(f2, want2d=True)
    assert rc == 0
    # the boundary facets the readers derive: grouped facets, group offsets, 2-D vertices and chain ends
    b3, b2 = R.gid_boundary(f3, want2d=False), R.gid_boundary(f2, want2d=True)
    bnd = {}
    for tag, b in (("tet", b3), ("tri", b2)):
        bnd[f"{tag}_bnd_facets"] = b["facets"]
        bnd[f"{tag}_bnd_group_ptr"] = np.cumsum([0] + [len(k) for k in b["groups"]])
        bnd[f"{tag}_bnd_vertices"] = b["vertices"]
        bnd[f"{tag}_bnd_ends"] = b["ends"]
    np.savez_compressed(os.path.join(path, "gidref_meshes.npz"), tet_coord=c3, tet_elem=e3, tri_coord=c2,
                        tri_elem=e2, **bnd)
    print(f"gid: {c3.shape[0]} nodes / {e3.shape[0]} tets, {c2.shape[0]} nodes / {e2.shape[0]} triangles")


if __name__ == "__main__":
    generate()
    generate_iluk()
    generate_zmat_text()
    generate_gid()
