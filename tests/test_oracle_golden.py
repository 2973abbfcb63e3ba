"""The oracle (oracle/dfm_oracle.c) against golden fixtures produced by the
reference itself (tests/golden/make_golden.py): pattern, assembled system,
Dirichlet elimination, ILU(0) factor, SpMV, preconditioner and the full Krylov
solve (x, iteration count, convergence ratio) must all be bit-identical."""
import glob
import os

import numpy as np
import pytest

from delfem_b200.meshes import Mesh
from oracle import port as P

_ALL = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))
ILUK = [p for p in _ALL if os.path.basename(p).startswith("iluk")]
GOLDEN = [p for p in _ALL if p not in ILUK and not os.path.basename(p).startswith(("zmatref", "gidref", "reference_solutions"))]
METHOD = {0: "pcg", 1: "pbicgstab", 2: "pcocg"}
POISSON2D, SOLID2D, SOLID3D, HELMHOLTZ2D = 1, 2, 3, 4


def _same(a, b, what):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape, (what, a.shape, b.shape)
    assert np.array_equal(a.view(np.uint64) if a.dtype == np.float64 else a,
                          b.view(np.uint64) if b.dtype == np.float64 else b), what


def _oracle_system(g):
    kind = int(g["kind"])
    m = Mesh(g["coord"], g["elem"], g["bnd"], {})
    rp, ci = P.pattern(m.nnode, m.elem)
    b = {POISSON2D: 1, SOLID2D: 2, SOLID3D: 3, HELMHOLTZ2D: 1}[kind]
    S = P.System(rp, ci, b, cplx=kind == HELMHOLTZ2D)
    p = g["params"]
    coef = g["coef"] if g["coef"].size else None
    if kind == POISSON2D:
        S.asm_poisson(m, p[0], p[1], coef)
    elif kind == SOLID2D:
        S.asm_solid2d(m, p[0], p[1], p[2], p[3], p[4], coef)
    elif kind == SOLID3D:
        S.asm_solid3d(m, p[0], p[1], p[2], p[3], p[4], p[5])
    else:
        S.asm_helmholtz(m, p[0])
    if g["load"].size:
        S.rhs += g["load"]
    if kind != HELMHOLTZ2D:
        S.apply_bc(P.bc_flags_from_bnd(m.nnode, b, m.bnd))
    return kind, m, S


def test_fixtures_present():
    assert len(GOLDEN) >= 6


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_oracle_matches_reference_fixture(path):
    g = np.load(path)
    kind, m, S = _oracle_system(g)
    _same(S.rowptr, g["rowptr"], "rowptr")
    _same(S.colind, g["colind"], "colind")
    if kind != HELMHOLTZ2D:
        _same(P.bc_flags_from_bnd(m.nnode, S.b, m.bnd), g["bcflag"], "bc flags")
    _same(S.diag, g["diag"], "diag")
    _same(S.off, g["off"], "off")
    _same(S.rhs, g["rhs"], "rhs")
    ns, fd, fo = S.ilu0()
    _same(fd, g["ilu_diag"], "ILU diag")
    _same(fo, g["ilu_off"], "ILU off")
    _same(S.spmv(1.0, g["vec"], 0.0, np.zeros_like(g["vec"])), g["spmv"], "spmv")
    if not S.cplx:
        _same(S.precond(fd, fo, g["vec"]), g["precond"], "precond")
    out = S.solve(fd, fo, method=METHOD[int(g["method"])], tol=float(g["tol"]), maxit=int(g["maxit"]))
    assert out["ok"] == bool(g["ok"])
    assert out["iters"] == int(g["iters"])
    assert out["conv"] == float(g["conv"])
    _same(out["x"], g["x"], "x")


def test_fixture_edge_case_maxit_is_recorded():
    """The max_iter fixture keeps the reference's exit values (true, iterations =
    max_iter, conv_ratio = its input tolerance)."""
    g = np.load([p for p in GOLDEN if p.endswith("maxit.npz")][0])
    assert bool(g["ok"]) and int(g["iters"]) == int(g["maxit"]) and float(g["conv"]) == float(g["tol"])


@pytest.mark.parametrize("path", ILUK, ids=[os.path.basename(p)[:-4] for p in ILUK])
def test_oracle_iluk_matches_reference_fixture(path):
    """ILU(k): the fill pattern (AddFracPtn), the factor on it and the
    ILU(k)-preconditioned Solve_PCG, bit-identical to the reference's."""
    g = np.load(path)
    S = P.System(g["rowptr"], g["colind"], int(g["b"]))
    S.diag[:] = g["diag"]
    S.off[:] = g["off"]
    S.rhs[:] = g["rhs"]
    ns, fpat, fd, fo = S.iluk(int(g["lev"]))
    _same(fpat[0], g["frowptr"], "fill rowptr")
    _same(fpat[1], g["fcolind"], "fill colind")
    _same(fd, g["ilu_diag"], "ILU(k) diagonal")
    _same(fo, g["ilu_off"], "ILU(k) off-diagonal")
    o = S.solve_fill(fpat, fd, fo, tol=float(g["tol"]), maxit=2000)
    _same(o["x"], g["x"], "x")
    assert o["iters"] == int(g["iters"]) and o["conv"] == float(g["conv"])
