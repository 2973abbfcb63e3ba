"""Pins the oracle's C restatement to the reference's own code on seeded cases
larger than the fixtures (skipped where the reference build, oracle/_ref/
libdfm_refshim.so, is absent): pattern, assembly, elimination, ILU(0),
preconditioner and solves must be bit-identical."""
import numpy as np
import pytest

from delfem_b200 import meshes
from oracle import port as P
from oracle import refshim as R
from tests import cases

pytestmark = pytest.mark.skipif(not R.available(), reason="reference build (oracle/_ref) not present")


def _eq(a, b):
    return np.array_equal(np.asarray(a).view(np.uint64), np.asarray(b).view(np.uint64))


CASES = [
    ("poisson", R.POISSON2D, lambda: meshes.unit_square_tri(20), [1.3, 0.7], True, False, "pcg"),
    ("solid2d", R.SOLID2D, lambda: meshes.unit_square_tri(12, bnd="left"),
     [cases.LAM2_PS, cases.MYU2, 0.5, 0.0, -1.0], True, True, "pcg"),
    ("solid3d", R.SOLID3D, lambda: meshes.box_tet(8, 3, 3), [cases.LAM3, cases.MYU3, 1.0, 0.0, 0.0, -1.0], False,
     False, "pbicgstab"),
    ("helmholtz", R.HELMHOLTZ2D, lambda: meshes.unit_disk_tri(16), [2 * 3.1416 / 6], False, True, "pcocg"),
]


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_oracle_pinned_to_reference(case):
    name, kind, mk, params, with_coef, with_load, method = case
    m = mk()
    rng = np.random.default_rng(11)
    coef = rng.lognormal(0, 0.7, m.elem.shape[0]) if with_coef else None
    load = None
    if with_load:
        load = meshes.gaussian_source_load(m) if kind == R.HELMHOLTZ2D else meshes.right_edge_traction(m, 12)
    ref = R.RefSystem(kind, m)
    rp, ci = ref.pattern()
    ref.assemble(params, coef, load)
    d, o, rhs = ref.system()
    ref.ilu()
    _, fd, fo = ref.ilu_factor()
    rc, x, it, conv, _ = ref.solve({"pcg": R.PCG, "pbicgstab": R.PBICGSTAB, "pcocg": R.PCOCG}[method], 1e-10, 3000)

    prp, pci = P.pattern(m.nnode, m.elem)
    assert np.array_equal(prp, rp) and np.array_equal(pci, ci)
    b = {R.POISSON2D: 1, R.SOLID2D: 2, R.SOLID3D: 3, R.HELMHOLTZ2D: 1}[kind]
    S = P.System(rp, ci, b, cplx=kind == R.HELMHOLTZ2D)
    if kind == R.POISSON2D:
        S.asm_poisson(m, *params, coef)
    elif kind == R.SOLID2D:
        S.asm_solid2d(m, *params, coef)
    elif kind == R.SOLID3D:
        S.asm_solid3d(m, *params)
    else:
        S.asm_helmholtz(m, params[0])
    if load is not None:
        S.rhs += np.asarray(load).ravel()
    if kind != R.HELMHOLTZ2D:
        flags = P.bc_flags_from_bnd(m.nnode, b, m.bnd)
        assert np.array_equal(flags, ref.bcflag())
        S.apply_bc(flags)
    assert _eq(S.diag, d) and _eq(S.off, o) and _eq(S.rhs, rhs)
    ns, pfd, pfo = S.ilu0()
    assert _eq(pfd, fd) and _eq(pfo, fo)
    out = S.solve(pfd, pfo, method=method, tol=1e-10, maxit=3000)
    assert out["iters"] == it and out["conv"] == conv and _eq(out["x"], x)
    assert out["ok"] == (rc == 0)


ILUK_SYSTEMS = {
    "poisson14": lambda: cases.poisson(14)[1],
    "poisson_coef": lambda: cases.poisson(10, np.random.default_rng(8).lognormal(0, 1, 2 * 10 * 10))[1],
    "solid2d": lambda: cases.solid2d(7, np.random.default_rng(9).lognormal(0, 0.5, 2 * 7 * 7))[1],
    "solid3d": lambda: cases.solid3d(5, 2, 2)[1],
    "random_b1": lambda: cases.random_spd_like(120, 1, seed=11),
    "random_b3": lambda: cases.random_spd_like(70, 3, seed=12),
}


@pytest.mark.parametrize("name", list(ILUK_SYSTEMS))
@pytest.mark.parametrize("lev", [1, 2, 3, -1])
def test_iluk_pinned_to_reference(name, lev):
    """ILU(k) symbolic fill (AddFracPtn, including its keep-the-first-level
    rule that makes ILU(3) smaller than ILU(2) on some meshes), the values'
    initialisation and the numeric factor on the fill pattern: bit-identical
    to CMatDiaFrac_BlkCrs(lev, A) + SetValue_Initialize + DoILUDecomp."""
    S = ILUK_SYSTEMS[name]()
    ns, (fr, fc, fdia), fd, fo = S.iluk(lev)
    rc, rfr, rfc, rfd, rfo = R.mat_iluk(S.N, S.b, S.rowptr, S.colind, S.diag, S.off, lev)
    assert rc == 0 and ns == 0
    assert np.array_equal(fr, rfr) and np.array_equal(fc, rfc)
    assert _eq(fd, rfd) and _eq(fo, rfo)
    assert fc.size >= S.colind.size


def _fill_rows(N, kind):
    """SetFillBlk lists: a few scattered rows, a contiguous run, the last row."""
    if kind == "scattered":
        return np.random.default_rng(N).choice(N, size=max(1, N // 15), replace=False).astype(np.uint32)
    if kind == "run":
        return np.arange(N // 3, N // 3 + max(2, N // 10), dtype=np.uint32)
    return np.array([N - 1, N - 1], np.uint32)  # the last row, listed twice


@pytest.mark.parametrize("name", ["poisson_coef", "solid2d", "solid3d", "random_b3"])
@pytest.mark.parametrize("lev", [0, 1, 2])
@pytest.mark.parametrize("kind", ["scattered", "run", "last"])
def test_iluk_fill_rows_pinned_to_reference(name, lev, kind):
    """CPreconditioner_ILU::SetFillBlk: AddFracPtn(lev, aBlkFill), where fill
    through or into a listed row is kept at any level (flag -1), over
    CMatDiaFrac_BlkCrs(0, A): the oracle's pattern, values and factor are
    bit-identical to the reference's."""
    S = ILUK_SYSTEMS[name]()
    rows = _fill_rows(S.N, kind)
    ns, (fr, fc, fdia), fd, fo = S.iluk(lev, rows)
    rc, rfr, rfc, rfd, rfo = R.mat_iluk(S.N, S.b, S.rowptr, S.colind, S.diag, S.off, lev, rows)
    assert rc == 0 and ns == 0
    assert np.array_equal(fr, rfr) and np.array_equal(fc, rfc)
    assert _eq(fd, rfd) and _eq(fo, rfo)
    if kind != "last":  # the last row's pivots have no upper part but itself
        _, (fr0, fc0, _), _, _ = S.iluk(lev)
        assert fc.size > fc0.size  # the listed rows took fill beyond level lev


@pytest.mark.parametrize("lev", [0, 1, 2])
def test_iluk_pcg_pinned_to_reference(lev):
    """Solve_PCG with CPreconditioner_ILU::SetFillInLevel(lev): the same x,
    iteration count and convergence ratio."""
    S = cases.solid3d(6, 3, 3)[1]
    ns, fpat, fd, fo = S.iluk(lev)
    o = S.solve_fill(fpat, fd, fo, tol=1e-10, maxit=2000)
    rc, x, it, conv, _, _ = R.mat_solve(S.N, S.b, S.rowptr, S.colind, S.diag, S.off, S.rhs, tol=1e-10, maxit=2000,
                                        lev=lev)
    assert rc == 0 and o["ok"]
    assert o["iters"] == it and _eq(o["x"], x) and o["conv"] == conv


@pytest.mark.parametrize("name,maxit", [("poisson", 5000), ("solid3d", 5000), ("solid2d", 5000), ("solid2d", 7)])
def test_cg_pinned_to_reference(name, maxit):
    """LsSol::Solve_CG (no preconditioner) through the reference's own
    CLinearSystem, against the oracle's restatement: x, iteration index and
    ratio bit-identical, including the max_iter exit (true, ratio left at the
    tolerance)."""
    S = {"poisson": lambda: cases.poisson(20)[1], "solid3d": lambda: cases.solid3d(6, 2, 2)[1],
         "solid2d": lambda: cases.solid2d(10)[1]}[name]()
    o = S.solve_cg(tol=1e-10, maxit=maxit)
    rc, x, it, conv, _, _ = R.mat_solve(S.N, S.b, S.rowptr, S.colind, S.diag, S.off, S.rhs, method=R.CG, tol=1e-10,
                                        maxit=maxit)
    assert rc == 0 and o["ok"]
    assert it == o["iters"] and _eq(conv, o["conv"]) and _eq(x, o["x"])
    if maxit == 7:
        assert it == 7 and conv == 1e-10


@pytest.mark.parametrize("nring,lev", [(16, 1), (16, 2), (40, 1), (24, -1)])
def test_complex_iluk_pinned_to_reference(nring, lev):
    """CZMatDiaFrac_BlkCrs(lev, A) (the fill path of CZPreconditioner_ILU::
    SetFillInLevel, src/matvec/zmatdiafrac_blkcrs.cpp:77-107, :263-441):
    pattern and factor of the oracle bit-identical to the reference's."""
    m, S = cases.helmholtz(nring)
    rc, fr, fc, fd, fo = R.zmat_iluk(S.N, S.rowptr, S.colind, S.diag, S.off, lev)
    ns, (pr, pc, pdia), od, oo = S.iluk(lev)
    assert np.array_equal(fr, pr) and np.array_equal(fc, pc)
    assert fc.size > S.colind.size  # fill entries exist
    assert _eq(fd, od) and _eq(fo, oo)


def test_complex_ilu1_cocg_pinned_to_reference():
    """The reference's Helmholtz demo runs CZPreconditioner_ILU with fill level
    1 (test_glut/helmholtz2d/main.cpp:87): its field-level ILU(1) + Solve_PCOCG
    against the oracle's, x, iteration count and ratio bit-identical."""
    m = meshes.unit_disk_tri(40)
    ref = R.RefSystem(R.HELMHOLTZ2D, m)
    ref.assemble([cases.WAVE_LENGTH], None, meshes.gaussian_source_load(m))
    ref.set_fill(1)
    ref.ilu()
    rc, x, it, conv, _ = ref.solve(R.PCOCG, 1e-10, 3000)
    m2, S = cases.helmholtz(40)
    ns, fpat, fd, fo = S.iluk(1)
    o = S.solve_fill(fpat, fd, fo, tol=1e-10, maxit=3000)
    assert rc == 0 and o["ok"]
    assert it == o["iters"] and _eq(conv, o["conv"]) and _eq(x, o["x"])
    assert fpat[1].size > S.colind.size  # a filled factor, not ILU(0)
