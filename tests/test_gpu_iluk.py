"""ILU(k) on the device (CPreconditioner_ILU::SetFillInLevel) against the
oracle, whose fill pattern and factor are pinned bit-exact to the reference's
CMatDiaFrac_BlkCrs(lev, A) (tests/test_oracle_pin.py, tests/golden/iluk*):
the fill pattern and its level sets are identical, the factor is
bit-identical, the sweeps agree to 1e-11 in every schedule, and the PCG
solution matches to 1e-8 at relative residual 1e-10."""
import numpy as np
import pytest

from oracle import port as P
from tests import cases

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

SYSTEMS = {
    "poisson16": lambda: cases.poisson(16)[1],
    "poisson_coef": lambda: cases.poisson(20, np.random.default_rng(3).lognormal(0, 1, 2 * 20 * 20))[1],
    "solid2d": lambda: cases.solid2d(10, np.random.default_rng(4).lognormal(0, 0.5, 2 * 10 * 10))[1],
    "solid3d": lambda: cases.solid3d(6, 3, 3)[1],
    "random_b2": lambda: cases.random_spd_like(150, 2, 2),
    "random_b3": lambda: cases.random_spd_like(120, 3, 3),
}
LEVELS = [1, 2, -1]


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float64)).cuda()


def _setup(ctx, S, lev):
    from delfem_b200 import lib
    A = lib.Matrix(ctx, S.rowptr, S.colind, S.b)
    A.set_values(S.diag, S.off)
    M = lib.ILU(A, fill_level=lev)
    return A, M


@pytest.mark.parametrize("name", list(SYSTEMS))
@pytest.mark.parametrize("lev", LEVELS)
def test_iluk_pattern_levels_and_factor(ctx, name, lev):
    S = SYSTEMS[name]()
    A, M = _setup(ctx, S, lev)
    ns, (fr, fc, fdia), fd, fo = S.iluk(lev)
    rp, ci = M.pattern()
    assert np.array_equal(rp, fr) and np.array_equal(ci, fc)
    lf, nf, lb, nb = M.levels()
    olf, onf, olb, onb = P.levels(fr, fc, fdia)
    assert nf == onf and nb == onb and np.array_equal(lf, olf) and np.array_equal(lb, olb)
    rc, gns = M.factor()
    assert gns == ns == 0
    gd, go = M.get_values()
    assert np.array_equal(gd, fd) and np.array_equal(go, fo)  # bit-identical to DoILUDecomp on the fill pattern


@pytest.mark.parametrize("name", ["poisson_coef", "solid2d", "solid3d", "random_b3"])
@pytest.mark.parametrize("sweep", [1, 2, 3, 4, 5, 6, 7, 8, 9, 10])
def test_iluk_apply_every_schedule(ctx, name, sweep):
    S = SYSTEMS[name]()
    A, M = _setup(ctx, S, 1)
    M.factor()
    M.sweep = sweep
    ns, (fr, fc, fdia), fd, fo = S.iluk(1)
    F = P.System(fr, fc, S.b)  # the oracle's sweeps over the fill pattern
    r = np.random.default_rng(5).standard_normal(S.N * S.b)
    ref = F.precond(fd, fo, r)
    z = torch.zeros(S.N * S.b, dtype=torch.float64, device="cuda")
    M.apply(_dev(r), z)
    got = z.cpu().numpy()
    assert np.allclose(got, ref, rtol=1e-11, atol=1e-12 * np.abs(ref).max())


@pytest.mark.parametrize("name", list(SYSTEMS))
@pytest.mark.parametrize("lev", [1, 2])
def test_iluk_pcg_matches_oracle(ctx, name, lev):
    from delfem_b200 import lib
    S = SYSTEMS[name]()
    A, M = _setup(ctx, S, lev)
    M.factor()
    ns, fpat, fd, fo = S.iluk(lev)
    ref = S.solve_fill(fpat, fd, fo, tol=1e-10, maxit=3000)
    assert ref["ok"]
    r = _dev(S.rhs)
    x = torch.zeros_like(r)
    rc, it, conv = lib.solve_pcg(A, M, r, x, tol=1e-10, maxit=3000)
    assert rc == lib.OK
    assert abs(it - ref["iters"]) <= max(2, ref["iters"] // 20), (it, ref["iters"])
    xr = ref["x"]
    assert np.linalg.norm(x.cpu().numpy() - xr) <= 1e-8 * np.linalg.norm(xr)


def test_iluk_fewer_iterations_than_ilu0(ctx):
    """A stronger preconditioner, as in the reference: ILU(1) and ILU(2) need
    fewer PCG iterations than ILU(0) on the 3-D elasticity system."""
    from delfem_b200 import lib
    S = cases.solid3d(8, 3, 3)[1]
    its = []
    for lev in (0, 1, 2):
        A, M = _setup(ctx, S, lev)
        M.factor()
        r = _dev(S.rhs)
        x = torch.zeros_like(r)
        rc, it, conv = lib.solve_pcg(A, M, r, x, tol=1e-10, maxit=3000)
        assert rc == lib.OK
        its.append(it)
    assert its[0] > its[1] > its[2], its


def test_iluk_refactor_with_new_values(ctx):
    """A second factorization with new values starts again from A's values in
    the fill pattern (the fill entries are zeroed), like SetValue."""
    S = SYSTEMS["solid2d"]()
    A, M = _setup(ctx, S, 2)
    M.factor()
    S2 = cases.solid2d(10, np.random.default_rng(9).lognormal(0, 0.5, 2 * 10 * 10))[1]
    assert np.array_equal(S2.rowptr, S.rowptr) and np.array_equal(S2.colind, S.colind)
    A.set_values(S2.diag, S2.off)
    M.factor()
    ns, fpat, fd, fo = S2.iluk(2)
    gd, go = M.get_values()
    assert np.array_equal(gd, fd) and np.array_equal(go, fo)


def test_iluk_mixed_and_bicgstab(ctx):
    """The other real solvers take an ILU(k) object too: PBiCGSTAB and the
    mixed-precision PCG reach the FP64 true residual."""
    from delfem_b200 import lib
    S = SYSTEMS["solid3d"]()
    A, M = _setup(ctx, S, 1)
    M.factor()
    for solve in (lib.solve_pbicgstab, lib.solve_pcg_mixed):
        r = _dev(S.rhs)
        x = torch.zeros_like(r)
        rc, it, conv = solve(A, M, r, x, tol=1e-10, maxit=3000)
        assert rc == lib.OK
        res = S.rhs - S.spmv(1.0, x.cpu().numpy(), 0.0, np.zeros_like(S.rhs))
        assert np.linalg.norm(res) < 2e-10 * np.linalg.norm(S.rhs)


def test_iluk_limits(ctx):
    """lev < -1 is rejected; a solve with another matrix than the
    preconditioner's is rejected."""
    from delfem_b200 import lib
    S = SYSTEMS["poisson16"]()
    A, M = _setup(ctx, S, 1)
    with pytest.raises(lib.DfmError):
        lib.ILU(A, fill_level=-2)
    B = lib.Matrix(ctx, S.rowptr, S.colind, S.b)
    B.set_values(S.diag, S.off)
    M.factor()
    r = _dev(S.rhs)
    x = torch.zeros_like(r)
    with pytest.raises(lib.DfmError):
        lib.solve_pcg(B, M, r, x, tol=1e-10, maxit=100, allow=(lib.OK,))


@pytest.mark.parametrize("nring,lev,solve", [(16, 1, False), (40, 1, True), (24, 2, False), (60, 2, True)])
def test_complex_iluk_factor_and_cocg(ctx, nring, lev, solve):
    """CZPreconditioner_ILU::SetFillInLevel(lev) on the device: the fill pattern
    and the complex factor bit-identical to the oracle (pinned to the
    reference's CZMatDiaFrac_BlkCrs), the preconditioner to 1e-11 in the range
    schedules, and ILU(k)-COCG to 1e-8 of the oracle's x on the cases where
    COCG converges (on rings 16 / lev 1 and 24 / lev 2 it stalls above 1e-10
    for 3000 iterations, the reference's Solve_PCOCG as well, and its
    iterates there are rounding noise)."""
    from delfem_b200 import lib
    m, Z = cases.helmholtz(nring)
    A = lib.Matrix(ctx, Z.rowptr, Z.colind, 1, lib.COMPLEX)
    A.set_values(Z.diag, Z.off)
    M = lib.ILU(A, fill_level=lev)
    M.factor()
    ns, (fr, fc, fdia), fd, fo = Z.iluk(lev)
    grp, gci = M.pattern()
    assert np.array_equal(grp, fr) and np.array_equal(gci, fc)
    gd, go = M.get_values()
    assert np.array_equal(gd, fd) and np.array_equal(go, fo)
    rng = np.random.default_rng(3)
    rv = rng.standard_normal(2 * Z.N)
    ref = Z.precond_fill((fr, fc, fdia), fd, fo, rv)
    for sweep in (1, 2, 3, 9, 10):
        M.sweep = sweep
        z = torch.zeros(2 * Z.N, dtype=torch.float64, device="cuda")
        M.apply(_dev(rv), z)
        assert np.allclose(z.cpu().numpy(), ref, rtol=1e-11, atol=1e-12 * np.abs(ref).max()), sweep
    if not solve:
        return
    o = Z.solve_fill((fr, fc, fdia), fd, fo, tol=1e-10, maxit=3000)
    assert o["iters"] < 3000  # converged (Solve_PCOCG returns true at max_iter too)
    r = _dev(Z.rhs)
    x = torch.zeros_like(r)
    rc, it, conv = lib.solve_pcocg(A, M, r, x, tol=1e-10, maxit=3000)
    assert rc == lib.OK and o["ok"]
    assert np.linalg.norm(x.cpu().numpy() - o["x"]) <= 1e-8 * np.linalg.norm(o["x"])


def _fill_rows(N, kind):
    if kind == "scattered":
        return np.random.default_rng(N).choice(N, size=max(1, N // 15), replace=False).astype(np.uint32)
    return np.arange(N // 3, N // 3 + max(2, N // 10), dtype=np.uint32)


@pytest.mark.parametrize("name", ["poisson_coef", "solid2d", "solid3d", "random_b3"])
@pytest.mark.parametrize("lev", [0, 1, 2])
@pytest.mark.parametrize("kind", ["scattered", "run"])
def test_iluk_fill_rows(ctx, name, lev, kind):
    """SetFillBlk (AddFracPtn(lev, aBlkFill)): the listed rows take fill at
    any level; pattern, level sets and factor identical to the oracle's (pinned
    to the reference's), the range-partitioned sweeps to 1e-11."""
    from delfem_b200 import lib
    S = SYSTEMS[name]()
    rows = _fill_rows(S.N, kind)
    A = lib.Matrix(ctx, S.rowptr, S.colind, S.b)
    A.set_values(S.diag, S.off)
    M = lib.ILU(A, fill_level=lev, fill_rows=rows)
    ns, (fr, fc, fdia), fd, fo = S.iluk(lev, rows)
    rp, ci = M.pattern()
    assert np.array_equal(rp, fr) and np.array_equal(ci, fc)
    lf, nf, lb, nb = M.levels()
    olf, onf, olb, onb = P.levels(fr, fc, fdia)
    assert nf == onf and nb == onb and np.array_equal(lf, olf) and np.array_equal(lb, olb)
    rc, gns = M.factor()
    assert gns == ns == 0
    gd, go = M.get_values()
    assert np.array_equal(gd, fd) and np.array_equal(go, fo)
    F = P.System(fr, fc, S.b)
    r = np.random.default_rng(6).standard_normal(S.N * S.b)
    ref = F.precond(fd, fo, r)
    for sweep in (1, 9):
        M.sweep = sweep
        z = torch.zeros(S.N * S.b, dtype=torch.float64, device="cuda")
        M.apply(_dev(r), z)
        got = z.cpu().numpy()
        assert np.allclose(got, ref, rtol=1e-11, atol=1e-12 * np.abs(ref).max())


def test_iluk_fill_rows_invalid(ctx):
    """A listed row at or past the bound, or a zero bound, is DFM_ERR_INVALID."""
    from delfem_b200 import lib
    S = SYSTEMS["poisson16"]()
    A = lib.Matrix(ctx, S.rowptr, S.colind, S.b)
    for rows, bound in (([S.N], None), ([3], 3), ([0], 0)):
        with pytest.raises(lib.DfmError):
            lib.ILU(A, fill_level=1, fill_rows=np.array(rows, np.uint32), fill_bound=bound)
