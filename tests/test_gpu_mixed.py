"""Mixed-precision PCG (FP32 values for SpMV and ILU sweeps, FP64 vectors,
dots, scalars and D^-1, FP64 residual replacement): the answer is judged by
the TRUE residual b - A x with the FP64 matrix and against the FP64 oracle's
solution at the same tolerance."""
import numpy as np
import pytest

from tests import cases

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float64)).cuda()


SYSTEMS = {
    "poisson64": lambda: cases.poisson(64)[1],
    "poisson_coef": lambda: cases.poisson(48, np.random.default_rng(1).lognormal(0, 1.0, 2 * 48 * 48))[1],
    "solid2d": lambda: cases.solid2d(16, np.random.default_rng(2).lognormal(0, 0.5, 2 * 16 * 16))[1],
    "solid3d": lambda: cases.solid3d(12, 3, 3)[1],
}


@pytest.fixture(params=[0, 1], ids=["fp64_operator", "fp32_operator"])
def op32(ctx, request):
    ctx.mixed_operator = request.param
    assert ctx.mixed_operator == request.param
    yield request.param
    ctx.mixed_operator = 0


@pytest.mark.parametrize("name", list(SYSTEMS))
@pytest.mark.parametrize("sweep", [1, 2, 3, 5, 7, 9, 10])
def test_mixed_true_residual_and_solution(ctx, op32, name, sweep):
    from delfem_b200 import lib
    S = SYSTEMS[name]()
    ns, fd, fo = S.ilu0()
    tol = 1e-10
    ref = S.solve(fd, fo, method="pcg", tol=tol, maxit=5000)
    A = lib.Matrix(ctx, S.rowptr, S.colind, S.b)
    A.set_values(S.diag, S.off)
    M = lib.ILU(A)
    M.factor()
    M.sweep = sweep
    r = _dev(S.rhs)
    x = torch.zeros_like(r)
    rc, it, conv = lib.solve_pcg_mixed(A, M, r, x, tol=tol, maxit=5000)
    assert rc == lib.OK, (rc, it, conv)
    xg = x.cpu().numpy()
    res = S.rhs - S.spmv(1.0, xg, 0.0, np.zeros_like(S.rhs))
    assert np.linalg.norm(res) < tol * np.linalg.norm(S.rhs)  # FP64 true residual
    assert conv < tol
    err = np.linalg.norm(xg - ref["x"]) / np.linalg.norm(ref["x"])
    assert err <= 1e-7, err
    if not op32:  # FP64 operator: no loss of conjugacy in A; the FP32 factor alone costs
        # up to ~50% more iterations (L and D^-1 U round separately, so the preconditioner
        # is not exactly symmetric; elasticity's ill-conditioned factors amplify that)
        assert it <= 2 * ref["iters"] + 5, (it, ref["iters"])
    # returned r is the final (true) residual, up to the rounding of b - A x in
    # another summation order: |dr| <= c eps (|b| + |A| |x|)
    absAx = S.spmv(1.0, np.abs(xg), 0.0, np.zeros_like(S.rhs), diag=np.abs(S.diag), off=np.abs(S.off))
    assert (np.abs(r.cpu().numpy() - res) <= 1e-13 * (np.abs(S.rhs) + absAx)).all()


def test_mixed_deterministic_and_host_entry(ctx):
    from delfem_b200 import lib
    S = SYSTEMS["poisson64"]()
    A = lib.Matrix(ctx, S.rowptr, S.colind, S.b)
    A.set_values(S.diag, S.off)
    M = lib.ILU(A)
    M.factor()
    out = []
    for _ in range(2):
        rc, x, it, conv = lib.solve_host(A, M, S.rhs, lib.PCG_MIXED, tol=1e-9, maxit=5000)
        assert rc == lib.OK
        out.append((x, it, conv))
    assert np.array_equal(out[0][0], out[1][0]) and out[0][1:] == out[1][1:]


def test_mixed_operator_switch_recaptures(ctx):
    """Switching the operator precision between solves re-captures the graph:
    both settings give the FP64 true residual, and the FP64 operator keeps the
    FP64 solve's iteration count."""
    from delfem_b200 import lib
    S = SYSTEMS["solid3d"]()
    ns, fd, fo = S.ilu0()
    ref = S.solve(fd, fo, method="pcg", tol=1e-10, maxit=5000)
    A = lib.Matrix(ctx, S.rowptr, S.colind, S.b)
    A.set_values(S.diag, S.off)
    M = lib.ILU(A)
    M.factor()
    for op in (0, 1, 0):
        ctx.mixed_operator = op
        r = _dev(S.rhs)
        x = torch.zeros_like(r)
        rc, it, conv = lib.solve_pcg_mixed(A, M, r, x, tol=1e-10, maxit=5000)
        assert rc == lib.OK
        res = S.rhs - S.spmv(1.0, x.cpu().numpy(), 0.0, np.zeros_like(S.rhs))
        assert np.linalg.norm(res) < 1e-10 * np.linalg.norm(S.rhs)
        if op == 0:
            assert it <= 2 * ref["iters"] + 5, (it, ref["iters"])
    ctx.mixed_operator = 0
    with pytest.raises(lib.DfmError):
        ctx.mixed_operator = 2


def test_mixed_follows_value_updates(ctx):
    """New values (set_values + refactor) reach the FP32 copies on the next solve."""
    from delfem_b200 import lib
    S = SYSTEMS["poisson64"]()
    A = lib.Matrix(ctx, S.rowptr, S.colind, S.b)
    A.set_values(S.diag, S.off)
    M = lib.ILU(A)
    M.factor()
    r = _dev(S.rhs)
    x = torch.zeros_like(r)
    lib.solve_pcg_mixed(A, M, r, x, tol=1e-9)
    A.set_values(S.diag * 2.0, S.off * 2.0)
    M.factor()
    r = _dev(S.rhs)
    x2 = torch.zeros_like(r)
    rc, it, conv = lib.solve_pcg_mixed(A, M, r, x2, tol=1e-9)
    assert rc == lib.OK
    assert np.allclose(x2.cpu().numpy() * 2.0, x.cpu().numpy(), rtol=1e-6, atol=1e-9)


@pytest.mark.parametrize("nring", [40])
@pytest.mark.parametrize("sweep", [1, 2, 3, 5, 7, 9, 10])
def test_cocg_mixed_true_residual(ctx, op32, nring, sweep):
    """complex64 values inside complex128 residual replacement (Helmholtz)."""
    from delfem_b200 import lib
    m, S = cases.helmholtz(nring, "bands")
    ns, fd, fo = S.ilu0()
    tol = 1e-8
    ref = S.solve(fd, fo, method="pcocg", tol=tol, maxit=5000)
    A = lib.Matrix(ctx, S.rowptr, S.colind, 1, lib.COMPLEX)
    A.set_values(S.diag, S.off)
    M = lib.ILU(A)
    M.factor()
    M.sweep = sweep
    r = _dev(S.rhs)
    x = torch.zeros_like(r)
    rc, it, conv = lib.solve_pcocg_mixed(A, M, r, x, tol=tol, maxit=5000)
    assert rc == lib.OK, (rc, it, conv)
    xg = x.cpu().numpy()
    res = S.rhs - S.spmv(1.0, xg, 0.0, np.zeros_like(S.rhs))
    assert np.linalg.norm(res) < tol * np.linalg.norm(S.rhs)
    err = np.linalg.norm(xg - ref["x"]) / np.linalg.norm(ref["x"])
    assert err <= 1e-5, err
