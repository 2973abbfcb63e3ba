"""Batched ILU(0)-PCG over uneven instances against one oracle solve per
instance (each instance: its own Solve_PCG): per-instance solutions to 1e-8
at relative residual 1e-10, iteration counts within a few, masks for
instances that stop early, per-instance max_iter, and argument checks."""
import numpy as np
import pytest

from delfem_b200 import meshes
from oracle import port as P

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _batch_problem(sizes, seed=0, zero_rhs=()):
    rng = np.random.default_rng(seed)
    ms = [meshes.unit_square_tri(int(n)) for n in sizes]
    big, noff, eoff = meshes.concat(ms)
    kappa = rng.lognormal(0.0, 1.0, big.elem.shape[0])
    rp, ci = P.pattern(big.nnode, big.elem)
    S = P.System(rp, ci, 1)
    S.asm_poisson(big, 1.0, 1.0, kappa)
    S.apply_bc(P.bc_flags_from_bnd(big.nnode, 1, big.bnd))
    for k in zero_rhs:
        S.rhs[noff[k]:noff[k + 1]] = 0.0
    inst = []
    for k, m in enumerate(ms):
        a, b = noff[k], noff[k + 1]
        Si = P.System(*P.pattern(m.nnode, m.elem), 1)
        Si.asm_poisson(m, 1.0, 1.0, kappa[eoff[k]:eoff[k + 1]])
        Si.apply_bc(P.bc_flags_from_bnd(m.nnode, 1, m.bnd))
        assert np.array_equal(Si.diag, S.diag[a:b])  # the union holds the instances unchanged
        Si.rhs[:] = S.rhs[a:b]
        inst.append(Si)
    return S, noff, inst


def _gpu_batch(ctx, S, noff):
    from delfem_b200 import lib
    A = lib.Matrix(ctx, S.rowptr, S.colind, 1)
    A.set_values(S.diag, S.off)
    M = lib.ILU(A)
    M.factor()
    return A, M, lib.Batch(M, noff)


@pytest.mark.parametrize("sweep,schedule", [(1, (1,)), (2, (1,)), (3, (1,)), (1, (2, 256, 2)), (1, (2, 512, 4)),
                                            (1, (2, 1024, 8)), (0, (0,))])
def test_batch_matches_per_instance_oracle(ctx, sweep, schedule):
    from delfem_b200 import lib
    sizes = [3, 17, 8, 30, 1, 12, 24, 5]
    S, noff, inst = _batch_problem(sizes, seed=1)
    A, M, B = _gpu_batch(ctx, S, noff)
    if sweep:
        M.sweep = sweep
    B.schedule = schedule
    rc, x, it, conv, st = B.solve(S.rhs, tol=1e-10, maxit=2000)
    assert rc == lib.OK and (st == lib.OK).all()
    for k, Si in enumerate(inst):
        ns, fd, fo = Si.ilu0()
        ref = Si.solve(fd, fo, method="pcg", tol=1e-10, maxit=2000)
        xk = x[noff[k]:noff[k + 1]]
        err = np.linalg.norm(xk - ref["x"]) / max(np.linalg.norm(ref["x"]), 1e-300)
        assert err <= 1e-8, (k, err)
        assert abs(int(it[k]) - ref["iters"]) <= 2, (k, it[k], ref["iters"])
        assert conv[k] < 1e-10


@pytest.mark.parametrize("schedule", [(1,), (2, 512, 4)])
def test_batch_masks_and_maxit(ctx, schedule):
    from delfem_b200 import lib
    sizes = [20, 4, 16, 9]
    S, noff, inst = _batch_problem(sizes, seed=2, zero_rhs=(2,))
    A, M, B = _gpu_batch(ctx, S, noff)
    B.schedule = schedule
    rc, x, it, conv, st = B.solve(S.rhs, tol=1e-10, maxit=12)
    assert rc == lib.NOT_CONVERGED
    assert st[2] == lib.OK and it[2] == 0 and np.all(x[noff[2]:noff[3]] == 0)  # zero rhs: stops at once
    for k in (0, 1, 3):
        ns, fd, fo = inst[k].ilu0()
        ref = inst[k].solve(fd, fo, method="pcg", tol=1e-10, maxit=12)
        if ref["ok"]:
            assert st[k] == lib.OK
        else:
            assert st[k] == lib.NOT_CONVERGED and it[k] == 12
            xk = x[noff[k]:noff[k + 1]]
            assert np.linalg.norm(xk - ref["x"]) <= 1e-9 * np.linalg.norm(ref["x"])


def test_batch_device_buffers_tuning_and_determinism(ctx):
    from delfem_b200 import lib
    S, noff, inst = _batch_problem([10, 25, 7], seed=3)
    A, M, B = _gpu_batch(ctx, S, noff)
    b = torch.from_numpy(S.rhs).cuda()
    outs = []
    for tune in [(0, 0), (8, 32), (32, 512), (4, 64)]:
        B.tuning = tune
        x = torch.zeros_like(b)
        rc, _, it, conv, st = B.solve(b, x, tol=1e-9)
        assert rc == lib.OK
        outs.append((x.cpu().numpy(), it.copy()))
        if tune != (0, 0):
            assert B.tuning == tune
    # the same tuning twice gives the same bits; other tunings agree to rounding
    B.tuning = (4, 64)
    x = torch.zeros_like(b)
    B.solve(b, x, tol=1e-9)
    assert np.array_equal(x.cpu().numpy(), outs[-1][0])
    for xo, ito in outs:
        assert np.allclose(xo, outs[0][0], rtol=1e-7, atol=1e-12)


def test_batch_rejects_cross_instance_entries(ctx):
    from delfem_b200 import lib
    S, noff, inst = _batch_problem([4, 4], seed=4)
    A, M, _ = _gpu_batch(ctx, S, noff)
    bad = noff.copy()
    bad[1] += 1  # cuts through instance 0's rows
    with pytest.raises(lib.DfmError):
        lib.Batch(M, bad)


def test_batch_schedules_agree(ctx):
    """Both schedules run the same per-instance algorithm: the same iteration
    counts up to reduction-order effects and solutions to rounding."""
    from delfem_b200 import lib
    S, noff, inst = _batch_problem([40, 9, 25, 64, 2], seed=7)
    A, M, B = _gpu_batch(ctx, S, noff)
    B.schedule = (1,)
    rc1, x1, it1, c1, st1 = B.solve(S.rhs, tol=1e-10)
    B.schedule = (2, 256, 4)
    rc2, x2, it2, c2, st2 = B.solve(S.rhs, tol=1e-10)
    assert rc1 == rc2 == lib.OK
    assert np.all(np.abs(it1.astype(int) - it2.astype(int)) <= 2)
    assert np.allclose(x1, x2, rtol=1e-7, atol=1e-12)
    B.schedule = (0,)
    B.solve(S.rhs, tol=1e-10)
    assert B.schedule[0] in (1, 2)  # autotuned
