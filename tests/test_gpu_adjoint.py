"""The hand-written adjoint of K(theta) u = f (plane-stress elasticity with
per-element Young's modulus) through torch.autograd: dL/dtheta from the device
(forward PCG, adjoint PCG with the same ILU(0) factorization, element kernel
-lambda_e^T K_e^0 u_e) against an FP64 reference gradient (direct sparse
solves) and against central finite differences (h = 1e-6, FP64) on sampled
elements, at the tolerance 1e-6 relative."""
import numpy as np
import pytest

from tests import cases
from tests.adjoint_ref import Reference

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _run(ctx, n, nsample, seed):
    from delfem_b200 import adjoint
    m, theta, theta_t, obs, fixed, load = cases.adjoint_case(n, seed=seed)
    R = Reference(m.coord, m.elem, fixed, load, cases.LAM2_PS, cases.MYU2)
    ut = R.solve(theta_t)[1]
    idx = np.concatenate([2 * obs, 2 * obs + 1])

    def gfun(u):
        g = np.zeros_like(u)
        g[idx] = u[idx] - ut[idx]
        return 0.5 * np.sum((u[idx] - ut[idx]) ** 2), g

    prob = adjoint.PlaneStressProblem(ctx, m.coord, m.elem, fixed, load, cases.LAM2_PS, cases.MYU2, tol=1e-12)
    th = torch.tensor(theta, dtype=torch.float64, device="cuda", requires_grad=True)
    u = adjoint.elastic_solve(th, prob)
    idx_t = torch.from_numpy(idx).cuda()
    ut_t = torch.from_numpy(ut).cuda()
    L = 0.5 * torch.sum((u[idx_t] - ut_t[idx_t]) ** 2)
    L.backward()
    g_dev = th.grad.cpu().numpy()
    L_ref, g_ref = R.grad(theta, gfun)
    assert abs(L.item() - L_ref) <= 1e-9 * abs(L_ref)
    err_ref = np.linalg.norm(g_dev - g_ref) / np.linalg.norm(g_ref)
    elems = np.random.default_rng(seed + 100).choice(m.elem.shape[0], nsample, replace=False)
    fd = R.fd(theta, idx, ut, elems, h=1e-6)
    err_fd = np.linalg.norm(g_dev[elems] - fd) / np.linalg.norm(fd)
    return err_ref, err_fd


def test_adjoint_small(ctx):
    err_ref, err_fd = _run(ctx, 32, 32, seed=5)
    assert err_ref <= 1e-8, err_ref
    assert err_fd <= 1e-6, err_fd


def test_adjoint_plane_stress_128(ctx):
    """The full configuration: 128 x 128 grid, 256 observed nodes, 64 sampled elements."""
    err_ref, err_fd = _run(ctx, 128, 64, seed=0)
    assert err_ref <= 1e-8, err_ref
    assert err_fd <= 1e-6, err_fd


def test_adjoint_reuses_factorization(ctx):
    """Backward after a second forward at another theta refactors for its own theta."""
    from delfem_b200 import adjoint
    m, theta, theta_t, obs, fixed, load = cases.adjoint_case(16, seed=6, nobs=40)
    R = Reference(m.coord, m.elem, fixed, load, cases.LAM2_PS, cases.MYU2)
    prob = adjoint.PlaneStressProblem(ctx, m.coord, m.elem, fixed, load, cases.LAM2_PS, cases.MYU2)
    th = torch.tensor(theta, device="cuda", requires_grad=True)
    u = adjoint.elastic_solve(th, prob)
    adjoint.elastic_solve(torch.tensor(theta_t, device="cuda"), prob)  # moves the factorization
    (0.5 * (u ** 2).sum()).backward()
    L, g_ref = R.grad(theta, lambda uu: (0.5 * np.sum(uu ** 2), np.where(R.fixed, 0.0, uu)))
    assert np.linalg.norm(th.grad.cpu().numpy() - g_ref) <= 1e-8 * np.linalg.norm(g_ref)
