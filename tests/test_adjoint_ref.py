"""The adjoint tests' CPU reference is itself checked: its eliminated K(theta)
equals the oracle's assembly (pinned to the reference) to rounding, and its
adjoint gradient agrees with central finite differences."""
import numpy as np

from oracle import port as P
from tests import cases
from tests.adjoint_ref import Reference


def test_reference_matrix_matches_oracle():
    m, theta, theta_t, obs, fixed, load = cases.adjoint_case(6, seed=3, nobs=10)
    R = Reference(m.coord, m.elem, fixed, load, cases.LAM2_PS, cases.MYU2)
    K = R.matrix(theta).tocsr()
    rp, ci = P.pattern(m.nnode, m.elem)
    S = P.System(rp, ci, 2)
    S.asm_solid2d(m, cases.LAM2_PS, cases.MYU2, 0.0, 0.0, 0.0, theta)
    S.rhs += load.ravel()
    S.apply_bc(P.bc_flags_from_bnd(m.nnode, 2, m.bnd))
    dense = np.zeros((2 * m.nnode, 2 * m.nnode))
    for i in range(m.nnode):
        dense[2 * i:2 * i + 2, 2 * i:2 * i + 2] = S.diag[4 * i:4 * i + 4].reshape(2, 2)
        for s in range(rp[i], rp[i + 1]):
            j = ci[s]
            dense[2 * i:2 * i + 2, 2 * j:2 * j + 2] = S.off[4 * s:4 * s + 4].reshape(2, 2)
    assert np.allclose(K.toarray(), dense, rtol=1e-13, atol=1e-14 * np.abs(dense).max())
    assert np.array_equal(R.f, S.rhs)


def test_reference_gradient_matches_finite_differences():
    m, theta, theta_t, obs, fixed, load = cases.adjoint_case(8, seed=4, nobs=20)
    R = Reference(m.coord, m.elem, fixed, load, cases.LAM2_PS, cases.MYU2)
    ut = R.solve(theta_t)[1]
    idx = np.concatenate([2 * obs, 2 * obs + 1])

    def gfun(u):
        g = np.zeros_like(u)
        g[idx] = u[idx] - ut[idx]
        return 0.5 * np.sum((u[idx] - ut[idx]) ** 2), g

    L, g = R.grad(theta, gfun)
    elems = np.random.default_rng(0).choice(m.elem.shape[0], 16, replace=False)
    fd = R.fd(theta, idx, ut, elems)
    assert np.linalg.norm(g[elems] - fd) <= 1e-6 * np.linalg.norm(fd)
