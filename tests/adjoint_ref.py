"""FP64 CPU reference for the adjoint tests (test infrastructure): the
plane-stress P1 element matrices at unit modulus, vectorised with numpy in the
order of the oracle's dfo_asm_solid2d_tri, the eliminated global matrix K(theta)
as a scipy sparse matrix, direct sparse solves, the adjoint gradient and
central finite differences of the loss."""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla


def element_matrices(coord, elem, lam, myu):
    """K_e^0[e, a, c, r, s] of every triangle (unit coefficient)."""
    p0, p1, p2 = coord[elem[:, 0]], coord[elem[:, 1]], coord[elem[:, 2]]
    area = 0.5 * ((p1[:, 0] - p0[:, 0]) * (p2[:, 1] - p0[:, 1]) - (p2[:, 0] - p0[:, 0]) * (p1[:, 1] - p0[:, 1]))
    t = 0.5 / area
    d = np.zeros((elem.shape[0], 3, 2))
    d[:, 0, 0] = t * (p1[:, 1] - p2[:, 1]); d[:, 1, 0] = t * (p2[:, 1] - p0[:, 1]); d[:, 2, 0] = t * (p0[:, 1] - p1[:, 1])
    d[:, 0, 1] = t * (p2[:, 0] - p1[:, 0]); d[:, 1, 1] = t * (p0[:, 0] - p2[:, 0]); d[:, 2, 1] = t * (p1[:, 0] - p0[:, 0])
    K = np.zeros((elem.shape[0], 3, 3, 2, 2))
    A = area[:, None, None]
    di, dj = d[:, :, None, :], d[:, None, :, :]
    K[..., 0, 0] = A * (lam + myu) * di[..., 0] * dj[..., 0]
    K[..., 0, 1] = A * (lam * di[..., 0] * dj[..., 1] + myu * dj[..., 0] * di[..., 1])
    K[..., 1, 0] = A * (lam * di[..., 1] * dj[..., 0] + myu * dj[..., 1] * di[..., 0])
    K[..., 1, 1] = A * (lam + myu) * di[..., 1] * dj[..., 1]
    dt = (di[..., 1] * dj[..., 1] + di[..., 0] * dj[..., 0]) * A * myu
    K[..., 0, 0] += dt
    K[..., 1, 1] += dt
    return K


class Reference:
    def __init__(self, coord, elem, fixed_nodes, load, lam, myu):
        self.coord, self.elem = coord, elem
        self.n = coord.shape[0]
        self.Ke = element_matrices(coord, elem, lam, myu)
        dof = (2 * elem[:, :, None] + np.arange(2)[None, None, :])  # [e, a, r]
        self.rows = np.broadcast_to(dof[:, :, None, :, None], self.Ke.shape).ravel()
        self.cols = np.broadcast_to(dof[:, None, :, None, :], self.Ke.shape).ravel()
        fixed = np.zeros(2 * self.n, bool)
        fixed[2 * np.asarray(fixed_nodes)] = True
        fixed[2 * np.asarray(fixed_nodes) + 1] = True
        self.fixed = fixed
        self.f = np.where(fixed, 0.0, np.asarray(load, np.float64).ravel())

    def matrix(self, theta):
        vals = (theta[:, None, None, None, None] * self.Ke).ravel()
        K = sp.coo_matrix((vals, (self.rows, self.cols)), shape=(2 * self.n, 2 * self.n)).tocsr()
        keep = sp.diags((~self.fixed).astype(np.float64))
        K = keep @ K @ keep + sp.diags(self.fixed.astype(np.float64))
        return K.tocsc()

    def solve(self, theta, rhs=None):
        lu = spla.splu(self.matrix(theta))
        return lu, lu.solve(self.f if rhs is None else rhs)

    def grad(self, theta, gfun):
        """(L, dL/dtheta) by the adjoint with direct solves; gfun(u) -> (L, dL/du)."""
        lu, u = self.solve(theta)
        L, gu = gfun(u)
        lam = lu.solve(np.where(self.fixed, 0.0, gu))
        le = lam[2 * self.elem[:, :, None] + np.arange(2)]
        ue = u[2 * self.elem[:, :, None] + np.arange(2)]
        return L, -np.einsum("ear,eacrs,ecs->e", le, self.Ke, ue)

    def fd(self, theta, idx, ut, elems, h=1e-6):
        """Central differences (L(theta + h e_k) - L(theta - h e_k)) / 2h of
        L = 1/2 sum_idx (u - ut)^2, each L(theta +- h e_k) evaluated exactly as
        L(theta) + (u - ut).d + 1/2 |d|^2 over idx with d = u(theta +- h e_k) - u
        solved directly from K(theta +- h e_k) d = -(+-h) K_e^0 u (an exact
        rearrangement: it avoids subtracting two nearly equal losses)."""
        _, u = self.solve(theta)
        w = u[idx] - ut[idx]
        out = []
        for e in elems:
            dofs = (2 * self.elem[e][:, None] + np.arange(2)).ravel()
            ke = self.Ke[e].transpose(0, 2, 1, 3).reshape(6, 6)
            du = np.zeros_like(u)
            du[dofs] = ke @ u[dofs]
            du[self.fixed] = 0.0
            dl = []
            for sgn in (1.0, -1.0):
                t = theta.copy()
                t[e] += sgn * h
                d = spla.splu(self.matrix(t)).solve(-sgn * h * du)
                dl.append(w @ d[idx] + 0.5 * d[idx] @ d[idx])
            out.append((dl[0] - dl[1]) / (2 * h))
        return np.array(out)
