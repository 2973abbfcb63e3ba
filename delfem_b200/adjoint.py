"""Differentiable linear elasticity solve: u = K(theta)^-1 f with a hand-written
adjoint, behind torch.autograd.Function.

K(theta) is the plane-stress P1 stiffness of AddLinSys_LinearSolid2D_Static_P1
(src/femeqn/eqn_linear_solid2d.cpp:505-598) with per-element Young's modulus
theta_e, i.e. lambda* and mu scaled by theta_e, so K_e(theta) = theta_e K_e^0.
Forward: device assembly (dfm_assemble_solid2d), Dirichlet elimination,
ILU(0) factorization and PCG, all through the C ABI.  Backward: one more PCG
with the SAME factorization (K is symmetric, so the transpose solve is the
solve), lambda = K^-1 dL/du, and the element kernel dfm_coef_grad_solid2d:
dL/dtheta_e = -lambda_e^T K_e^0 u_e.  There is no CPU path.
"""
from __future__ import annotations

import numpy as np
import torch

from . import lib


class PlaneStressProblem:
    """Device state of one plane-stress problem: mesh, pattern, Dirichlet flags,
    nodal load, and the factorization of the last assembled K(theta)."""

    def __init__(self, ctx: lib.Context, coord, elem, fixed_nodes, load, lam_star, myu, tol=1e-12, maxit=20000):
        self.ctx = ctx
        self.mesh = lib.Mesh(ctx, coord, elem)
        rp, ci = self.mesh.pattern()
        self.A = lib.Matrix(ctx, rp, ci, 2)
        self.M = lib.ILU(self.A)
        self.nnode = int(np.asarray(coord).shape[0])
        self.nelem = int(np.asarray(elem).shape[0])
        flags = np.zeros((self.nnode, 2), np.int32)
        flags[np.asarray(fixed_nodes, np.int64)] = 1
        self.flags = torch.from_numpy(flags.ravel()).cuda(ctx.device)
        self.load = torch.as_tensor(np.asarray(load, np.float64).ravel()).cuda(ctx.device)
        self.lam_star, self.myu = float(lam_star), float(myu)
        self.tol, self.maxit = tol, maxit
        self._theta = None  # theta of the current factorization

    def _prepare(self, theta: torch.Tensor):
        if self._theta is not None and self._theta.shape == theta.shape and torch.equal(self._theta, theta):
            return
        th = theta.detach().to(torch.float64).contiguous()
        self.rhs = torch.empty(2 * self.nnode, dtype=torch.float64, device=th.device)
        self.mesh.assemble_solid2d(self.A, self.lam_star, self.myu, 0.0, 0.0, 0.0, self.rhs, coef=th, load=self.load)
        lib.apply_dirichlet(self.A, self.flags, self.rhs)
        self.M.factor()
        self._theta = th.clone()

    def solve(self, theta: torch.Tensor, rhs: torch.Tensor | None = None) -> torch.Tensor:
        """u = K(theta)^-1 rhs (rhs defaults to the assembled load)."""
        self._prepare(theta)
        r = (self.rhs if rhs is None else rhs).detach().to(torch.float64).clone()
        x = torch.zeros_like(r)
        rc, it, conv = lib.solve_pcg(self.A, self.M, r, x, tol=self.tol, maxit=self.maxit)
        if rc != lib.OK:
            raise lib.DfmError(rc, "PlaneStressProblem.solve")
        self.last_iters = it
        return x

    def grad_theta(self, theta: torch.Tensor, u: torch.Tensor, gu: torch.Tensor) -> torch.Tensor:
        """dL/dtheta from dL/du by the adjoint solve and the element kernel."""
        self._prepare(theta)
        g = gu.detach().to(torch.float64).clone()
        g[self.flags.bool()] = 0.0  # eliminated DOFs carry no sensitivity
        lam = self.solve(theta, g)
        grad = torch.empty(self.nelem, dtype=torch.float64, device=u.device)
        lib.coef_grad_solid2d(self.mesh, self.lam_star, self.myu, lam, u.detach().contiguous(), grad)
        return grad


class ElasticSolve(torch.autograd.Function):
    """u = ElasticSolve.apply(theta, problem): differentiable in theta."""

    @staticmethod
    def forward(ctx, theta: torch.Tensor, problem: PlaneStressProblem):
        u = problem.solve(theta)
        ctx.problem = problem
        ctx.save_for_backward(theta.detach().clone(), u)
        return u

    @staticmethod
    def backward(ctx, gu):
        theta, u = ctx.saved_tensors
        return ctx.problem.grad_theta(theta, u, gu).to(theta.dtype), None


def elastic_solve(theta: torch.Tensor, problem: PlaneStressProblem) -> torch.Tensor:
    return ElasticSolve.apply(theta, problem)
