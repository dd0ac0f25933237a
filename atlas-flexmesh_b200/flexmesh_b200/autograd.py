"""Differentiable Newton solve: per-element Lame parameters -> displacements.

``NewtonSolve.apply(mu, lam, solver)`` runs the load path of ``solver`` on
the GPU (fm_newton_step per load level) with per-element mu_e, lambda_e and
returns the converged displacement u.  Its backward is the hand-written
adjoint (fm_adjoint): it solves K_exact^T w = dL/du on the free DOFs at the
converged state and returns dL/dmu_e = -w_e . df_e/dmu_e and the lambda
counterpart.  Both directions go through the C ABI; there is no PyTorch
re-implementation of the mechanics.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from . import _lib as L


@dataclass
class SolveSettings:
    n_steps: int
    rtol: float = 1e-10
    inner_tol: float = 1e-12
    prec: int = L.FM_FP64
    max_newton: int = 400
    adjoint_tol: float = 1e-10
    adjoint_inner_tol: float = 1e-12
    adjoint_prec: int = L.FM_FP64
    max_sweeps: int = 1000


class LameSolver:
    """A context bound to one mesh and its Dirichlet data; the material is
    supplied per call as per-element Lame parameters."""

    def __init__(self, xyz, conn, mask, bc_value, nu, settings: SolveSettings,
                 elem_volume=None, device: int = 0):
        self.ctx = L.Context(device)
        self.ctx.set_mesh(xyz, conn, elem_volume)
        self.ctx.set_bc(mask, bc_value)
        self.nu = nu
        self.s = settings
        self.device = device
        self.last = {}

    def solve(self, mu_e: np.ndarray, lam_e: np.ndarray) -> torch.Tensor:
        self.ctx.set_material_lame(mu_e, lam_e, self.nu)
        u = torch.zeros(self.ctx.n_dofs, dtype=torch.float64, device=f"cuda:{self.device}")
        newton = pcg = 0
        for s in range(1, self.s.n_steps + 1):
            r = self.ctx.newton_step(u, s / self.s.n_steps, rtol=self.s.rtol,
                                     inner_tol=self.s.inner_tol, max_newton=self.s.max_newton,
                                     prec=self.s.prec)
            newton += r["newton_iters"]
            pcg += r["pcg_iters"]
        self.last = {"newton_iters": newton, "pcg_iters": pcg}
        return u

    def adjoint(self, u, dLdu):
        gm, gl, w, sweeps, pcg = self.ctx.adjoint(u, dLdu, tol=self.s.adjoint_tol,
                                                  inner_tol=self.s.adjoint_inner_tol,
                                                  max_sweeps=self.s.max_sweeps,
                                                  prec=self.s.adjoint_prec)
        self.last.update({"adjoint_sweeps": sweeps, "adjoint_pcg": pcg})
        return gm, gl


class NewtonSolve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, mu, lam, solver: LameSolver):
        mu_h = mu.detach().double().cpu().numpy()
        lam_h = lam.detach().double().cpu().numpy()
        u = solver.solve(mu_h, lam_h)
        ctx.solver = solver
        ctx.mu_h, ctx.lam_h = mu_h, lam_h
        ctx.save_for_backward(u)
        return u

    @staticmethod
    def backward(ctx, grad_u):
        (u,) = ctx.saved_tensors
        solver = ctx.solver
        # the context's material must be the forward's one
        solver.ctx.set_material_lame(ctx.mu_h, ctx.lam_h, solver.nu)
        gm, gl = solver.adjoint(u, grad_u.detach().contiguous().double())
        return gm, gl, None


def newton_solve(mu, lam, solver: LameSolver):
    """u(mu, lam), differentiable in both per-element parameter arrays."""
    return NewtonSolve.apply(mu, lam, solver)
