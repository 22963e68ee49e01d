"""Differentiation form: gradients of the smoothed SpecAnn energy through the leading eigenvector.

No counterpart in the reference. With per-vertex normalisation exponents a (a_i = alpha + offset_i)
the operator is N_a = D_a^{-1/2} (J/c) D_a^{-1/2}; its leading pair (lambda, y) comes from the
alpha-solve kernel, the rounding vector is x = D_a^{-1/2} y (models/spectral_annealing.py:663) and
the smoothed energy is L = -1/2 tanh(beta x)^T J tanh(beta x). `SmoothedEnergy` is a
torch.autograd.Function whose backward is the hand-written adjoint (sa_adjoint: projected MINRES
for (lambda I - N_a) w = (I - y y^T) dL/dy, then two SpMVs), giving dL/dalpha and dL/da per
vertex. `EigenProblem.tangent` gives dy/dalpha, the direction of the tangent predictor.
"""
from __future__ import annotations

from typing import Optional, Tuple

import numpy as np
import scipy.sparse as sp
import torch

from . import _lib
from .engine import Engine
from .spectral_annealing import as_csr


class EigenProblem:
    """One instance on the GPU with what the differentiation form needs: the leading eigenpair at
    any exponents, the smoothed energy and its gradient, and the eigenvector tangent."""

    def __init__(self, J, precision: int = 32, ncv: int = 33, seed: int = 42):
        self.J = as_csr(J)
        n = self.J.shape[0]
        self.n = n
        self.engine = Engine(n, self.J.nnz, precision=precision, ncv_max=max(2, min(ncv, 64)), max_candidates=1)
        data = self.J.data.astype(np.float32 if precision == 32 else np.float64)
        self.info = self.engine.upload_csr(self.J.indptr, self.J.indices, data)
        # the operator layout the solver would choose (the eigenpair and the adjoint both use it)
        self.operator_layout = "worklist"
        if self.engine.panels_pay():
            self.engine.build_panels()
            self.operator_layout = "panel"
        deg = np.asarray(abs(self.J).sum(axis=1)).ravel()
        self.d = deg / deg.max()
        self.ncv = max(2, min(ncv, n - 1, 64))
        self.seed = int(seed)
        self.precision = precision

    def gershgorin(self, alpha: float, offsets: Optional[np.ndarray]) -> float:
        """g = max_i d_i^(1 - a_i) (models/spectral_annealing.py:579 with per-vertex exponents)."""
        a = alpha if offsets is None else alpha + offsets
        with np.errstate(divide="ignore"):
            return float(np.max(np.where(self.d > 0, self.d ** (1.0 - a), 0.0)))

    def eigenpair(self, alpha: float, offsets: Optional[torch.Tensor] = None, tol: float = 1e-6,
                  maxiter: int = 4000) -> Tuple[float, torch.Tensor]:
        """Leading eigenpair (lambda, unit y on the device) of N_a from a cold seeded start."""
        eng = self.engine
        eng.set_exponent_offsets(offsets)
        g = self.gershgorin(alpha, None if offsets is None else offsets.detach().cpu().numpy())
        rho = 1.001 * g
        rec = eng.alpha_solve(alpha=alpha, alpha_prev=alpha, rho=rho, gershgorin=g, tol=tol, pred_tol=1e-3,
                              maxiter=maxiter, ncv=self.ncv, start_mode=_lib.SA_START_RANDOM, seed=self.seed,
                              stream_id=0, align=False, residual_check=True)
        if rec.status not in (_lib.SA_OK, _lib.SA_ERR_NOT_CONVERGED):
            _lib.check("sa_alpha_solve", rec.status)
        self.last_record = rec
        return rho - rec.mu, eng.result_vector()

    def energy_and_gradient(self, alpha: float, offsets: Optional[torch.Tensor] = None, beta: float = 8.0,
                            tol: float = 1e-6, adj_tol: float = 1e-4, maxiter: int = 4000):
        """(L, dL/da per vertex as a float64 device tensor, dL/dalpha, adjoint result)."""
        lam, y = self.eigenpair(alpha, offsets, tol=tol, maxiter=maxiter)
        grad = torch.empty(self.n, dtype=torch.float64, device=self.engine.device)
        res = self.engine.adjoint(_lib.SA_ADJ_GRADIENT, alpha=alpha, lambda1=lam, y=y, beta=beta, tol=adj_tol,
                                  maxiter=maxiter, grad=grad)
        self.last_adjoint = res
        return res.loss, grad, res.dloss_dalpha, res

    def tangent(self, alpha: float, lambda1: float, y: torch.Tensor, tol: float = 1e-6, maxiter: int = 4000):
        """dy/dalpha at the eigenpair (orthogonal to y), on the device in the working precision."""
        out = torch.empty_like(y)
        res = self.engine.adjoint(_lib.SA_ADJ_TANGENT, alpha=alpha, lambda1=lambda1, y=y, tol=tol,
                                  maxiter=maxiter, out=out)
        self.last_adjoint = res
        return out, res

    def close(self):
        self.engine.close()


class SmoothedEnergy(torch.autograd.Function):
    """L(alpha, offsets) = -1/2 tanh(beta x)^T J tanh(beta x) with x = D_a^{-1/2} y(a); backward by the
    eigenvector adjoint. alpha: 0-d tensor; offsets: n-vector (float64, zeros for a = alpha)."""

    @staticmethod
    def forward(ctx, alpha: torch.Tensor, offsets: torch.Tensor, problem: EigenProblem, beta: float = 8.0,
                tol: float = 1e-6, adj_tol: float = 1e-4):
        L, grad, _, _ = problem.energy_and_gradient(float(alpha), offsets.detach(), beta=beta, tol=tol,
                                                    adj_tol=adj_tol)
        ctx.save_for_backward(grad)
        ctx.devices = (alpha.device, offsets.device)
        return torch.tensor(L, dtype=torch.float64, device=alpha.device)

    @staticmethod
    def backward(ctx, gL):
        (grad,) = ctx.saved_tensors
        g = grad * gL.to(grad.device)
        return g.sum().to(ctx.devices[0]), g.to(ctx.devices[1]), None, None, None, None


def smoothed_energy(problem: EigenProblem, alpha: torch.Tensor, offsets: Optional[torch.Tensor] = None,
                    beta: float = 8.0, tol: float = 1e-6, adj_tol: float = 1e-4) -> torch.Tensor:
    """tol: Lanczos tolerance of the eigenpair; adj_tol: MINRES tolerance of the adjoint (the
    adjoint cannot be resolved much below the eigenpair's own accuracy)."""
    if offsets is None:
        offsets = torch.zeros(problem.n, dtype=torch.float64, device=problem.engine.device)
    return SmoothedEnergy.apply(alpha, offsets, problem, beta, tol, adj_tol)
