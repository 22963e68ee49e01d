"""Dense FP64 oracle of the differentiation form (test infrastructure only: the tests use it as
the checker of the GPU adjoint; nothing in the product imports it).

The reference has no gradients, so this is a restatement of the mathematics, checked against
finite differences in tests/test_adjoint_oracle.py:
  d = |J| 1 / c, c = max_i sum_j |J_ij|; D_a = max(d^a, 1e-12) per vertex (the clamp of
  models/spectral_annealing.py:34); M = D_a^{-1/2} (J / c) D_a^{-1/2}; (lambda, y) its leading
  pair with |y| = 1; x = D_a^{-1/2} y (models/spectral_annealing.py:663);
  L = -1/2 tanh(beta x)^T J tanh(beta x).
Dense eigh and solves: for n up to a few thousand.
"""
from __future__ import annotations

import numpy as np
import scipy.linalg as sla
import scipy.sparse as sp

LOG2_CLAMP = np.log2(1e-12)


def _parts(J, a):
    J = sp.csr_matrix(J, dtype=np.float64)
    n = J.shape[0]
    deg = np.asarray(abs(J).sum(axis=1)).ravel()
    c = deg.max()
    d = deg / c
    a = np.broadcast_to(np.asarray(a, dtype=np.float64), (n,))
    ld = np.log2(d)
    logD = np.where(a == 0.0, 0.0, a * ld)
    active = logD > LOG2_CLAMP
    s = np.exp2(-0.5 * np.maximum(logD, LOG2_CLAMP))          # D^{-1/2}
    l = np.where(active, -0.5 * np.log(d), 0.0)               # d ln s_i / d a_i
    Jd = J.toarray()
    M = (s[:, None] * Jd * s[None, :]) / c
    return Jd, M, s, l


def leading_pair(M):
    n = M.shape[0]
    w, v = sla.eigh(M, subset_by_index=[n - 1, n - 1])
    return float(w[0]), v[:, 0]


def smoothed_energy(J, a, beta):
    Jd, M, s, _ = _parts(J, a)
    lam, y = leading_pair(M)
    t = np.tanh(beta * s * y)
    return float(-0.5 * t @ (Jd @ t))


def _projected_solve(M, lam, y, b):
    """w with (lam I - M) w = (I - y y^T) b and w orthogonal to y (lam I - M + y y^T is regular)."""
    n = M.shape[0]
    pb = b - (y @ b) * y
    A = lam * np.eye(n) - M + np.outer(y, y)
    w = sla.solve(A, pb, assume_a="sym")
    return w - (y @ w) * y


def energy_gradient(J, a, beta):
    """(L, dL/da per vertex, lambda, y) by the adjoint formula."""
    Jd, M, s, l = _parts(J, a)
    lam, y = leading_pair(M)
    x = s * y
    t = np.tanh(beta * x)
    Jt = Jd @ t
    L = float(-0.5 * t @ Jt)
    gx = -beta * (1.0 - t * t) * Jt
    gy = s * gx
    w = _projected_solve(M, lam, y, gy)
    grad = l * (y * (M @ w) + w * (M @ y)) + l * gx * x
    return L, grad, lam, y


def eigvec_tangent(J, alpha):
    """dy/dalpha for a = alpha 1 (orthogonal to y), with (lambda, y)."""
    _, M, s, l = _parts(J, alpha)
    lam, y = leading_pair(M)
    rhs = l * (M @ y) + M @ (l * y)
    return _projected_solve(M, lam, y, rhs), lam, y


def fd_alpha(J, alpha, beta, h=1e-5):
    return (smoothed_energy(J, alpha + h, beta) - smoothed_energy(J, alpha - h, beta)) / (2 * h)


def fd_direction(J, alpha, v, beta, h=1e-5):
    return (smoothed_energy(J, alpha + h * v, beta) - smoothed_energy(J, alpha - h * v, beta)) / (2 * h)
