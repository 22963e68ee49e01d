"""NumPy/SciPy restatement of the reference SpecAnn solver. TEST INFRASTRUCTURE ONLY.

Used by tests/ as the checker of the CUDA path, and by bench.py as the timed CPU baseline (the
reference pipeline run with SciPy eigsh and NumPy local search on host cores). Never imported by
the product package.

Each function cites the reference lines it restates (paths relative to the reference repository).
The eigensolver is SciPy's ARPACK ``eigsh`` on the same shifted operator S_rho; the reference uses
CuPy 13.6.0's thick-restart Lanczos (cupyx.scipy.sparse.linalg.eigsh, called from utils/eigsh.py:12),
which is not importable here, so eigenpairs are compared by eigenvalue and residual, not by
iteration trajectory.

Local search: the reference kernel updates spins in place from concurrent warps
(models/spectral_annealing.py:821-869), so its result depends on thread timing. This project
defines two deterministic pass semantics over the same node-selection stream (``oracle.selection``),
both decided from the spins at the start of the pass:
  * "priority" (default): a selected node that wants to flip (2 s_i (J s)_i < 0) flips unless a
    neighbour that also wants to flip comes earlier in the pass's permutation. The flips of a pass
    form an independent set, so each one lowers the energy by exactly its gain: the pass equals a
    sequential sweep of single flips (the in-order schedule of the reference kernel, with the blocked
    nodes deferred to the next pass). Energy decreases monotonically.
  * "snapshot": every wanting node flips (Jacobi). Adjacent nodes can flip together and undo each
    other, so on dense or large graphs it can oscillate and raise the energy.
``local_search`` implements both; the CUDA kernel matches it bit for bit for integer couplings.
``reference_kernel_pass`` restates the reference kernel's own arithmetic (fp32 lane-strided partial
sums and shuffle tree, in-place updates in warp order) so that differences can be counted.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from . import selection

PRED_MODES = ("diagonal", "secant", "prev")
SCHEDULES = ("sqrt", "linear")


class EigensolverBreakdown(RuntimeError):
    """models/spectral_annealing.py:70-71."""


class NumericalFailure(RuntimeError):
    """utils/failures.py:4-5."""


# ----------------------------------------------------------------------------------------------
# Prelude, schedule, operators, shift
# ----------------------------------------------------------------------------------------------

class ThreadedCSR:
    """Row-block parallel products of a CSR matrix for the timed CPU baseline: SciPy's sparse kernels
    release the GIL, so T row blocks multiplied on T threads use T host cores. Results equal the
    single-threaded product (each row's sum is computed the same way). `data`, `indices`, `indptr`
    and `shape` are those of the whole matrix."""

    def __init__(self, A, threads: int):
        from concurrent.futures import ThreadPoolExecutor
        self.A = sp.csr_matrix(A)
        self.shape, self.dtype = self.A.shape, self.A.dtype
        self.data, self.indices, self.indptr = self.A.data, self.A.indices, self.A.indptr
        n = self.A.shape[0]
        cuts = np.searchsorted(self.A.indptr, np.linspace(0, self.A.nnz, threads + 1)).clip(0, n)
        cuts[0], cuts[-1] = 0, n
        self.blocks = [self.A[a:b] for a, b in zip(cuts[:-1], cuts[1:]) if b > a]
        self.pool = ThreadPoolExecutor(max(1, len(self.blocks)))

    def __matmul__(self, X):
        parts = list(self.pool.map(lambda B: B @ X, self.blocks))
        return np.concatenate(parts, axis=0)


def threaded(A, threads: int):
    """A itself for one thread, else its row-block parallel wrapper."""
    return A if threads <= 1 else ThreadedCSR(A, threads)


@dataclass
class Prelude:
    J: sp.csr_matrix          # couplings in the working dtype (unscaled)
    Js: sp.csr_matrix         # J / c (fp32 division at precision 32)
    deg: np.ndarray           # sum_j |J_ij| in the working dtype
    c: float                  # max degree (normalisation factor)
    d: np.ndarray             # deg / c in the working dtype
    dtype: type
    op: object = None         # J / c for products (a row-block threaded wrapper for the CPU baseline)


def prelude(J, precision: int = 32, threads: int = 1) -> Prelude:
    """models/spectral_annealing.py:270-288: device CSR, absolute degrees, c = max degree, J/c, d."""
    dt = np.float32 if precision == 32 else np.float64
    Jc = sp.csr_matrix(J.astype(dt), dtype=dt)
    Jabs = Jc.copy()
    Jabs.data = np.abs(Jabs.data)
    deg = Jabs @ np.ones(Jc.shape[1], dtype=dt)
    c = deg.max()
    if precision == 32:
        Js = sp.csr_matrix((Jc.data / c, Jc.indices, Jc.indptr), shape=Jc.shape)
    else:
        Js = Jc / c
    d = deg / c
    return Prelude(J=Jc, Js=Js, deg=deg, c=float(c), d=d, dtype=dt, op=threaded(Js, threads))


def alpha_schedule(schedule: str = "sqrt", num_alphas: int = 128, interval=(0.0, 1.0)) -> List[float]:
    """models/spectral_annealing.py:549-555 (t = linspace in float64; alpha = sqrt(t) or t)."""
    t = np.linspace(float(interval[0]), float(interval[1]), int(num_alphas))
    return [float(x) for x in (np.sqrt(t) if schedule == "sqrt" else t)]


def d_inv_sqrt(d: np.ndarray, alpha: float) -> np.ndarray:
    """models/spectral_annealing.py:316 (D = d^alpha) and :34 (1/sqrt(max(D, 1e-12))), in d's dtype."""
    dt = d.dtype
    D = np.power(d, dt.type(alpha))
    return np.reciprocal(np.sqrt(np.maximum(D, dt.type(1e-12))))


def n_alpha_matvec(Js, dis, v):
    """models/spectral_annealing.py:38-41: N v = Dis (Js (Dis v))."""
    return dis * (Js @ (dis * v))


def s_rho_matvec(Js, dis, rho, v):
    """models/spectral_annealing.py:52-53: S v = rho v - N v."""
    return rho * v - n_alpha_matvec(Js, dis, v)


def scaled_operator_f64(J, deg, c, alpha):
    """The exact operator M(alpha) = D^{-a/2} (J/c) D^{-a/2} in float64 (the FP64 reference)."""
    J64 = sp.csr_matrix(J, dtype=np.float64)
    d = np.asarray(deg, dtype=np.float64) / float(c)
    with np.errstate(divide="ignore"):
        D = np.power(d, float(alpha))
    dis = 1.0 / np.sqrt(np.maximum(D, 1e-12))
    return (sp.diags(dis) @ (J64 / float(c)) @ sp.diags(dis)).tocsr(), dis


def gershgorin_bound(d, alpha) -> float:
    """models/spectral_annealing.py:579: g = max d^(1 - alpha)."""
    return float(np.max(np.power(d, d.dtype.type(1.0 - alpha))))


def compute_shift_rho(lambda1_prev, g, eps=1e-3) -> float:
    """models/spectral_annealing.py:56-67."""
    if lambda1_prev is None or not np.isfinite(lambda1_prev) or lambda1_prev <= 0:
        base = g
    else:
        base = max(lambda1_prev, g)
    rho = (1.0 + eps) * base
    if rho <= 0:
        rho = (1.0 + eps) * max(g, 1.0)
    return rho


# ----------------------------------------------------------------------------------------------
# Predictors (utils/predictors.py)
# ----------------------------------------------------------------------------------------------

def diagonal_predictor(y_last, d, delta_alpha, rng):
    """utils/predictors.py:6-26: normalise(max(d, 1e-12)^(delta_alpha/2) * y_last); random if ~0."""
    dt = y_last.dtype
    w = np.power(np.maximum(d, dt.type(1e-12)), dt.type(delta_alpha / 2.0))
    y = w * y_last
    nrm = np.linalg.norm(y)
    if nrm < 1e-12:
        z = rng.standard_normal(y.shape).astype(dt)
        return z / np.linalg.norm(z)
    return y / nrm


def secant_predictor(y_last, y_prev, gamma=1.0):
    """utils/predictors.py:29-56: normalise(y_last + gamma (y_last - sign-aligned y_prev))."""
    if y_prev is None:
        return y_last
    if np.dot(y_last, y_prev) < 0:
        y_prev = -y_prev
    s = y_last - y_prev
    if np.linalg.norm(s) < 1e-12:
        return y_last
    y = y_last + gamma * s
    nrm = np.linalg.norm(y)
    if nrm < 1e-12:
        return y_last
    return y / nrm


# ----------------------------------------------------------------------------------------------
# Eigensolve with predictor, shift, retry and checks
# ----------------------------------------------------------------------------------------------

def eigsh_smallest(matvec, n, v0, tol, maxiter, ncv, rng):
    """Smallest eigenpair of the symmetric operator with SciPy ARPACK in float64 (the reference calls
    CuPy's eigsh(S, k=1, which='SA', tol, maxiter, v0, ncv): models/spectral_annealing.py:671-677)."""
    op = spla.LinearOperator((n, n), matvec=lambda v: np.asarray(matvec(v), dtype=np.float64),
                             dtype=np.float64)
    if v0 is None:
        v0 = rng.standard_normal(n)
    kw = dict(k=1, which="SA", tol=tol, maxiter=maxiter, v0=np.asarray(v0, dtype=np.float64))
    if ncv is not None:
        kw["ncv"] = int(ncv)
    w, v = spla.eigsh(op, **kw)
    return w, v


def check_eigenpair(nu, y, rho, g, shift_eps):
    """models/spectral_annealing.py:679-691."""
    if not np.isfinite(nu):
        raise EigensolverBreakdown(f"non-finite eigenvalue {nu}")
    if not np.all(np.isfinite(y)):
        raise EigensolverBreakdown("non-finite eigenvector")
    lambda1 = rho - nu
    if lambda1 > g * (1.0 + max(0.5 * shift_eps, 1e-5)):
        raise EigensolverBreakdown(f"spurious eigenvalue {lambda1:.6g} above the Gershgorin bound {g:.6g}")


@dataclass
class AlphaResult:
    alpha: float
    lambda1: float
    rho: float
    g: float
    x: np.ndarray             # D^{-1/2} y (rounding vector)
    y: np.ndarray             # unit eigenvector, sign-aligned with y_last
    pred_residual: float
    pred_accepted: Optional[bool]
    retry: bool
    converged: bool
    residual: float


def solve_alpha(pre: Prelude, alpha, alpha_idx, alpha_prev, y_last, y_prev, lambda1_prev, *,
                pred_mode="diagonal", pred_tol=1e-3, shift_eps=1e-3, tol=1e-6, maxiter=1000, ncv=None,
                disable_warm_start=False, rng=None, start_vector=None) -> AlphaResult:
    """models/spectral_annealing.py:568-669 (_solve_eigenvalue_problem_pred), with SciPy's eigsh."""
    rng = rng if rng is not None else np.random.default_rng(0)
    dt = pre.dtype
    n = pre.d.size
    dis = d_inv_sqrt(pre.d, alpha)
    g = gershgorin_bound(pre.d, alpha)
    rho = compute_shift_rho(lambda1_prev, g, eps=shift_eps)

    def s_op(v):
        return s_rho_matvec(pre.op, dis, dt(rho), np.asarray(v, dtype=dt))

    pred_residual, pred_accepted = float("nan"), None
    if alpha_idx == 0 or disable_warm_start or y_last is None:
        y_init = (start_vector if start_vector is not None else rng.standard_normal(n)).astype(dt)
        y_init = y_init / np.linalg.norm(y_init)
    elif pred_mode == "prev":
        y_init = y_last
    else:
        delta = alpha - alpha_prev if alpha_prev is not None else 0.0
        if pred_mode == "diagonal":
            y_init = diagonal_predictor(y_last, pre.d, delta, rng)
        else:
            y_init = secant_predictor(y_last, y_prev)
        v = n_alpha_matvec(pre.op, dis, y_init)
        lam = float(np.dot(y_init, v))
        r = float(np.linalg.norm(v - lam * y_init))
        pred_residual, pred_accepted = r, not r > pred_tol
        if r > pred_tol:
            y_init = y_last

    retry = False
    try:
        w, Y = eigsh_smallest(s_op, n, y_init.copy(), tol, maxiter, ncv, rng)
        check_eigenpair(float(w[0]), Y, rho, g, shift_eps)
    except Exception:
        retry = True
        w, Y = eigsh_smallest(s_op, n, None, tol, maxiter, ncv, rng)
        check_eigenpair(float(w[0]), Y, rho, g, shift_eps)
    y = Y[:, 0].astype(dt)
    mu = float(w[0])
    resid = float(np.linalg.norm(s_op(y) - dt(mu) * y) / np.linalg.norm(y))
    converged = resid <= tol
    lambda1 = rho - mu
    if y_last is not None and float(np.dot(y, y_last)) < 0:
        y = -y
    nrm = np.linalg.norm(y)
    if nrm > 0:
        y = y / nrm
    x = y * dis
    return AlphaResult(alpha, lambda1, rho, g, x, y, pred_residual, pred_accepted, retry, converged, resid)


# ----------------------------------------------------------------------------------------------
# Rounding, signatures, energies
# ----------------------------------------------------------------------------------------------

def round_spins(x) -> np.ndarray:
    """models/spectral_annealing.py:345: +1 where x >= 0, else -1 (int8 here)."""
    return np.where(np.asarray(x) >= 0, 1, -1).astype(np.int8)


def signature(spins) -> bytes:
    """models/spectral_annealing.py:557-561: packbits(spins > 0) bytes (big-endian bit order)."""
    return np.packbits((np.asarray(spins) > 0).astype(np.uint8)).tobytes()


def pack_words(spins) -> np.ndarray:
    """Device layout of a rounded candidate: bit (j % 32) of uint32 word j // 32 is 1 iff s_j > 0."""
    s = np.asarray(spins)
    n = s.size
    nw = (n + 31) // 32
    bits = np.zeros(nw * 32, dtype=np.uint64)
    bits[:n] = (s > 0)
    bits = bits.reshape(nw, 32)
    return (bits << np.arange(32, dtype=np.uint64)).sum(axis=1).astype(np.uint32)


def unpack_words(words, n) -> np.ndarray:
    w = np.asarray(words, dtype=np.uint32).astype(np.uint64)
    bits = (w[:, None] >> np.arange(32, dtype=np.uint64)) & np.uint64(1)
    return np.where(bits.reshape(-1)[:n] == 1, 1, -1).astype(np.int8)


def exact_energy(J, spins) -> float:
    """E = -1/2 s^T J s in float64 from the input J (models/spectral_annealing.py:484-488)."""
    s = np.asarray(spins, dtype=np.float64)
    return float(-0.5 * s @ (sp.csr_matrix(J, dtype=np.float64) @ s))


def integer_energies(J, spins_kn) -> np.ndarray:
    """-1/2 s^T J s exactly (int64) for integer couplings; spins_kn is k x n."""
    Ji = sp.csr_matrix((np.rint(J.data).astype(np.int64), J.indices, J.indptr), shape=J.shape)
    S = np.asarray(spins_kn, dtype=np.int64).T
    H = Ji @ S
    return -(S * H).sum(axis=0) // 2


def fp32_energies(Js, spins_kn, c) -> np.ndarray:
    """models/spectral_annealing.py:925-976: fp32 couplings, fp64 accumulation per row, times -c/2."""
    S = np.asarray(spins_kn, dtype=np.float64).T
    H = sp.csr_matrix(Js, dtype=np.float64) @ S
    return -0.5 * c * (S * H).sum(axis=0)


# ----------------------------------------------------------------------------------------------
# Local search
# ----------------------------------------------------------------------------------------------

@dataclass
class LSResult:
    spins: np.ndarray         # k x n int8
    iterations: int           # main-loop passes (max_iters_used)
    energies_before: np.ndarray
    energies_after: np.ndarray
    flips: int


def is_integer_matrix(J) -> bool:
    data = np.asarray(J.data, dtype=np.float64)
    return bool(np.all(np.isfinite(data)) and np.all(data == np.rint(data)))


def local_search(J, spins_kn, seed: int, max_iterations: int = 1000, subset_fraction: float = 0.9,
                 final_sweep_fraction: float = 1.0, final_sweep_iters: int = 25,
                 num_rounds: int = 25, semantics: str = "priority", threads: int = 1) -> LSResult:
    """Batched local search with the control flow of flip_refinement and gpu_final_sweep
    (models/spectral_annealing.py:1039-1112, :983-1036).

    A pass over the selected nodes decides, from the spins at the start of the pass, which
    (node, candidate) pairs want to flip (energy change 2 s_i (J s)_i < 0); with "priority" a wanting
    node is held back when a wanting neighbour has a lower rank in the pass's permutation, with
    "snapshot" every wanting node flips. A candidate has a flip in a pass iff it has a wanting node
    (the lowest-ranked wanting node is never held back), so the stopping rules are those of the
    reference: the main loop stops when every candidate has had a pass without a flip (sticky mask,
    :1096-1100) or after max_iterations passes; then num_rounds rounds of up to final_sweep_iters
    passes, each round ending at the first pass in which no candidate flips (:1023-1034).
    """
    if semantics not in ("priority", "snapshot"):
        raise ValueError(semantics)
    S = np.asarray(spins_kn, dtype=np.int64).T.copy()      # n x k
    n, k = S.shape
    integer = is_integer_matrix(J)
    if integer:
        Jw = sp.csr_matrix((np.rint(J.data).astype(np.int64), J.indices, J.indptr), shape=J.shape)
    else:
        Jw = sp.csr_matrix(J, dtype=np.float64)
        S = S.astype(np.float64)
    Jw = threaded(Jw, threads)
    H = Jw @ S
    e_before = -(S * H).sum(axis=0)
    e_before = e_before // 2 if integer else 0.5 * e_before
    total = [0]
    coo = sp.csr_matrix(J).tocoo()

    def one_pass(sel, rank):
        nonlocal S, H
        dec = ((S * H) < 0) & sel[:, None]
        if semantics == "priority" and dec.any():
            earlier = rank[coo.col] < rank[coo.row]
            P = sp.csr_matrix((np.ones(int(earlier.sum())), (coo.row[earlier], coo.col[earlier])), shape=J.shape)
            blocked = (P @ dec.astype(np.float64)) > 0
            dec = dec & ~blocked
        counts = dec.sum(axis=0)
        if dec.any():
            dS = np.where(dec, -2 * S, 0)
            H = H + (Jw @ dS if integer else Jw @ dS.astype(np.float64))
            S = np.where(dec, -S, S)
            total[0] += int(counts.sum())
        return counts

    active = np.ones(k, dtype=bool)
    used = 0
    m_main = selection.num_selected(n, subset_fraction)
    for it in range(int(max_iterations)):
        used += 1
        rank = selection.ranks(n, seed, it)
        counts = one_pass(rank < m_main, rank)
        active &= counts > 0
        if not active.any():
            break
    m_final = selection.num_selected(n, final_sweep_fraction)
    for r in range(int(num_rounds)):
        rank = selection.ranks(n, seed, selection.FINAL_STREAM_BASE + r)
        sel = rank < m_final
        for _ in range(int(final_sweep_iters)):
            counts = one_pass(sel, rank)
            if not (counts > 0).any():
                break
    e_after = -(S * H).sum(axis=0)
    e_after = e_after // 2 if integer else 0.5 * e_after
    return LSResult(spins=S.T.astype(np.int8).copy(), iterations=used, energies_before=e_before,
                    energies_after=e_after, flips=total[0])


def _warp_sum_f32(vals: np.ndarray) -> np.float32:
    """fp32 sum in the order of the reference kernel: lane l accumulates elements l, l+32, ...,
    then __shfl_down_sync with offsets 16, 8, 4, 2, 1 (models/spectral_annealing.py:846-856)."""
    lanes = np.zeros(32, dtype=np.float32)
    for idx in range(vals.size):
        lanes[idx % 32] = np.float32(lanes[idx % 32] + vals[idx])
    off = 16
    while off > 0:
        lanes[:off] = (lanes[:off] + lanes[off:2 * off]).astype(np.float32)
        off //= 2
    return lanes[0]


def reference_kernel_pass(Js32, spins_kn, selected_nodes) -> np.ndarray:
    """One launch of update_spins_kernel_float32 (models/spectral_annealing.py:821-869) executed with
    warps in order (one legal schedule of the racy kernel): in place, fp32 arithmetic as the kernel
    does it. Returns the per-candidate flip counts; spins_kn (k x n int8) is updated in place."""
    k = spins_kn.shape[0]
    counts = np.zeros(k, dtype=np.int64)
    indptr, indices, data = Js32.indptr, Js32.indices, Js32.data.astype(np.float32)
    for node in np.asarray(selected_nodes):
        a, b = indptr[node], indptr[node + 1]
        for s in range(k):
            prod = (data[a:b] * spins_kn[s, indices[a:b]].astype(np.float32)).astype(np.float32)
            local = _warp_sum_f32(prod)
            si = spins_kn[s, node]
            delta = np.float32(2.0) * np.float32(si) * local
            if delta < 0:
                spins_kn[s, node] = -si
                counts[s] += 1
    return counts


def _reference_pass_all(Js32, Ji, S, order):
    """reference_kernel_pass for all candidates at once (S: k x n int8, updated in place), also
    comparing each decision with the exact integer gain at the same moment. Returns (flips per
    candidate, decisions whose fp32 sign differs from the exact gain's)."""
    k = S.shape[0]
    flips = np.zeros(k, dtype=np.int64)
    ties = 0
    ip, ix = Js32.indptr, Js32.indices
    dat = Js32.data.astype(np.float32)
    idat = Ji.data
    for node in order:
        a, b = ip[node], ip[node + 1]
        cols = ix[a:b]
        sv = S[:, cols]
        prod = dat[a:b][None, :] * sv.astype(np.float32)
        lanes = np.zeros((k, 32), dtype=np.float32)
        for e in range(b - a):                      # lane e % 32 accumulates in entry order
            lanes[:, e % 32] += prod[:, e]
        off = 16
        while off > 0:                               # __shfl_down_sync 16, 8, 4, 2, 1
            lanes[:, :off] = lanes[:, :off] + lanes[:, off:2 * off]
            off //= 2
        si = S[:, node].astype(np.float32)
        delta = np.float32(2.0) * si * lanes[:, 0]
        flip = delta < 0
        exact = 2 * S[:, node].astype(np.int64) * (sv.astype(np.int64) @ idat[a:b])
        ties += int(np.sum(flip != (exact < 0)))
        S[flip, node] = -S[flip, node]
        flips += flip
    return flips, ties


@dataclass
class LSDeviation:
    passes: int                    # main-loop passes compared
    decisions: int                 # (selected node, candidate) decisions per pass, summed
    schedule_differences: int      # decisions where the in-order in-place pass and the priority pass differ
    arithmetic_differences: int    # in-order decisions whose fp32 sign differs from the exact integer gain
    energy_reference: np.ndarray   # final energies of the in-order search (k)
    energy_priority: np.ndarray    # final energies of the priority search (k)


def ls_deviation(J, spins_kn, seed: int, max_passes: int = 1000, subset_fraction: float = 0.9) -> LSDeviation:
    """How the engine's local search departs from the reference kernel's (integer couplings).

    Both run the main loop of flip_refinement (models/spectral_annealing.py:1039-1100) over the same
    node-selection stream. Per pass, from the same starting spins, the decisions of one in-order
    in-place launch of update_spins_kernel_float32 (fp32 lane-strided sums and shuffle tree,
    :821-869, warps in rank order) are compared with the priority pass's, and every in-order decision
    is compared with the sign of the exact integer gain at that moment. Then each search continues on
    its own trajectory until it stops (sticky active mask) or max_passes; their final energies are
    returned. The final sweep is not included."""
    pre = prelude(J, 32)
    Ji = sp.csr_matrix((np.rint(J.data).astype(np.int64), J.indices, J.indptr), shape=J.shape)
    S0 = np.asarray(spins_kn, dtype=np.int8)
    k, n = S0.shape
    m = selection.num_selected(n, subset_fraction)
    coo = sp.csr_matrix(J).tocoo()
    S_ref = S0.copy()
    S_pri = S0.T.astype(np.int64).copy()            # n x k
    H_pri = Ji @ S_pri
    act_ref = np.ones(k, dtype=bool)
    act_pri = np.ones(k, dtype=bool)
    sched = arith = decisions = 0
    passes = 0
    for it in range(int(max_passes)):
        if not act_ref.any() and not act_pri.any():
            break
        passes += 1
        rank = selection.ranks(n, seed, it)
        sel = rank < m
        order = np.argsort(rank)[:m]
        # priority decisions from the snapshot
        dec = ((S_pri * H_pri) < 0) & sel[:, None]
        if dec.any():
            earlier = rank[coo.col] < rank[coo.row]
            P = sp.csr_matrix((np.ones(int(earlier.sum())), (coo.row[earlier], coo.col[earlier])), shape=J.shape)
            dec = dec & ~((P @ dec.astype(np.float64)) > 0)
        # the in-order pass from the same spins, to count schedule differences
        S_cmp = S_pri.T.astype(np.int8).copy()
        before = S_cmp.copy()
        _, t_cmp = _reference_pass_all(pre.Js, Ji, S_cmp, order)
        ref_dec = (S_cmp != before).T
        sched += int(np.sum(ref_dec != dec))
        decisions += m * k
        # advance both trajectories
        if act_ref.any():
            f, t = _reference_pass_all(pre.Js, Ji, S_ref, order)
            arith += t
            act_ref &= f > 0
        if act_pri.any():
            cnt = dec.sum(axis=0)
            if dec.any():
                dS = np.where(dec, -2 * S_pri, 0)
                H_pri = H_pri + Ji @ dS
                S_pri = np.where(dec, -S_pri, S_pri)
            act_pri &= cnt > 0
    e_ref = integer_energies(J, S_ref)
    e_pri = integer_energies(J, S_pri.T)
    return LSDeviation(passes=passes, decisions=decisions, schedule_differences=sched,
                       arithmetic_differences=arith, energy_reference=e_ref, energy_priority=e_pri)


# ----------------------------------------------------------------------------------------------
# Full solver (SpectralAnnealing.solve)
# ----------------------------------------------------------------------------------------------

@dataclass
class SolveResult:
    best_energy: float
    best_spins: np.ndarray
    best_alpha: Optional[float]
    alphas: List[float]
    records: List[dict] = field(default_factory=list)
    candidates: List[np.ndarray] = field(default_factory=list)
    ls: Optional[LSResult] = None


def solve(J, *, precision=32, schedule="sqrt", num_alphas=128, schedule_interval=(0.0, 1.0),
          pred_mode="diagonal", pred_tol=1e-3, shift_eps=1e-3, eigsh_tol=1e-6, eigsh_maxiter=1000,
          eigsh_ncv=None, disable_warm_start=False, use_local_search=True, max_local_iterations=1000,
          seed=42, alpha_subset=None, ls_semantics="priority", energy_mode="exact", threads=1) -> SolveResult:
    """models/spectral_annealing.py:262-525 with SciPy eigsh and the priority local search.

    ``alpha_subset`` (indices into the schedule) runs only those alphas, in order; the warm-start
    chain then links consecutive listed alphas. ``threads`` > 1 runs the sparse products on that
    many host threads (row blocks; same results).
    """
    rng = np.random.default_rng(seed)
    pre = prelude(J, precision, threads=threads)
    alphas = alpha_schedule(schedule, num_alphas, schedule_interval)
    order = list(range(len(alphas))) if alpha_subset is None else list(alpha_subset)
    y_last = y_prev = None
    lambda1_prev = alpha_prev = None
    records, uniq, cand_list = [], {}, []
    best_e, best_s, best_a = float("inf"), None, None
    for pos, ai in enumerate(order):
        alpha = alphas[ai]
        try:
            res = solve_alpha(pre, alpha, pos, alpha_prev, y_last, y_prev, lambda1_prev,
                              pred_mode=pred_mode, pred_tol=pred_tol, shift_eps=shift_eps, tol=eigsh_tol,
                              maxiter=eigsh_maxiter, ncv=eigsh_ncv, disable_warm_start=disable_warm_start,
                              rng=rng)
        except Exception:
            continue
        if not disable_warm_start:
            y_prev, y_last = y_last, res.y
            lambda1_prev, alpha_prev = res.lambda1, alpha
        spins = round_spins(res.x)
        key = signature(spins)
        if key not in uniq:
            uniq[key] = len(cand_list)
            cand_list.append(spins)
        if energy_mode == "exact":
            raw = exact_energy(J, spins)
        elif precision == 32:
            raw = float(fp32_energies(pre.Js, spins[None, :], pre.c)[0])
        else:
            raw = float(-0.5 * pre.c * spins.astype(np.float64) @ (pre.Js @ spins.astype(np.float64)))
        records.append(dict(alpha=alpha, lambda1=res.lambda1, rho=res.rho, candidate=uniq[key],
                            raw_energy=raw, energy=raw, pred_residual=res.pred_residual,
                            pred_accepted=res.pred_accepted, retry=res.retry, residual=res.residual))
        if raw < best_e:
            best_e, best_s, best_a = raw, spins.copy(), alpha
    ls = None
    if use_local_search and cand_list:
        ls = local_search(J, np.stack(cand_list), seed=seed, max_iterations=max_local_iterations,
                          semantics=ls_semantics, threads=threads)
        for rec in records:
            c = rec["candidate"]
            orig = rec["raw_energy"]
            refined = float(ls.energies_after[c])
            improved = orig if refined > orig else refined
            rec["energy"] = improved
            rec["refined"] = not refined > orig
        for rec in records:
            if rec["energy"] < best_e:
                best_e, best_a = rec["energy"], rec["alpha"]
                best_s = ls.spins[rec["candidate"]].copy() if rec["refined"] else cand_list[rec["candidate"]]
    if best_s is not None:
        best_e = exact_energy(J, best_s)
    return SolveResult(best_energy=best_e, best_spins=best_s, best_alpha=best_a, alphas=alphas,
                       records=records, candidates=cand_list, ls=ls)
