"""NumPy restatement of the reference's guarded local-search policies. TEST INFRASTRUCTURE ONLY.

The checker of the engine's guarded searches (specann_b200/csrc/guard.cu). Each function cites the
reference lines it restates (paths relative to the reference repository):

  * fixed_guard / adaptive_guard: safe_flip_refinement (models/spectral_annealing_safe.py:1035-1335)
    with the paper settings of models/local_search_guards/policies.py:22-38, i.e. its main phase
    (subset 0.9, max_iterations rounds) and final phase (subset 1.0, 25 x 25 rounds), each a loop of
    _run_guarded_phase (:281-797): a Jacobi ("immutable") proposal from the current spins over the
    selected nodes of every active candidate, its exact energy, acceptance only for a strict drop
    (models/safe_update_policy.py:4-29), per-candidate batch adaptation (:68-95) for the adaptive
    guard, and a patience of 3 rounds without acceptance;
  * independent_set: models/local_search_guards/conflict_free.py:80-367, flips restricted to one
    class of the greedy largest-first colouring (models/local_search_guards/common.py:136-159) per
    update, classes in a seeded random order per sweep, candidates retired after a sweep without
    flips;
  * sequential_oracle: models/local_search_guards/sequential_oracle.py:26-219, exact one-flip
    steepest descent (the first node of least energy change per step).

Differences from the reference, shared by the engine: node selection comes from this project's
counter-based stream (oracle.selection; the reference draws cp.random permutations), and decisions
use exact integer gains for integer couplings (the reference proposes with fp32 sums of J / c, so a
zero gain can round either way). With integer couplings the acceptance test
delta < -(1e-10 + 1e-12 max(1, |E|)) on energies in units of J / c is delta_int < 0 whenever
|E| / c < 1e10.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import scipy.sparse as sp

from . import selection
from .specann_oracle import integer_energies, is_integer_matrix

ABS_TOL, REL_TOL = 1e-10, 1e-12     # models/local_search_guards/policies.py:28-29
PATIENCE = 3                          # :32
MIN_FRACTION, SHRINK, GROWTH = 0.01, 0.5, 1.25   # :33-35


@dataclass
class GuardResult:
    spins: np.ndarray          # k x n int8
    energies: np.ndarray       # k energies of the refined spins (-1/2 s^T J s)
    rounds: int                # main-phase rounds (the policy's reported iterations)
    final_rounds: int
    accepted: int              # accepted candidate updates
    rejected: int


def _fields(J, S):
    """Couplings (int64 for integer J, else float64) and the fields H = J S (n x k)."""
    if is_integer_matrix(J):
        Jw = sp.csr_matrix((np.rint(J.data).astype(np.int64), J.indices, J.indptr), shape=J.shape)
        Sx = S.T.astype(np.int64)
    else:
        Jw = sp.csr_matrix(J, dtype=np.float64)
        Sx = S.T.astype(np.float64)
    return Jw, Sx, Jw @ Sx


def _tolerance(E_norm):
    """models/safe_update_policy.py:21-25."""
    return ABS_TOL + REL_TOL * np.maximum(1.0, np.abs(E_norm))


def _guarded_phase(Jw, S, H, E, c, seed, stream_base, max_rounds, fraction, adaptive):
    """models/spectral_annealing_safe.py:281-797 (one phase). S, H: n x k (updated in place);
    E: k energies in J units. Returns (rounds, accepted, rejected)."""
    n, k = S.shape
    active = np.ones(k, dtype=bool)
    streak = np.zeros(k, dtype=np.int64)
    frac = np.full(k, float(fraction))
    rounds = acc_n = rej_n = 0
    for r in range(int(max_rounds)):
        if not active.any():
            break
        rounds += 1
        if adaptive:
            counts = np.where(active, np.maximum(1, (frac * n).astype(np.int32)), 0)
        else:
            counts = np.where(active, max(1, int(fraction * n)), 0)
        rank = selection.ranks(n, seed, stream_base + r)
        allowed = rank[:, None] < counts[None, :]
        dec = ((S * H) < 0) & allowed                       # immutable proposal from the current spins
        has = dec.any(axis=0) & active
        dS = np.where(dec, -2 * S, 0)
        dH = Jw @ dS
        # E(S + dS) - E(S) = -(S^T J dS) - 1/2 dS^T J dS  (exact for integer couplings)
        dE = -(S * dH).sum(axis=0) - (dS * dH).sum(axis=0) / 2
        tol = _tolerance(E / c)
        accepted = has & (dE / c < -tol)
        rejected = has & ~accepted
        no_flips = active & ~has
        if accepted.any():
            S[:, accepted] = S[:, accepted] + dS[:, accepted]
            H[:, accepted] = H[:, accepted] + dH[:, accepted]
            E[accepted] = E[accepted] + dE[accepted]
        acc_n += int(accepted.sum())
        rej_n += int(rejected.sum())
        if adaptive:                                       # models/safe_update_policy.py:68-95
            smaller = np.maximum(MIN_FRACTION, frac * SHRINK)
            larger = np.minimum(float(fraction), frac * GROWTH)
            new = np.where(rejected, smaller, frac)
            new = np.where(accepted, larger, new)
            shrunk = rejected & (new < frac)
            frac = np.where(active, new, frac)
            stalled = no_flips | (rejected & ~shrunk)
        else:
            stalled = active & ~accepted
        streak = np.where(active, np.where(accepted, 0, np.where(stalled, streak + 1, 0)), streak)
        active = active & (streak < PATIENCE)
    return rounds, acc_n, rej_n


def guarded_search(J, spins_kn, seed, *, adaptive, max_iterations=1000, subset_fraction=0.9,
                   final_sweep_fraction=1.0, final_sweep_iters=25, num_rounds=25) -> GuardResult:
    """Fixed guard (adaptive=False) or adaptive guard (adaptive=True): models/spectral_annealing_safe.py:
    1035-1335 with models/local_search_guards/safe_common.py:12-41 (per-candidate adaptation, batch
    proposals, immutable semantics, no polish)."""
    S0 = np.asarray(spins_kn)
    Jw, S, H = _fields(J, S0)
    c = float(np.max(np.asarray(abs(J).sum(axis=1)).ravel()))
    E = -(S * H).sum(axis=0) / 2
    r1, a1, j1 = _guarded_phase(Jw, S, H, E, c, seed, 0, max_iterations, subset_fraction, adaptive)
    r2, a2, j2 = _guarded_phase(Jw, S, H, E, c, seed, selection.FINAL_STREAM_BASE,
                                int(final_sweep_iters) * int(num_rounds), final_sweep_fraction, adaptive)
    spins = S.T.astype(np.int8).copy()
    energies = integer_energies(J, spins).astype(np.float64) if is_integer_matrix(J) else E.astype(np.float64)
    return GuardResult(spins=spins, energies=energies, rounds=r1, final_rounds=r2, accepted=a1 + a2,
                       rejected=j1 + j2)


def greedy_coloring(J) -> np.ndarray:
    """Greedy largest-first proper colouring (models/local_search_guards/common.py:136-159): nodes by
    degree descending (ties by index), each given the smallest colour unused by its coloured
    neighbours."""
    A = sp.csr_matrix(J)
    n = A.shape[0]
    deg = np.diff(A.indptr)
    order = np.lexsort((np.arange(n), -deg))
    colors = np.full(n, -1, dtype=np.int32)
    seen = np.full(max(1, n), -1, dtype=np.int64)
    for stamp, v in enumerate(order):
        nb = colors[A.indices[A.indptr[v]:A.indptr[v + 1]]]
        nb = nb[nb >= 0]
        seen[nb] = stamp
        col = 0
        while seen[col] == stamp:
            col += 1
        colors[v] = col
    return colors


def color_sequence(num_colors: int, seed: int, updates: int) -> np.ndarray:
    """Colour class of each update: a fresh permutation of the classes per sweep from
    numpy.random.default_rng(seed) (models/local_search_guards/conflict_free.py:89, :235-236, :317)."""
    rng = np.random.default_rng(int(seed))
    out = []
    while len(out) < updates:
        out.extend(int(x) for x in rng.permutation(num_colors))
    return np.asarray(out[:updates], dtype=np.int32)


def independent_set_search(J, spins_kn, seed, *, max_iterations=1000, final_sweep_iters=25, num_rounds=25):
    """models/local_search_guards/conflict_free.py:80-367: per update, every node of one colour class
    flips in every active candidate where its gain is negative (a class is an independent set, so
    the joint change is the sum of the single ones); after each full sweep of the classes, candidates
    without a flip in it are retired."""
    S0 = np.asarray(spins_kn)
    Jw, S, H = _fields(J, S0)
    n, k = S.shape
    c = float(np.max(np.asarray(abs(J).sum(axis=1)).ravel()))
    colors = greedy_coloring(J)
    ncol = int(colors.max()) + 1 if n else 0
    limit = int(max_iterations) + int(final_sweep_iters) * int(num_rounds)
    seq = color_sequence(ncol, seed, limit)
    E = -(S * H).sum(axis=0) / 2
    active = np.ones(k, dtype=bool)
    sweep_flips = np.zeros(k, dtype=np.int64)
    updates = 0
    for u in range(limit):
        if not active.any():
            break
        updates += 1
        members = colors == seq[u]
        tol = _tolerance(E / c)
        gain = 2 * S * H                                    # energy change of each single flip
        dec = members[:, None] & active[None, :] & (gain / c < -tol[None, :])
        if dec.any():
            dS = np.where(dec, -2 * S, 0)
            dH = Jw @ dS
            E = E + np.where(dec, gain, 0).sum(axis=0)
            S += dS
            H += dH
        sweep_flips += dec.sum(axis=0)
        if (u + 1) % ncol == 0:
            done = (sweep_flips == 0) & active
            active &= ~done
            sweep_flips[:] = 0
    spins = S.T.astype(np.int8).copy()
    energies = integer_energies(J, spins).astype(np.float64) if is_integer_matrix(J) else E.astype(np.float64)
    return GuardResult(spins=spins, energies=energies, rounds=updates, final_rounds=0, accepted=0, rejected=0)


def sequential_oracle(J, spins_kn, max_steps_per_node: int = 100):
    """models/local_search_guards/sequential_oracle.py:26-219: per step and candidate, the single flip
    of least energy change (first node on ties) if it lowers the energy, until none does."""
    S0 = np.asarray(spins_kn)
    Jw, S, H = _fields(J, S0)
    n, k = S.shape
    c = float(np.max(np.asarray(abs(J).sum(axis=1)).ravel()))
    E = -(S * H).sum(axis=0) / 2
    steps = 0
    for _ in range(int(max_steps_per_node) * n):
        gain = 2 * S * H
        best = np.argmin(gain, axis=0)
        bg = gain[best, np.arange(k)]
        imp = bg / c < -_tolerance(E / c)
        if not imp.any():
            break
        steps += 1
        for cand in np.flatnonzero(imp):
            i = best[cand]
            s_old = S[i, cand]
            S[i, cand] = -s_old
            row = slice(Jw.indptr[i], Jw.indptr[i + 1])
            H[Jw.indices[row], cand] += -2 * s_old * Jw.data[row]
            E[cand] += bg[cand]
    spins = S.T.astype(np.int8).copy()
    energies = integer_energies(J, spins).astype(np.float64) if is_integer_matrix(J) else E.astype(np.float64)
    return GuardResult(spins=spins, energies=energies, rounds=steps, final_rounds=0, accepted=steps, rejected=0)
