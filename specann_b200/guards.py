"""Guarded local-search policies (ls_policy other than "default") for the solver classes: the
refiners of models/local_search_guards/policies.py:13-69 on the engine's kernels (sa_guard_search).

Policy names and iteration counts follow the reference (run_policy, policies.py:41-52): the guards
report their main-phase rounds, the independent set its updates and the oracle its steps. The
independent set's colouring (greedy largest-first, models/local_search_guards/common.py:136-159) is
computed on the host by the native host library, and its class order per sweep by
numpy.random.default_rng(seed) as in models/local_search_guards/conflict_free.py:89, :235-236.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib

POLICIES = {"fixed_guard": _lib.SA_GUARD_FIXED, "adaptive_guard": _lib.SA_GUARD_ADAPTIVE,
            "independent_set": _lib.SA_GUARD_INDEPENDENT_SET, "sequential_oracle": _lib.SA_GUARD_SEQUENTIAL}


def greedy_coloring(indptr: np.ndarray, indices: np.ndarray):
    """(colours int32[n], number of colours) of the CSR graph."""
    g = _lib.load_graphs()
    n = indptr.size - 1
    rp = np.ascontiguousarray(indptr, dtype=np.int64)
    col = np.ascontiguousarray(indices, dtype=np.int32)
    colors = np.empty(max(n, 1), dtype=np.int32)
    k = C.c_int32(0)
    st = g.sa_greedy_coloring(int(n), rp.ctypes.data_as(C.c_void_p), col.ctypes.data_as(C.c_void_p),
                              colors.ctypes.data_as(C.c_void_p), C.byref(k))
    if st != 0:
        raise ValueError("greedy colouring failed (invalid CSR)")
    return colors[:n], int(k.value)


def color_sequence(num_colors: int, seed: int, updates: int) -> np.ndarray:
    """Colour class of each update: one permutation of the classes per sweep."""
    rng = np.random.default_rng(int(seed))
    out = []
    while len(out) < updates:
        out.extend(int(x) for x in rng.permutation(num_colors))
    return np.asarray(out[:max(updates, 1)], dtype=np.int32)


def run_policy(engine, policy: str, k: int, *, max_iterations: int, seed: int, indptr=None, indices=None):
    """Refine candidate slots 0 .. k-1 with a guarded policy. Returns (energies before, energies
    after, iterations as the reference reports them, GuardResult)."""
    code = POLICIES[policy]
    extra = {}
    if code == _lib.SA_GUARD_INDEPENDENT_SET:
        colors, ncol = greedy_coloring(indptr, indices)
        seq = color_sequence(ncol, seed, int(max_iterations) + 25 * 25)
        extra = dict(colors=torch.from_numpy(colors).to(engine.device),
                     color_seq=torch.from_numpy(seq).to(engine.device), num_colors=ncol)
    eb, ea, res = engine.guard_search(code, k, max_iterations=max_iterations, seed=seed, **extra)
    if res.status not in (_lib.SA_OK, _lib.SA_ERR_NOT_CONVERGED):
        _lib.check("sa_guard_search", res.status)
    return eb, ea, int(res.rounds), res
