"""Seeded synthetic Ising instances (Barabasi-Albert, Erdos-Renyi) as SciPy CSR matrices.

Host C++ generators in libspecann_graphs.so (specann_b200/csrc/graphgen.cpp). Couplings:
  "unit"  J = -A (MaxCut weights), "pm1" +-1 from a fair coin per undirected edge,
  "int100" nonzero integers uniform in [-100, 100].
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import scipy.sparse as sp

from . import _lib

MODES = {"unit": 0, "pm1": 1, "int100": 2}


def _csr(n, nnz, fill):
    rowptr = np.empty(n + 1, dtype=np.int64)
    col = np.empty(nnz, dtype=np.int32)
    val = np.empty(nnz, dtype=np.float32)
    st = fill(rowptr.ctypes.data_as(C.c_void_p), col.ctypes.data_as(C.c_void_p), val.ctypes.data_as(C.c_void_p))
    if st != 0:
        raise ValueError("graph generation failed")
    return rowptr, col, val


def barabasi_albert_arrays(n: int, m: int, seed: int = 42, couplings: str = "unit"):
    """(rowptr int64, col int32, val float32) of a seeded BA(n, m) graph with 2 m (n - m) entries."""
    g = _lib.load_graphs()
    nnz = int(g.sa_graph_ba_nnz(int(n), int(m)))
    if nnz < 0:
        raise ValueError(f"invalid BA size n={n}, m={m}")
    return _csr(n, nnz, lambda r, c, v: g.sa_graph_ba(int(n), int(m), int(seed) & (2 ** 64 - 1), MODES[couplings], r, c, v))


def erdos_renyi_arrays(n: int, p: float, seed: int = 42, couplings: str = "unit"):
    g = _lib.load_graphs()
    nnz = int(g.sa_graph_er_nnz(int(n), float(p), int(seed) & (2 ** 64 - 1)))
    if nnz < 0:
        raise ValueError(f"invalid ER size n={n}, p={p}")
    return _csr(n, nnz, lambda r, c, v: g.sa_graph_er(int(n), float(p), int(seed) & (2 ** 64 - 1), MODES[couplings], r, c, v))


def to_scipy(rowptr, col, val, n, dtype=np.float64) -> sp.csr_matrix:
    idx = rowptr if rowptr[-1] > np.iinfo(np.int32).max else rowptr.astype(np.int32)
    return sp.csr_matrix((val.astype(dtype, copy=False), col, idx), shape=(n, n))


def barabasi_albert(n: int, m: int, seed: int = 42, couplings: str = "unit", dtype=np.float64) -> sp.csr_matrix:
    return to_scipy(*barabasi_albert_arrays(n, m, seed, couplings), n, dtype)


def erdos_renyi(n: int, p: float, seed: int = 42, couplings: str = "unit", dtype=np.float64) -> sp.csr_matrix:
    return to_scipy(*erdos_renyi_arrays(n, p, seed, couplings), n, dtype)


def drop_isolated(J: sp.csr_matrix) -> sp.csr_matrix:
    """Remove all-zero rows/columns (the reference loader does this, utils/data_loader.py:180-204)."""
    keep = np.flatnonzero(np.diff(J.indptr) > 0)
    if keep.size == J.shape[0]:
        return J
    return J[keep][:, keep].tocsr()


def ragged_batch(count: int = 64, seed: int = 2025, log2_min: int = 10, log2_max: int = 17):
    """The batched ragged workload: `count` instances with n log-uniform in [2^log2_min, 2^log2_max]
    (seeded); even-numbered ones Erdos-Renyi with expected degree 20, odd-numbered ones
    Barabasi-Albert with m = 10 or 20; +-1 couplings from a fair coin per undirected edge; isolated
    nodes removed. Returns a list of (name, CSR)."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(2.0 ** log2_min), np.log(2.0 ** log2_max), count)).astype(np.int64)
    ms = np.where(rng.random(count) < 0.5, 10, 20)
    out = []
    for i in range(count):
        n = int(sizes[i])
        gseed = int(rng.integers(1, 2 ** 62))
        if i % 2 == 0:
            J = erdos_renyi(n, 20.0 / (n - 1), seed=gseed, couplings="pm1")
            name = f"er_{n}_{i}"
        else:
            J = barabasi_albert(n, int(ms[i]), seed=gseed, couplings="pm1")
            name = f"ba_{n}_m{int(ms[i])}_{i}"
        out.append((name, drop_isolated(J)))
    return out
