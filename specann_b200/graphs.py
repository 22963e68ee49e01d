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
