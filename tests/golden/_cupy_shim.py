"""A NumPy/SciPy stand-in for the parts of CuPy 13.6 that the reference solvers use.

Fixture generation only (tests/golden/make_golden.py): it lets the reference's own solver files run
on the CPU of this container, where CuPy is absent, so that their outputs can be frozen as golden
vectors. Nothing in the product or in the GPU tests imports it.

What it stands in for, and how:
  * cupy array functions -> numpy (module __getattr__); cupy.random -> one numpy RandomState
    seeded by cupy.random.seed (so runs are reproducible, but the stream is not CuPy's);
  * cupyx.scipy.sparse -> scipy.sparse;
  * cupyx.scipy.sparse.linalg.eigsh -> SciPy ARPACK eigsh run in float64 on the operator and cast
    back to the operator's dtype (stock CuPy's eigsh returns two values, so the solvers take the
    "iteration count unknown" branch of utils/eigsh.py);
  * cupy.RawKernel -> NumPy executions of the reference kernels by name: the local-search update
    kernels run their warps one after another in launch order (a legal schedule of the racy
    in-place kernel, fp32 partial sums in the kernel's lane/shuffle order); the fp32 energy kernel
    keeps its float64 accumulation;
  * cupy.ElementwiseKernel -> the in-place row/column scaling of models/spec_signed_lap.py.
"""
import sys
import types

import numpy as np
import scipy.sparse as _sp
import scipy.sparse.linalg as _spla

LOG = {"ls_passes": []}      # filled by the update-kernel emulation when recording is on
RECORD_LS = [False]


class _Random:
    def __init__(self):
        self.rs = np.random.RandomState(0)

    def seed(self, s=None):
        self.rs = np.random.RandomState(None if s is None else int(s) % (2 ** 32))

    def randn(self, *shape):
        return self.rs.standard_normal(shape)

    def permutation(self, n):
        return self.rs.permutation(n)

    def random(self, size=None, dtype=np.float64):
        return self.rs.random_sample(size).astype(dtype)


def _lane_tree_sum(prod, dtype):
    """Rows of prod (k x L) summed as a warp does: lane l accumulates l, l+32, ... in order, then a
    shuffle-down tree with offsets 16, 8, 4, 2, 1."""
    k, L = prod.shape
    R = (L + 31) // 32
    pad = np.zeros((k, R * 32), dtype=dtype)
    pad[:, :L] = prod
    pad = pad.reshape(k, R, 32)
    lanes = np.zeros((k, 32), dtype=dtype)
    for r in range(R):
        lanes = (lanes + pad[:, r, :]).astype(dtype)
    off = 16
    while off > 0:
        lanes[:, :off] = (lanes[:, :off] + lanes[:, off:2 * off]).astype(dtype)
        off //= 2
    return lanes[:, 0]


def _update_spins(args, dtype):
    n_selected, n, k, selected, indptr, indices, data, spins, counts = args
    flat = spins.reshape(-1)
    data = np.asarray(data, dtype=dtype)
    sel = np.asarray(selected)[: int(n_selected)]
    before = flat.copy() if RECORD_LS[0] else None
    S = flat.reshape(int(k), int(n))
    for node in sel:
        a, b = indptr[node], indptr[node + 1]
        if b > a:
            prod = (data[a:b][None, :] * S[:, indices[a:b]].astype(dtype)).astype(dtype)
            local = _lane_tree_sum(prod, dtype)
        else:
            local = np.zeros(int(k), dtype=dtype)
        si = S[:, node].astype(dtype)
        delta = (dtype(2.0) * si * local).astype(dtype)
        flip = delta < 0
        S[flip, node] = -S[flip, node]
        counts[: int(k)] += flip.astype(counts.dtype)
    if RECORD_LS[0]:
        LOG["ls_passes"].append((sel.copy(), before.reshape(int(k), int(n)), S.copy()))


def _energy_rows(grid, block, args):
    n, indptr, indices, data, S, block_sums = args
    S = np.asarray(S)
    n = int(n)
    k = S.shape[1] if S.ndim == 2 else 1
    cols = S.reshape(n, k, order="F") if S.ndim == 2 else S.reshape(n, 1)
    wpb = int(block[1])
    gx = int(grid[0])
    data = np.asarray(data, dtype=np.float32).astype(np.float64)
    for c in range(k):
        s = cols[:, c].astype(np.float64)
        row_acc = np.zeros(n, dtype=np.float64)
        for row in range(n):
            a, b = indptr[row], indptr[row + 1]
            if b > a:
                prod = data[a:b] * s[indices[a:b]]
                row_acc[row] = _lane_tree_sum(prod[None, :], np.float64)[0]
        vals = row_acc * s
        for bx in range(gx):
            acc = 0.0
            for w in range(wpb):
                r = bx * wpb + w
                acc += vals[r] if r < n else 0.0
            block_sums[c, bx] = acc


class RawKernel:
    def __init__(self, code, name, *a, **kw):
        self.name = name

    def __call__(self, grid, block, args, **kw):
        if self.name in ("update_spins_kernel_float32", "update_spins_kernel"):
            return _update_spins(args, np.float32)
        if self.name == "update_spins_kernel_float64":
            return _update_spins(args, np.float64)
        if self.name == "energy_rows_kernel_float32":
            return _energy_rows(grid, block, args)
        raise NotImplementedError(f"kernel {self.name} is not emulated")


class ElementwiseKernel:
    def __init__(self, in_params, out_params, operation, name, *a, **kw):
        self.name = name

    def __call__(self, indptr, indices, d, data, size=None):
        if self.name != "specsignedlap_scale_rows_and_columns":
            raise NotImplementedError(self.name)
        dt = data.dtype.type
        for i in range(int(size)):
            di = d[i]
            for k in range(indptr[i], indptr[i + 1]):
                data[k] = dt(dt(di * data[k]) * d[indices[k]])
        return data


class _Pool:
    def total_bytes(self):
        return 0


class _Event:
    def record(self, *a, **k):
        pass

    def synchronize(self):
        pass


def _eigsh(A, k=6, which="LM", v0=None, ncv=None, maxiter=None, tol=0, return_eigenvectors=True):
    n = A.shape[0]
    dt = np.dtype(A.dtype)
    if _sp.issparse(A):
        A64 = A.astype(np.float64)
        op = _spla.aslinearoperator(A64)
    else:
        op = _spla.LinearOperator((n, n), dtype=np.float64,
                                  matvec=lambda v: np.asarray(A.matvec(np.asarray(v, dtype=dt)),
                                                              dtype=np.float64))
    if v0 is None:
        v0 = _random.rs.standard_normal(n)
    kw = dict(k=k, which=which, tol=tol, v0=np.asarray(v0, dtype=np.float64))
    if maxiter is not None:
        kw["maxiter"] = maxiter
    if ncv is not None:
        kw["ncv"] = ncv
    w, v = _spla.eigsh(op, **kw)
    return w.astype(dt), v.astype(dt)


_random = _Random()


def install():
    """Register cupy, cupyx, cupyx.scipy, cupyx.scipy.sparse(.linalg) in sys.modules."""
    cp = types.ModuleType("cupy")

    def _getattr(name):
        return getattr(np, name)

    cp.__getattr__ = _getattr
    cp.random = _random
    cp.RawKernel = RawKernel
    cp.ElementwiseKernel = ElementwiseKernel
    cp.asnumpy = lambda x, *a, **k: np.asarray(x)
    cp.get_default_memory_pool = lambda: _Pool()
    cp.get_default_pinned_memory_pool = lambda: _Pool()
    cuda = types.SimpleNamespace(
        Stream=types.SimpleNamespace(null=types.SimpleNamespace(synchronize=lambda: None)),
        Event=_Event, get_elapsed_time=lambda a, b: 0.0)
    cp.cuda = cuda
    cp.ndarray = np.ndarray

    cupyx = types.ModuleType("cupyx")
    cscipy = types.ModuleType("cupyx.scipy")
    csparse = types.ModuleType("cupyx.scipy.sparse")
    for name in ("csr_matrix", "identity", "diags", "coo_matrix", "issparse"):
        setattr(csparse, name, getattr(_sp, name))
    clinalg = types.ModuleType("cupyx.scipy.sparse.linalg")
    clinalg.LinearOperator = _spla.LinearOperator
    clinalg.eigsh = _eigsh
    cupyx.scipy = cscipy
    cscipy.sparse = csparse
    csparse.linalg = clinalg
    sys.modules.update({"cupy": cp, "cupyx": cupyx, "cupyx.scipy": cscipy,
                        "cupyx.scipy.sparse": csparse, "cupyx.scipy.sparse.linalg": clinalg})
    return cp
