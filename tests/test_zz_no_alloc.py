"""sa_spmv_scaled_noalloc, the allocation-free variant of the fused scaled operator.

Some callers cannot allocate device memory (a host framework whose pool allocator owns the whole
device; a latency-sensitive caller that must not pay for cudaMalloc's implicit synchronisation).
This entry point serves them with a fixed scratch array inside the library. Here it is called through
the C-ABI and compared with the handle-based sa_spmv_scaled on the same inputs, twice in a row
(the second call reuses the array the first one left behind). This file is collected last so that a
run that stops at the first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from specann_b200 import _lib, graphs  # noqa: E402
from specann_b200.engine import Engine  # noqa: E402


def _noalloc(lib, J, d_rp, d_col, d_val, alpha, rho, x):
    y = torch.empty_like(x)
    st = lib.sa_spmv_scaled_noalloc(J.shape[0], J.nnz, C.c_void_p(d_rp.data_ptr()), C.c_void_p(d_col.data_ptr()),
                                    C.c_void_p(d_val.data_ptr()), float(alpha), float(rho),
                                    C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()),
                                    C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == _lib.SA_OK, st
    torch.cuda.synchronize()
    return y


def test_noalloc_operator_matches_handle_operator_twice():
    lib = _lib.load()
    J = graphs.barabasi_albert(5000, 12, seed=7, couplings="int100")
    n = J.shape[0]
    d_rp = torch.from_numpy(J.indptr.astype(np.int32)).cuda()
    d_col = torch.from_numpy(J.indices.astype(np.int32)).cuda()
    d_val = torch.from_numpy(J.data.astype(np.float32)).cuda()
    eng = Engine(n, J.nnz, precision=32, ncv_max=33, max_candidates=1)
    eng.bind(d_rp, d_col, d_val)
    rng = np.random.default_rng(0)
    for alpha, rho in ((0.37, 1.001), (1.0, 0.5)):          # two calls in a row
        x = torch.tensor(rng.standard_normal(n), dtype=torch.float32, device="cuda")
        y_ref = eng.spmv(alpha, rho, x).double().cpu().numpy()
        y = _noalloc(lib, J, d_rp, d_col, d_val, alpha, rho, x).double().cpu().numpy()
        err = np.max(np.abs(y - y_ref)) / np.max(np.abs(y_ref))
        assert err < 3e-6, (alpha, err)


def test_noalloc_defined_on_zero_couplings_and_bad_columns():
    """All-zero couplings give y = rho x (no NaN); an out-of-range column is skipped."""
    lib = _lib.load()
    n = 64
    rp = np.arange(n + 1, dtype=np.int32)                    # one entry per row
    col = ((np.arange(n) + 1) % n).astype(np.int32)
    x = torch.linspace(-1, 1, n, dtype=torch.float32, device="cuda")
    d_rp = torch.from_numpy(rp).cuda()
    zero = torch.zeros(n, dtype=torch.float32, device="cuda")
    J = type("J", (), {"shape": (n, n), "nnz": n})
    y = _noalloc(lib, J, d_rp, torch.from_numpy(col).cuda(), zero, 0.5, 1.25, x)
    assert torch.equal(y, 1.25 * x)
    # a ring with one column out of range: that product is dropped, the other rows are untouched
    bad = col.copy()
    bad[3] = n + 1000
    ones = torch.ones(n, dtype=torch.float32, device="cuda")
    y_ok = _noalloc(lib, J, d_rp, torch.from_numpy(col).cuda(), ones, 0.0, 0.0, x)
    y_bad = _noalloc(lib, J, d_rp, torch.from_numpy(bad).cuda(), ones, 0.0, 0.0, x)
    assert torch.isfinite(y_bad).all()
    assert float(y_bad[3]) == 0.0
    keep = torch.arange(n, device="cuda") != 3
    assert torch.equal(y_bad[keep], y_ok[keep])


def test_noalloc_rejects_sizes_beyond_its_array():
    lib = _lib.load()
    x = torch.zeros(4, dtype=torch.float32, device="cuda")
    too_big = (1 << 20) + 1
    st = lib.sa_spmv_scaled_noalloc(too_big, 0, C.c_void_p(x.data_ptr()), None, None, 0.5, 1.0,
                                    C.c_void_p(x.data_ptr()), C.c_void_p(x.data_ptr()), None)
    assert st == _lib.SA_ERR_INVALID_ARG
