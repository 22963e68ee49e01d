"""Failure detection on the GPU without a fault: the bounded grid barrier of the persistent kernels is
made to run out (a barrier that expects one more CTA than the launch has, so nothing ever releases
it) with a short wait limit; the kernel returns SA_ERR_BARRIER_TIMEOUT to the host and the context
stays usable. The operator's status query reports a clean run after normal applications."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from oracle import specann_oracle as O  # noqa: E402
from specann_b200 import _lib, graphs  # noqa: E402
from specann_b200.engine import Engine  # noqa: E402


def selftest(blocks, expected, spin_limit):
    lib = _lib.load()
    scratch = torch.zeros(4096, dtype=torch.uint8, device="cuda")
    st, passed, epi = C.c_int32(-1), C.c_int32(-1), C.c_int32(-1)
    rc = lib.sa_barrier_selftest(blocks, expected, spin_limit, C.c_void_p(scratch.data_ptr()), scratch.numel(),
                                 C.byref(st), C.byref(passed), C.byref(epi),
                                 C.c_void_p(torch.cuda.current_stream().cuda_stream))
    return rc, st.value, passed.value, epi.value


def test_barrier_passes_when_every_cta_arrives():
    blocks = min(8, torch.cuda.get_device_properties(0).multi_processor_count)
    rc, st, passed, epi = selftest(blocks, blocks, 1 << 20)
    assert rc == _lib.SA_OK
    assert st == _lib.SA_OK and passed == blocks and epi == 1


def test_barrier_wait_runs_out_and_reports_timeout():
    blocks = min(8, torch.cuda.get_device_properties(0).multi_processor_count)
    rc, st, passed, epi = selftest(blocks, blocks + 1, 4096)      # nobody arrives last
    assert rc == _lib.SA_OK
    assert st == _lib.SA_ERR_BARRIER_TIMEOUT
    assert passed == 0 and epi == 0
    # the context is still usable: a normal barrier and an alpha solve afterwards
    rc, st, passed, epi = selftest(blocks, blocks, 1 << 20)
    assert st == _lib.SA_OK and passed == blocks
    J = graphs.erdos_renyi(512, 0.04, seed=3)
    eng = Engine(J.shape[0], J.nnz, precision=32, ncv_max=33, max_candidates=1)
    eng.upload_csr(J.indptr, J.indices, J.data.astype(np.float32))
    rec = eng.alpha_solve(alpha=0.5, alpha_prev=0.5, rho=1.001, gershgorin=1.0, tol=1e-6, pred_tol=1e-3,
                          maxiter=1000, ncv=33, start_mode=_lib.SA_START_RANDOM, seed=1, stream_id=0, align=False)
    assert rec.status == _lib.SA_OK


def test_barrier_selftest_rejects_unbounded_or_oversized_requests():
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    assert selftest(4, 4, (1 << 25) + 1)[0] == _lib.SA_ERR_INVALID_ARG
    assert selftest(sms + 1, sms + 1, 1000)[0] == _lib.SA_ERR_INVALID_ARG
    assert selftest(4, 4, 0)[0] == _lib.SA_ERR_INVALID_ARG


def test_operator_status_clean_after_panel_applications():
    J = graphs.barabasi_albert(1 << 15, 20, seed=8)
    n = J.shape[0]
    eng = Engine(n, J.nnz, precision=32, ncv_max=33, max_candidates=1)
    eng.upload_csr(J.indptr, J.indices, J.data.astype(np.float32))
    eng.build_panels()
    x = torch.tensor(np.random.default_rng(0).standard_normal(n), dtype=torch.float32, device="cuda")
    for _ in range(3):
        y = eng.spmv(0.3, 1.001, x)
    assert eng.operator_status() == _lib.SA_OK
    deg = np.asarray(abs(J).sum(axis=1)).ravel()
    M, _ = O.scaled_operator_f64(J, deg, deg.max(), 0.3)
    ref = 1.001 * x.double().cpu().numpy() - M @ x.double().cpu().numpy()
    assert np.max(np.abs(y.double().cpu().numpy() - ref)) / np.max(np.abs(ref)) < 3e-6
