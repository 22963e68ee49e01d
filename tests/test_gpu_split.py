"""L2 column splits of the operator (through the C-ABI): the standalone operator against the oracle's
FP64 operator and the work list for 2 to 8 splits (packed signed columns and the value stream, empty
rows, long rows), bit-exact repeats, the alpha solve through the splits, the solver's split layout,
and the switches between layouts."""
import numpy as np
import pytest
import scipy.sparse as sp

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from oracle import specann_oracle as O  # noqa: E402
from specann_b200 import _lib, graphs  # noqa: E402
from specann_b200.engine import Engine  # noqa: E402
from specann_b200.spectral_annealing import SpectralAnnealing  # noqa: E402


def engine_for(J, precision=32):
    J = sp.csr_matrix(J)
    eng = Engine(J.shape[0], J.nnz, precision=precision, ncv_max=33, max_candidates=4)
    data = J.data.astype(np.float32) if precision == 32 else J.data.astype(np.float64)
    eng.upload_csr(J.indptr, J.indices, data)
    return eng


def with_empty_rows(J, extra, seed=0):
    n = J.shape[0] + extra
    big = sp.block_diag([J, sp.csr_matrix((extra, extra))]).tocsr()
    p = np.random.default_rng(seed).permutation(n)
    P = sp.csr_matrix((np.ones(n), (np.arange(n), p)), shape=(n, n))
    return (P @ big @ P.T).tocsr()


def star_plus_ba(n, leaves):
    """A BA graph with one hub joined to `leaves` vertices: rows longer than a work-list chunk."""
    J = graphs.barabasi_albert(n, 8, seed=9).tolil()
    for j in range(1, leaves + 1):
        J[0, j] = -1.0
        J[j, 0] = -1.0
    return J.tocsr()


GRAPHS = {
    "ba65536": lambda: graphs.barabasi_albert(1 << 16, 20, seed=42),
    "ba30000_int": lambda: graphs.barabasi_albert(30000, 12, seed=4, couplings="int100"),
    "er5000_pm1": lambda: graphs.erdos_renyi(5000, 30 / 4999, seed=5, couplings="pm1"),
    "ba9000_empty": lambda: with_empty_rows(graphs.barabasi_albert(9000, 20, seed=6), 777),
    "hub": lambda: star_plus_ba(20000, 3000),
}


def operator_ref(J, alpha, rho, x):
    deg = np.asarray(abs(J).sum(axis=1)).ravel()
    M, _ = O.scaled_operator_f64(J, deg, deg.max(), alpha)
    return rho * x - M @ x


@pytest.mark.parametrize("gname", list(GRAPHS))
@pytest.mark.parametrize("precision,splits", [(32, 2), (32, 3), (32, 8), (64, 5)])
def test_split_operator_matches_fp64_and_worklist(gname, precision, splits):
    J = GRAPHS[gname]()
    eng = engine_for(J, precision)
    n = J.shape[0]
    dt = torch.float32 if precision == 32 else torch.float64
    x = torch.tensor(np.random.default_rng(7).standard_normal(n), dtype=dt, device="cuda")
    wl = {a: eng.spmv(a, 1.001, x).clone() for a in (0.0, 0.6, 1.0)}
    assert eng.build_splits(splits) == splits
    assert eng.split_count() == splits
    tol = 3e-6 if precision == 32 else 1e-13
    for a in (0.0, 0.6, 1.0):
        y = eng.spmv(a, 1.001, x)
        assert torch.equal(y, eng.spmv(a, 1.001, x))
        yr = operator_ref(J, a, 1.001, x.double().cpu().numpy())
        scale = np.max(np.abs(yr))
        assert np.max(np.abs(y.double().cpu().numpy() - yr)) / scale < tol, a
        assert (y.double() - wl[a].double()).abs().max().item() / scale < 2 * tol, a
    eng.enable_splits(False)
    assert eng.split_count() == 0
    assert torch.equal(eng.spmv(1.0, 1.001, x), wl[1.0])


@pytest.mark.parametrize("alpha", [0.0, 1.0])
def test_alpha_solve_through_splits(alpha):
    J = GRAPHS["ba65536"]()
    res = {}
    for layout in ("worklist", "split"):
        eng = engine_for(J)
        if layout == "split":
            eng.build_splits(3)
        rec = eng.alpha_solve(alpha=alpha, alpha_prev=alpha, rho=1.001, gershgorin=1.0, tol=1e-6, pred_tol=1e-3,
                              maxiter=3000, ncv=33, start_mode=_lib.SA_START_RANDOM, seed=42, stream_id=0,
                              align=False)
        assert rec.status == _lib.SA_OK, rec.status
        assert rec.residual < 1e-5
        res[layout] = 1.001 - rec.mu
        eng.close()
    assert res["split"] == pytest.approx(res["worklist"], abs=2e-6)


def test_solver_split_layout_energy():
    J = graphs.barabasi_albert(8192, 20, seed=11)
    out = {}
    for spmv in ("split", "worklist"):
        s = SpectralAnnealing("t", "t", random_seed=42, num_alphas=16, write_results=False, spmv=spmv)
        e, spins, _ = s.solve(J)
        assert s.operator_layout == spmv
        sv = np.asarray(spins, dtype=np.float64)
        assert e == pytest.approx(-0.5 * sv @ (J @ sv), rel=1e-9)
        out[spmv] = e
    assert out["split"] == pytest.approx(out["worklist"], rel=1e-2)


def test_layout_switches():
    J = GRAPHS["ba65536"]()
    eng = engine_for(J)
    eng.build_splits(2)
    eng.build_panels()                 # the panel layout takes over
    assert eng.split_count() == 0
    eng.enable_splits(True)            # and back
    assert eng.split_count() == 2
    eng.upload_csr(J.indptr, J.indices, J.data.astype(np.float32))   # a new matrix drops both
    assert eng.split_count() == 0
    with pytest.raises(_lib.SpecAnnError):
        eng.enable_splits(True)
