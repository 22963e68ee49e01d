"""Column-panel SpMV (through the C-ABI): the operator against the oracle's FP64 operator and against
the work-list path, bit-exact repeats, the value stream for couplings of several magnitudes, partial
last panels and empty rows; the alpha solve through the panel layout; the solver's operator choice;
and the packed signed-column stream of the work list (bit-exact against the unpacked stream)."""
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
    """J embedded among `extra` rows without entries, spread by a random permutation."""
    n = J.shape[0] + extra
    big = sp.block_diag([J, sp.csr_matrix((extra, extra))]).tocsr()
    p = np.random.default_rng(seed).permutation(n)
    P = sp.csr_matrix((np.ones(n), (np.arange(n), p)), shape=(n, n))
    return (P @ big @ P.T).tocsr()


GRAPHS = {
    "ba65536": lambda: graphs.barabasi_albert(1 << 16, 20, seed=42),           # 4 FP32 panels
    "ba40000_pm1": lambda: graphs.barabasi_albert(40000, 20, seed=3, couplings="pm1"),  # partial last panel
    "ba20000_int": lambda: graphs.barabasi_albert(20000, 20, seed=4, couplings="int100"),  # value stream
    "er5000": lambda: graphs.erdos_renyi(5000, 30 / 4999, seed=5),             # one panel, n % 4 != 0
    "ba9000_empty": lambda: with_empty_rows(graphs.barabasi_albert(9000, 20, seed=6), 777),
}


def operator_ref(J, alpha, rho, x):
    deg = np.asarray(abs(J).sum(axis=1)).ravel()
    M, _ = O.scaled_operator_f64(J, deg, deg.max(), alpha)
    return rho * x - M @ x


@pytest.mark.parametrize("gname", list(GRAPHS))
@pytest.mark.parametrize("precision", [32, 64])
def test_panel_operator_matches_fp64_and_worklist(gname, precision):
    J = GRAPHS[gname]()
    eng = engine_for(J, precision)
    n = J.shape[0]
    dt = torch.float32 if precision == 32 else torch.float64
    x = torch.tensor(np.random.default_rng(7).standard_normal(n), dtype=dt, device="cuda")
    wl = {a: eng.spmv(a, 1.001, x).clone() for a in (0.0, 0.5, 1.0)}
    nbytes = eng.build_panels()
    info = eng.panel_info()
    assert nbytes > 0 and info["blocks"] >= 1 and info["slots"] >= J.nnz and info["slots"] % 8 == 0
    assert info["panels"] == -(-n // info["width"])
    tol = 3e-6 if precision == 32 else 1e-13
    for a in (0.0, 0.5, 1.0):
        y = eng.spmv(a, 1.001, x)
        y2 = eng.spmv(a, 1.001, x)
        assert torch.equal(y, y2)   # fixed summation order
        yr = operator_ref(J, a, 1.001, x.double().cpu().numpy())
        scale = np.max(np.abs(yr))
        assert np.max(np.abs(y.double().cpu().numpy() - yr)) / scale < tol, a
        assert (y.double() - wl[a].double()).abs().max().item() / scale < 2 * tol, a
    # switching back gives the work-list result again, bit for bit
    eng.enable_panels(False)
    assert torch.equal(eng.spmv(1.0, 1.001, x), wl[1.0])


def test_panel_layout_dropped_by_new_matrix():
    J = GRAPHS["er5000"]()
    eng = engine_for(J)
    eng.build_panels()
    eng.upload_csr(J.indptr, J.indices, J.data.astype(np.float32))
    with pytest.raises(_lib.SpecAnnError):
        eng.enable_panels(True)


@pytest.mark.parametrize("alpha", [0.0, 1.0])
def test_alpha_solve_through_panels(alpha):
    J = GRAPHS["ba65536"]()
    res = {}
    for layout in ("worklist", "panel"):
        eng = engine_for(J)
        if layout == "panel":
            eng.build_panels()
        rec = eng.alpha_solve(alpha=alpha, alpha_prev=alpha, rho=1.001, gershgorin=1.0, tol=1e-6, pred_tol=1e-3,
                              maxiter=3000, ncv=33, start_mode=_lib.SA_START_RANDOM, seed=42, stream_id=0,
                              align=False)
        assert rec.status == _lib.SA_OK, rec.status
        assert rec.residual < 1e-5
        res[layout] = 1.001 - rec.mu
        eng.close()
    assert res["panel"] == pytest.approx(res["worklist"], abs=2e-6)


def test_solver_operator_choice_and_energy():
    J = graphs.barabasi_albert(8192, 20, seed=11)
    out = {}
    for spmv in ("auto", "worklist"):
        s = SpectralAnnealing("t", "t", random_seed=42, num_alphas=16, write_results=False, spmv=spmv)
        e, spins, _ = s.solve(J)
        out[spmv] = (s.operator_layout, e, spins)
        # the reported energy is the energy of the returned spins
        sv = np.asarray(spins, dtype=np.float64)
        assert e == pytest.approx(-0.5 * sv @ (J @ sv), rel=1e-9)
    assert out["auto"][0] == "panel" and out["worklist"][0] == "worklist"
    assert out["auto"][1] == pytest.approx(out["worklist"][1], rel=1e-2)


def test_solver_keeps_worklist_for_sparse_rows():
    J = graphs.erdos_renyi(6000, 6 / 5999, seed=12)
    s = SpectralAnnealing("t", "t", random_seed=1, num_alphas=4, write_results=False)
    s.solve(J)
    assert s.operator_layout == "worklist"


@pytest.mark.parametrize("couplings,packed", [("unit", True), ("pm1", True), ("int100", False)])
def test_packed_columns_bit_exact(couplings, packed):
    J = graphs.barabasi_albert(30000, 12, seed=13, couplings=couplings)
    eng = engine_for(J)
    pol = eng.spmv_policy()
    assert pol["packed_columns"] == packed
    assert pol["magnitude"] == (1.0 if packed else 0.0)
    x = torch.randn(J.shape[0], device="cuda")
    y_packed = eng.spmv(0.7, 1.001, x).clone()
    eng.set_spmv_policy(packed_columns=False)
    assert not eng.spmv_policy()["packed_columns"]
    assert torch.equal(eng.spmv(0.7, 1.001, x), y_packed)


def test_panel_layout_deterministic():
    """Two builds of the same matrix give the same entry stream, byte for byte (stable sort)."""
    J = GRAPHS["ba65536"]()
    words = []
    for _ in range(2):
        eng = engine_for(J)
        eng.build_panels()
        slots = eng.panel_info()["slots"]
        words.append(eng._panel_ws[: 4 * slots].clone())
        eng.close()
    assert torch.equal(words[0], words[1])
    w = words[0].view(torch.int32).cpu().numpy().view(np.uint32)
    real = w[w != 0xFFFF0000]
    assert len(real) == J.nnz
    assert np.all((real >> 16) < 16384) and np.all((real & 0x7FFF) < 16384)


def test_layout_tables_follow_the_restated_piece_rules():
    """The device-built entry stream and chunk table equal what the CPU restatement of the piece
    packing and warp cuts (tests/test_panel_pieces_logic.py) gives for every segment of a skewed
    graph with long hub rows."""
    from test_panel_pieces_logic import PIECE, WARPS, pieces, warp_starts
    J = graphs.barabasi_albert(20000, 8, seed=9).tolil()
    for j in range(1, 3001):                      # a hub of 3000 leaves: rows longer than a piece
        J[0, j] = -1.0
        J[j, 0] = -1.0
    J = J.tocsr()
    eng = engine_for(J, 32)
    eng.build_panels()
    info = eng.panel_info()
    ent, chunk, row0 = eng.panel_tables()
    nb, npn, width = info["blocks"], info["panels"], info["width"]
    assert chunk[nb * npn * WARPS] == info["slots"]
    pad = np.uint32(0xFFFF0000)
    for b in range(nb):
        r_lo, r_hi = int(row0[b]), int(row0[b + 1])
        a, e = J.indptr[r_lo], J.indptr[r_hi]
        rows = np.repeat(np.arange(r_lo, r_hi), np.diff(J.indptr[r_lo:r_hi + 1]))
        cols = J.indices[a:e]
        neg = J.data[a:e] < 0
        for p in range(npn):
            sel = (cols // width) == p
            seg_rows = rows[sel]
            words = ((seg_rows - r_lo).astype(np.uint32) << 16) | (neg[sel].astype(np.uint32) << 15) | \
                (cols[sel] - p * width).astype(np.uint32)
            pcs = pieces(seg_rows)
            st = warp_starts(seg_rows, pcs)
            q = (b * npn + p) * WARPS
            base = int(chunk[q])
            assert [int(x) for x in chunk[q:q + WARPS]] == [base + PIECE * t for t in st]
            assert int(chunk[q + WARPS]) == base + PIECE * len(pcs)
            for i, (s0, ln) in enumerate(pcs):
                slot = base + PIECE * i
                assert np.array_equal(ent[slot:slot + ln], words[s0:s0 + ln]), (b, p, i)
                assert np.all(ent[slot + ln:slot + PIECE] == pad)
