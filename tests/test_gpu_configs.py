"""Parity on the benchmark configurations, through the drop-in solver and the C-ABI.

  * C1, ER(1024, p = 20/1023, seed 42), 128 linear alphas, local search on:
      - FP32 (the configuration as published): every alpha's eigenpair against the exact FP64
        operator (dense eigh), rounding bit-exact given the GPU's own eigenvector, the local search,
        energies and selection bit-exact given the GPU's own candidates;
      - FP64 at eigsh_tol 1e-12: the candidates (up to a global sign) and the best energy equal the
        oracle pipeline's. At tol 1e-6 two eigensolvers may round tiny entries differently: the gap
        of C1's leading eigenvalue is ~1e-3 at every alpha, so a residual of 1e-6 leaves the vector
        uncertain by up to ~1e-3 while the smallest entries are ~1e-7 .. 1e-5.
  * The headline workload, BA(2^20, m = 20), 128 sqrt alphas, through the column-panel layout: six
    eigenpairs of the warm-started chain against the FP64 operator and SciPy's eigsh.
  * 64-bit row pointers forced on small matrices: the `long long` instantiations of the alpha,
    local-search, panel and split kernels give the same results as the int32 ones (up to the global
    sign of the eigenvector chain).
  * C2, BA(2^16, m = 20): FP32 with FP64 Ritz against all-FP64, per alpha.
The full-size C5 form (BA(2^25), int64 row pointers, FP32 against FP64) is the bench line's scale
block; here its row-pointer instantiations are checked on small matrices.
"""
import os

import numpy as np
import pytest
import scipy.linalg as sla
import scipy.sparse as sp
import scipy.sparse.linalg as spla

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from oracle import specann_oracle as O  # noqa: E402
from specann_b200 import graphs  # noqa: E402
from specann_b200.spectral_annealing import SpectralAnnealing  # noqa: E402


def c1_graph():
    return graphs.erdos_renyi(1024, 20 / 1023, seed=42)


def scaling(J, alpha):
    """FP64 sigma = D^{-alpha/2} / sqrt(c) of the exact operator M = sigma J sigma (1e-12 clamp)."""
    deg = np.asarray(abs(J).sum(axis=1)).ravel().astype(np.float64)
    c = deg.max()
    d = deg / c
    with np.errstate(divide="ignore"):
        D = np.power(d, float(alpha))
    return 1.0 / np.sqrt(np.maximum(D, 1e-12)) / np.sqrt(c)


def apply_M(J64, sig, v):
    return sig * (J64 @ (sig * v))


def leading_dense(J, alpha):
    """Leading eigenpair and the gap of the exact operator (dense, n <= a few thousand)."""
    sig = scaling(J, alpha)
    A = sp.diags(sig) @ sp.csr_matrix(J, dtype=np.float64) @ sp.diags(sig)
    n = J.shape[0]
    w, V = sla.eigh(A.toarray(), subset_by_index=[n - 2, n - 1])
    return float(w[1]), V[:, 1], float(w[1] - w[0])


def candidates(solver, k, refined=False):
    return np.stack([solver.engine.candidate_spins(c, refined=refined).cpu().numpy() for c in range(k)])


# ------------------------------------------------------------------------------------------------
# C1
# ------------------------------------------------------------------------------------------------

def test_c1_fp32_sweep_against_fp64_and_oracle():
    J = c1_graph()
    n = J.shape[0]
    s = SpectralAnnealing("c1.txt", "c1", random_seed=42, schedule="linear", num_alphas=128,
                          keep_vectors=range(128))
    energy, spins, _ = s.solve(J)
    rows = s.alpha_results
    assert len(rows) == 128 and s._alphas_skipped == 0
    J64 = sp.csr_matrix(J, dtype=np.float64)
    k = s._num_candidates
    cand = candidates(s, k)
    for i, r in enumerate(rows):
        alpha = r["alpha"]
        lam64, y64, gap = leading_dense(J, alpha)
        assert abs(r["lambda1"] - lam64) <= 1e-5, (i, r["lambda1"], lam64)
        assert r["eigsh_converged"] and r["eigsh_residual"] <= 1e-5, (i, r["eigsh_residual"])
        y, rho, mu = s.kept_vectors[i]
        y = y.double().cpu().numpy()
        sig = scaling(J, alpha)
        My = apply_M(J64, sig, y)
        lam_rq = float(y @ My) / float(y @ y)
        # the true residual of the GPU eigenvector against the exact FP64 operator
        assert np.linalg.norm(My - lam_rq * y) / np.linalg.norm(y) <= 1e-5, i
        assert abs(lam_rq - lam64) <= 1e-5
        # it is the leading eigenvector: sin(angle to y64) <= residual / gap <= 1e-2
        assert abs(float(y @ y64)) / np.linalg.norm(y) > 1 - 1e-4
        # rounding is bit-exact given the GPU's own (aligned) eigenvector
        assert np.array_equal(cand[r["candidate"]], np.where(y >= 0, 1, -1).astype(np.int8)), i
    # local search, energies and selection are exact given the GPU's candidates
    ls = O.local_search(J, cand, seed=42)
    raw = O.integer_energies(J, cand).astype(np.float64)
    assert np.array_equal(candidates(s, k, refined=True), ls.spins)
    best = np.inf
    for r in rows:
        c = r["candidate"]
        assert r["raw_energy"] == raw[c]
        assert r["energy"] == min(raw[c], float(ls.energies_after[c]))
        best = min(best, r["energy"])
    assert energy == best == O.exact_energy(J, spins)
    # the oracle pipeline (SciPy eigsh, its own eigenvectors) on the same instance: the same quality
    out = O.solve(J, seed=42, schedule="linear", num_alphas=128)
    assert abs(energy - out.best_energy) <= 0.01 * abs(out.best_energy)


def test_c1_fp64_tight_end_to_end_equals_oracle():
    """With both eigensolvers converged far below the smallest eigenvector entry, the whole pipeline
    (rounding, deduplication, local search, selection) gives the oracle's candidates and energy."""
    J = c1_graph()
    s = SpectralAnnealing("c1.txt", "c1", random_seed=42, schedule="linear", num_alphas=128, precision=64,
                          eigsh_tol=1e-12, write_results=False)
    energy, spins, _ = s.solve(J)
    out = O.solve(J, seed=42, schedule="linear", num_alphas=128, precision=64, eigsh_tol=1e-12)
    k = s._num_candidates
    assert k == len(out.candidates)
    cand = candidates(s, k)
    sign = 1 if np.array_equal(cand[0], out.candidates[0]) else -1
    for c in range(k):
        assert np.array_equal(cand[c], sign * out.candidates[c]), c
    assert [r["candidate"] for r in s.alpha_results] == [r["candidate"] for r in out.records]
    assert energy == out.best_energy
    assert O.exact_energy(J, spins) == energy


# ------------------------------------------------------------------------------------------------
# Headline workload through the column-panel layout
# ------------------------------------------------------------------------------------------------

def test_headline_ba2e20_panel_chain_against_fp64():
    J = graphs.barabasi_albert(1 << 20, 20, seed=42)
    keep = [0, 25, 51, 76, 102, 127]
    s = SpectralAnnealing("h.txt", "h", random_seed=42, keep_vectors=keep, write_results=False)
    energy, spins, _ = s.solve(J)
    assert s.operator_layout == "panel"
    assert s._alphas_skipped == 0
    assert O.exact_energy(J, spins) == energy
    J64 = sp.csr_matrix(J, dtype=np.float64)
    Jt = O.threaded(J64, os.cpu_count() or 1)      # row-block parallel products (same sums)
    k = s._num_candidates
    for i in keep:
        r = s.alpha_results[i]
        alpha = r["alpha"]
        y, rho, mu = s.kept_vectors[i]
        y = y.double().cpu().numpy()
        sig = scaling(J, alpha)
        My = sig * (Jt @ (sig * y))
        lam_rq = float(y @ My) / float(y @ y)
        res = np.linalg.norm(My - lam_rq * y) / np.linalg.norm(y)
        assert res <= 1e-5, (i, res)
        assert abs((rho - mu) - lam_rq) <= 1e-5
        op = spla.LinearOperator(J.shape, matvec=lambda v, sig=sig: sig * (Jt @ (sig * v)), dtype=np.float64)
        # started from the GPU vector, ARPACK (at the solver's own tolerance) confirms that it is the
        # leading eigenvalue
        w = spla.eigsh(op, k=1, which="LA", v0=y, tol=1e-6, ncv=32, maxiter=100, return_eigenvectors=False)
        assert abs(r["lambda1"] - float(w[0])) <= 1e-5, (i, r["lambda1"], float(w[0]))
        spins_i = s.engine.candidate_spins(r["candidate"]).cpu().numpy()
        assert np.array_equal(spins_i, np.where(y >= 0, 1, -1).astype(np.int8)), i
    assert k >= 1


# ------------------------------------------------------------------------------------------------
# 64-bit row pointers
# ------------------------------------------------------------------------------------------------

@pytest.mark.parametrize("layout,couplings", [("worklist", "pm1"), ("worklist", "int100"), ("panel", "unit"),
                                              ("split", "pm1")])
def test_rowptr64_matches_rowptr32(layout, couplings):
    J = graphs.barabasi_albert(1 << 13, 20, seed=3, couplings=couplings)
    out = {}
    for rp64 in (False, True):
        s = SpectralAnnealing("r.txt", "r", random_seed=7, num_alphas=16, spmv=layout, rowptr64=rp64,
                              keep_vectors=range(16), write_results=False)
        e, spins, _ = s.solve(J)
        assert s.engine.rowptr64 == rp64
        assert s.operator_layout == layout
        k = s._num_candidates
        out[rp64] = (e, spins, [r["lambda1"] for r in s.alpha_results], candidates(s, k),
                     candidates(s, k, refined=True), [r["eigsh_iterations"] for r in s.alpha_results])
    e32, s32, l32, c32, r32, it32 = out[False]
    e64, s64, l64, c64, r64, it64 = out[True]
    # the two instantiations are separate compiled code: the chain may come out with the other global
    # sign of the eigenvectors (both are eigenvectors), which negates every candidate and refined spin
    sign = 1 if np.array_equal(c32[0], c64[0]) else -1
    assert e32 == e64 and np.array_equal(s32, sign * s64)
    assert np.max(np.abs(np.array(l32) - np.array(l64))) <= 1e-6
    assert np.array_equal(c32, sign * c64) and np.array_equal(r32, sign * r64)


def test_rowptr64_split_operator_and_local_search_direct():
    """Standalone operator and energies through the int64 work-list and split kernels."""
    from specann_b200.engine import Engine
    J = graphs.barabasi_albert(20000, 12, seed=5, couplings="int100")
    n = J.shape[0]
    x = torch.tensor(np.random.default_rng(1).standard_normal(n), dtype=torch.float32, device="cuda")
    S = np.where(np.random.default_rng(2).random((5, n)) < 0.5, 1, -1).astype(np.int8)
    res = {}
    for rp64 in (False, True):
        eng = Engine(n, J.nnz, precision=32, ncv_max=33, max_candidates=8, rowptr64=rp64)
        eng.upload_csr(J.indptr, J.indices, J.data.astype(np.float32))
        y_wl = eng.spmv(0.4, 1.001, x).cpu().numpy()
        eng.build_splits(3)
        y_sp = eng.spmv(0.4, 1.001, x).cpu().numpy()
        for c in range(5):
            eng.set_candidate(c, S[c])
        eb, ea, r = eng.local_search(5, seed=11)
        refined = np.stack([eng.candidate_spins(c, refined=True).cpu().numpy() for c in range(5)])
        res[rp64] = (y_wl, y_sp, eb, ea, refined)
    for a, b in zip(res[False], res[True]):
        assert np.array_equal(a, b)
    ref = O.local_search(J, S, seed=11)
    assert np.array_equal(res[True][3], ref.energies_after.astype(np.float64))


# ------------------------------------------------------------------------------------------------
# C2: the precision form
# ------------------------------------------------------------------------------------------------

def test_c2_precision_fp32_ritz64_against_fp64():
    J = graphs.barabasi_albert(1 << 16, 20, seed=42)
    keep = [1, 40, 90, 127]
    runs = {}
    for prec in (32, 64):
        s = SpectralAnnealing("c2.txt", "c2", random_seed=42, precision=prec, keep_vectors=keep,
                              write_results=False)
        e, spins, _ = s.solve(J)
        assert s._alphas_skipped == 0
        runs[prec] = (e, s.alpha_results, s.kept_vectors)
    e32, rows32, kept32 = runs[32]
    e64, rows64, kept64 = runs[64]
    l32 = np.array([r["lambda1"] for r in rows32])
    l64 = np.array([r["lambda1"] for r in rows64])
    assert np.max(np.abs(l32 - l64)) <= 1e-6
    assert max(r["eigsh_residual"] for r in rows32) <= 1e-5
    assert max(r["eigsh_residual"] for r in rows64) <= 1e-5
    assert abs(e32 - e64) <= 1e-3 * abs(e64)
    # the FP64 run against SciPy's FP64 eigensolver on the exact operator
    J64 = sp.csr_matrix(J, dtype=np.float64)
    for i in keep:
        sig = scaling(J, rows64[i]["alpha"])
        op = spla.LinearOperator(J.shape, matvec=lambda v, sig=sig: apply_M(J64, sig, v), dtype=np.float64)
        y = kept64[i][0].cpu().numpy()
        w = spla.eigsh(op, k=1, which="LA", v0=y, tol=1e-12, ncv=20, maxiter=200, return_eigenvectors=False)
        assert abs(rows64[i]["lambda1"] - float(w[0])) <= 1e-8
        assert abs(rows32[i]["lambda1"] - float(w[0])) <= 1e-6
