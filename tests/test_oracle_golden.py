"""The CPU oracle against golden vectors produced by the reference's own solver code
(tests/golden/make_golden.py runs models/spectral_annealing.py, spec_adj.py and spec_signed_lap.py on
NumPy/SciPy through a CuPy stand-in). This pins the oracle before it is used as the checker."""
import json

import numpy as np
import pytest
import scipy.sparse as sp

from oracle import specann_oracle as O

SWEEP_CASES = ["tiny_ba20_specann32", "tiny_ba100_specann32", "tiny_ba190_specann64", "ba128_secant32",
               "er128_prev_linear32", "er1024_linear16_nols32"]


def _J(z):
    n = int(z["n"])
    return sp.csr_matrix((z["data"], z["indices"], z["indptr"]), shape=(n, n))


def _params(z):
    return json.loads(str(z["params"]))


@pytest.mark.parametrize("name", SWEEP_CASES)
def test_prelude_and_schedule(golden_cases, name):
    z = golden_cases[name]
    p = _params(z)
    pre = O.prelude(_J(z), p.get("precision", 32))
    assert pre.c == pytest.approx(float(z["normalization"]), rel=0, abs=0)
    alphas = O.alpha_schedule(p.get("schedule", "sqrt"), p.get("num_alphas", 128), (0.0, 1.0))
    assert np.array_equal(np.asarray(alphas), z["cap_alpha"])


@pytest.mark.parametrize("name", SWEEP_CASES)
def test_rounding_signature_energy_bit_exact(golden_cases, name):
    """Given the reference's own eigenvector at each alpha, the oracle's rounding equals the
    reference's spins bit for bit, and its fp32 energy equals the reference's raw energy."""
    z = golden_cases[name]
    p = _params(z)
    pre = O.prelude(_J(z), p.get("precision", 32))
    for a in range(z["cap_x"].shape[0]):
        spins = O.round_spins(z["cap_x"][a])
        if "cap_spins" in z:
            assert np.array_equal(spins, z["cap_spins"][a].astype(np.int8))
        raw = O.fp32_energies(pre.Js, spins[None, :], pre.c)[0] if p.get("precision", 32) == 32 else \
            -0.5 * pre.c * spins.astype(np.float64) @ (pre.Js @ spins.astype(np.float64))
        assert raw == pytest.approx(z["row_raw_energy"][a], rel=1e-12)
        assert O.exact_energy(_J(z), spins) == pytest.approx(z["row_raw_energy"][a], rel=1e-6)


@pytest.mark.parametrize("name", SWEEP_CASES)
def test_eigenpairs_and_predictor_against_reference(golden_cases, name):
    """Re-run each alpha of the reference sweep in the oracle from the reference's own warm-start
    chain: same shift, same predictor decision, same leading eigenvalue and eigenvector."""
    z = golden_cases[name]
    p = _params(z)
    prec = p.get("precision", 32)
    pre = O.prelude(_J(z), prec)
    alphas = z["cap_alpha"]
    ys = z["cap_y"]
    y_last = y_prev = None
    lam_prev = a_prev = None
    rng = np.random.default_rng(0)
    mismatched_accept = 0
    for a, alpha in enumerate(alphas):
        res = O.solve_alpha(pre, float(alpha), a, a_prev, y_last, y_prev, lam_prev,
                            pred_mode=p.get("pred_mode", "diagonal"), rng=rng)
        assert res.lambda1 == pytest.approx(z["row_lambda1"][a], abs=2e-5)
        # the eigenvector up to sign: |<y_oracle, y_ref>| ~ 1
        yr = ys[a] / np.linalg.norm(ys[a])
        assert abs(float(np.dot(res.y, yr))) > 1 - 1e-4
        ref_pr = z["row_pred_residual"][a]
        if np.isnan(ref_pr):
            assert np.isnan(res.pred_residual)
        else:
            assert res.pred_residual == pytest.approx(ref_pr, rel=2e-3, abs=1e-6)
            acc_ref = bool(z["row_pred_accepted"][a])
            if abs(ref_pr - 1e-3) > 1e-5:
                assert res.pred_accepted == acc_ref
            else:
                mismatched_accept += int(res.pred_accepted != acc_ref)
        y_prev, y_last = y_last, ys[a].astype(pre.dtype)
        lam_prev, a_prev = float(z["row_lambda1"][a]), float(alpha)
    assert mismatched_accept <= 1


def test_full_sweep_without_local_search_matches(golden_cases):
    """The oracle's full sweep (its own start vectors) reaches the reference's best energy."""
    z = golden_cases["er1024_linear16_nols32"]
    p = _params(z)
    out = O.solve(_J(z), schedule="linear", num_alphas=p["num_alphas"], use_local_search=False, seed=42)
    assert out.best_energy == pytest.approx(float(z["best_energy"]), rel=1e-9)


@pytest.mark.parametrize("name", ["tiny_ba20_specann32", "tiny_ba100_specann32", "tiny_ba190_specann64"])
def test_candidate_bookkeeping(golden_cases, name):
    """Deduplication: candidate ids in order of first appearance, identical spins <=> same id."""
    z = golden_cases[name]
    seen = {}
    for a in range(z["cap_spins"].shape[0]):
        key = O.signature(z["cap_spins"][a])
        if key not in seen:
            seen[key] = len(seen)
        assert seen[key] == z["row_candidate"][a]


@pytest.mark.parametrize("name", ["tiny_ba20_specann32", "tiny_ba100_specann32", "tiny_ba190_specann64",
                                  "ba128_secant32", "er128_prev_linear32"])
def test_reference_refined_energies_are_one_flip_stable(golden_cases, name):
    """The reference's local search returns (or keeps) spins whose energy is the per-alpha energy;
    the oracle's exact energy of the reference's best spins equals the reported best energy."""
    z = golden_cases[name]
    J = _J(z)
    assert O.exact_energy(J, z["best_spins"]) == pytest.approx(float(z["best_energy"]), rel=1e-12)
    assert float(z["best_energy"]) <= float(np.min(z["row_raw_energy"])) + 1e-6


@pytest.mark.parametrize("name", ["tiny_ba100_specadj32", "tiny_ba120_specsignedlap32"])
def test_fixed_alpha_endpoints(golden_cases, name):
    """SpecAdj / SpecSignedLap: the oracle's leading eigenvector at alpha 0 / 1, rounded and refined,
    reaches an energy no worse than the reference's unrefined rounding."""
    z = golden_cases[name]
    J = _J(z)
    alpha = 0.0 if "specadj" in name else 1.0
    pre = O.prelude(J, 32)
    res = O.solve_alpha(pre, alpha, 0, None, None, None, None, rng=np.random.default_rng(1))
    spins = O.round_spins(res.x)
    e = O.exact_energy(J, spins)
    ls = O.local_search(J, spins[None, :], seed=42)
    assert min(e, float(ls.energies_after[0])) <= float(z["best_energy"]) * (1 - 1e-3) or \
        min(e, float(ls.energies_after[0])) == pytest.approx(float(z["best_energy"]), rel=0.05)
