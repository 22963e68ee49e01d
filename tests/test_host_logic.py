"""Host-side logic of the drop-in classes (no GPU): constructor contract, schedule, shift, selection
stream, oracle local-search semantics."""
import inspect

import numpy as np
import pytest
import scipy.sparse as sp

from oracle import selection
from oracle import specann_oracle as O
from specann_b200 import graphs
from specann_b200.failures import NumericalFailure, is_out_of_memory
from specann_b200.selector import SOLVERS, get_solver_class
from specann_b200.spectral_annealing import (SpectralAnnealing, compute_shift_rho, default_ncv,
                                             gershgorin_bound)
from specann_b200.spec_adj import Alpha0GPU, Alpha1GPU

REFERENCE_SPECANN_PARAMS = ["instance_name", "dataset", "random_seed", "mode", "beta", "alpha", "use_local_search",
                            "max_local_iterations", "eigsh_tol", "eigsh_maxiter", "run_name", "disable_warm_start",
                            "precision", "pred_mode", "pred_tol", "shift_eps", "schedule", "num_alphas",
                            "schedule_interval", "eigsh_ncv", "fp32_spmv", "ls_policy", "ls_batch", "kwargs"]


def test_constructor_signature_matches_reference():
    params = list(inspect.signature(SpectralAnnealing.__init__).parameters)[1:]
    assert params == REFERENCE_SPECANN_PARAMS
    sig = inspect.signature(SpectralAnnealing.__init__).parameters
    assert sig["num_alphas"].default == 128 and sig["schedule"].default == "sqrt"
    assert sig["eigsh_tol"].default == 1e-6 and sig["pred_tol"].default == 1e-3
    a0 = list(inspect.signature(Alpha0GPU.__init__).parameters)[1:]
    assert a0 == ["instance_name", "dataset", "random_seed", "mode", "beta", "alpha", "use_local_search",
                  "max_local_iterations", "eigsh_tol", "eigsh_maxiter", "run_name", "ls_policy", "precision", "kwargs"]
    a1 = list(inspect.signature(Alpha1GPU.__init__).parameters)[1:]
    assert a1 == ["instance_name", "dataset", "random_seed", "mode", "beta", "use_local_search",
                  "max_local_iterations", "eigsh_tol", "eigsh_maxiter", "run_name", "ls_policy", "precision", "kwargs"]


@pytest.mark.parametrize("kw,msg", [
    ({"pred_mode": "bogus"}, "pred_mode must be one of"),
    ({"schedule": "cubic"}, "schedule must be one of"),
    ({"num_alphas": 1}, "need num_alphas >= 2"),
    ({"schedule_interval": (1.0, 0.5)}, "need num_alphas >= 2"),
    ({"precision": 16}, "precision must be 32 or 64"),
    ({"ls_policy": "nope"}, "ls_policy must be one of"),
    ({"ls_batch": False, "ls_policy": "fixed_guard"}, "ls_batch = False is only defined"),
    ({"precision": 64, "fp32_spmv": True}, "fp32_spmv needs precision 32"),
])
def test_constructor_validation(kw, msg):
    with pytest.raises(ValueError, match=msg):
        SpectralAnnealing("x.txt", "d", **kw)


def test_registry_names():
    assert sorted(SOLVERS) == ["spec_adj", "spec_signed_lap", "spectral_annealing"]
    assert get_solver_class("spectral_annealing") is SpectralAnnealing
    assert get_solver_class("spec_adj") is Alpha0GPU
    assert get_solver_class("spec_signed_lap") is Alpha1GPU
    with pytest.raises(ValueError):
        get_solver_class("nope")


def test_schedule_matches_oracle():
    s = SpectralAnnealing("x", "d", schedule="sqrt", num_alphas=51, schedule_interval=(0, 1.25))
    assert s._get_alpha_values(0) == O.alpha_schedule("sqrt", 51, (0, 1.25))
    s = SpectralAnnealing("x", "d", schedule="linear")
    assert s._get_alpha_values(0) == O.alpha_schedule("linear", 128, (0, 1))


def test_shift_and_gershgorin():
    assert compute_shift_rho(None, 1.0) == pytest.approx(1.001)
    assert compute_shift_rho(float("nan"), 1.0) == pytest.approx(1.001)
    assert compute_shift_rho(1.5, 1.0, eps=0.01) == pytest.approx(1.515)
    assert compute_shift_rho(-2.0, 0.5) == pytest.approx(0.5005)
    d = np.array([0.02, 0.5, 1.0])
    for a in (0.0, 0.3, 1.0, 1.2):
        assert gershgorin_bound(d.min(), d.max(), a) == pytest.approx(float(np.max(d ** (1 - a))))
    assert default_ncv(10, None) == 9 and default_ncv(1000, None) == 33 and default_ncv(2, None) == 2


def test_failure_mapping():
    assert is_out_of_memory(MemoryError())
    try:
        try:
            raise RuntimeError("CUDA out of memory. Tried to allocate")
        except RuntimeError as e:
            raise ValueError("wrapped") from e
    except ValueError as e:
        assert is_out_of_memory(e)
    assert not is_out_of_memory(NumericalFailure("x"))


@pytest.mark.parametrize("n", [1, 2, 3, 31, 32, 33, 1000, 4097])
def test_selection_is_exact_size_bijection(n):
    r = selection.ranks(n, seed=7, stream=3)
    assert sorted(r.tolist()) == list(range(n))
    m = selection.num_selected(n, 0.9)
    assert selection.selected_mask(n, 7, 3, m).sum() == m
    assert not np.array_equal(selection.ranks(n, 7, 4), r) or n <= 2


def test_num_selected_matches_reference_rounding():
    for n in (1, 9, 10, 11, 1025, 65536):
        assert selection.num_selected(n, 0.9) == max(1, int(0.9 * n))


def test_oracle_local_search_semantics():
    J = graphs.barabasi_albert(400, 4, seed=5, couplings="pm1")
    rng = np.random.default_rng(0)
    S = np.where(rng.random((3, 400)) < 0.5, 1, -1).astype(np.int8)
    res = O.local_search(J, S, seed=11)
    assert np.array_equal(res.energies_before, O.integer_energies(J, S))
    assert np.array_equal(res.energies_after, O.integer_energies(J, res.spins))
    assert np.all(res.energies_after <= res.energies_before)
    # determinism
    res2 = O.local_search(J, S, seed=11)
    assert np.array_equal(res.spins, res2.spins) and res.iterations == res2.iterations
    # zero passes: unchanged
    res0 = O.local_search(J, S, seed=11, max_iterations=0, num_rounds=0)
    assert np.array_equal(res0.spins, S) and res0.iterations == 0


def test_oracle_reference_kernel_emulation_counts():
    J = graphs.erdos_renyi(120, 0.1, seed=2, couplings="pm1")
    pre = O.prelude(J, 32)
    S = np.where(np.random.default_rng(1).random((2, 120)) < 0.5, 1, -1).astype(np.int8)
    S2 = S.copy()
    counts = O.reference_kernel_pass(pre.Js, S2, np.arange(120))
    assert counts.sum() == int((S2 != S).sum())
    # in-place sequential single flips never raise the energy
    assert np.all(O.integer_energies(J, S2) <= O.integer_energies(J, S))


def test_priority_local_search_is_monotone_and_stable():
    """Priority passes: flips form an independent set, so energy never rises and the result is a
    1-flip local minimum once the final sweep ends without flips."""
    J = graphs.barabasi_albert(2000, 8, seed=3, couplings="int100")
    S = np.where(np.random.default_rng(4).random((4, 2000)) < 0.5, 1, -1).astype(np.int8)
    res = O.local_search(J, S, seed=5)
    assert np.all(res.energies_after <= res.energies_before)
    Ji = sp.csr_matrix((np.rint(J.data).astype(np.int64), J.indices, J.indptr), shape=J.shape)
    H = Ji @ res.spins.T.astype(np.int64)
    assert np.all(res.spins.T.astype(np.int64) * H >= 0)      # no improving single flip left
    snap = O.local_search(J, S, seed=5, semantics="snapshot", max_iterations=50, num_rounds=2)
    assert snap.spins.shape == S.shape
