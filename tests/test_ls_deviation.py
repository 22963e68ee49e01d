"""How far the engine's local search is from the reference kernel's (CPU, oracle only).

The reference's update_spins_kernel_float32 (models/spectral_annealing.py:821-869) flips spins in
place from racing warps with fp32 sums, so its result depends on thread timing; the engine runs
deterministic priority passes with exact integer gains. oracle.ls_deviation runs both over the same
node-selection stream (the reference kernel with its warps in rank order, one legal schedule of it)
and counts, per pass and from the same spins, the decisions that differ in schedule and the
in-order decisions whose fp32 sign differs from the exact gain. The bounds below are the measured
figures rounded up; the numbers themselves are printed (pytest -s) and quoted in the design notes.
"""
import json

import numpy as np
import pytest
import scipy.sparse as sp

from oracle import specann_oracle as O


def _gold(golden_cases, name):
    z = golden_cases[name]
    n = int(z["n"])
    J = sp.csr_matrix((z["data"], z["indices"], z["indptr"]), shape=(n, n))
    keys, uniq = set(), []
    for s in z["cap_spins"]:
        if s.tobytes() not in keys:
            keys.add(s.tobytes())
            uniq.append(s)
    return J, np.stack(uniq)


@pytest.mark.parametrize("name,max_sched,max_arith", [("tiny_ba100_specann32", 0.03, 0),
                                                      ("tiny_ba190_specann64", 0.02, 10),
                                                      ("er128_prev_linear32", 0.03, 3),
                                                      ("ba128_secant32", 0.02, 2)])
def test_deviation_on_reference_goldens(golden_cases, name, max_sched, max_arith):
    J, S = _gold(golden_cases, name)
    d = O.ls_deviation(J, S, seed=42)
    frac = d.schedule_differences / d.decisions
    gap = (d.energy_reference - d.energy_priority) / np.abs(d.energy_priority)
    print(json.dumps({"case": name, "candidates": int(S.shape[0]), "passes": d.passes, "decisions": d.decisions,
                      "schedule_differences": d.schedule_differences, "fraction": round(frac, 5),
                      "arithmetic_differences": d.arithmetic_differences,
                      "best_reference": int(d.energy_reference.min()), "best_priority": int(d.energy_priority.min()),
                      "mean_rel_gap": float(gap.mean())}))
    assert frac <= max_sched
    assert d.arithmetic_differences <= max_arith
    # both are descents from the same candidates: neither ends above the starting energies
    e0 = O.integer_energies(J, S)
    assert np.all(d.energy_reference <= e0) and np.all(d.energy_priority <= e0)
    assert np.max(np.abs(gap)) < 0.1


def test_deviation_on_c1_candidates():
    """C1, ER(1024, 20/1023): the oracle sweep's candidates (16 of them, spread over the schedule)."""
    from specann_b200 import graphs
    J = graphs.erdos_renyi(1024, 20 / 1023, seed=42)
    out = O.solve(J, seed=42, schedule="linear", num_alphas=128, use_local_search=False)
    S = np.stack(out.candidates)[:: max(1, len(out.candidates) // 16)][:16]
    d = O.ls_deviation(J, S, seed=42)
    frac = d.schedule_differences / d.decisions
    print(json.dumps({"case": "c1", "candidates": int(S.shape[0]), "passes": d.passes, "decisions": d.decisions,
                      "schedule_differences": d.schedule_differences, "fraction": round(frac, 5),
                      "arithmetic_differences": d.arithmetic_differences,
                      "best_reference": int(d.energy_reference.min()), "best_priority": int(d.energy_priority.min())}))
    assert frac <= 0.02
    assert d.arithmetic_differences <= 0.002 * d.decisions
    assert abs(int(d.energy_reference.min()) - int(d.energy_priority.min())) <= 0.02 * abs(int(d.energy_priority.min()))


def test_reference_pass_restatement_matches_scalar_form():
    """The vectorised in-order pass equals the scalar restatement of the kernel, candidate by candidate."""
    from specann_b200 import graphs
    J = graphs.barabasi_albert(300, 6, seed=3, couplings="int100")
    pre = O.prelude(J, 32)
    Ji = sp.csr_matrix((np.rint(J.data).astype(np.int64), J.indices, J.indptr), shape=J.shape)
    S = np.where(np.random.default_rng(0).random((5, 300)) < 0.5, 1, -1).astype(np.int8)
    order = np.random.default_rng(1).permutation(300)[:270]
    A, B = S.copy(), S.copy()
    f_vec, _ = O._reference_pass_all(pre.Js, Ji, A, order)
    f_sca = O.reference_kernel_pass(pre.Js, B, order)
    assert np.array_equal(A, B) and np.array_equal(f_vec, f_sca)
