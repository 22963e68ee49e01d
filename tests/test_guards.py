"""Guarded local-search policies: the oracle's restatement (CPU) and the host pieces of the engine's
(colouring, class order), plus, on the GPU, the engine's kernels bit-exact against the oracle for
integer couplings and the solver classes with every ls_policy."""
import numpy as np
import pytest

from oracle import guards_oracle as G
from oracle import specann_oracle as O
from specann_b200 import graphs

GRAPHS = {
    "ba600_int": lambda: graphs.barabasi_albert(600, 6, seed=3, couplings="int100"),
    "er400_pm1": lambda: graphs.erdos_renyi(400, 0.05, seed=4, couplings="pm1"),
    "ba1500_unit": lambda: graphs.barabasi_albert(1500, 10, seed=5),
}


def candidates(J, k, seed):
    return np.where(np.random.default_rng(seed).random((k, J.shape[0])) < 0.5, 1, -1).astype(np.int8)


def test_host_coloring_matches_oracle_and_is_proper():
    from specann_b200.guards import color_sequence, greedy_coloring
    for mk in GRAPHS.values():
        J = mk()
        colors, k = greedy_coloring(J.indptr, J.indices)
        ref = G.greedy_coloring(J)
        assert np.array_equal(colors, ref) and k == int(ref.max()) + 1
        coo = J.tocoo()
        assert not np.any(colors[coo.row] == colors[coo.col])
    assert np.array_equal(color_sequence(7, 42, 30), G.color_sequence(7, 42, 30))


@pytest.mark.parametrize("policy", ["fixed", "adaptive", "independent", "oracle"])
def test_oracle_policies_are_monotone_descents(policy):
    J = GRAPHS["er400_pm1"]()
    S = candidates(J, 6, 1)
    fn = {"fixed": lambda: G.guarded_search(J, S, 7, adaptive=False),
          "adaptive": lambda: G.guarded_search(J, S, 7, adaptive=True),
          "independent": lambda: G.independent_set_search(J, S, 7),
          "oracle": lambda: G.sequential_oracle(J, S)}[policy]
    r = fn()
    e0 = O.integer_energies(J, S)
    assert np.array_equal(r.energies.astype(np.int64), O.integer_energies(J, r.spins))
    assert np.all(r.energies <= e0)
    if policy == "oracle":
        # a one-flip local optimum: no single flip lowers the energy
        H = (J @ r.spins.T.astype(np.float64))
        assert np.all(2 * r.spins.T * H >= 0)


torch = pytest.importorskip("torch")


def _engine(J, k):
    from specann_b200.engine import Engine
    eng = Engine(J.shape[0], J.nnz, precision=32, ncv_max=33, max_candidates=k)
    eng.upload_csr(J.indptr, J.indices, J.data.astype(np.float32))
    return eng


@pytest.mark.gpu
@pytest.mark.parametrize("gname", list(GRAPHS))
@pytest.mark.parametrize("policy", ["fixed_guard", "adaptive_guard", "independent_set", "sequential_oracle"])
def test_gpu_policy_bit_exact_against_oracle(gname, policy):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from specann_b200.guards import run_policy
    J = GRAPHS[gname]()
    k = 9
    S = candidates(J, k, 2)
    eng = _engine(J, k)
    for c in range(k):
        eng.set_candidate(c, S[c])
    eb, ea, iters, res = run_policy(eng, policy, k, max_iterations=1000, seed=11, indptr=J.indptr,
                                    indices=J.indices)
    ref = {"fixed_guard": lambda: G.guarded_search(J, S, 11, adaptive=False),
           "adaptive_guard": lambda: G.guarded_search(J, S, 11, adaptive=True),
           "independent_set": lambda: G.independent_set_search(J, S, 11),
           "sequential_oracle": lambda: G.sequential_oracle(J, S)}[policy]()
    assert res.integer_gains == 1
    assert np.array_equal(eb, O.integer_energies(J, S).astype(np.float64))
    assert np.array_equal(ea, ref.energies)
    assert iters == ref.rounds
    if policy in ("fixed_guard", "adaptive_guard"):
        assert res.final_rounds == ref.final_rounds
        assert (res.accepted, res.rejected) == (ref.accepted, ref.rejected)
    for c in range(k):
        assert np.array_equal(eng.candidate_spins(c, refined=True).cpu().numpy(), ref.spins[c]), c


@pytest.mark.gpu
@pytest.mark.parametrize("policy", ["fixed_guard", "adaptive_guard", "independent_set", "sequential_oracle"])
def test_gpu_solvers_with_guarded_policies(golden_cases, policy):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import json
    import scipy.sparse as sp
    from specann_b200.spec_adj import Alpha0GPU, Alpha1GPU
    from specann_b200.spectral_annealing import SpectralAnnealing
    z = golden_cases["tiny_ba100_specann32"]
    n = int(z["n"])
    J = sp.csr_matrix((z["data"], z["indices"], z["indptr"]), shape=(n, n))
    s = SpectralAnnealing("g.txt", "g", random_seed=42, num_alphas=16, ls_policy=policy)
    energy, spins, _ = s.solve(J)
    assert O.exact_energy(J, spins) == energy
    # the refined candidates are the oracle policy's on the solver's own candidates
    k = s._num_candidates
    cands = np.stack([s.engine.candidate_spins(c).cpu().numpy() for c in range(k)])
    ref = {"fixed_guard": lambda: G.guarded_search(J, cands, 42, adaptive=False),
           "adaptive_guard": lambda: G.guarded_search(J, cands, 42, adaptive=True),
           "independent_set": lambda: G.independent_set_search(J, cands, 42),
           "sequential_oracle": lambda: G.sequential_oracle(J, cands)}[policy]()
    raw = O.integer_energies(J, cands)
    assert energy == float(min(raw.min(), ref.energies.min()))
    for cls in (Alpha0GPU, Alpha1GPU):
        e, sp_, _ = cls("g.txt", "g", random_seed=42, ls_policy=policy).solve(J)
        assert O.exact_energy(J, sp_) == e
