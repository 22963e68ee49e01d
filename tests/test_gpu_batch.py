"""Batched sweeps (sa_batch_*): every (instance, seed) problem of one launch against the
single-problem path and the oracle. Eigenvalues agree with the single-problem solves to the
Lanczos tolerance (the reductions run in a different order, so vectors differ in the last bits);
the local search is bit-exact against the oracle on the batch's own candidates; graph replays
repeat a launch exactly; multi-CTA teams give the same answers as single-CTA teams."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from oracle import specann_oracle as O  # noqa: E402
from specann_b200 import graphs  # noqa: E402
from specann_b200.batch import BatchedSpectralAnnealing, unpack_words  # noqa: E402
from specann_b200.spectral_annealing import SpectralAnnealing  # noqa: E402


def instances():
    return [graphs.erdos_renyi(1024, 20 / 1023, seed=42, couplings="pm1"),
            graphs.barabasi_albert(3000, 5, seed=2, couplings="pm1"),
            graphs.erdos_renyi(700, 0.03, seed=5),
            graphs.barabasi_albert(5000, 10, seed=3, couplings="int100")]


PARAMS = dict(num_alphas=16, schedule="linear")


@pytest.fixture(scope="module")
def batch_run():
    Js = instances()
    b = BatchedSpectralAnnealing(seeds=(42, 7), **PARAMS)
    b.load(Js)
    b.sweep()
    res = b.results()
    yield b, Js, res
    b.close()


def candidates(b, p, k, n, refined=False):
    import ctypes as C
    out = []
    for c in range(k):
        w = torch.empty((n + 31) // 32, dtype=torch.int32, device="cuda")
        assert b.lib.sa_batch_candidate(b._batch, p, c, int(refined), C.c_void_p(w.data_ptr())) == 0
        out.append(unpack_words(w.cpu().numpy().view(np.uint32), n))
    return np.stack(out)


def test_every_problem_solved(batch_run):
    b, Js, res = batch_run
    assert len(res) == len(Js) * 2
    for r in res:
        assert r["status"] == 0 and r["num_candidates"] >= 1
        assert O.exact_energy(Js[r["instance"]], r["spins"]) == r["energy"]
        for row in r["rows"]:
            assert row["candidate"] >= 0 and row["eigsh_converged"], row
            assert row["eigsh_residual"] < 1e-4


def test_eigenvalues_match_single_problem_path(batch_run):
    b, Js, res = batch_run
    for r in res:
        J = Js[r["instance"]]
        s = SpectralAnnealing("b.txt", "batch", random_seed=r["seed"], write_results=False, **PARAMS)
        s.solve(J)
        lam_single = np.array([x["lambda1"] for x in s.alpha_results])
        lam_batch = np.array([x["lambda1"] for x in r["rows"]])
        assert np.max(np.abs(lam_single - lam_batch)) < 2e-5


def test_local_search_bit_exact_on_batch_candidates(batch_run):
    b, Js, res = batch_run
    for p, r in enumerate(res):
        J = Js[r["instance"]]
        n, k = J.shape[0], r["num_candidates"]
        S = candidates(b, p, k, n)
        # distinct candidates in order of first appearance
        assert len({s.tobytes() for s in S}) == k
        first = []
        for row in r["rows"]:
            if row["candidate"] not in first:
                first.append(row["candidate"])
        assert first == list(range(k))
        ref = O.local_search(J, S, seed=r["seed"])
        assert np.array_equal(r["energy_before"], ref.energies_before.astype(np.float64))
        assert np.array_equal(r["energy_after"], ref.energies_after.astype(np.float64))
        assert r["ls_iterations"] == ref.iterations
        assert np.array_equal(candidates(b, p, k, n, refined=True), ref.spins)


def test_graph_replay_repeats_the_launch(batch_run):
    b, Js, res = batch_run
    b.sweep()
    res2 = b.results()
    for r1, r2 in zip(res, res2):
        assert r1["energy"] == r2["energy"]
        assert [x["lambda1"] for x in r1["rows"]] == [x["lambda1"] for x in r2["rows"]]
        assert np.array_equal(r1["energy_after"], r2["energy_after"])


def test_multi_cta_teams_agree():
    Js = instances()
    runs = []
    for split in (1e-4, 1.0):            # one CTA per problem; large teams
        b = BatchedSpectralAnnealing(seeds=(42,), split=split, use_graph=False, **PARAMS)
        b.load(Js)
        b.sweep()
        runs.append((b.team_nb.max(), b.results()))
        b.close()
    assert runs[0][0] == 1 and runs[1][0] >= 2
    for r1, r2 in zip(runs[0][1], runs[1][1]):
        l1 = np.array([x["lambda1"] for x in r1["rows"]])
        l2 = np.array([x["lambda1"] for x in r2["rows"]])
        assert np.max(np.abs(l1 - l2)) < 2e-5
        J = Js[r2["instance"]]
        assert O.exact_energy(J, r2["spins"]) == r2["energy"]


def test_autotune_picks_a_measured_plan():
    Js = instances()[:2]
    b = BatchedSpectralAnnealing(seeds=(1, 2), num_alphas=8, schedule="linear")
    b.load(Js)
    times = b.autotune(splits=(0.5, 4.0), num_alphas=4)
    assert set(times) == {0.5, 4.0} and all(t > 0 for t in times.values())
    assert b._costs is not None and len(b._costs) == 4
    out = b.solve()
    assert len(out) == 4 and all(np.isfinite(e) for e, _, _ in out)
    b.close()


def test_c3_ragged_workload_at_its_shape():
    """C3: 64 ragged instances (n log-uniform in [2^10, 2^17], half ER degree 20, half BA m 10/20, +-1
    couplings) x 4 seeds x 128 sqrt alphas in one launch. Every problem solves with every alpha
    converged to a residual <= 1e-5; the smallest instances' eigenvalues match dense FP64 eigh at every
    alpha; the local search is bit-exact against the oracle on sampled problems' own candidates."""
    import scipy.linalg as sla
    import scipy.sparse as sp
    inst = graphs.ragged_batch()
    Js = [J for _, J in inst]
    assert len(Js) == 64
    b = BatchedSpectralAnnealing(seeds=(42, 43, 44, 45), num_alphas=128)
    b.load(Js)
    b.sweep()
    res = b.results()
    assert len(res) == 256
    for r in res:
        J = Js[r["instance"]]
        assert r["status"] == 0 and r["num_candidates"] >= 1
        assert O.exact_energy(J, r["spins"]) == r["energy"]
        assert len(r["rows"]) == 128
        for row in r["rows"]:
            assert row["eigsh_converged"] and row["eigsh_residual"] <= 1e-5, row
    small = sorted(range(64), key=lambda i: Js[i].shape[0])[:3]
    alphas = O.alpha_schedule("sqrt", 128)
    for i in small:
        J = Js[i]
        n = J.shape[0]
        deg = np.asarray(abs(J).sum(axis=1)).ravel()
        lam64 = []
        for a in alphas:
            M, _ = O.scaled_operator_f64(J, deg, deg.max(), a)
            lam64.append(float(sla.eigh(M.toarray(), eigvals_only=True, subset_by_index=[n - 1, n - 1])[0]))
        for r in res:
            if r["instance"] == i:
                lam = np.array([x["lambda1"] for x in r["rows"]])
                assert np.max(np.abs(lam - np.array(lam64))) <= 1e-5
    for p in range(0, 256, 37):
        r = res[p]
        J = Js[r["instance"]]
        S = candidates(b, p, r["num_candidates"], J.shape[0])
        ref = O.local_search(J, S, seed=r["seed"])
        assert np.array_equal(r["energy_after"], ref.energies_after.astype(np.float64))
        assert np.array_equal(candidates(b, p, r["num_candidates"], J.shape[0], refined=True), ref.spins)
    b.close()
