"""The instance matrix built on the device (sa_coo_to_csr) against the native host loader, whose CSR
equals the reference loader's (tests/test_loader.py): instance files written here in both formats
with duplicates (summed in file order), self-loops and out-of-range nodes (dropped), fields (a bias
node), comment and malformed lines, isolated nodes (removed) and couplings that cancel to zero."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from oracle import specann_oracle as O  # noqa: E402
from specann_b200 import loader  # noqa: E402
from specann_b200.spectral_annealing import SpectralAnnealing  # noqa: E402


def write_instance(path, n, edges, fields=None, extra_lines=()):
    with open(path, "w") as f:
        f.write(f"{n} {len(edges)}\n")
        if fields is not None:
            for h in fields:
                f.write(f"{h}\n")
        for i, j, w in edges:
            f.write(f"{i} {j} {w}\n")
        for line in extra_lines:
            f.write(line + "\n")


def random_edges(rng, n, m, weights):
    i = rng.integers(1, n + 1, m)
    j = rng.integers(1, n + 1, m)
    w = rng.choice(weights, m)
    return list(zip(i.tolist(), j.tolist(), w.tolist()))


def compare(path, gset):
    J, idx = loader.load_file(path, gset, return_index=True)
    rp, col, val, didx = loader.load_file_device(path, gset)
    assert rp.numel() == J.shape[0] + 1 and col.numel() == J.nnz
    assert np.array_equal(rp.cpu().numpy(), J.indptr.astype(np.int64))
    assert np.array_equal(col.cpu().numpy(), J.indices)
    assert np.array_equal(val.cpu().numpy(), J.data)
    assert np.array_equal(didx.node_ids, idx.node_ids)
    assert (didx.n_original, didx.n_solve, didx.bias_node_index) == (idx.n_original, idx.n_solve, idx.bias_node_index)
    return J, rp, col, val


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_gset_format(tmp_path, seed):
    rng = np.random.default_rng(seed)
    n = 700
    edges = random_edges(rng, n, 6000, [1, -1, 2, 0.5])
    edges += [(5, 5, 1.0), (0, 3, 1.0), (n + 1, 2, 1.0), (3, 9, 1.0), (9, 3, -1.0)]   # self-loop, out of range, cancel
    write_instance(tmp_path / "g.txt", n, edges, extra_lines=["# comment", "% other", "1 2", "x y z", ""])
    compare(tmp_path / "g.txt", True)


@pytest.mark.parametrize("seed", [3, 4])
def test_linear_bias_format(tmp_path, seed):
    rng = np.random.default_rng(seed)
    n = 900
    edges = random_edges(rng, n, 4000, [1, -1, 3, -2])
    fields = np.where(rng.random(n) < 0.3, rng.integers(-3, 4, n), 0)
    write_instance(tmp_path / "b.txt", n, edges, fields=fields.tolist())
    J, rp, col, val = compare(tmp_path / "b.txt", False)
    # the device CSR solves like the host one
    s = SpectralAnnealing("b.txt", "b", random_seed=1, num_alphas=8, precision=64, write_results=False)
    e, spins, _ = s.solve_device(rp, col, val)
    assert O.exact_energy(J, spins) == e


def test_empty_and_isolated(tmp_path):
    write_instance(tmp_path / "e.txt", 50, [(1, 2, 1.0), (2, 1, -1.0), (7, 8, 2.0)])   # 1-2 cancels: removed
    compare(tmp_path / "e.txt", True)
    write_instance(tmp_path / "z.txt", 20, [])                                      # no entries: all kept
    compare(tmp_path / "z.txt", True)


def test_larger_instance_and_sort_passes(tmp_path):
    rng = np.random.default_rng(9)
    n = 70000                                         # keys above 2^32: five radix passes
    edges = random_edges(rng, n, 300000, [1, -1])
    write_instance(tmp_path / "l.txt", n, edges)
    compare(tmp_path / "l.txt", True)
