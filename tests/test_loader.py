"""The native instance loader (specann_b200/loader.py over csrc/loader.cpp) against golden outputs of
the reference's utils/data_loader.py on synthetic files with irregular lines
(tests/golden/make_loader_golden.py)."""
import sys
from pathlib import Path

import numpy as np
import pytest

from specann_b200 import build, loader

GOLDEN = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(GOLDEN))
from make_loader_golden import write_instance_files  # noqa: E402


@pytest.fixture(scope="module")
def files(tmp_path_factory):
    build.build_all()
    root = tmp_path_factory.mktemp("instances")
    return root, write_instance_files(root)


def test_loader_matches_reference_outputs(files):
    root, fl = files
    z = np.load(GOLDEN / "loader_golden.npz")
    for k, (ds, name) in enumerate(fl):
        J, idx = loader.DataLoader(ds, datasets_path=str(root)).load_instance(name, return_index=True)
        assert tuple(J.shape) == tuple(z[f"f{k}_shape"])
        assert np.array_equal(J.indptr.astype(np.int64), z[f"f{k}_indptr"]), name
        assert np.array_equal(J.indices, z[f"f{k}_indices"]), name
        assert np.array_equal(J.data, z[f"f{k}_data"]), name
        assert np.array_equal(idx.node_ids, z[f"f{k}_node_ids"])
        meta = z[f"f{k}_meta"]
        assert (idx.n_original, idx.n_solve, idx.bias_node_index, int(idx.weights_negated)) == tuple(meta)
        assert idx.J_sum == pytest.approx(float(z[f"f{k}_J_sum"]), abs=1e-12)
        assert (J != J.T).nnz == 0


def test_loader_errors(tmp_path):
    (tmp_path / "ds").mkdir()
    (tmp_path / "ds" / "bad.txt").write_text("not a header\n")
    dl = loader.DataLoader("ds", datasets_path=str(tmp_path))
    with pytest.raises(loader.DataLoadError):
        dl.load_instance("bad.txt")
    with pytest.raises(FileNotFoundError):
        dl.load_instance("missing.txt")
    with pytest.raises(ValueError):
        loader.DataLoader("nope", datasets_path=str(tmp_path))
