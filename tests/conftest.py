import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA kernels")
    config.addinivalue_line("markers", "slow: larger CPU cases")


@pytest.fixture(scope="session")
def golden_cases():
    import numpy as np
    out = {}
    for p in sorted(GOLDEN.glob("*.npz")):
        out[p.stem] = dict(np.load(p, allow_pickle=False))
    return out


@pytest.fixture(autouse=True)
def _results_in_tmp(tmp_path, monkeypatch):
    """Solvers write results/<dataset>/... relative to the cwd: keep tests out of the repo."""
    monkeypatch.chdir(tmp_path)
    yield
