"""The C-ABI library loads without a GPU and exports every symbol include/specann_b200.h declares;
the ctypes binding covers exactly those symbols. No compute calls are made here."""
import ctypes
import re
from pathlib import Path

import pytest

from specann_b200 import _lib, build

ROOT = Path(__file__).resolve().parent.parent


def header_symbols():
    text = (ROOT / "include" / "specann_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sa_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib_path():
    build.build_all()
    return _lib.LIB_PATH


def test_library_loads_and_exports_every_declared_symbol(lib_path):
    lib = ctypes.CDLL(str(lib_path))
    syms = header_symbols()
    assert len(syms) >= 19
    for s in syms:
        assert hasattr(lib, s), s


def test_binding_matches_header():
    assert sorted(_lib.SIGNATURES) == header_symbols()


def test_version_string(lib_path):
    lib = _lib.load()
    assert b"sm_100a" in lib.sa_version()


def test_workspace_size_is_host_only(lib_path):
    lib = _lib.load()
    nbytes = ctypes.c_size_t()
    assert lib.sa_workspace_size(1 << 20, 41942240, 0, 32, 33, 128, ctypes.byref(nbytes)) == 0
    assert nbytes.value > 33 * (1 << 20) * 4
    assert lib.sa_workspace_size(0, 10, 0, 32, 33, 128, ctypes.byref(nbytes)) == _lib.SA_ERR_INVALID_ARG
    assert lib.sa_workspace_size(10, 10, 0, 16, 33, 128, ctypes.byref(nbytes)) == _lib.SA_ERR_INVALID_ARG


def test_struct_layouts_match_c():
    # sizes of the C structs on x86-64 (natural alignment)
    assert ctypes.sizeof(_lib.AlphaParams) == 7 * 8 + 4 * 4 + 8 + 8 + 8 + 4 * 4
    assert ctypes.sizeof(_lib.AlphaRecord) == 4 * 4 + 7 * 8 + 8 + 4 * 4 + 8 + 6 * 8
    assert ctypes.sizeof(_lib.LsParams) == 4 * 3 + 4 + 2 * 8 + 2 * 4 + 8 + 2 * 4
    assert ctypes.sizeof(_lib.LsResult) == 4 * 4 + 8 + 4 * 8
    assert ctypes.sizeof(_lib.GuardParams) == 4 * 4 + 2 * 8 + 2 * 4 + 8 + 2 * 8 + 2 * 4
    assert ctypes.sizeof(_lib.GuardResult) == 6 * 4 + 8


def test_graph_library():
    from specann_b200 import graphs
    import numpy as np
    J = graphs.barabasi_albert(300, 5, seed=3)
    assert J.nnz == 2 * 5 * (300 - 5)
    assert (J != J.T).nnz == 0 and J.diagonal().sum() == 0
    assert np.diff(J.indptr).min() >= 5
    J2 = graphs.barabasi_albert(300, 5, seed=3)
    assert (J != J2).nnz == 0
    E = graphs.erdos_renyi(500, 0.05, seed=1, couplings="pm1")
    assert set(np.unique(E.data)) <= {-1.0, 1.0} and (E != E.T).nnz == 0
    I = graphs.barabasi_albert(200, 3, seed=1, couplings="int100")
    assert np.all(np.abs(I.data) <= 100) and np.all(I.data != 0) and (I != I.T).nnz == 0
