"""Instance loader with the interface of the reference's utils/data_loader.py (DataLoader,
InstanceIndex, DataLoadError), parsed natively (specann_b200/csrc/loader.cpp): the Gset format and
the linear-bias format (fields carried by an extra bias node), duplicates summed, isolated nodes
removed. The matrix it returns is what SpectralAnnealing.solve takes (SciPy CSR, float64)."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from pathlib import Path
from typing import List

import numpy as np
import scipy.sparse as sp

from . import _lib

_ERRORS = {1: "bad arguments", 2: "file cannot be read", 3: "malformed header or field lines",
           4: "an infinite node number", 5: "more than 2^31 - 1 nodes"}


class DataLoadError(Exception):
    """An instance file could not be read (utils/data_loader.py:18-19)."""


@dataclass
class InstanceIndex:
    """Rows of the loaded matrix -> nodes of the file (utils/data_loader.py:22-36)."""
    n_original: int
    n_solve: int
    node_ids: np.ndarray
    bias_node_index: int = -1
    id_base: int = 1
    weights_negated: bool = False
    J_sum: float = 0.0


def load_file(path, gset: bool, return_index: bool = False):
    """Parse one instance file into a CSR matrix (and its InstanceIndex)."""
    g = _lib.load_graphs()
    h = C.c_void_p()
    n, nnz, n0, bias = C.c_int64(), C.c_int64(), C.c_int64(), C.c_int64()
    st = g.sa_instance_load(str(path).encode(), int(bool(gset)), C.byref(h), C.byref(n), C.byref(nnz),
                            C.byref(n0), C.byref(bias))
    if st != 0:
        kind = "Gset" if gset else "linear bias"
        raise DataLoadError(f"Error reading {kind} file {path}: {_ERRORS.get(st, st)}")
    rowptr = np.empty(n.value + 1, dtype=np.int64)
    col = np.empty(nnz.value, dtype=np.int32)
    val = np.empty(nnz.value, dtype=np.float64)
    ids = np.empty(n.value, dtype=np.int64)
    st = g.sa_instance_fetch(h, rowptr.ctypes.data_as(C.c_void_p), col.ctypes.data_as(C.c_void_p),
                             val.ctypes.data_as(C.c_void_p), ids.ctypes.data_as(C.c_void_p))
    if st != 0:
        raise DataLoadError(f"Error reading {path}: {_ERRORS.get(st, st)}")
    idx = rowptr.astype(np.int32) if nnz.value < 2 ** 31 else rowptr
    J = sp.csr_matrix((val, col, idx), shape=(n.value, n.value))
    if not return_index:
        return J
    index = InstanceIndex(n_original=int(n0.value), n_solve=int(n.value), node_ids=ids,
                          bias_node_index=int(bias.value), id_base=1, weights_negated=bool(gset),
                          J_sum=float(val.sum()))
    return J, index


class DataLoader:
    """Load the instances of one dataset folder (datasets/<name>); a name containing "gset" selects
    the Gset format, any other the linear-bias format (utils/data_loader.py:39-64)."""

    def __init__(self, dataset_name: str, datasets_path: str = "datasets"):
        self.dataset_name = dataset_name
        self.dataset_path = Path(datasets_path) / dataset_name
        if not self.dataset_path.exists():
            raise ValueError(f"Dataset path does not exist: {self.dataset_path}")
        self.dataset_format = 'gset' if 'gset' in dataset_name.lower() else 'graph_linear_bias'

    def list_instances(self) -> List[str]:
        return sorted(f.name for f in self.dataset_path.glob("*.txt"))

    def load_instance(self, instance_name: str, return_index: bool = False):
        path = self.dataset_path / instance_name
        if not path.exists():
            raise FileNotFoundError(f"Instance file not found: {path}")
        return load_file(path, self.dataset_format == 'gset', return_index)
