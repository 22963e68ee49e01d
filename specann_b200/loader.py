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


def load_file_device(path, gset: bool, device=None):
    """Parse one instance file on the host into its edge list and build the CSR on the device
    (sa_coo_to_csr). Returns (row pointers int64, columns int32, couplings float64) as device tensors
    and the InstanceIndex; the matrix equals load_file's."""
    import torch
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    g = _lib.load_graphs()
    h = C.c_void_p()
    ne, nv, n0, bias = C.c_int64(), C.c_int64(), C.c_int64(), C.c_int64()
    st = g.sa_instance_edges(str(path).encode(), int(bool(gset)), C.byref(h), C.byref(ne), C.byref(nv),
                             C.byref(n0), C.byref(bias))
    if st != 0:
        kind = "Gset" if gset else "linear bias"
        raise DataLoadError(f"Error reading {kind} file {path}: {_ERRORS.get(st, st)}")
    m = ne.value
    ei = np.empty(m, dtype=np.int64)
    ej = np.empty(m, dtype=np.int64)
    ew = np.empty(m, dtype=np.float64)
    if g.sa_instance_fetch_edges(h, ei.ctypes.data_as(C.c_void_p), ej.ctypes.data_as(C.c_void_p),
                                 ew.ctypes.data_as(C.c_void_p)) != 0:
        raise DataLoadError(f"Error reading {path}")
    lib = _lib.load()
    nbytes = C.c_size_t(0)
    _lib.check("sa_coo_workspace_size", lib.sa_coo_workspace_size(m, nv.value, C.byref(nbytes)))
    ws = torch.empty(nbytes.value + 256, dtype=torch.uint8, device=dev)
    wp = (ws.data_ptr() + 255) & ~255
    d_ei, d_ej, d_ew = (torch.from_numpy(a).to(dev) for a in (ei, ej, ew))
    rowptr = torch.empty(nv.value + 1, dtype=torch.int64, device=dev)
    col = torch.empty(max(1, 2 * m), dtype=torch.int32, device=dev)
    val = torch.empty(max(1, 2 * m), dtype=torch.float64, device=dev)
    ids = torch.empty(nv.value, dtype=torch.int64, device=dev)
    n_out, nnz_out = C.c_int64(), C.c_int64()
    stream = torch.cuda.current_stream(dev)
    _lib.check("sa_coo_to_csr", lib.sa_coo_to_csr(m, nv.value, C.c_void_p(d_ei.data_ptr()), C.c_void_p(d_ej.data_ptr()),
                                                 C.c_void_p(d_ew.data_ptr()), C.c_void_p(wp), nbytes.value,
                                                 C.c_void_p(rowptr.data_ptr()), C.c_void_p(col.data_ptr()),
                                                 C.c_void_p(val.data_ptr()), C.c_void_p(ids.data_ptr()),
                                                 C.byref(n_out), C.byref(nnz_out), C.c_void_p(stream.cuda_stream)))
    n, nnz = int(n_out.value), int(nnz_out.value)
    rowptr, col, val, ids = rowptr[:n + 1], col[:nnz], val[:nnz], ids[:n]
    node_ids = ids.cpu().numpy()
    b = int(bias.value)
    b_new = int(np.flatnonzero(node_ids == b)[0]) if b >= 0 and np.any(node_ids == b) else -1
    index = InstanceIndex(n_original=int(n0.value), n_solve=n, node_ids=node_ids, bias_node_index=b_new,
                          id_base=1, weights_negated=bool(gset), J_sum=float(val.sum().item()) if nnz else 0.0)
    return rowptr, col, val, index


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
