"""ctypes binding of libspecann_b200.so (the C-ABI declared in include/specann_b200.h).

The library is built in-tree by specann_b200/build.py. There is no CPU fallback: when the library is
missing or no CUDA device is present, every call that would compute raises.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

from .failures import EigensolverBreakdown, NumericalFailure, SpecAnnOutOfMemory

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libspecann_b200.so"
GRAPH_LIB_PATH = PKG / "libspecann_graphs.so"

SA_OK = 0
SA_ERR_BREAKDOWN = 1
SA_ERR_NONFINITE = 2
SA_ERR_NOT_CONVERGED = 3
SA_ERR_OOM = 4
SA_ERR_INVALID_ARG = 5
SA_ERR_CUDA = 6
SA_ERR_BARRIER_TIMEOUT = 7

STATUS_NAMES = {0: "OK", 1: "BREAKDOWN", 2: "NONFINITE", 3: "NOT_CONVERGED", 4: "OOM", 5: "INVALID_ARG",
                6: "CUDA_ERROR", 7: "BARRIER_TIMEOUT"}

SA_START_RANDOM, SA_START_PREV, SA_START_DIAGONAL, SA_START_SECANT, SA_START_GIVEN, SA_START_TANGENT = range(6)
NCV_MAX = 64          # largest Lanczos basis of the kernels


class AlphaParams(C.Structure):
    _fields_ = [("alpha", C.c_double), ("alpha_prev", C.c_double), ("rho", C.c_double),
                ("gershgorin", C.c_double), ("tol", C.c_double), ("pred_tol", C.c_double),
                ("secant_gamma", C.c_double), ("maxiter", C.c_int32), ("ncv", C.c_int32),
                ("start_mode", C.c_int32), ("align", C.c_int32), ("seed", C.c_uint64),
                ("stream_id", C.c_int64), ("v0", C.c_void_p), ("round", C.c_int32),
                ("residual_check", C.c_int32), ("restart_keep", C.c_int32), ("reserved", C.c_int32)]


class AlphaRecord(C.Structure):
    _fields_ = [("status", C.c_int32), ("iterations", C.c_int32), ("restarts", C.c_int32),
                ("pred_accepted", C.c_int32), ("mu", C.c_double), ("lambda1", C.c_double),
                ("residual", C.c_double), ("res_estimate", C.c_double), ("pred_residual", C.c_double),
                ("degree_scale", C.c_double), ("align_dot", C.c_double), ("signature", C.c_uint64),
                ("nonfinite", C.c_int32), ("basis_used", C.c_int32), ("spmv_count", C.c_int32),
                ("reserved", C.c_int32), ("alg_bytes", C.c_double), ("phase_ms", C.c_double * 6)]


class LsParams(C.Structure):
    _fields_ = [("k", C.c_int32), ("first_slot", C.c_int32), ("max_iterations", C.c_int32),
                ("subset_fraction", C.c_double),
                ("final_sweep_fraction", C.c_double), ("final_sweep_iters", C.c_int32),
                ("num_rounds", C.c_int32), ("seed", C.c_uint64), ("semantics", C.c_int32),
                ("reserved", C.c_int32)]


class LsResult(C.Structure):
    _fields_ = [("status", C.c_int32), ("iterations", C.c_int32), ("final_passes", C.c_int32),
                ("integer_gains", C.c_int32), ("total_flips", C.c_int64), ("phase_ms", C.c_double * 4)]


# name -> (restype, argtypes): every symbol include/specann_b200.h declares
SA_ADJ_GRADIENT, SA_ADJ_TANGENT, SA_ADJ_SOLVE = range(3)


SA_GUARD_FIXED, SA_GUARD_ADAPTIVE, SA_GUARD_INDEPENDENT_SET, SA_GUARD_SEQUENTIAL = 1, 2, 3, 4


class GuardParams(C.Structure):
    _fields_ = [("k", C.c_int32), ("first_slot", C.c_int32), ("policy", C.c_int32), ("max_iterations", C.c_int32),
                ("subset_fraction", C.c_double), ("final_sweep_fraction", C.c_double),
                ("final_sweep_iters", C.c_int32), ("num_rounds", C.c_int32), ("seed", C.c_uint64),
                ("colors", C.c_void_p), ("color_seq", C.c_void_p), ("num_colors", C.c_int32),
                ("reserved", C.c_int32)]


class GuardResult(C.Structure):
    _fields_ = [("status", C.c_int32), ("rounds", C.c_int32), ("final_rounds", C.c_int32), ("accepted", C.c_int32),
                ("rejected", C.c_int32), ("integer_gains", C.c_int32), ("flips", C.c_int64)]


class AdjointParams(C.Structure):
    _fields_ = [("alpha", C.c_double), ("lambda1", C.c_double), ("beta", C.c_double), ("tol", C.c_double),
                ("maxiter", C.c_int32), ("mode", C.c_int32), ("y", C.c_void_p), ("rhs", C.c_void_p),
                ("out", C.c_void_p), ("grad", C.c_void_p)]


class AdjointResult(C.Structure):
    _fields_ = [("status", C.c_int32), ("iterations", C.c_int32), ("spmv_count", C.c_int32),
                ("reserved", C.c_int32), ("residual", C.c_double), ("loss", C.c_double),
                ("dloss_dalpha", C.c_double)]


class BatchConfig(C.Structure):
    _fields_ = [("eigsh_tol", C.c_double), ("pred_tol", C.c_double), ("shift_eps", C.c_double),
                ("secant_gamma", C.c_double), ("subset_fraction", C.c_double), ("final_sweep_fraction", C.c_double),
                ("num_alphas", C.c_int32), ("maxiter", C.c_int32), ("ncv", C.c_int32), ("pred_mode", C.c_int32),
                ("warm_start", C.c_int32), ("residual_check", C.c_int32), ("use_local_search", C.c_int32),
                ("max_local_iterations", C.c_int32), ("final_sweep_iters", C.c_int32), ("num_rounds", C.c_int32),
                ("ls_semantics", C.c_int32), ("reserved", C.c_int32)]


class BatchAlphaRecord(C.Structure):
    _fields_ = [("alpha", C.c_double), ("lambda1", C.c_double), ("rho", C.c_double), ("gershgorin", C.c_double),
                ("residual", C.c_double), ("pred_residual", C.c_double), ("degree_scale", C.c_double),
                ("signature", C.c_uint64), ("status", C.c_int32), ("iterations", C.c_int32),
                ("restarts", C.c_int32), ("spmv_count", C.c_int32), ("pred_accepted", C.c_int32),
                ("retry", C.c_int32), ("converged", C.c_int32), ("candidate", C.c_int32)]


class BatchSummary(C.Structure):
    _fields_ = [("status", C.c_int32), ("num_candidates", C.c_int32), ("ls_iterations", C.c_int32),
                ("ls_final_passes", C.c_int32), ("alphas_skipped", C.c_int32), ("alphas_retried", C.c_int32),
                ("team_first_block", C.c_int32), ("team_blocks", C.c_int32), ("integer_gains", C.c_int32),
                ("reserved", C.c_int32), ("ls_total_flips", C.c_int64), ("device_ms", C.c_double),
                ("phase_ms", C.c_double * 6), ("ls_ms", C.c_double),
                ("energy_before", C.c_double * 128), ("energy_after", C.c_double * 128)]


_I32P = C.POINTER(C.c_int32)

SIGNATURES = {
    "sa_version": (C.c_char_p, []),
    "sa_spmv_scaled_noalloc": (C.c_int, [C.c_int64, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double,
                                         C.c_double, C.c_void_p, C.c_void_p, C.c_void_p]),
    "sa_kernel_launches": (C.c_uint64, []),
    "sa_workspace_size": (C.c_int, [C.c_int64, C.c_int64, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                    C.POINTER(C.c_size_t)]),
    "sa_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_int64, C.c_int64, C.c_int32, C.c_int32, C.c_int32,
                            C.c_int32, C.c_void_p, C.c_size_t, C.c_void_p]),
    "sa_destroy": (C.c_int, [C.c_void_p]),
    "sa_set_matrix": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_double),
                                C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_int32)]),
    "sa_spmv_scaled": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_void_p, C.c_void_p]),
    "sa_set_spmv_policy": (C.c_int, [C.c_void_p, C.c_int32]),
    "sa_operator_status": (C.c_int, [C.c_void_p, _I32P]),
    "sa_barrier_selftest": (C.c_int, [C.c_int32, C.c_int32, C.c_uint64, C.c_void_p, C.c_size_t, _I32P, _I32P,
                                      _I32P, C.c_void_p]),
    "sa_panel_workspace_size": (C.c_int, [C.c_void_p, C.POINTER(C.c_size_t), C.POINTER(C.c_int32)]),
    "sa_panel_build": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t]),
    "sa_panel_enable": (C.c_int, [C.c_void_p, C.c_int32]),
    "sa_split_workspace_size": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_size_t), C.POINTER(C.c_int32)]),
    "sa_split_build": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_size_t]),
    "sa_split_enable": (C.c_int, [C.c_void_p, C.c_int32]),
    "sa_split_count": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_double)]),
    "sa_panel_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                C.POINTER(C.c_int32), C.POINTER(C.c_double)]),
    "sa_get_spmv_policy": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_double)]),
    "sa_panel_tables": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]),
    "sa_alpha_solve": (C.c_int, [C.c_void_p, C.POINTER(AlphaParams), C.POINTER(AlphaRecord)]),
    "sa_result_vector": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "sa_commit_alpha": (C.c_int, [C.c_void_p]),
    "sa_set_last_vector": (C.c_int, [C.c_void_p, C.c_void_p]),
    "sa_round_vector": (C.c_int, [C.c_void_p, C.c_double, C.c_void_p, C.c_int32, C.POINTER(C.c_uint64)]),
    "sa_candidate_keep": (C.c_int, [C.c_void_p, C.c_int32]),
    "sa_candidate_equal": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_int32)]),
    "sa_candidate_set": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p]),
    "sa_candidate_get": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p]),
    "sa_candidate_unpack": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p]),
    "sa_ls_workspace_size": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_size_t)]),
    "sa_local_search": (C.c_int, [C.c_void_p, C.POINTER(LsParams), C.c_void_p, C.c_size_t,
                                  C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(LsResult)]),
    "sa_energies": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_size_t, C.POINTER(C.c_double)]),
    "sa_guard_workspace_size": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_size_t)]),
    "sa_guard_search": (C.c_int, [C.c_void_p, C.POINTER(GuardParams), C.c_void_p, C.c_size_t, C.POINTER(C.c_double),
                                  C.POINTER(C.c_double), C.POINTER(GuardResult)]),
    "sa_set_exponent_offsets": (C.c_int, [C.c_void_p, C.c_void_p]),
    "sa_adjoint_workspace_size": (C.c_int, [C.c_void_p, C.POINTER(C.c_size_t)]),
    "sa_adjoint": (C.c_int, [C.c_void_p, C.POINTER(AdjointParams), C.c_void_p, C.c_size_t,
                             C.POINTER(AdjointResult)]),
    "sa_batch_grid": (C.c_int, [C.c_int32, C.c_int32, _I32P]),
    "sa_batch_plan": (C.c_int, [C.c_int32, C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_double),
                                C.c_int32, C.c_double, C.c_double, _I32P, _I32P, _I32P, _I32P]),
    "sa_batch_workspace_size": (C.c_int, [C.c_int32, C.POINTER(C.c_void_p), C.c_int32, C.c_int32, C.c_int32,
                                          C.c_int32, _I32P, _I32P, _I32P, C.POINTER(C.c_size_t)]),
    "sa_batch_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_int32, C.POINTER(C.c_void_p), C.c_int32,
                                  C.POINTER(C.c_uint64), C.c_int32, C.c_int32, C.c_int32, _I32P, _I32P, _I32P,
                                  C.c_void_p, C.c_size_t, C.c_void_p]),
    "sa_batch_sweep": (C.c_int, [C.c_void_p, C.POINTER(BatchConfig), C.POINTER(C.c_double), C.c_int32]),
    "sa_batch_results": (C.c_int, [C.c_void_p, C.POINTER(BatchAlphaRecord), C.POINTER(BatchSummary)]),
    "sa_batch_candidate": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_void_p]),
    "sa_batch_destroy": (C.c_int, [C.c_void_p]),
    "sa_coo_workspace_size": (C.c_int, [C.c_int64, C.c_int64, C.POINTER(C.c_size_t)]),
    "sa_coo_to_csr": (C.c_int, [C.c_int64, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t,
                                C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_int64),
                                C.POINTER(C.c_int64), C.c_void_p]),
}

GRAPH_SIGNATURES = {
    "sa_graph_ba_nnz": (C.c_int64, [C.c_int64, C.c_int64]),
    "sa_graph_ba": (C.c_int, [C.c_int64, C.c_int64, C.c_uint64, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]),
    "sa_graph_er_nnz": (C.c_int64, [C.c_int64, C.c_double, C.c_uint64]),
    "sa_graph_er": (C.c_int, [C.c_int64, C.c_double, C.c_uint64, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]),
    "sa_instance_load": (C.c_int, [C.c_char_p, C.c_int32, C.POINTER(C.c_void_p), C.POINTER(C.c_int64),
                                   C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "sa_instance_fetch": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "sa_instance_edges": (C.c_int, [C.c_char_p, C.c_int32, C.POINTER(C.c_void_p), C.POINTER(C.c_int64),
                                    C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "sa_instance_fetch_edges": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "sa_greedy_coloring": (C.c_int, [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_int32)]),
}

_lib = None
_glib = None


class SpecAnnError(RuntimeError):
    def __init__(self, fn, status):
        super().__init__(f"{fn} failed with status {STATUS_NAMES.get(status, status)}")
        self.status = status


def load(path: Path = LIB_PATH):
    """Load the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not Path(path).exists():
            raise RuntimeError(f"{path} is missing: build it with `python -m specann_b200.build`")
        lib = C.CDLL(str(path))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def load_graphs(path: Path = GRAPH_LIB_PATH):
    global _glib
    if _glib is None:
        if not Path(path).exists():
            raise RuntimeError(f"{path} is missing: build it with `python -m specann_b200.build`")
        lib = C.CDLL(str(path))
        for name, (res, args) in GRAPH_SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _glib = lib
    return _glib


def check(fn: str, status: int):
    """Map a C-ABI status onto the exceptions of the reference (utils/failures.py, EigensolverBreakdown)."""
    if status == SA_OK:
        return
    if status == SA_ERR_OOM:
        raise SpecAnnOutOfMemory(f"{fn}: workspace too small (out of memory)")
    if status in (SA_ERR_BREAKDOWN, SA_ERR_NONFINITE):
        raise EigensolverBreakdown(f"{fn}: {STATUS_NAMES[status]}")
    if status == SA_ERR_NOT_CONVERGED:
        raise NumericalFailure(f"{fn}: not converged")
    raise SpecAnnError(fn, status)
