"""Device-side engine: one handle of libspecann_b200.so over torch-allocated device memory.

torch provides device memory and the stream; all arithmetic runs in the library's kernels. The
engine owns: the device CSR (row pointers int32 or int64, columns int32, couplings in the working
precision), the handle workspace, and the local-search workspace.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional, Tuple

import numpy as np
import torch

from . import _lib
from ._lib import AdjointParams, AdjointResult, AlphaParams, AlphaRecord, LsParams, LsResult, check


def _require_cuda():
    if not torch.cuda.is_available():
        raise RuntimeError("specann_b200 needs a CUDA device (there is no CPU fallback)")


@dataclass
class MatrixInfo:
    c: float
    d_min: float
    d_max: float
    integer: bool


class Engine:
    """A solver handle: workspace, bound matrix, candidate store."""

    def __init__(self, n: int, nnz: int, precision: int = 32, ncv_max: int = 33, max_candidates: int = 128,
                 device: Optional[torch.device] = None, stream: Optional[torch.cuda.Stream] = None,
                 rowptr64: Optional[bool] = None):
        """rowptr64: 64-bit row pointers (the kernels' `long long` instantiations); None chooses them
        only when nnz does not fit in int32."""
        _require_cuda()
        self.lib = _lib.load()
        self.n, self.nnz = int(n), int(nnz)
        self.precision = int(precision)
        self.rowptr64 = self.nnz > np.iinfo(np.int32).max if rowptr64 is None else bool(rowptr64)
        self.ncv_max = int(ncv_max)
        self.max_candidates = int(max_candidates)
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.stream = stream if stream is not None else torch.cuda.current_stream(self.device)
        self.vdtype = torch.float32 if self.precision == 32 else torch.float64
        nbytes = C.c_size_t(0)
        check("sa_workspace_size", self.lib.sa_workspace_size(self.n, self.nnz, int(self.rowptr64), self.precision,
                                                              self.ncv_max, self.max_candidates, C.byref(nbytes)))
        self.workspace = torch.empty(int(nbytes.value) + 256, dtype=torch.uint8, device=self.device)
        base = self.workspace.data_ptr()
        self._ws_ptr = (base + 255) & ~255
        self._ws_bytes = int(nbytes.value)
        h = C.c_void_p()
        check("sa_create", self.lib.sa_create(C.byref(h), self.n, self.nnz, int(self.rowptr64), self.precision,
                                              self.ncv_max, self.max_candidates, C.c_void_p(self._ws_ptr),
                                              self._ws_bytes, C.c_void_p(self.stream.cuda_stream)))
        self.h = h
        self.ls_workspace = None
        self.info: Optional[MatrixInfo] = None
        # optional per-kernel timing (CUDA events on the engine's stream) for roofline reports
        self.profile = False
        self.stats = {"alpha_ms": 0.0, "alpha_bytes": 0.0, "alpha_launches": 0, "spmvs": 0,
                      "ls_ms": 0.0, "ls_launches": 0}

    def close(self):
        if getattr(self, "h", None):
            self.lib.sa_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- matrix -----------------------------------------------------------------------------
    def upload_csr(self, indptr: np.ndarray, indices: np.ndarray, data: np.ndarray) -> MatrixInfo:
        """H2D copy of a host CSR and the prelude (degrees, c, d, work list)."""
        rp_dtype = np.int64 if self.rowptr64 else np.int32
        val_dtype = np.float32 if self.precision == 32 else np.float64
        self.d_rowptr = torch.from_numpy(np.ascontiguousarray(indptr, dtype=rp_dtype)).to(self.device, non_blocking=False)
        self.d_col = torch.from_numpy(np.ascontiguousarray(indices, dtype=np.int32)).to(self.device)
        self.d_val = torch.from_numpy(np.ascontiguousarray(data, dtype=val_dtype)).to(self.device)
        return self.bind(self.d_rowptr, self.d_col, self.d_val)

    def bind(self, rowptr: torch.Tensor, col: torch.Tensor, val: torch.Tensor) -> MatrixInfo:
        """Bind device CSR tensors (kept alive by the engine) and run the prelude."""
        want_rp = torch.int64 if self.rowptr64 else torch.int32
        want_val = torch.float32 if self.precision == 32 else torch.float64
        if rowptr.dtype != want_rp or col.dtype != torch.int32 or val.dtype != want_val:
            raise ValueError(f"device CSR must be rowptr {want_rp}, col torch.int32, val {want_val}; got "
                             f"{rowptr.dtype}, {col.dtype}, {val.dtype}")
        if rowptr.numel() != self.n + 1 or col.numel() != self.nnz or val.numel() != self.nnz:
            raise ValueError("device CSR sizes do not match the engine's n and nnz")
        self.d_rowptr, self.d_col, self.d_val = rowptr, col, val
        c = C.c_double()
        dmin = C.c_double()
        dmax = C.c_double()
        integer = C.c_int32()
        check("sa_set_matrix", self.lib.sa_set_matrix(self.h, C.c_void_p(rowptr.data_ptr()), C.c_void_p(col.data_ptr()),
                                                      C.c_void_p(val.data_ptr()), C.byref(c), C.byref(dmin),
                                                      C.byref(dmax), C.byref(integer)))
        self.info = MatrixInfo(c=c.value, d_min=dmin.value, d_max=dmax.value, integer=bool(integer.value))
        return self.info

    # ---- operator ---------------------------------------------------------------------------
    def spmv(self, alpha: float, rho: float, x: torch.Tensor, y: Optional[torch.Tensor] = None) -> torch.Tensor:
        if y is None:
            y = torch.empty_like(x)
        check("sa_spmv_scaled", self.lib.sa_spmv_scaled(self.h, float(alpha), float(rho), C.c_void_p(x.data_ptr()),
                                                        C.c_void_p(y.data_ptr())))
        return y

    def operator_status(self) -> int:
        """Status of the standalone operator applications since the last call (synchronises the
        engine's stream; SA_ERR_BARRIER_TIMEOUT if a panel wait ran out)."""
        st = C.c_int32(0)
        check("sa_operator_status", self.lib.sa_operator_status(self.h, C.byref(st)))
        return int(st.value)

    def set_spmv_policy(self, packed_columns: bool = True) -> None:
        """SpMV stream policy: packed signed columns for one-magnitude couplings."""
        check("sa_set_spmv_policy", self.lib.sa_set_spmv_policy(self.h, 1 if packed_columns else 0))

    def panel_plan(self) -> Tuple[int, int]:
        """(bytes, row blocks) of the column-panel layout of the bound matrix."""
        nb, blocks = C.c_size_t(0), C.c_int32(0)
        check("sa_panel_workspace_size", self.lib.sa_panel_workspace_size(self.h, C.byref(nb), C.byref(blocks)))
        return int(nb.value), int(blocks.value)

    def panels_pay(self) -> bool:
        """The column-panel SpMV is chosen in FP32 when rows average at least 16 entries and every
        SM holds one row block (in FP64 the persistent kernels spill with its shared-memory budget
        and the alpha solve measured slower: 15.6 against 11.5 ms on BA(2^18, 20))."""
        if self.precision != 32 or self.n < 4096 or self.nnz < 16 * self.n:
            return False
        sms = torch.cuda.get_device_properties(self.device).multi_processor_count
        try:
            blocks = self.panel_plan()[1]
        except _lib.SpecAnnError:      # more panels than the layout supports
            return False
        return blocks <= sms

    def build_panels(self) -> int:
        """Lay the bound matrix out for the column-panel SpMV (a device workspace owned by this
        engine until the next bind) and switch the operator kernels to it. Returns its bytes."""
        nb = C.c_size_t(0)
        check("sa_panel_workspace_size", self.lib.sa_panel_workspace_size(self.h, C.byref(nb), None))
        self._panel_ws = torch.empty(max(256, nb.value), dtype=torch.uint8, device=self.device)
        check("sa_panel_build", self.lib.sa_panel_build(self.h, C.c_void_p(self._panel_ws.data_ptr()),
                                                        C.c_size_t(self._panel_ws.numel())))
        return nb.value

    def panel_info(self) -> dict:
        slots, blocks, panels, width, nb = C.c_int64(0), C.c_int32(0), C.c_int32(0), C.c_int32(0), C.c_double(0.0)
        check("sa_panel_info", self.lib.sa_panel_info(self.h, C.byref(slots), C.byref(blocks), C.byref(panels),
                                                      C.byref(width), C.byref(nb)))
        return {"slots": int(slots.value), "blocks": int(blocks.value), "panels": int(panels.value),
                "width": int(width.value), "matrix_bytes": float(nb.value)}

    def panel_tables(self):
        """Host copies of the built panel layout's tables: (entry words uint32[slots], chunk starts
        int64[blocks * panels * 16 + 1], block first rows int32[blocks + 1])."""
        info = self.panel_info()
        e, ch, r0 = C.c_void_p(), C.c_void_p(), C.c_void_p()
        check("sa_panel_tables", self.lib.sa_panel_tables(self.h, C.byref(e), C.byref(ch), C.byref(r0)))
        nb, npn = info["blocks"], info["panels"]
        ent = device_view(e.value, info["slots"], torch.int32, self.device).cpu().numpy().view(np.uint32)
        chunk = device_view(ch.value, nb * npn * 16 + 1, torch.int64, self.device).cpu().numpy()
        row0 = device_view(r0.value, nb + 1, torch.int32, self.device).cpu().numpy()
        return ent, chunk, row0

    def build_splits(self, splits: int = 0) -> int:
        """Lay the bound matrix out as L2 column splits (0: one per 48 MB of the gathered vector)
        and switch the operator kernels to it. Returns the number of splits."""
        nb, used = C.c_size_t(0), C.c_int32(0)
        check("sa_split_workspace_size", self.lib.sa_split_workspace_size(self.h, int(splits), C.byref(nb),
                                                                          C.byref(used)))
        self._split_ws = torch.empty(max(256, nb.value), dtype=torch.uint8, device=self.device)
        check("sa_split_build", self.lib.sa_split_build(self.h, int(splits), C.c_void_p(self._split_ws.data_ptr()),
                                                        C.c_size_t(self._split_ws.numel())))
        return int(used.value)

    def enable_splits(self, on: bool = True) -> None:
        check("sa_split_enable", self.lib.sa_split_enable(self.h, 1 if on else 0))

    def split_count(self) -> int:
        k = C.c_int32(0)
        check("sa_split_count", self.lib.sa_split_count(self.h, C.byref(k), None))
        return int(k.value)

    def split_bytes(self) -> float:
        """Algorithmic bytes of one split SpMV's matrix stream and partial sums (0 when off)."""
        k, b = C.c_int32(0), C.c_double(0.0)
        check("sa_split_count", self.lib.sa_split_count(self.h, C.byref(k), C.byref(b)))
        return float(b.value)

    def splits_pay(self) -> bool:
        """L2 column splits are chosen when the gathered vector is larger than 48 MB (a third of L2)."""
        return self.n * (4 if self.precision == 32 else 8) > 48 * 1024 * 1024

    def enable_panels(self, on: bool = True) -> None:
        check("sa_panel_enable", self.lib.sa_panel_enable(self.h, 1 if on else 0))

    def spmv_policy(self) -> dict:
        packed, mag = C.c_int32(0), C.c_double(0.0)
        check("sa_get_spmv_policy", self.lib.sa_get_spmv_policy(self.h, C.byref(packed), C.byref(mag)))
        return {"packed_columns": bool(packed.value), "magnitude": mag.value}

    # ---- one alpha --------------------------------------------------------------------------
    def alpha_solve(self, *, alpha, alpha_prev, rho, gershgorin, tol, pred_tol, maxiter, ncv, start_mode,
                    seed, stream_id, align=True, v0: Optional[torch.Tensor] = None, secant_gamma=1.0,
                    round_spins=True, residual_check=True, restart_keep=0) -> AlphaRecord:
        p = AlphaParams(alpha=float(alpha), alpha_prev=float(alpha_prev), rho=float(rho),
                        gershgorin=float(gershgorin), tol=float(tol), pred_tol=float(pred_tol),
                        secant_gamma=float(secant_gamma), maxiter=int(maxiter), ncv=int(ncv),
                        start_mode=int(start_mode), align=int(bool(align)), seed=int(seed) & (2 ** 64 - 1),
                        stream_id=int(stream_id), v0=C.c_void_p(v0.data_ptr()) if v0 is not None else None,
                        round=int(bool(round_spins)), residual_check=int(bool(residual_check)),
                        restart_keep=int(restart_keep))
        rec = AlphaRecord()
        if self.profile:
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(self.stream)
        check("sa_alpha_solve", self.lib.sa_alpha_solve(self.h, C.byref(p), C.byref(rec)))
        if self.profile:
            e1.record(self.stream)
            e1.synchronize()
            self.stats["alpha_ms"] += e0.elapsed_time(e1)
            self.stats["alpha_bytes"] += rec.alg_bytes
            self.stats["alpha_launches"] += 1
            self.stats["spmvs"] += rec.spmv_count
            ph = self.stats.setdefault("phase_ms", [0.0] * 6)
            for q in range(6):
                ph[q] += rec.phase_ms[q]
        return rec

    def result_vector(self) -> torch.Tensor:
        """A copy of the last solve's eigenvector y (device)."""
        ptr = C.c_void_p()
        check("sa_result_vector", self.lib.sa_result_vector(self.h, C.byref(ptr)))
        return device_view(ptr.value, self.n, self.vdtype, self.device).clone()

    def commit(self):
        check("sa_commit_alpha", self.lib.sa_commit_alpha(self.h))

    def set_last_vector(self, y: torch.Tensor):
        check("sa_set_last_vector", self.lib.sa_set_last_vector(self.h, C.c_void_p(y.data_ptr())))

    def round_vector(self, alpha: float, y: torch.Tensor, align: bool = True) -> int:
        sig = C.c_uint64()
        check("sa_round_vector", self.lib.sa_round_vector(self.h, float(alpha), C.c_void_p(y.data_ptr()),
                                                          int(bool(align)), C.byref(sig)))
        return int(sig.value)

    # ---- candidates -------------------------------------------------------------------------
    def keep_candidate(self, slot: int):
        check("sa_candidate_keep", self.lib.sa_candidate_keep(self.h, int(slot)))

    def candidate_equal(self, slot: int) -> bool:
        eq = C.c_int32()
        check("sa_candidate_equal", self.lib.sa_candidate_equal(self.h, int(slot), C.byref(eq)))
        return bool(eq.value)

    def set_candidate(self, slot: int, spins: np.ndarray):
        words = torch.from_numpy(pack_words(spins).view(np.int32)).to(self.device)
        check("sa_candidate_set", self.lib.sa_candidate_set(self.h, int(slot), C.c_void_p(words.data_ptr())))
        self.stream.synchronize()

    def candidate_words(self, slot: int, refined: bool = False) -> np.ndarray:
        W = (self.n + 31) // 32
        out = torch.empty(W, dtype=torch.int32, device=self.device)
        check("sa_candidate_get", self.lib.sa_candidate_get(self.h, int(slot), int(refined), C.c_void_p(out.data_ptr())))
        return out.cpu().numpy().view(np.uint32)

    def candidate_spins(self, slot: int, refined: bool = False) -> torch.Tensor:
        out = torch.empty(self.n, dtype=torch.int8, device=self.device)
        check("sa_candidate_unpack", self.lib.sa_candidate_unpack(self.h, int(slot), int(refined),
                                                                  C.c_void_p(out.data_ptr())))
        return out

    # ---- local search and energies -----------------------------------------------------------
    def _ls_ws(self, k: int):
        nbytes = C.c_size_t(0)
        check("sa_ls_workspace_size", self.lib.sa_ls_workspace_size(self.h, int(k), C.byref(nbytes)))
        need = int(nbytes.value) + 256
        if self.ls_workspace is None or self.ls_workspace.numel() < need:
            self.ls_workspace = torch.empty(need, dtype=torch.uint8, device=self.device)
        base = self.ls_workspace.data_ptr()
        return (base + 255) & ~255, int(nbytes.value)

    def local_search(self, k: int, *, first_slot=0, max_iterations=1000, subset_fraction=0.9,
                     final_sweep_fraction=1.0, final_sweep_iters=25, num_rounds=25, seed=0,
                     semantics: str = "priority"):
        ptr, nbytes = self._ls_ws(k)
        p = LsParams(k=int(k), first_slot=int(first_slot), max_iterations=int(max_iterations),
                     subset_fraction=float(subset_fraction),
                     final_sweep_fraction=float(final_sweep_fraction), final_sweep_iters=int(final_sweep_iters),
                     num_rounds=int(num_rounds), seed=int(seed) & (2 ** 64 - 1),
                     semantics={"priority": 0, "snapshot": 1}[semantics])
        eb = (C.c_double * k)()
        ea = (C.c_double * k)()
        res = LsResult()
        if self.profile:
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(self.stream)
        check("sa_local_search", self.lib.sa_local_search(self.h, C.byref(p), C.c_void_p(ptr), nbytes, eb, ea,
                                                          C.byref(res)))
        if self.profile:
            e1.record(self.stream)
            e1.synchronize()
            self.stats["ls_ms"] += e0.elapsed_time(e1)
            self.stats["ls_launches"] += 1
            ph = self.stats.setdefault("ls_phase_ms", [0.0] * 4)
            for q in range(4):
                ph[q] += res.phase_ms[q]
        return np.array(eb[:]), np.array(ea[:]), res

    def guard_search(self, policy: int, k: int, *, first_slot=0, max_iterations=1000, subset_fraction=0.9,
                     final_sweep_fraction=1.0, final_sweep_iters=25, num_rounds=25, seed=0,
                     colors: Optional[torch.Tensor] = None, color_seq: Optional[torch.Tensor] = None,
                     num_colors: int = 0):
        """Guarded local search of candidate slots first_slot .. first_slot + k - 1 (policy: one of
        _lib.SA_GUARD_*). Returns (energies before, energies after, GuardResult)."""
        nbytes = C.c_size_t(0)
        check("sa_guard_workspace_size", self.lib.sa_guard_workspace_size(self.h, int(k), C.byref(nbytes)))
        need = int(nbytes.value) + 256
        if getattr(self, "guard_workspace", None) is None or self.guard_workspace.numel() < need:
            self.guard_workspace = torch.empty(need, dtype=torch.uint8, device=self.device)
        ptr = (self.guard_workspace.data_ptr() + 255) & ~255
        p = _lib.GuardParams(k=int(k), first_slot=int(first_slot), policy=int(policy),
                             max_iterations=int(max_iterations), subset_fraction=float(subset_fraction),
                             final_sweep_fraction=float(final_sweep_fraction), final_sweep_iters=int(final_sweep_iters),
                             num_rounds=int(num_rounds), seed=int(seed) & (2 ** 64 - 1),
                             colors=C.c_void_p(colors.data_ptr()) if colors is not None else None,
                             color_seq=C.c_void_p(color_seq.data_ptr()) if color_seq is not None else None,
                             num_colors=int(num_colors))
        eb = (C.c_double * k)()
        ea = (C.c_double * k)()
        res = _lib.GuardResult()
        check("sa_guard_search", self.lib.sa_guard_search(self.h, C.byref(p), C.c_void_p(ptr), int(nbytes.value),
                                                          eb, ea, C.byref(res)))
        return np.array(eb[:]), np.array(ea[:]), res

    def energies(self, k: int) -> np.ndarray:
        ptr, nbytes = self._ls_ws(k)
        e = (C.c_double * k)()
        check("sa_energies", self.lib.sa_energies(self.h, int(k), C.c_void_p(ptr), nbytes, e))
        return np.array(e[:])

    # ---- differentiation form ----------------------------------------------------------------
    def set_exponent_offsets(self, offsets: Optional[torch.Tensor]):
        """Per-vertex exponent offsets (a_i = alpha + offsets_i) of the following solves and
        adjoints; None clears them. The tensor (float64, on the device) is kept alive here."""
        self._offsets = None if offsets is None else offsets.to(self.device, torch.float64).contiguous()
        ptr = C.c_void_p(self._offsets.data_ptr()) if self._offsets is not None else None
        check("sa_set_exponent_offsets", self.lib.sa_set_exponent_offsets(self.h, ptr))

    def adjoint(self, mode: int, *, alpha: float, lambda1: float, y: torch.Tensor, beta: float = 8.0,
                tol: float = 1e-6, maxiter: int = 2000, rhs: Optional[torch.Tensor] = None,
                out: Optional[torch.Tensor] = None, grad: Optional[torch.Tensor] = None) -> AdjointResult:
        nbytes = C.c_size_t(0)
        check("sa_adjoint_workspace_size", self.lib.sa_adjoint_workspace_size(self.h, C.byref(nbytes)))
        need = int(nbytes.value) + 256
        if getattr(self, "adj_workspace", None) is None or self.adj_workspace.numel() < need:
            self.adj_workspace = torch.empty(need, dtype=torch.uint8, device=self.device)
        ptr = (self.adj_workspace.data_ptr() + 255) & ~255
        p = AdjointParams(alpha=float(alpha), lambda1=float(lambda1), beta=float(beta), tol=float(tol),
                          maxiter=int(maxiter), mode=int(mode), y=C.c_void_p(y.data_ptr()),
                          rhs=C.c_void_p(rhs.data_ptr()) if rhs is not None else None,
                          out=C.c_void_p(out.data_ptr()) if out is not None else None,
                          grad=C.c_void_p(grad.data_ptr()) if grad is not None else None)
        res = AdjointResult()
        check("sa_adjoint", self.lib.sa_adjoint(self.h, C.byref(p), C.c_void_p(ptr), int(nbytes.value), C.byref(res)))
        if res.status not in (_lib.SA_OK, _lib.SA_ERR_NOT_CONVERGED):
            check("sa_adjoint", res.status)
        return res


class _CudaArray:
    """Minimal __cuda_array_interface__ holder for a raw device pointer."""

    def __init__(self, ptr: int, n: int, typestr: str):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3, "strides": None}


_TYPESTR = {torch.float32: "<f4", torch.float64: "<f8", torch.int8: "|i1", torch.int32: "<i4",
            torch.uint8: "|u1", torch.int64: "<i8"}


def device_view(ptr: int, n: int, dtype: torch.dtype, device) -> torch.Tensor:
    """Zero-copy torch view of n elements at a device pointer owned by the engine's workspace."""
    return torch.as_tensor(_CudaArray(ptr, n, _TYPESTR[dtype]), device=device)


def pack_words(spins: np.ndarray) -> np.ndarray:
    """Device layout of a rounded candidate: bit (j % 32) of uint32 word j // 32 is 1 iff s_j > 0."""
    s = np.asarray(spins)
    n = s.size
    nw = (n + 31) // 32
    bits = np.zeros(nw * 32, dtype=np.uint64)
    bits[:n] = s > 0
    return (bits.reshape(nw, 32) << np.arange(32, dtype=np.uint64)).sum(axis=1).astype(np.uint32)
