"""Batched SpecAnn: many (instance, seed) solves in one persistent launch.

The reference runs one solver object per (instance, seed) in a host loop (utils/core.py:103-105,
each a models/spectral_annealing.py:262-525 solve). `BatchedSpectralAnnealing` takes the same
solver parameters as `SpectralAnnealing` and a list of instances; every (instance, seed) problem
runs its full sweep (shift, predictor, alpha solve, cold retry, deduplication, warm start) and the
local search of its distinct candidates inside one cooperative kernel (sa_batch_sweep), optionally
replayed from a captured CUDA graph. Results per problem have the shape of SpectralAnnealing.solve:
(best energy, best spins, seconds) plus the per-alpha rows.

Which CTAs work on which problems is a plan (sa_batch_plan: LPT over a cost model, large problems
split over teams of CTAs); `autotune` measures a few plans on a short schedule and keeps the
fastest, so the SpMV / local-search tile-to-CTA mapping of a workload is picked by measurement.
"""
from __future__ import annotations

import ctypes as C
import time
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np
import scipy.sparse as sp
import torch

from . import _lib
from ._lib import BatchAlphaRecord, BatchConfig, BatchSummary, check
from .engine import Engine
from .failures import NumericalFailure
from .spectral_annealing import PRED_MODES, SCHEDULES, as_csr

_PRED = {"diagonal": _lib.SA_START_DIAGONAL, "secant": _lib.SA_START_SECANT, "prev": _lib.SA_START_PREV}

# plans measured by autotune, keyed by the workload's shape
_TUNED: Dict[tuple, float] = {}


def unpack_words(words: np.ndarray, n: int) -> np.ndarray:
    w = np.asarray(words, dtype=np.uint32).astype(np.uint64)
    bits = (w[:, None] >> np.arange(32, dtype=np.uint64)) & np.uint64(1)
    return np.where(bits.reshape(-1)[:n] == 1, 1, -1).astype(np.int8)


def plan(n: Sequence[int], nnz: Sequence[int], blocks: int, split: float = 1.0, barrier_cost: float = 0.05,
         cost: Optional[Sequence[float]] = None):
    """Host-side plan of problems onto contiguous teams of CTAs (no GPU needed); `cost`: measured
    CTA-time per problem (else the size model). Returns (team_of[P], team_b0[T], team_nb[T])."""
    lib = _lib.load()
    P = len(n)
    na = np.ascontiguousarray(n, dtype=np.int64)
    za = np.ascontiguousarray(nnz, dtype=np.int64)
    ca = None if cost is None else np.ascontiguousarray(cost, dtype=np.float64)
    team_of = np.zeros(P, dtype=np.int32)
    b0 = np.zeros(max(1, blocks), dtype=np.int32)
    nb = np.zeros(max(1, blocks), dtype=np.int32)
    nt = C.c_int32(0)
    I64 = C.POINTER(C.c_int64)
    I32 = C.POINTER(C.c_int32)
    cptr = None if ca is None else ca.ctypes.data_as(C.POINTER(C.c_double))
    check("sa_batch_plan", lib.sa_batch_plan(P, na.ctypes.data_as(I64), za.ctypes.data_as(I64), cptr, int(blocks),
                                             float(split), float(barrier_cost), team_of.ctypes.data_as(I32),
                                             b0.ctypes.data_as(I32), nb.ctypes.data_as(I32), C.byref(nt)))
    return team_of, b0[:nt.value].copy(), nb[:nt.value].copy()


class BatchedSpectralAnnealing:
    """SpecAnn over a list of instances x seeds in one launch. Parameters as SpectralAnnealing
    (precision, pred_mode, pred_tol, shift_eps, schedule, num_alphas, schedule_interval, eigsh_tol,
    eigsh_maxiter, eigsh_ncv, use_local_search, max_local_iterations, disable_warm_start), plus
    `seeds` (per instance), `split` (None: the default plan, or the autotuned one when autotune
    ran), `use_graph` and `ls_semantics`."""

    def __init__(self, seeds: Sequence[int] = (42,), precision: int = 32, pred_mode: str = "diagonal",
                 pred_tol: float = 1e-3, shift_eps: float = 1e-3, schedule: str = "sqrt", num_alphas: int = 128,
                 schedule_interval=(0.0, 1.0), eigsh_tol: float = 1e-6, eigsh_maxiter: int = 1000,
                 eigsh_ncv: Optional[int] = None, use_local_search: bool = True, max_local_iterations: int = 1000,
                 disable_warm_start: bool = False, ls_semantics: str = "priority", split: Optional[float] = None,
                 barrier_cost: float = 0.05, use_graph: bool = True, residual_check: bool = True):
        if pred_mode not in PRED_MODES:
            raise ValueError(f"pred_mode must be one of {PRED_MODES}, got {pred_mode!r}")
        if schedule not in SCHEDULES:
            raise ValueError(f"schedule must be one of {SCHEDULES}, got {schedule!r}")
        if precision not in (32, 64):
            raise ValueError(f"precision must be 32 or 64, got {precision}")
        t_min, t_max = (float(v) for v in schedule_interval)
        if int(num_alphas) < 2 or int(num_alphas) > 128 or not 0.0 <= t_min < t_max:
            raise ValueError(f"need 2 <= num_alphas <= 128 and 0 <= start < end, got {num_alphas}, {schedule_interval}")
        if ls_semantics not in ("priority", "snapshot"):
            raise ValueError(f"ls_semantics must be 'priority' or 'snapshot', got {ls_semantics!r}")
        self.seeds = [int(s) & (2 ** 64 - 1) for s in seeds]
        self.precision = int(precision)
        self.pred_mode = pred_mode
        self.pred_tol = float(pred_tol)
        self.shift_eps = float(shift_eps)
        self.schedule = schedule
        self.num_alphas = int(num_alphas)
        self.schedule_interval = (t_min, t_max)
        self.eigsh_tol = float(eigsh_tol)
        self.eigsh_maxiter = int(eigsh_maxiter)
        self.eigsh_ncv = eigsh_ncv
        self.use_local_search = bool(use_local_search)
        self.max_local_iterations = int(max_local_iterations)
        self.disable_warm_start = bool(disable_warm_start)
        self.ls_semantics = ls_semantics
        self.split = split
        self.barrier_cost = float(barrier_cost)
        self.use_graph = bool(use_graph)
        self.residual_check = bool(residual_check)
        self.lib = _lib.load()
        self._batch = None
        self._ws = None
        self._costs = None          # measured CTA-time per problem (autotune), else the size model
        self.engines: List[Engine] = []
        self.Js: List[sp.csr_matrix] = []
        self.last_ms = None

    # ---- set-up ------------------------------------------------------------------------------
    def alphas(self, num_alphas: Optional[int] = None) -> np.ndarray:
        k = self.num_alphas if num_alphas is None else int(num_alphas)
        t = np.linspace(*self.schedule_interval, k)
        return np.sqrt(t) if self.schedule == "sqrt" else t

    def load(self, instances: Sequence) -> "BatchedSpectralAnnealing":
        """Upload the instances (SciPy CSR, symmetric, zero diagonal) and run their preludes."""
        self.close()
        self.Js = [as_csr(J) for J in instances]
        for J in self.Js:
            if J.nnz >= 2 ** 31:
                raise ValueError("batched instances need fewer than 2^31 stored entries")
            eng = Engine(J.shape[0], J.nnz, precision=self.precision, ncv_max=2, max_candidates=1)
            data = J.data.astype(np.float32 if self.precision == 32 else np.float64, copy=False)
            eng.upload_csr(J.indptr, J.indices, data)
            self.engines.append(eng)
        return self

    @property
    def n_problems(self) -> int:
        return len(self.Js) * len(self.seeds)

    def grid(self) -> int:
        b = C.c_int32(0)
        check("sa_batch_grid", self.lib.sa_batch_grid(self.precision, 0, C.byref(b)))
        return int(b.value)

    def _sizes(self):
        S = len(self.seeds)
        n = [J.shape[0] for J in self.Js for _ in range(S)]
        z = [J.nnz for J in self.Js for _ in range(S)]
        return n, z

    def _key(self):
        return (self.precision, len(self.seeds)) + tuple((J.shape[0], J.nnz) for J in self.Js)

    def _build(self, split: float):
        """Plan, workspace and batch object for one split factor."""
        if self._batch is not None:
            self.lib.sa_batch_destroy(self._batch)
            self._batch = None
        blocks = self.grid()
        n, z = self._sizes()
        team_of, b0, nb = plan(n, z, blocks, split, self.barrier_cost, cost=self._costs)
        self.team_of, self.team_b0, self.team_nb = team_of, b0, nb
        I32 = C.POINTER(C.c_int32)
        handles = (C.c_void_p * len(self.engines))(*[e.h.value for e in self.engines])
        ncv_max = min(_lib.NCV_MAX, max(2, self.eigsh_ncv or 33))
        cap = 128
        nbytes = C.c_size_t(0)
        check("sa_batch_workspace_size", self.lib.sa_batch_workspace_size(
            len(self.engines), handles, len(self.seeds), ncv_max, cap, len(b0), b0.ctypes.data_as(I32),
            nb.ctypes.data_as(I32), team_of.ctypes.data_as(I32), C.byref(nbytes)))
        dev = self.engines[0].device
        self._ws = None
        torch.cuda.empty_cache()
        self._ws = torch.empty(int(nbytes.value) + 256, dtype=torch.uint8, device=dev)
        ptr = (self._ws.data_ptr() + 255) & ~255
        seeds = np.array([s for _ in self.Js for s in self.seeds], dtype=np.uint64)
        b = C.c_void_p()
        self._stream = torch.cuda.current_stream(dev)
        check("sa_batch_create", self.lib.sa_batch_create(
            C.byref(b), len(self.engines), handles, len(self.seeds), seeds.ctypes.data_as(C.POINTER(C.c_uint64)),
            ncv_max, cap, len(b0), b0.ctypes.data_as(I32), nb.ctypes.data_as(I32), team_of.ctypes.data_as(I32),
            C.c_void_p(ptr), int(nbytes.value), C.c_void_p(self._stream.cuda_stream)))
        self._batch = b
        self._built_split = split
        self.workspace_bytes = int(nbytes.value)

    def config(self, num_alphas: Optional[int] = None) -> BatchConfig:
        return BatchConfig(
            eigsh_tol=self.eigsh_tol, pred_tol=self.pred_tol, shift_eps=self.shift_eps, secant_gamma=1.0,
            subset_fraction=0.9, final_sweep_fraction=1.0,
            num_alphas=self.num_alphas if num_alphas is None else int(num_alphas), maxiter=self.eigsh_maxiter,
            ncv=int(self.eigsh_ncv or 0), pred_mode=_PRED[self.pred_mode],
            warm_start=0 if self.disable_warm_start else 1, residual_check=int(self.residual_check),
            use_local_search=int(self.use_local_search), max_local_iterations=self.max_local_iterations,
            final_sweep_iters=25, num_rounds=25, ls_semantics=0 if self.ls_semantics == "priority" else 1,
            reserved=0)

    # ---- runs ----------------------------------------------------------------------------------
    def sweep(self, num_alphas: Optional[int] = None, use_graph: Optional[bool] = None) -> float:
        """One batched launch over every problem; returns its device time in ms (CUDA events on
        the batch's stream)."""
        if self._batch is None:
            self._build(self._choose_split())
        cfg = self.config(num_alphas)
        al = np.ascontiguousarray(self.alphas(cfg.num_alphas), dtype=np.float64)
        g = self.use_graph if use_graph is None else bool(use_graph)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(self._stream)
        check("sa_batch_sweep", self.lib.sa_batch_sweep(self._batch, C.byref(cfg),
                                                        al.ctypes.data_as(C.POINTER(C.c_double)), int(g)))
        e1.record(self._stream)
        e1.synchronize()
        self.last_ms = e0.elapsed_time(e1)
        self._last_num_alphas = cfg.num_alphas
        return self.last_ms

    def _choose_split(self) -> float:
        if self.split is not None:
            return float(self.split)
        tuned = _TUNED.get(self._key())
        if tuned is not None:
            self._costs = tuned[1]
            return tuned[0]
        return 1.0

    def summaries(self) -> List[BatchSummary]:
        """Per-problem summaries of the last launch (no candidate copies)."""
        sums = (BatchSummary * self.n_problems)()
        check("sa_batch_results", self.lib.sa_batch_results(self._batch, None, sums))
        return list(sums)

    def autotune(self, splits=(1.0, 2.0, 4.0), num_alphas: int = 8, repeats: int = 1) -> Dict[float, float]:
        """Measure, then choose. A short schedule runs once with the size-model plan; each problem's
        device time x its team's CTAs becomes its measured cost. Plans built from those costs with
        each split are then timed on the same short schedule, and the fastest is kept for this
        workload shape. Returns {split: ms}."""
        self._costs = None
        self._build(1.0)
        self.sweep(num_alphas, use_graph=False)
        self._costs = [max(1e-3, z.device_ms) * max(1, z.team_blocks) for z in self.summaries()]
        times = {}
        seen = {}
        for s in splits:
            self._build(float(s))
            sig = (tuple(self.team_of), tuple(self.team_b0), tuple(self.team_nb))
            if sig in seen:                      # the same plan as an earlier split
                times[float(s)] = times[seen[sig]]
                continue
            self.sweep(num_alphas, use_graph=False)
            t = min(self.sweep(num_alphas, use_graph=False) for _ in range(max(1, repeats)))
            times[float(s)] = t
            seen[sig] = float(s)
        best = min(times, key=times.get)
        _TUNED[self._key()] = (best, list(self._costs))
        self._build(best)
        self.tuned = times
        return times

    def results(self) -> List[dict]:
        """Per problem: best energy / spins (selection of models/spectral_annealing.py:446-520, the
        FP64 energy of the returned spins from the input J), per-alpha rows and counters."""
        P = self.n_problems
        recs = (BatchAlphaRecord * (P * 128))()
        sums = (BatchSummary * P)()
        check("sa_batch_results", self.lib.sa_batch_results(self._batch, recs, sums))
        S = len(self.seeds)
        out = []
        dev = self.engines[0].device
        for p in range(P):
            inst, seed = p // S, self.seeds[p % S]
            J = self.Js[inst]
            n = J.shape[0]
            z = sums[p]
            k = int(z.num_candidates)
            rows = []
            for a in range(self._last_num_alphas):
                r = recs[p * 128 + a]
                rows.append({"alpha": r.alpha, "lambda1": r.lambda1, "rho": r.rho, "gershgorin": r.gershgorin,
                             "eigsh_residual": r.residual, "pred_residual": r.pred_residual,
                             "pred_accepted": None if r.pred_accepted < 0 else bool(r.pred_accepted),
                             "degree_scale": r.degree_scale, "eigsh_iterations": int(r.iterations),
                             "eigsh_restarts": int(r.restarts), "eigsh_spmvs": int(r.spmv_count),
                             "eigsh_retry": bool(r.retry), "eigsh_converged": bool(r.converged),
                             "status": int(r.status), "candidate": int(r.candidate), "signature": int(r.signature)})
            res = {"instance": inst, "seed": seed, "n": n, "status": int(z.status), "num_candidates": k,
                   "ls_iterations": int(z.ls_iterations), "ls_final_passes": int(z.ls_final_passes),
                   "alphas_skipped": int(z.alphas_skipped), "alphas_retried": int(z.alphas_retried),
                   "team": (int(z.team_first_block), int(z.team_blocks)), "device_ms": float(z.device_ms),
                   "phase_ms": [float(x) for x in z.phase_ms], "ls_ms": float(z.ls_ms),
                   "rows": rows, "energy_before": np.array(z.energy_before[:k]),
                   "energy_after": np.array(z.energy_after[:k])}
            best, src = float("inf"), None
            eb, ea = res["energy_before"], res["energy_after"]
            for r in rows:
                c = r["candidate"]
                if c < 0:
                    continue
                raw = float(eb[c])
                r["raw_energy"] = raw
                r["energy"] = raw
                if raw < best:
                    best, src = raw, (False, c)
            if self.use_local_search:
                for r in rows:
                    c = r["candidate"]
                    if c < 0:
                        continue
                    refined = not (ea[c] > eb[c])
                    e = float(ea[c] if refined else eb[c])
                    r["energy"] = e
                    if e < best:
                        best, src = e, (refined, c)
            if src is None:
                res.update(energy=None, spins=None, best_alpha=None)
            else:
                words = torch.empty((n + 31) // 32, dtype=torch.int32, device=dev)
                check("sa_batch_candidate", self.lib.sa_batch_candidate(self._batch, p, src[1], int(src[0]),
                                                                        C.c_void_p(words.data_ptr())))
                spins = unpack_words(words.cpu().numpy().view(np.uint32), n)
                s64 = spins.astype(np.float64)
                res.update(spins=spins, device_energy=best, energy=float(-0.5 * s64 @ (J @ s64)),
                           best_source=("refined" if src[0] else "original", src[1]))
            out.append(res)
        return out

    def solve(self, instances: Optional[Sequence] = None) -> List[Tuple[float, np.ndarray, float]]:
        """(best energy, best spins, seconds) per (instance, seed), instance-major: the return of
        SpectralAnnealing.solve for each problem; the seconds are the batch's wall time."""
        t0 = time.time()
        if instances is not None:
            self.load(instances)
        self.sweep()
        self.last_results = self.results()
        dt = time.time() - t0
        out = []
        for r in self.last_results:
            if r["energy"] is None:
                raise NumericalFailure(f"instance {r['instance']} seed {r['seed']}: no alpha produced a solution")
            out.append((r["energy"], r["spins"], dt))
        return out

    def close(self):
        if getattr(self, "_batch", None) is not None:
            self.lib.sa_batch_destroy(self._batch)
            self._batch = None
        self._ws = None
        for e in getattr(self, "engines", []):
            e.close()
        self.engines = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
