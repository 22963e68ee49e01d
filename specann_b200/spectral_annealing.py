"""SpectralAnnealing: drop-in replacement of the reference solver class
(models/spectral_annealing.py:132-525) running the alpha sweep on the B200 engine.

Same constructor signature, defaults and validation errors; same solve(J) contract (returns
(best energy, best spins, seconds)) and the same result CSVs. What runs where:
  * per alpha, one cooperative kernel launch (sa_alpha_solve): predictor and its residual test,
    warm-started thick-restart Lanczos on S_rho, checks, alignment, true residual, rounding and
    the candidate signature; the host keeps the reference's control flow (shift, schedule, cold
    retry, skipped alphas, deduplication bookkeeping);
  * after the sweep, one cooperative launch for the batched local search over all distinct
    candidates, which also yields every candidate's energy before and after (exact integers for
    integer couplings).
"""
from __future__ import annotations

import os
import time
from datetime import datetime
from typing import List, Optional

import numpy as np
import scipy.sparse as sp
import torch

from . import _lib
from .failures import EigensolverBreakdown, NumericalFailure, is_numerical, is_out_of_memory
from . import results as _results

# "tangent" (first-order step along dy/dalpha from the eigenvector adjoint) has no reference
# counterpart; the other three are utils/predictors.py and models/spectral_annealing.py:589-612
PRED_MODES = ("diagonal", "secant", "prev", "tangent")
LS_POLICIES = ("default", "fixed_guard", "adaptive_guard", "independent_set", "sequential_oracle")
SCHEDULES = ("sqrt", "linear")


def compute_shift_rho(lambda1_prev, gershgorin_bound, eps=1e-3):
    """rho = (1 + eps) max(lambda1_prev, g) (models/spectral_annealing.py:56-67)."""
    if lambda1_prev is None or not np.isfinite(lambda1_prev) or lambda1_prev <= 0:
        base = gershgorin_bound
    else:
        base = max(lambda1_prev, gershgorin_bound)
    rho = (1.0 + eps) * base
    if rho <= 0:
        rho = (1.0 + eps) * max(gershgorin_bound, 1.0)
    return rho


def gershgorin_bound(d_min: float, d_max: float, alpha: float) -> float:
    """g = max_i d_i^(1 - alpha) (models/spectral_annealing.py:579) from the extremes of d in (0, 1]."""
    e = 1.0 - float(alpha)
    vals = []
    for d in (d_min, d_max):
        if d > 0:
            vals.append(d ** e)
        else:
            vals.append(0.0 if e > 0 else (1.0 if e == 0 else float("inf")))
    return float(max(vals))


def default_ncv(n: int, ncv: Optional[int]) -> int:
    """CuPy's default basis min(max(2k, k + 32), n - 1) for k = 1, at least 2."""
    if ncv is None:
        ncv = min(33, n - 1)
    return int(max(2, min(int(ncv), max(2, n))))


def as_csr(J) -> sp.csr_matrix:
    if sp.issparse(J):
        return J.tocsr()
    return sp.csr_matrix(np.asarray(J))


def _seed_value(random_seed) -> int:
    if random_seed is None:
        return int.from_bytes(os.urandom(8), "little")
    return int(random_seed)


class _Candidates:
    """Distinct rounded candidates of a sweep (the reference's dict keyed by packed spins,
    models/spectral_annealing.py:362-370): signature -> slots of the device store, with an exact
    comparison on a signature match."""

    def __init__(self, engine, capacity: int):
        self.engine = engine
        self.capacity = capacity
        self.by_sig = {}
        self.count = 0

    def add_scratch(self, signature: int) -> int:
        for slot in self.by_sig.get(signature, []):
            if self.engine.candidate_equal(slot):
                return slot
        if self.count >= self.capacity:
            raise NumericalFailure(f"more than {self.capacity} distinct candidates in one sweep")
        slot = self.count
        self.engine.keep_candidate(slot)
        self.by_sig.setdefault(signature, []).append(slot)
        self.count += 1
        return slot


class SpectralAnnealing:
    """SpecAnn solver (B200 engine). Parameters as models/spectral_annealing.py:140-170."""

    def __init__(self, instance_name: str, dataset: str, random_seed: int = None,
                 mode: int = 0, beta: float = None, alpha: float = None,
                 use_local_search: bool = True, max_local_iterations: int = 1000,
                 eigsh_tol: float = 1e-6, eigsh_maxiter: int = 1000, run_name: str = None,
                 disable_warm_start: bool = False, precision: int = 32,
                 pred_mode: str = "diagonal", pred_tol: float = 1e-3, shift_eps: float = 1e-3,
                 schedule: str = "sqrt", num_alphas: int = 128, schedule_interval=(0.0, 1.0),
                 eigsh_ncv: int = None, fp32_spmv: bool = None, ls_policy: str = "default",
                 ls_batch: bool = True, **kwargs):
        self.instance_name = instance_name
        self.dataset = dataset
        self.random_seed = random_seed
        self.mode = mode
        self.beta = beta
        self.alpha = alpha
        self.use_local_search = use_local_search
        self.max_local_iterations = max_local_iterations
        self.eigsh_tol = float(eigsh_tol)
        self.eigsh_maxiter = int(eigsh_maxiter)
        self.eigsh_ncv = None if eigsh_ncv is None else int(eigsh_ncv)
        self.disable_warm_start = disable_warm_start
        if pred_mode not in PRED_MODES:
            raise ValueError(f"pred_mode must be one of {PRED_MODES}, got {pred_mode!r}")
        self.pred_mode = pred_mode
        self.pred_tol = float(pred_tol)
        self.shift_eps = float(shift_eps)
        t_min, t_max = (float(v) for v in schedule_interval)
        if schedule not in SCHEDULES:
            raise ValueError(f"schedule must be one of {SCHEDULES}, got {schedule!r}")
        if int(num_alphas) < 2 or not 0.0 <= t_min < t_max:
            raise ValueError(f"need num_alphas >= 2 and 0 <= start < end, got {num_alphas}, {schedule_interval}")
        self.schedule = schedule
        self.num_alphas = int(num_alphas)
        self.schedule_interval = (t_min, t_max)
        if precision == 32:
            self.dtype = np.float32
        elif precision == 64:
            self.dtype = np.float64
        else:
            raise ValueError(f"precision must be 32 or 64, got {precision}")
        self.precision = precision
        self.fp32_spmv = (precision == 32) if fp32_spmv is None else bool(fp32_spmv)
        if ls_policy not in LS_POLICIES:
            raise ValueError(f"ls_policy must be one of {LS_POLICIES}, got {ls_policy!r}")
        self.ls_policy = ls_policy
        self.ls_batch = bool(ls_batch)
        if not self.ls_batch and ls_policy != "default":
            raise ValueError("ls_batch = False is only defined for ls_policy 'default'")
        if self.fp32_spmv and precision != 32:
            raise ValueError("fp32_spmv needs precision 32")
        self.solver_name = run_name if run_name else "spectral_annealing_pred"
        self.residual_check = bool(kwargs.pop("residual_check", True))
        self.verbose = bool(kwargs.pop("verbose", False))
        # write_results=False skips the result CSVs (the reference writes them after its timer)
        self.write_results = bool(kwargs.pop("write_results", True))
        self.profile = bool(kwargs.pop("profile", False))
        # MINRES tolerance of the tangent predictor's direction (pred_mode "tangent")
        self.tangent_tol = float(kwargs.pop("tangent_tol", 1e-2))
        # Ritz vectors kept by an implicit restart of the Lanczos basis (0: the kernel's default, 8)
        self.restart_keep = int(kwargs.pop("restart_keep", 0))
        # operator layout: "auto" (column panels when rows average >= 16 entries and the row
        # blocks fit the SMs; L2 column splits when the gathered vector is larger than 48 MB; else
        # the work list), "panel", "split" or "worklist"
        self.spmv = str(kwargs.pop("spmv", "auto"))
        if self.spmv not in ("auto", "panel", "split", "worklist"):
            raise ValueError(f"spmv must be 'auto', 'panel', 'split' or 'worklist', got {self.spmv!r}")
        # local-search pass semantics: "priority" (independent flips, monotone) or "snapshot"
        self.ls_semantics = str(kwargs.pop("ls_semantics", "priority"))
        # 64-bit row pointers for solve(J) (None: only when nnz does not fit in int32); solve_device
        # follows the dtype of the row-pointer tensor it is given
        rp64 = kwargs.pop("rowptr64", None)
        self.rowptr64 = None if rp64 is None else bool(rp64)
        # alpha indices whose eigenvector (device copy), shift and Ritz value are kept after the
        # solve in self.kept_vectors[idx] = (y, rho, mu) (checks against an FP64 eigensolver)
        self.keep_vectors = frozenset(int(i) for i in kwargs.pop("keep_vectors", ()))
        self.kept_vectors = {}
        if self.ls_semantics not in ("priority", "snapshot"):
            raise ValueError(f"ls_semantics must be 'priority' or 'snapshot', got {self.ls_semantics!r}")
        self._extra_kwargs = kwargs
        self.engine = None
        if self.verbose:
            print(f"Initialized {self.solver_name} solver (B200 engine): precision {precision}, "
                  f"fp32_spmv {self.fp32_spmv}, schedule {schedule} x {num_alphas}, pred_mode {pred_mode}")

    # -- schedule ---------------------------------------------------------------------------------
    def _get_alpha_values(self, mode: int) -> list:
        """models/spectral_annealing.py:549-555."""
        if mode == 0:
            t = np.linspace(*self.schedule_interval, self.num_alphas)
            return [float(x) for x in (np.sqrt(t) if self.schedule == "sqrt" else t)]
        raise ValueError(f"Unknown mode {mode}")

    # -- one alpha ---------------------------------------------------------------------------------
    def _attempt(self, eng, alpha, alpha_prev, rho, g, start_mode, stream_id, ncv):
        v0 = self._tangent if start_mode == _lib.SA_START_TANGENT else None
        rec = eng.alpha_solve(alpha=alpha, alpha_prev=alpha if alpha_prev is None else alpha_prev, rho=rho,
                              gershgorin=g, tol=self.eigsh_tol, pred_tol=self.pred_tol,
                              maxiter=self.eigsh_maxiter, ncv=ncv, start_mode=start_mode, seed=self._seed,
                              stream_id=stream_id, align=True, residual_check=self.residual_check, v0=v0,
                              restart_keep=self.restart_keep)
        if rec.status in (_lib.SA_ERR_BREAKDOWN, _lib.SA_ERR_NONFINITE) or rec.nonfinite:
            raise EigensolverBreakdown(f"Lanczos failed: {_lib.STATUS_NAMES.get(rec.status, rec.status)}")
        if rec.status not in (_lib.SA_OK, _lib.SA_ERR_NOT_CONVERGED):
            raise RuntimeError(f"alpha kernel failed: {_lib.STATUS_NAMES.get(rec.status, rec.status)}")
        nu = rec.mu
        if not np.isfinite(nu):
            raise EigensolverBreakdown(f"non-finite eigenvalue {nu}")
        lambda1 = rho - nu
        if lambda1 > g * (1.0 + max(0.5 * self.shift_eps, 1e-5)):
            raise EigensolverBreakdown(f"spurious eigenvalue {lambda1:.6g} above the Gershgorin bound {g:.6g}")
        return rec

    def _solve_alpha(self, eng, alpha_idx, alpha, alpha_prev, lambda1_prev, info, ncv, warm):
        g = gershgorin_bound(info.d_min, info.d_max, alpha)
        rho = compute_shift_rho(lambda1_prev, g, eps=self.shift_eps)
        if alpha_idx == 0 or self.disable_warm_start or not warm:
            mode = _lib.SA_START_RANDOM
        elif self.pred_mode == "prev":
            mode = _lib.SA_START_PREV
        elif self.pred_mode == "diagonal":
            mode = _lib.SA_START_DIAGONAL
        elif self.pred_mode == "tangent":
            mode = _lib.SA_START_TANGENT if self._tangent is not None else _lib.SA_START_PREV
        else:
            mode = _lib.SA_START_SECANT
        retry = False
        try:
            rec = self._attempt(eng, alpha, alpha_prev, rho, g, mode, 4 * alpha_idx, ncv)
            first = rec
        except EigensolverBreakdown as e:
            if self.verbose:
                print(f"Warning: eigensolver failed for alpha={alpha}, rho={rho}: {e}")
            retry = True
            first = None
            rec = self._attempt(eng, alpha, alpha_prev, rho, g, _lib.SA_START_RANDOM, 4 * alpha_idx + 1, ncv)
        pred_rec = first if first is not None else rec
        converged = rec.status == _lib.SA_OK or (np.isfinite(rec.residual) and rec.residual <= self.eigsh_tol)
        return rec, rho, g, retry, converged, pred_rec

    # -- solve --------------------------------------------------------------------------------------
    def solve(self, J):
        """Run SpecAnn on J (SciPy CSR or dense, symmetric, zero diagonal); write the CSVs.
        Returns (best energy, best spins as a NumPy array of +-1 in the solver dtype, seconds)."""
        start_time = time.time()
        self._check_runnable()
        Jc = as_csr(J)
        n = Jc.shape[0]
        self._host_csr = (Jc.indptr, Jc.indices)
        eng = self._make_engine(n, Jc.nnz, self.rowptr64)
        data = Jc.data.astype(np.float32, copy=False) if (self.precision == 32) else Jc.data
        info = eng.upload_csr(Jc.indptr, Jc.indices, data)
        self._choose_operator(eng)
        return self._sweep(eng, info, Jc, start_time)

    def solve_device(self, rowptr, col, val):
        """The same solve on a CSR already in device memory (torch CUDA tensors: row pointers int32
        or int64, columns int32, couplings float32 at precision 32 / float64 at 64). The reported
        energy is the device energy of the best spins (exact for integer couplings)."""
        start_time = time.time()
        self._check_runnable()
        n = int(rowptr.numel()) - 1
        self._host_csr = None
        eng = self._make_engine(n, int(col.numel()), rowptr.dtype == torch.int64)
        info = eng.bind(rowptr, col, val)
        self._choose_operator(eng)
        return self._sweep(eng, info, None, start_time)

    def _choose_operator(self, eng):
        """Lay the operator out as column panels (spmv 'panel', or 'auto' when they pay) or keep
        the CSR work list."""
        self.operator_layout = "worklist"
        if self.spmv == "panel" or (self.spmv == "auto" and eng.panels_pay()):
            eng.build_panels()
            self.operator_layout = "panel"
        elif self.spmv == "split" or (self.spmv == "auto" and eng.splits_pay()):
            eng.build_splits()
            self.operator_layout = "split"

    def _check_runnable(self):
        if self.alpha is not None:
            raise ValueError("Alpha is not set")

    def _make_engine(self, n, nnz, rowptr64=None):
        from .engine import Engine
        self._seed = _seed_value(self.random_seed)
        eng_prec = 32 if self.fp32_spmv else 64
        self._capacity = min(128, self.num_alphas)
        self._ncv = default_ncv(n, self.eigsh_ncv)
        eng = Engine(n, nnz, precision=eng_prec, ncv_max=max(self._ncv, 2), max_candidates=self._capacity,
                     rowptr64=rowptr64)
        eng.profile = self.profile
        self.engine = eng
        return eng

    def _sweep(self, eng, info, Jc, start_time):
        n = eng.n
        ncv = self._ncv
        capacity = self._capacity
        self._normalization_factor = info.c
        alpha_list = self._get_alpha_values(self.mode)
        cands = _Candidates(eng, capacity)
        alpha_results: List[dict] = []
        row_cand: List[int] = []
        lambda1_prev = alpha_prev = None
        warm = False
        self._alphas_skipped = 0
        self._alphas_retried = 0
        self._alpha_errors = 0
        self._last_alpha_error = None
        self._tangent = None
        self.kept_vectors = {}
        for alpha_idx, alpha in enumerate(alpha_list):
            t_alpha = time.time()
            try:
                rec, rho, g, retry, converged, pred_rec = self._solve_alpha(
                    eng, alpha_idx, alpha, alpha_prev, lambda1_prev, info, ncv, warm)
            except Exception as e:
                if is_out_of_memory(e):
                    raise
                if self.verbose:
                    print(f"Alpha {alpha} failed: {e}")
                self._alphas_skipped += 1
                if not is_numerical(e):
                    self._alpha_errors += 1
                    self._last_alpha_error = e
                continue
            self._alphas_retried += int(retry)
            lambda1 = rho - rec.mu
            bound = (-0.5 * lambda1 * rec.degree_scale * info.c) if converged else float("nan")
            slot = cands.add_scratch(rec.signature)
            if alpha_idx in self.keep_vectors:
                self.kept_vectors[alpha_idx] = (eng.result_vector(), rho, rec.mu)
            tangent_spmvs = 0
            if self.pred_mode == "tangent" and not self.disable_warm_start:
                # dy/dalpha at this eigenpair (the next alpha's start is y + dalpha t)
                y_now = eng.result_vector()
                t = torch.empty_like(y_now)
                tres = eng.adjoint(_lib.SA_ADJ_TANGENT, alpha=alpha, lambda1=lambda1, y=y_now,
                                   tol=self.tangent_tol, maxiter=self.eigsh_maxiter, out=t)
                self._tangent = t
                tangent_spmvs = int(tres.spmv_count)
            if not self.disable_warm_start:
                eng.commit()
                warm = True
                lambda1_prev = lambda1
                alpha_prev = alpha
            pred_acc = None if pred_rec.pred_accepted < 0 else bool(pred_rec.pred_accepted)
            alpha_results.append({
                'instance_name': self.instance_name, 'dataset': self.dataset, 'seed': self.random_seed,
                'solver_name': self.solver_name, 'alpha': alpha, 'beta': None, 'energy': None,
                'raw_energy': None, 'time': time.time() - t_alpha, 'mode': self.mode,
                'use_local_search': self.use_local_search, 'local_search_iterations': 0,
                'eigsh_iterations': int(rec.iterations), 'eigsh_retry': retry, 'eigsh_converged': converged,
                'warm_start': not self.disable_warm_start, 'alpha_index': alpha_idx,
                'precision': self.precision, 'fp32_spmv': self.fp32_spmv, 'lambda1': lambda1,
                'degree_scale': rec.degree_scale, 'energy_bound': bound, 'pred_mode': self.pred_mode,
                'pred_residual': pred_rec.pred_residual, 'pred_accepted': pred_acc,
                'candidate': slot if self.use_local_search else None,
                'eigsh_residual': rec.residual, 'eigsh_restarts': int(rec.restarts),
                'eigsh_spmvs': int(rec.spmv_count), 'alg_bytes': float(rec.alg_bytes),
                'tangent_spmvs': tangent_spmvs,
                'timestamp': datetime.now().strftime('%Y-%m-%d %H:%M:%S')})
            row_cand.append(slot)
        sweep_end = time.time()
        k = cands.count
        self._num_candidates = k if self.use_local_search else None
        best_energy, best_src, best_alpha, best_iters = float("inf"), None, None, 0
        local_iterations = 0
        if k > 0:
            if self.use_local_search:
                raw, refined, local_iterations = self._refine(eng, k)
            else:
                raw, refined = eng.energies(k), None
            for i, res in enumerate(alpha_results):
                e = float(raw[row_cand[i]])
                res['raw_energy'] = e
                res['energy'] = e
                if e < best_energy:
                    best_energy, best_src, best_alpha = e, ('original', row_cand[i]), res['alpha']
            if refined is not None:
                for i, res in enumerate(alpha_results):
                    c = row_cand[i]
                    kind = 'original' if refined[c] > raw[c] else 'refined'
                    e = float(raw[c] if kind == 'original' else refined[c])
                    res['energy'] = e
                    res['local_search_iterations'] = local_iterations
                    if e < best_energy:
                        best_energy, best_src, best_alpha = e, (kind, c), res['alpha']
                        best_iters = local_iterations
        best_spins = None
        if best_src is not None:
            kind, c = best_src
            best_spins = eng.candidate_spins(c, refined=(kind == 'refined')).cpu().numpy().astype(self.dtype)
        total_time = time.time() - start_time
        if best_spins is not None and Jc is not None and not (info.integer and abs(best_energy) < 2.0 ** 52):
            # the reported energy is -1/2 s^T J s in FP64 from the input J (models/spectral_annealing.py:
            # 484-488); for integer couplings the device energy is already that number exactly (int64
            # sums of int32 fields), so the host product is only needed for non-integer J
            s64 = best_spins.astype(np.float64)
            best_energy = float(-0.5 * s64 @ (Jc @ s64))
        self._sweep_time = sweep_end - start_time
        self._post_sweep_time = total_time - self._sweep_time
        self._gpu_pool_bytes = int(torch.cuda.memory_reserved())
        if best_alpha is None:
            if self.write_results:
                self._store_timing_results(alpha_results)
            message = f"no alpha produced a solution ({self._alphas_skipped} of {len(alpha_list)} skipped)"
            if self._alpha_errors:
                last = self._last_alpha_error
                raise RuntimeError(f"{message}; {self._alpha_errors} of them raised a non-numerical error, "
                                   f"the last {type(last).__name__}: {last}") from last
            raise NumericalFailure(message)
        self.alpha_results = alpha_results
        if self.write_results:
            self._store_general_results(best_energy, best_alpha, None, total_time, best_iters)
            self._store_timing_results(alpha_results)
        return best_energy, best_spins, total_time

    def _refine(self, eng, k):
        """Local search of the distinct candidates: (energies before, energies after, passes)."""
        if self.ls_policy != "default":
            # guarded policies (models/spectral_annealing.py:540-547 -> local_search_guards.run_policy)
            from .guards import run_policy
            indptr = indices = None
            if self.ls_policy == "independent_set":
                indptr, indices = self._host_structure(eng)
            eb, ea, iters, res = run_policy(eng, self.ls_policy, k, max_iterations=self.max_local_iterations,
                                            seed=self._seed, indptr=indptr, indices=indices)
            self._ls_passes = iters + int(res.final_rounds)
            self._last_ls_summary = {"rounds": int(res.rounds), "final_rounds": int(res.final_rounds),
                                     "accepted_updates": int(res.accepted), "rejected_updates": int(res.rejected),
                                     "status": int(res.status)}
            return eb, ea, iters
        if self.ls_batch:
            eb, ea, res = eng.local_search(k, max_iterations=self.max_local_iterations, seed=self._seed,
                                           semantics=self.ls_semantics)
            self._ls_passes = int(res.iterations) + int(res.final_passes)
            return eb, ea, int(res.iterations)
        eb = np.empty(k)
        ea = np.empty(k)
        used = 0
        for c in range(k):
            b, a, res = eng.local_search(1, first_slot=c, max_iterations=self.max_local_iterations, seed=self._seed,
                                         semantics=self.ls_semantics)
            eb[c], ea[c] = b[0], a[0]
            used = max(used, int(res.iterations))
        return eb, ea, used

    def _host_structure(self, eng):
        """Host row pointers and columns of the bound matrix (the independent set's colouring)."""
        if getattr(self, "_host_csr", None) is not None:
            return self._host_csr
        return eng.d_rowptr.cpu().numpy(), eng.d_col.cpu().numpy()

    # -- CSVs -----------------------------------------------------------------------------------------
    def _store_general_results(self, energy, alpha, beta, time_taken, local_search_iterations=0):
        row = {
            'instance_name': self.instance_name, 'dataset': self.dataset, 'seed': self.random_seed,
            'solver_name': self.solver_name, 'energy': energy, 'time': time_taken,
            'local_search': self.use_local_search, 'local_search_iterations': local_search_iterations,
            'alpha': alpha, 'beta': beta, 'mode': self.mode, 'precision': self.precision,
            'fp32_spmv': self.fp32_spmv, 'ls_policy': self.ls_policy,
            'alphas_skipped': getattr(self, '_alphas_skipped', 0),
            'alphas_retried': getattr(self, '_alphas_retried', 0),
            'num_candidates': getattr(self, '_num_candidates', None),
            'sweep_time': getattr(self, '_sweep_time', None),
            'post_sweep_time': getattr(self, '_post_sweep_time', None),
            'gpu_pool_bytes': getattr(self, '_gpu_pool_bytes', None),
            'timestamp': datetime.now().strftime('%Y-%m-%d %H:%M:%S')}
        try:
            _results.store_general(self.dataset, self.solver_name, self.instance_name, row)
        except Exception as e:
            print(f"Error saving general results: {e}")

    def _store_timing_results(self, alpha_results):
        _results.store_alphas(self.dataset, self.solver_name, self.instance_name, self.random_seed, alpha_results)
