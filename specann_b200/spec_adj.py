"""Alpha0GPU (SpecAdj, the alpha = 0 end of the path) and Alpha1GPU (SpecSignedLap, alpha = 1) on the
B200 engine: drop-in replacements of models/spec_adj.py:21-154 and models/spec_signed_lap.py:21-170.

Both solve one eigenproblem with the same kernels as the sweep, without materialising S:
  SpecAdj:        S = I - J/c                          (models/spec_adj.py:155-160)  -> alpha 0, rho 1
  SpecSignedLap:  S = D^{-1/2} (D - J/c) D^{-1/2}        (models/spec_signed_lap.py:174-208)
                    = I - D^{-1/2} (J/c) D^{-1/2}       -> alpha 1, rho 1
(the reference clamps D at 1e-7 for SpecSignedLap and the fused operator at 1e-12; they agree
whenever every normalised degree d = deg/c is at least 1e-7, i.e. max/min degree ratio <= 1e7).
A cold start (two tries, models/spec_adj.py:351-363), the rounding s = sign(x >= 0) of
x = D^{-alpha/2} y, then the batched local search on the one candidate, kept only if it lowers the
energy (models/spec_adj.py:120-142).
"""
from __future__ import annotations

import time
from datetime import datetime

import numpy as np

from . import _lib
from . import results as _results
from .failures import NumericalFailure
from .spectral_annealing import LS_POLICIES, _seed_value, as_csr, default_ncv


class _FixedAlpha:
    _alpha_value = 0.0
    _default_name = "alpha0_gpu"
    _beta_value = 1.0

    def _init_common(self, instance_name, dataset, random_seed, mode, beta, use_local_search,
                     max_local_iterations, eigsh_tol, eigsh_maxiter, run_name, ls_policy, precision, kwargs):
        self.instance_name = instance_name
        if ls_policy not in LS_POLICIES:
            raise ValueError(f"ls_policy must be one of {LS_POLICIES}, got {ls_policy!r}")
        self.ls_policy = ls_policy
        self.dataset = dataset
        self.random_seed = random_seed
        self.mode = mode
        self.beta = beta
        self.use_local_search = use_local_search
        self.max_local_iterations = max_local_iterations
        self.eigsh_tol = float(eigsh_tol)
        self.eigsh_maxiter = int(eigsh_maxiter)
        if precision not in (32, 64):
            raise ValueError(f"precision must be 32 or 64, got {precision}")
        self.precision = int(precision)
        self.dtype = np.float32 if self.precision == 32 else np.float64
        self.solver_name = run_name if run_name else self._default_name
        self.verbose = bool(kwargs.pop("verbose", False))
        self.ls_semantics = str(kwargs.pop("ls_semantics", "priority"))
        self.engine = None

    def _solve_eigen(self, eng, n):
        """Two cold tries (models/spec_adj.py:351-363 _eigsh_finite); residual-checked convergence."""
        ncv = default_ncv(n, None)
        for attempt in (0, 1):
            rec = eng.alpha_solve(alpha=self._alpha_value, alpha_prev=self._alpha_value, rho=1.0, gershgorin=1.0,
                                  tol=self.eigsh_tol, pred_tol=0.0, maxiter=self.eigsh_maxiter, ncv=ncv,
                                  start_mode=_lib.SA_START_RANDOM, seed=self._seed, stream_id=attempt,
                                  align=False, residual_check=True)
            if rec.status in (_lib.SA_OK, _lib.SA_ERR_NOT_CONVERGED) and not rec.nonfinite and np.isfinite(rec.mu):
                self._eigsh_iterations = int(rec.iterations)
                self._eigsh_converged = rec.status == _lib.SA_OK or rec.residual <= self.eigsh_tol
                return rec
            if self.verbose:
                print(f"Warning: eigensolver returned a non-finite eigenpair (try {attempt + 1} of 2)")
        raise NumericalFailure("eigensolver returned a non-finite eigenpair twice")

    def solve(self, J):
        """Solve the instance with couplings J. Returns (energy, spins, time in seconds)."""
        from .engine import Engine
        start_time = time.time()
        Jc = as_csr(J)
        n = Jc.shape[0]
        self._seed = _seed_value(self.random_seed)
        data = Jc.data.astype(np.float32, copy=False) if self.precision == 32 else Jc.data
        eng = Engine(n, Jc.nnz, precision=self.precision, ncv_max=default_ncv(n, None), max_candidates=1)
        self.engine = eng
        info = eng.upload_csr(Jc.indptr, Jc.indices, data)
        self._normalization_factor = info.c
        self._prepare(info)
        self._solve_eigen(eng, n)
        eng.keep_candidate(0)
        local_iterations = 0
        use_refined = False
        if self.use_local_search:
            if self.ls_policy == "default":
                eb, ea, res = eng.local_search(1, max_iterations=self.max_local_iterations, seed=self._seed,
                                               semantics=self.ls_semantics)
                local_iterations = int(res.iterations)
            else:
                # models/spec_adj.py:130-133, models/spec_signed_lap.py (refine_candidates)
                from .guards import run_policy
                eb, ea, local_iterations, _ = run_policy(eng, self.ls_policy, 1,
                                                         max_iterations=self.max_local_iterations,
                                                         seed=self._seed, indptr=Jc.indptr, indices=Jc.indices)
            energy = float(eb[0])
            if ea[0] < eb[0]:
                energy = float(ea[0])
                use_refined = True
        else:
            energy = float(eng.energies(1)[0])
        spins = eng.candidate_spins(0, refined=use_refined).cpu().numpy().astype(self.dtype)
        total_time = time.time() - start_time
        s64 = spins.astype(np.float64)
        energy = float(-0.5 * s64 @ (Jc @ s64))
        self._store_general_results(energy, self._alpha_value, self._beta_value, total_time, local_iterations)
        return energy, spins, total_time

    def _prepare(self, info):
        pass

    def _store_general_results(self, energy, alpha, beta, time_taken, local_iterations):
        row = {'instance_name': self.instance_name, 'dataset': self.dataset, 'seed': self.random_seed,
               'solver_name': self.solver_name, 'energy': energy, 'time': time_taken,
               'local_search': self.use_local_search, 'local_search_iterations': local_iterations,
               'alpha': alpha, 'beta': beta, 'mode': self.mode, 'precision': self.precision,
               'eigsh_maxiter': self.eigsh_maxiter, 'eigsh_iterations': getattr(self, '_eigsh_iterations', None),
               'eigsh_converged': getattr(self, '_eigsh_converged', None),
               'timestamp': datetime.now().strftime('%Y-%m-%d %H:%M:%S')}
        _results.store_general(self.dataset, self.solver_name, self.instance_name, row)


class Alpha0GPU(_FixedAlpha):
    """SpecAdj solver (alpha = 0). Parameters as models/spec_adj.py:21-42."""
    _alpha_value = 0
    _default_name = "alpha0_gpu"
    _beta_value = 1.0

    def __init__(self, instance_name: str, dataset: str, random_seed: int = None,
                 mode: int = 0, beta: float = None, alpha: float = 0,
                 use_local_search: bool = True, max_local_iterations: int = 1000,
                 eigsh_tol: float = 1e-6, eigsh_maxiter: int = 1000, run_name: str = None,
                 ls_policy: str = "default", precision: int = 32, **kwargs):
        self._init_common(instance_name, dataset, random_seed, mode, beta, use_local_search,
                          max_local_iterations, eigsh_tol, eigsh_maxiter, run_name, ls_policy, precision, kwargs)
        self.alpha = 0


class Alpha1GPU(_FixedAlpha):
    """SpecSignedLap solver (alpha = 1). Parameters as models/spec_signed_lap.py:21-44."""
    _alpha_value = 1.0
    _default_name = "alpha1_gpu"
    _beta_value = 1.0

    def __init__(self, instance_name: str, dataset: str, random_seed: int = None,
                 mode: int = 0, beta: float = None,
                 use_local_search: bool = True, max_local_iterations: int = 1000,
                 eigsh_tol: float = 1e-6, eigsh_maxiter: int = 1000, run_name: str = None,
                 ls_policy: str = "default", precision: int = 32, **kwargs):
        self._init_common(instance_name, dataset, random_seed, mode, beta, use_local_search,
                          max_local_iterations, eigsh_tol, eigsh_maxiter, run_name, ls_policy, precision, kwargs)
        self.alpha = 1.0

    def _prepare(self, info):
        self.beta = 1.0
