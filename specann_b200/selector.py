"""Solver registry with the reference's names (utils/selector.py:4-16), mapped to the B200 classes."""
import importlib

SOLVERS = {
    'spectral_annealing': ('specann_b200.spectral_annealing', 'SpectralAnnealing'),   # SpecAnn
    'spec_adj': ('specann_b200.spec_adj', 'Alpha0GPU'),                               # SpecAdj (alpha = 0)
    'spec_signed_lap': ('specann_b200.spec_signed_lap', 'Alpha1GPU'),                 # SpecSignedLap (alpha = 1)
}


def get_solver_class(solver_name: str):
    """Import and return the class of a solver name."""
    if solver_name not in SOLVERS:
        raise ValueError(f"Unknown solver {solver_name!r}; choose one of {sorted(SOLVERS)}")
    module, cls = SOLVERS[solver_name]
    return getattr(importlib.import_module(module), cls)
