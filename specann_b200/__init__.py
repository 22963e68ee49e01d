"""B200-native SpecAnn engine: the alpha-sweep hot path of Vgueca/SpecAnn as hand-written sm_100a
kernels behind a C-ABI (include/specann_b200.h), with drop-in solver classes."""
from .failures import EigensolverBreakdown, NumericalFailure, is_out_of_memory  # noqa: F401

__all__ = ["SpectralAnnealing", "Alpha0GPU", "Alpha1GPU", "EigensolverBreakdown", "NumericalFailure"]


def __getattr__(name):
    if name == "SpectralAnnealing":
        from .spectral_annealing import SpectralAnnealing
        return SpectralAnnealing
    if name in ("Alpha0GPU", "Alpha1GPU"):
        from . import spec_adj
        return getattr(spec_adj, name)
    raise AttributeError(name)
