"""Alpha1GPU (SpecSignedLap) lives in spec_adj.py beside Alpha0GPU; this module keeps the reference's
module name (models/spec_signed_lap.py) for the solver registry."""
from .spec_adj import Alpha1GPU

__all__ = ["Alpha1GPU"]
