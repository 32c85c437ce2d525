"""elegant_b200: B200-native particle tracking for elegant's hot path
(DRIF/EDRIFT, KQUAD/KSEXT, CSBEND, RFCA, MAXAMP; CSRCSBEND/CSRDRIFT).

The compute path is the CUDA library ``libelegant_b200.so`` behind the C ABI
in ``include/elegant_b200.h``; this package is its Python host layer.
"""
from .beam import Beam, gaussian_beam, p_central_from_momentum_mev  # noqa: F401
from .lattice import Element, Lattice, LatticeError, parse_lte  # noqa: F401
from .track import Tracker, TrackResult, track  # noqa: F401

__all__ = ["Beam", "gaussian_beam", "p_central_from_momentum_mev", "Element", "Lattice", "LatticeError",
           "parse_lte", "Tracker", "TrackResult", "track"]
