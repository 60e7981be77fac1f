"""B200-native structured 2D shallow-water step (drop-in for Rakali's C ABI).

``Rakali`` mirrors the reference's structured Python front end over
``librakali.so``, a hand-written sm_100a CUDA implementation of the SSP-RK2
barotropic step (hydrostatic/minmod reconstruction, HLL/HLLC, Manning
friction, CFL reduction).  Build the library with
``python -m rakali_b200.build``.
"""
from .core import Rakali, kwargs_to_namelist, validate_namelist

__version__ = "0.1.0"
__all__ = ["Rakali", "kwargs_to_namelist", "validate_namelist", "__version__"]
