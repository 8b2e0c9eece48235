"""bmc_b200 -- the Bloch-McConnell forward model and Levenberg-Marquardt fit of BMC-JAX, on B200.

The public API mirrors BMC-JAX (simulation, sequences, fitting, design, mrf, settings); the
computation runs in libbmc_b200.so, hand-written CUDA for sm_100a behind a C ABI
(include/bmc_b200.h). See `simulation` for the forward model and `fitting` for the fits.
"""
from . import settings                       # noqa: F401
from ._lib import lib as _load_library       # noqa: F401

__version__ = "0.1.0"
