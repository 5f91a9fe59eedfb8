"""B200 (sm_100a) implementation of the QCMaquis DMRG hot path: symmetry-blocked
H·psi and left/right boundary steps behind the libdmrgb200 C ABI."""
from . import _capi  # noqa: F401  (loads libdmrgb200.so, fails loudly when missing)

__all__ = ["_capi", "models", "mps", "engine"]
