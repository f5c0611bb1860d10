"""Host side of the B200 two-phase substep: ctypes mirror of include/pvof.h,
case builders and the ``Solver`` wrapper around the CUDA library."""
from . import abi, cases  # noqa: F401
from .runtime import PvofError, Solver, load  # noqa: F401
