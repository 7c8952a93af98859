"""scatrs_b200: the size-distribution ensemble path of usask-arg/scatrs on NVIDIA B200.

The compute path is libscatrs_b200.so (hand-written sm_100a CUDA behind the C ABI of
include/scatrs_b200.h); this package binds it (``_native``), mirrors the reference's binding
surface for the ensemble (``_scatrs``) and its exceptions (``errors``), and draws the seeded
benchmark inputs (``workloads``).
"""

from . import errors
from ._native import ensemble_fixed, gauss_legendre, launch_count, mie

__all__ = ["ensemble_fixed", "errors", "gauss_legendre", "launch_count", "mie"]
