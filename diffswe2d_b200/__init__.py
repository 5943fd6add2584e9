"""diffswe2d_b200 -- DiffSWE2d's explicit finite-volume step on NVIDIA B200.

The package mirrors the reference's call surface (``SWEConfig``, ``SWE2D``
and the numerical operators) and runs the step as hand-written sm_100a CUDA
kernels behind the C ABI of ``include/swe_b200.h``.
"""
from .config import SWEConfig
from .solver import SWE2D

__all__ = ["SWEConfig", "SWE2D"]
__version__ = "0.1.0"
