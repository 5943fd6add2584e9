"""diffswe2d_b200 -- DiffSWE2d's explicit finite-volume step on NVIDIA B200.

The package mirrors the reference's call surface (``SWEConfig``, ``SWE2D``
and the numerical operators) and runs the step as hand-written sm_100a CUDA
kernels behind the C ABI of ``include/swe_b200.h``.
"""
from .boundary import add_ghost_cells
from .config import SWEConfig
from .forcing import RainfallForcing
from .friction import apply_manning_friction, apply_roughness_length_friction
from .numerics import limited_increment, minmod3
from .reconstruction import bflood_cn_reconstruction
from .riemann import bflood_hllc_flux, primitive
from .solver import SWE2D

__all__ = [
    "SWEConfig",
    "SWE2D",
    "RainfallForcing",
    "add_ghost_cells",
    "bflood_cn_reconstruction",
    "bflood_hllc_flux",
    "primitive",
    "minmod3",
    "limited_increment",
    "apply_manning_friction",
    "apply_roughness_length_friction",
]
__version__ = "0.1.0"
