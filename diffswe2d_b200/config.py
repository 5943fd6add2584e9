"""SWEConfig: numerical configuration of the structured-grid solver.

Same fields, defaults and meaning as the reference's ``SWEConfig``
(``src/config.py:4-28``), so a reference config can be passed unchanged.
"""
from dataclasses import dataclass


@dataclass
class SWEConfig:
    """Numerical configuration for the structured-grid solver."""

    gravity: float = 9.81
    dry_depth: float = 1.0e-6
    epsilon: float = 1.0e-12
    cfl: float = 0.5
    limiter_theta: float = 1.3
    # "wall", "constant", "water_level", "transmissive", "periodic" or "absorbing"
    boundary_left: str = "water_level"
    boundary_right: str = "water_level"
    boundary_top: str = "water_level"
    boundary_bottom: str = "water_level"
    constant_value: float = 0.0  # for "constant" boundaries
    constant_level: float = 0.0  # for "water_level" boundaries
    water_slope_reset: bool = True
    positivity_limiter: bool = True
    apply_friction: bool = True
    frictionmodel: str = "manning"
    rainfall_outside_domain: str = "zero"
