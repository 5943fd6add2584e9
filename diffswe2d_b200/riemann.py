"""Riemann solver on the B200 kernels: drop-ins for ``primitive`` and
``bflood_hllc_flux`` (``src/riemann.py:20-105``)."""
from __future__ import annotations

import torch

from . import _native as nat


def primitive(U, gravity: float, epsilon: float, dry_depth: float):
    """[h, hu, hv] -> depth, velocities and celerity (src/riemann.py:20-38)."""
    if U.ndim != 4 or U.shape[1] != 3:
        raise ValueError(f"U must have shape [batch, 3, ny, nx], got {tuple(U.shape)}.")
    if gravity <= 0 or epsilon <= 0 or dry_depth < 0:
        raise ValueError("Require gravity > 0, epsilon > 0, dry_depth >= 0.")
    U = nat.require_cuda_f32("U", U)
    B, _, H, W = U.shape
    outs = [torch.empty((B, 1, H, W), dtype=U.dtype, device=U.device) for _ in range(4)]
    p = nat.params_basic(gravity, epsilon, dry_depth)
    rc = nat.lib().swe_primitive_f32(nat.ptr(U), B, H, W, p, *[nat.ptr(o) for o in outs],
                                     nat.stream_handle(U.device))
    nat.check(rc, "primitive")
    return tuple(outs)


def bflood_hllc_flux(UL, UR, normal: str, gravity: float, epsilon: float, dry_depth: float):
    """B-Flood two-wave HLL flux with dry-front treatment (src/riemann.py:41-105).

    Returns ``(flux, max_wave_speed)``.
    """
    if normal not in ("x", "y"):
        raise ValueError("normal must be 'x' or 'y'.")
    if UL.shape != UR.shape:
        raise ValueError(f"UL and UR shapes differ: {UL.shape} != {UR.shape}.")
    if UL.ndim != 4 or UL.shape[1] != 3:
        raise ValueError(f"U must have shape [batch, 3, ny, nx], got {tuple(UL.shape)}.")
    if gravity <= 0 or epsilon <= 0 or dry_depth < 0:
        raise ValueError("Require gravity > 0, epsilon > 0, dry_depth >= 0.")
    UL = nat.require_cuda_f32("UL", UL)
    UR = nat.require_cuda_f32("UR", UR)
    B, _, H, W = UL.shape
    flux = torch.empty_like(UL)
    speed = torch.empty((B, 1, H, W), dtype=UL.dtype, device=UL.device)
    p = nat.params_basic(gravity, epsilon, dry_depth)
    rc = nat.lib().swe_hll_flux_f32(nat.ptr(UL), nat.ptr(UR), B, H, W, 1 if normal == "y" else 0, p,
                                    nat.ptr(flux), nat.ptr(speed), nat.stream_handle(UL.device))
    nat.check(rc, "bflood_hllc_flux")
    return flux, speed
