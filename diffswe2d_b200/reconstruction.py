"""Hydrostatic reconstruction on the B200 kernels: drop-in for
``bflood_cn_reconstruction`` (``src/reconstruction.py:18-108``)."""
from __future__ import annotations

import torch

from . import _native as nat


def bflood_cn_reconstruction(U, bed, dim, gravity, epsilon, dry_depth, theta=1.3,
                             water_slope_reset=True):
    """B-Flood combined CN hydrostatic reconstruction along ``dim``.

    ``U`` is a (padded) state [B,3,H,W], ``bed`` [1|B,1,H,W]; ``dim`` is -1
    (x) or -2 (y).  Values at the two array ends use torch.roll wrap-around as
    the reference does.  Returns ``(UL, UR, source_L, source_R)``.
    """
    if U.ndim != 4 or U.shape[1] != 3:
        raise ValueError(f"U must have shape [batch, 3, ny, nx], got {tuple(U.shape)}.")
    if gravity <= 0 or epsilon <= 0 or dry_depth < 0:
        raise ValueError("Require gravity > 0, epsilon > 0, dry_depth >= 0.")
    d = dim if dim < 0 else dim - 4
    if d not in (-1, -2):
        raise ValueError(f"dim must select x (-1) or y (-2), got {dim}.")
    if bed.ndim == 2:
        bed = bed[None, None]
    if bed.ndim != 4 or bed.shape[1] != 1 or bed.shape[-2:] != U.shape[-2:] or \
            bed.shape[0] not in (1, U.shape[0]):
        raise ValueError(f"bed must have shape [1|B,1,H,W] matching U, got {tuple(bed.shape)}.")
    U = nat.require_cuda_f32("U", U)
    bed = nat.require_cuda_f32("bed", bed)
    B, _, H, W = U.shape
    UL, UR = torch.empty_like(U), torch.empty_like(U)
    sL = torch.empty((B, 1, H, W), dtype=U.dtype, device=U.device)
    sR = torch.empty_like(sL)
    p = nat.params_basic(gravity, epsilon, dry_depth, theta, water_slope_reset)
    rc = nat.lib().swe_reconstruction_f32(nat.ptr(U), nat.ptr(bed), B, bed.shape[0], H, W, d, p,
                                          nat.ptr(UL), nat.ptr(UR), nat.ptr(sL), nat.ptr(sR),
                                          nat.stream_handle(U.device))
    nat.check(rc, "bflood_cn_reconstruction")
    return UL, UR, sL, sR
