"""Limiter primitives on the B200 kernels: drop-ins for ``minmod3`` and
``limited_increment`` (``src/numerics.py:4-27``)."""
from __future__ import annotations

import torch

from . import _native as nat


def minmod3(a: torch.Tensor, b: torch.Tensor, c: torch.Tensor) -> torch.Tensor:
    """Three-argument minmod limiter (broadcasting like the reference)."""
    a, b, c = torch.broadcast_tensors(a, b, c)
    a = nat.require_cuda_f32("a", a)
    b = nat.require_cuda_f32("b", b)
    c = nat.require_cuda_f32("c", c)
    out = torch.empty_like(a)
    rc = nat.lib().swe_minmod3_f32(nat.ptr(a), nat.ptr(b), nat.ptr(c), a.numel(), nat.ptr(out),
                                   nat.stream_handle(a.device))
    nat.check(rc, "minmod3")
    return out


def limited_increment(q: torch.Tensor, dim: int, theta: float = 1.3) -> torch.Tensor:
    """Limited cell increment Delta q along ``dim`` (one of the last two axes),
    with torch.roll wrap-around at the ends."""
    if q.ndim < 2:
        raise ValueError("limited_increment needs at least a 2-D tensor")
    d = dim if dim < 0 else dim - q.ndim
    if d not in (-1, -2):
        raise ValueError(f"dim must be one of the last two axes, got {dim}.")
    q = nat.require_cuda_f32("q", q)
    H, W = q.shape[-2:]
    outer = q.numel() // max(H * W, 1)
    out = torch.empty_like(q)
    rc = nat.lib().swe_limited_increment_f32(nat.ptr(q), outer, H, W, d, float(theta), nat.ptr(out),
                                             nat.stream_handle(q.device))
    nat.check(rc, "limited_increment")
    return out
