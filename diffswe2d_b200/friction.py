"""Friction updates on the B200 kernels: drop-ins for
``apply_manning_friction`` (``src/friction.py:102-131``) and
``apply_roughness_length_friction`` (``src/friction.py:69-99``)."""
from __future__ import annotations

import torch

from . import _native as nat


def _dt_value(dt) -> float:
    if torch.is_tensor(dt):
        if dt.numel() != 1:
            raise ValueError("dt must be a scalar")
        return float(dt.detach().to(torch.float32).item())
    return float(torch.tensor(float(dt), dtype=torch.float32).item())


def _apply(U, field, dt, dry_depth, epsilon, model, name):
    if U.ndim != 4 or U.shape[1] != 3:
        raise ValueError(f"U must have shape [batch, 3, ny, nx], got {tuple(U.shape)}.")
    if field.ndim == 2:
        field = field[None, None]
    B, _, ny, nx = U.shape
    if field.ndim != 4 or field.shape[1] != 1 or field.shape[-2:] != (ny, nx) or \
            field.shape[0] not in (1, B):
        field = torch.broadcast_to(field, (B, 1, ny, nx))
    U = nat.require_cuda_f32("U", U)
    field = nat.require_cuda_f32(name, field)
    out = torch.empty_like(U)
    p = nat.params_basic(epsilon=epsilon, dry_depth=dry_depth)
    rc = nat.lib().swe_friction_f32(nat.ptr(U), nat.ptr(field), field.shape[0], B, ny, nx,
                                    _dt_value(dt), model, p, nat.ptr(out),
                                    nat.stream_handle(U.device))
    nat.check(rc, "friction")
    return out


def apply_manning_friction(U, n, dt, dry_depth=1e-6, epsilon=1e-12):
    """Semi-implicit Manning friction: momentum / (1 + Cf |u| dt / h)."""
    return _apply(U, n, dt, dry_depth, epsilon, 0, "n")


def apply_roughness_length_friction(U, roughness_length, dt, dry_depth=1e-6, epsilon=1e-12):
    """Semi-implicit BG-Flood roughness-length friction."""
    return _apply(U, roughness_length, dt, dry_depth, epsilon, 1, "roughness_length")
