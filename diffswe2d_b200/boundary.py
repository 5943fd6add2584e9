"""Ghost cells on the B200 kernels: drop-in for ``add_ghost_cells``
(``src/boundary.py:150-413``), same arguments, validation and results
(corner cells included)."""
from __future__ import annotations

from typing import Union

import torch

from . import _native as nat

ScalarOrTensor = Union[float, int, torch.Tensor]

_VALID_BOUNDARY_TYPES = set(nat.BC_CODES)


def _validate_inputs(U, bed, ng, boundaries):
    """Same checks and messages as src/boundary.py:46-110."""
    if U.ndim != 4:
        raise ValueError("U must be a four-dimensional tensor with shape "
                         f"[batch, 3, ny, nx]. Received shape {tuple(U.shape)}.")
    if U.shape[1] != 3:
        raise ValueError("U must contain three channels [h, hu, hv]. "
                         f"Received {U.shape[1]} channels.")
    if bed.ndim != 4:
        raise ValueError("bed must be a four-dimensional tensor with shape "
                         f"[batch or 1, 1, ny, nx]. Received shape {tuple(bed.shape)}.")
    if bed.shape[1] != 1:
        raise ValueError(f"bed must contain one elevation channel. Received {bed.shape[1]} channels.")
    if U.shape[-2:] != bed.shape[-2:]:
        raise ValueError("U and bed must have identical spatial dimensions. "
                         f"U has {tuple(U.shape[-2:])}; bed has {tuple(bed.shape[-2:])}.")
    if bed.shape[0] not in (1, U.shape[0]):
        raise ValueError("The bed batch dimension must be either 1 or equal to the state batch "
                         f"size. U batch={U.shape[0]}, bed batch={bed.shape[0]}.")
    if not isinstance(ng, int) or isinstance(ng, bool) or ng <= 0:
        raise ValueError(f"ng must be a positive integer. Received {ng!r}.")
    ny, nx = U.shape[-2:]
    if ng > ny or ng > nx:
        raise ValueError("ng cannot exceed either interior grid dimension. "
                         f"Received ng={ng}, ny={ny}, nx={nx}.")
    for side, boundary_type in boundaries.items():
        if boundary_type not in _VALID_BOUNDARY_TYPES:
            raise ValueError(f"Unsupported {side} boundary type {boundary_type!r}. "
                             f"Valid types are {sorted(_VALID_BOUNDARY_TYPES)}.")


def _boundary_values(value: ScalarOrTensor, reference: torch.Tensor):
    """Scalar, one-element or per-batch value (src/boundary.py:113-147)."""
    t = (value.to(dtype=reference.dtype, device=reference.device) if torch.is_tensor(value)
         else reference.new_tensor(value))
    if t.ndim == 0 or t.numel() == 1:
        return t.detach().reshape(1).contiguous(), 1
    if t.ndim == 1 and t.shape[0] == reference.shape[0]:
        return t.detach().contiguous(), reference.shape[0]
    raise ValueError("Boundary values must be a scalar, a one-element tensor, or a tensor with "
                     f"one value per batch member. Received shape {tuple(t.shape)}.")


def add_ghost_cells(U: torch.Tensor, bed: torch.Tensor, ng: int,
                    boundary_left: str = "transmissive", boundary_right: str = "transmissive",
                    boundary_top: str = "transmissive", boundary_bottom: str = "transmissive",
                    constant_value: ScalarOrTensor = 0.0, constant_level: ScalarOrTensor = 0.0):
    """Pad the SWE state and bed with ``ng`` ghost layers; returns ``(Up, zp)``."""
    boundaries = {"left": boundary_left, "right": boundary_right, "top": boundary_top,
                  "bottom": boundary_bottom}
    _validate_inputs(U, bed, ng, boundaries)
    U = nat.require_cuda_f32("U", U)
    bed = nat.require_cuda_f32("bed", bed)
    B, _, ny, nx = U.shape
    level, levelB = _boundary_values(constant_level, U)
    cval, cvalB = _boundary_values(constant_value, U)
    Up = torch.empty((B, 3, ny + 2 * ng, nx + 2 * ng), dtype=U.dtype, device=U.device)
    zp = torch.empty((bed.shape[0], 1, ny + 2 * ng, nx + 2 * ng), dtype=U.dtype, device=U.device)
    p = nat.params_basic(bcs=(boundary_left, boundary_right, boundary_top, boundary_bottom))
    rc = nat.lib().swe_ghost_cells_f32(nat.ptr(U), nat.ptr(bed), B, bed.shape[0], ny, nx, ng, p,
                                       nat.ptr(level), levelB, nat.ptr(cval), cvalB, nat.ptr(Up),
                                       nat.ptr(zp), nat.stream_handle(U.device))
    nat.check(rc, "add_ghost_cells")
    return Up, zp
