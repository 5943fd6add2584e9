"""SWE2D: the reference's solver module with its step on the B200 kernels.

Drop-in for ``SWE2D`` of ``src/solver.py`` (DiffSWE2d) on the forward path:
same constructor, buffers and parameter, same ``spatial_operator`` /
``stable_dt`` / ``step`` / ``forward`` signatures, return types and
exceptions.  ``step`` runs as the two fused sm_100a kernels of
``csrc/swe_step.cu``; the host reads one 8-byte word pair per step (status
and dt), where the reference synchronises three times.
"""
from __future__ import annotations

from numbers import Integral, Real
from typing import Optional, Union

import numpy as np
import torch
import torch.nn as nn

from . import _native as nat
from .config import SWEConfig

ScalarOrTensor = Union[float, int, torch.Tensor]


class SWE2D(nn.Module):
    """Differentiable B-Flood-style 2-D shallow-water solver (state [h, hu, hv]).

    ``forward(..., t_end=...)`` interprets ``t_end`` as the duration of that
    call, as the reference does (``src/solver.py:40-47``).

    ``arithmetic`` (not in the reference) selects the step kernels: "exact"
    evaluates every float32 operation of the reference's step in its order
    with IEEE rounding; "fast" is the tolerance mode (fused multiply-adds,
    hardware approximations, about twice the throughput), within FP32
    rounding of the reference.  ``rainfall`` is an object with
    ``at(time) -> rate`` (``RainfallForcing``); as in the reference, stage 1
    of a step uses the rate at the step's start and stage 2 the rate half a
    step later, so a step with rainfall reads dt between its two kernels.
    """

    def __init__(self, bed_reference, roughness_length, dx, dy, config=None, train_dem=True,
                 maximum_dem_correction=None, valid_mask=None, x=None, y=None, rainfall=None,
                 arithmetic="exact"):
        super().__init__()
        nat.arithmetic_code(arithmetic)
        self.arithmetic = arithmetic
        self.cfg = config or SWEConfig()
        self.dx, self.dy = float(dx), float(dy)
        if self.dx <= 0.0 or self.dy <= 0.0:
            raise ValueError(f"dx and dy must be positive, got {self.dx}, {self.dy}.")
        if bed_reference.ndim == 2:
            bed_reference = bed_reference[None, None]
        if roughness_length.ndim == 2:
            roughness_length = roughness_length[None, None]
        if bed_reference.ndim != 4 or bed_reference.shape[1] != 1:
            raise ValueError(f"bed_reference must have shape [ny,nx] or [B,1,ny,nx], "
                             f"got {tuple(bed_reference.shape)}.")
        if roughness_length.ndim != 4:
            raise ValueError(f"roughness_length must be 2-D or 4-D, "
                             f"got {tuple(roughness_length.shape)}.")
        if bed_reference.shape != roughness_length.shape:
            raise ValueError(f"DEM and roughness shapes differ: {bed_reference.shape} "
                             f"!= {roughness_length.shape}.")
        if not torch.isfinite(bed_reference).all():
            raise ValueError("bed_reference contains non-finite values.")
        if not torch.isfinite(roughness_length).all():
            raise ValueError("roughness_length contains non-finite values.")
        self.register_buffer("bed_reference", bed_reference.clone())
        self.register_buffer("roughness_length", roughness_length.clone())
        mask = (torch.ones_like(bed_reference, dtype=torch.bool) if valid_mask is None
                else valid_mask.reshape_as(bed_reference).bool())
        self.register_buffer("valid_mask", mask)
        if x is not None:
            self.register_buffer("x", x.clone())
        if y is not None:
            self.register_buffer("y", y.clone())
        self.maximum_dem_correction = maximum_dem_correction
        self.dem_correction_parameter = nn.Parameter(torch.zeros_like(bed_reference),
                                                     requires_grad=bool(train_dem))
        self.train_dem = bool(train_dem)
        self.rainfall = rainfall
        self.use_dynamic_bc = False
        self.bc_times = None
        self.bc_wls = None
        self.track_gauges = False
        self.gauge_indices = {}
        self.bed_elevations = {}
        self.ts_time, self.ts_dt = [], []
        self.ts_h, self.ts_z = {}, {}

    # ------------------------------------------------------------- properties
    @property
    def bed(self):
        """Current bed: bed_reference + correction * mask (src/solver.py:134-147)."""
        correction = self.dem_correction_parameter
        if self.maximum_dem_correction is not None:
            correction = float(self.maximum_dem_correction) * torch.tanh(correction)
        return self.bed_reference + correction * self.valid_mask.to(self.bed_reference.dtype)

    def dem_regularization(self, prior_weight=1.0, slope_weight=0.0, curvature_weight=0.0):
        """Prior, slope and curvature penalty of the DEM-correction inversion
        (src/solver.py:807-836): mean squared correction, mean squared first
        differences of the bed along x and y, mean squared second
        differences; PyTorch operations on the bed (autograd supplies their
        gradient, the hand-written adjoint the simulation's)."""
        bed = self.bed
        correction = bed - self.bed_reference
        d_x = bed[..., 1:] - bed[..., :-1]
        d_y = bed[..., 1:, :] - bed[..., :-1, :]
        prior = correction.square().mean()
        slope = d_x.square().mean() + d_y.square().mean()
        zero = bed.new_zeros(())
        curv_x = (d_x[..., 1:] - d_x[..., :-1]).square().mean() if d_x.shape[-1] >= 2 else zero
        curv_y = (d_y[..., 1:, :] - d_y[..., :-1, :]).square().mean() if d_y.shape[-2] >= 2 else zero
        return (float(prior_weight) * prior + float(slope_weight) * slope
                + float(curvature_weight) * (curv_x + curv_y))

    # ------------------------------------------------------ configuration
    def set_dynamic_boundary(self, times: torch.Tensor, water_levels: torch.Tensor,
                             enabled: bool = True) -> None:
        """Time-varying boundary level (src/solver.py:329-354)."""
        if not torch.is_tensor(times) or not torch.is_tensor(water_levels):
            raise TypeError("times and water_levels must be tensors.")
        if times.ndim != 1 or water_levels.ndim != 1:
            raise ValueError("times and water_levels must be one-dimensional.")
        if times.numel() == 0 or times.numel() != water_levels.numel():
            raise ValueError("Boundary arrays must be non-empty and equal length.")
        if times.numel() > 1 and not torch.all(times[1:] > times[:-1]):
            raise ValueError("Dynamic boundary times must be strictly increasing.")
        if not torch.isfinite(times).all() or not torch.isfinite(water_levels).all():
            raise ValueError("Dynamic boundary arrays contain non-finite values.")
        self.bc_times, self.bc_wls = times, water_levels
        self.use_dynamic_bc = bool(enabled)

    def clear_dynamic_boundary(self) -> None:
        self.use_dynamic_bc = False
        self.bc_times = self.bc_wls = None

    def reset_gauge_tracking(self) -> None:
        self.ts_time, self.ts_dt = [], []
        self.ts_h = {name: [] for name in self.gauge_indices}
        self.ts_z = {name: [] for name in self.gauge_indices}

    @staticmethod
    def _expand(field: torch.Tensor, batch: int) -> torch.Tensor:
        if field.shape[0] == batch:
            return field
        if field.shape[0] != 1:
            raise ValueError(f"Field batch must be 1 or {batch}, got {field.shape[0]}.")
        return field.expand(batch, -1, -1, -1)

    @staticmethod
    def _prepare_boundary_level(level: ScalarOrTensor, reference: torch.Tensor) -> torch.Tensor:
        if torch.is_tensor(level):
            return level.to(dtype=reference.dtype, device=reference.device)
        return reference.new_tensor(level)

    def _interpolate_dynamic_boundary(self, current_time: float,
                                      reference: torch.Tensor) -> torch.Tensor:
        """Linear interpolation of the boundary series (src/solver.py:391-415)."""
        if self.bc_times is None or self.bc_wls is None:
            raise RuntimeError("Dynamic boundary forcing is not configured.")
        times = self.bc_times.to(dtype=reference.dtype, device=reference.device)
        levels = self.bc_wls.to(dtype=reference.dtype, device=reference.device)
        time = reference.new_tensor(current_time)
        index = torch.searchsorted(times, time, right=False)
        index = torch.clamp(index, 1, times.numel() - 1)
        t0, t1 = times[index - 1], times[index]
        w0, w1 = levels[index - 1], levels[index]
        weight = (time - t0) / torch.clamp(t1 - t0, min=torch.finfo(times.dtype).eps)
        return w0 + weight * (w1 - w0)

    def _resolve_boundary_level(self, current_time: float, U: torch.Tensor,
                                explicit_boundary_level: Optional[ScalarOrTensor]) -> torch.Tensor:
        if explicit_boundary_level is not None:
            return self._prepare_boundary_level(explicit_boundary_level, U)
        if self.use_dynamic_bc:
            return self._interpolate_dynamic_boundary(current_time, U)
        return self._prepare_boundary_level(self.cfg.constant_level, U)

    # ------------------------------------------------------ argument packing
    def _params(self):
        return nat.params(self.cfg, self.dx, self.dy, self.arithmetic)

    @staticmethod
    def _level_arg(level: torch.Tensor, batch: int):
        """Boundary value forms of src/boundary.py:113-147 -> (tensor, count)."""
        lv = level.detach().reshape(-1) if level.ndim > 0 else level.detach().reshape(1)
        if lv.numel() == 1:
            return lv.contiguous(), 1
        if level.ndim == 1 and lv.numel() == batch:
            return lv.contiguous(), batch
        raise ValueError("Boundary values must be a scalar, a one-element tensor, or a tensor "
                         f"with one value per batch member. Received shape {tuple(level.shape)}.")

    @staticmethod
    def _forcing_arg(value, h: torch.Tensor):
        """Rain / infiltration argument -> (tensor or None, mode, batch)."""
        if value is None:
            return None, nat.FORCING_NONE, 1
        t = (value.to(dtype=h.dtype, device=h.device) if torch.is_tensor(value)
             else h.new_tensor(value))
        if t.numel() == 1:
            return t.detach().reshape(1).contiguous(), nat.FORCING_SCALAR, 1
        B, _, ny, nx = h.shape
        t = t.detach()
        while t.ndim < 4:
            t = t.unsqueeze(0)
        if t.shape[-2:] != (ny, nx) or t.shape[1] != 1 or t.shape[0] not in (1, B):
            t = torch.broadcast_to(t, (B, 1, ny, nx))
        return t.contiguous(), nat.FORCING_FIELD, t.shape[0]

    def _check_state(self, U):
        if U.ndim != 4 or U.shape[1] != 3:
            raise ValueError(f"U must have shape [batch,3,ny,nx], got {tuple(U.shape)}.")
        ny, nx = U.shape[-2:]
        if self.bed_reference.shape[-2:] != (ny, nx):
            raise ValueError("U and bed must have identical spatial dimensions. "
                             f"U has {(ny, nx)}; bed has {tuple(self.bed_reference.shape[-2:])}.")
        if ny < 2 or nx < 2:
            raise ValueError(f"ng cannot exceed either interior grid dimension. "
                             f"Received ng=2, ny={ny}, nx={nx}.")

    def _fields(self, U):
        B = U.shape[0]
        bed = nat.require_cuda_f32("bed", self.bed.detach())
        if bed.shape[0] not in (1, B):
            raise ValueError(f"Field batch must be 1 or {B}, got {bed.shape[0]}.")
        n = nat.require_cuda_f32("roughness_length", self.roughness_length.detach())
        if n.shape[0] not in (1, B):
            raise ValueError(f"Field batch must be 1 or {B}, got {n.shape[0]}.")
        return bed, n

    # ------------------------------------------------------ spatial operator
    def spatial_operator(self, U, rainfall_rate=None, infiltration=None, return_wave_speed=False,
                         boundary_level=None):
        """Conservative SWE tendency (src/solver.py:448-531)."""
        self._check_state(U)
        U = nat.require_cuda_f32("U", U)
        B, _, ny, nx = U.shape
        bed, _ = self._fields(U)
        level = self._prepare_boundary_level(
            self.cfg.constant_level if boundary_level is None else boundary_level, U)
        lv, levelB = self._level_arg(level, B)
        h = U[:, 0:1]
        rain, rmode, rB = self._forcing_arg(rainfall_rate, h)
        infil, imode, iB = self._forcing_arg(infiltration, h)
        rhs = torch.empty_like(U)
        red = torch.empty(nat.RED_WORDS, dtype=torch.int32, device=U.device)
        p = self._params()
        rc = nat.lib().swe_spatial_operator_f32(
            nat.ptr(U), nat.ptr(bed), B, bed.shape[0], ny, nx, p, nat.ptr(lv), levelB,
            nat.ptr(rain), rmode, rB, nat.ptr(infil), imode, iB, nat.ptr(rhs), nat.ptr(red),
            nat.stream_handle(U.device))
        nat.check(rc, "spatial_operator")
        if return_wave_speed:
            ax, ay = red[0:2].view(torch.float32).unbind(0)
            return rhs, ax, ay
        return rhs

    def stable_dt(self, U, boundary_level=None):
        """CFL-stable time step (src/solver.py:537-545)."""
        _, ax, ay = self.spatial_operator(U, return_wave_speed=True, boundary_level=boundary_level)
        denominator = torch.clamp(ax / self.dx + ay / self.dy, min=self.cfg.epsilon)
        return self.cfg.cfl / denominator

    def _clean_and_limit(self, old, candidate):
        """Positivity preservation and dry-cell momentum removal (src/solver.py:547-570)."""
        old = nat.require_cuda_f32("old", old)
        candidate = nat.require_cuda_f32("candidate", candidate)
        if old.shape != candidate.shape or old.ndim != 4 or old.shape[1] != 3:
            raise ValueError(f"old and candidate must both be [B,3,ny,nx], got "
                             f"{tuple(old.shape)} and {tuple(candidate.shape)}.")
        B, _, ny, nx = old.shape
        out = torch.empty_like(old)
        rc = nat.lib().swe_clean_and_limit_f32(nat.ptr(old), nat.ptr(candidate), B, ny, nx,
                                               self._params(), nat.ptr(out),
                                               nat.stream_handle(old.device))
        nat.check(rc, "_clean_and_limit")
        return out

    # ------------------------------------------------------------------ step
    def step(self, U, model_time, max_dt, infiltration=None, boundary_level=None):
        """One adaptive midpoint predictor-corrector step (src/solver.py:572-663).

        Returns ``(U_new, dt_float)``.  The CFL time step is detached, as in
        the reference.
        """
        self._check_state(U)
        if self._needs_adjoint(U, boundary_level):
            if self.rainfall is not None:
                raise NotImplementedError("the step adjoint has no rainfall source; differentiate "
                                          "a model without rainfall")
            from .adjoint import step_with_adjoint
            return step_with_adjoint(self, U, model_time, max_dt, infiltration, boundary_level)
        U = nat.require_cuda_f32("U", U)
        B, _, ny, nx = U.shape
        max_dt_f = float((max_dt.to(dtype=torch.float32) if torch.is_tensor(max_dt)
                          else torch.tensor(float(max_dt), dtype=torch.float32)).item())
        level = self._prepare_boundary_level(
            self.cfg.constant_level if boundary_level is None else boundary_level, U)
        if self.rainfall is not None:
            # model_time is taken in U's dtype first (src/solver.py:593-597, :608)
            time_float = float(np.float32(self._scalar_float(model_time, "model_time")))
            U_new, status, dt = self._launch_step_rain(U, level, max_dt_f, infiltration, time_float)
        else:
            U_new, status, dt = self._launch_step(U, level, max_dt_f, infiltration)
        self._raise_on_status(status, dt)
        return U_new, dt

    def _needs_adjoint(self, U, boundary_level) -> bool:
        """A step is differentiated when autograd is on and the state, the
        boundary level, the roughness field or the DEM correction requires
        grad."""
        if not torch.is_grad_enabled():
            return False
        return bool(U.requires_grad or self.roughness_length.requires_grad
                    or self.dem_correction_parameter.requires_grad
                    or (torch.is_tensor(boundary_level) and boundary_level.requires_grad))

    def _launch_step(self, U, level, max_dt_f, infiltration, red=None, scratch=None):
        """Enqueue one step; returns (U_new, status, dt) with one host read."""
        B, _, ny, nx = U.shape
        bed, n = self._fields(U)
        lv, levelB = self._level_arg(level, B)
        infil, imode, iB = self._forcing_arg(infiltration, U[:, 0:1])
        U_out = torch.empty_like(U)
        scratch = torch.empty_like(U) if scratch is None else scratch
        red = torch.empty(nat.RED_WORDS, dtype=torch.int32, device=U.device) if red is None else red
        p = self._params()
        rc = nat.lib().swe_step_f32(
            nat.ptr(U), nat.ptr(bed), bed.shape[0], nat.ptr(n), n.shape[0], B, ny, nx, p,
            nat.ptr(lv), levelB, max_dt_f, nat.ptr(infil), imode, iB, nat.ptr(scratch),
            nat.ptr(red), nat.ptr(U_out), nat.stream_handle(U.device))
        nat.check(rc, "step")
        host = red[2:4].cpu()
        status = int(host[0].item()) & 0xFFFFFFFF
        dt = float(host[1:2].view(torch.float32).item())
        return U_out, status, dt

    def _host_dt(self, red_host: torch.Tensor, max_dt_f: float) -> float:
        """The step's dt from the stage-1 maxima, in float32 as the kernels and
        the reference compute it (src/solver.py:620-626)."""
        ax, ay = (float(v) for v in red_host[0:2].view(torch.float32))
        f = np.float32
        den = max(f(f(ax) / f(self.dx)) + f(f(ay) / f(self.dy)), f(self.cfg.epsilon))
        stable = f(f(1.0) / f(den)) * f(self.cfg.cfl)
        return float(stable if np.isnan(stable) else min(stable, f(max_dt_f)))

    def _launch_step_rain(self, U, level, max_dt_f, infiltration, time_float):
        """One step with the rainfall source: stage 1 with the rate at the
        step's start, dt read on the host, stage 2 with the rate at t + dt/2
        (src/solver.py:609-643)."""
        B, _, ny, nx = U.shape
        bed, n = self._fields(U)
        lv, levelB = self._level_arg(level, B)
        h = U[:, 0:1]
        infil, imode, iB = self._forcing_arg(infiltration, h)
        U_out = torch.empty_like(U)
        scratch = torch.empty_like(U)
        red = torch.empty(nat.RED_WORDS, dtype=torch.int32, device=U.device)
        p = self._params()
        st = nat.stream_handle(U.device)
        lib = nat.lib()

        def stage(k, rate):
            rain, rmode, rB = self._forcing_arg(rate, h)
            rc = lib.swe_step_stage_forced_f32(
                k, nat.ptr(U), nat.ptr(bed), bed.shape[0], nat.ptr(n), n.shape[0], B, ny, nx, p,
                nat.ptr(lv), levelB, max_dt_f, nat.ptr(rain), rmode, rB, nat.ptr(infil), imode, iB,
                nat.ptr(scratch), nat.ptr(red), nat.ptr(U_out), st)
            nat.check(rc, "step")
            return rain  # kept alive until the kernel has read it

        keep = stage(1, self.rainfall.at(time_float))
        host = red.cpu()
        status = int(host[2].item()) & 0xFFFFFFFF
        if status & nat.S_NONFINITE_STATE:
            return U_out, status, float("nan")
        dt = self._host_dt(host, max_dt_f)
        if not np.isfinite(dt) or not dt > 0.0:
            return U_out, nat.S_NONFINITE_DT if not np.isfinite(dt) else nat.S_NONPOSITIVE_DT, dt
        keep = stage(2, self.rainfall.at(time_float + 0.5 * dt))
        host = red[2:4].cpu()
        del keep
        status = int(host[0].item()) & 0xFFFFFFFF
        return U_out, status, float(host[1:2].view(torch.float32).item())

    @staticmethod
    def _raise_on_status(status: int, dt: float) -> None:
        if status & (nat.S_NONFINITE_DT | nat.S_NONFINITE_STATE):
            raise FloatingPointError("The calculated timestep is non-finite.")
        if status & nat.S_NONPOSITIVE_DT:
            raise FloatingPointError(f"Non-positive timestep: {dt}.")

    # --------------------------------------------------------------- forward
    @staticmethod
    def _scalar_float(value, name: str) -> float:
        if torch.is_tensor(value):
            if value.numel() != 1:
                raise ValueError(f"{name} must be scalar.")
            return float(value.detach().cpu())
        if isinstance(value, Real):
            return float(value)
        raise TypeError(f"{name} must be a real scalar or scalar tensor.")

    def forward(self, U0, t_end, start_time=0.0, max_steps=1_000_000, infiltration=None,
                callback=None, boundary_level=None, max_dt_cap=None):
        """Advance the model for ``t_end`` seconds (src/solver.py:680-779).

        Returns ``(U, hmax)``.
        """
        if U0.ndim != 4 or U0.shape[1] != 3:
            raise ValueError(f"U0 must have shape [batch,3,ny,nx], got {tuple(U0.shape)}.")
        duration = self._scalar_float(t_end, "t_end")
        absolute_start = self._scalar_float(start_time, "start_time")
        if not isinstance(max_steps, Integral) or isinstance(max_steps, bool) or max_steps <= 0:
            raise ValueError(f"max_steps must be positive, got {max_steps!r}.")
        if duration < 0.0:
            raise ValueError(f"t_end duration cannot be negative: {duration}.")
        if duration == 0.0:
            return U0, U0[:, 0].clone()
        if self._device_loop_ok(U0, callback, boundary_level, max_dt_cap):
            return self._forward_device(U0, duration, absolute_start, int(max_steps), infiltration,
                                        boundary_level, max_dt_cap)
        U, hmax, elapsed = U0, U0[:, 0].clone(), 0.0
        tolerance = max(1e-12, 1e-12 * abs(duration))
        for iteration in range(max_steps):
            remaining = duration - elapsed
            if remaining <= tolerance:
                self.last_forward_steps = iteration
                return U, hmax
            step_max_dt = remaining
            if max_dt_cap is not None:
                step_max_dt = min(remaining, self._scalar_float(max_dt_cap, "max_dt_cap"))
            current_time = absolute_start + elapsed
            level = self._resolve_boundary_level(current_time, U, boundary_level)
            U, dt_value = self.step(U, model_time=current_time, max_dt=step_max_dt,
                                    infiltration=infiltration, boundary_level=level)
            hmax = torch.maximum(hmax, U[:, 0])
            elapsed += dt_value
            if elapsed > duration and elapsed - duration <= tolerance:
                elapsed = duration
            if self.track_gauges:
                self._record_gauges(U, absolute_start + elapsed, dt_value)
            if callback is not None:
                callback(iteration, absolute_start + elapsed, U)
        raise RuntimeError(f"max_steps={max_steps} reached after {elapsed:.8f} s; "
                           f"requested duration={duration:.8f} s.")

    # ------------------------------------------------ device-driven forward
    #: steps per CUDA-graph replay of the device-driven loop (even: the state
    #: ping-pongs between two buffers and ends each chunk in the first)
    steps_per_chunk = 32

    def _device_loop_ok(self, U0, callback, boundary_level, max_dt_cap) -> bool:
        """The device loop serves forward() calls that need no host work per
        step: no callback, no autograd, and a positive max_dt cap if any."""
        if callback is not None or not U0.is_cuda or U0.dtype != torch.float32:
            return False
        if self.rainfall is not None:  # rates are evaluated on the host per stage
            return False
        if self._needs_adjoint(U0, boundary_level) or (
                torch.is_grad_enabled() and boundary_level is None and self.use_dynamic_bc
                and self.bc_wls.requires_grad):
            return False
        if max_dt_cap is not None and not self._scalar_float(max_dt_cap, "max_dt_cap") > 0.0:
            return False
        return True

    def _forward_device(self, U0, duration, absolute_start, max_steps, infiltration,
                        boundary_level, max_dt_cap):
        """forward() with the time loop on the device (src/solver.py:680-779).

        Each chunk of ``steps_per_chunk`` steps is one replay of a CUDA graph
        of [stage 1, stage 2, clock] launches; the host reads the 72-byte
        clock once per chunk.  The graph and its buffers are captured once per
        shape and configuration (``_DeviceLoop``) and reused by later calls.
        Results are those of the host loop bit for bit.
        """
        self._check_state(U0)
        U0 = nat.require_cuda_f32("U0", U0.detach())
        dev = U0.device
        B, _, ny, nx = U0.shape
        bed, n = self._fields(U0)
        if boundary_level is not None:
            lv, levelB = self._level_arg(self._prepare_boundary_level(boundary_level, U0), B)
            series = None
        elif self.use_dynamic_bc:
            lv, levelB = None, 1
            series = (self.bc_times.detach().to(dtype=torch.float32, device=dev),
                      self.bc_wls.detach().to(dtype=torch.float32, device=dev))
        else:
            lv, levelB = self._level_arg(self._prepare_boundary_level(self.cfg.constant_level, U0), B)
            series = None
        infil, imode, iB = self._forcing_arg(infiltration, U0[:, 0:1])
        names = list(self.gauge_indices) if self.track_gauges else []
        cells = []
        for name in names:
            iy, ix = self.gauge_indices[name]
            if not (0 <= iy < ny and 0 <= ix < nx):
                raise ValueError(f"gauge cell {(iy, ix)} outside the {ny}x{nx} grid")
            cells.append((int(iy), int(ix)))
        p = self._params()
        key = (B, ny, nx, str(dev), bed.shape[0], n.shape[0], levelB,
               None if series is None else series[0].numel(), tuple(cells), imode, iB,
               None if infil is None else tuple(infil.shape), self.steps_per_chunk, bytes(p))
        loops = self.__dict__.setdefault("_device_loops", {})
        loop = loops.get(key)
        if loop is None:
            loop = _DeviceLoop(self, key, B, ny, nx, dev, bed.shape, n.shape, levelB, series, cells,
                               infil, imode, iB, p, self.steps_per_chunk)
            loops[key] = loop
        cap = self._scalar_float(max_dt_cap, "max_dt_cap") if max_dt_cap is not None else 0.0
        clock = nat.SweClock(duration, absolute_start, max(1e-12, 1e-12 * abs(duration)), cap, 0.0,
                             max_steps, 0, 0, 0, 0, 0.0, 0.0, 0.0)
        steps_seen = 0
        bed_at = {}
        if names:
            bed0 = self.bed.detach()[0, 0]
            bed_at = {name: float(bed0[iy, ix]) for name, (iy, ix) in zip(names, cells)}
        for state, c in loop.run(U0, bed, n, lv, series, infil, clock):
            if names and c.steps > steps_seen:
                rows = loop.gbuf.cpu().numpy()
                for k in range(steps_seen, c.steps):
                    r = rows[k % loop.chunk]
                    self.ts_time.append(float(r[0]))
                    self.ts_dt.append(float(r[1]))
                    for g, name in enumerate(names):
                        depth = float(r[2 + g])
                        self.ts_h.setdefault(name, []).append(depth)
                        self.ts_z.setdefault(name, []).append(depth + bed_at[name])
            steps_seen = c.steps
            if c.state == nat.CLOCK_FAILED:
                self._raise_on_status(c.dt_status, float(c.last_dt))
            if c.state == nat.CLOCK_MAXSTEPS:
                raise RuntimeError(f"max_steps={max_steps} reached after {c.elapsed:.8f} s; "
                                   f"requested duration={duration:.8f} s.")
        self.last_forward_steps = steps_seen
        return loop.bufs[0].clone(), loop.hmax.clone()

    def _record_gauges(self, U: torch.Tensor, absolute_time: float, dt_value: float) -> None:
        """Micro-step gauge records (src/solver.py:781-801)."""
        self.ts_time.append(absolute_time)
        self.ts_dt.append(dt_value)
        current_bed = self.bed
        for name, (iy, ix) in self.gauge_indices.items():
            self.ts_h.setdefault(name, [])
            self.ts_z.setdefault(name, [])
            depth = float(U[0, 0, iy, ix].detach().cpu())
            bed = float(current_bed[0, 0, iy, ix].detach().cpu())
            self.ts_h[name].append(depth)
            self.ts_z[name].append(depth + bed)


def replay_lengths(chunk: int):
    """Step counts of the device loop's graphs: ``chunk`` and its halvings
    while they stay even (32 -> [32, 16, 8, 4, 2]); every length is even so
    that a replay leaves the state in the first of the two buffers."""
    sizes = [int(chunk)]
    while sizes[-1] > 2 and sizes[-1] % 4 == 0:
        sizes.append(sizes[-1] // 2)
    return sizes


def replay_length(sizes, left: float) -> int:
    """The longest of ``sizes`` (descending) that ``left`` more steps fill,
    else the shortest."""
    return next((m for m in sizes if m <= left), sizes[-1])


class _DeviceLoop:
    """Buffers and captured CUDA graph of the device-driven forward() loop for
    one (shape, configuration) of a model.  Inputs are copied into the
    buffers at each call; the graph runs ``chunk`` steps per replay."""

    def __init__(self, model, key, B, ny, nx, dev, bed_shape, n_shape, levelB, series, cells, infil,
                 imode, iB, params, chunk):
        self.chunk = int(chunk)
        self.bufs = [torch.empty((B, 3, ny, nx), device=dev), torch.empty((B, 3, ny, nx), device=dev)]
        self.scratch = torch.empty((B, 3, ny, nx), device=dev)
        self.red = torch.zeros(nat.RED_WORDS, dtype=torch.int32, device=dev)
        self.hmax = torch.empty((B, ny, nx), device=dev)
        self.bed = torch.empty(bed_shape, device=dev)
        self.n = torch.empty(n_shape, device=dev)
        self.lv = torch.zeros(levelB, device=dev)
        self.nseries = 0 if series is None else series[0].numel()
        self.series_t = None if series is None else torch.empty(self.nseries, device=dev)
        self.series_w = None if series is None else torch.empty(self.nseries, device=dev)
        self.infil = None if infil is None else torch.empty_like(infil)
        self.imode, self.iB = imode, iB
        self.ncells = len(cells)
        self.cells = (torch.tensor(cells, dtype=torch.int32, device=dev).reshape(-1).contiguous()
                      if cells else None)
        self.gbuf = (torch.zeros((self.chunk, 2 + self.ncells), dtype=torch.float64, device=dev)
                     if cells else None)
        self.clock = torch.zeros(72, dtype=torch.uint8, device=dev)
        self.clock_host = torch.zeros(72, dtype=torch.uint8).pin_memory()
        self.params = params
        self.arithmetic = model.arithmetic
        self.B, self.ny, self.nx, self.levelB, self.dev = B, ny, nx, levelB, dev
        # graphs of `chunk` steps and of the shorter tail lengths (halving, down
        # to 2): near the end of a call the host replays the longest one that
        # the remaining time still fills, so that few steps run inactive
        # (an inactive step still copies the state through)
        self.sizes = replay_lengths(self.chunk)
        self.graphs = {}
        self.dt_hint = 0.0  # mean step of the calls so far (sizes a call's first replay)

    def _clock_tick(self, state):
        rc = nat.lib().swe_clock_f32(
            nat.ptr(self.clock), nat.ptr(self.red), nat.ptr(self.series_t), nat.ptr(self.series_w),
            self.nseries, nat.ptr(self.lv), nat.ptr(state), self.ny, self.nx, nat.ptr(self.cells),
            self.ncells, nat.ptr(self.gbuf), self.chunk if self.ncells else 0,
            nat.stream_handle(self.dev))
        nat.check(rc, "forward clock")

    def _step(self, src, dst):
        rc = nat.lib().swe_step_clocked_f32(
            3, nat.ptr(src), nat.ptr(self.bed), self.bed.shape[0], nat.ptr(self.n), self.n.shape[0],
            self.B, self.ny, self.nx, self.params, nat.ptr(self.lv), self.levelB,
            nat.ptr(self.clock), nat.ptr(self.infil), self.imode, self.iB, nat.ptr(self.scratch),
            nat.ptr(self.red), nat.ptr(dst), nat.ptr(self.hmax), nat.stream_handle(self.dev))
        nat.check(rc, "forward step")
        self._clock_tick(dst)

    def run(self, U0, bed, n, lv, series, infil, clock):
        """Yields (state buffer, clock) after each replay until the call ends."""
        self.bufs[0].copy_(U0)
        self.hmax.copy_(U0[:, 0])
        self.bed.copy_(bed)
        self.n.copy_(n)
        if lv is not None:
            self.lv.copy_(lv.reshape(-1))
        if series is not None:
            self.series_t.copy_(series[0])
            self.series_w.copy_(series[1])
        if infil is not None:
            self.infil.copy_(infil)
        self.clock_host.copy_(torch.frombuffer(bytearray(bytes(clock)), dtype=torch.uint8))
        self.clock.copy_(self.clock_host, non_blocking=True)
        self._clock_tick(self.bufs[0])  # sets up the first step
        if not self.graphs:
            from .autotune import sweep_rows, tuned_rows_for_shape
            nat.load_kernels()
            rows = tuned_rows_for_shape(self.B, self.ny, self.nx, self.dev,
                                        arithmetic=self.arithmetic)
            with sweep_rows(rows):
                for n in self.sizes:  # even lengths: the state ends in bufs[0]
                    graph = torch.cuda.CUDAGraph()
                    with torch.cuda.graph(graph):
                        for s in range(n):
                            self._step(self.bufs[s % 2], self.bufs[1 - s % 2])
                    self.graphs[n] = graph
        def size_for(left):
            return replay_length(self.sizes, left)

        n = size_for(clock.duration / self.dt_hint) if self.dt_hint > 0 else self.chunk
        while True:
            self.graphs[n].replay()
            c = nat.SweClock.from_buffer_copy(self.clock.cpu().numpy().tobytes())
            if c.steps > 0 and c.elapsed > 0:
                self.dt_hint = float(c.elapsed) / c.steps
            yield self.bufs[0], c
            if c.state != nat.CLOCK_RUNNING:
                return
            # the steps the remaining time needs at the mean step so far
            n = size_for((c.duration - c.elapsed) / self.dt_hint if self.dt_hint > 0 else float("inf"))
