"""Hand-written adjoint of the step behind ``torch.autograd``.

The reference differentiates its step with PyTorch autograd (inversions in
``Examples/inverse/**/bc_inversion_train.py``: BPTT through ``SWE2D.forward``,
optionally with ``torch.utils.checkpoint`` per output chunk, ``:332-349``).
Here the vector-Jacobian product of one step is the sm_100a kernels of
``csrc/swe_adjoint.cu`` (same derivative conventions as autograd, dt
detached as in ``src/solver.py:626``), wrapped in two autograd Functions:

* ``step_with_adjoint`` -- ``SWE2D.step`` when its state or boundary level
  requires grad: saves the step's input and recomputes the stage
  intermediates in backward;
* ``forward_checkpointed`` -- a whole ``SWE2D.forward`` call as one node: the
  forward pass runs the device-driven time loop and keeps only the chunk's
  initial state; the backward pass recomputes the chunk's states (its
  checkpoint interval is the chunk) and runs the adjoint steps in reverse.

Gradients flow to the state, the boundary level and the roughness field.
The bed (``dem_correction_parameter``) is not differentiated.
"""
from __future__ import annotations

import torch

from . import _native as nat

LEVEL_BLOCKS = 64


def _check_no_bed_grad(model):
    if torch.is_grad_enabled() and model.dem_correction_parameter.requires_grad:
        raise NotImplementedError(
            "gradients with respect to the bed (dem_correction_parameter) are not provided by "
            "the B200 adjoint; construct the model with train_dem=False")


class AdjointWorkspace:
    """Scratch buffers of adjoint_step for one state shape (reused across steps)."""

    def __init__(self, B, ny, nx, dev):
        shape = (B, 3, ny, nx)
        self.K1, self.K2, self.P = (torch.empty(shape, device=dev) for _ in range(3))
        self.lam_k = torch.empty(shape, device=dev)
        self.lam_P = torch.empty(shape, device=dev)
        self.red = torch.empty(nat.RED_WORDS, dtype=torch.int32, device=dev)
        self.cx = torch.empty(B * ny * (nx + 1) * 12, device=dev)
        self.cy = torch.empty(B * (ny + 1) * nx * 12, device=dev)
        self.part = torch.empty(B * LEVEL_BLOCKS, device=dev)
        self.key = (B, ny, nx, str(dev))


def adjoint_step(model, U, level, n, dt, lam_out, infiltration=None, ws=None, lam_U=None,
                 lam_n=None):
    """VJP of one step at input state ``U`` with time step ``dt``.

    Returns ``(lam_U, lam_level, lam_n)``: adjoints of the state
    [B,3,ny,nx], the level vector (1 or B values) and the roughness field
    (same shape as ``n``; None when friction is off).  ``ws`` is an optional
    AdjointWorkspace; ``lam_U`` / ``lam_n`` optional zeroed outputs that the
    step accumulates into.
    """
    U = nat.require_cuda_f32("U", U.detach())
    lam_out = nat.require_cuda_f32("lam_out", lam_out)
    B, _, ny, nx = U.shape
    dev = U.device
    bed, _ = model._fields(U)
    n = nat.require_cuda_f32("n", n.detach())
    lv, levelB = model._level_arg(level.detach(), B)
    infil, imode, iB = model._forcing_arg(infiltration, U[:, 0:1])
    p = model._params()
    lib, st = nat.lib(), nat.stream_handle(dev)
    if ws is None or ws.key != (B, ny, nx, str(dev)):
        ws = AdjointWorkspace(B, ny, nx, dev)
    K1, K2, P, red = ws.K1, ws.K2, ws.P, ws.red

    def tendency(S, out):
        rc = lib.swe_spatial_operator_f32(nat.ptr(S), nat.ptr(bed), B, bed.shape[0], ny, nx, p,
                                          nat.ptr(lv), levelB, None, nat.FORCING_NONE, 1,
                                          nat.ptr(infil), imode, iB, nat.ptr(out), nat.ptr(red), st)
        nat.check(rc, "adjoint recompute")

    # recompute the step's stage intermediates (solver.py:613-646)
    tendency(U, K1)
    rc = lib.swe_adj_pointwise_f32(2, nat.ptr(U), nat.ptr(K1), None, 1, B, ny, nx, p, float(dt),
                                   None, None, None, None, nat.ptr(P), st)
    nat.check(rc, "adjoint predictor")
    tendency(P, K2)
    lam_U = torch.zeros_like(U) if lam_U is None else lam_U
    lam_k = ws.lam_k
    lam_P = ws.lam_P
    lam_P.zero_()
    fric = bool(model.cfg.apply_friction)
    if fric and lam_n is None:
        lam_n = torch.zeros_like(n)
    cx, cy, part = ws.cx, ws.cy, ws.part
    # corrector + friction
    rc = lib.swe_adj_pointwise_f32(0, nat.ptr(U), nat.ptr(K2), nat.ptr(n), n.shape[0], B, ny, nx, p,
                                   float(dt), nat.ptr(lam_out), nat.ptr(lam_U), nat.ptr(lam_k),
                                   nat.ptr(lam_n), None, st)
    nat.check(rc, "adjoint corrector")
    # spatial operator at the predictor
    rc = lib.swe_adj_spatial_f32(nat.ptr(P), nat.ptr(bed), bed.shape[0], B, ny, nx, p, nat.ptr(lv),
                                 levelB, nat.ptr(lam_k), nat.ptr(cx), nat.ptr(cy), nat.ptr(lam_P),
                                 nat.ptr(part), LEVEL_BLOCKS, st)
    nat.check(rc, "adjoint spatial operator (stage 2)")
    lam_level = part.view(B, LEVEL_BLOCKS).sum(1)
    # predictor
    rc = lib.swe_adj_pointwise_f32(1, nat.ptr(U), nat.ptr(K1), None, 1, B, ny, nx, p, float(dt),
                                   nat.ptr(lam_P), nat.ptr(lam_U), nat.ptr(lam_k), None, None, st)
    nat.check(rc, "adjoint predictor")
    # spatial operator at the input state
    rc = lib.swe_adj_spatial_f32(nat.ptr(U), nat.ptr(bed), bed.shape[0], B, ny, nx, p, nat.ptr(lv),
                                 levelB, nat.ptr(lam_k), nat.ptr(cx), nat.ptr(cy), nat.ptr(lam_U),
                                 nat.ptr(part), LEVEL_BLOCKS, st)
    nat.check(rc, "adjoint spatial operator (stage 1)")
    lam_level = lam_level + part.view(B, LEVEL_BLOCKS).sum(1)
    if levelB == 1:
        lam_level = lam_level.sum(0, keepdim=True)
    return lam_U, lam_level, lam_n


class _StepFunction(torch.autograd.Function):
    """One SWE2D.step as an autograd node (inputs: state, level vector, roughness)."""

    @staticmethod
    def forward(ctx, U, level_vec, n, model, max_dt_f, infiltration, dt_out):
        U_new, status, dt = model._launch_step(U.detach(), level_vec.detach(), max_dt_f, infiltration)
        model._raise_on_status(status, dt)
        dt_out.append(dt)
        ctx.model, ctx.dt, ctx.infiltration = model, dt, infiltration
        ctx.save_for_backward(U, level_vec, n)
        return U_new

    @staticmethod
    def backward(ctx, gU):
        U, level_vec, n = ctx.saved_tensors
        lam_U, lam_level, lam_n = adjoint_step(ctx.model, U, level_vec, n, ctx.dt, gU.contiguous(),
                                               ctx.infiltration)
        g_level = lam_level.reshape(level_vec.shape) if ctx.needs_input_grad[1] else None
        g_n = lam_n.reshape(n.shape) if (ctx.needs_input_grad[2] and lam_n is not None) else None
        return lam_U, g_level, g_n, None, None, None, None


def step_with_adjoint(model, U, model_time, max_dt, infiltration=None, boundary_level=None):
    """SWE2D.step under autograd: returns (U_new, dt_float) like the reference."""
    _check_no_bed_grad(model)
    max_dt_f = float((max_dt.to(dtype=torch.float32) if torch.is_tensor(max_dt)
                      else torch.tensor(float(max_dt), dtype=torch.float32)).item())
    level = model._prepare_boundary_level(
        model.cfg.constant_level if boundary_level is None else boundary_level, U)
    level_vec = level.reshape(-1) if level.ndim > 0 else level.reshape(1)
    dt_out = []
    U_new = _StepFunction.apply(U, level_vec, model.roughness_length, model, max_dt_f, infiltration,
                                dt_out)
    return U_new, dt_out[0]


class _ChunkFunction(torch.autograd.Function):
    """A whole forward() call (explicit boundary level) as one autograd node."""

    @staticmethod
    def forward(ctx, U0, level_vec, n, model, t_end, start_time, max_dt_cap, max_steps, steps_out):
        with torch.no_grad():
            U, _ = model.forward(U0.detach(), t_end=t_end, start_time=start_time,
                                 boundary_level=level_vec.detach(), max_dt_cap=max_dt_cap,
                                 max_steps=max_steps)
        steps = getattr(model, "last_forward_steps", None)
        steps_out.append(steps)
        ctx.model, ctx.t_end, ctx.max_dt_cap, ctx.max_steps = model, t_end, max_dt_cap, max_steps
        ctx.start_time, ctx.steps = start_time, steps
        ctx.save_for_backward(U0, level_vec, n)
        return U

    @staticmethod
    def backward(ctx, gU):
        U0, level_vec, n = ctx.saved_tensors
        model = ctx.model
        states, dts = _recompute_chunk(model, U0.detach(), level_vec.detach(), float(ctx.t_end),
                                       float(ctx.start_time), ctx.max_dt_cap, ctx.steps)
        lam = gU.contiguous()
        lam_level = torch.zeros_like(level_vec)
        lam_n = torch.zeros_like(n) if model.cfg.apply_friction else None
        B, _, ny, nx = U0.shape
        ws = AdjointWorkspace(B, ny, nx, U0.device)
        for U_s, dt_s in zip(reversed(states), reversed(dts)):
            lam, l_lev, lam_n = adjoint_step(model, U_s, level_vec, n, dt_s, lam, ws=ws, lam_n=lam_n)
            lam_level += l_lev.reshape(lam_level.shape)
        g_level = lam_level if ctx.needs_input_grad[1] else None
        g_n = lam_n if (ctx.needs_input_grad[2] and lam_n is not None) else None
        return lam, g_level, g_n, None, None, None, None, None, None


def _recompute_chunk(model, U0, level_vec, duration, start_time, max_dt_cap, steps):
    """States entering each step of one forward() call and their time steps,
    recomputed with the device clock (same kernels and bookkeeping as the
    forward pass, so the same states bit for bit) and one host read."""
    dev = U0.device
    B, _, ny, nx = U0.shape
    bed, n = model._fields(U0)
    lv, levelB = model._level_arg(level_vec, B)
    p = model._params()
    lib, st = nat.lib(), nat.stream_handle(dev)
    cap = float(max_dt_cap) if max_dt_cap is not None else 0.0
    clock_host = nat.SweClock(duration, start_time, max(1e-12, 1e-12 * abs(duration)), cap, 0.0,
                              int(steps), 0, 0, 0, 0, 0.0, 0.0, 0.0)
    clock = torch.frombuffer(bytearray(bytes(clock_host)), dtype=torch.uint8).to(dev)
    red = torch.zeros(nat.RED_WORDS, dtype=torch.int32, device=dev)
    scratch = torch.empty_like(U0)
    rec = torch.zeros((max(int(steps), 1), 2), dtype=torch.float64, device=dev)

    def tick(state):
        rc = lib.swe_clock_f32(nat.ptr(clock), nat.ptr(red), None, None, 0, nat.ptr(lv), nat.ptr(state),
                               ny, nx, None, 0, nat.ptr(rec), int(steps), st)
        nat.check(rc, "recompute clock")

    tick(U0)
    states = [U0]
    for _ in range(int(steps)):
        out = torch.empty_like(U0)
        rc = lib.swe_step_clocked_f32(3, nat.ptr(states[-1]), nat.ptr(bed), bed.shape[0], nat.ptr(n),
                                      n.shape[0], B, ny, nx, p, nat.ptr(lv), levelB, nat.ptr(clock),
                                      None, nat.FORCING_NONE, 1, nat.ptr(scratch), nat.ptr(red),
                                      nat.ptr(out), None, st)
        nat.check(rc, "recompute step")
        tick(out)
        states.append(out)
    c = nat.SweClock.from_buffer_copy(clock.cpu().numpy().tobytes())
    if c.state == nat.CLOCK_FAILED:
        model._raise_on_status(c.dt_status, float(c.last_dt))
    dts = [float(x) for x in rec[:, 1].cpu().tolist()][: c.steps]
    return states[: c.steps], dts


def forward_checkpointed(model, U0, t_end, start_time=0.0, boundary_level=None, max_dt_cap=None,
                         max_steps=1_000_000):
    """``model.forward`` over ``t_end`` seconds with a constant (explicit or
    configured) boundary level, differentiable with respect to U0, the level
    and the roughness field; only U0 is kept for the backward pass."""
    _check_no_bed_grad(model)
    level = model._prepare_boundary_level(
        model.cfg.constant_level if boundary_level is None else boundary_level, U0)
    level_vec = level.reshape(-1) if level.ndim > 0 else level.reshape(1)
    steps_out = []
    U = _ChunkFunction.apply(U0, level_vec, model.roughness_length, model, float(t_end),
                             float(start_time), max_dt_cap, int(max_steps), steps_out)
    return U
