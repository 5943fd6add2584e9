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

Gradients flow to the state, the boundary level, the roughness field and,
when ``dem_correction_parameter`` requires grad, the bed (``model.bed`` is an
autograd input, so the gradient reaches the correction parameter through
the reference's ``tanh`` bound and valid mask, ``src/solver.py:134-147``).
"""
from __future__ import annotations

import torch

from . import _native as nat

def level_blocks(ny: int, nx: int) -> int:
    """Blocks per batch member of the spatial adjoint's gather launch (one
    cell per thread of 256, at most 1024 blocks): each writes one partial
    sum of the level adjoint, summed in a fixed order afterwards."""
    return max(1, min(1024, -(-ny * nx // 256)))


def bed_input(model):
    """``model.bed`` as an autograd input when the DEM correction requires
    grad (and autograd is on), else None."""
    if torch.is_grad_enabled() and model.dem_correction_parameter.requires_grad:
        return model.bed
    return None


class AdjointStepper:
    """The step adjoint's kernels for one model, state shape and level form,
    with their scratch buffers allocated once (a run's backward pass calls
    it once per step)."""

    def __init__(self, model, B, ny, nx, dev, levelB, infiltration=None, bed_grad=False):
        shape = (B, 3, ny, nx)
        self.model = model
        self.B, self.ny, self.nx, self.levelB = B, ny, nx, levelB
        self.bed_grad = bool(bed_grad)
        rec = 16 if self.bed_grad else 12  # floats per face record
        self.K1, self.K2, self.P = (torch.empty(shape, device=dev) for _ in range(3))
        self.lam_k = torch.empty(shape, device=dev)
        self.red = torch.empty(nat.RED_WORDS, dtype=torch.int32, device=dev)
        self.cx = torch.empty(B * ny * (nx + 1) * rec, device=dev)
        self.cy = torch.empty(B * (ny + 1) * nx * rec, device=dev)
        # bed adjoint per batch member, accumulated over the steps of a pass
        self.lam_bed = torch.zeros((B, ny, nx), device=dev) if self.bed_grad else None
        self.level_blocks = level_blocks(ny, nx)
        self.part = torch.empty((2, B * self.level_blocks), device=dev)
        probe = torch.empty((B, 1, ny, nx), device=dev)
        self.bed, self.n = model._fields(probe.expand(B, 3, ny, nx))
        self.infil, self.imode, self.iB = model._forcing_arg(infiltration, probe)
        self.p = model._params()
        self.fric = bool(model.cfg.apply_friction)
        self.lib, self.dev = nat.lib(), dev
        self.key = (B, ny, nx, str(dev), levelB, self.bed_grad)

    @property
    def st(self):
        # the current stream at each call, so launches inside a CUDA-graph
        # capture land in the graph
        return nat.stream_handle(self.dev)

    def _tendency(self, S, lv, out):
        rc = self.lib.swe_spatial_operator_f32(
            nat.ptr(S), nat.ptr(self.bed), self.B, self.bed.shape[0], self.ny, self.nx, self.p,
            nat.ptr(lv), self.levelB, None, nat.FORCING_NONE, 1, nat.ptr(self.infil), self.imode,
            self.iB, nat.ptr(out), nat.ptr(self.red), self.st)
        nat.check(rc, "adjoint recompute")

    def _spatial(self, S, lv, lam_rhs, lam_S, part, what):
        args = (nat.ptr(S), nat.ptr(self.bed), self.bed.shape[0], self.B, self.ny, self.nx, self.p,
                nat.ptr(lv), self.levelB, nat.ptr(lam_rhs), nat.ptr(self.cx), nat.ptr(self.cy),
                nat.ptr(lam_S), nat.ptr(part), self.level_blocks)
        if self.bed_grad:
            rc = self.lib.swe_adj_spatial_bed_f32(*args, nat.ptr(self.lam_bed), self.st)
        else:
            rc = self.lib.swe_adj_spatial_f32(*args, self.st)
        nat.check(rc, what)

    def _stage2(self, P, U, K1, lv, dt, lam_U):
        """Spatial adjoint at the predictor P (lam_rhs = self.lam_k, the
        adjoint of k2) and the predictor's adjoint in one call: lam_U += ...,
        self.lam_k = adjoint of k1 (written after the last read of k2's)."""
        dev_dt = torch.is_tensor(dt)
        rc = self.lib.swe_adj_stage2_f32(
            nat.ptr(P), nat.ptr(U), nat.ptr(K1), nat.ptr(self.bed), self.bed.shape[0], self.B, self.ny,
            self.nx, self.p, nat.ptr(lv), self.levelB, nat.ptr(self.lam_k), nat.ptr(self.cx),
            nat.ptr(self.cy), 0.0 if dev_dt else float(dt), nat.ptr(dt) if dev_dt else None,
            nat.ptr(lam_U), nat.ptr(self.lam_k), nat.ptr(self.part[0]), self.level_blocks,
            nat.ptr(self.lam_bed) if self.bed_grad else None, self.st)
        nat.check(rc, "adjoint spatial operator and predictor (stage 2)")

    def bed_adjoint(self):
        """The accumulated bed adjoint in the bed's batch form
        [bedB, 1, ny, nx] (summed over the batch for a shared bed)."""
        lb = self.lam_bed
        if self.bed.shape[0] == 1:
            lb = lb.sum(0, keepdim=True)
        return lb.unsqueeze(1)

    def _pointwise(self, mode, U, k, dt, lam_out, lam_U, lam_n, P_out):
        n = self.n
        corrector = mode in (0, 3)
        nptr = nat.ptr(n) if corrector else None
        lnptr = nat.ptr(lam_n) if (corrector and self.fric) else None
        if torch.is_tensor(dt):  # device time step (graph-captured backward passes)
            rc = self.lib.swe_adj_pointwise_dev_f32(
                mode, nat.ptr(U), nat.ptr(k), nptr, n.shape[0], self.B, self.ny, self.nx, self.p,
                nat.ptr(dt), nat.ptr(lam_out), nat.ptr(lam_U), nat.ptr(self.lam_k), lnptr,
                nat.ptr(P_out), self.st)
        else:
            rc = self.lib.swe_adj_pointwise_f32(
                mode, nat.ptr(U), nat.ptr(k), nptr, n.shape[0], self.B, self.ny, self.nx, self.p,
                float(dt), nat.ptr(lam_out), nat.ptr(lam_U), nat.ptr(self.lam_k), lnptr,
                nat.ptr(P_out), self.st)
        nat.check(rc, ("adjoint corrector", "adjoint predictor", "adjoint predictor",
                       "adjoint corrector")[mode])

    def __call__(self, U, lv, dt, lam_out, lam_U, lam_n, K1=None, overwrite=False, K2=None):
        """lam_U += (d U_new / d U)^T lam_out and lam_n += the roughness
        adjoint (when friction is on) for the step at input state U with
        level vector lv and time step dt (a float, or a one-element device
        tensor); returns the level adjoint's partial sums
        [2, B * level_blocks] (their sum per batch member is that member's
        level adjoint).  K1, if given, is the step's stage-1 tendency kept
        from the forward recompute (else it is recomputed here); K2 likewise
        the step's stage-2 tendency.  With overwrite, lam_U's previous
        contents are ignored (lam_U = ... rather than +=)."""
        P, lam_k = self.P, self.lam_k
        # recompute the step's stage intermediates (solver.py:613-646)
        if K1 is None:
            K1 = self.K1
            self._tendency(U, lv, K1)
        self._pointwise(2, U, K1, dt, None, None, None, P)
        if K2 is None:
            K2 = self.K2
            self._tendency(P, lv, K2)
        # corrector + friction: lam_k = adjoint of k2
        self._pointwise(3 if overwrite else 0, U, K2, dt, lam_out, lam_U, lam_n, None)
        # spatial operator at the predictor, then the predictor: lam_k = adjoint of k1
        self._stage2(P, U, K1, lv, dt, lam_U)
        # spatial operator at the input state
        self._spatial(U, lv, lam_k, lam_U, self.part[1], "adjoint spatial operator (stage 1)")
        return self.part

    def level_adjoint(self, part):
        """Level adjoint [levelB] from the partial sums of one step."""
        lam = part.view(2, self.B, self.level_blocks).sum(dim=(0, 2))
        return lam.sum(0, keepdim=True) if self.levelB == 1 else lam


def adjoint_step(model, U, level, n, dt, lam_out, infiltration=None, ws=None, lam_U=None,
                 lam_n=None, bed_grad=False):
    """VJP of one step at input state ``U`` with time step ``dt``.

    Returns ``(lam_U, lam_level, lam_n, lam_bed)``: adjoints of the state
    [B,3,ny,nx], the level vector (1 or B values), the roughness field (same
    shape as ``n``; None when friction is off) and, with ``bed_grad``, the
    bed ([bedB,1,ny,nx]; else None).  ``ws`` is an optional AdjointStepper
    built for the same model and shapes; ``lam_U`` / ``lam_n`` optional
    zeroed outputs that the step accumulates into.
    """
    U = nat.require_cuda_f32("U", U.detach())
    lam_out = nat.require_cuda_f32("lam_out", lam_out)
    B, _, ny, nx = U.shape
    dev = U.device
    lv, levelB = model._level_arg(level.detach(), B)
    if ws is None or ws.key != (B, ny, nx, str(dev), levelB, bool(bed_grad)):
        ws = AdjointStepper(model, B, ny, nx, dev, levelB, infiltration, bed_grad)
    lam_U = torch.zeros_like(U) if lam_U is None else lam_U
    if ws.fric and lam_n is None:
        lam_n = torch.zeros_like(ws.n)
    if ws.bed_grad:
        ws.lam_bed.zero_()
    part = ws(U, lv, dt, lam_out, lam_U, lam_n)
    lam_bed = ws.bed_adjoint() if ws.bed_grad else None
    return lam_U, ws.level_adjoint(part), (lam_n if ws.fric else None), lam_bed


class _StepFunction(torch.autograd.Function):
    """One SWE2D.step as an autograd node (inputs: state, level vector,
    roughness, bed or None)."""

    @staticmethod
    def forward(ctx, U, level_vec, n, bed, model, max_dt_f, infiltration, dt_out):
        U_new, status, dt = model._launch_step(U.detach(), level_vec.detach(), max_dt_f, infiltration)
        model._raise_on_status(status, dt)
        dt_out.append(dt)
        ctx.model, ctx.dt, ctx.infiltration = model, dt, infiltration
        ctx.bed_shape = None if bed is None else bed.shape
        ctx.save_for_backward(U, level_vec, n)
        return U_new

    @staticmethod
    def backward(ctx, gU):
        U, level_vec, n = ctx.saved_tensors
        need_bed = ctx.bed_shape is not None and ctx.needs_input_grad[3]
        lam_U, lam_level, lam_n, lam_bed = adjoint_step(ctx.model, U, level_vec, n, ctx.dt,
                                                        gU.contiguous(), ctx.infiltration,
                                                        bed_grad=need_bed)
        g_level = lam_level.reshape(level_vec.shape) if ctx.needs_input_grad[1] else None
        g_n = lam_n.reshape(n.shape) if (ctx.needs_input_grad[2] and lam_n is not None) else None
        g_bed = lam_bed.reshape(ctx.bed_shape) if need_bed else None
        return lam_U, g_level, g_n, g_bed, None, None, None, None


def step_with_adjoint(model, U, model_time, max_dt, infiltration=None, boundary_level=None):
    """SWE2D.step under autograd: returns (U_new, dt_float) like the reference."""
    max_dt_f = float((max_dt.to(dtype=torch.float32) if torch.is_tensor(max_dt)
                      else torch.tensor(float(max_dt), dtype=torch.float32)).item())
    level = model._prepare_boundary_level(
        model.cfg.constant_level if boundary_level is None else boundary_level, U)
    level_vec = level.reshape(-1) if level.ndim > 0 else level.reshape(1)
    dt_out = []
    U_new = _StepFunction.apply(U, level_vec, model.roughness_length, bed_input(model), model,
                                max_dt_f, infiltration, dt_out)
    return U_new, dt_out[0]


class _ChunkFunction(torch.autograd.Function):
    """A whole forward() call (explicit boundary level) as one autograd node
    (inputs: initial state, level vector, roughness, bed or None)."""

    @staticmethod
    def forward(ctx, U0, level_vec, n, bed, model, t_end, start_time, max_dt_cap, max_steps,
                steps_out):
        with torch.no_grad():
            U, _ = model.forward(U0.detach(), t_end=t_end, start_time=start_time,
                                 boundary_level=level_vec.detach(), max_dt_cap=max_dt_cap,
                                 max_steps=max_steps)
        steps = getattr(model, "last_forward_steps", None)
        steps_out.append(steps)
        ctx.model, ctx.t_end, ctx.max_dt_cap, ctx.max_steps = model, t_end, max_dt_cap, max_steps
        ctx.start_time, ctx.steps = start_time, steps
        ctx.bed_shape = None if bed is None else bed.shape
        ctx.save_for_backward(U0, level_vec, n)
        return U

    @staticmethod
    def backward(ctx, gU):
        U0, level_vec, n = ctx.saved_tensors
        model = ctx.model
        need_bed = ctx.bed_shape is not None and ctx.needs_input_grad[3]
        states, dts = _recompute_chunk(model, U0.detach(), level_vec.detach(), float(ctx.t_end),
                                       float(ctx.start_time), ctx.max_dt_cap, ctx.steps)
        lam = gU.contiguous()
        lam_level = torch.zeros_like(level_vec)
        lam_n = torch.zeros_like(n) if model.cfg.apply_friction else None
        B, _, ny, nx = U0.shape
        ws = AdjointStepper(model, B, ny, nx, U0.device, model._level_arg(level_vec, B)[1],
                            bed_grad=need_bed)
        lv = model._level_arg(level_vec.detach(), B)[0]
        for U_s, dt_s in zip(reversed(states), reversed(dts)):
            lam_out, lam = lam, torch.zeros_like(lam)
            part = ws(U_s, lv, dt_s, lam_out, lam, lam_n)
            lam_level += ws.level_adjoint(part).reshape(lam_level.shape)
        g_level = lam_level if ctx.needs_input_grad[1] else None
        g_n = lam_n if (ctx.needs_input_grad[2] and lam_n is not None) else None
        g_bed = ws.bed_adjoint().reshape(ctx.bed_shape) if need_bed else None
        return lam, g_level, g_n, g_bed, None, None, None, None, None, None


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
    configured) boundary level, differentiable with respect to U0, the level,
    the roughness field and (when the DEM correction requires grad) the bed;
    only U0 is kept for the backward pass."""
    level = model._prepare_boundary_level(
        model.cfg.constant_level if boundary_level is None else boundary_level, U0)
    level_vec = level.reshape(-1) if level.ndim > 0 else level.reshape(1)
    steps_out = []
    U = _ChunkFunction.apply(U0, level_vec, model.roughness_length, bed_input(model), model,
                             float(t_end), float(start_time), max_dt_cap, int(max_steps), steps_out)
    return U
