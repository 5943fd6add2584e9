"""A whole gauge run -- the model advanced through ``n_out`` output intervals,
each with its own boundary level, gauges read after each interval -- as one
autograd node.

The reference's inversion script runs this loop in Python
(``Examples/inverse/Monai_Valley/Monai_Velley_BC_inversion_spline_lr002/
bc_inversion_train.py:332-411``): one ``SWE2D.forward(U, t_end=dt_out,
boundary_level=series[i])`` call per output interval, gauges read from the
state after each call, autograd through everything (optionally
``torch.utils.checkpoint`` per chunk).  Here:

* forward: the device-driven time loop (``swe_run_clock_f32`` between
  clocked steps) captured in a CUDA graph of ``graph_steps`` steps and
  replayed until the clock reports the end; every interval's level is read
  on the device, every step's dt and interval are recorded on the device,
  and the state is copied to a checkpoint every ``checkpoint_every`` steps.
  No host synchronisation inside the run except one clock read per replay.
* backward: segment by segment in reverse, the segment's states and both
  stage tendencies are recomputed from its checkpoint in replay mode (bit
  for bit the forward's), then the hand-written step adjoint runs in
  reverse over the segment with the gauge cotangents injected at the end of
  each interval (it re-evaluates only the predictor).  When the whole
  trajectory fits in device memory (``store_states``, decided by free
  memory by default), the forward pass keeps every step's output state and
  stage tendencies instead (its graphs write two alternating rings, copied
  into the store on a copy stream), and the backward pass copies a
  segment's states into place rather than recomputing them.

Gradients flow to the initial state, the per-interval levels and the
roughness field, as through the reference's loop (dt detached).
"""
from __future__ import annotations

import ctypes
from typing import Optional, Sequence, Tuple

import torch

from . import _native as nat
from .adjoint import AdjointStepper, bed_input

GRAPH_STEPS = 32
CHECKPOINT_EVERY = 128
# Kernels of this library per solver step: forward (stage 1, stage 2, the
# run clock) and adjoint with both stage tendencies kept (cursor set-up,
# predictor, corrector adjoint, stage-2 spatial + predictor adjoint (2),
# stage-1 spatial adjoint (2), cursor finish).
FORWARD_KERNELS_PER_STEP = 3
ADJOINT_KERNELS_PER_STEP = 8


class GaugeRunWorkspace:
    """Device buffers and captured graphs of gauge runs of one model, state
    shape, interval count and gauge set."""

    def __init__(self, model, B: int, ny: int, nx: int, dev, levelB: int, n_out: int,
                 gauges: Sequence[Tuple[int, int]], graph_steps: int = GRAPH_STEPS,
                 checkpoint_every: int = CHECKPOINT_EVERY, record_cap: Optional[int] = None,
                 store_states: Optional[bool] = None):
        if graph_steps < 2 or graph_steps % 2:
            raise ValueError("graph_steps must be even and >= 2")
        if checkpoint_every < graph_steps or checkpoint_every % graph_steps:
            raise ValueError("checkpoint_every must be a multiple of graph_steps")
        self.model = model
        self.B, self.ny, self.nx, self.dev = B, ny, nx, dev
        self.levelB, self.n_out = levelB, n_out
        self.G, self.k = graph_steps, checkpoint_every
        shape = (B, 3, ny, nx)
        self.bufs = [torch.empty(shape, device=dev), torch.empty(shape, device=dev)]
        self.scratch = torch.empty(shape, device=dev)
        self.red = torch.zeros(nat.RED_WORDS, dtype=torch.int32, device=dev)
        probe = torch.empty(shape, device=dev)
        bed, n = model._fields(probe)
        self.bed = torch.empty_like(bed)
        self.n = torch.empty_like(n)
        self.levels = torch.zeros((n_out, levelB), device=dev)
        self.lv = torch.zeros(levelB, device=dev)
        self.ngauge = len(gauges)
        self.gauge_cells = [(int(iy), int(ix)) for iy, ix in gauges]
        for iy, ix in gauges:
            if not (0 <= iy < ny and 0 <= ix < nx):
                raise ValueError(f"gauge cell {(iy, ix)} outside the {ny}x{nx} grid")
        self.cells = torch.tensor([v for g in gauges for v in g] or [0, 0], dtype=torch.int32,
                                  device=dev)
        self.gauge_out = torch.zeros((B, n_out, max(self.ngauge, 1)), device=dev)
        self.record_cap = int(record_cap) if record_cap else max(4096, 64 * n_out)
        self.step_dt = torch.zeros(self.record_cap, device=dev)
        self.step_code = torch.zeros(self.record_cap, dtype=torch.int32, device=dev)
        self.clock = torch.zeros(ctypes.sizeof(nat.SweRunClock), dtype=torch.uint8, device=dev)
        self.params = model._params()
        self.ckpts = []
        self.seg = None
        self.fwd_graph = None
        self.replay_graph = None
        self.last_steps = 0
        self.generation = 0
        self.kernel_launches = 0  # kernels of this library enqueued or replayed so far
        self.stepper = None
        # full-trajectory storage (None: when free device memory allows)
        self.store_mode = store_states
        self.rings = None  # two (state, k1, k2) rings of graph_steps items, used alternately
        self.copy_stream = None
        self.ring_done = self.ring_free = None
        self.fwd_store_graphs = None
        self.store, self.store_k1, self.store_k2 = [], [], []
        self.stored = False
        from .autotune import tuned_rows_for_shape
        self.rows = tuned_rows_for_shape(B, ny, nx, dev, arithmetic=model.arithmetic)

    # ------------------------------------------------------------ launches
    def _tick(self, state):
        rc = nat.lib().swe_run_clock_f32(
            nat.ptr(self.clock), nat.ptr(self.red), nat.ptr(self.levels), self.levelB,
            nat.ptr(self.lv), nat.ptr(state), nat.ptr(self.bed), self.bed.shape[0], self.B, self.ny,
            self.nx, nat.ptr(self.cells), self.ngauge, nat.ptr(self.gauge_out), nat.ptr(self.step_dt),
            nat.ptr(self.step_code), nat.stream_handle(self.dev))
        nat.check(rc, "gauge-run clock")

    def _step(self, src, dst, k1=None, k2=None):
        """One clocked step src -> dst; its stage-1 tendency goes to k1 (the
        shared scratch if None), its stage-2 tendency to k2 (if given) and
        the clock advances."""
        k1 = self.scratch if k1 is None else k1
        args = (3, nat.ptr(src), nat.ptr(self.bed), self.bed.shape[0], nat.ptr(self.n), self.n.shape[0],
                self.B, self.ny, self.nx, self.params, nat.ptr(self.lv), self.levelB,
                nat.ptr(self.clock), None, nat.FORCING_NONE, 1, nat.ptr(k1), nat.ptr(self.red),
                nat.ptr(dst), None)
        if k2 is None:
            rc = nat.lib().swe_step_clocked_f32(*args, nat.stream_handle(self.dev))
        else:
            rc = nat.lib().swe_step_clocked_k2_f32(*args, nat.ptr(k2), nat.stream_handle(self.dev))
        nat.check(rc, "gauge-run step")
        self._tick(dst)

    def _set_clock(self, **fields):
        c = nat.SweRunClock()
        c.base.duration = self.out_dt
        c.base.tolerance = max(1e-12, 1e-12 * abs(self.out_dt))
        c.base.max_dt_cap = self.max_dt_cap
        c.base.max_steps = self.max_steps
        c.out_dt = self.out_dt
        c.n_out = self.n_out
        c.record_cap = self.record_cap
        for k, v in fields.items():
            if k in ("steps", "active"):
                setattr(c.base, k, v)
            else:
                setattr(c, k, v)
        self.clock.copy_(torch.frombuffer(bytearray(bytes(c)), dtype=torch.uint8))

    def _read_clock(self) -> nat.SweRunClock:
        return nat.SweRunClock.from_buffer_copy(self.clock.cpu().numpy().tobytes())

    # ------------------------------------------------------------- forward
    def run(self, U0, levels, out_dt: float, max_dt_cap=None, max_steps: int = 1_000_000):
        """Forward gauge run; returns (gauges [B, n_out, ngauge], final state).
        Both are views of workspace buffers (valid until the next run)."""
        bed, n = self.model._fields(U0)
        self.bed.copy_(bed)
        self.n.copy_(n)
        self.levels.copy_(levels)
        self.out_dt = float(out_dt)
        self.max_dt_cap = float(max_dt_cap) if max_dt_cap is not None else 0.0
        self.max_steps = int(max_steps)
        self.generation += 1
        self.bufs[0].copy_(U0)
        self.gauge_out.zero_()
        self._set_clock()
        self._tick(self.bufs[0])
        self.kernel_launches += 1
        if self.fwd_graph is None:
            from .autotune import sweep_rows
            nat.load_kernels()
            g = torch.cuda.CUDAGraph()
            with sweep_rows(self.rows), torch.cuda.graph(g):
                for s in range(self.G):
                    self._step(self.bufs[s % 2], self.bufs[1 - s % 2])
            self.fwd_graph = g
        storing = self.store_mode is not False
        if storing and self.fwd_store_graphs is None:
            # two rings: replay r writes ring r % 2 while the copy stream moves
            # ring (r - 1) % 2 into the store
            from .autotune import sweep_rows
            shape = (self.G,) + tuple(self.bufs[0].shape)
            self.rings = [tuple(torch.empty(shape, device=self.dev) for _ in range(3)) for _ in range(2)]
            self.copy_stream = torch.cuda.Stream(self.dev)
            self.ring_done = [torch.cuda.Event() for _ in range(2)]
            self.ring_free = [torch.cuda.Event() for _ in range(2)]
            graphs = []
            for st, k1, k2 in self.rings:
                g = torch.cuda.CUDAGraph()
                with sweep_rows(self.rows), torch.cuda.graph(g):
                    for s in range(self.G):
                        self._step(self.bufs[0] if s == 0 else st[s - 1], st[s], k1[s], k2[s])
                    self.bufs[0].copy_(st[self.G - 1])
                graphs.append(g)
            self.fwd_store_graphs = graphs
        cur = torch.cuda.current_stream(self.dev)
        per_ckpt = self.k // self.G
        replay = 0
        while True:
            if replay % per_ckpt == 0:
                j = replay // per_ckpt
                if j == len(self.ckpts):
                    self.ckpts.append(torch.empty_like(self.bufs[0]))
                self.ckpts[j].copy_(self.bufs[0])
            if storing:
                i = replay % 2
                if replay >= 2:
                    cur.wait_event(self.ring_free[i])  # its previous contents are in the store
                self.fwd_store_graphs[i].replay()
                self.ring_done[i].record(cur)
                storing = self._keep_replay(replay, i)
            else:
                self.fwd_graph.replay()
            self.kernel_launches += self.G * FORWARD_KERNELS_PER_STEP
            replay += 1
            c = self._read_clock()
            if c.base.state != nat.CLOCK_RUNNING:
                break
        if self.copy_stream is not None:
            cur.wait_stream(self.copy_stream)  # the store is complete before the backward pass
        self.stored = storing
        if c.base.state == nat.CLOCK_FAILED:
            self.model._raise_on_status(int(c.base.dt_status), float(c.base.last_dt))
        if c.base.state == nat.CLOCK_MAXSTEPS:
            raise RuntimeError(f"Reached max_steps={self.max_steps} before an output interval of "
                               f"{self.out_dt} s was complete.")
        if c.base.state == nat.CLOCK_RECORD_FULL:
            raise _RecordFull(int(c.base.steps))
        self.last_steps = int(c.base.steps)
        return self.gauge_out[..., : self.ngauge], self.bufs[0]

    # ------------------------------------------------------------ backward
    def _keep_replay(self, r: int, i: int) -> bool:
        """Copy replay r's step outputs and stage tendencies (ring i) into
        the store on the copy stream; False (stop storing) when the store
        would leave too little device memory or storage is switched off."""
        ring = self.rings[i]
        if r == len(self.store):
            need = 3 * ring[0].numel() * 4
            if self.store_mode is None:
                free, total = torch.cuda.mem_get_info(self.dev)
                if free - need < max(8 << 30, int(0.15 * total)):
                    return False
            self.store.append(torch.empty_like(ring[0]))
            self.store_k1.append(torch.empty_like(ring[1]))
            self.store_k2.append(torch.empty_like(ring[2]))
        cs = self.copy_stream
        cs.wait_event(self.ring_done[i])
        with torch.cuda.stream(cs):
            for dst, src in zip((self.store[r], self.store_k1[r], self.store_k2[r]), ring):
                dst.copy_(src)
                dst.record_stream(cs)
            self.ring_free[i].record(cs)
        return True

    def _copy_steps(self, dst, d0: int, chunks, s0: int, n: int):
        """dst[d0 : d0+n] = step items s0 .. s0+n-1 of a store kept in chunks
        of graph_steps items."""
        while n > 0:
            c, o = divmod(s0, self.G)
            m = min(n, self.G - o)
            dst[d0:d0 + m].copy_(chunks[c][o:o + m])
            d0, s0, n = d0 + m, s0 + m, n - m

    def _stored_segment(self, j: int, s0: int, s1: int):
        """The segment's states and stage tendencies copied from the store."""
        self._alloc_segment()
        n = s1 - s0
        self.seg[0].copy_(self.ckpts[j])
        if n > 1:
            self._copy_steps(self.seg, 1, self.store, s0, n - 1)  # outputs of s0 .. s1-2
        self._copy_steps(self.seg_k1, 0, self.store_k1, s0, n)
        self._copy_steps(self.seg_k2, 0, self.store_k2, s0, n)

    def _alloc_segment(self):
        if self.seg is None:
            shape = tuple(self.bufs[0].shape)
            self.seg = torch.empty((self.k + 1,) + shape, device=self.dev)
            self.seg_k1 = torch.empty((self.k,) + shape, device=self.dev)
            self.seg_k2 = torch.empty((self.k,) + shape, device=self.dev)

    def _recompute_segment(self, j: int, s0: int, s1: int):
        """States entering steps s0 .. s1-1 into self.seg[0 .. s1-s0-1] and
        their stage tendencies into self.seg_k1 / self.seg_k2 (the adjoint
        reuses them: the same kernels on the same state and level give the
        same bits)."""
        self._alloc_segment()
        self.seg[0].copy_(self.ckpts[j])
        self._set_clock(replay=1, replay_end=s1, steps=s0, active=0)
        self._tick(self.seg[0])
        self.kernel_launches += 1 + self.k * FORWARD_KERNELS_PER_STEP
        if self.replay_graph is None:
            from .autotune import sweep_rows
            g = torch.cuda.CUDAGraph()
            with sweep_rows(self.rows), torch.cuda.graph(g):
                for i in range(self.k):
                    self._step(self.seg[i], self.seg[i + 1], self.seg_k1[i], self.seg_k2[i])
            self.replay_graph = g
        self.replay_graph.replay()

    def _alloc_backward(self, bed_grad: bool):
        dev, shape = self.dev, self.bufs[0].shape
        self.stepper = AdjointStepper(self.model, self.B, self.ny, self.nx, dev, self.levelB,
                                      bed_grad=bed_grad)
        self.lam = [torch.empty(shape, device=dev), torch.empty(shape, device=dev)]
        self.g_gauge = torch.zeros_like(self.gauge_out)
        self.g_levels = torch.zeros_like(self.levels)
        self.lam_n = torch.zeros_like(self.n) if self.stepper.fric else None
        self.cursor = torch.zeros(1, dtype=torch.int32, device=dev)
        self.dt_cur = torch.zeros(1, device=dev)
        self.lv_cur = torch.zeros(self.levelB, device=dev)
        self.adj_graph = None

    def _adjoint_steps(self, count):
        """Enqueue the adjoint of the steps in seg slots count-1 .. 0, the
        step index taken from the device cursor (decremented per step); lam
        alternates lam[0] -> lam[1] -> ..., starting from lam[0]."""
        lib, st, stp = nat.lib(), nat.stream_handle(self.dev), self.stepper
        for q, i in enumerate(range(count - 1, -1, -1)):
            lam_in, lam_out = self.lam[q % 2], self.lam[1 - q % 2]
            rc = lib.swe_gauge_adjoint_prep_f32(
                nat.ptr(self.cursor), nat.ptr(self.step_dt), nat.ptr(self.step_code),
                nat.ptr(self.levels), self.levelB, nat.ptr(self.dt_cur), nat.ptr(self.lv_cur),
                nat.ptr(lam_in), self.B, self.ny, self.nx, nat.ptr(self.cells), self.ngauge,
                nat.ptr(self.g_gauge), self.n_out, self.record_cap, st)
            nat.check(rc, "gauge-run adjoint setup")
            part = stp(self.seg[i], self.lv_cur, self.dt_cur, lam_in, lam_out, self.lam_n,
                       K1=self.seg_k1[i], K2=self.seg_k2[i], overwrite=True)
            rc = lib.swe_gauge_adjoint_post_f32(
                nat.ptr(self.cursor), nat.ptr(self.step_code), nat.ptr(part), 2, self.B,
                stp.level_blocks, self.levelB, nat.ptr(self.g_levels), self.record_cap, st)
            nat.check(rc, "gauge-run adjoint finish")

    def backward(self, g_gauges, g_final, bed_grad: bool = False):
        """Adjoints of U0, the levels [n_out, levelB], the roughness field and
        (bed_grad) the bed for the cotangents of the gauges [B, n_out, ngauge]
        and of the final state (either may be None).  The last segment's
        adjoint steps are enqueued directly; every full segment replays one
        captured graph of checkpoint_every adjoint steps.  No host
        synchronisation."""
        total = self.last_steps
        if self.stepper is None or self.stepper.bed_grad != bool(bed_grad):
            self._alloc_backward(bool(bed_grad))
        if self.stepper.bed_grad:
            self.stepper.lam_bed.zero_()
        if g_final is None:
            self.lam[0].zero_()
        else:
            self.lam[0].copy_(g_final)
        if g_gauges is None:
            self.g_gauge.zero_()
        else:
            self.g_gauge[..., : self.ngauge].copy_(g_gauges)
        self.g_levels.zero_()
        if self.lam_n is not None:
            self.lam_n.zero_()
        nseg = (total + self.k - 1) // self.k
        from .autotune import sweep_rows
        with sweep_rows(self.rows):
            self._backward_segments(nseg, total)
        lam_n = self.lam_n.clone() if self.lam_n is not None else None
        lam_bed = self.stepper.bed_adjoint().clone() if self.stepper.bed_grad else None
        return self.lam[0].clone(), self.g_levels.clone(), lam_n, lam_bed

    def _backward_segments(self, nseg, total):
        for j in range(nseg - 1, -1, -1):
            s0, s1 = j * self.k, min((j + 1) * self.k, total)
            if self.stored:
                self._stored_segment(j, s0, s1)
            else:
                self._recompute_segment(j, s0, s1)
            self.cursor.fill_(s1 - 1)
            count = s1 - s0
            self.kernel_launches += count * ADJOINT_KERNELS_PER_STEP
            if count < self.k:
                self._adjoint_steps(count)
                if count % 2:
                    self.lam[0].copy_(self.lam[1])
                continue
            if self.adj_graph is None:
                g = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g):
                    self._adjoint_steps(self.k)
                self.adj_graph = g
                self.cursor.fill_(s1 - 1)  # the capture ran nothing; keep the cursor explicit
            self.adj_graph.replay()


class _RecordFull(RuntimeError):
    def __init__(self, steps):
        super().__init__(f"gauge run needs more than {steps} recorded steps")
        self.steps = steps


class _GaugeRunFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, U0, levels, n, bed, ws, out_dt, max_dt_cap, max_steps):
        lv = levels.detach().t() if levels.ndim == 2 else levels.detach().reshape(-1, 1)
        gauges, final = ws.run(U0.detach(), lv, out_dt, max_dt_cap, max_steps)
        ctx.ws, ctx.generation = ws, ws.generation
        ctx.levels_shape = levels.shape
        ctx.bed_shape = None if bed is None else bed.shape
        return gauges.clone(), final.clone()

    @staticmethod
    def backward(ctx, g_gauges, g_final):
        ws = ctx.ws
        if ws.generation != ctx.generation:
            raise RuntimeError("the gauge-run workspace ran again before this run's backward pass; "
                               "call backward before the next gauge_run of the same shape")
        need_bed = ctx.bed_shape is not None and ctx.needs_input_grad[3]
        lam, g_levels, lam_n, lam_bed = ws.backward(g_gauges, g_final, need_bed)
        g_lv = None
        if ctx.needs_input_grad[1]:
            g_lv = (g_levels.t() if len(ctx.levels_shape) == 2 else g_levels).reshape(ctx.levels_shape)
        g_n = lam_n if (ctx.needs_input_grad[2] and lam_n is not None) else None
        g_bed = None
        if need_bed:
            # eta = h + bed at the gauges: the bed term's adjoint (summed over intervals)
            if g_gauges is not None and ws.ngauge:
                per = g_gauges.sum(dim=1)  # [B, ngauge]
                if lam_bed.shape[0] == 1:
                    per = per.sum(dim=0, keepdim=True)
                for q, (iy, ix) in enumerate(ws.gauge_cells):
                    lam_bed[:, 0, iy, ix] += per[:, q]
            g_bed = lam_bed.reshape(ctx.bed_shape)
        return lam if ctx.needs_input_grad[0] else None, g_lv, g_n, g_bed, None, None, None, None


_WORKSPACES = {}


def gauge_run(model, U0: torch.Tensor, levels: torch.Tensor, out_dt: float,
              gauges: Sequence[Tuple[int, int]], max_dt_cap=None, max_steps: int = 1_000_000,
              graph_steps: int = GRAPH_STEPS, checkpoint_every: Optional[int] = CHECKPOINT_EVERY,
              store_states: Optional[bool] = None):
    """Advance ``U0`` through ``n_out`` output intervals of ``out_dt``
    seconds; interval i runs exactly like ``model(U, t_end=out_dt,
    boundary_level=level_i)``, with level_i = ``levels[:, i]`` for levels
    [B, n_out] (one series per batch member) or ``levels[i]`` for [n_out].

    Returns ``(gauges, U_final)``: eta = h + bed at the gauge cells (row,
    column) after every interval, [B, n_out, len(gauges)], and the final
    state.  Differentiable with respect to U0, levels, the roughness field
    and (when the DEM correction requires grad) the bed.

    ``checkpoint_every=None`` takes the interval from the autotuner
    (``autotune.tuned_checkpoint_every``: timed on this run's shape the first
    time, then cached)."""
    if checkpoint_every is None:
        from .autotune import tuned_checkpoint_every
        checkpoint_every = tuned_checkpoint_every(model, U0, levels, out_dt, gauges,
                                                  max_dt_cap=max_dt_cap, store_states=store_states)
    model._check_state(U0)
    U0 = nat.require_cuda_f32("U0", U0)
    B, _, ny, nx = U0.shape
    if levels.ndim == 2:
        if levels.shape[0] != B:
            raise ValueError(f"levels [B, n_out] must have B={B} rows, got {tuple(levels.shape)}")
        levelB, n_out = B, levels.shape[1]
    elif levels.ndim == 1:
        levelB, n_out = 1, levels.shape[0]
    else:
        raise ValueError("levels must be [n_out] or [B, n_out]")
    if n_out < 1:
        raise ValueError("need at least one output interval")
    if not out_dt > 0:
        raise ValueError("out_dt must be positive")
    key = (id(model), B, ny, nx, str(U0.device), levelB, n_out, tuple(map(tuple, gauges)),
           graph_steps, checkpoint_every, store_states)
    ws = _WORKSPACES.get(key)
    if ws is None or ws.model is not model:
        ws = GaugeRunWorkspace(model, B, ny, nx, U0.device, levelB, n_out, gauges, graph_steps,
                               checkpoint_every, store_states=store_states)
        _WORKSPACES.clear()
        _WORKSPACES[key] = ws
    levels_f = levels.to(dtype=torch.float32)
    while True:
        try:
            return _GaugeRunFunction.apply(U0, levels_f, model.roughness_length, bed_input(model), ws,
                                           float(out_dt), max_dt_cap, int(max_steps))
        except _RecordFull as e:
            ws = GaugeRunWorkspace(model, B, ny, nx, U0.device, levelB, n_out, gauges, graph_steps,
                                   checkpoint_every, record_cap=4 * e.steps,
                                   store_states=store_states)
            _WORKSPACES.clear()
            _WORKSPACES[key] = ws


__all__ = ["gauge_run", "GaugeRunWorkspace", "GRAPH_STEPS", "CHECKPOINT_EVERY"]
