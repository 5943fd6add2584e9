"""Ensembles of independent scenarios in one persistent, CUDA-graph-captured launch.

The reference batches scenarios through its batch dimension, which needs equal
grid sizes and shares one time step across the batch (``src/solver.py:367-376``,
``:527-530``).  ``Ensemble`` runs scenarios of different grid sizes, each with
its own configuration, roughness, boundary series, CFL time step and step
count, in one launch of the persistent kernel of ``csrc/swe_step.cu``
(``swe_ensemble_run_f32``); the launch (with its control-state reset) is
captured in a CUDA graph and replayed.  Each scenario's result is bit for bit
what ``SWE2D.step`` gives for that scenario alone.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import List, Optional, Sequence

import torch

from . import _native as nat
from .config import SWEConfig


@dataclass
class EnsembleResult:
    states: List[torch.Tensor]   # final [1,3,ny,nx] state of each scenario
    steps: List[int]
    times: List[float]           # simulated time advanced
    hmax: Optional[List[torch.Tensor]]
    elapsed_ms: float            # device time of the persistent launch
    cell_updates: int
    failed: List[int]            # scenarios whose time step failed (run(strict=False))
    status: List[int]            # SWE_S_* bits of each scenario (0: no failure)

    @property
    def mcells_per_s(self) -> float:
        return self.cell_updates / (self.elapsed_ms * 1e-3) / 1e6


class Ensemble:
    """Scenarios (``diffswe2d_b200.scenarios.Scenario`` or compatible) on one GPU.

    ``rows`` fixes the sweep tile height of every scenario; by default it is
    the autotuner's ensemble value (``autotune.tuned_ensemble_rows``).
    ``arithmetic`` selects the step kernels ("exact": IEEE operation for
    operation as the reference; "fast": the tolerance mode).  ``stall_ns``
    is the persistent kernel's idle limit (None: the library's 2 s): a launch
    in which no scenario completes a phase for that long stops with an error.
    """

    def __init__(self, scenarios: Sequence, device="cuda", steps: Optional[int] = None,
                 rows: Optional[int] = None, track_hmax: bool = False, max_dt: float = 1.0e9,
                 arithmetic: str = "exact", stall_ns: Optional[int] = None):
        from .autotune import tuned_ensemble_rows
        self.arith = nat.arithmetic_code(arithmetic)
        self.stall_ns = 0 if stall_ns is None else int(stall_ns)
        if self.stall_ns < 0:
            raise ValueError("stall_ns must be positive")
        self.device = torch.device(device)
        self.count = len(scenarios)
        if not 1 <= self.count <= 1024:
            raise ValueError("an ensemble holds 1 to 1024 scenarios")
        self._keep = []  # tensors referenced by the device member table
        members = (nat.SweEnsembleMember * self.count)()
        fric = None
        self.cells = []
        self.steps = []
        self.U_a, self.U_b, self.hmax = [], [], []
        for m, sc in enumerate(scenarios):
            cfg = SWEConfig(**sc.config)
            f = (1 + (0 if cfg.frictionmodel == "manning" else 1)) if cfg.apply_friction else 0
            if fric is None:
                fric = f
            elif f != fric:
                raise ValueError("all scenarios of an ensemble must use the same friction law")
            ny, nx = sc.bed.shape
            dev = self.device
            bed = torch.as_tensor(sc.bed, dtype=torch.float32, device=dev).contiguous()
            n = torch.as_tensor(sc.roughness, dtype=torch.float32, device=dev).contiguous()
            Ua = torch.as_tensor(sc.U0, dtype=torch.float32, device=dev).reshape(3, ny, nx).clone()
            Ub = torch.empty_like(Ua)
            k1 = torch.empty_like(Ua)
            hm = Ua[0].clone() if track_hmax else None
            st = sw = None
            nser = 0
            if sc.bc_times is not None:
                st = torch.as_tensor(sc.bc_times, dtype=torch.float32, device=dev).contiguous()
                sw = torch.as_tensor(sc.bc_levels, dtype=torch.float32, device=dev).contiguous()
                nser = st.numel()
            steps_m = int(sc.steps if steps is None else steps)
            r = int(rows) if rows is not None else tuned_ensemble_rows(dev, arithmetic)
            mem = members[m]
            mem.bed, mem.n = bed.data_ptr(), n.data_ptr()
            mem.U_a, mem.U_b, mem.k1 = Ua.data_ptr(), Ub.data_ptr(), k1.data_ptr()
            mem.hmax = hm.data_ptr() if hm is not None else None
            mem.series_t = st.data_ptr() if st is not None else None
            mem.series_w = sw.data_ptr() if sw is not None else None
            mem.nseries, mem.ny, mem.nx, mem.steps, mem.rows = nser, ny, nx, steps_m, r
            mem.level = float(cfg.constant_level)
            mem.start_time = 0.0
            mem.max_dt = float(max_dt)
            mem.params = nat.params(cfg, sc.dx, sc.dy, arithmetic)
            self._keep += [bed, n, Ua, Ub, k1, hm, st, sw]
            self.U_a.append(Ua)
            self.U_b.append(Ub)
            self.hmax.append(hm)
            self.cells.append(ny * nx)
            self.steps.append(steps_m)
        self.friction = fric
        self.initial = [u.clone() for u in self.U_a]
        lib = nat.lib()
        nbytes = lib.swe_ensemble_workspace_bytes(self.count)
        if nbytes < 0:
            raise ValueError("invalid ensemble size")
        self.workspace = torch.empty(int(nbytes), dtype=torch.uint8, device=self.device)
        self.results_dev = torch.empty(self.count * ctypes.sizeof(nat.SweEnsembleResult),
                                       dtype=torch.uint8, device=self.device)
        self.error_dev = torch.zeros(1, dtype=torch.int32, device=self.device)
        rc = lib.swe_ensemble_prepare_f32(members, self.count, nat.ptr(self.workspace),
                                          nat.stream_handle(self.device))
        nat.check(rc, "ensemble prepare")
        props = torch.cuda.get_device_properties(self.device)
        self.blocks = props.multi_processor_count * 6
        self._graph = None

    def _launch(self):
        lib, st = nat.lib(), nat.stream_handle(self.device)
        nat.check(lib.swe_ensemble_reset_f32(nat.ptr(self.workspace), self.count, st), "ensemble reset")
        nat.check(lib.swe_ensemble_run_f32(nat.ptr(self.workspace), self.count, self.friction,
                                           self.arith, self.blocks, self.stall_ns, st), "ensemble run")

    def run(self, strict: bool = True) -> EnsembleResult:
        """Run every scenario from its initial state; returns final states.

        A scenario whose time step fails (non-finite state or dt) stops on
        its own; the others run to the end.  With ``strict`` the failure
        raises FloatingPointError, otherwise it is listed in ``failed``."""
        for Ua, U0 in zip(self.U_a, self.initial):
            Ua.copy_(U0)
        for hm, U0 in zip(self.hmax, self.initial):
            if hm is not None:
                hm.copy_(U0[0])
        if self._graph is None:
            nat.load_kernels()
            self._graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(self._graph):
                self._launch()
            for Ua, U0 in zip(self.U_a, self.initial):  # capture ran nothing; keep inputs
                Ua.copy_(U0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        self._graph.replay()
        e1.record()
        lib = nat.lib()
        nat.check(lib.swe_ensemble_results_f32(nat.ptr(self.workspace), self.count,
                                               nat.ptr(self.results_dev), nat.ptr(self.error_dev),
                                               nat.stream_handle(self.device)), "ensemble results")
        torch.cuda.synchronize(self.device)
        raw = bytes(self.results_dev.cpu().numpy())
        res = (nat.SweEnsembleResult * self.count).from_buffer_copy(raw)
        if int(self.error_dev.item()) != 0:
            raise RuntimeError("ensemble kernel stopped: idle limit reached")
        states, steps, times, failed, status = [], [], [], [], []
        for m in range(self.count):
            r = res[m]
            if r.finished == 2:
                if strict:
                    raise FloatingPointError(f"scenario {m}: time step failed (status {r.status})")
                failed.append(m)
            status.append(int(r.status))
            buf = self.U_a[m] if r.steps % 2 == 0 else self.U_b[m]
            states.append(buf.clone().unsqueeze(0))
            steps.append(int(r.steps))
            times.append(float(r.time))
        hmax = [h.clone() if h is not None else None for h in self.hmax] if any(
            h is not None for h in self.hmax) else None
        total = sum(c * s for c, s in zip(self.cells, steps))
        return EnsembleResult(states, steps, times, hmax, e0.elapsed_time(e1), total, failed, status)


@dataclass
class GaugeEnsembleResult:
    gauges: torch.Tensor   # [M, n_out, ngauge] eta after each output interval
    states: torch.Tensor   # [M, 3, ny, nx] final states
    steps: List[int]
    times: List[float]
    elapsed_ms: float      # device time of the persistent launch
    cell_updates: int

    @property
    def mcells_per_s(self) -> float:
        return self.cell_updates / (self.elapsed_ms * 1e-3) / 1e6


class GaugeEnsemble:
    """Members of one grid shape in interval mode: member m runs ``n_out``
    output intervals of ``out_dt`` seconds with levels ``out_levels[m]``, each
    interval exactly like ``SWE2D.forward(U, t_end=out_dt,
    boundary_level=level)`` with its own CFL steps, and records eta = h + bed
    at the gauge cells after every interval -- the run of
    ``gauge_run`` for a batch of one, for up to 1024 members in one persistent
    launch (the solver-generated training runs of the learned warm start).

    bed [M, ny, nx]; n [M or 1, ny, nx]; U0 [M, 3, ny, nx]; out_levels
    [M, n_out] (float32, device tensors).
    """

    def __init__(self, bed: torch.Tensor, n: torch.Tensor, U0: torch.Tensor, out_levels: torch.Tensor,
                 out_dt: float, gauges: Sequence, config: SWEConfig, dx: float, dy: Optional[float] = None,
                 rows: Optional[int] = None, max_steps: int = 1 << 30, max_dt_cap: float = 0.0,
                 arithmetic: str = "exact"):
        from .autotune import tuned_ensemble_rows
        self.arith = nat.arithmetic_code(arithmetic)
        M, ny, nx = bed.shape
        if not 1 <= M <= 1024:
            raise ValueError("a gauge ensemble holds 1 to 1024 members")
        if U0.shape != (M, 3, ny, nx) or out_levels.ndim != 2 or out_levels.shape[0] != M:
            raise ValueError("U0 must be [M,3,ny,nx] and out_levels [M,n_out] for bed [M,ny,nx]")
        if n.ndim != 3 or n.shape[0] not in (1, M) or n.shape[1:] != (ny, nx):
            raise ValueError("n must be [1 or M, ny, nx]")
        if not out_dt > 0:
            raise ValueError("out_dt must be positive")
        if not 0 <= len(gauges) <= 64:
            raise ValueError("at most 64 gauges")
        for iy, ix in gauges:
            if not (0 <= iy < ny and 0 <= ix < nx):
                raise ValueError(f"gauge cell {(iy, ix)} outside the {ny}x{nx} grid")
        dev = bed.device
        self.device = dev
        self.M, self.ny, self.nx = M, ny, nx
        self.n_out = out_levels.shape[1]
        self.ngauge = len(gauges)
        self.bed = nat.require_cuda_f32("bed", bed)
        self.n = nat.require_cuda_f32("n", n)
        self.levels = nat.require_cuda_f32("out_levels", out_levels)
        self.initial = nat.require_cuda_f32("U0", U0)
        self.Ua = self.initial.clone()
        self.Ub = torch.empty_like(self.Ua)
        self.k1 = torch.empty_like(self.Ua)
        self.cells = torch.tensor([v for g in gauges for v in g] or [0, 0], dtype=torch.int32,
                                  device=dev)
        self.gauge_out = torch.zeros((M, self.n_out, max(self.ngauge, 1)), device=dev)
        self.friction = (1 + (0 if config.frictionmodel == "manning" else 1)) if config.apply_friction else 0
        r = int(rows) if rows is not None else tuned_ensemble_rows(dev, arithmetic)
        p = nat.params(config, dx, dx if dy is None else dy, arithmetic)
        members = (nat.SweEnsembleMember * M)()
        for m in range(M):
            mem = members[m]
            mem.bed = self.bed[m].data_ptr()
            mem.n = self.n[m if self.n.shape[0] == M else 0].data_ptr()
            mem.U_a, mem.U_b, mem.k1 = self.Ua[m].data_ptr(), self.Ub[m].data_ptr(), self.k1[m].data_ptr()
            mem.hmax = None
            mem.nseries, mem.ny, mem.nx, mem.steps, mem.rows = 0, ny, nx, int(max_steps), r
            mem.level = 0.0
            mem.start_time = 0.0
            mem.max_dt = float(max_dt_cap)
            mem.params = p
            mem.out_dt = float(out_dt)
            mem.n_out = self.n_out
            mem.ngauge = self.ngauge
            mem.out_levels = self.levels[m].data_ptr()
            mem.gauge_cells = self.cells.data_ptr()
            mem.gauge_out = self.gauge_out[m].data_ptr()
        lib = nat.lib()
        self.workspace = torch.empty(int(lib.swe_ensemble_workspace_bytes(M)), dtype=torch.uint8,
                                     device=dev)
        self.results_dev = torch.empty(M * ctypes.sizeof(nat.SweEnsembleResult), dtype=torch.uint8,
                                       device=dev)
        self.error_dev = torch.zeros(1, dtype=torch.int32, device=dev)
        nat.check(lib.swe_ensemble_prepare_f32(members, M, nat.ptr(self.workspace),
                                               nat.stream_handle(dev)), "gauge ensemble prepare")
        self.blocks = torch.cuda.get_device_properties(dev).multi_processor_count * 6

    def run(self) -> GaugeEnsembleResult:
        lib, st = nat.lib(), nat.stream_handle(self.device)
        self.Ua.copy_(self.initial)
        self.gauge_out.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        nat.check(lib.swe_ensemble_reset_f32(nat.ptr(self.workspace), self.M, st), "ensemble reset")
        e0.record()
        nat.check(lib.swe_ensemble_run_f32(nat.ptr(self.workspace), self.M, self.friction, self.arith,
                                           self.blocks, 0, st), "ensemble run")
        e1.record()
        nat.check(lib.swe_ensemble_results_f32(nat.ptr(self.workspace), self.M,
                                               nat.ptr(self.results_dev), nat.ptr(self.error_dev), st),
                  "ensemble results")
        torch.cuda.synchronize(self.device)
        res = (nat.SweEnsembleResult * self.M).from_buffer_copy(bytes(self.results_dev.cpu().numpy()))
        if int(self.error_dev.item()) != 0:
            raise RuntimeError("ensemble kernel stopped: idle limit reached")
        steps, times = [], []
        final = torch.empty_like(self.Ua)
        for m in range(self.M):
            r = res[m]
            if r.finished == 2:
                if r.status & nat.S_STEP_LIMIT:
                    raise RuntimeError(f"member {m}: step cap reached before the last output interval")
                raise FloatingPointError(f"member {m}: time step failed (status {r.status})")
            final[m] = self.Ua[m] if r.steps % 2 == 0 else self.Ub[m]
            steps.append(int(r.steps))
            times.append(float(r.time))
        cells = self.ny * self.nx
        return GaugeEnsembleResult(self.gauge_out[..., : self.ngauge].clone(), final, steps, times,
                                   e0.elapsed_time(e1), cells * sum(steps))
