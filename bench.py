#!/usr/bin/env python
"""Throughput of the fused FP32 shallow-water step on B200.

Metric: Mcell-updates/s (one cell-update = one full RK2 step of one cell,
friction included) and its fraction of the HBM roofline.

Workload: the runup scenario (plane beach + 20 seeded Gaussian bumps, west
water-level inflow from a leading-depression N-wave, walls elsewhere,
Manning n = 0.01, dx = 0.014 m) after 8 s of simulated time (waves and
wet/dry fronts), tiled to 4096 x 4096 cells; synthetic data.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                  [--arithmetic fast|exact]

One process per GPU (torchrun for N > 1).  Each rank steps its own replica of
the grid -- the single-grid step has no exchange (weak scaling) -- and rank 0
prints one JSON line.  ``value`` is device-timed with CUDA events around K
steps of the tolerance-mode kernels (``--arithmetic``; the IEEE kernels are
timed too and reported under ``exact_arithmetic``) with inputs resident in
HBM; ``e2e`` is the same metric through the public ``SWE2D.forward`` call
with the state copied from pinned host memory and back inside the timed
region.  Outside the timed regions: ``parity`` (three steps of a crop, IEEE
kernels bit for bit against the CPU oracle, tolerance mode's error),
``cpu_baseline`` and ``reference_torch`` (the reference's own PyTorch step,
eager on the host cores and eager / compiled on the GPU).
``--impl reference`` times the CPU oracle (a C restatement of the reference
step, all host threads) on a bounded crop of the same workload.
"""
from __future__ import annotations

import argparse
import contextlib
import ctypes
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np
import torch

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

BYTES_PER_CELL_UPDATE = 32  # read h,hu,hv,z,n once, write h,hu,hv once
STAGE2_BYTES_PER_CELL = 44  # stage-2 kernel: read U, k1, z, n; write U
# DRAM bytes per cell of one stage-2 launch, from ncu captures of the same
# kernel on a smaller grid of the same workload (traffic grows with the
# cells, so a launch of the bench's grid moves this many bytes per cell).
STAGE2_DRAM_BYTES_PER_CELL = {
    # IEEE kernels: 302.1 MB read + 95.9 MB written over 3072^2 cells
    "exact": (302.098944e6 + 95.926016e6) / (3072 * 3072),
    # tolerance mode (tile height 32, as tuned at 4096^2): 333.4 MB read +
    # 93.1 MB written over 3072^2 cells
    "fast": (333.448192e6 + 93.130496e6) / (3072 * 3072),
}
STAGE2_TRAFFIC_SOURCE = {
    "exact": "ncu dram__bytes_read+write of the IEEE stage-2 kernel at 3072^2, scaled by cells",
    "fast": "ncu dram__bytes_read+write of the tolerance-mode stage-2 kernel at 3072^2 (32-row "
            "tiles), scaled by cells",
}
L2_BYTES = 126 * 2 ** 20


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--arithmetic", choices=["exact", "fast"], default="fast",
                    help="step kernels of the headline number (the other mode is reported too)")
    ap.add_argument("--ny", type=int, default=4096)
    ap.add_argument("--nx", type=int, default=4096)
    ap.add_argument("--no-cpu-baseline", action="store_true",
                    help="skip the CPU oracle timing and the parity check on a crop")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-reference-context", action="store_true",
                    help="skip timing the reference's own PyTorch step (baseline/_ref)")
    ap.add_argument("--reference-context", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--rows", type=int, default=0,
                    help="sweep tile height to use instead of the autotuner's (0: autotune)")
    ap.add_argument("--workload", choices=["runup4096", "ensemble", "inversion", "warmstart",
                                           "adjoint"],
                    default="runup4096",
                    help="runup4096: the headline single-grid step; ensemble: 64 scenarios of "
                         "uneven sizes in one persistent launch vs 64 sequential runs")
    ap.add_argument("--ensemble-steps", type=int, default=2000)
    ap.add_argument("--ensemble-count", type=int, default=64)
    ap.add_argument("--ens-arithmetic", choices=["exact", "fast"], default="fast",
                    help="ensemble: step kernels of the scenarios")
    ap.add_argument("--inv-cases", type=int, default=4,
                    help="inversion: runup cases inverted together")
    ap.add_argument("--inv-grid", default="244x393x0.014", help="inversion: ny x nx x dx")
    ap.add_argument("--inv-duration", type=float, default=22.5, help="inversion: seconds simulated")
    ap.add_argument("--inv-arithmetic", choices=["exact", "fast"], default="fast",
                    help="inversion: step kernels of the forward run and its recompute")
    ap.add_argument("--ws-train", type=int, default=20000, help="warmstart: training runs")
    ap.add_argument("--ws-cases", type=int, default=100, help="warmstart: held-out cases")
    ap.add_argument("--ws-epochs", type=int, default=30)
    ap.add_argument("--ws-grid", default="244x393x0.014",
                    help="warmstart: ny x nx x dx of the runup family (the runup config's grid)")
    ap.add_argument("--ws-arithmetic", choices=["exact", "fast"], default="fast",
                    help="warmstart: step kernels of the training runs and inversions")
    ap.add_argument("--ws-cold-cases", type=int, default=8,
                    help="warmstart at full scale: held-out cases also inverted from the cold start")
    ap.add_argument("--ws-cold-iters", type=int, default=40)
    ap.add_argument("--ws-warm-iters", type=int, default=20)
    return ap.parse_args()


def world_size() -> int:
    return int(os.environ.get("WORLD_SIZE", "1"))


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        backend = "nccl" if args.impl == "b200" else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def workload(ny, nx):
    from diffswe2d_b200 import scenarios
    return scenarios.throughput_workload(ny, nx)


def level_at(sc, t: float) -> float:
    """Float32 linear interpolation of the west boundary series at time t."""
    times, levels = sc.bc_times, sc.bc_levels
    i = int(np.searchsorted(times, np.float32(t), side="left"))
    i = min(max(i, 1), len(times) - 1)
    w = (np.float32(t) - times[i - 1]) / max(times[i] - times[i - 1], np.float32(1.1920929e-07))
    return float(levels[i - 1] + np.float32(w) * (levels[i] - levels[i - 1]))


class Clocks:
    """SM clock and clock-event (throttle) reasons sampled every few
    milliseconds through NVML while a region runs (read only; nothing is
    changed)."""

    REASONS = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20,
               "sw_power_cap": 0x4}

    def __init__(self, index: int, period_s: float = 0.005):
        self.index, self.period = index, period_s
        self.samples, self.max_mhz, self.reasons = [], None, set()
        self.error = None

    def _poll(self):
        try:
            import pynvml
            h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))
            while not self._stop.is_set():
                self.samples.append(float(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)))
                bits = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
                for name, bit in self.REASONS.items():
                    if bits & bit:
                        self.reasons.add(name)
                self._stop.wait(self.period)
        except Exception as e:  # sampling must never break the measurement
            self.error = repr(e)

    def __enter__(self):
        import threading
        self._stop = threading.Event()
        self._thread = None
        try:
            import pynvml
            pynvml.nvmlInit()
            self._thread = threading.Thread(target=self._poll, daemon=True)
            self._thread.start()
        except Exception as e:
            self.error = repr(e)
        return self

    def __exit__(self, *exc):
        if self._thread is not None:
            self._stop.set()
            self._thread.join(timeout=5)
        return False

    def summary(self):
        out = {"sm_mhz": statistics.median(self.samples) if self.samples else None,
               "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons),
               "samples": len(self.samples), "source": "NVML, every 5 ms during the timed region"}
        if self.error:
            out["error"] = self.error
        return out


def measured_peaks():
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def crop_of(sc, crop):
    """The top-left crop x crop block of a scenario as a scenario of its own
    (same configuration: west water level, walls elsewhere)."""
    from diffswe2d_b200.scenarios import Scenario
    return Scenario(f"{sc.name}_crop{crop}", np.ascontiguousarray(sc.bed[:crop, :crop]),
                    np.ascontiguousarray(sc.roughness[:crop, :crop]),
                    np.ascontiguousarray(sc.U0[:, :, :crop, :crop]), sc.dx, sc.dy, dict(sc.config),
                    sc.bc_times, sc.bc_levels, sc.steps, dict(sc.meta))


def cpu_baseline(sc, max_seconds=12.0, crop=1024):
    """The CPU oracle (C restatement of the reference step, all host threads)
    on a crop of the workload."""
    sys.path.insert(0, str(REPO / "oracle"))
    from oracle import OracleSWE, num_threads
    from diffswe2d_b200.config import SWEConfig
    c = crop_of(sc, crop)
    m = OracleSWE(c.bed, c.roughness, c.dx, c.dy, SWEConfig(**c.config))
    t = c.meta.get("start_time", 0.0)
    U, dt = m.step(c.U0, t, 1.0e9, boundary_level=level_at(c, t))  # warm caches
    t += dt
    steps, t0 = 0, time.perf_counter()
    while True:
        U, dt = m.step(U, t, 1.0e9, boundary_level=level_at(c, t))
        t += dt
        steps += 1
        el = time.perf_counter() - t0
        if el > max_seconds or steps >= 200:
            break
    cells = c.bed.size
    return {"value": cells * steps / el / 1e6, "unit": "Mcell-updates/s", "cores": num_threads(),
            "kind": "port",
            "sample": f"{steps} steps of a {crop}x{crop} crop of the workload ({el:.1f} s)"}


def parity_on_crop(sc, dev, crop=1024, steps=3):
    """Outside the timed region: `steps` steps of a crop of the workload by
    the IEEE kernels (bit for bit against the CPU oracle) and by the
    tolerance-mode kernels (normwise error against the oracle, wet/dry
    mask), through SWE2D.step."""
    sys.path.insert(0, str(REPO / "oracle"))
    from oracle import OracleSWE
    from diffswe2d_b200 import SWE2D, SWEConfig
    c = crop_of(sc, crop)
    cfg = SWEConfig(**c.config)
    om = OracleSWE(c.bed, c.roughness, c.dx, c.dy, cfg)
    t0 = c.meta.get("start_time", 0.0)
    U, t, ref, dts = c.U0, t0, [], []
    for _ in range(steps):
        U, dt = om.step(U, t, 1.0e9, boundary_level=level_at(c, t))
        t += dt
        ref.append(U)
        dts.append(dt)
    out = {"crop": [crop, crop], "steps": steps}
    for mode in ("exact", "fast"):
        m = SWE2D(torch.from_numpy(c.bed).to(dev), torch.from_numpy(c.roughness).to(dev), c.dx, c.dy,
                  config=cfg, train_dem=False, arithmetic=mode)
        Ug, t, same_dt = torch.from_numpy(c.U0).to(dev), t0, True
        with torch.no_grad():
            for k in range(steps):
                Ug, dt = m.step(Ug, t, 1.0e9, boundary_level=level_at(c, t))
                same_dt &= dt == dts[k]
                t += dt
        Uh = Ug.cpu().numpy()
        if mode == "exact":
            out["exact_bitwise_vs_oracle"] = bool(np.array_equal(Uh.view(np.uint32),
                                                                 ref[-1].view(np.uint32)) and same_dt)
        else:
            errs = []
            for ch in range(3):
                a, b = Uh[:, ch].astype(np.float64), ref[-1][:, ch].astype(np.float64)
                errs.append(float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30)))
            out["fast_normwise_vs_oracle"] = errs
            out["fast_wet_mask_equal"] = bool(np.array_equal(Uh[:, 0] > 1e-6, ref[-1][:, 0] > 1e-6))
    return out


def time_single_grid(sc, args, dev, arithmetic, clocks=None):
    """K device-timed steps of the single-grid step (the two stage kernels
    enqueued through the C ABI, a CUDA event after each) on the workload,
    after W untimed ones; inputs resident in HBM and larger than L2."""
    from diffswe2d_b200 import SWEConfig, autotune
    from diffswe2d_b200 import _native as nat
    ny, nx = sc.bed.shape
    cells = ny * nx
    cfg = SWEConfig(**sc.config)
    if args.rows > 0:
        tuning, rows = {}, args.rows
    else:
        # tile height timed on this very shape (cached per device), as the
        # device loop of SWE2D.forward picks it
        tuning = autotune.tune(dev, arithmetic=arithmetic)
        rows = autotune.tuned_rows_for_shape(1, ny, nx, dev, arithmetic=arithmetic)
    lib = nat.lib()
    nat.check(lib.swe_tune_sweep_rows(rows), "tuned rows")
    p = nat.params(cfg, sc.dx, sc.dy, arithmetic)
    bed = torch.from_numpy(sc.bed).to(dev)
    n = torch.from_numpy(sc.roughness).to(dev)
    U = [torch.from_numpy(sc.U0).to(dev), torch.empty((1, 3, ny, nx), device=dev)]
    k1 = torch.empty_like(U[0])
    red = torch.zeros(nat.RED_WORDS, dtype=torch.int32, device=dev)
    stream = nat.stream_handle(dev)
    total = args.warmup + args.steps
    lev = torch.zeros(total, dtype=torch.float32, device=dev)

    def launch(i, src, dst, stage):
        rc = lib.swe_step_stage_f32(stage, nat.ptr(src), nat.ptr(bed), 1, nat.ptr(n), 1, 1, ny, nx, p,
                                    ctypes.c_void_p(lev.data_ptr() + 4 * i), 1, 1.0e9, None, 0, 1,
                                    nat.ptr(k1), nat.ptr(red), nat.ptr(dst), stream)
        nat.check(rc, "step")

    # Host-side replica of the model time so every step sees the inflow level
    # of its own time, staged on the device before the timed region: the CFL
    # step barely changes over a few hundred steps, one probe step fixes it.
    t = sc.meta.get("start_time", 0.0)
    lev.fill_(level_at(sc, t))
    launch(0, U[0], U[1], 3)
    dt_probe = float(red[3:4].view(torch.float32).item())
    lev.copy_(torch.tensor([level_at(sc, t + i * dt_probe) for i in range(total)], dtype=torch.float32))
    src = 0
    for i in range(args.warmup):
        launch(i, U[src], U[1 - src], 3)
        src = 1 - src
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2 * args.steps + 1)]
    if world_size() > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize(dev)
    with clocks if clocks is not None else contextlib.nullcontext():
        ev[0].record()
        for k in range(args.steps):
            i = args.warmup + k
            launch(i, U[src], U[1 - src], 1)
            ev[2 * k + 1].record()
            launch(i, U[src], U[1 - src], 2)
            ev[2 * k + 2].record()
            src = 1 - src
        torch.cuda.synchronize(dev)
    total_ms = ev[0].elapsed_time(ev[-1])
    s1 = [ev[2 * k].elapsed_time(ev[2 * k + 1]) for k in range(args.steps)]
    s2 = [ev[2 * k + 1].elapsed_time(ev[2 * k + 2]) for k in range(args.steps)]
    return {"total_ms": total_ms, "stage1_ms": statistics.mean(s1), "stage2_ms": statistics.mean(s2),
            "rows": rows,
            "tuned_rows": tuning.get("rows" if arithmetic == "exact" else f"rows_{arithmetic}"),
            "status": int(red[2].item()), "finite": bool(torch.isfinite(U[src]).all().item()),
            "dt_probe": dt_probe}


def end_to_end(sc, args, dev, world, arithmetic, dt_probe):
    """The same metric through the public API: each call is SWE2D.forward(U0,
    t_end = about 100 CFL steps) on a state copied in from pinned host
    memory, with the result copied back to pinned host memory, every copy
    inside the timed region.  Two forms are timed:
      * sequential: copy in, forward, copy out, one call after another;
      * pipelined (the reported value): the copies run on a copy stream,
        the next call's input copy and the previous call's result copy
        overlapping the current call's compute (two device input buffers;
        the first input copy and the last result copy are not overlapped)."""
    from diffswe2d_b200 import SWE2D, SWEConfig
    from diffswe2d_b200.sharding import reduce_over_ranks
    ny, nx = sc.bed.shape
    model = SWE2D(torch.from_numpy(sc.bed).to(dev), torch.from_numpy(sc.roughness).to(dev),
                  sc.dx, sc.dy, config=SWEConfig(**sc.config), train_dem=False, arithmetic=arithmetic)
    model.set_dynamic_boundary(torch.from_numpy(sc.bc_times).to(dev),
                               torch.from_numpy(sc.bc_levels).to(dev))
    t0 = sc.meta.get("start_time", 0.0)
    host_in = torch.from_numpy(sc.U0).pin_memory()
    host_out = [torch.empty_like(host_in).pin_memory() for _ in range(2)]
    span = 100 * dt_probe
    for _ in range(2):  # warm-up (captures the device loop's graph)
        Uf, _ = model(host_in.to(dev, non_blocking=True), t_end=span, start_time=t0)
        host_out[0].copy_(Uf, non_blocking=True)

    def timed(fn):
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        counts = fn(e0)
        e1.record()
        torch.cuda.synchronize(dev)
        return reduce_over_ranks([e0.elapsed_time(e1)], "max", dev)[0], counts

    def sequential(_e0, calls=3):
        counts = []
        for _ in range(calls):
            Uf, _ = model(host_in.to(dev, non_blocking=True), t_end=span, start_time=t0)
            host_out[0].copy_(Uf, non_blocking=True)
            counts.append(model.last_forward_steps)
        return counts

    def pipelined(e0, calls=6):
        comp, cs = torch.cuda.current_stream(dev), torch.cuda.Stream(dev)
        ins = [torch.empty(host_in.shape, device=dev) for _ in range(2)]
        copied = [torch.cuda.Event() for _ in range(2)]   # input i % 2 on the device
        consumed = [torch.cuda.Event() for _ in range(2)]  # call done with input i % 2
        cs.wait_event(e0)
        with torch.cuda.stream(cs):
            ins[0].copy_(host_in, non_blocking=True)
            copied[0].record(cs)
        counts, pending = [], []
        for i in range(calls):
            if i + 1 < calls:  # the next call's input, behind this call's compute
                with torch.cuda.stream(cs):
                    if i >= 1:
                        cs.wait_event(consumed[(i + 1) % 2])
                    ins[(i + 1) % 2].copy_(host_in, non_blocking=True)
                    copied[(i + 1) % 2].record(cs)
            comp.wait_event(copied[i % 2])
            Uf, _ = model(ins[i % 2], t_end=span, start_time=t0)
            consumed[i % 2].record(comp)
            counts.append(model.last_forward_steps)
            with torch.cuda.stream(cs):  # this call's result, behind the next call's compute
                cs.wait_event(consumed[i % 2])
                host_out[i % 2].copy_(Uf, non_blocking=True)
                Uf.record_stream(cs)
            pending.append(Uf)
        comp.wait_stream(cs)
        return counts

    nbytes = host_in.numel() * 4
    seq_runs = sorted((timed(sequential) for _ in range(3)), key=lambda r: r[0])
    ms_seq, counts_seq = seq_runs[1]
    runs = [timed(pipelined) for _ in range(3)]  # the median of three: copies share the host's PCIe
    rates = [world * ny * nx * sum(c) / (m * 1e-3) / 1e6 for m, c in runs]
    order = sorted(range(3), key=lambda r: rates[r])
    ms, counts = runs[order[1]]
    steps, steps_seq = sum(counts), sum(counts_seq)
    return {"value": world * ny * nx * steps / (ms * 1e-3) / 1e6, "unit": "Mcell-updates/s",
            "pipelined_values": rates,
            "h2d_bytes_per_step": nbytes * len(counts) / steps,
            "d2h_bytes_per_step": nbytes * len(counts) / steps,
            "h2d_bytes_per_call": nbytes, "d2h_bytes_per_call": nbytes,
            "internal_steps_per_call": counts,
            "sequential_value": world * ny * nx * steps_seq / (ms_seq * 1e-3) / 1e6,
            "api": "SWE2D.forward(U0 copied from pinned host, t_end = about 100 CFL steps; "
                   "device-driven time loop) + state copied back to pinned host, per call, 6 calls "
                   "with the copies on a copy stream overlapping the neighbouring calls' compute, "
                   "the median of three such runs (pipelined_values: all three; sequential_value: the "
                   "median of three runs of 3 calls, copy in / forward / copy out one after another); "
                   "bytes per step are the per-call copies divided by the solver steps of the call"}


REFERENCE_TARGET = REPO / "baseline" / "_ref"


def reference_context(args, timeout_s=420):
    """The reference's own PyTorch step (installed into baseline/_ref), timed
    in a child process outside every timed region of this run: eager on the
    host cores (a crop), eager on the GPU and torch.compile'd on the GPU
    (the full grid).  Context for the kernels' numbers, not a bench line."""
    if not (REFERENCE_TARGET / "diffswe2d" / "solver.py").exists():
        return {"unavailable": "the reference is not installed in baseline/_ref"}
    cmd = [sys.executable, str(Path(__file__).resolve()), "--reference-context",
           "--ny", str(args.ny), "--nx", str(args.nx)]
    note = None
    env = dict(os.environ)
    for var, path in (("CC", "/usr/bin/gcc"), ("CXX", "/usr/bin/g++")):  # compilers with OpenMP
        if os.path.exists(path):
            env[var] = path
    try:
        out = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout_s, env=env)
        stdout, stderr = out.stdout, out.stderr
    except subprocess.TimeoutExpired as e:
        stdout = e.stdout.decode() if isinstance(e.stdout, bytes) else (e.stdout or "")
        stderr = ""
        note = f"stopped after {timeout_s} s"
    for line in reversed(stdout.splitlines()):
        if line.startswith("{"):
            res = json.loads(line)
            if note:
                res["note"] = note
            elif "cuda_compile" not in res and stderr.strip():
                res["note"] = "stopped: " + stderr.strip().splitlines()[-1]
            return res
    return {"unavailable": note or ("reference timing failed: "
                                    + (stderr.strip().splitlines() or ["?"])[-1])}


def _import_reference():
    import importlib.machinery
    import types
    if "xarray" not in sys.modules:
        try:
            import xarray  # noqa: F401
        except ImportError:  # only the reference's NetCDF reader needs it
            stub = types.ModuleType("xarray")
            stub.__spec__ = importlib.machinery.ModuleSpec("xarray", None)
            sys.modules["xarray"] = stub
    sys.path.insert(0, str(REFERENCE_TARGET))
    import diffswe2d
    return diffswe2d


def run_reference_context(args):
    """Child process of reference_context: prints one JSON object."""
    ref = _import_reference()
    sc = workload(args.ny, args.nx)
    t0 = sc.meta.get("start_time", 0.0)
    res = {"code": "reference SWE2D (baseline/_ref, unmodified), float32"}

    def model_on(dev, c):
        m = ref.SWE2D(torch.from_numpy(c.bed).to(dev), torch.from_numpy(c.roughness).to(dev), c.dx, c.dy,
                      config=ref.SWEConfig(**c.config), train_dem=False)
        m.set_dynamic_boundary(torch.from_numpy(c.bc_times).to(dev), torch.from_numpy(c.bc_levels).to(dev))
        return m

    # eager, host cores, on a crop
    crop = 512
    c = crop_of(sc, crop)
    torch.set_num_threads(os.cpu_count() or 1)
    m = model_on("cpu", c)
    U, t = torch.from_numpy(c.U0), t0
    with torch.no_grad():
        U, dt = m.step(U, t, 1.0e9, boundary_level=m._interpolate_dynamic_boundary(t, U))
        t += dt
        steps, start = 0, time.perf_counter()
        while time.perf_counter() - start < 8.0 and steps < 50:
            U, dt = m.step(U, t, 1.0e9, boundary_level=m._interpolate_dynamic_boundary(t, U))
            t += dt
            steps += 1
        el = time.perf_counter() - start
    res["cpu_eager"] = {"value": crop * crop * steps / el / 1e6, "unit": "Mcell-updates/s",
                        "threads": torch.get_num_threads(), "sample": f"{steps} steps, {crop}x{crop} crop"}
    print(json.dumps(res), flush=True)
    if not torch.cuda.is_available():
        return
    dev = torch.device("cuda", 0)
    ny, nx = sc.bed.shape
    m = model_on(dev, sc)
    U0 = torch.from_numpy(sc.U0).to(dev)

    def timed(fn, count):
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        steps = fn(count)
        e1.record()
        torch.cuda.synchronize(dev)
        return ny * nx * steps / (e0.elapsed_time(e1) * 1e-3) / 1e6

    def eager(count):
        U, t = U0, t0
        with torch.no_grad():
            for _ in range(count):
                U, dt = m.step(U, t, 1.0e9, boundary_level=m._interpolate_dynamic_boundary(t, U))
                t += dt
        return count

    eager(2)
    res["cuda_eager"] = {"value": timed(eager, 10), "unit": "Mcell-updates/s",
                         "sample": f"10 steps of the {ny}x{nx} grid"}
    print(json.dumps(res), flush=True)
    # the reference's own usage: torch.compile(model) around forward(), with
    # the boundary level given per call as its inversion script does (the
    # series lookup of _interpolate_dynamic_boundary does not trace)
    level0 = level_at(sc, t0)
    dt0 = float(m.stable_dt(U0, boundary_level=level0))
    counted = []
    try:
        cm = torch.compile(m)
        start = time.perf_counter()

        def compiled(count):
            counted.clear()
            with torch.no_grad():
                cm(U0, t_end=count * dt0, start_time=t0, boundary_level=level0,
                   callback=lambda i, t, U: counted.append(i))
            return len(counted)

        compiled(3)
        res["cuda_compile_seconds"] = time.perf_counter() - start
        res["cuda_compile"] = {"value": timed(compiled, 10), "unit": "Mcell-updates/s",
                               "sample": f"forward() of about 10 steps of the {ny}x{nx} grid, "
                                         "torch.compile(model) as the reference's examples do"}
    except Exception as e:  # report why, keep the other numbers
        lines = [l for l in str(e).splitlines() if l.strip()]
        res["cuda_compile"] = {"unavailable": f"torch.compile of the reference failed: "
                                              f"{type(e).__name__}: {(lines or ['?'])[0][:300]}"}
    print(json.dumps(res), flush=True)


def run_reference(args, world, rank):
    """--impl reference: the CPU oracle port of the reference step (all host
    threads), rank 0 only, on a 1024x1024 crop of the workload."""
    if rank != 0:
        return
    sc = workload(args.ny, args.nx)
    sys.path.insert(0, str(REPO / "oracle"))
    from oracle import OracleSWE, num_threads
    from diffswe2d_b200.config import SWEConfig
    crop = 1024
    c = crop_of(sc, crop)
    m = OracleSWE(c.bed, c.roughness, c.dx, c.dy, SWEConfig(**c.config))
    U, t = c.U0, c.meta.get("start_time", 0.0)
    for _ in range(args.warmup):
        U, dt = m.step(U, t, 1.0e9, boundary_level=level_at(c, t))
        t += dt
    t0 = time.perf_counter()
    for _ in range(args.steps):
        U, dt = m.step(U, t, 1.0e9, boundary_level=level_at(c, t))
        t += dt
    el = time.perf_counter() - t0
    value = crop * crop * args.steps / el / 1e6
    line = {
        "impl": "reference", "metric": "Mcell-updates/s & %HBM peak", "value": value,
        "unit": "Mcell-updates/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": el / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"runup_tiled_{args.ny}x{args.nx}", "sample": f"{crop}x{crop} crop",
                   "dx": sc.dx},
        "cpu_baseline": {"value": value, "unit": "Mcell-updates/s", "cores": num_threads(),
                         "kind": "port",
                         "sample": f"{args.steps} steps of a {crop}x{crop} crop of the workload"},
        "e2e": {"value": value, "unit": "Mcell-updates/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ensemble(args, world, rank, local):
    """Config 4: scenarios with sides log-uniform in [128, 1024], each its own
    bed, forcing, Manning n and CFL step, `--ensemble-steps` steps each, in one
    persistent CUDA-graph-captured launch; against the same scenarios run one
    after another with the single-grid step (two launches per step).  Under
    torchrun each rank runs its own shard of the scenarios."""
    from diffswe2d_b200 import scenarios
    from diffswe2d_b200 import _native as nat
    from diffswe2d_b200.autotune import tune
    from diffswe2d_b200.config import SWEConfig
    from diffswe2d_b200.ensemble import Ensemble
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    sizes = scenarios.ensemble_sizes(args.ensemble_count, seed=0)
    from diffswe2d_b200.sharding import reduce_over_ranks, shard_indices
    mine = [(k, sizes[k]) for k in shard_indices(len(sizes), world, rank)]
    members = []
    for k, (ny, nx) in mine:
        sc = scenarios.ensemble_member(ny, nx, seed=k)
        sc.steps = args.ensemble_steps
        members.append(sc)
    arith = args.ens_arithmetic
    tuning = tune(dev, arithmetic=arith)
    ens = Ensemble(members, device=dev, arithmetic=arith)
    ens.run()  # warm-up (also captures the graph)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    res = ens.run()
    ms = res.elapsed_ms
    # sequential single-grid runs of the same scenarios
    lib = nat.lib()
    st = nat.stream_handle(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    seq_ms = 0.0
    from diffswe2d_b200.autotune import tuned_rows
    for sc in members:
        ny, nx = sc.bed.shape
        nat.check(lib.swe_tune_sweep_rows(tuned_rows(ny * nx, dev, arith)), "tuned rows")
        cfg = SWEConfig(**sc.config)
        p = nat.params(cfg, sc.dx, sc.dy, arith)
        bed = torch.from_numpy(sc.bed).to(dev)
        n = torch.from_numpy(sc.roughness).to(dev)
        U = [torch.from_numpy(sc.U0).to(dev), torch.empty((1, 3, ny, nx), device=dev)]
        k1 = torch.empty_like(U[0])
        red = torch.empty(nat.RED_WORDS, dtype=torch.int32, device=dev)
        lev = torch.full((1,), float(sc.bc_levels[0]) if sc.bc_levels is not None else 0.0, device=dev)
        torch.cuda.synchronize(dev)
        e0.record()
        for s in range(sc.steps):
            nat.check(lib.swe_step_f32(nat.ptr(U[s % 2]), nat.ptr(bed), 1, nat.ptr(n), 1, 1, ny, nx, p,
                                       nat.ptr(lev), 1, 1.0e9, None, 0, 1, nat.ptr(k1), nat.ptr(red),
                                       nat.ptr(U[1 - s % 2]), st), "sequential step")
        e1.record()
        torch.cuda.synchronize(dev)
        seq_ms += e0.elapsed_time(e1)
    cells = res.cell_updates
    ms, seq_ms = reduce_over_ranks([ms, seq_ms], "max", dev)
    cells = int(reduce_over_ranks([cells], "sum", dev)[0])
    line = {
        "metric": "Mcell-updates/s (ensemble)", "value": cells / (ms * 1e-3) / 1e6,
        "unit": "Mcell-updates/s", "n_gpus": world, "steps": args.ensemble_steps, "warmup": 1,
        "ms_per_step": ms / args.ensemble_steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"ensemble_{args.ensemble_count}_sides_128_1024",
                   "scenarios": len(sizes), "steps_each": args.ensemble_steps,
                   "cells_total": int(sum(a * b for a, b in sizes)),
                   "ensemble_tile_rows": tuning.get("ensemble_rows" if arith == "exact"
                                                    else f"ensemble_rows_{arith}"),
                   "arithmetic": arith,
                   "parallelism": f"scenario shards x{world}"},
        "sequential_single_grid": {"value": cells / (seq_ms * 1e-3) / 1e6, "unit": "Mcell-updates/s",
                                   "ms": seq_ms},
        "persistent_ms": ms,
        "gpu_launches": 2,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


def run_inversion(args, world, rank, local):
    """Config 3: boundary-inflow inversion on the runup grid (default 244 x
    393, dx 0.014 m; 16 controls, 6 gauges every 0.02 s over 22.5 s, Adam lr
    0.002): time per Adam iteration (one gauge run forward + its checkpointed
    adjoint) for `--inv-cases` cases inverted together.  A step of the metric
    is one iteration; cell-updates count forward steps only."""
    from diffswe2d_b200.inversion import make_runup_problem
    from diffswe2d_b200.gauge_run import _WORKSPACES
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    gy, gx, gdx = args.inv_grid.split("x")
    gy, gx, gdx = int(gy), int(gx), float(gdx)
    problem, raw_true = make_runup_problem(cases=args.inv_cases, seed=0, ny=gy, nx=gx, dx=gdx,
                                           duration=args.inv_duration, dt_out=0.02, device=dev,
                                           arithmetic=args.inv_arithmetic)
    raw = torch.zeros_like(raw_true).requires_grad_(True)
    opt = torch.optim.Adam([raw], lr=0.002)
    clk = Clocks(local)

    def iteration():
        opt.zero_grad(set_to_none=True)
        sim = problem.simulate(problem.series(raw))
        loss = ((sim - problem.targets) ** 2).mean(dim=(1, 2)).sum()
        loss.backward()
        opt.step()
        return loss

    for _ in range(max(args.warmup, 1)):
        iteration()
    torch.cuda.synchronize(dev)
    ws = list(_WORKSPACES.values())[0]
    launches0 = ws.kernel_launches
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with clk:
        e0.record()
        for _ in range(args.steps):
            loss = iteration()
        e1.record()
        torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / args.steps
    assert list(_WORKSPACES.values())[0] is ws
    steps = ws.last_steps
    cells = args.inv_cases * gy * gx * steps
    line = {
        "metric": "adjoint inversion: seconds per Adam iteration (config 3)",
        "value": ms / 1e3, "unit": "s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"runup_inversion_{gy}x{gx}", "dx": gdx, "cases": args.inv_cases,
                   "controls": 16, "gauges": 6, "dt_out": 0.02, "duration_s": args.inv_duration,
                   "lr": 0.002,
                   "solver_steps_per_run": steps, "checkpoint_every": ws.k,
                   "checkpoint_every_source": "autotuner (timed k in 32/64/128/256)",
                   "arithmetic": args.inv_arithmetic,
                   "backward_states": "kept from the forward pass" if ws.stored
                   else "recomputed from checkpoints",
                   "l2": "per-iteration working set (states, checkpoints, face buffers) > L2"},
        "forward_plus_adjoint_mcell_per_s": cells / (ms * 1e-3) / 1e6,
        "loss": float(loss.detach()), "clocks": clk.summary(),
        "gpu_launches": ws.kernel_launches - launches0,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_adjoint(args, world, rank, local):
    """The step adjoint alone at the inversion's shape (--inv-cases runup
    cases of --inv-grid, --inv-arithmetic): time per adjoint step as the
    gauge run's backward pass runs it (predictor and k2 re-evaluated, k1
    kept; corrector, stage-2 and stage-1 spatial adjoints), on a state after
    0.3 s of inflow.  The timed loop is bracketed by cudaProfilerStart/Stop
    (for `ncu --profile-from-start off`).  A step of the metric is one
    adjoint step."""
    from diffswe2d_b200.adjoint import AdjointStepper
    from diffswe2d_b200.autotune import sweep_rows, tuned_rows_for_shape
    from diffswe2d_b200.inversion import make_runup_problem
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    gy, gx, gdx = args.inv_grid.split("x")
    gy, gx, gdx = int(gy), int(gx), float(gdx)
    problem, _ = make_runup_problem(cases=args.inv_cases, seed=0, ny=gy, nx=gx, dx=gdx, duration=1.0,
                                    dt_out=0.02, device=dev, arithmetic=args.inv_arithmetic)
    m = problem.model
    B = args.inv_cases
    with torch.no_grad():
        U, _ = m(problem.U0.clone(), t_end=0.3, boundary_level=torch.tensor(0.02, device=dev))
    stp = AdjointStepper(m, B, gy, gx, dev, 1)
    lv = torch.tensor([0.01], device=dev)
    gen = torch.Generator(device="cpu").manual_seed(0)
    lam_out = (torch.randn(U.shape, generator=gen) * 1e-3).to(dev)
    lam_U = torch.zeros_like(U)
    lam_n = torch.zeros_like(stp.n)
    dt = torch.tensor([1e-3], device=dev)
    K1 = torch.empty_like(U)
    rows = tuned_rows_for_shape(B, gy, gx, dev, arithmetic=args.inv_arithmetic)
    clk = Clocks(local)
    with sweep_rows(rows):
        stp._tendency(U, lv, K1)
        for _ in range(max(args.warmup, 1)):
            stp(U, lv, dt, lam_out, lam_U, lam_n, K1=K1)
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.profiler.start()
        with clk:
            e0.record()
            for _ in range(args.steps):
                stp(U, lv, dt, lam_out, lam_U, lam_n, K1=K1)
            e1.record()
            torch.cuda.synchronize(dev)
        torch.cuda.profiler.stop()
    us = e0.elapsed_time(e1) / args.steps * 1e3
    line = {
        "metric": "step adjoint time (inversion shape)", "value": us, "unit": "us",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": us / 1e3,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": f"runup_adjoint_{gy}x{gx}", "cases": B, "dx": gdx, "tile_rows": rows,
                   "arithmetic": args.inv_arithmetic,
                   "per_step": "predictor + k2 re-evaluation, corrector adjoint, stage-2 spatial + "
                               "predictor adjoint, stage-1 spatial adjoint (k1 kept)"},
        "adjoint_mcell_per_s": B * gy * gx / us,
        "gradient_finite": bool(torch.isfinite(lam_U).all()),
        "gpu_launches": 7 * args.steps, "clocks": clk.summary(),
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_warmstart(args, world, rank, local):
    """Config 5: learned warm start + adjoint inversion against the plain
    (cold-start) inversion, Adam lr 0.002, tolerance gauge RMSE <= 1e-4 m, on
    the runup family of --ws-grid (default the runup config's 244 x 393 grid
    at dx 0.014 m).  Training runs come from the persistent ensemble kernel;
    the network is trained by the project's own kernels.  At the full grid a
    batched adjoint iteration over the 100 held-out cases costs about a
    minute, so the warm start is evaluated on every held-out case and the
    cold start on --ws-cold-cases of them (compare_at_scale).  value = median
    wall time to tolerance per warm-started case (inference and its forward
    evaluation included)."""
    from diffswe2d_b200.inversion import RunupFamily
    from diffswe2d_b200.warmstart import WarmStartNet
    from diffswe2d_b200.warmstart_study import compare_at_scale, generate, train
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    ny, nx, dx = args.ws_grid.split("x")
    fam = RunupFamily(int(ny), int(nx), float(dx), seed=0, device=str(dev), arithmetic=args.ws_arithmetic)
    clk = Clocks(local)
    with clk:
        # training runs and held-out cases are sharded over the ranks (no
        # communication during the runs, one gather at the end); every rank
        # trains the same network on the gathered data
        data = generate(fam, args.ws_train, seed=1, world=world, rank=rank)
        net = WarmStartNet(dev, seed=0)
        log = train(net, data, epochs=args.ws_epochs, batch=256, lr=2e-3)
        res = compare_at_scale(fam, net, cases=args.ws_cases, seed=12345, lr=0.002, tol=1e-4,
                               warm_max_iters=args.ws_warm_iters, cold_cases=args.ws_cold_cases,
                               cold_max_iters=args.ws_cold_iters, world=world, rank=rank)
    w, c = res["warm"], res["cold"]
    warm_t = [t for t in w["seconds_to_tol"] if t is not None]
    cold_per_case_s = c["seconds_per_iteration_per_case"]
    line = {
        "metric": "inversion wall-time to gauge RMSE <= 1e-4 m (learned warm start)",
        "value": float(np.median(warm_t)) if warm_t else None, "unit": "s per case", "n_gpus": world,
        "steps": w["median_iterations"], "warmup": 0,
        "ms_per_step": None, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": f"f32 solver ({args.ws_arithmetic} arithmetic) and adjoint; bf16 products with "
                 "fp32 accumulation in the network",
        "data": "synthetic (solver-generated runs)",
        "config": {"workload": f"runup_warmstart_{ny}x{nx}", "dx": float(dx),
                   "training_runs": args.ws_train, "held_out_cases": args.ws_cases, "tol_m": 1e-4,
                   "lr": 0.002, "samples": fam.n_out, "gauges": fam.n_gauges,
                   "controls": fam.n_controls, "arithmetic": args.ws_arithmetic},
        "warm": {"cases": args.ws_cases, "reached": w["reached"],
                 "reached_at_iteration_0": w["reached_at_iteration_0"],
                 "median_iterations": w["median_iterations"],
                 "max_iterations": max([i for i in w["iterations"] if i is not None], default=None),
                 "median_seconds_to_tol": float(np.median(warm_t)) if warm_t else None,
                 "max_seconds_to_tol": max(warm_t) if warm_t else None,
                 "median_initial_rmse": float(np.median(w["initial_rmse"])),
                 "forward_eval_s_per_case": w["forward_eval_s_per_case"],
                 "inference_s": res["inference_s"]},
        "cold": {"cases": c["cases"], "reached": c["reached"], "max_iters": c["max_iters"],
                 "iterations": c["iterations"],
                 "seconds_per_iteration_per_case": cold_per_case_s,
                 "seconds_at_cap_per_case": (cold_per_case_s * (c["max_iters"] + 1)
                                             if cold_per_case_s else None),
                 "median_initial_rmse": float(np.median(c["initial_rmse"])),
                 "median_final_rmse": float(np.median(c["final_rmse"]))},
        "predicted_control_rmse_m": res["pred_control_rmse_m"],
        "training": {"runs": args.ws_train, "generation_s": data.seconds,
                     "generation_mcell_per_s": data.cell_updates / data.seconds / 1e6,
                     "epochs": log.epochs, "steps": log.steps, "train_s": log.seconds,
                     "val_control_rmse_m": log.val_rmse_m},
        "clocks": clk.summary(),
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.reference_context:
        run_reference_context(args)
        return
    world, rank, local = dist_setup(args)
    if args.workload == "ensemble" and args.impl == "b200":
        run_ensemble(args, world, rank, local)
        return
    if args.workload == "warmstart" and args.impl == "b200":
        run_warmstart(args, world, rank, local)
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()
        return
    if args.workload in ("inversion", "adjoint") and args.impl == "b200":
        if rank == 0:
            (run_inversion if args.workload == "inversion" else run_adjoint)(args, world, rank, local)
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()
        return
    if args.impl == "reference":
        run_reference(args, world, rank)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA device")
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    from diffswe2d_b200 import SWE2D, SWEConfig
    from diffswe2d_b200 import _native as nat

    sc = workload(args.ny, args.nx)
    ny, nx = sc.bed.shape
    cells = ny * nx
    modes = [args.arithmetic] + [m for m in ("fast", "exact") if m != args.arithmetic]
    runs, clk = {}, None
    for mode in modes:
        c = Clocks(local)
        runs[mode] = time_single_grid(sc, args, dev, mode, c)
        if mode == args.arithmetic:
            clk = c
    head = runs[args.arithmetic]
    from diffswe2d_b200.sharding import reduce_over_ranks
    for r in runs.values():
        r["total_ms"] = reduce_over_ranks([r["total_ms"]], "max", dev)[0]  # max over ranks
        r["value"] = world * cells * args.steps / (r["total_ms"] * 1e-3) / 1e6
        r["ms_per_step"] = r["total_ms"] / args.steps

    e2e = None
    if not args.no_e2e:
        e2e = end_to_end(sc, args, dev, world, args.arithmetic, head["dt_probe"])

    peak, peak_kind = measured_peaks()

    def roofline(r, mode):
        achieved = STAGE2_BYTES_PER_CELL * cells / (r["stage2_ms"] * 1e-3) / 1e9
        step_achieved = BYTES_PER_CELL_UPDATE * cells / (r["ms_per_step"] * 1e-3) / 1e9
        traffic = STAGE2_DRAM_BYTES_PER_CELL.get(mode)
        return {"bound": "hbm", "kernel": f"stage 2 ({mode} arithmetic): predictor + tendency + "
                                          "corrector + friction",
                "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": None if traffic is None else traffic * cells,
                "traffic_source": STAGE2_TRAFFIC_SOURCE.get(mode),
                "peak_kind": peak_kind, "bytes_per_cell": STAGE2_BYTES_PER_CELL,
                "stage1_ms": r["stage1_ms"], "stage2_ms": r["stage2_ms"],
                "step_achieved_gbs": step_achieved, "step_frac": step_achieved / peak,
                "step_bytes_per_cell_update": BYTES_PER_CELL_UPDATE}

    line = {
        "metric": "Mcell-updates/s & %HBM peak",
        "value": head["value"],
        "unit": "Mcell-updates/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": head["ms_per_step"],
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": f"runup_tiled_{ny}x{nx}", "grid": [ny, nx], "dx": sc.dx,
                   "state": f"runup scenario after {sc.meta.get('start_time', 0.0):g} s of simulated "
                            "time (waves, wet/dry fronts), tiled",
                   "boundaries": "west water_level (N-wave), walls", "manning": 0.01,
                   "arithmetic": args.arithmetic,
                   "l2": "inputs larger than L2: state 201 MB + k1 201 MB + bed/n 134 MB per replica",
                   "parallelism": f"replicas x{world}", "sweep_tile_rows": head["rows"],
                   "tuned_rows_by_size_class": head["tuned_rows"]},
        "roofline": roofline(head, args.arithmetic),
        "gpu_launches": 2 * args.steps,
        "clocks": clk.summary() if clk is not None else None,
        "status_word": head["status"],
        "state_finite": head["finite"],
    }
    for mode, r in runs.items():
        if mode != args.arithmetic:
            line[f"{mode}_arithmetic"] = {"value": r["value"], "unit": "Mcell-updates/s",
                                          "ms_per_step": r["ms_per_step"],
                                          "sweep_tile_rows": r["rows"],
                                          "roofline": roofline(r, mode),
                                          "status_word": r["status"], "state_finite": r["finite"]}
    if e2e is not None:
        line["e2e"] = e2e
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(sc)
        line["parity"] = parity_on_crop(sc, dev)
    if rank == 0 and world == 1 and not args.no_reference_context:
        line["reference_torch"] = reference_context(args)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
