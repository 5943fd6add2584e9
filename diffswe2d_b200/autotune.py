"""Autotuner for the step kernels' launch shape.

Two knobs are tuned by timing them on the GPU in use:

* the sweep tile height (output rows per warp strip) per grid-size class --
  taller tiles recompute fewer halo rows, shorter ones give more tiles to
  fill the 148 SMs on small grids and a shorter serial chain per warp; used
  by the single-grid kernels (``swe_tune_sweep_rows``); one throughput-tuned
  value for the persistent ensemble kernel (``tuned_ensemble_rows``); and per
  exact (batch, ny, nx) shape for the captured time loops of gauge runs and
  ``SWE2D.forward`` (``tuned_rows_for_shape``);
* the number of steps per CUDA-graph replay of ``SWE2D.forward``'s device
  loop -- more steps per replay mean fewer host reads, more no-op steps at
  the end of a call;
* the checkpoint interval k of a differentiated gauge run
  (``tuned_checkpoint_every``) -- memory O(steps/k + k) states; a longer k
  means fewer checkpoints but a longer recomputed (or copied) segment held
  at once and longer captured graphs -- timed on the run itself.

Tile heights are tuned separately for the two arithmetic modes of the step
kernels ("exact" and "fast"), whose register use and cost per cell differ.
Results are kept per device name in memory and in
``$XDG_CACHE_HOME/diffswe2d_b200/autotune.json`` (default ``~/.cache``).
"""
from __future__ import annotations

import json
import os
import time
from pathlib import Path
from typing import Dict, Optional

import torch

from . import _native as nat

SIZE_CLASSES = ((0, 1 << 16), (1 << 16, 1 << 18), (1 << 18, 1 << 20), (1 << 20, 1 << 62))
ROW_CHOICES = (4, 8, 16, 32, 64, 128)
DEFAULT_ROWS = (16, 32, 64, 64)
CHUNK_CHOICES = (8, 16, 32, 64)

_tuned: Dict[str, dict] = {}


def _cache_file() -> Path:
    base = os.environ.get("XDG_CACHE_HOME") or str(Path.home() / ".cache")
    return Path(base) / "diffswe2d_b200" / "autotune.json"


def _device_key(device) -> str:
    props = torch.cuda.get_device_properties(torch.device(device))
    return f"{props.name}/{props.multi_processor_count}"


def _load(device) -> dict:
    key = _device_key(device)
    if key not in _tuned:
        try:
            _tuned[key] = json.loads(_cache_file().read_text()).get(key, {})
        except (OSError, ValueError):
            _tuned[key] = {}
    return _tuned[key]


def _store(device, entry: dict) -> None:
    key = _device_key(device)
    _tuned[key] = entry
    path = _cache_file()
    try:
        data = json.loads(path.read_text()) if path.exists() else {}
        data[key] = entry
        path.parent.mkdir(parents=True, exist_ok=True)
        path.write_text(json.dumps(data, indent=1))
    except OSError:
        pass


def size_class(cells: int) -> int:
    for k, (lo, hi) in enumerate(SIZE_CLASSES):
        if lo <= cells < hi:
            return k
    return len(SIZE_CLASSES) - 1


def _mode_key(name: str, arithmetic: str) -> str:
    nat.arithmetic_code(arithmetic)
    return name if arithmetic == "exact" else f"{name}_{arithmetic}"


def tuned_rows(cells: int, device="cuda", arithmetic: str = "exact") -> int:
    """Tile height for a grid of `cells` cells (the default if not tuned)."""
    k = size_class(cells)
    rows = _load(device).get(_mode_key("rows", arithmetic))
    return int(rows[k]) if rows else DEFAULT_ROWS[k]


def _time_steps(side_y: int, side_x: int, rows: int, device, steps: int, batch: int = 1,
                arithmetic: str = "exact") -> float:
    """ms per step of the single-grid step kernels on a runup-recipe grid
    (``batch`` copies of it)."""
    from . import scenarios
    from .config import SWEConfig
    sc = scenarios.tiled(scenarios.runup(seed=0), side_y, side_x)
    dev = torch.device(device)
    lib = nat.lib()
    p = nat.params(SWEConfig(**sc.config), sc.dx, sc.dy, arithmetic)
    bed = torch.from_numpy(sc.bed).to(dev)
    n = torch.from_numpy(sc.roughness).to(dev)
    U0 = torch.from_numpy(sc.U0).to(dev).expand(batch, 3, side_y, side_x).contiguous()
    U = [U0, torch.empty_like(U0)]
    k = torch.empty_like(U[0])
    red = torch.empty(nat.RED_WORDS, dtype=torch.int32, device=dev)
    lev = torch.full((1,), 0.005, device=dev)
    st = nat.stream_handle(dev)
    nat.check(lib.swe_tune_sweep_rows(rows), "tune rows")

    def run(count):
        for s in range(count):
            rc = lib.swe_step_f32(nat.ptr(U[s % 2]), nat.ptr(bed), 1, nat.ptr(n), 1, batch, side_y, side_x,
                                  p, nat.ptr(lev), 1, 1.0e9, None, 0, 1, nat.ptr(k), nat.ptr(red),
                                  nat.ptr(U[1 - s % 2]), st)
            nat.check(rc, "tune step")

    run(2)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    run(steps)
    e1.record()
    torch.cuda.synchronize(dev)
    return e0.elapsed_time(e1) / steps


def tune(device="cuda", steps: int = 8, force: bool = False, arithmetic: str = "exact") -> dict:
    """Time every tile height on one representative grid per size class
    (kernels of the given arithmetic), the ensemble tile height and the
    graph chunk length on a small grid; store and return the choice."""
    entry = dict(_load(device))
    rkey = _mode_key("rows", arithmetic)
    if entry.get(rkey) and not force:
        return entry
    t0 = time.perf_counter()
    reps = ((96, 160), (384, 512), (1024, 960), (2048, 2048))
    rows_choice, timing = [], {}
    for k, (ny, nx) in enumerate(reps):
        best, best_ms = None, None
        for r in ROW_CHOICES:
            ms = _time_steps(ny, nx, r, device, steps, arithmetic=arithmetic)
            timing[f"{ny}x{nx}/rows{r}"] = ms
            if best_ms is None or ms < best_ms:
                best, best_ms = r, ms
        rows_choice.append(best)
    nat.check(nat.lib().swe_tune_sweep_rows(64), "tune rows")
    entry[rkey] = rows_choice
    if not entry.get("chunk") or force:
        entry["chunk"] = _tune_chunk(device)
    entry[_mode_key("ensemble_rows", arithmetic)] = _tune_ensemble_rows(device, arithmetic=arithmetic)
    entry[_mode_key("timing_ms", arithmetic)] = timing
    entry[_mode_key("seconds", arithmetic)] = time.perf_counter() - t0
    _store(device, entry)
    return entry


ENSEMBLE_ROW_CHOICES = (8, 16, 32, 64)


def _tune_ensemble_rows(device, count: int = 24, steps: int = 30, arithmetic: str = "exact") -> int:
    """Tile height for the persistent ensemble kernel, where many scenarios
    fill the GPU together (throughput, not per-step latency, decides): one
    value for all scenarios, timed on `count` seeded scenarios with sides
    log-uniform in [128, 1024]."""
    from . import scenarios
    from .ensemble import Ensemble
    sizes = scenarios.ensemble_sizes(count, seed=99)
    members = []
    for k, (ny, nx) in enumerate(sizes):
        sc = scenarios.ensemble_member(ny, nx, seed=1000 + k)
        sc.steps = steps
        members.append(sc)
    best, best_ms = None, None
    for r in ENSEMBLE_ROW_CHOICES:
        ens = Ensemble(members, device=device, rows=r, arithmetic=arithmetic)
        ens.run()
        ms = ens.run().elapsed_ms
        if best_ms is None or ms < best_ms:
            best, best_ms = r, ms
        del ens
    return int(best)


def tuned_ensemble_rows(device="cuda", arithmetic: str = "exact") -> int:
    """The ensemble kernel's tile height (16 if not tuned)."""
    return int(_load(device).get(_mode_key("ensemble_rows", arithmetic), 16))


def _tune_chunk(device) -> int:
    from . import scenarios
    from .config import SWEConfig
    from .solver import SWE2D
    sc = scenarios.runup(ny=122, nx=196, dx=0.028, seed=1)
    dev = torch.device(device)
    m = SWE2D(torch.from_numpy(sc.bed).to(dev), torch.from_numpy(sc.roughness).to(dev), sc.dx, sc.dy,
              config=SWEConfig(**sc.config), train_dem=False)
    U0 = torch.from_numpy(sc.U0).to(dev)
    best, best_t = None, None
    for chunk in CHUNK_CHOICES:
        m.steps_per_chunk = chunk
        with torch.no_grad():
            m(U0, t_end=0.2, boundary_level=0.005)
            torch.cuda.synchronize(dev)
            t = time.perf_counter()
            m(U0, t_end=0.5, boundary_level=0.005)
            torch.cuda.synchronize(dev)
            t = time.perf_counter() - t
        if best_t is None or t < best_t:
            best, best_t = chunk, t
    return int(best)


def tuned_rows_for_shape(batch: int, ny: int, nx: int, device="cuda", steps: int = 6,
                         arithmetic: str = "exact") -> int:
    """Tile height for a time loop over [batch, 3, ny, nx] states: timed on
    that shape (runup recipe) the first time it is asked for, then cached."""
    entry = _load(device)
    key = f"{batch}x{ny}x{nx}" if arithmetic == "exact" else f"{arithmetic}/{batch}x{ny}x{nx}"
    shapes = entry.setdefault("shapes", {})
    if key in shapes:
        return int(shapes[key])
    prev = int(nat.lib().swe_sweep_rows())
    best, best_ms = None, None
    try:
        for r in ROW_CHOICES:
            if r > 2 * ny and best is not None:
                break
            ms = _time_steps(ny, nx, r, device, steps, batch, arithmetic)
            if best_ms is None or ms < best_ms:
                best, best_ms = r, ms
    finally:
        nat.check(nat.lib().swe_tune_sweep_rows(prev), "tune rows")
    shapes[key] = int(best)
    _store(device, entry)
    return int(best)


CHECKPOINT_CHOICES = (32, 64, 128, 256)


def tuned_checkpoint_every(model, U0, levels, out_dt: float, gauges, max_dt_cap=None,
                           store_states=None, budget_frac: float = 0.25, force: bool = False) -> int:
    """Checkpoint interval k of ``gauge_run`` for this model, state shape,
    interval count and storage mode: the k in CHECKPOINT_CHOICES whose
    forward + backward gauge run is fastest, timed on the first intervals of
    the caller's own run (about 1500 solver steps), among the k whose
    segment and checkpoint buffers fit in ``budget_frac`` of the free device
    memory.  Cached per device like the tile heights."""
    from .gauge_run import CHECKPOINT_EVERY, GRAPH_STEPS, gauge_run
    dev = U0.device
    B, _, ny, nx = U0.shape
    lv = levels.detach()
    n_out = lv.shape[-1]
    entry = _load(dev)
    key = (f"{model.arithmetic}/{B}x{ny}x{nx}/{n_out}x{float(out_dt):.6g}/"
           f"{len(gauges)}g/{'store' if store_states else 'auto' if store_states is None else 'recompute'}")
    table = entry.setdefault("checkpoint_every", {})
    if key in table and not force:
        return int(table[key]["k"])
    Ud = U0.detach()
    # steps per interval, from one forward pass of a few intervals
    probe = lv[..., : min(n_out, 4)]
    with torch.no_grad():
        gauge_run(model, Ud, probe, out_dt, gauges, max_dt_cap=max_dt_cap,
                  checkpoint_every=CHECKPOINT_EVERY, store_states=False)
    from .gauge_run import _WORKSPACES
    per_interval = max(1, list(_WORKSPACES.values())[0].last_steps // probe.shape[-1])
    n_t = max(1, min(n_out, -(-1536 // per_interval)))
    lv_t = lv[..., :n_t].contiguous()
    state_bytes = 4 * 3 * B * ny * nx
    est_steps = per_interval * n_out
    free, _ = torch.cuda.mem_get_info(dev)
    timings = {}
    best, best_ms = None, None
    for k in CHECKPOINT_CHOICES:
        if k % GRAPH_STEPS:
            continue
        need = (2 * k + 1 + -(-est_steps // k)) * state_bytes
        if need > budget_frac * free and best is not None:
            continue
        U = Ud.clone().requires_grad_(True)
        L = lv_t.clone().requires_grad_(True)
        ms = []
        with torch.enable_grad():
            for rep in range(2):  # the first run captures the graphs
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                g, _ = gauge_run(model, U, L, out_dt, gauges, max_dt_cap=max_dt_cap,
                                 checkpoint_every=k, store_states=store_states)
                g.square().sum().backward()
                e1.record()
                torch.cuda.synchronize(dev)
                ms.append(e0.elapsed_time(e1))
        timings[str(k)] = ms[-1]
        if best_ms is None or ms[-1] < best_ms:
            best, best_ms = k, ms[-1]
    table[key] = {"k": int(best), "timing_ms": timings, "intervals_timed": n_t}
    _store(dev, entry)
    return int(best)


def checkpoint_tuning(device, key_prefix: str = "") -> dict:
    """The cached checkpoint-interval choices (and their timings) of a device."""
    return {k: v for k, v in _load(device).get("checkpoint_every", {}).items() if k.startswith(key_prefix)}


class sweep_rows:
    """Context manager: the single-grid kernels use ``rows`` inside (e.g.
    while a CUDA graph is captured), the previous value after."""

    def __init__(self, rows: int):
        self.rows = int(rows)

    def __enter__(self):
        self.prev = int(nat.lib().swe_sweep_rows())
        nat.check(nat.lib().swe_tune_sweep_rows(self.rows), "tune rows")
        return self

    def __exit__(self, *exc):
        nat.check(nat.lib().swe_tune_sweep_rows(self.prev), "tune rows")
        return False


def apply(device="cuda", cells: Optional[int] = None, arithmetic: str = "exact") -> None:
    """Use the tuned values: tile height for grids of `cells` cells (single-grid
    kernels of the given arithmetic) and the forward() chunk length."""
    entry = _load(device)
    if cells is not None:
        nat.check(nat.lib().swe_tune_sweep_rows(tuned_rows(cells, device, arithmetic)), "tune rows")
    if entry.get("chunk"):
        from .solver import SWE2D
        SWE2D.steps_per_chunk = int(entry["chunk"])


__all__ = ["tune", "tuned_rows", "tuned_ensemble_rows", "tuned_rows_for_shape", "sweep_rows", "apply",
           "tuned_checkpoint_every", "checkpoint_tuning", "CHECKPOINT_CHOICES",
           "size_class",
           "SIZE_CLASSES", "ROW_CHOICES"]
