"""Seeded synthetic scenarios with the shapes of the benchmark workloads.

The reference validates on laboratory benchmarks (Monai Valley runup, CEA
2008 rainfall-runoff) whose data are not part of this package.  These
recipes stand in for them with the same grid shapes, spacings, forcing
lengths and value ranges:

* ``gaussian_island`` -- 256x256, dx = 1 m, walls: sloping bed with one
  Gaussian island, Gaussian hump of water, Manning n = 0.025.
* ``runup`` -- 244x393 (ny x nx), dx = 0.014 m: plane beach from 0.13 m
  depth (west) to 0.10 m above still water (east) plus 20 seeded Gaussian
  valleys/ridges, west ``water_level`` inflow from a leading-depression
  N-wave sampled at 50 Hz for 22.5 s, other sides walls, Manning n = 0.01.
* ``tiled`` -- any scenario tiled to a larger grid (4096x4096 for the
  HBM-roofline runs).
* ``ensemble`` -- many runup/hump scenarios of uneven sizes.

All arrays are built in float64 with numpy's PCG64 generator and returned
as float32 numpy arrays; tests keep the float32 inputs they use in their
fixtures, so results never depend on a platform's libm.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from pathlib import Path
from typing import Optional

import numpy as np


@dataclass
class Scenario:
    name: str
    bed: np.ndarray            # [ny, nx] float32
    roughness: np.ndarray      # [ny, nx] float32 (Manning n)
    U0: np.ndarray             # [1, 3, ny, nx] float32
    dx: float
    dy: float
    config: dict               # SWEConfig keyword arguments
    bc_times: Optional[np.ndarray] = None   # dynamic west boundary (seconds)
    bc_levels: Optional[np.ndarray] = None  # water levels (m)
    steps: int = 1000
    meta: dict = field(default_factory=dict)

    @property
    def shape(self):
        return self.bed.shape

    def make_config(self, cls):
        return cls(**self.config)


def _centres(n: int, d: float) -> np.ndarray:
    return (np.arange(n, dtype=np.float64) + 0.5) * d


def gaussian_island(n: int = 256, seed: int = 0, dx: float = 1.0) -> Scenario:
    """Config 1: walls, z = -10 + 0.02 x + 2 exp(-r^2/(2*20^2)), hump 0.5 m, sigma 15 m."""
    rng = np.random.default_rng(seed)
    x = _centres(n, dx)
    X, Y = np.meshgrid(x, x)  # Y varies along rows (axis 0)
    L = n * dx
    cx, cy = rng.uniform(0.25 * L, 0.75 * L, size=2)
    z = -10.0 + 0.02 * X + 2.0 * np.exp(-((X - cx) ** 2 + (Y - cy) ** 2) / (2 * 20.0 ** 2))
    eta = 0.5 * np.exp(-((X - L / 2) ** 2 + (Y - L / 2) ** 2) / (2 * 15.0 ** 2))
    h = np.maximum(eta - z, 0.0)
    U0 = np.stack([h, np.zeros_like(h), np.zeros_like(h)])[None]
    cfg = dict(boundary_left="wall", boundary_right="wall", boundary_top="wall",
               boundary_bottom="wall", cfl=0.5, limiter_theta=1.3, frictionmodel="manning")
    return Scenario("gaussian_island", z.astype(np.float32), np.full_like(z, 0.025, np.float32),
                    U0.astype(np.float32), dx, dx, cfg, steps=1000,
                    meta=dict(seed=seed, island=(float(cx), float(cy))))


def n_wave(t: np.ndarray, trough: float = -0.01, crest: float = 0.015,
           period: float = 15.0) -> np.ndarray:
    """Leading-depression N-wave: trough then crest over one period, zero after."""
    s = np.asarray(t, dtype=np.float64) / period
    w = np.where(s < 0.5, trough * np.sin(2 * np.pi * s), -crest * np.sin(2 * np.pi * s))
    return np.where((s >= 0.0) & (s <= 1.0), w, 0.0)


def runup_bed(ny: int, nx: int, dx: float, rng, n_bumps: int = 20) -> np.ndarray:
    x, y = _centres(nx, dx), _centres(ny, dx)
    X, Y = np.meshgrid(x, y)
    Lx, Ly = nx * dx, ny * dx
    z = -0.13 + 0.23 * X / Lx
    for _ in range(n_bumps):
        cx, cy = rng.uniform(0.0, Lx), rng.uniform(0.0, Ly)
        amp = rng.uniform(0.01, 0.05) * (1.0 if rng.uniform() < 0.5 else -1.0)
        sig = rng.uniform(0.05, 0.3)
        z = z + amp * np.exp(-((X - cx) ** 2 + (Y - cy) ** 2) / (2 * sig ** 2))
    return z


RUNUP_SAMPLES = 1125  # 22.5 s at 50 Hz
RUNUP_DT_SAMPLE = 0.02


def runup(ny: int = 244, nx: int = 393, dx: float = 0.014, seed: int = 0,
          n_bumps: int = 20, manning: float = 0.01) -> Scenario:
    """Config 2: plane beach + Gaussian bumps, west N-wave water level, walls elsewhere."""
    rng = np.random.default_rng(seed)
    z = runup_bed(ny, nx, dx, rng, n_bumps)
    h = np.maximum(-z, 0.0)
    U0 = np.stack([h, np.zeros_like(h), np.zeros_like(h)])[None]
    times = np.arange(RUNUP_SAMPLES, dtype=np.float64) * RUNUP_DT_SAMPLE
    levels = n_wave(times)
    cfg = dict(boundary_left="water_level", boundary_right="wall", boundary_top="wall",
               boundary_bottom="wall", cfl=0.5, limiter_theta=1.3, frictionmodel="manning")
    return Scenario("runup", z.astype(np.float32), np.full_like(z, manning, np.float32),
                    U0.astype(np.float32), dx, dx, cfg, times.astype(np.float32),
                    levels.astype(np.float32), steps=1000, meta=dict(seed=seed))


def tiled(base: Scenario, ny: int, nx: int) -> Scenario:
    """The base scenario's bed/state/roughness tiled periodically to ny x nx."""
    by, bx = base.bed.shape
    reps = (math.ceil(ny / by), math.ceil(nx / bx))
    bed = np.tile(base.bed, reps)[:ny, :nx]
    n = np.tile(base.roughness, reps)[:ny, :nx]
    U0 = np.tile(base.U0, (1, 1) + reps)[:, :, :ny, :nx]
    return Scenario(f"{base.name}_tiled_{ny}x{nx}", np.ascontiguousarray(bed),
                    np.ascontiguousarray(n), np.ascontiguousarray(U0), base.dx, base.dy,
                    dict(base.config), base.bc_times, base.bc_levels, base.steps,
                    dict(base.meta, tiled_from=base.name))


def ensemble_sizes(count: int = 64, lo: int = 128, hi: int = 1024, seed: int = 0):
    """Grid sides drawn log-uniform in [lo, hi] (non-square allowed)."""
    rng = np.random.default_rng(seed)
    sides = np.exp(rng.uniform(math.log(lo), math.log(hi), size=(count, 2)))
    return [(int(round(a)), int(round(b))) for a, b in sides]


def ensemble_member(ny: int, nx: int, seed: int) -> Scenario:
    """One ensemble scenario: plane beach + Gaussians, hump or N-wave forcing, n in [0.01,0.035]."""
    rng = np.random.default_rng(seed)
    dx = 0.014 * 393 / max(nx, 1)
    z = runup_bed(ny, nx, dx, rng, n_bumps=int(rng.integers(5, 21)))
    manning = float(rng.uniform(0.01, 0.035))
    hump = rng.uniform() < 0.5
    h = np.maximum(-z, 0.0)
    if hump:
        x, y = _centres(nx, dx), _centres(ny, dx)
        X, Y = np.meshgrid(x, y)
        cx, cy = rng.uniform(0.1, 0.5) * nx * dx, rng.uniform(0.2, 0.8) * ny * dx
        sig = rng.uniform(0.05, 0.2) * min(nx, ny) * dx
        eta = 0.02 * np.exp(-((X - cx) ** 2 + (Y - cy) ** 2) / (2 * sig ** 2))
        h = np.where(h > 0.0, np.maximum(eta - z, 0.0), 0.0)
    U0 = np.stack([h, np.zeros_like(h), np.zeros_like(h)])[None]
    cfg = dict(boundary_left="water_level" if not hump else "wall", boundary_right="wall",
               boundary_top="wall", boundary_bottom="wall", cfl=0.5, limiter_theta=1.3,
               frictionmodel="manning")
    times = levels = None
    if not hump:
        times = (np.arange(RUNUP_SAMPLES) * RUNUP_DT_SAMPLE).astype(np.float32)
        levels = n_wave(times.astype(np.float64)).astype(np.float32)
    return Scenario(f"ensemble_{ny}x{nx}_{seed}", z.astype(np.float32),
                    np.full_like(z, manning, np.float32), U0.astype(np.float32), dx, dx, cfg,
                    times, levels, steps=2000, meta=dict(seed=seed, hump=bool(hump)))


def spun_up(base: Scenario, seconds: float, device="cuda", arithmetic: str = "exact") -> Scenario:
    """The scenario advanced ``seconds`` of simulated time by ``SWE2D.forward``
    on the GPU (its boundary series included), as a new scenario whose
    initial state is that state and whose ``meta["start_time"]`` is
    ``seconds``: a state with waves and moving wet/dry fronts instead of
    water at rest, e.g. to tile into the 4096x4096 throughput workload."""
    import torch

    from .config import SWEConfig
    from .solver import SWE2D
    dev = torch.device(device)
    model = SWE2D(torch.from_numpy(base.bed).to(dev), torch.from_numpy(base.roughness).to(dev),
                  base.dx, base.dy, config=SWEConfig(**base.config), train_dem=False,
                  arithmetic=arithmetic)
    if base.bc_times is not None:
        model.set_dynamic_boundary(torch.from_numpy(base.bc_times).to(dev),
                                   torch.from_numpy(base.bc_levels).to(dev))
    with torch.no_grad():
        U, _ = model(torch.from_numpy(base.U0).to(dev), t_end=float(seconds), start_time=0.0)
    U0 = U.cpu().numpy().astype(np.float32)
    return Scenario(f"{base.name}_at_{seconds:g}s", base.bed, base.roughness, U0, base.dx, base.dy,
                    dict(base.config), base.bc_times, base.bc_levels, base.steps,
                    dict(base.meta, start_time=float(seconds), spun_up_from=base.name))


#: simulated seconds of the runup scenario before it is tiled into the
#: throughput workload: the N-wave's trough has run down the beach and its
#: crest is arriving (waves and wet/dry fronts across the domain)
WORKLOAD_SPIN_UP_S = 8.0


WORKLOAD_STATE = Path(__file__).resolve().parent / "data" / "runup_state_8s.npz"


def runup_at_spin_up() -> Scenario:
    """The 244x393 runup scenario (seed 0) at WORKLOAD_SPIN_UP_S seconds: its
    state then is stored in ``data/runup_state_8s.npz`` (computed by the
    reference's step, see tests/golden/make_workload_state.py), so no GPU
    is needed to build the workload."""
    base = runup(seed=0)
    d = np.load(WORKLOAD_STATE)
    if float(d["seconds"]) != WORKLOAD_SPIN_UP_S or d["U"].shape != base.U0.shape:
        raise ValueError(f"{WORKLOAD_STATE} does not hold the runup state at {WORKLOAD_SPIN_UP_S} s")
    return Scenario(f"{base.name}_at_{WORKLOAD_SPIN_UP_S:g}s", base.bed, base.roughness,
                    np.ascontiguousarray(d["U"], dtype=np.float32), base.dx, base.dy,
                    dict(base.config), base.bc_times, base.bc_levels, base.steps,
                    dict(base.meta, start_time=WORKLOAD_SPIN_UP_S, spun_up_from=base.name,
                         spin_up_steps=int(d["steps"])))


def throughput_workload(ny: int = 4096, nx: int = 4096) -> Scenario:
    """The throughput workload: the runup scenario after WORKLOAD_SPIN_UP_S
    seconds (waves, wet/dry fronts) tiled (bed, roughness and state) to
    ny x nx; its boundary series continues from that time
    (``meta["start_time"]``)."""
    return tiled(runup_at_spin_up(), ny, nx)
