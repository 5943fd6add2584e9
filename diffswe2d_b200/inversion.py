"""Boundary-inflow inversion on the B200 step and its hand-written adjoint.

Restates the inversion workflow of the reference's example
``Examples/inverse/**/bc_inversion_train.py``: the west-edge water level is a
clamped cubic B-spline of a few controls bounded by a sigmoid (``:165-242``),
the model runs in output chunks with the chunk's spline value as the
boundary level (``:332-411``), gauges read eta = h + bed at gauge cells after
each chunk, the loss is the mean squared gauge misfit (``:427-452``) and Adam
updates the raw controls (``:637-720``).  Differences: many cases (one per
batch member, each with its own bed, controls and targets) are inverted at
once; gradients come from ``adjoint.forward_checkpointed`` (one checkpoint per
chunk, states recomputed in the backward pass); regularisation terms and
gradient clipping of the reference script are optional and off by default.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np
import torch

from .adjoint import forward_checkpointed


# ------------------------------------------------------------------ spline
def clamped_bspline_basis(sample_times: torch.Tensor, number_of_controls: int, degree: int = 3):
    """Basis matrix [T, n], knot vector and Greville abscissae of a clamped
    B-spline with uniform interior knots, by the Cox-de Boor recursion
    (bc_inversion_train.py:189-231).  The last sample is assigned to the last
    basis function so every row sums to one."""
    if degree < 1 or number_of_controls < degree + 1:
        raise ValueError("Require degree >= 1 and number_of_controls >= degree + 1.")
    if sample_times.ndim != 1 or sample_times.numel() < 2:
        raise ValueError("sample_times must be a one-dimensional tensor with at least two values.")
    t = sample_times.to(torch.float64)
    t0, t1 = t[0], t[-1]
    n_int = number_of_controls - degree - 1
    interior = (torch.linspace(float(t0), float(t1), n_int + 2, dtype=torch.float64)[1:-1]
                if n_int > 0 else t.new_empty(0))
    knots = torch.cat((t0.repeat(degree + 1), interior, t1.repeat(degree + 1)))
    x = t[:, None]
    basis = ((x >= knots[:-1]) & (x < knots[1:])).to(torch.float64)
    eps = torch.finfo(torch.float64).eps
    for order in range(1, degree + 1):
        cols = knots.numel() - order - 1
        ld = knots[order:order + cols] - knots[:cols]
        rd = knots[order + 1:order + 1 + cols] - knots[1:1 + cols]
        left = torch.where(ld > 0, (x - knots[:cols]) / ld.clamp_min(eps), 0.0)
        right = torch.where(rd > 0, (knots[order + 1:order + 1 + cols] - x) / rd.clamp_min(eps), 0.0)
        basis = left * basis[:, :cols] + right * basis[:, 1:cols + 1]
    basis[-1].zero_()
    basis[-1, -1] = 1.0
    if not torch.allclose(basis.sum(1), torch.ones(basis.shape[0], dtype=torch.float64),
                          atol=1e-10, rtol=1e-10):
        raise RuntimeError("B-spline basis does not form a partition of unity.")
    greville = torch.stack([knots[i + 1:i + degree + 1].mean() for i in range(number_of_controls)])
    return basis, knots, greville


BC_MINIMUM, BC_MAXIMUM = -0.02, 0.05


def bounded_controls(raw: torch.Tensor, lo: float = BC_MINIMUM, hi: float = BC_MAXIMUM):
    """lo + (hi - lo) sigmoid(raw) (bc_inversion_train.py:181-182)."""
    return lo + (hi - lo) * torch.sigmoid(raw)


def raw_from_controls(values: torch.Tensor, lo: float = BC_MINIMUM, hi: float = BC_MAXIMUM):
    """Inverse of bounded_controls, clamped inside the open interval."""
    eps = torch.finfo(values.dtype).eps
    frac = ((values - lo) / (hi - lo)).clamp(eps, 1.0 - eps)
    return torch.logit(frac)


# ------------------------------------------------------------------ problem
@dataclass
class InversionProblem:
    """``model`` holds the cases in its batch (bed [B,1,ny,nx] or shared);
    gauges are (row, column) cells; ``n_out`` output chunks of ``dt_out``
    seconds; ``basis`` maps controls to the chunk levels."""
    model: "object"
    U0: torch.Tensor                      # [B,3,ny,nx]
    gauges: Sequence[Tuple[int, int]]
    dt_out: float
    n_out: int
    basis: torch.Tensor                   # [n_out, n_controls] float32 on the device
    targets: Optional[torch.Tensor] = None  # [B, n_out, n_gauges]
    lo: float = BC_MINIMUM
    hi: float = BC_MAXIMUM

    @property
    def batch(self) -> int:
        return int(self.U0.shape[0])

    def series(self, raw: torch.Tensor) -> torch.Tensor:
        """Chunk levels [B, n_out] from raw controls [B, n_controls]."""
        return bounded_controls(raw, self.lo, self.hi) @ self.basis.t()

    def gauge_eta(self, U: torch.Tensor) -> torch.Tensor:
        bed = self.model.bed.detach()
        B = U.shape[0]
        vals = []
        for iy, ix in self.gauges:
            z = bed[:, 0, iy, ix] if bed.shape[0] == B else bed[0, 0, iy, ix].expand(B)
            vals.append(U[:, 0, iy, ix] + z)
        return torch.stack(vals, dim=-1)  # [B, n_gauges]

    def simulate(self, series: torch.Tensor, differentiable: bool = True) -> torch.Tensor:
        """Gauge eta [B, n_out, n_gauges] after each output chunk; the chunk's
        level is series[:, i] (held over the chunk, as the reference does)."""
        U = self.U0
        out = []
        for i in range(self.n_out):
            if differentiable:
                U = forward_checkpointed(self.model, U, t_end=self.dt_out, start_time=i * self.dt_out,
                                         boundary_level=series[:, i])
            else:
                with torch.no_grad():
                    U, _ = self.model(U, t_end=self.dt_out, start_time=i * self.dt_out,
                                      boundary_level=series[:, i])
            out.append(self.gauge_eta(U))
        return torch.stack(out, dim=1)


@dataclass
class InversionResult:
    raw: torch.Tensor                      # final raw controls [B, n_controls]
    iterations_to_tol: List[Optional[int]]  # per case, None if not reached
    rmse_history: List[List[float]]        # per iteration, per case
    seconds_per_iteration: float
    seconds_to_tol: List[Optional[float]]
    wall_seconds: float = 0.0
    losses: List[float] = field(default_factory=list)


def gauge_rmse(sim: torch.Tensor, targets: torch.Tensor) -> torch.Tensor:
    """Per-case RMSE [B] over all chunks and gauges."""
    return ((sim - targets) ** 2).mean(dim=(1, 2)).sqrt()


def invert(problem: InversionProblem, raw0: torch.Tensor, lr: float = 0.002, max_iters: int = 200,
           rmse_tol: float = 1e-4, stop_when_all_converged: bool = True,
           log_every: int = 0) -> InversionResult:
    """Adam on the raw spline controls of every case until each case's gauge
    RMSE is at most ``rmse_tol`` metres (or ``max_iters``).  The loss is the
    sum over cases of each case's mean squared gauge misfit, so each case's
    controls see their own MSE gradient."""
    if problem.targets is None:
        raise ValueError("the problem has no targets")
    raw = raw0.detach().clone().to(problem.U0.device).requires_grad_(True)
    opt = torch.optim.Adam([raw], lr=lr)
    B = problem.batch
    reached: List[Optional[int]] = [None] * B
    history: List[List[float]] = []
    losses: List[float] = []
    t_start = time.perf_counter()
    for it in range(max_iters + 1):
        opt.zero_grad(set_to_none=True)
        sim = problem.simulate(problem.series(raw))
        mse = ((sim - problem.targets) ** 2).mean(dim=(1, 2))
        rmse = mse.detach().sqrt().cpu().tolist()
        history.append(rmse)
        losses.append(float(mse.sum()))
        for b in range(B):
            if reached[b] is None and rmse[b] <= rmse_tol:
                reached[b] = it
        if log_every and it % log_every == 0:
            print(f"iter {it:4d}  rmse " + " ".join(f"{r:.2e}" for r in rmse), flush=True)
        if it == max_iters or (stop_when_all_converged and all(r is not None for r in reached)):
            break
        mse.sum().backward()
        opt.step()
    wall = time.perf_counter() - t_start
    per_it = wall / max(len(history), 1)
    return InversionResult(raw.detach(), reached, history, per_it,
                           [None if r is None else r * per_it for r in reached], wall, losses)


def make_runup_problem(cases: int = 4, seed: int = 0, ny: int = 122, nx: int = 196,
                       dx: float = 0.028, duration: float = 22.5, dt_out: float = 0.1,
                       n_controls: int = 16, n_gauges: int = 6, device="cuda",
                       bathy_perturb: float = 0.01):
    """Config 3 at a chosen resolution: the runup bathymetry (each case with
    its own seeded Gaussian perturbation of the bed), walls except the west
    water level, Manning n = 0.01, still water at rest, 16-control spline over
    `duration` seconds sampled every `dt_out`, `n_gauges` seeded gauge cells
    in the wet part.  Returns (problem, true raw controls [cases, n_controls])."""
    from . import scenarios
    from .config import SWEConfig
    from .solver import SWE2D
    rng = np.random.default_rng(seed)
    base = scenarios.runup(ny=ny, nx=nx, dx=dx, seed=seed)
    beds = []
    for c in range(cases):
        z = base.bed.astype(np.float64).copy()
        if bathy_perturb > 0:
            X, Y = np.meshgrid((np.arange(nx) + 0.5) * dx, (np.arange(ny) + 0.5) * dx)
            for _ in range(3):
                cx, cy = rng.uniform(0.1, 0.9) * nx * dx, rng.uniform(0.1, 0.9) * ny * dx
                amp = rng.uniform(-bathy_perturb, bathy_perturb)
                sig = rng.uniform(0.05, 0.2)
                z += amp * np.exp(-((X - cx) ** 2 + (Y - cy) ** 2) / (2 * sig ** 2))
        beds.append(z.astype(np.float32))
    bed = torch.tensor(np.stack(beds)[:, None], device=device)
    n = torch.full_like(bed, 0.01)
    cfg = SWEConfig(**base.config)
    model = SWE2D(bed, n, dx, dx, config=cfg, train_dem=False)
    h0 = torch.clamp(-bed, min=0.0)
    U0 = torch.cat([h0, torch.zeros_like(h0), torch.zeros_like(h0)], dim=1).contiguous()
    wet = np.argwhere(np.stack(beds).max(0) < -0.03)
    pick = rng.choice(len(wet), size=n_gauges, replace=False)
    gauges = [tuple(int(v) for v in wet[i]) for i in pick]
    n_out = int(round(duration / dt_out))
    times = torch.arange(n_out, dtype=torch.float64) * dt_out
    basis, _, _ = clamped_bspline_basis(times, n_controls, 3)
    problem = InversionProblem(model, U0, gauges, dt_out, n_out, basis.float().to(device))
    truth = torch.tensor(rng.uniform(-0.012, 0.015, size=(cases, n_controls)), dtype=torch.float32,
                         device=device)
    raw_true = raw_from_controls(truth)
    with torch.no_grad():
        problem.targets = problem.simulate(problem.series(raw_true), differentiable=False)
    return problem, raw_true


__all__ = ["clamped_bspline_basis", "bounded_controls", "raw_from_controls", "InversionProblem",
           "InversionResult", "invert", "gauge_rmse", "make_runup_problem", "math"]
