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

import time
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np
import torch

from .adjoint import forward_checkpointed
from .gauge_run import gauge_run


# ------------------------------------------------------------------ spline
def clamped_bspline_basis(sample_times: torch.Tensor, number_of_controls: int, degree: int = 3):
    """Basis matrix [T, n], knot vector and Greville abscissae of the clamped
    B-spline the reference's inversion script uses (bc_inversion_train.py:
    189-231): ``degree + 1`` repeated knots at the first and last sample
    time, ``n - degree - 1`` uniform interior knots.  The basis is SciPy's
    B-spline design matrix (de Boor's algorithm) on the sample times, the
    last sample belonging to the last interval, so every row sums to one;
    the Greville abscissa of control i is the mean of knots i+1 .. i+degree."""
    from scipy.interpolate import BSpline
    if degree < 1:
        raise ValueError(f"degree must be at least 1, got {degree}")
    if number_of_controls < degree + 1:
        raise ValueError(f"a degree-{degree} spline needs at least {degree + 1} controls, "
                         f"got {number_of_controls}")
    if sample_times.ndim != 1 or sample_times.numel() < 2:
        raise ValueError("sample_times must be 1-D with at least two times")
    t = sample_times.detach().to(torch.float64).cpu().numpy()
    interior = np.linspace(t[0], t[-1], number_of_controls - degree + 1)[1:-1]
    knots = np.concatenate([np.full(degree + 1, t[0]), interior, np.full(degree + 1, t[-1])])
    basis = BSpline.design_matrix(t, knots, degree, extrapolate=False).toarray()
    if not np.allclose(basis.sum(axis=1), 1.0, rtol=0, atol=1e-10):
        raise RuntimeError("the B-spline basis rows do not sum to one")
    greville = np.array([knots[i + 1:i + degree + 1].mean() for i in range(number_of_controls)])
    dev = sample_times.device
    return (torch.from_numpy(basis).to(dev), torch.from_numpy(knots).to(dev),
            torch.from_numpy(greville).to(dev))


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
    checkpoint_every: Optional[int] = None  # None: the autotuner's choice for this run

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
        level is series[:, i] (held over the chunk, as the reference does).
        One gauge_run: a device-driven run with a checkpointed adjoint."""
        if differentiable:
            if self.checkpoint_every is None:
                from .autotune import tuned_checkpoint_every
                self.checkpoint_every = tuned_checkpoint_every(self.model, self.U0, series,
                                                               self.dt_out, self.gauges)
            return gauge_run(self.model, self.U0, series, self.dt_out, self.gauges,
                             checkpoint_every=self.checkpoint_every)[0]
        # a forward-only run keeps no segments: k only sets the checkpoint copies
        from .gauge_run import CHECKPOINT_EVERY
        with torch.no_grad():
            return gauge_run(self.model, self.U0, series.detach(), self.dt_out, self.gauges,
                             checkpoint_every=self.checkpoint_every or CHECKPOINT_EVERY)[0]

    def simulate_chunked(self, series: torch.Tensor, differentiable: bool = True) -> torch.Tensor:
        """The same run as the reference's script writes it: one forward()
        call (one autograd node, forward_checkpointed) per output chunk."""
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
        losses.append(float(mse.sum().detach()))
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


@dataclass
class RunupFamily:
    """The runup cases of one resolution: the runup bathymetry of the
    scenario recipe (seeded) perturbed per case by three seeded Gaussian
    bumps of amplitude up to ``bathy_perturb`` metres, walls except the west
    water level, Manning n = 0.01, still water at rest; gauges at
    ``n_gauges`` seeded cells deeper than 3 cm in the unperturbed bed (the
    same cells for every case); a clamped cubic spline of ``n_controls``
    controls sampled every ``dt_out`` seconds over ``duration``."""
    ny: int = 122
    nx: int = 196
    dx: float = 0.028
    seed: int = 0
    duration: float = 22.5
    dt_out: float = 0.02
    n_controls: int = 16
    n_gauges: int = 6
    bathy_perturb: float = 0.01
    device: str = "cuda"
    arithmetic: str = "exact"  # step kernels of the runs and inversions ("exact" or "fast")

    def __post_init__(self):
        from . import scenarios
        from .config import SWEConfig
        self.base = scenarios.runup(ny=self.ny, nx=self.nx, dx=self.dx, seed=self.seed)
        self.config = SWEConfig(**self.base.config)
        rng = np.random.default_rng(self.seed + 7919)
        wet = np.argwhere(self.base.bed < -0.03)
        pick = rng.choice(len(wet), size=self.n_gauges, replace=False)
        self.gauges = [tuple(int(v) for v in wet[i]) for i in sorted(pick)]
        self.n_out = int(round(self.duration / self.dt_out))
        times = torch.arange(self.n_out, dtype=torch.float64) * self.dt_out
        basis, _, _ = clamped_bspline_basis(times, self.n_controls, 3)
        self.basis = basis.float().to(self.device)

    def beds(self, count: int, rng) -> np.ndarray:
        """[count, ny, nx] float32 perturbed beds."""
        X, Y = np.meshgrid((np.arange(self.nx) + 0.5) * self.dx, (np.arange(self.ny) + 0.5) * self.dx)
        out = np.empty((count, self.ny, self.nx), np.float32)
        for c in range(count):
            z = self.base.bed.astype(np.float64).copy()
            if self.bathy_perturb > 0:
                for _ in range(3):
                    cx = rng.uniform(0.1, 0.9) * self.nx * self.dx
                    cy = rng.uniform(0.1, 0.9) * self.ny * self.dx
                    amp = rng.uniform(-self.bathy_perturb, self.bathy_perturb)
                    sig = rng.uniform(0.05, 0.2)
                    z += amp * np.exp(-((X - cx) ** 2 + (Y - cy) ** 2) / (2 * sig ** 2))
            out[c] = z
        return out

    def controls(self, count: int, rng) -> np.ndarray:
        """[count, n_controls] control values uniform in [-0.012, 0.015] m."""
        return rng.uniform(-0.012, 0.015, size=(count, self.n_controls)).astype(np.float32)

    def problem(self, beds: np.ndarray, truth: Optional[np.ndarray] = None):
        """InversionProblem over the cases of `beds` (batched); targets from
        the forward run with control values `truth`, if given."""
        from .solver import SWE2D
        bed = torch.tensor(beds[:, None], device=self.device)
        n = torch.full_like(bed, 0.01)
        model = SWE2D(bed, n, self.dx, self.dx, config=self.config, train_dem=False,
                      arithmetic=self.arithmetic)
        h0 = torch.clamp(-bed, min=0.0)
        U0 = torch.cat([h0, torch.zeros_like(h0), torch.zeros_like(h0)], dim=1).contiguous()
        problem = InversionProblem(model, U0, self.gauges, self.dt_out, self.n_out, self.basis)
        if truth is not None:
            raw = raw_from_controls(torch.as_tensor(truth, device=self.device))
            with torch.no_grad():
                problem.targets = problem.simulate(problem.series(raw), differentiable=False)
        return problem

    def ensemble_gauges(self, beds: np.ndarray, values: np.ndarray, rows: Optional[int] = None):
        """Gauge eta [count, n_out, n_gauges] of independent runs (each its own
        CFL steps), in persistent-kernel launches of up to 1024 runs."""
        from .ensemble import GaugeEnsemble
        out = []
        n = torch.full((1, self.ny, self.nx), 0.01, device=self.device)
        for s in range(0, beds.shape[0], 1024):
            bed = torch.tensor(beds[s:s + 1024], device=self.device)
            h0 = torch.clamp(-bed, min=0.0)
            U0 = torch.stack([h0, torch.zeros_like(h0), torch.zeros_like(h0)], dim=1).contiguous()
            v = torch.as_tensor(values[s:s + 1024], device=self.device)
            levels = (v @ self.basis.t()).contiguous()
            ens = GaugeEnsemble(bed, n, U0, levels, self.dt_out, self.gauges, self.config, self.dx,
                                rows=rows, arithmetic=self.arithmetic)
            res = ens.run()
            out.append(res.gauges)
            self.last_ensemble = res
            del ens
        return torch.cat(out)


def make_runup_problem(cases: int = 4, seed: int = 0, ny: int = 122, nx: int = 196,
                       dx: float = 0.028, duration: float = 22.5, dt_out: float = 0.1,
                       n_controls: int = 16, n_gauges: int = 6, device="cuda",
                       bathy_perturb: float = 0.01, arithmetic: str = "exact"):
    """Config 3 at a chosen resolution (a RunupFamily): `cases` perturbed beds
    and seeded true controls.  Returns (problem, true raw controls
    [cases, n_controls])."""
    fam = RunupFamily(ny, nx, dx, seed, duration, dt_out, n_controls, n_gauges, bathy_perturb,
                      str(device), arithmetic)
    rng = np.random.default_rng(seed)
    beds = fam.beds(cases, rng)
    truth = fam.controls(cases, rng)
    problem = fam.problem(beds, truth)
    return problem, raw_from_controls(torch.as_tensor(truth, device=device))


__all__ = ["clamped_bspline_basis", "bounded_controls", "raw_from_controls", "InversionProblem",
           "InversionResult", "invert", "gauge_rmse", "make_runup_problem", "RunupFamily"]
