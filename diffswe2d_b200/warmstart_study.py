"""Learned warm start against the plain inversion.

1. Training runs: ``count`` forward runs of a RunupFamily with random spline
   inflows (controls uniform in [-0.012, 0.015] m) and random bathymetry
   perturbations, generated by the persistent ensemble kernel (interval
   mode, gauges every ``dt_out``).
2. The network (``warmstart.WarmStartNet``) is trained on (gauge series ->
   normalised controls) with its own kernels.
3. Held-out cases (their own seeds) are inverted twice with the same Adam
   settings: from the reference's cold start (every control at the initial
   boundary value 0.0 m, ``bc_inversion_train.py:632-636``) and from the
   network's prediction.  Reported: iterations and wall time until each
   case's gauge RMSE is at most the tolerance.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np
import torch

from .inversion import RunupFamily, invert, raw_from_controls
from .warmstart import WarmStartNet, normalise_controls


@dataclass
class Dataset:
    x: torch.Tensor          # [count, gauges, n_out] gauge eta (m)
    y: torch.Tensor          # [count, n_controls] control values (m)
    seconds: float
    cell_updates: int


def generate(fam: RunupFamily, count: int, seed: int, rows: Optional[int] = None) -> Dataset:
    rng = np.random.default_rng(seed)
    xs, ys, cells = [], [], 0
    t0 = time.perf_counter()
    for s in range(0, count, 1024):
        m = min(1024, count - s)
        beds = fam.beds(m, rng)
        values = fam.controls(m, rng)
        g = fam.ensemble_gauges(beds, values, rows=rows)   # [m, n_out, G]
        xs.append(g.transpose(1, 2).contiguous())
        ys.append(torch.as_tensor(values, device=g.device))
        cells += fam.last_ensemble.cell_updates
    torch.cuda.synchronize()
    return Dataset(torch.cat(xs), torch.cat(ys), time.perf_counter() - t0, cells)


@dataclass
class TrainLog:
    epochs: int
    steps: int
    seconds: float
    train_loss: List[float] = field(default_factory=list)
    val_loss: List[float] = field(default_factory=list)
    val_rmse_m: float = 0.0      # control RMSE on the validation split (m)


def train(net: WarmStartNet, data: Dataset, epochs: int = 30, batch: int = 256, lr: float = 1e-3,
          val_frac: float = 0.05, seed: int = 0) -> TrainLog:
    n = data.x.shape[0]
    nval = max(1, int(n * val_frac))
    g = torch.Generator(device=data.x.device).manual_seed(seed)
    perm = torch.randperm(n, device=data.x.device, generator=g)
    val, tr = perm[:nval], perm[nval:]
    y_norm = normalise_controls(data.y)
    log = TrainLog(epochs, 0, 0.0)
    t0 = time.perf_counter()
    for ep in range(epochs):
        order = tr[torch.randperm(tr.numel(), device=tr.device, generator=g)]
        lr_ep = lr * 0.5 * (1 + np.cos(np.pi * ep / epochs))  # cosine schedule
        tot = torch.zeros((), device=data.x.device)
        nb = 0
        for s in range(0, order.numel() - batch + 1, batch):
            idx = order[s:s + batch]
            tot += net.train_step(data.x[idx].contiguous(), y_norm[idx].contiguous(), lr=lr_ep)[0]
            nb += 1
            log.steps += 1
        log.train_loss.append(float(tot) / max(nb, 1))
        pred = net.predict_controls(data.x[val].contiguous())
        log.val_loss.append(float(((normalise_controls(pred) - y_norm[val]) ** 2).mean()))
    torch.cuda.synchronize()
    net.check_errors()
    log.seconds = time.perf_counter() - t0
    pred = net.predict_controls(data.x[val].contiguous())
    log.val_rmse_m = float(((pred - data.y[val]) ** 2).mean().sqrt())
    return log


def compare(fam: RunupFamily, net: WarmStartNet, cases: int, seed: int, lr: float = 0.002,
            max_iters: int = 400, tol: float = 1e-4, extra_cold_lrs=()) -> Dict:
    """Cold and warm inversions of `cases` held-out cases (batched), both
    with Adam at `lr`; `extra_cold_lrs` adds cold-start runs at other
    learning rates (e.g. 0.02, the inversion script's own setting)."""
    rng = np.random.default_rng(seed)
    beds = fam.beds(cases, rng)
    truth = fam.controls(cases, rng)
    problem = fam.problem(beds, truth)
    B = cases
    cold_raw = raw_from_controls(torch.zeros((B, fam.n_controls), device=problem.U0.device))
    res_cold = invert(problem, cold_raw, lr=lr, max_iters=max_iters, rmse_tol=tol)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    pred = net.predict_controls(problem.targets.transpose(1, 2).contiguous())
    eps = 1e-4
    warm_raw = raw_from_controls(pred.clamp(problem.lo + eps, problem.hi - eps))
    torch.cuda.synchronize()
    t_inf = time.perf_counter() - t0
    res_warm = invert(problem, warm_raw, lr=lr, max_iters=max_iters, rmse_tol=tol)
    truth_t = torch.as_tensor(truth, device=pred.device)
    extra = {}
    for lr2 in extra_cold_lrs:
        extra[f"cold_lr{lr2:g}"] = _summary(
            invert(problem, cold_raw, lr=lr2, max_iters=max_iters, rmse_tol=tol), 0.0)
    return {
        **extra,
        "cases": B,
        "tol_m": tol,
        "lr": lr,
        "max_iters": max_iters,
        "inference_s": t_inf,
        "pred_control_rmse_m": float(((pred - truth_t) ** 2).mean().sqrt()),
        "cold": _summary(res_cold, 0.0),
        "warm": _summary(res_warm, t_inf),
    }


def _summary(res, extra_s: float) -> Dict:
    its = res.iterations_to_tol
    reached = [i for i in its if i is not None]
    return {
        "iterations": its,
        "reached": len(reached),
        "median_iterations": float(np.median(reached)) if reached else None,
        "seconds_per_iteration": res.seconds_per_iteration,
        "seconds_to_tol": [None if s is None else s + extra_s for s in res.seconds_to_tol],
        "wall_seconds": res.wall_seconds + extra_s,
        "initial_rmse": res.rmse_history[0],
        "final_rmse": res.rmse_history[-1],
    }


__all__ = ["Dataset", "generate", "train", "compare", "TrainLog"]
