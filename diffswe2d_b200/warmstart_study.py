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


def run_inputs(fam: RunupFamily, index: int, seed: int):
    """Bed [ny, nx] and control values [n_controls] of run `index`: drawn from
    a generator seeded by (seed, index), so a run does not depend on which
    rank makes it or in which batch."""
    rng = np.random.default_rng([seed, index])
    return fam.beds(1, rng)[0], fam.controls(1, rng)[0]


def generate(fam: RunupFamily, count: int, seed: int, rows: Optional[int] = None,
             world: int = 1, rank: int = 0, simulate=None) -> Dataset:
    """`count` training runs; with world > 1 each rank runs its round-robin
    share (no communication during the runs) and the dataset is gathered
    once at the end, in run order, on every rank -- the same dataset as one
    rank makes.  `simulate(beds, values) -> gauges [m, n_out, G]` defaults
    to the family's persistent ensemble launch."""
    from .sharding import gather_rows, shard_indices
    mine = shard_indices(count, world, rank)
    sim = simulate or (lambda b, v: fam.ensemble_gauges(b, v, rows=rows))
    xs, ys, cells = [], [], 0
    t0 = time.perf_counter()
    for s in range(0, len(mine), 1024):
        part = [run_inputs(fam, k, seed) for k in mine[s:s + 1024]]
        beds = np.stack([p[0] for p in part])
        values = np.stack([p[1] for p in part])
        g = sim(beds, values)   # [m, n_out, G]
        xs.append(g.transpose(1, 2).contiguous())
        ys.append(torch.as_tensor(values, device=g.device))
        if simulate is None:
            cells += fam.last_ensemble.cell_updates
    x = torch.cat(xs) if xs else None
    y = torch.cat(ys) if ys else None
    if torch.cuda.is_available():
        torch.cuda.synchronize()
    seconds = time.perf_counter() - t0
    if world > 1:
        x, y = gather_rows(count, mine, [x, y], world)
        from .sharding import reduce_over_ranks
        seconds = reduce_over_ranks([seconds], "max")[0]
        cells = int(reduce_over_ranks([cells], "sum")[0])
    return Dataset(x, y, seconds, cells)


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


def compare_at_scale(fam: RunupFamily, net: WarmStartNet, cases: int, seed: int, lr: float = 0.002,
                     tol: float = 1e-4, warm_max_iters: int = 20, cold_cases: int = 8,
                     cold_max_iters: int = 40, world: int = 1, rank: int = 0) -> Dict:
    """The comparison for grids where a batched adjoint iteration over every
    held-out case costs minutes: the warm start is evaluated on all `cases`
    (one batched forward run of the predicted controls; only the cases not
    yet within `tol` are inverted further, as a batch, for up to
    `warm_max_iters` iterations), the cold start on the first `cold_cases`
    of them for up to `cold_max_iters` iterations (its cost per case is the
    same for every case: each iteration is one forward + adjoint run).
    Held-out case c is drawn from a generator seeded by (seed, c); with
    world > 1 each rank takes its round-robin share of the cases and the
    per-case results are gathered once at the end.  Times are this rank's
    wall times, shared out per case of a batch."""
    from .sharding import shard_indices
    mine = shard_indices(cases, world, rank)
    recs = {}
    t_inf = 0.0
    if mine:
        inputs = [run_inputs(fam, c, seed) for c in mine]
        beds = np.stack([p[0] for p in inputs])
        truth = np.stack([p[1] for p in inputs])
        problem = fam.problem(beds, truth)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        pred = net.predict_controls(problem.targets.transpose(1, 2).contiguous())
        eps = 1e-4
        warm_vals = pred.clamp(problem.lo + eps, problem.hi - eps)
        torch.cuda.synchronize()
        t_inf = time.perf_counter() - t0
        t0 = time.perf_counter()
        with torch.no_grad():
            sim = problem.simulate(problem.series(raw_from_controls(warm_vals)), differentiable=False)
        rmse0 = ((sim - problem.targets) ** 2).mean(dim=(1, 2)).sqrt().cpu().numpy()
        torch.cuda.synchronize()
        per_case_eval = (time.perf_counter() - t0) / len(mine)
        err2 = ((pred - torch.as_tensor(truth, device=pred.device)) ** 2).sum(dim=1).cpu().numpy()
        for j, c in enumerate(mine):
            ok = bool(rmse0[j] <= tol)
            recs[c] = {"rmse0": float(rmse0[j]), "warm_it": 0 if ok else None,
                       "warm_s": t_inf / len(mine) + per_case_eval if ok else None,
                       "eval_s": per_case_eval, "err2": float(err2[j])}
        left = [j for j, c in enumerate(mine) if rmse0[j] > tol]
        if left and warm_max_iters > 0:
            sub = fam.problem(beds[left], truth[left])
            res = invert(sub, raw_from_controls(warm_vals[left]), lr=lr, max_iters=warm_max_iters,
                         rmse_tol=tol)
            for q, j in enumerate(left):
                r = recs[mine[j]]
                r["warm_iter_s"] = res.seconds_per_iteration / len(left)
                if res.iterations_to_tol[q] is not None:
                    r["warm_it"] = res.iterations_to_tol[q]
                    r["warm_s"] = t_inf / len(mine) + per_case_eval + res.seconds_to_tol[q] / len(left)
        cold_local = [j for j, c in enumerate(mine) if c < cold_cases]
        if cold_local:
            cold = fam.problem(beds[cold_local], truth[cold_local])
            raw0 = raw_from_controls(torch.zeros((len(cold_local), fam.n_controls),
                                                 device=problem.U0.device))
            rc = invert(cold, raw0, lr=lr, max_iters=cold_max_iters, rmse_tol=tol)
            for q, j in enumerate(cold_local):
                recs[mine[j]].update(cold_it=rc.iterations_to_tol[q],
                                     cold_iter_s=rc.seconds_per_iteration / len(cold_local),
                                     cold_rmse0=rc.rmse_history[0][q], cold_rmse=rc.rmse_history[-1][q])
    if world > 1:
        import torch.distributed as dist
        parts = [None] * world
        dist.all_gather_object(parts, (recs, t_inf))
        recs = {k: v for part, _ in parts for k, v in part.items()}
        t_inf = max(t for _, t in parts)
    order = list(range(cases))
    warm_iters = [recs[c]["warm_it"] for c in order]
    reached = [i for i in warm_iters if i is not None]
    cold = [recs[c] for c in order if "cold_it" in recs[c]]
    iter_s = [r["warm_iter_s"] for r in recs.values() if "warm_iter_s" in r]
    return {
        "cases": cases, "tol_m": tol, "lr": lr, "inference_s": t_inf,
        "pred_control_rmse_m": float(np.sqrt(sum(recs[c]["err2"] for c in order)
                                             / (cases * fam.n_controls))),
        "warm": {
            "reached": len(reached),
            "reached_at_iteration_0": int(sum(1 for i in warm_iters if i == 0)),
            "median_iterations": float(np.median(reached)) if reached else None,
            "iterations": warm_iters,
            "seconds_to_tol": [recs[c]["warm_s"] for c in order],
            "initial_rmse": [recs[c]["rmse0"] for c in order],
            "forward_eval_s_per_case": float(np.mean([recs[c]["eval_s"] for c in order])),
            "seconds_per_iteration_per_case": float(np.mean(iter_s)) if iter_s else None,
            "max_iters": warm_max_iters,
        },
        "cold": {
            "cases": len(cold), "max_iters": cold_max_iters,
            "reached": sum(1 for r in cold if r["cold_it"] is not None),
            "iterations": [r["cold_it"] for r in cold],
            "seconds_per_iteration_per_case": float(np.mean([r["cold_iter_s"] for r in cold]))
            if cold else None,
            "initial_rmse": [r["cold_rmse0"] for r in cold],
            "final_rmse": [r["cold_rmse"] for r in cold],
        },
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


__all__ = ["Dataset", "generate", "train", "compare", "compare_at_scale", "TrainLog"]
