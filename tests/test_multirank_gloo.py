"""The multi-GPU host logic on two CPU processes (gloo): every scenario of an
ensemble lands on exactly one rank, timings combine as the max over ranks
and work as the sum, and the CPU reference arm does its work on rank 0
only."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from diffswe2d_b200 import scenarios
from diffswe2d_b200.sharding import reduce_over_ranks, shard_indices


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sizes = scenarios.ensemble_sizes(64, seed=0)
        mine = shard_indices(len(sizes), world, rank)
        cells = sum(a * b for a, b in (sizes[k] for k in mine))
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        t_max = reduce_over_ranks([1.0 + rank, 10.0 * (rank + 1)], "max")
        work = reduce_over_ranks([cells], "sum")[0]
        out[rank] = (gathered, t_max, work, sum(a * b for a, b in sizes))
    finally:
        dist.destroy_process_group()


def test_sharding_and_reductions_on_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, start_method="spawn")
    for rank in range(2):
        gathered, t_max, work, total = out[rank]
        flat = sorted(i for part in gathered for i in part)
        assert flat == list(range(64))                       # each scenario once
        assert not set(gathered[0]) & set(gathered[1])
        assert t_max == [2.0, 20.0]                           # max over ranks
        assert work == total                                  # sum over ranks


def _fake_runs(beds, values):
    """Stand-in for the ensemble launch (CPU): gauges [m, n_out, 6] that
    depend on each run's bed and controls only."""
    m = beds.shape[0]
    base = torch.from_numpy(beds.reshape(m, -1).mean(axis=1) + values.sum(axis=1)).float()
    return base.view(m, 1, 1).expand(m, 1125, 6) + torch.arange(1125.0).view(1, 1125, 1)


def _gen_worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from diffswe2d_b200.inversion import RunupFamily
        from diffswe2d_b200.warmstart_study import generate
        fam = RunupFamily(ny=12, nx=20, dx=0.3, device="cpu")
        data = generate(fam, 37, seed=4, world=world, rank=rank, simulate=_fake_runs)
        out[rank] = (data.x.numpy(), data.y.numpy())
    finally:
        dist.destroy_process_group()


def test_training_runs_sharded_and_gathered_equal_one_rank():
    """Config 5's training runs on two ranks: each run is made on exactly one
    rank (run k's inputs depend on k only) and the gathered dataset equals
    the single-rank one, in run order, on both ranks."""
    import numpy as np
    from diffswe2d_b200.inversion import RunupFamily
    from diffswe2d_b200.warmstart_study import generate
    fam = RunupFamily(ny=12, nx=20, dx=0.3, device="cpu")
    ref = generate(fam, 37, seed=4, simulate=_fake_runs)
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    mp.start_processes(_gen_worker, args=(2, _free_port(), out), nprocs=2, start_method="spawn")
    for rank in range(2):
        x, y = out[rank]
        assert x.shape == (37, 6, 1125)
        assert np.array_equal(x, ref.x.numpy()) and np.array_equal(y, ref.y.numpy())
    assert shard_indices(37, 2, 0) == list(range(0, 37, 2))


def test_reductions_are_identity_without_a_process_group():
    assert reduce_over_ranks([3.0, 4.0], "max") == [3.0, 4.0]
    with pytest.raises(ValueError):
        shard_indices(10, 2, 2)


def test_reference_arm_runs_on_rank_zero_only(capsys):
    import bench
    ns = type("A", (), dict(ny=64, nx=64, steps=1, warmup=0, gpus=2))()
    assert bench.run_reference(ns, 2, 1) is None             # rank 1: no work, no line
    assert capsys.readouterr().out == ""
