"""The persistent ensemble kernel against each scenario run alone.

Scenarios of different grid sizes, configurations and step counts run in one
launch; every scenario's final state, step count and simulated time must be
bit for bit those of SWE2D.step run on that scenario by itself (its own CFL
time steps and its own boundary series).
"""
import pytest
import torch

from diffswe2d_b200 import SWE2D, SWEConfig, scenarios
from diffswe2d_b200.autotune import ROW_CHOICES, size_class, tuned_rows
from diffswe2d_b200.ensemble import Ensemble

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def _members():
    sizes = [(40, 70), (128, 96), (33, 200), (200, 150), (64, 64), (257, 131)]
    out = []
    for k, (ny, nx) in enumerate(sizes):
        sc = scenarios.ensemble_member(ny, nx, seed=100 + k)
        sc.steps = 12 + 5 * k
        out.append(sc)
    return out


def _alone(sc):
    cfg = SWEConfig(**sc.config)
    m = SWE2D(torch.from_numpy(sc.bed).to(DEV), torch.from_numpy(sc.roughness).to(DEV), sc.dx, sc.dy,
              config=cfg, train_dem=False)
    if sc.bc_times is not None:
        m.set_dynamic_boundary(torch.from_numpy(sc.bc_times).to(DEV),
                               torch.from_numpy(sc.bc_levels).to(DEV))
    U, t = torch.from_numpy(sc.U0).to(DEV), 0.0
    with torch.no_grad():
        for _ in range(sc.steps):
            level = m._resolve_boundary_level(t, U, None)
            U, dt = m.step(U, t, 1.0e9, boundary_level=level)
            t += dt
    return U, t


@pytest.mark.parametrize("rows", [None, 16])
def test_ensemble_matches_each_scenario_alone(rows):
    members = _members()
    ens = Ensemble(members, device=DEV, rows=rows, track_hmax=True)
    res = ens.run()
    for m, sc in enumerate(members):
        U, t = _alone(sc)
        assert res.steps[m] == sc.steps
        assert res.times[m] == t
        assert torch.equal(res.states[m], U), f"scenario {m} ({sc.bed.shape})"
    # a second replay of the captured graph gives the same result
    res2 = ens.run()
    for a, b in zip(res.states, res2.states):
        assert torch.equal(a, b)
    assert res.mcells_per_s > 0


def test_size_classes_and_default_rows():
    assert size_class(1000) == 0 and size_class(1 << 17) == 1 and size_class(1 << 30) == 3
    assert tuned_rows(96 * 96, DEV) in ROW_CHOICES


def test_gauge_ensemble_matches_gauge_run_per_member():
    """Interval mode: each member's gauges and final state are bit for bit
    those of gauge_run on that member alone (its own CFL steps)."""
    from diffswe2d_b200.ensemble import GaugeEnsemble
    from diffswe2d_b200.gauge_run import gauge_run
    sc = scenarios.runup(ny=61, nx=98, dx=0.056, seed=5)
    cfg = SWEConfig(**sc.config)
    M, n_out, out_dt = 3, 9, 0.3
    base = torch.from_numpy(sc.bed).to(DEV)
    bed = torch.stack([base + 0.003 * m for m in range(M)]).contiguous()
    h0 = torch.clamp(-bed, min=0.0)
    U0 = torch.stack([h0, torch.zeros_like(h0), torch.zeros_like(h0)], dim=1).contiguous()
    t = torch.arange(n_out, device=DEV, dtype=torch.float32)
    levels = torch.stack([0.01 * torch.sin(0.5 * t + m) for m in range(M)]).contiguous()
    gauges = [(10, 20), (30, 40), (50, 10)]
    n = torch.from_numpy(sc.roughness).to(DEV)[None]
    ens = GaugeEnsemble(bed, n, U0, levels, out_dt, gauges, cfg, sc.dx)
    res = ens.run()
    for m in range(M):
        model = SWE2D(bed[m], n[0], sc.dx, sc.dy, config=cfg, train_dem=False)
        with torch.no_grad():
            g, U = gauge_run(model, U0[m:m + 1], levels[m], out_dt, gauges)
        assert torch.equal(res.gauges[m], g[0]), f"member {m}"
        assert torch.equal(res.states[m], U[0])
    res2 = ens.run()
    assert torch.equal(res.gauges, res2.gauges)
    capped = GaugeEnsemble(bed, n, U0, levels, out_dt, gauges, cfg, sc.dx, max_steps=5)
    with pytest.raises(RuntimeError, match="step cap"):
        capped.run()


def test_nan_member_fails_alone():
    """A member that starts with a NaN fails by itself (status non-finite
    state); every other member runs to its end, bit for bit as alone."""
    members = _members()[:4]
    bad = 2
    members[bad].U0 = members[bad].U0.copy()
    members[bad].U0[0, 0, 5, 7] = float("nan")
    res = Ensemble(members, device=DEV, rows=8).run(strict=False)
    assert res.failed == [bad]
    assert res.status[bad] & 1  # SWE_S_NONFINITE_STATE
    for m, sc in enumerate(members):
        if m == bad:
            continue
        U, t = _alone(sc)
        assert res.steps[m] == sc.steps and res.status[m] == 0
        assert torch.equal(res.states[m], U), f"scenario {m}"
    with pytest.raises(FloatingPointError, match="scenario 2"):
        Ensemble(members, device=DEV, rows=8).run()


def test_idle_limit_surfaces_as_error_and_kernel_returns():
    """The persistent kernel's idle limit at one microsecond: blocks that find
    no work see no phase completed within it (a phase takes longer), set the
    launch's error bit and leave; the launch ends and the error surfaces as
    a Python exception.  The same ensemble with the default limit runs."""
    sc = scenarios.ensemble_member(96, 96, seed=7)
    sc.steps = 40
    with pytest.raises(RuntimeError, match="idle limit"):
        Ensemble([sc], device=DEV, rows=8, stall_ns=1000).run()
    res = Ensemble([sc], device=DEV, rows=8).run()
    assert res.steps == [40]
