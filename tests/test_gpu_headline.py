"""Parity on the throughput workload itself: the 244x393 runup scenario after
8 s of simulated time (waves and wet/dry fronts), tiled to 4096x4096
(16.8 M cells, state and inputs larger than L2), at the tile height the
autotuner picks for that size -- the launch that bench.py times.

* IEEE kernels: three steps equal the CPU oracle bit for bit (state and dt),
  at the tuned tile height and at the smallest one.
* Tolerance-mode kernels: the same three steps within 1e-5 (depth) and 1e-4
  (momenta) of the oracle, normwise, with the oracle's wet/dry mask.
"""
import numpy as np
import pytest
import torch

from conftest import field_errors, wet_mask
from oracle import OracleSWE

from diffswe2d_b200 import SWE2D, SWEConfig, autotune, scenarios
from diffswe2d_b200 import _native as nat

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda", 0)
STEPS = 3


@pytest.fixture(scope="module")
def workload():
    autotune.tune(DEV)  # the tile heights bench.py uses (cached per device)
    autotune.tune(DEV, arithmetic="fast")
    sc = scenarios.throughput_workload(4096, 4096)
    cfg = SWEConfig(**sc.config)
    t0 = sc.meta["start_time"]
    om = OracleSWE(sc.bed, sc.roughness, sc.dx, sc.dy, cfg)
    om.set_dynamic_boundary(sc.bc_times, sc.bc_levels)
    U, t, states, dts = sc.U0, t0, [], []
    for _ in range(STEPS):
        U, dt = om.step(U, t, 1.0e9, boundary_level=om.interpolate_boundary(t))
        t += dt
        states.append(U)
        dts.append(dt)
    return sc, cfg, states, dts


def _gpu_steps(sc, cfg, arithmetic, rows):
    m = SWE2D(torch.from_numpy(sc.bed).to(DEV), torch.from_numpy(sc.roughness).to(DEV), sc.dx, sc.dy,
              config=cfg, train_dem=False, arithmetic=arithmetic)
    m.set_dynamic_boundary(torch.from_numpy(sc.bc_times).to(DEV), torch.from_numpy(sc.bc_levels).to(DEV))
    lib = nat.lib()
    prev = int(lib.swe_sweep_rows())
    nat.check(lib.swe_tune_sweep_rows(rows), "rows")
    try:
        U, t, out = torch.from_numpy(sc.U0).to(DEV), sc.meta["start_time"], []
        with torch.no_grad():
            for _ in range(STEPS):
                U, dt = m.step(U, t, 1.0e9, boundary_level=m._interpolate_dynamic_boundary(t, U))
                t += dt
                out.append((U.cpu().numpy(), dt))
    finally:
        nat.check(lib.swe_tune_sweep_rows(prev), "rows")
    return out


def test_stored_spun_up_state_is_what_the_kernels_compute():
    """The workload's stored initial state (the runup scenario at 8 s,
    computed on the CPU) equals SWE2D.forward's IEEE kernels run for 8 s
    from the scenario's initial state, bit for bit."""
    sc = scenarios.spun_up(scenarios.runup(seed=0), scenarios.WORKLOAD_SPIN_UP_S, DEV)
    stored = scenarios.runup_at_spin_up()
    assert np.array_equal(sc.U0.view(np.uint32), stored.U0.view(np.uint32))


def test_workload_is_not_at_rest(workload):
    sc, _, _, _ = workload
    assert sc.bed.shape == (4096, 4096)
    speed = np.abs(sc.U0[0, 1]).max()
    wet = (sc.U0[0, 0] > 1e-6).mean()
    assert speed > 1e-3 and 0.2 < wet < 0.95


@pytest.mark.parametrize("which", ["tuned", "smallest"])
def test_ieee_kernels_bitwise_on_workload(workload, which):
    sc, cfg, states, dts = workload
    rows = autotune.tuned_rows(4096 * 4096, DEV) if which == "tuned" else autotune.ROW_CHOICES[0]
    for k, (U, dt) in enumerate(_gpu_steps(sc, cfg, "exact", rows)):
        assert dt == dts[k], f"step {k + 1}: dt differs (rows {rows})"
        assert np.array_equal(U.view(np.uint32), states[k].view(np.uint32)), f"step {k + 1} (rows {rows})"


def test_fast_kernels_on_workload(workload):
    sc, cfg, states, dts = workload
    rows = autotune.tuned_rows(4096 * 4096, DEV, "fast")
    out = _gpu_steps(sc, cfg, "fast", rows)
    for k, (U, dt) in enumerate(out):
        assert abs(dt - dts[k]) <= 1e-5 * dts[k]
    U = out[-1][0]
    err = field_errors(U, states[-1])
    print("fast vs oracle on the 4096^2 workload after", STEPS, "steps:", err,
          "wet cells differing:", int((wet_mask(U) != wet_mask(states[-1])).sum()))
    assert err[0] <= 1e-5 and err[1] <= 1e-4 and err[2] <= 1e-4
    assert np.array_equal(wet_mask(U), wet_mask(states[-1]))
