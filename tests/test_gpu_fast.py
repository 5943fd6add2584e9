"""The tolerance-mode step kernels (SWE2D(..., arithmetic="fast"),
csrc/swe_fast.cu) against the reference.

The bar is the one the reference's own FP32 arithmetic sets: after 1000
steps of the 256x256 island case and 200 steps of the runup case every field
stays within 1.5x the reference's FP32-vs-FP64 difference of the FP64
reference (normwise, max|a-b| / max|b|), with the stock FP32 reference's
wet/dry mask; short runs on the operator fixtures and random states stay
within the normwise bounds written in each test of the CPU oracle.  Results
of the tolerance mode do not depend on the launch shape: an ensemble member
and the device-driven forward() loop equal the single step bit for bit.
"""
import numpy as np
import pytest
import torch

from conftest import BC_CASES, bc_kwargs, field_errors, normwise, wet_mask
from oracle import OracleSWE

from diffswe2d_b200 import SWE2D, SWEConfig, scenarios
from diffswe2d_b200 import _native as nat

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def _t(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


def _np(t):
    return t.detach().cpu().numpy()


def _model(bed, n, dx, dy, cfg, arithmetic="fast"):
    return SWE2D(_t(bed), _t(n), dx, dy, config=cfg, train_dem=False, arithmetic=arithmetic)


def _run(m, U, nsteps, dynamic=False):
    t, dts = 0.0, []
    with torch.no_grad():
        for _ in range(nsteps):
            level = m._interpolate_dynamic_boundary(t, U) if dynamic else None
            U, dt = m.step(U, t, 1.0e9, boundary_level=level)
            t += dt
            dts.append(dt)
    return U, np.array(dts)


def test_island_1000_steps_within_fp32_floor(golden):
    """Config 1 (256x256, walls, Manning 0.025): 1000 steps."""
    d = golden("c1_island")
    cfg = SWEConfig(boundary_left="wall", boundary_right="wall", boundary_top="wall",
                    boundary_bottom="wall")
    U, dts = _run(_model(d["bed"], d["n"], 1.0, 1.0, cfg), _t(d["U0"]), 1000)
    U = _np(U)
    floor = field_errors(d["f32_1000"], d["f64_1000"])
    err64 = field_errors(U, d["f64_1000"])
    err32 = field_errors(U, d["f32_1000"])
    print("fast: vs FP64", err64, "vs stock FP32", err32, "FP32 floor", floor)
    for e, f in zip(err64, floor):
        assert e <= 1.5 * f
    assert np.array_equal(wet_mask(U), wet_mask(d["f32_1000"]))
    assert np.allclose(dts, d["f32_dts"], rtol=1e-4)


def test_runup_200_steps_within_fp32_floor(golden):
    """Config 2 (244x393, west water level from the N-wave series): 200 steps;
    the FP64 reference is the FP64 oracle (pinned to the reference's FP64 run
    in tests/test_oracle.py)."""
    d = golden("c2_runup")
    cfg = SWEConfig(boundary_left="water_level", boundary_right="wall", boundary_top="wall",
                    boundary_bottom="wall")
    dx = float(d["dx"])
    m = _model(d["bed"], d["n"], dx, dx, cfg)
    m.set_dynamic_boundary(_t(d["bc_times"]), _t(d["bc_levels"]))
    U, dts = _run(m, _t(d["U0"]), 200, dynamic=True)
    U = _np(U)
    o64 = OracleSWE(d["bed"], d["n"], dx, dx, cfg, dtype=np.float64)
    o64.set_dynamic_boundary(d["bc_times"], d["bc_levels"])
    Uo, t = d["U0"].astype(np.float64), 0.0
    for _ in range(200):
        Uo, dt = o64.step(Uo, t, 1.0e9, boundary_level=o64.interpolate_boundary(t))
        t += dt
    floor = field_errors(d["f32_200"], Uo)
    err64 = field_errors(U, Uo)
    print("fast runup: vs FP64", err64, "vs stock FP32", field_errors(U, d["f32_200"]), "floor", floor)
    for e, f in zip(err64, floor):
        assert e <= 1.5 * f
    assert np.array_equal(wet_mask(U), wet_mask(d["f32_200"]))
    assert np.allclose(dts, d["f32_dts"], rtol=1e-4)


@pytest.mark.parametrize("case", sorted(BC_CASES))
def test_five_steps_each_boundary(golden, case):
    """Random wet/dry states (a quarter dry, films below the dry depth),
    every boundary type: five steps within 1e-5 (depth) / 1e-4 (momenta)
    of the oracle, normwise, and the same time steps to 1e-5."""
    d = golden("ops")
    cfg = SWEConfig(**bc_kwargs(case), constant_value=0.05, constant_level=0.2)
    m = _model(d["bed1"][0, 0], d["n"][0, 0], 0.05, 0.04, cfg)
    om = OracleSWE(d["bed1"], d["n"], 0.05, 0.04, cfg)
    U, Uo = _t(d["U"]), d["U"]
    for _ in range(5):
        U, dt = m.step(U, 0.0, 0.05, boundary_level=0.2)
        Uo, dto = om.step(Uo, 0.0, 0.05, boundary_level=0.2)
        assert abs(dt - dto) <= 1e-5 * dto
    err = field_errors(_np(U), Uo)
    print(case, err)
    assert err[0] <= 1e-5 and err[1] <= 1e-4 and err[2] <= 1e-4


def test_spatial_operator_fast(golden):
    d = golden("ops")
    cfg = SWEConfig(**bc_kwargs("mixed_a"), constant_value=0.05, constant_level=0.2)
    m = _model(d["bed1"][0, 0], d["n"][0, 0], 0.05, 0.04, cfg)
    rhs, ax, ay = m.spatial_operator(_t(d["U"]), return_wave_speed=True, boundary_level=0.2)
    from oracle import Oracle
    orhs, oax, oay = Oracle().spatial_operator(d["U"], d["bed1"], cfg, 0.05, 0.04, 0.2)
    assert normwise(_np(rhs), orhs) <= 1e-5
    assert abs(float(ax) - float(oax)) <= 1e-6 * float(oax)
    assert abs(float(ay) - float(oay)) <= 1e-6 * float(oay)


@pytest.mark.parametrize("model", ["manning", "roughness"])
def test_friction_models_and_batched_fields(golden, model):
    """Per-batch bed, roughness and level, both friction laws, wsr and the
    positivity limiter off and on."""
    d = golden("ops")
    for wsr, pos in ((True, True), (False, False)):
        cfg = SWEConfig(boundary_left="water_level", boundary_right="wall", boundary_top="wall",
                        boundary_bottom="water_level", frictionmodel=model,
                        water_slope_reset=wsr, positivity_limiter=pos)
        n = d["stb_n"] if model == "manning" else np.full_like(d["stb_n"], 0.01)
        m = SWE2D(_t(d["bed"]), _t(n), 0.05, 0.04, config=cfg, train_dem=False, arithmetic="fast")
        om = OracleSWE(d["bed"], n, 0.05, 0.04, cfg)
        U, Uo = _t(d["U"]), d["U"]
        for _ in range(3):
            U, dt = m.step(U, 0.0, 0.05, boundary_level=_t(d["level_b"]))
            Uo, dto = om.step(Uo, 0.0, 0.05, boundary_level=d["level_b"])
        err = field_errors(_np(U), Uo)
        print(model, wsr, pos, err)
        assert err[0] <= 1e-5 and err[1] <= 1e-4 and err[2] <= 1e-4


@pytest.mark.parametrize("shape", [(2, 2), (3, 7), (9, 40), (37, 53), (65, 129), (300, 257)])
def test_odd_and_tile_straddling_sizes(shape):
    ny, nx = shape
    rng = np.random.default_rng(ny * 1000 + nx)
    B = 2
    h = rng.uniform(0, 0.5, (B, ny, nx))
    h[rng.uniform(size=h.shape) < 0.3] = 0.0
    U = np.stack([h, rng.normal(0, 0.1, h.shape) * (h > 0), rng.normal(0, 0.1, h.shape) * (h > 0)],
                 axis=1).astype(np.float32)
    bed = rng.normal(-0.2, 0.1, (1, 1, ny, nx)).astype(np.float32)
    n = np.full_like(bed, 0.02)
    cfg = SWEConfig(boundary_left="water_level", boundary_right="wall", boundary_top="periodic",
                    boundary_bottom="periodic", constant_level=0.05)
    m = _model(bed[0, 0], n[0, 0], 0.1, 0.1, cfg)
    om = OracleSWE(bed, n, 0.1, 0.1, cfg)
    Ug, Uo = _t(U), U
    for _ in range(3):
        Ug, dt = m.step(Ug, 0.0, 0.01)
        Uo, dto = om.step(Uo, 0.0, 0.01)
        assert abs(dt - dto) <= 1e-5 * dto
    err = field_errors(_np(Ug), Uo)
    assert err[0] <= 1e-5 and err[1] <= 1e-4 and err[2] <= 1e-4, err


def test_tiny_and_subnormal_operands():
    """Momenta of draining films (tiny and subnormal), depths below the dry
    depth: the tolerance mode flushes subnormals, the result stays within
    the bound and finite."""
    rng = np.random.default_rng(11)
    B, ny, nx = 1, 96, 160
    h = rng.uniform(0.05, 0.5, (B, ny, nx))
    hu = rng.normal(0, 0.05, h.shape)
    hv = rng.normal(0, 0.05, h.shape)
    pick = rng.uniform(size=h.shape)
    hu[pick < 0.05] = 1e-36
    hv[(pick >= 0.05) & (pick < 0.08)] = -3e-39
    h[(pick >= 0.08) & (pick < 0.10)] = 1e-30
    U = np.stack([h, hu, hv], axis=1).astype(np.float32)
    bed = rng.normal(-0.2, 0.05, (1, 1, ny, nx)).astype(np.float32)
    n = np.full_like(bed, 0.03)
    cfg = SWEConfig(boundary_left="water_level", boundary_right="wall", boundary_top="wall",
                    boundary_bottom="wall", constant_level=0.05)
    m = _model(bed[0, 0], n[0, 0], 0.05, 0.05, cfg)
    om = OracleSWE(bed, n, 0.05, 0.05, cfg)
    Ug, Uo = _t(U), U
    for _ in range(3):
        Ug, dt = m.step(Ug, 0.0, 0.01)
        Uo, dto = om.step(Uo, 0.0, 0.01)
    err = field_errors(_np(Ug), Uo)
    assert np.isfinite(_np(Ug)).all()
    assert err[0] <= 1e-5 and err[1] <= 1e-4 and err[2] <= 1e-4, err


def test_errors_raise_like_reference():
    bed = torch.full((8, 8), -1.0, device=DEV)
    m = SWE2D(bed, torch.full_like(bed, 0.02), 1.0, 1.0, config=SWEConfig(), train_dem=False,
              arithmetic="fast")
    U = torch.zeros(1, 3, 8, 8, device=DEV)
    U[:, 0] = 1.0
    with pytest.raises(FloatingPointError, match="Non-positive"):
        m.step(U, 0.0, 0.0)
    U[0, 1, 3, 3] = float("inf")
    with pytest.raises(FloatingPointError, match="non-finite"):
        m.step(U, 0.0, 1.0)


def test_forward_device_loop_equals_host_loop(golden):
    """forward() in the tolerance mode: the captured device loop and the host
    loop (callback) give the same state, hmax and step count."""
    d = golden("c2_runup")
    cfg = SWEConfig(boundary_left="water_level", boundary_right="wall", boundary_top="wall",
                    boundary_bottom="wall")
    dx = float(d["dx"])
    m = _model(d["bed"], d["n"], dx, dx, cfg)
    m.set_dynamic_boundary(_t(d["bc_times"]), _t(d["bc_levels"]))
    times = []
    with torch.no_grad():
        U1, h1 = m(_t(d["f32cr_200"]), t_end=0.2, start_time=1.0, callback=lambda i, t, U: times.append(t))
        U2, h2 = m(_t(d["f32cr_200"]), t_end=0.2, start_time=1.0)
    assert m.last_forward_steps == len(times)
    assert torch.equal(U1, U2) and torch.equal(h1, h2)


def test_ensemble_members_equal_single_steps():
    """Each member of a tolerance-mode ensemble equals SWE2D.step (tolerance
    mode) run on it alone, bit for bit."""
    from diffswe2d_b200.ensemble import Ensemble
    members = []
    for k, (ny, nx) in enumerate([(70, 130), (129, 64), (200, 201)]):
        sc = scenarios.ensemble_member(ny, nx, seed=50 + k)
        sc.steps = 12
        members.append(sc)
    res = Ensemble(members, device=DEV, rows=8, arithmetic="fast").run()
    for sc, U_ens, steps in zip(members, res.states, res.steps):
        m = SWE2D(_t(sc.bed), _t(sc.roughness), sc.dx, sc.dy, config=SWEConfig(**sc.config),
                  train_dem=False, arithmetic="fast")
        if sc.bc_times is not None:
            m.set_dynamic_boundary(_t(sc.bc_times), _t(sc.bc_levels))
        U, t = _t(sc.U0), 0.0
        with torch.no_grad():
            for _ in range(steps):
                level = m._interpolate_dynamic_boundary(t, U) if sc.bc_times is not None else None
                U, dt = m.step(U, t, 1.0e9, boundary_level=level)
                t += dt
        assert torch.equal(U, U_ens)


def test_launch_shape_does_not_change_results():
    """The tolerance-mode kernels give the same bits for every tile height."""
    sc = scenarios.tiled(scenarios.runup(seed=2), 300, 500)
    cfg = SWEConfig(**sc.config)
    m = _model(sc.bed, sc.roughness, sc.dx, sc.dy, cfg)
    outs = []
    lib = nat.lib()
    prev = int(lib.swe_sweep_rows())
    try:
        for rows in (4, 16, 128):
            nat.check(lib.swe_tune_sweep_rows(rows), "rows")
            U = _t(sc.U0)
            for _ in range(3):
                U, _ = m.step(U, 0.0, 1.0e9, boundary_level=0.005)
            outs.append(U)
    finally:
        nat.check(lib.swe_tune_sweep_rows(prev), "rows")
    assert torch.equal(outs[0], outs[1]) and torch.equal(outs[0], outs[2])
