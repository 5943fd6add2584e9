"""Rainfall and infiltration sources on the GPU (src/solver.py:437-446,
:520-525, :607-643), against fixtures of the reference's own runs made with
correctly-rounded sqrt/pow (tests/golden/forcing.npz): the IEEE kernels are
bit for bit those, the tolerance-mode kernels within the bound written in
each test."""
import numpy as np
import pytest
import torch

from conftest import field_errors
from oracle import OracleSWE, rainfall_at

from diffswe2d_b200 import RainfallForcing, SWE2D, SWEConfig

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
CFG = dict(boundary_left="water_level", boundary_right="wall", boundary_top="wall",
           boundary_bottom="transmissive", constant_level=0.2)


def _t(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


def _np(t):
    return t.detach().cpu().numpy()


def _model(d, arithmetic="exact", rainfall=None):
    return SWE2D(_t(d["bed1"][0, 0]), _t(d["n"][0, 0]), 0.05, 0.04, config=SWEConfig(**CFG),
                 train_dem=False, rainfall=rainfall, arithmetic=arithmetic)


def _case(d, tag):
    if tag == "scalar":
        return 1.5e-3, 4e-4
    return _t(d[f"rain_{tag}"]), _t(d[f"infil_{tag}"])


@pytest.mark.parametrize("tag", ["scalar", "field", "batch"])
def test_spatial_operator_rain_and_infiltration_bitwise(golden, tag):
    d = golden("forcing")
    rain, infil = _case(d, tag)
    rhs, ax, ay = _model(d).spatial_operator(_t(d["U"]), rainfall_rate=rain, infiltration=infil,
                                             return_wave_speed=True, boundary_level=0.2)
    assert np.array_equal(_np(rhs), d[f"socr_{tag}"])
    assert np.array_equal(np.array([float(ax), float(ay)], np.float32), d[f"socr_{tag}_axay"])


@pytest.mark.parametrize("tag", ["scalar", "field", "batch"])
def test_steps_with_infiltration_bitwise(golden, tag):
    d = golden("forcing")
    infil = 4e-4 if tag == "scalar" else _t(d[f"infil_{tag}"])
    m = _model(d)
    U, dts = _t(d["U"]), []
    for _ in range(5):
        U, dt = m.step(U, 0.0, 0.05, infiltration=infil, boundary_level=0.2)
        dts.append(dt)
    assert np.array_equal(_np(U), d[f"stcr_infil_{tag}"])
    assert np.array_equal(np.array(dts), d[f"stcr_infil_{tag}_dts"])


def test_rainfall_forcing_rates_bitwise(golden):
    d = golden("forcing")
    rf = RainfallForcing(_t(d["r_times"]), _t(d["r_rates"]))
    for k, t in enumerate((0.0, 0.001, 0.0137, 0.5)):
        assert np.array_equal(_np(rf.at(t)), d["rf_at"][k])


def test_steps_with_rainfall_forcing_bitwise(golden):
    """Stage 1 sees the rate at the step's start, stage 2 the rate half a step
    later; five steps equal the reference's bit for bit."""
    d = golden("forcing")
    m = _model(d, rainfall=RainfallForcing(_t(d["r_times"]), _t(d["r_rates"])))
    U, dts, t = _t(d["U"]), [], 0.0
    for _ in range(5):
        U, dt = m.step(U, t, 0.05, infiltration=_t(d["infil_field"]), boundary_level=0.2)
        dts.append(dt)
        t += dt
    assert np.array_equal(_np(U), d["stcr_rainfall"])
    assert np.array_equal(np.array(dts), d["stcr_rainfall_dts"])


def test_forward_with_rainfall_equals_its_steps(golden):
    """forward() of a model with rainfall runs the host loop (the rates are
    evaluated per stage on the host): same result as stepping by hand."""
    d = golden("forcing")
    rf = RainfallForcing(_t(d["r_times"]), _t(d["r_rates"]))
    m = _model(d, rainfall=rf)
    steps = []
    with torch.no_grad():
        U, _ = m(_t(d["U"]), t_end=6e-5, boundary_level=0.2, callback=lambda i, t, U: steps.append(t))
        V, _ = m(_t(d["U"]), t_end=6e-5, boundary_level=0.2)
    assert torch.equal(U, V) and len(steps) >= 3


def test_rainfall_with_autograd_is_refused(golden):
    d = golden("forcing")
    m = _model(d, rainfall=RainfallForcing(_t(d["r_times"]), _t(d["r_rates"])))
    U = _t(d["U"]).requires_grad_(True)
    with pytest.raises(NotImplementedError):
        m.step(U, 0.0, 0.05, boundary_level=0.2)


def test_fast_arithmetic_with_rain_and_infiltration(golden):
    """Tolerance mode: five rainfall-forced steps with per-batch infiltration
    stay within 1e-5 (depth) and 1e-4 (momenta) of the oracle, normwise."""
    d = golden("forcing")
    rf = RainfallForcing(_t(d["r_times"]), _t(d["r_rates"]))
    m = _model(d, arithmetic="fast", rainfall=rf)
    om = OracleSWE(d["bed1"], d["n"], 0.05, 0.04, SWEConfig(**CFG))
    U, Uo, t, to = _t(d["U"]), d["U"], 0.0, 0.0
    for _ in range(5):
        U, dt = m.step(U, t, 0.05, infiltration=_t(d["infil_batch"]), boundary_level=0.2)
        Uo, dto = om.step(Uo, to, 0.05, boundary_level=0.2, infiltration=d["infil_batch"],
                          rainfall=lambda tt: rainfall_at(d["r_times"], d["r_rates"], tt))
        t, to = t + dt, to + dto
        assert abs(dt - dto) <= 1e-5 * dto
    err = field_errors(_np(U), Uo)
    print("fast vs oracle after 5 forced steps", err)
    assert err[0] <= 1e-5 and err[1] <= 1e-4 and err[2] <= 1e-4
