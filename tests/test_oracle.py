"""The CPU oracle against golden outputs of the reference itself.

The oracle (oracle/swe_oracle.c) uses correctly-rounded arithmetic; the
reference's PyTorch CPU build evaluates sqrt and pow to within an ulp but not
always correctly rounded.  Operators without sqrt/pow must match bit for bit;
those with them must agree to a few ulps, and multi-step runs to the
normwise tolerances written in each test.
"""
import numpy as np
import pytest

from conftest import BC_CASES, bc_kwargs, field_errors, normwise, wet_mask
from oracle import Oracle, OracleSWE

from diffswe2d_b200.config import SWEConfig


@pytest.fixture(scope="module")
def o32():
    return Oracle(np.float32)


def test_primitive_bit_exact(golden, o32):
    d = golden("ops")
    h, u, v, c = o32.primitive(d["U"], SWEConfig())
    assert np.array_equal(h, d["prim_h"]) and np.array_equal(u, d["prim_u"])
    assert np.array_equal(v, d["prim_v"]) and np.array_equal(c, d["prim_c"])


def test_limited_increment_bit_exact(golden, o32):
    d = golden("ops")
    assert np.array_equal(o32.limited_increment(d["li_q"], -1), d["li_x"])
    assert np.array_equal(o32.limited_increment(d["li_q"], -2), d["li_y"])


@pytest.mark.parametrize("case", sorted(BC_CASES))
@pytest.mark.parametrize("lname", ["s", "b"])
@pytest.mark.parametrize("bname", ["bB", "b1"])
def test_ghost_cells_bit_exact(golden, o32, case, lname, bname):
    d = golden("ops")
    cfg = SWEConfig(**bc_kwargs(case), constant_value=0.05)
    bed = d["bed"] if bname == "bB" else d["bed1"]
    level = 0.2 if lname == "s" else d["level_b"]
    Up, zp = o32.ghost_cells(d["U"], bed, 2, cfg, level, 0.05)
    key = f"gc_{case}_{lname}_{bname}"
    assert np.array_equal(Up, d[key + "_Up"])
    assert np.array_equal(zp, d[key + "_zp"])


@pytest.mark.parametrize("tag,dim", [("x", -1), ("y", -2)])
@pytest.mark.parametrize("wsr", [1, 0])
def test_reconstruction_bit_exact(golden, o32, tag, dim, wsr):
    d = golden("ops")
    cfg = SWEConfig(water_slope_reset=bool(wsr))
    UL, UR, sL, sR = o32.reconstruction(d["rc_Up"], d["rc_zp"], dim, cfg)
    key = f"rc_{tag}_{wsr}"
    for name, a in (("UL", UL), ("UR", UR), ("sL", sL), ("sR", sR)):
        assert np.array_equal(a, d[f"{key}_{name}"]), name


@pytest.mark.parametrize("tag", ["x", "y"])
def test_hll_flux_within_sqrt_ulps(golden, o32, tag):
    d = golden("ops")
    F, s = o32.hll_flux(d[f"hll_{tag}_UL"], d[f"hll_{tag}_UR"], tag, SWEConfig())
    # the reference's sqrt can be one ulp off; fluxes inherit a few ulps
    assert np.allclose(F, d[f"hll_{tag}_F"], rtol=1e-6, atol=1e-7)
    assert np.allclose(s, d[f"hll_{tag}_s"], rtol=1e-6, atol=0)
    assert (F != d[f"hll_{tag}_F"]).mean() < 0.02


def test_friction(golden, o32):
    d = golden("ops")
    assert np.allclose(o32.manning(d["U"], d["n"], d["fr_dt"]), d["fr_manning"], rtol=1e-6, atol=1e-9)
    assert np.allclose(o32.roughness_friction(d["U"], d["fr_z0"], d["fr_dt"]), d["fr_rough"],
                       rtol=1e-6, atol=1e-9)


def test_clean_and_limit_bit_exact(golden, o32):
    d = golden("ops")
    assert np.array_equal(o32.clean_and_limit(d["U"], d["cl_cand"], SWEConfig()), d["cl_out"])


@pytest.mark.parametrize("case", sorted(BC_CASES))
def test_spatial_operator_and_steps(golden, o32, case):
    d = golden("ops")
    cfg = SWEConfig(**bc_kwargs(case), constant_value=0.05, constant_level=0.2)
    rhs, ax, ay = o32.spatial_operator(d["U"], d["bed1"], cfg, 0.05, 0.04, 0.2)
    assert normwise(rhs, d[f"so_{case}_rhs"]) < 1e-6
    assert np.allclose([ax, ay], d[f"so_{case}_axay"], rtol=1e-6)
    m = OracleSWE(d["bed1"], d["n"], 0.05, 0.04, cfg)
    U = d["U"]
    dts = []
    for k in range(5):
        U, dt = m.step(U, 0.0, 0.05, boundary_level=0.2)
        dts.append(dt)
        if k == 0:
            assert max(field_errors(U, d[f"st_{case}_1"])) < 1e-6
    assert max(field_errors(U, d[f"st_{case}_5"])) < 1e-5
    assert np.array_equal(wet_mask(U), wet_mask(d[f"st_{case}_5"]))
    assert np.allclose(dts, d[f"st_{case}_dts"], rtol=1e-5)


def test_batched_bed_and_level(golden):
    d = golden("ops")
    cfg = SWEConfig(boundary_left="water_level", boundary_right="wall", boundary_top="wall",
                    boundary_bottom="water_level")
    m = OracleSWE(d["bed"], d["stb_n"], 0.05, 0.04, cfg)
    U, dt = m.step(d["U"], 0.0, 0.05, boundary_level=d["level_b"])
    assert max(field_errors(U, d["stb_U"])) < 1e-6
    assert dt == pytest.approx(float(d["stb_dt"]), rel=1e-6)


def test_oracle_step_errors():
    """Non-finite and non-positive dt raise FloatingPointError (src/solver.py:627-632)."""
    bed = np.full((8, 8), -1.0, np.float32)
    m = OracleSWE(bed, np.full_like(bed, 0.02), 1.0, 1.0, SWEConfig(boundary_left="wall"))
    U = np.zeros((1, 3, 8, 8), np.float32)
    U[:, 0] = 1.0
    with pytest.raises(FloatingPointError, match="Non-positive"):
        m.step(U, 0.0, 0.0)
    U[0, 1, 3, 3] = np.nan
    with pytest.raises(FloatingPointError, match="non-finite"):
        m.step(U, 0.0, 1.0)


@pytest.mark.parametrize("fixture", ["adj_run", "adj_run_wet"])
def test_thirty_step_loss_matches_reference(golden, fixture):
    """The 30-step loss of the adjoint fixtures: the FP64 oracle against the
    reference's FP64 run, the FP32 oracle against its FP32 run with
    correctly-rounded sqrt/pow (the finite-difference checks of the adjoint
    differentiate this oracle loss)."""
    d = golden(fixture)
    cfg = SWEConfig(boundary_left="water_level", boundary_right="wall", boundary_top="wall",
                    boundary_bottom="wall")
    for dtype, key, rel in ((np.float64, "f64_loss", 1e-12), (np.float32, "f32_loss", 1e-6)):
        om = OracleSWE(d["bed"], d["n"], float(d["dx"]), float(d["dx"]), cfg, dtype=dtype)
        U = d["U0"].astype(dtype)
        L = dtype(0.0)
        for s in range(len(d["levels"])):
            U, _ = om.step(U, 0.0, 2.0e-3, boundary_level=dtype(d["levels"][s]))
            for iy, ix in d["gauges"]:
                eta = U[0, 0, iy, ix] + dtype(d["bed"][iy, ix])
                L = L + eta * eta
        L = L + dtype(1e-3) * (U * U).sum(dtype=dtype)
        assert float(L) == pytest.approx(float(d[key]), rel=rel)


# ------------------------------------------------------------ rain / infiltration
FORCING_CFG = dict(boundary_left="water_level", boundary_right="wall", boundary_top="wall",
                   boundary_bottom="transmissive", constant_level=0.2)


def _forcing_case(d, tag):
    if tag == "scalar":
        return np.float32(1.5e-3), np.float32(4e-4)
    if tag == "field":
        return d["rain_field"], d["infil_field"]
    return d["rain_batch"], d["infil_batch"]


@pytest.mark.parametrize("tag", ["scalar", "field", "batch"])
def test_spatial_operator_with_rain_and_infiltration(golden, o32, tag):
    """src/solver.py:520-525: rhs[:,0] + rain - clamp(infiltration, min=0)."""
    d = golden("forcing")
    rain, infil = _forcing_case(d, tag)
    rhs, ax, ay = o32.spatial_operator(d["U"], d["bed1"], SWEConfig(**FORCING_CFG), 0.05, 0.04,
                                       0.2, rain, infil)
    assert np.array_equal(rhs, d[f"socr_{tag}"])
    assert np.array_equal(np.array([ax, ay], np.float32), d[f"socr_{tag}_axay"])
    assert normwise(rhs, d[f"so_{tag}"]) < 1e-6  # stock sqrt within an ulp


@pytest.mark.parametrize("tag", ["scalar", "field", "batch"])
def test_steps_with_infiltration(golden, tag):
    d = golden("forcing")
    infil = np.float32(4e-4) if tag == "scalar" else d[f"infil_{tag}"]
    om = OracleSWE(d["bed1"], d["n"], 0.05, 0.04, SWEConfig(**FORCING_CFG))
    U, dts = d["U"], []
    for _ in range(5):
        U, dt = om.step(U, 0.0, 0.05, boundary_level=0.2, infiltration=infil)
        dts.append(dt)
    assert np.array_equal(U, d[f"stcr_infil_{tag}"])
    assert np.array_equal(np.array(dts), d[f"stcr_infil_{tag}_dts"])


def test_rainfall_interpolation_matches_reference(golden):
    from oracle import rainfall_at
    d = golden("forcing")
    for k, t in enumerate((0.0, 0.001, 0.0137, 0.5)):
        assert np.array_equal(rainfall_at(d["r_times"], d["r_rates"], t), d["rf_at"][k])


def test_steps_with_rainfall_forcing(golden):
    """Stage 1 at the rate of the step's start, stage 2 half a step later
    (src/solver.py:607-643)."""
    from oracle import rainfall_at
    d = golden("forcing")
    om = OracleSWE(d["bed1"], d["n"], 0.05, 0.04, SWEConfig(**FORCING_CFG))
    U, dts, t = d["U"], [], 0.0
    for _ in range(5):
        U, dt = om.step(U, t, 0.05, boundary_level=0.2, infiltration=d["infil_field"],
                        rainfall=lambda tt: rainfall_at(d["r_times"], d["r_rates"], tt))
        dts.append(dt)
        t += dt
    assert np.array_equal(U, d["stcr_rainfall"])
    assert np.array_equal(np.array(dts), d["stcr_rainfall_dts"])


def test_cea_dem_fixture_from_the_reference_reader(golden):
    """The CEA DEM as the reference's io_ascii reader grids it: the example's
    254 x 200 grid at 0.01 m, finite, the raster's elevation range."""
    d = golden("cea_topo")
    bed = d["bed"]
    assert bed.shape == (254, 200) and float(d["dx"]) == 0.01
    assert np.isfinite(bed).all() and -0.51 < bed.min() and bed.max() < 0.11
