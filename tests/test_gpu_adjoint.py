"""The hand-written adjoint against the reference's autograd gradients and
against finite differences of the FP64 oracle.

Bar: adjoint gradients match the reference autograd to 1e-4
(normwise relative, per gradient).  Fixtures: tests/golden/adj_*.npz, made by
the reference itself (make_golden_adjoint.py) in float32 with
correctly-rounded sqrt/pow and in float64.
"""
import numpy as np
import pytest
import torch

from oracle import OracleSWE

from diffswe2d_b200 import SWE2D, SWEConfig
from diffswe2d_b200.adjoint import forward_checkpointed

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
TOL = 1e-4

STEP_CASES = {
    "walls": dict(boundary_left="wall", boundary_right="wall", boundary_top="wall",
                  boundary_bottom="wall"),
    "water_level": dict(boundary_left="water_level", boundary_right="water_level",
                        boundary_top="water_level", boundary_bottom="water_level"),
    "transmissive": dict(boundary_left="transmissive", boundary_right="transmissive",
                         boundary_top="transmissive", boundary_bottom="transmissive"),
    "periodic": dict(boundary_left="periodic", boundary_right="periodic", boundary_top="periodic",
                     boundary_bottom="periodic"),
    "mixed_a": dict(boundary_left="water_level", boundary_right="wall", boundary_top="periodic",
                    boundary_bottom="absorbing"),
    "mixed_b": dict(boundary_left="constant", boundary_right="transmissive", boundary_top="wall",
                    boundary_bottom="water_level"),
    "roughness_law": dict(boundary_left="water_level", boundary_right="wall", boundary_top="wall",
                          boundary_bottom="wall", frictionmodel="roughness_length"),
    "no_friction": dict(boundary_left="water_level", boundary_right="wall", boundary_top="wall",
                        boundary_bottom="wall", apply_friction=False),
    "no_reset_no_limiter": dict(boundary_left="water_level", boundary_right="wall",
                                boundary_top="wall", boundary_bottom="wall",
                                water_slope_reset=False, positivity_limiter=False),
}


def _t(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


def _rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    s = np.abs(b).max()
    return float(np.abs(a - b).max() / s) if s > 0 else float(np.abs(a - b).max())


@pytest.mark.parametrize("case", sorted(STEP_CASES))
def test_one_step_vjp_matches_reference_autograd(golden, case):
    d = golden("adj_step")
    kw = STEP_CASES[case]
    field = d["z0"] if kw.get("frictionmodel") == "roughness_length" else d["n"]
    cfg = SWEConfig(**kw, constant_value=0.05)
    m = SWE2D(_t(d["bed"]), _t(field), 0.05, 0.04, config=cfg, train_dem=False)
    m.roughness_length.requires_grad_(True)
    U = _t(d["U"]).requires_grad_(True)
    lv = torch.tensor(0.18, device=DEV, requires_grad=True)
    Un, dt = m.step(U, 0.0, 0.01, boundary_level=lv)
    assert dt == pytest.approx(float(d[f"{case}_dt"]), rel=1e-6)
    (Un * _t(d["w"])).sum().backward()
    gU = U.grad.cpu().numpy()
    eU = _rel(gU, d[f"{case}_gU"])
    el = abs(float(lv.grad) - float(d[f"{case}_glevel"])) / max(abs(float(d[f"{case}_glevel"])), 1e-30)
    print(case, "dL/dU", eU, "vs FP64", _rel(gU, d[f"{case}_gU64"]), "dL/dlevel", el)
    assert eU <= TOL
    if float(d[f"{case}_glevel"]) != 0.0:
        assert el <= TOL
    else:
        assert float(lv.grad) == 0.0
    if kw.get("apply_friction", True):
        gn = m.roughness_length.grad.cpu().numpy()
        assert _rel(gn, d[f"{case}_gn"]) <= TOL


@pytest.mark.parametrize("case", sorted(STEP_CASES))
def test_one_step_vjp_fast_arithmetic(golden, case):
    """The tolerance-mode adjoint (hardware reciprocal / square root, FMA
    contraction) at the tolerance-mode step: within 1e-4 of the reference's
    FP32 autograd, or, where the reference's own FP32 and FP64 gradients
    differ by more, within 1.5x that difference of the FP64 gradient."""
    d = golden("adj_step")
    kw = STEP_CASES[case]
    field = d["z0"] if kw.get("frictionmodel") == "roughness_length" else d["n"]
    cfg = SWEConfig(**kw, constant_value=0.05)
    m = SWE2D(_t(d["bed"]), _t(field), 0.05, 0.04, config=cfg, train_dem=False, arithmetic="fast")
    m.roughness_length.requires_grad_(True)
    U = _t(d["U"]).requires_grad_(True)
    lv = torch.tensor(0.18, device=DEV, requires_grad=True)
    Un, dt = m.step(U, 0.0, 0.01, boundary_level=lv)
    assert dt == pytest.approx(float(d[f"{case}_dt"]), rel=1e-5)
    (Un * _t(d["w"])).sum().backward()
    gU = U.grad.cpu().numpy()
    eU, eU64 = _rel(gU, d[f"{case}_gU"]), _rel(gU, d[f"{case}_gU64"])
    floor = _rel(d[f"{case}_gU"], d[f"{case}_gU64"])
    print(case, "fast dL/dU vs FP32 autograd", eU, "vs FP64", eU64, "FP32-vs-FP64", floor)
    assert eU <= TOL or eU64 <= 1.5 * floor
    gl, rl = float(lv.grad), float(d[f"{case}_glevel"])
    if rl != 0.0:
        assert abs(gl - rl) <= TOL * abs(rl)
    else:
        assert gl == 0.0
    if kw.get("apply_friction", True):
        assert _rel(m.roughness_length.grad.cpu().numpy(), d[f"{case}_gn"]) <= TOL


@pytest.mark.parametrize("arithmetic", ["exact", "fast"])
@pytest.mark.parametrize("bed_grad", [False, True])
def test_stage2_entry_equals_spatial_then_predictor(golden, arithmetic, bed_grad):
    """swe_adj_stage2_f32 (spatial adjoint at P with the predictor adjoint
    fused into its gather) against swe_adj_spatial(_bed)_f32 into a zeroed
    lam_P followed by swe_adj_pointwise_f32 mode 1: the same adjoints of U,
    k1, the level and the bed -- bit for bit in the IEEE mode, within 1e-6
    (normwise) in the tolerance mode."""
    from diffswe2d_b200 import _native as nat
    from diffswe2d_b200.adjoint import level_blocks
    d = golden("adj_step")
    cfg = SWEConfig(**STEP_CASES["mixed_a"], constant_value=0.05)
    m = SWE2D(_t(d["bed"]), _t(d["n"]), 0.05, 0.04, config=cfg, train_dem=False,
              arithmetic=arithmetic)
    lib, st, p = nat.lib(), nat.stream_handle(torch.device(DEV)), m._params()
    U = _t(d["U"])
    B, _, ny, nx = U.shape
    bed = m.bed.detach().reshape(1, 1, ny, nx).contiguous()
    lv = torch.tensor([0.18], device=DEV)
    red = torch.zeros(nat.RED_WORDS, dtype=torch.int32, device=DEV)
    K1, P = torch.empty_like(U), torch.empty_like(U)
    nat.check(lib.swe_spatial_operator_f32(nat.ptr(U), nat.ptr(bed), B, 1, ny, nx, p, nat.ptr(lv), 1,
                                           None, nat.FORCING_NONE, 1, None, nat.FORCING_NONE, 1,
                                           nat.ptr(K1), nat.ptr(red), st), "k1")
    dt = 2.5e-3
    nat.check(lib.swe_adj_pointwise_f32(2, nat.ptr(U), nat.ptr(K1), None, 1, B, ny, nx, p, dt, None,
                                        None, None, None, nat.ptr(P), st), "predictor")
    g = torch.Generator(device="cpu").manual_seed(3)
    lk2 = torch.randn(U.shape, generator=g).to(DEV)
    base = torch.randn(U.shape, generator=g).to(DEV)
    rec = 16 if bed_grad else 12
    LEVEL_BLOCKS = level_blocks(ny, nx)
    cx = torch.empty(B * ny * (nx + 1) * rec, device=DEV)
    cy = torch.empty(B * (ny + 1) * nx * rec, device=DEV)

    def run(fused):
        lamU, lk1 = base.clone(), torch.zeros_like(U)
        part = torch.zeros(B * LEVEL_BLOCKS, device=DEV)
        lbed = torch.zeros((B, ny, nx), device=DEV) if bed_grad else None
        if fused:
            rc = lib.swe_adj_stage2_f32(nat.ptr(P), nat.ptr(U), nat.ptr(K1), nat.ptr(bed), 1, B, ny, nx,
                                        p, nat.ptr(lv), 1, nat.ptr(lk2), nat.ptr(cx), nat.ptr(cy), dt,
                                        None, nat.ptr(lamU), nat.ptr(lk1), nat.ptr(part), LEVEL_BLOCKS,
                                        nat.ptr(lbed) if bed_grad else None, st)
            nat.check(rc, "stage 2")
        else:
            lamP = torch.zeros_like(U)
            args = (nat.ptr(P), nat.ptr(bed), 1, B, ny, nx, p, nat.ptr(lv), 1, nat.ptr(lk2), nat.ptr(cx),
                    nat.ptr(cy), nat.ptr(lamP), nat.ptr(part), LEVEL_BLOCKS)
            if bed_grad:
                nat.check(lib.swe_adj_spatial_bed_f32(*args, nat.ptr(lbed), st), "spatial")
            else:
                nat.check(lib.swe_adj_spatial_f32(*args, st), "spatial")
            nat.check(lib.swe_adj_pointwise_f32(1, nat.ptr(U), nat.ptr(K1), None, 1, B, ny, nx, p, dt,
                                                nat.ptr(lamP), nat.ptr(lamU), nat.ptr(lk1), None, None,
                                                st), "predictor adjoint")
        torch.cuda.synchronize()
        out = [lamU, lk1, part] + ([lbed] if bed_grad else [])
        return [x.cpu().numpy() for x in out]

    fused, split = run(True), run(False)
    assert np.abs(split[1]).max() > 0 and np.abs(split[2]).max() > 0
    for a, b in zip(fused, split):
        if arithmetic == "exact":
            assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
        else:
            assert _rel(a, b) <= 1e-6


@pytest.mark.parametrize("arithmetic", ["exact", "fast"])
def test_corrector_adjoint_overwrite_mode(golden, arithmetic):
    """swe_adj_pointwise_f32 mode 3 (lam_U written) equals mode 0 (lam_U
    accumulated) into a zeroed lam_U, value for value (0 + x turns a -0
    into +0), whatever lam_U held."""
    from diffswe2d_b200 import _native as nat
    d = golden("adj_step")
    cfg = SWEConfig(**STEP_CASES["walls"], constant_value=0.05)
    m = SWE2D(_t(d["bed"]), _t(d["n"]), 0.05, 0.04, config=cfg, train_dem=False,
              arithmetic=arithmetic)
    lib, st, p = nat.lib(), nat.stream_handle(torch.device(DEV)), m._params()
    U = _t(d["U"])
    B, _, ny, nx = U.shape
    n = m.roughness_length.detach().reshape(1, 1, ny, nx).contiguous()
    g = torch.Generator(device="cpu").manual_seed(5)
    k2 = (torch.randn(U.shape, generator=g) * 0.1).to(DEV)
    lout = torch.randn(U.shape, generator=g).to(DEV)
    outs = []
    for mode, start in ((0, torch.zeros_like(U)), (3, torch.randn(U.shape, generator=g).to(DEV))):
        lamU, lamk, lamn = start.clone(), torch.zeros_like(U), torch.zeros_like(n)
        nat.check(lib.swe_adj_pointwise_f32(mode, nat.ptr(U), nat.ptr(k2), nat.ptr(n), 1, B, ny, nx, p,
                                            2.5e-3, nat.ptr(lout), nat.ptr(lamU), nat.ptr(lamk),
                                            nat.ptr(lamn), None, st), f"mode {mode}")
        torch.cuda.synchronize()
        outs.append([x.cpu().numpy() for x in (lamU, lamk, lamn)])
    assert np.abs(outs[0][0]).max() > 0
    for a, b in zip(*outs):
        assert np.array_equal(a, b)


def _run_model(d, requires=True, arithmetic="exact"):
    cfg = SWEConfig(boundary_left="water_level", boundary_right="wall", boundary_top="wall",
                    boundary_bottom="wall")
    m = SWE2D(_t(d["bed"]), _t(d["n"]), float(d["dx"]), float(d["dx"]), config=cfg, train_dem=False,
              arithmetic=arithmetic)
    m.roughness_length.requires_grad_(requires)
    return m


def _run_loss(m, U0, levels, gauges, bed):
    U, loss = U0, 0.0
    for s in range(levels.shape[0]):
        U, _ = m.step(U, 0.0, 2.0e-3, boundary_level=levels[s])
        for iy, ix in gauges:
            eta = U[0, 0, iy, ix] + bed[iy, ix]
            loss = loss + eta * eta
    return loss + 1e-3 * (U * U).sum()


@pytest.mark.parametrize("fixture", ["adj_run", "adj_run_wet"])
def test_thirty_step_gradients_match_reference_autograd(golden, fixture):
    d = golden(fixture)
    m = _run_model(d)
    U0 = _t(d["U0"]).requires_grad_(True)
    lv = _t(d["levels"]).requires_grad_(True)
    loss = _run_loss(m, U0, lv, d["gauges"], _t(d["bed"]))
    loss.backward()
    assert float(loss.detach()) == pytest.approx(float(d["f32_loss"]), rel=1e-6)
    errs = {
        "U0": _rel(U0.grad.cpu().numpy(), d["f32_gU0"]),
        "levels": _rel(lv.grad.cpu().numpy(), d["f32_glevels"]),
        "n": _rel(m.roughness_length.grad.cpu().numpy(), d["f32_gn"]),
    }
    errs64 = {
        "U0": _rel(U0.grad.cpu().numpy(), d["f64_gU0"]),
        "levels": _rel(lv.grad.cpu().numpy(), d["f64_glevels"]),
        "n": _rel(m.roughness_length.grad.cpu().numpy(), d["f64_gn"]),
    }
    print("vs reference autograd FP32", errs, "vs FP64", errs64)
    for k, e in errs.items():
        assert e <= TOL, k


@pytest.mark.parametrize("fixture", ["adj_run", "adj_run_wet"])
def test_thirty_step_gradients_with_fast_forward(golden, fixture):
    """The tolerance-mode forward kernels (inversions run on them): the
    adjoint, evaluated at their states, matches the reference's autograd to
    the 1e-4 bar, except where the reference's own FP32 and FP64 gradients
    differ by more (dL/dU0 of the wet crop: 6.8 %, limiter branches switch
    with the last bits of the state): there it stays within 1.5x that
    difference of the FP64 gradient."""
    d = golden(fixture)
    m = _run_model(d, arithmetic="fast")
    U0 = _t(d["U0"]).requires_grad_(True)
    lv = _t(d["levels"]).requires_grad_(True)
    loss = _run_loss(m, U0, lv, d["gauges"], _t(d["bed"]))
    loss.backward()
    assert float(loss.detach()) == pytest.approx(float(d["f32_loss"]), rel=1e-5)
    errs = {
        "U0": _rel(U0.grad.cpu().numpy(), d["f32_gU0"]),
        "levels": _rel(lv.grad.cpu().numpy(), d["f32_glevels"]),
        "n": _rel(m.roughness_length.grad.cpu().numpy(), d["f32_gn"]),
    }
    ref = {"U0": U0.grad.cpu().numpy(), "levels": lv.grad.cpu().numpy(),
           "n": m.roughness_length.grad.cpu().numpy()}
    key = {"U0": "gU0", "levels": "glevels", "n": "gn"}
    for k, g in ref.items():
        floor = _rel(d[f"f32_{key[k]}"], d[f"f64_{key[k]}"])
        e64 = _rel(g, d[f"f64_{key[k]}"])
        print("fast forward", k, "vs FP32 autograd", errs[k], "vs FP64", e64, "FP32-vs-FP64", floor)
        assert errs[k] <= TOL or e64 <= 1.5 * floor, k


def test_level_gradient_matches_fp64_finite_differences(golden):
    """Central differences (eps 1e-4) of the same loss with the FP64 oracle."""
    d = golden("adj_run")
    m = _run_model(d, requires=False)
    U0 = _t(d["U0"])
    lv = _t(d["levels"]).requires_grad_(True)
    _run_loss(m, U0, lv, d["gauges"], _t(d["bed"])).backward()
    g = lv.grad.cpu().numpy()
    cfg = SWEConfig(boundary_left="water_level", boundary_right="wall", boundary_top="wall",
                    boundary_bottom="wall")
    om = OracleSWE(d["bed"], d["n"], float(d["dx"]), float(d["dx"]), cfg, dtype=np.float64)

    def loss64(levels):
        U = d["U0"].astype(np.float64)
        L = 0.0
        for s in range(len(levels)):
            U, _ = om.step(U, 0.0, 2.0e-3, boundary_level=levels[s])
            for iy, ix in d["gauges"]:
                L += (U[0, 0, iy, ix] + float(d["bed"][iy, ix])) ** 2
        return L + 1e-3 * float((U * U).sum())

    eps = 1e-4
    checked = 0
    for s in np.argsort(-np.abs(g))[:4]:  # the levels the loss is most sensitive to
        up = d["levels"].astype(np.float64).copy()
        dn = up.copy()
        up[s] += eps
        dn[s] -= eps
        fd = (loss64(up) - loss64(dn)) / (2 * eps)
        print("level", s, "adjoint", g[s], "FD64", fd)
        assert g[s] != 0.0
        assert abs(g[s] - fd) <= 1e-3 * abs(fd)
        checked += 1
    assert checked == 4


def test_state_and_roughness_gradients_match_fp64_finite_differences(golden):
    """Central differences of the 30-step loss w.r.t. entries of U0 and n, on
    the crop across the shoreline (adj_run_wet).  Momentum entries and n are
    smooth at the FD scale (eps 1e-7 absolute for U0, 1e-4 relative for n;
    bar 1e-3).  Depth entries sit on a piecewise-smooth surface -- the
    minmod/limiter branches of 30 steps switch inside any usable eps, and the
    reference's own FP32 and FP64 autograd gradients differ by about 1 % there
    -- so they get a 2 % bar."""
    d = golden("adj_run_wet")
    m = _run_model(d)
    U0 = _t(d["U0"]).requires_grad_(True)
    lv = _t(d["levels"])
    _run_loss(m, U0, lv, d["gauges"], _t(d["bed"])).backward()
    gU, gn = U0.grad.cpu().numpy(), m.roughness_length.grad.cpu().numpy()
    cfg = SWEConfig(boundary_left="water_level", boundary_right="wall", boundary_top="wall",
                    boundary_bottom="wall")

    def loss64(U0v, nv):
        om = OracleSWE(d["bed"], nv, float(d["dx"]), float(d["dx"]), cfg, dtype=np.float64)
        U = U0v.astype(np.float64)
        L = 0.0
        for s in range(len(d["levels"])):
            U, _ = om.step(U, 0.0, 2.0e-3, boundary_level=float(d["levels"][s]))
            for iy, ix in d["gauges"]:
                L += (U[0, 0, iy, ix] + float(d["bed"][iy, ix])) ** 2
        return L + 1e-3 * float((U * U).sum())

    n64 = d["n"].astype(np.float64)
    U064 = d["U0"].astype(np.float64)
    cells = U064.shape[2] * U064.shape[3]
    wet = U064[0, 0].ravel() > 5e-3
    order = np.argsort(-np.abs(gU).ravel())
    momentum = [i for i in order if i >= cells and wet[i % cells]][:3]
    depth = [i for i in order if i < cells and wet[i]][:3]
    for idx, bar in [(i, 1e-3) for i in momentum] + [(i, 2e-2) for i in depth]:
        e = 1e-7
        up, dn = U064.ravel().copy(), U064.ravel().copy()
        up[idx] += e
        dn[idx] -= e
        fd = (loss64(up.reshape(U064.shape), n64) - loss64(dn.reshape(U064.shape), n64)) / (2 * e)
        print("U0", idx, gU.ravel()[idx], fd)
        assert abs(gU.ravel()[idx] - fd) <= bar * abs(fd)
    for idx in np.argsort(-np.abs(gn).ravel())[:2]:
        e = 1e-4 * float(d["n"].ravel()[idx])
        up, dn = n64.ravel().copy(), n64.ravel().copy()
        up[idx] += e
        dn[idx] -= e
        fd = (loss64(U064, up.reshape(n64.shape)) - loss64(U064, dn.reshape(n64.shape))) / (2 * e)
        print("n", idx, gn.ravel()[idx], fd)
        assert abs(gn.ravel()[idx] - fd) <= 1e-3 * abs(fd)


def test_checkpointed_chunk_matches_stepwise_autograd(golden):
    """forward_checkpointed (one autograd node per forward() call, states
    recomputed in backward) gives the stepwise adjoint's gradients."""
    d = golden("adj_run")
    grads = []
    for mode in ("chunk", "steps"):
        m = _run_model(d)
        U0 = _t(d["U0"]).requires_grad_(True)
        lv = torch.tensor(0.008, device=DEV, requires_grad=True)
        if mode == "chunk":
            U = forward_checkpointed(m, U0, t_end=0.03, boundary_level=lv)
        else:
            U, _ = m(U0, t_end=0.03, boundary_level=lv, callback=lambda it, t, U: None)
        (U[0, 0, 20, 30] ** 2 + 1e-3 * (U * U).sum()).backward()
        grads.append((U0.grad.cpu().numpy(), float(lv.grad), m.roughness_length.grad.cpu().numpy(),
                      U.detach().cpu().numpy()))
    (g0c, glc, gnc, Uc), (g0s, gls, gns, Us) = grads
    assert np.array_equal(Uc, Us)
    assert _rel(g0c, g0s) <= 1e-6
    assert abs(glc - gls) <= 1e-6 * max(abs(gls), 1e-30)
    assert _rel(gnc, gns) <= 1e-6


# ---------------------------------------------------------------- bed (DEM)
def _bed_model(cfg_kw, bed, field, dx, dy, max_corr=None, mask=None, corr0=None):
    cfg = SWEConfig(**cfg_kw, constant_value=0.05)
    m = SWE2D(_t(bed), _t(field), dx, dy, config=cfg, train_dem=True, maximum_dem_correction=max_corr,
              valid_mask=None if mask is None else torch.from_numpy(mask).to(DEV))
    if corr0 is not None:
        with torch.no_grad():
            m.dem_correction_parameter.copy_(_t(corr0).reshape(m.dem_correction_parameter.shape))
    return m


@pytest.mark.parametrize("case", sorted(STEP_CASES) + ["tanh_mask"])
def test_one_step_bed_gradient_matches_reference_autograd(golden, case):
    """d(sum w U_new)/d(dem_correction_parameter): the bed's adjoint through
    the spatial operator (eta, increments, Audusse bed, sources, ghost cells)
    chained by autograd through the tanh bound and mask."""
    d, g = golden("adj_step"), golden("adj_bed")
    if case == "tanh_mask":
        m = _bed_model(STEP_CASES["water_level"], d["bed"], d["n"], 0.05, 0.04, 0.05, g["mask"], g["corr0"])
    else:
        kw = STEP_CASES[case]
        field = d["z0"] if kw.get("frictionmodel") == "roughness_length" else d["n"]
        m = _bed_model(kw, d["bed"], field, 0.05, 0.04)
    Un, _ = m.step(_t(d["U"]), 0.0, 0.01, boundary_level=torch.tensor(0.18, device=DEV))
    (Un * _t(d["w"])).sum().backward()
    gb = m.dem_correction_parameter.grad.cpu().numpy()
    e = _rel(gb, g[f"{case}_gbed"])
    print(case, "d/dbed", e, "vs FP64", _rel(gb, g[f"{case}_gbed64"]))
    assert e <= TOL


def test_thirty_step_bed_gradient_with_regulariser_matches_reference(golden):
    """30 steps on the shoreline crop, gauge loss + dem_regularization(1, 0.1,
    0.01), bounded correction: the gradient w.r.t. dem_correction_parameter,
    stepwise autograd nodes and one forward_checkpointed node."""
    r, g = golden("adj_run_wet"), golden("adj_bed")
    cfg_kw = dict(boundary_left="water_level", boundary_right="wall", boundary_top="wall",
                  boundary_bottom="wall")
    for mode in ("steps", "chunk"):
        m = SWE2D(_t(r["bed"]), _t(r["n"]), float(r["dx"]), float(r["dx"]), config=SWEConfig(**cfg_kw),
                  train_dem=True, maximum_dem_correction=0.05)
        with torch.no_grad():
            m.dem_correction_parameter.copy_(_t(g["run_corr0"]).reshape(m.dem_correction_parameter.shape))
        if mode == "steps":
            loss = _run_loss(m, _t(r["U0"]), _t(r["levels"]), r["gauges"], m.bed[0, 0])
        else:  # one node per step (constant levels differ per step, so chunk = 1 step each)
            U, loss = _t(r["U0"]), 0.0
            for s in range(r["levels"].shape[0]):
                U = forward_checkpointed(m, U, t_end=2.0e-3, boundary_level=_t(r["levels"])[s])
                for iy, ix in r["gauges"]:
                    loss = loss + (U[0, 0, iy, ix] + m.bed[0, 0, iy, ix]) ** 2
            loss = loss + 1e-3 * (U * U).sum()
        loss = loss + m.dem_regularization(1.0, 0.1, 0.01)
        loss.backward()
        assert float(loss.detach()) == pytest.approx(float(g["run_f32_loss"]), rel=2e-6)
        gc = m.dem_correction_parameter.grad.cpu().numpy()
        e = _rel(gc, g["run_f32_gcorr"])
        print(mode, "d/dcorrection", e, "vs FP64", _rel(gc, g["run_f64_gcorr"]))
        assert e <= TOL


def test_bed_gradient_matches_fp64_finite_differences(golden):
    """Central differences (eps 1e-7 m) of the 30-step gauge loss w.r.t. bed
    entries of wet cells, FP64 oracle.  The loss is piecewise smooth in the
    bed as in the depth (eta = h + z feeds the limiters), so the bar is the
    depth entries' 2 %."""
    d = golden("adj_run_wet")
    cfg = SWEConfig(boundary_left="water_level", boundary_right="wall", boundary_top="wall",
                    boundary_bottom="wall")
    m = SWE2D(_t(d["bed"]), _t(d["n"]), float(d["dx"]), float(d["dx"]), config=cfg, train_dem=True)
    _run_loss(m, _t(d["U0"]), _t(d["levels"]), d["gauges"], m.bed[0, 0]).backward()
    gb = m.dem_correction_parameter.grad.cpu().numpy().reshape(d["bed"].shape)

    def loss64(bed):
        om = OracleSWE(bed, d["n"].astype(np.float64), float(d["dx"]), float(d["dx"]), cfg,
                       dtype=np.float64)
        U = d["U0"].astype(np.float64)
        L = 0.0
        for s in range(len(d["levels"])):
            U, _ = om.step(U, 0.0, 2.0e-3, boundary_level=float(d["levels"][s]))
            for iy, ix in d["gauges"]:
                L += (U[0, 0, iy, ix] + float(bed[iy, ix])) ** 2
        return L + 1e-3 * float((U * U).sum())

    bed64 = d["bed"].astype(np.float64)
    wet = (d["U0"][0, 0] > 5e-3).ravel()
    order = [i for i in np.argsort(-np.abs(gb).ravel()) if wet[i]][:4]
    for idx in order:
        up, dn = bed64.ravel().copy(), bed64.ravel().copy()
        up[idx] += 1e-7
        dn[idx] -= 1e-7
        fd = (loss64(up.reshape(bed64.shape)) - loss64(dn.reshape(bed64.shape))) / 2e-7
        print("bed", idx, gb.ravel()[idx], fd)
        assert abs(gb.ravel()[idx] - fd) <= 2e-2 * abs(fd)
