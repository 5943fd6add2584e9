"""Golden gradients of the reference step from PyTorch autograd (adj_*.npz).

Called by make_golden.py (``--only adj``).  Every case is run twice: in
float32 with correctly-rounded sqrt/pow (the arithmetic the kernels
reproduce, see make_golden.py) and in float64 (the accuracy oracle).

adj_step.npz  one step, random state with wet, dry and near-dry cells, for
              several boundary / friction configurations: L = sum(w * U_new)
              for a seeded random w; gradients w.r.t. U, the level and the
              roughness field.
adj_run.npz   30 steps of a 40x56 crop of the runup bathymetry above the
              shoreline (dry at the start, flooded from the west), west water
              level given per step (30 values), fixed max_dt = 2e-3 (below the
              CFL step, so dt is the same in every evaluation); L = sum over
              steps and three gauges of eta^2 plus 1e-3 sum(U_final^2);
              gradients w.r.t. U0, the 30 levels and n.
adj_run_wet.npz  the same on a crop across the shoreline (92 % wet at the
              start), where U0 and n have smooth gradients for finite
              differences (every U0 entry of the dry crop sits on the wet/dry
              kink).
adj_bed.npz   gradients w.r.t. dem_correction_parameter (the bed of the
              DEM-correction inversion, src/solver.py:111-147): the one-step
              cases of adj_step.npz with train_dem=True, one case with the
              tanh bound (maximum_dem_correction=0.05), a partial valid mask
              and a nonzero correction; and the 30-step loss of
              adj_run_wet.npz plus dem_regularization(1.0, 0.1, 0.01)
              (src/solver.py:807-836) with the same bound.
"""
from __future__ import annotations

import numpy as np
import torch

from make_golden import correctly_rounded_elementary, random_bed, random_state

from diffswe2d_b200 import scenarios

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


def _grads_step(ref, dtype, cfg_kw, U, bed, n, level, w, dx, dy, max_dt):
    cfg = ref.SWEConfig(**cfg_kw, constant_value=0.05)
    m = ref.SWE2D(torch.from_numpy(bed).to(dtype), torch.from_numpy(n).to(dtype), dx, dy, config=cfg,
                  train_dem=False)
    m.roughness_length.requires_grad_(True)
    Ut = torch.from_numpy(U).to(dtype).requires_grad_(True)
    lv = torch.tensor(level, dtype=dtype, requires_grad=True)
    Un, dt = m.step(Ut, 0.0, max_dt, boundary_level=lv)
    loss = (Un * torch.from_numpy(w).to(dtype)).sum()
    loss.backward()
    gl = float(lv.grad) if lv.grad is not None else 0.0
    gn = (m.roughness_length.grad.numpy().astype(np.float64) if m.roughness_length.grad is not None
          else np.zeros((1, 1) + n.shape, np.float64))
    return Ut.grad.numpy().astype(np.float64), gl, gn, dt


def _grads_step_bed(ref, dtype, cfg_kw, U, bed, n, level, w, dx, dy, max_dt, max_corr=None,
                    mask=None, corr0=None):
    cfg = ref.SWEConfig(**cfg_kw, constant_value=0.05)
    m = ref.SWE2D(torch.from_numpy(bed).to(dtype), torch.from_numpy(n).to(dtype), dx, dy, config=cfg,
                  train_dem=True, maximum_dem_correction=max_corr,
                  valid_mask=None if mask is None else torch.from_numpy(mask))
    if corr0 is not None:
        with torch.no_grad():
            m.dem_correction_parameter.copy_(torch.from_numpy(corr0).to(dtype).reshape(
                m.dem_correction_parameter.shape))
    Un, _ = m.step(torch.from_numpy(U).to(dtype), 0.0, max_dt, boundary_level=level)
    (Un * torch.from_numpy(w).to(dtype)).sum().backward()
    return m.dem_correction_parameter.grad.numpy().astype(np.float64)


def make_bed_grads(ref, out):
    d = dict(np.load(out / "adj_step.npz"))
    rng = np.random.default_rng(78)
    mask = rng.uniform(size=d["bed"].shape) > 0.2
    corr0 = (rng.normal(size=d["bed"].shape) * 0.5).astype(np.float32)
    g = {"mask": mask, "corr0": corr0}
    for name, kw in STEP_CASES.items():
        field = d["z0"] if kw.get("frictionmodel") == "roughness_length" else d["n"]
        args = (kw, d["U"], d["bed"], field, 0.18, d["w"], 0.05, 0.04, 0.01)
        with correctly_rounded_elementary():
            g[f"{name}_gbed"] = _grads_step_bed(ref, torch.float32, *args)
        g[f"{name}_gbed64"] = _grads_step_bed(ref, torch.float64, *args)
    kw = STEP_CASES["water_level"]
    args = (kw, d["U"], d["bed"], d["n"], 0.18, d["w"], 0.05, 0.04, 0.01)
    with correctly_rounded_elementary():
        g["tanh_mask_gbed"] = _grads_step_bed(ref, torch.float32, *args, 0.05, mask, corr0)
    g["tanh_mask_gbed64"] = _grads_step_bed(ref, torch.float64, *args, 0.05, mask, corr0)
    # 30-step run on the shoreline crop with the DEM regulariser
    r = dict(np.load(out / "adj_run_wet.npz"))
    corr_run = (rng.normal(size=r["bed"].shape) * 0.3).astype(np.float32)
    g["run_corr0"] = corr_run
    kw = dict(boundary_left="water_level", boundary_right="wall", boundary_top="wall",
              boundary_bottom="wall")
    for dtype, tag, cr in ((torch.float32, "f32", True), (torch.float64, "f64", False)):
        m = ref.SWE2D(torch.from_numpy(r["bed"]).to(dtype), torch.from_numpy(r["n"]).to(dtype),
                      float(r["dx"]), float(r["dx"]), config=ref.SWEConfig(**kw), train_dem=True,
                      maximum_dem_correction=0.05)
        with torch.no_grad():
            m.dem_correction_parameter.copy_(torch.from_numpy(corr_run).to(dtype).reshape(
                m.dem_correction_parameter.shape))
        ctx = correctly_rounded_elementary() if cr else _Null()
        with ctx:
            loss = run_loss(m, dtype, torch.from_numpy(r["U0"]).to(dtype),
                            torch.from_numpy(r["levels"]).to(dtype), RUN_GAUGES, m.bed[0, 0], None,
                            None, float(r["dx"]))
            loss = loss + m.dem_regularization(1.0, 0.1, 0.01)
            loss.backward()
        g[f"run_{tag}_loss"] = float(loss)
        g[f"run_{tag}_gcorr"] = m.dem_correction_parameter.grad.numpy().astype(np.float64)
    np.savez_compressed(out / "adj_bed.npz", **g)
    print("adj_bed.npz", g["run_f32_loss"], g["run_f64_loss"])


def make_step_grads(ref, out):
    rng = np.random.default_rng(77)
    ny, nx = 11, 14
    d = {}
    U = random_state(rng, 1, ny, nx)
    bed = random_bed(rng, 1, ny, nx)[0, 0]
    n = rng.uniform(0.005, 0.04, size=(ny, nx)).astype(np.float32)
    z0 = rng.uniform(0.0005, 0.01, size=(ny, nx)).astype(np.float32)
    w = rng.normal(size=U.shape).astype(np.float32)
    d["U"], d["bed"], d["n"], d["z0"], d["w"] = U, bed, n, z0, w
    level = 0.18
    for name, kw in STEP_CASES.items():
        field = z0 if kw.get("frictionmodel") == "roughness_length" else n
        with correctly_rounded_elementary():
            gU, gl, gn, dt = _grads_step(ref, torch.float32, kw, U, bed, field, level, w, 0.05, 0.04, 0.01)
        d[f"{name}_gU"], d[f"{name}_glevel"], d[f"{name}_gn"], d[f"{name}_dt"] = gU, gl, gn, dt
        gU, gl, gn, dt = _grads_step(ref, torch.float64, kw, U, bed, field, level, w, 0.05, 0.04, 0.01)
        d[f"{name}_gU64"], d[f"{name}_glevel64"], d[f"{name}_gn64"] = gU, gl, gn
    np.savez_compressed(out / "adj_step.npz", **d)
    print("adj_step.npz", len(STEP_CASES), "cases")


RUN_STEPS = 30
RUN_GAUGES = ((10, 20), (20, 30), (30, 44))


def run_loss(ref_or_model, dtype, U0, levels, gauges, bed, n, crop_cfg, dx, steps=RUN_STEPS):
    """Shared definition of the multi-step loss (reference side)."""
    m = ref_or_model
    Ut = U0
    loss = 0.0
    for s in range(steps):
        Ut, _ = m.step(Ut, 0.0, 2.0e-3, boundary_level=levels[s])
        for (iy, ix) in gauges:
            eta = Ut[0, 0, iy, ix] + bed[iy, ix]
            loss = loss + eta * eta
    return loss + 1e-3 * (Ut * Ut).sum()


def make_run_grads(ref, out, name="adj_run", r0=100, c0=296):
    sc = scenarios.runup(seed=0)
    bed = np.ascontiguousarray(sc.bed[r0:r0 + 40, c0:c0 + 56])
    n = np.ascontiguousarray(sc.roughness[r0:r0 + 40, c0:c0 + 56])
    U0 = np.ascontiguousarray(sc.U0[:, :, r0:r0 + 40, c0:c0 + 56])
    dx = sc.dx
    levels = (0.004 + 0.01 * np.sin(np.linspace(0.0, 3.0, RUN_STEPS))).astype(np.float32)
    d = dict(bed=bed, n=n, U0=U0, levels=levels, dx=np.float64(dx),
             gauges=np.array(RUN_GAUGES, np.int32))
    kw = dict(boundary_left="water_level", boundary_right="wall", boundary_top="wall",
              boundary_bottom="wall")
    for dtype, tag, cr in ((torch.float32, "f32", True), (torch.float64, "f64", False)):
        cfg = ref.SWEConfig(**kw)
        m = ref.SWE2D(torch.from_numpy(bed).to(dtype), torch.from_numpy(n).to(dtype), dx, dx, config=cfg,
                      train_dem=False)
        m.roughness_length.requires_grad_(True)
        Ut = torch.from_numpy(U0).to(dtype).requires_grad_(True)
        lv = torch.from_numpy(levels).to(dtype).requires_grad_(True)
        bed_t = torch.from_numpy(bed).to(dtype)
        ctx = correctly_rounded_elementary() if cr else _Null()
        with ctx:
            loss = run_loss(m, dtype, Ut, lv, RUN_GAUGES, bed_t, None, None, dx)
            loss.backward()
        d[f"{tag}_loss"] = float(loss)
        d[f"{tag}_gU0"] = Ut.grad.numpy().astype(np.float64)
        d[f"{tag}_glevels"] = lv.grad.numpy().astype(np.float64)
        d[f"{tag}_gn"] = m.roughness_length.grad.numpy().astype(np.float64)
    np.savez_compressed(out / f"{name}.npz", **d)
    print(f"{name}.npz", d["f32_loss"], d["f64_loss"])


class _Null:
    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False


def make_adjoint(ref, out):
    make_step_grads(ref, out)
    make_run_grads(ref, out)
    make_run_grads(ref, out, "adj_run_wet", 100, 170)
    make_bed_grads(ref, out)
