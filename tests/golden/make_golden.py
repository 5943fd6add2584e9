"""Generate the golden fixtures of tests/golden/ from the DiffSWE2d reference.

Run where the reference's source tree is available, given by --ref or the
environment variable DIFFSWE2D_REFERENCE; the fixtures it writes are what the
tests read, so the reference itself never has to be present where the tests
run:

    python tests/golden/make_golden.py --ref <reference checkout> [--only ops,c1,c2,forcing,cea,adj]

The reference is imported as the package ``diffswe2d`` from its ``src/``
directory.  Its ``io_netcdf`` module imports ``xarray`` at load time, which
the step never uses; when xarray is absent a stub module is registered so the
import succeeds.  All reference runs use PyTorch on the CPU.

Fixtures (numpy .npz, float32 unless noted):
  ops.npz         operator-level inputs/outputs on small random grids
  c1_island.npz   256x256 Gaussian-island config, FP32 states at steps
                  1/10/100/1000 and the FP64 reference (rounded to float32)
  c2_runup.npz    244x393 runup config with dynamic west water level,
                  FP32 states at steps 1/50/200 and a forward() chunk
  adj_step.npz, adj_run.npz   reference autograd gradients (make_golden_adjoint.py)
  spline.npz      clamped B-spline basis and bounded controls of the
                  reference's inversion script
  cea_topo.npz    the CEA 2008 DEM (an ESRI ASCII raster of the reference's
                  examples) as the reference's io_ascii reader grids it
  forcing.npz     rainfall and infiltration sources: spatial_operator with
                  scalar / field / per-batch rates, steps with infiltration,
                  and steps of a model forced by RainfallForcing
"""
from __future__ import annotations

import argparse
import importlib.machinery
import importlib.util
import pathlib
import sys
import time
import types

import numpy as np
import torch

HERE = pathlib.Path(__file__).resolve().parent
REPO = HERE.parent.parent
sys.path.insert(0, str(REPO))

from diffswe2d_b200 import scenarios  # noqa: E402


def load_reference(root: str):
    src = pathlib.Path(root) / "src"
    if "xarray" not in sys.modules:
        try:
            import xarray  # noqa: F401
        except ImportError:
            stub = types.ModuleType("xarray")
            stub.__spec__ = importlib.machinery.ModuleSpec("xarray", None)
            sys.modules["xarray"] = stub
    spec = importlib.util.spec_from_file_location(
        "diffswe2d", src / "__init__.py", submodule_search_locations=[str(src)])
    pkg = importlib.util.module_from_spec(spec)
    sys.modules["diffswe2d"] = pkg
    spec.loader.exec_module(pkg)
    import diffswe2d.boundary as boundary
    import diffswe2d.friction as friction
    import diffswe2d.numerics as numerics
    import diffswe2d.reconstruction as reconstruction
    import diffswe2d.riemann as riemann
    return types.SimpleNamespace(pkg=pkg, SWE2D=pkg.SWE2D, SWEConfig=pkg.SWEConfig,
                                 boundary=boundary, friction=friction, numerics=numerics,
                                 reconstruction=reconstruction, riemann=riemann)


BC_TYPES = ["transmissive", "periodic", "constant", "water_level", "wall", "absorbing"]
BC_CASES = [
    ("all_" + t, dict(boundary_left=t, boundary_right=t, boundary_top=t, boundary_bottom=t))
    for t in BC_TYPES
] + [
    ("mixed_a", dict(boundary_left="water_level", boundary_right="wall", boundary_top="periodic",
                     boundary_bottom="absorbing")),
    ("mixed_b", dict(boundary_left="constant", boundary_right="transmissive", boundary_top="wall",
                     boundary_bottom="water_level")),
    ("mixed_c", dict(boundary_left="periodic", boundary_right="periodic", boundary_top="wall",
                     boundary_bottom="wall")),
]


def random_state(rng, B, ny, nx, dry_frac=0.25):
    h = rng.uniform(0.0, 1.0, size=(B, ny, nx))
    h[rng.uniform(size=h.shape) < dry_frac] = 0.0
    h[rng.uniform(size=h.shape) < 0.05] = 1e-7  # below dry_depth
    hu = rng.normal(0.0, 0.3, size=h.shape) * (h > 0)
    hv = rng.normal(0.0, 0.3, size=h.shape) * (h > 0)
    U = np.stack([h, hu, hv], axis=1).astype(np.float32)
    return U


def random_bed(rng, B, ny, nx):
    y, x = np.meshgrid(np.linspace(0, 1, ny), np.linspace(0, 1, nx), indexing="ij")
    base = -0.5 + 0.8 * x + 0.2 * np.sin(6 * y)
    bed = base[None, None] + rng.normal(0.0, 0.05, size=(B, 1, ny, nx))
    return bed.astype(np.float32)


def t32(a):
    return torch.from_numpy(np.ascontiguousarray(a))


def make_ops(ref, out):
    rng = np.random.default_rng(1234)
    B, ny, nx = 2, 9, 13
    d = {}
    U = random_state(rng, B, ny, nx)
    bed = random_bed(rng, B, ny, nx)
    bed1 = bed[:1]
    n = rng.uniform(0.0, 0.05, size=(1, 1, ny, nx)).astype(np.float32)
    d["U"], d["bed"], d["bed1"], d["n"] = U, bed, bed1, n
    level_b = np.array([0.15, 0.3], dtype=np.float32)
    d["level_b"] = level_b
    cfg0 = ref.SWEConfig()
    g, eps, dry = cfg0.gravity, cfg0.epsilon, cfg0.dry_depth
    with torch.no_grad():
        # primitive / limited increment / minmod
        h, u, v, c = ref.riemann.primitive(t32(U), g, eps, dry)
        d["prim_h"], d["prim_u"], d["prim_v"], d["prim_c"] = (x.numpy() for x in (h, u, v, c))
        q = rng.normal(size=(B, 3, ny, nx)).astype(np.float32)
        q[:, :, ::3, ::2] = 0.0
        d["li_q"] = q
        d["li_x"] = ref.numerics.limited_increment(t32(q), -1, 1.3).numpy()
        d["li_y"] = ref.numerics.limited_increment(t32(q), -2, 1.3).numpy()
        # ghost cells for each boundary case, scalar and per-batch level
        for name, bcs in BC_CASES:
            for lname, lev in (("s", 0.2), ("b", t32(level_b))):
                for bname, bb in (("bB", bed), ("b1", bed1)):
                    Up, zp = ref.boundary.add_ghost_cells(t32(U), t32(bb), 2, constant_value=0.05,
                                                          constant_level=lev, **bcs)
                    d[f"gc_{name}_{lname}_{bname}_Up"] = Up.numpy()
                    d[f"gc_{name}_{lname}_{bname}_zp"] = zp.numpy()
        # reconstruction + flux on a padded wall grid
        Up, zp = ref.boundary.add_ghost_cells(t32(U), t32(bed), 2, "wall", "water_level", "wall",
                                              "transmissive", constant_level=0.2)
        d["rc_Up"], d["rc_zp"] = Up.numpy(), zp.numpy()
        for dim, tag in ((-1, "x"), (-2, "y")):
            for wsr in (True, False):
                UL, UR, sL, sR = ref.reconstruction.bflood_cn_reconstruction(
                    Up, zp, dim, g, eps, dry, 1.3, wsr)
                k = f"rc_{tag}_{int(wsr)}"
                d[k + "_UL"], d[k + "_UR"], d[k + "_sL"], d[k + "_sR"] = (
                    x.numpy() for x in (UL, UR, sL, sR))
            UL, UR, _, _ = ref.reconstruction.bflood_cn_reconstruction(Up, zp, dim, g, eps, dry)
            F, s = ref.riemann.bflood_hllc_flux(UL, UR, tag, g, eps, dry)
            d[f"hll_{tag}_UL"], d[f"hll_{tag}_UR"] = UL.numpy(), UR.numpy()
            d[f"hll_{tag}_F"], d[f"hll_{tag}_s"] = F.numpy(), s.numpy()
        # friction
        dt = torch.tensor(0.01, dtype=torch.float32)
        d["fr_dt"] = np.float32(0.01)
        d["fr_manning"] = ref.friction.apply_manning_friction(t32(U), t32(n), dt).numpy()
        z0 = rng.uniform(0.0, 0.02, size=(1, 1, ny, nx)).astype(np.float32)
        d["fr_z0"] = z0
        d["fr_rough"] = ref.friction.apply_roughness_length_friction(t32(U), t32(z0), dt).numpy()
        # spatial operator, clean_and_limit and one/five steps per boundary case
        for name, bcs in BC_CASES:
            cfg = ref.SWEConfig(**bcs, constant_value=0.05, constant_level=0.2)
            m = ref.SWE2D(t32(bed1[0, 0]), t32(n[0, 0]), 0.05, 0.04, config=cfg, train_dem=False)
            rhs, ax, ay = m.spatial_operator(t32(U), return_wave_speed=True, boundary_level=0.2)
            d[f"so_{name}_rhs"], d[f"so_{name}_axay"] = rhs.numpy(), np.array([ax, ay], np.float32)
            Us, dts = t32(U), []
            for k in range(5):
                Us, dt_k = m.step(Us, 0.0, 0.05, boundary_level=0.2)
                dts.append(dt_k)
                if k == 0:
                    d[f"st_{name}_1"] = Us.numpy()
            d[f"st_{name}_5"], d[f"st_{name}_dts"] = Us.numpy(), np.array(dts, np.float64)
        cand = U + rng.normal(0, 0.2, size=U.shape).astype(np.float32)
        d["cl_cand"] = cand
        cfg = ref.SWEConfig()
        m = ref.SWE2D(t32(bed1[0, 0]), t32(n[0, 0]), 0.05, 0.04, config=cfg, train_dem=False)
        d["cl_out"] = m._clean_and_limit(t32(U), t32(cand)).numpy()
        # per-batch bed and level with a batch of two
        cfg = ref.SWEConfig(boundary_left="water_level", boundary_right="wall",
                            boundary_top="wall", boundary_bottom="water_level")
        m = ref.SWE2D(t32(bed), t32(np.broadcast_to(n, bed.shape)), 0.05, 0.04, config=cfg,
                      train_dem=False)
        Us, dt_k = m.step(t32(U), 0.0, 0.05, boundary_level=t32(level_b))
        d["stb_U"], d["stb_dt"] = Us.numpy(), np.float64(dt_k)
        d["stb_n"] = np.ascontiguousarray(np.broadcast_to(n, bed.shape))
    np.savez_compressed(out / "ops.npz", **d)
    print("ops.npz", len(d), "arrays")


class correctly_rounded_elementary:
    """Context manager: evaluate the reference's float32 sqrt and pow correctly
    rounded (through float64), leaving every other operation untouched.

    PyTorch's CPU build computes float32 sqrt (MKL VML) and pow (SLEEF) to
    within an ulp but not always correctly rounded; under this patch the
    reference's step is the exact function that correctly-rounded FP32
    arithmetic defines, so fixtures made with it pin a correctly-rounded
    implementation bit for bit.
    """

    def __enter__(self):
        self._sqrt, self._pow = torch.sqrt, torch.Tensor.pow
        sqrt, pow_ = self._sqrt, self._pow

        def cr_sqrt(x, *args, **kwargs):
            if torch.is_tensor(x) and x.dtype == torch.float32 and not args and not kwargs:
                return sqrt(x.double()).float()
            return sqrt(x, *args, **kwargs)

        def cr_pow(self_, exponent):
            if self_.dtype == torch.float32 and not torch.is_tensor(exponent):
                return pow_(self_.double(), float(np.float32(exponent))).float()
            return pow_(self_, exponent)

        torch.sqrt, torch.Tensor.pow = cr_sqrt, cr_pow
        return self

    def __exit__(self, *exc):
        torch.sqrt, torch.Tensor.pow = self._sqrt, self._pow
        return False


def run_steps(m, U, nsteps, keep, dyn=None, max_dt=1.0e9):
    """Drive step() as forward() does for a dynamic boundary, recording states."""
    states, dts, t = {}, [], 0.0
    with torch.no_grad():
        for i in range(1, nsteps + 1):
            level = None if dyn is None else m._interpolate_dynamic_boundary(t, U)
            U, dt = m.step(U, t, max_dt, boundary_level=level)
            t += dt
            dts.append(dt)
            if i in keep:
                states[i] = U.numpy().copy()
    return states, np.array(dts, np.float64)


def make_c1(ref, out):
    """Gaussian island, 256x256, 1000 steps: stock FP32 and FP64 reference, and
    the FP32 reference with correctly-rounded sqrt/pow ("f32cr")."""
    sc = scenarios.gaussian_island(256, seed=0)
    d = dict(bed=sc.bed, n=sc.roughness, U0=sc.U0, dx=np.float64(sc.dx))
    keep = (1, 1000)
    runs = ((torch.float32, "f32", False), (torch.float64, "f64", False), (torch.float32, "f32cr", True))
    for dtype, tag, cr in runs:
        cfg = ref.SWEConfig(**sc.config)
        m = ref.SWE2D(t32(sc.bed).to(dtype), t32(sc.roughness).to(dtype), sc.dx, sc.dy, config=cfg,
                      train_dem=False)
        t0 = time.perf_counter()
        if cr:
            with correctly_rounded_elementary():
                states, dts = run_steps(m, t32(sc.U0).to(dtype), 1000, keep)
        else:
            states, dts = run_steps(m, t32(sc.U0).to(dtype), 1000, keep)
        print(f"c1 {tag}: 1000 steps in {time.perf_counter() - t0:.1f}s")
        for k, v in states.items():
            if tag != "f32cr" or k == 1000:
                d[f"{tag}_{k}"] = v.astype(np.float32)
        d[f"{tag}_dts"] = dts
    np.savez_compressed(out / "c1_island.npz", **d)


def make_c2(ref, out):
    """Runup, 244x393, dynamic west level: 200 steps (stock and "cr") and a
    forward() chunk of 0.2 s."""
    sc = scenarios.runup(seed=0)
    d = dict(bed=sc.bed, n=sc.roughness, U0=sc.U0, dx=np.float64(sc.dx), bc_times=sc.bc_times,
             bc_levels=sc.bc_levels)
    cfg = ref.SWEConfig(**sc.config)
    m = ref.SWE2D(t32(sc.bed), t32(sc.roughness), sc.dx, sc.dy, config=cfg, train_dem=False)
    m.set_dynamic_boundary(t32(sc.bc_times), t32(sc.bc_levels))
    t0 = time.perf_counter()
    states, dts = run_steps(m, t32(sc.U0), 200, (1, 200), dyn=True)
    print(f"c2 f32: 200 steps in {time.perf_counter() - t0:.1f}s")
    for k, v in states.items():
        d[f"f32_{k}"] = v
    d["f32_dts"] = dts
    with correctly_rounded_elementary():
        cr_states, cr_dts = run_steps(m, t32(sc.U0), 200, (200,), dyn=True)
        d["f32cr_200"], d["f32cr_dts"] = cr_states[200], cr_dts
        # forward() chunk of 0.2 s from the 200-step state, starting at 1.0 s
        count = []
        with torch.no_grad():
            U, hmax = m(t32(cr_states[200]), t_end=0.2, start_time=1.0,
                        callback=lambda it, t, U: count.append(t))
    d["fwcr_U"], d["fwcr_hmax"], d["fwcr_times"] = U.numpy(), hmax.numpy(), np.array(count, np.float64)
    np.savez_compressed(out / "c2_runup.npz", **d)


def make_forcing(ref, out):
    """Rainfall and infiltration (src/solver.py:437-446, :520-525, :607-643):
    the tendency with scalar, field and per-batch rates, five steps with
    infiltration, and five steps of a model with a RainfallForcing, all
    with correctly-rounded sqrt/pow ("cr"), plus the stock tendency."""
    import diffswe2d.forcing as forcing
    rng = np.random.default_rng(4321)
    B, ny, nx = 2, 24, 40
    U = random_state(rng, B, ny, nx, dry_frac=0.15)
    bed1 = random_bed(rng, 1, ny, nx)
    n = rng.uniform(0.01, 0.04, size=(1, 1, ny, nx)).astype(np.float32)
    rain_field = rng.uniform(0.0, 2e-3, size=(1, 1, ny, nx)).astype(np.float32)
    rain_batch = rng.uniform(0.0, 2e-3, size=(B, 1, ny, nx)).astype(np.float32)
    infil_field = rng.uniform(-5e-4, 1e-3, size=(1, 1, ny, nx)).astype(np.float32)
    infil_batch = rng.uniform(-5e-4, 1e-3, size=(B, 1, ny, nx)).astype(np.float32)
    r_times = np.array([0.0, 0.004, 0.02], np.float32)
    r_rates = rng.uniform(0.0, 5e-3, size=(3, 1, ny, nx)).astype(np.float32)
    d = dict(U=U, bed1=bed1, n=n, rain_field=rain_field, rain_batch=rain_batch,
             infil_field=infil_field, infil_batch=infil_batch, r_times=r_times, r_rates=r_rates)
    cfg = ref.SWEConfig(boundary_left="water_level", boundary_right="wall", boundary_top="wall",
                        boundary_bottom="transmissive", constant_level=0.2)
    cases = {
        "scalar": (1.5e-3, 4e-4),
        "field": (rain_field, infil_field),
        "batch": (rain_batch, infil_batch),
    }
    with torch.no_grad():
        m = ref.SWE2D(t32(bed1[0, 0]), t32(n[0, 0]), 0.05, 0.04, config=cfg, train_dem=False)
        for tag, (rain, infil) in cases.items():
            r = rain if np.isscalar(rain) else t32(rain)
            i = infil if np.isscalar(infil) else t32(infil)
            rhs = m.spatial_operator(t32(U), rainfall_rate=r, infiltration=i, boundary_level=0.2)
            d[f"so_{tag}"] = rhs.numpy()
            with correctly_rounded_elementary():
                rhs, ax, ay = m.spatial_operator(t32(U), rainfall_rate=r, infiltration=i,
                                                 boundary_level=0.2, return_wave_speed=True)
            d[f"socr_{tag}"] = rhs.numpy()
            d[f"socr_{tag}_axay"] = np.array([ax, ay], np.float32)
        for tag, infil in (("scalar", 4e-4), ("field", infil_field), ("batch", infil_batch)):
            i = infil if np.isscalar(infil) else t32(infil)
            Us, dts = t32(U), []
            with correctly_rounded_elementary():
                for _ in range(5):
                    Us, dt = m.step(Us, 0.0, 0.05, infiltration=i, boundary_level=0.2)
                    dts.append(dt)
            d[f"stcr_infil_{tag}"], d[f"stcr_infil_{tag}_dts"] = Us.numpy(), np.array(dts, np.float64)
        rf = forcing.RainfallForcing(t32(r_times), t32(r_rates))
        mr = ref.SWE2D(t32(bed1[0, 0]), t32(n[0, 0]), 0.05, 0.04, config=cfg, train_dem=False,
                       rainfall=rf)
        Us, dts, t = t32(U), [], 0.0
        with correctly_rounded_elementary():
            for _ in range(5):
                Us, dt = mr.step(Us, t, 0.05, infiltration=t32(infil_field), boundary_level=0.2)
                dts.append(dt)
                t += dt
        d["stcr_rainfall"], d["stcr_rainfall_dts"] = Us.numpy(), np.array(dts, np.float64)
        d["rf_at"] = np.stack([rf.at(tt).numpy() for tt in (0.0, 0.001, 0.0137, 0.5)])
    np.savez_compressed(out / "forcing.npz", **d)
    print("forcing.npz", len(d), "arrays")


def make_cea(ref_root, out):
    """The CEA 2008 rainfall-runoff DEM (Examples/forward/Cea2008/
    Cea2008_C1_new/topo.asc, ESRI ASCII) read and regridded by the
    reference's own reader onto the example's model grid (example_run.py:
    ModelGrid.from_bounds(0.02, 2.02, -0.005, 2.535, 0.01), float64)."""
    import diffswe2d.io_ascii as io_ascii
    from diffswe2d.io_netcdf import ModelGrid
    path = pathlib.Path(ref_root) / "Examples/forward/Cea2008/Cea2008_C1_new/topo.asc"
    grid = ModelGrid.from_bounds(xmin=0.02, xmax=2.02, ymin=-0.005, ymax=2.535, resolution=0.01,
                                 dtype=torch.float64, device="cpu")
    bed, spec = io_ascii.ascii_to_tensor(path, grid, dtype=torch.float64)
    np.savez_compressed(out / "cea_topo.npz", bed=bed.numpy(), dx=np.float64(spec.resolution),
                        bounds=np.array([spec.xmin, spec.xmax, spec.ymin, spec.ymax]))
    print("cea_topo.npz", tuple(bed.shape))


def main():
    import os
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("DIFFSWE2D_REFERENCE"),
                    help="checkout of the reference (or set DIFFSWE2D_REFERENCE)")
    ap.add_argument("--only", default="ops,c1,c2,forcing")
    args = ap.parse_args()
    if not args.ref:
        ap.error("give the reference checkout with --ref or DIFFSWE2D_REFERENCE")
    torch.set_num_threads(max(1, torch.get_num_threads()))
    ref = load_reference(args.ref)
    groups = set(args.only.split(","))
    if "ops" in groups:
        make_ops(ref, HERE)
    if "c1" in groups:
        make_c1(ref, HERE)
    if "c2" in groups:
        make_c2(ref, HERE)
    if "forcing" in groups:
        make_forcing(ref, HERE)
    if "cea" in groups:
        make_cea(args.ref, HERE)
    if "adj" in groups:
        from make_golden_adjoint import make_adjoint  # noqa: E402
        make_adjoint(ref, HERE)
    if "spline" in groups:
        make_spline(args.ref, HERE)



def make_spline(ref_root, out):
    """Clamped cubic B-spline basis of the reference's inversion script
    (Examples/inverse/**/bc_inversion_train.py:189-231) for two sample grids."""
    import importlib.util
    import pathlib as _pl
    script = next(_pl.Path(ref_root).glob("Examples/inverse/*/*_6simg/bc_inversion_train.py"))
    spec = importlib.util.spec_from_file_location("bc_inversion_train", script)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    d = {}
    for tag, (t_end, n, ctl) in {"a": (22.5, 1125, 16), "b": (29.8, 150, 20), "c": (22.5, 226, 16)}.items():
        times = torch.linspace(0.0, t_end, n, dtype=torch.float64)
        basis, knots, greville = mod.build_clamped_bspline_basis(times, ctl, 3)
        d[f"{tag}_times"] = times.numpy()
        d[f"{tag}_basis"] = basis.numpy()
        d[f"{tag}_knots"] = knots.numpy()
        d[f"{tag}_greville"] = greville.numpy()
        raw = torch.linspace(-2.0, 2.0, ctl, dtype=torch.float64)
        d[f"{tag}_raw"] = raw.numpy()
        d[f"{tag}_bounded"] = mod.bounded_control_values(raw).numpy()
    np.savez_compressed(out / "spline.npz", **d)
    print("spline.npz", len(d))


if __name__ == "__main__":
    main()
