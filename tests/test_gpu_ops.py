"""Operator-level drop-ins on the GPU against the reference's golden outputs
(bit-exact where the operator has no sqrt/pow) and against the CPU oracle
(bit-exact everywhere)."""
import numpy as np
import pytest
import torch

from conftest import BC_CASES, bc_kwargs
from oracle import Oracle

import diffswe2d_b200 as d2
from diffswe2d_b200 import SWE2D, SWEConfig

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def _t(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


def _np(t):
    return t.detach().cpu().numpy()


@pytest.mark.parametrize("case", sorted(BC_CASES))
@pytest.mark.parametrize("lname", ["s", "b"])
@pytest.mark.parametrize("bname", ["bB", "b1"])
def test_add_ghost_cells(golden, case, lname, bname):
    d = golden("ops")
    bed = d["bed"] if bname == "bB" else d["bed1"]
    level = 0.2 if lname == "s" else _t(d["level_b"])
    Up, zp = d2.add_ghost_cells(_t(d["U"]), _t(bed), 2, constant_value=0.05, constant_level=level,
                                **bc_kwargs(case))
    key = f"gc_{case}_{lname}_{bname}"
    assert np.array_equal(_np(Up), d[key + "_Up"])
    assert np.array_equal(_np(zp), d[key + "_zp"])


def test_add_ghost_cells_validation():
    U = torch.zeros(1, 3, 4, 4, device=DEV)
    bed = torch.zeros(1, 1, 4, 4, device=DEV)
    with pytest.raises(ValueError, match="Unsupported left"):
        d2.add_ghost_cells(U, bed, 2, boundary_left="nope")
    with pytest.raises(ValueError, match="ng cannot exceed"):
        d2.add_ghost_cells(U, bed, 5)
    with pytest.raises(ValueError, match="three channels"):
        d2.add_ghost_cells(torch.zeros(1, 2, 4, 4, device=DEV), bed, 2)


def test_primitive(golden):
    d = golden("ops")
    outs = d2.primitive(_t(d["U"]), 9.81, 1e-12, 1e-6)
    ref = Oracle().primitive(d["U"], SWEConfig())
    for o, r, name in zip(outs, ref, ("h", "u", "v", "c")):
        assert np.array_equal(_np(o), r), name
        assert np.allclose(_np(o), d[f"prim_{name}"], rtol=2e-7, atol=0)
    with pytest.raises(ValueError):
        d2.primitive(_t(d["U"]), -1.0, 1e-12, 1e-6)


def test_limited_increment_and_minmod(golden):
    d = golden("ops")
    assert np.array_equal(_np(d2.limited_increment(_t(d["li_q"]), -1)), d["li_x"])
    assert np.array_equal(_np(d2.limited_increment(_t(d["li_q"]), -2)), d["li_y"])
    rng = np.random.default_rng(5)
    a, b, c = (rng.normal(size=(4, 7)).astype(np.float32) for _ in range(3))
    a[0, :3] = 0.0
    sa, sb, sc = np.sign(a), np.sign(b), np.sign(c)
    same = (sa == sb) & (sb == sc)
    want = np.where(same, sa * np.minimum(np.abs(a), np.minimum(np.abs(b), np.abs(c))), 0.0)
    assert np.array_equal(_np(d2.minmod3(_t(a), _t(b), _t(c))), want.astype(np.float32))


@pytest.mark.parametrize("tag,dim", [("x", -1), ("y", -2)])
@pytest.mark.parametrize("wsr", [1, 0])
def test_reconstruction(golden, tag, dim, wsr):
    d = golden("ops")
    UL, UR, sL, sR = d2.bflood_cn_reconstruction(_t(d["rc_Up"]), _t(d["rc_zp"]), dim, 9.81, 1e-12,
                                                 1e-6, 1.3, bool(wsr))
    key = f"rc_{tag}_{wsr}"
    for name, a in (("UL", UL), ("UR", UR), ("sL", sL), ("sR", sR)):
        assert np.array_equal(_np(a), d[f"{key}_{name}"]), name


@pytest.mark.parametrize("tag", ["x", "y"])
def test_hll_flux(golden, tag):
    d = golden("ops")
    F, s = d2.bflood_hllc_flux(_t(d[f"hll_{tag}_UL"]), _t(d[f"hll_{tag}_UR"]), tag, 9.81, 1e-12, 1e-6)
    Fo, so = Oracle().hll_flux(d[f"hll_{tag}_UL"], d[f"hll_{tag}_UR"], tag, SWEConfig())
    assert np.array_equal(_np(F), Fo) and np.array_equal(_np(s), so)
    assert np.allclose(_np(F), d[f"hll_{tag}_F"], rtol=1e-6, atol=1e-7)


def test_friction(golden):
    d = golden("ops")
    o = Oracle()
    man = d2.apply_manning_friction(_t(d["U"]), _t(d["n"]), float(d["fr_dt"]))
    assert np.array_equal(_np(man), o.manning(d["U"], d["n"], d["fr_dt"]))
    assert np.allclose(_np(man), d["fr_manning"], rtol=1e-6, atol=1e-9)
    rough = d2.apply_roughness_length_friction(_t(d["U"]), _t(d["fr_z0"]), torch.tensor(0.01))
    assert np.array_equal(_np(rough), o.roughness_friction(d["U"], d["fr_z0"], d["fr_dt"]))
    assert np.allclose(_np(rough), d["fr_rough"], rtol=1e-6, atol=1e-9)


def test_clean_and_limit(golden):
    d = golden("ops")
    bed = torch.zeros(4, 4, device=DEV)
    m = SWE2D(bed, bed + 0.02, 1.0, 1.0, config=SWEConfig(), train_dem=False)
    out = m._clean_and_limit(_t(d["U"]), _t(d["cl_cand"]))
    assert np.array_equal(_np(out), d["cl_out"])
