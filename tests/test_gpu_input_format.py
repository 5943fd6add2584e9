"""A DEM from the reference's own input format: the CEA 2008 rainfall-runoff
raster (an ESRI ASCII file of the reference's examples), read and regridded
by the reference's io_ascii.ascii_to_tensor onto the example's model grid
(tests/golden/cea_topo.npz), stepped by SWE2D with the example's boundaries
and Manning n: the IEEE kernels bit for bit against the CPU oracle, the
tolerance mode within its bound."""
import numpy as np
import pytest
import torch

from conftest import field_errors
from oracle import OracleSWE

from diffswe2d_b200 import SWE2D, SWEConfig

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
# Examples/forward/Cea2008/Cea2008_C1_new/example_run.py: boundaries, friction
CFG = dict(boundary_left="wall", boundary_right="wall", boundary_top="wall",
           boundary_bottom="transmissive", frictionmodel="manning")


def _case(golden):
    d = golden("cea_topo")
    bed = d["bed"].astype(np.float32)  # float32 model from the reader's float64 grid
    ny, nx = bed.shape
    y, x = np.meshgrid(np.arange(ny) * 0.01, np.arange(nx) * 0.01, indexing="ij")
    hump = 0.03 * np.exp(-((x - 1.0) ** 2 + (y - 1.6) ** 2) / (2 * 0.15 ** 2))
    h = np.maximum(-0.1 + hump - bed.astype(np.float64), 0.0)
    U0 = np.stack([h, np.zeros_like(h), np.zeros_like(h)])[None].astype(np.float32)
    n = np.full_like(bed, 0.012)
    return bed, n, U0, float(d["dx"])


@pytest.mark.parametrize("arithmetic", ["exact", "fast"])
def test_cea_dem_steps(golden, arithmetic):
    bed, n, U0, dx = _case(golden)
    assert bed.shape == (254, 200)
    cfg = SWEConfig(**CFG)
    m = SWE2D(torch.from_numpy(bed).to(DEV), torch.from_numpy(n).to(DEV), dx, dx, config=cfg,
              train_dem=False, arithmetic=arithmetic)
    om = OracleSWE(bed, n, dx, dx, cfg)
    U, Uo, t = torch.from_numpy(U0).to(DEV), U0, 0.0
    for k in range(20):
        U, dt = m.step(U, t, 1.0e9)
        Uo, dto = om.step(Uo, t, 1.0e9)
        t += dto
        if arithmetic == "exact":
            assert dt == dto and np.array_equal(U.cpu().numpy(), Uo), f"step {k + 1}"
    err = field_errors(U.cpu().numpy(), Uo)
    print(arithmetic, "after 20 steps", err)
    assert err[0] <= 1e-5 and err[1] <= 1e-4 and err[2] <= 1e-4
