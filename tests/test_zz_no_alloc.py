"""The step entry point that allocates nothing, swe_step_noalloc_f32.

Some callers cannot give the step its scratch buffers: their process's device
memory is owned by another allocator (a framework's caching allocator or a
memory pool they do not control), or they run a loop that must not allocate
after start-up.  For them the library keeps the step's scratch (stage-1
tendency and reduction words) in a static device array of
SWE_NOALLOC_MAX_CELLS cells and the call takes only inputs and outputs.

These tests call it through the C ABI and check it against swe_step_f32 --
the entry point with caller-owned scratch -- for two calls in a row, with the
tolerance the step's other parity tests use (bit-identical), and check that a
grid beyond the static scratch is rejected before anything runs.  This file
sorts last so that a run stopping at its first failure has run every other
test already.
"""
import ctypes

import pytest
import torch

from diffswe2d_b200 import SWEConfig, scenarios
from diffswe2d_b200 import _native as nat

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda", 0)
MAX_CELLS = 1 << 20  # SWE_NOALLOC_MAX_CELLS
ETOOLARGE = 3        # SWE_ETOOLARGE


def _setup():
    sc = scenarios.runup(ny=120, nx=200, dx=0.014 * 393 / 200, seed=7)
    cfg = SWEConfig(**sc.config)
    p = nat.params(cfg, sc.dx, sc.dy)
    bed = torch.from_numpy(sc.bed).to(DEV)
    n = torch.from_numpy(sc.roughness).to(DEV)
    level = torch.tensor([0.012], dtype=torch.float32, device=DEV)
    U0 = torch.from_numpy(sc.U0).to(DEV)
    return sc, p, bed, n, level, U0


def _regular_step(lib, p, U, bed, n, level, stream):
    B, _, ny, nx = U.shape
    out = torch.empty_like(U)
    scratch = torch.empty_like(U)
    red = torch.empty(nat.RED_WORDS, dtype=torch.int32, device=DEV)
    rc = lib.swe_step_f32(nat.ptr(U), nat.ptr(bed), 1, nat.ptr(n), 1, B, ny, nx, p, nat.ptr(level),
                          1, 0.05, None, 0, 1, nat.ptr(scratch), nat.ptr(red), nat.ptr(out), stream)
    assert rc == nat.SWE_OK
    return out, red[2:4].clone()


def _noalloc_step(lib, p, U, bed, n, level, stream):
    B, _, ny, nx = U.shape
    out = torch.empty_like(U)
    status_dt = torch.full((2,), -1, dtype=torch.int32, device=DEV)
    rc = lib.swe_step_noalloc_f32(nat.ptr(U), nat.ptr(bed), 1, nat.ptr(n), 1, B, ny, nx, p,
                                  nat.ptr(level), 1, 0.05, None, 0, 1, nat.ptr(out),
                                  nat.ptr(status_dt), stream)
    assert rc == nat.SWE_OK
    return out, status_dt


def test_noalloc_step_matches_step_with_caller_scratch_twice():
    lib = nat.lib()
    sc, p, bed, n, level, U0 = _setup()
    stream = nat.stream_handle(DEV)
    U_reg, U_na = U0, U0
    for call in range(2):
        U_reg, sd_reg = _regular_step(lib, p, U_reg, bed, n, level, stream)
        U_na, sd_na = _noalloc_step(lib, p, U_na, bed, n, level, stream)
        torch.cuda.synchronize(DEV)
        assert torch.equal(U_na, U_reg), f"call {call + 1}: state differs"
        assert torch.equal(sd_na, sd_reg), f"call {call + 1}: status/dt differ"
        assert int(sd_na[0]) == 0
        dt = float(sd_na[1:2].view(torch.float32).item())
        assert 0.0 < dt <= 0.05
    assert bool(torch.isfinite(U_na).all())


@pytest.mark.parametrize("arithmetic", ["exact", "fast"])
def test_noalloc_step_at_the_size_limit_twice(arithmetic):
    """A batch of four 512x512 grids fills the static scratch exactly
    (SWE_NOALLOC_MAX_CELLS cells); two calls in a row equal swe_step_f32,
    for both arithmetic modes."""
    lib = nat.lib()
    base = scenarios.tiled(scenarios.runup_at_spin_up(), 512, 512)
    cfg = SWEConfig(**base.config)
    p = nat.params(cfg, base.dx, base.dy, arithmetic)
    bed = torch.from_numpy(base.bed).to(DEV)
    n = torch.from_numpy(base.roughness).to(DEV)
    level = torch.tensor([0.004], dtype=torch.float32, device=DEV)
    U0 = torch.from_numpy(base.U0).to(DEV)
    U0 = torch.cat([U0, U0.flip(-1), U0.flip(-2), U0 * 0.5]).contiguous()
    assert U0.shape[0] * 512 * 512 == MAX_CELLS
    stream = nat.stream_handle(DEV)
    U_reg, U_na = U0, U0
    for call in range(2):
        U_reg, sd_reg = _regular_step(lib, p, U_reg, bed, n, level, stream)
        U_na, sd_na = _noalloc_step(lib, p, U_na, bed, n, level, stream)
        torch.cuda.synchronize(DEV)
        assert torch.equal(U_na, U_reg), f"call {call + 1}: state differs"
        assert torch.equal(sd_na, sd_reg), f"call {call + 1}: status/dt differ"
        assert int(sd_na[0]) == 0


def test_noalloc_step_rejects_grids_beyond_static_scratch():
    lib = nat.lib()
    p = nat.params(SWEConfig(), 1.0, 1.0)
    status_dt = torch.zeros(2, dtype=torch.int32, device=DEV)
    null = ctypes.c_void_p(0)
    ny, nx = 1025, 1024  # one row more than SWE_NOALLOC_MAX_CELLS allows
    assert ny * nx > MAX_CELLS
    rc = lib.swe_step_noalloc_f32(null, null, 1, null, 1, 1, ny, nx, p, null, 1, 0.05, null, 0, 1,
                                  null, nat.ptr(status_dt), nat.stream_handle(DEV))
    assert rc == ETOOLARGE
    rc = lib.swe_step_noalloc_f32(null, null, 1, null, 1, 2, 512, 1025, p, null, 1, 0.05, null, 0,
                                  1, null, nat.ptr(status_dt), nat.stream_handle(DEV))
    assert rc == ETOOLARGE
