"""Device self-test of the step's shared-reciprocal division and square root
against CUDA's IEEE operations (swe_selftest_arith_f32).

The step's quotients must equal IEEE correctly-rounded division bit for bit,
since the reference's float32 tensors divide that way.  The reciprocal and
square root are checked exhaustively over the range the step uses; the
corrected division on random operands and on operands built next to rounding
midpoints.
"""
import numpy as np
import pytest
import torch

from diffswe2d_b200 import _native as nat

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda", 0)


def _selftest(which, n=0, seed=12345):
    fn = nat.lib().swe_selftest_arith_f32
    count = torch.zeros(1, dtype=torch.int64, device=DEV)
    first = torch.zeros(2, dtype=torch.int32, device=DEV)
    rc = fn(which, n, seed, nat.ptr(count), nat.ptr(first), nat.stream_handle(DEV))
    assert rc == nat.SWE_OK
    torch.cuda.synchronize(DEV)
    bad = int(count.item())
    a, b = (int(x) & 0xFFFFFFFF for x in first.tolist())
    return bad, (hex(a), hex(b))


def test_reciprocal_exhaustive():
    bad, first = _selftest(0)
    assert bad == 0, f"{bad} reciprocal mismatches, first input {first}"


def test_square_root_exhaustive():
    bad, first = _selftest(3)
    assert bad == 0, f"{bad} square-root mismatches, first input {first}"


@pytest.mark.parametrize("seed", [1, 2])
def test_division_random_operands(seed):
    bad, first = _selftest(1, n=1 << 34, seed=seed)
    assert bad == 0, f"{bad} division mismatches, first (a, b) = {first}"


def test_division_near_midpoints():
    bad, first = _selftest(2, n=1 << 30, seed=7)
    assert bad == 0, f"{bad} division mismatches, first (a, b) = {first}"



def _f32_bits(v):
    return int(np.array(v, dtype=np.float32).view(np.uint32))


def test_friction_power_exhaustive():
    """pow_pos, the friction's h ** (1/3), against CUDA's double pow rounded
    to float, for every float h in [2^-40, 2^14)."""
    bad, first = _selftest(4, seed=_f32_bits(np.float32(1.0 / 3.0)))
    assert bad == 0, f"{bad} power mismatches, first (x, got) = {first}"


def test_friction_power_derivative_exponent():
    """The adjoint's h ** (1/3 - 1) (exponent rounded to float as the
    kernel rounds it): at most a handful of near-midpoint cases may round
    the other way, a one-ulp difference in a derivative."""
    bad, first = _selftest(4, seed=_f32_bits(np.float32(1.0 / 3.0) - np.float32(1.0)))
    assert bad <= 8, f"{bad} power mismatches, first (x, got) = {first}"


def test_division_tiny_numerators():
    """The shared-reciprocal quotient on numerators below 2^-62, subnormals
    included, which it scales by 2^64 (subnormal quotients take the IEEE
    division): it equals IEEE division."""
    bad, first = _selftest(5, n=1 << 28, seed=3)
    assert bad == 0, f"{bad} division mismatches, first (a, b) = {first}"
