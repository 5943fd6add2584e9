"""The friction's power h ** (1/3) (pow_pos in swe_math.cuh), compiled for
the host with g++, against the host's double pow rounded to float.

The kernels evaluate the Manning coefficient's h ** (1/3) with pow_pos, a
double-double exp(t ln x); the oracle (and the reference's CPU arithmetic it
restates) uses the C library's pow.  The same source compiled for the host
must give the same float for every input the friction sees; this test runs
it over a strided sample of all floats in [2^-40, 2^14) (every 61st
significand of every binade), for the friction's exponent and the adjoint's.
The device build is checked exhaustively against CUDA's pow by
tests/test_gpu_arith.py.
"""
import shutil
import subprocess
from pathlib import Path

import pytest

CSRC = Path(__file__).resolve().parents[1] / "diffswe2d_b200" / "csrc"

HARNESS = r"""
#include "swe_math.cuh"
#include <cstdio>
#include <cstdlib>
using namespace swe;
int main(int argc, char** argv) {
    const float t = u2f((uint32_t)strtoul(argv[1], nullptr, 16));
    unsigned long long bad = 0, n = 0;
    for (uint32_t e = 87; e < 141; ++e)
        for (uint32_t sig = 0; sig < (1u << 23); sig += 61) {
            const float x = u2f((e << 23) | sig);
            ++n;
            if (f2u(pow_pos(x, t)) != f2u((float)pow((double)x, (double)t))) {
                if (bad == 0) printf("first mismatch x=%a\n", x);
                ++bad;
            }
        }
    printf("%llu %llu\n", n, bad);
    return 0;
}
"""


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    d = tmp_path_factory.mktemp("pow")
    (d / "h.cpp").write_text(HARNESS)
    exe = d / "h"
    subprocess.run([gxx, "-std=c++17", "-O2", "-ffp-contract=off", "-I", str(CSRC), "-o", str(exe),
                    str(d / "h.cpp"), "-lm"], check=True)
    return exe


def _run(exe, t_bits):
    out = subprocess.run([str(exe), f"{t_bits:08x}"], check=True, capture_output=True, text=True).stdout
    n, bad = (int(v) for v in out.strip().splitlines()[-1].split())
    return n, bad, out


def test_power_one_third(harness):
    n, bad, out = _run(harness, 0x3EAAAAAB)  # float(1/3)
    assert n > 7_000_000
    assert bad == 0, out


def test_power_derivative_exponent(harness):
    n, bad, out = _run(harness, 0xBF2AAAAA)  # float(1/3) - 1 in float
    assert bad <= 2, out
