"""Write diffswe2d_b200/data/runup_state_8s.npz: the state of the 244x393
runup scenario (scenarios.runup(seed=0)) after 8 s of simulated time, the
initial state of the 4096x4096 throughput workload (scenarios.
throughput_workload), which tiles it.

The state is computed by the CPU oracle (pinned bit for bit to the
reference's step in tests/test_oracle.py) driving forward() exactly as the
reference does (src/solver.py:680-779, dynamic west boundary); the GPU test
tests/test_gpu_headline.py checks that SWE2D's IEEE kernels reproduce it
bit for bit.

    python tests/golden/make_workload_state.py
"""
from __future__ import annotations

import sys
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent.parent.parent
sys.path.insert(0, str(REPO))
sys.path.insert(0, str(REPO / "oracle"))

from oracle import OracleSWE  # noqa: E402

from diffswe2d_b200 import scenarios  # noqa: E402
from diffswe2d_b200.config import SWEConfig  # noqa: E402


def main():
    base = scenarios.runup(seed=0)
    seconds = scenarios.WORKLOAD_SPIN_UP_S
    om = OracleSWE(base.bed, base.roughness, base.dx, base.dy, SWEConfig(**base.config))
    om.set_dynamic_boundary(base.bc_times, base.bc_levels)
    t0 = time.perf_counter()
    U, hmax, dts = om.forward(base.U0, t_end=seconds, start_time=0.0)
    print(f"{len(dts)} steps in {time.perf_counter() - t0:.1f} s")
    out = REPO / "diffswe2d_b200" / "data" / "runup_state_8s.npz"
    np.savez_compressed(out, U=U.astype(np.float32), seconds=np.float64(seconds),
                        steps=np.int64(len(dts)))
    print("wrote", out)


if __name__ == "__main__":
    main()
