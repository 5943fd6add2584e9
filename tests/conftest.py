"""Shared fixtures and markers.

``gpu`` marks tests that need a CUDA device (they run the sm_100a kernels).
Everything else runs on the CPU: the oracle against the reference's golden
outputs, the host-side logic, and the C ABI's exported symbols.
"""
import sys
from pathlib import Path

import numpy as np
import pytest

REPO = Path(__file__).resolve().parent.parent
GOLDEN = REPO / "tests" / "golden"
sys.path.insert(0, str(REPO))
sys.path.insert(0, str(REPO / "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs the sm_100a kernels)")
    config.addinivalue_line("markers", "slow: long-running CPU test")


def pytest_collection_modifyitems(config, items):
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:  # pragma: no cover
        has_gpu = False
    if has_gpu:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session")
def golden():
    """Lazy loader of the golden .npz fixtures."""
    cache = {}

    def load(name):
        if name not in cache:
            cache[name] = dict(np.load(GOLDEN / f"{name}.npz"))
        return cache[name]

    return load


def normwise(a, b):
    """max|a-b| / max|b| in float64 (the parity metric used throughout)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = np.abs(b).max()
    diff = np.abs(a - b).max()
    return float(diff / scale) if scale > 0 else float(diff)


def field_errors(a, b):
    """Normwise relative error of h, hu, hv for [B,3,ny,nx] states."""
    return [normwise(np.asarray(a)[:, c], np.asarray(b)[:, c]) for c in range(3)]


def wet_mask(U, dry=1e-6):
    return np.asarray(U)[:, 0] > np.float32(dry)


BC_CASES = {
    "all_transmissive": ("transmissive",) * 4,
    "all_periodic": ("periodic",) * 4,
    "all_constant": ("constant",) * 4,
    "all_water_level": ("water_level",) * 4,
    "all_wall": ("wall",) * 4,
    "all_absorbing": ("absorbing",) * 4,
    "mixed_a": ("water_level", "wall", "periodic", "absorbing"),
    "mixed_b": ("constant", "transmissive", "wall", "water_level"),
    "mixed_c": ("periodic", "periodic", "wall", "wall"),
}


def bc_kwargs(case):
    l, r, t, b = BC_CASES[case]
    return dict(boundary_left=l, boundary_right=r, boundary_top=t, boundary_bottom=b)
