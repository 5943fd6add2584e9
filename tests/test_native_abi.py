"""The C-ABI library builds, loads without a GPU and exports every entry point
that include/*.h declares; the host-side argument checks reject bad input
before any launch."""
import ctypes
import re
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parent.parent


def declared_symbols():
    names = []
    for header in sorted((REPO / "include").glob("*.h")):
        text = header.read_text()
        names += re.findall(r"^\s*int\s+(swe_\w+|nn_\w+)\s*\(", text, flags=re.M)
    return names


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "swe_step_f32" in names and "swe_spatial_operator_f32" in names


def test_library_exports_every_declared_symbol():
    from diffswe2d_b200 import _native
    lib = ctypes.CDLL(str(_native.LIB_PATH))
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header():
    from diffswe2d_b200 import _native
    assert set(declared_symbols()) <= set(_native.exported_symbols())


def test_params_struct_layout_matches_header():
    from diffswe2d_b200 import _native
    # 8 doubles + 10 int32 = 104 bytes, no padding
    assert ctypes.sizeof(_native.SweParams) == 104
    assert _native.SweParams.arithmetic.offset == 96


def test_arithmetic_mode_checked():
    """An unknown arithmetic name raises; an unknown code is rejected by the
    library before any launch."""
    from diffswe2d_b200 import _native as nat
    from diffswe2d_b200.config import SWEConfig
    with pytest.raises(ValueError):
        nat.params(SWEConfig(), 1.0, 1.0, "approximate")
    assert nat.params(SWEConfig(), 1.0, 1.0, "fast").arithmetic == nat.ARITH_FAST
    p = nat.params(SWEConfig(), 1.0, 1.0)
    p.arithmetic = 7
    buf = ctypes.c_void_p(16)  # never dereferenced: the parameters are checked first
    rc = nat.lib().swe_step_f32(buf, buf, 1, buf, 1, 1, 8, 8, p, buf, 1, 1.0, None, 0, 1, buf, buf,
                                buf, None)
    assert rc == nat.SWE_EARG
    rc = nat.lib().swe_ensemble_run_f32(buf, 1, 0, 7, 1, 0, None)
    assert rc == nat.SWE_EARG
    rc = nat.lib().swe_ensemble_run_f32(buf, 1, 0, 0, 1, -1, None)
    assert rc == nat.SWE_EARG


def test_invalid_arguments_rejected_without_launch():
    """Null pointers and bad shapes return SWE_EARG before touching the GPU."""
    from diffswe2d_b200 import _native as nat
    from diffswe2d_b200.config import SWEConfig
    lib = nat.lib()
    p = nat.params(SWEConfig(), 1.0, 1.0)
    null = ctypes.c_void_p(0)
    rc = lib.swe_step_f32(null, null, 1, null, 1, 1, 8, 8, p, null, 1, 1.0, null, 0, 1, null,
                          null, null, null)
    assert rc == nat.SWE_EARG
    rc = lib.swe_spatial_operator_f32(null, null, 1, 1, 8, 8, p, null, 1, null, 0, 1, null, 0, 1,
                                      null, null, null)
    assert rc == nat.SWE_EARG


def test_cpu_tensor_fails_loudly():
    import torch
    from diffswe2d_b200 import SWE2D, SWEConfig
    from diffswe2d_b200._native import NativeLibraryError
    bed = torch.zeros(8, 8)
    m = SWE2D(bed, torch.full_like(bed, 0.02), 1.0, 1.0, config=SWEConfig(), train_dem=False)
    U = torch.zeros(1, 3, 8, 8)
    with pytest.raises(NativeLibraryError):
        m.step(U, 0.0, 1.0)
