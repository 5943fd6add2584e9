"""ctypes binding of libswe_b200.so, the sm_100a kernels behind the C ABI
declared in ``include/swe_b200.h``.

There is no fallback: if the library is missing, or a tensor is not a
contiguous float32 CUDA tensor, the call raises.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import torch

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libswe_b200.so"

SWE_OK, SWE_EARG, SWE_ECUDA = 0, 1, 2
#: swe_params.arithmetic: IEEE operation-for-operation kernels, or the
#: tolerance-mode kernels
ARITH_EXACT, ARITH_FAST = 0, 1
ARITHMETIC = {"exact": ARITH_EXACT, "fast": ARITH_FAST}
S_NONFINITE_STATE, S_NONFINITE_DT, S_NONPOSITIVE_DT, S_STEP_LIMIT = 1, 2, 4, 8
RED_WORDS = 8
FORCING_NONE, FORCING_SCALAR, FORCING_FIELD = 0, 1, 2
NN_GEMM_WAIT_NS = 1_000_000_000  # nn_gemm_bf16's normal wait limit (include/nn_b200.h)

BC_CODES = {
    "transmissive": 0,
    "periodic": 1,
    "constant": 2,
    "water_level": 3,
    "wall": 4,
    "absorbing": 5,
}


class NativeLibraryError(RuntimeError):
    """The CUDA library is missing or a call into it failed."""


class SweParams(ctypes.Structure):
    _fields_ = [
        ("gravity", ctypes.c_double),
        ("dry_depth", ctypes.c_double),
        ("epsilon", ctypes.c_double),
        ("cfl", ctypes.c_double),
        ("theta", ctypes.c_double),
        ("dx", ctypes.c_double),
        ("dy", ctypes.c_double),
        ("constant_value", ctypes.c_double),
        ("bc_left", ctypes.c_int32),
        ("bc_right", ctypes.c_int32),
        ("bc_top", ctypes.c_int32),
        ("bc_bottom", ctypes.c_int32),
        ("water_slope_reset", ctypes.c_int32),
        ("positivity_limiter", ctypes.c_int32),
        ("apply_friction", ctypes.c_int32),
        ("friction_model", ctypes.c_int32),
        ("arithmetic", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
    ]


class SweClock(ctypes.Structure):
    """swe_clock of include/swe_b200.h (72 bytes)."""
    _fields_ = [
        ("duration", ctypes.c_double),
        ("start", ctypes.c_double),
        ("tolerance", ctypes.c_double),
        ("max_dt_cap", ctypes.c_double),
        ("elapsed", ctypes.c_double),
        ("max_steps", ctypes.c_int32),
        ("steps", ctypes.c_int32),
        ("active", ctypes.c_int32),
        ("state", ctypes.c_int32),
        ("dt_status", ctypes.c_uint32),
        ("max_dt", ctypes.c_float),
        ("level", ctypes.c_float),
        ("last_dt", ctypes.c_float),
    ]


CLOCK_RUNNING, CLOCK_DONE, CLOCK_MAXSTEPS, CLOCK_FAILED, CLOCK_RECORD_FULL = 0, 1, 2, 3, 4


class SweRunClock(ctypes.Structure):
    """swe_run_clock of include/swe_b200.h (104 bytes)."""
    _fields_ = [
        ("base", SweClock),
        ("out_dt", ctypes.c_double),
        ("n_out", ctypes.c_int32),
        ("chunk", ctypes.c_int32),
        ("chunk_steps", ctypes.c_int32),
        ("record_cap", ctypes.c_int32),
        ("replay", ctypes.c_int32),
        ("replay_end", ctypes.c_int32),
    ]


class SweEnsembleMember(ctypes.Structure):
    """swe_ensemble_member of include/swe_b200.h."""
    _fields_ = [
        ("bed", ctypes.c_void_p),
        ("n", ctypes.c_void_p),
        ("U_a", ctypes.c_void_p),
        ("U_b", ctypes.c_void_p),
        ("k1", ctypes.c_void_p),
        ("hmax", ctypes.c_void_p),
        ("series_t", ctypes.c_void_p),
        ("series_w", ctypes.c_void_p),
        ("nseries", ctypes.c_int32),
        ("ny", ctypes.c_int32),
        ("nx", ctypes.c_int32),
        ("steps", ctypes.c_int32),
        ("rows", ctypes.c_int32),
        ("level", ctypes.c_float),
        ("start_time", ctypes.c_double),
        ("max_dt", ctypes.c_double),
        ("params", SweParams),
        ("out_dt", ctypes.c_double),
        ("n_out", ctypes.c_int32),
        ("ngauge", ctypes.c_int32),
        ("out_levels", ctypes.c_void_p),
        ("gauge_cells", ctypes.c_void_p),
        ("gauge_out", ctypes.c_void_p),
    ]


class SweEnsembleResult(ctypes.Structure):
    """swe_ensemble_result of include/swe_b200.h (24 bytes)."""
    _fields_ = [
        ("steps", ctypes.c_int32),
        ("finished", ctypes.c_int32),
        ("status", ctypes.c_uint32),
        ("dt_last", ctypes.c_float),
        ("time", ctypes.c_double),
    ]

_P = ctypes.c_void_p
_I = ctypes.c_int
_F = ctypes.c_float

# name -> argtypes, in the order of include/swe_b200.h
_SIGNATURES = {
    "swe_spatial_operator_f32": [_P, _P, _I, _I, _I, _I, ctypes.POINTER(SweParams), _P, _I,
                                 _P, _I, _I, _P, _I, _I, _P, _P, _P],
    "swe_step_f32": [_P, _P, _I, _P, _I, _I, _I, _I, ctypes.POINTER(SweParams), _P, _I, _F,
                     _P, _I, _I, _P, _P, _P, _P],
    "swe_step_stage_f32": [_I, _P, _P, _I, _P, _I, _I, _I, _I, ctypes.POINTER(SweParams), _P, _I,
                           _F, _P, _I, _I, _P, _P, _P, _P],
    "swe_step_stage_forced_f32": [_I, _P, _P, _I, _P, _I, _I, _I, _I, ctypes.POINTER(SweParams), _P,
                                  _I, _F, _P, _I, _I, _P, _I, _I, _P, _P, _P, _P],
    "swe_clock_f32": [_P, _P, _P, _P, _I, _P, _P, _I, _I, _P, _I, _P, _I, _P],
    "swe_run_clock_f32": [_P, _P, _P, _I, _P, _P, _P, _I, _I, _I, _I, _P, _I, _P, _P, _P, _P],
    "swe_gauge_adjoint_f32": [_P, _I, _I, _I, _P, _I, _P, _I, _I, _P],
    "swe_step_clocked_f32": [_I, _P, _P, _I, _P, _I, _I, _I, _I, ctypes.POINTER(SweParams), _P, _I,
                             _P, _P, _I, _I, _P, _P, _P, _P, _P],
    "swe_step_clocked_k2_f32": [_I, _P, _P, _I, _P, _I, _I, _I, _I, ctypes.POINTER(SweParams), _P,
                                _I, _P, _P, _I, _I, _P, _P, _P, _P, _P, _P],
    "swe_adj_spatial_f32": [_P, _P, _I, _I, _I, _I, ctypes.POINTER(SweParams), _P, _I, _P, _P, _P,
                            _P, _P, _I, _P],
    "swe_adj_spatial_bed_f32": [_P, _P, _I, _I, _I, _I, ctypes.POINTER(SweParams), _P, _I, _P, _P,
                                _P, _P, _P, _I, _P, _P],
    "swe_adj_stage2_f32": [_P, _P, _P, _P, _I, _I, _I, _I, ctypes.POINTER(SweParams), _P, _I, _P,
                           _P, _P, _F, _P, _P, _P, _P, _I, _P, _P],
    "swe_adj_pointwise_f32": [_I, _P, _P, _P, _I, _I, _I, _I, ctypes.POINTER(SweParams), _F, _P,
                              _P, _P, _P, _P, _P],
    "swe_adj_pointwise_dev_f32": [_I, _P, _P, _P, _I, _I, _I, _I, ctypes.POINTER(SweParams), _P,
                                  _P, _P, _P, _P, _P, _P],
    "swe_gauge_adjoint_prep_f32": [_P, _P, _P, _P, _I, _P, _P, _P, _I, _I, _I, _P, _I, _P, _I, _I,
                                   _P],
    "swe_gauge_adjoint_post_f32": [_P, _P, _P, _I, _I, _I, _I, _P, _I, _P],
    "swe_step_noalloc_f32": [_P, _P, _I, _P, _I, _I, _I, _I, ctypes.POINTER(SweParams), _P, _I,
                             _F, _P, _I, _I, _P, _P, _P],
    "swe_ghost_cells_f32": [_P, _P, _I, _I, _I, _I, _I, ctypes.POINTER(SweParams), _P, _I, _P, _I,
                            _P, _P, _P],
    "swe_reconstruction_f32": [_P, _P, _I, _I, _I, _I, _I, ctypes.POINTER(SweParams), _P, _P, _P,
                               _P, _P],
    "swe_hll_flux_f32": [_P, _P, _I, _I, _I, _I, ctypes.POINTER(SweParams), _P, _P, _P],
    "swe_primitive_f32": [_P, _I, _I, _I, ctypes.POINTER(SweParams), _P, _P, _P, _P, _P],
    "swe_limited_increment_f32": [_P, _I, _I, _I, _I, ctypes.c_double, _P, _P],
    "swe_minmod3_f32": [_P, _P, _P, ctypes.c_longlong, _P, _P],
    "swe_clean_and_limit_f32": [_P, _P, _I, _I, _I, ctypes.POINTER(SweParams), _P, _P],
    "swe_friction_f32": [_P, _P, _I, _I, _I, _I, _F, _I, ctypes.POINTER(SweParams), _P, _P],
    "swe_selftest_arith_f32": [_I, ctypes.c_longlong, ctypes.c_ulonglong, _P, _P, _P],
    "swe_ensemble_prepare_f32": [ctypes.POINTER(SweEnsembleMember), _I, _P, _P],
    "swe_ensemble_reset_f32": [_P, _I, _P],
    "swe_ensemble_run_f32": [_P, _I, _I, _I, _I, ctypes.c_longlong, _P],
    "swe_ensemble_results_f32": [_P, _I, _P, _P, _P],
    "swe_tune_sweep_rows": [_I],
    "swe_sweep_rows": [],
    "swe_load_kernels": [],
    # include/nn_b200.h
    "nn_gemm_bf16": [_P, _I, _P, _I, _I, _I, _I, _P, _I, _P, _P, _P, _I, _I, _P, ctypes.c_longlong,
                     _P, _P],
    "nn_im2col": [_P, _P, _I, _I, _I, _I, _I, _I, _I, _I, _I, _I, _F, _F, _P, _I, _P],
    "nn_col2im": [_P, _I, _I, _I, _I, _I, _I, _I, _I, _P, _P],
    "nn_act_backward": [_P, _P, _I, _I, _I, _I, _P, _I, _P, _I, _P, _P],
    "nn_colsum": [_P, _I, _I, _I, _P, _P],
    "nn_transpose_bf16": [_P, _I, _I, _I, _P, _I, _P],
    "nn_cast_bf16": [_P, _I, _I, _I, _P, _I, _P, _I, _P],
    "nn_mse": [_P, _P, _I, _I, _P, _P, _P],
    "nn_adam": [_P, _P, _P, _P, ctypes.c_longlong, _F, _F, _F, _F, _I, _P],
}

_lib = None


def lib() -> ctypes.CDLL:
    """Load the library once; raise NativeLibraryError if it is absent."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise NativeLibraryError(
                f"{LIB_PATH} is missing; build it with `make -C diffswe2d_b200/csrc` "
                "(or __graft_entry__.build())")
        handle = ctypes.CDLL(str(LIB_PATH))
        for name, args in _SIGNATURES.items():
            fn = getattr(handle, name)
            fn.argtypes = args
            fn.restype = ctypes.c_int
        handle.swe_ensemble_workspace_bytes.argtypes = [_I]
        handle.swe_ensemble_workspace_bytes.restype = ctypes.c_longlong
        _lib = handle
    return _lib


_kernels_loaded = False


def load_kernels() -> None:
    """Load the kernels' modules once (before the first CUDA-graph capture)."""
    global _kernels_loaded
    if not _kernels_loaded:
        check(lib().swe_load_kernels(), "loading kernels")
        _kernels_loaded = True


def exported_symbols():
    return list(_SIGNATURES)


def arithmetic_code(arithmetic: str) -> int:
    if arithmetic not in ARITHMETIC:
        raise ValueError(f"arithmetic must be one of {sorted(ARITHMETIC)}, got {arithmetic!r}")
    return ARITHMETIC[arithmetic]


def params(cfg, dx: float, dy: float, arithmetic: str = "exact") -> SweParams:
    for side in ("left", "right", "top", "bottom"):
        name = getattr(cfg, f"boundary_{side}")
        if name not in BC_CODES:
            raise ValueError(f"Unsupported {side} boundary type {name!r}. "
                             f"Valid types are {sorted(BC_CODES)}.")
    # As in src/solver.py:654-661, every friction model name other than
    # "manning" selects the roughness-length law.
    return SweParams(
        float(cfg.gravity), float(cfg.dry_depth), float(cfg.epsilon), float(cfg.cfl),
        float(cfg.limiter_theta), float(dx), float(dy), float(cfg.constant_value),
        BC_CODES[cfg.boundary_left], BC_CODES[cfg.boundary_right],
        BC_CODES[cfg.boundary_top], BC_CODES[cfg.boundary_bottom],
        int(bool(cfg.water_slope_reset)), int(bool(cfg.positivity_limiter)),
        int(bool(cfg.apply_friction)), 0 if cfg.frictionmodel == "manning" else 1,
        arithmetic_code(arithmetic), 0,
    )


def require_cuda_f32(name: str, t: torch.Tensor) -> torch.Tensor:
    if not torch.is_tensor(t):
        raise TypeError(f"{name} must be a tensor")
    if not t.is_cuda:
        raise NativeLibraryError(
            f"{name} is on {t.device}; the B200 kernels only run on CUDA tensors")
    if t.dtype != torch.float32:
        raise TypeError(f"{name} must be float32 for the FP32 kernels, got {t.dtype}")
    return t.contiguous()


def stream_handle(device: torch.device) -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def ptr(t) -> ctypes.c_void_p:
    return ctypes.c_void_p(0 if t is None else t.data_ptr())


def check(rc: int, what: str) -> None:
    if rc == SWE_OK:
        return
    if rc == SWE_EARG:
        raise ValueError(f"{what}: invalid argument rejected by the CUDA library")
    raise NativeLibraryError(f"{what}: CUDA error (code {rc})")


def params_basic(gravity=9.81, epsilon=1e-12, dry_depth=1e-6, theta=1.3,
                 water_slope_reset=True, positivity_limiter=True, bcs=None,
                 constant_value=0.0) -> SweParams:
    """Parameters for the operator-level entry points (no grid spacing)."""
    l, r, t, b = bcs if bcs is not None else ("transmissive",) * 4
    return SweParams(float(gravity), float(dry_depth), float(epsilon), 0.5, float(theta), 1.0, 1.0,
                     float(constant_value), BC_CODES[l], BC_CODES[r], BC_CODES[t], BC_CODES[b],
                     int(bool(water_slope_reset)), int(bool(positivity_limiter)), 1, 0, ARITH_EXACT, 0)
