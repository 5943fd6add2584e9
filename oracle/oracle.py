"""CPU oracle for DiffSWE2d's explicit finite-volume step.

TEST INFRASTRUCTURE ONLY.  This module is the checker: only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` import
it.  The product package ``diffswe2d_b200`` never imports, links or calls it.

It wraps ``libswe_oracle.so`` (``swe_oracle.c``), a plain-C restatement of
the reference's numerical operators in float32 and float64, with numpy
arrays in and out.  ``OracleSWE`` restates the host-side logic of the
reference's ``SWE2D`` (``src/solver.py``): the step's dt handling, the
duration loop of ``forward`` and the dynamic boundary interpolation.

Parity of this oracle with the reference is pinned in
``tests/test_oracle.py`` against golden outputs of the reference itself
(``tests/golden/``, made by ``tests/golden/make_golden.py``).
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_LIB_PATH = _HERE / "_build" / "libswe_oracle.so"

BC_CODES = {
    "transmissive": 0,
    "periodic": 1,
    "constant": 2,
    "water_level": 3,
    "wall": 4,
    "absorbing": 5,
}


class _Params(ctypes.Structure):
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
    ]


def build() -> Path:
    """Compile the oracle library with its Makefile (gcc, no FMA contraction)."""
    subprocess.run(["make", "-s", "-C", str(_HERE)], check=True)
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not _LIB_PATH.exists():
            build()
        _lib = ctypes.CDLL(str(_LIB_PATH))
    return _lib


def num_threads() -> int:
    return int(lib().orc_num_threads())


def make_params(cfg, dx: float, dy: float) -> _Params:
    """Pack an SWEConfig-like object (attribute names of src/config.py)."""
    return _Params(
        float(cfg.gravity), float(cfg.dry_depth), float(cfg.epsilon), float(cfg.cfl),
        float(cfg.limiter_theta), float(dx), float(dy), float(cfg.constant_value),
        BC_CODES[cfg.boundary_left], BC_CODES[cfg.boundary_right],
        BC_CODES[cfg.boundary_top], BC_CODES[cfg.boundary_bottom],
        int(bool(cfg.water_slope_reset)), int(bool(cfg.positivity_limiter)),
        int(bool(cfg.apply_friction)), 0 if cfg.frictionmodel == "manning" else 1,
    )


def _sfx(dtype) -> str:
    return "f32" if np.dtype(dtype) == np.float32 else "f64"


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def _arr(a, dtype) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=dtype))


def _batch_values(value, B: int, dtype) -> np.ndarray:
    v = np.asarray(value, dtype=np.float64).reshape(-1)
    if v.size == 1:
        v = np.repeat(v, B)
    if v.size != B:
        raise ValueError(f"need 1 or {B} boundary values, got {v.size}")
    return _arr(v, dtype)


def _f(dtype, x):
    """A Python float rounded to the working precision."""
    return np.dtype(dtype).type(x)


class Oracle:
    """Array-level restatements of the reference's operators."""

    def __init__(self, dtype=np.float32):
        self.dtype = np.dtype(dtype)
        self.sfx = _sfx(dtype)
        self.L = lib()

    def _fn(self, name):
        return getattr(self.L, f"orc_{name}_{self.sfx}")

    def _scalar(self, x):
        return (ctypes.c_float if self.sfx == "f32" else ctypes.c_double)(float(x))

    # src/boundary.py:150
    def ghost_cells(self, U, bed, ng, cfg, level=0.0, cval=0.0):
        U, bed = _arr(U, self.dtype), _arr(bed, self.dtype)
        B, _, ny, nx = U.shape
        bedB = bed.shape[0]
        Up = np.empty((B, 3, ny + 2 * ng, nx + 2 * ng), self.dtype)
        zp = np.empty((bedB, 1, ny + 2 * ng, nx + 2 * ng), self.dtype)
        p = make_params(cfg, 1.0, 1.0)
        lv, cv = _batch_values(level, B, self.dtype), _batch_values(cval, B, self.dtype)
        self._fn("ghost_cells")(_ptr(U), _ptr(bed), B, bedB, ny, nx, ng, ctypes.byref(p),
                                _ptr(lv), _ptr(cv), _ptr(Up), _ptr(zp))
        return Up, zp

    # src/reconstruction.py:18
    def reconstruction(self, Up, zp, dim, cfg):
        Up, zp = _arr(Up, self.dtype), _arr(zp, self.dtype)
        B, _, H, W = Up.shape
        UL, UR = np.empty_like(Up), np.empty_like(Up)
        sL, sR = np.empty((B, 1, H, W), self.dtype), np.empty((B, 1, H, W), self.dtype)
        p = make_params(cfg, 1.0, 1.0)
        rc = self._fn("reconstruction")(_ptr(Up), _ptr(zp), B, zp.shape[0], H, W, int(dim),
                                        ctypes.byref(p), _ptr(UL), _ptr(UR), _ptr(sL), _ptr(sR))
        if rc:
            raise MemoryError("oracle reconstruction failed")
        return UL, UR, sL, sR

    # src/riemann.py:41
    def hll_flux(self, UL, UR, normal, cfg):
        UL, UR = _arr(UL, self.dtype), _arr(UR, self.dtype)
        B, _, H, W = UL.shape
        F = np.empty_like(UL)
        s = np.empty((B, 1, H, W), self.dtype)
        p = make_params(cfg, 1.0, 1.0)
        self._fn("hll_flux")(_ptr(UL), _ptr(UR), B, H, W, 1 if normal == "y" else 0,
                             ctypes.byref(p), _ptr(F), _ptr(s))
        return F, s

    # src/riemann.py:20
    def primitive(self, U, cfg):
        U = _arr(U, self.dtype)
        B, _, H, W = U.shape
        outs = [np.empty((B, 1, H, W), self.dtype) for _ in range(4)]
        p = make_params(cfg, 1.0, 1.0)
        self._fn("primitive")(_ptr(U), B, H, W, ctypes.byref(p), *[_ptr(o) for o in outs])
        return tuple(outs)

    # src/numerics.py:16
    def limited_increment(self, q, dim, theta=1.3):
        q = _arr(q, self.dtype)
        B, C, H, W = q.shape
        out = np.empty_like(q)
        self._fn("limited_increment")(_ptr(q), B, C, H, W, int(dim), ctypes.c_double(theta), _ptr(out))
        return out

    # src/solver.py:448
    def spatial_operator(self, U, bed, cfg, dx, dy, level=0.0, rain=None, infil=None):
        U, bed = _arr(U, self.dtype), _arr(bed, self.dtype)
        B, _, ny, nx = U.shape
        rhs = np.empty_like(U)
        ax, ay = self._scalar(0), self._scalar(0)
        p = make_params(cfg, dx, dy)
        lv = _batch_values(level, B, self.dtype)
        rn = None if rain is None else _arr(np.broadcast_to(rain, (B, 1, ny, nx)), self.dtype)
        inf = None if infil is None else _arr(np.broadcast_to(infil, (B, 1, ny, nx)), self.dtype)
        rc = self._fn("spatial_operator")(
            _ptr(U), _ptr(bed), B, bed.shape[0], ny, nx, ctypes.byref(p), _ptr(lv),
            None if rn is None else _ptr(rn), None if inf is None else _ptr(inf),
            _ptr(rhs), ctypes.byref(ax), ctypes.byref(ay))
        if rc:
            raise MemoryError("oracle spatial operator failed")
        return rhs, self.dtype.type(ax.value), self.dtype.type(ay.value)

    # src/solver.py:547
    def clean_and_limit(self, old, cand, cfg):
        old, cand = _arr(old, self.dtype), _arr(cand, self.dtype)
        B, _, ny, nx = old.shape
        out = np.empty_like(old)
        p = make_params(cfg, 1.0, 1.0)
        self._fn("clean_and_limit")(_ptr(old), _ptr(cand), B, ny, nx, ctypes.byref(p), _ptr(out))
        return out

    # src/friction.py:102
    def manning(self, U, n, dt, dry_depth=1e-6, epsilon=1e-12):
        U, n = _arr(U, self.dtype), _arr(n, self.dtype)
        B, _, ny, nx = U.shape
        out = np.empty_like(U)
        self._fn("manning")(_ptr(U), _ptr(n), B, n.shape[0], ny, nx, self._scalar(dt),
                            ctypes.c_double(dry_depth), ctypes.c_double(epsilon), _ptr(out))
        return out

    # src/friction.py:69
    def roughness_friction(self, U, z0, dt, dry_depth=1e-6, epsilon=1e-12):
        U, z0 = _arr(U, self.dtype), _arr(z0, self.dtype)
        B, _, ny, nx = U.shape
        out = np.empty_like(U)
        self._fn("roughness_friction")(_ptr(U), _ptr(z0), B, z0.shape[0], ny, nx, self._scalar(dt),
                                       ctypes.c_double(dry_depth), ctypes.c_double(epsilon), _ptr(out))
        return out

    # src/solver.py:572 (array part): returns (U_new, dt in working precision).
    # rain0 / rain1: rainfall rates of stage 1 / stage 2 (broadcast to [B,1,ny,nx]).
    def step(self, U, bed, n, cfg, dx, dy, level, max_dt, infil=None, rain0=None, rain1=None):
        U, bed, n = _arr(U, self.dtype), _arr(bed, self.dtype), _arr(n, self.dtype)
        B, _, ny, nx = U.shape
        out = np.empty_like(U)
        dt = self._scalar(0)
        p = make_params(cfg, dx, dy)
        lv = _batch_values(level, B, self.dtype)

        def field(a):
            return None if a is None else _arr(np.broadcast_to(a, (B, 1, ny, nx)), self.dtype)

        inf, r0, r1 = field(infil), field(rain0), field(rain1)
        rc = self._fn("step_forced")(_ptr(U), _ptr(bed), bed.shape[0], _ptr(n), n.shape[0], B, ny,
                                     nx, ctypes.byref(p), _ptr(lv),
                                     self._scalar(_f(self.dtype, max_dt)),
                                     None if r0 is None else _ptr(r0),
                                     None if r1 is None else _ptr(r1),
                                     None if inf is None else _ptr(inf), _ptr(out), ctypes.byref(dt))
        if rc == 2:
            raise FloatingPointError("The calculated timestep is non-finite.")
        if rc == 3:
            raise FloatingPointError(f"Non-positive timestep: {float(dt.value)}.")
        if rc:
            raise MemoryError("oracle step failed")
        return out, self.dtype.type(dt.value)


class OracleSWE:
    """Restatement of the host logic of SWE2D (src/solver.py) over the oracle.

    ``bed`` and ``roughness`` are [ny,nx] or [1|B,1,ny,nx] arrays; the state
    is [B,3,ny,nx].  ``dtype`` selects float32 or float64 arithmetic.
    """

    def __init__(self, bed, roughness, dx, dy, config, dtype=np.float32):
        self.dtype = np.dtype(dtype)
        bed = np.asarray(bed, dtype=self.dtype)
        roughness = np.asarray(roughness, dtype=self.dtype)
        if bed.ndim == 2:
            bed = bed[None, None]
        if roughness.ndim == 2:
            roughness = roughness[None, None]
        self.bed = np.ascontiguousarray(bed)
        self.roughness = np.ascontiguousarray(roughness)
        self.dx, self.dy = float(dx), float(dy)
        self.cfg = config
        self.o = Oracle(self.dtype)
        self.bc_times = self.bc_wls = None
        self.use_dynamic_bc = False

    def set_dynamic_boundary(self, times, water_levels):
        self.bc_times = np.asarray(times, dtype=np.float64)
        self.bc_wls = np.asarray(water_levels, dtype=np.float64)
        self.use_dynamic_bc = True

    # src/solver.py:391-415
    def interpolate_boundary(self, current_time: float):
        t = np.asarray(self.bc_times, dtype=self.dtype)
        w = np.asarray(self.bc_wls, dtype=self.dtype)
        time = self.dtype.type(current_time)
        idx = int(np.searchsorted(t, time, side="left"))
        idx = min(max(idx, 1), t.size - 1)
        t0, t1, w0, w1 = t[idx - 1], t[idx], w[idx - 1], w[idx]
        eps = self.dtype.type(np.finfo(self.dtype).eps)
        span = t1 - t0
        weight = (time - t0) / (span if span > eps else eps)
        return w0 + weight * (w1 - w0)

    def resolve_level(self, current_time, explicit=None):
        if explicit is not None:
            return explicit
        if self.use_dynamic_bc:
            return self.interpolate_boundary(current_time)
        return self.cfg.constant_level

    def spatial_operator(self, U, boundary_level=None):
        level = self.cfg.constant_level if boundary_level is None else boundary_level
        return self.o.spatial_operator(U, self.bed, self.cfg, self.dx, self.dy, level)

    # src/solver.py:572-663 -> (U_new, dt as Python float).  ``rainfall`` is a
    # callable time -> rate ([1,1,ny,nx] or scalar), evaluated at the step's
    # start (model time in the working precision) for stage 1 and half a
    # step later for stage 2 (:607-643).
    def step(self, U, model_time, max_dt, boundary_level=None, infiltration=None, rainfall=None):
        level = self.cfg.constant_level if boundary_level is None else boundary_level
        rain0 = rain1 = None
        if rainfall is not None:
            R = self.dtype.type
            t = float(R(model_time))
            rain0 = rainfall(t)
            _, ax, ay = self.o.spatial_operator(U, self.bed, self.cfg, self.dx, self.dy, level,
                                                rain0, infiltration)
            den = max(R(ax) / R(self.dx) + R(ay) / R(self.dy), R(self.cfg.epsilon))
            stable = (R(1) / den) * R(self.cfg.cfl)
            dt = stable if np.isnan(stable) else min(stable, R(max_dt))
            if np.isfinite(dt) and dt > 0:
                rain1 = rainfall(t + 0.5 * float(dt))
        out, dt = self.o.step(U, self.bed, self.roughness, self.cfg, self.dx, self.dy,
                              level, max_dt, infiltration, rain0, rain1)
        return out, float(dt)

    # src/solver.py:680-779 -> (U, hmax, list of dt)
    def forward(self, U0, t_end, start_time=0.0, max_steps=1_000_000, boundary_level=None,
                max_dt_cap=None, callback=None):
        duration, absolute_start = float(t_end), float(start_time)
        U = np.asarray(U0, dtype=self.dtype)
        hmax = U[:, 0].copy()
        if duration == 0.0:
            return U, hmax, []
        elapsed, dts = 0.0, []
        tolerance = max(1e-12, 1e-12 * abs(duration))
        for iteration in range(max_steps):
            remaining = duration - elapsed
            if remaining <= tolerance:
                return U, hmax, dts
            step_max_dt = remaining
            if max_dt_cap is not None:
                step_max_dt = min(remaining, float(max_dt_cap))
            current_time = absolute_start + elapsed
            level = self.resolve_level(current_time, boundary_level)
            U, dt = self.step(U, current_time, step_max_dt, boundary_level=level)
            hmax = np.maximum(hmax, U[:, 0])
            elapsed += dt
            if elapsed > duration and elapsed - duration <= tolerance:
                elapsed = duration
            dts.append(dt)
            if callback is not None:
                callback(iteration, absolute_start + elapsed, U)
        raise RuntimeError(f"max_steps={max_steps} reached after {elapsed:.8f} s; "
                           f"requested duration={duration:.8f} s.")


def rainfall_at(times, rates, time, dtype=np.float32):
    """Rain rate [1,1,ny,nx] at ``time`` from records ``rates`` [nt,1,ny,nx]
    at ``times`` [nt]: linear interpolation, held outside the series
    (RainfallForcing.at, src/forcing.py:24-37), in ``dtype``."""
    R = np.dtype(dtype).type
    times = np.asarray(times, dtype=dtype)
    rates = np.asarray(rates, dtype=dtype)
    nt = times.size
    if nt == 1:
        return rates[0:1]
    t = R(time)
    right = min(max(int(np.searchsorted(times, t, side="left")), 1), nt - 1)
    left = right - 1
    width = max(times[right] - times[left], R(1.0e-12))
    weight = (t - times[left]) / width
    out = (R(1.0) - weight) * rates[left] + weight * rates[right]
    if t <= times[0]:
        out = rates[0]
    if t >= times[-1]:
        out = rates[-1]
    return np.ascontiguousarray(out[None])


def isclose_report(a, b):
    """Normwise and pointwise relative differences used by the parity tests."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = np.abs(b).max()
    normwise = float(np.abs(a - b).max() / scale) if scale > 0 else float(np.abs(a - b).max())
    return normwise


if os.environ.get("SWE_ORACLE_BUILD_ON_IMPORT"):
    build()

__all__ = ["Oracle", "OracleSWE", "BC_CODES", "build", "lib", "num_threads", "isclose_report",
           "rainfall_at", "math"]
