// swe_common.cuh -- host/device plumbing shared by the step kernels.
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "../../include/swe_b200.h"
#include "swe_math.cuh"

namespace swe {

// RN(1/b) for a finite float b != 0, exactly: the candidate from double
// division and its two float neighbours are compared by the exact residual
// |1 - b y| (a product of two floats is exact in double).
inline float host_rcp_cr(float b) {
    float y = (float)(1.0 / (double)b);
    float best = y;
    double best_err = fabs(1.0 - (double)b * (double)y);
    for (int d = -1; d <= 1; d += 2) {
        float c = nextafterf(y, d < 0 ? -INFINITY : INFINITY);
        double err = fabs(1.0 - (double)b * (double)c);
        if (err < best_err) {
            best = c;
            best_err = err;
        }
    }
    return best;
}

// Derives the float32 constants of swe_params as the reference rounds its
// Python scalars (see SweConsts).
inline SweConsts make_consts(const swe_params& p) {
    SweConsts k;
    double pf = 1.0e-6;  // float32 precision floor, riemann.py:6-11
    double fh = p.epsilon > p.dry_depth ? p.epsilon : p.dry_depth;
    fh = fh > pf ? fh : pf;
    double fe = p.epsilon > pf ? p.epsilon : pf;
    if (fe < 0.0) fe = 0.0;
    k.g = (float)p.gravity;
    k.half_g = (float)(0.5 * p.gravity);
    k.dry = (float)p.dry_depth;
    k.floor_h = (float)fh;
    k.den_floor = (float)fe;
    k.theta = (float)p.theta;
    k.eps = (float)p.epsilon;
    k.cfl = (float)p.cfl;
    k.dx = (float)p.dx;
    k.dy = (float)p.dy;
    k.fr_vs = (float)fh;
    k.fr_e = (float)fe;
    k.fr_e2 = (float)(fe * fe);
    k.third = (float)(1.0 / 3.0);
    k.absorb_lim = 1e-4f;
    k.absorb_min = 1e-6f;
    k.g981 = 9.81f;
    k.rdx = host_rcp_cr(k.dx);
    k.rdy = host_rcp_cr(k.dy);
    return k;
}

inline bool valid_bc(int c) { return c >= SWE_BC_TRANSMISSIVE && c <= SWE_BC_ABSORBING; }

inline bool valid_params(const swe_params* p) {
    if (!p) return false;
    if (!(p->gravity > 0.0) || !(p->epsilon > 0.0) || !(p->dry_depth >= 0.0)) return false;
    if (!(p->dx > 0.0) || !(p->dy > 0.0)) return false;
    return valid_bc(p->bc_left) && valid_bc(p->bc_right) && valid_bc(p->bc_top) &&
           valid_bc(p->bc_bottom) && (p->friction_model == 0 || p->friction_model == 1) &&
           (p->arithmetic == SWE_ARITH_EXACT || p->arithmetic == SWE_ARITH_FAST);
}

// Chained launches (programmatic dependent launch, sm_90 and later).  The
// kernels of a time step and of its adjoint form a chain in which each one
// reads what the one before it wrote.  They are launched with
// launch_chained(), which lets the launch of the next kernel of the stream
// overlap the end of the current one, and each calls chain_start() before
// its first memory access: it waits until the preceding kernel has
// completed and its writes are visible (at once for a kernel launched the
// ordinary way).  The kernels do not signal their dependents early: blocks
// of the next kernel waiting beside the running ones slowed the forward
// loop at the inversion's grid size (44.7 against 39.7 us per step).
__device__ __forceinline__ void chain_start() {
#if defined(__CUDA_ARCH__)
    asm volatile("griddepcontrol.wait;" ::: "memory");
#endif
}

template <typename... K, typename... A>
inline cudaError_t launch_chained(void (*kernel)(K...), dim3 grid, dim3 block, cudaStream_t s,
                                  A&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, static_cast<K>(args)...);
}

}  // namespace swe
