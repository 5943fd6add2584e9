// swe_common.cuh -- host/device plumbing shared by the step kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/swe_b200.h"
#include "swe_math.cuh"

namespace swe {

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
    k.wall_pad0 = k.wall_pad1 = 0.0f;
    return k;
}

inline bool valid_bc(int c) { return c >= SWE_BC_TRANSMISSIVE && c <= SWE_BC_ABSORBING; }

inline bool valid_params(const swe_params* p) {
    if (!p) return false;
    if (!(p->gravity > 0.0) || !(p->epsilon > 0.0) || !(p->dry_depth >= 0.0)) return false;
    if (!(p->dx > 0.0) || !(p->dy > 0.0)) return false;
    return valid_bc(p->bc_left) && valid_bc(p->bc_right) && valid_bc(p->bc_top) &&
           valid_bc(p->bc_bottom) && (p->friction_model == 0 || p->friction_model == 1);
}

}  // namespace swe
