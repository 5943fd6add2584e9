// swe_sweep.cuh -- launch arguments and padded-cell access shared by the
// step kernels of both arithmetic modes (swe_step.cu: IEEE, operation for
// operation as the reference; swe_fast.cu: tolerance mode).
//
// The row-sweep kernels give each warp a strip of 32 columns (SW_OUT output
// columns plus a two-cell halo either side) and a number of output rows; a
// block holds SW_WARPS strips side by side.  Cells outside the interior are
// the ghost cells of add_ghost_cells (src/boundary.py:150-413), evaluated on
// the fly by sweep_cell.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "swe_common.cuh"

namespace swe {

constexpr int SW_OUT = 28;    // output columns per warp
constexpr int SW_ROWS = 64;   // default output rows per warp
constexpr int SW_WARPS = 4;   // warps per block (side by side in x)

// Arguments of one stage launch (one step = stage 1 + stage 2).
struct StepArgs {
    const float* U;
    const float* bed;
    const float* n;
    const float* level;
    const float* rain;
    const float* infil;
    float* tend;   // stage 1: k1 output; stage 2: k1 input
    float* U_out;  // stage 2 output
    uint32_t* red;
    const swe_clock* clk;  // device clock of forward(), or null for a plain step
    float* hmax;           // running max depth [B,ny,nx], or null
    float* k2_out;         // stage 2: its tendency k2 [B,3,ny,nx], or null
    int rows;              // output rows per sweep tile
    float max_dt, cval;
    int B, bedB, nB, levelB, ny, nx;
    int rain_mode, rain_batch, infil_mode, infil_batch;
    int bc[4];
    int wsr, positivity, friction, friction_model;
    SweConsts kc;
};

namespace {

__device__ __forceinline__ size_t at3(int b, int c, int j, int i, int ny, int nx) {
    return (((size_t)b * 3 + c) * ny + j) * nx + i;
}
__device__ __forceinline__ size_t at1(int b, int j, int i, int ny, int nx) {
    return ((size_t)b * ny + j) * nx + i;
}

__device__ __forceinline__ float forcing(const float* f, int mode, int fb, int b, int j, int i,
                                         int ny, int nx) {
    if (mode == SWE_FORCING_SCALAR) return f[0];
    if (mode == SWE_FORCING_FIELD) return f[at1(fb == 1 ? 0 : b, j, i, ny, nx)];
    return 0.0f;
}

__device__ __forceinline__ float bed_at(const StepArgs& a, int b, int j, int i) {
    return a.bed[at1(a.bedB == 1 ? 0 : b, j, i, a.ny, a.nx)];
}

// Loads of the state and the tendency.  CG = true bypasses L1 (ld.global.cg):
// needed when another block of the same launch wrote the data (the
// persistent ensemble kernel), since L1 is not coherent across blocks.
template <bool CG>
__device__ __forceinline__ float ld_state(const float* p) {
    return CG ? __ldcg(p) : *p;
}

// The predictor of stage 2, clean(U, U + dt/2 k1) (solver.py:639), in the
// arithmetic of the including file: P::predict(u, k1, dt/2, consts,
// positivity) with k1 given as three floats.

// The second source cell of a wall ghost two cells out (rare: domain edge
// only), kept out of line to keep the sweep kernels' code small.
template <int STAGE, bool CG, class P>
__device__ __noinline__ State mirror_state(const float* __restrict__ U, const float* __restrict__ tend,
                                           int ny, int nx, int b, int j, int i, float hdt, float eps,
                                           float dry, int positivity) {
    const size_t plane = (size_t)ny * nx;
    const size_t o = at3(b, 0, j, i, ny, nx);
    const State u{ld_state<CG>(U + o), ld_state<CG>(U + o + plane), ld_state<CG>(U + o + 2 * plane)};
    if (STAGE == 1) return u;
    SweConsts k{};
    k.eps = eps;
    k.dry = dry;
    return P::predict(u, ld_state<CG>(tend + o), ld_state<CG>(tend + o + plane),
                      ld_state<CG>(tend + o + 2 * plane), hdt, k, positivity);
}

// Cell (j, i) of the padded state for the sweep (interior coordinates,
// -2 <= j < ny+2, -2 <= i < nx+2), with the ghost rules of add_ghost_cells.
// Only the four "arms" of the padding are ever used by the stencil (corner
// ghosts feed no face of an interior row or column), so a cell outside the
// interior in both directions, or beyond the two-cell padding, gets its
// clamped neighbour's value and is never read.  Also returns the raw U of
// the source cell.
template <int STAGE, bool CG, class P>
__device__ __forceinline__ void sweep_cell(const StepArgs& a, int b, int j, int i, float hdt,
                                           State& s, float& z, State& uraw) {
    const int ny = a.ny, nx = a.nx;
    const bool jin = (unsigned)j < (unsigned)ny, iin = (unsigned)i < (unsigned)nx;
    int js = min(max(j, 0), ny - 1), is = min(max(i, 0), nx - 1);
    const bool xarm = jin && !iin && i >= -2 && i < nx + 2;
    const bool yarm = iin && !jin && j >= -2 && j < ny + 2;
    int code = -1, side = 0;
    if (xarm || yarm) {
        side = xarm ? (i < 0 ? 0 : 1) : (j < 0 ? 2 : 3);
        code = a.bc[side];
        if (code == SWE_BC_PERIODIC) {  // boundary.py:247-257, :301-302
            if (xarm) is = i < 0 ? nx + i : i - nx;
            else js = j < 0 ? ny + j : j - ny;
        }
    }
    const size_t plane = (size_t)ny * nx;
    const size_t o = at3(b, 0, js, is, ny, nx);
    uraw = State{ld_state<CG>(a.U + o), ld_state<CG>(a.U + o + plane), ld_state<CG>(a.U + o + 2 * plane)};
    if (STAGE == 1) {
        s = uraw;
    } else {  // predictor clean(U, U + dt/2 k1), solver.py:639
        s = P::predict(uraw, ld_state<CG>(a.tend + o), ld_state<CG>(a.tend + o + plane),
                       ld_state<CG>(a.tend + o + 2 * plane), hdt, a.kc, a.positivity);
    }
    z = bed_at(a, b, js, is);
    if (code < 0 || code == SWE_BC_TRANSMISSIVE || code == SWE_BC_PERIODIC) return;
    const float lev = ld_state<CG>(a.level + (a.levelB == 1 ? 0 : b));
    if (code == SWE_BC_CONSTANT) {  // boundary.py:304-305
        s = State{a.cval, a.cval, a.cval};
    } else if (code == SWE_BC_WATER_LEVEL) {  // boundary.py:279-282, :307-310
        s.h = fmaxf(lev - z, 0.0f);
    } else if (code == SWE_BC_WALL) {  // boundary.py:312-316: flip of the first/last two lines
        const int jm = xarm ? j : (j < 0 ? -1 - j : 2 * ny - 1 - j);
        const int im = xarm ? (i < 0 ? -1 - i : 2 * nx - 1 - i) : i;
        float mirror;
        if (jm == js && im == is) {
            mirror = xarm ? s.hu : s.hv;
        } else {
            const State m = mirror_state<STAGE, CG, P>(a.U, a.tend, ny, nx, b, jm, im, hdt, a.kc.eps,
                                                       a.kc.dry, a.positivity);
            mirror = xarm ? m.hu : m.hv;
        }
        if (xarm) s.hu = -mirror;
        else s.hv = -mirror;
    } else if (code == SWE_BC_ABSORBING) {  // boundary.py:318-328
        const float hr = fmaxf(lev - z, 0.0f);
        const float hg = s.h;
        const float hc = hr > a.kc.absorb_lim ? hr : hg;
        const float c = sqrtf(a.kc.g981 * fmaxf(hc, a.kc.absorb_min));
        const float val = ((side == 0 || side == 2) ? -c : c) * (hg - hr);
        if (xarm) s.hu = val;
        else s.hv = val;
    }
}

__device__ __forceinline__ float shfl_up1(float v) { return __shfl_up_sync(0xffffffffu, v, 1); }
__device__ __forceinline__ float shfl_dn1(float v) { return __shfl_down_sync(0xffffffffu, v, 1); }
__device__ __forceinline__ uint32_t warp_max_u32(uint32_t v) { return __reduce_max_sync(0xffffffffu, v); }

// Stable time step of stage 2 from the stage-1 maxima (solver.py:620-632;
// torch.minimum propagates a NaN stable dt); the first thread of the grid
// records dt and its status bits.
template <bool CG>
__device__ __forceinline__ float stage2_dt(const StepArgs& a, bool first) {
    const uint32_t ax = CG ? __ldcg(a.red) : a.red[0];
    const uint32_t ay = CG ? __ldcg(a.red + 1) : a.red[1];
    const float st = stable_dt(u2f(ax), u2f(ay), a.kc);
    const float max_dt = a.clk != nullptr ? a.clk->max_dt : a.max_dt;
    const float dt = st != st ? st : fminf(st, max_dt);
    if (first) {
        uint32_t st_bits = 0;
        if (!isfinite(dt)) st_bits |= SWE_S_NONFINITE_DT;
        else if (!(dt > 0.0f)) st_bits |= SWE_S_NONPOSITIVE_DT;
        if (st_bits) atomicOr(&a.red[2], st_bits);
        a.red[3] = f2u(dt);
    }
    return dt;
}

}  // namespace

// Kernels of the tolerance mode (swe_fast.cu): enqueue stage 1 and/or 2
// (stage bit 1 / bit 2) of a step whose reduction words are already cleared.
int fast_launch_stages(int stage, const StepArgs& a, dim3 grid, cudaStream_t s);
// Touch every tolerance-mode kernel (module load before stream capture).
int fast_load_kernels();

}  // namespace swe
