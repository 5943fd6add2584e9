// swe_adjoint_kernels.cuh -- kernels of the step adjoint, templated on the
// arithmetic policy M of swe_adjoint.cuh and instantiated twice: with
// ExactMath in swe_adjoint.cu (IEEE flags) and with FastMath in
// swe_adjoint_fast.cu (compiled like the tolerance-mode step).
//
// The spatial-operator adjoint is two launches: adj_face_kernel, one thread
// per face (x faces, then y faces, in one grid), computes the face's reverse
// mode (swe_adjoint.cuh) and writes its contributions to its four stencil
// cells into face-record planes; adj_gather_kernel, one thread per cell,
// sums them in a fixed order and folds the adjoints of ghost cells back into
// the interior cells and boundary level they were made from (the adjoint of
// add_ghost_cells, src/boundary.py:150-413), and, for stage 2, goes on
// through the predictor's adjoint.  No float atomics: results are
// deterministic.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "swe_adjoint.cuh"
#include "swe_common.cuh"

namespace swe {

constexpr int ADJ_THREADS = 256;
// Blocks per SM the kernels are compiled for (register budgets): the face
// kernel at three (80 registers, a few hundred bytes of spills) measured
// 2.5-9 % faster per inversion iteration than at two (no spills) and 3 %
// faster than at four; the gather kernel is memory-latency bound and runs
// 7 % faster per adjoint step at eight (32 registers) than at three.
#ifndef SWE_ADJ_FACE_MINB
#define SWE_ADJ_FACE_MINB 3
#endif
#ifndef SWE_ADJ_GATHER_MINB
#define SWE_ADJ_GATHER_MINB 8
#endif

struct AdjArgs {
    const float* S;      // state whose tendency is differentiated, [B,3,ny,nx]
    const float* bed;    // [bedB,1,ny,nx]
    const float* level;  // [levelB]
    const float* lrhs;   // adjoint of the tendency, [B,3,ny,nx]
    float* cx;           // x-face contributions [12 or 16 planes][B][ny][nx+1]
    float* cy;           // y-face contributions [12 or 16 planes][B][ny+1][nx]
    float* lS;           // adjoint of S, accumulated (+=)
    float* llevel_part;  // per-block partial level adjoints [B][gridDim.x]
    float* lbed;         // adjoint of the bed [B,ny,nx], accumulated (+=); BEDG only
    int B, bedB, levelB, ny, nx;
    int bc[4];
    float cval;
    int wsr;
    SweConsts kc;
    // Predictor adjoint fused into the gather (adj_gather_kernel with PRED;
    // S is then the predictor P = clean(U, U + dt/2 k1)): the cell's adjoint
    // of P is not stored but taken through the clean-up's adjoint at once.
    const float* U;       // step input [B,3,ny,nx]
    const float* k1;      // stage-1 tendency [B,3,ny,nx]
    const float* dt_dev;  // the step's dt in device memory, or null: dt
    float dt;
    float* lU;            // adjoint of U, accumulated (+=)
    float* lk1;           // adjoint of k1 (written)
    int positivity;
};

struct PwArgs {
    const float* U;     // step input
    const float* k;     // tendency (k2 for modes 0 and 3, k1 for modes 1 and 2)
    const float* n;     // roughness (modes 0, 3)
    const float* lout;  // adjoint of the step output (modes 0, 3) or of P (mode 1)
    float* lU;          // adjoint of U, accumulated (+=; written in mode 3)
    float* lk;          // adjoint of the tendency (written)
    float* ln;          // adjoint of the roughness field, accumulated (+=) [nB,ny,nx]
    float* P;           // mode 2: predictor output
    float scale;        // dt (modes 0, 3) or dt/2 (modes 1, 2)
    float dt;
    const float* dt_dev;  // if set: dt read from device memory (scale derived here)
    int B, nB, ny, nx, mode, positivity, friction, friction_model;
    SweConsts kc;
};

namespace {

__device__ __forceinline__ size_t a3(int b, int c, int j, int i, int ny, int nx) {
    return (((size_t)b * 3 + c) * ny + j) * nx + i;
}

__device__ __forceinline__ float bed_of(const AdjArgs& a, int b, int j, int i) {
    return a.bed[((size_t)(a.bedB == 1 ? 0 : b) * a.ny + j) * a.nx + i];
}

// Padded cell (j, i) of S with the ghost rules (arm cells only; corners are
// never part of an interior face's stencil).
template <class M>
__device__ PrimRec padded_prim(const AdjArgs& a, int b, int j, int i) {
    const int ny = a.ny, nx = a.nx;
    const bool jin = (unsigned)j < (unsigned)ny, iin = (unsigned)i < (unsigned)nx;
    int js = min(max(j, 0), ny - 1), is = min(max(i, 0), nx - 1);
    const bool xarm = jin && !iin, yarm = iin && !jin;
    int code = -1, side = 0;
    if (xarm || yarm) {
        side = xarm ? (i < 0 ? 0 : 1) : (j < 0 ? 2 : 3);
        code = a.bc[side];
        if (code == SWE_BC_PERIODIC) {
            if (xarm) is = i < 0 ? nx + i : i - nx;
            else js = j < 0 ? ny + j : j - ny;
        }
    }
    const size_t plane = (size_t)ny * nx;
    const size_t o = a3(b, 0, js, is, ny, nx);
    float U0 = a.S[o], U1 = a.S[o + plane], U2 = a.S[o + 2 * plane];
    const float z = bed_of(a, b, js, is);
    const float lev = a.level[a.levelB == 1 ? 0 : b];
    if (code == SWE_BC_CONSTANT) {
        U0 = U1 = U2 = a.cval;
    } else if (code == SWE_BC_WATER_LEVEL) {
        U0 = fmaxf(lev - z, 0.0f);
    } else if (code == SWE_BC_WALL) {
        const int jm = xarm ? j : (j < 0 ? -1 - j : 2 * ny - 1 - j);
        const int im = xarm ? (i < 0 ? -1 - i : 2 * nx - 1 - i) : i;
        const size_t om = a3(b, xarm ? 1 : 2, jm, im, ny, nx);
        if (xarm) U1 = -a.S[om];
        else U2 = -a.S[om];
    } else if (code == SWE_BC_ABSORBING) {
        const float hr = fmaxf(lev - z, 0.0f);
        const float hg = U0;
        const float hc = hr > a.kc.absorb_lim ? hr : hg;
        const float c = M::sqrt(a.kc.g981 * fmaxf(hc, a.kc.absorb_min));
        const float val = ((side == 0 || side == 2) ? -c : c) * (hg - hr);
        if (xarm) U1 = val;
        else U2 = val;
    }
    return prim_rec<M>(U0, U1, U2, z, a.kc);
}

// Face records: 4 cells x (U0, U1, U2[, Z]) floats per face, stored as
// planes (plane p = cell * C + channel, C = 3 or 4; within a plane, face t of
// the launch at t) so that consecutive faces' writes and consecutive cells'
// reads are coalesced.
template <bool BEDG>
__host__ __device__ constexpr int rec_floats() { return BEDG ? 16 : 12; }

__device__ __forceinline__ size_t xfaces(const AdjArgs& a) { return (size_t)a.B * a.ny * (a.nx + 1); }
__device__ __forceinline__ size_t yfaces(const AdjArgs& a) { return (size_t)a.B * (a.ny + 1) * a.nx; }

// Faces of one direction, one thread per face, over blocks [blk, blk + nblk)
// of the launch.
template <bool DIRY, bool BEDG, class M>
__device__ __forceinline__ void face_dir(const AdjArgs& a, int blk, int nblk) {
    const int ny = a.ny, nx = a.nx;
    const long long nfaces = DIRY ? (long long)(ny + 1) * nx : (long long)ny * (nx + 1);
    const long long total = nfaces * a.B;
    const size_t plane = (size_t)ny * nx;
    for (long long t = blk * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)nblk * blockDim.x) {
        const int b = (int)(t / nfaces);
        const long long r = t - (long long)b * nfaces;
        int row, f;  // x: row j, face f in [0, nx]; y: face f in [0, ny], column i (row var)
        if (DIRY) {
            f = (int)(r / nx);
            row = (int)(r - (long long)f * nx);
        } else {
            row = (int)(r / (nx + 1));
            f = (int)(r - (long long)row * (nx + 1));
        }
        PrimRec P[4];
        if (f >= 2 && f <= (DIRY ? ny : nx) - 2) {  // the stencil's four cells are interior
            const size_t o0 = DIRY ? a3(b, 0, f - 2, row, ny, nx) : a3(b, 0, row, f - 2, ny, nx);
            const size_t z0 = DIRY ? ((size_t)(a.bedB == 1 ? 0 : b) * ny + (f - 2)) * nx + row
                                   : ((size_t)(a.bedB == 1 ? 0 : b) * ny + row) * nx + (f - 2);
            const size_t step = DIRY ? (size_t)nx : 1;
            for (int s = 0; s < 4; ++s) {
                const size_t o = o0 + s * step;
                P[s] = prim_rec<M>(a.S[o], a.S[o + plane], a.S[o + 2 * plane], a.bed[z0 + s * step], a.kc);
            }
        } else {
            for (int s = 0; s < 4; ++s)
                P[s] = DIRY ? padded_prim<M>(a, b, f - 2 + s, row) : padded_prim<M>(a, b, row, f - 2 + s);
        }
        // adjoints of the face outputs from the tendencies of the two cells
        // sharing the face: (F_right(f) - F_left(f+1)) / d
        const float d = DIRY ? a.kc.dy : a.kc.dx;
        const float rd = DIRY ? a.kc.rdy : a.kc.rdx;  // RN(1/d): lrhs / d below is exact RN
        const int n = DIRY ? ny : nx;
        float r0p = 0.0f, r1p = 0.0f, r2p = 0.0f, r0m = 0.0f, r1m = 0.0f, r2m = 0.0f;
        if (f < n) {  // cell f: this face is its left/top face
            const size_t o = DIRY ? a3(b, 0, f, row, ny, nx) : a3(b, 0, row, f, ny, nx);
            r0p = M::div(a.lrhs[o], d, rd);
            r1p = M::div(a.lrhs[o + plane], d, rd);
            r2p = M::div(a.lrhs[o + 2 * plane], d, rd);
        }
        if (f >= 1) {  // cell f-1: this face is its right/bottom face
            const size_t o = DIRY ? a3(b, 0, f - 1, row, ny, nx) : a3(b, 0, row, f - 1, ny, nx);
            r0m = M::div(a.lrhs[o], d, rd);
            r1m = M::div(a.lrhs[o + plane], d, rd);
            r2m = M::div(a.lrhs[o + 2 * plane], d, rd);
        }
        const float l_mass = r0p - r0m;
        // x: channel 1 normal, 2 tangential; y: channel 1 tangential, 2 normal
        const float l_nR = DIRY ? r2p : r1p;
        const float l_nL = DIRY ? -r2m : -r1m;
        const float l_tan = DIRY ? (r1p - r1m) : (r2p - r2m);
        CellAdj out[4];
        face_vjp<BEDG, M>(P, l_mass, l_nL, l_nR, l_tan, DIRY, a.kc, a.wsr != 0, out);
        constexpr int C = BEDG ? 4 : 3;
        const size_t np = DIRY ? yfaces(a) : xfaces(a);
        float* dst = (DIRY ? a.cy : a.cx) + t;
        for (int s = 0; s < 4; ++s) {
            dst[(C * s) * np] = out[s].U0;
            dst[(C * s + 1) * np] = out[s].U1;
            dst[(C * s + 2) * np] = out[s].U2;
            if (BEDG) dst[(C * s + 3) * np] = out[s].Z;
        }
    }
}

// The x faces on the first xblocks blocks, the y faces on the rest.
template <bool BEDG, class M>
__global__ void __launch_bounds__(ADJ_THREADS, SWE_ADJ_FACE_MINB) adj_face_kernel(const AdjArgs a, int xblocks) {
    chain_start();
    if ((int)blockIdx.x < xblocks) face_dir<false, BEDG, M>(a, blockIdx.x, xblocks);
    else face_dir<true, BEDG, M>(a, blockIdx.x - xblocks, gridDim.x - xblocks);
}

// Sum of the face contributions to padded cell (row j, column col) along x
// (l[3], the bed channel, with BEDG only).
template <bool BEDG>
__device__ void lam_x(const AdjArgs& a, int b, int j, int col, float l[4]) {
    constexpr int C = BEDG ? 4 : 3;
    const size_t np = xfaces(a);
    l[0] = l[1] = l[2] = l[3] = 0.0f;
    for (int f = col - 1; f <= col + 2; ++f) {
        if (f < 0 || f > a.nx) continue;
        const float* c = a.cx + (((size_t)b * a.ny + j) * (a.nx + 1) + f) + C * (col - f + 2) * np;
        l[0] += c[0];
        l[1] += c[np];
        l[2] += c[2 * np];
        if (BEDG) l[3] += c[3 * np];
    }
}

template <bool BEDG>
__device__ void lam_y(const AdjArgs& a, int b, int row, int i, float l[4]) {
    constexpr int C = BEDG ? 4 : 3;
    const size_t np = yfaces(a);
    l[0] = l[1] = l[2] = l[3] = 0.0f;
    for (int f = row - 1; f <= row + 2; ++f) {
        if (f < 0 || f > a.ny) continue;
        const float* c = a.cy + (((size_t)b * (a.ny + 1) + f) * a.nx + i) + C * (row - f + 2) * np;
        l[0] += c[0];
        l[1] += c[np];
        l[2] += c[2 * np];
        if (BEDG) l[3] += c[3 * np];
    }
}

// Folds the adjoint lg of ghost g (side `side`; g its column for left/right,
// row for top/bottom) into cell (j, i) if the ghost was made from it, and
// adds the level adjoint once per ghost (in the thread of the ghost's
// clamped source cell).  BEDG: lg[3] is the ghost's bed adjoint, folded into
// the cell its bed was copied from (replicate, or periodic), plus the bed
// terms of the forced ghost depth max(level - z, 0) -> lzc.
template <bool BEDG, class M>
__device__ void fold_ghost(const AdjArgs& a, int b, int side, int g, const float lg[4], int j,
                           int i, float lam[3], float& llev, float& lzc) {
    const int ny = a.ny, nx = a.nx;
    const bool xs = side < 2;
    const int n = xs ? nx : ny;
    const int pos = xs ? i : j;  // this cell's index along the side's direction
    const int clamp_src = g < 0 ? 0 : n - 1;
    const int mirror = g < 0 ? -1 - g : 2 * n - 1 - g;
    const int periodic = g < 0 ? n + g : g - n;
    const int normal = xs ? 1 : 2;  // momentum channel reflected by a wall
    const int code = a.bc[side];
    if (BEDG && pos == (code == SWE_BC_PERIODIC ? periodic : clamp_src)) lzc += lg[3];
    switch (code) {
    case SWE_BC_TRANSMISSIVE:
        if (pos == clamp_src) {
            lam[0] += lg[0];
            lam[1] += lg[1];
            lam[2] += lg[2];
        }
        break;
    case SWE_BC_PERIODIC:
        if (pos == periodic) {
            lam[0] += lg[0];
            lam[1] += lg[1];
            lam[2] += lg[2];
        }
        break;
    case SWE_BC_CONSTANT:
        break;
    case SWE_BC_WATER_LEVEL:
        if (pos == clamp_src) {
            lam[1] += lg[1];
            lam[2] += lg[2];
            const float z = bed_of(a, b, xs ? j : clamp_src, xs ? clamp_src : i);
            const float lev = a.level[a.levelB == 1 ? 0 : b];
            if (lev - z >= 0.0f) {  // clamp(level - z, min=0)
                llev += lg[0];
                if (BEDG) lzc -= lg[0];
            }
        }
        break;
    case SWE_BC_WALL:
        if (pos == clamp_src) {
            lam[0] += lg[0];
            lam[3 - normal] += lg[3 - normal];
        }
        if (pos == mirror) lam[normal] -= lg[normal];
        break;
    case SWE_BC_ABSORBING:
        if (pos == clamp_src) {
            lam[3 - normal] += lg[3 - normal];
            lam[0] += lg[0];
            // value = s c (hg - hr), hr = max(level - z, 0),
            // c = sqrt(9.81 max(where(hr > 1e-4, hr, hg), 1e-6))
            const size_t plane = (size_t)ny * nx;
            const int jj = xs ? j : clamp_src, ii = xs ? clamp_src : i;
            const float hg = a.S[a3(b, 0, jj, ii, ny, nx)];
            (void)plane;
            const float z = bed_of(a, b, jj, ii);
            const float lev = a.level[a.levelB == 1 ? 0 : b];
            const float hr = fmaxf(lev - z, 0.0f);
            const bool use_hr = hr > a.kc.absorb_lim;
            const float hc = use_hr ? hr : hg;
            const float cm = fmaxf(hc, a.kc.absorb_min);
            const float c = M::sqrt(a.kc.g981 * cm);
            const float s = (side == 0 || side == 2) ? -1.0f : 1.0f;
            const float lv = lg[normal];
            const float l_c = lv * (s * (hg - hr));
            const float l_diff = lv * (s * c);
            float l_hc = 0.0f;
            if (hc >= a.kc.absorb_min) {
                const float c2 = 2.0f * c;
                l_hc = a.kc.g981 * M::div(l_c, c2, M::rcp(c2));
            }
            float l_hg = l_diff + (use_hr ? 0.0f : l_hc);
            float l_hr = -l_diff + (use_hr ? l_hc : 0.0f);
            lam[0] += l_hg;
            if (lev - z >= 0.0f) {
                llev += l_hr;
                if (BEDG) lzc -= l_hr;
            }
        }
        break;
    default:
        break;
    }
}

// _clean_and_limit (solver.py:547-570) in the arithmetic M.
template <class M>
__device__ __forceinline__ State clean_fwd(const State& o, State c, const SweConsts& k, bool positivity) {
    if (positivity) {
        const float d0 = c.h - o.h, d1 = c.hu - o.hu, d2 = c.hv - o.hv;
        const float safe = fmaxf(-d0, k.eps);
        const float th = d0 < 0.0f ? fminf(M::div(o.h, safe, M::rcp(safe)), 1.0f) : 1.0f;
        c.h = o.h + th * d0;
        c.hu = o.hu + th * d1;
        c.hv = o.hv + th * d2;
    }
    State r;
    r.h = fmaxf(c.h, 0.0f);
    const bool wet = r.h > k.dry;
    r.hu = wet ? c.hu : 0.0f;
    r.hv = wet ? c.hv : 0.0f;
    return r;
}

// Adjoint of _clean_and_limit (solver.py:547-570): returns lam_old, lam_cand.
template <class M>
__device__ void clean_bwd(const State& o, const State& c, const State& lout, const SweConsts& k,
                          bool positivity, State& lold, State& lcand) {
    State cp = c;
    float d0 = 0.0f, d1 = 0.0f, d2 = 0.0f, th = 1.0f, ratio = 0.0f, safe = 0.0f, ysafe = 0.0f;
    bool theta_branch = false;
    if (positivity) {
        d0 = c.h - o.h;
        d1 = c.hu - o.hu;
        d2 = c.hv - o.hv;
        safe = fmaxf(-d0, k.eps);
        ysafe = M::rcp(safe);
        ratio = M::div(o.h, safe, ysafe);
        theta_branch = d0 < 0.0f;
        th = theta_branch ? fminf(ratio, 1.0f) : 1.0f;
        cp.h = o.h + th * d0;
        cp.hu = o.hu + th * d1;
        cp.hv = o.hv + th * d2;
    }
    const float h = fmaxf(cp.h, 0.0f);
    const bool wet = h > k.dry;
    State lcp;
    lcp.h = cp.h >= 0.0f ? lout.h : 0.0f;
    lcp.hu = wet ? lout.hu : 0.0f;
    lcp.hv = wet ? lout.hv : 0.0f;
    if (!positivity) {
        lold = State{0.0f, 0.0f, 0.0f};
        lcand = lcp;
        return;
    }
    // cand' = old + th * delta
    const float l_th = lcp.h * d0 + lcp.hu * d1 + lcp.hv * d2;
    float ld0 = lcp.h * th, ld1 = lcp.hu * th, ld2 = lcp.hv * th;
    lold = lcp;
    if (theta_branch && ratio <= 1.0f) {  // th = clamp(old_h / safe, max=1)
        lold.h += M::div(l_th, safe, ysafe);
        const float l_safe = -l_th * M::div(ratio, safe, ysafe);
        if (-d0 >= k.eps) ld0 -= l_safe;  // safe = clamp(-dh, min=eps)
    }
    lcand = State{ld0, ld1, ld2};
    lold.h -= ld0;
    lold.hu -= ld1;
    lold.hv -= ld2;
}

// Adjoint of the friction update (friction.py:12-131) w.r.t. its input state
// and the roughness field.
template <class M>
__device__ void friction_bwd(const State& s0, float n, float dt, int model, const SweConsts& k,
                             const State& lout, State& ls, float& ln) {
    const float h = fmaxf(s0.h, 0.0f);
    const bool wet = h > k.dry;
    const float safe = fmaxf(h, k.fr_vs);
    const float ys = M::rcp(safe);
    const float u = M::div(wet ? s0.hu : 0.0f, safe, ys), v = M::div(wet ? s0.hv : 0.0f, safe, ys);
    const float sp2 = u * u + v * v;
    const bool moving = wet && sp2 > 0.0f;
    const float S = fmaxf(sp2, k.fr_e2);
    const float speed = moving ? M::sqrt(S) : 0.0f;
    float cf;
    // cf and d cf / d h, d cf / d n (as autograd evaluates them)
    float dcf_dpre = 0.0f, dcf_dn = 0.0f, hpre = 0.0f;
    bool h_pass = false, n_pass = false;
    if (model == 0) {
        const float nn = fmaxf(n, 0.0f);
        hpre = fmaxf(h, k.fr_e);
        const float pw = M::pow(hpre, k.third);
        const float num = k.g981 * (nn * nn);
        const float ypw = M::rcp(pw);
        cf = M::div(num, pw, ypw);
        // d/d pw: -cf / pw ; d pw / d hpre = third * hpre^(third - 1)
        const float dpw = k.third * M::pow(hpre, k.third - 1.0f);
        dcf_dpre = -M::div(cf, pw, ypw) * dpw;
        dcf_dn = M::div(k.g981 * (2.0f * nn), pw, ypw);
        h_pass = h >= k.fr_e;
        n_pass = n >= 0.0f;
    } else {
        const float zz = fmaxf(n, k.fr_e);
        hpre = fmaxf(h, k.fr_e);
        const float yzz = M::rcp(zz);
        const float ratio = M::div(hpre, zz, yzz);
        const float shallow_den = fmaxf(0.46f * ratio, k.fr_e);
        const float rc = fmaxf(ratio, k.fr_e);
        const float lg = M::ln(rc);
        const float inv_rc = M::inv(rc);
        const float lt = 2.5f * ((lg - 1.0f) + inv_rc * 1.359f);
        const float deep_den = fmaxf(lt * lt, k.fr_e);
        const bool shallow_b = ratio < 2.71828182845904523536f;
        cf = shallow_b ? M::inv(shallow_den) : M::inv(deep_den);
        float dcf_dratio;
        if (shallow_b) {
            dcf_dratio = (0.46f * ratio >= k.fr_e) ? -(cf * cf) * 0.46f : 0.0f;
        } else {
            float dlt = 0.0f;
            if (ratio >= k.fr_e) dlt = 2.5f * (inv_rc - 1.359f * inv_rc * inv_rc);
            dcf_dratio = (lt * lt >= k.fr_e) ? -(cf * cf) * (2.0f * lt) * dlt : 0.0f;
        }
        dcf_dpre = M::div(dcf_dratio, zz, yzz);
        dcf_dn = -dcf_dratio * M::div(ratio, zz, yzz);
        h_pass = h >= k.fr_e;
        n_pass = n >= k.fr_e;
    }
    const float X = M::div((cf * speed) * dt, safe, ys);
    const float fac = M::inv(1.0f + X);
    ls.h = lout.h;
    ls.hu = wet ? lout.hu * fac : 0.0f;
    ls.hv = wet ? lout.hv * fac : 0.0f;
    float l_fac = wet ? lout.hu * s0.hu + lout.hv * s0.hv : 0.0f;
    const float l_D = -l_fac * (fac * fac);
    const float l_num = M::div(l_D, safe, ys);  // d/d((cf speed) dt)
    float l_safe = -l_D * M::div(X, safe, ys);
    const float l_cs = l_num * dt;
    const float l_cf = l_cs * speed;
    const float l_speed = l_cs * cf;
    float l_u = 0.0f, l_v = 0.0f;
    if (moving) {
        const float s2 = 2.0f * speed;
        const float l_S = M::div(l_speed, s2, M::rcp(s2));
        if (sp2 >= k.fr_e2) {
            l_u = l_S * (2.0f * u);
            l_v = l_S * (2.0f * v);
        }
    }
    if (wet) {
        ls.hu += M::div(l_u, safe, ys);
        ls.hv += M::div(l_v, safe, ys);
    }
    l_safe -= l_u * M::div(u, safe, ys) + l_v * M::div(v, safe, ys);
    float l_h = 0.0f;
    if (h >= k.fr_vs) l_h += l_safe;
    if (h_pass) l_h += l_cf * dcf_dpre;
    ln = n_pass ? l_cf * dcf_dn : 0.0f;
    if (s0.h >= 0.0f) ls.h += l_h;
}

template <bool BEDG, bool PRED, class M>
__global__ void __launch_bounds__(ADJ_THREADS, SWE_ADJ_GATHER_MINB) adj_gather_kernel(const AdjArgs a) {
    chain_start();
    const int ny = a.ny, nx = a.nx;
    const int b = blockIdx.y;
    const long long ncell = (long long)ny * nx;
    const size_t plane = (size_t)ny * nx;
    float llev = 0.0f;
    float scale = 0.0f;
    if (PRED) scale = 0.5f * (a.dt_dev != nullptr ? *a.dt_dev : a.dt);
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < ncell;
         t += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(t / nx), i = (int)(t - (long long)(t / nx) * nx);
        float lam[4], l[4];
        lam_x<BEDG>(a, b, j, i, lam);
        lam_y<BEDG>(a, b, j, i, l);
        lam[0] += l[0];
        lam[1] += l[1];
        lam[2] += l[2];
        float lz = BEDG ? lam[3] + l[3] : 0.0f;
        if (i < 2 || i >= nx - 2) {
            const int gx[4] = {-1, -2, nx, nx + 1};
            for (int q = 0; q < 4; ++q) {
                lam_x<BEDG>(a, b, j, gx[q], l);
                fold_ghost<BEDG, M>(a, b, q < 2 ? 0 : 1, gx[q], l, j, i, lam, llev, lz);
            }
        }
        if (j < 2 || j >= ny - 2) {
            const int gy[4] = {-1, -2, ny, ny + 1};
            for (int q = 0; q < 4; ++q) {
                lam_y<BEDG>(a, b, gy[q], i, l);
                fold_ghost<BEDG, M>(a, b, q < 2 ? 2 : 3, gy[q], l, j, i, lam, llev, lz);
            }
        }
        const size_t o = a3(b, 0, j, i, ny, nx);
        if (PRED) {  // predictor P = clean(U, U + dt/2 k1), solver.py:639
            const State u{a.U[o], a.U[o + plane], a.U[o + 2 * plane]};
            const State cand{u.h + scale * a.k1[o], u.hu + scale * a.k1[o + plane],
                             u.hv + scale * a.k1[o + 2 * plane]};
            State lold, lcand;
            clean_bwd<M>(u, cand, State{lam[0], lam[1], lam[2]}, a.kc, a.positivity != 0, lold,
                         lcand);
            a.lU[o] += lold.h + lcand.h;
            a.lU[o + plane] += lold.hu + lcand.hu;
            a.lU[o + 2 * plane] += lold.hv + lcand.hv;
            a.lk1[o] = lcand.h * scale;
            a.lk1[o + plane] = lcand.hu * scale;
            a.lk1[o + 2 * plane] = lcand.hv * scale;
        } else {
            a.lS[o] += lam[0];
            a.lS[o + plane] += lam[1];
            a.lS[o + 2 * plane] += lam[2];
        }
        if (BEDG) a.lbed[(size_t)b * plane + (size_t)j * nx + i] += lz;
    }
    // per-block partial sum of the level adjoint (fixed order)
    __shared__ float s_part[ADJ_THREADS / 32];
    for (int off = 16; off > 0; off >>= 1) llev += __shfl_down_sync(0xffffffffu, llev, off);
    if ((threadIdx.x & 31) == 0) s_part[threadIdx.x >> 5] = llev;
    __syncthreads();
    if (threadIdx.x == 0) {
        float sum = 0.0f;
        for (int w = 0; w < ADJ_THREADS / 32; ++w) sum += s_part[w];
        a.llevel_part[(size_t)b * gridDim.x + blockIdx.x] = sum;
    }
}

// ------------------------------------------------------- pointwise adjoints

template <class M>
__global__ void adj_pointwise_kernel(const PwArgs a) {
    chain_start();
    const long long plane = (long long)a.ny * a.nx;
    const long long total = plane * a.B;
    float dt = a.dt, scale = a.scale;
    if (a.dt_dev != nullptr) {
        dt = *a.dt_dev;
        scale = (a.mode == 0 || a.mode == 3) ? dt : 0.5f * dt;
    }
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const int b = (int)(t / plane);
        const long long i = t - (long long)b * plane;
        const size_t o = (size_t)b * 3 * plane + i;
        const State u{a.U[o], a.U[o + plane], a.U[o + 2 * plane]};
        const State cand{u.h + scale * a.k[o], u.hu + scale * a.k[o + plane],
                         u.hv + scale * a.k[o + 2 * plane]};
        if (a.mode == 2) {  // predictor forward, solver.py:639
            const State p = clean_fwd<M>(u, cand, a.kc, a.positivity != 0);
            a.P[o] = p.h;
            a.P[o + plane] = p.hu;
            a.P[o + 2 * plane] = p.hv;
            continue;
        }
        State lq{a.lout[o], a.lout[o + plane], a.lout[o + 2 * plane]};
        if ((a.mode == 0 || a.mode == 3) && a.friction) {
            const State q = clean_fwd<M>(u, cand, a.kc, a.positivity != 0);
            const size_t on = (size_t)(a.nB == 1 ? 0 : b) * plane + i;
            State lqi;
            float ln = 0.0f;
            friction_bwd<M>(q, a.n[on], dt, a.friction_model, a.kc, lq, lqi, ln);
            lq = lqi;
            if (a.nB == 1 && a.B > 1) atomicAdd(&a.ln[on], ln);
            else a.ln[on] += ln;
        }
        State lold, lcand;
        clean_bwd<M>(u, cand, lq, a.kc, a.positivity != 0, lold, lcand);
        // cand = U + scale * k; mode 3 writes the adjoint of U instead of adding to it
        if (a.mode == 3) {
            a.lU[o] = lold.h + lcand.h;
            a.lU[o + plane] = lold.hu + lcand.hu;
            a.lU[o + 2 * plane] = lold.hv + lcand.hv;
        } else {
            a.lU[o] += lold.h + lcand.h;
            a.lU[o + plane] += lold.hu + lcand.hu;
            a.lU[o + 2 * plane] += lold.hv + lcand.hv;
        }
        a.lk[o] = lcand.h * scale;
        a.lk[o + plane] = lcand.hu * scale;
        a.lk[o + 2 * plane] = lcand.hv * scale;
    }
}

inline int blocks_for(long long n) {
    long long b = (n + ADJ_THREADS - 1) / ADJ_THREADS;
    if (b < 1) b = 1;
    return (int)(b > 148LL * 32 ? 148LL * 32 : b);
}

// Enqueue the spatial adjoint of a (a.lbed set: with the bed's adjoint;
// pred: the stage-2 form, the predictor adjoint fused into the gather).
template <class M>
int launch_adj_spatial(const AdjArgs& a, int level_blocks, bool pred, cudaStream_t s) {
    const int gx = blocks_for((long long)a.B * a.ny * (a.nx + 1));
    const int gy = blocks_for((long long)a.B * (a.ny + 1) * a.nx);
    const dim3 gg(level_blocks, a.B), gf(gx + gy), th(ADJ_THREADS);
    cudaError_t e;
    if (a.lbed) {
        e = launch_chained(adj_face_kernel<true, M>, gf, th, s, a, gx);
        if (e == cudaSuccess)
            e = pred ? launch_chained(adj_gather_kernel<true, true, M>, gg, th, s, a)
                     : launch_chained(adj_gather_kernel<true, false, M>, gg, th, s, a);
    } else {
        e = launch_chained(adj_face_kernel<false, M>, gf, th, s, a, gx);
        if (e == cudaSuccess)
            e = pred ? launch_chained(adj_gather_kernel<false, true, M>, gg, th, s, a)
                     : launch_chained(adj_gather_kernel<false, false, M>, gg, th, s, a);
    }
    return e == cudaSuccess && cudaGetLastError() == cudaSuccess ? SWE_OK : SWE_ECUDA;
}

template <class M>
int launch_adj_pointwise(const PwArgs& a, cudaStream_t s) {
    const cudaError_t e = launch_chained(adj_pointwise_kernel<M>, dim3(blocks_for((long long)a.B * a.ny * a.nx)),
                                         dim3(ADJ_THREADS), s, a);
    return e == cudaSuccess && cudaGetLastError() == cudaSuccess ? SWE_OK : SWE_ECUDA;
}

}  // namespace

// The FastMath instantiations (swe_adjoint_fast.cu).
int fast_launch_adj_spatial(const AdjArgs& a, int level_blocks, bool pred, cudaStream_t s);
int fast_launch_adj_pointwise(const PwArgs& a, cudaStream_t s);

}  // namespace swe
