// swe_ops.cu -- the reference's numerical operators as standalone sm_100a
// kernels (the drop-in call surface of boundary.py, reconstruction.py,
// riemann.py, numerics.py, friction.py and SWE2D._clean_and_limit).
//
// Each kernel is elementwise (one thread per output cell, grid-stride) and
// uses the same FP32 functions as the fused step (swe_math.cuh), so an
// operator applied to the same inputs gives bit-identical values to the
// step's internal ones.
#include <cuda_runtime.h>

#include "swe_common.cuh"

namespace swe {
namespace {

constexpr int OPS_THREADS = 256;

inline int blocks_for(long long n) {
    long long b = (n + OPS_THREADS - 1) / OPS_THREADS;
    if (b < 1) b = 1;
    return (int)(b > 148LL * 64 ? 148LL * 64 : b);
}

// ------------------------------------------------------------ ghost cells
struct GcArgs {
    const float* U;
    const float* bed;
    const float* level;
    const float* cval;
    float* Up;
    float* zp;
    int B, bedB, levelB, cvalB, ny, nx, ng, H, W;
    int bc[4];
    SweConsts kc;
};

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return min(max(v, lo), hi); }

__device__ __forceinline__ float u_at(const GcArgs& a, int b, int ch, int j, int i) {
    return a.U[(((size_t)b * 3 + ch) * a.ny + j) * a.nx + i];
}

// Padded bed: replicate, then the periodic arms (boundary.py:234-257).
__device__ float zp_at(const GcArgs& a, int bb, int q, int p) {
    const int ng = a.ng, H = a.H, W = a.W;
    int j = clampi(q - ng, 0, a.ny - 1), i = clampi(p - ng, 0, a.nx - 1);
    const bool rows = q >= ng && q < H - ng, cols = p >= ng && p < W - ng;
    if (a.bc[0] == SWE_BC_PERIODIC && p < ng && rows) i = a.nx - ng + p;
    if (a.bc[1] == SWE_BC_PERIODIC && p >= W - ng && rows) i = p - (W - ng);
    if (a.bc[2] == SWE_BC_PERIODIC && q < ng && cols) j = a.ny - ng + q;
    if (a.bc[3] == SWE_BC_PERIODIC && q >= H - ng && cols) j = q - (H - ng);
    return a.bed[((size_t)bb * a.ny + j) * a.nx + i];
}

// forced_h = clamp(level - zp, min=0), boundary.py:279-282
__device__ __forceinline__ float forced(const GcArgs& a, int b, int q, int p) {
    const float lev = a.level[a.levelB == 1 ? 0 : b];
    return fmaxf(lev - zp_at(a, a.bedB == 1 ? 0 : b, q, p), 0.0f);
}

__device__ __forceinline__ float cval(const GcArgs& a, int b) { return a.cval[a.cvalB == 1 ? 0 : b]; }

// Flather radiation value -c (h_ghost - h_ref) (sign < 0) or +c (...),
// boundary.py:318-328.
__device__ __forceinline__ float absorbing(const GcArgs& a, float hg, float hr, bool negative) {
    const float hc = hr > a.kc.absorb_lim ? hr : hg;
    const float c = sqrtf(a.kc.g981 * fmaxf(hc, a.kc.absorb_min));
    return (negative ? -c : c) * (hg - hr);
}

// The padded state after each of the reference's sequential overwrites.
__device__ float v0(const GcArgs& a, int b, int ch, int q, int p) {
    return u_at(a, b, ch, clampi(q - a.ng, 0, a.ny - 1), clampi(p - a.ng, 0, a.nx - 1));
}

__device__ float v_left(const GcArgs& a, int b, int ch, int q, int p) {  // boundary.py:301-328
    const int ng = a.ng;
    if (p >= ng) return v0(a, b, ch, q, p);
    switch (a.bc[0]) {
    case SWE_BC_PERIODIC:
        if (q >= ng && q < a.H - ng) return u_at(a, b, ch, q - ng, a.nx - ng + p);
        return v0(a, b, ch, q, p);
    case SWE_BC_CONSTANT: return cval(a, b);
    case SWE_BC_WATER_LEVEL: return ch == 0 ? forced(a, b, q, p) : v0(a, b, ch, q, p);
    case SWE_BC_WALL: return ch == 1 ? -v0(a, b, 1, q, 2 * ng - 1 - p) : v0(a, b, ch, q, p);
    case SWE_BC_ABSORBING:
        return ch == 1 ? absorbing(a, v0(a, b, 0, q, p), forced(a, b, q, p), true) : v0(a, b, ch, q, p);
    default: return v0(a, b, ch, q, p);
    }
}

__device__ float v_right(const GcArgs& a, int b, int ch, int q, int p) {  // boundary.py:336-357
    const int ng = a.ng, W = a.W;
    if (p < W - ng) return v_left(a, b, ch, q, p);
    switch (a.bc[1]) {
    case SWE_BC_PERIODIC:
        if (q >= ng && q < a.H - ng) return u_at(a, b, ch, q - ng, p - (W - ng));
        return v_left(a, b, ch, q, p);
    case SWE_BC_CONSTANT: return cval(a, b);
    case SWE_BC_WATER_LEVEL: return ch == 0 ? forced(a, b, q, p) : v_left(a, b, ch, q, p);
    case SWE_BC_WALL:
        return ch == 1 ? -v_left(a, b, 1, q, 2 * (W - ng) - 1 - p) : v_left(a, b, ch, q, p);
    case SWE_BC_ABSORBING:
        return ch == 1 ? absorbing(a, v_left(a, b, 0, q, p), forced(a, b, q, p), false)
                       : v_left(a, b, ch, q, p);
    default: return v_left(a, b, ch, q, p);
    }
}

__device__ float v_top(const GcArgs& a, int b, int ch, int q, int p) {  // boundary.py:363-384
    const int ng = a.ng;
    if (q >= ng) return v_right(a, b, ch, q, p);
    switch (a.bc[2]) {
    case SWE_BC_PERIODIC:
        if (p >= ng && p < a.W - ng) return u_at(a, b, ch, a.ny - ng + q, p - ng);
        return v_right(a, b, ch, q, p);
    case SWE_BC_CONSTANT: return cval(a, b);
    case SWE_BC_WATER_LEVEL: return ch == 0 ? forced(a, b, q, p) : v_right(a, b, ch, q, p);
    case SWE_BC_WALL: return ch == 2 ? -v_right(a, b, 2, 2 * ng - 1 - q, p) : v_right(a, b, ch, q, p);
    case SWE_BC_ABSORBING:
        return ch == 2 ? absorbing(a, v_right(a, b, 0, q, p), forced(a, b, q, p), true)
                       : v_right(a, b, ch, q, p);
    default: return v_right(a, b, ch, q, p);
    }
}

__device__ float v_bottom(const GcArgs& a, int b, int ch, int q, int p) {  // boundary.py:390-411
    const int ng = a.ng, H = a.H;
    if (q < H - ng) return v_top(a, b, ch, q, p);
    switch (a.bc[3]) {
    case SWE_BC_PERIODIC:
        if (p >= ng && p < a.W - ng) return u_at(a, b, ch, q - (H - ng), p - ng);
        return v_top(a, b, ch, q, p);
    case SWE_BC_CONSTANT: return cval(a, b);
    case SWE_BC_WATER_LEVEL: return ch == 0 ? forced(a, b, q, p) : v_top(a, b, ch, q, p);
    case SWE_BC_WALL:
        return ch == 2 ? -v_top(a, b, 2, 2 * (H - ng) - 1 - q, p) : v_top(a, b, ch, q, p);
    case SWE_BC_ABSORBING:
        return ch == 2 ? absorbing(a, v_top(a, b, 0, q, p), forced(a, b, q, p), false)
                       : v_top(a, b, ch, q, p);
    default: return v_top(a, b, ch, q, p);
    }
}

__global__ void ghost_cells_kernel(const GcArgs a) {
    const long long plane = (long long)a.H * a.W;
    const long long nb = (long long)max(a.B, a.bedB) * plane;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nb;
         t += (long long)gridDim.x * blockDim.x) {
        const int b = (int)(t / plane);
        const int rem = (int)(t - (long long)b * plane);
        const int q = rem / a.W, p = rem - (rem / a.W) * a.W;
        if (b < a.B)
            for (int ch = 0; ch < 3; ++ch)
                a.Up[((size_t)b * 3 + ch) * plane + rem] = v_bottom(a, b, ch, q, p);
        if (b < a.bedB) a.zp[(size_t)b * plane + rem] = zp_at(a, b, q, p);
    }
}

// --------------------------------------------------------- reconstruction
struct RcArgs {
    const float* Up;
    const float* zp;
    float *UL, *UR, *sL, *sR;
    int B, zB, H, W, dim_x, wsr;
    SweConsts kc;
};

__device__ __forceinline__ Prim rc_prim(const RcArgs& a, int b, int q, int p) {
    const size_t plane = (size_t)a.H * a.W;
    const size_t o = (size_t)q * a.W + p;
    const float* U = a.Up + (size_t)b * 3 * plane;
    return make_prim(U[o], U[plane + o], U[2 * plane + o], a.zp[(size_t)(a.zB == 1 ? 0 : b) * plane + o], a.kc);
}

__global__ void reconstruction_kernel(const RcArgs a) {
    const long long plane = (long long)a.H * a.W;
    const long long total = (long long)a.B * plane;
    const int len = a.dim_x ? a.W : a.H;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const int b = (int)(t / plane);
        const int rem = (int)(t - (long long)b * plane);
        const int q = rem / a.W, p = rem - (rem / a.W) * a.W;
        const int k = a.dim_x ? p : q;
        Prim c[4];  // cells k-1, k, k+1, k+2 along the line, torch.roll wrap-around
        for (int s = 0; s < 4; ++s) {
            const int kk = (k - 1 + s + 2 * len) % len;
            c[s] = a.dim_x ? rc_prim(a, b, q, kk) : rc_prim(a, b, kk, p);
        }
        const Sides L = make_sides(c[0], c[1], c[2], a.kc, a.wsr != 0);
        const Sides R = make_sides(c[1], c[2], c[3], a.kc, a.wsr != 0);
        const FaceStates f = face_states(L.p, c[1].h, c[1].z, R.m, c[2].h, c[2].z, a.kc);
        const size_t o3 = (size_t)b * 3 * plane + rem;
        a.UL[o3] = f.L0;
        a.UL[o3 + plane] = f.L1;
        a.UL[o3 + 2 * plane] = f.L2;
        a.UR[o3] = f.R0;
        a.UR[o3 + plane] = f.R1;
        a.UR[o3 + 2 * plane] = f.R2;
        a.sL[(size_t)b * plane + rem] = f.srcL;
        a.sR[(size_t)b * plane + rem] = f.srcR;
    }
}

// ---------------------------------------------------------------- HLL flux
__global__ void hll_kernel(const float* UL, const float* UR, float* F, float* speed, int B,
                           long long plane, int normal_y, const SweConsts kc) {
    const long long total = (long long)B * plane;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const long long b = t / plane, i = t - b * plane;
        const size_t o = (size_t)b * 3 * plane + i;
        const Hll h = hll_flux(UL[o], UL[o + plane], UL[o + 2 * plane], UR[o], UR[o + plane],
                               UR[o + 2 * plane], normal_y != 0, kc);
        F[o] = h.fh;
        F[o + plane] = normal_y ? h.ft : h.fq;
        F[o + 2 * plane] = normal_y ? h.fq : h.ft;
        speed[t] = u2f(h.speed_bits);
    }
}

// --------------------------------------------------------------- primitive
__global__ void primitive_kernel(const float* U, float* h, float* u, float* v, float* c, int B,
                                 long long plane, const SweConsts kc) {
    const long long total = (long long)B * plane;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const long long b = t / plane, i = t - b * plane;
        const size_t o = (size_t)b * 3 * plane + i;
        float hh, uu, vv, cc;
        face_primitive(U[o], U[o + plane], U[o + 2 * plane], kc, hh, uu, vv, cc);
        h[t] = hh;
        u[t] = uu;
        v[t] = vv;
        c[t] = cc;
    }
}

// ------------------------------------------------------ limited increment
__global__ void limited_increment_kernel(const float* q, float* out, long long lines_outer, int H,
                                         int W, int dim_x, float theta) {
    const long long plane = (long long)H * W;
    const long long total = lines_outer * plane;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const long long bc = t / plane;
        const int rem = (int)(t - bc * plane);
        const int r = rem / W, x = rem - (rem / W) * W;
        const float* base = q + bc * plane;
        float qm, qp;
        if (dim_x) {
            qm = base[(size_t)r * W + (x - 1 + W) % W];
            qp = base[(size_t)r * W + (x + 1) % W];
        } else {
            qm = base[(size_t)((r - 1 + H) % H) * W + x];
            qp = base[(size_t)((r + 1) % H) * W + x];
        }
        out[t] = limited_increment(qm, base[rem], qp, theta);
    }
}

__global__ void minmod3_kernel(const float* a, const float* b, const float* c, float* out,
                               long long n) {
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x)
        out[t] = minmod3(a[t], b[t], c[t]);
}

// ------------------------------------------------- clean / limit, friction
__global__ void clean_kernel(const float* old, const float* cand, float* out, int B,
                             long long plane, int positivity, const SweConsts kc) {
    const long long total = (long long)B * plane;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const long long b = t / plane, i = t - b * plane;
        const size_t o = (size_t)b * 3 * plane + i;
        const State r = clean_and_limit(State{old[o], old[o + plane], old[o + 2 * plane]},
                                        State{cand[o], cand[o + plane], cand[o + 2 * plane]}, kc,
                                        positivity != 0);
        out[o] = r.h;
        out[o + plane] = r.hu;
        out[o + 2 * plane] = r.hv;
    }
}

__global__ void friction_kernel(const float* U, const float* n, int nB, float* out, int B,
                                long long plane, float dt, int model, const SweConsts kc) {
    const long long total = (long long)B * plane;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const long long b = t / plane, i = t - b * plane;
        const size_t o = (size_t)b * 3 * plane + i;
        const float nv = n[(size_t)(nB == 1 ? 0 : b) * plane + i];
        const State s{U[o], U[o + plane], U[o + 2 * plane]};
        const State r = model == 0 ? manning(s, nv, dt, kc) : roughness_friction(s, nv, dt, kc);
        out[o] = r.h;
        out[o + plane] = r.hu;
        out[o + 2 * plane] = r.hv;
    }
}

bool batch_ok(int x, int B) { return x == 1 || x == B; }

int launch_result() { return cudaGetLastError() == cudaSuccess ? SWE_OK : SWE_ECUDA; }

}  // namespace
}  // namespace swe

using namespace swe;

extern "C" int swe_ghost_cells_f32(const float* U, const float* bed, int B, int bedB, int ny,
                                   int nx, int ng, const swe_params* p, const float* level,
                                   int levelB, const float* constant_value, int cvalB, float* Up,
                                   float* zp, void* stream) {
    if (!U || !bed || !level || !constant_value || !Up || !zp || !valid_params(p)) return SWE_EARG;
    if (B < 1 || ng < 1 || ng > ny || ng > nx) return SWE_EARG;  // boundary.py:91-102
    if (!batch_ok(bedB, B) || !batch_ok(levelB, B) || !batch_ok(cvalB, B)) return SWE_EARG;
    GcArgs a{};
    a.U = U;
    a.bed = bed;
    a.level = level;
    a.cval = constant_value;
    a.Up = Up;
    a.zp = zp;
    a.B = B;
    a.bedB = bedB;
    a.levelB = levelB;
    a.cvalB = cvalB;
    a.ny = ny;
    a.nx = nx;
    a.ng = ng;
    a.H = ny + 2 * ng;
    a.W = nx + 2 * ng;
    a.bc[0] = p->bc_left;
    a.bc[1] = p->bc_right;
    a.bc[2] = p->bc_top;
    a.bc[3] = p->bc_bottom;
    a.kc = make_consts(*p);
    const long long n = (long long)(B > bedB ? B : bedB) * a.H * a.W;
    ghost_cells_kernel<<<blocks_for(n), OPS_THREADS, 0, (cudaStream_t)stream>>>(a);
    return launch_result();
}

extern "C" int swe_reconstruction_f32(const float* Up, const float* zp, int B, int zB, int H, int W,
                                      int dim, const swe_params* p, float* UL, float* UR,
                                      float* sL, float* sR, void* stream) {
    if (!Up || !zp || !UL || !UR || !sL || !sR || !valid_params(p)) return SWE_EARG;
    if (B < 1 || H < 1 || W < 1 || !batch_ok(zB, B) || (dim != -1 && dim != -2)) return SWE_EARG;
    RcArgs a{};
    a.Up = Up;
    a.zp = zp;
    a.UL = UL;
    a.UR = UR;
    a.sL = sL;
    a.sR = sR;
    a.B = B;
    a.zB = zB;
    a.H = H;
    a.W = W;
    a.dim_x = dim == -1;
    a.wsr = p->water_slope_reset;
    a.kc = make_consts(*p);
    reconstruction_kernel<<<blocks_for((long long)B * H * W), OPS_THREADS, 0, (cudaStream_t)stream>>>(a);
    return launch_result();
}

extern "C" int swe_hll_flux_f32(const float* UL, const float* UR, int B, int H, int W, int normal_y,
                                const swe_params* p, float* flux, float* speed, void* stream) {
    if (!UL || !UR || !flux || !speed || !valid_params(p) || B < 1 || H < 1 || W < 1) return SWE_EARG;
    const long long plane = (long long)H * W;
    hll_kernel<<<blocks_for(B * plane), OPS_THREADS, 0, (cudaStream_t)stream>>>(
        UL, UR, flux, speed, B, plane, normal_y ? 1 : 0, make_consts(*p));
    return launch_result();
}

extern "C" int swe_primitive_f32(const float* U, int B, int H, int W, const swe_params* p, float* h,
                                 float* u, float* v, float* c, void* stream) {
    if (!U || !h || !u || !v || !c || !valid_params(p) || B < 1 || H < 1 || W < 1) return SWE_EARG;
    const long long plane = (long long)H * W;
    primitive_kernel<<<blocks_for(B * plane), OPS_THREADS, 0, (cudaStream_t)stream>>>(
        U, h, u, v, c, B, plane, make_consts(*p));
    return launch_result();
}

extern "C" int swe_limited_increment_f32(const float* q, int outer, int H, int W, int dim,
                                         double theta, float* out, void* stream) {
    if (!q || !out || outer < 1 || H < 1 || W < 1 || (dim != -1 && dim != -2)) return SWE_EARG;
    limited_increment_kernel<<<blocks_for((long long)outer * H * W), OPS_THREADS, 0,
                               (cudaStream_t)stream>>>(q, out, outer, H, W, dim == -1, (float)theta);
    return launch_result();
}

extern "C" int swe_minmod3_f32(const float* a, const float* b, const float* c, long long n,
                               float* out, void* stream) {
    if (!a || !b || !c || !out || n < 0) return SWE_EARG;
    if (n == 0) return SWE_OK;
    minmod3_kernel<<<blocks_for(n), OPS_THREADS, 0, (cudaStream_t)stream>>>(a, b, c, out, n);
    return launch_result();
}

extern "C" int swe_clean_and_limit_f32(const float* old, const float* cand, int B, int ny, int nx,
                                       const swe_params* p, float* out, void* stream) {
    if (!old || !cand || !out || !valid_params(p) || B < 1 || ny < 1 || nx < 1) return SWE_EARG;
    const long long plane = (long long)ny * nx;
    clean_kernel<<<blocks_for(B * plane), OPS_THREADS, 0, (cudaStream_t)stream>>>(
        old, cand, out, B, plane, p->positivity_limiter, make_consts(*p));
    return launch_result();
}

extern "C" int swe_friction_f32(const float* U, const float* n, int nB, int B, int ny, int nx,
                                float dt, int model, const swe_params* p, float* out, void* stream) {
    if (!U || !n || !out || !valid_params(p) || B < 1 || ny < 1 || nx < 1) return SWE_EARG;
    if (!batch_ok(nB, B) || (model != 0 && model != 1)) return SWE_EARG;
    const long long plane = (long long)ny * nx;
    friction_kernel<<<blocks_for(B * plane), OPS_THREADS, 0, (cudaStream_t)stream>>>(
        U, n, nB, out, B, plane, dt, model, make_consts(*p));
    return launch_result();
}
