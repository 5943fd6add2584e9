// swe_fast.cu -- tolerance-mode FP32 step of the DiffSWE2d finite-volume
// solver on sm_100a (swe_params.arithmetic = SWE_ARITH_FAST).
//
// The same step as swe_step.cu (SWE2D.step, src/solver.py:572-663: two
// launches, stage 1 = tendency k1 and the global wave-speed maxima, stage 2
// = dt, predictor, k2, corrector, friction), the same launch shape (row
// sweep: one warp per 28-column strip, a register window sliding down the
// rows, x neighbours by shuffles) and the same ghost cells, but evaluated
// for speed within FP32 rounding of the reference instead of operation for
// operation:
//   * the file is compiled with -fmad=true -ftz=true: products and sums
//     contract to FMAs;
//   * quotients are products with the hardware reciprocal (rcp.approx), the
//     wave celerity uses sqrt.approx, h^(1/3) is ex2.approx(lg2.approx(h)/3);
//   * algebraic identities of the reference's expressions are used where
//     they save work: a face's velocity (h_cn u)/h_cn is u itself, the
//     limiter's centred difference is the sum of the two one-sided ones,
//     minmod3 is max(min(a,b,c), 0) + min(max(a,b,c), 0), the positivity
//     limiter scales the increment dt*k directly;
//   * the one-sided differences along y are carried from row to row, those
//     along x exchanged with one shuffle per field; the x-direction part of
//     a row's tendency is formed one row before the row is written.
// The time step, its status bits and the stage-1 non-finite check are
// computed as in the IEEE kernels.  The accuracy bar (tests/
// test_gpu_fast.py): after 1000 steps of the 256^2 island case and 200
// steps of the runup case, every field within 1.5x the reference's own
// FP32-vs-FP64 difference of the FP64 reference, identical wet/dry masks.
#include <cuda_runtime.h>
#include <stdlib.h>
#include <string.h>

#include "swe_ensemble.cuh"
#include "swe_sweep.cuh"

namespace swe {
namespace {

__device__ __forceinline__ float rcpa(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float sqrta(float x) {
    float y;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float ex2a(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float lg2a(float x) {
    float y;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
// Three-input minimum / maximum (sm_100).
__device__ __forceinline__ float min3f(float a, float b, float c) {
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}
__device__ __forceinline__ float max3f(float a, float b, float c) {
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

// Constants of the tolerance mode, derived from SweConsts in each thread.
struct FK {
    float g, half_g, dry, floor_h, rfloor, den_floor, ht, eps, rdx, rdy;
    bool floor_above_dry;  // floor_h > dry: a wet face's h_cn may be below floor_h
    bool clamp;            // theta > 16: the +-10 clamp of the velocity factor can act
};

__device__ __forceinline__ FK make_fk(const SweConsts& k) {
    FK f;
    f.g = k.g;
    f.half_g = k.half_g;
    f.dry = k.dry;
    f.floor_h = k.floor_h;
    f.rfloor = rcpa(k.floor_h);
    f.den_floor = k.den_floor;
    f.ht = 0.5f * k.theta;
    f.eps = k.eps;
    f.rdx = k.rdx;
    f.rdy = k.rdy;
    f.floor_above_dry = k.floor_h > k.dry;
    // |0.5 dh / h| <= theta/2 for non-negative depths, so the clamp of
    // reconstruction.py:90-91 only acts when theta/2 can reach 9.
    f.clamp = k.theta > 16.0f;
    return f;
}

// primitive() of a cell (riemann.py:20-38) with eta = h + z; rw is the
// reciprocal of the safe depth on wet cells and 0 on dry ones.
struct FPrim {
    float h, u, v, eta, z, rw;
};

__device__ __forceinline__ FPrim fprim(float U0, float U1, float U2, float z, const FK& k) {
    FPrim p;
    p.h = fmaxf(U0, 0.0f);
    const float r = rcpa(fmaxf(p.h, k.floor_h));
    p.rw = p.h > k.dry ? r : 0.0f;
    p.u = U1 * p.rw;
    p.v = U2 * p.rw;
    p.eta = p.h + z;
    p.z = z;
    return p;
}

// One-sided differences of h, eta, z, u, v between two neighbouring cells.
struct FDiff {
    float h, e, z, u, v;
};

__device__ __forceinline__ FDiff fdiff(const FPrim& hi, const FPrim& lo) {
    return FDiff{hi.h - lo.h, hi.eta - lo.eta, hi.z - lo.z, hi.u - lo.u, hi.v - lo.v};
}

// Half of limited_increment (numerics.py:4-27) from the backward and forward
// differences: 0.5 minmod3(theta b, (b+f)/2, theta f).
__device__ __forceinline__ float half_inc(float b, float f, const FK& k) {
    const float x = k.ht * b, y = k.ht * f, c = 0.25f * (b + f);
    return fmaxf(min3f(x, c, y), 0.0f) + fminf(max3f(x, c, y), 0.0f);
}

struct FSide {
    float hlin, eta, bed, u, v;
};
struct FSides {
    FSide p, m;  // p faces +direction (UL of face k+1/2), m faces -direction
};

// Face-side values of a cell in one direction (reconstruction.py:26-96).
__device__ __forceinline__ FSides fsides(const FPrim& c, const FDiff& b, const FDiff& f, const FK& k,
                                         bool wsr) {
    const float dh = half_inc(b.h, f.h, k);
    const float dz = half_inc(b.z, f.z, k);
    const float du = half_inc(b.u, f.u, k);
    const float dv = half_inc(b.v, f.v, k);
    float de = half_inc(b.e, f.e, k);
    if (wsr) {  // reconstruction.py:32-42 (base eta - h taken as z)
        const float half = de - dh;
        const bool reset = fabsf(de) > fabsf(dz) &&
                           (c.z - half > c.eta - b.e || c.z + half > c.eta + f.e);
        de = reset ? dh + dz : de;
    }
    const float q = dh * c.rw;  // 0.5 dh / safe_h on wet cells, 0 on dry ones
    float fl = 1.0f - q, fr = 1.0f + q;
    if (k.clamp) {  // reconstruction.py:90-91
        fl = fminf(fmaxf(fl, -10.0f), 10.0f);
        fr = fminf(fmaxf(fr, -10.0f), 10.0f);
    }
    FSides s;
    s.p.hlin = c.h + dh;
    s.m.hlin = c.h - dh;
    s.p.eta = c.eta + de;
    s.m.eta = c.eta - de;
    s.p.bed = c.z + dz;
    s.m.bed = c.z - dz;
    s.p.u = c.u + fl * du;
    s.p.v = c.v + fl * dv;
    s.m.u = c.u - fr * du;
    s.m.v = c.v - fr * dv;
    return s;
}

// One face: hydrostatic reconstruction (reconstruction.py:59-106), HLL flux
// (riemann.py:41-105) and the source split of spatial_operator
// (solver.py:503-509).  NY selects the y-direction conventions.
struct FFace {
    float fmass, fnorm_L, fnorm_R, ftan;
    uint32_t speed_bits;
};

template <bool NY>
__device__ __forceinline__ FFace fface(const FSide& L, float hLc, float zLc, const FSide& R, float hRc,
                                       float zRc, const FK& k) {
    const float bcn = min3f(fmaxf(L.bed, R.bed), L.eta, R.eta);
    const float hL = fmaxf(fminf(L.eta - bcn, L.hlin), 0.0f);
    const float hR = fmaxf(fminf(R.eta - bcn, R.hlin), 0.0f);
    const float srcL = k.half_g * (hLc + hL) * (zLc - bcn);
    const float srcR = k.half_g * (hR + hRc) * (zRc - bcn);
    // primitive() of the face states: (h u)/max(h, floor) is u when h >= floor
    const bool wL = hL > k.dry, wR = hR > k.dry;
    float sL = 1.0f, sR = 1.0f;
    if (k.floor_above_dry) {
        sL = fminf(hL * k.rfloor, 1.0f);
        sR = fminf(hR * k.rfloor, 1.0f);
    }
    const float unL = wL ? (NY ? L.v : L.u) * sL : 0.0f;
    const float utL = wL ? (NY ? L.u : L.v) * sL : 0.0f;
    const float unR = wR ? (NY ? R.v : R.u) * sR : 0.0f;
    const float utR = wR ? (NY ? R.u : R.v) * sR : 0.0f;
    const float cL = wL ? sqrta(k.g * fmaxf(hL, k.floor_h)) : 0.0f;
    const float cR = wR ? sqrta(k.g * fmaxf(hR, k.floor_h)) : 0.0f;
    const float us = 0.5f * (unL + unR) + cL - cR;
    const float cs = 0.5f * (cL + cR) + 0.25f * (unL - unR);
    const float SL = wL ? fminf(unL - cL, us - cs) : unR - 2.0f * cR;
    const float SR = wR ? fmaxf(unR + cR, us + cs) : unL + 2.0f * cL;
    const float fhL = hL * unL, fhR = hR * unR;
    const float fqL = fhL * unL + k.half_g * hL * hL;
    const float fqR = fhR * unR + k.half_g * hR * hR;
    const float rden = rcpa(fmaxf(SR - SL, k.den_floor));
    const float SLSR = SL * SR;
    const float fhs = (SR * fhL - SL * fhR + SLSR * (hR - hL)) * rden;
    const float fqs = (SR * fqL - SL * fqR + SLSR * (fhR - fhL)) * rden;
    const bool lf = SL >= 0.0f, rf = SR <= 0.0f;
    const float fh = lf ? fhL : (rf ? fhR : fhs);
    float fq = lf ? fqL : (rf ? fqR : fqs);
    fq = (wL || wR) ? fq : 0.0f;  // both sides dry: zero flux (the others vanish by themselves)
    FFace F;
    F.fmass = fh;
    F.ftan = (fh > 0.0f ? utL : utR) * fh;
    F.fnorm_L = fq - srcL;
    F.fnorm_R = fq - srcR;
    F.speed_bits = max(f2u(SL) & 0x7fffffffu, f2u(SR) & 0x7fffffffu);
    return F;
}

// clean(o, o + s*k) (solver.py:547-570) given the increment's factor s and
// tendency k: the positivity limiter scales s, then depth >= 0 and dry
// cells lose their momentum.
__device__ __forceinline__ State fclean(const State& o, float k0, float k1, float k2, float s, float eps,
                                        float dry, int positivity) {
    float ts = s;
    if (positivity) {
        const float d0 = s * k0;
        const float th = fminf(o.h * rcpa(fmaxf(-d0, eps)), 1.0f);
        ts = d0 < 0.0f ? s * th : s;
    }
    State r;
    r.h = fmaxf(o.h + ts * k0, 0.0f);
    const bool wet = r.h > dry;
    r.hu = wet ? o.hu + ts * k1 : 0.0f;
    r.hv = wet ? o.hv + ts * k2 : 0.0f;
    return r;
}

struct FastPredict {
    static __device__ __forceinline__ State predict(const State& u, float k0, float k1, float k2,
                                                    float hdt, const SweConsts& k, int positivity) {
        return fclean(u, k0, k1, k2, hdt, k.eps, k.dry, positivity);
    }
};

// Semi-implicit friction (friction.py:12-38, :69-131) on a cleaned state
// (h >= 0, no momentum on dry cells).  FRIC 1: Manning, 2: roughness length.
template <int FRIC>
__device__ __forceinline__ State ffriction(State s, float n, float dt, const SweConsts& k) {
    const bool wet = s.h > k.dry;
    const float rs = rcpa(fmaxf(s.h, k.fr_vs));
    const float u = s.hu * rs, v = s.hv * rs;
    const float sp2 = u * u + v * v;
    const float speed = (wet && sp2 > 0.0f) ? sqrta(fmaxf(sp2, k.fr_e2)) : 0.0f;
    float cf;
    if (FRIC == 1) {  // 9.81 n^2 / h^(1/3), friction.py:62-66
        const float nn = fmaxf(n, 0.0f);
        cf = k.g981 * (nn * nn) * ex2a(-k.third * lg2a(fmaxf(s.h, k.fr_e)));
    } else {  // friction.py:41-59
        const float ratio = fmaxf(s.h, k.fr_e) * rcpa(fmaxf(n, k.fr_e));
        const float shallow = rcpa(fmaxf(0.46f * ratio, k.fr_e));
        const float rc = fmaxf(ratio, k.fr_e);
        const float lt = 2.5f * ((0.69314718f * lg2a(rc) - 1.0f) + rcpa(rc) * 1.359f);
        const float deep = rcpa(fmaxf(lt * lt, k.fr_e));
        cf = ratio < 2.71828182845904523536f ? shallow : deep;
    }
    const float fac = rcpa(1.0f + cf * speed * dt * rs);
    s.hu *= fac;  // 0 on dry cells already
    s.hv *= fac;
    return s;
}

// One tile of the sweep (SW_WARPS strips side by side, `rows` output rows)
// of batch member b.  At row iteration k the warp holds the primitives of
// rows k-1 and k, the y-differences between rows k-2 and k-1, the y-side
// and cell values of row k-2, the y-face above row k-2 and the x-part of
// row k-2's tendency; it forms row k-1's y-sides, the y-face between rows
// k-2 and k-1, writes row k-2, and forms row k-1's x-faces.
template <int STAGE, int FRIC, bool CG>
__device__ __forceinline__ void fast_tile(const StepArgs& a, int bx, int by, int b, int rows) {
    const SweConsts& kc = a.kc;
    const int lane = threadIdx.x & 31;
    const int strip = bx * SW_WARPS + (threadIdx.x >> 5);
    const int i0 = strip * SW_OUT;
    const int j0 = by * rows;
    if (i0 >= a.nx) return;  // whole warp
    const int ny = a.ny, nx = a.nx;
    const int c = i0 - 2 + lane;  // this lane's column
    const bool out_lane = lane >= 2 && lane < 2 + SW_OUT && c < nx;
    const int jend = min(j0 + rows, ny);
    const size_t plane = (size_t)ny * nx;

    if (a.clk != nullptr && !a.clk->active) {
        if (STAGE == 2 && out_lane)
            for (int j = j0; j < jend; ++j) {
                const size_t o = at3(b, 0, j, c, ny, nx);
                a.U_out[o] = a.U[o];
                a.U_out[o + plane] = a.U[o + plane];
                a.U_out[o + 2 * plane] = a.U[o + 2 * plane];
            }
        return;
    }
    float dt = 0.0f, hdt = 0.0f;
    if (STAGE == 2) {
        dt = stage2_dt<CG>(a, threadIdx.x == 0 && bx == 0 && by == 0 && b == 0);
        hdt = 0.5f * dt;
    }
    const FK k = make_fk(kc);
    const bool wsr = a.wsr != 0;
    const bool xin = i0 >= 2 && i0 + 29 < nx;  // every lane's column is interior
    const float* Ub = a.U + (size_t)b * 3 * plane;
    const float* Tb = a.tend + (size_t)b * 3 * plane;
    const float* Zb = a.bed + (a.bedB == 1 ? (size_t)0 : (size_t)b * plane);

    FPrim pB{}, pC{};        // rows k-1, k
    FDiff dA{};              // row k-1 minus row k-2
    FSide sA{};              // y-side "p" of row k-2
    float hA = 0.0f, zA = 0.0f;                   // row k-2 depth, bed
    float fyA0 = 0.0f, fyA1 = 0.0f, fyA2 = 0.0f;  // y-face above row k-2: mass, tangential, normal (R)
    float rxA0 = 0.0f, rxA1 = 0.0f, rxA2 = 0.0f;  // x-part of row k-2's tendency
    uint32_t axb = 0u, ayb = 0u;
    bool bad = false;
    for (int kk = j0 - 2, it = 0; kk < jend + 2; ++kk, ++it) {
        // ---- row kk: state (predictor on stage 2) and primitives
        float s0, s1, s2, z;
        if (xin && (unsigned)kk < (unsigned)ny) {
            const size_t o = (size_t)kk * nx + c;
            const State u{ld_state<CG>(Ub + o), ld_state<CG>(Ub + o + plane), ld_state<CG>(Ub + o + 2 * plane)};
            z = Zb[o];
            if (STAGE == 1) {
                s0 = u.h;
                s1 = u.hu;
                s2 = u.hv;
                bad |= (__fsub_rn(u.h, u.h) + __fsub_rn(u.hu, u.hu) + __fsub_rn(u.hv, u.hv)) != 0.0f;
            } else {
                const State p = fclean(u, ld_state<CG>(Tb + o), ld_state<CG>(Tb + o + plane),
                                       ld_state<CG>(Tb + o + 2 * plane), hdt, k.eps, k.dry, a.positivity);
                s0 = p.h;
                s1 = p.hu;
                s2 = p.hv;
            }
        } else {
            State s, ur;
            sweep_cell<STAGE, CG, FastPredict>(a, b, kk, c, hdt, s, z, ur);
            s0 = s.h;
            s1 = s.hu;
            s2 = s.hv;
            if (STAGE == 1 && (unsigned)kk < (unsigned)ny && (unsigned)c < (unsigned)nx)
                bad |= (__fsub_rn(s0, s0) + __fsub_rn(s1, s1) + __fsub_rn(s2, s2)) != 0.0f;
        }
        pC = fprim(s0, s1, s2, z, k);
        const FDiff dB = fdiff(pC, pB);  // row kk minus row kk-1
        if (it >= 2) {
            // ---- y-sides of row kk-1
            const FSides sy = fsides(pB, dA, dB, k, wsr);
            if (it >= 3) {
                // ---- y-face between rows kk-2 and kk-1
                const FFace fy = fface<true>(sA, hA, zA, sy.m, pB.h, pB.z, k);
                if (STAGE == 1 && out_lane && kk - 1 >= 0 && kk - 1 <= ny) ayb = max(ayb, fy.speed_bits);
                if (it >= 4) {
                    // ---- row o = kk-2 is complete
                    const int o = kk - 2;
                    if (out_lane) {
                        float r0 = rxA0 + (fyA0 - fy.fmass) * k.rdy;
                        const float r1 = rxA1 + (fyA1 - fy.ftan) * k.rdy;
                        const float r2 = rxA2 + (fyA2 - fy.fnorm_L) * k.rdy;
                        if (a.rain_mode != SWE_FORCING_NONE)
                            r0 += forcing(a.rain, a.rain_mode, a.rain_batch, b, o, c, ny, nx);
                        if (a.infil_mode != SWE_FORCING_NONE)
                            r0 -= fmaxf(forcing(a.infil, a.infil_mode, a.infil_batch, b, o, c, ny, nx), 0.0f);
                        const size_t oo = at3(b, 0, o, c, ny, nx);
                        if (STAGE == 1) {
                            a.tend[oo] = r0;
                            a.tend[oo + plane] = r1;
                            a.tend[oo + 2 * plane] = r2;
                        } else {
                            const State u{ld_state<CG>(a.U + oo), ld_state<CG>(a.U + oo + plane),
                                          ld_state<CG>(a.U + oo + 2 * plane)};
                            State upd = fclean(u, r0, r1, r2, dt, k.eps, k.dry, a.positivity);
                            if (FRIC != 0)
                                upd = ffriction<FRIC>(upd, a.n[at1(a.nB == 1 ? 0 : b, o, c, ny, nx)], dt, kc);
                            a.U_out[oo] = upd.h;
                            a.U_out[oo + plane] = upd.hu;
                            a.U_out[oo + 2 * plane] = upd.hv;
                            if (a.hmax != nullptr) {  // torch.maximum(hmax, U[:, 0]), NaN-propagating
                                float* mp = a.hmax + at1(b, o, c, ny, nx);
                                const float m = ld_state<CG>(mp);
                                *mp = (upd.h > m || upd.h != upd.h) ? upd.h : m;
                            }
                        }
                    }
                }
                fyA0 = fy.fmass;
                fyA1 = fy.ftan;
                fyA2 = fy.fnorm_R;
                // ---- x-faces of row kk-1 (an output row for it <= rows + 2)
                if (kk - 1 < jend) {
                    const float hr = shfl_dn1(pB.h), er = shfl_dn1(pB.eta), zr = shfl_dn1(pB.z);
                    const float ur = shfl_dn1(pB.u), vr = shfl_dn1(pB.v);
                    const FDiff fx{hr - pB.h, er - pB.eta, zr - pB.z, ur - pB.u, vr - pB.v};
                    const FDiff bx_{shfl_up1(fx.h), shfl_up1(fx.e), shfl_up1(fx.z), shfl_up1(fx.u),
                                    shfl_up1(fx.v)};
                    const FSides sx = fsides(pB, bx_, fx, k, wsr);
                    const FSide rm{shfl_dn1(sx.m.hlin), shfl_dn1(sx.m.eta), shfl_dn1(sx.m.bed),
                                   shfl_dn1(sx.m.u), shfl_dn1(sx.m.v)};
                    const FFace fx_ = fface<false>(sx.p, pB.h, pB.z, rm, hr, zr, k);
                    if (STAGE == 1 && lane >= 1 && lane < 2 + SW_OUT && c >= -1 && c < nx)
                        axb = max(axb, fx_.speed_bits);
                    const float lm = shfl_up1(fx_.fmass), ln = shfl_up1(fx_.fnorm_R), lt = shfl_up1(fx_.ftan);
                    rxA0 = (lm - fx_.fmass) * k.rdx;
                    rxA1 = (ln - fx_.fnorm_L) * k.rdx;
                    rxA2 = (lt - fx_.ftan) * k.rdx;
                }
            }
            sA = sy.p;
            hA = pB.h;
            zA = pB.z;
        }
        pB = pC;
        dA = dB;
    }
    if (STAGE == 1) {
        axb = warp_max_u32(axb);
        ayb = warp_max_u32(ayb);
        if (lane == 0) {
            if (axb) atomicMax(&a.red[0], axb);
            if (ayb) atomicMax(&a.red[1], ayb);
        }
        if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(&a.red[2], SWE_S_NONFINITE_STATE);
    }
}

// ---------------------------------------------------------------------------
// Paired form of the tile: the x- and y-direction face sides of a row, and
// its x-face and the y-face above it, are evaluated together as float2
// pairs (x, y) with sm_100's two-wide FP32 add / multiply / fused
// multiply-add (one instruction for both directions); minima, maxima and
// selections stay per component.
__device__ __forceinline__ float2 f2(float x, float y) { return make_float2(x, y); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, f2(-1.0f, -1.0f), a); }
__device__ __forceinline__ float2 splat(float s) { return f2(s, s); }

// half_inc for both directions.
__device__ __forceinline__ float2 half_inc2(float2 b, float2 f, const FK& k) {
    const float2 x = mul2(splat(k.ht), b), y = mul2(splat(k.ht), f);
    const float2 c = fma2(b, splat(0.25f), mul2(f, splat(0.25f)));
    return add2(f2(fmaxf(min3f(x.x, c.x, y.x), 0.0f), fmaxf(min3f(x.y, c.y, y.y), 0.0f)),
                f2(fminf(max3f(x.x, c.x, y.x), 0.0f), fminf(max3f(x.y, c.y, y.y), 0.0f)));
}

struct FSide2 {
    float2 hlin, eta, bed, u, v;
};
struct FSides2 {
    FSide2 p, m;
};

// fsides for both directions of cell c: b, f hold the backward / forward
// differences as (x, y) pairs.
__device__ __forceinline__ FSides2 fsides2(const FPrim& c, const float2 (&b)[5], const float2 (&f)[5],
                                           const FK& k, bool wsr) {
    const float2 dh = half_inc2(b[0], f[0], k);
    const float2 dz = half_inc2(b[2], f[2], k);
    const float2 du = half_inc2(b[3], f[3], k);
    const float2 dv = half_inc2(b[4], f[4], k);
    float2 de = half_inc2(b[1], f[1], k);
    const float2 eta = splat(c.eta), z = splat(c.z), h = splat(c.h);
    if (wsr) {
        const float2 half = sub2(de, dh);
        const float2 bm = sub2(z, half), bp = add2(z, half);
        const float2 ea = sub2(eta, b[1]), eb = add2(eta, f[1]);
        const float2 alt = add2(dh, dz);
        de.x = (fabsf(de.x) > fabsf(dz.x) && (bm.x > ea.x || bp.x > eb.x)) ? alt.x : de.x;
        de.y = (fabsf(de.y) > fabsf(dz.y) && (bm.y > ea.y || bp.y > eb.y)) ? alt.y : de.y;
    }
    const float2 q = mul2(dh, splat(c.rw));
    float2 fl = sub2(splat(1.0f), q), fr = add2(splat(1.0f), q);
    if (k.clamp) {
        fl = f2(fminf(fmaxf(fl.x, -10.0f), 10.0f), fminf(fmaxf(fl.y, -10.0f), 10.0f));
        fr = f2(fminf(fmaxf(fr.x, -10.0f), 10.0f), fminf(fmaxf(fr.y, -10.0f), 10.0f));
    }
    FSides2 s;
    s.p.hlin = add2(h, dh);
    s.m.hlin = sub2(h, dh);
    s.p.eta = add2(eta, de);
    s.m.eta = sub2(eta, de);
    s.p.bed = add2(z, dz);
    s.m.bed = sub2(z, dz);
    s.p.u = fma2(fl, du, splat(c.u));
    s.p.v = fma2(fl, dv, splat(c.v));
    s.m.u = fma2(f2(-fr.x, -fr.y), du, splat(c.u));
    s.m.v = fma2(f2(-fr.x, -fr.y), dv, splat(c.v));
    return s;
}

struct FFace2 {
    float2 fmass, fnorm_L, fnorm_R, ftan;
    uint32_t speed_x, speed_y;
};

// The x-face (component x: L = this cell's +x side, R = the right neighbour's
// -x side) and the y-face (component y: L = the row above's +y side, R = this
// cell's -y side) at once.
__device__ __forceinline__ FFace2 fface2(const FSide2& L, float2 hLc, float2 zLc, const FSide2& R,
                                         float2 hRc, float2 zRc, const FK& k) {
    const float2 bcn = f2(min3f(fmaxf(L.bed.x, R.bed.x), L.eta.x, R.eta.x),
                          min3f(fmaxf(L.bed.y, R.bed.y), L.eta.y, R.eta.y));
    const float2 eL = sub2(L.eta, bcn), eR = sub2(R.eta, bcn);
    const float2 hL = f2(fmaxf(fminf(eL.x, L.hlin.x), 0.0f), fmaxf(fminf(eL.y, L.hlin.y), 0.0f));
    const float2 hR = f2(fmaxf(fminf(eR.x, R.hlin.x), 0.0f), fmaxf(fminf(eR.y, R.hlin.y), 0.0f));
    const float2 hg = splat(k.half_g);
    const float2 srcL = mul2(mul2(hg, add2(hLc, hL)), sub2(zLc, bcn));
    const float2 srcR = mul2(mul2(hg, add2(hR, hRc)), sub2(zRc, bcn));
    const bool wLx = hL.x > k.dry, wLy = hL.y > k.dry, wRx = hR.x > k.dry, wRy = hR.y > k.dry;
    float2 sL = splat(1.0f), sR = splat(1.0f);
    if (k.floor_above_dry) {
        sL = f2(fminf(hL.x * k.rfloor, 1.0f), fminf(hL.y * k.rfloor, 1.0f));
        sR = f2(fminf(hR.x * k.rfloor, 1.0f), fminf(hR.y * k.rfloor, 1.0f));
    }
    // normal velocity: u across x-faces, v across y-faces
    const float2 mL = f2(wLx ? sL.x : 0.0f, wLy ? sL.y : 0.0f);
    const float2 mR = f2(wRx ? sR.x : 0.0f, wRy ? sR.y : 0.0f);
    const float2 unL = mul2(f2(L.u.x, L.v.y), mL), utL = mul2(f2(L.v.x, L.u.y), mL);
    const float2 unR = mul2(f2(R.u.x, R.v.y), mR), utR = mul2(f2(R.v.x, R.u.y), mR);
    const float2 gL = mul2(splat(k.g), f2(fmaxf(hL.x, k.floor_h), fmaxf(hL.y, k.floor_h)));
    const float2 gR = mul2(splat(k.g), f2(fmaxf(hR.x, k.floor_h), fmaxf(hR.y, k.floor_h)));
    const float2 cL = f2(wLx ? sqrta(gL.x) : 0.0f, wLy ? sqrta(gL.y) : 0.0f);
    const float2 cR = f2(wRx ? sqrta(gR.x) : 0.0f, wRy ? sqrta(gR.y) : 0.0f);
    const float2 us = sub2(fma2(splat(0.5f), add2(unL, unR), cL), cR);
    const float2 cs = fma2(splat(0.25f), sub2(unL, unR), mul2(splat(0.5f), add2(cL, cR)));
    const float2 a1 = sub2(unL, cL), a2 = sub2(us, cs), a3 = fma2(splat(-2.0f), cR, unR);
    const float2 b1 = add2(unR, cR), b2 = add2(us, cs), b3 = fma2(splat(2.0f), cL, unL);
    const float2 SL = f2(wLx ? fminf(a1.x, a2.x) : a3.x, wLy ? fminf(a1.y, a2.y) : a3.y);
    const float2 SR = f2(wRx ? fmaxf(b1.x, b2.x) : b3.x, wRy ? fmaxf(b1.y, b2.y) : b3.y);
    const float2 fhL = mul2(hL, unL), fhR = mul2(hR, unR);
    const float2 fqL = fma2(fhL, unL, mul2(mul2(hg, hL), hL));
    const float2 fqR = fma2(fhR, unR, mul2(mul2(hg, hR), hR));
    const float2 den = sub2(SR, SL);
    const float2 rden = f2(rcpa(fmaxf(den.x, k.den_floor)), rcpa(fmaxf(den.y, k.den_floor)));
    const float2 SLSR = mul2(SL, SR);
    const float2 fhs = mul2(fma2(SLSR, sub2(hR, hL), sub2(mul2(SR, fhL), mul2(SL, fhR))), rden);
    const float2 fqs = mul2(fma2(SLSR, sub2(fhR, fhL), sub2(mul2(SR, fqL), mul2(SL, fqR))), rden);
    float2 fh, fq;
    fh.x = SL.x >= 0.0f ? fhL.x : (SR.x <= 0.0f ? fhR.x : fhs.x);
    fh.y = SL.y >= 0.0f ? fhL.y : (SR.y <= 0.0f ? fhR.y : fhs.y);
    fq.x = SL.x >= 0.0f ? fqL.x : (SR.x <= 0.0f ? fqR.x : fqs.x);
    fq.y = SL.y >= 0.0f ? fqL.y : (SR.y <= 0.0f ? fqR.y : fqs.y);
    fq.x = (wLx || wRx) ? fq.x : 0.0f;
    fq.y = (wLy || wRy) ? fq.y : 0.0f;
    FFace2 F;
    F.fmass = fh;
    F.ftan = mul2(f2(fh.x > 0.0f ? utL.x : utR.x, fh.y > 0.0f ? utL.y : utR.y), fh);
    F.fnorm_L = sub2(fq, srcL);
    F.fnorm_R = sub2(fq, srcR);
    F.speed_x = max(f2u(SL.x) & 0x7fffffffu, f2u(SR.x) & 0x7fffffffu);
    F.speed_y = max(f2u(SL.y) & 0x7fffffffu, f2u(SR.y) & 0x7fffffffu);
    return F;
}

// The tile of fast_tile with the paired evaluation above.
template <int STAGE, int FRIC, bool CG>
__device__ __forceinline__ void fast_tile_x2(const StepArgs& a, int bx, int by, int b, int rows) {
    const SweConsts& kc = a.kc;
    const int lane = threadIdx.x & 31;
    const int strip = bx * SW_WARPS + (threadIdx.x >> 5);
    const int i0 = strip * SW_OUT;
    const int j0 = by * rows;
    if (i0 >= a.nx) return;  // whole warp
    const int ny = a.ny, nx = a.nx;
    const int c = i0 - 2 + lane;  // this lane's column
    const bool out_lane = lane >= 2 && lane < 2 + SW_OUT && c < nx;
    const int jend = min(j0 + rows, ny);
    const size_t plane = (size_t)ny * nx;

    if (a.clk != nullptr && !a.clk->active) {
        if (STAGE == 2 && out_lane)
            for (int j = j0; j < jend; ++j) {
                const size_t o = at3(b, 0, j, c, ny, nx);
                a.U_out[o] = a.U[o];
                a.U_out[o + plane] = a.U[o + plane];
                a.U_out[o + 2 * plane] = a.U[o + 2 * plane];
            }
        return;
    }
    float dt = 0.0f, hdt = 0.0f;
    if (STAGE == 2) {
        dt = stage2_dt<CG>(a, threadIdx.x == 0 && bx == 0 && by == 0 && b == 0);
        hdt = 0.5f * dt;
    }
    const FK k = make_fk(kc);
    const bool wsr = a.wsr != 0;
    const bool xin = i0 >= 2 && i0 + 29 < nx;  // every lane's column is interior
    const float* Ub = a.U + (size_t)b * 3 * plane;
    const float* Tb = a.tend + (size_t)b * 3 * plane;
    const float* Zb = a.bed + (a.bedB == 1 ? (size_t)0 : (size_t)b * plane);

    FPrim pB{}, pC{};        // rows k-1, k
    FDiff dA{};              // row k-1 minus row k-2
    FSide sA{};              // y-side "p" of row k-2
    float hA = 0.0f, zA = 0.0f;                   // row k-2 depth, bed
    float fyA0 = 0.0f, fyA1 = 0.0f, fyA2 = 0.0f;  // y-face above row k-2: mass, tangential, normal (R)
    float rxA0 = 0.0f, rxA1 = 0.0f, rxA2 = 0.0f;  // x-part of row k-2's tendency
    uint32_t axb = 0u, ayb = 0u;
    bool bad = false;
    for (int kk = j0 - 2, it = 0; kk < jend + 2; ++kk, ++it) {
        // ---- row kk: state (predictor on stage 2) and primitives
        float s0, s1, s2, z;
        if (xin && (unsigned)kk < (unsigned)ny) {
            const size_t o = (size_t)kk * nx + c;
            const State u{ld_state<CG>(Ub + o), ld_state<CG>(Ub + o + plane), ld_state<CG>(Ub + o + 2 * plane)};
            z = Zb[o];
            if (STAGE == 1) {
                s0 = u.h;
                s1 = u.hu;
                s2 = u.hv;
                bad |= (__fsub_rn(u.h, u.h) + __fsub_rn(u.hu, u.hu) + __fsub_rn(u.hv, u.hv)) != 0.0f;
            } else {
                const State p = fclean(u, ld_state<CG>(Tb + o), ld_state<CG>(Tb + o + plane),
                                       ld_state<CG>(Tb + o + 2 * plane), hdt, k.eps, k.dry, a.positivity);
                s0 = p.h;
                s1 = p.hu;
                s2 = p.hv;
            }
        } else {
            State s, ur;
            sweep_cell<STAGE, CG, FastPredict>(a, b, kk, c, hdt, s, z, ur);
            s0 = s.h;
            s1 = s.hu;
            s2 = s.hv;
            if (STAGE == 1 && (unsigned)kk < (unsigned)ny && (unsigned)c < (unsigned)nx)
                bad |= (__fsub_rn(s0, s0) + __fsub_rn(s1, s1) + __fsub_rn(s2, s2)) != 0.0f;
        }
        pC = fprim(s0, s1, s2, z, k);
        const FDiff dB = fdiff(pC, pB);  // row kk minus row kk-1
        if (it >= 2) {
            // ---- both directions' sides of row kk-1: x differences by shuffles
            const float hr = shfl_dn1(pB.h), er = shfl_dn1(pB.eta), zr = shfl_dn1(pB.z);
            const float ur = shfl_dn1(pB.u), vr = shfl_dn1(pB.v);
            const FDiff fx{hr - pB.h, er - pB.eta, zr - pB.z, ur - pB.u, vr - pB.v};
            const float2 Bk[5] = {f2(shfl_up1(fx.h), dA.h), f2(shfl_up1(fx.e), dA.e),
                                  f2(shfl_up1(fx.z), dA.z), f2(shfl_up1(fx.u), dA.u),
                                  f2(shfl_up1(fx.v), dA.v)};
            const float2 Fw[5] = {f2(fx.h, dB.h), f2(fx.e, dB.e), f2(fx.z, dB.z), f2(fx.u, dB.u),
                                  f2(fx.v, dB.v)};
            const FSides2 sd = fsides2(pB, Bk, Fw, k, wsr);
            if (it >= 3) {
                // ---- x-face of row kk-1 and the y-face between rows kk-2 and kk-1
                const FSide2 L{f2(sd.p.hlin.x, sA.hlin), f2(sd.p.eta.x, sA.eta), f2(sd.p.bed.x, sA.bed),
                               f2(sd.p.u.x, sA.u), f2(sd.p.v.x, sA.v)};
                const FSide2 R{f2(shfl_dn1(sd.m.hlin.x), sd.m.hlin.y), f2(shfl_dn1(sd.m.eta.x), sd.m.eta.y),
                               f2(shfl_dn1(sd.m.bed.x), sd.m.bed.y), f2(shfl_dn1(sd.m.u.x), sd.m.u.y),
                               f2(shfl_dn1(sd.m.v.x), sd.m.v.y)};
                const FFace2 F = fface2(L, f2(pB.h, hA), f2(pB.z, zA), R, f2(hr, pB.h), f2(zr, pB.z), k);
                if (STAGE == 1 && out_lane && kk - 1 >= 0 && kk - 1 <= ny) ayb = max(ayb, F.speed_y);
                if (it >= 4) {
                    // ---- row o = kk-2 is complete
                    const int o = kk - 2;
                    if (out_lane) {
                        float r0 = rxA0 + (fyA0 - F.fmass.y) * k.rdy;
                        const float r1 = rxA1 + (fyA1 - F.ftan.y) * k.rdy;
                        const float r2 = rxA2 + (fyA2 - F.fnorm_L.y) * k.rdy;
                        if (a.rain_mode != SWE_FORCING_NONE)
                            r0 += forcing(a.rain, a.rain_mode, a.rain_batch, b, o, c, ny, nx);
                        if (a.infil_mode != SWE_FORCING_NONE)
                            r0 -= fmaxf(forcing(a.infil, a.infil_mode, a.infil_batch, b, o, c, ny, nx), 0.0f);
                        const size_t oo = at3(b, 0, o, c, ny, nx);
                        if (STAGE == 1) {
                            a.tend[oo] = r0;
                            a.tend[oo + plane] = r1;
                            a.tend[oo + 2 * plane] = r2;
                        } else {
                            const State u{ld_state<CG>(a.U + oo), ld_state<CG>(a.U + oo + plane),
                                          ld_state<CG>(a.U + oo + 2 * plane)};
                            State upd = fclean(u, r0, r1, r2, dt, k.eps, k.dry, a.positivity);
                            if (FRIC != 0)
                                upd = ffriction<FRIC>(upd, a.n[at1(a.nB == 1 ? 0 : b, o, c, ny, nx)], dt, kc);
                            a.U_out[oo] = upd.h;
                            a.U_out[oo + plane] = upd.hu;
                            a.U_out[oo + 2 * plane] = upd.hv;
                            if (a.hmax != nullptr) {  // torch.maximum(hmax, U[:, 0]), NaN-propagating
                                float* mp = a.hmax + at1(b, o, c, ny, nx);
                                const float m = ld_state<CG>(mp);
                                *mp = (upd.h > m || upd.h != upd.h) ? upd.h : m;
                            }
                        }
                    }
                }
                fyA0 = F.fmass.y;
                fyA1 = F.ftan.y;
                fyA2 = F.fnorm_R.y;
                if (kk - 1 < jend) {  // row kk-1 is an output row: keep its x-part
                    if (STAGE == 1 && lane >= 1 && lane < 2 + SW_OUT && c >= -1 && c < nx)
                        axb = max(axb, F.speed_x);
                    const float lm = shfl_up1(F.fmass.x), ln = shfl_up1(F.fnorm_R.x);
                    const float lt = shfl_up1(F.ftan.x);
                    rxA0 = (lm - F.fmass.x) * k.rdx;
                    rxA1 = (ln - F.fnorm_L.x) * k.rdx;
                    rxA2 = (lt - F.ftan.x) * k.rdx;
                }
            }
            sA = FSide{sd.p.hlin.y, sd.p.eta.y, sd.p.bed.y, sd.p.u.y, sd.p.v.y};
            hA = pB.h;
            zA = pB.z;
        }
        pB = pC;
        dA = dB;
    }
    if (STAGE == 1) {
        axb = warp_max_u32(axb);
        ayb = warp_max_u32(ayb);
        if (lane == 0) {
            if (axb) atomicMax(&a.red[0], axb);
            if (ayb) atomicMax(&a.red[1], ayb);
        }
        if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(&a.red[2], SWE_S_NONFINITE_STATE);
    }
}

template <int STAGE, int FRIC, bool X2>
__global__ void __launch_bounds__(SW_WARPS * 32, 8) fast_kernel(const StepArgs a) {
    if (X2) fast_tile_x2<STAGE, FRIC, false>(a, blockIdx.x, blockIdx.y, blockIdx.z, a.rows);
    else fast_tile<STAGE, FRIC, false>(a, blockIdx.x, blockIdx.y, blockIdx.z, a.rows);
}

template <bool X2>
struct FastTile {
    template <int STAGE, int FRIC>
    static __device__ __forceinline__ void run(const StepArgs& a, int bx, int by, int rows) {
        if (X2) fast_tile_x2<STAGE, FRIC, true>(a, bx, by, 0, rows);
        else fast_tile<STAGE, FRIC, true>(a, bx, by, 0, rows);
    }
};

template <int FRIC, bool X2>
__global__ void __launch_bounds__(SW_WARPS * 32, 6)
fast_ensemble_kernel(const StepArgs* __restrict__ args, EnsCtl* ctl, int count, EnsGlobal* g,
                     unsigned long long stall_ns) {
    ensemble_body<FRIC, FastTile<X2>>(args, ctl, count, g, stall_ns);
}

}  // namespace

namespace {

// Tile form of the single-grid tolerance-mode kernels: the paired form
// unless SWE_FAST_TILE=scalar (read once per process).
bool use_paired_tile() {
    static const bool paired = [] {
        const char* v = getenv("SWE_FAST_TILE");
        return !(v != nullptr && strcmp(v, "scalar") == 0);
    }();
    return paired;
}

template <bool X2>
void launch_fast(int stage, const StepArgs& a, dim3 grid, cudaStream_t s) {
    const int threads = SW_WARPS * 32;
    if (stage & 1) fast_kernel<1, 0, X2><<<grid, threads, 0, s>>>(a);
    if (stage & 2) {
        if (!a.friction) fast_kernel<2, 0, X2><<<grid, threads, 0, s>>>(a);
        else if (a.friction_model == 0) fast_kernel<2, 1, X2><<<grid, threads, 0, s>>>(a);
        else fast_kernel<2, 2, X2><<<grid, threads, 0, s>>>(a);
    }
}

}  // namespace

int fast_launch_stages(int stage, const StepArgs& a, dim3 grid, cudaStream_t s) {
    if (use_paired_tile()) launch_fast<true>(stage, a, grid, s);
    else launch_fast<false>(stage, a, grid, s);
    return cudaGetLastError() == cudaSuccess ? SWE_OK : SWE_ECUDA;
}

namespace {
template <bool X2>
void launch_fast_ensemble(int friction, int blocks, const StepArgs* args, EnsCtl* ctl, int count,
                          EnsGlobal* g, unsigned long long stall_ns, cudaStream_t s) {
    const int threads = SW_WARPS * 32;
    if (friction == 0)
        fast_ensemble_kernel<0, X2><<<blocks, threads, 0, s>>>(args, ctl, count, g, stall_ns);
    else if (friction == 1)
        fast_ensemble_kernel<1, X2><<<blocks, threads, 0, s>>>(args, ctl, count, g, stall_ns);
    else
        fast_ensemble_kernel<2, X2><<<blocks, threads, 0, s>>>(args, ctl, count, g, stall_ns);
}
}  // namespace

// The ensemble uses the same tile form as the single-grid kernels, so a
// member's result equals the single-grid step's bit for bit.
int fast_launch_ensemble(int friction, int blocks, const StepArgs* args, EnsCtl* ctl, int count,
                         EnsGlobal* g, unsigned long long stall_ns, cudaStream_t s) {
    if (use_paired_tile()) launch_fast_ensemble<true>(friction, blocks, args, ctl, count, g, stall_ns, s);
    else launch_fast_ensemble<false>(friction, blocks, args, ctl, count, g, stall_ns, s);
    return cudaGetLastError() == cudaSuccess ? SWE_OK : SWE_ECUDA;
}

int fast_load_kernels() {
    cudaFuncAttributes at;
    const void* fns[] = {
        (const void*)fast_kernel<1, 0, false>, (const void*)fast_kernel<2, 0, false>,
        (const void*)fast_kernel<2, 1, false>, (const void*)fast_kernel<2, 2, false>,
        (const void*)fast_kernel<1, 0, true>,  (const void*)fast_kernel<2, 0, true>,
        (const void*)fast_kernel<2, 1, true>,  (const void*)fast_kernel<2, 2, true>,
        (const void*)fast_ensemble_kernel<0, false>, (const void*)fast_ensemble_kernel<1, false>,
        (const void*)fast_ensemble_kernel<2, false>, (const void*)fast_ensemble_kernel<0, true>,
        (const void*)fast_ensemble_kernel<1, true>,  (const void*)fast_ensemble_kernel<2, true>,
    };
    for (const void* f : fns)
        if (cudaFuncGetAttributes(&at, f) != cudaSuccess) return SWE_ECUDA;
    return SWE_OK;
}

}  // namespace swe
