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
//     minmod3 is max(min(a,b,c), min(max(a,b,c), 0)), the positivity
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

#include "swe_approx.cuh"
#include "swe_ensemble.cuh"
#include "swe_sweep.cuh"

namespace swe {
namespace {

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
// differences: 0.5 minmod3(theta b, (b+f)/2, theta f).  minmod3 of values
// whose minimum is lo and maximum hi is max(lo, min(hi, 0)).
__device__ __forceinline__ float half_inc(float b, float f, const FK& k) {
    const float x = k.ht * b, y = k.ht * f, c = 0.25f * (b + f);
    // the median of (min, 0, max): the minimum if all three are positive,
    // the maximum if all are negative, else 0
    return fmaxf(min3f(x, c, y), fminf(max3f(x, c, y), 0.0f));
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
    // primitive() of the face states: (h u)/max(h, floor) is u min(h/floor, 1)
    // on wet states and 0 on dry ones -- a mask multiplied in (1 or 0, with
    // the floor's factor when the floor exceeds the dry depth)
    const bool wL = hL > k.dry, wR = hR > k.dry;
    const float wmL = wL ? 1.0f : 0.0f, wmR = wR ? 1.0f : 0.0f;
    float mL = wmL, mR = wmR;
    if (k.floor_above_dry) {
        mL *= fminf(hL * k.rfloor, 1.0f);
        mR *= fminf(hR * k.rfloor, 1.0f);
    }
    const float unL = (NY ? L.v : L.u) * mL;
    const float utL = (NY ? L.u : L.v) * mL;
    const float unR = (NY ? R.v : R.u) * mR;
    const float utR = (NY ? R.u : R.v) * mR;
    const float cL = sqrta(k.g * fmaxf(hL, k.floor_h)) * wmL;
    const float cR = sqrta(k.g * fmaxf(hR, k.floor_h)) * wmR;
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
                            if (a.k2_out != nullptr) {
                                a.k2_out[oo] = r0;
                                a.k2_out[oo + plane] = r1;
                                a.k2_out[oo + 2 * plane] = r2;
                            }
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

template <int STAGE, int FRIC>
__global__ void __launch_bounds__(SW_WARPS * 32, 8) fast_kernel(const StepArgs a) {
    chain_start();
    fast_tile<STAGE, FRIC, false>(a, blockIdx.x, blockIdx.y, blockIdx.z, a.rows);
}

struct FastTile {
    template <int STAGE, int FRIC>
    static __device__ __forceinline__ void run(const StepArgs& a, int bx, int by, int rows) {
        fast_tile<STAGE, FRIC, true>(a, bx, by, 0, rows);
    }
};

template <int FRIC>
__global__ void __launch_bounds__(SW_WARPS * 32, 6)
fast_ensemble_kernel(const StepArgs* __restrict__ args, EnsCtl* ctl, int count, EnsGlobal* g,
                     unsigned long long stall_ns) {
    ensemble_body<FRIC, FastTile>(args, ctl, count, g, stall_ns);
}

}  // namespace

int fast_launch_stages(int stage, const StepArgs& a, dim3 grid, cudaStream_t s) {
    const dim3 threads(SW_WARPS * 32);
    cudaError_t e = cudaSuccess;
    if (stage & 1) e = launch_chained(fast_kernel<1, 0>, grid, threads, s, a);
    if ((stage & 2) && e == cudaSuccess) {
        if (!a.friction) e = launch_chained(fast_kernel<2, 0>, grid, threads, s, a);
        else if (a.friction_model == 0) e = launch_chained(fast_kernel<2, 1>, grid, threads, s, a);
        else e = launch_chained(fast_kernel<2, 2>, grid, threads, s, a);
    }
    return e == cudaSuccess && cudaGetLastError() == cudaSuccess ? SWE_OK : SWE_ECUDA;
}

int fast_launch_ensemble(int friction, int blocks, const StepArgs* args, EnsCtl* ctl, int count,
                         EnsGlobal* g, unsigned long long stall_ns, cudaStream_t s) {
    const int threads = SW_WARPS * 32;
    if (friction == 0) fast_ensemble_kernel<0><<<blocks, threads, 0, s>>>(args, ctl, count, g, stall_ns);
    else if (friction == 1) fast_ensemble_kernel<1><<<blocks, threads, 0, s>>>(args, ctl, count, g, stall_ns);
    else fast_ensemble_kernel<2><<<blocks, threads, 0, s>>>(args, ctl, count, g, stall_ns);
    return cudaGetLastError() == cudaSuccess ? SWE_OK : SWE_ECUDA;
}

int fast_load_kernels() {
    cudaFuncAttributes at;
    const void* fns[] = {
        (const void*)fast_kernel<1, 0>,       (const void*)fast_kernel<2, 0>,
        (const void*)fast_kernel<2, 1>,       (const void*)fast_kernel<2, 2>,
        (const void*)fast_ensemble_kernel<0>, (const void*)fast_ensemble_kernel<1>,
        (const void*)fast_ensemble_kernel<2>,
    };
    for (const void* f : fns)
        if (cudaFuncGetAttributes(&at, f) != cudaSuccess) return SWE_ECUDA;
    return SWE_OK;
}

}  // namespace swe
