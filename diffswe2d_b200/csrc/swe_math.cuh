// swe_math.cuh -- FP32 arithmetic of the DiffSWE2d finite-volume step.
//
// Every function evaluates the same expression tree, in the same order and
// with the same rounding points, as the PyTorch code it cites (paths are
// relative to the DiffSWE2d project).  The file is compiled with
// -fmad=false -prec-div=true -prec-sqrt=true -ftz=false, so each +,-,*,/
// and sqrt is one IEEE correctly-rounded operation: the results are those of
// the reference's float32 tensors op for op.
//
// Python scalars that the reference multiplies into float32 tensors are
// rounded to float32 first (PyTorch casts a wrapped scalar to the tensor's
// dtype); they arrive pre-rounded in SweConsts.
#pragma once

#include <math.h>
#include <stdint.h>

#if defined(__CUDACC__)
#define SWE_HD __host__ __device__ __forceinline__
#else
#define SWE_HD inline
#endif

namespace swe {

// Constants of one configuration, rounded to float32 as the reference rounds
// them at each use.
struct SweConsts {
    float g;          // float(gravity)                  riemann.py:36, :76
    float half_g;     // 0.5 * gravity                    reconstruction.py:101, riemann.py:76
    float dry;        // dry_depth                        riemann.py:29
    float floor_h;    // max(eps, dry, 1e-6)              riemann.py:6-11, reconstruction.py:12-15
    float den_floor;  // max(eps, 1e-6)                   riemann.py:14-17
    float theta;      // limiter_theta                    numerics.py:27
    float eps;        // epsilon                          solver.py:552, :621
    float cfl;        // cfl                              solver.py:623
    float dx, dy;     // grid spacing                     solver.py:514, :518
    float fr_vs;      // friction _floor(h, eps, dry)     friction.py:17
    float fr_e;       // friction _floor(h, eps)          friction.py:63
    float fr_e2;      // _floor(h, eps) ** 2              friction.py:27
    float third;      // 1.0 / 3.0                        friction.py:66
    float absorb_lim; // 1e-4                             boundary.py:325
    float absorb_min; // 1e-6                             boundary.py:326
    float g981;       // 9.81 (hard-coded)                friction.py:66, boundary.py:326
    float rdx, rdy;   // RN(1/dx), RN(1/dy) for the tendency's divisions
};

// ------------------------------------------------ correctly rounded division
// Quotients are IEEE correctly rounded, as the reference's float32 "/"
// is.  On the device several quotients that share a denominator b share one
// reciprocal y = RN(1/b): the hardware approximation rcp.approx refined by
// one Newton-Raphson step y1 = y0 + y0 (1 - b y0), then each quotient is
// q = RN(a y) corrected once with the exact FMA remainder r = a - q b,
// q' = RN(q + r y) (P. Markstein, "Computation of elementary functions on
// the IBM RISC System/6000 processor", IBM J. Res. Dev. 34(1), 1990).  The
// device self-test swe_selftest_arith_f32 checks rcp_cr against CUDA's
// rcp.rn for every float in the range used and div_by against div.rn on
// random and near-halfway operands, and on tiny numerators.  Quotients
// outside [2^-100, 2^100] or below 2^-125 (zero excepted) and non-finite
// operands take the IEEE division instead.
#if defined(__CUDA_ARCH__)
// IEEE fallbacks for operands outside the range the fast forms are checked
// for.  Out of line: one copy shared by every call site keeps the kernels'
// code small (the branch to them is almost never taken).
__device__ __noinline__ float ieee_div_slow(float a, float b) { return __fdiv_rn(a, b); }
__device__ __noinline__ float ieee_rcp_slow(float b) { return __frcp_rn(b); }
__device__ __noinline__ float ieee_sqrt_slow(float x) { return __fsqrt_rn(x); }
#endif

SWE_HD float rcp_cr(float b) {
#if defined(__CUDA_ARCH__)
    float y0;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y0) : "f"(b));
    const float e = __fmaf_rn(-b, y0, 1.0f);
    const float y1 = __fmaf_rn(y0, e, y0);
    const float ab = fabsf(b);
    return (ab >= 0x1p-100f && ab < 0x1p+100f) ? y1 : ieee_rcp_slow(b);
#else
    return 1.0f / b;
#endif
}

// a / b given y = rcp_cr(b).  The FMA remainder r = a - q b must not
// underflow, so a numerator below 2^-62 in magnitude (tiny and subnormal
// momenta are common where thin films drain under friction) is scaled by
// 2^64 first, exactly, and the quotient scaled back by 2^-64, exactly while
// it stays at least 2^-126: the range test on the scaled quotient (at least
// 2^-61) ensures that.  Subnormal quotients take the IEEE division.
SWE_HD float div_by(float a, float b, float y) {
#if defined(__CUDA_ARCH__)
    const bool tiny = fabsf(a) < 0x1p-62f;
    const float as = tiny ? __fmul_rn(a, 0x1p+64f) : a;
    const float q = __fmul_rn(as, y);
    const float r = __fmaf_rn(-q, b, as);
    const float q1 = __fmaf_rn(r, y, q);
    const float aq = fabsf(q);
    const bool safe = (aq >= (tiny ? 0x1p-61f : 0x1p-100f) && aq <= 0x1p+100f) || a == 0.0f;
    return safe ? (tiny ? __fmul_rn(q1, 0x1p-64f) : q1) : ieee_div_slow(a, b);
#else
    (void)y;
    return a / b;
#endif
}

// Correctly rounded square root for finite x > 0: s = x y and h = y/2 from
// the hardware approximation y ~ 1/sqrt(x) (rsqrt.approx), corrected once
// with the exact FMA remainder r = x - s s, s' = RN(s + r h) (Markstein's
// method for the square root, same reference).  Checked exhaustively
// against sqrt.rn over [2^-100, 2^100) by swe_selftest_arith_f32; other
// arguments take the IEEE square root.
SWE_HD float sqrt_cr(float x) {
#if defined(__CUDA_ARCH__)
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    const float s = __fmul_rn(x, y);
    const float h = __fmul_rn(0.5f, y);
    const float r = __fmaf_rn(-s, s, x);
    const float s1 = __fmaf_rn(r, h, s);
    const bool safe = x >= 0x1p-100f && x < 0x1p+100f;
    return safe ? s1 : ieee_sqrt_slow(x);
#else
    return sqrtf(x);
#endif
}

// The step's quotients, reciprocals and square roots.  With SWE_FAST_DIV the
// shared-reciprocal forms above are used, otherwise CUDA's IEEE operations;
// both give the same correctly-rounded values.
#ifndef SWE_FAST_DIV
#define SWE_FAST_DIV 1
#endif

// Reciprocal of a denominator shared by several quotients (unused when
// SWE_FAST_DIV is off).
SWE_HD float shared_rcp(float b) {
#if SWE_FAST_DIV
    return rcp_cr(b);
#else
    (void)b;
    return 0.0f;
#endif
}

// a / b with y = shared_rcp(b).
SWE_HD float quot(float a, float b, float y) {
#if SWE_FAST_DIV
    return div_by(a, b, y);
#else
    (void)y;
    return a / b;
#endif
}

// 1 / b (PyTorch's reciprocal()).
SWE_HD float recip(float b) {
#if SWE_FAST_DIV
    return rcp_cr(b);
#else
    return 1.0f / b;
#endif
}

SWE_HD float root(float x) {
#if SWE_FAST_DIV
    return sqrt_cr(x);
#else
    return sqrtf(x);
#endif
}

// ---------------------------------------------------------------- numerics
// minmod3, numerics.py:4-13.  With lo = min(a,b,c) and hi = max(a,b,c):
// all three positive <=> lo > 0, and then sign(a)*min|.| = lo exactly; all
// negative <=> hi < 0, and then the result is -min(-a,-b,-c) = hi exactly;
// any zero or mixed signs gives 0.
SWE_HD float minmod3(float a, float b, float c) {
    float lo = fminf(a, fminf(b, c));
    float hi = fmaxf(a, fmaxf(b, c));
    return lo > 0.0f ? lo : (hi < 0.0f ? hi : 0.0f);
}

// limited_increment, numerics.py:16-27, for a cell with neighbours qm, qp.
SWE_HD float limited_increment(float qm, float q, float qp, float theta) {
    float backward = q - qm;
    float centred = 0.5f * (qp - qm);
    float forward = qp - q;
    return minmod3(theta * backward, centred, theta * forward);
}

// Per-cell primitive values (riemann.py:20-38) plus eta = h + bed
// (reconstruction.py:23-24).
struct Prim {
    float h, u, v, eta, z;
};

SWE_HD Prim make_prim(float U0, float U1, float U2, float z, const SweConsts& k) {
    Prim p;
    p.h = fmaxf(U0, 0.0f);
    bool wet = p.h > k.dry;
    float safe = fmaxf(p.h, k.floor_h);
    float y = shared_rcp(safe);
    p.u = wet ? quot(U1, safe, y) : 0.0f;
    p.v = wet ? quot(U2, safe, y) : 0.0f;
    p.eta = p.h + z;
    p.z = z;
    return p;
}

// Face-side values a cell contributes to the two faces across it in one
// direction (reconstruction.py:26-96).  "p" is the side facing +direction
// (the left state UL of the face k+1/2), "m" the side facing -direction (the
// right state UR of the face k-1/2).
struct Side {
    float hlin;  // h +/- 0.5 dh
    float eta;   // eta +/- 0.5 deta
    float bed;   // z +/- 0.5 dz
    float u, v;  // u +/- 0.5 factor du
};

struct Sides {
    Side p, m;
    float h, z;  // cell depth and bed for the well-balanced sources
};

// c is the cell, a its neighbour in -direction, b in +direction.
SWE_HD Sides make_sides(const Prim& a, const Prim& c, const Prim& b, const SweConsts& k,
                        bool water_slope_reset) {
    float dh = limited_increment(a.h, c.h, b.h, k.theta);        // :26
    float deta = limited_increment(a.eta, c.eta, b.eta, k.theta); // :27
    float dz = limited_increment(a.z, c.z, b.z, k.theta);        // :28
    float du = limited_increment(a.u, c.u, b.u, k.theta);        // :29
    float dv = limited_increment(a.v, c.v, b.v, k.theta);        // :30
    if (water_slope_reset) {                                     // :32-42
        float half = 0.5f * (deta - dh);
        float base = c.eta - c.h;
        float bed_minus = base - half;
        float bed_plus = base + half;
        bool reset = (deta * deta > dz * dz) && ((bed_minus > a.eta) || (bed_plus > b.eta));
        if (reset) deta = dh + dz;
    }
    Sides s;
    float hdh = 0.5f * dh, hdeta = 0.5f * deta, hdz = 0.5f * dz;
    s.p.hlin = c.h + hdh;   // :50
    s.m.hlin = c.h - hdh;   // :51
    s.p.eta = c.eta + hdeta;  // :53
    s.m.eta = c.eta - hdeta;  // :54
    s.p.bed = c.z + hdz;    // :56
    s.m.bed = c.z - hdz;    // :57
    float safe = fmaxf(c.h, k.floor_h);  // :71-73
    float q = quot(hdh, safe, shared_rcp(safe));  // 0.5 * dh / safe_h, :75-76
    bool wet = c.h > k.dry;              // :78-87
    float fL = wet ? 1.0f - q : 1.0f;
    float fR = wet ? 1.0f + q : 1.0f;
    fL = fminf(fmaxf(fL, -10.0f), 10.0f);  // :90-91
    fR = fminf(fmaxf(fR, -10.0f), 10.0f);
    float hfL = 0.5f * fL, hfR = 0.5f * fR;
    s.p.u = c.u + hfL * du;  // :93-96
    s.p.v = c.v + hfL * dv;
    s.m.u = c.u - hfR * du;
    s.m.v = c.v - hfR * dv;
    s.h = c.h;
    s.z = c.z;
    return s;
}

// Result of one face: HLL flux (riemann.py:41-105) with the two
// well-balanced source terms (reconstruction.py:101-106) already folded into
// the normal-momentum channel as spatial_operator does (solver.py:503-509).
struct FaceFlux {
    float fmass;    // mass flux
    float fnorm_L;  // normal momentum flux minus source_L (used as "left" flux)
    float fnorm_R;  // normal momentum flux minus source_R (used as "right" flux)
    float ftan;     // tangential momentum flux
    uint32_t speed_bits;  // bit pattern of max(|SL|,|SR|) (>= 0, NaN stays NaN)
};

// primitive() of a reconstructed face state (riemann.py:20-38).
SWE_HD void face_primitive(float h0, float hu, float hv, const SweConsts& k, float& h, float& u,
                           float& v, float& c) {
    h = fmaxf(h0, 0.0f);
    bool wet = h > k.dry;
    float safe = fmaxf(h, k.floor_h);
    float y = shared_rcp(safe);
    u = wet ? quot(hu, safe, y) : 0.0f;
    v = wet ? quot(hv, safe, y) : 0.0f;
    c = wet ? root(k.g * safe) : 0.0f;
}

SWE_HD uint32_t f2u(float x) {
#if defined(__CUDA_ARCH__)
    return __float_as_uint(x);
#else
    union { float f; uint32_t u; } t;
    t.f = x;
    return t.u;
#endif
}

SWE_HD float u2f(uint32_t x) {
#if defined(__CUDA_ARCH__)
    return __uint_as_float(x);
#else
    union { float f; uint32_t u; } t;
    t.u = x;
    return t.f;
#endif
}

// Reconstructed states either side of one face and its two well-balanced
// sources (reconstruction.py:59-106).
struct FaceStates {
    float L0, L1, L2;  // UL = (h_cn_L, h_cn_L u_L, h_cn_L v_L)
    float R0, R1, R2;  // UR
    float srcL, srcR;  // source_L, source_R
};

// Lp is L's "p" side, Rm is R's "m" side; hL_c, zL_c, hR_c, zR_c are the two
// cells' depth and bed.
SWE_HD FaceStates face_states(const Side& Lp, float hL_c, float zL_c, const Side& Rm, float hR_c,
                              float zR_c, const SweConsts& k) {
    FaceStates s;
    // reconstruction.py:59-69
    float baud = fmaxf(Lp.bed, Rm.bed);
    float bcn = fminf(baud, fminf(Lp.eta, Rm.eta));
    float hcL = fmaxf(fminf(Lp.eta - bcn, Lp.hlin), 0.0f);
    float hcR = fmaxf(fminf(Rm.eta - bcn, Rm.hlin), 0.0f);
    // reconstruction.py:98-106
    s.L0 = hcL;
    s.L1 = hcL * Lp.u;
    s.L2 = hcL * Lp.v;
    s.R0 = hcR;
    s.R1 = hcR * Rm.u;
    s.R2 = hcR * Rm.v;
    s.srcL = (k.half_g * (hL_c + hcL)) * (zL_c - bcn);
    s.srcR = (k.half_g * (hcR + hR_c)) * (zR_c - bcn);
    return s;
}

// HLL flux of one face (riemann.py:41-105).  Returns the flux in channel
// order (mass, normal, tangential) via fh/fq/ft (already zeroed where both
// sides are dry) and the wave speed's bit pattern.
struct Hll {
    float fh, fq, ft;
    uint32_t speed_bits;
};

SWE_HD Hll hll_flux(float L0, float L1, float L2, float R0, float R1, float R2, bool normal_y,
                    const SweConsts& k) {
    // riemann.py:57-105
    float hL, uL, vL, cL, hR, uR, vR, cR;
    face_primitive(L0, L1, L2, k, hL, uL, vL, cL);
    face_primitive(R0, R1, R2, k, hR, uR, vR, cR);
    float unL = normal_y ? vL : uL, utL = normal_y ? uL : vL;
    float unR = normal_y ? vR : uR, utR = normal_y ? uR : vR;
    float us = (0.5f * (unL + unR) + cL) - cR;
    float cs = 0.5f * (cL + cR) + 0.25f * (unL - unR);
    float SLw = fminf(unL - cL, us - cs);
    float SRw = fmaxf(unR + cR, us + cs);
    bool ldry = hL <= k.dry, rdry = hR <= k.dry;
    float SL = ldry ? unR - 2.0f * cR : SLw;
    float SR = rdry ? unL + 2.0f * cL : SRw;
    float fhL = hL * unL, fhR = hR * unR;
    float fqL = hL * (unL * unL + k.half_g * hL);
    float fqR = hR * (unR * unR + k.half_g * hR);
    float den = fmaxf(SR - SL, k.den_floor);
    float yden = shared_rcp(den);
    float SLSR = SL * SR;
    float fhs = quot((SR * fhL - SL * fhR) + SLSR * (hR - hL), den, yden);
    float fqs = quot((SR * fqL - SL * fqR) + SLSR * (hR * unR - hL * unL), den, yden);
    bool lf = SL >= 0.0f, rf = SR <= 0.0f;
    float fh = lf ? fhL : (rf ? fhR : fhs);
    float fq = lf ? fqL : (rf ? fqR : fqs);
    float ft = (fh > 0.0f ? utL : utR) * fh;
    bool both = ldry && rdry;
    Hll r;
    r.fh = both ? 0.0f : fh;
    r.fq = both ? 0.0f : fq;
    r.ft = both ? 0.0f : ft;
    uint32_t a = f2u(SL) & 0x7fffffffu, b = f2u(SR) & 0x7fffffffu;
    r.speed_bits = both ? 0u : (a > b ? a : b);
    return r;
}

// One face between cell L and cell R: reconstruction, HLL flux and the
// source split of spatial_operator (solver.py:503-509).  normal_y selects
// the y-direction conventions of riemann.py:60-61, :199-203.
SWE_HD FaceFlux face_flux(const Side& Lp, float hL_c, float zL_c, const Side& Rm, float hR_c,
                          float zR_c, bool normal_y, const SweConsts& k) {
    const FaceStates s = face_states(Lp, hL_c, zL_c, Rm, hR_c, zR_c, k);
    const Hll h = hll_flux(s.L0, s.L1, s.L2, s.R0, s.R1, s.R2, normal_y, k);
    FaceFlux F;
    F.fmass = h.fh;
    F.ftan = h.ft;
    // Fx_left = F - sL, Fx_right = F - sR on the normal channel.
    F.fnorm_L = h.fq - s.srcL;
    F.fnorm_R = h.fq - s.srcR;
    F.speed_bits = h.speed_bits;
    return F;
}

// One cell's tendency (solver.py:511-525) from its four faces.  xm/xp are the
// faces at x-1/2 and x+1/2, ym/yp at y-1/2 and y+1/2.
struct Rhs {
    float r0, r1, r2;
};

SWE_HD Rhs cell_rhs(const FaceFlux& xm, const FaceFlux& xp, const FaceFlux& ym,
                    const FaceFlux& yp, const SweConsts& k, float rain, float loss) {
    Rhs r;
    // x: (Fx_right[x-1/2] - Fx_left[x+1/2]) / dx; channel order (fh, fq, ft)
    float x0 = quot(xm.fmass - xp.fmass, k.dx, k.rdx);
    float x1 = quot(xm.fnorm_R - xp.fnorm_L, k.dx, k.rdx);
    float x2 = quot(xm.ftan - xp.ftan, k.dx, k.rdx);
    // y: (Gy_top[y-1/2] - Gy_bottom[y+1/2]) / dy; channel order (fh, ft, fq)
    float y0 = quot(ym.fmass - yp.fmass, k.dy, k.rdy);
    float y1 = quot(ym.ftan - yp.ftan, k.dy, k.rdy);
    float y2 = quot(ym.fnorm_R - yp.fnorm_L, k.dy, k.rdy);
    r.r0 = ((x0 + y0) + rain) - loss;
    r.r1 = x1 + y1;
    r.r2 = x2 + y2;
    return r;
}

// _clean_and_limit, solver.py:547-570
struct State {
    float h, hu, hv;
};

SWE_HD State clean_and_limit(const State& o, State c, const SweConsts& k, bool positivity) {
    if (positivity) {
        float d0 = c.h - o.h, d1 = c.hu - o.hu, d2 = c.hv - o.hv;
        float safe = fmaxf(-d0, k.eps);
        float th = d0 < 0.0f ? fminf(quot(o.h, safe, shared_rcp(safe)), 1.0f) : 1.0f;
        c.h = o.h + th * d0;
        c.hu = o.hu + th * d1;
        c.hv = o.hv + th * d2;
    }
    State r;
    r.h = fmaxf(c.h, 0.0f);
    bool wet = r.h > k.dry;
    r.hu = wet ? c.hu : 0.0f;
    r.hv = wet ? c.hv : 0.0f;
    return r;
}

SWE_HD uint64_t d2u(double x) {
#if defined(__CUDA_ARCH__)
    return (uint64_t)__double_as_longlong(x);
#else
    union { double d; uint64_t u; } t;
    t.d = x;
    return t.u;
#endif
}

SWE_HD double u2d(uint64_t x) {
#if defined(__CUDA_ARCH__)
    return __longlong_as_double((long long)x);
#else
    union { double d; uint64_t u; } t;
    t.u = x;
    return t.d;
#endif
}

// x ** t for float x and t, as the double power x^t rounded once to float,
// i.e. the value of (float)pow((double)x, (double)t), for positive normal x
// and |t ln x| <= 700 (other arguments call pow itself).  The power is
// exp(t ln x), evaluated in double with double-double intermediates:
//   ln x = e ln 2 + ln m, m in [sqrt(1/2), sqrt(2)), ln m = 2 atanh(s) with
//   s = (m - 1)/(m + 1) carried as s + s_lo (exact FMA remainder), and
//   atanh(s)/s = sum s^2k/(2k+1) to k = 10 (|s| <= 0.1716: the first term
//   left out is below 2^-60); ln 2 split in a 32-bit head (exact products
//   with the exponent) and a tail (Cody and Waite, "Software Manual for the
//   Elementary Functions", 1980);
//   y = t ln x as a double-double, y = n ln 2 + r with n = rint(y / ln 2),
//   |r| <= ln 2 / 2, exp(r) from its Taylor series to degree 13 (remainder
//   below 2^-57), exp(y) = 2^n exp(r).
// The double result is within about 2^-54 relative of x^t, so it rounds to
// the same float as a correctly rounded double pow except for x^t within
// that distance of a float rounding midpoint.  swe_selftest_arith_f32
// (which = 4) compares it with CUDA's pow for every float x in a range.
SWE_HD float pow_pos(float x, float t) {
    const uint32_t xb = f2u(x);
    if (xb - 0x00800000u >= 0x7f000000u) return (float)pow((double)x, (double)t);
    constexpr double kLn2Hi = 0x1.62e42feep-1;              // 32 significant bits
    constexpr double kLn2Lo = 0x1.a39ef35793c76p-33;        // ln 2 - kLn2Hi
    constexpr double kInvLn2 = 0x1.71547652b82fep+0;        // 1 / ln 2
    int e = (int)(xb >> 23) - 127;
    uint32_t mb = (xb & 0x007fffffu) | 0x3f800000u;         // m in [1, 2)
    if (mb > 0x3fb504f3u) {                                 // m > sqrt(2): halve it
        mb -= 0x00800000u;
        e += 1;
    }
    const double m = (double)u2f(mb);
    const double num = m - 1.0, den = m + 1.0;              // both exact
    const double inv = 1.0 / den;
    const double s = num * inv;
    const double s_lo = fma(-s, den, num) * inv;            // num/den = s + s_lo
    const double s2 = s * s;
    double q = 1.0 / 21;
    q = fma(q, s2, 1.0 / 19);
    q = fma(q, s2, 1.0 / 17);
    q = fma(q, s2, 1.0 / 15);
    q = fma(q, s2, 1.0 / 13);
    q = fma(q, s2, 1.0 / 11);
    q = fma(q, s2, 1.0 / 9);
    q = fma(q, s2, 1.0 / 7);
    q = fma(q, s2, 1.0 / 5);
    q = fma(q, s2, 1.0 / 3);
    // ln m = a_hi + a_lo
    const double a_hi = 2.0 * s;
    const double a_lo = fma((2.0 * s) * s2, q, 2.0 * s_lo);
    // ln x = L_hi + L_lo (two-sum of e ln2_hi, exact, and a_hi)
    const double E = (double)e;
    const double p = E * kLn2Hi;
    const double L_hi = p + a_hi;
    const double bb = L_hi - p;
    const double L_lo = ((p - (L_hi - bb)) + (a_hi - bb)) + fma(E, kLn2Lo, a_lo);
    // y = t ln x = y_hi + y_lo
    const double td = (double)t;
    const double y_hi = td * L_hi;
    if (!(fabs(y_hi) <= 700.0)) return (float)pow((double)x, (double)t);
    const double y_lo = fma(td, L_hi, -y_hi) + td * L_lo;
    const double n = rint(y_hi * kInvLn2);
    const double r = fma(-n, kLn2Hi, y_hi) + fma(-n, kLn2Lo, y_lo);
    double c = 1.0 / 6227020800.0;                          // 1/13!
    c = fma(c, r, 1.0 / 479001600.0);
    c = fma(c, r, 1.0 / 39916800.0);
    c = fma(c, r, 1.0 / 3628800.0);
    c = fma(c, r, 1.0 / 362880.0);
    c = fma(c, r, 1.0 / 40320.0);
    c = fma(c, r, 1.0 / 5040.0);
    c = fma(c, r, 1.0 / 720.0);
    c = fma(c, r, 1.0 / 120.0);
    c = fma(c, r, 1.0 / 24.0);
    c = fma(c, r, 1.0 / 6.0);
    c = fma(c, r, 0.5);
    const double er = 1.0 + fma(r * r, c, r);               // exp(r)
    const double scale = u2d((uint64_t)((int)n + 1023) << 52);
    return (float)(er * scale);
}

// x ** (float)(1/3) rounded to float (friction.py:66): the double power
// rounded once.  PyTorch's CPU pow agrees with this value on all but a
// small fraction of inputs, where it differs by one ulp.
SWE_HD float pow_third(float x, float third) {
#if defined(__CUDA_ARCH__)
    return pow_pos(x, third);
#else
    return (float)pow((double)x, (double)third);
#endif
}

// Semi-implicit friction factor shared by both friction models
// (friction.py:12-38 and :89, :122).
SWE_HD State apply_friction_factor(const State& s, float cf_of_h, float dt, const SweConsts& k,
                                   float speed, float safe, bool wet) {
    float fac = recip(1.0f + quot((cf_of_h * speed) * dt, safe, shared_rcp(safe)));
    State r;
    r.h = s.h;
    r.hu = wet ? s.hu * fac : 0.0f;
    r.hv = wet ? s.hv * fac : 0.0f;
    return r;
}

// apply_manning_friction, friction.py:102-131 (with :12-38, :62-66).  s.h is
// clamp(U[:,0], min=0) already applied by the caller or here.
SWE_HD State manning(State s, float n, float dt, const SweConsts& k) {
    s.h = fmaxf(s.h, 0.0f);
    bool wet = s.h > k.dry;
    float safe = fmaxf(s.h, k.fr_vs);
    float ys = shared_rcp(safe);
    float u = quot(wet ? s.hu : 0.0f, safe, ys);
    float v = quot(wet ? s.hv : 0.0f, safe, ys);
    float sp2 = u * u + v * v;
    bool moving = wet && (sp2 > 0.0f);
    float speed = moving ? root(fmaxf(sp2, k.fr_e2)) : 0.0f;
    float nn = fmaxf(n, 0.0f);
    float pw = pow_third(fmaxf(s.h, k.fr_e), k.third);
    float cf = quot(k.g981 * (nn * nn), pw, shared_rcp(pw));
    return apply_friction_factor(s, cf, dt, k, speed, safe, wet);
}

// apply_roughness_length_friction, friction.py:69-99 (with :41-59).
SWE_HD State roughness_friction(State s, float z0, float dt, const SweConsts& k) {
    s.h = fmaxf(s.h, 0.0f);
    bool wet = s.h > k.dry;
    float safe = fmaxf(s.h, k.fr_vs);
    float ys = shared_rcp(safe);
    float u = quot(wet ? s.hu : 0.0f, safe, ys);
    float v = quot(wet ? s.hv : 0.0f, safe, ys);
    float sp2 = u * u + v * v;
    bool moving = wet && (sp2 > 0.0f);
    float speed = moving ? root(fmaxf(sp2, k.fr_e2)) : 0.0f;
    float zz = fmaxf(z0, k.fr_e);
    float ratio = quot(fmaxf(s.h, k.fr_e), zz, shared_rcp(zz));
    float shallow = recip(fmaxf(0.46f * ratio, k.fr_e));
    float rc = fmaxf(ratio, k.fr_e);
    float lt = 2.5f * (((float)log((double)rc) - 1.0f) + recip(rc) * 1.359f);
    float deep = recip(fmaxf(lt * lt, k.fr_e));
    float cf = ratio < 2.71828182845904523536f ? shallow : deep;
    return apply_friction_factor(s, cf, dt, k, speed, safe, wet);
}

// stable dt, solver.py:620-626: cfl / clamp(ax/dx + ay/dy, min=eps), where
// PyTorch evaluates `scalar / tensor` as tensor.reciprocal() * scalar.
SWE_HD float stable_dt(float ax, float ay, const SweConsts& k) {
#if defined(__CUDA_ARCH__)
    // IEEE divisions whatever the file's division flags (the tolerance-mode
    // kernels are compiled with approximate "/").
    float den = fmaxf(__fadd_rn(__fdiv_rn(ax, k.dx), __fdiv_rn(ay, k.dy)), k.eps);
    return __fmul_rn(__frcp_rn(den), k.cfl);
#else
    float den = fmaxf(ax / k.dx + ay / k.dy, k.eps);
    return (1.0f / den) * k.cfl;
#endif
}

}  // namespace swe
