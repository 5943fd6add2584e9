// swe_adjoint.cuh -- hand-written reverse mode of the FP32 step's face
// function, with the derivative conventions of PyTorch's autograd so the
// adjoint equals the reference's autograd gradient (src/solver.py:572-663
// differentiated by PyTorch, dt detached):
//   torch.where              gradient to the selected branch only
//   torch.minimum / maximum  gradient to the smaller/larger input, halved
//                            between the two on an exact tie
//   torch.clamp              gradient passes where min <= x <= max (bounds
//                            included), zero outside
//   abs, sign                sign(x) and 0 (both 0 at x = 0)
//   sqrt                     grad / (2 sqrt(x)); x / y: grad / y and
//                            -grad (x / y) / y
// The bed is differentiated on request (template flag BEDG: the gradient
// of the DEM-correction inversion, src/solver.py:111-147); without it the
// bed's adjoint is not formed.
#pragma once

#include <math.h>

#include "swe_approx.cuh"
#include "swe_math.cuh"

namespace swe {

// Gradient shares of torch.minimum(a, b) (or maximum with larger = true).
SWE_HD void minmax_shares(float a, float b, bool larger, float& sa, float& sb) {
    sa = a == b ? 0.5f : (((a < b) != larger) ? 1.0f : 0.0f);
    sb = 1.0f - sa;
}

// limited_increment of the middle of three values with the shares of each
// of the three minmod3 arguments (numerics.py:4-27 under autograd).
struct Incr {
    float val;
    float sa, sb, sc;  // d val / d(theta*backward), d/d(centred), d/d(theta*forward)
};

SWE_HD Incr incr_fwd(float qm, float q, float qp, float theta) {
    const float a = theta * (q - qm);
    const float b = 0.5f * (qp - qm);
    const float c = theta * (qp - q);
    Incr r;
    r.val = minmod3(a, b, c);
    // minmod3 passes gradient only when all three share a sign (a NaN
    // compares false: no gradient), to the smallest of |a|, min(|b|, |c|)
    // with torch.minimum's tie rule (half each on a tie): the shares of
    // minmax_shares, written branch-free (s_in = 1 - s_a, s_c = 1 - s_b).
    const bool same = (a > 0.0f && b > 0.0f && c > 0.0f) || (a < 0.0f && b < 0.0f && c < 0.0f);
    const float aa = fabsf(a), ab = fabsf(b), ac = fabsf(c);
    const float inner = fminf(ab, ac);
    const float s_a = aa == inner ? 0.5f : (aa < inner ? 1.0f : 0.0f);
    const float s_b = ab == ac ? 0.5f : (ab < ac ? 1.0f : 0.0f);
    const float s_in = same ? 1.0f - s_a : 0.0f;
    r.sa = same ? s_a : 0.0f;
    r.sb = s_in * s_b;
    r.sc = s_in * (1.0f - s_b);
    return r;
}

// Adjoint of an increment: adds to the three values' adjoints.
SWE_HD void incr_bwd(const Incr& r, float lam, float theta, float& lqm, float& lq, float& lqp) {
    const float la = (lam * r.sa) * theta;  // d/d(q - qm)
    const float lb = (lam * r.sb) * 0.5f;   // d/d(qp - qm)
    const float lc = (lam * r.sc) * theta;  // d/d(qp - q)
    lq += la - lc;
    lqm -= la + lb;
    lqp += lb + lc;
}

// Arithmetic of the adjoint's quotients, reciprocals and roots, a policy
// class M of every function below:
//   ExactMath: the correctly-rounded forms of the IEEE step (swe_math.cuh),
//              for adjoints of runs made with SWE_ARITH_EXACT;
//   FastMath:  the hardware approximations of the tolerance-mode step
//              (swe_approx.cuh), for runs made with SWE_ARITH_FAST.
// div(a, b, y) is a / b with y = rcp(b) shared by the quotients of one
// denominator; pow(x, t) is x^t for positive normal x.
struct ExactMath {
    static SWE_HD float rcp(float b) { return shared_rcp(b); }
    static SWE_HD float div(float a, float b, float y) { return quot(a, b, y); }
    static SWE_HD float sqrt(float x) { return root(x); }
    static SWE_HD float inv(float b) { return recip(b); }
    static SWE_HD float pow(float x, float t) { return pow_pos(x, t); }
    static SWE_HD float ln(float x) { return (float)::log((double)x); }
};

struct FastMath {
#if defined(__CUDA_ARCH__)
    static __device__ __forceinline__ float rcp(float b) { return rcpa(b); }
    static __device__ __forceinline__ float div(float a, float, float y) { return a * y; }
    static __device__ __forceinline__ float sqrt(float x) { return sqrta(x); }
    static __device__ __forceinline__ float inv(float b) { return rcpa(b); }
    static __device__ __forceinline__ float pow(float x, float t) { return ex2a(t * lg2a(x)); }
    static __device__ __forceinline__ float ln(float x) { return 0.69314718f * lg2a(x); }
#else
    static inline float rcp(float b) { return 1.0f / b; }
    static inline float div(float a, float b, float) { return a / b; }
    static inline float sqrt(float x) { return ::sqrtf(x); }
    static inline float inv(float b) { return 1.0f / b; }
    static inline float pow(float x, float t) { return ::powf(x, t); }
    static inline float ln(float x) { return ::logf(x); }
#endif
};

// Forward values of one cell kept for the backward pass.
struct PrimRec {
    float U0, U1, U2, z;
    float h, safe, u, v, eta;
    float rsafe;  // M::rcp(safe): every quotient by safe uses it
    bool wet;
};

template <class M>
SWE_HD PrimRec prim_rec(float U0, float U1, float U2, float z, const SweConsts& k) {
    PrimRec p;
    p.U0 = U0;
    p.U1 = U1;
    p.U2 = U2;
    p.z = z;
    p.h = fmaxf(U0, 0.0f);
    p.wet = p.h > k.dry;
    p.safe = fmaxf(p.h, k.floor_h);
    p.rsafe = M::rcp(p.safe);
    p.u = p.wet ? M::div(U1, p.safe, p.rsafe) : 0.0f;
    p.v = p.wet ? M::div(U2, p.safe, p.rsafe) : 0.0f;
    p.eta = p.h + z;
    return p;
}

// Adjoint of primitive() + eta = h + bed (riemann.py:20-38,
// reconstruction.py:23-24, :71-73): lh includes everything that reached h
// (directly, via eta and via the reconstruction's own clamp of h).
template <class M>
SWE_HD void prim_bwd(const PrimRec& p, float lh, float lsafe, float lu, float lv, float leta,
                     const SweConsts& k, float& lU0, float& lU1, float& lU2, float& lz) {
    lh += leta;
    lz += leta;  // eta = h + bed
    if (p.wet) {
        lU1 += M::div(lu, p.safe, p.rsafe);
        lU2 += M::div(lv, p.safe, p.rsafe);
        lsafe -= lu * M::div(p.u, p.safe, p.rsafe) + lv * M::div(p.v, p.safe, p.rsafe);
    }
    if (p.h >= k.floor_h) lh += lsafe;
    if (p.U0 >= 0.0f) lU0 += lh;
}

// One side of a cell in one direction (reconstruction.py:26-96) with what
// the backward pass needs.  plus = true: the "p" side (h + dh/2 ...),
// false: the "m" side.
struct SideRec {
    Incr ih, ie, iz, iu, iv;
    bool reset;
    float q, f_raw, f;  // 0.5 dh / safe, factor before and after the clamp
    Side s;
};

template <class M>
SWE_HD SideRec side_fwd(const PrimRec& a, const PrimRec& c, const PrimRec& b, bool plus,
                        const SweConsts& k, bool wsr) {
    SideRec r;
    r.ih = incr_fwd(a.h, c.h, b.h, k.theta);
    r.ie = incr_fwd(a.eta, c.eta, b.eta, k.theta);
    r.iz = incr_fwd(a.z, c.z, b.z, k.theta);
    r.iu = incr_fwd(a.u, c.u, b.u, k.theta);
    r.iv = incr_fwd(a.v, c.v, b.v, k.theta);
    const float dh = r.ih.val, dz = r.iz.val;
    float deta = r.ie.val;
    r.reset = false;
    if (wsr) {
        const float half = 0.5f * (deta - dh);
        const float base = c.eta - c.h;
        const float bm = base - half, bp = base + half;
        r.reset = (deta * deta > dz * dz) && ((bm > a.eta) || (bp > b.eta));
        if (r.reset) deta = dh + dz;
    }
    const float hdh = 0.5f * dh;
    r.q = M::div(hdh, c.safe, c.rsafe);
    if (plus) {
        r.s.hlin = c.h + hdh;
        r.s.eta = c.eta + 0.5f * deta;
        r.s.bed = c.z + 0.5f * dz;
        r.f_raw = c.h > k.dry ? 1.0f - r.q : 1.0f;
    } else {
        r.s.hlin = c.h - hdh;
        r.s.eta = c.eta - 0.5f * deta;
        r.s.bed = c.z - 0.5f * dz;
        r.f_raw = c.h > k.dry ? 1.0f + r.q : 1.0f;
    }
    r.f = fminf(fmaxf(r.f_raw, -10.0f), 10.0f);
    const float hf = 0.5f * r.f;
    if (plus) {
        r.s.u = c.u + hf * r.iu.val;
        r.s.v = c.v + hf * r.iv.val;
    } else {
        r.s.u = c.u - hf * r.iu.val;
        r.s.v = c.v - hf * r.iv.val;
    }
    return r;
}

// Adjoints of the three cells' primitives (h, safe, u, v, eta per cell).
struct PrimAdj {
    float h, safe, u, v, eta, z;
};

template <bool BEDG, class M>
SWE_HD void side_bwd(const SideRec& r, const PrimRec& c, bool plus, float l_hlin, float l_eta,
                     float l_u, float l_v, float l_bed, const SweConsts& k, PrimAdj& la,
                     PrimAdj& lc, PrimAdj& lb) {
    const float sg = plus ? 1.0f : -1.0f;
    // u_side = u +/- (0.5 f) du ; v likewise
    const float hf = 0.5f * r.f;
    lc.u += l_u;
    lc.v += l_v;
    float l_du = sg * (l_u * hf);
    float l_dv = sg * (l_v * hf);
    float l_hf = sg * (l_u * r.iu.val + l_v * r.iv.val);
    float l_f = 0.5f * l_hf;
    // clamp(-10, 10) then where(h > dry, 1 -/+ q, 1)
    float l_fraw = (r.f_raw >= -10.0f && r.f_raw <= 10.0f) ? l_f : 0.0f;
    float l_q = c.h > k.dry ? -sg * l_fraw : 0.0f;
    // q = (0.5 dh) / safe
    float l_dh = 0.5f * M::div(l_q, c.safe, c.rsafe);
    lc.safe -= l_q * M::div(r.q, c.safe, c.rsafe);
    // hlin = h +/- 0.5 dh ; eta_side = eta +/- 0.5 deta
    lc.h += l_hlin;
    l_dh += sg * (0.5f * l_hlin);
    lc.eta += l_eta;
    float l_deta = sg * (0.5f * l_eta);
    float l_dz = 0.0f;
    if (BEDG) {  // bed_side = bed +/- 0.5 dz
        lc.z += l_bed;
        l_dz = sg * (0.5f * l_bed);
    }
    if (r.reset) {  // deta = dh + dz
        l_dh += l_deta;
        if (BEDG) l_dz += l_deta;
        l_deta = 0.0f;
    }
    if (BEDG) incr_bwd(r.iz, l_dz, k.theta, la.z, lc.z, lb.z);
    incr_bwd(r.ih, l_dh, k.theta, la.h, lc.h, lb.h);
    incr_bwd(r.ie, l_deta, k.theta, la.eta, lc.eta, lb.eta);
    incr_bwd(r.iu, l_du, k.theta, la.u, lc.u, lb.u);
    incr_bwd(r.iv, l_dv, k.theta, la.v, lc.v, lb.v);
}

// Adjoint of the face function for cells (p0, p1 | p2, p3) along a line: the
// face lies between p1 and p2.  Inputs: adjoints of the face outputs
// (mass flux, normal flux minus source_L, normal flux minus source_R,
// tangential flux).  Outputs: adjoints of (U0, U1, U2) of the four cells.
struct CellAdj {
    float U0, U1, U2, Z;  // Z: adjoint of the cell's bed (BEDG only)
};

template <bool BEDG, class M>
SWE_HD void face_vjp(const PrimRec P[4], float l_mass, float l_nL, float l_nR, float l_tan,
                     bool normal_y, const SweConsts& k, bool wsr, CellAdj out[4]) {
    // ---- forward: sides of p1 ("p") and p2 ("m")
    const SideRec SL_ = side_fwd<M>(P[0], P[1], P[2], true, k, wsr);
    const SideRec SR_ = side_fwd<M>(P[1], P[2], P[3], false, k, wsr);
    const Side& Lp = SL_.s;
    const Side& Rm = SR_.s;
    // face reconstruction (reconstruction.py:59-106)
    const float baud = fmaxf(Lp.bed, Rm.bed);
    const float inner = fminf(Lp.eta, Rm.eta);
    const float bcn = fminf(baud, inner);
    const float AL = Lp.eta - bcn, AR = Rm.eta - bcn;
    const float mL = fminf(AL, Lp.hlin), mR = fminf(AR, Rm.hlin);
    const float hcL = fmaxf(mL, 0.0f), hcR = fmaxf(mR, 0.0f);
    const float UL1 = hcL * Lp.u, UL2 = hcL * Lp.v, UR1 = hcR * Rm.u, UR2 = hcR * Rm.v;
    const float sL1 = k.half_g * (P[1].h + hcL), sL2 = P[1].z - bcn;
    const float sR1 = k.half_g * (hcR + P[2].h), sR2 = P[2].z - bcn;
    // HLL (riemann.py:57-105)
    const float hL = fmaxf(hcL, 0.0f), hR = fmaxf(hcR, 0.0f);
    const bool wetL = hL > k.dry, wetR = hR > k.dry;
    const float safeL = fmaxf(hL, k.floor_h), safeR = fmaxf(hR, k.floor_h);
    const float ysL = M::rcp(safeL), ysR = M::rcp(safeR);
    const float uL = wetL ? M::div(UL1, safeL, ysL) : 0.0f, vL = wetL ? M::div(UL2, safeL, ysL) : 0.0f;
    const float uR = wetR ? M::div(UR1, safeR, ysR) : 0.0f, vR = wetR ? M::div(UR2, safeR, ysR) : 0.0f;
    const float cL = wetL ? M::sqrt(k.g * safeL) : 0.0f, cR = wetR ? M::sqrt(k.g * safeR) : 0.0f;
    const float unL = normal_y ? vL : uL, utL = normal_y ? uL : vL;
    const float unR = normal_y ? vR : uR, utR = normal_y ? uR : vR;
    const float us = (0.5f * (unL + unR) + cL) - cR;
    const float cs = 0.5f * (cL + cR) + 0.25f * (unL - unR);
    const float t1 = unL - cL, t2 = us - cs, t3 = unR + cR, t4 = us + cs;
    const float SLw = fminf(t1, t2), SRw = fmaxf(t3, t4);
    const bool ldry = hL <= k.dry, rdry = hR <= k.dry;
    const float SL = ldry ? unR - 2.0f * cR : SLw;
    const float SR = rdry ? unL + 2.0f * cL : SRw;
    const float fhL = hL * unL, fhR = hR * unR;
    const float wL = unL * unL + k.half_g * hL, wR = unR * unR + k.half_g * hR;
    const float fqL = hL * wL, fqR = hR * wR;
    const float dd = SR - SL;
    const float den = fmaxf(dd, k.den_floor);
    const float SLSR = SL * SR;
    const float numh = (SR * fhL - SL * fhR) + SLSR * (hR - hL);
    const float mom = hR * unR - hL * unL;
    const float numq = (SR * fqL - SL * fqR) + SLSR * mom;
    const float yden = M::rcp(den);
    const float fhs = M::div(numh, den, yden), fqs = M::div(numq, den, yden);
    const bool lf = SL >= 0.0f, rf = SR <= 0.0f;
    const float fh = lf ? fhL : (rf ? fhR : fhs);
    const bool both = ldry && rdry;

    // ---- backward
    // outputs: mass = fh, nL = fq - srcL, nR = fq - srcR, tan = (fh>0 ? utL : utR) * fh
    float l_fh = 0.0f, l_fq = 0.0f, l_utL = 0.0f, l_utR = 0.0f;
    if (!both) {
        l_fh = l_mass;
        l_fq = l_nL + l_nR;
        const float ut = fh > 0.0f ? utL : utR;
        l_fh += l_tan * ut;
        if (fh > 0.0f) l_utL += l_tan * fh;
        else l_utR += l_tan * fh;
    }
    const float l_srcL = -l_nL, l_srcR = -l_nR;
    // fh / fq selection
    float l_fhL = 0.0f, l_fhR = 0.0f, l_fhs = 0.0f, l_fqL = 0.0f, l_fqR = 0.0f, l_fqs = 0.0f;
    if (lf) {
        l_fhL = l_fh;
        l_fqL = l_fq;
    } else if (rf) {
        l_fhR = l_fh;
        l_fqR = l_fq;
    } else {
        l_fhs = l_fh;
        l_fqs = l_fq;
    }
    // fhs = numh / den, fqs = numq / den
    const float l_numh = M::div(l_fhs, den, yden), l_numq = M::div(l_fqs, den, yden);
    const float l_den = -(l_fhs * M::div(fhs, den, yden)) - l_fqs * M::div(fqs, den, yden);
    float l_SL = 0.0f, l_SR = 0.0f, l_hL = 0.0f, l_hR = 0.0f, l_unL = 0.0f, l_unR = 0.0f;
    float l_cL = 0.0f, l_cR = 0.0f;
    // numh = (SR fhL - SL fhR) + SLSR (hR - hL)
    l_SR += l_numh * fhL;
    l_fhL += l_numh * SR;
    l_SL -= l_numh * fhR;
    l_fhR -= l_numh * SL;
    float l_SLSR = l_numh * (hR - hL);
    l_hR += l_numh * SLSR;
    l_hL -= l_numh * SLSR;
    // numq = (SR fqL - SL fqR) + SLSR (hR unR - hL unL)
    l_SR += l_numq * fqL;
    l_fqL += l_numq * SR;
    l_SL -= l_numq * fqR;
    l_fqR -= l_numq * SL;
    l_SLSR += l_numq * mom;
    const float l_mom = l_numq * SLSR;
    l_hR += l_mom * unR;
    l_unR += l_mom * hR;
    l_hL -= l_mom * unL;
    l_unL -= l_mom * hL;
    l_SL += l_SLSR * SR;
    l_SR += l_SLSR * SL;
    if (dd >= k.den_floor) {  // den = clamp(SR - SL, min=floor)
        l_SR += l_den;
        l_SL -= l_den;
    }
    // fqL = hL (unL^2 + g/2 hL), fhL = hL unL (and R)
    l_hL += l_fqL * wL;
    {
        const float l_w = l_fqL * hL;
        l_unL += l_w * (2.0f * unL);
        l_hL += l_w * k.half_g;
    }
    l_hR += l_fqR * wR;
    {
        const float l_w = l_fqR * hR;
        l_unR += l_w * (2.0f * unR);
        l_hR += l_w * k.half_g;
    }
    l_hL += l_fhL * unL;
    l_unL += l_fhL * hL;
    l_hR += l_fhR * unR;
    l_unR += l_fhR * hR;
    // SL = ldry ? unR - 2 cR : min(t1, t2);  SR = rdry ? unL + 2 cL : max(t3, t4)
    float l_t1 = 0.0f, l_t2 = 0.0f, l_t3 = 0.0f, l_t4 = 0.0f;
    if (ldry) {
        l_unR += l_SL;
        l_cR -= 2.0f * l_SL;
    } else {
        float s1, s2;
        minmax_shares(t1, t2, false, s1, s2);
        l_t1 = l_SL * s1;
        l_t2 = l_SL * s2;
    }
    if (rdry) {
        l_unL += l_SR;
        l_cL += 2.0f * l_SR;
    } else {
        float s3, s4;
        minmax_shares(t3, t4, true, s3, s4);
        l_t3 = l_SR * s3;
        l_t4 = l_SR * s4;
    }
    l_unL += l_t1;
    l_cL -= l_t1;
    l_unR += l_t3;
    l_cR += l_t3;
    const float l_us = l_t2 + l_t4, l_cs = l_t4 - l_t2;
    // us = (0.5 (unL + unR) + cL) - cR ; cs = 0.5 (cL + cR) + 0.25 (unL - unR)
    l_unL += 0.5f * l_us + 0.25f * l_cs;
    l_unR += 0.5f * l_us - 0.25f * l_cs;
    l_cL += l_us + 0.5f * l_cs;
    l_cR += 0.5f * l_cs - l_us;
    // un / ut back to u / v
    const float l_uL = normal_y ? l_utL : l_unL, l_vL = normal_y ? l_unL : l_utL;
    const float l_uR = normal_y ? l_utR : l_unR, l_vR = normal_y ? l_unR : l_utR;
    // primitive() of the face states
    float l_UL1 = 0.0f, l_UL2 = 0.0f, l_UR1 = 0.0f, l_UR2 = 0.0f, l_safeL = 0.0f, l_safeR = 0.0f;
    if (wetL) {
        l_UL1 = M::div(l_uL, safeL, ysL);
        l_UL2 = M::div(l_vL, safeL, ysL);
        l_safeL -= l_uL * M::div(uL, safeL, ysL) + l_vL * M::div(vL, safeL, ysL);
        const float c2 = 2.0f * cL;
        l_safeL += k.g * M::div(l_cL, c2, M::rcp(c2));
    }
    if (wetR) {
        l_UR1 = M::div(l_uR, safeR, ysR);
        l_UR2 = M::div(l_vR, safeR, ysR);
        l_safeR -= l_uR * M::div(uR, safeR, ysR) + l_vR * M::div(vR, safeR, ysR);
        const float c2 = 2.0f * cR;
        l_safeR += k.g * M::div(l_cR, c2, M::rcp(c2));
    }
    if (hL >= k.floor_h) l_hL += l_safeL;
    if (hR >= k.floor_h) l_hR += l_safeR;
    float l_hcL = hcL >= 0.0f ? l_hL : 0.0f;
    float l_hcR = hcR >= 0.0f ? l_hR : 0.0f;
    // UL = (hcL, hcL uL_side, hcL vL_side)
    l_hcL += l_UL1 * Lp.u + l_UL2 * Lp.v;
    l_hcR += l_UR1 * Rm.u + l_UR2 * Rm.v;
    const float l_Lu = l_UL1 * hcL, l_Lv = l_UL2 * hcL;
    const float l_Ru = l_UR1 * hcR, l_Rv = l_UR2 * hcR;
    // sources: srcL = (g/2 (h1 + hcL)) (z1 - bcn)
    float l_bcn = 0.0f;
    PrimAdj la[4] = {};
    {
        const float l_s1 = l_srcL * sL2;
        l_bcn -= l_srcL * sL1;
        la[1].h += k.half_g * l_s1;
        l_hcL += k.half_g * l_s1;
        const float l_s2 = l_srcR * sR2;
        l_bcn -= l_srcR * sR1;
        la[2].h += k.half_g * l_s2;
        l_hcR += k.half_g * l_s2;
        if (BEDG) {  // srcL = (g/2 (h1 + hcL)) (z1 - bcn), srcR likewise with z2
            la[1].z += l_srcL * sL1;
            la[2].z += l_srcR * sR1;
        }
    }
    // hc = clamp(min(eta_side - bcn, hlin), min=0)
    const float l_mL = mL >= 0.0f ? l_hcL : 0.0f;
    const float l_mR = mR >= 0.0f ? l_hcR : 0.0f;
    float sa, sb;
    minmax_shares(AL, Lp.hlin, false, sa, sb);
    const float l_AL = l_mL * sa, l_Lhlin = l_mL * sb;
    minmax_shares(AR, Rm.hlin, false, sa, sb);
    const float l_AR = l_mR * sa, l_Rhlin = l_mR * sb;
    float l_Leta = l_AL, l_Reta = l_AR;
    l_bcn -= l_AL + l_AR;
    // bcn = min(baud, min(etaL, etaR)); baud = max(bedL, bedR)
    minmax_shares(baud, inner, false, sa, sb);
    const float l_inner = l_bcn * sb;
    float l_Lbed = 0.0f, l_Rbed = 0.0f;
    if (BEDG) {
        const float l_baud = l_bcn * sa;
        float ba, bb;
        minmax_shares(Lp.bed, Rm.bed, true, ba, bb);
        l_Lbed = l_baud * ba;
        l_Rbed = l_baud * bb;
    }
    minmax_shares(Lp.eta, Rm.eta, false, sa, sb);
    l_Leta += l_inner * sa;
    l_Reta += l_inner * sb;
    // sides -> primitives of the four cells
    side_bwd<BEDG, M>(SL_, P[1], true, l_Lhlin, l_Leta, l_Lu, l_Lv, l_Lbed, k, la[0], la[1], la[2]);
    side_bwd<BEDG, M>(SR_, P[2], false, l_Rhlin, l_Reta, l_Ru, l_Rv, l_Rbed, k, la[1], la[2], la[3]);
    for (int i = 0; i < 4; ++i) {
        out[i].U0 = out[i].U1 = out[i].U2 = 0.0f;
        out[i].Z = la[i].z;  // sources, increments, face beds; prim_bwd adds the eta term
        prim_bwd<M>(P[i], la[i].h, la[i].safe, la[i].u, la[i].v, la[i].eta, k, out[i].U0, out[i].U1,
                 out[i].U2, out[i].Z);
    }
}

}  // namespace swe
