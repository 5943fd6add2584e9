/*
 * swe_oracle_impl.h -- TEST INFRASTRUCTURE ONLY.  Included twice by
 * swe_oracle.c, once with R=float (suffix f32) and once with R=double
 * (suffix f64).  Each function restates the reference function named in its
 * comment, one array operation per line, in the reference's evaluation
 * order.  Python scalars that the reference multiplies into a tensor are
 * rounded to R first, as PyTorch does for a wrapped scalar.
 */

#define FN(name) CAT(name, SFX)
#define CAT(a, b) CAT2(a, b)
#define CAT2(a, b) a##_##b

/* The reference's dtype-dependent floors (src/riemann.py:6-11,
 * src/reconstruction.py:12-15, src/friction.py:4-9). */
static double FN(precision_floor)(void) { return sizeof(R) == 4 ? 1.0e-6 : 1.0e-10; }

static double FN(depth_floor)(double eps, double dry) {
    double f = eps > dry ? eps : dry;
    double pf = FN(precision_floor)();
    return f > pf ? f : pf;
}

/* torch.minimum / torch.maximum / torch.clamp propagate NaN. */
static inline R FN(tmin)(R a, R b) { return (a != a || b != b) ? (R)NAN : (a < b ? a : b); }
static inline R FN(tmax)(R a, R b) { return (a != a || b != b) ? (R)NAN : (a > b ? a : b); }
static inline R FN(clamp_min)(R x, R m) { return x != x ? x : (x < m ? m : x); }
static inline R FN(clamp_max)(R x, R m) { return x != x ? x : (x > m ? m : x); }
static inline R FN(tsign)(R a) { return a != a ? a : (R)((a > 0) - (a < 0)); }
static inline R FN(tabs)(R a) { return a < 0 ? -a : (a == 0 ? (R)0 : a); }

/* minmod3, src/numerics.py:4-13 */
static inline R FN(minmod3)(R a, R b, R c) {
    R sa = FN(tsign)(a), sb = FN(tsign)(b), sc = FN(tsign)(c);
    int same = (sa == sb) && (sb == sc);
    R mag = FN(tmin)(FN(tabs)(a), FN(tmin)(FN(tabs)(b), FN(tabs)(c)));
    return same ? sa * mag : (R)0;
}

/* limited_increment, src/numerics.py:16-27, on one line of length W with
 * torch.roll wrap-around.  q[k*stride]. */
static void FN(limited_increment_line)(const R* q, int W, long stride, R theta, R* out, long ostride) {
    for (int k = 0; k < W; ++k) {
        R qm = q[(long)((k - 1 + W) % W) * stride];
        R qp = q[(long)((k + 1) % W) * stride];
        R qc = q[(long)k * stride];
        R backward = qc - qm;
        R centred = (R)0.5 * (qp - qm);
        R forward = qp - qc;
        out[(long)k * ostride] = FN(minmod3)(theta * backward, centred, theta * forward);
    }
}

int FN(orc_limited_increment)(const R* q, int B, int C, int H, int W, int dim, double theta, R* out) {
    R th = (R)theta;
    long plane = (long)H * W;
#pragma omp parallel for collapse(2) schedule(static)
    for (int b = 0; b < B * C; ++b)
        for (int line = 0; line < (dim == -1 ? H : W); ++line) {
            const R* base = q + (long)b * plane;
            R* ob = out + (long)b * plane;
            if (dim == -1)
                FN(limited_increment_line)(base + (long)line * W, W, 1, th, ob + (long)line * W, 1);
            else
                FN(limited_increment_line)(base + line, H, W, th, ob + line, W);
        }
    return 0;
}

/* primitive, src/riemann.py:20-38 */
static inline void FN(primitive1)(R U0, R U1, R U2, R g, R dry, R floor_, R* h, R* u, R* v, R* c) {
    R hh = FN(clamp_min)(U0, (R)0);
    int wet = hh > dry;
    R safe = FN(clamp_min)(hh, floor_);
    *h = hh;
    *u = wet ? U1 / safe : (R)0;
    *v = wet ? U2 / safe : (R)0;
    *c = wet ? (R)sqrt(g * safe) : (R)0;
}

int FN(orc_primitive)(const R* U, int B, int H, int W, const orc_params* p, R* h, R* u, R* v, R* c) {
    long plane = (long)H * W;
    R g = (R)p->gravity, dry = (R)p->dry_depth, fl = (R)FN(depth_floor)(p->epsilon, p->dry_depth);
#pragma omp parallel for schedule(static)
    for (int b = 0; b < B; ++b)
        for (long i = 0; i < plane; ++i) {
            const R* Ub = U + (long)b * 3 * plane;
            FN(primitive1)(Ub[i], Ub[plane + i], Ub[2 * plane + i], g, dry, fl,
                           h + b * plane + i, u + b * plane + i, v + b * plane + i, c + b * plane + i);
        }
    return 0;
}

/* add_ghost_cells, src/boundary.py:150-413.  level and cval hold one value
 * per batch member (a scalar is repeated by the caller).  Up is
 * [B,3,ny+2ng,nx+2ng]; zp is [bedB,1,ny+2ng,nx+2ng]. */
int FN(orc_ghost_cells)(const R* U, const R* bed, int B, int bedB, int ny, int nx, int ng,
                        const orc_params* p, const R* level, const R* cval, R* Up, R* zp) {
    int H = ny + 2 * ng, W = nx + 2 * ng;
    long plane = (long)H * W, iplane = (long)ny * nx;
    int bcs[4] = {p->bc_left, p->bc_right, p->bc_top, p->bc_bottom};
#define UP(b, ch, q, x) Up[((long)(b) * 3 + (ch)) * plane + (long)(q) * W + (x)]
#define ZP(b, q, x) zp[(long)(b) * plane + (long)(q) * W + (x)]
#define UI(b, ch, q, x) U[((long)(b) * 3 + (ch)) * iplane + (long)(q) * nx + (x)]
#define BI(b, q, x) bed[(long)(b) * iplane + (long)(q) * nx + (x)]
    /* replicate padding (F.pad mode="replicate"), :227-238 */
    for (int b = 0; b < B; ++b)
        for (int ch = 0; ch < 3; ++ch)
            for (int q = 0; q < H; ++q)
                for (int x = 0; x < W; ++x) {
                    int qi = q - ng < 0 ? 0 : (q - ng >= ny ? ny - 1 : q - ng);
                    int xi = x - ng < 0 ? 0 : (x - ng >= nx ? nx - 1 : x - ng);
                    UP(b, ch, q, x) = UI(b, ch, qi, xi);
                }
    for (int b = 0; b < bedB; ++b)
        for (int q = 0; q < H; ++q)
            for (int x = 0; x < W; ++x) {
                int qi = q - ng < 0 ? 0 : (q - ng >= ny ? ny - 1 : q - ng);
                int xi = x - ng < 0 ? 0 : (x - ng >= nx ? nx - 1 : x - ng);
                ZP(b, q, x) = BI(b, qi, xi);
            }
    /* periodic bed, :247-257 */
    for (int b = 0; b < bedB; ++b) {
        if (bcs[0] == ORC_BC_PERIODIC)
            for (int q = ng; q < H - ng; ++q)
                for (int x = 0; x < ng; ++x) ZP(b, q, x) = BI(b, q - ng, nx - ng + x);
        if (bcs[1] == ORC_BC_PERIODIC)
            for (int q = ng; q < H - ng; ++q)
                for (int x = 0; x < ng; ++x) ZP(b, q, W - ng + x) = BI(b, q - ng, x);
        if (bcs[2] == ORC_BC_PERIODIC)
            for (int q = 0; q < ng; ++q)
                for (int x = ng; x < W - ng; ++x) ZP(b, q, x) = BI(b, ny - ng + q, x - ng);
        if (bcs[3] == ORC_BC_PERIODIC)
            for (int q = 0; q < ng; ++q)
                for (int x = ng; x < W - ng; ++x) ZP(b, H - ng + q, x) = BI(b, q, x - ng);
    }
    /* forced_h = clamp(level - zp, min=0), :270-282, evaluated lazily */
#define FORCED(b, q, x) FN(clamp_min)(level[b] - ZP(bedB == 1 ? 0 : (b), q, x), (R)0)
    R g981 = (R)9.81, lim = (R)1e-4, hmin = (R)1e-6;
    for (int b = 0; b < B; ++b) {
        /* left, :301-328 */
        switch (bcs[0]) {
        case ORC_BC_PERIODIC:
            for (int ch = 0; ch < 3; ++ch)
                for (int q = ng; q < H - ng; ++q)
                    for (int x = 0; x < ng; ++x) UP(b, ch, q, x) = UI(b, ch, q - ng, nx - ng + x);
            break;
        case ORC_BC_CONSTANT:
            for (int ch = 0; ch < 3; ++ch)
                for (int q = 0; q < H; ++q)
                    for (int x = 0; x < ng; ++x) UP(b, ch, q, x) = cval[b];
            break;
        case ORC_BC_WATER_LEVEL:
            for (int q = 0; q < H; ++q)
                for (int x = 0; x < ng; ++x) UP(b, 0, q, x) = FORCED(b, q, x);
            break;
        case ORC_BC_WALL:
            for (int q = 0; q < H; ++q)
                for (int x = 0; x < ng; ++x) UP(b, 1, q, x) = -UP(b, 1, q, 2 * ng - 1 - x);
            break;
        case ORC_BC_ABSORBING:
            for (int q = 0; q < H; ++q)
                for (int x = 0; x < ng; ++x) {
                    R hg = UP(b, 0, q, x), hr = FORCED(b, q, x);
                    R hc = hr > lim ? hr : hg;
                    R c = (R)sqrt(g981 * FN(clamp_min)(hc, hmin));
                    UP(b, 1, q, x) = -c * (hg - hr);
                }
            break;
        default: break;
        }
        /* right, :336-357 */
        switch (bcs[1]) {
        case ORC_BC_PERIODIC:
            for (int ch = 0; ch < 3; ++ch)
                for (int q = ng; q < H - ng; ++q)
                    for (int x = 0; x < ng; ++x) UP(b, ch, q, W - ng + x) = UI(b, ch, q - ng, x);
            break;
        case ORC_BC_CONSTANT:
            for (int ch = 0; ch < 3; ++ch)
                for (int q = 0; q < H; ++q)
                    for (int x = W - ng; x < W; ++x) UP(b, ch, q, x) = cval[b];
            break;
        case ORC_BC_WATER_LEVEL:
            for (int q = 0; q < H; ++q)
                for (int x = W - ng; x < W; ++x) UP(b, 0, q, x) = FORCED(b, q, x);
            break;
        case ORC_BC_WALL:
            for (int q = 0; q < H; ++q)
                for (int x = W - ng; x < W; ++x) UP(b, 1, q, x) = -UP(b, 1, q, 2 * (W - ng) - 1 - x);
            break;
        case ORC_BC_ABSORBING:
            for (int q = 0; q < H; ++q)
                for (int x = W - ng; x < W; ++x) {
                    R hg = UP(b, 0, q, x), hr = FORCED(b, q, x);
                    R hc = hr > lim ? hr : hg;
                    R c = (R)sqrt(g981 * FN(clamp_min)(hc, hmin));
                    UP(b, 1, q, x) = c * (hg - hr);
                }
            break;
        default: break;
        }
        /* top, :363-384 */
        switch (bcs[2]) {
        case ORC_BC_PERIODIC:
            for (int ch = 0; ch < 3; ++ch)
                for (int q = 0; q < ng; ++q)
                    for (int x = ng; x < W - ng; ++x) UP(b, ch, q, x) = UI(b, ch, ny - ng + q, x - ng);
            break;
        case ORC_BC_CONSTANT:
            for (int ch = 0; ch < 3; ++ch)
                for (int q = 0; q < ng; ++q)
                    for (int x = 0; x < W; ++x) UP(b, ch, q, x) = cval[b];
            break;
        case ORC_BC_WATER_LEVEL:
            for (int q = 0; q < ng; ++q)
                for (int x = 0; x < W; ++x) UP(b, 0, q, x) = FORCED(b, q, x);
            break;
        case ORC_BC_WALL:
            for (int q = 0; q < ng; ++q)
                for (int x = 0; x < W; ++x) UP(b, 2, q, x) = -UP(b, 2, 2 * ng - 1 - q, x);
            break;
        case ORC_BC_ABSORBING:
            for (int q = 0; q < ng; ++q)
                for (int x = 0; x < W; ++x) {
                    R hg = UP(b, 0, q, x), hr = FORCED(b, q, x);
                    R hc = hr > lim ? hr : hg;
                    R c = (R)sqrt(g981 * FN(clamp_min)(hc, hmin));
                    UP(b, 2, q, x) = -c * (hg - hr);
                }
            break;
        default: break;
        }
        /* bottom, :390-411 */
        switch (bcs[3]) {
        case ORC_BC_PERIODIC:
            for (int ch = 0; ch < 3; ++ch)
                for (int q = 0; q < ng; ++q)
                    for (int x = ng; x < W - ng; ++x) UP(b, ch, H - ng + q, x) = UI(b, ch, q, x - ng);
            break;
        case ORC_BC_CONSTANT:
            for (int ch = 0; ch < 3; ++ch)
                for (int q = H - ng; q < H; ++q)
                    for (int x = 0; x < W; ++x) UP(b, ch, q, x) = cval[b];
            break;
        case ORC_BC_WATER_LEVEL:
            for (int q = H - ng; q < H; ++q)
                for (int x = 0; x < W; ++x) UP(b, 0, q, x) = FORCED(b, q, x);
            break;
        case ORC_BC_WALL:
            for (int q = H - ng; q < H; ++q)
                for (int x = 0; x < W; ++x) UP(b, 2, q, x) = -UP(b, 2, 2 * (H - ng) - 1 - q, x);
            break;
        case ORC_BC_ABSORBING:
            for (int q = H - ng; q < H; ++q)
                for (int x = 0; x < W; ++x) {
                    R hg = UP(b, 0, q, x), hr = FORCED(b, q, x);
                    R hc = hr > lim ? hr : hg;
                    R c = (R)sqrt(g981 * FN(clamp_min)(hc, hmin));
                    UP(b, 2, q, x) = c * (hg - hr);
                }
            break;
        default: break;
        }
    }
#undef FORCED
#undef UP
#undef ZP
#undef UI
#undef BI
    return 0;
}

/* bflood_cn_reconstruction, src/reconstruction.py:18-108, for one line of
 * length W (elements at stride `st`).  Work arrays hold W values each. */
static void FN(recon_line)(const R* U0, const R* U1, const R* U2, const R* z, long st, int W,
                           const orc_params* p, R* w, R* UL0, R* UL1, R* UL2, R* UR0, R* UR1,
                           R* UR2, R* sL, R* sR) {
    R g = (R)p->gravity, dry = (R)p->dry_depth, th = (R)p->theta;
    R fl = (R)FN(depth_floor)(p->epsilon, p->dry_depth);
    R* h = w;
    R* u = w + W;
    R* v = w + 2 * W;
    R* eta = w + 3 * W;
    R* zz = w + 4 * W;
    R* dh = w + 5 * W;
    R* deta = w + 6 * W;
    R* dz = w + 7 * W;
    R* du = w + 8 * W;
    R* dv = w + 9 * W;
    for (int k = 0; k < W; ++k) {
        R c;
        FN(primitive1)(U0[k * st], U1[k * st], U2[k * st], g, dry, fl, &h[k], &u[k], &v[k], &c);
        zz[k] = z[k * st];
        eta[k] = h[k] + zz[k]; /* :24 */
    }
    FN(limited_increment_line)(h, W, 1, th, dh, 1); /* :26-30 */
    FN(limited_increment_line)(eta, W, 1, th, deta, 1);
    FN(limited_increment_line)(zz, W, 1, th, dz, 1);
    FN(limited_increment_line)(u, W, 1, th, du, 1);
    FN(limited_increment_line)(v, W, 1, th, dv, 1);
    if (p->water_slope_reset) { /* :32-42 */
        for (int k = 0; k < W; ++k) {
            R em = eta[(k - 1 + W) % W], ep = eta[(k + 1) % W];
            R half = (R)0.5 * (deta[k] - dh[k]);
            R bm = (eta[k] - h[k]) - half;
            R bp = (eta[k] - h[k]) + half;
            int reset = (deta[k] * deta[k] > dz[k] * dz[k]) && ((bm > em) || (bp > ep));
            if (reset) deta[k] = dh[k] + dz[k];
        }
    }
    R halfg = (R)(0.5 * p->gravity);
    for (int k = 0; k < W; ++k) {
        int n = (k + 1) % W;
        R hlL = h[k] + (R)0.5 * dh[k]; /* :50-51 */
        R hlR = h[n] - (R)0.5 * dh[n];
        R eL = eta[k] + (R)0.5 * deta[k]; /* :53-54 */
        R eR = eta[n] - (R)0.5 * deta[n];
        R bL = zz[k] + (R)0.5 * dz[k]; /* :56-57 */
        R bR = zz[n] - (R)0.5 * dz[n];
        R baud = FN(tmax)(bL, bR); /* :59-60 */
        R bcn = FN(tmin)(baud, FN(tmin)(eL, eR));
        R hcL = FN(clamp_min)(FN(tmin)(eL - bcn, hlL), (R)0); /* :62-69 */
        R hcR = FN(clamp_min)(FN(tmin)(eR - bcn, hlR), (R)0);
        R sfL = FN(clamp_min)(h[k], fl); /* :71-73 */
        R sfR = FN(clamp_min)(h[n], fl);
        R fLr = (R)1 - ((R)0.5 * dh[k]) / sfL; /* :75-76 */
        R fRr = (R)1 + ((R)0.5 * dh[n]) / sfR;
        R fL = h[k] > dry ? fLr : (R)1; /* :78-87 */
        R fR = h[n] > dry ? fRr : (R)1;
        fL = FN(clamp_max)(FN(clamp_min)(fL, (R)-10), (R)10); /* :90-91 */
        fR = FN(clamp_max)(FN(clamp_min)(fR, (R)-10), (R)10);
        R uL = u[k] + ((R)0.5 * fL) * du[k]; /* :93-96 */
        R vL = v[k] + ((R)0.5 * fL) * dv[k];
        R uR = u[n] - ((R)0.5 * fR) * du[n];
        R vR = v[n] - ((R)0.5 * fR) * dv[n];
        UL0[k * st] = hcL; /* :98-99 */
        UL1[k * st] = hcL * uL;
        UL2[k * st] = hcL * vL;
        UR0[k * st] = hcR;
        UR1[k * st] = hcR * uR;
        UR2[k * st] = hcR * vR;
        sL[k * st] = (halfg * (h[k] + hcL)) * (zz[k] - bcn); /* :101-106 */
        sR[k * st] = (halfg * (hcR + h[n])) * (zz[n] - bcn);
    }
}

int FN(orc_reconstruction)(const R* Up, const R* zp, int B, int zB, int H, int W, int dim,
                           const orc_params* p, R* UL, R* UR, R* sL, R* sR) {
    long plane = (long)H * W;
    int nlines = dim == -1 ? H : W, len = dim == -1 ? W : H;
    long st = dim == -1 ? 1 : W;
    R* work = (R*)malloc(sizeof(R) * 10 * (size_t)len * (size_t)(B * nlines));
    if (!work) return 1;
#pragma omp parallel for collapse(2) schedule(static)
    for (int b = 0; b < B; ++b)
        for (int line = 0; line < nlines; ++line) {
            long off = dim == -1 ? (long)line * W : line;
            const R* Ub = Up + (long)b * 3 * plane;
            const R* zb = zp + (long)(zB == 1 ? 0 : b) * plane;
            R* ULb = UL + (long)b * 3 * plane;
            R* URb = UR + (long)b * 3 * plane;
            FN(recon_line)(Ub + off, Ub + plane + off, Ub + 2 * plane + off, zb + off, st, len, p,
                           work + (size_t)10 * len * ((size_t)b * nlines + line), ULb + off,
                           ULb + plane + off, ULb + 2 * plane + off, URb + off, URb + plane + off,
                           URb + 2 * plane + off, sL + (long)b * plane + off, sR + (long)b * plane + off);
        }
    free(work);
    return 0;
}

/* bflood_hllc_flux, src/riemann.py:41-105, one face. */
static inline void FN(hll1)(R L0, R L1, R L2, R R0, R R1, R R2, int normal_y, R g, R dry, R fl,
                            R den_floor, R halfg, R* F0, R* F1, R* F2, R* speed) {
    R hL, uL, vL, cL, hR, uR, vR, cR;
    FN(primitive1)(L0, L1, L2, g, dry, fl, &hL, &uL, &vL, &cL);
    FN(primitive1)(R0, R1, R2, g, dry, fl, &hR, &uR, &vR, &cR);
    R unL = normal_y ? vL : uL, utL = normal_y ? uL : vL; /* :60-61 */
    R unR = normal_y ? vR : uR, utR = normal_y ? uR : vR;
    R us = ((R)0.5 * (unL + unR) + cL) - cR; /* :63-64 */
    R cs = (R)0.5 * (cL + cR) + (R)0.25 * (unL - unR);
    R SLw = FN(tmin)(unL - cL, us - cs); /* :66-67 */
    R SRw = FN(tmax)(unR + cR, us + cs);
    int ldry = hL <= dry, rdry = hR <= dry; /* :69-70 */
    R SL = ldry ? unR - (R)2 * cR : SLw; /* :72-73 */
    R SR = rdry ? unL + (R)2 * cL : SRw;
    R fhL = hL * unL, fhR = hR * unR; /* :75-77 */
    R fqL = hL * (unL * unL + halfg * hL);
    R fqR = hR * (unR * unR + halfg * hR);
    R den = FN(clamp_min)(SR - SL, den_floor); /* :79 */
    R fhs = ((SR * fhL - SL * fhR) + (SL * SR) * (hR - hL)) / den; /* :80-82 */
    R fqs = ((SR * fqL - SL * fqR) + (SL * SR) * (hR * unR - hL * unL)) / den; /* :83-86 */
    int lf = SL >= 0, rf = SR <= 0; /* :88-89 */
    R fh = lf ? fhL : (rf ? fhR : fhs);
    R fq = lf ? fqL : (rf ? fqR : fqs);
    R ft = (fh > 0 ? utL : utR) * fh; /* :97 */
    int both = ldry && rdry; /* :105-106 */
    if (both) { fh = 0; fq = 0; ft = 0; }
    *F0 = fh;
    *F1 = normal_y ? ft : fq;
    *F2 = normal_y ? fq : ft;
    R sp = FN(tmax)(FN(tabs)(SL), FN(tabs)(SR)); /* :108-111 */
    *speed = both ? (R)0 : sp;
}

int FN(orc_hll_flux)(const R* UL, const R* UR, int B, int H, int W, int normal_y, const orc_params* p,
                     R* flux, R* speed) {
    long plane = (long)H * W;
    R g = (R)p->gravity, dry = (R)p->dry_depth, fl = (R)FN(depth_floor)(p->epsilon, p->dry_depth);
    double pf = FN(precision_floor)();
    R den_floor = (R)(p->epsilon > pf ? p->epsilon : pf);
    R halfg = (R)(0.5 * p->gravity);
#pragma omp parallel for schedule(static)
    for (int b = 0; b < B; ++b)
        for (long i = 0; i < plane; ++i) {
            const R* L = UL + (long)b * 3 * plane;
            const R* Rr = UR + (long)b * 3 * plane;
            R* F = flux + (long)b * 3 * plane;
            FN(hll1)(L[i], L[plane + i], L[2 * plane + i], Rr[i], Rr[plane + i], Rr[2 * plane + i],
                     normal_y, g, dry, fl, den_floor, halfg, &F[i], &F[plane + i], &F[2 * plane + i],
                     &speed[(long)b * plane + i]);
        }
    return 0;
}

/* SWE2D.spatial_operator, src/solver.py:448-531, with return_wave_speed.
 * rain and infil are per-cell [B,1,ny,nx] arrays or NULL. */
int FN(orc_spatial_operator)(const R* U, const R* bed, int B, int bedB, int ny, int nx,
                             const orc_params* p, const R* level, const R* rain, const R* infil,
                             R* rhs, R* ax, R* ay) {
    int ng = 2, H = ny + 4, W = nx + 4;
    long plane = (long)H * W, iplane = (long)ny * nx;
    size_t n3 = (size_t)B * 3 * plane, n1 = (size_t)B * plane;
    R* Up = (R*)malloc(sizeof(R) * n3);
    R* zp = (R*)malloc(sizeof(R) * (size_t)bedB * plane);
    R* ULx = (R*)malloc(sizeof(R) * n3);
    R* URx = (R*)malloc(sizeof(R) * n3);
    R* ULy = (R*)malloc(sizeof(R) * n3);
    R* URy = (R*)malloc(sizeof(R) * n3);
    R* sxL = (R*)malloc(sizeof(R) * n1);
    R* sxR = (R*)malloc(sizeof(R) * n1);
    R* syL = (R*)malloc(sizeof(R) * n1);
    R* syR = (R*)malloc(sizeof(R) * n1);
    R* Fx = (R*)malloc(sizeof(R) * n3);
    R* Gy = (R*)malloc(sizeof(R) * n3);
    R* axf = (R*)malloc(sizeof(R) * n1);
    R* ayf = (R*)malloc(sizeof(R) * n1);
    R* cval = (R*)malloc(sizeof(R) * (size_t)B);
    int rc = 1;
    if (cval)
        for (int b = 0; b < B; ++b) cval[b] = (R)p->constant_value;
    if (!Up || !zp || !ULx || !URx || !ULy || !URy || !sxL || !sxR || !syL || !syR || !Fx || !Gy ||
        !axf || !ayf || !cval)
        goto done;
    FN(orc_ghost_cells)(U, bed, B, bedB, ny, nx, ng, p, level, cval, Up, zp); /* :474-484 */
    FN(orc_reconstruction)(Up, zp, B, bedB, H, W, -1, p, ULx, URx, sxL, sxR); /* :493-494 */
    FN(orc_reconstruction)(Up, zp, B, bedB, H, W, -2, p, ULy, URy, syL, syR);
    FN(orc_hll_flux)(ULx, URx, B, H, W, 0, p, Fx, axf); /* :496-501 */
    FN(orc_hll_flux)(ULy, URy, B, H, W, 1, p, Gy, ayf);
    {
        R dxr = (R)p->dx, dyr = (R)p->dy;
        R axm = 0, aym = 0;
        int first = 1;
        for (int b = 0; b < B; ++b) {
            const R* F = Fx + (long)b * 3 * plane;
            const R* G = Gy + (long)b * 3 * plane;
            const R* sxl = sxL + (long)b * plane;
            const R* sxr = sxR + (long)b * plane;
            const R* syl = syL + (long)b * plane;
            const R* syr = syR + (long)b * plane;
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) {
                    int q = j + 2, x = i + 2;
                    long cidx = (long)q * W + x;
                    long fxm = cidx - 1, fym = cidx - W; /* faces x-1/2 and y-1/2 */
                    R out[3];
                    for (int ch = 0; ch < 3; ++ch) {
                        /* Fx_right[:, :, 2:2+ny, 1:1+nx] - Fx_left[:, :, 2:2+ny, 2:2+nx], :504-514 */
                        R fr = F[ch * plane + fxm], flf = F[ch * plane + cidx];
                        if (ch == 1) { fr = fr - sxr[fxm]; flf = flf - sxl[cidx]; }
                        R r = (fr - flf) / dxr;
                        /* Gy_top[:, :, 1:1+ny, 2:2+nx] - Gy_bottom[:, :, 2:2+ny, 2:2+nx], :515-518 */
                        R gt = G[ch * plane + fym], gb = G[ch * plane + cidx];
                        if (ch == 2) { gt = gt - syr[fym]; gb = gb - syl[cidx]; }
                        R s = (gt - gb) / dyr;
                        out[ch] = r + s;
                    }
                    long o = (long)j * nx + i;
                    R rn = rain ? rain[(long)b * iplane + o] : (R)0; /* :520-525 */
                    R ls = infil ? FN(clamp_min)(infil[(long)b * iplane + o], (R)0) : (R)0;
                    rhs[((long)b * 3 + 0) * iplane + o] = (out[0] + rn) - ls;
                    rhs[((long)b * 3 + 1) * iplane + o] = out[1];
                    rhs[((long)b * 3 + 2) * iplane + o] = out[2];
                }
            /* ax[:, :, 2:2+ny, 1:2+nx].amax(), ay[:, :, 1:2+ny, 2:2+nx].amax(), :527-530 */
            for (int q = 2; q < 2 + ny; ++q)
                for (int x = 1; x < 2 + nx; ++x) {
                    R s = axf[(long)b * plane + (long)q * W + x];
                    axm = first ? s : FN(tmax)(axm, s);
                    first = 0;
                }
        }
        first = 1;
        for (int b = 0; b < B; ++b)
            for (int q = 1; q < 2 + ny; ++q)
                for (int x = 2; x < 2 + nx; ++x) {
                    R s = ayf[(long)b * plane + (long)q * W + x];
                    aym = first ? s : FN(tmax)(aym, s);
                    first = 0;
                }
        *ax = axm;
        *ay = aym;
    }
    rc = 0;
done:
    free(Up); free(zp); free(ULx); free(URx); free(ULy); free(URy); free(sxL); free(sxR);
    free(syL); free(syR); free(Fx); free(Gy); free(axf); free(ayf); free(cval);
    return rc;
}

/* SWE2D._clean_and_limit, src/solver.py:547-570 */
int FN(orc_clean_and_limit)(const R* old, const R* cand, int B, int ny, int nx, const orc_params* p, R* out) {
    long ip = (long)ny * nx;
    R eps = (R)p->epsilon, dry = (R)p->dry_depth;
#pragma omp parallel for schedule(static)
    for (int b = 0; b < B; ++b)
        for (long i = 0; i < ip; ++i) {
            const R* o = old + (long)b * 3 * ip;
            const R* c = cand + (long)b * 3 * ip;
            R c0 = c[i], c1 = c[ip + i], c2 = c[2 * ip + i];
            if (p->positivity_limiter) {
                R d0 = c0 - o[i], d1 = c1 - o[ip + i], d2 = c2 - o[2 * ip + i];
                R safe = FN(clamp_min)(-d0, eps);
                R th = d0 < 0 ? FN(clamp_max)(o[i] / safe, (R)1) : (R)1;
                c0 = o[i] + th * d0;
                c1 = o[ip + i] + th * d1;
                c2 = o[2 * ip + i] + th * d2;
            }
            R h = FN(clamp_min)(c0, (R)0);
            int wet = h > dry;
            R* ob = out + (long)b * 3 * ip;
            ob[i] = h;
            ob[ip + i] = wet ? c1 : (R)0;
            ob[2 * ip + i] = wet ? c2 : (R)0;
        }
    return 0;
}

/* pow(x, (R)(1/3)) correctly rounded in R.  The reference's CPU pow agrees
 * with this value except for an ulp on a small fraction of inputs. */
static inline R FN(cbrt_pow)(R x) { return (R)pow((double)x, (double)(R)(1.0 / 3.0)); }

/* apply_manning_friction, src/friction.py:102-131 (+ :12-38, :62-66) */
int FN(orc_manning)(const R* U, const R* n, int B, int nB, int ny, int nx, R dt, double dry_depth,
                    double epsilon, R* out) {
    long ip = (long)ny * nx;
    double pf = FN(precision_floor)();
    double f_vs = FN(depth_floor)(epsilon, dry_depth); /* _floor(h, eps, dry) */
    double f_e = epsilon > pf ? epsilon : pf;          /* _floor(h, eps) */
    if (0.0 > f_e) f_e = 0.0;
    R dry = (R)dry_depth, fvs = (R)f_vs, fe = (R)f_e, fe2 = (R)(f_e * f_e), g981 = (R)9.81;
#pragma omp parallel for schedule(static)
    for (int b = 0; b < B; ++b)
        for (long i = 0; i < ip; ++i) {
            const R* Ub = U + (long)b * 3 * ip;
            R h = FN(clamp_min)(Ub[i], (R)0), hu = Ub[ip + i], hv = Ub[2 * ip + i];
            int wet = h > dry;
            R safe = FN(clamp_min)(h, fvs);
            R u = (wet ? hu : (R)0) / safe;
            R v = (wet ? hv : (R)0) / safe;
            R sp2 = u * u + v * v;
            int moving = wet && (sp2 > 0);
            R speed = moving ? (R)sqrt(FN(clamp_min)(sp2, fe2)) : (R)0;
            R nn = FN(clamp_min)(n[(long)(nB == 1 ? 0 : b) * ip + i], (R)0);
            R cf = (g981 * (nn * nn)) / FN(cbrt_pow)(FN(clamp_min)(h, fe));
            R fac = (R)1 / ((R)1 + ((cf * speed) * dt) / safe);
            R* o = out + (long)b * 3 * ip;
            o[i] = h;
            o[ip + i] = wet ? hu * fac : (R)0;
            o[2 * ip + i] = wet ? hv * fac : (R)0;
        }
    return 0;
}

/* apply_roughness_length_friction, src/friction.py:69-99 (+ :41-59) */
int FN(orc_roughness_friction)(const R* U, const R* z0, int B, int nB, int ny, int nx, R dt,
                               double dry_depth, double epsilon, R* out) {
    long ip = (long)ny * nx;
    double pf = FN(precision_floor)();
    double f_vs = FN(depth_floor)(epsilon, dry_depth);
    double f_e = epsilon > pf ? epsilon : pf;
    R dry = (R)dry_depth, fvs = (R)f_vs, fe = (R)f_e, fe2 = (R)(f_e * f_e);
    R c046 = (R)0.46, c25 = (R)2.5, c1359 = (R)1.359, e = (R)2.718281828459045;
#pragma omp parallel for schedule(static)
    for (int b = 0; b < B; ++b)
        for (long i = 0; i < ip; ++i) {
            const R* Ub = U + (long)b * 3 * ip;
            R h = FN(clamp_min)(Ub[i], (R)0), hu = Ub[ip + i], hv = Ub[2 * ip + i];
            int wet = h > dry;
            R safe = FN(clamp_min)(h, fvs);
            R u = (wet ? hu : (R)0) / safe;
            R v = (wet ? hv : (R)0) / safe;
            R sp2 = u * u + v * v;
            int moving = wet && (sp2 > 0);
            R speed = moving ? (R)sqrt(FN(clamp_min)(sp2, fe2)) : (R)0;
            R zz = FN(clamp_min)(z0[(long)(nB == 1 ? 0 : b) * ip + i], fe);
            R ratio = FN(clamp_min)(h, fe) / zz;
            R shallow = (R)1 / FN(clamp_min)(c046 * ratio, fe);
            R rc = FN(clamp_min)(ratio, fe);
            R lt = c25 * (((R)log((double)rc) - (R)1) + ((R)1 / rc) * c1359);
            R deep = (R)1 / FN(clamp_min)(lt * lt, fe);
            R cf = ratio < e ? shallow : deep;
            R fac = (R)1 / ((R)1 + ((cf * speed) * dt) / safe);
            R* o = out + (long)b * 3 * ip;
            o[i] = h;
            o[ip + i] = wet ? hu * fac : (R)0;
            o[2 * ip + i] = wet ? hv * fac : (R)0;
        }
    return 0;
}

/* SWE2D.step, src/solver.py:572-663.  level holds B values.  rain0 / rain1
 * (the rainfall rate of stage 1 and of stage 2, :609-643) and infil are
 * per-cell [B,1,ny,nx] arrays or NULL.  *dt_out receives dt in R. */
int FN(orc_step_forced)(const R* U, const R* bed, int bedB, const R* n, int nB, int B, int ny,
                        int nx, const orc_params* p, const R* level, R max_dt, const R* rain0,
                        const R* rain1, const R* infil, R* U_out, R* dt_out) {
    size_t n3 = (size_t)B * 3 * ny * nx;
    R* k = (R*)malloc(sizeof(R) * n3);
    R* cand = (R*)malloc(sizeof(R) * n3);
    R* pred = (R*)malloc(sizeof(R) * n3);
    int rc = 1;
    if (!k || !cand || !pred) goto done;
    R ax, ay;
    if (FN(orc_spatial_operator)(U, bed, B, bedB, ny, nx, p, level, rain0, infil, k, &ax, &ay)) goto done;
    {
        /* :620-626: denominator = clamp(ax/dx + ay/dy, min=eps); cfl/den is
         * den.reciprocal() * cfl in PyTorch; dt = minimum(stable, max_dt). */
        R den = FN(clamp_min)(ax / (R)p->dx + ay / (R)p->dy, (R)p->epsilon);
        R stable = ((R)1 / den) * (R)p->cfl;
        R dt = FN(tmin)(stable, max_dt);
        *dt_out = dt;
        if (!(dt == dt) || dt == (R)INFINITY || dt == -(R)INFINITY) { rc = 2; goto done; }
        if (!(dt > 0)) { rc = 3; goto done; }
        R hdt = (R)0.5 * dt; /* :639 */
        for (size_t i = 0; i < n3; ++i) cand[i] = U[i] + hdt * k[i];
        FN(orc_clean_and_limit)(U, cand, B, ny, nx, p, pred);
        if (FN(orc_spatial_operator)(pred, bed, B, bedB, ny, nx, p, level, rain1, infil, k, &ax, &ay)) goto done;
        for (size_t i = 0; i < n3; ++i) cand[i] = U[i] + dt * k[i]; /* :646 */
        if (p->apply_friction) {
            FN(orc_clean_and_limit)(U, cand, B, ny, nx, p, pred);
            if (p->friction_model == 0)
                FN(orc_manning)(pred, n, B, nB, ny, nx, dt, p->dry_depth, p->epsilon, U_out);
            else
                FN(orc_roughness_friction)(pred, n, B, nB, ny, nx, dt, p->dry_depth, p->epsilon, U_out);
        } else {
            FN(orc_clean_and_limit)(U, cand, B, ny, nx, p, U_out);
        }
    }
    rc = 0;
done:
    free(k); free(cand); free(pred);
    return rc;
}

/* The step without rainfall. */
int FN(orc_step)(const R* U, const R* bed, int bedB, const R* n, int nB, int B, int ny, int nx,
                 const orc_params* p, const R* level, R max_dt, const R* infil, R* U_out, R* dt_out) {
    return FN(orc_step_forced)(U, bed, bedB, n, nB, B, ny, nx, p, level, max_dt, NULL, NULL, infil,
                               U_out, dt_out);
}

#undef FN
#undef CAT
#undef CAT2
