/*
 * orc_markers.c -- TEST INFRASTRUCTURE (CPU oracle).  Restatement of the reference's marker
 * operations in plain C, single-threaded:
 *
 *   cell search ............ m1serch/m2serch/m3serch  mark3mg.c:1021-1087
 *   velocity at a point .... vxyzcalc1                mark3mg.c:2347-2530
 *   strain rate/stress ..... epscalc1                 mark3mg.c:2535-2838
 *   temperature ............ tkcalc1                  mark3mg.c:2844-2910
 *   pressure ............... prcalc1                  mark3mg.c:2917-3001
 *   density ................ dencalc1                 mark3mg.c:3006-3024
 *   viscosity .............. viscalc (rheologies A-F + brittle) mark3mg.c:1114-1693
 *   RK4 advection .......... movemark                 mark3mg.c:2-397 (rock markers)
 *   marker -> node ......... ronurecalc               mark3mg.c:404-1015
 *   temperature boundaries . tkrecalc                 heat3mg.c:849-899
 *
 * The marker -> node sums are accumulated in FP64 (the reference accumulates most of them
 * in its FP32 node arrays, in racy OpenMP order); results are normalised and stored as FP32.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "orc_internal.h"

#define MAXV(a, b) ((a) >= (b) ? (a) : (b))
#define ABSV(a) ((a) >= 0 ? (a) : -(a))

enum { R_N0, R_N1, R_S0, R_S1, R_NU, R_DH, R_DV, R_SS, R_MM, R_LL, R_A0, R_A1, R_B0, R_B1, R_E0, R_E1,
       R_RO, R_BB, R_AA, R_CP, R_KT, R_KF, R_KP, R_HT };

static long bsearch_g(const double *g, long n, double x)
{
    long a = 0, b = n - 1, m;
    do {
        m = (a + b) / 2;
        if (g[m] > x) b = m; else a = m;
    } while ((b - a) > 1);
    if (a > n - 2) a = n - 2;
    return a;
}
long orc_m1serch(const orc_ctx *o, double x) { return bsearch_g(o->gx, o->nx, x); }
long orc_m2serch(const orc_ctx *o, double y) { return bsearch_g(o->gy, o->ny, y); }
long orc_m3serch(const orc_ctx *o, double z) { return bsearch_g(o->gz, o->nz, z); }

/* vxyzcalc1: staggered trilinear velocity (mark3mg.c:2347-2530) */
void orc_vxyz(const orc_ctx *o, double x, double y, double z, double *v, long *wn)
{
    const double *gx = o->gx, *gy = o->gy, *gz = o->gz;
    long X = o->nx, Y = o->ny, Z = o->nz, XY = X * Y;
    v[0] = v[1] = v[2] = 0;
    if (x < 0) x = 0; if (x > o->m.xsize) x = o->m.xsize;
    if (y < 0) y = 0; if (y > o->m.ysize) y = o->m.ysize;
    if (z < 0) z = 0; if (z > o->m.zsize) z = o->m.zsize;
    long m1 = wn[0] = orc_m1serch(o, x), m2 = wn[1] = orc_m2serch(o, y), m3 = wn[2] = orc_m3serch(o, z);
    long a, b, c, k1, k2, k3;
    double dx, dy, dz, ddx, ddy, ddz;
    /* Vx */
    a = m1; if (a < 0) a = 0; if (a > X - 2) a = X - 2;
    b = m2; if (y < (gy[b] + gy[b + 1]) / 2.0) b -= 1; if (b < 0) b = 0; if (b > Y - 3) b = Y - 3;
    c = m3; if (z < (gz[c] + gz[c + 1]) / 2.0) c -= 1; if (c < 0) c = 0; if (c > Z - 3) c = Z - 3;
    dx = gx[a + 1] - gx[a]; dy = (gy[b + 2] - gy[b]) / 2.0; dz = (gz[c + 2] - gz[c]) / 2.0;
    for (k3 = c; k3 <= c + 1; k3++) {
        ddz = ((gz[k3] + gz[k3 + 1]) / 2.0 - z) / dz; if (k3 == c) ddz = -ddz; ddz = 1.0 - ddz;
        for (k1 = a; k1 <= a + 1; k1++) {
            ddx = (gx[k1] - x) / dx; if (k1 == a) ddx = -ddx; ddx = 1.0 - ddx;
            for (k2 = b; k2 <= b + 1; k2++) {
                ddy = ((gy[k2] + gy[k2 + 1]) / 2.0 - y) / dy; if (k2 == b) ddy = -ddy; ddy = 1.0 - ddy;
                v[0] += o->vx[k3 * XY + k1 * Y + k2] * (ddx * ddy * ddz);
            }
        }
    }
    /* Vy */
    a = m1; if (x < (gx[a] + gx[a + 1]) / 2.0) a -= 1; if (a < 0) a = 0; if (a > X - 3) a = X - 3;
    b = m2; if (b < 0) b = 0; if (b > Y - 2) b = Y - 2;
    c = m3; if (z < (gz[c] + gz[c + 1]) / 2.0) c -= 1; if (c < 0) c = 0; if (c > Z - 3) c = Z - 3;
    dx = (gx[a + 2] - gx[a]) / 2.0; dy = gy[b + 1] - gy[b]; dz = (gz[c + 2] - gz[c]) / 2.0;
    for (k3 = c; k3 <= c + 1; k3++) {
        ddz = ((gz[k3] + gz[k3 + 1]) / 2.0 - z) / dz; if (k3 == c) ddz = -ddz; ddz = 1.0 - ddz;
        for (k1 = a; k1 <= a + 1; k1++) {
            ddx = ((gx[k1] + gx[k1 + 1]) / 2.0 - x) / dx; if (k1 == a) ddx = -ddx; ddx = 1.0 - ddx;
            for (k2 = b; k2 <= b + 1; k2++) {
                ddy = (gy[k2] - y) / dy; if (k2 == b) ddy = -ddy; ddy = 1.0 - ddy;
                v[1] += o->vy[k3 * XY + k1 * Y + k2] * (ddx * ddy * ddz);
            }
        }
    }
    /* Vz */
    a = m1; if (x < (gx[a] + gx[a + 1]) / 2.0) a -= 1; if (a < 0) a = 0; if (a > X - 3) a = X - 3;
    b = m2; if (y < (gy[b] + gy[b + 1]) / 2.0) b -= 1; if (b < 0) b = 0; if (b > Y - 3) b = Y - 3;
    c = m3; if (c < 0) c = 0; if (c > Z - 2) c = Z - 2;
    dx = (gx[a + 2] - gx[a]) / 2.0; dy = (gy[b + 2] - gy[b]) / 2.0; dz = gz[c + 1] - gz[c];
    for (k3 = c; k3 <= c + 1; k3++) {
        ddz = (gz[k3] - z) / dz; if (k3 == c) ddz = -ddz; ddz = 1.0 - ddz;
        for (k1 = a; k1 <= a + 1; k1++) {
            ddx = ((gx[k1] + gx[k1 + 1]) / 2.0 - x) / dx; if (k1 == a) ddx = -ddx; ddx = 1.0 - ddx;
            for (k2 = b; k2 <= b + 1; k2++) {
                ddy = ((gy[k2] + gy[k2 + 1]) / 2.0 - y) / dy; if (k2 == b) ddy = -ddy; ddy = 1.0 - ddy;
                v[2] += o->vz[k3 * XY + k1 * Y + k2] * (ddx * ddy * ddz);
            }
        }
    }
}

static double clamp01(double d) { if (d < 0) d = 0; if (d > 1.0) d = 1.0; return d; }

/* epscalc1 with the cell given (mark3mg.c:2535-2838): e[0..6] = exx eyy ezz exy exz eyz P,
 * s[0..5] = sxx syy szz sxy sxz syz, *dis = dissipation */
static void eps_at(const orc_ctx *o, double x, double y, double z, const long *wn, double *e, double *s, double *dis)
{
    const double *gx = o->gx, *gy = o->gy, *gz = o->gz;
    long X = o->nx, Y = o->ny, Z = o->nz, XY = X * Y;
    for (int i = 0; i < 7; i++) e[i] = 0;
    for (int i = 0; i < 6; i++) s[i] = 0;
    *dis = 0;
    if (x < 0) x = 0; if (x > o->m.xsize) x = o->m.xsize;
    if (y < 0) y = 0; if (y > o->m.ysize) y = o->m.ysize;
    if (z < 0) z = 0; if (z > o->m.zsize) z = o->m.zsize;
    long m1 = wn[0], m2 = wn[1], m3 = wn[2], a, b, c, k1, k2, k3, n;
    double dx, dy, dz, ddx, ddy, ddz, w;
    /* normal components and P at cell centres */
    a = m1; if (x > (gx[a] + gx[a + 1]) / 2.0) a += 1; if (a < 1) a = 1; if (a > X - 2) a = X - 2;
    b = m2; if (y > (gy[b] + gy[b + 1]) / 2.0) b += 1; if (b < 1) b = 1; if (b > Y - 2) b = Y - 2;
    c = m3; if (z > (gz[c] + gz[c + 1]) / 2.0) c += 1; if (c < 1) c = 1; if (c > Z - 2) c = Z - 2;
    dx = (gx[a + 1] - gx[a - 1]) / 2.0; dy = (gy[b + 1] - gy[b - 1]) / 2.0; dz = (gz[c + 1] - gz[c - 1]) / 2.0;
    for (k3 = c; k3 <= c + 1; k3++) {
        ddz = ((gz[k3 - 1] + gz[k3]) / 2.0 - z) / dz; if (k3 == c) ddz = -ddz; ddz = clamp01(1.0 - ddz);
        for (k1 = a; k1 <= a + 1; k1++) {
            ddx = ((gx[k1 - 1] + gx[k1]) / 2.0 - x) / dx; if (k1 == a) ddx = -ddx; ddx = clamp01(1.0 - ddx);
            for (k2 = b; k2 <= b + 1; k2++) {
                ddy = ((gy[k2 - 1] + gy[k2]) / 2.0 - y) / dy; if (k2 == b) ddy = -ddy; ddy = clamp01(1.0 - ddy);
                n = k3 * XY + k1 * Y + k2;
                w = ddx * ddy * ddz;
                e[0] += o->exx[n] * w; e[1] += o->eyy[n] * w; e[2] += o->ezz[n] * w;
                s[0] += o->sxx[n] * w; s[1] += o->syy[n] * w; s[2] += o->szz[n] * w;
                *dis += (o->sxx[n] * o->exx[n] + o->syy[n] * o->eyy[n] + o->szz[n] * o->ezz[n]) * w;
                e[6] += o->pr[n] * w;
            }
        }
    }
    /* xy at z-edges */
    a = m1; if (a < 1) a = 1; if (a > X - 3) a = X - 3;
    b = m2; if (b < 1) b = 1; if (b > Y - 3) b = Y - 3;
    c = m3; if (z < (gz[c] + gz[c + 1]) / 2.0) c -= 1; if (c < 0) c = 0; if (c > Z - 3) c = Z - 3;
    dx = gx[a + 1] - gx[a]; dy = gy[b + 1] - gy[b]; dz = (gz[c + 2] - gz[c]) / 2.0;
    for (k3 = c; k3 <= c + 1; k3++) {
        ddz = ((gz[k3] + gz[k3 + 1]) / 2.0 - z) / dz; if (k3 == c) ddz = -ddz; ddz = clamp01(1.0 - ddz);
        for (k1 = a; k1 <= a + 1; k1++) {
            ddx = (gx[k1] - x) / dx; if (k1 == a) ddx = -ddx; ddx = clamp01(1.0 - ddx);
            for (k2 = b; k2 <= b + 1; k2++) {
                ddy = (gy[k2] - y) / dy; if (k2 == b) ddy = -ddy; ddy = clamp01(1.0 - ddy);
                n = k3 * XY + k1 * Y + k2;
                w = ddx * ddy * ddz;
                e[3] += o->exy[n] * w; s[3] += o->sxy[n] * w;
                *dis += 2.0 * o->sxy[n] * o->exy[n] * w;
            }
        }
    }
    /* xz at y-edges */
    a = m1; if (a < 1) a = 1; if (a > X - 3) a = X - 3;
    b = m2; if (y < (gy[b] + gy[b + 1]) / 2.0) b -= 1; if (b < 0) b = 0; if (b > Y - 3) b = Y - 3;
    c = m3; if (c < 1) c = 1; if (c > Z - 3) c = Z - 3;
    dx = gx[a + 1] - gx[a]; dy = (gy[b + 2] - gy[b]) / 2.0; dz = gz[c + 1] - gz[c];
    for (k3 = c; k3 <= c + 1; k3++) {
        ddz = (gz[k3] - z) / dz; if (k3 == c) ddz = -ddz; ddz = clamp01(1.0 - ddz);
        for (k1 = a; k1 <= a + 1; k1++) {
            ddx = (gx[k1] - x) / dx; if (k1 == a) ddx = -ddx; ddx = clamp01(1.0 - ddx);
            for (k2 = b; k2 <= b + 1; k2++) {
                ddy = ((gy[k2] + gy[k2 + 1]) / 2.0 - y) / dy; if (k2 == b) ddy = -ddy; ddy = clamp01(1.0 - ddy);
                n = k3 * XY + k1 * Y + k2;
                w = ddx * ddy * ddz;
                e[4] += o->exz[n] * w; s[4] += o->sxz[n] * w;
                *dis += 2.0 * o->sxz[n] * o->exz[n] * w;
            }
        }
    }
    /* yz at x-edges */
    a = m1; if (x < (gx[a] + gx[a + 1]) / 2.0) a -= 1; if (a < 0) a = 0; if (a > X - 3) a = X - 3;
    b = m2; if (b < 1) b = 1; if (b > Y - 3) b = Y - 3;
    c = m3; if (c < 1) c = 1; if (c > Z - 3) c = Z - 3;
    dx = (gx[a + 2] - gx[a]) / 2.0; dy = gy[b + 1] - gy[b]; dz = gz[c + 1] - gz[c];
    for (k3 = c; k3 <= c + 1; k3++) {
        ddz = (gz[k3] - z) / dz; if (k3 == c) ddz = -ddz; ddz = clamp01(1.0 - ddz);
        for (k1 = a; k1 <= a + 1; k1++) {
            ddx = ((gx[k1] + gx[k1 + 1]) / 2.0 - x) / dx; if (k1 == a) ddx = -ddx; ddx = clamp01(1.0 - ddx);
            for (k2 = b; k2 <= b + 1; k2++) {
                ddy = (gy[k2] - y) / dy; if (k2 == b) ddy = -ddy; ddy = clamp01(1.0 - ddy);
                n = k3 * XY + k1 * Y + k2;
                w = ddx * ddy * ddz;
                e[5] += o->eyz[n] * w; s[5] += o->syz[n] * w;
                *dis += 2.0 * o->syz[n] * o->eyz[n] * w;
            }
        }
    }
}

/* prcalc1 (mark3mg.c:2917-3001) */
static double pr_at(const orc_ctx *o, double x, double y, double z, long *wn)
{
    const double *gx = o->gx, *gy = o->gy, *gz = o->gz;
    long X = o->nx, Y = o->ny, Z = o->nz, XY = X * Y;
    if (x < 0) x = 0; if (x > o->m.xsize) x = o->m.xsize;
    if (y < 0) y = 0; if (y > o->m.ysize) y = o->m.ysize;
    if (z < 0) z = 0; if (z > o->m.zsize) z = o->m.zsize;
    long m1 = wn[0] = orc_m1serch(o, x), m2 = wn[1] = orc_m2serch(o, y), m3 = wn[2] = orc_m3serch(o, z);
    long a, b, c, k1, k2, k3;
    a = m1; if (x > (gx[a] + gx[a + 1]) / 2.0) a += 1; if (a < 1) a = 1; if (a > X - 2) a = X - 2;
    b = m2; if (y > (gy[b] + gy[b + 1]) / 2.0) b += 1; if (b < 1) b = 1; if (b > Y - 2) b = Y - 2;
    c = m3; if (z > (gz[c] + gz[c + 1]) / 2.0) c += 1; if (c < 1) c = 1; if (c > Z - 2) c = Z - 2;
    double dx = (gx[a + 1] - gx[a - 1]) / 2.0, dy = (gy[b + 1] - gy[b - 1]) / 2.0, dz = (gz[c + 1] - gz[c - 1]) / 2.0;
    double p = 0, ddx, ddy, ddz;
    for (k3 = c; k3 <= c + 1; k3++) {
        ddz = ((gz[k3 - 1] + gz[k3]) / 2.0 - z) / dz; if (k3 == c) ddz = -ddz; ddz = 1.0 - ddz;
        for (k1 = a; k1 <= a + 1; k1++) {
            ddx = ((gx[k1 - 1] + gx[k1]) / 2.0 - x) / dx; if (k1 == a) ddx = -ddx; ddx = 1.0 - ddx;
            for (k2 = b; k2 <= b + 1; k2++) {
                ddy = ((gy[k2 - 1] + gy[k2]) / 2.0 - y) / dy; if (k2 == b) ddy = -ddy; ddy = 1.0 - ddy;
                p += o->pr[k3 * XY + k1 * Y + k2] * (ddx * ddy * ddz);
            }
        }
    }
    return p;
}

/* dencalc1 (mark3mg.c:3006-3024); *bb = thermal expansion term */
static double den_at(const orc_ctx *o, double mtk, double mpb, int mm2, double *bb)
{
    double **R = (double **)o->rock;
    *bb = 0;
    if (o->p.densimod == 0) return R[R_RO][mm2];
    *bb = R[R_BB][mm2] / (1.0 - R[R_BB][mm2] * (mtk - 298.15));
    return R[R_RO][mm2] * (1.0 - R[R_BB][mm2] * (mtk - 298.15)) * (1.0 + R[R_AA][mm2] * (mpb - 1.0) * 1e-3);
}

/* viscalc (mark3mg.c:1114-1693): rheologies A-D, F and the brittle limit; returns -1 for
 * the grain-damage rheology (markdh < 0), which is not restated */
static double visc(orc_ctx *o, double mtk, double mpb, long mm1, int mm2, double epsin, double sigin,
                   double markrii1)
{
    double **R = (double **)o->rock;
    (void)sigin;
    double rt = 8.314 * mtk, e1, k1, sduct, sbrit;
    double strain = ABSV(o->me[mm1]);
    double lamb = 1.0, abrit = R[R_A0][mm2], bbrit = R[R_B0][mm2];
    if (strain > R[R_E1][mm2]) { abrit = R[R_A1][mm2]; bbrit = R[R_B1][mm2]; }
    else if (strain > R[R_E0][mm2] && R[R_E1][mm2] > R[R_E0][mm2]) {
        abrit = R[R_A0][mm2] + (R[R_A1][mm2] - R[R_A0][mm2]) * (strain - R[R_E0][mm2]) / (R[R_E1][mm2] - R[R_E0][mm2]);
        bbrit = R[R_B0][mm2] + (R[R_B1][mm2] - R[R_B0][mm2]) * (strain - R[R_E0][mm2]) / (R[R_E1][mm2] - R[R_E0][mm2]);
    }
    double mpf = mpb * 1e+5, nubrit = 0;
    if (epsin > 0 && (bbrit > 0 || abrit * lamb > 0) && mm2 > 1) {
        sbrit = abrit + bbrit * mpf * lamb;
        if (mpf < 0) sbrit = abrit + mpf;
        if (sbrit > 0) nubrit = 1.0 / (0.5 * sbrit / epsin / markrii1);
        else { nubrit = 1.0 / R[R_N0][mm2]; sbrit = 0; }
    }
    double nunewt = 0, nupowl = 0;
    double nu = R[R_NU][mm2], dh = R[R_DH][mm2], dv = R[R_DV][mm2], ss = R[R_SS][mm2], mm = R[R_MM][mm2];
    if (nu) {
        if (dh == 0 && dv == 0 && (ss == 0 || mm == 1.0)) nunewt = 1.0 / nu;
        if ((dh != 0 || dv != 0) && (ss == 0 || mm == 1.0)) {
            e1 = (dh + dv * mpb) / rt;
            if (e1 > 150.0) e1 = 150.0;
            if (dh < 0 && dv > 0) { e1 = dh * (mtk - dv); if (e1 < -150.0) e1 = -150.0; }
            if (dh < 0 && dv < 0) { e1 = (-dh) * (1.0 - (mtk - (-dv)) / (-dv)) / 8.314 / (-dv); if (e1 > 150.0) e1 = 150.0; }
            nunewt = 1.0 / (nu * exp(e1));
        }
        if ((dh == 0 && dv == 0) && ss != 0 && mm != 1.0) {
            k1 = nu / pow(ss, mm - 1.0);
            nunewt = 1.0 / (0.5 * k1);
            sduct = pow(nu * epsin, 1.0 / mm);
            if (epsin > 0) nupowl = 1.0 / (0.5 * sduct / epsin);
        }
        if (nu > 0 && dh > 0 && (dh != 0 || dv != 0) && ss != 0 && mm != 1.0) {
            e1 = (dh + dv * mpb) / rt;
            if (e1 > 150.0) e1 = 150.0;
            e1 = exp(e1);
            k1 = nu / pow(ss, mm - 1.0);
            nunewt = 1.0 / (0.5 * k1 * e1);
            sduct = pow(nu * e1 * epsin, 1.0 / mm);
            if (epsin > 0) nupowl = 1.0 / (0.5 * sduct / epsin);
        }
        if (nu < 0) {
            double mnu2 = 1.0;
            e1 = (ss + mpb * R[R_LL][mm2]) / rt;
            if (e1 > 150.0) e1 = 150.0;
            e1 = exp(e1);
            nunewt = 1.0 / (0.5 * pow(mnu2 * 1e-3 / 5e-10, 2.5) * 8e+10 / R[R_S1][mm2] * e1);
            nupowl = 0;
            if (epsin > 0) {
                e1 = (dh + dv * mpb) / rt / mm;
                if (e1 > 150.0) e1 = 150.0;
                e1 = exp(e1);
                nupowl = 1.0 / (0.5 * pow(epsin, 1.0 / mm - 1.0) * 8e+10 / pow(-nu, 1.0 / mm) * e1);
            }
        }
        if (dh < 0) return -1;
    }
    double nueff = nunewt + nupowl;
    if (mm2 == 7 || mm2 == 8 || mm2 == 9 || mm2 == 10) {
        if (mtk > 1300.0) o->mft[mm1] = 0;
        else if (o->mft[mm1] <= 0) o->mft[mm1] = o->m.timesum;
    }
    if (nubrit > nueff) {
        nueff = nubrit;
        if (o->me[mm1] == 0) o->me[mm1] = 1e-20;
        o->me[mm1] = ABSV(o->me[mm1]);
    } else {
        o->me[mm1] = -ABSV(o->me[mm1]);
    }
    if (nueff <= 0) nueff = 1.0 / R[R_N1][mm2];
    nueff = 1.0 / nueff;
    if (nueff < R[R_N0][mm2]) nueff = R[R_N0][mm2];
    if (nueff > R[R_N1][mm2]) nueff = R[R_N1][mm2];
    if (nueff < o->p.nubeg) nueff = o->p.nubeg;
    if (nueff > o->p.nuend) nueff = o->p.nuend;
    return nueff;
}

static int inbox_strict(const orc_ctx *o, long mm1)
{
    return o->mx[mm1] > 0 && o->my[mm1] > 0 && o->mz[mm1] > 0 && (double)o->mx[mm1] < o->m.xsize &&
           (double)o->my[mm1] < o->m.ysize && (double)o->mz[mm1] < o->m.zsize;
}

/* movemark (mark3mg.c:2-310) for rock markers (types < 50) with RK4 (markmod 2) or Euler */
int orc_move_markers(orc_ctx *o, double timestep)
{
    for (long mm1 = 0; mm1 < o->marknum; mm1++) {
        int t = o->mt[mm1];
        int inbox = o->mx[mm1] >= 0 && o->my[mm1] >= 0 && o->mz[mm1] >= 0 && (double)o->mx[mm1] <= o->m.xsize &&
                    (double)o->my[mm1] <= o->m.ysize && (double)o->mz[mm1] <= o->m.zsize;
        if (!(inbox || (o->p.outgrid != 1 && (t < 50 || t >= 100)))) continue;
        if (t >= 50) { snprintf(o->err, sizeof o->err, "marker type %d is not supported", t); return I3G_E_UNSUPPORTED; }
        double xold = o->mx[mm1], yold = o->my[mm1];
        double v1[3], e[7], s[6], dis;
        long wn[3];
        orc_vxyz(o, o->mx[mm1], o->my[mm1], o->mz[mm1], v1, wn);
        eps_at(o, o->mx[mm1], o->my[mm1], o->mz[mm1], wn, e, s, &dis);
        double eii = pow(0.5 * (e[0] * e[0] + e[1] * e[1] + e[2] * e[2]) + e[3] * e[3] + e[4] * e[4] + e[5] * e[5], 0.5);
        double sii = pow(0.5 * (s[0] * s[0] + s[1] * s[1] + s[2] * s[2]) + s[3] * s[3] + s[4] * s[4] + s[5] * s[5], 0.5);
        double mpb = e[6] * 1e-5, mtk = o->mk[mm1];
        if (t < 50 && mtk > 0) {
            double rii = 1.0;
            if (o->mv[mm1] > 0 && o->mx[mm1] > o->gx[3] && o->mx[mm1] < o->gx[o->nx - 4] && o->my[mm1] > o->gy[3] &&
                o->my[mm1] < o->gy[o->ny - 4] && o->mz[mm1] > o->gz[3] && o->mz[mm1] < o->gz[o->nz - 4])
                rii *= pow(0.5 * sii / eii / o->mv[mm1], 0.87);
            double mnu = visc(o, mtk, mpb, mm1, t, eii, sii, rii);
            if (mnu < 0) { snprintf(o->err, sizeof o->err, "grain-damage rheology (markdh < 0) is not supported"); return I3G_E_UNSUPPORTED; }
            o->mv[mm1] = mnu;
            if (o->me[mm1] > 0) o->me[mm1] += timestep * eii;
            if (o->me[mm1] > 0) { o->me[mm1] -= timestep * o->p.healrate; if (o->me[mm1] < 0) o->me[mm1] = 0; }
            else { o->me[mm1] += timestep * o->p.healrate; if (o->me[mm1] > 0) o->me[mm1] = 0; }
        }
        double v[3];
        if (o->p.markmod == 1) { v[0] = v1[0]; v[1] = v1[1]; v[2] = v1[2]; }
        else {
            double v2[3], v3[3], v4[3];
            orc_vxyz(o, o->mx[mm1] + v1[0] * timestep / 2.0, o->my[mm1] + v1[1] * timestep / 2.0, o->mz[mm1] + v1[2] * timestep / 2.0, v2, wn);
            orc_vxyz(o, o->mx[mm1] + v2[0] * timestep / 2.0, o->my[mm1] + v2[1] * timestep / 2.0, o->mz[mm1] + v2[2] * timestep / 2.0, v3, wn);
            orc_vxyz(o, o->mx[mm1] + v3[0] * timestep, o->my[mm1] + v3[1] * timestep, o->mz[mm1] + v3[2] * timestep, v4, wn);
            for (int k = 0; k < 3; k++) v[k] = (v1[k] + 2.0 * v2[k] + 2.0 * v3[k] + v4[k]) / 6.0;
        }
        if (o->p.outgrid == 2) {
            if (o->mx[mm1] < 0 || (double)o->mx[mm1] > o->m.xsize) v[1] = v[2] = 0;
            if (o->my[mm1] < 0 || (double)o->my[mm1] > o->m.ysize) v[0] = v[2] = 0;
            if (o->mz[mm1] < 0 || (double)o->mz[mm1] > o->m.zsize) v[0] = v[1] = 0;
        }
        double zdeep = o->p.zdeep, vdeep = o->p.vdeep, tdeep = o->p.tdeep;
        if (o->my[mm1] > zdeep && v[1] < 0 && o->mk[mm1] < tdeep && o->mt[mm1] == 10) o->mk[mm1] = tdeep;
        if (o->my[mm1] > zdeep && v[1] < 0 && o->mt[mm1] != 10) { o->mt[mm1] = 10; o->mw[mm1] = 0; }
        if (o->my[mm1] > zdeep && o->mt[mm1] != 10 && o->mt[mm1] != 9) { o->mt[mm1] = 9; o->mw[mm1] = 0; }
        o->mx[mm1] += timestep * v[0] - 0.0;
        o->my[mm1] += timestep * v[1];
        o->mz[mm1] += timestep * v[2];
        if ((yold > vdeep && o->my[mm1] < vdeep) || (yold > zdeep && o->my[mm1] < zdeep)) {
            if (o->mk[mm1] < tdeep) o->mk[mm1] = tdeep;
            o->mt[mm1] = 10;
        }
        (void)xold;
        if (o->mx[mm1] < 0 || o->my[mm1] < 0 || o->mz[mm1] < 0 || (double)o->mx[mm1] > o->m.xsize ||
            (double)o->my[mm1] > o->m.ysize || (double)o->mz[mm1] > o->m.zsize) {
            o->mk[mm1] = 0;
            o->mv[mm1] = 0;
        }
    }
    return 0;
}

/* tkrecalc (heat3mg.c:849-899): temperature boundary rows on level 0 */
void orc_tkrecalc(orc_ctx *o)
{
    float *tk1 = malloc(sizeof(float) * o->nodenum);
    memcpy(tk1, o->tk, sizeof(float) * o->nodenum);
    for (long n = 0; n < o->nodenum; n++) {
        int b = o->bcid_t[n];
        if (b < 0) continue;
        o->tk[n] = (float)o->bc_c[b];
        if (o->bc_p[b] >= 0) o->tk[n] += (float)o->bc_k[b] * tk1[o->bc_p[b]];   /* FP32 like bondv1 */
    }
    free(tk1);
}

/* ronurecalc (mark3mg.c:404-1015) for rock markers; FP64 sums */
int orc_markers_to_nodes(orc_ctx *o, double timestep)
{
    long N = o->nodenum, X = o->nx, Y = o->ny, XY = X * Y;
    enum { A_NU, W_NU, A_XX, W_XX, A_XY, W_XY, A_XZ, W_XZ, A_YZ, W_YZ, A_RO, A_CP, A_KT, A_HT, A_ET, A_TK, A_RR, W_P, NA };
    double *acc = calloc((size_t)N * NA, sizeof(double));
    double **R = (double **)o->rock;
    int vm = o->p.viscmod;
    for (long mm1 = 0; mm1 < o->marknum; mm1++) {
        if (!(inbox_strict(o, mm1) && o->mt[mm1] < 50 && o->mk[mm1] > 0)) continue;
        int mm2 = o->mt[mm1];
        if (mm2 > 1 && o->my[mm1] < o->p.eroslev) mm2 = o->mt[mm1] = 0;
        if (mm2 < 2 && o->my[mm1] > o->p.sedilev) { free(acc); snprintf(o->err, sizeof o->err, "sedimentation is not supported"); return I3G_E_UNSUPPORTED; }
        if (mm2 < 2 && o->p.waterlev >= 0) { free(acc); snprintf(o->err, sizeof o->err, "water/air markers are not supported"); return I3G_E_UNSUPPORTED; }
        if (mm2 > 20) { free(acc); snprintf(o->err, sizeof o->err, "molten rock types are not supported"); return I3G_E_UNSUPPORTED; }
        if (o->p.densimod >= 2) { free(acc); snprintf(o->err, sizeof o->err, "densimod >= 2 is not supported"); return I3G_E_UNSUPPORTED; }
        long wn[3];
        double mpb = pr_at(o, o->mx[mm1], o->my[mm1], o->mz[mm1], wn) * 1e-5;
        double mtk = o->mk[mm1];
        double mnu = o->mv[mm1];
        if (mnu <= 0 || timestep <= 0) {
            double e[7], s[6], dis;
            eps_at(o, o->mx[mm1], o->my[mm1], o->mz[mm1], wn, e, s, &dis);
            double eii = pow(0.5 * (e[0] * e[0] + e[1] * e[1] + e[2] * e[2]) + e[3] * e[3] + e[4] * e[4] + e[5] * e[5], 0.5);
            double sii = pow(0.5 * (s[0] * s[0] + s[1] * s[1] + s[2] * s[2]) + s[3] * s[3] + s[4] * s[4] + s[5] * s[5], 0.5);
            mnu = visc(o, mtk, mpb, mm1, mm2, eii, sii, 1.0);
            if (mnu < 0) { free(acc); snprintf(o->err, sizeof o->err, "grain-damage rheology is not supported"); return I3G_E_UNSUPPORTED; }
            o->mv[mm1] = mnu;
        }
        double mbb, mro = den_at(o, mtk, mpb, mm2, &mbb);
        if ((mm2 >= 7 && mm2 <= 8) || (mm2 >= 16 && mm2 <= 18)) {
            double rokf = 1.0;
            double p_ga_in = -9222.0 + mtk * 14.0; if (p_ga_in < 2000.0) p_ga_in = 2000.0;
            double p_pl_out = -1460.0 + mtk * 20.0; if (p_pl_out < 12000.0) p_pl_out = 12000.0;
            if (mpb > p_ga_in) { if (mpb >= p_pl_out) rokf *= 1.16; else rokf *= 1.0 + 0.16 * (mpb - p_ga_in) / (p_pl_out - p_ga_in); }
            double p_st_in = 59100.0 + mtk * 22.6;
            if (mpb > p_st_in) rokf *= 1.06;
            double p_sp_out = 354000.0 - mtk * 40.0, p_pv_in = 352000.0 - mtk * 40.0;
            if (mpb > p_pv_in) { if (mpb >= p_sp_out) rokf *= 1.08; else rokf *= 1.0 + 0.08 * (mpb - p_pv_in) / (p_sp_out - p_pv_in); }
            if (mtk < o->p.teclmax) { if (mtk < o->p.teclmin) rokf = 1.00; else rokf = 1.0 + (rokf - 1.0) * (mtk - o->p.teclmin) / (o->p.teclmax - o->p.teclmin); }
            mro *= rokf;
        }
        if (mm2 >= 9 && mm2 <= 14) {
            double rokf = 1.0;
            double p_ol_out = 91000.0 + mtk * 27.0, p_sp_in = 66000.0 + mtk * 39.0;
            if (p_sp_in > p_ol_out - 2000.0) p_sp_in = p_ol_out - 2000.0;
            if (mpb > p_sp_in) { if (mpb >= p_ol_out) rokf *= 1.06; else rokf *= 1.0 + 0.06 * (mpb - p_sp_in) / (p_ol_out - p_sp_in); }
            double p_sp_out = 304000.0 - mtk * 40.0, p_pv_in = 302000.0 - mtk * 40.0;
            if (mpb > p_pv_in) { if (mpb >= p_sp_out) rokf *= 1.11; else rokf *= 1.0 + 0.11 * (mpb - p_pv_in) / (p_sp_out - p_pv_in); }
            if (mtk < o->p.teclmax) { if (mtk < o->p.teclmin) rokf = 1.00; else rokf = 1.0 + (rokf - 1.0) * (mtk - o->p.teclmin) / (o->p.teclmax - o->p.teclmin); }
            mro *= rokf;
        }
        double mcp = R[R_CP][mm2];
        double mkt = (R[R_KT][mm2] + R[R_KF][mm2] / (mtk + 77.0)) * exp(R[R_KP][mm2] * mpb);
        double mht = R[R_HT][mm2];
        if (o->my[mm1] > o->p.vdeep && mnu > o->p.nudeep) mnu = o->p.nudeep;
        if (o->my[mm1] < 5e+4 && o->mx[mm1] > o->m.xsize - 1e+4 && o->mz[mm1] > 1.5e+5 && o->mz[mm1] < 8.7e+5 && mnu > 1e+19) mnu = 1e+19;
        long m10 = wn[0], m20 = wn[1], m30 = wn[2];
        double dx = o->gx[m10 + 1] - o->gx[m10], dy = o->gy[m20 + 1] - o->gy[m20], dz = o->gz[m30 + 1] - o->gz[m30];
        double vnu = vm == 0 ? mnu : vm == 1 ? log(mnu) : 1.0 / mnu;
        for (long m3 = m30; m3 <= m30 + 1; m3++) {
            double ddz = (o->gz[m3] - o->mz[mm1]) / dz; ddz = 1.0 - ABSV(ddz);
            for (long m1 = m10; m1 <= m10 + 1; m1++) {
                double ddx = (o->gx[m1] - o->mx[mm1]) / dx; ddx = 1.0 - ABSV(ddx);
                for (long m2 = m20; m2 <= m20 + 1; m2++) {
                    double ddy = (o->gy[m2] - o->my[mm1]) / dy; ddy = 1.0 - ABSV(ddy);
                    double swt = ddx * ddy * ddz, swt1;
                    double *a = acc + (m3 * XY + m1 * Y + m2) * NA;
                    if (ddx > o->p.nukoef && ddy > o->p.nukoef && ddz > o->p.nukoef) { a[A_NU] += vnu * swt; a[W_NU] += swt; }
                    if (m1 > m10 && m2 > m20 && m3 > m30) {
                        swt1 = 8.0 * (0.5 - ABSV(ddx - 0.5)) * (0.5 - ABSV(ddy - 0.5)) * (0.5 - ABSV(ddz - 0.5));
                        a[A_XX] += vnu * swt1; a[W_XX] += swt1;
                    }
                    if (m3 == m30 && ddx > 0.5 && ddy > 0.5) {
                        swt1 = 8.0 * (ddx - 0.5) * (ddy - 0.5) * (0.5 - ABSV(ddz - 0.5));
                        a[A_XY] += vnu * swt1; a[W_XY] += swt1;
                    }
                    if (m2 == m20 && ddx > 0.5 && ddz > 0.5) {
                        swt1 = 8.0 * (ddx - 0.5) * (0.5 - ABSV(ddy - 0.5)) * (ddz - 0.5);
                        a[A_XZ] += vnu * swt1; a[W_XZ] += swt1;
                    }
                    if (m1 == m10 && ddy > 0.5 && ddz > 0.5) {
                        swt1 = 8.0 * (0.5 - ABSV(ddx - 0.5)) * (ddy - 0.5) * (ddz - 0.5);
                        a[A_YZ] += vnu * swt1; a[W_YZ] += swt1;
                    }
                    if (swt > 0) {
                        a[A_RO] += mro * swt; a[A_CP] += mcp * mro * swt; a[A_KT] += mkt * swt;
                        a[A_HT] += mht * swt; a[A_ET] += mbb * swt; a[A_TK] += mtk * swt;
                        a[A_RR] += o->mrr[mm1] * swt; a[W_P] += swt;
                    }
                }
            }
        }
    }
    for (long n = 0; n < N; n++) {
        double *a = acc + n * NA;
#define FIN(field, A, W) if (a[W] > 0.01) { double v_ = a[A] / a[W]; if (vm == 1) v_ = exp(v_); if (vm == 2) v_ = 1.0 / v_; o->field[n] = (float)v_; }
        FIN(nu, A_NU, W_NU);
        FIN(nxx, A_XX, W_XX);
        FIN(nxy, A_XY, W_XY);
        FIN(nxz, A_XZ, W_XZ);
        FIN(nyz, A_YZ, W_YZ);
#undef FIN
        if (a[W_P] > 0.01) {
            o->ro[n] = (float)(a[A_RO] / a[W_P]);
            o->cp[n] = (float)(a[A_CP] / a[W_P] / o->ro[n]);
            o->kt[n] = (float)(a[A_KT] / a[W_P]);
            o->ht[n] = (float)(a[A_HT] / a[W_P]);
            o->et[n] = (float)(a[A_ET] / a[W_P]);
            o->tk[n] = (float)(a[A_TK] / a[W_P]);
            o->rr[n] = (float)(a[A_RR] / a[W_P]);
        }
        if (o->nu[n] < o->p.nubeg) o->nu[n] = o->p.nubeg;
        if (o->nu[n] > o->p.nuend) o->nu[n] = o->p.nuend;
    }
    free(acc);
    orc_tkrecalc(o);
    return 0;
}
