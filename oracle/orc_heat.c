/*
 * orc_heat.c -- TEST INFRASTRUCTURE (CPU oracle).  Restatement of the reference's heat step
 * titerate (heat3mg.c:287-788), single-threaded:
 *
 *   explicit right-hand side and rate limit ... heaterr mode 0   heat3mg.c:40-183, 310-367
 *   implicit 7-point rows ..................... heaterr mode 1   heat3mg.c:193-241
 *   boundary rows ............................. tbonderr         heat3mg.c:794-843
 *   relaxation ................................ gausmatt         heat3mg.c:906-961
 *   substep loop .............................. titerate         heat3mg.c:380-585
 *   marker temperature + subgrid diffusion .... titerate         heat3mg.c:592-782
 *
 * The stopping rule is the relative residual ||b - A T|| / ||b|| over non-boundary rows
 * (heat_rtol), shared with the CUDA library.  Only adiabyn 0/1 are restated.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "orc_internal.h"

#define ABSV(a) ((a) >= 0 ? (a) : -(a))
#define MAXV(a, b) ((a) >= (b) ? (a) : (b))
#define MINV(a, b) ((a) <= (b) ? (a) : (b))

/* heaterr mode 0 (heat3mg.c:40-183) for a non-boundary node: right-hand side rate */
static double rhs0(orc_ctx *o, long m1, long m2, long m3, const float *tk0)
{
    long X = o->nx, Y = o->ny, XY = X * Y;
    long v3 = m3 * XY + m1 * Y + m2;
    double ival = o->ht[v3];
    double xkf = 2.0 / (o->gx[m1 + 1] - o->gx[m1 - 1]);
    double ykf = 2.0 / (o->gy[m2 + 1] - o->gy[m2 - 1]);
    double zkf = 2.0 / (o->gz[m3 + 1] - o->gz[m3 - 1]);
    double x = (o->gx[m1] - o->gx[m1 - 1]) / 2.0 * xkf;
    double y = (o->gy[m2] - o->gy[m2 - 1]) / 2.0 * ykf;
    double z = (o->gz[m3] - o->gz[m3 - 1]) / 2.0 * zkf;
    double v[3] = {0, 0, 0};
    long wn[3];
    if (o->p.adiabyn) orc_vxyz(o, o->gx[m1], o->gy[m2], o->gz[m3], v, wn);
    if (o->p.adiabyn == 1 && o->ro[v3] > 2e+3 && o->gy[m2] < o->m.ysize - o->p.stp100)
        ival += o->et[v3] * tk0[v3] * o->ro[v3] * (v[0] * o->m.gxkoef + v[1] * o->m.gykoef + v[2] * o->m.gzkoef);
    if (o->p.frictyn && o->ro[v3] > 2e+3 && o->gy[m2] < o->m.ysize - o->p.stp100) {
        long p[8];
        p[0] = v3; p[1] = p[0] + 1; p[2] = p[0] + Y; p[3] = p[2] + 1;
        p[4] = p[0] + XY; p[5] = p[4] + 1; p[6] = p[4] + Y; p[7] = p[6] + 1;
        double w8[8] = {(1.0 - x) * (1.0 - y) * (1.0 - z), (1.0 - x) * (y) * (1.0 - z), (x) * (1.0 - y) * (1.0 - z),
                        (x) * (y) * (1.0 - z), (1.0 - x) * (1.0 - y) * (z), (1.0 - x) * (y) * (z),
                        (x) * (1.0 - y) * (z), (x) * (y) * (z)};
        double ev = 0;
        for (int q = 0; q < 8; q++)
            ev += w8[q] * (o->sxx[p[q]] * o->exx[p[q]] + o->syy[p[q]] * o->eyy[p[q]] + o->szz[p[q]] * o->ezz[p[q]]);
        long v0 = v3 - XY, v1 = v3 - Y, v2 = v3 - 1;
        ev += 2.0 * ((1.0 - z) * (o->sxy[v0] * o->exy[v0]) + z * (o->sxy[v3] * o->exy[v3]));
        ev += 2.0 * ((1.0 - y) * (o->sxz[v2] * o->exz[v2]) + y * (o->sxz[v3] * o->exz[v3]));
        ev += 2.0 * ((1.0 - x) * (o->syz[v1] * o->eyz[v1]) + x * (o->syz[v3] * o->eyz[v3]));
        ival += ev;
    }
    return ival;
}

/* Assemble level-0 rows (heat3mg.c:407-453); T rows: 7 slots; boundary rows 1-2 slots */
static void assemble(orc_ctx *o, double dt, const float *tk0)
{
    long X = o->nx, Y = o->ny, Z = o->nz, XY = X * Y, N = o->nodenum, pos = 0;
    for (long m3 = 0; m3 < Z; m3++)
        for (long m1 = 0; m1 < X; m1++)
            for (long m2 = 0; m2 < Y; m2++) {
                long n = m3 * XY + m1 * Y + m2;
                o->trowptr[n] = pos;
                int b = o->bcid_t[n];
                if (b >= 0) {
                    double c = o->bc_c[b];
                    if (o->m.timesum > o->p.timebeg && m2 == Y - 1) {
                        if (o->m.timesum >= o->p.timeend) c = o->p.tempend;
                        else c = c + (o->p.tempend - c) / (o->p.timeend - o->p.timebeg) * (o->m.timesum - o->p.timebeg);
                    }
                    o->tfre1[n] = c;
                    o->tcol[pos] = n; o->tval[pos] = 1.0; pos++;
                    if (o->bc_p[b] >= 0) { o->tcol[pos] = o->bc_p[b]; o->tval[pos] = -o->bc_k[b]; pos++; }
                } else {
                    double xkf = 2.0 / (o->gx[m1 + 1] - o->gx[m1 - 1]);
                    double ykf = 2.0 / (o->gy[m2 + 1] - o->gy[m2 - 1]);
                    double zkf = 2.0 / (o->gz[m3 + 1] - o->gz[m3 - 1]);
                    double rocpkf = o->ro[n] * o->cp[n];
                    const float *kt = o->kt;
                    long v0 = n - XY, v1 = n - Y, v2 = n - 1, v4 = n + 1, v5 = n + Y, v6 = n + XY;
                    o->tfre1[n] = o->tk1[n] + tk0[n] / dt * rocpkf;
                    double d = rocpkf / dt, iv;
                    long base = pos;
                    pos += 7;
                    o->tcol[base] = n;
                    iv = (kt[v1] + kt[n]) / 2.0 * xkf / (o->gx[m1] - o->gx[m1 - 1]);
                    o->tcol[base + 1] = v1; o->tval[base + 1] = -iv; d += iv;
                    iv = (kt[n] + kt[v5]) / 2.0 * xkf / (o->gx[m1 + 1] - o->gx[m1]);
                    d += iv; o->tcol[base + 2] = v5; o->tval[base + 2] = -iv;
                    iv = (kt[v2] + kt[n]) / 2.0 * ykf / (o->gy[m2] - o->gy[m2 - 1]);
                    o->tcol[base + 3] = v2; o->tval[base + 3] = -iv; d += iv;
                    iv = (kt[n] + kt[v4]) / 2.0 * ykf / (o->gy[m2 + 1] - o->gy[m2]);
                    d += iv; o->tcol[base + 4] = v4; o->tval[base + 4] = -iv;
                    iv = (kt[v0] + kt[n]) / 2.0 * zkf / (o->gz[m3] - o->gz[m3 - 1]);
                    o->tcol[base + 5] = v0; o->tval[base + 5] = -iv; d += iv;
                    iv = (kt[n] + kt[v6]) / 2.0 * zkf / (o->gz[m3 + 1] - o->gz[m3]);
                    d += iv; o->tcol[base + 6] = v6; o->tval[base + 6] = -iv;
                    o->tval[base] = d;
                }
                o->trowptr[n + 1] = pos;
            }
    (void)N;
}

static double heat_relres(orc_ctx *o)
{
    double rr = 0, bb = 0;
    for (long n = 0; n < o->nodenum; n++) {
        if (o->bcid_t[n] >= 0) continue;
        double r = o->tfre1[n];
        for (long e = o->trowptr[n]; e < o->trowptr[n + 1]; e++) r -= o->tval[e] * o->tsol[o->tcol[e]];
        rr += r * r; bb += o->tfre1[n] * o->tfre1[n];
    }
    return bb > 0 ? sqrt(rr / bb) : sqrt(rr);
}

/* gausmatt sweeps (heat3mg.c:921-942) */
static void gausmatt(orc_ctx *o, int am)
{
    for (int s = 0; s < am; s++)
        for (long n = 0; n < o->nodenum; n++) {
            long a = o->trowptr[n], b = o->trowptr[n + 1];
            if (a == b) continue;
            double iv = -o->tfre1[n], d = o->tval[a];
            for (long e = a; e < b; e++) iv += o->tval[e] * o->tsol[o->tcol[e]];
            o->tsol[n] -= iv / d * o->p.t0koef;
        }
}

/* tkcalc1 (mark3mg.c:2844-2910): T0, T1, T, T2 at a point with cell, spacings and weights */
static void tk_at(orc_ctx *o, double x, double y, double z, const float *tk0, const float *tk1f, const float *tk2,
                  double *e, long *wn, double *wi)
{
    long XY = o->nx * o->ny, Y = o->ny;
    long m10 = wn[0] = orc_m1serch(o, x), m20 = wn[1] = orc_m2serch(o, y), m30 = wn[2] = orc_m3serch(o, z);
    double dx = wi[0] = o->gx[m10 + 1] - o->gx[m10];
    double dy = wi[1] = o->gy[m20 + 1] - o->gy[m20];
    double dz = wi[2] = o->gz[m30 + 1] - o->gz[m30];
    e[0] = e[1] = e[2] = e[3] = 0;
    int q = 0;
    for (long m3 = m30; m3 <= m30 + 1; m3++) {
        double ddz = (o->gz[m3] - z) / dz; ddz = 1.0 - ABSV(ddz);
        for (long m1 = m10; m1 <= m10 + 1; m1++) {
            double ddx = (o->gx[m1] - x) / dx; ddx = 1.0 - ABSV(ddx);
            for (long m2 = m20; m2 <= m20 + 1; m2++) {
                double ddy = (o->gy[m2] - y) / dy; ddy = 1.0 - ABSV(ddy);
                double swt = wi[3 + q] = ddx * ddy * ddz;
                long m4 = wn[3 + q] = m3 * XY + m1 * Y + m2;
                e[0] += swt * tk0[m4]; e[1] += swt * tk1f[m4]; e[2] += swt * o->tk[m4]; e[3] += swt * tk2[m4];
                q++;
            }
        }
    }
}

/* titerate (heat3mg.c:287-788) with the relative-residual stop */
int orc_heat(orc_ctx *o, double *timestep)
{
    long N = o->nodenum, X = o->nx, Y = o->ny, Z = o->nz, XY = X * Y;
    if (o->p.adiabyn > 1) { snprintf(o->err, sizeof o->err, "adiabyn %d is not supported", o->p.adiabyn); return I3G_E_UNSUPPORTED; }
    if (!o->trowptr) {
        o->trowptr = calloc(N + 1, sizeof(long));
        o->tcol = calloc(7 * N, sizeof(long));
        o->tval = calloc(7 * N, sizeof(double));
        o->tfre1 = calloc(N, sizeof(double));
        o->tsol = calloc(N, sizeof(double));
    }
    float *tk0 = malloc(sizeof(float) * N), *tk1f = malloc(sizeof(float) * N), *tk2 = malloc(sizeof(float) * N);
    memcpy(tk0, o->tk, sizeof(float) * N);
    double maxrate = 0;
    memset(tk1f, 0, sizeof(float) * N);
    for (long m3 = 0; m3 < Z; m3++)
        for (long m1 = 0; m1 < X; m1++)
            for (long m2 = 0; m2 < Y; m2++) {
                long n = m3 * XY + m1 * Y + m2;
                if (o->bcid_t[n] >= 0) continue;
                double iv = rhs0(o, m1, m2, m3, tk0);
                tk1f[n] = (float)iv;
                double rocpkf = o->ro[n] * o->cp[n];
                maxrate = MAXV(maxrate, ABSV(iv / rocpkf));
            }
    for (long n = 0; n < N; n++) o->tk1[n] = tk1f[n];
    double tkstep = 1e30;
    if (maxrate) tkstep = o->f.maxtkstep / maxrate;
    if (*timestep == 0 || tkstep == 0) { free(tk0); free(tk1f); free(tk2); return 0; }
    memcpy(tk2, o->tk, sizeof(float) * N);
    double total = *timestep, done = 0;
    double rtol = o->p.heat_rtol > 0 ? o->p.heat_rtol : 1e-10;
    int maxc = o->p.heat_maxcyc > 0 ? o->p.heat_maxcyc : 2000, cycles = 0, subs = 0;
    double rel = 0;
    do {
        double dt = MINV(total, tkstep);
        if (dt > total - done) dt = total - done;
        memcpy(tk0, o->tk, sizeof(float) * N);
        for (long n = 0; n < N; n++) o->tsol[n] = o->tk[n];
        assemble(o, dt, tk0);
        int it = 0;
        do {
            gausmatt(o, o->p.multittt0 > 0 ? o->p.multittt0 : 30);
            rel = heat_relres(o);
            it++;
        } while (rel > rtol && it < maxc);
        cycles += it;
        for (long n = 0; n < N; n++) o->tk[n] = (float)o->tsol[n];
        if (rel > rtol) {
            free(tk0); free(tk1f); free(tk2);
            snprintf(o->err, sizeof o->err, "heat: no convergence (%g)", rel);
            return I3G_E_NOCONV;
        }
        done += dt;
        subs++;
    } while (done < total);
    o->st.heat_cycles = cycles;
    o->st.heat_substeps = subs;
    o->st.heat_rel = rel;
    /* marker temperatures (heat3mg.c:592-782); timestep is the full step again */
    double dtm = total;
    double *w0 = calloc(N, sizeof(double)), *w1 = calloc(N, sizeof(double));
    for (long mm = 0; mm < o->marknum; mm++) {
        if (!(o->mt[mm] < 50 && o->mx[mm] > 0 && o->my[mm] > 0 && o->mz[mm] > 0 && (double)o->mx[mm] < o->m.xsize &&
              (double)o->my[mm] < o->m.ysize && (double)o->mz[mm] < o->m.zsize)) continue;
        double e[4], wi[11];
        long wn[11];
        tk_at(o, o->mx[mm], o->my[mm], o->mz[mm], tk0, tk1f, tk2, e, wn, wi);
        if (o->mk[mm] <= 0) {
            o->mk[mm] = (float)e[3];
            if (o->my[mm] > o->p.zdeep && o->mk[mm] < o->p.tdeep) o->mk[mm] = o->p.tdeep;
        }
        if (o->p.heatdif) {
            double mkt = 0, rocp = 0, mtk = o->tk[wn[3]];
            for (int q = 0; q < 8; q++) {
                long m4 = wn[3 + q];
                mkt += o->kt[m4] * wi[3 + q];
                rocp += o->ro[m4] * o->cp[m4] * wi[3 + q];
                mtk = MAXV(mtk, o->tk[m4]);
            }
            if ((wn[0] <= 0 || wn[0] >= X - 2 || wn[1] <= 0 || wn[1] >= Y - 2 || wn[2] <= 0 || wn[2] >= Z - 2) &&
                (o->mk[mm] + e[2] - e[3]) > mtk)
                o->mk[mm] = mtk - e[2] + e[3];
            double dtk = e[3] - (double)o->mk[mm];
            double dtk1 = -o->p.heatdif * mkt / rocp * 2.0 * (1.0 / wi[0] / wi[0] + 1.0 / wi[1] / wi[1] + 1.0 / wi[2] / wi[2]) * dtm;
            if (dtk1 < -150.0) dtk1 = -150.0;
            dtk1 = dtk * (1.0 - exp(dtk1));
            o->mk[mm] += (float)dtk1;
            for (int q = 0; q < 8; q++) {
                w1[wn[3 + q]] += dtk1 * wi[3 + q];
                w0[wn[3 + q]] += wi[3 + q];
            }
        }
        o->mk[mm] += (float)(e[2] - e[3]);
    }
    if (o->p.heatdif) {
        for (long n = 0; n < N; n++) if (w0[n]) w1[n] /= w0[n];
        for (long mm = 0; mm < o->marknum; mm++) {
            if (!(o->mt[mm] < 50 && o->mx[mm] > 0 && o->my[mm] > 0 && o->mz[mm] > 0 && (double)o->mx[mm] < o->m.xsize &&
                  (double)o->my[mm] < o->m.ysize && (double)o->mz[mm] < o->m.zsize)) continue;
            double e[4], wi[11];
            long wn[11];
            tk_at(o, o->mx[mm], o->my[mm], o->mz[mm], tk0, tk1f, tk2, e, wn, wi);
            double iv = 0;
            for (int q = 0; q < 8; q++) iv -= w1[wn[3 + q]] * wi[3 + q];
            o->mk[mm] += (float)iv;
        }
    }
    free(w0); free(w1); free(tk0); free(tk1f); free(tk2);
    return 0;
}
