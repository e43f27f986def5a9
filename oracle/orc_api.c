/*
 * orc_api.c -- TEST INFRASTRUCTURE (CPU oracle).  Context set-up and the vpiterate driver
 * restated in C (move3mg.c:1585-2636), exported with the same call shapes as include/i3g.h
 * under an orc_ prefix so the tests can run the oracle and the CUDA library on one model.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "orc_internal.h"

#define MINV(a, b) ((a) <= (b) ? (a) : (b))
#define MAXV(a, b) ((a) >= (b) ? (a) : (b))
#define ABSV(a) ((a) >= 0 ? (a) : -(a))

static void *xcalloc(size_t n, size_t s)
{
    void *p = calloc(n ? n : 1, s);
    if (!p) { fprintf(stderr, "oracle: out of memory\n"); abort(); }
    return p;
}

static float *fdup(const float *a, long n)
{
    float *p = xcalloc(n, sizeof(float));
    if (a) memcpy(p, a, n * sizeof(float));
    return p;
}

void orc_destroy(orc_ctx *o);

int orc_create(const i3g_model *m, const i3g_params *p, orc_ctx **out)
{
    orc_ctx *o = xcalloc(1, sizeof(orc_ctx));
    o->m = *m;
    o->p = *p;
    o->nx = m->xnumx; o->ny = m->ynumy; o->nz = m->znumz;
    long N = o->nodenum = o->nx * o->ny * o->nz;
    o->gx = xcalloc(o->nx, 8); o->gy = xcalloc(o->ny, 8); o->gz = xcalloc(o->nz, 8);
    for (long i = 0; i < o->nx; i++) o->gx[i] = m->gx[i];
    for (long i = 0; i < o->ny; i++) o->gy[i] = m->gy[i];
    for (long i = 0; i < o->nz; i++) o->gz[i] = m->gz[i];
    o->pr = xcalloc(N, 8);
    memcpy(o->pr, m->pr, N * 8);
    o->vx = fdup(m->vx, N); o->vy = fdup(m->vy, N); o->vz = fdup(m->vz, N);
    o->ro = fdup(m->ro, N); o->nu = fdup(m->nu, N);
    o->nxx = fdup(m->nxx, N); o->nxy = fdup(m->nxy, N); o->nxz = fdup(m->nxz, N); o->nyz = fdup(m->nyz, N);
    o->tk = fdup(m->tk, N); o->cp = fdup(m->cp, N); o->et = fdup(m->et, N);
    o->kt = fdup(m->kt, N); o->ht = fdup(m->ht, N); o->rr = fdup(m->rr, N);
    o->exx = fdup(m->exx, N); o->eyy = fdup(m->eyy, N); o->ezz = fdup(m->ezz, N);
    o->exy = fdup(m->exy, N); o->exz = fdup(m->exz, N); o->eyz = fdup(m->eyz, N);
    o->sxx = fdup(m->sxx, N); o->syy = fdup(m->syy, N); o->szz = fdup(m->szz, N);
    o->sxy = fdup(m->sxy, N); o->sxz = fdup(m->sxz, N); o->syz = fdup(m->syz, N);
    o->tk0 = xcalloc(N, 8); o->tk1 = xcalloc(N, 8); o->tk2 = xcalloc(N, 8);
    long M = o->marknum = m->marknum;
    o->mx = fdup(m->markx, M); o->my = fdup(m->marky, M); o->mz = fdup(m->markz, M);
    o->mk = fdup(m->markk, M); o->mw = fdup(m->markw, M); o->md = fdup(m->markd, M);
    o->mv = fdup(m->markv, M); o->me = fdup(m->marke, M); o->mex = fdup(m->markex, M);
    o->mft = fdup(m->markft, M); o->mrr = fdup(m->markrr, M); o->mrn = fdup(m->markrn, M);
    o->mt = xcalloc(M, 1);
    memcpy(o->mt, m->markt, M);
    o->rocknum = m->rocknum;
    for (int k = 0; k < 24; k++) {
        o->rock[k] = xcalloc(m->rocknum, 8);
        memcpy(o->rock[k], m->rock[k], m->rocknum * 8);
    }
    /* gridcheck (load3mg.c:1220-1282) */
    o->nlev = p->multimax + 1;
    if (o->nlev < 1 || o->nlev > ORC_MAXLEV) { snprintf(o->err, sizeof o->err, "bad multimax"); *out = o; return I3G_E_ARG; }
    o->mgx[0] = o->nx; o->mgy[0] = o->ny; o->mgz[0] = o->nz; o->mgp[0] = 0;
    for (int l = 0; l < o->nlev; l++) {
        if (l) {
            o->mgx[l] = (o->mgx[l - 1] - 5) / 2 + 5;
            o->mgy[l] = (o->mgy[l - 1] - 5) / 2 + 5;
            o->mgz[l] = (o->mgz[l - 1] - 5) / 2 + 5;
            o->mgp[l] = o->mgp[l - 1] + o->mgn[l - 1];
        }
        o->mgxy[l] = o->mgx[l] * o->mgy[l];
        o->mgn[l] = o->mgxy[l] * o->mgz[l];
        long s = 1L << l;
        double *g[3] = {o->gx, o->gy, o->gz};
        long n0[3] = {o->nx, o->ny, o->nz}, nl[3] = {o->mgx[l], o->mgy[l], o->mgz[l]};
        double **dst[3] = {o->mggx, o->mggy, o->mggz};
        for (int d = 0; d < 3; d++) {
            double *c = xcalloc(nl[d], 8);
            c[0] = g[d][0]; c[1] = g[d][1]; c[2] = g[d][2];
            c[nl[d] - 1] = g[d][n0[d] - 1]; c[nl[d] - 2] = g[d][n0[d] - 2]; c[nl[d] - 3] = g[d][n0[d] - 3];
            for (long i = 3; i < nl[d] - 3; i++) c[i] = g[d][(i - 2) * s + 2];
            dst[d][l] = c;
        }
    }
    o->ntot = o->mgp[o->nlev - 1] + o->mgn[o->nlev - 1];
    long R = o->ntot * 4;
    o->bcid = xcalloc(R, 4); o->bcid_t = xcalloc(o->ntot, 4);
    for (long r = 0; r < R; r++) o->bcid[r] = -1;
    for (long r = 0; r < o->ntot; r++) o->bcid_t[r] = -1;
    o->nbc = m->bondnum;
    o->bc_c = xcalloc(o->nbc, 8); o->bc_k = xcalloc(o->nbc, 8); o->bc_p = xcalloc(o->nbc, 8);
    for (long b = 0; b < o->nbc; b++) {
        long row = m->bond_row[b];
        o->bc_c[b] = m->bond_c[b];
        o->bc_k[b] = m->bond_k[b];
        long pp = m->bond_partner1[b] - 1;
        if (row >= 8 * N) {
            long nd = row - 8 * N;
            if (nd >= o->ntot) continue;
            o->bcid_t[nd] = (int32_t)b;
            o->bc_p[b] = pp;   /* node index (or -1) */
        } else {
            if (row >= R) continue;
            o->bcid[row] = (int32_t)b;
            o->bc_p[b] = pp;
        }
    }
    o->nul = xcalloc(o->ntot, 4);
    o->nd = xcalloc(o->ntot, 4);
    o->sol = xcalloc(R, 8); o->fre1 = xcalloc(R, 8); o->fre0 = xcalloc(R, 8); o->wsum = xcalloc(R, 8);
    o->rowptr = xcalloc(R + 1, 8);
    o->col = xcalloc(o->ntot * 57 + 1, 8);
    o->val = xcalloc(o->ntot * 57 + 1, 8);
    o->f.multinum = p->multimax;
    o->f.p0koef = p->p0koef; o->f.p1koef = p->p1koef; o->f.p2koef = p->p2koef;
    o->f.p0koef2 = p->p0koef; o->f.p1koef2 = p->p1koef; o->f.p2koef2 = p->p2koef;
    o->f.multinum2 = p->multimax; o->f.multstp = 1 << 30;
    o->f.nubeg = p->nubeg; o->f.nuend = p->nuend;
    *out = o;
    return 0;
}

void orc_destroy(orc_ctx *o)
{
    if (!o) return;
    void *ptrs[] = {o->gx, o->gy, o->gz, o->pr, o->vx, o->vy, o->vz, o->ro, o->nu, o->nxx, o->nxy, o->nxz,
                    o->nyz, o->tk, o->cp, o->et, o->kt, o->ht, o->rr, o->exx, o->eyy, o->ezz, o->exy, o->exz,
                    o->eyz, o->sxx, o->syy, o->szz, o->sxy, o->sxz, o->syz, o->tk0, o->tk1, o->tk2,
                    o->mx, o->my, o->mz, o->mk, o->mw, o->md, o->mv, o->me, o->mex, o->mft, o->mrr, o->mrn,
                    o->mt, o->bcid, o->bcid_t, o->bc_c, o->bc_k, o->bc_p, o->nul, o->nd, o->sol, o->fre1,
                    o->fre0, o->wsum, o->rowptr, o->col, o->val, o->trowptr, o->tcol, o->tval, o->tfre1, o->tsol};
    for (size_t i = 0; i < sizeof ptrs / sizeof ptrs[0]; i++) free(ptrs[i]);
    for (int k = 0; k < 24; k++) free(o->rock[k]);
    for (int l = 0; l < o->nlev; l++) { free(o->mggx[l]); free(o->mggy[l]); free(o->mggz[l]); }
    free(o);
}

const char *orc_last_error(const orc_ctx *o) { return o ? o->err : "no context"; }

int orc_set_file_params(orc_ctx *o, const i3g_file_params *f)
{
    o->f = *f;
    o->p.nubeg = f->nubeg; o->p.nuend = f->nuend;
    o->p.p0koef = f->p0koef; o->p.p1koef = f->p1koef; o->p.p2koef = f->p2koef;
    return 0;
}

int orc_stokes_setup(orc_ctx *o)
{
    if (o->p.p2koef != 0) { snprintf(o->err, sizeof o->err, "p2koef != 0 is not supported"); return I3G_E_UNSUPPORTED; }
    return orc_stokes_build(o);
}

int orc_stokes_vcycles(orc_ctx *o, int n)
{
    for (int i = 0; i < n; i++) orc_vcycle(o, o->f.multinum);
    return 0;
}
int orc_stokes_smooth(orc_ctx *o, int level, int n) { orc_smooth_mc(o, level, n); return 0; }
int orc_stokes_smooth_ref(orc_ctx *o, int level, int n) { orc_smooth_ref(o, level, n); return 0; }
int orc_stokes_residual(orc_ctx *o, int level) { orc_residual(o, level); return 0; }
int orc_stokes_restrict(orc_ctx *o, int level) { orc_restrict(o, level); return 0; }
int orc_stokes_prolong(orc_ctx *o, int level) { orc_prolong(o, level); return 0; }
int orc_stokes_relres(orc_ctx *o, double *mom, double *cont) { orc_relres(o, mom, cont); return 0; }

int orc_get_array(orc_ctx *o, int which, int level, void *dst, int64_t nbytes)
{
    if (level < 0 || level >= o->nlev) return I3G_E_ARG;
    long n = o->mgn[level], p = o->mgp[level];
    switch (which) {
    case I3G_A_SOL: if (nbytes != n * 32) return I3G_E_ARG; memcpy(dst, o->sol + 4 * p, n * 32); return 0;
    case I3G_A_RHS: if (nbytes != n * 32) return I3G_E_ARG; memcpy(dst, o->fre1 + 4 * p, n * 32); return 0;
    case I3G_A_RES: if (nbytes != n * 32) return I3G_E_ARG; memcpy(dst, o->fre0 + 4 * p, n * 32); return 0;
    case I3G_A_NU: if (nbytes != n * 4) return I3G_E_ARG; memcpy(dst, o->nul + p, n * 4); return 0;
    case I3G_A_ETA: if (nbytes != n * 32) return I3G_E_ARG; orc_eta(o, level, (double *)dst); return 0;
    case I3G_A_TK: if (nbytes != o->nodenum * 8 || !o->tsol) return I3G_E_ARG; memcpy(dst, o->tsol, nbytes); return 0;
    }
    return I3G_E_ARG;
}

int orc_set_array(orc_ctx *o, int which, int level, const void *src, int64_t nbytes)
{
    if (level < 0 || level >= o->nlev) return I3G_E_ARG;
    long n = o->mgn[level], p = o->mgp[level];
    switch (which) {
    case I3G_A_SOL: if (nbytes != n * 32) return I3G_E_ARG; memcpy(o->sol + 4 * p, src, n * 32); return 0;
    case I3G_A_RHS: if (nbytes != n * 32) return I3G_E_ARG; memcpy(o->fre1 + 4 * p, src, n * 32); return 0;
    case I3G_A_RES: if (nbytes != n * 32) return I3G_E_ARG; memcpy(o->fre0 + 4 * p, src, n * 32); return 0;
    }
    return I3G_E_ARG;
}

/* Strain rates and stresses from the FP32 velocities (sxxcalc..syzcalc with ynval = 0,
 * as recomputed at move3mg.c:2320-2359). */
static void eps_sig(orc_ctx *o, double *numin, double *numax)
{
    long m1, m2, m3;
    long X = o->nx, Y = o->ny, Z = o->nz, XY = X * Y;
    double out4[4];
    double *eta = xcalloc(o->nodenum * 4, 8);
    orc_eta(o, 0, eta);
    *numin = 1e50; *numax = -1e50;
    for (m3 = 0; m3 < Z; m3++)
        for (m1 = 0; m1 < X; m1++)
            for (m2 = 0; m2 < Y; m2++) {
                long n = m3 * XY + m1 * Y + m2;
                (void)out4;
                if (m1 > 0 && m2 > 0 && m3 > 0) {
                    long v0 = n - XY - Y - 1;
                    double ne = eta[n * 4];
                    double xkf = 1.0 / (o->gx[m1] - o->gx[m1 - 1]);
                    double ykf = 1.0 / (o->gy[m2] - o->gy[m2 - 1]);
                    double zkf = 1.0 / (o->gz[m3] - o->gz[m3 - 1]);
                    double e;
                    e = (o->vx[v0 + Y] - o->vx[v0]) * xkf; o->exx[n] = e; o->sxx[n] = 2.0 * ne * e;
                    e = (o->vy[v0 + 1] - o->vy[v0]) * ykf; o->eyy[n] = e; o->syy[n] = 2.0 * ne * e;
                    e = (o->vz[v0 + XY] - o->vz[v0]) * zkf; o->ezz[n] = e; o->szz[n] = 2.0 * ne * e;
                    *numin = MINV(*numin, ne); *numax = MAXV(*numax, ne);
                }
                if (m1 > 0 && m1 < X - 1 && m2 > 0 && m2 < Y - 1 && m3 < Z - 1) {
                    double xkf = 1.0 / (o->gx[m1 + 1] - o->gx[m1 - 1]);
                    double ykf = 1.0 / (o->gy[m2 + 1] - o->gy[m2 - 1]);
                    long v1 = n - Y, v2 = n - 1;   /* (m1-1,m2,m3), (m1,m2-1,m3) */
                    double e = (o->vx[n] - o->vx[v2]) * ykf + (o->vy[n] - o->vy[v1]) * xkf;
                    o->exy[n] = e; o->sxy[n] = 2.0 * eta[n * 4 + 1] * e;
                }
                if (m1 > 0 && m1 < X - 1 && m2 < Y - 1 && m3 > 0 && m3 < Z - 1) {
                    double xkf = 1.0 / (o->gx[m1 + 1] - o->gx[m1 - 1]);
                    double zkf = 1.0 / (o->gz[m3 + 1] - o->gz[m3 - 1]);
                    long v2 = n - XY, v4 = n - Y;   /* (m1,m2,m3-1), (m1-1,m2,m3) */
                    double e = (o->vx[n] - o->vx[v2]) * zkf + (o->vz[n] - o->vz[v4]) * xkf;
                    o->exz[n] = e; o->sxz[n] = 2.0 * eta[n * 4 + 2] * e;
                }
                if (m1 < X - 1 && m2 > 0 && m2 < Y - 1 && m3 > 0 && m3 < Z - 1) {
                    double ykf = 1.0 / (o->gy[m2 + 1] - o->gy[m2 - 1]);
                    double zkf = 1.0 / (o->gz[m3 + 1] - o->gz[m3 - 1]);
                    long v1 = n - XY, v4 = n - 1;   /* (m1,m2,m3-1), (m1,m2-1,m3) */
                    double e = (o->vy[n] - o->vy[v1]) * zkf + (o->vz[n] - o->vz[v4]) * ykf;
                    o->eyz[n] = e; o->syz[n] = 2.0 * eta[n * 4 + 3] * e;
                }
            }
    free(eta);
}

/* copy the level-0 solution back to the FP32 fields with pressure pinning
 * (move3mg.c:2248-2314); returns min/max of the velocity components */
static int copy_back(orc_ctx *o, double *vmin, double *vmax)
{
    long m1, m2, m3;
    long X = o->nx, Y = o->ny, Z = o->nz;
    long pc = orc_node(o, 0, o->m.pxinit, o->m.pyinit, o->m.pzinit) * 4;
    double shift = o->m.pinit - o->sol[pc];
    for (int k = 0; k < 3; k++) { vmin[k] = 1e30; vmax[k] = -1e30; }
    for (m3 = 0; m3 < Z; m3++)
        for (m1 = 0; m1 < X; m1++)
            for (m2 = 0; m2 < Y; m2++) {
                long n = orc_node(o, 0, m1, m2, m3);
                if (m1 && m2 && m3) {
                    o->pr[n] = o->sol[n * 4] + shift;
                    if (o->pr[n] > 1e12) { snprintf(o->err, sizeof o->err, "pressure too big %e", o->pr[n]); return I3G_E_PRESSURE; }
                }
                if (m2 < Y - 1 && m3 < Z - 1) { o->vx[n] = o->sol[n * 4 + 1]; vmin[0] = MINV(vmin[0], o->vx[n]); vmax[0] = MAXV(vmax[0], o->vx[n]); }
                if (m1 < X - 1 && m3 < Z - 1) { o->vy[n] = o->sol[n * 4 + 2]; vmin[1] = MINV(vmin[1], o->vy[n]); vmax[1] = MAXV(vmax[1], o->vy[n]); }
                if (m1 < X - 1 && m2 < Y - 1) { o->vz[n] = o->sol[n * 4 + 3]; vmin[2] = MINV(vmin[2], o->vz[n]); vmax[2] = MAXV(vmax[2], o->vz[n]); }
            }
    return 0;
}

/* vpiterate (move3mg.c:1585-2636) with the relative-residual stopping rule when
 * stokes_rtol > 0.  The reference's absolute-norm rule is not restated here. */
int orc_stokes(orc_ctx *o, int n0, double *timestep)
{
    (void)n0;
    int rc = orc_stokes_setup(o);
    if (rc) return rc;
    double mom, cont, vmin[3], vmax[3], numin, numax;
    int maxc = o->p.stokes_maxcyc > 0 ? o->p.stokes_maxcyc : 2000;
    double rtol = o->p.stokes_rtol > 0 ? o->p.stokes_rtol : 1e-8;
    int multinum = o->f.multinum, cycles = 0, outer = 0;
    orc_relres(o, &mom, &cont);
    o->st.stokes_rel0 = MAXV(mom, cont);
    int conv = 0;
    while (cycles < maxc) {
        int ncyc = o->p.multicyc > 0 ? o->p.multicyc : 1;
        for (int i = 0; i < ncyc && cycles < maxc; i++) {
            orc_vcycle(o, multinum);
            cycles++;
            orc_relres(o, &mom, &cont);
            if (!(mom == mom) || !(cont == cont)) { snprintf(o->err, sizeof o->err, "NaN in Stokes solve"); return I3G_E_NAN; }
            if (mom <= rtol && cont <= rtol) { conv = 1; break; }
        }
        outer++;
        if (outer >= o->f.multstp) {   /* move3mg.c:2585-2593 */
            multinum = o->f.multinum2;
            o->p.p0koef = o->f.p0koef2; o->p.p1koef = o->f.p1koef2;
        }
        if (conv) break;
    }
    o->p.p0koef = o->f.p0koef; o->p.p1koef = o->f.p1koef;
    rc = copy_back(o, vmin, vmax);
    if (rc) return rc;
    eps_sig(o, &numin, &numax);
    o->st.stokes_cycles = cycles; o->st.stokes_outer = outer;
    o->st.stokes_rel = MAXV(mom, cont); o->st.stokes_mom_rel = mom; o->st.stokes_cont_rel = cont;
    /* CFL time step (move3mg.c:2608-2632) */
    for (int k = 0; k < 3; k++) {
        double vm = MAXV(ABSV(vmin[k]), ABSV(vmax[k]));
        if (vm) { vm = o->f.maxxystep / vm; if (*timestep > vm) *timestep = vm; }
    }
    if (!conv) { snprintf(o->err, sizeof o->err, "Stokes: %d V-cycles without reaching %g", cycles, rtol); return I3G_E_NOCONV; }
    return 0;
}

int orc_get_stats(const orc_ctx *o, i3g_stats *s) { *s = o->st; return 0; }

int orc_download(orc_ctx *o, i3g_model *m, unsigned mask)
{
    long N = o->nodenum, M = o->marknum;
#define CP(dst, src, n, sz) do { if (dst) memcpy(dst, src, (size_t)(n) * (sz)); } while (0)
    if (mask & I3G_SYNC_NODES) {
        CP(m->pr, o->pr, N, 8);
        CP(m->vx, o->vx, N, 4); CP(m->vy, o->vy, N, 4); CP(m->vz, o->vz, N, 4);
        CP(m->ro, o->ro, N, 4); CP(m->nu, o->nu, N, 4); CP(m->nxx, o->nxx, N, 4); CP(m->nxy, o->nxy, N, 4);
        CP(m->nxz, o->nxz, N, 4); CP(m->nyz, o->nyz, N, 4); CP(m->tk, o->tk, N, 4); CP(m->cp, o->cp, N, 4);
        CP(m->et, o->et, N, 4); CP(m->kt, o->kt, N, 4); CP(m->ht, o->ht, N, 4); CP(m->rr, o->rr, N, 4);
    }
    if (mask & I3G_SYNC_STRESS) {
        CP(m->exx, o->exx, N, 4); CP(m->eyy, o->eyy, N, 4); CP(m->ezz, o->ezz, N, 4);
        CP(m->exy, o->exy, N, 4); CP(m->exz, o->exz, N, 4); CP(m->eyz, o->eyz, N, 4);
        CP(m->sxx, o->sxx, N, 4); CP(m->syy, o->syy, N, 4); CP(m->szz, o->szz, N, 4);
        CP(m->sxy, o->sxy, N, 4); CP(m->sxz, o->sxz, N, 4); CP(m->syz, o->syz, N, 4);
    }
    if (mask & I3G_SYNC_MARKERS) {
        CP(m->markx, o->mx, M, 4); CP(m->marky, o->my, M, 4); CP(m->markz, o->mz, M, 4);
        CP(m->markk, o->mk, M, 4); CP(m->markw, o->mw, M, 4); CP(m->markd, o->md, M, 4);
        CP(m->markv, o->mv, M, 4); CP(m->marke, o->me, M, 4); CP(m->markex, o->mex, M, 4);
        CP(m->markft, o->mft, M, 4); CP(m->markrr, o->mrr, M, 4); CP(m->markrn, o->mrn, M, 4);
        CP(m->markt, o->mt, M, 1);
    }
#undef CP
    return 0;
}

int orc_upload(orc_ctx *o, const i3g_model *m, unsigned mask)
{
    long N = o->nodenum;
    if (mask & I3G_SYNC_NODES) {
        memcpy(o->pr, m->pr, N * 8);
        float *d[15] = {o->vx, o->vy, o->vz, o->ro, o->nu, o->nxx, o->nxy, o->nxz, o->nyz, o->tk, o->cp, o->et, o->kt, o->ht, o->rr};
        float *s[15] = {m->vx, m->vy, m->vz, m->ro, m->nu, m->nxx, m->nxy, m->nxz, m->nyz, m->tk, m->cp, m->et, m->kt, m->ht, m->rr};
        for (int i = 0; i < 15; i++) if (s[i]) memcpy(d[i], s[i], N * 4);
    }
    if (mask & I3G_SYNC_STRESS) {
        float *d[12] = {o->exx, o->eyy, o->ezz, o->exy, o->exz, o->eyz, o->sxx, o->syy, o->szz, o->sxy, o->sxz, o->syz};
        float *s[12] = {m->exx, m->eyy, m->ezz, m->exy, m->exz, m->eyz, m->sxx, m->syy, m->szz, m->sxy, m->sxz, m->syz};
        for (int i = 0; i < 12; i++) if (s[i]) memcpy(d[i], s[i], N * 4);
    }
    if (mask & I3G_SYNC_MARKERS) {
        long M = o->marknum;
        float *d[12] = {o->mx, o->my, o->mz, o->mk, o->mw, o->md, o->mv, o->me, o->mex, o->mft, o->mrr, o->mrn};
        float *s[12] = {m->markx, m->marky, m->markz, m->markk, m->markw, m->markd, m->markv, m->marke, m->markex, m->markft, m->markrr, m->markrn};
        for (int i = 0; i < 12; i++) if (s[i]) memcpy(d[i], s[i], M * 4);
        memcpy(o->mt, m->markt, M);
    }
    return 0;
}

/* V-cycles with the multicolour relaxation of the CUDA library (same schedule as
 * move3mg.c:2173-2213; a level with zero down-leg sweeps still forms its residual). */
int orc_stokes_vcycles_mc(orc_ctx *o, int n)
{
    int mn = o->f.multinum < o->nlev - 1 ? o->f.multinum : o->nlev - 1;
    for (int i = 0; i < n; i++) {
        for (int l = 0; l < mn; l++) {
            if (o->p.multinnn[0][l] > 0) orc_smooth_mc(o, l, o->p.multinnn[0][l]);
            else orc_residual(o, l);
            orc_restrict(o, l + 1);
        }
        for (int l = mn; l > 0; l--) {
            if (o->p.multinnn[1][l] > 0) orc_smooth_mc(o, l, o->p.multinnn[1][l]);
            orc_prolong(o, l);
        }
        if (o->p.multinnn[1][0] > 0) orc_smooth_mc(o, 0, o->p.multinnn[1][0]);
    }
    return 0;
}
