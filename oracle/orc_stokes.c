/*
 * orc_stokes.c -- TEST INFRASTRUCTURE (CPU oracle).  Restatement of the reference's
 * staggered-grid Stokes multigrid in plain C, single-threaded, so that it is deterministic
 * (the reference's OpenMP Gauss-Seidel races: move3mg.c:3089-3130).
 *
 *   effective viscosity at stress points ......... sxxcalc..syzcalc  move3mg.c:3-710
 *   momentum rows (17 entries, same entry order) .. x/y/zstokserr      move3mg.c:718-1301
 *   continuity row + nd ........................... continerr          move3mg.c:1310-1425
 *   boundary rows ................................. bonderr            move3mg.c:1532-1579
 *   row store ..................................... gausmat2           gaus3mg.c:67-127
 *   relaxation + residual ......................... gausmat4           move3mg.c:3068-3159
 *   restriction / prolongation .................... vprestrict/vpprolong move3mg.c:3165-3520 / 2748-3063
 *   viscosity restriction ......................... ronurestrict       move3mg.c:2642-2741
 *   V-cycle schedule .............................. vpiterate          move3mg.c:2170-2223
 *
 * Expressions keep the reference's operand order (sums of FP32 fields are formed in FP32,
 * as C evaluates them) so that the assembled rows agree bit for bit.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "orc_internal.h"

#define ABSV(a) ((a) >= 0 ? (a) : -(a))

long orc_node(const orc_ctx *o, int l, long m1, long m2, long m3)
{
    return o->mgp[l] + m3 * o->mgxy[l] + m1 * o->mgy[l] + m2;
}

static double clampnu(const orc_ctx *o, double n)
{
    if (n > o->p.nuend) n = o->p.nuend;
    if (n < o->p.nubeg) n = o->p.nubeg;
    return n;
}

/* average of 8 nodal viscosities by viscmod; v[] in the reference's corner order */
static double avg8(const orc_ctx *o, const long *v)
{
    const float *nu = o->nul;
    double r = 0;
    if (o->p.viscmod == 0)
        r = (nu[v[0]] + nu[v[1]] + nu[v[2]] + nu[v[3]] + nu[v[4]] + nu[v[5]] + nu[v[6]] + nu[v[7]]) / 8.0;
    else if (o->p.viscmod == 1)
        r = exp((log(nu[v[0]]) + log(nu[v[1]]) + log(nu[v[2]]) + log(nu[v[3]]) + log(nu[v[4]]) +
                 log(nu[v[5]]) + log(nu[v[6]]) + log(nu[v[7]])) / 8.0);
    else
        r = 1.0 / ((1.0 / nu[v[0]] + 1.0 / nu[v[1]] + 1.0 / nu[v[2]] + 1.0 / nu[v[3]] + 1.0 / nu[v[4]] +
                    1.0 / nu[v[5]] + 1.0 / nu[v[6]] + 1.0 / nu[v[7]]) / 8.0);
    return r;
}

static double avg2(const orc_ctx *o, long a, long b)
{
    const float *nu = o->nul;
    if (o->p.viscmod == 0) return (nu[a] + nu[b]) / 2.0;
    if (o->p.viscmod == 1) return exp((log(nu[a]) + log(nu[b])) / 2.0);
    return 1.0 / ((1.0 / nu[a] + 1.0 / nu[b]) / 2.0);
}

static void corners(const orc_ctx *o, int l, long base, long *v)
{
    v[0] = base; v[1] = v[0] + 1;
    v[2] = v[0] + o->mgy[l]; v[3] = v[2] + 1;
    v[4] = v[0] + o->mgxy[l]; v[5] = v[4] + 1;
    v[6] = v[4] + o->mgy[l]; v[7] = v[6] + 1;
}

/* normal-stress viscosity of the cell whose upper corner is (m1,m2,m3): sxxcalc nueff */
static double eta_c(const orc_ctx *o, int l, long m1, long m2, long m3)
{
    long v[8];
    corners(o, l, orc_node(o, l, m1 - 1, m2 - 1, m3 - 1), v);
    double n;
    if (l == 0 && m1 > 3 && m2 > 3 && m3 > 3 && m1 < o->mgx[l] - 3 && m2 < o->mgy[l] - 3 && m3 < o->mgz[l] - 3)
        n = o->nxx[v[7]];
    else
        n = avg8(o, v);
    return clampnu(o, n);
}

/* shear viscosities at the sxy / sxz / syz points (m1,m2,m3) */
static double eta_xy(const orc_ctx *o, int l, long m1, long m2, long m3)
{
    long v[8];
    corners(o, l, orc_node(o, l, m1 - 1, m2 - 1, m3), v);
    double n;
    if (l == 0 && m1 > 3 && m2 > 3 && m3 > 2 && m1 < o->mgx[l] - 4 && m2 < o->mgy[l] - 4 && m3 < o->mgz[l] - 4)
        n = o->nxy[v[3]];
    else
        n = avg2(o, v[3], v[7]);
    return clampnu(o, n);
}

static double eta_xz(const orc_ctx *o, int l, long m1, long m2, long m3)
{
    long v[8];
    corners(o, l, orc_node(o, l, m1 - 1, m2, m3 - 1), v);
    double n;
    if (l == 0 && m1 > 3 && m2 > 2 && m3 > 3 && m1 < o->mgx[l] - 4 && m2 < o->mgy[l] - 4 && m3 < o->mgz[l] - 4)
        n = o->nxz[v[6]];
    else
        n = avg2(o, v[6], v[7]);
    return clampnu(o, n);
}

static double eta_yz(const orc_ctx *o, int l, long m1, long m2, long m3)
{
    long v[8];
    corners(o, l, orc_node(o, l, m1, m2 - 1, m3 - 1), v);
    double n;
    if (l == 0 && m1 > 2 && m2 > 3 && m3 > 3 && m1 < o->mgx[l] - 4 && m2 < o->mgy[l] - 4 && m3 < o->mgz[l] - 4)
        n = o->nyz[v[5]];
    else
        n = avg2(o, v[5], v[7]);
    return clampnu(o, n);
}

/* Stress-point viscosities of one level, 4 per node: cell, xy, xz, yz (0 where undefined). */
void orc_eta(orc_ctx *o, int l, double *out)
{
    long m1, m2, m3;
    for (m3 = 0; m3 < o->mgz[l]; m3++)
        for (m1 = 0; m1 < o->mgx[l]; m1++)
            for (m2 = 0; m2 < o->mgy[l]; m2++) {
                long n = (m3 * o->mgxy[l] + m1 * o->mgy[l] + m2) * 4;
                out[n] = out[n + 1] = out[n + 2] = out[n + 3] = 0;
                if (m1 > 0 && m2 > 0 && m3 > 0) out[n] = eta_c(o, l, m1, m2, m3);
                if (m1 > 0 && m1 < o->mgx[l] - 1 && m2 > 0 && m2 < o->mgy[l] - 1 && m3 < o->mgz[l] - 1)
                    out[n + 1] = eta_xy(o, l, m1, m2, m3);
                if (m1 > 0 && m1 < o->mgx[l] - 1 && m3 > 0 && m3 < o->mgz[l] - 1 && m2 < o->mgy[l] - 1)
                    out[n + 2] = eta_xz(o, l, m1, m2, m3);
                if (m2 > 0 && m2 < o->mgy[l] - 1 && m3 > 0 && m3 < o->mgz[l] - 1 && m1 < o->mgx[l] - 1)
                    out[n + 3] = eta_yz(o, l, m1, m2, m3);
            }
}

/* ---- row builders ------------------------------------------------------------------ */
/* A stress term contributes entries e[0..5] (normal) or e[0..3] (shear) with the
 * coefficient forms of sxxcalc..syzcalc: -ynval*nueff*2*dk and +ynval*nueff*2*dk. */
typedef struct { long col[6]; double val[6]; } sterm;

static void t_sxx(const orc_ctx *o, int l, long m1, long m2, long m3, double yn, sterm *t)
{
    double xkf = 1.0 / (o->mggx[l][m1] - o->mggx[l][m1 - 1]);
    long v[8];
    corners(o, l, orc_node(o, l, m1 - 1, m2 - 1, m3 - 1), v);
    double n = eta_c(o, l, m1, m2, m3);
    t->col[0] = v[0] * 4 + 1; t->val[0] = -yn * n * 2.0 * xkf;
    t->col[1] = v[2] * 4 + 1; t->val[1] = +yn * n * 2.0 * xkf;
    t->col[2] = v[0] * 4 + 2; t->val[2] = 0;
    t->col[3] = v[1] * 4 + 2; t->val[3] = 0;
    t->col[4] = v[0] * 4 + 3; t->val[4] = 0;
    t->col[5] = v[4] * 4 + 3; t->val[5] = 0;
}

static void t_syy(const orc_ctx *o, int l, long m1, long m2, long m3, double yn, sterm *t)
{
    double ykf = 1.0 / (o->mggy[l][m2] - o->mggy[l][m2 - 1]);
    long v[8];
    corners(o, l, orc_node(o, l, m1 - 1, m2 - 1, m3 - 1), v);
    double n = eta_c(o, l, m1, m2, m3);
    t->col[0] = v[0] * 4 + 1; t->val[0] = 0;
    t->col[1] = v[2] * 4 + 1; t->val[1] = 0;
    t->col[2] = v[0] * 4 + 2; t->val[2] = -yn * n * 2.0 * ykf;
    t->col[3] = v[1] * 4 + 2; t->val[3] = +yn * n * 2.0 * ykf;
    t->col[4] = v[0] * 4 + 3; t->val[4] = 0;
    t->col[5] = v[4] * 4 + 3; t->val[5] = 0;
}

static void t_szz(const orc_ctx *o, int l, long m1, long m2, long m3, double yn, sterm *t)
{
    double zkf = 1.0 / (o->mggz[l][m3] - o->mggz[l][m3 - 1]);
    long v[8];
    corners(o, l, orc_node(o, l, m1 - 1, m2 - 1, m3 - 1), v);
    double n = eta_c(o, l, m1, m2, m3);
    t->col[0] = v[0] * 4 + 1; t->val[0] = 0;
    t->col[1] = v[2] * 4 + 1; t->val[1] = 0;
    t->col[2] = v[0] * 4 + 2; t->val[2] = 0;
    t->col[3] = v[1] * 4 + 2; t->val[3] = 0;
    t->col[4] = v[0] * 4 + 3; t->val[4] = -yn * n * 2.0 * zkf;
    t->col[5] = v[4] * 4 + 3; t->val[5] = +yn * n * 2.0 * zkf;
}

static void t_sxy(const orc_ctx *o, int l, long m1, long m2, long m3, double yn, sterm *t)
{
    double xkf = 1.0 / (o->mggx[l][m1 + 1] - o->mggx[l][m1 - 1]);
    double ykf = 1.0 / (o->mggy[l][m2 + 1] - o->mggy[l][m2 - 1]);
    long v[8];
    corners(o, l, orc_node(o, l, m1 - 1, m2 - 1, m3), v);
    double n = eta_xy(o, l, m1, m2, m3);
    t->col[0] = v[2] * 4 + 1; t->val[0] = -yn * n * 2.0 * ykf;
    t->col[1] = v[3] * 4 + 1; t->val[1] = +yn * n * 2.0 * ykf;
    t->col[2] = v[1] * 4 + 2; t->val[2] = -yn * n * 2.0 * xkf;
    t->col[3] = v[3] * 4 + 2; t->val[3] = +yn * n * 2.0 * xkf;
}

static void t_sxz(const orc_ctx *o, int l, long m1, long m2, long m3, double yn, sterm *t)
{
    double xkf = 1.0 / (o->mggx[l][m1 + 1] - o->mggx[l][m1 - 1]);
    double zkf = 1.0 / (o->mggz[l][m3 + 1] - o->mggz[l][m3 - 1]);
    long v[8];
    corners(o, l, orc_node(o, l, m1 - 1, m2, m3 - 1), v);
    double n = eta_xz(o, l, m1, m2, m3);
    t->col[0] = v[2] * 4 + 1; t->val[0] = -yn * n * 2.0 * zkf;
    t->col[1] = v[6] * 4 + 1; t->val[1] = +yn * n * 2.0 * zkf;
    t->col[2] = v[4] * 4 + 3; t->val[2] = -yn * n * 2.0 * xkf;
    t->col[3] = v[6] * 4 + 3; t->val[3] = +yn * n * 2.0 * xkf;
}

static void t_syz(const orc_ctx *o, int l, long m1, long m2, long m3, double yn, sterm *t)
{
    double ykf = 1.0 / (o->mggy[l][m2 + 1] - o->mggy[l][m2 - 1]);
    double zkf = 1.0 / (o->mggz[l][m3 + 1] - o->mggz[l][m3 - 1]);
    long v[8];
    corners(o, l, orc_node(o, l, m1, m2 - 1, m3 - 1), v);
    double n = eta_yz(o, l, m1, m2, m3);
    t->col[0] = v[1] * 4 + 2; t->val[0] = -yn * n * 2.0 * zkf;
    t->col[1] = v[5] * 4 + 2; t->val[1] = +yn * n * 2.0 * zkf;
    t->col[2] = v[4] * 4 + 3; t->val[2] = -yn * n * 2.0 * ykf;
    t->col[3] = v[5] * 4 + 3; t->val[3] = +yn * n * 2.0 * ykf;
}

/* set slot s from term entry e, or accumulate into it */
#define SET(s, e) (col[s] = t.col[e], val[s] = t.val[e])
#define ACC(s, e) (val[s] += t.val[e])

/* x-momentum row, slots 1..17 (xstokserr, move3mg.c:718-903) */
static double row_x(const orc_ctx *o, int l, long m1, long m2, long m3, long *col, double *val)
{
    double XK = 2.0 / (o->mggx[l][m1 + 1] - o->mggx[l][m1 - 1]);
    double YK = 1.0 / (o->mggy[l][m2 + 1] - o->mggy[l][m2]);
    double ZK = 1.0 / (o->mggz[l][m3 + 1] - o->mggz[l][m3]);
    long v[8];
    corners(o, l, orc_node(o, l, m1, m2, m3), v);
    const float *ro = o->ro;
    /* coarse right-hand sides are replaced by restricted residuals (move3mg.c:3508-3518) */
    double rhs = l ? 0.0 : -o->m.gxkoef * (ro[v[0]] + ro[v[1]] + ro[v[4]] + ro[v[5]]) / 4.0;
    sterm t;
    col[16] = v[5] * 4; val[16] = +XK;
    col[17] = v[7] * 4; val[17] = -XK;
    t_sxx(o, l, m1, m2 + 1, m3 + 1, -XK, &t);
    SET(2, 0); SET(1, 1); SET(8, 2); SET(9, 3); SET(12, 4); SET(13, 5);
    t_sxx(o, l, m1 + 1, m2 + 1, m3 + 1, XK, &t);
    ACC(1, 0); SET(3, 1); SET(10, 2); SET(11, 3); SET(14, 4); SET(15, 5);
    t_sxy(o, l, m1, m2, m3, -YK, &t);
    ACC(1, 1); SET(4, 0); ACC(8, 2); ACC(10, 3);
    t_sxy(o, l, m1, m2 + 1, m3, YK, &t);
    ACC(1, 0); SET(5, 1); ACC(9, 2); ACC(11, 3);
    t_sxz(o, l, m1, m2, m3, -ZK, &t);
    ACC(1, 1); SET(6, 0); ACC(12, 2); ACC(14, 3);
    t_sxz(o, l, m1, m2, m3 + 1, ZK, &t);
    ACC(1, 0); SET(7, 1); ACC(13, 2); ACC(15, 3);
    return rhs;
}

/* y-momentum row (ystokserr, move3mg.c:910-1101) */
static double row_y(const orc_ctx *o, int l, long m1, long m2, long m3, long *col, double *val)
{
    double XK = 1.0 / (o->mggx[l][m1 + 1] - o->mggx[l][m1]);
    double YK = 2.0 / (o->mggy[l][m2 + 1] - o->mggy[l][m2 - 1]);
    double ZK = 1.0 / (o->mggz[l][m3 + 1] - o->mggz[l][m3]);
    long v[8];
    corners(o, l, orc_node(o, l, m1, m2, m3), v);
    const float *ro = o->ro;
    /* coarse right-hand sides are replaced by restricted residuals (move3mg.c:3508-3518) */
    double rhs = l ? 0.0 : -o->m.gykoef * (ro[v[0]] + ro[v[2]] + ro[v[4]] + ro[v[6]]) / 4.0;
    sterm t;
    col[16] = v[6] * 4; val[16] = +YK;
    col[17] = v[7] * 4; val[17] = -YK;
    t_syy(o, l, m1 + 1, m2, m3 + 1, -YK, &t);
    SET(8, 0); SET(10, 1); SET(4, 2); SET(1, 3); SET(12, 4); SET(14, 5);
    t_syy(o, l, m1 + 1, m2 + 1, m3 + 1, YK, &t);
    SET(9, 0); SET(11, 1); ACC(1, 2); SET(5, 3); SET(13, 4); SET(15, 5);
    t_sxy(o, l, m1, m2, m3, -XK, &t);
    ACC(8, 0); ACC(9, 1); SET(2, 2); ACC(1, 3);
    t_sxy(o, l, m1 + 1, m2, m3, XK, &t);
    ACC(10, 0); ACC(11, 1); ACC(1, 2); SET(3, 3);
    t_syz(o, l, m1, m2, m3, -ZK, &t);
    SET(6, 0); ACC(1, 1); ACC(12, 2); ACC(13, 3);
    t_syz(o, l, m1, m2, m3 + 1, ZK, &t);
    ACC(1, 0); SET(7, 1); ACC(14, 2); ACC(15, 3);
    return rhs;
}

/* z-momentum row (zstokserr, move3mg.c:1109-1301) */
static double row_z(const orc_ctx *o, int l, long m1, long m2, long m3, long *col, double *val)
{
    double XK = 1.0 / (o->mggx[l][m1 + 1] - o->mggx[l][m1]);
    double YK = 1.0 / (o->mggy[l][m2 + 1] - o->mggy[l][m2]);
    double ZK = 2.0 / (o->mggz[l][m3 + 1] - o->mggz[l][m3 - 1]);
    long v[8];
    corners(o, l, orc_node(o, l, m1, m2, m3), v);
    const float *ro = o->ro;
    /* coarse right-hand sides are replaced by restricted residuals (move3mg.c:3508-3518) */
    double rhs = l ? 0.0 : -o->m.gzkoef * (ro[v[0]] + ro[v[1]] + ro[v[2]] + ro[v[3]]) / 4.0;
    sterm t;
    col[16] = v[3] * 4; val[16] = +ZK;
    col[17] = v[7] * 4; val[17] = -ZK;
    t_szz(o, l, m1 + 1, m2 + 1, m3, -ZK, &t);
    SET(12, 0); SET(14, 1); SET(8, 2); SET(9, 3); SET(6, 4); SET(1, 5);
    t_szz(o, l, m1 + 1, m2 + 1, m3 + 1, ZK, &t);
    SET(13, 0); SET(15, 1); SET(10, 2); SET(11, 3); ACC(1, 4); SET(7, 5);
    t_sxz(o, l, m1, m2, m3, -XK, &t);
    ACC(12, 0); ACC(13, 1); SET(2, 2); ACC(1, 3);
    t_sxz(o, l, m1 + 1, m2, m3, XK, &t);
    ACC(14, 0); ACC(15, 1); ACC(1, 2); SET(3, 3);
    t_syz(o, l, m1, m2, m3, -YK, &t);
    ACC(8, 0); ACC(10, 1); SET(4, 2); ACC(1, 3);
    t_syz(o, l, m1, m2 + 1, m3, YK, &t);
    ACC(9, 0); ACC(11, 1); ACC(1, 2); SET(5, 3);
    return rhs;
}
#undef SET
#undef ACC

/* continuity row of the cell with upper corner (m1,m2,m3) (continerr, move3mg.c:1310-1425) */
static void row_c(orc_ctx *o, int l, long m1, long m2, long m3, long *col, double *val)
{
    double xkf = 1.0 / (o->mggx[l][m1] - o->mggx[l][m1 - 1]);
    double ykf = 1.0 / (o->mggy[l][m2] - o->mggy[l][m2 - 1]);
    double zkf = 1.0 / (o->mggz[l][m3] - o->mggz[l][m3 - 1]);
    long v[8];
    corners(o, l, orc_node(o, l, m1 - 1, m2 - 1, m3 - 1), v);
    o->nd[v[7]] = (float)eta_c(o, l, m1, m2, m3);
    col[1] = v[0] * 4 + 1; val[1] = -xkf;
    col[2] = v[2] * 4 + 1; val[2] = +xkf;
    col[3] = v[0] * 4 + 2; val[3] = -ykf;
    col[4] = v[1] * 4 + 2; val[4] = +ykf;
    col[5] = v[0] * 4 + 3; val[5] = -zkf;
    col[6] = v[4] * 4 + 3; val[6] = +zkf;
}

static int row_exists(const orc_ctx *o, int l, long m1, long m2, long m3, int var)
{
    switch (var) {
    case 0: return m1 && m2 && m3;
    case 1: return m2 < o->mgy[l] - 1 && m3 < o->mgz[l] - 1;
    case 2: return m1 < o->mgx[l] - 1 && m3 < o->mgz[l] - 1;
    default: return m1 < o->mgx[l] - 1 && m2 < o->mgy[l] - 1;
    }
}

/* ronurestrict(mgi) (move3mg.c:2642-2741): volume-weighted viscosity restriction */
static void ronurestrict(orc_ctx *o, int mgi)
{
    long m1, m2, m3, m10, m20, m30;
    double *w = o->wsum;
    for (m1 = o->mgp[mgi]; m1 < o->mgp[mgi] + o->mgn[mgi]; m1++) { o->nul[m1] = 0; w[m1] = 0; }
    int f = mgi - 1;
    for (m3 = 0; m3 < o->mgz[f]; m3++)
        for (m1 = 0; m1 < o->mgx[f]; m1++)
            for (m2 = 0; m2 < o->mgy[f]; m2++) {
                long m4 = orc_node(o, f, m1, m2, m3);
                long a = (m1 - 2) / 2 + 2, b = (m2 - 2) / 2 + 2, c = (m3 - 2) / 2 + 2;
                if (m1 < 3) a = m1;
                if (m1 > o->mgx[f] - 4) a = o->mgx[mgi] - (o->mgx[f] - m1);
                if (a > o->mgx[mgi] - 2) a = o->mgx[mgi] - 2;
                if (m2 < 3) b = m2;
                if (m2 > o->mgy[f] - 4) b = o->mgy[mgi] - (o->mgy[f] - m2);
                if (b > o->mgy[mgi] - 2) b = o->mgy[mgi] - 2;
                if (m3 < 3) c = m3;
                if (m3 > o->mgz[f] - 4) c = o->mgz[mgi] - (o->mgz[f] - m3);
                if (c > o->mgz[mgi] - 2) c = o->mgz[mgi] - 2;
                double dx = o->mggx[mgi][a + 1] - o->mggx[mgi][a];
                double dy = o->mggy[mgi][b + 1] - o->mggy[mgi][b];
                double dz = o->mggz[mgi][c + 1] - o->mggz[mgi][c];
                for (m30 = c; m30 <= c + 1; m30++) {
                    double ddz = (o->mggz[mgi][m30] - o->mggz[f][m3]) / dz;
                    ddz = 1.0 - ABSV(ddz);
                    for (m10 = a; m10 <= a + 1; m10++) {
                        double ddx = (o->mggx[mgi][m10] - o->mggx[f][m1]) / dx;
                        ddx = 1.0 - ABSV(ddx);
                        for (m20 = b; m20 <= b + 1; m20++) {
                            double ddy = (o->mggy[mgi][m20] - o->mggy[f][m2]) / dy;
                            ddy = 1.0 - ABSV(ddy);
                            long m40 = orc_node(o, mgi, m10, m20, m30);
                            double swt = ddx * ddy * ddz, iv = 0;
                            if (o->p.viscmod == 0) iv = o->nul[m4] * swt;
                            if (o->p.viscmod == 1) iv = log(o->nul[m4]) * swt;
                            if (o->p.viscmod == 2) iv = 1.0 / o->nul[m4] * swt;
                            o->nul[m40] += iv;   /* FP32 accumulator, as nu[] */
                            w[m40] += swt;
                        }
                    }
                }
            }
    for (m1 = o->mgp[mgi]; m1 < o->mgp[mgi] + o->mgn[mgi]; m1++) {
        o->nul[m1] /= w[m1];
        if (o->p.viscmod == 1) o->nul[m1] = exp(o->nul[m1]);
        if (o->p.viscmod == 2) o->nul[m1] = 1.0 / o->nul[m1];
        w[m1] = 0;
    }
}

/* Assemble rows of all levels and load v,P into the level-0 solution
 * (vpiterate set-up, move3mg.c:1948-2159). */
int orc_stokes_build(orc_ctx *o)
{
    int l;
    long m1, m2, m3, k;
    long nrow = o->ntot * 4;
    for (k = 0; k < o->nodenum; k++) o->nul[k] = o->nu[k];
    for (l = 1; l < o->nlev; l++) ronurestrict(o, l);
    memset(o->sol, 0, sizeof(double) * nrow);
    for (m3 = 0; m3 < o->mgz[0]; m3++)
        for (m1 = 0; m1 < o->mgx[0]; m1++)
            for (m2 = 0; m2 < o->mgy[0]; m2++) {
                long n = orc_node(o, 0, m1, m2, m3);
                if (row_exists(o, 0, m1, m2, m3, 0)) o->sol[n * 4 + 0] = o->pr[n];
                if (row_exists(o, 0, m1, m2, m3, 1)) o->sol[n * 4 + 1] = o->vx[n];
                if (row_exists(o, 0, m1, m2, m3, 2)) o->sol[n * 4 + 2] = o->vy[n];
                if (row_exists(o, 0, m1, m2, m3, 3)) o->sol[n * 4 + 3] = o->vz[n];
            }
    long pos = 0;
    long col[24];
    double val[24];
    for (l = 0; l < o->nlev; l++)
        for (m3 = 0; m3 < o->mgz[l]; m3++)
            for (m1 = 0; m1 < o->mgx[l]; m1++)
                for (m2 = 0; m2 < o->mgy[l]; m2++) {
                    long n = orc_node(o, l, m1, m2, m3);
                    for (int var = 0; var < 4; var++) {
                        long r = n * 4 + var;
                        o->rowptr[r] = pos;
                        if (!row_exists(o, l, m1, m2, m3, var)) { o->rowptr[r + 1] = pos; continue; }
                        int cnt;
                        double rhs = 0;
                        int b = o->bcid[r];
                        if (b >= 0) {
                            col[1] = r; val[1] = 1.0; cnt = 1;
                            if (o->bc_p[b] >= 0) { col[2] = o->bc_p[b]; val[2] = -o->bc_k[b]; cnt = 2; }
                            rhs = o->bc_c[b];
                        } else if (var == 0) {
                            row_c(o, l, m1, m2, m3, col, val); cnt = 6;
                        } else {
                            if (var == 1) rhs = row_x(o, l, m1, m2, m3, col, val);
                            else if (var == 2) rhs = row_y(o, l, m1, m2, m3, col, val);
                            else rhs = row_z(o, l, m1, m2, m3, col, val);
                            cnt = 17;
                        }
                        for (int e = 1; e <= cnt; e++) { o->col[pos] = col[e]; o->val[pos] = val[e]; pos++; }
                        o->fre1[r] = rhs;
                        o->rowptr[r + 1] = pos;
                    }
                }
    return 0;
}

/* gausmat4 relaxation in the reference's lexicographic order (move3mg.c:3087-3131) */
void orc_smooth_ref(orc_ctx *o, int l, int nsweeps)
{
    long beg = o->mgp[l] * 4, end = (o->mgp[l] + o->mgn[l]) * 4;
    for (int s = 0; s < nsweeps; s++)
        for (long r = beg; r < end; r++) {
            long a = o->rowptr[r], b = o->rowptr[r + 1];
            if (a == b) continue;
            double iv = -o->fre1[r];
            double diag = o->val[a];
            for (long e = a; e < b; e++) iv += o->val[e] * o->sol[o->col[e]];
            if (r % 4 == 0) {
                if (o->bcid[r] < 0) o->sol[r] -= iv * o->nd[r / 4] * o->p.p0koef;
                else o->sol[r] -= iv;
            } else {
                if (o->bcid[r] < 0) o->sol[r] -= iv / diag * o->p.v0koef;
                else o->sol[r] -= iv;
            }
        }
    orc_residual(o, l);
}

/* fre0 = fre1 - A sol0 on one level (move3mg.c:3136-3157) */
void orc_residual(orc_ctx *o, int l)
{
    long beg = o->mgp[l] * 4, end = (o->mgp[l] + o->mgn[l]) * 4;
    for (long r = beg; r < end; r++) {
        long a = o->rowptr[r], b = o->rowptr[r + 1];
        if (a == b) continue;
        double iv = o->fre1[r];
        for (long e = a; e < b; e++) iv -= o->val[e] * o->sol[o->col[e]];
        o->fre0[r] = iv;
    }
}

/* Flattened boundary value: follow partner links to a row that is not a boundary row
 * (the fixed point of the reference's boundary rows, bonderr move3mg.c:1532-1579). */
static double bc_value(const orc_ctx *o, long r, int depth)
{
    int b = o->bcid[r];
    if (b < 0) return o->sol[r];
    if (depth > 16) return 0;
    double c = o->fre1[r];             /* c on level 0, 0 on coarse levels after restriction */
    if (o->bc_p[b] < 0) return c;
    long pr = o->bc_p[b];
    if (o->rowptr[pr] == o->rowptr[pr + 1]) return c + o->bc_k[b] * o->sol[pr];
    return c + o->bc_k[b] * bc_value(o, pr, depth + 1);
}

/* Multicolour sweep (the CUDA library's order): for each velocity component red then black
 * interior rows, then that component's boundary rows; then all interior pressure rows,
 * then pressure boundary rows.  Each row uses the gausmat4 update formula. */
void orc_smooth_mc(orc_ctx *o, int l, int nsweeps)
{
    long m1, m2, m3;
    long NX = o->mgx[l], NY = o->mgy[l], NZ = o->mgz[l];
    double *tmp = o->wsum;
    for (int s = 0; s < nsweeps; s++) {
        for (int var = 1; var <= 4; var++) {
            int v = var & 3;   /* 1,2,3 then 0 (pressure) */
            for (int color = 0; color < (v ? 2 : 1); color++) {
                /* compute all updates of this colour from the same state, then apply */
                for (m3 = 0; m3 < NZ; m3++)
                    for (m1 = 0; m1 < NX; m1++)
                        for (m2 = 0; m2 < NY; m2++) {
                            long r = orc_node(o, l, m1, m2, m3) * 4 + v;
                            if (v && ((m1 + m2 + m3) & 1) != color) continue;
                            long a = o->rowptr[r], b = o->rowptr[r + 1];
                            if (a == b || o->bcid[r] >= 0) continue;
                            double iv = -o->fre1[r];
                            for (long e = a; e < b; e++) iv += o->val[e] * o->sol[o->col[e]];
                            if (v == 0) tmp[r / 4] = o->sol[r] - iv * o->nd[r / 4] * o->p.p0koef;
                            else tmp[r / 4] = o->sol[r] - iv / o->val[a] * o->p.v0koef;
                        }
                for (m3 = 0; m3 < NZ; m3++)
                    for (m1 = 0; m1 < NX; m1++)
                        for (m2 = 0; m2 < NY; m2++) {
                            long r = orc_node(o, l, m1, m2, m3) * 4 + v;
                            if (v && ((m1 + m2 + m3) & 1) != color) continue;
                            if (o->rowptr[r] == o->rowptr[r + 1] || o->bcid[r] >= 0) continue;
                            o->sol[r] = tmp[r / 4];
                        }
            }
            /* boundary rows of this component (partners are interior after flattening) */
            for (m3 = 0; m3 < NZ; m3++)
                for (m1 = 0; m1 < NX; m1++)
                    for (m2 = 0; m2 < NY; m2++) {
                        long r = orc_node(o, l, m1, m2, m3) * 4 + v;
                        if (o->rowptr[r] == o->rowptr[r + 1] || o->bcid[r] < 0) continue;
                        tmp[r / 4] = bc_value(o, r, 0);
                    }
            for (m3 = 0; m3 < NZ; m3++)
                for (m1 = 0; m1 < NX; m1++)
                    for (m2 = 0; m2 < NY; m2++) {
                        long r = orc_node(o, l, m1, m2, m3) * 4 + v;
                        if (o->rowptr[r] == o->rowptr[r + 1] || o->bcid[r] < 0) continue;
                        o->sol[r] = tmp[r / 4];
                    }
        }
        for (long k = o->mgp[l]; k < o->mgp[l] + o->mgn[l]; k++) tmp[k] = 0;
    }
    orc_residual(o, l);
}

/* Index of the lower of the two coarse nodes used for fine index m, in one direction, for
 * a quantity living on grid lines (staggered == 0), on mid-points (staggered == 1) or on
 * cell centres (staggered == 2), with the boundary rules of move3mg.c:2769-2782 etc. */
static long cmin_idx(const orc_ctx *o, int lc, long m, const double *gf, const double *gc, long nf, long nc, int stag)
{
    long a = (m - 2) / 2 + 2;
    if (m < 3) a = m;
    if (m > nf - 4) a = nc - (nf - m);
    if (stag == 0) { if (a > nc - 2) a = nc - 2; }
    else if (stag == 1) {
        if (a > nc - 3) a = nc - 3;
        if ((gf[m] + gf[m + 1]) / 2.0 < (gc[a] + gc[a + 1]) / 2.0 && a > 0) a -= 1;
    } else {
        if (a > nc - 2) a = nc - 2;
        if ((gf[m] + gf[m - 1]) / 2.0 < (gc[a] + gc[a - 1]) / 2.0 && a > 1) a -= 1;
    }
    (void)lc;
    return a;
}

/* one-dimensional weights (ddx of the reference) for coarse index k in {a, a+1} */
static double w1(long k, long a, const double *gf, const double *gc, long m, int stag, double d)
{
    double dd;
    if (stag == 0) dd = (gc[k] - gf[m]) / d;
    else if (stag == 1) dd = (gc[k] + gc[k + 1] - gf[m] - gf[m + 1]) / 2.0 / d;
    else dd = (gc[k] + gc[k - 1] - gf[m] - gf[m - 1]) / 2.0 / d;
    if (k == a) dd = -dd;
    return 1.0 - dd;
}

static double span(const double *gc, long a, int stag)
{
    if (stag == 0) return gc[a + 1] - gc[a];
    if (stag == 1) return (gc[a + 2] - gc[a]) / 2.0;
    return (gc[a + 1] - gc[a - 1]) / 2.0;
}

/* staggering of variable var along each axis: 0 grid line, 1 mid-point, 2 cell centre */
static const int STAG[4][3] = {{2, 2, 2}, {0, 1, 1}, {1, 0, 1}, {1, 1, 0}};

/* vprestrict(mgi) (move3mg.c:3165-3520) */
void orc_restrict(orc_ctx *o, int mgi)
{
    int f = mgi - 1;
    long m1, m2, m3, r;
    for (r = o->mgp[mgi] * 4; r < (o->mgp[mgi] + o->mgn[mgi]) * 4; r++) { o->fre1[r] = 0; o->wsum[r] = 0; }
    for (m3 = 0; m3 < o->mgz[f]; m3++)
        for (m1 = 0; m1 < o->mgx[f]; m1++)
            for (m2 = 0; m2 < o->mgy[f]; m2++) {
                long m4 = orc_node(o, f, m1, m2, m3);
                for (int var = 1; var <= 4; var++) {
                    int v = var & 3;
                    if (!row_exists(o, f, m1, m2, m3, v) || o->bcid[m4 * 4 + v] >= 0) continue;
                    const int *s = STAG[v];
                    long a = cmin_idx(o, mgi, m1, o->mggx[f], o->mggx[mgi], o->mgx[f], o->mgx[mgi], s[0]);
                    long b = cmin_idx(o, mgi, m2, o->mggy[f], o->mggy[mgi], o->mgy[f], o->mgy[mgi], s[1]);
                    long c = cmin_idx(o, mgi, m3, o->mggz[f], o->mggz[mgi], o->mgz[f], o->mgz[mgi], s[2]);
                    double dx = span(o->mggx[mgi], a, s[0]), dy = span(o->mggy[mgi], b, s[1]), dz = span(o->mggz[mgi], c, s[2]);
                    for (long k3 = c; k3 <= c + 1; k3++) {
                        double ddz = w1(k3, c, o->mggz[f], o->mggz[mgi], m3, s[2], dz);
                        for (long k1 = a; k1 <= a + 1; k1++) {
                            double ddx = w1(k1, a, o->mggx[f], o->mggx[mgi], m1, s[0], dx);
                            for (long k2 = b; k2 <= b + 1; k2++) {
                                double ddy = w1(k2, b, o->mggy[f], o->mggy[mgi], m2, s[1], dy);
                                long m40 = orc_node(o, mgi, k1, k2, k3);
                                if (o->bcid[m40 * 4 + v] >= 0) continue;
                                double swt = ddx * ddy * ddz;
                                double iv;
                                if (v == 0) iv = o->fre0[m4 * 4] * o->nd[m4] / o->nd[m40] * swt;
                                else iv = o->fre0[m4 * 4 + v] * swt;
                                o->fre1[m40 * 4 + v] += iv;
                                o->wsum[m40 * 4 + v] += swt;
                            }
                        }
                    }
                }
            }
    for (r = o->mgp[mgi] * 4; r < (o->mgp[mgi] + o->mgn[mgi]) * 4; r++) {
        if (o->wsum[r]) { o->fre1[r] /= o->wsum[r]; o->wsum[r] = 0; }
        o->sol[r] = 0;
    }
}

/* vpprolong(mgi, 0) (move3mg.c:2748-3063) */
void orc_prolong(orc_ctx *o, int mgi)
{
    int f = mgi - 1;
    long m1, m2, m3;
    for (m3 = 0; m3 < o->mgz[f]; m3++)
        for (m1 = 0; m1 < o->mgx[f]; m1++)
            for (m2 = 0; m2 < o->mgy[f]; m2++) {
                long m4 = orc_node(o, f, m1, m2, m3);
                for (int var = 1; var <= 4; var++) {
                    int v = var & 3;
                    if (!row_exists(o, f, m1, m2, m3, v)) continue;
                    const int *s = STAG[v];
                    long a = cmin_idx(o, mgi, m1, o->mggx[f], o->mggx[mgi], o->mgx[f], o->mgx[mgi], s[0]);
                    long b = cmin_idx(o, mgi, m2, o->mggy[f], o->mggy[mgi], o->mgy[f], o->mgy[mgi], s[1]);
                    long c = cmin_idx(o, mgi, m3, o->mggz[f], o->mggz[mgi], o->mgz[f], o->mgz[mgi], s[2]);
                    double dx = span(o->mggx[mgi], a, s[0]), dy = span(o->mggy[mgi], b, s[1]), dz = span(o->mggz[mgi], c, s[2]);
                    double kf = v ? o->p.v1koef : o->p.p1koef;
                    for (long k3 = c; k3 <= c + 1; k3++) {
                        double ddz = w1(k3, c, o->mggz[f], o->mggz[mgi], m3, s[2], dz);
                        for (long k1 = a; k1 <= a + 1; k1++) {
                            double ddx = w1(k1, a, o->mggx[f], o->mggx[mgi], m1, s[0], dx);
                            for (long k2 = b; k2 <= b + 1; k2++) {
                                double ddy = w1(k2, b, o->mggy[f], o->mggy[mgi], m2, s[1], dy);
                                long m40 = orc_node(o, mgi, k1, k2, k3);
                                double swt = ddx * ddy * ddz;
                                o->sol[m4 * 4 + v] += o->sol[m40 * 4 + v] * swt * kf;
                            }
                        }
                    }
                }
            }
}

/* V-cycle of move3mg.c:2173-2213 with the reference's relaxation */
void orc_vcycle(orc_ctx *o, int multinum)
{
    int l;
    for (l = 0; l < multinum; l++) {
        if (o->p.multinnn[0][l] > 0) orc_smooth_ref(o, l, o->p.multinnn[0][l]);
        orc_restrict(o, l + 1);
    }
    for (l = multinum; l > 0; l--) {
        if (o->p.multinnn[1][l] > 0) orc_smooth_ref(o, l, o->p.multinnn[1][l]);
        orc_prolong(o, l);
    }
    if (o->p.multinnn[1][0] > 0) orc_smooth_ref(o, 0, o->p.multinnn[1][0]);
}

/* Relative residuals of the level-0 system: momentum ||b - A x|| / ||b|| over non-boundary
 * velocity rows; continuity RMS(div v) * mean spacing / RMS(v). */
void orc_relres(orc_ctx *o, double *mom, double *cont)
{
    double rb = 0, bb = 0, rc = 0, vv = 0, nc = 0, nv = 0;
    for (long r = 0; r < o->mgn[0] * 4; r++) {
        long a = o->rowptr[r], b = o->rowptr[r + 1];
        if (a == b) continue;
        if (r % 4) { vv += o->sol[r] * o->sol[r]; nv += 1; }
        if (o->bcid[r] >= 0) continue;
        double x = o->fre1[r];
        for (long e = a; e < b; e++) x -= o->val[e] * o->sol[o->col[e]];
        if (r % 4) { rb += x * x; bb += o->fre1[r] * o->fre1[r]; }
        else { rc += x * x; nc += 1; }
    }
    double h = (o->m.xsize / (o->nx - 1) + o->m.ysize / (o->ny - 1) + o->m.zsize / (o->nz - 1)) / 3.0;
    *mom = bb > 0 ? sqrt(rb / bb) : sqrt(rb);
    *cont = (nc > 0 && vv > 0) ? sqrt(rc / nc) * h / sqrt(vv / nv) : sqrt(rc);
}

/* Assembled rows of one level (for exact comparison with the reference's row store). */
int orc_get_csr(orc_ctx *o, int l, int64_t *counts, int64_t *cols, double *vals)
{
    long beg = o->mgp[l] * 4, end = (o->mgp[l] + o->mgn[l]) * 4, k = 0;
    for (long r = beg; r < end; r++) {
        long a = o->rowptr[r], b = o->rowptr[r + 1];
        if (counts) counts[r - beg] = b - a;
        for (long e = a; e < b; e++, k++) {
            if (cols) cols[k] = o->col[e];
            if (vals) vals[k] = o->val[e];
        }
    }
    return 0;
}
