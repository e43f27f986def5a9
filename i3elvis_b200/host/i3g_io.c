/*
 * i3g_io.c -- .prn, mode.t3c and file.t3c for the C host loop.
 *
 * .prn byte layout (native little-endian, sizeof(long) == 8, no padding; load3mg.c:704-892
 * reads it, load3mg.c:898-1063 writes it):
 *   4 bytes  sizes of int, long, float, double
 *   header   xnumx ynumy znumz mnumx mnumy mnumz (i64), xsize ysize zsize (f64),
 *            pxinit pyinit pzinit (i64), pinit gxkoef gykoef gzkoef (f64), rocknum (i32),
 *            bondnum marknum (i64), cycle (i32), timesum in years, gridcur, gridtot (f64)
 *   rocks    24 tables of rocknum doubles
 *   nodes    16 floats per node: pr vx vy vz ro nu nxx nxy nxz nyz tk cp et kt ht rr
 *   grid     gx[xnumx] gy[ynumy] gz[znumz] as floats
 *   bonds    bondnum records: row (i64), id (i64), c (f32), k (f32), partner row + 1 (i64)
 *   markers  marknum records: x y z k w d v e ex ft rr rn (f32) and the rock type (char)
 */
#include "i3g_io.h"

#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static int failf(char *err, const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(err, 256, fmt, ap);
    va_end(ap);
    return -1;
}

#define RD(ptr, size, n)                                                                       \
    do {                                                                                       \
        if ((long)fread((ptr), (size), (n), fl) != (long)(n)) {                                \
            fclose(fl);                                                                        \
            return failf(err, "%s: truncated file", path);                                     \
        }                                                                                      \
    } while (0)

#define WR(ptr, size, n)                                                                       \
    do {                                                                                       \
        if ((long)fwrite((ptr), (size), (n), fl) != (long)(n)) {                               \
            fclose(fl);                                                                        \
            return failf(err, "%s: write failed", path);                                       \
        }                                                                                      \
    } while (0)

static void *xcalloc(long n, long size) { return calloc(n > 0 ? n : 1, size); }

static void *(*g_alloc)(int64_t) = NULL;
static void (*g_release)(void *) = NULL;

void prn_set_allocator(void *(*alloc)(int64_t bytes), void (*release)(void *))
{
    g_alloc = alloc && release ? alloc : NULL;
    g_release = alloc && release ? release : NULL;
}

/* large arrays: the installed allocator (page-locked memory in the host loop), else calloc */
static void *big_alloc(const prn_file *p, long n, long size)
{
    if (p->release != free && g_alloc) return g_alloc((int64_t)(n > 0 ? n : 1) * size);
    return xcalloc(n, size);
}

static void big_free(const prn_file *p, void *a)
{
    if (a) (p->release ? p->release : free)(a);
}

/* the large arrays of an image */
static int alloc_arrays(prn_file *p, long nn, long mn)
{
    p->release = g_alloc ? g_release : free;
    p->pr = (double *)big_alloc(p, nn, 8);
    int ok = p->pr != NULL;
    for (int f = 0; f < 15; f++) ok &= (p->node[f] = (float *)big_alloc(p, nn, 4)) != NULL;
    for (int f = 0; f < 12; f++) ok &= (p->stress[f] = (float *)big_alloc(p, nn, 4)) != NULL;
    for (int f = 0; f < 12; f++) ok &= (p->mark[f] = (float *)big_alloc(p, mn, 4)) != NULL;
    ok &= (p->markt = (int8_t *)big_alloc(p, mn, 1)) != NULL;
    return ok ? 0 : -1;
}

/* i3g_model pointers of an image to its own arrays */
static void bind_model(prn_file *p)
{
    i3g_model *m = &p->m;
    for (int t = 0; t < 24; t++) m->rock[t] = p->rock[t];
    m->gx = p->gxf; m->gy = p->gyf; m->gz = p->gzf;
    m->pr = p->pr;
    float **nf[15] = {&m->vx, &m->vy, &m->vz, &m->ro, &m->nu, &m->nxx, &m->nxy, &m->nxz, &m->nyz,
                      &m->tk, &m->cp, &m->et, &m->kt, &m->ht, &m->rr};
    for (int f = 0; f < 15; f++) *nf[f] = p->node[f];
    float **sf[12] = {&m->exx, &m->eyy, &m->ezz, &m->exy, &m->exz, &m->eyz,
                      &m->sxx, &m->syy, &m->szz, &m->sxy, &m->sxz, &m->syz};
    for (int f = 0; f < 12; f++) *sf[f] = p->stress[f];
    m->bond_row = p->brow; m->bond_c = p->bc; m->bond_k = p->bk; m->bond_partner1 = p->bp1;
    float **mf[12] = {&m->markx, &m->marky, &m->markz, &m->markk, &m->markw, &m->markd, &m->markv,
                      &m->marke, &m->markex, &m->markft, &m->markrr, &m->markrn};
    for (int f = 0; f < 12; f++) *mf[f] = p->mark[f];
    m->markt = p->markt;
}

int prn_read(const char *path, prn_file *p, char *err)
{
    memset(p, 0, sizeof *p);
    FILE *fl = fopen(path, "rb");
    if (!fl) return failf(err, "cannot open %s", path);
    unsigned char sz[4];
    RD(sz, 1, 4);
    if (sz[0] != 4 || sz[1] != 8 || sz[2] != 4 || sz[3] != 8) {
        fclose(fl);
        return failf(err, "%s: type sizes %d %d %d %d differ from int 4, long 8, float 4, double 8", path, sz[0], sz[1], sz[2], sz[3]);
    }
    i3g_model *m = &p->m;
    double timesum_yr;
    RD(&m->xnumx, 8, 1); RD(&m->ynumy, 8, 1); RD(&m->znumz, 8, 1);
    RD(&m->mnumx, 8, 1); RD(&m->mnumy, 8, 1); RD(&m->mnumz, 8, 1);
    RD(&m->xsize, 8, 1); RD(&m->ysize, 8, 1); RD(&m->zsize, 8, 1);
    RD(&m->pxinit, 8, 1); RD(&m->pyinit, 8, 1); RD(&m->pzinit, 8, 1);
    RD(&m->pinit, 8, 1); RD(&m->gxkoef, 8, 1); RD(&m->gykoef, 8, 1); RD(&m->gzkoef, 8, 1);
    RD(&m->rocknum, 4, 1); RD(&m->bondnum, 8, 1); RD(&m->marknum, 8, 1); RD(&p->cycle, 4, 1);
    RD(&timesum_yr, 8, 1); RD(&p->gridcur, 8, 1); RD(&p->gridtot, 8, 1);
    m->timesum = timesum_yr * I3G_YEAR;
    if (m->xnumx < 5 || m->ynumy < 5 || m->znumz < 5 || m->rocknum < 0 || m->bondnum < 0 || m->marknum < 0) {
        fclose(fl);
        return failf(err, "%s: implausible header", path);
    }
    const long rn = m->rocknum, nn = (long)(m->xnumx * m->ynumy * m->znumz);
    const long bn = (long)m->bondnum, mn = (long)m->marknum;
    for (int t = 0; t < 24; t++) {
        p->rock[t] = (double *)xcalloc(rn, 8);
        RD(p->rock[t], 8, rn);
        m->rock[t] = p->rock[t];
    }
    if (alloc_arrays(p, nn, mn)) { fclose(fl); prn_free(p); return failf(err, "%s: out of host memory", path); }
    {
        const long chunk = 1 << 16;
        float *buf = (float *)malloc(sizeof(float) * 16 * chunk);
        for (long a = 0; a < nn; a += chunk) {
            const long n = nn - a < chunk ? nn - a : chunk;
            if ((long)fread(buf, 64, n, fl) != n) { free(buf); fclose(fl); return failf(err, "%s: truncated nodes", path); }
            for (long q = 0; q < n; q++) {
                p->pr[a + q] = (double)buf[16 * q];
                for (int f = 0; f < 15; f++) p->node[f][a + q] = buf[16 * q + 1 + f];
            }
        }
        free(buf);
    }
    p->gxf = (float *)xcalloc(m->xnumx, 4); p->gyf = (float *)xcalloc(m->ynumy, 4); p->gzf = (float *)xcalloc(m->znumz, 4);
    RD(p->gxf, 4, m->xnumx); RD(p->gyf, 4, m->ynumy); RD(p->gzf, 4, m->znumz);
    p->brow = (int64_t *)xcalloc(bn, 8); p->bond_id = (int64_t *)xcalloc(bn, 8); p->bp1 = (int64_t *)xcalloc(bn, 8);
    p->bc = (float *)xcalloc(bn, 4); p->bk = (float *)xcalloc(bn, 4);
    for (long b = 0; b < bn; b++) {
        RD(&p->brow[b], 8, 1); RD(&p->bond_id[b], 8, 1); RD(&p->bc[b], 4, 1); RD(&p->bk[b], 4, 1); RD(&p->bp1[b], 8, 1);
    }
    {
        const long chunk = 1 << 16;
        unsigned char *buf = (unsigned char *)malloc(49 * chunk);
        for (long a = 0; a < mn; a += chunk) {
            const long n = mn - a < chunk ? mn - a : chunk;
            if ((long)fread(buf, 49, n, fl) != n) { free(buf); fclose(fl); return failf(err, "%s: truncated markers", path); }
            for (long q = 0; q < n; q++) {
                for (int f = 0; f < 12; f++) memcpy(&p->mark[f][a + q], buf + 49 * q + 4 * f, 4);
                p->markt[a + q] = (int8_t)buf[49 * q + 48];
            }
        }
        free(buf);
    }
    fclose(fl);
    bind_model(p);
    return 0;
}

int prn_alloc_like(const prn_file *src, prn_file *p, char *err)
{
    memset(p, 0, sizeof *p);
    p->m = src->m;
    p->cycle = src->cycle;
    p->gridcur = src->gridcur;
    p->gridtot = src->gridtot;
    const i3g_model *m = &src->m;
    const long rn = m->rocknum, nn = (long)(m->xnumx * m->ynumy * m->znumz), bn = (long)m->bondnum, mn = (long)m->marknum;
    for (int t = 0; t < 24; t++) {
        p->rock[t] = (double *)xcalloc(rn, 8);
        memcpy(p->rock[t], src->rock[t], 8 * rn);
    }
    p->gxf = (float *)xcalloc(m->xnumx, 4); p->gyf = (float *)xcalloc(m->ynumy, 4); p->gzf = (float *)xcalloc(m->znumz, 4);
    memcpy(p->gxf, src->gxf, 4 * m->xnumx); memcpy(p->gyf, src->gyf, 4 * m->ynumy); memcpy(p->gzf, src->gzf, 4 * m->znumz);
    p->brow = (int64_t *)xcalloc(bn, 8); p->bond_id = (int64_t *)xcalloc(bn, 8); p->bp1 = (int64_t *)xcalloc(bn, 8);
    p->bc = (float *)xcalloc(bn, 4); p->bk = (float *)xcalloc(bn, 4);
    memcpy(p->brow, src->brow, 8 * bn); memcpy(p->bp1, src->bp1, 8 * bn);
    memcpy(p->bc, src->bc, 4 * bn); memcpy(p->bk, src->bk, 4 * bn);
    if (src->bond_id) memcpy(p->bond_id, src->bond_id, 8 * bn);
    if (alloc_arrays(p, nn, mn)) { prn_free(p); return failf(err, "out of host memory for a staging image"); }
    bind_model(p);
    return 0;
}

int prn_write(const char *path, const prn_file *p, char *err)
{
    FILE *fl = fopen(path, "wb");
    if (!fl) return failf(err, "cannot create %s", path);
    const i3g_model *m = &p->m;
    const unsigned char sz[4] = {4, 8, 4, 8};
    const double timesum_yr = m->timesum / I3G_YEAR;
    WR(sz, 1, 4);
    WR(&m->xnumx, 8, 1); WR(&m->ynumy, 8, 1); WR(&m->znumz, 8, 1);
    WR(&m->mnumx, 8, 1); WR(&m->mnumy, 8, 1); WR(&m->mnumz, 8, 1);
    WR(&m->xsize, 8, 1); WR(&m->ysize, 8, 1); WR(&m->zsize, 8, 1);
    WR(&m->pxinit, 8, 1); WR(&m->pyinit, 8, 1); WR(&m->pzinit, 8, 1);
    WR(&m->pinit, 8, 1); WR(&m->gxkoef, 8, 1); WR(&m->gykoef, 8, 1); WR(&m->gzkoef, 8, 1);
    WR(&m->rocknum, 4, 1); WR(&m->bondnum, 8, 1); WR(&m->marknum, 8, 1); WR(&p->cycle, 4, 1);
    WR(&timesum_yr, 8, 1); WR(&p->gridcur, 8, 1); WR(&p->gridtot, 8, 1);
    for (int t = 0; t < 24; t++) WR(m->rock[t], 8, m->rocknum);
    const long nn = (long)(m->xnumx * m->ynumy * m->znumz), bn = (long)m->bondnum, mn = (long)m->marknum;
    const float *nf[15] = {m->vx, m->vy, m->vz, m->ro, m->nu, m->nxx, m->nxy, m->nxz, m->nyz,
                           m->tk, m->cp, m->et, m->kt, m->ht, m->rr};
    {
        const long chunk = 1 << 16;
        float *buf = (float *)malloc(sizeof(float) * 16 * chunk);
        for (long a = 0; a < nn; a += chunk) {
            const long n = nn - a < chunk ? nn - a : chunk;
            for (long q = 0; q < n; q++) {
                buf[16 * q] = (float)m->pr[a + q];
                for (int f = 0; f < 15; f++) buf[16 * q + 1 + f] = nf[f][a + q];
            }
            if ((long)fwrite(buf, 64, n, fl) != n) { free(buf); fclose(fl); return failf(err, "%s: write failed", path); }
        }
        free(buf);
    }
    WR(m->gx, 4, m->xnumx); WR(m->gy, 4, m->ynumy); WR(m->gz, 4, m->znumz);
    for (long b = 0; b < bn; b++) {
        const int64_t id = p->bond_id ? p->bond_id[b] : b + 1;
        WR(&m->bond_row[b], 8, 1); WR(&id, 8, 1); WR(&m->bond_c[b], 4, 1); WR(&m->bond_k[b], 4, 1);
        WR(&m->bond_partner1[b], 8, 1);
    }
    const float *mf[12] = {m->markx, m->marky, m->markz, m->markk, m->markw, m->markd, m->markv,
                           m->marke, m->markex, m->markft, m->markrr, m->markrn};
    {
        const long chunk = 1 << 16;
        unsigned char *buf = (unsigned char *)malloc(49 * chunk);
        for (long a = 0; a < mn; a += chunk) {
            const long n = mn - a < chunk ? mn - a : chunk;
            for (long q = 0; q < n; q++) {
                for (int f = 0; f < 12; f++) memcpy(buf + 49 * q + 4 * f, &mf[f][a + q], 4);
                buf[49 * q + 48] = (unsigned char)m->markt[a + q];
            }
            if ((long)fwrite(buf, 49, n, fl) != n) { free(buf); fclose(fl); return failf(err, "%s: write failed", path); }
        }
        free(buf);
    }
    if (fclose(fl)) return failf(err, "%s: close failed", path);
    return 0;
}

void prn_free(prn_file *p)
{
    for (int t = 0; t < 24; t++) free(p->rock[t]);
    big_free(p, p->pr);
    for (int f = 0; f < 15; f++) big_free(p, p->node[f]);
    for (int f = 0; f < 12; f++) big_free(p, p->stress[f]);
    free(p->gxf); free(p->gyf); free(p->gzf);
    free(p->brow); free(p->bond_id); free(p->bp1); free(p->bc); free(p->bk);
    for (int f = 0; f < 12; f++) big_free(p, p->mark[f]);
    big_free(p, p->markt);
    memset(p, 0, sizeof *p);
}

/* ---- mode.t3c ---------------------------------------------------------------------- */
/* Whitespace-separated tokens; a token that starts with '/' is a comment (ffscanf,
 * load3mg.c:1102-1127).  Values are read with atoi/atof, which stop at the first character
 * that does not belong to the number ("1e-04-DIVVMIN" reads as 1e-4). */
typedef struct toks {
    FILE *fl;
    char t[512];
    int eof;
} toks;

static const char *next_tok(toks *s)
{
    for (;;) {
        if (fscanf(s->fl, "%511s", s->t) != 1) {
            s->eof = 1;
            s->t[0] = 0;
            return s->t;
        }
        if (s->t[0] != '/') return s->t;
    }
}

static double tf(toks *s) { return atof(next_tok(s)); }
static int ti(toks *s) { return atoi(next_tok(s)); }

int mode_read(const char *path, mode_t3c *md, char *err)
{
    memset(md, 0, sizeof *md);
    toks s;
    memset(&s, 0, sizeof s);
    s.fl = fopen(path, "rt");
    if (!s.fl) return failf(err, "cannot open %s", path);
    i3g_params *p = &md->p;
    /* input file name and type (load3mg.c:19-22) */
    snprintf(md->infile, sizeof md->infile, "%s", next_tok(&s));
    next_tok(&s);
    /* output file rows up to '~' (load3mg.c:24-58) */
    const char *t = next_tok(&s);
    while (!s.eof && t[0] != '~') {
        if (md->nfiles >= MODE_MAXFILES) { fclose(s.fl); return failf(err, "%s: more than %d output files", path, MODE_MAXFILES); }
        mode_file *f = &md->files[md->nfiles++];
        snprintf(f->name, sizeof f->name, "%s", t);
        next_tok(&s);
        f->fp.cyc0max = ti(&s);
        f->fp.maxxystep = tf(&s);
        f->fp.maxtkstep = tf(&s);
        f->fp.maxtmstep = tf(&s) * I3G_YEAR;
        f->fp.nubeg = tf(&s);
        f->fp.nuend = tf(&s);
        f->fp.p0koef = tf(&s); f->fp.p1koef = tf(&s); f->fp.p2koef = tf(&s);
        f->fp.p0koef2 = tf(&s); f->fp.p1koef2 = tf(&s); f->fp.p2koef2 = tf(&s);
        f->fp.multinum = ti(&s); f->fp.multstp = ti(&s); f->fp.multinum2 = ti(&s);
        t = next_tok(&s);
    }
    /* general block (load3mg.c:61-76) */
    p->printmod = ti(&s); p->movemod = ti(&s); p->tempmod = ti(&s); p->markmod = ti(&s);
    p->gridmod = ti(&s); p->outgrid = ti(&s); p->densimod = ti(&s);
    p->stp100 = tf(&s);
    md->filesjob = ti(&s);
    p->eroslev = tf(&s); p->sedilev = tf(&s); p->waterlev = tf(&s);
    md->cyc1max = ti(&s);
    /* V_P block (load3mg.c:79-100) */
    p->DIVVMIN = tf(&s); p->STOKSMIN = tf(&s); p->DIVVMAX = tf(&s); p->STOKSMAX = tf(&s);
    p->multimax = ti(&s);
    p->multicyc = ti(&s);
    if (p->multimax < 0 || p->multimax >= I3G_MAXLEV) { fclose(s.fl); return failf(err, "%s: multinum %d outside 0..%d", path, p->multimax, I3G_MAXLEV - 1); }
    for (int l = 0; l <= p->multimax; l++) p->multinnn[0][l] = ti(&s);
    for (int l = 0; l <= p->multimax; l++) p->multinnn[1][l] = ti(&s);
    p->p0koef = tf(&s); p->p1koef = tf(&s); p->p2koef = tf(&s); p->v0koef = tf(&s); p->v1koef = tf(&s);
    p->nubeg = tf(&s); p->nuend = tf(&s); p->nukoef = tf(&s);
    p->viscmod = ti(&s);
    ti(&s);                                   /* spheryn */
    ti(&s);                                   /* cyc2max */
    /* T block (load3mg.c:103-116) */
    p->HEATMIN = tf(&s);
    const int multinumt = ti(&s);
    p->multicyct = ti(&s);
    if (multinumt < 0 || multinumt >= 100) { fclose(s.fl); return failf(err, "%s: multinumt %d out of range", path, multinumt); }
    for (int l = 0; l <= multinumt; l++) { const int v = ti(&s); if (l == 0) p->multittt0 = v; }
    for (int l = 0; l <= multinumt; l++) ti(&s);
    p->t0koef = tf(&s);
    tf(&s);                                   /* t1koef */
    p->heatdif = tf(&s);
    p->frictyn = (int32_t)tf(&s);
    p->adiabyn = (int32_t)tf(&s);
    /* water / melt block, 29 values (load3mg.c:119-147); the time step uses a few */
    double w[29];
    for (int i = 0; i < 29; i++) w[i] = tf(&s);
    p->tdeep = w[5]; p->zdeep = w[8]; p->vdeep = w[9]; p->nudeep = w[10];
    p->healrate = w[23]; p->teclmin = w[27]; p->teclmax = w[28];
    tf(&s); tf(&s);                           /* xvolc, xtkplut (load3mg.c:149-156) */
    p->timebeg = tf(&s) * I3G_YEAR;
    p->timeend = tf(&s) * I3G_YEAR;
    tf(&s);                                   /* tempbeg */
    tf(&s);                                   /* convend */
    p->tempend = 0.0;
    const int bad = s.eof;
    fclose(s.fl);
    if (bad) return failf(err, "%s: ended before all parameters were read", path);
    return 0;
}

int file_t3c_read(const char *path)
{
    FILE *fl = fopen(path, "rt");
    if (!fl) return -1;
    char t[64] = {0};
    int ok = fscanf(fl, "%63s", t) == 1;
    fclose(fl);
    return ok ? atoi(t) : -1;
}

int file_t3c_write(const char *path, int index)
{
    FILE *fl = fopen(path, "wt");
    if (!fl) return -1;
    fprintf(fl, "%d \n", index);
    return fclose(fl) ? -1 : 0;
}
