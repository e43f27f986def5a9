/*
 * ref_harness.c -- TEST INFRASTRUCTURE.  Drives the reference's own functions so that the
 * CPU oracle (i3g_oracle.c) and the CUDA library can be checked against the reference
 * itself.  It is compiled by build_ref.sh together with the reference sources where they
 * lie; only the array-size macros of head3mg.c are shrunk (the shipped sizes need 78 GB of
 * static storage).  Nothing in the product links this file.
 *
 * Commands (run in a directory holding mode.t3c, file.t3c and the input .prn, stdin closed
 * because the reference's interpolation checks call getchar()):
 *
 *   prepare OUT.prn            ronurecalc, hydrostatic pressure, ronurecalc (in3mg.c:990-1031)
 *   assemble PREFIX            vpiterate set-up (move3mg.c:1948-2159): writes PREFIX.csr
 *   vcycles N PREFIX           set-up + N V-cycles (move3mg.c:2170-2223): PREFIX.sol
 *   solve RTOL MAXC PREFIX     set-up + V-cycles until the relative residual <= RTOL
 *   heat DT RTOL MAXC PREFIX   titerate set-up (heat3mg.c:310-453) + gausmatt to RTOL
 *   stokes PREFIX              vpiterate(0,0) as is; writes PREFIX.fields (v, P, stresses)
 *   move DT PREFIX             loads PREFIX.fields, movemark(); writes PREFIX.marks
 *   r2n PREFIX                 ronurecalc() on the loaded markers; writes PREFIX.nodes
 *   mover2n DT PREFIX          loads PREFIX.fields, movemark(), ronurecalc(); marks + nodes
 *   titerate DT PREFIX [CAP]   loads PREFIX.fields, titerate(0) (at most CAP iteration blocks); marks + nodes
 *   steps RTOL MAXC REPS PREP HEATCAP [DT]   whole timed steps, V-cycles to RTOL (see below)
 *   step OUT.prn               one full i3mg time step (i3mg.c:80-147), wall time per phase
 */
#include <stdio.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <omp.h>
#include <time.h>

/* cap on titerate's outer iteration blocks (see build_ref.sh); unlimited by default */
static long i3g_heat_blocks = 0, i3g_heat_block_cap = 0x7fffffffffffffffL;
#include "head3mg.c"
#include "load3mg.c"
#include "move3mg.c"
#include "mark3mg.c"
#include "gaus3mg.c"
#include "heat3mg.c"

static void file_params(int f0)
{
    /* i3mg.c:64-77 */
    cyc0max = fl0cyc[f0][0];
    maxxystep = fl0stp[f0][0];
    maxtkstep = fl0stp[f0][1];
    maxtmstep = fl0stp[f0][2];
    nubeg = fl0stp[f0][3];
    nuend = fl0stp[f0][4];
    p0koef = fl0stp[f0][5];
    p1koef = fl0stp[f0][6];
    p2koef = fl0stp[f0][7];
    multinum = fl0cyc[f0][1];
}

static void wr(FILE *f, const void *p, size_t sz, size_t n)
{
    if (fwrite(p, sz, n, f) != n) { fprintf(stderr, "write failed\n"); exit(3); }
}

static FILE *openw(const char *prefix, const char *ext)
{
    char nm[512];
    snprintf(nm, sizeof nm, "%s.%s", prefix, ext);
    FILE *f = fopen(nm, "wb");
    if (!f) { fprintf(stderr, "cannot open %s\n", nm); exit(3); }
    return f;
}

/* Set-up part of vpiterate (move3mg.c:1948-2159), using the reference's row builders. */
static void stokes_assemble(void)
{
    long m1, m2, m3, mcmax, mcmax1, pos0cur1;
    long un1[MAXPOS];
    double ui1[MAXPOS], eps1[100];
    int mgi;
    for (mgi = 1; mgi <= multimax; mgi++) ronurestrict(mgi);
    for (m1 = 0; m1 < (mgp[multimax] + mgn[multimax]) * 4; m1++) { sol0[m1] = 0; num0[m1] = 0; }
    mgi = 0;
    for (m3 = 0; m3 < mgz[0]; m3++)
        for (m1 = 0; m1 < mgx[0]; m1++)
            for (m2 = 0; m2 < mgy[0]; m2++) {
                mcmax1 = m3 * mgxy[0] + m1 * mgy[0] + m2;
                if (m1 && m2 && m3) sol0[mcmax1 * 4 + 0] = pr[mcmax1];
                if (m2 < mgy[0] - 1 && m3 < mgz[0] - 1) sol0[mcmax1 * 4 + 1] = vx[mcmax1];
                if (m1 < mgx[0] - 1 && m3 < mgz[0] - 1) sol0[mcmax1 * 4 + 2] = vy[mcmax1];
                if (m1 < mgx[0] - 1 && m2 < mgy[0] - 1) sol0[mcmax1 * 4 + 3] = vz[mcmax1];
            }
    for (mgi = 0; mgi <= multimax; mgi++)
        for (m3 = 0; m3 < mgz[mgi]; m3++)
            for (m1 = 0; m1 < mgx[mgi]; m1++)
                for (m2 = 0; m2 < mgy[mgi]; m2++) {
                    mcmax1 = mgp[mgi] + m3 * mgxy[mgi] + m1 * mgy[mgi] + m2;
                    mcmax = mcmax1 * 4;
                    pos0cur1 = mcmax1 * 57;
                    if (m1 && m2 && m3) {
                        if (!bondm[mcmax + 0]) continerr(m1, m2, m3, 0, mgi, eps1, un1, ui1);
                        else bonderr(mcmax + 0, 0, eps1, un1, ui1);
                        gausmat2(1, mcmax + 0, pos0cur1, un1, ui1);
                    }
                    if (m2 < mgy[mgi] - 1 && m3 < mgz[mgi] - 1) {
                        if (!bondm[mcmax + 1]) xstokserr(m1, m2, m3, 0, mgi, eps1, un1, ui1);
                        else bonderr(mcmax + 1, 0, eps1, un1, ui1);
                        gausmat2(1, mcmax + 1, pos0cur1 + 6, un1, ui1);
                    }
                    if (m1 < mgx[mgi] - 1 && m3 < mgz[mgi] - 1) {
                        if (!bondm[mcmax + 2]) ystokserr(m1, m2, m3, 0, mgi, eps1, un1, ui1);
                        else bonderr(mcmax + 2, 0, eps1, un1, ui1);
                        gausmat2(1, mcmax + 2, pos0cur1 + 23, un1, ui1);
                    }
                    if (m1 < mgx[mgi] - 1 && m2 < mgy[mgi] - 1) {
                        if (!bondm[mcmax + 3]) zstokserr(m1, m2, m3, 0, mgi, eps1, un1, ui1);
                        else bonderr(mcmax + 3, 0, eps1, un1, ui1);
                        gausmat2(1, mcmax + 3, pos0cur1 + 40, un1, ui1);
                    }
                }
}

/* One V-cycle with the schedule of move3mg.c:2173-2213. */
static void vcycle(void)
{
    int n2, mgi;
    for (n2 = 0; n2 < multinum; n2++) {
        mgi = n2;
        if (multinnn[0][mgi] > 0) gausmat4(multinnn[0][mgi], (mgp[mgi] + mgn[mgi]) * 4 - 1, mgp[mgi] * 4, mgi);
        vprestrict(mgi + 1);
    }
    for (n2 = multinum; n2 > 0; n2--) {
        mgi = n2;
        if (multinnn[1][mgi] > 0) gausmat4(multinnn[1][mgi], (mgp[mgi] + mgn[mgi]) * 4 - 1, mgp[mgi] * 4, mgi);
        vpprolong(mgi, 0);
    }
    if (multinnn[1][0] > 0) gausmat4(multinnn[1][0], mgn[0] * 4 - 1, 0, 0);
}

/* Relative residuals of the level-0 system (the stopping rule shared with the oracle and
 * the CUDA library): momentum ||b-Ax||/||b|| over non-boundary velocity rows; continuity
 * RMS(div v) * mean spacing / RMS(v) over non-boundary pressure rows. */
static void relres(double *mom, double *cont)
{
    long m, e;
    double rb = 0, bb = 0, rc = 0, vv = 0, nc = 0, nv = 0, h;
#pragma omp parallel for private(e) reduction(+ : rb, bb, rc, vv, nc, nv) schedule(static)
    for (m = 0; m < mgn[0] * 4; m++) {
        if (!num0[m]) continue;
        if (m % 4) { vv += sol0[m] * sol0[m]; nv += 1; }
        if (bondm[m]) continue;
        double r = fre1[m];
        for (e = 0; e < num0[m]; e++) r -= val1[pos0[m] + e] * sol0[lin0[pos0[m] + e]];
        if (m % 4) { rb += r * r; bb += fre1[m] * fre1[m]; }
        else { rc += r * r; nc += 1; }
    }
    h = (xsize / (xnumx - 1) + ysize / (ynumy - 1) + zsize / (znumz - 1)) / 3.0;
    *mom = bb > 0 ? sqrt(rb / bb) : sqrt(rb);
    if (nc > 0 && vv > 0) *cont = sqrt(rc / nc) * h / sqrt(vv / nv);
    else *cont = sqrt(rc);
}

static void dump_csr(const char *prefix, long nrows)
{
    FILE *f = openw(prefix, "csr");
    long m, e, nnz = 0;
    for (m = 0; m < nrows; m++) nnz += num0[m];
    wr(f, &nrows, 8, 1);
    wr(f, &nnz, 8, 1);
    for (m = 0; m < nrows; m++) { long n = num0[m]; wr(f, &n, 8, 1); }
    for (m = 0; m < nrows; m++)
        for (e = 0; e < num0[m]; e++) { long c = lin0[pos0[m] + e]; wr(f, &c, 8, 1); }
    for (m = 0; m < nrows; m++)
        for (e = 0; e < num0[m]; e++) wr(f, &val1[pos0[m] + e], 8, 1);
    wr(f, fre1, 8, nrows);
    long nn = nrows / 4;
    wr(f, nd, 4, nn);
    wr(f, nu, 4, nn);
    fclose(f);
}

static void dump_sol(const char *prefix, long n, double *hist, int nh)
{
    FILE *f = openw(prefix, "sol");
    long nn = n;
    wr(f, &nn, 8, 1);
    wr(f, sol0, 8, n);
    long h = nh;
    wr(f, &h, 8, 1);
    if (nh) wr(f, hist, 8, nh);
    fclose(f);
}

static void dump_fields(const char *prefix)
{
    FILE *f = openw(prefix, "fields");
    long n = nodenum;
    wr(f, &n, 8, 1);
    wr(f, pr, 8, n);
    float *a[15] = {vx, vy, vz, exx, eyy, ezz, exy, exz, eyz, sxx, syy, szz, sxy, sxz, syz};
    for (int i = 0; i < 15; i++) wr(f, a[i], 4, n);
    wr(f, &timestep, 8, 1);
    fclose(f);
}

static void load_fields(const char *prefix)
{
    char nm[512];
    snprintf(nm, sizeof nm, "%s.fields", prefix);
    FILE *f = fopen(nm, "rb");
    long n;
    if (!f || fread(&n, 8, 1, f) != 1 || n != nodenum) { fprintf(stderr, "bad fields file\n"); exit(3); }
    if (fread(pr, 8, n, f) != (size_t)n) exit(3);
    float *a[15] = {vx, vy, vz, exx, eyy, ezz, exy, exz, eyz, sxx, syy, szz, sxy, sxz, syz};
    for (int i = 0; i < 15; i++) if (fread(a[i], 4, n, f) != (size_t)n) exit(3);
    fclose(f);
}

static void dump_marks(const char *prefix)
{
    FILE *f = openw(prefix, "marks");
    long n = marknum;
    wr(f, &n, 8, 1);
    float *a[12] = {markx, marky, markz, markk, markw, markd, markv, marke, markex, markft, markrr, markrn};
    for (int i = 0; i < 12; i++) wr(f, a[i], 4, n);
    wr(f, markt, 1, n);
    fclose(f);
}

static void dump_nodes(const char *prefix)
{
    FILE *f = openw(prefix, "nodes");
    long n = nodenum;
    wr(f, &n, 8, 1);
    float *a[15] = {ro, nu, nxx, nxy, nxz, nyz, tk, cp, et, kt, ht, rr, vx, vy, vz};
    for (int i = 0; i < 15; i++) wr(f, a[i], 4, n);
    fclose(f);
}

/* The initial-condition passes of in3mg.c:990-1031: nodes from markers, hydrostatic
 * pressure (in3mg.c:1010-1021), nodes from markers again. */
static void prepare_state(void)
{
    long m1, m3, m4, m2;
    double ts = timestep;
    timestep = 0;
    ronurecalc();
    if (GYKOEF > 0)
        for (m3 = 1; m3 < znumz; m3++)
            for (m1 = 1; m1 < xnumx; m1++) {
                m4 = xynumxy * m3 + m1 * ynumy + 1;
                pr[m4] = pinit;
                for (m2 = 2; m2 < ynumy; m2++) {
                    m4++;
                    pr[m4] = pr[m4 - 1] + (gy[m2] - gy[m2 - 2]) / 2.0 * GYKOEF *
                             (ro[m4 - 1] + ro[m4 - ynumy - 1] + ro[m4 - xynumxy - 1] + ro[m4 - xynumxy - ynumy - 1]) / 4.0;
                }
            }
    ronurecalc();
    gridcheck();
    timestep = ts;
}

/* Level-0 pressure and velocities from sol0 into pr, vx, vy, vz (move3mg.c:2246-2317) and the
 * marker time step limit maxxystep / max|v| (move3mg.c:2608-2632). */
static double sample_vmax = 0;

static void velocities_and_cfl(void)
{
    long m1, m2, m3, n;
    double vmax[3] = {0, 0, 0};
    /* pressure shifted to pinit in the pinning cell (move3mg.c:2248-2269) */
    const double ival = pinit - sol0[(pzinit * xynumxy + pxinit * ynumy + pyinit) * 4];
    for (m3 = 1; m3 < znumz; m3++)
        for (m1 = 1; m1 < xnumx; m1++)
            for (m2 = 1; m2 < ynumy; m2++) {
                n = m3 * xynumxy + m1 * ynumy + m2;
                pr[n] = sol0[4 * n] + ival;
            }
    for (m3 = 0; m3 < znumz; m3++)
        for (m1 = 0; m1 < xnumx; m1++)
            for (m2 = 0; m2 < ynumy; m2++) {
                n = m3 * xynumxy + m1 * ynumy + m2;
                if (m2 < ynumy - 1 && m3 < znumz - 1) { vx[n] = (float)sol0[4 * n + 1]; if (fabs(vx[n]) > vmax[0]) vmax[0] = fabs(vx[n]); }
                if (m1 < xnumx - 1 && m3 < znumz - 1) { vy[n] = (float)sol0[4 * n + 2]; if (fabs(vy[n]) > vmax[1]) vmax[1] = fabs(vy[n]); }
                if (m1 < xnumx - 1 && m2 < ynumy - 1) { vz[n] = (float)sol0[4 * n + 3]; if (fabs(vz[n]) > vmax[2]) vmax[2] = fabs(vz[n]); }
            }
    for (int k = 0; k < 3; k++)
        if (vmax[k] > 0 && timestep > maxxystep / vmax[k]) timestep = maxxystep / vmax[k];
    sample_vmax = fmax(vmax[0], fmax(vmax[1], vmax[2]));
}

int main(int argc, char **argv)
{
    if (argc < 2) { fprintf(stderr, "usage: ref_harness CMD ...\n"); return 2; }
    const char *cmd = argv[1];
    double tl = omp_get_wtime();
    loadconf();
    loader();
    file_params(0);
    timestep = maxtmstep;
    fprintf(stderr, "loaded in %.1f s\n", omp_get_wtime() - tl);
    if (!strcmp(cmd, "prepare") && argc == 3) {
        prepare_state();
        snprintf(fl1out, sizeof fl1out, "%s", argv[2]);
        saver(0, 0);
        return 0;
    }
    if (!strcmp(cmd, "assemble") && argc == 3) {
        stokes_assemble();
        dump_csr(argv[2], (mgp[multimax] + mgn[multimax]) * 4);
        return 0;
    }
    if (!strcmp(cmd, "vcycles") && argc == 4) {
        int n = atoi(argv[2]);
        stokes_assemble();
        double hist[2 * 4096];
        int nh = 0;
        for (int i = 0; i < n; i++) {
            vcycle();
            if (nh < 4096) { relres(&hist[2 * nh], &hist[2 * nh + 1]); nh++; }
        }
        dump_sol(argv[3], (mgp[multimax] + mgn[multimax]) * 4, hist, 2 * nh);
        return 0;
    }
    if (!strcmp(cmd, "solve") && argc == 5) {
        double rtol = atof(argv[2]);
        int maxc = atoi(argv[3]);
        stokes_assemble();
        double *hist = malloc(sizeof(double) * 2 * (maxc + 1));
        int nh = 0;
        double mom, cont;
        relres(&mom, &cont);
        hist[0] = mom; hist[1] = cont; nh = 1;
        double t0 = omp_get_wtime();
        for (int i = 0; i < maxc; i++) {
            vcycle();
            relres(&mom, &cont);
            hist[2 * nh] = mom; hist[2 * nh + 1] = cont; nh++;
            if (mom <= rtol && cont <= rtol) break;
        }
        double t1 = omp_get_wtime();
        printf("{\"cycles\": %d, \"mom\": %.6e, \"cont\": %.6e, \"seconds\": %.4f, \"threads\": %d}\n",
               nh - 1, mom, cont, t1 - t0, omp_get_max_threads());
        dump_sol(argv[4], mgn[0] * 4, hist, 2 * nh);
        return 0;
    }
    if (!strcmp(cmd, "heat") && argc == 6) {
        long m1, m2, m3, mcmax, mcmax1, pos0cur1, e;
        long un1[MAXPOS];
        double ui1[MAXPOS], eps1[100];
        timestep = atof(argv[2]);
        double rtol = atof(argv[3]);
        int maxc = atoi(argv[4]);
        /* heat3mg.c:310-335: old T and right-hand-side pass (heaterr mode 0 fills tk1) */
        for (m1 = 0; m1 < nodenum; m1++) tk0[m1] = tk[m1];
        for (m3 = 0; m3 < mgz[0]; m3++)
            for (m1 = 0; m1 < mgx[0]; m1++)
                for (m2 = 0; m2 < mgy[0]; m2++) {
                    mcmax = m3 * mgxy[0] + m1 * mgy[0] + m2;
                    if (bondm[mcmax + nodenum8] == 0) heaterr(m1, m2, m3, 0, 0, eps1, un1, ui1);
                }
        for (m1 = 0; m1 < nodenum; m1++) { tk2[m1] = tk[m1]; tk0[m1] = tk[m1]; sol0[m1] = tk[m1]; }
        /* heat3mg.c:407-453, level 0 */
        for (m3 = 0; m3 < mgz[0]; m3++)
            for (m1 = 0; m1 < mgx[0]; m1++)
                for (m2 = 0; m2 < mgy[0]; m2++) {
                    mcmax = m3 * mgxy[0] + m1 * mgy[0] + m2;
                    mcmax1 = mcmax + nodenum8;
                    pos0cur1 = mcmax * 7;
                    if (bondm[mcmax1] == 0) heaterr(m1, m2, m3, 1, 0, eps1, un1, ui1);
                    else tbonderr(mcmax, 0, eps1, un1, ui1);
                    gausmat2(1, mcmax, pos0cur1, un1, ui1);
                }
        double rel = 1, hist[8192];
        int nh = 0;
        for (int it = 0; it < maxc; it++) {
            gausmatt(multittt[0][0], nodenum - 1, 0);
            double rr = 0, bb = 0;
            for (m1 = 0; m1 < nodenum; m1++) {
                if (bondm[m1 + nodenum8]) continue;
                double r = fre1[m1];
                for (e = 0; e < num0[m1]; e++) r -= val1[pos0[m1] + e] * sol0[lin0[pos0[m1] + e]];
                rr += r * r; bb += fre1[m1] * fre1[m1];
            }
            rel = sqrt(rr / bb);
            if (nh < 8192) hist[nh++] = rel;
            if (rel <= rtol) break;
        }
        printf("{\"cycles\": %d, \"rel\": %.6e}\n", nh, rel);
        dump_csr(argv[5], nodenum);
        dump_sol(argv[5], nodenum, hist, nh);
        return 0;
    }
    if (!strcmp(cmd, "stokes") && argc == 3) {
        vpiterate(0, 0);
        dump_fields(argv[2]);
        return 0;
    }
    if (!strcmp(cmd, "move") && argc == 4) {
        load_fields(argv[3]);
        timestep = atof(argv[2]);
        movemark();
        dump_marks(argv[3]);
        return 0;
    }
    if (!strcmp(cmd, "mover2n") && argc == 4) {
        load_fields(argv[3]);
        timestep = atof(argv[2]);
        movemark();
        dump_marks(argv[3]);
        ronurecalc();
        dump_nodes(argv[3]);
        return 0;
    }
    if (!strcmp(cmd, "titerate") && (argc == 4 || argc == 5)) {
        load_fields(argv[3]);
        timestep = atof(argv[2]);
        if (argc == 5 && atol(argv[4]) > 0) i3g_heat_block_cap = atol(argv[4]);
        i3g_heat_blocks = 0;
        double t0 = omp_get_wtime();
        titerate(0);
        printf("{\"heat_blocks\": %ld, \"seconds\": %.4f, \"timestep\": %.9e}\n", i3g_heat_blocks + 1,
               omp_get_wtime() - t0, timestep);
        dump_marks(argv[3]);
        dump_nodes(argv[3]);
        return 0;
    }
    if (!strcmp(cmd, "r2n") && argc == 3) {
        ronurecalc();
        dump_nodes(argv[2]);
        return 0;
    }
    if (!strcmp(cmd, "sample") && argc >= 3) {
        /* Bounded timing sample of time steps: SAMPLE NCYC [REPS [PREP [HEATCAP [DT]]]].  Optionally the
         * initial-condition passes first (PREP=1, timed apart); then REPS times: the reference's
         * vpiterate set-up (ronurestrict and row assembly, move3mg.c:1948-2159) and NCYC V-cycles,
         * the velocities and CFL time step from that iterate (or DT seconds when given), titerate (at most HEATCAP outer
         * iteration blocks), movemark and ronurecalc.  Wall clock, one JSON line per repetition. */
        int ncyc = atoi(argv[2]);
        int reps = argc >= 4 ? atoi(argv[3]) : 1;
        if (argc >= 6 && atol(argv[5]) > 0) i3g_heat_block_cap = atol(argv[5]);
        const double dt_fixed = argc >= 7 ? atof(argv[6]) : 0.0;
        double tp = 0;
        if (argc >= 5 && atoi(argv[4])) {
            double a = omp_get_wtime();
            prepare_state();
            tp = omp_get_wtime() - a;
        }
        fprintf(stderr, "sample: prepared in %.1f s\n", tp);
        for (int r = 0; r < reps; r++) {
            timestep = maxtmstep;
            double t0 = omp_get_wtime();
            stokes_assemble();
            double t1 = omp_get_wtime();
            fprintf(stderr, "sample %d: set-up %.1f s\n", r, t1 - t0);
            for (int i = 0; i < ncyc; i++) vcycle();
            double t2 = omp_get_wtime();
            fprintf(stderr, "sample %d: %d V-cycles %.1f s\n", r, ncyc, t2 - t1);
            velocities_and_cfl();
            if (dt_fixed > 0) timestep = dt_fixed;
            i3g_heat_blocks = 0;
            if (tempmod) titerate(0);
            double t3 = omp_get_wtime();
            fprintf(stderr, "sample %d: titerate %.1f s\n", r, t3 - t2);
            if (markmod) movemark();
            double t4 = omp_get_wtime();
            fprintf(stderr, "sample %d: movemark %.1f s\n", r, t4 - t3);
            if (gridmod) ronurecalc();
            double t5 = omp_get_wtime();
            printf("{\"rep\": %d, \"assemble_s\": %.4f, \"vcycle_s\": %.4f, \"ncyc\": %d, \"heat_s\": %.4f, "
                   "\"move_s\": %.4f, \"r2n_s\": %.4f, \"prepare_s\": %.4f, \"timestep\": %.6e, \"vmax\": %.3e, "
                   "\"heat_blocks\": %ld, \"threads\": %d}\n",
                   r, t1 - t0, (t2 - t1) / (ncyc > 0 ? ncyc : 1), ncyc, t3 - t2, t4 - t3, t5 - t4, tp, timestep,
                   sample_vmax, i3g_heat_blocks + 1, omp_get_max_threads());
            fflush(stdout);
        }
        return 0;
    }
    if (!strcmp(cmd, "steps") && argc >= 7) {
        /* Whole time steps of the reference on all OpenMP threads, timed by wall clock:
         * STEPS RTOL MAXC REPS PREP HEATCAP [DT].  Optionally the initial-condition passes first
         * (PREP=1, timed apart).  Then REPS times: vpiterate's set-up (ronurestrict and row
         * assembly, move3mg.c:1948-2159); V-cycles (move3mg.c:2170-2223), each followed by the
         * relative residual of the level-0 rows, until momentum and continuity are <= RTOL or
         * MAXC cycles; after the file row's multstp cycles (fl0cyc[0][2]) -- or as soon as the
         * residual is 30 times above the best one seen, the divergence the library also
         * reacts to -- the row's second relaxation set (move3mg.c:2585-2593); the velocities
         * and CFL time step (or DT seconds when given), titerate (at most HEATCAP iteration
         * blocks), movemark, ronurecalc.  One JSON line per repetition. */
        const double rtol = atof(argv[2]);
        const int maxc = atoi(argv[3]);
        const int reps = atoi(argv[4]);
        if (atol(argv[6]) > 0) i3g_heat_block_cap = atol(argv[6]);
        const double dt_fixed = argc >= 8 ? atof(argv[7]) : 0.0;
        double tp = 0;
        if (atoi(argv[5])) {
            double a = omp_get_wtime();
            prepare_state();
            tp = omp_get_wtime() - a;
        }
        fprintf(stderr, "steps: prepared in %.1f s\n", tp);
        for (int r = 0; r < reps; r++) {
            timestep = maxtmstep;
            p0koef = fl0stp[0][5];
            p1koef = fl0stp[0][6];
            multinum = fl0cyc[0][1];
            double t0 = omp_get_wtime();
            stokes_assemble();
            double t1 = omp_get_wtime();
            double mom = 0, cont = 0, best = 1e300, rel0;
            relres(&mom, &cont);
            rel0 = fmax(mom, cont);
            int ncyc = 0, switched = 0;
            while (ncyc < maxc && !(mom <= rtol && cont <= rtol)) {
                vcycle();
                ncyc++;
                relres(&mom, &cont);
                const double cur = fmax(mom, cont);
                if (!(cur == cur)) break;
                if (cur < best) best = cur;
                if (!switched && (ncyc >= fl0cyc[0][2] || cur > 30.0 * best)) {
                    multinum = fl0cyc[0][3];
                    p0koef = fl0stp[0][8];
                    p1koef = fl0stp[0][9];
                    switched = 1;
                    best = cur;
                }
            }
            double t2 = omp_get_wtime();
            fprintf(stderr, "steps %d: set-up %.1f s, %d V-cycles %.1f s, rel %.3e\n", r, t1 - t0, ncyc, t2 - t1, fmax(mom, cont));
            velocities_and_cfl();
            if (dt_fixed > 0) timestep = dt_fixed;
            i3g_heat_blocks = 0;
            if (tempmod) titerate(0);
            double t3 = omp_get_wtime();
            if (markmod) movemark();
            double t4 = omp_get_wtime();
            if (gridmod) ronurecalc();
            double t5 = omp_get_wtime();
            timesum += timestep;
            printf("{\"rep\": %d, \"step_s\": %.4f, \"assemble_s\": %.4f, \"stokes_s\": %.4f, \"ncyc\": %d, "
                   "\"rel0\": %.3e, \"rel\": %.3e, \"switched\": %d, \"heat_s\": %.4f, \"move_s\": %.4f, "
                   "\"r2n_s\": %.4f, \"prepare_s\": %.4f, \"timestep\": %.6e, \"vmax\": %.3e, \"heat_blocks\": %ld, "
                   "\"threads\": %d}\n",
                   r, t5 - t0, t1 - t0, t2 - t1, ncyc, rel0, fmax(mom, cont), switched, t3 - t2, t4 - t3, t5 - t4, tp,
                   timestep, sample_vmax, i3g_heat_blocks + 1, omp_get_max_threads());
            fflush(stdout);
        }
        return 0;
    }
    if (!strcmp(cmd, "step") && argc == 3) {
        double t[5];
        t[0] = omp_get_wtime();
        if (movemod) vpiterate(0, 0);
        t[1] = omp_get_wtime();
        if (tempmod && timestep) titerate(0);
        t[2] = omp_get_wtime();
        if (markmod && timestep) movemark();
        t[3] = omp_get_wtime();
        if (gridmod) ronurecalc();
        t[4] = omp_get_wtime();
        timesum += timestep;
        printf("{\"stokes_s\": %.4f, \"heat_s\": %.4f, \"move_s\": %.4f, \"r2n_s\": %.4f, "
               "\"total_s\": %.4f, \"timestep\": %.9e, \"threads\": %d}\n",
               t[1] - t[0], t[2] - t[1], t[3] - t[2], t[4] - t[3], t[4] - t[0], timestep,
               omp_get_max_threads());
        snprintf(fl1out, sizeof fl1out, "%s", argv[2]);
        saver(1, 0);
        return 0;
    }
    fprintf(stderr, "unknown command or arguments\n");
    return 2;
}
