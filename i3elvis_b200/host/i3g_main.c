/*
 * i3g_main.c -- the reference's host program (i3mg.c) over the B200 library.
 *
 * Run in a directory holding file.t3c, mode.t3c and the input .prn, like the reference:
 *
 *     i3g [-rtol R] [-heat-rtol R] [-maxcyc N] [-mixed] [-krylov M] [-warm W] [-exact] [-files N]
 *     i3g -roundtrip in.prn out.prn      (read and rewrite a .prn; no GPU used)
 *     i3g -dump-mode mode.t3c            (print the parsed parameters; no GPU used)
 *
 * Sequence (i3mg.c:24-160): loadconf + loader, the optional reset of v, P and stresses
 * with a marker->node pass when cyc1max < 0 (i3mg.c:40-52), then for each output file its
 * parameter row (i3mg.c:64-77) and cyc0max time steps of
 *     Stokes (vpiterate) -> heat (titerate) -> markers (movemark) -> nodes (ronurecalc)
 * (i3mg.c:80-147), then saver and file.t3c.  Solver controls that the reference does not
 * have (relative stopping tolerances, precision, FGMRES, the extrapolated Stokes start -warm 2|3,
 * the marker kernels in the reference's operation order -exact) come from the command line.
 *
 * Saving overlaps the computation: the model images live in page-locked memory, each output
 * file's state is downloaded into a staging image, and a writer thread writes the .prn file and
 * then file.t3c (so a restart never names an incomplete file) while the GPU already runs the
 * next file's steps.  The reference writes synchronously inside the loop (i3mg.c:150-160).
 */
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "i3g_io.h"

/* one asynchronous save: the staging image, its file name and the file.t3c index after it */
typedef struct saver_job {
    prn_file img;
    char name[256];
    int next_index;
    int busy, rc;
    char err[256];
    pthread_t th;
} saver_job;

static void *saver_run(void *arg)
{
    saver_job *j = (saver_job *)arg;
    j->rc = prn_write(j->name, &j->img, j->err);
    if (!j->rc && file_t3c_write("file.t3c", j->next_index)) {
        snprintf(j->err, sizeof j->err, "cannot write file.t3c");
        j->rc = -1;
    }
    return NULL;
}

/* wait for the save in flight; non-zero if it failed */
static int saver_wait(saver_job *j)
{
    if (!j->busy) return 0;
    pthread_join(j->th, NULL);
    j->busy = 0;
    if (j->rc) fprintf(stderr, "i3g: %s\n", j->err);
    return j->rc;
}

static int check(int rc, i3g_ctx *c, const char *what)
{
    if (rc) fprintf(stderr, "i3g: %s failed (%d): %s\n", what, rc, i3g_last_error(c));
    return rc;
}

/* Print the parsed mode.t3c as "name value" lines (for checking the parser). */
static int dump_mode(const char *path)
{
    char err[256];
    static mode_t3c md;
    if (mode_read(path, &md, err)) { fprintf(stderr, "i3g: %s\n", err); return 1; }
    const i3g_params *p = &md.p;
    printf("infile %s\nnfiles %d\nfilesjob %d\ncyc1max %d\n", md.infile, md.nfiles, md.filesjob, md.cyc1max);
    for (int f = 0; f < md.nfiles; f++) {
        const i3g_file_params *q = &md.files[f].fp;
        printf("file %s %d %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %d %d %d\n",
               md.files[f].name, q->cyc0max, q->maxxystep, q->maxtkstep, q->maxtmstep, q->nubeg, q->nuend,
               q->p0koef, q->p1koef, q->p2koef, q->p0koef2, q->p1koef2, q->p2koef2, q->multinum, q->multstp,
               q->multinum2);
    }
    printf("printmod %d\nmovemod %d\ntempmod %d\nmarkmod %d\ngridmod %d\noutgrid %d\ndensimod %d\n", p->printmod,
           p->movemod, p->tempmod, p->markmod, p->gridmod, p->outgrid, p->densimod);
    printf("stp100 %.17g\neroslev %.17g\nsedilev %.17g\nwaterlev %.17g\n", p->stp100, p->eroslev, p->sedilev, p->waterlev);
    printf("DIVVMIN %.17g\nSTOKSMIN %.17g\nDIVVMAX %.17g\nSTOKSMAX %.17g\n", p->DIVVMIN, p->STOKSMIN, p->DIVVMAX, p->STOKSMAX);
    printf("multinum %d\nmulticyc %d\nmultinnn", p->multimax, p->multicyc);
    for (int i = 0; i < 2; i++)
        for (int l = 0; l <= p->multimax; l++) printf(" %d", p->multinnn[i][l]);
    printf("\np0koef %.17g\np1koef %.17g\np2koef %.17g\nv0koef %.17g\nv1koef %.17g\n", p->p0koef, p->p1koef,
           p->p2koef, p->v0koef, p->v1koef);
    printf("nubeg %.17g\nnuend %.17g\nnukoef %.17g\nviscmod %d\nHEATMIN %.17g\nmulticyct %d\nmultittt0 %d\n",
           p->nubeg, p->nuend, p->nukoef, p->viscmod, p->HEATMIN, p->multicyct, p->multittt0);
    printf("t0koef %.17g\nheatdif %.17g\nfrictyn %d\nadiabyn %d\n", p->t0koef, p->heatdif, p->frictyn, p->adiabyn);
    printf("zdeep %.17g\nvdeep %.17g\ntdeep %.17g\nnudeep %.17g\nhealrate %.17g\nteclmin %.17g\nteclmax %.17g\n",
           p->zdeep, p->vdeep, p->tdeep, p->nudeep, p->healrate, p->teclmin, p->teclmax);
    printf("timebeg %.17g\ntimeend %.17g\n", p->timebeg, p->timeend);
    return 0;
}

static int roundtrip(const char *in, const char *out)
{
    char err[256];
    prn_file p;
    if (prn_read(in, &p, err) || prn_write(out, &p, err)) {
        fprintf(stderr, "i3g: %s\n", err);
        return 1;
    }
    prn_free(&p);
    return 0;
}

int main(int argc, char **argv)
{
    double rtol = 1e-8, heat_rtol = 1e-10;
    int maxcyc = 2000, precision = 0, max_files = -1, krylov = 0, warm = 1, exact = 0;
    for (int a = 1; a < argc; a++) {
        if (!strcmp(argv[a], "-roundtrip") && a + 2 < argc) return roundtrip(argv[a + 1], argv[a + 2]);
        else if (!strcmp(argv[a], "-dump-mode") && a + 1 < argc) return dump_mode(argv[a + 1]);
        else if (!strcmp(argv[a], "-rtol") && a + 1 < argc) rtol = atof(argv[++a]);
        else if (!strcmp(argv[a], "-heat-rtol") && a + 1 < argc) heat_rtol = atof(argv[++a]);
        else if (!strcmp(argv[a], "-maxcyc") && a + 1 < argc) maxcyc = atoi(argv[++a]);
        else if (!strcmp(argv[a], "-mixed")) precision = 1;
        else if (!strcmp(argv[a], "-krylov") && a + 1 < argc) krylov = atoi(argv[++a]);
        else if (!strcmp(argv[a], "-warm") && a + 1 < argc) warm = atoi(argv[++a]);
        else if (!strcmp(argv[a], "-exact")) exact = 1;
        else if (!strcmp(argv[a], "-files") && a + 1 < argc) max_files = atoi(argv[++a]);
        else {
            fprintf(stderr, "usage: i3g [-rtol R] [-heat-rtol R] [-maxcyc N] [-mixed] [-krylov M] [-warm W] [-exact] [-files N]\n"
                            "       i3g -roundtrip in.prn out.prn\n");
            return 2;
        }
    }
    char err[256];
    static mode_t3c md;
    if (mode_read("mode.t3c", &md, err)) { fprintf(stderr, "i3g: %s\n", err); return 1; }
    /* file.t3c names the next output file; its predecessor is the input (load3mg.c:9-11, 161-169) */
    int fln3 = file_t3c_read("file.t3c") - 1;
    const char *infile = md.infile;
    if (fln3 >= 0 && fln3 < md.nfiles) infile = md.files[fln3].name;
    else fln3 = -1;
    /* page-locked images when a GPU is there (calloc otherwise: the allocator returns NULL) */
    void *probe = i3g_host_alloc(1);
    if (probe) {
        i3g_host_free(probe);
        prn_set_allocator(i3g_host_alloc, i3g_host_free);
    }
    prn_file p;
    if (prn_read(infile, &p, err)) { fprintf(stderr, "i3g: %s\n", err); return 1; }
    static saver_job sv;
    if (prn_alloc_like(&p, &sv.img, err)) { fprintf(stderr, "i3g: %s\n", err); prn_free(&p); return 1; }
    md.p.stokes_rtol = rtol;
    md.p.stokes_maxcyc = maxcyc;
    md.p.heat_rtol = heat_rtol;
    md.p.heat_maxcyc = maxcyc;
    md.p.precision = precision;
    md.p.warm_start = warm;
    md.p.krylov = krylov;
    md.p.marker_exact = exact;
    i3g_ctx *c = NULL;
    if (check(i3g_create(&p.m, &md.p, &c), NULL, "i3g_create")) return 1;
    int rc = 0;
    if (md.cyc1max < 0) {
        /* reset v, P, strain rates and stresses, then nodes from markers (i3mg.c:40-52) */
        const long nn = (long)(p.m.xnumx * p.m.ynumy * p.m.znumz);
        memset(p.pr, 0, sizeof(double) * nn);
        for (int f = 0; f < 3; f++) memset(p.node[f], 0, sizeof(float) * nn);
        for (int f = 0; f < 12; f++) memset(p.stress[f], 0, sizeof(float) * nn);
        rc = check(i3g_upload(c, &p.m, I3G_SYNC_NODES | I3G_SYNC_STRESS), c, "i3g_upload");
        if (!rc) rc = check(i3g_markers_to_nodes(c, 0.0), c, "i3g_markers_to_nodes");
    }
    int last = fln3 + 1 + md.filesjob;
    if (last > md.nfiles) last = md.nfiles;
    if (max_files >= 0 && last > fln3 + 1 + max_files) last = fln3 + 1 + max_files;
    const i3g_params *P = &md.p;
    for (int f0 = fln3 + 1; f0 < last && !rc; f0++) {
        const mode_file *F = &md.files[f0];
        if ((rc = check(i3g_set_file_params(c, &F->fp), c, "i3g_set_file_params"))) break;
        int n0 = 0;
        for (n0 = 0; n0 < F->fp.cyc0max && !rc; n0++) {
            if (P->printmod) printf("\n! FILE %s  STEP %d\n", F->name, n0 + 1);
            double timestep = F->fp.maxtmstep;
            if (P->movemod && (rc = check(i3g_stokes(c, n0, &timestep), c, "i3g_stokes"))) break;
            if (P->tempmod && timestep != 0 && (rc = check(i3g_heat(c, n0, &timestep), c, "i3g_heat"))) break;
            if (P->markmod && timestep != 0 && (rc = check(i3g_move_markers(c, timestep), c, "i3g_move_markers"))) break;
            if (P->gridmod && (rc = check(i3g_markers_to_nodes(c, timestep), c, "i3g_markers_to_nodes"))) break;
            if ((rc = check(i3g_add_time(c, timestep), c, "i3g_add_time"))) break;
            if (P->printmod) {
                i3g_stats s;
                i3g_get_stats(c, &s);
                printf(" step %e years: Stokes %d V-cycles (rel %.3e) %.1f ms, heat %d cycles %.1f ms, "
                       "markers %.1f ms, nodes %.1f ms\n", timestep / I3G_YEAR, s.stokes_cycles, s.stokes_rel,
                       s.ms_stokes, s.heat_cycles, s.ms_heat, s.ms_move, s.ms_r2n);
            }
        }
        if (rc) break;
        /* ParaView output every 50th file (saver_paraview, i3mg.c:159) */
        if ((f0 + 1) % 50 == 0) {
            char vtr[300];
            snprintf(vtr, sizeof vtr, "%s.vtr", F->name);
            if ((rc = check(i3g_write_vtr(c, vtr), c, "i3g_write_vtr"))) break;
        }
        /* the previous file's writer must be done with the staging image */
        if ((rc = saver_wait(&sv))) break;
        if ((rc = check(i3g_download(c, &sv.img.m, I3G_SYNC_ALL), c, "i3g_download"))) break;
        sv.img.cycle = F->fp.cyc0max - 1;
        snprintf(sv.name, sizeof sv.name, "%s", F->name);
        sv.next_index = f0 + 1;
        if (pthread_create(&sv.th, NULL, saver_run, &sv)) {
            saver_run(&sv);   /* no thread: write in line */
            if ((rc = sv.rc)) { fprintf(stderr, "i3g: %s\n", sv.err); break; }
        } else {
            sv.busy = 1;
        }
        if (P->printmod) printf("\n saving %s\n", F->name);
    }
    if (saver_wait(&sv)) rc = 1;
    i3g_destroy(c);
    prn_free(&sv.img);
    prn_free(&p);
    return rc ? 1 : 0;
}
