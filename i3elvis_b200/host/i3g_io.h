/*
 * i3g_io.h -- the reference's run files for the C host loop: binary .prn restart files
 * (loader / saver, load3mg.c:704-1063), mode.t3c (loadconf, load3mg.c:2-170) and
 * file.t3c (load3mg.c:9-11, 1065-1068).
 */
#ifndef I3G_IO_H
#define I3G_IO_H

#include <stdint.h>
#include "../../include/i3g.h"

#define I3G_YEAR 3.15576e7     /* seconds per year (load3mg.c:44) */

/* .prn image: the i3g_model points into the arrays owned here. */
typedef struct prn_file {
    i3g_model m;
    int32_t cycle;                      /* header: time-step counter of the file        */
    double gridcur, gridtot;            /* header: grid-refinement bookkeeping (kept)   */
    int64_t *bond_id;                   /* second field of each boundary record (kept)  */
    /* storage */
    float *gxf, *gyf, *gzf;
    double *pr;
    float *node[15];                    /* vx vy vz ro nu nxx nxy nxz nyz tk cp et kt ht rr */
    float *stress[12];                  /* exx eyy ezz exy exz eyz sxx syy szz sxy sxz syz  */
    int64_t *brow, *bp1;
    float *bc, *bk;
    float *mark[12];                    /* x y z k w d v e ex ft rr rn                      */
    int8_t *markt;
    double *rock[24];
    void (*release)(void *);            /* frees the nodal and marker arrays (set by prn_read) */
} prn_file;

/* Allocator of the large arrays (nodes, stresses, markers) of the images that prn_read and
 * prn_alloc_like make from now on; NULL restores calloc/free.  The host loop passes
 * i3g_host_alloc / i3g_host_free so that uploads and downloads run at full bus speed from
 * page-locked memory.  The allocator must return zeroed memory or NULL. */
void prn_set_allocator(void *(*alloc)(int64_t bytes), void (*release)(void *));

/* 0 on success; on failure -1 with a message in err[256]. */
int prn_read(const char *path, prn_file *p, char *err);
int prn_write(const char *path, const prn_file *p, char *err);
/* An image with the header, grid, rocks and boundary records of src and its own (zeroed)
 * nodal, stress and marker arrays: the staging image of an asynchronous save. */
int prn_alloc_like(const prn_file *src, prn_file *p, char *err);
void prn_free(prn_file *p);

#define MODE_MAXFILES 1000

typedef struct mode_file {
    char name[256];
    i3g_file_params fp;
} mode_file;

typedef struct mode_t3c {
    char infile[256];
    int nfiles;
    mode_file files[MODE_MAXFILES];
    int32_t filesjob, cyc1max;
    i3g_params p;                       /* solver controls left at 0: the caller sets them */
} mode_t3c;

int mode_read(const char *path, mode_t3c *m, char *err);
/* 1-based index of the next output file stored in file.t3c; -1 when unreadable. */
int file_t3c_read(const char *path);
int file_t3c_write(const char *path, int index);

#endif
