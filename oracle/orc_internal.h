/*
 * orc_internal.h -- TEST INFRASTRUCTURE.  Shared declarations of the CPU oracle: a plain C
 * restatement of the reference's per-time-step algorithms, used only by tests/, by the
 * smoke check and by the benchmark's CPU-baseline leg as the thing results are checked
 * against.  Nothing in the product links it.
 */
#ifndef ORC_INTERNAL_H
#define ORC_INTERNAL_H
#include <stdint.h>
#include "../include/i3g.h"

#define ORC_MAXLEV I3G_MAXLEV

typedef struct orc_ctx {
    /* model copy (reference layout) */
    i3g_model m;
    i3g_params p;
    i3g_file_params f;
    long nx, ny, nz, nodenum;
    double *gx, *gy, *gz;             /* grid lines promoted to double (load3mg.c:814-825) */
    double *pr;                       /* level 0 pressure (double)                         */
    float *vx, *vy, *vz;              /* level 0 velocities                                */
    float *ro, *nu, *nxx, *nxy, *nxz, *nyz, *tk, *cp, *et, *kt, *ht, *rr;
    float *exx, *eyy, *ezz, *exy, *exz, *eyz, *sxx, *syy, *szz, *sxy, *sxz, *syz;
    double *tk0, *tk1, *tk2;          /* heat solve scratch (head3mg.c:78 keeps them float) */
    /* markers */
    long marknum;
    float *mx, *my, *mz, *mk, *mw, *md, *mv, *me, *mex, *mft, *mrr, *mrn;
    int8_t *mt;
    double *rock[24];
    int rocknum;
    /* multigrid geometry (gridcheck, load3mg.c:1200-1282) */
    int nlev;                          /* multimax + 1 */
    long mgx[ORC_MAXLEV], mgy[ORC_MAXLEV], mgz[ORC_MAXLEV], mgxy[ORC_MAXLEV], mgn[ORC_MAXLEV], mgp[ORC_MAXLEV];
    double *mggx[ORC_MAXLEV], *mggy[ORC_MAXLEV], *mggz[ORC_MAXLEV];
    long ntot;                         /* nodes over all levels */
    /* boundary rows: bcid[row] = index into bc_* or -1; rows: 4*node+var (Stokes),
     * bcid_t[node] for temperature */
    int32_t *bcid, *bcid_t;
    long nbc;
    double *bc_c, *bc_k;
    long *bc_p;                        /* partner row or -1 */
    /* level arrays */
    float *nul;                        /* nu over all levels (level 0 = nu)                */
    float *nd;                         /* continuity viscosity, all levels (float like nd[]) */
    double *sol, *fre1, *fre0, *wsum;  /* 4*ntot                                          */
    /* assembled rows (CSR over all 4*ntot rows) */
    long *rowptr;
    long *col;
    double *val;
    /* heat rows (level 0) */
    long *trowptr, *tcol;
    double *tval, *tfre1, *tsol;
    /* statistics */
    i3g_stats st;
    char err[512];
} orc_ctx;

/* stokes.c */
int orc_stokes_build(orc_ctx *o);
void orc_vcycle(orc_ctx *o, int multinum);
void orc_smooth_ref(orc_ctx *o, int level, int nsweeps);
void orc_smooth_mc(orc_ctx *o, int level, int nsweeps);
void orc_residual(orc_ctx *o, int level);
void orc_restrict(orc_ctx *o, int level);
void orc_prolong(orc_ctx *o, int level);
void orc_relres(orc_ctx *o, double *mom, double *cont);
void orc_eta(orc_ctx *o, int level, double *out4);
long orc_node(const orc_ctx *o, int l, long m1, long m2, long m3);

/* markers.c */
long orc_m1serch(const orc_ctx *o, double x);
long orc_m2serch(const orc_ctx *o, double y);
long orc_m3serch(const orc_ctx *o, double z);
void orc_vxyz(const orc_ctx *o, double x, double y, double z, double *v, long *wn);
int orc_move_markers(orc_ctx *o, double timestep);
int orc_markers_to_nodes(orc_ctx *o, double timestep);
void orc_tkrecalc(orc_ctx *o);

/* heat.c */
int orc_heat(orc_ctx *o, double *timestep);

#endif
