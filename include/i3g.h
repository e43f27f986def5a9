/*
 * i3g.h -- C ABI of the B200 time-step library for I3ELVIS-style marker-in-cell models.
 *
 * The reference has no plugin interface: its time step is four internal calls made by the
 * host loop, which share state through static arrays (head3mg.c:33-288):
 *
 *     vpiterate(n0, f0)   i3mg.c:98    Stokes + continuity multigrid   (move3mg.c:1585-2636)
 *     titerate(n0)        i3mg.c:112   implicit heat solve + marker T  (heat3mg.c:287-788)
 *     movemark()          i3mg.c:125   RK4 marker advection + rheology (mark3mg.c:2-397)
 *     ronurecalc()        i3mg.c:137   marker -> node averaging        (mark3mg.c:404-1015)
 *
 * This header replaces those globals with one explicit model description (i3g_model, plain
 * pointers to host arrays in the .prn layout) and one opaque context that owns the device
 * copies.  Every entry point returns 0 on success or a negative I3G_E* code; the message of
 * the last failure is available from i3g_last_error().  The reference reports failures with
 * printf + exit(0) (gaus3mg.c:86-90, move3mg.c:2272); here nothing exits.
 *
 * All calls are made from one host thread and are ordered on the context's CUDA stream.
 * Host arrays are read by i3g_create()/i3g_upload() and written by i3g_download() only.
 */
#ifndef I3G_H
#define I3G_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define I3G_MAXLEV 12

/* ---- error codes ------------------------------------------------------------------ */
enum {
    I3G_OK = 0,
    I3G_E_ARG = -1,          /* invalid argument or size                                    */
    I3G_E_CUDA = -2,         /* CUDA runtime error (message has the CUDA error string)     */
    I3G_E_NOMEM = -3,        /* device allocation failed                                   */
    I3G_E_UNSUPPORTED = -4,  /* model feature outside the implemented physics              */
    I3G_E_NOCONV = -5,       /* iteration cap reached before the tolerance                 */
    I3G_E_NAN = -6,          /* NaN or Inf detected in a solution vector                   */
    I3G_E_PRESSURE = -7,     /* |P| > 1e12 Pa after a solve (reference exits: move3mg.c:2272) */
    I3G_E_BC = -8            /* boundary-condition table inconsistent (cycle, bad partner) */
};

/* ---- model: host image of one .prn file (load3mg.c:704-892) ----------------------- */
typedef struct i3g_model {
    /* grid (load3mg.c:739-751) */
    int64_t xnumx, ynumy, znumz;        /* nodes along x, y (vertical, y fastest), z     */
    int64_t mnumx, mnumy, mnumz;        /* markers per cell (used by the water level test)*/
    double xsize, ysize, zsize;         /* box size, m                                   */
    int64_t pxinit, pyinit, pzinit;     /* pressure-pinning cell                          */
    double pinit;                       /* pressure in that cell, Pa                     */
    double gxkoef, gykoef, gzkoef;      /* gravity, m/s^2                                */
    double timesum;                     /* model time, s                                 */
    const float *gx, *gy, *gz;          /* grid lines as stored in the file (FP32)      */
    /* nodal fields, level 0, node = z*(xnumx*ynumy) + x*ynumy + y (head3mg.c:70-80)     */
    double *pr;                         /* pressure (FP64 like the reference)            */
    float *vx, *vy, *vz;
    float *ro, *nu, *nxx, *nxy, *nxz, *nyz;
    float *tk, *cp, *et, *kt, *ht, *rr;
    /* stresses and strain rates written by the Stokes step (head3mg.c:81-82); may be NULL */
    float *exx, *eyy, *ezz, *exy, *exz, *eyz;
    float *sxx, *syy, *szz, *sxy, *sxz, *syz;
    /* boundary rows (load3mg.c:828-838): row index into bondm, x_row = c + k*x_(partner1-1) */
    int64_t bondnum;
    const int64_t *bond_row;
    const float *bond_c, *bond_k;
    const int64_t *bond_partner1;       /* 0 = no partner                                */
    /* markers (load3mg.c:845-859), structure of arrays */
    int64_t marknum;
    float *markx, *marky, *markz, *markk, *markw, *markd, *markv, *marke;
    float *markex, *markft, *markrr, *markrn;
    int8_t *markt;
    /* rock types: 24 tables of rocknum doubles in file order n0 n1 s0 s1 nu dh dv ss mm ll
     * a0 a1 b0 b1 e0 e1 ro bb aa cp kt kf kp ht (load3mg.c:766-789)                     */
    int32_t rocknum;
    const double *rock[24];
} i3g_model;

/* ---- run parameters: mode.t3c (load3mg.c:2-170) ------------------------------------ */
typedef struct i3g_params {
    int32_t printmod, movemod, tempmod, markmod, gridmod, outgrid, densimod;
    double stp100, eroslev, sedilev, waterlev;
    double DIVVMIN, STOKSMIN, DIVVMAX, STOKSMAX;
    int32_t multimax;                   /* levels built (multinum of the V_P block)      */
    int32_t multicyc;                   /* V-cycles per convergence check                */
    int32_t multinnn[2][I3G_MAXLEV];    /* sweeps per level: [0] down leg, [1] up leg    */
    double p0koef, p1koef, p2koef, v0koef, v1koef;
    double nubeg, nuend, nukoef;
    int32_t viscmod;                    /* 0 arithmetic, 1 geometric, 2 harmonic          */
    double HEATMIN;
    int32_t multicyct, multittt0;       /* heat: cycles per check, sweeps per cycle      */
    double t0koef, heatdif;
    int32_t frictyn, adiabyn;
    double zdeep, vdeep, tdeep, nudeep, healrate, teclmin, teclmax;
    double timebeg, timeend, tempend;   /* plume BC schedule, s / K                       */
    /* ---- solver controls of this library (no reference counterpart) ---- */
    double stokes_rtol;                 /* > 0: stop on relative residual (see i3g_stokes)*/
    int32_t stokes_maxcyc;              /* cap on V-cycles per solve (0 = 2000)          */
    double heat_rtol;                   /* > 0: stop on relative heat residual           */
    int32_t heat_maxcyc;                /* cap on heat V-cycles (0 = 2000)               */
    int32_t precision;                  /* 0: FP64 multigrid, 1: FP32 MG inside FP64 defect correction */
    int32_t warm_start;                 /* 0: zero start; 1: the previous step's v,P (reference behaviour);
                                         * 2: linear extrapolation in time from the last two converged
                                         * solutions (falls back to 1 until two exist; an upload of nodal
                                         * fields whose v, P differ from the last solution as downloaded
                                         * resets it, an upload of exactly that state keeps it);
                                         * 3: quadratic extrapolation from the last three (linear while
                                         * only two exist), same reset rule */
    int32_t krylov;                     /* > 0: restarted FGMRES(krylov) (<= 16) on the FP64 residual,
                                         * preconditioned by one V-cycle of this precision (precision 1:
                                         * the FP32 V-cycle on the scaled correction system; precision 0:
                                         * the FP64 V-cycle); 0: one V-cycle per iteration, the
                                         * reference's iteration (with FP64 defect correction for 1) */
    int32_t marker_exact;               /* marker kernels (movemark, ronurecalc, marker temperatures):
                                         * 1: the reference's operation order (divisions, separate
                                         * multiply and add), marker positions bit-identical to the
                                         * reference's; 0: reciprocal spacings and fused multiply-adds,
                                         * interpolated values within ~1e-16 relative of those, FP32
                                         * positions equal except within ~1e-13 m of a rounding boundary */
} i3g_params;

/* ---- per output file row (load3mg.c:25-58, applied at i3mg.c:64-77) ---------------- */
typedef struct i3g_file_params {
    int32_t cyc0max;
    double maxxystep, maxtkstep, maxtmstep;   /* m, K, s */
    double nubeg, nuend;
    double p0koef, p1koef, p2koef;             /* until multstp outer iterations          */
    double p0koef2, p1koef2, p2koef2;          /* afterwards (move3mg.c:2585-2593)        */
    int32_t multinum, multstp, multinum2;
} i3g_file_params;

/* ---- statistics of the last solves -------------------------------------------------- */
typedef struct i3g_stats {
    int32_t stokes_cycles;              /* V-cycles in the last i3g_stokes                */
    int32_t stokes_outer;               /* outer (defect-correction / check) iterations   */
    double stokes_rel0, stokes_rel;     /* relative residual before / after               */
    double stokes_mom_rel, stokes_cont_rel;
    int32_t heat_cycles, heat_substeps;
    double heat_rel;
    double ms_stokes, ms_heat, ms_move, ms_r2n;   /* device time of the last calls        */
    int64_t kernel_launches;            /* kernels launched by this context so far        */
    int32_t stokes_start;               /* start of the last i3g_stokes: 0 the nodal v, P
                                           (uploaded or the last solution), 1 extrapolated
                                           from the last two solutions (warm_start 2), 2 the
                                           staged guess (i3g_unet_predict), 3 extrapolated
                                           from the last three (warm_start 3)              */
} i3g_stats;

typedef struct i3g_ctx i3g_ctx;

/* Create a context on the current CUDA device: checks the model, builds the multigrid
 * geometry (gridcheck, load3mg.c:1162-1283), flattens boundary rows and uploads all
 * arrays.  Replaces loader()+gridcheck() state setup for the device. */
int i3g_create(const i3g_model *m, const i3g_params *p, i3g_ctx **out);
void i3g_destroy(i3g_ctx *c);
const char *i3g_last_error(const i3g_ctx *c);   /* valid for c == NULL too */

/* Per-output-file parameters (i3mg.c:64-77). */
int i3g_set_file_params(i3g_ctx *c, const i3g_file_params *f);

/* Replace the run parameters (no reference counterpart: the reference reads mode.t3c once,
 * load3mg.c:2-170).  The level count (multimax) must stay the one the context was built with;
 * the current file row's nubeg, nuend and p*koef keep overriding the mode values. */
int i3g_set_params(i3g_ctx *c, const i3g_params *p);

/* vpiterate(n0,f0) (move3mg.c:1585-2636): Stokes + continuity on the staggered grid.
 * Stops when the relative residual (momentum ||b-Ax||/||b|| and continuity
 * ||div v|| * h / ||v||, both <= stokes_rtol) is met, or -- when stokes_rtol <= 0 -- on the
 * reference's absolute criteria (move3mg.c:2596).  Lowers *timestep to the CFL limit
 * maxxystep / max|v| (move3mg.c:2608-2632).  Writes v, P, stresses, strain rates. */
int i3g_stokes(i3g_ctx *c, int n0, double *timestep);

/* titerate(n0) (heat3mg.c:287-788): implicit heat step with substeps limited by
 * maxtkstep, geometric multigrid solve, then the marker temperature update with subgrid
 * diffusion.  *timestep is left unchanged on return, as in the reference. */
int i3g_heat(i3g_ctx *c, int n0, double *timestep);

/* movemark() (mark3mg.c:2-397): per-marker rheology update and RK4 advection. */
int i3g_move_markers(i3g_ctx *c, double timestep);

/* ronurecalc() (mark3mg.c:404-1015): marker -> node averages + tkrecalc T boundaries. */
int i3g_markers_to_nodes(i3g_ctx *c, double timestep);

/* Advance model time (i3mg.c:146). */
int i3g_add_time(i3g_ctx *c, double timestep);

/* Host <-> device copies of the model arrays.  mask: I3G_SYNC_* bits.
 * I3G_SYNC_ASYNC (upload only): the marker copies run on the context's copy stream and i3g_upload
 * returns once the nodal copies are done; the Stokes solve then overlaps the marker copies, and
 * the first call that needs the markers (i3g_heat's marker update, i3g_move_markers,
 * i3g_markers_to_nodes, a marker download) waits for them on the device.  The host marker
 * arrays must stay unchanged until such a call has returned.  (The reference keeps the state in
 * static arrays and copies nothing: head3mg.c:33-101.) */
enum { I3G_SYNC_NODES = 1, I3G_SYNC_STRESS = 2, I3G_SYNC_MARKERS = 4, I3G_SYNC_ALL = 7, I3G_SYNC_ASYNC = 8 };
int i3g_download(i3g_ctx *c, i3g_model *m, unsigned mask);
int i3g_upload(i3g_ctx *c, const i3g_model *m, unsigned mask);

int i3g_get_stats(const i3g_ctx *c, i3g_stats *s);

/* Page-locked host memory for model images (no reference counterpart: the reference keeps
 * its state in static arrays, head3mg.c:33-101).  Uploads and downloads from such buffers run
 * at full bus speed and asynchronously to the host thread.  Returns zeroed memory, or NULL
 * (also without a GPU); free with i3g_host_free. */
void *i3g_host_alloc(int64_t bytes);
void i3g_host_free(void *p);

/* ParaView output of the nodal fields (saver_paraview's nodal part, i3vis_output_paraview.c:
 * 700-792 and 887-975, called every 50th output file at i3mg.c:159): a VTK XML RectilinearGrid
 * file with raw appended data -- Float64 grid lines, then viscosity, temperature, density, vy,
 * vx, vz (Float32) and pressure (Float64) in VTK point order (x fastest), reordered on the GPU
 * from the device arrays. */
int i3g_write_vtr(i3g_ctx *c, const char *path);

/* ---- initial conditions on the GPU (in3mg.c, the reference's separate generator) ------- */
/* A rock body of init.t3c (in3mg.c:548-797); coordinates relative to the box size.
 * shape 0: a box whose six faces are bilinear surfaces through its corners 0..7 (corner bits:
 *          1 larger y, 2 larger x, 4 larger z);
 * shape 1: an ellipsoid shell, centre = point 0, axis scales = point 7, scaled radius between
 *          x[2] and x[5];  shape 2: the same as a cylinder along y, |y - y0| <= scale y. */
#define I3G_INIT_MAX_BODIES 256
typedef struct i3g_body {
    int32_t rock, shape;
    double x[8], y[8], z[8];
    double ex, e;                       /* markex and marke of the body's markers          */
} i3g_body;
typedef struct i3g_init {
    int32_t nonstab;                    /* jitter resolution n (0: none), in3mg.c:177-186  */
    double xnonstab, ynonstab, znonstab;/* jitter amplitude, fraction of the marker spacing */
    uint64_t seed;                      /* of the counter-based jitter generator            */
    int32_t background;                 /* rock type of markers outside every body          */
    double t_top, t_bottom;             /* marker temperature, linear in y between these    */
    int32_t nbodies;
    const i3g_body *bodies;             /* applied in order: later bodies win               */
} i3g_init;
/* Replace c's markers by in3mg's initial markers: mnumx x mnumy x mnumz per cell on the
 * placement grid size/(n-1) (in3mg.c:131-175), jittered by (r mod (2n+1) - n)/n x amplitude with
 * r 31-bit numbers from SplitMix64(seed, 3 * marker + axis) (the reference uses rand()), then
 * the bodies.  Rock types >= 50 (fluid, immobile) are rejected as I3G_E_UNSUPPORTED. */
int i3g_init_markers(i3g_ctx *c, const i3g_init *s);
/* The initial-condition passes of in3mg.c:990-1031 on the device: nodes from markers,
 * hydrostatic pressure (in3mg.c:1010-1021), nodes from markers again. */
int i3g_prepare(i3g_ctx *c);

/* ---- kernel-level entry points (parity tests and benchmarks) ------------------------- */
/* Level arrays addressable by i3g_get_array / i3g_set_array (element type in brackets). */
enum {
    I3G_A_SOL = 0,      /* [double, 4*N_l] unknowns P,Vx,Vy,Vz interleaved per node (sol0) */
    I3G_A_RHS = 1,      /* [double, 4*N_l] right-hand sides (fre1)                        */
    I3G_A_RES = 2,      /* [double, 4*N_l] residual b - A x (fre0)                        */
    I3G_A_NU = 3,       /* [float, N_l] nodal viscosity (nu, restricted on l > 0)          */
    I3G_A_ETA = 4,      /* [double, 4*N_l] clamped stress-point viscosities c, xy, xz, yz  */
    I3G_A_TK = 5        /* [double, N_0] temperature solution                              */
};
int i3g_get_array(i3g_ctx *c, int which, int level, void *dst, int64_t nbytes);
int i3g_set_array(i3g_ctx *c, int which, int level, const void *src, int64_t nbytes);

/* Build level operators for the current nodal fields: ronurestrict (move3mg.c:2642-2741),
 * stress-point viscosities, right-hand side (move3mg.c:2029-2159) and load the current
 * v,P into the level-0 solution (move3mg.c:1969-2019). */
int i3g_stokes_setup(i3g_ctx *c);
/* fre0 = fre1 - A sol0 on a level (gausmat4 residual pass, move3mg.c:3136-3157). */
int i3g_stokes_residual(i3g_ctx *c, int level);
/* nsweeps multicolour relaxation sweeps on a level (gausmat4 relaxation formula,
 * move3mg.c:3087-3131, in red-black order per velocity component, then pressure). */
int i3g_stokes_smooth(i3g_ctx *c, int level, int nsweeps);
/* vprestrict(level) (move3mg.c:3165-3520) and vpprolong(level,0) (move3mg.c:2748-3063). */
int i3g_stokes_restrict(i3g_ctx *c, int level);
int i3g_stokes_prolong(i3g_ctx *c, int level);
/* ncycles V-cycles with the schedule of move3mg.c:2170-2223. */
int i3g_stokes_vcycles(i3g_ctx *c, int ncycles);
/* Relative residuals of the level-0 system for the current solution. */
int i3g_stokes_relres(i3g_ctx *c, double *mom_rel, double *cont_rel);
/* Strain rates exx..eyz and stresses sxx..syz of the current level-0 velocities and nodal
 * viscosities: sxxcalc..syzcalc with ynval = 0 (move3mg.c:3-710), as vpiterate recomputes
 * them after its iterations (move3mg.c:2405-2555).  Builds the level operators first, like
 * i3g_stokes_setup; read the result with i3g_download(I3G_SYNC_STRESS). */
int i3g_stokes_stresses(i3g_ctx *c);

/* Time reps launches of one kernel class on the level-0 data with CUDA events on the
 * context stream; returns the mean duration per launch and the algorithmic bytes that one
 * launch must move.  kind: 0 smoother sweep, 1 residual, 2 restriction, 3 prolongation,
 * 4 marker->node, 5 RK4 advection, 6 heat sweep, 7 one FP32 velocity colour, 8 one FP32
 * level-0 sweep, 9 marker temperatures, 10 one FP64 level-0 sweep (kinds 0-10 with L2
 * flushed before every launch); with warm caches: 11 one FP32 V-cycle of the solver's schedule,
 * 12 its coarse tail kernel, 13 + l - 1 one FP32 sweep of level l >= 1, 19 one FP32 sweep of
 * level 0. */
int i3g_time_kernel(i3g_ctx *c, int kind, int reps, double *ms_per_launch, double *bytes_per_launch);

/* Device-side stopwatch on the context stream (no reference counterpart: the reference
 * times phases with clock(), i3mg.c:96-139).  op 0 records the start event; op 1 records
 * the stop event, waits for it and returns the elapsed milliseconds in *ms. */
int i3g_timer(i3g_ctx *c, int op, double *ms);

/* ---- learned warm start: 3-D U-Net (no counterpart in the reference) ---------------- */
/* The reference starts every Stokes solve from the previous step's v, P
 * (move3mg.c:1969-2019).  The network maps log10 viscosity, density and that previous
 * velocity on the level-0 node grid to a correction (dP, dVx, dVy, dVz) of that start; the
 * solver keeps the corrected start only when its relative residual is lower and then iterates
 * to the same tolerance, so the network changes the cycle count, never the converged answer.
 * 4 levels of 16/32/64/128 channels, 15 convolutions of 3x3x3 on tcgen05 tensor cores (BF16
 * operands, FP32 accumulation), Adam on FP32 master weights.  Every grid axis needs n >= 9
 * and n-1 divisible by 8.  Host arrays of nodal data are planar in the solver's node order
 * (node = z*nx*ny + x*ny + y): in5 = [5][n] log10 eta, rho, vx, vy, vz; tg4 / out4 = [4][n]
 * dP, dVx, dVy, dVz.  The handle owns its device memory and its own stream; calls that take a
 * context first wait for the context's stream.  Errors: i3g_last_error(NULL). */
typedef struct i3g_unet i3g_unet;
/* capacity: training samples kept on the device (36 bytes per node each). */
int i3g_unet_create(int nx, int ny, int nz, int capacity, uint64_t seed, i3g_unet **out);
void i3g_unet_destroy(i3g_unet *u);
int i3g_unet_nparams(const i3g_unet *u, int64_t *n);
/* Flat FP32 parameters: per layer W[27][cout][cin] (tap = (dz+1)*9 + (dx+1)*3 + (dy+1)) then b[cout]. */
int i3g_unet_get_params(i3g_unet *u, float *host, int64_t n);
int i3g_unet_set_params(i3g_unet *u, const float *host, int64_t n);   /* also resets Adam */
/* s = {log10-eta mean, 1/std, rho mean, 1/std, velocity scale, pressure scale} */
int i3g_unet_set_scales(i3g_unet *u, const float s[6]);
int i3g_unet_set_sample(i3g_unet *u, int slot, const float *in5, const float *tg4);
int i3g_unet_get_sample(i3g_unet *u, int slot, float *in5, float *tg4);
/* Record the inputs of c's next Stokes solve (before i3g_stokes) and, after it, the target:
 * converged v, P minus that start. */
int i3g_unet_capture_input(i3g_unet *u, i3g_ctx *c, int slot);
int i3g_unet_capture_target(i3g_unet *u, i3g_ctx *c, int slot);
/* One Adam step on the mean loss of the listed samples; *loss = that mean before the step. */
int i3g_unet_train_step(i3g_unet *u, const int *slots, int nslots, float lr, double *loss);
int i3g_unet_loss(i3g_unet *u, const int *slots, int nslots, double *loss);
/* Host data in and out: out4 = correction for in5; with tg4, *loss and (grads != NULL) the
 * parameter gradients of that one sample's loss. */
int i3g_unet_eval_host(i3g_unet *u, const float *in5, const float *tg4, float *out4, float *grads, double *loss);
/* Stage previous v, P + correction as the start of c's next i3g_stokes, which scales the
 * correction by the residual-minimising factor and keeps the result only when its relative
 * residual is lower than the default start's (see i3g_stokes_guess_info). */
int i3g_unet_predict(i3g_unet *u, i3g_ctx *c);
/* Mean device time of one training step on sample slot 0 and of one forward pass. */
int i3g_unet_time(i3g_unet *u, int reps, double *ms_train, double *ms_forward);
/* Mean device time of the forward convolution of layer 0..14 (inputs of the last forward
 * pass) and its algorithmic bytes (interior rows of input, output and skip tensor, weights). */
int i3g_unet_time_conv(i3g_unet *u, int layer, int reps, double *ms, double *bytes);
/* One tensor-core convolution on host BF16 bit patterns over a padded (nz+2)(nx+2)(ny+2) grid:
 * in [rows][cin], w [27][cout][cin], bias [cout] or NULL, add [rows][cout] or NULL; out FP32
 * [rows][cout], interior rows only.  cin, cout in {16, 32, 64, 128} as the network pairs them. */
int i3g_unet_conv_host(int cin, int cout, int nx, int ny, int nz, const uint16_t *in, const uint16_t *w,
                       const float *bias, const uint16_t *add, int relu, float *out);
/* Weight and bias gradients of one convolution layer on host BF16 bit patterns over the same
 * padded grid: x [rows][cin] the layer's input, g [rows][cout] the gradient of its output (zero
 * on halo rows); dw [27][cout][cin] = sum_rows g[row][co] x[row + tap offset][ci] and db [cout]
 * in FP32 (tcgen05 for cin, cout in {16, 32}, CUDA cores otherwise).  No reference counterpart
 * (the reference has no network); used by the tests. */
int i3g_unet_wgrad_host(int cin, int cout, int nx, int ny, int nz, const uint16_t *x, const uint16_t *g, float *dw,
                        float *db);
/* Last i3g_stokes: used = -1 no staged start, 0 rejected, 1 used; relative residuals of the
 * staged start (after scaling its correction by alpha) and of the default start; alpha is the
 * factor a >= 0 minimising the row-weighted residual of default + a (staged - default). */
int i3g_stokes_guess_info(const i3g_ctx *c, int *used, double *rel_guess, double *rel_default, double *alpha);

/* ---- allocation-free stopping test (no counterpart in the reference) --------------- */
/* For host codes that may not allocate device memory after start-up (they give all of it
 * to their own pool allocator, or cannot let a cudaMalloc synchronise the device under work
 * they have queued) and so cannot create a context.  Computes the two numbers of
 * i3g_stokes_relres() -- momentum ||b - Ax|| / ||b|| and continuity RMS(div v) * h / RMS(v)
 * over the non-boundary rows -- from a level-0 system in the caller's device memory, in
 * the library's layout (node = z*nx*ny + x*ny + y; one array per component):
 *   res[4]  device residuals of the P, Vx, Vy, Vz rows (b - Ax)
 *   rhs[4], sol[4]  device right-hand sides and solution (index 0, pressure, is not read)
 *   bc      device byte per node, bit v set when row v of that node is a boundary row
 *   h       mean grid spacing, (xsize/(nx-1) + ysize/(ny-1) + zsize/(nz-1)) / 3
 *   out     device, 2 doubles: momentum, continuity
 *   stream  cudaStream_t the two kernels are queued on (NULL: the legacy default stream);
 *           the call returns without waiting for them.
 * It allocates nothing: its scratch is a static device array of I3G_NOALLOC_MAX_COLUMNS x 6
 * doubles (3 MiB, held by every GPU that loads the library until the process exits), one
 * slot per x-z grid column, so grids with nx*nz > I3G_NOALLOC_MAX_COLUMNS are rejected with
 * I3G_E_ARG.  The first call on each device looks up the array's device address (make it
 * before any stream capture on that device).  All calls share the array: calls whose kernels
 * may overlap on the GPU race.  Errors are read with i3g_last_error(NULL). */
#define I3G_NOALLOC_MAX_COLUMNS 65536
int i3g_stokes_relres_noalloc(int nx, int ny, int nz, double h, const uint8_t *bc,
                              const double *const res[4], const double *const rhs[4],
                              const double *const sol[4], double *out, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* I3G_H */
