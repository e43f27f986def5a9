// i3g_internal.cuh -- device-side data layout of the B200 time-step library.
//
// Every multigrid level keeps the reference's node numbering (node = z*NX*NY + x*NY + y,
// y fastest: move3mg.c:1632) so that a warp reads consecutive y.  Unknowns are stored as
// separate arrays per component (P, Vx, Vy, Vz) instead of the reference's interleaved
// sol0[4*node+k] (head3mg.c:33), which keeps every component load unit-stride.
#pragma once
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <utility>
#include <cuda_runtime.h>
#include "../../include/i3g.h"

#define I3G_CUDA(call)                                                                   \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess) return cuda_fail(c, e_, #call, __FILE__, __LINE__);        \
    } while (0)

namespace i3g {

// Programmatic dependent launch: kernels launched through launch_pdl() are scheduled while their
// predecessor on the stream still runs; each such kernel must start with pdl_enter(), which waits
// for the predecessor's completion (and memory) before any data is touched and then lets its own
// successor launch.  On latency-bound launches this hides most of the launch gap.
__device__ __forceinline__ void pdl_enter()
{
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

inline bool pdl_enabled()
{
    static const bool on = getenv("I3G_PDL") == nullptr || atoi(getenv("I3G_PDL")) != 0;
    return on;
}

template <typename... KArgs, typename... Args>
inline void launch_pdl(cudaStream_t st, void (*kern)(KArgs...), dim3 grid, dim3 block, Args &&...args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = pdl_enabled() ? 1 : 0;
    cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}

constexpr int kMaxBcDepth = 4;   // boundary chains x_a = c + k x_b, x_b = c' + k' x_c, ...

// Boundary rows of one component on one level, flattened to an interior partner.
struct BcList {
    int n = 0;
    int *node = nullptr;        // row node (level-local)
    int *pnode = nullptr;       // interior partner node, -1: constant
    int *depth = nullptr;       // number of (c,k) pairs in the chain (1..kMaxBcDepth)
    double *c = nullptr;        // [n*kMaxBcDepth] chain constants, outermost first
    double *k = nullptr;        // [n*kMaxBcDepth] chain factors
    int *onode = nullptr;       // original partner node (unflattened), -1: none
    int *ocomp = nullptr;       // original partner component
    double *oc = nullptr, *ok = nullptr;   // original constant and factor (level 0 residual)
    // Rows written inside the relaxation kernel that finalises the component in a sweep
    // (na >= 0): entries [0, na) are sorted by their writer, a row of that kernel, and written by
    // the writer's thread right after its own update (bit 4 + v of the level's bc byte marks
    // writers, first[node] is a writer's first entry); entries [na, n) run on extra blocks of
    // that kernel.  na = -1: a separate boundary pass after the kernel.
    int na = -1;
    int *first = nullptr;
    int *writer = nullptr;
};

template <typename T>
struct Fields {
    T *u[4] = {nullptr, nullptr, nullptr, nullptr};    // solution: P, Vx, Vy, Vz
    T *f[4] = {nullptr, nullptr, nullptr, nullptr};    // right-hand side (fre1)
    T *r[4] = {nullptr, nullptr, nullptr, nullptr};    // residual (fre0)
    T *etac = nullptr, *etaxy = nullptr, *etaxz = nullptr, *etayz = nullptr;
    T *ix[2] = {nullptr, nullptr};   // per axis x: [0] 1/(g[i]-g[i-1]), [1] 1/(g[i+1]-g[i-1])
    T *iy[2] = {nullptr, nullptr};
    T *iz[2] = {nullptr, nullptr};
    float *nd = nullptr;             // pressure relaxation viscosity (FP32 like the reference's nd[])
};

// Separable 1-D transfer stencils between a fine level and the next coarse level.
// For fine index f: coarse cell index a[f] and weights w0[f] (to a) and w1[f] (to a+1).
// For the gather form, coarse index c lists its fine contributors (ascending f) in
// [gptr[c], gptr[c+1]) with fine index gf and weight gw.
struct Transfer1D {
    int nf = 0, nc = 0;
    int *a = nullptr;
    double *w0 = nullptr, *w1 = nullptr;
    int *gptr = nullptr, *gf = nullptr;
    double *gw = nullptr;
};

// staggering kinds: 0 grid line, 1 mid-point, 2 cell centre, 3 grid line with |d| weights
// (viscosity restriction)
constexpr int kStagLine = 0, kStagMid = 1, kStagCell = 2, kStagAbs = 3;

struct Level {
    int nx = 0, ny = 0, nz = 0;
    long n = 0;
    double *gx = nullptr, *gy = nullptr, *gz = nullptr;   // level coordinates (host)
    float *nu = nullptr;               // nodal viscosity of this level
    uint8_t *bc = nullptr;             // bit v: row v (0 P, 1 Vx, 2 Vy, 3 Vz) is a boundary row;
                                       // bit 4 + v: partner of in-kernel boundary rows of v (BcList::na)
    Fields<double> d;
    Fields<float> s;                    // scaled FP32 copy for the mixed-precision solver
    BcList bcl[4];
    Transfer1D tr[3][4];               // to the next coarser level: axis x,y,z; staggering
    long scratch_n = 0;
    double *red = nullptr;             // reduction scratch
};

// Two CUDA events for a device-time measurement, destroyed on every return path.
struct EventPair {
    cudaEvent_t a = nullptr, b = nullptr;
    EventPair() = default;
    EventPair(const EventPair &) = delete;
    EventPair &operator=(const EventPair &) = delete;
    cudaError_t create()
    {
        cudaError_t e = cudaEventCreate(&a);
        return e == cudaSuccess ? cudaEventCreate(&b) : e;
    }
    ~EventPair()
    {
        if (a) cudaEventDestroy(a);
        if (b) cudaEventDestroy(b);
    }
};

}  // namespace i3g

struct i3g_ctx {
    i3g_model m;
    i3g_params p;
    i3g_file_params f;
    int dev = 0;
    cudaStream_t st = nullptr;
    cudaStream_t cst = nullptr;                 // copy stream of asynchronous marker uploads
    long nodenum = 0, marknum = 0;
    int nlev = 0;
    i3g::Level lev[I3G_MAXLEV];
    // level-0 physical fields (device)
    double *pr = nullptr;
    float *vx = nullptr, *vy = nullptr, *vz = nullptr;
    float *ro = nullptr, *nxx = nullptr, *nxy = nullptr, *nxz = nullptr, *nyz = nullptr;
    float *tk = nullptr, *cp = nullptr, *et = nullptr, *kt = nullptr, *ht = nullptr, *rr = nullptr;
    float *eps[6] = {}, *sig[6] = {};   // exx eyy ezz exy exz eyz / sxx ...
    double *gx0 = nullptr, *gy0 = nullptr, *gz0 = nullptr;   // level-0 grid lines (device)
    // host copies of the grid lines
    double *hgx = nullptr, *hgy = nullptr, *hgz = nullptr;
    // reductions
    double *dred = nullptr, *hred = nullptr;    // device scratch and pinned host mirror
    double *hstage = nullptr;                   // pinned host staging (4 * red_blocks doubles)
    int red_blocks = 0;
    double ncont = 0, nvel = 0;                 // level-0 row counts for the continuity norm
    float **deps = nullptr, **dsig = nullptr;   // device arrays of the 6+6 stress/strain pointers
    // bookkeeping
    bool stokes_ready = false;
    double eta_ref = 1.0, h_ref = 1.0;
    i3g_stats st_;
    char err[512] = {0};
    int64_t launches = 0;
    cudaEvent_t tev[2] = {nullptr, nullptr};   // i3g_timer
    // captured Stokes iteration (one V-cycle + norms) and the parameters it was built with
    cudaGraphExec_t sgraph = nullptr;
    int sg_multinum = -1, sg_prec = -1;
    double sg_p0 = 0, sg_p1 = 0, sg_v0 = 0, sg_v1 = 0;
    long sg_nodes = 0;
    double *dscale = nullptr;                   // device scale factors of the FP32 correction solve
    void *flush = nullptr;                      // 256 MiB written between cold-cache timings (L2 is 126 MB)
    long tail_nodes = 2000;                     // levels up to this size run in the one-block V-cycle tail
    long coop_nodes = 0;                        // > 0: levels up to this size run in the cooperative coarse kernel
    int tail_cluster = 1;                       // CTAs of the V-cycle tail (> 1: one thread-block cluster)
    int fuse = 1;                               // boundary rows inside the relaxation kernels of levels >= 1
                                                // (3: level 0 too), residual and four-component transfer
                                                // launches (0: one launch per pass)
    int coop_blocks = 0;                        // its grid: every CTA resident at once (0: no cooperative launch)
    unsigned *dbar = nullptr;                   // its grid barrier: arrival count, generation
    int *dbar_err = nullptr;                    // set when a grid barrier wait timed out
    // FP32 smoother's pressure scale: the face rows' harmonic-mean viscosity where it exceeds the
    // cell viscosity by more than this factor (k_nd_schur; 0: the cell viscosity everywhere)
    int nd_schur = 10;
    double *hist[3][4] = {};                    // last three converged level-0 solutions, newest last
                                                // (warm_start 2 and 3)
    int hist_check = 0;                         // an upload is being compared with the last solution
    int *dflag = nullptr, *hflag = nullptr;     // its result: device flag and pinned host mirror
    double hist_dt[3] = {0, 0, 0};              // time steps taken after them
    int nhist = 0;
    // staged start for the next Stokes solve (i3g_unet_predict); kept only when its relative
    // residual is below the default start's
    double *guess[4] = {};
    double *gsave[8] = {};                      // default start (0..3) and its residual (4..7)
    double *gdots = nullptr;                    // 2 device doubles: weighted <r0,dr>, <dr,dr>
    int guess_pending = 0;
    int guess_used = -1;                        // last solve: -1 none staged, 0 rejected, 1 used
    double guess_rel[2] = {0, 0};               // relative residual of the staged / default start
    double guess_alpha = 0;                     // factor applied to the staged correction
    void *kry = nullptr;       // FGMRES state of the mixed-precision Stokes solve
    void *heat = nullptr;      // heat-solver state
    void *mk = nullptr;        // marker state
};

int cuda_fail(i3g_ctx *c, cudaError_t e, const char *what, const char *file, int line);

namespace i3g {
constexpr size_t kFlushBytes = 256ull << 20;

// Mean device time of `launch()` with an empty L2: before every repetition a buffer of twice the
// L2 size is overwritten on the stream, outside the timed interval, so each timed launch reads
// its data from HBM.  Every repetition has its own event pair.
template <typename F>
int cold_time(i3g_ctx *c, int reps, F launch, double *ms)
{
    if (!c->flush) I3G_CUDA(cudaMalloc(&c->flush, kFlushBytes));
    cudaEvent_t ev[2 * 64];
    if (reps > 64) reps = 64;
    for (int i = 0; i < 2 * reps; i++) ev[i] = nullptr;
    int rc = 0;
    for (int i = 0; i < 2 * reps && !rc; i++)
        if (cudaEventCreate(&ev[i]) != cudaSuccess) rc = 1;
    for (int r = 0; r < reps && !rc; r++) {
        if (cudaMemsetAsync(c->flush, r & 0xff, kFlushBytes, c->st) != cudaSuccess) rc = 1;
        cudaEventRecord(ev[2 * r], c->st);
        if (!rc) rc = launch();
        cudaEventRecord(ev[2 * r + 1], c->st);
    }
    double tot = 0;
    if (!rc && cudaEventSynchronize(ev[2 * reps - 1]) != cudaSuccess) rc = 1;
    for (int r = 0; r < reps && !rc; r++) {
        float t = 0;
        cudaEventElapsedTime(&t, ev[2 * r], ev[2 * r + 1]);
        tot += t;
    }
    for (int i = 0; i < 2 * reps; i++)
        if (ev[i]) cudaEventDestroy(ev[i]);
    if (rc) {
        cudaError_t e = cudaGetLastError();
        return e != cudaSuccess ? cuda_fail(c, e, "cold_time", __FILE__, __LINE__) : rc;
    }
    *ms = tot / reps;
    return 0;
}
}  // namespace i3g
int set_error(i3g_ctx *c, int code, const char *fmt, ...);
int set_global_error(int code, const char *fmt, ...);

namespace i3g {
// stokes.cu
int stokes_alloc(i3g_ctx *c);
void stokes_free(i3g_ctx *c);
void stokes_graph_free(i3g_ctx *c);
void stokes_params_changed(i3g_ctx *c);
int stokes_setup(i3g_ctx *c);
int stokes_upload_check(i3g_ctx *c);
int stokes_residual(i3g_ctx *c, int level);
int stokes_smooth(i3g_ctx *c, int level, int nsweeps);
int stokes_restrict(i3g_ctx *c, int level);
int stokes_prolong(i3g_ctx *c, int level);
int stokes_vcycle(i3g_ctx *c, int multinum);
int stokes_relres(i3g_ctx *c, double *mom, double *cont);
int stokes_stresses(i3g_ctx *c);
int stokes_solve(i3g_ctx *c, double *timestep);
int stokes_time_kernel(i3g_ctx *c, int kind, int reps, double *ms, double *bytes);
}  // namespace i3g
