// i3g_api.cu -- the extern "C" boundary declared in include/i3g.h.
//
// Owns the device copies of the reference's global arrays (head3mg.c:33-101) for one model
// and dispatches the four time-step calls of the host loop (i3mg.c:98-137).  Host arrays are
// touched only by i3g_create / i3g_upload / i3g_download.
#include <cstdarg>
#include <cstring>
#include <vector>
#include "i3g_internal.cuh"
#include "heat_markers.cuh"

int set_error(i3g_ctx *c, int code, const char *fmt, ...)
{
    if (c) {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(c->err, sizeof c->err, fmt, ap);
        va_end(ap);
    }
    return code;
}

int cuda_fail(i3g_ctx *c, cudaError_t e, const char *what, const char *file, int line)
{
    const int code = (e == cudaErrorMemoryAllocation) ? I3G_E_NOMEM : I3G_E_CUDA;
    return set_error(c, code, "%s: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
}

static thread_local char g_err[512];

// failures of entry points that have no context (reported by i3g_last_error(NULL))
int set_global_error(int code, const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
    return code;
}

template <typename T>
static int dup_to_device(i3g_ctx *c, T *&dst, const T *src, long n)
{
    if (cudaMalloc((void **)&dst, sizeof(T) * (n > 0 ? n : 1)) != cudaSuccess)
        return set_error(c, I3G_E_NOMEM, "cudaMalloc of %ld elements failed", n);
    if (src) I3G_CUDA(cudaMemcpyAsync(dst, src, sizeof(T) * n, cudaMemcpyHostToDevice, c->st));
    else I3G_CUDA(cudaMemsetAsync(dst, 0, sizeof(T) * n, c->st));
    return 0;
}

extern "C" {

const char *i3g_last_error(const i3g_ctx *c) { return c ? c->err : g_err; }

void i3g_destroy(i3g_ctx *c)
{
    if (!c) return;
    cudaStreamSynchronize(c->st);
    i3g::markers_free(c);
    i3g::heat_free(c);
    i3g::stokes_free(c);
    void *f[] = {c->pr, c->vx, c->vy, c->vz, c->ro, c->nxx, c->nxy, c->nxz, c->nyz, c->tk, c->cp, c->et,
                 c->kt, c->ht, c->rr, c->gx0, c->gy0, c->gz0, c->lev[0].nu, c->deps, c->dsig};
    for (void *p : f) cudaFree(p);
    for (int a = 0; a < 6; a++) { cudaFree(c->eps[a]); cudaFree(c->sig[a]); }
    for (int v = 0; v < 4; v++) cudaFree(c->guess[v]);
    for (int v = 0; v < 8; v++) cudaFree(c->gsave[v]);
    cudaFree(c->gdots);
    if (c->hstage) cudaFreeHost(c->hstage);
    if (c->tev[0]) { cudaEventDestroy(c->tev[0]); cudaEventDestroy(c->tev[1]); }
    delete[] c->hgx; delete[] c->hgy; delete[] c->hgz;
    cudaFree(c->flush);
    if (c->st) cudaStreamDestroy(c->st);
    if (c->cst) cudaStreamDestroy(c->cst);
    delete c;
}

int i3g_create(const i3g_model *m, const i3g_params *p, i3g_ctx **out)
{
    if (!out) return I3G_E_ARG;
    *out = nullptr;
    if (!m || !p) { snprintf(g_err, sizeof g_err, "null model or params"); return I3G_E_ARG; }
    if (m->xnumx < 5 || m->ynumy < 5 || m->znumz < 5) { snprintf(g_err, sizeof g_err, "grid must have at least 5 nodes per axis"); return I3G_E_ARG; }
    if (!m->gx || !m->gy || !m->gz || !m->pr || !m->vx || !m->vy || !m->vz || !m->ro || !m->nu || !m->nxx ||
        !m->nxy || !m->nxz || !m->nyz || !m->tk) { snprintf(g_err, sizeof g_err, "missing nodal field pointer"); return I3G_E_ARG; }
    if (p->multimax < 0 || p->multimax + 1 > I3G_MAXLEV) { snprintf(g_err, sizeof g_err, "multimax %d out of range", p->multimax); return I3G_E_ARG; }
    if (m->marknum < 0 || (m->marknum > 0 && (!m->markx || !m->marky || !m->markz || !m->markt))) { snprintf(g_err, sizeof g_err, "bad marker arrays"); return I3G_E_ARG; }
    i3g_ctx *c = new i3g_ctx();
    c->m = *m;
    c->p = *p;
    c->f.multinum = p->multimax; c->f.multinum2 = p->multimax; c->f.multstp = 0;
    c->f.nubeg = p->nubeg; c->f.nuend = p->nuend;
    c->f.p0koef = c->f.p0koef2 = p->p0koef; c->f.p1koef = c->f.p1koef2 = p->p1koef; c->f.p2koef = c->f.p2koef2 = p->p2koef;
    c->f.maxxystep = 0; c->f.maxtkstep = 1e30; c->f.maxtmstep = 1e30; c->f.cyc0max = 1;
    cudaGetDevice(&c->dev);
    if (cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->cst, cudaStreamNonBlocking) != cudaSuccess) {
        snprintf(g_err, sizeof g_err, "cannot create a CUDA stream (is a GPU present?)");
        if (c->st) cudaStreamDestroy(c->st);
        delete c;
        return I3G_E_CUDA;
    }
    c->nodenum = m->xnumx * m->ynumy * m->znumz;
    c->marknum = m->marknum;
    c->nlev = p->multimax + 1;
    const long N = c->nodenum;
    c->hgx = new double[m->xnumx]; c->hgy = new double[m->ynumy]; c->hgz = new double[m->znumz];
    for (long i = 0; i < m->xnumx; i++) c->hgx[i] = m->gx[i];
    for (long i = 0; i < m->ynumy; i++) c->hgy[i] = m->gy[i];
    for (long i = 0; i < m->znumz; i++) c->hgz[i] = m->gz[i];
    int rc = 0;
    if ((rc = dup_to_device(c, c->pr, m->pr, N)) || (rc = dup_to_device(c, c->vx, m->vx, N)) ||
        (rc = dup_to_device(c, c->vy, m->vy, N)) || (rc = dup_to_device(c, c->vz, m->vz, N)) ||
        (rc = dup_to_device(c, c->ro, m->ro, N)) || (rc = dup_to_device(c, c->lev[0].nu, (const float *)m->nu, N)) ||
        (rc = dup_to_device(c, c->nxx, m->nxx, N)) || (rc = dup_to_device(c, c->nxy, m->nxy, N)) ||
        (rc = dup_to_device(c, c->nxz, m->nxz, N)) || (rc = dup_to_device(c, c->nyz, m->nyz, N)) ||
        (rc = dup_to_device(c, c->tk, m->tk, N)) || (rc = dup_to_device(c, c->cp, (const float *)m->cp, N)) ||
        (rc = dup_to_device(c, c->et, (const float *)m->et, N)) || (rc = dup_to_device(c, c->kt, (const float *)m->kt, N)) ||
        (rc = dup_to_device(c, c->ht, (const float *)m->ht, N)) || (rc = dup_to_device(c, c->rr, (const float *)m->rr, N)) ||
        (rc = dup_to_device(c, c->gx0, c->hgx, m->xnumx)) || (rc = dup_to_device(c, c->gy0, c->hgy, m->ynumy)) ||
        (rc = dup_to_device(c, c->gz0, c->hgz, m->znumz))) {
        snprintf(g_err, sizeof g_err, "%s", c->err);
        i3g_destroy(c);
        return rc;
    }
    const float *he[6] = {m->exx, m->eyy, m->ezz, m->exy, m->exz, m->eyz};
    const float *hs[6] = {m->sxx, m->syy, m->szz, m->sxy, m->sxz, m->syz};
    for (int a = 0; a < 6 && !rc; a++) {
        rc = dup_to_device(c, c->eps[a], he[a], N);
        if (!rc) rc = dup_to_device(c, c->sig[a], hs[a], N);
    }
    if (!rc) {
        if (cudaMalloc((void **)&c->deps, 6 * sizeof(float *)) != cudaSuccess ||
            cudaMalloc((void **)&c->dsig, 6 * sizeof(float *)) != cudaSuccess) rc = set_error(c, I3G_E_NOMEM, "cudaMalloc failed");
        else {
            cudaMemcpyAsync(c->deps, c->eps, 6 * sizeof(float *), cudaMemcpyHostToDevice, c->st);
            cudaMemcpyAsync(c->dsig, c->sig, 6 * sizeof(float *), cudaMemcpyHostToDevice, c->st);
        }
    }
    if (!rc) rc = i3g::stokes_alloc(c);
    if (!rc && cudaMallocHost((void **)&c->hstage, sizeof(double) * 4 * (c->red_blocks + 64)) != cudaSuccess)
        rc = set_error(c, I3G_E_NOMEM, "pinned staging allocation failed");
    if (!rc) rc = i3g::heat_alloc(c);
    if (!rc) rc = i3g::markers_alloc(c);
    if (!rc && cudaStreamSynchronize(c->st) != cudaSuccess) rc = set_error(c, I3G_E_CUDA, "%s", cudaGetErrorString(cudaGetLastError()));
    if (rc) {
        snprintf(g_err, sizeof g_err, "%s", c->err);
        i3g_destroy(c);
        return rc;
    }
    *out = c;
    return 0;
}

int i3g_set_file_params(i3g_ctx *c, const i3g_file_params *f)
{
    if (!c || !f) return I3G_E_ARG;
    c->f = *f;
    c->p.nubeg = f->nubeg;
    c->p.nuend = f->nuend;
    c->p.p0koef = f->p0koef;
    c->p.p1koef = f->p1koef;
    c->p.p2koef = f->p2koef;
    return 0;
}

int i3g_set_params(i3g_ctx *c, const i3g_params *p)
{
    if (!c || !p) return I3G_E_ARG;
    if (p->multimax != c->p.multimax)
        return set_error(c, I3G_E_ARG, "multimax %d differs from the %d levels the context was built with", p->multimax,
                         c->p.multimax);
    c->p = *p;
    // the current output-file row keeps overriding these (i3mg.c:64-77)
    c->p.nubeg = c->f.nubeg;
    c->p.nuend = c->f.nuend;
    c->p.p0koef = c->f.p0koef;
    c->p.p1koef = c->f.p1koef;
    c->p.p2koef = c->f.p2koef;
    i3g::stokes_params_changed(c);
    return 0;
}

int i3g_stokes(i3g_ctx *c, int n0, double *timestep)
{
    (void)n0;
    if (!c || !timestep) return I3G_E_ARG;
    return i3g::stokes_solve(c, timestep);
}

int i3g_heat(i3g_ctx *c, int n0, double *timestep)
{
    (void)n0;
    if (!c || !timestep) return I3G_E_ARG;
    return i3g::heat_solve(c, timestep);
}

int i3g_move_markers(i3g_ctx *c, double timestep)
{
    if (!c) return I3G_E_ARG;
    return i3g::markers_move(c, timestep);
}

int i3g_markers_to_nodes(i3g_ctx *c, double timestep)
{
    if (!c) return I3G_E_ARG;
    return i3g::markers_to_nodes(c, timestep);
}

int i3g_add_time(i3g_ctx *c, double timestep)
{
    if (!c) return I3G_E_ARG;
    c->m.timesum += timestep;
    return 0;
}

#define D2H(dst, src, n, sz) do { if (dst) I3G_CUDA(cudaMemcpyAsync(dst, src, (size_t)(n) * (sz), cudaMemcpyDeviceToHost, c->st)); } while (0)
#define H2D(dst, src, n, sz) do { if (src) I3G_CUDA(cudaMemcpyAsync(dst, src, (size_t)(n) * (sz), cudaMemcpyHostToDevice, c->st)); } while (0)

int i3g_download(i3g_ctx *c, i3g_model *m, unsigned mask)
{
    if (!c || !m) return I3G_E_ARG;
    const long N = c->nodenum;
    if (mask & I3G_SYNC_NODES) {
        D2H(m->pr, c->pr, N, 8);
        D2H(m->vx, c->vx, N, 4); D2H(m->vy, c->vy, N, 4); D2H(m->vz, c->vz, N, 4);
        D2H(m->ro, c->ro, N, 4); D2H(m->nu, c->lev[0].nu, N, 4);
        D2H(m->nxx, c->nxx, N, 4); D2H(m->nxy, c->nxy, N, 4); D2H(m->nxz, c->nxz, N, 4); D2H(m->nyz, c->nyz, N, 4);
        D2H(m->tk, c->tk, N, 4); D2H(m->cp, c->cp, N, 4); D2H(m->et, c->et, N, 4);
        D2H(m->kt, c->kt, N, 4); D2H(m->ht, c->ht, N, 4); D2H(m->rr, c->rr, N, 4);
    }
    if (mask & I3G_SYNC_STRESS) {
        float *he[6] = {m->exx, m->eyy, m->ezz, m->exy, m->exz, m->eyz};
        float *hs[6] = {m->sxx, m->syy, m->szz, m->sxy, m->sxz, m->syz};
        for (int a = 0; a < 6; a++) { D2H(he[a], c->eps[a], N, 4); D2H(hs[a], c->sig[a], N, 4); }
    }
    if (mask & I3G_SYNC_MARKERS) {
        int rc = i3g::markers_download(c, m);
        if (rc) return rc;
    }
    m->timesum = c->m.timesum;
    I3G_CUDA(cudaStreamSynchronize(c->st));
    return 0;
}

int i3g_upload(i3g_ctx *c, const i3g_model *m, unsigned mask)
{
    if (!c || !m) return I3G_E_ARG;
    const long N = c->nodenum;
    if (mask & I3G_SYNC_NODES) {
        H2D(c->pr, m->pr, N, 8);
        H2D(c->vx, m->vx, N, 4); H2D(c->vy, m->vy, N, 4); H2D(c->vz, m->vz, N, 4);
        H2D(c->ro, m->ro, N, 4); H2D(c->lev[0].nu, m->nu, N, 4);
        H2D(c->nxx, m->nxx, N, 4); H2D(c->nxy, m->nxy, N, 4); H2D(c->nxz, m->nxz, N, 4); H2D(c->nyz, m->nyz, N, 4);
        H2D(c->tk, m->tk, N, 4); H2D(c->cp, m->cp, N, 4); H2D(c->et, m->et, N, 4);
        H2D(c->kt, m->kt, N, 4); H2D(c->ht, m->ht, N, 4); H2D(c->rr, m->rr, N, 4);
        // the extrapolation history survives only an upload of the library's own last solution
        int rc = i3g::stokes_upload_check(c);
        if (rc) return rc;
    }
    if (mask & I3G_SYNC_STRESS) {
        const float *he[6] = {m->exx, m->eyy, m->ezz, m->exy, m->exz, m->eyz};
        const float *hs[6] = {m->sxx, m->syy, m->szz, m->sxy, m->sxz, m->syz};
        for (int a = 0; a < 6; a++) { H2D(c->eps[a], he[a], N, 4); H2D(c->sig[a], hs[a], N, 4); }
    }
    if (mask & I3G_SYNC_MARKERS) {
        int rc = i3g::markers_upload(c, m, (mask & I3G_SYNC_ASYNC) != 0);
        if (rc) return rc;
    }
    c->m.timesum = m->timesum;
    I3G_CUDA(cudaStreamSynchronize(c->st));
    return 0;
}

void *i3g_host_alloc(int64_t bytes)
{
    if (bytes <= 0) return nullptr;
    void *p = nullptr;
    if (cudaMallocHost(&p, (size_t)bytes) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    memset(p, 0, (size_t)bytes);
    return p;
}

void i3g_host_free(void *p)
{
    if (p) cudaFreeHost(p);
}

int i3g_get_stats(const i3g_ctx *c, i3g_stats *s)
{
    if (!c || !s) return I3G_E_ARG;
    *s = c->st_;
    s->kernel_launches = c->launches;
    return 0;
}

// ---- kernel-level entry points ----
static int level_ok(i3g_ctx *c, int level)
{
    if (level < 0 || level >= c->nlev) return set_error(c, I3G_E_ARG, "level %d out of range", level);
    return 0;
}

int i3g_get_array(i3g_ctx *c, int which, int level, void *dst, int64_t nbytes)
{
    if (!c || !dst) return I3G_E_ARG;
    int rc = level_ok(c, level);
    if (rc) return rc;
    i3g::Level &L = c->lev[level];
    const long n = L.n;
    if (which == I3G_A_NU) {
        if (nbytes != n * 4) return set_error(c, I3G_E_ARG, "size mismatch");
        I3G_CUDA(cudaMemcpyAsync(dst, L.nu, n * 4, cudaMemcpyDeviceToHost, c->st));
        I3G_CUDA(cudaStreamSynchronize(c->st));
        return 0;
    }
    if (which == I3G_A_TK) return i3g::heat_get_solution(c, dst, nbytes);
    if (nbytes != n * 32) return set_error(c, I3G_E_ARG, "size mismatch (%lld != %ld)", (long long)nbytes, n * 32);
    double *src[4];
    switch (which) {
    case I3G_A_SOL: for (int v = 0; v < 4; v++) src[v] = L.d.u[v]; break;
    case I3G_A_RHS: for (int v = 0; v < 4; v++) src[v] = L.d.f[v]; break;
    case I3G_A_RES: for (int v = 0; v < 4; v++) src[v] = L.d.r[v]; break;
    case I3G_A_ETA: src[0] = L.d.etac; src[1] = L.d.etaxy; src[2] = L.d.etaxz; src[3] = L.d.etayz; break;
    default: return set_error(c, I3G_E_ARG, "unknown array %d", which);
    }
    std::vector<double> h(4 * n);
    for (int v = 0; v < 4; v++) I3G_CUDA(cudaMemcpyAsync(h.data() + v * n, src[v], n * 8, cudaMemcpyDeviceToHost, c->st));
    I3G_CUDA(cudaStreamSynchronize(c->st));
    double *o = (double *)dst;
    for (long q = 0; q < n; q++)
        for (int v = 0; v < 4; v++) o[4 * q + v] = h[v * n + q];
    return 0;
}

int i3g_set_array(i3g_ctx *c, int which, int level, const void *src, int64_t nbytes)
{
    if (!c || !src) return I3G_E_ARG;
    int rc = level_ok(c, level);
    if (rc) return rc;
    i3g::Level &L = c->lev[level];
    const long n = L.n;
    if (nbytes != n * 32) return set_error(c, I3G_E_ARG, "size mismatch");
    double *dst[4];
    switch (which) {
    case I3G_A_SOL: for (int v = 0; v < 4; v++) dst[v] = L.d.u[v]; break;
    case I3G_A_RHS: for (int v = 0; v < 4; v++) dst[v] = L.d.f[v]; break;
    case I3G_A_RES: for (int v = 0; v < 4; v++) dst[v] = L.d.r[v]; break;
    default: return set_error(c, I3G_E_ARG, "array %d is read-only", which);
    }
    std::vector<double> h(4 * n);
    const double *s = (const double *)src;
    for (long q = 0; q < n; q++)
        for (int v = 0; v < 4; v++) h[v * n + q] = s[4 * q + v];
    for (int v = 0; v < 4; v++) I3G_CUDA(cudaMemcpyAsync(dst[v], h.data() + v * n, n * 8, cudaMemcpyHostToDevice, c->st));
    I3G_CUDA(cudaStreamSynchronize(c->st));
    return 0;
}

int i3g_stokes_setup(i3g_ctx *c)
{
    if (!c) return I3G_E_ARG;
    int rc = i3g::stokes_setup(c);
    if (rc) return rc;
    I3G_CUDA(cudaStreamSynchronize(c->st));
    return 0;
}

#define LEVEL_CALL(fn)                                                                    \
    if (!c) return I3G_E_ARG;                                                             \
    int rc = level_ok(c, level);                                                          \
    if (rc) return rc;                                                                    \
    rc = fn;                                                                              \
    if (rc) return rc;                                                                    \
    I3G_CUDA(cudaStreamSynchronize(c->st));                                               \
    return 0

int i3g_stokes_residual(i3g_ctx *c, int level) { LEVEL_CALL(i3g::stokes_residual(c, level)); }
int i3g_stokes_smooth(i3g_ctx *c, int level, int nsweeps) { LEVEL_CALL(i3g::stokes_smooth(c, level, nsweeps)); }
int i3g_stokes_restrict(i3g_ctx *c, int level)
{
    if (c && level == 0) return set_error(c, I3G_E_ARG, "restriction targets a coarse level (>= 1)");
    LEVEL_CALL(i3g::stokes_restrict(c, level));
}
int i3g_stokes_prolong(i3g_ctx *c, int level)
{
    if (c && level == 0) return set_error(c, I3G_E_ARG, "prolongation starts from a coarse level (>= 1)");
    LEVEL_CALL(i3g::stokes_prolong(c, level));
}

int i3g_stokes_vcycles(i3g_ctx *c, int ncycles)
{
    if (!c || ncycles < 0) return I3G_E_ARG;
    const int mn = c->f.multinum > 0 ? (c->f.multinum < c->nlev - 1 ? c->f.multinum : c->nlev - 1) : c->nlev - 1;
    for (int i = 0; i < ncycles; i++) {
        int rc = i3g::stokes_vcycle(c, mn);
        if (rc) return rc;
    }
    I3G_CUDA(cudaStreamSynchronize(c->st));
    return 0;
}

int i3g_stokes_stresses(i3g_ctx *c)
{
    if (!c) return I3G_E_ARG;
    return i3g::stokes_stresses(c);
}

int i3g_stokes_relres(i3g_ctx *c, double *mom_rel, double *cont_rel)
{
    if (!c || !mom_rel || !cont_rel) return I3G_E_ARG;
    return i3g::stokes_relres(c, mom_rel, cont_rel);
}

int i3g_time_kernel(i3g_ctx *c, int kind, int reps, double *ms_per_launch, double *bytes_per_launch)
{
    if (!c || reps <= 0 || !ms_per_launch || !bytes_per_launch) return I3G_E_ARG;
    if (kind == 4 || kind == 5 || kind == 9) return i3g::markers_time_kernel(c, kind, reps, ms_per_launch, bytes_per_launch);
    if (kind == 6) return i3g::heat_time_kernel(c, reps, ms_per_launch, bytes_per_launch);
    return i3g::stokes_time_kernel(c, kind, reps, ms_per_launch, bytes_per_launch);
}

int i3g_stokes_guess_info(const i3g_ctx *c, int *used, double *rel_guess, double *rel_default, double *alpha)
{
    if (!c) return I3G_E_ARG;
    if (alpha) *alpha = c->guess_alpha;
    if (used) *used = c->guess_used;
    if (rel_guess) *rel_guess = c->guess_rel[0];
    if (rel_default) *rel_default = c->guess_rel[1];
    return 0;
}

int i3g_timer(i3g_ctx *c, int op, double *ms)
{
    if (!c) return I3G_E_ARG;
    if (!c->tev[0]) {
        I3G_CUDA(cudaEventCreate(&c->tev[0]));
        I3G_CUDA(cudaEventCreate(&c->tev[1]));
    }
    if (op == 0) {
        I3G_CUDA(cudaEventRecord(c->tev[0], c->st));
        return 0;
    }
    if (op != 1 || !ms) return I3G_E_ARG;
    I3G_CUDA(cudaEventRecord(c->tev[1], c->st));
    I3G_CUDA(cudaEventSynchronize(c->tev[1]));
    float t = 0;
    I3G_CUDA(cudaEventElapsedTime(&t, c->tev[0], c->tev[1]));
    *ms = t;
    return 0;
}

}  // extern "C"
