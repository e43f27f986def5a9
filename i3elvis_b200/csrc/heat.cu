// heat.cu -- implicit heat step (titerate, heat3mg.c:287-788) for sm_100a.
//
// The reference assembles the 7-point rows of heaterr (heat3mg.c:193-241) and relaxes only
// level 0 with point Gauss-Seidel (gausmatt, heat3mg.c:906-961).  Here the rows are applied
// matrix-free and solved by a geometric multigrid on the Stokes level hierarchy: red-black
// relaxation with the reference's damped update, node-centred weighted restriction of the
// residual, trilinear prolongation, and conductivity / heat capacity restricted with the
// viscosity-restriction weights.  The converged temperature is that of the reference's rows.
// FP64 arithmetic uses explicitly rounded operations in the reference's operand order.
#include <algorithm>
#include <cmath>
#include <vector>
#include "heat_markers.cuh"

namespace i3g {

struct HeatLevel {
    double *u = nullptr, *f = nullptr, *r = nullptr;
    float *kt = nullptr;            // level 0 points at the context's kt
    double *rocp = nullptr;
    double *dx = nullptr, *dy = nullptr, *dz = nullptr;   // raw spacings g[i]-g[i-1] (i >= 1)
    uint8_t *bc = nullptr;
    int nbc = 0;
    int *bnode = nullptr, *bpn = nullptr, *bdep = nullptr;
    double *bcc = nullptr, *bck = nullptr;     // flattened chain
    int *bon = nullptr;                        // original partner (residual)
    double *boc = nullptr, *bok = nullptr;
};

struct HeatState {
    HeatLevel L[I3G_MAXLEV];
    float *tk0 = nullptr, *tk1 = nullptr, *tk2 = nullptr;
    double *part = nullptr;
    bool ready = false;
};

static HeatState *hs(i3g_ctx *c) { return (HeatState *)c->heat; }

struct HView {
    int nx, ny, nz;
    long nxy;
    double *u, *f, *r;
    const float *kt;
    const double *rocp;
    const double *isx, *isy, *isz;    // 1/(g[i+1]-g[i-1])
    const double *dx, *dy, *dz;       // g[i]-g[i-1]
    const uint8_t *bc;
    double dt;
};

// diagonal and neighbour coefficients of the heat row at n (heaterr mode 1)
struct HRow { double d, c[6]; };

__device__ __forceinline__ double kflux(float ka, float kb, double xkf, double h)
{
    // (kt_a + kt_b)/2.0 * xkf / h, the FP32 sum first as in C
    return __ddiv_rn(__dmul_rn(__ddiv_rn((double)__fadd_rn(ka, kb), 2.0), xkf), h);
}

__device__ __forceinline__ HRow hrow(const HView &V, int i, int j, int k, long n)
{
    HRow R;
    const long NY = V.ny, NXY = V.nxy;
    const double xkf = __dmul_rn(2.0, V.isx[i]), ykf = __dmul_rn(2.0, V.isy[j]), zkf = __dmul_rn(2.0, V.isz[k]);
    const float kn = V.kt[n];
    double d = __ddiv_rn(V.rocp[n], V.dt), iv;
    iv = kflux(V.kt[n - NY], kn, xkf, V.dx[i]);     R.c[0] = -iv; d = __dadd_rn(d, iv);   // v1 (x-)
    iv = kflux(kn, V.kt[n + NY], xkf, V.dx[i + 1]); d = __dadd_rn(d, iv); R.c[1] = -iv;   // v5 (x+)
    iv = kflux(V.kt[n - 1], kn, ykf, V.dy[j]);      R.c[2] = -iv; d = __dadd_rn(d, iv);   // v2 (y-)
    iv = kflux(kn, V.kt[n + 1], ykf, V.dy[j + 1]);  d = __dadd_rn(d, iv); R.c[3] = -iv;   // v4 (y+)
    iv = kflux(V.kt[n - NXY], kn, zkf, V.dz[k]);    R.c[4] = -iv; d = __dadd_rn(d, iv);   // v0 (z-)
    iv = kflux(kn, V.kt[n + NXY], zkf, V.dz[k + 1]); d = __dadd_rn(d, iv); R.c[5] = -iv;  // v6 (z+)
    R.d = d;
    return R;
}

// slots in the reference's order: centre, x-, x+, y-, y+, z-, z+
template <bool RES>
__device__ __forceinline__ double hsum(const HView &V, const HRow &R, long n, double s)
{
    const long NY = V.ny, NXY = V.nxy;
    const double x[7] = {V.u[n], V.u[n - NY], V.u[n + NY], V.u[n - 1], V.u[n + 1], V.u[n - NXY], V.u[n + NXY]};
    const double a[7] = {R.d, R.c[0], R.c[1], R.c[2], R.c[3], R.c[4], R.c[5]};
    for (int q = 0; q < 7; q++) s = RES ? __dsub_rn(s, __dmul_rn(a[q], x[q])) : __dadd_rn(s, __dmul_rn(a[q], x[q]));
    return s;
}

__global__ void __launch_bounds__(256) k_heat_relax(HView V, int color, double koef)
{
    pdl_enter();
    const int hy = (V.ny + 1) >> 1;
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)hy * V.nx * V.nz) return;
    const int jh = (int)(t % hy);
    const long rest = t / hy;
    const int i = (int)(rest % V.nx), k = (int)(rest / V.nx);
    const int j = 2 * jh + ((i + k + color) & 1);
    if (j >= V.ny) return;
    const long n = (long)k * V.nxy + (long)i * V.ny + j;
    if (V.bc[n]) return;
    const HRow R = hrow(V, i, j, k, n);
    const double s = hsum<false>(V, R, n, -V.f[n]);
    V.u[n] = __dsub_rn(V.u[n], __dmul_rn(__ddiv_rn(s, R.d), koef));
}

__global__ void k_heat_residual(HView V)
{
    pdl_enter();
    const long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= V.nxy * V.nz) return;
    if (V.bc[n]) return;
    const int j = (int)(n % V.ny);
    const long rest = n / V.ny;
    const int i = (int)(rest % V.nx), k = (int)(rest / V.nx);
    const HRow R = hrow(V, i, j, k, n);
    V.r[n] = hsum<true>(V, R, n, V.f[n]);
}

__global__ void k_heat_bc(double *u, int n, const int *node, const int *pn, const int *dep, const double *cc,
                          const double *kk, int use_c)
{
    pdl_enter();
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    double v = pn[t] >= 0 ? u[pn[t]] : 0.0;
    for (int d = dep[t] - 1; d >= 0; d--)
        v = __dadd_rn(use_c ? cc[t * kMaxBcDepth + d] : 0.0, __dmul_rn(kk[t * kMaxBcDepth + d], v));
    u[node[t]] = v;
}

__global__ void k_heat_bc_res(const double *u, const double *f, double *r, int n, const int *node, const int *on, const double *ok)
{
    pdl_enter();
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int nd = node[t];
    double s = __dsub_rn(f[nd], __dmul_rn(1.0, u[nd]));
    if (on[t] >= 0) s = __dsub_rn(s, __dmul_rn(-ok[t], u[on[t]]));
    r[nd] = s;
}

struct TrV { const int *gptr, *gf; const double *gw; const int *a; const double *w0, *w1; };

// node-centred residual restriction, weight-normalised, boundary rows excluded
__global__ void k_heat_restrict(HView F, HView Cc, TrV tx, TrV ty, TrV tz)
{
    pdl_enter();
    const long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= Cc.nxy * Cc.nz) return;
    const int j = (int)(n % Cc.ny);
    const long rest = n / Cc.ny;
    const int i = (int)(rest % Cc.nx), k = (int)(rest / Cc.nx);
    Cc.u[n] = 0.0;
    if (Cc.bc[n]) { Cc.f[n] = 0.0; return; }
    double s = 0, ws = 0;
    for (int ez = tz.gptr[k]; ez < tz.gptr[k + 1]; ez++)
        for (int ex = tx.gptr[i]; ex < tx.gptr[i + 1]; ex++)
            for (int ey = ty.gptr[j]; ey < ty.gptr[j + 1]; ey++) {
                const long m = (long)tz.gf[ez] * F.nxy + (long)tx.gf[ex] * F.ny + ty.gf[ey];
                if (F.bc[m]) continue;
                const double w = __dmul_rn(__dmul_rn(tx.gw[ex], ty.gw[ey]), tz.gw[ez]);
                s = __dadd_rn(s, __dmul_rn(F.r[m], w));
                ws = __dadd_rn(ws, w);
            }
    Cc.f[n] = ws != 0 ? __ddiv_rn(s, ws) : 0.0;
}

__global__ void k_heat_prolong(HView F, HView Cc, TrV tx, TrV ty, TrV tz, double koef)
{
    pdl_enter();
    const long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= F.nxy * F.nz) return;
    const int j = (int)(n % F.ny);
    const long rest = n / F.ny;
    const int i = (int)(rest % F.nx), k = (int)(rest / F.nx);
    const int a = tx.a[i], b = ty.a[j], c = tz.a[k];
    const double wx[2] = {tx.w0[i], tx.w1[i]}, wy[2] = {ty.w0[j], ty.w1[j]}, wz[2] = {tz.w0[k], tz.w1[k]};
    double s = F.u[n];
    for (int dz = 0; dz < 2; dz++)
        for (int dx = 0; dx < 2; dx++)
            for (int dy = 0; dy < 2; dy++) {
                const long m = (long)(c + dz) * Cc.nxy + (long)(a + dx) * Cc.ny + (b + dy);
                s = __dadd_rn(s, __dmul_rn(__dmul_rn(Cc.u[m], __dmul_rn(__dmul_rn(wx[dx], wy[dy]), wz[dz])), koef));
            }
    F.u[n] = s;
}

// conductivity and volumetric heat capacity of a coarse level (volume weights)
__global__ void k_heat_coef_restrict(HView F, HView Cc, float *ktc, double *rocpc, TrV tx, TrV ty, TrV tz)
{
    pdl_enter();
    const long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= Cc.nxy * Cc.nz) return;
    const int j = (int)(n % Cc.ny);
    const long rest = n / Cc.ny;
    const int i = (int)(rest % Cc.nx), k = (int)(rest / Cc.nx);
    double sk = 0, sr = 0, ws = 0;
    for (int ez = tz.gptr[k]; ez < tz.gptr[k + 1]; ez++)
        for (int ex = tx.gptr[i]; ex < tx.gptr[i + 1]; ex++)
            for (int ey = ty.gptr[j]; ey < ty.gptr[j + 1]; ey++) {
                const long m = (long)tz.gf[ez] * F.nxy + (long)tx.gf[ex] * F.ny + ty.gf[ey];
                const double w = tx.gw[ex] * ty.gw[ey] * tz.gw[ez];
                sk += (double)F.kt[m] * w;
                sr += F.rocp[m] * w;
                ws += w;
            }
    ktc[n] = (float)(sk / ws);
    rocpc[n] = sr / ws;
}

// level-0 set-up: explicit heat-source right-hand side (heaterr mode 0, no adiabatic terms),
// rho*cp, old temperature; per-block maximum of |rate|
struct H0Args {
    int nx, ny, nz;
    const float *tk, *ro, *cp, *ht, *kt;
    const float *e[6], *s[6];
    const double *isx, *isy, *isz, *dx, *dy, *dz;
    const double *gy;
    double ysize, stp100;
    int frictyn;
    const uint8_t *bc;
    float *tk0, *tk1, *tk2;
    double *rocp, *u, *part;
};

__global__ void k_heat_setup0(H0Args a)
{
    pdl_enter();
    __shared__ double sh[8];
    const long NY = a.ny, NXY = (long)a.nx * a.ny, N = NXY * a.nz;
    double m = 0;
    for (long n = (long)blockIdx.x * blockDim.x + threadIdx.x; n < N; n += (long)gridDim.x * blockDim.x) {
        const float tkn = a.tk[n];
        a.tk0[n] = tkn; a.tk2[n] = tkn;
        a.u[n] = tkn;
        const float rocpf = __fmul_rn(a.ro[n], a.cp[n]);
        a.rocp[n] = rocpf;
        if (a.bc[n]) { a.tk1[n] = 0; continue; }
        const int j = (int)(n % NY);
        const long rest = n / NY;
        const int i = (int)(rest % a.nx), k = (int)(rest / a.nx);
        double iv = a.ht[n];
        if (a.frictyn && a.ro[n] > 2e+3 && a.gy[j] < a.ysize - a.stp100) {
            const double xkf = 2.0 * a.isx[i], ykf = 2.0 * a.isy[j], zkf = 2.0 * a.isz[k];
            const double x = a.dx[i] / 2.0 * xkf, y = a.dy[j] / 2.0 * ykf, z = a.dz[k] / 2.0 * zkf;
            const long p[8] = {n, n + 1, n + NY, n + NY + 1, n + NXY, n + NXY + 1, n + NXY + NY, n + NXY + NY + 1};
            const double w8[8] = {(1.0 - x) * (1.0 - y) * (1.0 - z), (1.0 - x) * (y) * (1.0 - z), (x) * (1.0 - y) * (1.0 - z),
                                  (x) * (y) * (1.0 - z), (1.0 - x) * (1.0 - y) * (z), (1.0 - x) * (y) * (z),
                                  (x) * (1.0 - y) * (z), (x) * (y) * (z)};
            double ev = 0;
            for (int q = 0; q < 8; q++)
                ev += w8[q] * (double)__fadd_rn(__fadd_rn(__fmul_rn(a.s[0][p[q]], a.e[0][p[q]]), __fmul_rn(a.s[1][p[q]], a.e[1][p[q]])),
                                                __fmul_rn(a.s[2][p[q]], a.e[2][p[q]]));
            ev += 2.0 * ((1.0 - z) * (double)__fmul_rn(a.s[3][n - NXY], a.e[3][n - NXY]) + z * (double)__fmul_rn(a.s[3][n], a.e[3][n]));
            ev += 2.0 * ((1.0 - y) * (double)__fmul_rn(a.s[4][n - 1], a.e[4][n - 1]) + y * (double)__fmul_rn(a.s[4][n], a.e[4][n]));
            ev += 2.0 * ((1.0 - x) * (double)__fmul_rn(a.s[5][n - NY], a.e[5][n - NY]) + x * (double)__fmul_rn(a.s[5][n], a.e[5][n]));
            iv += ev;
        }
        a.tk1[n] = (float)iv;
        m = fmax(m, fabs(iv / (double)rocpf));
    }
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); w++) m = fmax(m, sh[w]);
        a.part[blockIdx.x] = m;
    }
}

// per substep: old temperature, solution start and level-0 right-hand side
__global__ void k_heat_substep0(long N, const float *tk, float *tk0, const float *tk1, const double *rocp, const uint8_t *bc,
                                double *u, double *f, double dt)
{
    pdl_enter();
    const long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    const float t = tk[n];
    tk0[n] = t;
    u[n] = t;
    if (!bc[n]) f[n] = __dadd_rn((double)tk1[n], __dmul_rn(__ddiv_rn((double)t, dt), rocp[n]));
}

// level-0 boundary constants (tbonderr, heat3mg.c:817-824)
__global__ void k_bc_rhs_heat(double *f, int n, const int *node, const double *oc)
{
    pdl_enter();
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) f[node[t]] = oc[t];
}

__global__ void k_heat_store(long N, const double *u, float *tk)
{
    pdl_enter();
    const long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n < N) tk[n] = (float)u[n];
}

__global__ void k_heat_norm_part(HView V, double *part)
{
    pdl_enter();
    __shared__ double sh[2][8];
    double q[2] = {0, 0};
    const long N = V.nxy * V.nz;
    for (long n = (long)blockIdx.x * blockDim.x + threadIdx.x; n < N; n += (long)gridDim.x * blockDim.x) {
        if (V.bc[n]) continue;
        const int j = (int)(n % V.ny);
        const long rest = n / V.ny;
        const int i = (int)(rest % V.nx), k = (int)(rest / V.nx);
        const HRow R = hrow(V, i, j, k, n);
        const double r = hsum<true>(V, R, n, V.f[n]);
        q[0] += r * r;
        q[1] += V.f[n] * V.f[n];
    }
    for (int a = 0; a < 2; a++) {
        double v = q[a];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0) sh[a][threadIdx.x >> 5] = v;
    }
    __syncthreads();
    if (threadIdx.x < 2) {
        double v = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) v += sh[threadIdx.x][w];
        part[blockIdx.x * 2 + threadIdx.x] = v;
    }
}

// ------------------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------------------
static inline unsigned nb(long n, int t = 256) { return (unsigned)((n + t - 1) / t); }

#define LAUNCH(kern, grid, block, ...)                                                     \
    do {                                                                                   \
        launch_pdl(c->st, kern, dim3(grid), dim3(block), __VA_ARGS__);                     \
        c->launches++;                                                                     \
    } while (0)

template <typename T>
static int up(i3g_ctx *c, T *&d, const std::vector<T> &h)
{
    I3G_CUDA(cudaMalloc((void **)&d, sizeof(T) * std::max<size_t>(h.size(), 1)));
    if (!h.empty()) I3G_CUDA(cudaMemcpyAsync(d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice, c->st));
    return 0;
}

static TrV trv(const Transfer1D &t) { return TrV{t.gptr, t.gf, t.gw, t.a, t.w0, t.w1}; }

static HView hview(i3g_ctx *c, int l, double dt)
{
    Level &L = c->lev[l];
    HeatLevel &H = hs(c)->L[l];
    HView V;
    V.nx = L.nx; V.ny = L.ny; V.nz = L.nz; V.nxy = (long)L.nx * L.ny;
    V.u = H.u; V.f = H.f; V.r = H.r; V.kt = l == 0 ? c->kt : H.kt; V.rocp = H.rocp;
    V.isx = L.d.ix[1]; V.isy = L.d.iy[1]; V.isz = L.d.iz[1];
    V.dx = H.dx; V.dy = H.dy; V.dz = H.dz;
    V.bc = H.bc;
    V.dt = dt;
    return V;
}

int heat_alloc(i3g_ctx *c)
{
    HeatState *S = new HeatState();
    c->heat = S;
    const long N0 = c->nodenum;
    long mgp[I3G_MAXLEV], ntot = 0;
    for (int l = 0; l < c->nlev; l++) { mgp[l] = ntot; ntot += c->lev[l].n; }
    // temperature rows: bondm[8*nodenum + node] with node counting all levels
    std::vector<int> rid(ntot, -1);
    for (long b = 0; b < c->m.bondnum; b++) {
        const long row = c->m.bond_row[b];
        if (row >= 8 * N0 && row - 8 * N0 < ntot) rid[row - 8 * N0] = (int)b;
    }
    for (int l = 0; l < c->nlev; l++) {
        Level &L = c->lev[l];
        HeatLevel &H = S->L[l];
        I3G_CUDA(cudaMalloc((void **)&H.u, sizeof(double) * L.n));
        I3G_CUDA(cudaMalloc((void **)&H.f, sizeof(double) * L.n));
        I3G_CUDA(cudaMalloc((void **)&H.r, sizeof(double) * L.n));
        I3G_CUDA(cudaMemsetAsync(H.r, 0, sizeof(double) * L.n, c->st));
        I3G_CUDA(cudaMemsetAsync(H.f, 0, sizeof(double) * L.n, c->st));
        I3G_CUDA(cudaMalloc((void **)&H.rocp, sizeof(double) * L.n));
        if (l > 0) I3G_CUDA(cudaMalloc((void **)&H.kt, sizeof(float) * L.n));
        const double *g[3] = {L.gx, L.gy, L.gz};
        const int nn[3] = {L.nx, L.ny, L.nz};
        double **dd[3] = {&H.dx, &H.dy, &H.dz};
        for (int d = 0; d < 3; d++) {
            std::vector<double> h(nn[d] + 1, 0.0);
            for (int i = 1; i < nn[d]; i++) h[i] = g[d][i] - g[d][i - 1];
            int rc = up(c, *dd[d], h);
            if (rc) return rc;
        }
        std::vector<uint8_t> mask(L.n, 0);
        std::vector<int> bn, bp, bdp, bon;
        std::vector<double> bcc, bck, boc, bok;
        for (long q = 0; q < L.n; q++) {
            const int b = rid[mgp[l] + q];
            const int j = (int)(q % L.ny), i = (int)((q / L.ny) % L.nx), k = (int)(q / ((long)L.ny * L.nx));
            if (b < 0) {
                if (i < 1 || i > L.nx - 2 || j < 1 || j > L.ny - 2 || k < 1 || k > L.nz - 2)
                    return set_error(c, I3G_E_BC, "level %d: temperature row at (%d,%d,%d) has no boundary condition but its stencil leaves the grid", l, i, j, k);
                continue;
            }
            mask[q] = 1;
            bn.push_back((int)q);
            const long p1 = c->m.bond_partner1[b];
            bon.push_back(p1 > 0 ? (int)(p1 - 1 - mgp[l]) : -1);
            boc.push_back(c->m.bond_c[b]);
            bok.push_back(c->m.bond_k[b]);
            double chc[kMaxBcDepth], chk[kMaxBcDepth];
            int dep = 0, pn = -1;
            long cur = mgp[l] + q;
            for (;;) {
                const int bb = rid[cur];
                if (dep >= kMaxBcDepth) return set_error(c, I3G_E_BC, "temperature boundary chain too long (cycle?)");
                chc[dep] = c->m.bond_c[bb];
                const long q1 = c->m.bond_partner1[bb];
                chk[dep] = q1 > 0 ? (double)c->m.bond_k[bb] : 0.0;
                dep++;
                if (q1 <= 0) break;
                const long pr = q1 - 1;
                if (pr < mgp[l] || pr >= mgp[l] + L.n) return set_error(c, I3G_E_BC, "temperature boundary partner on another level");
                if (rid[pr] < 0) { pn = (int)(pr - mgp[l]); break; }
                cur = pr;
            }
            bp.push_back(pn);
            bdp.push_back(dep);
            for (int d = 0; d < kMaxBcDepth; d++) { bcc.push_back(d < dep ? chc[d] : 0.0); bck.push_back(d < dep ? chk[d] : 0.0); }
        }
        H.nbc = (int)bn.size();
        int rc;
        if ((rc = up(c, H.bc, mask)) || (rc = up(c, H.bnode, bn)) || (rc = up(c, H.bpn, bp)) || (rc = up(c, H.bdep, bdp)) ||
            (rc = up(c, H.bcc, bcc)) || (rc = up(c, H.bck, bck)) || (rc = up(c, H.bon, bon)) || (rc = up(c, H.boc, boc)) ||
            (rc = up(c, H.bok, bok)))
            return rc;
    }
    I3G_CUDA(cudaMalloc((void **)&S->tk0, sizeof(float) * N0));
    I3G_CUDA(cudaMalloc((void **)&S->tk1, sizeof(float) * N0));
    I3G_CUDA(cudaMalloc((void **)&S->tk2, sizeof(float) * N0));
    I3G_CUDA(cudaMalloc((void **)&S->part, sizeof(double) * 2 * (c->red_blocks + 8)));
    I3G_CUDA(cudaStreamSynchronize(c->st));
    return 0;
}

void heat_free(i3g_ctx *c)
{
    HeatState *S = hs(c);
    if (!S) return;
    for (int l = 0; l < c->nlev; l++) {
        HeatLevel &H = S->L[l];
        void *p[] = {H.u, H.f, H.r, H.rocp, H.dx, H.dy, H.dz, H.bc, H.bnode, H.bpn, H.bdep, H.bcc, H.bck, H.bon, H.boc, H.bok};
        for (void *q : p) cudaFree(q);
        if (l > 0) cudaFree(H.kt);
    }
    cudaFree(S->tk0); cudaFree(S->tk1); cudaFree(S->tk2); cudaFree(S->part);
    delete S;
    c->heat = nullptr;
}

static void hbc(i3g_ctx *c, int l, bool use_c)
{
    HeatLevel &H = hs(c)->L[l];
    if (H.nbc) LAUNCH(k_heat_bc, nb(H.nbc), 256, H.u, H.nbc, (const int *)H.bnode, (const int *)H.bpn, (const int *)H.bdep,
                      (const double *)H.bcc, (const double *)H.bck, (int)use_c);
}

static void hsmooth(i3g_ctx *c, int l, int n, double dt, bool res)
{
    Level &L = c->lev[l];
    HView V = hview(c, l, dt);
    const long tot = (long)((L.ny + 1) / 2) * L.nx * L.nz;
    for (int s = 0; s < n; s++) {
        LAUNCH(k_heat_relax, nb(tot), 256, V, 0, c->p.t0koef);
        LAUNCH(k_heat_relax, nb(tot), 256, V, 1, c->p.t0koef);
        hbc(c, l, l == 0);
    }
    if (res) {
        LAUNCH(k_heat_residual, nb(L.n), 256, V);
        HeatLevel &H = hs(c)->L[l];
        if (H.nbc) LAUNCH(k_heat_bc_res, nb(H.nbc), 256, (const double *)H.u, (const double *)H.f, H.r, H.nbc,
                          (const int *)H.bnode, (const int *)H.bon, (const double *)H.bok);
    }
}

static void hvcycle(i3g_ctx *c, double dt)
{
    const int L = c->nlev - 1;
    for (int l = 0; l < L; l++) {
        hsmooth(c, l, 2, dt, true);
        Level &F = c->lev[l];
        LAUNCH(k_heat_restrict, nb(c->lev[l + 1].n), 256, hview(c, l, dt), hview(c, l + 1, dt), trv(F.tr[0][kStagLine]),
               trv(F.tr[1][kStagLine]), trv(F.tr[2][kStagLine]));
    }
    hsmooth(c, L, 16, dt, false);
    for (int l = L; l > 0; l--) {
        Level &F = c->lev[l - 1];
        LAUNCH(k_heat_prolong, nb(F.n), 256, hview(c, l - 1, dt), hview(c, l, dt), trv(F.tr[0][kStagLine]),
               trv(F.tr[1][kStagLine]), trv(F.tr[2][kStagLine]), 1.0);
        hsmooth(c, l - 1, 2, dt, false);
    }
}

static int hrelres(i3g_ctx *c, double dt, double *rel)
{
    HeatState *S = hs(c);
    LAUNCH(k_heat_norm_part, c->red_blocks, 256, hview(c, 0, dt), S->part);
    I3G_CUDA(cudaMemcpyAsync(c->hstage, S->part, sizeof(double) * 2 * c->red_blocks, cudaMemcpyDeviceToHost, c->st));
    I3G_CUDA(cudaStreamSynchronize(c->st));
    double rr = 0, bb = 0;
    for (int b = 0; b < c->red_blocks; b++) { rr += c->hstage[2 * b]; bb += c->hstage[2 * b + 1]; }
    *rel = bb > 0 ? std::sqrt(rr / bb) : std::sqrt(rr);
    return 0;
}

int heat_solve(i3g_ctx *c, double *timestep)
{
    HeatState *S = hs(c);
    if (c->p.adiabyn) return set_error(c, I3G_E_UNSUPPORTED, "adiabatic heating (adiabyn %d) is not supported on the GPU", c->p.adiabyn);
    if (c->m.timesum > c->p.timebeg)
        return set_error(c, I3G_E_UNSUPPORTED, "the bottom-temperature schedule (timebeg, heat3mg.c:433-446) is not supported");
    EventPair ev;
    I3G_CUDA(ev.create());
    cudaEvent_t e0 = ev.a, e1 = ev.b;
    I3G_CUDA(cudaEventRecord(e0, c->st));
    Level &L0 = c->lev[0];
    HeatLevel &H0 = S->L[0];
    H0Args a;
    a.nx = L0.nx; a.ny = L0.ny; a.nz = L0.nz;
    a.tk = c->tk; a.ro = c->ro; a.cp = c->cp; a.ht = c->ht; a.kt = c->kt;
    for (int q = 0; q < 6; q++) { a.e[q] = c->eps[q]; a.s[q] = c->sig[q]; }
    a.isx = L0.d.ix[1]; a.isy = L0.d.iy[1]; a.isz = L0.d.iz[1];
    a.dx = H0.dx; a.dy = H0.dy; a.dz = H0.dz;
    a.gy = c->gy0; a.ysize = c->m.ysize; a.stp100 = c->p.stp100; a.frictyn = c->p.frictyn;
    a.bc = H0.bc;
    a.tk0 = S->tk0; a.tk1 = S->tk1; a.tk2 = S->tk2; a.rocp = H0.rocp; a.u = H0.u; a.part = S->part;
    LAUNCH(k_heat_setup0, c->red_blocks, 256, a);
    I3G_CUDA(cudaMemcpyAsync(c->hstage, S->part, sizeof(double) * c->red_blocks, cudaMemcpyDeviceToHost, c->st));
    // coarse-level coefficients
    for (int l = 1; l < c->nlev; l++) {
        Level &F = c->lev[l - 1];
        LAUNCH(k_heat_coef_restrict, nb(c->lev[l].n), 256, hview(c, l - 1, 1.0), hview(c, l, 1.0), S->L[l].kt, S->L[l].rocp,
               trv(F.tr[0][kStagAbs]), trv(F.tr[1][kStagAbs]), trv(F.tr[2][kStagAbs]));
    }
    I3G_CUDA(cudaStreamSynchronize(c->st));
    double maxrate = 0;
    for (int b = 0; b < c->red_blocks; b++) maxrate = std::max(maxrate, c->hstage[b]);
    double tkstep = 1e30;
    if (maxrate > 0) tkstep = c->f.maxtkstep / maxrate;
    if (*timestep == 0 || tkstep == 0) return 0;
    const double total = *timestep;
    double done = 0, rel = 0;
    const double rtol = c->p.heat_rtol > 0 ? c->p.heat_rtol : 1e-10;
    const int maxc = c->p.heat_maxcyc > 0 ? c->p.heat_maxcyc : 2000;
    int cycles = 0, subs = 0;
    do {
        double dt = std::min(total, tkstep);
        if (dt > total - done) dt = total - done;
        LAUNCH(k_heat_substep0, nb(L0.n), 256, L0.n, (const float *)c->tk, S->tk0, (const float *)S->tk1,
               (const double *)H0.rocp, (const uint8_t *)H0.bc, H0.u, H0.f, dt);
        if (H0.nbc) LAUNCH(k_bc_rhs_heat, nb(H0.nbc), 256, H0.f, H0.nbc, (const int *)H0.bnode, (const double *)H0.boc);
        hbc(c, 0, true);
        int it = 0;
        for (;;) {
            hvcycle(c, dt);
            it++;
            int rc = hrelres(c, dt, &rel);
            if (rc) return rc;
            if (!(rel == rel)) return set_error(c, I3G_E_NAN, "NaN in the heat solve");
            if (rel <= rtol || it >= maxc) break;
        }
        cycles += it;
        LAUNCH(k_heat_store, nb(L0.n), 256, L0.n, (const double *)H0.u, c->tk);
        if (rel > rtol) return set_error(c, I3G_E_NOCONV, "heat: %d V-cycles without reaching %g (%g)", it, rtol, rel);
        done += dt;
        subs++;
    } while (done < total);
    c->st_.heat_cycles = cycles;
    c->st_.heat_substeps = subs;
    c->st_.heat_rel = rel;
    int rc = markers_heat_update(c, total, S->tk0, S->tk1, S->tk2);
    if (rc) return rc;
    I3G_CUDA(cudaEventRecord(e1, c->st));
    I3G_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    c->st_.ms_heat = ms;
    S->ready = true;
    return 0;
}

int heat_get_solution(i3g_ctx *c, void *dst, int64_t nbytes)
{
    if (nbytes != c->nodenum * 8) return set_error(c, I3G_E_ARG, "size mismatch");
    I3G_CUDA(cudaMemcpyAsync(dst, hs(c)->L[0].u, nbytes, cudaMemcpyDeviceToHost, c->st));
    I3G_CUDA(cudaStreamSynchronize(c->st));
    return 0;
}

int heat_time_kernel(i3g_ctx *c, int reps, double *ms, double *bytes)
{
    Level &L0 = c->lev[0];
    HView V = hview(c, 0, 1e13);
    const long tot = (long)((L0.ny + 1) / 2) * L0.nx * L0.nz;
    // one full sweep (both colours) with an empty L2; 32 B per node: T read and written (FP64),
    // k and rho cp (FP32), right-hand side (FP64)
    int rc = cold_time(c, reps, [&]() -> int {
        LAUNCH(k_heat_relax, nb(tot), 256, V, 0, 1.0);
        LAUNCH(k_heat_relax, nb(tot), 256, V, 1, 1.0);
        return 0;
    }, ms);
    if (rc) return rc;
    *bytes = (double)L0.n * 32.0;
    return 0;
}

}  // namespace i3g
