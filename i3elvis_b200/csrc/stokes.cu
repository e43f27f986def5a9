// stokes.cu -- staggered-grid variable-viscosity Stokes multigrid for sm_100a.
//
// Replaces vpiterate (move3mg.c:1585-2636).  The reference assembles every row into a
// 57-slot CSR store (gausmat2, gaus3mg.c:67-127; 684 B/node of matrix traffic per sweep)
// and relaxes it lexicographically.  Here the rows are never stored: each kernel rebuilds
// a row's 17 coefficients from the four stress-point viscosity arrays and the 1-D grid
// tables, and the relaxation runs in multicolour order (red/black per velocity component,
// then all pressure rows), which parallelises without the data race of the reference's
// OpenMP sweep (move3mg.c:3089-3130).
//
// FP64 arithmetic uses explicitly rounded operations in the reference's operand order, so
// rows, residuals and relaxation updates agree bit for bit with the CPU oracle.  The FP32
// path (mixed precision) uses the same stencil code on viscosity and geometry scaled to O(1).
//
// Solve drivers (stokes_solve): the reference's FP64 V-cycle iteration; FP32 V-cycles inside
// FP64 defect correction; or FGMRES(m) (i3g_params.krylov) with the FP32 V-cycle as the
// preconditioner and fused Gram-Schmidt kernels (k_kr_proj).  The FP32 smoother's pressure
// update of weak cells enclosed by stiff material is scaled by their faces' viscosity
// (k_nd_schur).  The start is the previous solution, its linear or quadratic extrapolation
// (k_extrapolate3), or a staged learned correction, whichever has the smaller residual.  An
// iteration (and each FGMRES step index) is captured as a CUDA graph and replayed, captured
// again only when the level count, the precision or the relaxation factors change.
#include <algorithm>
#include <type_traits>
#include <cmath>
#include <cstring>
#include <utility>
#include <vector>
#include "i3g_internal.cuh"

namespace i3g {

// ------------------------------------------------------------------------------------
// arithmetic policies
// ------------------------------------------------------------------------------------
template <typename T>
struct Ar;
template <>
struct Ar<double> {
    static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
    static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
    static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
    static __device__ __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }
};
template <>
struct Ar<float> {
    static __device__ __forceinline__ float mul(float a, float b) { return a * b; }
    static __device__ __forceinline__ float add(float a, float b) { return a + b; }
    static __device__ __forceinline__ float sub(float a, float b) { return a - b; }
    static __device__ __forceinline__ float div(float a, float b) { return a / b; }
};

// floor(n / d) for 0 <= n < 2^31 by one multiply-high and a shift (Granlund and Montgomery,
// "Division by invariant integers using multiplication", PLDI 1994, Theorem 4.2 with N = 31):
// l = ceil(log2 d), m = ceil(2^(31+l) / d) < 2^32, q = umulhi(n, m) >> (l - 1); d = 1: m = 0.
struct FastDiv {
    unsigned m = 0, s = 0;
    static FastDiv of(unsigned d)
    {
        FastDiv f;
        if (d <= 1) return f;
        const unsigned l = 32u - (unsigned)__builtin_clz(d - 1u);
        f.m = (unsigned)((((unsigned long long)1 << (31 + l)) + d - 1) / d);
        f.s = l - 1;
        return f;
    }
    __device__ __forceinline__ unsigned div(unsigned n) const { return m ? __umulhi(n, m) >> s : n; }
};

// Level view passed by value to kernels.
template <typename T>
struct View {
    int nx, ny, nz;
    long nxy;
    FastDiv dnx, dny, dhy;          // division by nx, ny and (ny + 1) / 2 for index decomposition
    const uint8_t *bc;
    T *u0, *u1, *u2, *u3;
    T *f0, *f1, *f2, *f3;
    T *r0, *r1, *r2, *r3;
    const T *etac, *etaxy, *etaxz, *etayz;
    const T *icx, *isx, *icy, *isy, *icz, *isz;
    const float *nd;
};

// (i, j, k) of node n = (k * nx + i) * ny + j of a level (n < 2^31)
template <typename T>
__device__ __forceinline__ void node_ijk(const View<T> &L, long n, int &i, int &j, int &k)
{
    const unsigned u = (unsigned)n;
    const unsigned r = L.dny.div(u);
    j = (int)(u - r * (unsigned)L.ny);
    const unsigned q = L.dnx.div(r);
    i = (int)(r - q * (unsigned)L.nx);
    k = (int)q;
}

template <typename T>
static View<T> view(Level &L, Fields<T> &F)
{
    View<T> v;
    v.nx = L.nx; v.ny = L.ny; v.nz = L.nz; v.nxy = (long)L.nx * L.ny;
    v.dnx = FastDiv::of((unsigned)L.nx); v.dny = FastDiv::of((unsigned)L.ny); v.dhy = FastDiv::of((unsigned)((L.ny + 1) / 2));
    v.bc = L.bc;
    v.u0 = F.u[0]; v.u1 = F.u[1]; v.u2 = F.u[2]; v.u3 = F.u[3];
    v.f0 = F.f[0]; v.f1 = F.f[1]; v.f2 = F.f[2]; v.f3 = F.f[3];
    v.r0 = F.r[0]; v.r1 = F.r[1]; v.r2 = F.r[2]; v.r3 = F.r[3];
    v.etac = F.etac; v.etaxy = F.etaxy; v.etaxz = F.etaxz; v.etayz = F.etayz;
    v.icx = F.ix[0]; v.isx = F.ix[1]; v.icy = F.iy[0]; v.isy = F.iy[1]; v.icz = F.iz[0]; v.isz = F.iz[1];
    v.nd = F.nd;
    return v;
}

// row existence (vpiterate loop guards, move3mg.c:2057-2141)
__host__ __device__ __forceinline__ bool row_exists(int v, int i, int j, int k, int nx, int ny, int nz)
{
    switch (v) {
    case 0: return i > 0 && j > 0 && k > 0;
    case 1: return j < ny - 1 && k < nz - 1;
    case 2: return i < nx - 1 && k < nz - 1;
    default: return i < nx - 1 && j < ny - 1;
    }
}

// accumulate one slot: smoother form s += c*x (starting from -f), residual form s -= c*x
template <typename T, bool RES>
__device__ __forceinline__ void acc(T &s, T c, T x)
{
    if (RES) s = Ar<T>::sub(s, Ar<T>::mul(c, x));
    else s = Ar<T>::add(s, Ar<T>::mul(c, x));
}

template <typename T>
__device__ __forceinline__ T cf(T a, T n, T k)   // ((a*n)*2)*k: -ynval*nueff*2.0*dk
{
    return Ar<T>::mul(Ar<T>::mul(Ar<T>::mul(a, n), T(2)), k);
}

// x-momentum row at node n = (i,j,k) (xstokserr, move3mg.c:718-903): accumulates the 17
// slots in the reference's order into s and returns the diagonal.
template <typename T, bool RES>
__device__ __forceinline__ T xrow(const View<T> &L, int i, int j, int k, long n, T &s)
{
    using A = Ar<T>;
    const long NY = L.ny, NXY = L.nxy;
    const T XK = A::mul(T(2), L.isx[i]), YK = L.icy[j + 1], ZK = L.icz[k + 1];
    const T cA = cf(XK, L.etac[n + NXY + 1], L.icx[i]);
    const T cB = cf(XK, L.etac[n + NXY + NY + 1], L.icx[i + 1]);
    const T nS = L.etaxy[n], nN = L.etaxy[n + 1], xkS = L.isx[i];
    const T cSy = cf(YK, nS, L.isy[j]), cSx = cf(YK, nS, xkS);
    const T cNy = cf(YK, nN, L.isy[j + 1]), cNx = cf(YK, nN, xkS);
    const T nF = L.etaxz[n], nK = L.etaxz[n + NXY];
    const T cFz = cf(ZK, nF, L.isz[k]), cFx = cf(ZK, nF, xkS);
    const T cKz = cf(ZK, nK, L.isz[k + 1]), cKx = cf(ZK, nK, xkS);
    T d = -cA;
    d = A::add(d, -cB); d = A::add(d, -cSy); d = A::add(d, -cNy); d = A::add(d, -cFz); d = A::add(d, -cKz);
    const T *vx = L.u1, *vy = L.u2, *vz = L.u3, *p = L.u0;
    acc<T, RES>(s, d, vx[n]);
    acc<T, RES>(s, cA, vx[n - NY]);
    acc<T, RES>(s, cB, vx[n + NY]);
    acc<T, RES>(s, cSy, vx[n - 1]);
    acc<T, RES>(s, cNy, vx[n + 1]);
    acc<T, RES>(s, cFz, vx[n - NXY]);
    acc<T, RES>(s, cKz, vx[n + NXY]);
    acc<T, RES>(s, cSx, vy[n - NY]);
    acc<T, RES>(s, -cNx, vy[n - NY + 1]);
    acc<T, RES>(s, -cSx, vy[n]);
    acc<T, RES>(s, cNx, vy[n + 1]);
    acc<T, RES>(s, cFx, vz[n - NY]);
    acc<T, RES>(s, -cKx, vz[n - NY + NXY]);
    acc<T, RES>(s, -cFx, vz[n]);
    acc<T, RES>(s, cKx, vz[n + NXY]);
    acc<T, RES>(s, XK, p[n + NXY + 1]);
    acc<T, RES>(s, -XK, p[n + NXY + NY + 1]);
    return d;
}

// y-momentum row (ystokserr, move3mg.c:910-1101)
template <typename T, bool RES>
__device__ __forceinline__ T yrow(const View<T> &L, int i, int j, int k, long n, T &s)
{
    using A = Ar<T>;
    const long NY = L.ny, NXY = L.nxy;
    const T XK = L.icx[i + 1], YK = A::mul(T(2), L.isy[j]), ZK = L.icz[k + 1];
    const T cA = cf(YK, L.etac[n + NY + NXY], L.icy[j]);
    const T cB = cf(YK, L.etac[n + NY + 1 + NXY], L.icy[j + 1]);
    const T nW = L.etaxy[n], nE = L.etaxy[n + NY], ykW = L.isy[j];
    const T cWy = cf(XK, nW, ykW), cWx = cf(XK, nW, L.isx[i]);
    const T cEy = cf(XK, nE, ykW), cEx = cf(XK, nE, L.isx[i + 1]);
    const T nF = L.etayz[n], nK = L.etayz[n + NXY];
    const T cFz = cf(ZK, nF, L.isz[k]), cFy = cf(ZK, nF, ykW);
    const T cKz = cf(ZK, nK, L.isz[k + 1]), cKy = cf(ZK, nK, ykW);
    T d = -cA;
    d = A::add(d, -cB); d = A::add(d, -cWx); d = A::add(d, -cEx); d = A::add(d, -cFz); d = A::add(d, -cKz);
    const T *vx = L.u1, *vy = L.u2, *vz = L.u3, *p = L.u0;
    acc<T, RES>(s, d, vy[n]);
    acc<T, RES>(s, cWx, vy[n - NY]);
    acc<T, RES>(s, cEx, vy[n + NY]);
    acc<T, RES>(s, cA, vy[n - 1]);
    acc<T, RES>(s, cB, vy[n + 1]);
    acc<T, RES>(s, cFz, vy[n - NXY]);
    acc<T, RES>(s, cKz, vy[n + NXY]);
    acc<T, RES>(s, cWy, vx[n - 1]);
    acc<T, RES>(s, -cWy, vx[n]);
    acc<T, RES>(s, -cEy, vx[n + NY - 1]);
    acc<T, RES>(s, cEy, vx[n + NY]);
    acc<T, RES>(s, cFy, vz[n - 1]);
    acc<T, RES>(s, -cFy, vz[n]);
    acc<T, RES>(s, -cKy, vz[n - 1 + NXY]);
    acc<T, RES>(s, cKy, vz[n + NXY]);
    acc<T, RES>(s, YK, p[n + NY + NXY]);
    acc<T, RES>(s, -YK, p[n + NY + 1 + NXY]);
    return d;
}

// z-momentum row (zstokserr, move3mg.c:1109-1301)
template <typename T, bool RES>
__device__ __forceinline__ T zrow(const View<T> &L, int i, int j, int k, long n, T &s)
{
    using A = Ar<T>;
    const long NY = L.ny, NXY = L.nxy;
    const T XK = L.icx[i + 1], YK = L.icy[j + 1], ZK = A::mul(T(2), L.isz[k]);
    const T cA = cf(ZK, L.etac[n + NY + 1], L.icz[k]);
    const T cB = cf(ZK, L.etac[n + NY + 1 + NXY], L.icz[k + 1]);
    const T nW = L.etaxz[n], nE = L.etaxz[n + NY], zkW = L.isz[k];
    const T cWz = cf(XK, nW, zkW), cWx = cf(XK, nW, L.isx[i]);
    const T cEz = cf(XK, nE, zkW), cEx = cf(XK, nE, L.isx[i + 1]);
    const T nS = L.etayz[n], nN = L.etayz[n + 1];
    const T cSz = cf(YK, nS, zkW), cSy = cf(YK, nS, L.isy[j]);
    const T cNz = cf(YK, nN, zkW), cNy = cf(YK, nN, L.isy[j + 1]);
    T d = -cA;
    d = A::add(d, -cB); d = A::add(d, -cWx); d = A::add(d, -cEx); d = A::add(d, -cSy); d = A::add(d, -cNy);
    const T *vx = L.u1, *vy = L.u2, *vz = L.u3, *p = L.u0;
    acc<T, RES>(s, d, vz[n]);
    acc<T, RES>(s, cWx, vz[n - NY]);
    acc<T, RES>(s, cEx, vz[n + NY]);
    acc<T, RES>(s, cSy, vz[n - 1]);
    acc<T, RES>(s, cNy, vz[n + 1]);
    acc<T, RES>(s, cA, vz[n - NXY]);
    acc<T, RES>(s, cB, vz[n + NXY]);
    acc<T, RES>(s, cSz, vy[n - NXY]);
    acc<T, RES>(s, -cNz, vy[n + 1 - NXY]);
    acc<T, RES>(s, -cSz, vy[n]);
    acc<T, RES>(s, cNz, vy[n + 1]);
    acc<T, RES>(s, cWz, vx[n - NXY]);
    acc<T, RES>(s, -cWz, vx[n]);
    acc<T, RES>(s, -cEz, vx[n + NY - NXY]);
    acc<T, RES>(s, cEz, vx[n + NY]);
    acc<T, RES>(s, ZK, p[n + NY + 1]);
    acc<T, RES>(s, -ZK, p[n + NY + 1 + NXY]);
    return d;
}

// continuity row of the cell with upper corner n = (i,j,k) (continerr, move3mg.c:1310-1425)
template <typename T, bool RES>
__device__ __forceinline__ void crow(const View<T> &L, int i, int j, int k, long n, T &s)
{
    const long NY = L.ny, NXY = L.nxy;
    const long v0 = n - NXY - NY - 1;
    const T xk = L.icx[i], yk = L.icy[j], zk = L.icz[k];
    acc<T, RES>(s, -xk, L.u1[v0]);
    acc<T, RES>(s, xk, L.u1[v0 + NY]);
    acc<T, RES>(s, -yk, L.u2[v0]);
    acc<T, RES>(s, yk, L.u2[v0 + 1]);
    acc<T, RES>(s, -zk, L.u3[v0]);
    acc<T, RES>(s, zk, L.u3[v0 + NXY]);
}

// ------------------------------------------------------------------------------------
// relaxation kernels
// ------------------------------------------------------------------------------------
// One colour of one velocity component: thread t handles the row of colour `color` in the
// y-pair (2*jh, 2*jh+1) of line (i,k), so a warp covers 64 consecutive y.
// Node of thread t's row of colour `color` (the y-pair (2*jh, 2*jh+1) of line (i,k)); -1 when
// the row does not exist.
template <int V, typename T>
__device__ __forceinline__ long vel_row_node(const View<T> &L, long t, int color, int &i, int &j, int &k)
{
    const unsigned hy = (unsigned)((L.ny + 1) >> 1), u = (unsigned)t;
    const unsigned rest = L.dhy.div(u);
    const int jh = (int)(u - rest * hy);
    const unsigned q = L.dnx.div(rest);
    i = (int)(rest - q * (unsigned)L.nx); k = (int)q;
    j = 2 * jh + ((i + k + color) & 1);
    if (j >= L.ny || !row_exists(V, i, j, k, L.nx, L.ny, L.nz)) return -1;
    return (long)k * L.nxy + (long)i * L.ny + j;
}

// the relaxation update of velocity row n; returns the new value
template <typename T, int V>
__device__ __forceinline__ T relax_vel_row(const View<T> &L, int i, int j, int k, long n, T koef)
{
    using A = Ar<T>;
    T s, d, u;
    if (V == 1) { s = -L.f1[n]; d = xrow<T, false>(L, i, j, k, n, s); u = L.u1[n] = A::sub(L.u1[n], A::mul(A::div(s, d), koef)); }
    if (V == 2) { s = -L.f2[n]; d = yrow<T, false>(L, i, j, k, n, s); u = L.u2[n] = A::sub(L.u2[n], A::mul(A::div(s, d), koef)); }
    if (V == 3) { s = -L.f3[n]; d = zrow<T, false>(L, i, j, k, n, s); u = L.u3[n] = A::sub(L.u3[n], A::mul(A::div(s, d), koef)); }
    return u;
}

template <typename T, int V>
__device__ __forceinline__ void relax_vel_at(const View<T> &L, long t, int color, T koef)
{
    int i, j, k;
    const long n = vel_row_node<V>(L, t, color, i, j, k);
    if (n < 0 || (L.bc[n] & (1 << V))) return;
    relax_vel_row<T, V>(L, i, j, k, n, koef);
}

template <typename T, int V>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 6 : 4) k_relax_vel(View<T> L, int color, T koef)
{
    pdl_enter();
    long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)((L.ny + 1) >> 1) * L.nx * L.nz) return;
    relax_vel_at<T, V>(L, t, color, koef);
}

// All interior pressure rows: p -= (div v - f) * nd * p0koef (move3mg.c:3105-3116)
// Relaxes pressure row n if it exists; *b receives its bc byte, *u the new value.
template <typename T>
__device__ __forceinline__ bool relax_p_at(const View<T> &L, long n, T koef, uint8_t *b = nullptr, T *u = nullptr)
{
    using A = Ar<T>;
    int i, j, k;
    node_ijk(L, n, i, j, k);
    const uint8_t bb = L.bc[n];
    if (!(i > 0 && j > 0 && k > 0) || (bb & 1)) return false;
    T s = -L.f0[n];
    crow<T, false>(L, i, j, k, n, s);
    const T un = L.u0[n] = A::sub(L.u0[n], A::mul(A::mul(s, (T)L.nd[n]), koef));
    if (b) *b = bb;
    if (u) *u = un;
    return true;
}

template <typename T>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 6 : 4) k_relax_p(View<T> L, T koef)
{
    pdl_enter();
    long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= L.nxy * L.nz) return;
    relax_p_at<T>(L, n, koef);
}

// Boundary rows of one component: x = c1 + k1*(c2 + k2*(... x_partner)) evaluated from the
// innermost link outwards (the fixed point of bonderr rows, move3mg.c:1532-1579).
template <typename T>
__device__ __forceinline__ void bc_apply_at(T *u, int t, const int *node, const int *pnode, const int *depth,
                                            const double *cc, const double *kk, int use_c)
{
    using A = Ar<T>;
    const int p = pnode[t];
    T val = p >= 0 ? u[p] : T(0);
    for (int d = depth[t] - 1; d >= 0; d--) {
        const T c0 = use_c ? (T)cc[t * kMaxBcDepth + d] : T(0);
        val = A::add(c0, A::mul((T)kk[t * kMaxBcDepth + d], val));
    }
    u[node[t]] = val;
}

template <typename T>
__global__ void k_bc_apply(T *u, int n, const int *node, const int *pnode, const int *depth,
                           const double *cc, const double *kk, int use_c)
{
    pdl_enter();
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    bc_apply_at<T>(u, t, node, pnode, depth, cc, kk, use_c);
}

// Device view of a component's boundary rows (BcList).
struct BcDev {
    int n, na;
    const int *node, *pnode, *depth, *onode, *ocomp, *first, *writer;
    const double *c, *k, *ok;
};

// In-kernel boundary rows (BcList::na >= 0).  A sweep's separate boundary pass writes each
// boundary node from its interior partner after the kernel that finalises the component.  Here
// the same values are written inside that kernel, by one of its rows' threads right after that
// row's update (entries [0, na), sorted by writer) or by extra blocks (entries [na, n)).  The
// writer is the partner when the kernel updates the partner; otherwise the one row of the
// kernel that reads the boundary node, if there is one.  Set-up admits a component only if
// every boundary node is read by no row of the kernel other than its writer, whose read comes
// before its write, so all rows see the values the separate pass would leave and the results
// are bit-identical.
//
// The writer's entries are fetched through the read-only path before its own update (e0 =
// first entry), so their loads overlap the row's; a partner that is the writer itself takes the
// value just computed (un), any other partner is final in this kernel.
template <typename T>
__device__ __forceinline__ void bc_writer_rows(T *u, const BcDev &B, int e0, long n, T un, int use_c)
{
    using A = Ar<T>;
    for (int e = e0; e < B.na && __ldg(B.writer + e) == (int)n; e++) {
        const int p = __ldg(B.pnode + e);
        T val = p < 0 ? T(0) : p == (int)n ? un : __ldg(u + p);
        for (int d = __ldg(B.depth + e) - 1; d >= 0; d--) {
            const T c0 = use_c ? (T)__ldg(B.c + e * kMaxBcDepth + d) : T(0);
            val = A::add(c0, A::mul((T)__ldg(B.k + e * kMaxBcDepth + d), val));
        }
        u[__ldg(B.node + e)] = val;
    }
}

// Colour 1 of velocity component V with the component's boundary rows; blocks from rowblocks on
// write entries [na, n).
template <typename T, int V>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 6 : 4) k_relax_vel_bc(View<T> L, T koef, BcDev B, int use_c,
                                                                               unsigned rowblocks)
{
    pdl_enter();
    T *u = V == 1 ? L.u1 : V == 2 ? L.u2 : L.u3;
    if (blockIdx.x >= rowblocks) {
        const int e = B.na + (int)(blockIdx.x - rowblocks) * (int)blockDim.x + (int)threadIdx.x;
        if (e < B.n) bc_apply_at<T>(u, e, B.node, B.pnode, B.depth, B.c, B.k, use_c);
        return;
    }
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)((L.ny + 1) >> 1) * L.nx * L.nz) return;
    int i, j, k;
    const long n = vel_row_node<V>(L, t, 1, i, j, k);
    if (n < 0) return;
    const uint8_t b = L.bc[n];
    if (b & (1 << V)) return;
    const int e0 = (b & (16 << V)) ? __ldg(B.first + n) : B.na;
    const T un = relax_vel_row<T, V>(L, i, j, k, n, koef);
    if (e0 < B.na) bc_writer_rows<T>(u, B, e0, n, un, use_c);
}

// All pressure rows with the pressure boundary rows (no pressure row reads another pressure).
template <typename T>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 6 : 4) k_relax_p_bc(View<T> L, T koef, BcDev B, int use_c,
                                                                             unsigned rowblocks)
{
    pdl_enter();
    if (blockIdx.x >= rowblocks) {
        const int e = B.na + (int)(blockIdx.x - rowblocks) * (int)blockDim.x + (int)threadIdx.x;
        if (e < B.n) bc_apply_at<T>(L.u0, e, B.node, B.pnode, B.depth, B.c, B.k, use_c);
        return;
    }
    const long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= L.nxy * L.nz) return;
    const int e0 = (L.bc[n] & 16) ? __ldg(B.first + n) : B.na;
    uint8_t b = 0;
    T un = 0;
    if (relax_p_at<T>(L, n, koef, &b, &un) && e0 < B.na) bc_writer_rows<T>(L.u0, B, e0, n, un, use_c);
}

// ------------------------------------------------------------------------------------
// residual (gausmat4 residual pass, move3mg.c:3136-3157)
// ------------------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void residual_at(const View<T> &L, long n)
{
    int i, j, k;
    node_ijk(L, n, i, j, k);
    const uint8_t b = L.bc[n];
    if (row_exists(0, i, j, k, L.nx, L.ny, L.nz) && !(b & 1)) { T s = L.f0[n]; crow<T, true>(L, i, j, k, n, s); L.r0[n] = s; }
    if (row_exists(1, i, j, k, L.nx, L.ny, L.nz) && !(b & 2)) { T s = L.f1[n]; xrow<T, true>(L, i, j, k, n, s); L.r1[n] = s; }
    if (row_exists(2, i, j, k, L.nx, L.ny, L.nz) && !(b & 4)) { T s = L.f2[n]; yrow<T, true>(L, i, j, k, n, s); L.r2[n] = s; }
    if (row_exists(3, i, j, k, L.nx, L.ny, L.nz) && !(b & 8)) { T s = L.f3[n]; zrow<T, true>(L, i, j, k, n, s); L.r3[n] = s; }
}

template <typename T>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 4 : 1) k_residual(View<T> L)
{
    pdl_enter();
    long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= L.nxy * L.nz) return;
    residual_at<T>(L, n);
}

// residual of boundary rows with their original (unflattened) partner
template <typename T>
__device__ __forceinline__ void bc_residual_at(const View<T> &L, int V, int t, const int *node, const int *onode,
                                               const int *ocomp, const double *ok)
{
    using A = Ar<T>;
    T *u[4] = {L.u0, L.u1, L.u2, L.u3};
    T *f[4] = {L.f0, L.f1, L.f2, L.f3};
    T *r[4] = {L.r0, L.r1, L.r2, L.r3};
    const int nd = node[t];
    T s = f[V][nd];
    s = A::sub(s, A::mul(T(1), u[V][nd]));
    if (onode[t] >= 0) s = A::sub(s, A::mul((T)(-ok[t]), u[ocomp[t]][onode[t]]));
    r[V][nd] = s;
}

template <typename T>
__global__ void k_bc_residual(View<T> L, int V, int n, const int *node, const int *onode, const int *ocomp,
                              const double *ok)
{
    pdl_enter();
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    bc_residual_at<T>(L, V, t, node, onode, ocomp, ok);
}

// Residual of all rows; blocks from rowblocks on take the boundary rows of the four components
// (they write only boundary nodes, which the row threads skip, and read no residual).
struct BcDev4 {
    BcDev b[4];
};

// Residual of all rows; blocks from rowblocks on take the boundary rows of the four components
// (they write only boundary nodes, which the row threads skip, and read no residual).  One thread
// computes the four rows of a node, which share most of their loads (one thread per row and
// component took 25 % longer with a cold L2).
template <typename T>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 4 : 1) k_residual_bc(View<T> L, BcDev4 B, unsigned rowblocks)
{
    pdl_enter();
    if (blockIdx.x >= rowblocks) {
        int t = (int)(blockIdx.x - rowblocks) * (int)blockDim.x + (int)threadIdx.x;
        for (int v = 0; v < 4; v++) {
            if (t < B.b[v].n) {
                bc_residual_at<T>(L, v, t, B.b[v].node, B.b[v].onode, B.b[v].ocomp, B.b[v].ok);
                return;
            }
            t -= B.b[v].n;
        }
        return;
    }
    const long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= L.nxy * L.nz) return;
    residual_at<T>(L, n);
}

// ------------------------------------------------------------------------------------
// grid transfers in gather form
// ------------------------------------------------------------------------------------
struct TrView {
    const int *gptr, *gf;
    const double *gw;
    const int *a;
    const double *w0, *w1;
};

static TrView trview(const Transfer1D &t)
{
    return TrView{t.gptr, t.gf, t.gw, t.a, t.w0, t.w1};
}

// vprestrict (move3mg.c:3165-3520): coarse row = sum over fine contributors (fine rows that
// exist and are not boundary rows), weight-normalised; pressure residuals scaled by
// nd_fine/nd_coarse.  Contributions are summed in the fine lexicographic order of the
// reference's scatter loop.  Coarse solution is zeroed.
template <typename T, int V>
__device__ __forceinline__ void restrict_at(const View<T> &F, const View<T> &Cc, const TrView &tx, const TrView &ty,
                                            const TrView &tz, long n)
{
    using A = Ar<T>;
    int i, j, k;
    node_ijk(Cc, n, i, j, k);
    T *cu = V == 0 ? Cc.u0 : V == 1 ? Cc.u1 : V == 2 ? Cc.u2 : Cc.u3;
    T *cf_ = V == 0 ? Cc.f0 : V == 1 ? Cc.f1 : V == 2 ? Cc.f2 : Cc.f3;
    const T *fr = V == 0 ? F.r0 : V == 1 ? F.r1 : V == 2 ? F.r2 : F.r3;
    cu[n] = T(0);
    if (!row_exists(V, i, j, k, Cc.nx, Cc.ny, Cc.nz) || (Cc.bc[n] & (1 << V))) { cf_[n] = T(0); return; }
    T sum = 0, ws = 0;
    const T ndc = V == 0 ? (T)Cc.nd[n] : T(1);
    for (int ez = tz.gptr[k]; ez < tz.gptr[k + 1]; ez++) {
        const int fk = tz.gf[ez];
        const T wz = (T)tz.gw[ez];
        for (int ex = tx.gptr[i]; ex < tx.gptr[i + 1]; ex++) {
            const int fi = tx.gf[ex];
            const T wx = (T)tx.gw[ex];
            for (int ey = ty.gptr[j]; ey < ty.gptr[j + 1]; ey++) {
                const int fj = ty.gf[ey];
                if (!row_exists(V, fi, fj, fk, F.nx, F.ny, F.nz)) continue;
                const long m = (long)fk * F.nxy + (long)fi * F.ny + fj;
                if (F.bc[m] & (1 << V)) continue;
                const T swt = A::mul(A::mul(wx, (T)ty.gw[ey]), wz);
                T term;
                if (V == 0) term = A::mul(A::div(A::mul(fr[m], (T)F.nd[m]), ndc), swt);
                else term = A::mul(fr[m], swt);
                sum = A::add(sum, term);
                ws = A::add(ws, swt);
            }
        }
    }
    cf_[n] = ws != T(0) ? A::div(sum, ws) : sum;
}

template <typename T, int V>
__global__ void __launch_bounds__(256) k_restrict(View<T> F, View<T> Cc, TrView tx, TrView ty, TrView tz)
{
    pdl_enter();
    long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= Cc.nxy * Cc.nz) return;
    restrict_at<T, V>(F, Cc, tx, ty, tz, n);
}

// FP32 restriction with four lanes per coarse row (the FP32 V-cycle's restriction): lane q of a
// group sums the fine contributors of the z-entries gptr[k] + q, + q + 4, ..., the group's partial
// sums and weights are added by two shuffles, and the pressure rows' 1 / nd_coarse is applied once
// to the sum instead of to every term.  A coarse row gathers up to 4 x 4 x 4 contributors, so one
// thread per row is a long chain of dependent loads; four shorten it and fill small levels.  The
// FP32 sums come out in a different order than the FP64 restriction's (which follows the
// reference's scatter order bit for bit); the FP32 V-cycle is a preconditioner only.
template <int V>
__device__ __forceinline__ void restrict_split_at(const View<float> &F, const View<float> &Cc, const TrView &tx,
                                                  const TrView &ty, const TrView &tz, long n, int q, bool live)
{
    int i = 0, j = 0, k = 0;
    float sum = 0.f, ws = 0.f;
    bool row = false;
    const float *fr = V == 0 ? F.r0 : V == 1 ? F.r1 : V == 2 ? F.r2 : F.r3;
    if (live) {
        node_ijk(Cc, n, i, j, k);
        row = row_exists(V, i, j, k, Cc.nx, Cc.ny, Cc.nz) && !(Cc.bc[n] & (1 << V));
        if (row) {
            for (int ez = tz.gptr[k] + q; ez < tz.gptr[k + 1]; ez += 4) {
                const int fk = tz.gf[ez];
                const float wz = (float)tz.gw[ez];
                for (int ex = tx.gptr[i]; ex < tx.gptr[i + 1]; ex++) {
                    const int fi = tx.gf[ex];
                    const float wx = (float)tx.gw[ex];
                    for (int ey = ty.gptr[j]; ey < ty.gptr[j + 1]; ey++) {
                        const int fj = ty.gf[ey];
                        if (!row_exists(V, fi, fj, fk, F.nx, F.ny, F.nz)) continue;
                        const long m = (long)fk * F.nxy + (long)fi * F.ny + fj;
                        if (F.bc[m] & (1 << V)) continue;
                        const float swt = wx * (float)ty.gw[ey] * wz;
                        sum += (V == 0 ? fr[m] * F.nd[m] : fr[m]) * swt;
                        ws += swt;
                    }
                }
            }
        }
    }
    sum += __shfl_xor_sync(0xffffffffu, sum, 1);
    ws += __shfl_xor_sync(0xffffffffu, ws, 1);
    sum += __shfl_xor_sync(0xffffffffu, sum, 2);
    ws += __shfl_xor_sync(0xffffffffu, ws, 2);
    if (!live || q != 0) return;
    float *cu = V == 0 ? Cc.u0 : V == 1 ? Cc.u1 : V == 2 ? Cc.u2 : Cc.u3;
    float *cf_ = V == 0 ? Cc.f0 : V == 1 ? Cc.f1 : V == 2 ? Cc.f2 : Cc.f3;
    cu[n] = 0.f;
    if (!row) { cf_[n] = 0.f; return; }
    if (V == 0) sum /= Cc.nd[n];
    cf_[n] = ws != 0.f ? sum / ws : sum;
}

// vpprolong (move3mg.c:2748-3063): fine += sum_8 coarse * weight * koef
template <typename T, int V>
__device__ __forceinline__ void prolong_at(const View<T> &F, const View<T> &Cc, const TrView &tx, const TrView &ty,
                                           const TrView &tz, T koef, long n)
{
    using A = Ar<T>;
    int i, j, k;
    node_ijk(F, n, i, j, k);
    if (!row_exists(V, i, j, k, F.nx, F.ny, F.nz)) return;
    T *fu = V == 0 ? F.u0 : V == 1 ? F.u1 : V == 2 ? F.u2 : F.u3;
    const T *cu = V == 0 ? Cc.u0 : V == 1 ? Cc.u1 : V == 2 ? Cc.u2 : Cc.u3;
    const int a = tx.a[i], b = ty.a[j], c = tz.a[k];
    const T wx[2] = {(T)tx.w0[i], (T)tx.w1[i]};
    const T wy[2] = {(T)ty.w0[j], (T)ty.w1[j]};
    const T wz[2] = {(T)tz.w0[k], (T)tz.w1[k]};
    T s = fu[n];
    for (int dz = 0; dz < 2; dz++)
        for (int dx = 0; dx < 2; dx++)
            for (int dy = 0; dy < 2; dy++) {
                const long m = (long)(c + dz) * Cc.nxy + (long)(a + dx) * Cc.ny + (b + dy);
                const T swt = A::mul(A::mul(wx[dx], wy[dy]), wz[dz]);
                s = A::add(s, A::mul(A::mul(cu[m], swt), koef));
            }
    fu[n] = s;
}

template <typename T, int V>
__global__ void __launch_bounds__(256) k_prolong(View<T> F, View<T> Cc, TrView tx, TrView ty, TrView tz, T koef)
{
    pdl_enter();
    long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= F.nxy * F.nz) return;
    prolong_at<T, V>(F, Cc, tx, ty, tz, koef, n);
}

// The four components' transfers in one launch (blockIdx.y = component); the components read
// and write disjoint arrays.
struct Tr4 {
    TrView t[4][3];      // [component][axis]
};

template <typename T>
__global__ void __launch_bounds__(256) k_restrict4(View<T> F, View<T> Cc, Tr4 R)
{
    pdl_enter();
    const long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= Cc.nxy * Cc.nz) return;
    switch (blockIdx.y) {
    case 0: restrict_at<T, 0>(F, Cc, R.t[0][0], R.t[0][1], R.t[0][2], n); break;
    case 1: restrict_at<T, 1>(F, Cc, R.t[1][0], R.t[1][1], R.t[1][2], n); break;
    case 2: restrict_at<T, 2>(F, Cc, R.t[2][0], R.t[2][1], R.t[2][2], n); break;
    default: restrict_at<T, 3>(F, Cc, R.t[3][0], R.t[3][1], R.t[3][2], n); break;
    }
}

// four components (blockIdx.y), four lanes per coarse row
__global__ void __launch_bounds__(256) k_restrict4_f32(View<float> F, View<float> Cc, Tr4 R)
{
    pdl_enter();
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long n = t >> 2;
    const int q = (int)(t & 3);
    const bool live = n < Cc.nxy * Cc.nz;
    switch (blockIdx.y) {
    case 0: restrict_split_at<0>(F, Cc, R.t[0][0], R.t[0][1], R.t[0][2], n, q, live); break;
    case 1: restrict_split_at<1>(F, Cc, R.t[1][0], R.t[1][1], R.t[1][2], n, q, live); break;
    case 2: restrict_split_at<2>(F, Cc, R.t[2][0], R.t[2][1], R.t[2][2], n, q, live); break;
    default: restrict_split_at<3>(F, Cc, R.t[3][0], R.t[3][1], R.t[3][2], n, q, live); break;
    }
}

template <typename T>
__global__ void __launch_bounds__(256) k_prolong4(View<T> F, View<T> Cc, Tr4 R, T kv, T kp)
{
    pdl_enter();
    const long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= F.nxy * F.nz) return;
    switch (blockIdx.y) {
    case 0: prolong_at<T, 0>(F, Cc, R.t[0][0], R.t[0][1], R.t[0][2], kp, n); break;
    case 1: prolong_at<T, 1>(F, Cc, R.t[1][0], R.t[1][1], R.t[1][2], kv, n); break;
    case 2: prolong_at<T, 2>(F, Cc, R.t[2][0], R.t[2][1], R.t[2][2], kv, n); break;
    default: prolong_at<T, 3>(F, Cc, R.t[3][0], R.t[3][1], R.t[3][2], kv, n); break;
    }
}

// ------------------------------------------------------------------------------------
// coarse tail of a V-cycle in one thread block
// ------------------------------------------------------------------------------------
// On levels of a few thousand nodes every relaxation phase is a kernel of a few hundred
// rows, so the V-cycle there is bound by kernel-to-kernel latency (11 dependent launches per
// sweep, up to 64 sweeps per level).  The tail kernel runs the whole lower part of the
// V-cycle -- down sweeps, residuals, restrictions, coarsest sweeps, prolongations and up
// sweeps of the small levels -- in one block of 512 threads, with __syncthreads() where the
// multi-kernel version has a kernel boundary.  Each phase applies the same per-row functions
// to the same rows, and rows within a phase are independent, so results are bit-identical.
// The small levels stay resident in L1/L2.
constexpr int kTailMax = 6;
constexpr int kTailThreads = 512;

template <typename T>
struct TailLevel {
    View<T> v;
    BcDev bc[4];
    TrView tr[4][3];     // transfer to the next coarser level: [component][axis]
    int down, up;        // sweeps on the way down (0: residual only) and on the way up
};

template <typename T>
struct TailArgs {
    int nl;
    T v0, p0, kv, kp;
    TailLevel<T> L[kTailMax];
};

template <typename T>
__device__ __forceinline__ T *comp(const View<T> &L, int v)
{
    return v == 0 ? L.u0 : v == 1 ? L.u1 : v == 2 ? L.u2 : L.u3;
}

// The threads that run the tail, and their barrier: one block (the one-block tail kernel) or the
// whole co-resident grid of a cooperative launch (the coarse-level kernel).
struct BlockTeam {
    __device__ __forceinline__ long rank() const { return threadIdx.x; }
    __device__ __forceinline__ long size() const { return blockDim.x; }
    __device__ __forceinline__ void sync() const { __syncthreads(); }
};

// The CTAs of one thread-block cluster (up to 16, on distinct SMs of one GPC) and the hardware
// cluster barrier, whose release/acquire orders the global-memory writes of one phase before the
// reads of the next across the cluster.
struct ClusterTeam {
    __device__ __forceinline__ long rank() const
    {
        unsigned r;
        asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
        return (long)r * blockDim.x + threadIdx.x;
    }
    __device__ __forceinline__ long size() const
    {
        unsigned n;
        asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(n));
        return (long)n * blockDim.x;
    }
    __device__ __forceinline__ void sync() const
    {
        asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
    }
};

// Grid-wide barrier of a cooperative launch (all CTAs resident by construction).  The last CTA
// to arrive resets the counter and advances the generation; the others wait for the generation,
// each for at most 2 s (then the launch's error flag is set and the wait gives up, so a broken
// launch can never hang the GPU; the host reports the flag as an error).
struct GridTeam {
    unsigned *count;
    unsigned *gen;
    int *err;
    __device__ __forceinline__ long rank() const { return (long)blockIdx.x * blockDim.x + threadIdx.x; }
    __device__ __forceinline__ long size() const { return (long)gridDim.x * blockDim.x; }
    __device__ void sync() const
    {
        __syncthreads();
        if (threadIdx.x == 0) {
            volatile unsigned *vg = gen;
            const unsigned g = *vg;   // cannot advance before this CTA arrives
            __threadfence();
            if (atomicAdd(count, 1u) == gridDim.x - 1) {
                atomicExch(count, 0u);
                __threadfence();
                atomicAdd(gen, 1u);
            } else {
                uint64_t t0;
                asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
                while (*vg == g) {
                    uint64_t t;
                    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
                    if (t - t0 > 2000000000ull) {
                        atomicOr(err, 1);
                        break;
                    }
                }
            }
            __threadfence();
        }
        __syncthreads();
    }
};

template <typename T, typename Team>
__device__ void tail_bc(const TailLevel<T> &TL, int v, const Team &tm)
{
    const BcDev &B = TL.bc[v];
    if (B.n == 0) return;   // uniform over the team
    T *u = comp(TL.v, v);
    for (long t = tm.rank(); t < B.n; t += tm.size()) bc_apply_at<T>(u, (int)t, B.node, B.pnode, B.depth, B.c, B.k, 0);
    tm.sync();
}

template <typename T, int V, typename Team>
__device__ void tail_colours(const TailLevel<T> &TL, T v0, const Team &tm)
{
    const View<T> &L = TL.v;
    const long total = (long)((L.ny + 1) >> 1) * L.nx * L.nz;
    for (int color = 0; color < 2; color++) {
        for (long t = tm.rank(); t < total; t += tm.size()) relax_vel_at<T, V>(L, t, color, v0);
        tm.sync();
    }
    tail_bc<T>(TL, V, tm);
}

template <typename T, typename Team>
__device__ void tail_smooth(const TailLevel<T> &TL, int nsweeps, T v0, T p0, const Team &tm)
{
    const View<T> &L = TL.v;
    const long N = L.nxy * L.nz;
    for (int s = 0; s < nsweeps; s++) {
        tail_colours<T, 1>(TL, v0, tm);
        tail_colours<T, 2>(TL, v0, tm);
        tail_colours<T, 3>(TL, v0, tm);
        for (long n = tm.rank(); n < N; n += tm.size()) relax_p_at<T>(L, n, p0);
        tm.sync();
        tail_bc<T>(TL, 0, tm);
    }
}

template <typename T, typename Team>
__device__ void tail_residual(const TailLevel<T> &TL, const Team &tm)
{
    const View<T> &L = TL.v;
    const long N = L.nxy * L.nz;
    for (long n = tm.rank(); n < N; n += tm.size()) residual_at<T>(L, n);
    for (int v = 0; v < 4; v++) {
        const BcDev &B = TL.bc[v];
        for (long t = tm.rank(); t < B.n; t += tm.size()) bc_residual_at<T>(L, v, (int)t, B.node, B.onode, B.ocomp, B.ok);
    }
    tm.sync();
}

template <typename T, typename Team>
__device__ void tail_restrict(const TailLevel<T> &F, const TailLevel<T> &C, const Team &tm)
{
    const long N = C.v.nxy * C.v.nz;
    for (long n = tm.rank(); n < N; n += tm.size()) {
        restrict_at<T, 1>(F.v, C.v, F.tr[1][0], F.tr[1][1], F.tr[1][2], n);
        restrict_at<T, 2>(F.v, C.v, F.tr[2][0], F.tr[2][1], F.tr[2][2], n);
        restrict_at<T, 3>(F.v, C.v, F.tr[3][0], F.tr[3][1], F.tr[3][2], n);
        restrict_at<T, 0>(F.v, C.v, F.tr[0][0], F.tr[0][1], F.tr[0][2], n);
    }
    tm.sync();
}

template <typename T, typename Team>
__device__ void tail_prolong(const TailLevel<T> &F, const TailLevel<T> &C, T kv, T kp, const Team &tm)
{
    const long N = F.v.nxy * F.v.nz;
    for (long n = tm.rank(); n < N; n += tm.size()) {
        prolong_at<T, 1>(F.v, C.v, F.tr[1][0], F.tr[1][1], F.tr[1][2], kv, n);
        prolong_at<T, 2>(F.v, C.v, F.tr[2][0], F.tr[2][1], F.tr[2][2], kv, n);
        prolong_at<T, 3>(F.v, C.v, F.tr[3][0], F.tr[3][1], F.tr[3][2], kv, n);
        prolong_at<T, 0>(F.v, C.v, F.tr[0][0], F.tr[0][1], F.tr[0][2], kp, n);
    }
    tm.sync();
}

// Levels a.L[0..nl-1] (fine to coarse) of the V-cycle schedule of move3mg.c:2173-2213, from
// the down sweeps of a.L[0] to its up sweeps.
template <typename T, typename Team>
__device__ void tail_body(const TailArgs<T> &a, const Team &tm)
{
    for (int q = 0; q + 1 < a.nl; q++) {
        if (a.L[q].down > 0) tail_smooth<T>(a.L[q], a.L[q].down, a.v0, a.p0, tm);
        tail_residual<T>(a.L[q], tm);
        tail_restrict<T>(a.L[q], a.L[q + 1], tm);
    }
    for (int q = a.nl - 1; q > 0; q--) {
        if (a.L[q].up > 0) tail_smooth<T>(a.L[q], a.L[q].up, a.v0, a.p0, tm);
        tail_prolong<T>(a.L[q - 1], a.L[q], a.kv, a.kp, tm);
    }
    if (a.L[0].up > 0) tail_smooth<T>(a.L[0], a.L[0].up, a.v0, a.p0, tm);
}

template <typename T>
__global__ void __launch_bounds__(kTailThreads, 1) k_vcycle_tail(const __grid_constant__ TailArgs<T> a)
{
    pdl_enter();
    tail_body<T>(a, BlockTeam());
}

// The same schedule over the whole grid of a cooperative launch: every phase spreads its rows
// over all resident threads and ends at a grid barrier instead of a kernel boundary, so the
// coarse levels run as one launch without being confined to one SM.
constexpr int kCoopThreads = 256;

template <typename T>
__global__ void __launch_bounds__(kCoopThreads) k_vcycle_coop(const __grid_constant__ TailArgs<T> a, GridTeam tm)
{
    pdl_enter();
    tail_body<T>(a, tm);
}

// The same schedule on one cluster of CTAs: the small coarse levels run on several SMs with a
// hardware barrier between phases instead of on one SM (the one-block tail) or the whole grid.
template <typename T>
__global__ void __launch_bounds__(kTailThreads, 1) k_vcycle_cluster(const __grid_constant__ TailArgs<T> a)
{
    pdl_enter();
    tail_body<T>(a, ClusterTeam());
}

// ronurestrict (move3mg.c:2642-2741): FP32 accumulator as in nu[], FP64 weights
__global__ void k_nu_restrict(const float *nuf, int fnx, int fny, int fnz, float *nuc, int cnx, int cny, int cnz,
                              TrView tx, TrView ty, TrView tz, int viscmod)
{
    pdl_enter();
    long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long N = (long)cnx * cny * cnz;
    if (n >= N) return;
    const int j = (int)(n % cny);
    const long rest = n / cny;
    const int i = (int)(rest % cnx), k = (int)(rest / cnx);
    float accu = 0.f;
    double ws = 0;
    for (int ez = tz.gptr[k]; ez < tz.gptr[k + 1]; ez++) {
        const int fk = tz.gf[ez];
        const double wz = tz.gw[ez];
        for (int ex = tx.gptr[i]; ex < tx.gptr[i + 1]; ex++) {
            const int fi = tx.gf[ex];
            const double wx = tx.gw[ex];
            for (int ey = ty.gptr[j]; ey < ty.gptr[j + 1]; ey++) {
                const int fj = ty.gf[ey];
                const double swt = __dmul_rn(__dmul_rn(wx, ty.gw[ey]), wz);
                const float nf = nuf[(long)fk * fnx * fny + (long)fi * fny + fj];
                double iv = viscmod == 0 ? __dmul_rn((double)nf, swt)
                          : viscmod == 1 ? __dmul_rn(log((double)nf), swt) : __dmul_rn(__ddiv_rn(1.0, (double)nf), swt);
                accu = (float)__dadd_rn((double)accu, iv);
                ws = __dadd_rn(ws, swt);
            }
        }
    }
    float r = (float)__ddiv_rn((double)accu, ws);
    if (viscmod == 1) r = (float)exp((double)r);
    if (viscmod == 2) r = (float)__ddiv_rn(1.0, (double)r);
    nuc[n] = r;
}

// ------------------------------------------------------------------------------------
// operator set-up: stress-point viscosities (sxxcalc..syzcalc nueff, move3mg.c:30-46, 402-412)
// ------------------------------------------------------------------------------------
struct EtaArgs {
    int nx, ny, nz, lev0, viscmod;
    const float *nu, *nxx, *nxy, *nxz, *nyz;
    double nubeg, nuend;
    double *etac, *etaxy, *etaxz, *etayz;
    float *nd;
};

__device__ __forceinline__ double avg8(const float *nu, long v0, long NY, long NXY, int viscmod)
{
    const long v[8] = {v0, v0 + 1, v0 + NY, v0 + NY + 1, v0 + NXY, v0 + NXY + 1, v0 + NXY + NY, v0 + NXY + NY + 1};
    if (viscmod == 0) {
        float s = nu[v[0]];
        for (int q = 1; q < 8; q++) s = __fadd_rn(s, nu[v[q]]);
        return __ddiv_rn((double)s, 8.0);
    }
    double s = 0;
    if (viscmod == 1) {
        s = log((double)nu[v[0]]);
        for (int q = 1; q < 8; q++) s = __dadd_rn(s, log((double)nu[v[q]]));
        return exp(__ddiv_rn(s, 8.0));
    }
    s = __ddiv_rn(1.0, (double)nu[v[0]]);
    for (int q = 1; q < 8; q++) s = __dadd_rn(s, __ddiv_rn(1.0, (double)nu[v[q]]));
    return __ddiv_rn(1.0, __ddiv_rn(s, 8.0));
}

__device__ __forceinline__ double avg2(const float *nu, long a, long b, int viscmod)
{
    if (viscmod == 0) return __ddiv_rn((double)__fadd_rn(nu[a], nu[b]), 2.0);
    if (viscmod == 1) return exp(__ddiv_rn(__dadd_rn(log((double)nu[a]), log((double)nu[b])), 2.0));
    return __ddiv_rn(1.0, __ddiv_rn(__dadd_rn(__ddiv_rn(1.0, (double)nu[a]), __ddiv_rn(1.0, (double)nu[b])), 2.0));
}

__device__ __forceinline__ double clampnu(double n, double b, double e)
{
    if (n > e) n = e;
    if (n < b) n = b;
    return n;
}

__global__ void k_eta(EtaArgs a)
{
    pdl_enter();
    long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long NY = a.ny, NXY = (long)a.nx * a.ny, N = NXY * a.nz;
    if (n >= N) return;
    const int m2 = (int)(n % NY);
    const long rest = n / NY;
    const int m1 = (int)(rest % a.nx), m3 = (int)(rest / a.nx);
    double ec = 0, exy = 0, exz = 0, eyz = 0;
    if (m1 > 0 && m2 > 0 && m3 > 0) {
        double v;
        if (a.lev0 && m1 > 3 && m2 > 3 && m3 > 3 && m1 < a.nx - 3 && m2 < a.ny - 3 && m3 < a.nz - 3) v = a.nxx[n];
        else v = avg8(a.nu, n - NXY - NY - 1, NY, NXY, a.viscmod);
        ec = clampnu(v, a.nubeg, a.nuend);
    }
    if (m1 > 0 && m1 < a.nx - 1 && m2 > 0 && m2 < a.ny - 1 && m3 < a.nz - 1) {
        double v;
        if (a.lev0 && m1 > 3 && m2 > 3 && m3 > 2 && m1 < a.nx - 4 && m2 < a.ny - 4 && m3 < a.nz - 4) v = a.nxy[n];
        else v = avg2(a.nu, n, n + NXY, a.viscmod);
        exy = clampnu(v, a.nubeg, a.nuend);
    }
    if (m1 > 0 && m1 < a.nx - 1 && m3 > 0 && m3 < a.nz - 1 && m2 < a.ny - 1) {
        double v;
        if (a.lev0 && m1 > 3 && m2 > 2 && m3 > 3 && m1 < a.nx - 4 && m2 < a.ny - 4 && m3 < a.nz - 4) v = a.nxz[n];
        else v = avg2(a.nu, n, n + 1, a.viscmod);
        exz = clampnu(v, a.nubeg, a.nuend);
    }
    if (m2 > 0 && m2 < a.ny - 1 && m3 > 0 && m3 < a.nz - 1 && m1 < a.nx - 1) {
        double v;
        if (a.lev0 && m1 > 2 && m2 > 3 && m3 > 3 && m1 < a.nx - 4 && m2 < a.ny - 4 && m3 < a.nz - 4) v = a.nyz[n];
        else v = avg2(a.nu, n, n + NY, a.viscmod);
        eyz = clampnu(v, a.nubeg, a.nuend);
    }
    a.etac[n] = ec; a.etaxy[n] = exy; a.etaxz[n] = exz; a.etayz[n] = eyz;
    a.nd[n] = (float)ec;
}

// scaled FP32 copies of the level operator data
__global__ void k_eta_f32(long n, const double *ec, const double *exy, const double *exz, const double *eyz,
                          const float *nd, float *fc, float *fxy, float *fxz, float *fyz, float *fnd, double inv_ref)
{
    pdl_enter();
    long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    fc[t] = (float)(ec[t] * inv_ref);
    fxy[t] = (float)(exy[t] * inv_ref);
    fxz[t] = (float)(exz[t] * inv_ref);
    fyz[t] = (float)(eyz[t] * inv_ref);
    fnd[t] = (float)((double)nd[t] * inv_ref);
}

// Pressure-update scale of the FP32 preconditioner's smoother.  The reference scales a cell's
// pressure correction by the cell's own viscosity (nd = etac, p -= r nd p0koef).  The diagonal of
// the pressure Schur complement B diag(A)^-1 B^T is the sum over the cell's six faces of
// (1/h)^2 / diag(face velocity row), so its inverse scales with the harmonic mean of the face rows'
// viscosities: a weak cell enclosed by stiff material (a weak layer's cell inside a 1e24
// lithosphere) needs corrections set by its stiff neighbours, and the cell viscosity makes them
// 1e5 times too small (its divergence stalls; the subduction model's continuity residual stopped
// at 1e-3).  In regions of smooth viscosity the two scales agree.
//
// weighted mean of a velocity row's six stencil viscosities: the row's diagonal over the one it has
// with unit viscosity (xrow, yrow, zrow coefficients)
__device__ double vrow_eta(const View<double> &L, int V, int i, int j, int k, long n)
{
    const long NY = L.ny, NXY = L.nxy;
    double w[6], e[6];
    if (V == 1) {
        const double XK = 2.0 * L.isx[i], YK = L.icy[j + 1], ZK = L.icz[k + 1];
        w[0] = XK * L.icx[i]; w[1] = XK * L.icx[i + 1]; w[2] = YK * L.isy[j]; w[3] = YK * L.isy[j + 1];
        w[4] = ZK * L.isz[k]; w[5] = ZK * L.isz[k + 1];
        e[0] = L.etac[n + NXY + 1]; e[1] = L.etac[n + NXY + NY + 1]; e[2] = L.etaxy[n]; e[3] = L.etaxy[n + 1];
        e[4] = L.etaxz[n]; e[5] = L.etaxz[n + NXY];
    } else if (V == 2) {
        const double XK = L.icx[i + 1], YK = 2.0 * L.isy[j], ZK = L.icz[k + 1];
        w[0] = YK * L.icy[j]; w[1] = YK * L.icy[j + 1]; w[2] = XK * L.isx[i]; w[3] = XK * L.isx[i + 1];
        w[4] = ZK * L.isz[k]; w[5] = ZK * L.isz[k + 1];
        e[0] = L.etac[n + NY + NXY]; e[1] = L.etac[n + NY + 1 + NXY]; e[2] = L.etaxy[n]; e[3] = L.etaxy[n + NY];
        e[4] = L.etayz[n]; e[5] = L.etayz[n + NXY];
    } else {
        const double XK = L.icx[i + 1], YK = L.icy[j + 1], ZK = 2.0 * L.isz[k];
        w[0] = ZK * L.icz[k]; w[1] = ZK * L.icz[k + 1]; w[2] = XK * L.isx[i]; w[3] = XK * L.isx[i + 1];
        w[4] = YK * L.isy[j]; w[5] = YK * L.isy[j + 1];
        e[0] = L.etac[n + NY + 1]; e[1] = L.etac[n + NY + 1 + NXY]; e[2] = L.etaxz[n]; e[3] = L.etaxz[n + NY];
        e[4] = L.etayz[n]; e[5] = L.etayz[n + 1];
    }
    double sw = 0, se = 0;
#pragma unroll
    for (int q = 0; q < 6; q++) { sw += w[q]; se += w[q] * e[q]; }
    return sw > 0 ? se / sw : 0.0;
}

// fnd[cell] = the harmonic mean over the cell's interior face rows of vrow_eta where it exceeds the
// cell viscosity by more than the factor ratio, scaled like the FP32 copy; the cell viscosity
// otherwise.  Only a weak cell (nearly) enclosed by stiff material reaches a large ratio; on the
// boundary of a weak inclusion the weak faces keep the harmonic mean within a few times the cell
// viscosity, and changing the scale there costs the inclusion models a V-cycle per step.
__global__ void k_nd_schur(View<double> L, float *fnd, double inv_ref, double ratio)
{
    pdl_enter();
    const long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= L.nxy * L.nz) return;
    int i, j, k;
    node_ijk(L, n, i, j, k);
    if (!row_exists(0, i, j, k, L.nx, L.ny, L.nz)) return;
    const long v0 = n - L.nxy - L.ny - 1;
    const int fi[6] = {i - 1, i, i - 1, i - 1, i - 1, i - 1}, fj[6] = {j - 1, j - 1, j - 1, j, j - 1, j - 1},
              fk[6] = {k - 1, k - 1, k - 1, k - 1, k - 1, k}, fv[6] = {1, 1, 2, 2, 3, 3};
    const long fm[6] = {v0, v0 + L.ny, v0, v0 + 1, v0, v0 + L.nxy};
    double inv = 0;
    int cnt = 0;
#pragma unroll
    for (int q = 0; q < 6; q++) {
        if (!row_exists(fv[q], fi[q], fj[q], fk[q], L.nx, L.ny, L.nz) || (L.bc[fm[q]] & (1 << fv[q]))) continue;
        const double e = vrow_eta(L, fv[q], fi[q], fj[q], fk[q], fm[q]);
        if (e > 0) { inv += 1.0 / e; cnt++; }
    }
    const double h = cnt ? (double)cnt / inv : 0.0;
    if (h > ratio * L.etac[n]) fnd[n] = (float)(h * inv_ref);
}

// level-0 right-hand side (move3mg.c:751, 942, 1140) and boundary constants
__global__ void k_rhs0(View<double> L, const float *ro, double gx, double gy, double gz)
{
    pdl_enter();
    long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long NY = L.ny, NXY = L.nxy, N = NXY * L.nz;
    if (n >= N) return;
    const int j = (int)(n % NY);
    const long rest = n / NY;
    const int i = (int)(rest % L.nx), k = (int)(rest / L.nx);
    const uint8_t b = L.bc[n];
    L.f0[n] = 0;
    L.f1[n] = 0; L.f2[n] = 0; L.f3[n] = 0;
    if (row_exists(1, i, j, k, L.nx, L.ny, L.nz) && !(b & 2)) {
        const float s = __fadd_rn(__fadd_rn(__fadd_rn(ro[n], ro[n + 1]), ro[n + NXY]), ro[n + NXY + 1]);
        L.f1[n] = __ddiv_rn(__dmul_rn(-gx, (double)s), 4.0);
    }
    if (row_exists(2, i, j, k, L.nx, L.ny, L.nz) && !(b & 4)) {
        const float s = __fadd_rn(__fadd_rn(__fadd_rn(ro[n], ro[n + NY]), ro[n + NXY]), ro[n + NXY + NY]);
        L.f2[n] = __ddiv_rn(__dmul_rn(-gy, (double)s), 4.0);
    }
    if (row_exists(3, i, j, k, L.nx, L.ny, L.nz) && !(b & 8)) {
        const float s = __fadd_rn(__fadd_rn(__fadd_rn(ro[n], ro[n + 1]), ro[n + NY]), ro[n + NY + 1]);
        L.f3[n] = __ddiv_rn(__dmul_rn(-gz, (double)s), 4.0);
    }
}

__global__ void k_bc_rhs(double *f, int n, const int *node, const double *oc)
{
    pdl_enter();
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) f[node[t]] = oc[t];
}

// load the current v,P into the level-0 solution (move3mg.c:1969-2019)
__global__ void k_load_sol(View<double> L, const double *pr, const float *vx, const float *vy, const float *vz)
{
    pdl_enter();
    long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long NY = L.ny, N = L.nxy * L.nz;
    if (n >= N) return;
    const int j = (int)(n % NY);
    const long rest = n / NY;
    const int i = (int)(rest % L.nx), k = (int)(rest / L.nx);
    L.u0[n] = row_exists(0, i, j, k, L.nx, L.ny, L.nz) ? pr[n] : 0.0;
    L.u1[n] = row_exists(1, i, j, k, L.nx, L.ny, L.nz) ? (double)vx[n] : 0.0;
    L.u2[n] = row_exists(2, i, j, k, L.nx, L.ny, L.nz) ? (double)vy[n] : 0.0;
    L.u3[n] = row_exists(3, i, j, k, L.nx, L.ny, L.nz) ? (double)vz[n] : 0.0;
}

// ------------------------------------------------------------------------------------
// norms (deterministic two-pass block reduction)
// ------------------------------------------------------------------------------------
constexpr int kRedThreads = 256;
constexpr int kRedQ = 4;   // quantities: sum r_mom^2, sum f_mom^2, sum r_cont^2, sum v^2

__device__ __forceinline__ double warp_sum(double v)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_relres_part(View<T> L, double *part)
{
    pdl_enter();
    __shared__ double sh[kRedQ][kRedThreads / 32];
    double q[kRedQ] = {0, 0, 0, 0};
    const long N = L.nxy * L.nz;
    for (long n = (long)blockIdx.x * blockDim.x + threadIdx.x; n < N; n += (long)gridDim.x * blockDim.x) {
        int i, j, k;
        node_ijk(L, n, i, j, k);
        const uint8_t b = L.bc[n];
        if (row_exists(0, i, j, k, L.nx, L.ny, L.nz) && !(b & 1)) {
            T s = L.f0[n]; crow<T, true>(L, i, j, k, n, s); q[2] += (double)s * (double)s;
        }
        if (row_exists(1, i, j, k, L.nx, L.ny, L.nz)) {
            q[3] += (double)L.u1[n] * (double)L.u1[n];
            if (!(b & 2)) { T s = L.f1[n]; xrow<T, true>(L, i, j, k, n, s); q[0] += (double)s * s; q[1] += (double)L.f1[n] * L.f1[n]; }
        }
        if (row_exists(2, i, j, k, L.nx, L.ny, L.nz)) {
            q[3] += (double)L.u2[n] * (double)L.u2[n];
            if (!(b & 4)) { T s = L.f2[n]; yrow<T, true>(L, i, j, k, n, s); q[0] += (double)s * s; q[1] += (double)L.f2[n] * L.f2[n]; }
        }
        if (row_exists(3, i, j, k, L.nx, L.ny, L.nz)) {
            q[3] += (double)L.u3[n] * (double)L.u3[n];
            if (!(b & 8)) { T s = L.f3[n]; zrow<T, true>(L, i, j, k, n, s); q[0] += (double)s * s; q[1] += (double)L.f3[n] * L.f3[n]; }
        }
    }
    const int w = threadIdx.x >> 5, ln = threadIdx.x & 31;
    for (int a = 0; a < kRedQ; a++) {
        double v = warp_sum(q[a]);
        if (ln == 0) sh[a][w] = v;
    }
    __syncthreads();
    if (threadIdx.x < kRedQ) {
        double v = 0;
        for (int a = 0; a < kRedThreads / 32; a++) v += sh[threadIdx.x][a];
        part[(long)blockIdx.x * kRedQ + threadIdx.x] = v;
    }
}

__global__ void k_red_final(const double *part, int nblk, int nq, double *out)
{
    pdl_enter();
    // one warp per quantity, fixed order
    const int qi = threadIdx.x >> 5, ln = threadIdx.x & 31;
    if (qi >= nq) return;
    double v = 0;
    for (int b = ln; b < nblk; b += 32) v += part[(long)b * nq + qi];
    v = warp_sum(v);
    if (ln == 0) out[qi] = v;
}

// ------------------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------------------
static inline unsigned nblk(long n, int t = 256) { return (unsigned)((n + t - 1) / t); }

template <typename T>
static T *dalloc(long n)
{
    void *p = nullptr;
    if (cudaMalloc(&p, sizeof(T) * (n > 0 ? n : 1)) != cudaSuccess) return nullptr;
    return (T *)p;
}

#define ALLOC(ptr, T, n)                                                                   \
    do {                                                                                   \
        ptr = dalloc<T>(n);                                                                \
        if (!ptr) return set_error(c, I3G_E_NOMEM, "cudaMalloc of %ld x %zu bytes failed", (long)(n), sizeof(T)); \
    } while (0)

template <typename T>
static int upload(i3g_ctx *c, T *&dst, const std::vector<T> &src)
{
    ALLOC(dst, T, (long)src.size());
    if (!src.empty()) I3G_CUDA(cudaMemcpyAsync(dst, src.data(), sizeof(T) * src.size(), cudaMemcpyHostToDevice, c->st));
    I3G_CUDA(cudaStreamSynchronize(c->st));
    return 0;
}

// one-dimensional transfer stencil (host, FP64, the reference's expressions)
static void build_transfer(const double *gf, int nf, const double *gc, int nc, int stag, Transfer1D &t,
                           std::vector<int> &ha, std::vector<double> &hw0, std::vector<double> &hw1,
                           std::vector<int> &gptr, std::vector<int> &gfv, std::vector<double> &gwv)
{
    ha.assign(nf, 0); hw0.assign(nf, 0); hw1.assign(nf, 0);
    for (int m = 0; m < nf; m++) {
        long a = (m - 2) / 2 + 2;
        if (m < 3) a = m;
        if (m > nf - 4) a = nc - (nf - m);
        double d;
        if (stag == kStagLine || stag == kStagAbs) {
            if (a > nc - 2) a = nc - 2;
            d = gc[a + 1] - gc[a];
        } else if (stag == kStagMid) {
            if (a > nc - 3) a = nc - 3;
            if (m + 1 < nf && (gf[m] + gf[m + 1]) / 2.0 < (gc[a] + gc[a + 1]) / 2.0 && a > 0) a -= 1;
            d = (gc[a + 2] - gc[a]) / 2.0;
        } else {
            if (a > nc - 2) a = nc - 2;
            if (m > 0 && (gf[m] + gf[m - 1]) / 2.0 < (gc[a] + gc[a - 1]) / 2.0 && a > 1) a -= 1;
            d = (gc[a + 1] - gc[a - 1]) / 2.0;
        }
        double w[2];
        for (int q = 0; q < 2; q++) {
            long k = a + q;
            double dd;
            if (stag == kStagAbs) {
                dd = (gc[k] - gf[m]) / d;
                dd = 1.0 - (dd >= 0 ? dd : -dd);
            } else {
                if (stag == kStagLine) dd = (gc[k] - gf[m]) / d;
                else if (stag == kStagMid) dd = (m + 1 < nf && k + 1 < nc) ? (gc[k] + gc[k + 1] - gf[m] - gf[m + 1]) / 2.0 / d : 0.0;
                else dd = (m > 0 && k > 0) ? (gc[k] + gc[k - 1] - gf[m] - gf[m - 1]) / 2.0 / d : 0.0;
                if (k == a) dd = -dd;
                dd = 1.0 - dd;
            }
            w[q] = dd;
        }
        ha[m] = (int)a; hw0[m] = w[0]; hw1[m] = w[1];
    }
    gptr.assign(nc + 1, 0);
    std::vector<std::vector<std::pair<int, double>>> lists(nc);
    for (int m = 0; m < nf; m++) {
        if (ha[m] >= 0 && ha[m] < nc) lists[ha[m]].push_back({m, hw0[m]});
        if (ha[m] + 1 >= 0 && ha[m] + 1 < nc) lists[ha[m] + 1].push_back({m, hw1[m]});
    }
    gfv.clear(); gwv.clear();
    for (int q = 0; q < nc; q++) {
        gptr[q] = (int)gfv.size();
        for (auto &e : lists[q]) { gfv.push_back(e.first); gwv.push_back(e.second); }
    }
    gptr[nc] = (int)gfv.size();
    t.nf = nf; t.nc = nc;
}

static int upload_transfer(i3g_ctx *c, const double *gf, int nf, const double *gc, int nc, int stag, Transfer1D &t)
{
    std::vector<int> ha, gptr, gfv;
    std::vector<double> w0, w1, gwv;
    build_transfer(gf, nf, gc, nc, stag, t, ha, w0, w1, gptr, gfv, gwv);
    int rc;
    if ((rc = upload(c, t.a, ha)) || (rc = upload(c, t.w0, w0)) || (rc = upload(c, t.w1, w1)) ||
        (rc = upload(c, t.gptr, gptr)) || (rc = upload(c, t.gf, gfv)) || (rc = upload(c, t.gw, gwv)))
        return rc;
    return 0;
}

// staggering of each unknown along x, y, z (P cell centre; V along its own axis on grid lines)
static const int kStag[4][3] = {{kStagCell, kStagCell, kStagCell}, {kStagLine, kStagMid, kStagMid},
                                {kStagMid, kStagLine, kStagMid}, {kStagMid, kStagMid, kStagLine}};

// inverse spacing tables: [0] 1/(g[i]-g[i-1]) at i >= 1, [1] 1/(g[i+1]-g[i-1]) at 1 <= i <= n-2
static void inv_tables(const double *g, int n, std::vector<double> &ic, std::vector<double> &is)
{
    ic.assign(n + 1, 0.0); is.assign(n + 1, 0.0);
    for (int i = 1; i < n; i++) ic[i] = 1.0 / (g[i] - g[i - 1]);
    for (int i = 1; i < n - 1; i++) is[i] = 1.0 / (g[i + 1] - g[i - 1]);
}

static int upload_f32_scaled(i3g_ctx *c, float *&dst, const std::vector<double> &src, double scale)
{
    std::vector<float> f(src.size());
    for (size_t i = 0; i < src.size(); i++) f[i] = (float)(src[i] * scale);
    return upload(c, dst, f);
}

// Boundary rows: flatten chains to an interior partner; reject cycles, partners that are
// not rows of the system and interior rows whose stencil leaves the grid.
static int build_bc(i3g_ctx *c)
{
    const i3g_model &m = c->m;
    const long N0 = c->nodenum;
    long ntot = 0, mgp[I3G_MAXLEV];
    for (int l = 0; l < c->nlev; l++) { mgp[l] = ntot; ntot += c->lev[l].n; }
    // row -> bc record index
    std::vector<int> rid(4 * ntot, -1);
    for (long b = 0; b < m.bondnum; b++) {
        long row = m.bond_row[b];
        if (row < 0) return set_error(c, I3G_E_BC, "negative boundary row %ld", row);
        if (row >= 8 * N0) continue;   // temperature rows are handled by the heat solver
        if (row >= 4 * ntot) return set_error(c, I3G_E_BC, "boundary row %ld beyond the multigrid levels", row);
        rid[row] = (int)b;
    }
    for (int l = 0; l < c->nlev; l++) {
        Level &L = c->lev[l];
        std::vector<uint8_t> mask(L.n, 0);
        std::vector<int> node[4], pnode[4], depth[4], onode[4], ocomp[4];
        std::vector<double> cc[4], kk[4], oc[4], ok[4];
        for (long q = 0; q < L.n; q++) {
            const int j = (int)(q % L.ny), i = (int)((q / L.ny) % L.nx), k = (int)(q / ((long)L.ny * L.nx));
            for (int v = 0; v < 4; v++) {
                long row = (mgp[l] + q) * 4 + v;
                if (!row_exists(v, i, j, k, L.nx, L.ny, L.nz)) continue;
                int b = rid[row];
                if (l == 0) {
                    if (v) c->nvel += 1;
                    else if (b < 0) c->ncont += 1;
                }
                if (b < 0) {
                    // interior row: its stencil must stay on the grid
                    bool ok_ = true;
                    if (v == 1) ok_ = i >= 1 && i <= L.nx - 2 && j >= 1 && j <= L.ny - 3 && k >= 1 && k <= L.nz - 3;
                    if (v == 2) ok_ = i >= 1 && i <= L.nx - 3 && j >= 1 && j <= L.ny - 2 && k >= 1 && k <= L.nz - 3;
                    if (v == 3) ok_ = i >= 1 && i <= L.nx - 3 && j >= 1 && j <= L.ny - 3 && k >= 1 && k <= L.nz - 2;
                    if (!ok_) return set_error(c, I3G_E_BC, "level %d: row %d at (%d,%d,%d) has no boundary condition but its stencil leaves the grid", l, v, i, j, k);
                    continue;
                }
                mask[q] |= (uint8_t)(1 << v);
                node[v].push_back((int)q);
                // original partner
                long p1 = m.bond_partner1[b];
                if (p1 > 0) {
                    long pr = p1 - 1;
                    if (pr / 4 < mgp[l] || pr / 4 >= mgp[l] + L.n) return set_error(c, I3G_E_BC, "boundary row %ld partners row %ld on another level", row, pr);
                    onode[v].push_back((int)(pr / 4 - mgp[l])); ocomp[v].push_back((int)(pr % 4));
                } else { onode[v].push_back(-1); ocomp[v].push_back(0); }
                oc[v].push_back((double)m.bond_c[b]);
                ok[v].push_back((double)m.bond_k[b]);
                // flatten
                double chc[kMaxBcDepth], chk[kMaxBcDepth];
                int dep = 0;
                long cur = row;
                int pn = -1;
                for (;;) {
                    int bb = rid[cur];
                    if (dep >= kMaxBcDepth) return set_error(c, I3G_E_BC, "boundary chain from row %ld longer than %d (cycle?)", row, kMaxBcDepth);
                    chc[dep] = (double)m.bond_c[bb];
                    long q1 = m.bond_partner1[bb];
                    chk[dep] = q1 > 0 ? (double)m.bond_k[bb] : 0.0;
                    dep++;
                    if (q1 <= 0) { pn = -1; break; }
                    long pr = q1 - 1;
                    if (pr % 4 != v) return set_error(c, I3G_E_BC, "boundary row %ld partners another component", row);
                    long pq = pr / 4 - mgp[l];
                    const int pj = (int)(pq % L.ny), pi = (int)((pq / L.ny) % L.nx), pk = (int)(pq / ((long)L.ny * L.nx));
                    if (!row_exists(v, pi, pj, pk, L.nx, L.ny, L.nz)) { pn = -1; break; }   // value stays 0
                    if (rid[pr] < 0) { pn = (int)pq; break; }
                    cur = pr;
                }
                pnode[v].push_back(pn);
                depth[v].push_back(dep);
                for (int d = 0; d < kMaxBcDepth; d++) {
                    cc[v].push_back(d < dep ? chc[d] : 0.0);
                    kk[v].push_back(d < dep ? chk[d] : 0.0);
                }
            }
        }
        // In-kernel boundary rows (k_relax_vel_bc, k_relax_p_bc).  The finalising kernel of a
        // velocity component updates its colour-1 rows (i + j + k odd), which read only their even
        // neighbours; the pressure kernel updates every pressure row and reads no pressure.  Per
        // boundary row b with partner p, R = the kernel's rows that read b:
        //   p updated by the kernel: writer p, admitted if R is within {p};
        //   otherwise (p final or constant): no reader -> extra blocks; one reader r -> writer r;
        // two or more readers: the component keeps the separate pass.
        int na[4] = {-1, -1, -1, -1};
        std::vector<int> first[4], writer[4];
        auto is_row = [&](long q, int v) {
            const int j = (int)(q % L.ny), i = (int)((q / L.ny) % L.nx), k = (int)(q / ((long)L.ny * L.nx));
            return row_exists(v, i, j, k, L.nx, L.ny, L.nz) && !(mask[q] & (1 << v));
        };
        auto odd = [&](long q) {
            const int j = (int)(q % L.ny), i = (int)((q / L.ny) % L.nx), k = (int)(q / ((long)L.ny * L.nx));
            return ((i + j + k) & 1) != 0;
        };
        for (int v = 0; c->fuse && v < 4; v++) {
            const int nb = (int)node[v].size();
            std::vector<int> A, Bo, wr(nb, -1);
            bool admit = true;
            for (int e = 0; e < nb && admit; e++) {
                const int p = pnode[v][e];
                int R[6], nr = 0;
                if (v > 0) {
                    const long q = node[v][e];
                    const int j = (int)(q % L.ny), i = (int)((q / L.ny) % L.nx), k = (int)(q / ((long)L.ny * L.nx));
                    const int di[6] = {-1, 1, 0, 0, 0, 0}, dj[6] = {0, 0, -1, 1, 0, 0}, dk[6] = {0, 0, 0, 0, -1, 1};
                    for (int d = 0; d < 6; d++) {
                        const int i2 = i + di[d], j2 = j + dj[d], k2 = k + dk[d];
                        if (i2 < 0 || j2 < 0 || k2 < 0 || i2 >= L.nx || j2 >= L.ny || k2 >= L.nz) continue;
                        const long r = ((long)k2 * L.nx + i2) * L.ny + j2;
                        if (is_row(r, v) && odd(r)) R[nr++] = (int)r;
                    }
                }
                if (p >= 0 && is_row(p, v) && (v == 0 || odd(p))) {
                    for (int q = 0; q < nr; q++)
                        if (R[q] != p) admit = false;
                    wr[e] = p;
                    A.push_back(e);
                } else if (nr == 0) {
                    Bo.push_back(e);
                } else if (nr == 1) {
                    wr[e] = R[0];
                    A.push_back(e);
                } else {
                    admit = false;
                }
            }
            if (!admit) continue;
            std::stable_sort(A.begin(), A.end(), [&](int x, int y) { return wr[x] < wr[y]; });
            std::vector<int> perm(A);
            perm.insert(perm.end(), Bo.begin(), Bo.end());
            auto permute = [&](auto &vec, int width) {
                auto old = vec;
                for (size_t e = 0; e < perm.size(); e++)
                    for (int w = 0; w < width; w++) vec[e * width + w] = old[(size_t)perm[e] * width + w];
            };
            permute(node[v], 1); permute(pnode[v], 1); permute(depth[v], 1); permute(onode[v], 1);
            permute(ocomp[v], 1); permute(oc[v], 1); permute(ok[v], 1); permute(wr, 1);
            permute(cc[v], kMaxBcDepth); permute(kk[v], kMaxBcDepth);
            na[v] = (int)A.size();
            if (na[v] > 0) {
                writer[v].assign(wr.begin(), wr.begin() + na[v]);
                first[v].assign(L.n, -1);
                for (int e = na[v] - 1; e >= 0; e--) {
                    first[v][wr[e]] = e;
                    mask[wr[e]] |= (uint8_t)(16 << v);
                }
            }
        }
        if (getenv("I3G_TRACE"))
            for (int v = 0; v < 4; v++)
                fprintf(stderr, "i3g: level %d component %d: %zu boundary rows, %s (%d by a row's thread)\n", l, v,
                        node[v].size(), na[v] >= 0 ? "in-kernel" : "separate pass", na[v]);
        int rc = upload(c, L.bc, mask);
        if (rc) return rc;
        for (int v = 0; v < 4; v++) {
            BcList &B = L.bcl[v];
            B.n = (int)node[v].size();
            B.na = na[v];
            if (na[v] > 0 && ((rc = upload(c, B.first, first[v])) || (rc = upload(c, B.writer, writer[v])))) return rc;
            if ((rc = upload(c, B.node, node[v])) || (rc = upload(c, B.pnode, pnode[v])) ||
                (rc = upload(c, B.depth, depth[v])) || (rc = upload(c, B.c, cc[v])) || (rc = upload(c, B.k, kk[v])) ||
                (rc = upload(c, B.onode, onode[v])) || (rc = upload(c, B.ocomp, ocomp[v])) ||
                (rc = upload(c, B.oc, oc[v])) || (rc = upload(c, B.ok, ok[v])))
                return rc;
        }
    }
    return 0;
}

int stokes_alloc(i3g_ctx *c)
{
    // size limit of the one-block V-cycle tail (I3G_TAIL_NODES=0 turns it off)
    if (const char *e = getenv("I3G_TAIL_NODES")) c->tail_nodes = atol(e);
    // cooperative coarse-level kernel: levels up to this size (I3G_COOP_NODES, 0 = off) run in
    // one launch over the whole grid; its size is what every SM can hold at once
    if (const char *e = getenv("I3G_COOP_NODES")) c->coop_nodes = atol(e);
    // CTAs of the tail (I3G_TAIL_CLUSTER, 1: the one-block kernel; 2..16: one thread-block cluster)
    if (const char *e = getenv("I3G_TAIL_CLUSTER")) c->tail_cluster = std::max(1, std::min(16, atoi(e)));
    // I3G_FUSE: 0 one launch per boundary pass, residual part and transfer component; 1 boundary
    // rows in-kernel on levels >= 1 (default); 3 on level 0 too
    if (const char *e = getenv("I3G_FUSE")) c->fuse = atoi(e);
    if (const char *e = getenv("I3G_ND_SCHUR")) c->nd_schur = std::max(0, atoi(e));
    if (c->tail_cluster > 8) {
        I3G_CUDA(cudaFuncSetAttribute(k_vcycle_cluster<float>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
        I3G_CUDA(cudaFuncSetAttribute(k_vcycle_cluster<double>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    }
    {
        int dev = 0, sms = 0, coop = 0, a = 0, b = 0;
        I3G_CUDA(cudaGetDevice(&dev));
        I3G_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        I3G_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
        I3G_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_vcycle_coop<float>, kCoopThreads, 0));
        I3G_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_vcycle_coop<double>, kCoopThreads, 0));
        c->coop_blocks = coop ? sms * std::min(a, b) : 0;
        I3G_CUDA(cudaMalloc((void **)&c->dbar, 2 * sizeof(unsigned)));
        I3G_CUDA(cudaMalloc((void **)&c->dbar_err, sizeof(int)));
        I3G_CUDA(cudaMemsetAsync(c->dbar, 0, 2 * sizeof(unsigned), c->st));
        I3G_CUDA(cudaMemsetAsync(c->dbar_err, 0, sizeof(int), c->st));
    }
    // level geometry (gridcheck, load3mg.c:1220-1282)
    for (int l = 0; l < c->nlev; l++) {
        Level &L = c->lev[l];
        if (l == 0) { L.nx = (int)c->m.xnumx; L.ny = (int)c->m.ynumy; L.nz = (int)c->m.znumz; }
        else {
            L.nx = (c->lev[l - 1].nx - 5) / 2 + 5;
            L.ny = (c->lev[l - 1].ny - 5) / 2 + 5;
            L.nz = (c->lev[l - 1].nz - 5) / 2 + 5;
        }
        if (L.nx < 5 || L.ny < 5 || L.nz < 5) return set_error(c, I3G_E_ARG, "level %d has fewer than 5 nodes along an axis", l);
        L.n = (long)L.nx * L.ny * L.nz;
        const long s = 1L << l;
        const double *g0[3] = {c->hgx, c->hgy, c->hgz};
        const int n0[3] = {(int)c->m.xnumx, (int)c->m.ynumy, (int)c->m.znumz};
        const int nl[3] = {L.nx, L.ny, L.nz};
        double **dst[3] = {&L.gx, &L.gy, &L.gz};
        for (int d = 0; d < 3; d++) {
            double *g = new double[nl[d]];
            g[0] = g0[d][0]; g[1] = g0[d][1]; g[2] = g0[d][2];
            g[nl[d] - 1] = g0[d][n0[d] - 1]; g[nl[d] - 2] = g0[d][n0[d] - 2]; g[nl[d] - 3] = g0[d][n0[d] - 3];
            for (int i = 3; i < nl[d] - 3; i++) g[i] = g0[d][(i - 2) * s + 2];
            *dst[d] = g;
        }
    }
    double hsum = 0;
    hsum = (c->m.xsize / (c->m.xnumx - 1) + c->m.ysize / (c->m.ynumy - 1) + c->m.zsize / (c->m.znumz - 1)) / 3.0;
    c->h_ref = hsum;
    for (int l = 0; l < c->nlev; l++) {
        Level &L = c->lev[l];
        const long n = L.n;
        if (l > 0) ALLOC(L.nu, float, n);
        for (int v = 0; v < 4; v++) {
            ALLOC(L.d.u[v], double, n); ALLOC(L.d.f[v], double, n); ALLOC(L.d.r[v], double, n);
            ALLOC(L.s.u[v], float, n); ALLOC(L.s.f[v], float, n); ALLOC(L.s.r[v], float, n);
            I3G_CUDA(cudaMemsetAsync(L.d.u[v], 0, n * 8, c->st)); I3G_CUDA(cudaMemsetAsync(L.d.f[v], 0, n * 8, c->st));
            I3G_CUDA(cudaMemsetAsync(L.d.r[v], 0, n * 8, c->st));
            I3G_CUDA(cudaMemsetAsync(L.s.u[v], 0, n * 4, c->st)); I3G_CUDA(cudaMemsetAsync(L.s.f[v], 0, n * 4, c->st));
            I3G_CUDA(cudaMemsetAsync(L.s.r[v], 0, n * 4, c->st));
        }
        ALLOC(L.d.etac, double, n); ALLOC(L.d.etaxy, double, n); ALLOC(L.d.etaxz, double, n); ALLOC(L.d.etayz, double, n);
        ALLOC(L.s.etac, float, n); ALLOC(L.s.etaxy, float, n); ALLOC(L.s.etaxz, float, n); ALLOC(L.s.etayz, float, n);
        ALLOC(L.s.nd, float, n);
        ALLOC(L.d.nd, float, n);
        const double *g[3] = {L.gx, L.gy, L.gz};
        const int nn[3] = {L.nx, L.ny, L.nz};
        double **di[3][2] = {{&L.d.ix[0], &L.d.ix[1]}, {&L.d.iy[0], &L.d.iy[1]}, {&L.d.iz[0], &L.d.iz[1]}};
        float **fi[3][2] = {{&L.s.ix[0], &L.s.ix[1]}, {&L.s.iy[0], &L.s.iy[1]}, {&L.s.iz[0], &L.s.iz[1]}};
        for (int d = 0; d < 3; d++) {
            std::vector<double> ic, is;
            inv_tables(g[d], nn[d], ic, is);
            int rc;
            if ((rc = upload(c, *di[d][0], ic)) || (rc = upload(c, *di[d][1], is)) ||
                (rc = upload_f32_scaled(c, *fi[d][0], ic, c->h_ref)) || (rc = upload_f32_scaled(c, *fi[d][1], is, c->h_ref)))
                return rc;
        }
    }
    for (int l = 0; l + 1 < c->nlev; l++) {
        Level &F = c->lev[l], &Cc = c->lev[l + 1];
        const double *gf[3] = {F.gx, F.gy, F.gz}, *gc[3] = {Cc.gx, Cc.gy, Cc.gz};
        const int nf[3] = {F.nx, F.ny, F.nz}, ncn[3] = {Cc.nx, Cc.ny, Cc.nz};
        for (int d = 0; d < 3; d++)
            for (int s = 0; s < 4; s++) {
                int rc = upload_transfer(c, gf[d], nf[d], gc[d], ncn[d], s, F.tr[d][s]);
                if (rc) return rc;
            }
    }
    c->red_blocks = 2 * 148;
    ALLOC(c->dred, double, (long)c->red_blocks * kRedQ + 16);
    if (!c->hred) I3G_CUDA(cudaMallocHost((void **)&c->hred, 64 * sizeof(double)));
    int rc = build_bc(c);
    if (rc) return rc;
    I3G_CUDA(cudaStreamSynchronize(c->st));
    return 0;
}

static void kry_free(i3g_ctx *c);

void stokes_free(i3g_ctx *c)
{
    cudaFree(c->dbar);
    cudaFree(c->dbar_err);
    c->dbar = nullptr;
    c->dbar_err = nullptr;
    stokes_graph_free(c);
    kry_free(c);
    for (int h = 0; h < 3; h++)
        for (int v = 0; v < 4; v++) { cudaFree(c->hist[h][v]); c->hist[h][v] = nullptr; }
    for (int l = 0; l < c->nlev; l++) {
        Level &L = c->lev[l];
        delete[] L.gx; delete[] L.gy; delete[] L.gz;
        L.gx = L.gy = L.gz = nullptr;
        if (l > 0) cudaFree(L.nu);
        cudaFree(L.bc);
        for (int v = 0; v < 4; v++) {
            cudaFree(L.d.u[v]); cudaFree(L.d.f[v]); cudaFree(L.d.r[v]);
            cudaFree(L.s.u[v]); cudaFree(L.s.f[v]); cudaFree(L.s.r[v]);
            BcList &B = L.bcl[v];
            cudaFree(B.node); cudaFree(B.pnode); cudaFree(B.depth); cudaFree(B.c); cudaFree(B.k);
            cudaFree(B.onode); cudaFree(B.ocomp); cudaFree(B.oc); cudaFree(B.ok); cudaFree(B.first); cudaFree(B.writer);
        }
        cudaFree(L.d.etac); cudaFree(L.d.etaxy); cudaFree(L.d.etaxz); cudaFree(L.d.etayz); cudaFree(L.d.nd);
        cudaFree(L.s.etac); cudaFree(L.s.etaxy); cudaFree(L.s.etaxz); cudaFree(L.s.etayz); cudaFree(L.s.nd);
        for (int a = 0; a < 2; a++) {
            cudaFree(L.d.ix[a]); cudaFree(L.d.iy[a]); cudaFree(L.d.iz[a]);
            cudaFree(L.s.ix[a]); cudaFree(L.s.iy[a]); cudaFree(L.s.iz[a]);
        }
        for (int d = 0; d < 3; d++)
            for (int s = 0; s < 4; s++) {
                Transfer1D &t = L.tr[d][s];
                cudaFree(t.a); cudaFree(t.w0); cudaFree(t.w1); cudaFree(t.gptr); cudaFree(t.gf); cudaFree(t.gw);
            }
    }
    cudaFree(c->dred);
    if (c->hred) cudaFreeHost(c->hred);
    c->hred = nullptr;
}

#define LAUNCH(kern, grid, block, ...)                                                     \
    do {                                                                                   \
        launch_pdl(c->st, kern, dim3(grid), dim3(block), __VA_ARGS__);                     \
        c->launches++;                                                                     \
    } while (0)

int stokes_setup(i3g_ctx *c)
{
    Level &L0 = c->lev[0];
    // restricted viscosity of coarse levels
    for (int l = 1; l < c->nlev; l++) {
        Level &F = c->lev[l - 1], &Cc = c->lev[l];
        const float *nuf = l == 1 ? c->lev[0].nu : F.nu;
        LAUNCH(k_nu_restrict, nblk(Cc.n), 256, nuf, F.nx, F.ny, F.nz, Cc.nu, Cc.nx, Cc.ny, Cc.nz,
               trview(F.tr[0][kStagAbs]), trview(F.tr[1][kStagAbs]), trview(F.tr[2][kStagAbs]), c->p.viscmod);
    }
    double emin = c->p.nubeg, emax = c->p.nuend;
    c->eta_ref = std::sqrt(emin * emax);
    for (int l = 0; l < c->nlev; l++) {
        Level &L = c->lev[l];
        EtaArgs a;
        a.nx = L.nx; a.ny = L.ny; a.nz = L.nz; a.lev0 = l == 0; a.viscmod = c->p.viscmod;
        a.nu = L.nu; a.nxx = c->nxx; a.nxy = c->nxy; a.nxz = c->nxz; a.nyz = c->nyz;
        a.nubeg = c->p.nubeg; a.nuend = c->p.nuend;
        a.etac = L.d.etac; a.etaxy = L.d.etaxy; a.etaxz = L.d.etaxz; a.etayz = L.d.etayz;
        a.nd = L.d.nd;
        LAUNCH(k_eta, nblk(L.n), 256, a);
        LAUNCH(k_eta_f32, nblk(L.n), 256, L.n, L.d.etac, L.d.etaxy, L.d.etaxz, L.d.etayz, (const float *)a.nd,
               L.s.etac, L.s.etaxy, L.s.etaxz, L.s.etayz, L.s.nd, 1.0 / c->eta_ref);
        if (c->nd_schur > 0)
            LAUNCH(k_nd_schur, nblk(L.n), 256, view<double>(L, L.d), L.s.nd, 1.0 / c->eta_ref, (double)c->nd_schur);
        for (int v = 0; v < 4; v++) {
            I3G_CUDA(cudaMemsetAsync(L.d.u[v], 0, L.n * 8, c->st));
            I3G_CUDA(cudaMemsetAsync(L.d.f[v], 0, L.n * 8, c->st));
            I3G_CUDA(cudaMemsetAsync(L.d.r[v], 0, L.n * 8, c->st));
        }
    }
    View<double> V0 = view<double>(L0, L0.d);
    LAUNCH(k_rhs0, nblk(L0.n), 256, V0, (const float *)c->ro, c->m.gxkoef, c->m.gykoef, c->m.gzkoef);
    for (int v = 0; v < 4; v++) {
        BcList &B = L0.bcl[v];
        if (B.n) LAUNCH(k_bc_rhs, nblk(B.n), 256, L0.d.f[v], B.n, (const int *)B.node, (const double *)B.oc);
    }
    LAUNCH(k_load_sol, nblk(L0.n), 256, V0, (const double *)c->pr, (const float *)c->vx, (const float *)c->vy, (const float *)c->vz);
    I3G_CUDA(cudaGetLastError());
    c->stokes_ready = true;
    return 0;
}

// ------------------------------------------------------------------------------------
// solver drivers
// ------------------------------------------------------------------------------------
template <typename T>
static Fields<T> &fields(Level &L);
template <>
Fields<double> &fields<double>(Level &L) { return L.d; }
template <>
Fields<float> &fields<float>(Level &L) { return L.s; }

template <typename T>
static void bc_apply(i3g_ctx *c, int l, int v, bool use_c)
{
    Level &L = c->lev[l];
    BcList &B = L.bcl[v];
    if (!B.n) return;
    LAUNCH(k_bc_apply<T>, nblk(B.n), 256, fields<T>(L).u[v], B.n, (const int *)B.node, (const int *)B.pnode,
           (const int *)B.depth, (const double *)B.c, (const double *)B.k, (int)use_c);
}

static BcDev bcdev(const BcList &B)
{
    return BcDev{B.n, B.na, B.node, B.pnode, B.depth, B.onode, B.ocomp, B.first, B.writer, B.c, B.k, B.ok};
}

template <typename T>
static void residual_t(i3g_ctx *c, int l)
{
    Level &L = c->lev[l];
    View<T> V = view<T>(L, fields<T>(L));
    if (c->fuse) {
        BcDev4 B;
        long nb = 0;
        for (int v = 0; v < 4; v++) { B.b[v] = bcdev(L.bcl[v]); nb += L.bcl[v].n; }
        const unsigned rows = nblk(L.n);
        LAUNCH(k_residual_bc<T>, rows + nblk(nb), 256, V, B, rows);
        return;
    }
    LAUNCH(k_residual<T>, nblk(L.n), 256, V);
    for (int v = 0; v < 4; v++) {
        BcList &B = L.bcl[v];
        if (B.n) LAUNCH(k_bc_residual<T>, nblk(B.n), 256, V, v, B.n, (const int *)B.node, (const int *)B.onode,
                        (const int *)B.ocomp, (const double *)B.ok);
    }
}

// nsweeps multicolour sweeps (gausmat4 update formula, move3mg.c:3087-3131)
template <typename T>
static void smooth_t(i3g_ctx *c, int l, int nsweeps, bool homogeneous, bool with_residual)
{
    Level &L = c->lev[l];
    View<T> V = view<T>(L, fields<T>(L));
    const long total = (long)((L.ny + 1) / 2) * L.nx * L.nz;
    const T v0 = (T)c->p.v0koef, p0 = (T)c->p.p0koef;
    const bool use_c = l == 0 && !homogeneous;
    const unsigned rows = nblk(total), prows = nblk(L.n);
    // in-kernel boundary rows: coarse levels always (latency-bound launches), level 0 with
    // I3G_FUSE=3 (its launches are bandwidth-bound and the writers' loads lengthen them)
    const bool inkernel = c->fuse && (l > 0 || c->fuse >= 3);
    // colour 1 of a component, with its boundary rows when set-up admitted them in-kernel
#define LAST_COLOUR(V_)                                                                                 \
    do {                                                                                                \
        const BcList &B = L.bcl[V_];                                                                    \
        if (inkernel && B.na >= 0)                                                                      \
            LAUNCH((k_relax_vel_bc<T, V_>), rows + nblk(B.n - B.na), 256, V, v0, bcdev(B), (int)use_c, rows); \
        else {                                                                                          \
            LAUNCH((k_relax_vel<T, V_>), rows, 256, V, 1, v0);                                          \
            bc_apply<T>(c, l, V_, use_c);                                                               \
        }                                                                                               \
    } while (0)
    for (int s = 0; s < nsweeps; s++) {
        LAUNCH((k_relax_vel<T, 1>), rows, 256, V, 0, v0);
        LAST_COLOUR(1);
        LAUNCH((k_relax_vel<T, 2>), rows, 256, V, 0, v0);
        LAST_COLOUR(2);
        LAUNCH((k_relax_vel<T, 3>), rows, 256, V, 0, v0);
        LAST_COLOUR(3);
        const BcList &B = L.bcl[0];
        if (inkernel && B.na >= 0)
            LAUNCH(k_relax_p_bc<T>, prows + nblk(B.n - B.na), 256, V, p0, bcdev(B), (int)use_c, prows);
        else {
            LAUNCH(k_relax_p<T>, prows, 256, V, p0);
            bc_apply<T>(c, l, 0, use_c);
        }
    }
#undef LAST_COLOUR
    if (with_residual) residual_t<T>(c, l);
}

template <typename T>
static void restrict_t(i3g_ctx *c, int l)
{
    Level &F = c->lev[l - 1], &Cc = c->lev[l];
    View<T> VF = view<T>(F, fields<T>(F)), VC = view<T>(Cc, fields<T>(Cc));
    if (c->fuse) {
        Tr4 R;
        for (int v = 0; v < 4; v++)
            for (int ax = 0; ax < 3; ax++) R.t[v][ax] = trview(F.tr[ax][kStag[v][ax]]);
        if constexpr (std::is_same<T, float>::value)
            LAUNCH(k_restrict4_f32, dim3(nblk(4 * Cc.n), 4), 256, VF, VC, R);
        else
            LAUNCH(k_restrict4<T>, dim3(nblk(Cc.n), 4), 256, VF, VC, R);
        return;
    }
#define RST(V_) LAUNCH((k_restrict<T, V_>), nblk(Cc.n), 256, VF, VC, trview(F.tr[0][kStag[V_][0]]), \
                       trview(F.tr[1][kStag[V_][1]]), trview(F.tr[2][kStag[V_][2]]))
    RST(1); RST(2); RST(3); RST(0);
#undef RST
}

template <typename T>
static void prolong_t(i3g_ctx *c, int l)
{
    Level &F = c->lev[l - 1], &Cc = c->lev[l];
    View<T> VF = view<T>(F, fields<T>(F)), VC = view<T>(Cc, fields<T>(Cc));
    const T kv = (T)c->p.v1koef, kp = (T)c->p.p1koef;
    if (c->fuse) {
        Tr4 R;
        for (int v = 0; v < 4; v++)
            for (int ax = 0; ax < 3; ax++) R.t[v][ax] = trview(F.tr[ax][kStag[v][ax]]);
        LAUNCH(k_prolong4<T>, dim3(nblk(F.n), 4), 256, VF, VC, R, kv, kp);
        return;
    }
#define PRL(V_, K_) LAUNCH((k_prolong<T, V_>), nblk(F.n), 256, VF, VC, trview(F.tr[0][kStag[V_][0]]), \
                           trview(F.tr[1][kStag[V_][1]]), trview(F.tr[2][kStag[V_][2]]), K_)
    PRL(1, kv); PRL(2, kv); PRL(3, kv); PRL(0, kp);
#undef PRL
}

// First level of the one-block tail: the coarsest levels (>= 1) with at most tail_nodes nodes;
// multinum + 1 when none qualifies.  With the cooperative coarse-level kernel enabled
// (coop_nodes > 0) the same rule applies with its larger size limit, and all those levels run in
// that kernel instead.
static int tail_start(const i3g_ctx *c, int multinum)
{
    const long lim = c->coop_nodes > 0 && c->coop_blocks > 0 ? c->coop_nodes : c->tail_nodes;
    int lc = multinum + 1;
    for (int l = multinum; l >= 1 && l > multinum - kTailMax; l--) {
        if (c->lev[l].n > lim) break;
        lc = l;
    }
    return lc;
}

template <typename T>
static void tail_launch(i3g_ctx *c, int lc, int multinum)
{
    TailArgs<T> a;
    memset(&a, 0, sizeof a);
    a.nl = multinum - lc + 1;
    a.v0 = (T)c->p.v0koef; a.p0 = (T)c->p.p0koef; a.kv = (T)c->p.v1koef; a.kp = (T)c->p.p1koef;
    for (int q = 0; q < a.nl; q++) {
        Level &L = c->lev[lc + q];
        TailLevel<T> &TL = a.L[q];
        TL.v = view<T>(L, fields<T>(L));
        for (int v = 0; v < 4; v++) {
            const BcList &B = L.bcl[v];
            TL.bc[v] = bcdev(B);
            if (q + 1 < a.nl)
                for (int ax = 0; ax < 3; ax++) TL.tr[v][ax] = trview(L.tr[ax][kStag[v][ax]]);
        }
        TL.down = c->p.multinnn[0][lc + q];
        TL.up = c->p.multinnn[1][lc + q];
    }
    if (c->coop_nodes > 0 && c->coop_blocks > 0) {
        // one cooperative launch over all resident CTAs; the barrier counter starts at zero
        cudaMemsetAsync(c->dbar, 0, 2 * sizeof(unsigned), c->st);
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)c->coop_blocks);
        cfg.blockDim = dim3(kCoopThreads);
        cfg.stream = c->st;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeCooperative;
        at[0].val.cooperative = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        cudaLaunchKernelEx(&cfg, k_vcycle_coop<T>, a, GridTeam{c->dbar, c->dbar + 1, c->dbar_err});
        c->launches++;
        return;
    }
    if (c->tail_cluster > 1) {
        // one cluster of tail_cluster CTAs (non-portable sizes above 8 are enabled at set-up)
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)c->tail_cluster);
        cfg.blockDim = dim3(kTailThreads);
        cfg.stream = c->st;
        cudaLaunchAttribute at[2];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = (unsigned)c->tail_cluster;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        at[1].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = at;
        cfg.numAttrs = pdl_enabled() ? 2 : 1;
        cudaLaunchKernelEx(&cfg, k_vcycle_cluster<T>, a);
        c->launches++;
        return;
    }
    LAUNCH(k_vcycle_tail<T>, 1, kTailThreads, a);
}

// V-cycle with the schedule of move3mg.c:2173-2213; the small coarse levels run in the
// one-block tail kernel.
template <typename T>
static void vcycle_t(i3g_ctx *c, int multinum, bool homogeneous)
{
    const int lc = tail_start(c, multinum);
    for (int l = 0; l < multinum && l < lc; l++) {
        const int n = c->p.multinnn[0][l];
        if (n > 0) smooth_t<T>(c, l, n, homogeneous, true);
        else residual_t<T>(c, l);
        restrict_t<T>(c, l + 1);
    }
    if (lc <= multinum) tail_launch<T>(c, lc, multinum);
    for (int l = std::min(lc, multinum); l > 0; l--) {
        const int n = c->p.multinnn[1][l];
        if (n > 0 && l != lc) smooth_t<T>(c, l, n, homogeneous, false);
        prolong_t<T>(c, l);
    }
    if (c->p.multinnn[1][0] > 0) smooth_t<T>(c, 0, c->p.multinnn[1][0], homogeneous, false);
}

int stokes_residual(i3g_ctx *c, int level) { residual_t<double>(c, level); I3G_CUDA(cudaGetLastError()); return 0; }
int stokes_smooth(i3g_ctx *c, int level, int nsweeps) { smooth_t<double>(c, level, nsweeps, false, true); I3G_CUDA(cudaGetLastError()); return 0; }
int stokes_restrict(i3g_ctx *c, int level) { restrict_t<double>(c, level); I3G_CUDA(cudaGetLastError()); return 0; }
int stokes_prolong(i3g_ctx *c, int level) { prolong_t<double>(c, level); I3G_CUDA(cudaGetLastError()); return 0; }
int stokes_vcycle(i3g_ctx *c, int multinum) { vcycle_t<double>(c, multinum, false); I3G_CUDA(cudaGetLastError()); return 0; }

// relative residuals of the level-0 system (same definition as the oracle)
// norms into the pinned host mirror (enqueued; read after the stream has passed them)
static int relres_enqueue(i3g_ctx *c)
{
    Level &L = c->lev[0];
    View<double> V = view<double>(L, L.d);
    LAUNCH(k_relres_part<double>, c->red_blocks, kRedThreads, V, c->dred);
    LAUNCH(k_red_final, 1, 32 * kRedQ, (const double *)c->dred, c->red_blocks, kRedQ, c->dred + (long)c->red_blocks * kRedQ);
    I3G_CUDA(cudaMemcpyAsync(c->hred, c->dred + (long)c->red_blocks * kRedQ, kRedQ * sizeof(double), cudaMemcpyDeviceToHost, c->st));
    return 0;
}

static void relres_read(i3g_ctx *c, double *mom, double *cont)
{
    const double *q = c->hred;
    *mom = q[1] > 0 ? std::sqrt(q[0] / q[1]) : std::sqrt(q[0]);
    const double ncont = c->ncont, nvel = c->nvel;
    *cont = (ncont > 0 && q[3] > 0) ? std::sqrt(q[2] / ncont) * c->h_ref / std::sqrt(q[3] / nvel) : std::sqrt(q[2]);
}

int stokes_relres(i3g_ctx *c, double *mom, double *cont)
{
    int rc = relres_enqueue(c);
    if (rc) return rc;
    I3G_CUDA(cudaStreamSynchronize(c->st));
    relres_read(c, mom, cont);
    return 0;
}

// ------------------------------------------------------------------------------------
// mixed precision: FP32 multigrid on the correction inside FP64 defect correction
// ------------------------------------------------------------------------------------
__global__ void k_max_abs(const double *a, long n, double *part)
{
    pdl_enter();
    __shared__ double sh[8];
    double m = 0;
    for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) m = fmax(m, fabs(a[t]));
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); w++) m = fmax(m, sh[w]);
        part[blockIdx.x] = m;
    }
}

// Scale factors of the FP32 correction solve from the largest momentum residual r:
// e_v = sv * e_v', e_p = sp * e_p' with sv = r h^2 / eta_ref and sp = eta_ref sv / h, so that
// the scaled rows (viscosity / eta_ref, lengths / h) have right-hand sides of order one.
// scale = {momentum rhs factor, continuity rhs factor, sp, sv}
__global__ void k_scale(const double *part, int nparts, double h, double er, double *scale)
{
    pdl_enter();
    __shared__ double sh[32];
    double m = 0;
    for (int i = threadIdx.x; i < nparts; i += blockDim.x) m = fmax(m, part[i]);
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); w++) m = fmax(m, sh[w]);
        if (!(m > 0)) m = 1.0;
        const double sv = m * h * h / er, sp = er * sv / h;
        scale[0] = h * h / (er * sv);
        scale[1] = h / sv;
        scale[2] = sp;
        scale[3] = sv;
    }
}

// FP32 scaled right-hand side from the FP64 residual; boundary rows get 0
__global__ void k_to_f32(long n, const double *r0, const double *r1, const double *r2, const double *r3,
                         float *f0, float *f1, float *f2, float *f3, float *u0, float *u1, float *u2, float *u3,
                         const uint8_t *bc, const double *scale)
{
    pdl_enter();
    long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const double sm = scale[0], sc = scale[1];
    const uint8_t b = bc[t];
    f0[t] = (b & 1) ? 0.f : (float)(r0[t] * sc);
    f1[t] = (b & 2) ? 0.f : (float)(r1[t] * sm);
    f2[t] = (b & 4) ? 0.f : (float)(r2[t] * sm);
    f3[t] = (b & 8) ? 0.f : (float)(r3[t] * sm);
    u0[t] = 0.f; u1[t] = 0.f; u2[t] = 0.f; u3[t] = 0.f;
}

__global__ void k_add_correction(long n, double *x0, double *x1, double *x2, double *x3, const float *e0,
                                 const float *e1, const float *e2, const float *e3, const double *scale)
{
    pdl_enter();
    long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const double sp = scale[2], sv = scale[3];
    x0[t] += sp * (double)e0[t];
    x1[t] += sv * (double)e1[t];
    x2[t] += sv * (double)e2[t];
    x3[t] += sv * (double)e3[t];
}

// ------------------------------------------------------------------------------------
// after the solve: FP32 fields, pressure pinning, stresses, CFL (move3mg.c:2248-2632)
// ------------------------------------------------------------------------------------
__global__ void k_copy_back(View<double> L, long pin, double pinit, double *pr, float *vx, float *vy, float *vz, double *part)
{
    pdl_enter();
    __shared__ double sh[4][8];
    double m[4] = {0, 0, 0, -1e300};
    const long N = L.nxy * L.nz;
    const double shift = pinit - L.u0[pin];
    for (long n = (long)blockIdx.x * blockDim.x + threadIdx.x; n < N; n += (long)gridDim.x * blockDim.x) {
        int i, j, k;
        node_ijk(L, n, i, j, k);
        if (row_exists(0, i, j, k, L.nx, L.ny, L.nz)) { pr[n] = L.u0[n] + shift; m[3] = fmax(m[3], pr[n]); }
        if (row_exists(1, i, j, k, L.nx, L.ny, L.nz)) { vx[n] = (float)L.u1[n]; m[0] = fmax(m[0], fabs((double)vx[n])); }
        if (row_exists(2, i, j, k, L.nx, L.ny, L.nz)) { vy[n] = (float)L.u2[n]; m[1] = fmax(m[1], fabs((double)vy[n])); }
        if (row_exists(3, i, j, k, L.nx, L.ny, L.nz)) { vz[n] = (float)L.u3[n]; m[2] = fmax(m[2], fabs((double)vz[n])); }
    }
    for (int a = 0; a < 4; a++) {
        double v = m[a];
        for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
        if ((threadIdx.x & 31) == 0) sh[a][threadIdx.x >> 5] = v;
    }
    __syncthreads();
    if (threadIdx.x < 4) {
        double v = sh[threadIdx.x][0];
        for (int w = 1; w < (int)(blockDim.x >> 5); w++) v = fmax(v, sh[threadIdx.x][w]);
        part[(long)blockIdx.x * 4 + threadIdx.x] = v;
    }
}

// *flag = 1 where the node arrays differ from what k_copy_back writes for the level-0
// solution x (pinned pressure shift included): the uploaded state is not the last solution.
__global__ void k_same_solution(View<double> L, long pin, double pinit, const double *x0, const double *x1,
                                const double *x2, const double *x3, const double *pr, const float *vx, const float *vy,
                                const float *vz, int *flag)
{
    const long N = L.nxy * L.nz;
    const double shift = pinit - x0[pin];
    bool diff = false;
    for (long n = (long)blockIdx.x * blockDim.x + threadIdx.x; n < N; n += (long)gridDim.x * blockDim.x) {
        int i, j, k;
        node_ijk(L, n, i, j, k);
        if (row_exists(0, i, j, k, L.nx, L.ny, L.nz) && !(pr[n] == x0[n] + shift)) diff = true;
        if (row_exists(1, i, j, k, L.nx, L.ny, L.nz) && !(vx[n] == (float)x1[n])) diff = true;
        if (row_exists(2, i, j, k, L.nx, L.ny, L.nz) && !(vy[n] == (float)x2[n])) diff = true;
        if (row_exists(3, i, j, k, L.nx, L.ny, L.nz) && !(vz[n] == (float)x3[n])) diff = true;
    }
    if (__any_sync(0xffffffffu, diff) && (threadIdx.x & 31) == 0) *flag = 1;
}

// After an upload of nodal fields: keep the extrapolation history only if the uploaded v, P are
// exactly the last converged solution as the library returned it (a host loop that downloads
// and re-uploads the state every step); the comparison's result is read at the next solve.
int stokes_upload_check(i3g_ctx *c)
{
    c->hist_check = 0;
    if (c->nhist == 0 || !c->hist[2][0]) { c->nhist = 0; return 0; }
    if (!c->dflag) {
        I3G_CUDA(cudaMalloc((void **)&c->dflag, sizeof(int)));
        I3G_CUDA(cudaMallocHost((void **)&c->hflag, sizeof(int)));
    }
    Level &L0 = c->lev[0];
    const long pin = ((long)c->m.pzinit * L0.nx + c->m.pxinit) * L0.ny + c->m.pyinit;
    I3G_CUDA(cudaMemsetAsync(c->dflag, 0, sizeof(int), c->st));
    k_same_solution<<<std::min<long>(nblk(L0.n), 4L * 148), 256, 0, c->st>>>(
        view<double>(L0, L0.d), pin, c->m.pinit, c->hist[2][0], c->hist[2][1], c->hist[2][2], c->hist[2][3], c->pr,
        c->vx, c->vy, c->vz, c->dflag);
    c->launches++;
    I3G_CUDA(cudaMemcpyAsync(c->hflag, c->dflag, sizeof(int), cudaMemcpyDeviceToHost, c->st));
    c->hist_check = 1;
    I3G_CUDA(cudaGetLastError());
    return 0;
}

// strain rates and stresses from the FP32 velocities (sxxcalc..syzcalc with ynval = 0)
__global__ void k_eps_sig(int nx, int ny, int nz, const float *vx, const float *vy, const float *vz,
                          const double *etac, const double *etaxy, const double *etaxz, const double *etayz,
                          const double *icx, const double *isx, const double *icy, const double *isy,
                          const double *icz, const double *isz, float **eps, float **sig)
{
    pdl_enter();
    const long NY = ny, NXY = (long)nx * ny, N = NXY * nz;
    long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    const int m2 = (int)(n % NY);
    const long rest = n / NY;
    const int m1 = (int)(rest % nx), m3 = (int)(rest / nx);
    if (m1 > 0 && m2 > 0 && m3 > 0) {
        const long v0 = n - NXY - NY - 1;
        const double ne = etac[n];
        double e;
        e = __dmul_rn((double)__fsub_rn(vx[v0 + NY], vx[v0]), icx[m1]); eps[0][n] = (float)e; sig[0][n] = (float)__dmul_rn(__dmul_rn(2.0, ne), e);
        e = __dmul_rn((double)__fsub_rn(vy[v0 + 1], vy[v0]), icy[m2]); eps[1][n] = (float)e; sig[1][n] = (float)__dmul_rn(__dmul_rn(2.0, ne), e);
        e = __dmul_rn((double)__fsub_rn(vz[v0 + NXY], vz[v0]), icz[m3]); eps[2][n] = (float)e; sig[2][n] = (float)__dmul_rn(__dmul_rn(2.0, ne), e);
    }
    if (m1 > 0 && m1 < nx - 1 && m2 > 0 && m2 < ny - 1 && m3 < nz - 1) {
        double e = __dadd_rn(__dmul_rn((double)__fsub_rn(vx[n], vx[n - 1]), isy[m2]),
                             __dmul_rn((double)__fsub_rn(vy[n], vy[n - NY]), isx[m1]));
        eps[3][n] = (float)e; sig[3][n] = (float)__dmul_rn(__dmul_rn(2.0, etaxy[n]), e);
    }
    if (m1 > 0 && m1 < nx - 1 && m2 < ny - 1 && m3 > 0 && m3 < nz - 1) {
        double e = __dadd_rn(__dmul_rn((double)__fsub_rn(vx[n], vx[n - NXY]), isz[m3]),
                             __dmul_rn((double)__fsub_rn(vz[n], vz[n - NY]), isx[m1]));
        eps[4][n] = (float)e; sig[4][n] = (float)__dmul_rn(__dmul_rn(2.0, etaxz[n]), e);
    }
    if (m1 < nx - 1 && m2 > 0 && m2 < ny - 1 && m3 > 0 && m3 < nz - 1) {
        double e = __dadd_rn(__dmul_rn((double)__fsub_rn(vy[n], vy[n - NXY]), isz[m3]),
                             __dmul_rn((double)__fsub_rn(vz[n], vz[n - 1]), isy[m2]));
        eps[5][n] = (float)e; sig[5][n] = (float)__dmul_rn(__dmul_rn(2.0, etayz[n]), e);
    }
}

// strain rates and stresses of the level-0 FP32 velocities into c->eps / c->sig
static void eps_sig_launch(i3g_ctx *c)
{
    Level &L = c->lev[0];
    LAUNCH(k_eps_sig, nblk(L.n), 256, L.nx, L.ny, L.nz, (const float *)c->vx, (const float *)c->vy, (const float *)c->vz,
           (const double *)L.d.etac, (const double *)L.d.etaxy, (const double *)L.d.etaxz, (const double *)L.d.etayz,
           (const double *)L.d.ix[0], (const double *)L.d.ix[1], (const double *)L.d.iy[0], (const double *)L.d.iy[1],
           (const double *)L.d.iz[0], (const double *)L.d.iz[1], c->deps, c->dsig);
}

// sxxcalc..syzcalc with ynval = 0 (move3mg.c:3-710) for the current nodal velocities and
// viscosities, as vpiterate recomputes them after its iterations (move3mg.c:2405-2555)
int stokes_stresses(i3g_ctx *c)
{
    int rc = stokes_setup(c);
    if (rc) return rc;
    eps_sig_launch(c);
    I3G_CUDA(cudaGetLastError());
    I3G_CUDA(cudaStreamSynchronize(c->st));
    return 0;
}

static int finish_solve(i3g_ctx *c, double *timestep)
{
    Level &L = c->lev[0];
    View<double> V = view<double>(L, L.d);
    const long pin = (long)c->m.pzinit * L.nx * L.ny + (long)c->m.pxinit * L.ny + c->m.pyinit;
    const int nb = c->red_blocks;
    LAUNCH(k_copy_back, nb, 256, V, pin, c->m.pinit, c->pr, c->vx, c->vy, c->vz, c->dred);
    I3G_CUDA(cudaMemcpyAsync(c->hstage, c->dred, sizeof(double) * 4 * nb, cudaMemcpyDeviceToHost, c->st));
    eps_sig_launch(c);
    I3G_CUDA(cudaStreamSynchronize(c->st));
    double vm[4] = {0, 0, 0, -1e300};
    for (int b = 0; b < nb; b++)
        for (int a = 0; a < 4; a++) vm[a] = std::max(vm[a], c->hstage[b * 4 + a]);
    if (vm[3] > 1e12) return set_error(c, I3G_E_PRESSURE, "pressure is too big %e", vm[3]);
    if (!(vm[0] == vm[0]) || !(vm[1] == vm[1]) || !(vm[2] == vm[2])) return set_error(c, I3G_E_NAN, "NaN velocity after the Stokes solve");
    for (int a = 0; a < 3; a++)
        if (vm[a] > 0) {
            const double t = c->f.maxxystep / vm[a];
            if (*timestep > t) *timestep = t;
        }
    return 0;
}

// One solver iteration: an FP64 V-cycle, or (mixed precision) r = b - A x in FP64, one FP32
// V-cycle on the scaled correction system and x += e; then the level-0 norms to the host.
static int enqueue_iteration(i3g_ctx *c, int multinum)
{
    Level &L0 = c->lev[0];
    if (c->p.precision == 1) {
        residual_t<double>(c, 0);
        const int nb = c->red_blocks;
        LAUNCH(k_max_abs, nb, 256, (const double *)L0.d.r[1], L0.n, c->dred);
        LAUNCH(k_max_abs, nb, 256, (const double *)L0.d.r[2], L0.n, c->dred + nb);
        LAUNCH(k_max_abs, nb, 256, (const double *)L0.d.r[3], L0.n, c->dred + 2 * nb);
        LAUNCH(k_scale, 1, 1024, (const double *)c->dred, 3 * nb, c->h_ref, c->eta_ref, c->dscale);
        LAUNCH(k_to_f32, nblk(L0.n), 256, L0.n, (const double *)L0.d.r[0], (const double *)L0.d.r[1],
               (const double *)L0.d.r[2], (const double *)L0.d.r[3], L0.s.f[0], L0.s.f[1], L0.s.f[2], L0.s.f[3],
               L0.s.u[0], L0.s.u[1], L0.s.u[2], L0.s.u[3], (const uint8_t *)L0.bc, (const double *)c->dscale);
        vcycle_t<float>(c, multinum, true);
        LAUNCH(k_add_correction, nblk(L0.n), 256, L0.n, L0.d.u[0], L0.d.u[1], L0.d.u[2], L0.d.u[3],
               (const float *)L0.s.u[0], (const float *)L0.s.u[1], (const float *)L0.s.u[2], (const float *)L0.s.u[3],
               (const double *)c->dscale);
    } else {
        vcycle_t<double>(c, multinum, false);
    }
    return relres_enqueue(c);
}

// Capture the iteration into a CUDA graph, re-capturing when its parameters change.
static int iteration_graph(i3g_ctx *c, int multinum)
{
    if (c->sgraph && c->sg_multinum == multinum && c->sg_prec == c->p.precision && c->sg_p0 == c->p.p0koef &&
        c->sg_p1 == c->p.p1koef && c->sg_v0 == c->p.v0koef && c->sg_v1 == c->p.v1koef)
        return 0;
    if (c->sgraph) { cudaGraphExecDestroy(c->sgraph); c->sgraph = nullptr; }
    if (!c->dscale) I3G_CUDA(cudaMalloc((void **)&c->dscale, 16 * sizeof(double)));
    const int64_t l0 = c->launches;
    cudaGraph_t g = nullptr;
    I3G_CUDA(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
    int rc = enqueue_iteration(c, multinum);
    cudaError_t e = cudaStreamEndCapture(c->st, &g);
    if (rc) { if (g) cudaGraphDestroy(g); return rc; }
    if (e != cudaSuccess) return cuda_fail(c, e, "cudaStreamEndCapture", __FILE__, __LINE__);
    e = cudaGraphInstantiate(&c->sgraph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_fail(c, e, "cudaGraphInstantiate", __FILE__, __LINE__);
    c->sg_nodes = c->launches - l0;
    c->launches = l0;
    c->sg_multinum = multinum; c->sg_prec = c->p.precision;
    c->sg_p0 = c->p.p0koef; c->sg_p1 = c->p.p1koef; c->sg_v0 = c->p.v0koef; c->sg_v1 = c->p.v1koef;
    return 0;
}

void stokes_graph_free(i3g_ctx *c)
{
    if (c->sgraph) cudaGraphExecDestroy(c->sgraph);
    c->sgraph = nullptr;
    cudaFree(c->dscale);
    c->dscale = nullptr;
}

// ------------------------------------------------------------------------------------
// FGMRES acceleration of the mixed-precision correction solve
// ------------------------------------------------------------------------------------
// With krylov = m > 0 the FP64 defect correction is restarted FGMRES(m) (Saad 1993, flexible
// right preconditioning) whose preconditioner is the FP32 V-cycle on the scaled correction
// problem.  The Krylov vectors live in a row-scaled residual space, D r with D = 1/||b_mom||
// on velocity rows and h / (sqrt(#continuity rows) RMS(v)) on pressure rows, so that the
// minimised norm ||D r||^2 = mom^2 + cont^2 matches the stopping test.  Each Arnoldi step (the
// V-cycle, the FP64 operator and classical Gram-Schmidt with one re-orthogonalisation) is one
// CUDA graph per step index; the host applies the Givens rotations between steps.
constexpr int kKryMax = 16;
constexpr int kKryNq = kKryMax + 2;

struct KrylovState {
    int m = 0;
    long N = 0;
    double *V = nullptr;     // m+1 basis vectors, vector j component v at V + (4j + v) N
    double *Z = nullptr;     // m preconditioned directions, same layout
    double *W = nullptr;     // work vector (4N)
    double *F0 = nullptr;    // zero right-hand side (4N)
    double *part = nullptr;  // partial dot products [blocks][kKryNq]
    double *hdev = nullptr;  // [3][kKryNq]: first and second projection, squared norm; then 2 weights
    double *hhost = nullptr; // pinned mirror of hdev
    double *save = nullptr;  // FP64 preconditioner: level-0 solution and right-hand side set aside (8N)
    cudaGraphExec_t g[kKryMax] = {};
    long g_nodes[kKryMax] = {};   // kernels per captured step
    int g_multinum = -1, g_prec = -1;
    double g_p0 = 0, g_p1 = 0, g_v0 = 0, g_v1 = 0;
};

static KrylovState *kry(i3g_ctx *c) { return (KrylovState *)c->kry; }

// FP64 preconditioner input: the vector to precondition (in the residual arrays) becomes the
// right-hand side of the correction system, zero on boundary rows, with a zero start
__global__ void k_corr64_in(long n, const double *r0, const double *r1, const double *r2, const double *r3, double *f0,
                            double *f1, double *f2, double *f3, double *u0, double *u1, double *u2, double *u3,
                            const uint8_t *bc)
{
    pdl_enter();
    long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const uint8_t b = bc[t];
    f0[t] = (b & 1) ? 0.0 : r0[t];
    f1[t] = (b & 2) ? 0.0 : r1[t];
    f2[t] = (b & 4) ? 0.0 : r2[t];
    f3[t] = (b & 8) ? 0.0 : r3[t];
    u0[t] = 0.0; u1[t] = 0.0; u2[t] = 0.0; u3[t] = 0.0;
}

__global__ void k_kr_store64(long N, double *z, const double *e0, const double *e1, const double *e2, const double *e3)
{
    pdl_enter();
    long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= N) return;
    z[t] = e0[t]; z[N + t] = e1[t]; z[2 * N + t] = e2[t]; z[3 * N + t] = e3[t];
}

// d[0] = velocity-row weight, d[1] = pressure-row weight (device, so that the captured steps
// stay valid when the weights change between restarts)
__global__ void k_kr_from_r(long N, const double *r0, const double *r1, const double *r2, const double *r3, double *v,
                            const double *d)
{
    pdl_enter();
    long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= N) return;
    const double dv = d[0], dp = d[1];
    v[t] = dp * r0[t]; v[N + t] = dv * r1[t]; v[2 * N + t] = dv * r2[t]; v[3 * N + t] = dv * r3[t];
}

__global__ void k_kr_to_r(long N, const double *v, double *r0, double *r1, double *r2, double *r3, const double *d)
{
    pdl_enter();
    long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= N) return;
    const double dv = d[0], dp = d[1];
    r0[t] = v[t] / dp; r1[t] = v[N + t] / dv; r2[t] = v[2 * N + t] / dv; r3[t] = v[3 * N + t] / dv;
}

// z = scaled FP32 correction (the FP64 image of the V-cycle's result)
__global__ void k_kr_store(long N, double *z, const float *e0, const float *e1, const float *e2, const float *e3,
                           const double *scale)
{
    pdl_enter();
    long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= N) return;
    const double sp = scale[2], sv = scale[3];
    z[t] = sp * (double)e0[t]; z[N + t] = sv * (double)e1[t]; z[2 * N + t] = sv * (double)e2[t]; z[3 * N + t] = sv * (double)e3[t];
}

// One classical Gram-Schmidt pass over the 4N-vector w and the basis v_0..v_{NV-1}, per element
//   MODE 0: x = w;
//   MODE 1: x = -d w with the stopping test's row weight of the element's component (pressure
//           rows d[1], velocity rows d[0]), stored back into w (the residual -A z becomes D A z);
//   MODE 2: x = w - sum_i h_i v_i, stored back into w (the first projection removed);
// and the block partial sums of x . v_i (i < NV) and x . x (slot NV).  A grid of a few CTAs per
// SM with two elements in flight per thread keeps HBM busy; the basis is read once per pass.
constexpr int kKrBlocks = 4 * 148;
template <int NV, int MODE>
__global__ void __launch_bounds__(256) k_kr_proj(double *__restrict__ w, const double *__restrict__ V, long N, long n4,
                                                 const double *__restrict__ h, const double *__restrict__ d,
                                                 double *__restrict__ part)
{
    pdl_enter();
    __shared__ double sh[NV + 1][8];
    double q[NV + 1];
#pragma unroll
    for (int i = 0; i <= NV; i++) q[i] = 0;
    double hh[NV > 0 ? NV : 1];
#pragma unroll
    for (int i = 0; i < NV; i++) hh[i] = MODE == 2 ? h[i] : 0.0;
    const double dp = MODE == 1 ? -d[1] : 0.0, dv = MODE == 1 ? -d[0] : 0.0;
    const long stride = (long)gridDim.x * blockDim.x;
    for (long t0 = (long)blockIdx.x * blockDim.x + threadIdx.x; t0 < n4; t0 += 2 * stride) {
        double x[2], v[2][NV > 0 ? NV : 1];
        bool in[2];
#pragma unroll
        for (int u = 0; u < 2; u++) {
            const long t = t0 + u * stride;
            in[u] = t < n4;
            x[u] = in[u] ? w[t] : 0.0;
#pragma unroll
            for (int i = 0; i < NV; i++) v[u][i] = in[u] ? __ldg(V + i * n4 + t) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 2; u++) {
            const long t = t0 + u * stride;
            double y = x[u];
            if (MODE == 1) y *= t < N ? dp : dv;
            if (MODE == 2)
#pragma unroll
                for (int i = 0; i < NV; i++) y -= hh[i] * v[u][i];
            if (MODE != 0 && in[u]) w[t] = y;
#pragma unroll
            for (int i = 0; i < NV; i++) q[i] += y * v[u][i];
            q[NV] += y * y;
        }
    }
    const int wi = threadIdx.x >> 5, ln = threadIdx.x & 31;
#pragma unroll
    for (int i = 0; i <= NV; i++) {
        const double r = warp_sum(q[i]);
        if (ln == 0) sh[i][wi] = r;
    }
    __syncthreads();
    if ((int)threadIdx.x <= NV) {
        double r = 0;
        for (int a = 0; a < 8; a++) r += sh[threadIdx.x][a];
        part[(long)blockIdx.x * kKryNq + threadIdx.x] = r;
    }
}

__global__ void k_kr_dot_final(const double *part, int nblk, int nq, double *out)
{
    pdl_enter();
    const int qi = threadIdx.x >> 5, ln = threadIdx.x & 31;
    if (qi >= nq) return;
    double v = 0;
    for (int b = ln; b < nblk; b += 32) v += part[(long)b * kKryNq + qi];
    v = warp_sum(v);
    if (ln == 0) out[qi] = v;
}


// v = (w - sum_i h_i v_i) / |.|, the squared norm taken as w.w - sum_i h_i^2 (hw[nv] = w.w from
// the projection pass; v_0..v_{nv-1} are orthonormal)
__global__ void k_kr_axpy_normalize(double *v, const double *w, const double *V, int nv, long n4, const double *hw)
{
    pdl_enter();
    long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n4) return;
    double nrm2 = hw[nv];
    for (int i = 0; i < nv; i++) nrm2 -= hw[i] * hw[i];
    double x = w[t];
    for (int i = 0; i < nv; i++) x -= hw[i] * V[i * n4 + t];
    v[t] = x / sqrt(nrm2);
}

// v = w / sqrt(nrm2)
__global__ void k_kr_normalize(long n4, const double *w, double *v, const double *nrm2)
{
    pdl_enter();
    long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n4) return;
    v[t] = w[t] / sqrt(*nrm2);
}

struct KrY { double y[kKryMax]; };

// x += sum_j y_j z_j
__global__ void k_kr_update(long N, double *x0, double *x1, double *x2, double *x3, const double *Z, int k, KrY y)
{
    pdl_enter();
    long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= N) return;
    double a0 = 0, a1 = 0, a2 = 0, a3 = 0;
    for (int j = 0; j < k; j++) {
        const double *z = Z + (long)j * 4 * N;
        a0 += y.y[j] * z[t]; a1 += y.y[j] * z[N + t]; a2 += y.y[j] * z[2 * N + t]; a3 += y.y[j] * z[3 * N + t];
    }
    x0[t] += a0; x1[t] += a1; x2[t] += a2; x3[t] += a3;
}

// u = a + r (a - b): the next solution predicted from the last two
__global__ void k_extrapolate(long n, double *u, const double *a, const double *b, double r)
{
    pdl_enter();
    long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    u[t] = a[t] + r * (a[t] - b[t]);
}

// u = wa a + wb b + wc c: the next solution predicted from the last three
__global__ void k_extrapolate3(long n, double *u, const double *a, const double *b, const double *cc, double wa, double wb,
                               double wc)
{
    pdl_enter();
    long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    u[t] = wa * a[t] + wb * b[t] + wc * cc[t];
}

// Row-weighted dots of a staged start's residual change dr = r0 - r (r0: the default start's
// residual, r = L.r: the staged start's) over the rows of the stopping test: out[0] += <r0, dr>,
// out[1] += <dr, dr>, weight wm on non-boundary velocity rows and wc on pressure rows.
__global__ void __launch_bounds__(256) k_guess_dots(View<double> L, const double *a0, const double *a1, const double *a2,
                                                    const double *a3, double wm, double wc, double *out)
{
    pdl_enter();
    __shared__ double sh[2][8];
    double x = 0, y = 0;
    const long N = L.nxy * L.nz;
    for (long n = (long)blockIdx.x * blockDim.x + threadIdx.x; n < N; n += (long)gridDim.x * blockDim.x) {
        int i, j, k;
        node_ijk(L, n, i, j, k);
        const uint8_t b = L.bc[n];
        if (row_exists(0, i, j, k, L.nx, L.ny, L.nz) && !(b & 1)) { const double d = a0[n] - L.r0[n]; x += wc * a0[n] * d; y += wc * d * d; }
        if (row_exists(1, i, j, k, L.nx, L.ny, L.nz) && !(b & 2)) { const double d = a1[n] - L.r1[n]; x += wm * a1[n] * d; y += wm * d * d; }
        if (row_exists(2, i, j, k, L.nx, L.ny, L.nz) && !(b & 4)) { const double d = a2[n] - L.r2[n]; x += wm * a2[n] * d; y += wm * d * d; }
        if (row_exists(3, i, j, k, L.nx, L.ny, L.nz) && !(b & 8)) { const double d = a3[n] - L.r3[n]; x += wm * a3[n] * d; y += wm * d * d; }
    }
    x = warp_sum(x);
    y = warp_sum(y);
    const int w = threadIdx.x >> 5, ln = threadIdx.x & 31;
    if (ln == 0) { sh[0][w] = x; sh[1][w] = y; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int q = 1; q < (int)(blockDim.x >> 5); q++) { x += sh[0][q]; y += sh[1][q]; }
        atomicAdd(out, x);
        atomicAdd(out + 1, y);
    }
}

// k_kr_proj<nv, mode> for a run-time basis size nv <= kKryMax
template <int MODE>
static void kr_proj_launch(i3g_ctx *c, int nv, double *w, const double *V, long N, long n4, const double *h, const double *d,
                           double *part)
{
    switch (nv) {
#define KR_CASE(k) case k: LAUNCH((k_kr_proj<k, MODE>), kKrBlocks, 256, w, V, N, n4, h, d, part); break;
    KR_CASE(0) KR_CASE(1) KR_CASE(2) KR_CASE(3) KR_CASE(4) KR_CASE(5) KR_CASE(6) KR_CASE(7) KR_CASE(8)
    KR_CASE(9) KR_CASE(10) KR_CASE(11) KR_CASE(12) KR_CASE(13) KR_CASE(14) KR_CASE(15) KR_CASE(16)
#undef KR_CASE
    default: break;
    }
}

static int kr_proj(i3g_ctx *c, int nv, int mode, double *w, long N, long n4, const double *h, const double *d, double *part)
{
    if (nv < 0 || nv > kKryMax) return set_error(c, I3G_E_ARG, "Krylov basis of %d vectors above %d", nv, kKryMax);
    const double *V = kry(c)->V;
    if (mode == 0) kr_proj_launch<0>(c, nv, w, V, N, n4, h, d, part);
    else if (mode == 1) kr_proj_launch<1>(c, nv, w, V, N, n4, h, d, part);
    else kr_proj_launch<2>(c, nv, w, V, N, n4, h, d, part);
    return 0;
}

static int kry_alloc(i3g_ctx *c, int m)
{
    KrylovState *K = kry(c);
    if (K && K->m == m && (K->save || c->p.precision != 0)) return 0;
    if (K) kry_free(c);
    K = new KrylovState();
    c->kry = K;
    K->m = m;
    K->N = c->lev[0].n;
    const long n4 = 4 * K->N;
    ALLOC(K->V, double, (m + 1) * n4);
    ALLOC(K->Z, double, m * n4);
    ALLOC(K->W, double, n4);
    ALLOC(K->F0, double, n4);
    ALLOC(K->part, double, (long)kKrBlocks * kKryNq);
    ALLOC(K->hdev, double, 3 * kKryNq + 2);
    if (c->p.precision == 0) ALLOC(K->save, double, 2 * n4);
    I3G_CUDA(cudaMallocHost((void **)&K->hhost, (3 * kKryNq + 2) * sizeof(double)));
    I3G_CUDA(cudaMemsetAsync(K->W, 0, n4 * 8, c->st));
    I3G_CUDA(cudaMemsetAsync(K->F0, 0, n4 * 8, c->st));
    return 0;
}

static void kry_free(i3g_ctx *c)
{
    KrylovState *K = kry(c);
    if (!K) return;
    for (int j = 0; j < kKryMax; j++) if (K->g[j]) cudaGraphExecDestroy(K->g[j]);
    cudaFree(K->V); cudaFree(K->Z); cudaFree(K->W); cudaFree(K->F0); cudaFree(K->part); cudaFree(K->hdev);
    cudaFree(K->save);
    cudaFreeHost(K->hhost);
    delete K;
    c->kry = nullptr;
}

// Captured iterations depend on the sweep counts and relaxation factors: drop them.
void stokes_params_changed(i3g_ctx *c)
{
    if (c->sgraph) cudaGraphExecDestroy(c->sgraph);
    c->sgraph = nullptr;
    KrylovState *K = kry(c);
    if (K)
        for (int q = 0; q < kKryMax; q++)
            if (K->g[q]) { cudaGraphExecDestroy(K->g[q]); K->g[q] = nullptr; }
}

// Arnoldi step j: z_j = M^-1 D^-1 v_j, w = D A z_j orthogonalised against v_0..v_j, v_{j+1} = w/|w|;
// projections and the squared norm land in hhost.
static int kry_enqueue_step(i3g_ctx *c, int j, int multinum)
{
    KrylovState *K = kry(c);
    Level &L0 = c->lev[0];
    const long N = K->N, n4 = 4 * N;
    double *vj = K->V + (long)j * n4, *zj = K->Z + (long)j * n4;
    // preconditioner: the V-cycle of this precision on the unscaled vector
    const double *d = K->hdev + 3 * kKryNq;
    LAUNCH(k_kr_to_r, nblk(N), 256, N, (const double *)vj, L0.d.r[0], L0.d.r[1], L0.d.r[2], L0.d.r[3], d);
    const int nb = c->red_blocks;
    if (c->p.precision == 0) {
        // FP64 V-cycle from zero on level 0's own arrays, whose solution and right-hand side
        // are set aside meanwhile (no scaling: the system is already FP64)
        for (int v = 0; v < 4; v++) {
            I3G_CUDA(cudaMemcpyAsync(K->save + v * N, L0.d.u[v], N * 8, cudaMemcpyDeviceToDevice, c->st));
            I3G_CUDA(cudaMemcpyAsync(K->save + (4 + v) * N, L0.d.f[v], N * 8, cudaMemcpyDeviceToDevice, c->st));
        }
        LAUNCH(k_corr64_in, nblk(N), 256, N, (const double *)L0.d.r[0], (const double *)L0.d.r[1],
               (const double *)L0.d.r[2], (const double *)L0.d.r[3], L0.d.f[0], L0.d.f[1], L0.d.f[2], L0.d.f[3],
               L0.d.u[0], L0.d.u[1], L0.d.u[2], L0.d.u[3], (const uint8_t *)L0.bc);
        vcycle_t<double>(c, multinum, true);
        LAUNCH(k_kr_store64, nblk(N), 256, N, zj, (const double *)L0.d.u[0], (const double *)L0.d.u[1],
               (const double *)L0.d.u[2], (const double *)L0.d.u[3]);
        for (int v = 0; v < 4; v++) {
            I3G_CUDA(cudaMemcpyAsync(L0.d.u[v], K->save + v * N, N * 8, cudaMemcpyDeviceToDevice, c->st));
            I3G_CUDA(cudaMemcpyAsync(L0.d.f[v], K->save + (4 + v) * N, N * 8, cudaMemcpyDeviceToDevice, c->st));
        }
    } else {
        LAUNCH(k_max_abs, nb, 256, (const double *)L0.d.r[1], N, c->dred);
        LAUNCH(k_max_abs, nb, 256, (const double *)L0.d.r[2], N, c->dred + nb);
        LAUNCH(k_max_abs, nb, 256, (const double *)L0.d.r[3], N, c->dred + 2 * nb);
        LAUNCH(k_scale, 1, 1024, (const double *)c->dred, 3 * nb, c->h_ref, c->eta_ref, c->dscale);
        LAUNCH(k_to_f32, nblk(N), 256, N, (const double *)L0.d.r[0], (const double *)L0.d.r[1],
               (const double *)L0.d.r[2], (const double *)L0.d.r[3], L0.s.f[0], L0.s.f[1], L0.s.f[2], L0.s.f[3],
               L0.s.u[0], L0.s.u[1], L0.s.u[2], L0.s.u[3], (const uint8_t *)L0.bc, (const double *)c->dscale);
        vcycle_t<float>(c, multinum, true);
        LAUNCH(k_kr_store, nblk(N), 256, N, zj, (const float *)L0.s.u[0], (const float *)L0.s.u[1],
               (const float *)L0.s.u[2], (const float *)L0.s.u[3], (const double *)c->dscale);
    }
    // w = D A z_j: the FP64 residual of z_j with a zero right-hand side is -A z_j
    View<double> Vz = view<double>(L0, L0.d);
    Vz.u0 = zj; Vz.u1 = zj + N; Vz.u2 = zj + 2 * N; Vz.u3 = zj + 3 * N;
    Vz.f0 = K->F0; Vz.f1 = K->F0 + N; Vz.f2 = K->F0 + 2 * N; Vz.f3 = K->F0 + 3 * N;
    Vz.r0 = K->W; Vz.r1 = K->W + N; Vz.r2 = K->W + 2 * N; Vz.r3 = K->W + 3 * N;
    if (c->fuse) {
        BcDev4 B;
        long nb = 0;
        for (int v = 0; v < 4; v++) { B.b[v] = bcdev(L0.bcl[v]); nb += L0.bcl[v].n; }
        LAUNCH(k_residual_bc<double>, nblk(N) + nblk(nb), 256, Vz, B, nblk(N));
    } else {
        LAUNCH(k_residual<double>, nblk(N), 256, Vz);
        for (int v = 0; v < 4; v++) {
            BcList &B = L0.bcl[v];
            if (B.n) LAUNCH(k_bc_residual<double>, nblk(B.n), 256, Vz, v, B.n, (const int *)B.node, (const int *)B.onode,
                            (const int *)B.ocomp, (const double *)B.ok);
        }
    }
    // classical Gram-Schmidt, twice: the first pass also applies the row weights (w = D A z), the
    // second subtracts the first projection while it forms the second one and w.w, from which the
    // last kernel takes the norm while it subtracts the second projection and normalises
    double *h1 = K->hdev, *h2 = K->hdev + kKryNq;
    if (int rc = kr_proj(c, j + 1, 1, K->W, N, n4, nullptr, d, K->part)) return rc;
    LAUNCH(k_kr_dot_final, 1, 32 * (j + 2), (const double *)K->part, kKrBlocks, j + 2, h1);
    if (int rc = kr_proj(c, j + 1, 2, K->W, N, n4, h1, d, K->part)) return rc;
    LAUNCH(k_kr_dot_final, 1, 32 * (j + 2), (const double *)K->part, kKrBlocks, j + 2, h2);
    LAUNCH(k_kr_axpy_normalize, nblk(n4), 256, K->V + (long)(j + 1) * n4, (const double *)K->W, (const double *)K->V,
           j + 1, n4, (const double *)h2);
    I3G_CUDA(cudaMemcpyAsync(K->hhost, K->hdev, 2 * kKryNq * sizeof(double), cudaMemcpyDeviceToHost, c->st));
    return 0;
}

static int kry_graph(i3g_ctx *c, int j, int multinum)
{
    KrylovState *K = kry(c);
    if (K->g_multinum != multinum || K->g_p0 != c->p.p0koef || K->g_p1 != c->p.p1koef || K->g_v0 != c->p.v0koef ||
        K->g_v1 != c->p.v1koef || K->g_prec != c->p.precision) {
        for (int q = 0; q < kKryMax; q++) if (K->g[q]) { cudaGraphExecDestroy(K->g[q]); K->g[q] = nullptr; }
        K->g_multinum = multinum; K->g_p0 = c->p.p0koef; K->g_p1 = c->p.p1koef; K->g_v0 = c->p.v0koef;
        K->g_v1 = c->p.v1koef; K->g_prec = c->p.precision;
    }
    if (K->g[j]) return 0;
    const int64_t l0 = c->launches;
    cudaGraph_t g = nullptr;
    I3G_CUDA(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
    int rc = kry_enqueue_step(c, j, multinum);
    cudaError_t e = cudaStreamEndCapture(c->st, &g);
    if (rc) { if (g) cudaGraphDestroy(g); return rc; }
    if (e != cudaSuccess) return cuda_fail(c, e, "cudaStreamEndCapture", __FILE__, __LINE__);
    e = cudaGraphInstantiate(&K->g[j], g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_fail(c, e, "cudaGraphInstantiate", __FILE__, __LINE__);
    K->g_nodes[j] = c->launches - l0;
    c->launches = l0;
    return 0;
}

// One FGMRES restart cycle from the current level-0 solution; *steps += Arnoldi steps taken.
static int kry_cycle(i3g_ctx *c, int multinum, double rtol, int maxsteps, int *steps)
{
    KrylovState *K = kry(c);
    Level &L0 = c->lev[0];
    const long N = K->N, n4 = 4 * N;
    const int m = K->m;
    // weights from the current norms (relres_enqueue has filled hred)
    const double *q = c->hred;
    const double dv = q[1] > 0 ? 1.0 / std::sqrt(q[1]) : 1.0;
    const double rmsv = (c->nvel > 0 && q[3] > 0) ? std::sqrt(q[3] / c->nvel) : 0.0;
    const double dp = (c->ncont > 0 && rmsv > 0) ? c->h_ref / (std::sqrt(c->ncont) * rmsv) : 1.0;
    // weights to the device, then v_0 = D r / |D r|
    K->hhost[3 * kKryNq] = dv;
    K->hhost[3 * kKryNq + 1] = dp;
    I3G_CUDA(cudaMemcpyAsync(K->hdev + 3 * kKryNq, K->hhost + 3 * kKryNq, 2 * sizeof(double), cudaMemcpyHostToDevice, c->st));
    const double *d = K->hdev + 3 * kKryNq;
    residual_t<double>(c, 0);
    LAUNCH(k_kr_from_r, nblk(N), 256, N, (const double *)L0.d.r[0], (const double *)L0.d.r[1],
           (const double *)L0.d.r[2], (const double *)L0.d.r[3], K->V, d);
    double *nrm = K->hdev + 2 * kKryNq;
    if (int rc = kr_proj(c, 0, 0, K->V, N, n4, nullptr, d, K->part)) return rc;
    LAUNCH(k_kr_dot_final, 1, 32, (const double *)K->part, kKrBlocks, 1, nrm);
    I3G_CUDA(cudaMemcpyAsync(K->hhost + 2 * kKryNq, nrm, sizeof(double), cudaMemcpyDeviceToHost, c->st));
    LAUNCH(k_kr_normalize, nblk(n4), 256, n4, (const double *)K->V, K->V, (const double *)nrm);
    I3G_CUDA(cudaStreamSynchronize(c->st));
    const double beta = std::sqrt(K->hhost[2 * kKryNq]);
    if (!(beta > 0)) return 0;
    double H[kKryMax + 1][kKryMax], cs[kKryMax], sn[kKryMax], g[kKryMax + 1];
    for (int i = 0; i <= m; i++) g[i] = 0;
    g[0] = beta;
    int k = 0;
    for (int j = 0; j < m && *steps < maxsteps; j++) {
        int rc = kry_graph(c, j, multinum);
        if (rc) return rc;
        I3G_CUDA(cudaGraphLaunch(K->g[j], c->st));
        c->launches += K->g_nodes[j];
        I3G_CUDA(cudaStreamSynchronize(c->st));
        (*steps)++;
        k = j + 1;
        const double *h = K->hhost;
        for (int i = 0; i <= j; i++) H[i][j] = h[i] + h[kKryNq + i];
        double hn2 = h[kKryNq + j + 1];   // w.w before the second projection
        for (int i = 0; i <= j; i++) hn2 -= h[kKryNq + i] * h[kKryNq + i];
        const double hn = std::sqrt(std::max(0.0, hn2));
        // previous rotations, then a new one that zeroes H[j+1][j]
        for (int i = 0; i < j; i++) {
            const double a = H[i][j], b = H[i + 1][j];
            H[i][j] = cs[i] * a + sn[i] * b;
            H[i + 1][j] = -sn[i] * a + cs[i] * b;
        }
        const double a = H[j][j], r = std::hypot(a, hn);
        cs[j] = r > 0 ? a / r : 1.0;
        sn[j] = r > 0 ? hn / r : 0.0;
        H[j][j] = r;
        g[j + 1] = -sn[j] * g[j];
        g[j] = cs[j] * g[j];
        if (!(g[j + 1] == g[j + 1])) return set_error(c, I3G_E_NAN, "NaN in the FGMRES step");
        // |g[j+1]| = ||D r||, and ||D r||^2 = mom^2 + cont^2: both criteria hold once it is <= rtol
        if (std::fabs(g[j + 1]) <= rtol || !(hn > 0)) break;
    }
    // y = R^-1 g, x += Z y
    KrY y;
    for (int i = k - 1; i >= 0; i--) {
        double sum = g[i];
        for (int l = i + 1; l < k; l++) sum -= H[i][l] * y.y[l];
        y.y[i] = H[i][i] != 0 ? sum / H[i][i] : 0.0;
    }
    LAUNCH(k_kr_update, nblk(N), 256, N, L0.d.u[0], L0.d.u[1], L0.d.u[2], L0.d.u[3], (const double *)K->Z, k, y);
    return 0;
}

int stokes_solve(i3g_ctx *c, double *timestep)
{
    if (c->p.p2koef != 0 || c->f.p2koef != 0 || c->f.p2koef2 != 0)
        return set_error(c, I3G_E_UNSUPPORTED, "p2koef != 0 (grad div terms, move3mg.c:860-889) is not supported");
    EventPair ev;
    I3G_CUDA(ev.create());
    cudaEvent_t e0 = ev.a, e1 = ev.b;
    I3G_CUDA(cudaEventRecord(e0, c->st));
    int rc = stokes_setup(c);
    if (rc) return rc;
    Level &L0 = c->lev[0];
    if (!c->p.warm_start)
        for (int v = 0; v < 4; v++) I3G_CUDA(cudaMemsetAsync(L0.d.u[v], 0, L0.n * 8, c->st));
    if (c->hist_check) {
        // the upload comparison was enqueued before this solve: its flag is ready after a sync
        I3G_CUDA(cudaStreamSynchronize(c->st));
        if (*c->hflag) c->nhist = 0;
        c->hist_check = 0;
    }
    c->st_.stokes_start = 0;
    if (c->p.warm_start == 3 && c->nhist == 3 && c->hist_dt[0] > 0 && c->hist_dt[1] > 0) {
        c->st_.stokes_start = 3;
        // quadratic (Lagrange) extrapolation in time from the last three converged solutions at
        // t0 < t1 < t2 to t3 = t2 + dt, with h1 = t1 - t0, h2 = t2 - t1, h3 = dt (the step taken
        // after the newest solution); equal steps give 3 x2 - 3 x1 + x0
        const double h1 = c->hist_dt[0], h2 = c->hist_dt[1], h3 = c->hist_dt[2];
        const double w0 = h3 * (h2 + h3) / (h1 * (h1 + h2));
        const double w1 = -h3 * (h1 + h2 + h3) / (h1 * h2);
        const double w2 = (h1 + h2 + h3) * (h2 + h3) / ((h1 + h2) * h2);
        for (int v = 0; v < 4; v++)
            LAUNCH(k_extrapolate3, nblk(L0.n), 256, L0.n, L0.d.u[v], (const double *)c->hist[2][v],
                   (const double *)c->hist[1][v], (const double *)c->hist[0][v], w2, w1, w0);
    } else if (c->p.warm_start >= 2 && c->nhist >= 2 && c->hist_dt[1] > 0) {
        c->st_.stokes_start = 1;
        // linear extrapolation in time from the last two converged solutions
        const double r = c->hist_dt[2] / c->hist_dt[1];
        for (int v = 0; v < 4; v++)
            LAUNCH(k_extrapolate, nblk(L0.n), 256, L0.n, L0.d.u[v], (const double *)c->hist[2][v],
                   (const double *)c->hist[1][v], r);
    }
    // boundary rows of the initial guess consistent with their partners
    for (int v = 0; v < 4; v++) bc_apply<double>(c, 0, v, true);
    const int maxc = c->p.stokes_maxcyc > 0 ? c->p.stokes_maxcyc : 2000;
    const double rtol = c->p.stokes_rtol > 0 ? c->p.stokes_rtol : 1e-8;
    int multinum = c->f.multinum > 0 ? std::min(c->f.multinum, c->nlev - 1) : std::min(c->p.multimax, c->nlev - 1);
    double mom, cont;
    if ((rc = stokes_relres(c, &mom, &cont))) return rc;
    c->guess_used = -1;
    if (c->guess_pending) {
        // A staged (learned) start g competes with the default start d.  The correction g - d is
        // first scaled by the factor that minimises the stopping test's row-weighted residual
        // along it: r(d + a (g - d)) = r0 - a dr with dr = r0 - r(g), a = <r0,dr> / <dr,dr>.
        // The scaled start is kept only if its relative residual is below the default start's.
        c->guess_pending = 0;
        const double q1 = c->hred[1], q3 = c->hred[3];   // sum b_mom^2 and sum v^2 of the default start
        double *const *su = c->gsave, *const *sr = c->gsave + 4;
        residual_t<double>(c, 0);
        for (int v = 0; v < 4; v++) {
            I3G_CUDA(cudaMemcpyAsync(sr[v], L0.d.r[v], L0.n * 8, cudaMemcpyDeviceToDevice, c->st));
            I3G_CUDA(cudaMemcpyAsync(su[v], L0.d.u[v], L0.n * 8, cudaMemcpyDeviceToDevice, c->st));
            I3G_CUDA(cudaMemcpyAsync(L0.d.u[v], c->guess[v], L0.n * 8, cudaMemcpyDeviceToDevice, c->st));
        }
        for (int v = 0; v < 4; v++) bc_apply<double>(c, 0, v, true);
        residual_t<double>(c, 0);
        const double wm = q1 > 0 ? 1.0 / q1 : 1.0;
        const double wc = (c->ncont > 0 && q3 > 0) ? c->h_ref * c->h_ref * c->nvel / (c->ncont * q3) : 1.0;
        I3G_CUDA(cudaMemsetAsync(c->gdots, 0, 2 * sizeof(double), c->st));
        LAUNCH(k_guess_dots, c->red_blocks, 256, view<double>(L0, L0.d), (const double *)sr[0], (const double *)sr[1],
               (const double *)sr[2], (const double *)sr[3], wm, wc, c->gdots);
        double dots[2] = {0, 0};
        I3G_CUDA(cudaMemcpyAsync(dots, c->gdots, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->st));
        I3G_CUDA(cudaStreamSynchronize(c->st));
        double alpha = dots[1] > 0 ? dots[0] / dots[1] : 0.0;
        if (!(alpha > 0)) alpha = 0.0;   // also for NaN
        alpha = std::min(alpha, 4.0);
        c->guess_alpha = alpha;
        // u = d + alpha (g - d)
        for (int v = 0; v < 4; v++)
            LAUNCH(k_extrapolate, nblk(L0.n), 256, L0.n, L0.d.u[v], (const double *)su[v], (const double *)c->guess[v], -alpha);
        for (int v = 0; v < 4; v++) bc_apply<double>(c, 0, v, true);
        double gm, gc;
        if ((rc = stokes_relres(c, &gm, &gc))) return rc;
        const double rg = std::max(gm, gc), rdef = std::max(mom, cont);
        c->guess_rel[0] = rg;
        c->guess_rel[1] = rdef;
        c->guess_used = (alpha > 0 && rg < rdef) ? 1 : 0;   // false for a NaN residual too
        if (c->guess_used) {
            c->st_.stokes_start = 2;
            mom = gm;
            cont = gc;
        } else {
            // back to the default start; the norms are recomputed so that everything derived from
            // them (the FGMRES row scaling) is the default start's again
            for (int v = 0; v < 4; v++)
                I3G_CUDA(cudaMemcpyAsync(L0.d.u[v], su[v], L0.n * 8, cudaMemcpyDeviceToDevice, c->st));
            if ((rc = stokes_relres(c, &mom, &cont))) return rc;
        }
    }
    c->st_.stokes_rel0 = std::max(mom, cont);
    int cycles = 0, outer = 0;
    bool conv = mom <= rtol && cont <= rtol;
    const double p0_save = c->p.p0koef, p1_save = c->p.p1koef;
    const int ncyc = c->p.multicyc > 0 ? c->p.multicyc : 1;
    double best = std::max(mom, cont);
    bool switched = false;
    static const bool trace = getenv("I3G_TRACE") != nullptr;   // per-cycle residuals on stderr
    if (c->p.krylov > 0) {
        if (c->p.krylov > kKryMax) return set_error(c, I3G_E_ARG, "krylov restart length %d above %d", c->p.krylov, kKryMax);
        if ((rc = kry_alloc(c, c->p.krylov))) return rc;
        if (!c->dscale) I3G_CUDA(cudaMalloc((void **)&c->dscale, 16 * sizeof(double)));
        while (!conv && cycles < maxc) {
            if ((rc = kry_cycle(c, multinum, rtol, maxc, &cycles))) return rc;
            outer++;
            if ((rc = stokes_relres(c, &mom, &cont))) return rc;
            if (!(mom == mom) || !(cont == cont)) return set_error(c, I3G_E_NAN, "NaN residual after %d V-cycles", cycles);
            conv = mom <= rtol && cont <= rtol;
            if (trace) fprintf(stderr, "i3g stokes fgmres restart %d cycles %d mom %.3e cont %.3e\n", outer, cycles, mom, cont);
        }
    }
    while (!conv && cycles < maxc) {
        for (int i = 0; i < ncyc && cycles < maxc && !conv; i++) {
            if ((rc = iteration_graph(c, multinum))) return rc;
            I3G_CUDA(cudaGraphLaunch(c->sgraph, c->st));
            c->launches += c->sg_nodes;
            I3G_CUDA(cudaStreamSynchronize(c->st));
            cycles++;
            relres_read(c, &mom, &cont);
            if (!(mom == mom) || !(cont == cont)) return set_error(c, I3G_E_NAN, "NaN residual after %d V-cycles", cycles);
            conv = mom <= rtol && cont <= rtol;
            if (trace) fprintf(stderr, "i3g stokes cycle %d mom %.3e cont %.3e p0 %.3g p1 %.3g multinum %d\n", cycles, mom, cont,
                               c->p.p0koef, c->p.p1koef, multinum);
            // Safeguard: a residual 30x above the best one seen in this solve means the cycle
            // diverges (transient rises of a convergent cycle stay far below that); switch to the
            // file row's second relaxation set early (the reference switches after multstp
            // iterations, move3mg.c:2585-2593).
            const double cur = std::max(mom, cont);
            best = std::min(best, cur);
            if (cur > 30.0 * best && !switched && (c->p.p0koef != c->f.p0koef2 || c->p.p1koef != c->f.p1koef2)) {
                c->p.p0koef = c->f.p0koef2;
                c->p.p1koef = c->f.p1koef2;
                multinum = std::min(c->f.multinum2 > 0 ? c->f.multinum2 : multinum, c->nlev - 1);
                switched = true;
                best = cur;
            }
        }
        outer++;
        if (outer >= c->f.multstp && c->f.multstp > 0 && !switched) {   // move3mg.c:2585-2593
            multinum = std::min(c->f.multinum2 > 0 ? c->f.multinum2 : multinum, c->nlev - 1);
            c->p.p0koef = c->f.p0koef2;
            c->p.p1koef = c->f.p1koef2;
            switched = true;
        }
    }
    c->p.p0koef = p0_save;
    c->p.p1koef = p1_save;
    c->st_.stokes_cycles = cycles;
    c->st_.stokes_outer = outer;
    c->st_.stokes_rel = std::max(mom, cont);
    c->st_.stokes_mom_rel = mom;
    c->st_.stokes_cont_rel = cont;
    const bool keep = c->p.warm_start >= 2 && conv;
    if (keep) {
        // the oldest slot takes the new solution, which becomes the newest (slot 2)
        const int nh = c->p.warm_start == 3 ? 3 : 2;
        for (int h = 3 - nh; h < 3; h++)
            for (int v = 0; v < 4; v++)
                if (!c->hist[h][v]) ALLOC(c->hist[h][v], double, L0.n);
        for (int v = 0; v < 4; v++) {
            double *old = c->hist[3 - nh][v];
            for (int h = 3 - nh; h < 2; h++) c->hist[h][v] = c->hist[h + 1][v];
            c->hist[2][v] = old;
            I3G_CUDA(cudaMemcpyAsync(c->hist[2][v], L0.d.u[v], L0.n * 8, cudaMemcpyDeviceToDevice, c->st));
        }
    }
    if ((rc = finish_solve(c, timestep))) return rc;
    if (keep) {
        c->hist_dt[0] = c->hist_dt[1];
        c->hist_dt[1] = c->hist_dt[2];
        c->hist_dt[2] = *timestep;
        c->nhist = std::min(c->nhist + 1, c->p.warm_start == 3 ? 3 : 2);
    }
    I3G_CUDA(cudaEventRecord(e1, c->st));
    I3G_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    c->st_.ms_stokes = ms;
    if (c->dbar_err && c->coop_nodes > 0) {
        int berr = 0;
        I3G_CUDA(cudaMemcpy(&berr, c->dbar_err, sizeof(int), cudaMemcpyDeviceToHost));
        if (berr) return set_error(c, I3G_E_CUDA, "Stokes: a grid barrier of the coarse-level kernel timed out");
    }
    if (!conv) return set_error(c, I3G_E_NOCONV, "Stokes: %d V-cycles without reaching relative residual %g (mom %.3e cont %.3e)", cycles, rtol, mom, cont);
    return 0;
}

// Timing of kernel classes on level 0 with an empty L2 before every repetition (cold_time).
// Bytes are the algorithmic (compulsory) bytes of the unit timed: per node of level 0,
//   0 / 7  one colour of Vx (FP64 / FP32): vx, vy, vz, P and three viscosity arrays read, the
//          right-hand side and the writes of half the rows, the boundary mask;
//   8 / 10 one full sweep (FP32 / FP64: Vx, Vy, Vz red and black, boundary rows, pressure):
//          4 unknowns read and written, 4 right-hand sides read, 5 FP32 viscosities: 68 / 116 B;
//   1      FP64 residual: 116 B;  2  restriction: 4 s (1 + 1/8) B;  3  prolongation: 4 s (2 + 1/8) B.
constexpr int kMaxLevWarm = 6;
constexpr int kWarmLevel0 = 19;

int stokes_time_kernel(i3g_ctx *c, int kind, int reps, double *ms, double *bytes)
{
    if (!c->stokes_ready) {
        int rc = stokes_setup(c);
        if (rc) return rc;
    }
    Level &L = c->lev[0];
    const double N = (double)L.n;
    View<double> V = view<double>(L, L.d);
    View<float> Vf = view<float>(L, L.s);
    const long total = (long)((L.ny + 1) / 2) * L.nx * L.nz;
    int r = 0;
    auto launch = [&]() -> int {
        switch (kind) {
        case 0: LAUNCH((k_relax_vel<double, 1>), nblk(total), 256, V, r & 1, c->p.v0koef); break;
        case 7: LAUNCH((k_relax_vel<float, 1>), nblk(total), 256, Vf, r & 1, (float)c->p.v0koef); break;
        case 8: smooth_t<float>(c, 0, 1, true, false); break;
        case 10: smooth_t<double>(c, 0, 1, false, false); break;
        case 1: LAUNCH(k_residual<double>, nblk(L.n), 256, V); break;
        case 2: if (c->nlev > 1) restrict_t<double>(c, 1); break;
        case 3: if (c->nlev > 1) prolong_t<double>(c, 1); break;
        default: break;
        }
        r++;
        return 0;
    };
    // warm-cache kinds (the coarse levels of a V-cycle stay in L2): 11 one FP32 V-cycle of the
    // solver's schedule, 12 its coarse tail kernel alone, 13 + l - 1 one FP32 sweep of level l
    if ((kind >= 11 && kind <= 12 + kMaxLevWarm) || kind == kWarmLevel0) {
        const int mn = c->f.multinum > 0 ? std::min(c->f.multinum, c->nlev - 1) : std::min(c->p.multimax, c->nlev - 1);
        const int lc = tail_start(c, mn);
        const int l = kind == kWarmLevel0 ? 0 : kind - 12;
        if (kind >= 13 && l >= c->nlev) return set_error(c, I3G_E_ARG, "level %d does not exist", l);
        auto warm = [&]() {
            if (kind == 11) vcycle_t<float>(c, mn, true);
            else if (kind == 12) { if (lc <= mn) tail_launch<float>(c, lc, mn); }
            else smooth_t<float>(c, l, 1, true, false);
        };
        for (int w = 0; w < 2; w++) warm();
        EventPair e;
        I3G_CUDA(e.create());
        I3G_CUDA(cudaEventRecord(e.a, c->st));
        for (int q = 0; q < reps; q++) warm();
        I3G_CUDA(cudaEventRecord(e.b, c->st));
        I3G_CUDA(cudaEventSynchronize(e.b));
        float t = 0;
        I3G_CUDA(cudaEventElapsedTime(&t, e.a, e.b));
        *ms = t / reps;
        *bytes = kind >= 13 || kind == kWarmLevel0 ? 68.0 * (double)c->lev[l].n : 0.0;
        I3G_CUDA(cudaGetLastError());
        return 0;
    }
    for (int w = 0; w < 2; w++) launch();   // warm-up (instruction caches, first-touch)
    int rc = cold_time(c, reps, launch, ms);
    if (rc) return rc;
    switch (kind) {
    case 0: *bytes = N * (8.0 * 7 + 8.0 * 0.5 + 8.0 * 0.5 + 1.0); break;
    case 7: *bytes = N * (4.0 * 7 + 4.0 * 0.5 + 4.0 * 0.5 + 1.0); break;
    case 8: *bytes = N * 68.0; break;
    case 10: *bytes = N * 116.0; break;
    case 1: *bytes = N * 116.0; break;
    case 2: *bytes = N * 4.0 * 8.0 * (1.0 + 1.0 / 8.0); break;
    case 3: *bytes = N * 4.0 * 8.0 * (2.0 + 1.0 / 8.0); break;
    default: *bytes = 0;
    }
    I3G_CUDA(cudaGetLastError());
    return 0;
}

}  // namespace i3g
