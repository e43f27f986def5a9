// markers.cu -- marker advection (movemark, mark3mg.c:2-397) and marker -> node averaging
// (ronurecalc, mark3mg.c:404-1015) for sm_100a.
//
// Markers live on the device as structure-of-arrays, sorted by cell inside cell tiles
// (4 x 32 x 4 cells): after every advection a counting sort by (tile, cell) regroups them.
// The marker -> node pass gives each CTA one tile and each warp one cell: the warp computes
// its markers' properties, then sums them per node of the cell in registers, and adds the
// per-cell sums to the tile's FP64 node sums in shared memory in 8 parity classes of cells
// that share no node -- no atomics inside the tile.  Each tile writes its box of node sums to
// a staging buffer and k_r2n_gather adds, per node, the boxes of the tiles holding it in a
// fixed order: no atomics at all, the same sums on every run.  The reference's scatter
// (mark3mg.c:848-924) adds into shared node arrays from many threads without atomics.  The
// only atomics of the file are the counters of the (tile, cell) sort.  An original-index
// array lets downloads return markers in the reference's order.
//
// Two arithmetic variants of the interpolation and rheology (template parameter EX, chosen by
// i3g_params.marker_exact): the reference's operation order (EX = true), and reciprocal tables,
// distance-form weights, factorised trilinear sums and explicit fused multiply-adds (EX = false,
// about twice as fast).  This file is compiled with -fmad=false so that the exact variant
// rounds like the CPU restatement (transcendentals may still differ in the last unit); the fast
// variant's fused operations are written out.

#include <algorithm>
#include <cmath>
#include <vector>
#include "heat_markers.cuh"

namespace i3g {

constexpr int TX = 4, TY = 32, TZ = 4;                       // cells per tile
constexpr int NBX = TX + 1, NBY = TY + 1, NBZ = TZ + 1;       // nodes per tile box
constexpr int NBOX = NBX * NBY * NBZ;
enum { A_NU, W_NU, A_XX, W_XX, A_XY, W_XY, A_XZ, W_XZ, A_YZ, W_YZ, A_RO, A_CP, A_KT, A_HT, A_ET, A_TK, A_RR, W_P, NACC };
enum { R_N0, R_N1, R_S0, R_S1, R_NU, R_DH, R_DV, R_SS, R_MM, R_LL, R_A0, R_A1, R_B0, R_B1, R_E0, R_E1,
       R_RO, R_BB, R_AA, R_CP, R_KT, R_KF, R_KP, R_HT };
enum { ERR_TYPE = 1, ERR_GRAIN = 2, ERR_WATER = 4, ERR_MELT = 8, ERR_DENSI = 16 };

struct Marks {
    float *x, *y, *z, *k, *w, *d, *v, *e, *ex, *ft, *rr, *rn;
    int8_t *t;
    int *id;
};

struct MarkerState {
    long n = 0;
    Marks a{}, b{};                 // current arrays and the sort target
    int *key = nullptr;             // sort key per marker: tile * cells per tile + cell in tile
    int *cnt = nullptr, *coff = nullptr, *cur = nullptr;   // per cell (+ inactive bin)
    int *off = nullptr;             // per tile: first marker (ntiles + 1 entries)
    int *bsum = nullptr;            // scan chunk sums
    int ntx = 0, nty = 0, ntz = 0, ntiles = 0;
    long nbins = 0;                 // cells of all tiles + inactive bin + end
    double *acc = nullptr;          // [2 * nodenum] node sums of the marker temperature change
    double *stage = nullptr;        // [ntiles][NACC][NBOX] per-tile node-box sums (no atomics)
    float *tk1 = nullptr;           // copy of T before boundary rows
    double *rock = nullptr;         // [24 * rocknum]
    int *err = nullptr, *herr = nullptr;
    int tbc_n = 0;                  // temperature boundary rows (level 0)
    int *tbc_node = nullptr, *tbc_p = nullptr;
    double *tbc_c = nullptr, *tbc_k = nullptr;
    bool sorted = false;
    // register caps of the FP64-latency-bound marker kernels (resident CTAs per SM they allow)
    int move_minb = 2;              // k_move: 2 (128 registers), 3 or 4 (I3G_MOVE_OCC)
    // k_heat_mark_cells: 2 CTAs per SM (64 registers; 4.5 ms instead of 6.6 ms at 129^3 with 56.6 M
    // markers on B200, its FP64 dependency chains need the extra warps), 1 with I3G_HEAT_OCC=1
    int heat_minb = 2;
    unsigned move_blocks = 1;       // persistent grid of k_move: resident CTAs on all SMs
    unsigned key_blocks = 1;        // the same for k_tile_key and k_heat_mark_anti
    cudaEvent_t up_ev = nullptr;    // end of an asynchronous upload on the copy stream
    bool up_pending = false;        // the compute stream has not waited for it yet
};

static MarkerState *ms(i3g_ctx *c) { return (MarkerState *)c->mk; }

// ------------------------------------------------------------------------------------
// device-side physics (same expressions as the CPU restatement)
// ------------------------------------------------------------------------------------
struct Grid {
    int nx, ny, nz;
    double xsize, ysize, zsize;
    const double *gx, *gy, *gz;     // shared-memory copies inside kernels
    double ux, uy, uz;              // 1 / spacing of a uniform axis, 0 when not uniform
    // per-axis tables of the fast arithmetic (shared memory, filled by load_grid<false>), index
    // 0 = x, 1 = y, 2 = z: mid-points (g[i] + g[i+1]) / 2, 1 / (g[i+1] - g[i]) and
    // 1 / ((g[i+2] - g[i]) / 2)
    const double *gm[3], *rl[3], *rm[3];
};

// Interpolation arithmetic of the marker kernels, chosen per launch by the template flag EX:
//  * EX = true: the reference's expressions in its operation order -- one correctly rounded
//    division per weight, separate multiply and add (this file is compiled with -fmad=false),
//    sums over the 8 corners in the reference's loop order.  Marker positions, strains and
//    types come out bit-identical to the reference's movemark.
//  * EX = false: the same weights from per-interval reciprocal tables, written as the distance
//    to the other node times 1 / spacing (so a point on a node gets exactly zero weight for the
//    other one, like the reference: a marker on a wall keeps its exactly zero wall velocity),
//    fused multiply-adds and factorised trilinear sums (y, then x, then z).  Each interpolated
//    value differs from the exact one by a few units in the last place of FP64 times the sum of
//    |node value x weight|; the new FP32 positions x + dt v differ only when that double lies
//    within ~1e-12 m of an FP32 rounding boundary.  Node averages and marker temperatures are
//    compared with tolerances either way.
template <bool EX>
__device__ __forceinline__ double quot(double a, double b, double rb) { return EX ? a / b : a * rb; }

__device__ __forceinline__ int bsearch_g(const double *g, int n, double x)
{
    int a = 0, b = n - 1, m;
    do {
        m = (a + b) / 2;
        if (g[m] > x) b = m; else a = m;
    } while ((b - a) > 1);
    if (a > n - 2) a = n - 2;
    return a;
}

// bsearch_g's result without the search on (nearly) uniform axes: a guess from the spacing,
// accepted only if it or a neighbour brackets x exactly as the search would; otherwise the
// search.  Identical results for any strictly increasing grid.
__device__ __forceinline__ int locate(const double *g, int n, double x, double inv)
{
    if (inv > 0) {
        const double t = (x - g[0]) * inv;
        if (t >= 0 && t < (double)n) {   // false for NaN
            int m = (int)t;
            if (m > n - 2) m = n - 2;
            if (g[m] <= x && (m == n - 2 || x < g[m + 1])) return m;
            if (m > 0 && g[m - 1] <= x && x < g[m]) return m - 1;
            if (m + 1 <= n - 2 && g[m + 1] <= x && (m + 1 == n - 2 || x < g[m + 2])) return m + 1;
        }
    }
    return bsearch_g(g, n, x);
}

__device__ __forceinline__ double clamp01(double d) { return d < 0 ? 0.0 : (d > 1.0 ? 1.0 : d); }

struct NodeF {
    const float *vx, *vy, *vz;
    const float *e[6], *s[6];
    const double *pr;
    long NY, NXY;
};

// One axis of a trilinear stencil: first node index i and the weights of nodes i and i + 1,
// computed with the reference's expressions (one correctly rounded division per weight).  The
// three staggered velocity components, and the four strain-rate groups, use a few distinct
// kinds per axis; computing each kind once per point, instead of once per corner, removes most
// of the FP64 divisions of the advection without changing a single rounding.
struct Ax {
    int i;
    double w0, w1;
};

__device__ __forceinline__ Ax clamped(Ax a) { return Ax{a.i, clamp01(a.w0), clamp01(a.w1)}; }

// node-line stencil of a component along its own axis (vxyzcalc1, e.g. Vx in x,
// mark3mg.c:2370-2395): i = cell clamped to [lo, n - 2 - hi_off]
// (axis q: 0 = x, 1 = y, 2 = z; the fast tables of that axis)
template <bool EX>
__device__ __forceinline__ Ax ax_line(const Grid &G, int q, const double *g, int n, int m, double x, int lo, int hi)
{
    int a = m;
    if (a < lo) a = lo;
    if (a > n - hi) a = n - hi;
    if (!EX) {
        // each weight is the distance to the other node times 1 / spacing: a point on a node
        // gets exactly 0 for the other one, as in the reference (a wall node's zero velocity
        // then stays exactly zero)
        const double r = G.rl[q][a];
        return Ax{a, (g[a + 1] - x) * r, (x - g[a]) * r};
    }
    const double d = g[a + 1] - g[a];
    double t0 = (g[a] - x) / d, t1 = (g[a + 1] - x) / d;
    t0 = -t0;
    return Ax{a, 1.0 - t0, 1.0 - t1};
}

// mid-point stencil across a staggered axis (vxyzcalc1, e.g. Vx in y): i = cell, minus one below
// the cell's mid-point, clamped to [0, n - 3]; nodes are the mid-points (g[k] + g[k+1]) / 2
template <bool EX>
__device__ __forceinline__ Ax ax_mid(const Grid &G, int q, const double *g, int n, int m, double x)
{
    int b = m;
    if (!EX) {
        const double *gm = G.gm[q];   // the same mid-point values, bit for bit
        if (x < gm[b]) b -= 1;
        if (b < 0) b = 0;
        if (b > n - 3) b = n - 3;
        const double r = G.rm[q][b];
        return Ax{b, (gm[b + 1] - x) * r, (x - gm[b]) * r};
    }
    if (x < (g[b] + g[b + 1]) / 2.0) b -= 1;
    if (b < 0) b = 0;
    if (b > n - 3) b = n - 3;
    const double d = (g[b + 2] - g[b]) / 2.0;
    double t0 = ((g[b] + g[b + 1]) / 2.0 - x) / d, t1 = ((g[b + 1] + g[b + 2]) / 2.0 - x) / d;
    t0 = -t0;
    return Ax{b, 1.0 - t0, 1.0 - t1};
}

// cell-centre stencil of epscalc1's normal components (mark3mg.c:2562-2600): i = cell, plus one
// above the mid-point, clamped to [1, n - 2]; nodes are (g[k-1] + g[k]) / 2; weights in [0, 1]
__device__ __forceinline__ Ax ax_cent_raw(const Grid &G, int q, int n, int m, double x)
{
    const double *gm = G.gm[q];
    int a = m;
    if (x > gm[a]) a += 1;
    if (a < 1) a = 1;
    if (a > n - 2) a = n - 2;
    const double r = G.rm[q][a - 1];   // 1 / ((g[a+1] - g[a-1]) / 2)
    return Ax{a, (gm[a] - x) * r, (x - gm[a - 1]) * r};
}

template <bool EX>
__device__ __forceinline__ Ax ax_cent(const Grid &G, int q, const double *g, int n, int m, double x)
{
    if (!EX) return clamped(ax_cent_raw(G, q, n, m, x));
    int a = m;
    if (x > (g[a] + g[a + 1]) / 2.0) a += 1;
    if (a < 1) a = 1;
    if (a > n - 2) a = n - 2;
    const double d = (g[a + 1] - g[a - 1]) / 2.0;
    double t0 = ((g[a - 1] + g[a]) / 2.0 - x) / d, t1 = ((g[a] + g[a + 1]) / 2.0 - x) / d;
    t0 = -t0;
    return Ax{a, clamp01(1.0 - t0), clamp01(1.0 - t1)};
}

// factorised trilinear sum of val(node) from node n0 (fast arithmetic): pairs along y, then x,
// then z, 14 FP64 operations instead of 28
template <class Fn>
__device__ __forceinline__ double tri_fact(int n0, int NY, int NXY, const Ax &X, const Ax &Y, const Ax &Z, Fn val)
{
    double u[2];
#pragma unroll
    for (int k3 = 0; k3 < 2; k3++) {
        const int b = n0 + k3 * NXY;
        const double a0 = fma(val(b + 1), Y.w1, val(b) * Y.w0);
        const double a1 = fma(val(b + NY + 1), Y.w1, val(b + NY) * Y.w0);
        u[k3] = fma(a1, X.w1, a0 * X.w0);
    }
    return fma(u[1], Z.w1, u[0] * Z.w0);
}

// sum over the 8 corners of f * ((ddx * ddy) * ddz) in the reference's loop order z, x, y (EX)
// or factorised (fast); node offsets in 32 bits (a level-0 grid has fewer than 2^31 nodes)
template <bool EX>
__device__ __forceinline__ double tri(const float *__restrict__ f, int NY, int NXY, const Ax &X, const Ax &Y, const Ax &Z)
{
    const int n0 = Z.i * NXY + X.i * NY + Y.i;
    if (!EX) return tri_fact(n0, NY, NXY, X, Y, Z, [&](int n) { return (double)__ldg(f + n); });
    const float *p = f + n0;
    double s = 0;
#pragma unroll
    for (int k3 = 0; k3 < 2; k3++) {
        const double ddz = k3 ? Z.w1 : Z.w0;
#pragma unroll
        for (int k1 = 0; k1 < 2; k1++) {
            const double ddx = k1 ? X.w1 : X.w0;
            const int base = k3 * NXY + k1 * NY;
#pragma unroll
            for (int k2 = 0; k2 < 2; k2++) {
                const double ddy = k2 ? Y.w1 : Y.w0;
                s += (double)__ldg(p + base + k2) * (ddx * ddy * ddz);
            }
        }
    }
    return s;
}

// Stencils of one point for vxyzcalc1: node-line and mid-point kinds on each axis.
struct VStencil {
    Ax lx, ly, lz, mx, my, mz;
};

// vxyzcalc1 (mark3mg.c:2347-2530): staggered trilinear velocity at a point.  Vx uses
// (line x, mid y, mid z), Vy (mid x, line y, mid z), Vz (mid x, mid y, line z).
template <bool EX>
__device__ __forceinline__ void vxyz(const Grid &G, const NodeF &F, double x, double y, double z, double *v, int *wn,
                                     VStencil *out = nullptr)
{
    const double *gx = G.gx, *gy = G.gy, *gz = G.gz;
    const int X = G.nx, Y = G.ny, Z = G.nz;
    if (x < 0) x = 0; if (x > G.xsize) x = G.xsize;
    if (y < 0) y = 0; if (y > G.ysize) y = G.ysize;
    if (z < 0) z = 0; if (z > G.zsize) z = G.zsize;
    const int m1 = wn[0] = locate(gx, X, x, G.ux), m2 = wn[1] = locate(gy, Y, y, G.uy), m3 = wn[2] = locate(gz, Z, z, G.uz);
    VStencil S;
    S.lx = ax_line<EX>(G, 0, gx, X, m1, x, 0, 2);
    S.ly = ax_line<EX>(G, 1, gy, Y, m2, y, 0, 2);
    S.lz = ax_line<EX>(G, 2, gz, Z, m3, z, 0, 2);
    S.mx = ax_mid<EX>(G, 0, gx, X, m1, x);
    S.my = ax_mid<EX>(G, 1, gy, Y, m2, y);
    S.mz = ax_mid<EX>(G, 2, gz, Z, m3, z);
    const int NY = (int)F.NY, NXY = (int)F.NXY;
    v[0] = tri<EX>(F.vx, NY, NXY, S.lx, S.my, S.mz);
    v[1] = tri<EX>(F.vy, NY, NXY, S.mx, S.ly, S.mz);
    v[2] = tri<EX>(F.vz, NY, NXY, S.mx, S.my, S.lz);
    if (out) *out = S;
}

// one shear group of epscalc1: strain rate, stress and the dissipation term 2 s e w
template <bool EX>
__device__ __forceinline__ void edge_group(const float *__restrict__ fe, const float *__restrict__ fs, int NY, int NXY,
                                           const Ax &AX, const Ax &AY, const Ax &AZ, double &e, double &s, double &d)
{
    const int n0 = AZ.i * NXY + AX.i * NY + AY.i;
    if (!EX) {
        e += tri_fact(n0, NY, NXY, AX, AY, AZ, [&](int n) { return (double)__ldg(fe + n); });
        s += tri_fact(n0, NY, NXY, AX, AY, AZ, [&](int n) { return (double)__ldg(fs + n); });
        d += tri_fact(n0, NY, NXY, AX, AY, AZ, [&](int n) { return 2.0 * (double)__ldg(fs + n) * (double)__ldg(fe + n); });
        return;
    }
#pragma unroll
    for (int k3 = 0; k3 < 2; k3++) {
        const double ddz = k3 ? AZ.w1 : AZ.w0;
#pragma unroll
        for (int k1 = 0; k1 < 2; k1++) {
            const double ddx = k1 ? AX.w1 : AX.w0;
#pragma unroll
            for (int k2 = 0; k2 < 2; k2++) {
                const double ddy = k2 ? AY.w1 : AY.w0;
                const int n = n0 + k3 * NXY + k1 * NY + k2;
                const double w = ddx * ddy * ddz;
                const float ev = __ldg(fe + n), sv = __ldg(fs + n);
                e += ev * w;
                s += sv * w;
                d += 2.0 * sv * ev * w;
            }
        }
    }
}

// epscalc1 (mark3mg.c:2535-2838) at the point of the first vxyz call, from its cell and
// mid-point stencils: normal strain rates, stresses and pressure at cell centres, the three
// shear groups on their edges, and the dissipation sum, each with weights clamped to [0, 1].
template <bool EX>
__device__ __forceinline__ void eps_from(const Grid &G, const NodeF &F, double x, double y, double z, const int *wn,
                                         const VStencil &S, double *e, double *s, double *dis)
{
    const double *gx = G.gx, *gy = G.gy, *gz = G.gz;
    const int X = G.nx, Y = G.ny, Z = G.nz;
    if (x < 0) x = 0; if (x > G.xsize) x = G.xsize;
    if (y < 0) y = 0; if (y > G.ysize) y = G.ysize;
    if (z < 0) z = 0; if (z > G.zsize) z = G.zsize;
    const int NY = (int)F.NY, NXY = (int)F.NXY;
    for (int i = 0; i < 7; i++) e[i] = 0;
    for (int i = 0; i < 6; i++) s[i] = 0;
    double d = 0;
    if (!EX) {
        const Ax cx = ax_cent<false>(G, 0, gx, X, wn[0], x), cy = ax_cent<false>(G, 1, gy, Y, wn[1], y),
                 cz = ax_cent<false>(G, 2, gz, Z, wn[2], z);
        const int n0 = cz.i * NXY + cx.i * NY + cy.i;
#pragma unroll
        for (int q = 0; q < 3; q++) {
            e[q] = tri_fact(n0, NY, NXY, cx, cy, cz, [&](int n) { return (double)__ldg(F.e[q] + n); });
            s[q] = tri_fact(n0, NY, NXY, cx, cy, cz, [&](int n) { return (double)__ldg(F.s[q] + n); });
        }
        e[6] = tri_fact(n0, NY, NXY, cx, cy, cz, [&](int n) { return __ldg(F.pr + n); });
        // the dissipation of the normal components: the FP32 sum of the three products per corner
        d = tri_fact(n0, NY, NXY, cx, cy, cz, [&](int n) {
            return (double)__fadd_rn(__fadd_rn(__fmul_rn(__ldg(F.s[0] + n), __ldg(F.e[0] + n)),
                                               __fmul_rn(__ldg(F.s[1] + n), __ldg(F.e[1] + n))),
                                     __fmul_rn(__ldg(F.s[2] + n), __ldg(F.e[2] + n)));
        });
        const Ax ix = clamped(ax_line<false>(G, 0, gx, X, wn[0], x, 1, 3)), iy = clamped(ax_line<false>(G, 1, gy, Y, wn[1], y, 1, 3)),
                 iz = clamped(ax_line<false>(G, 2, gz, Z, wn[2], z, 1, 3));
        const Ax qx = clamped(S.mx), qy = clamped(S.my), qz = clamped(S.mz);
        edge_group<false>(F.e[3], F.s[3], NY, NXY, ix, iy, qz, e[3], s[3], d);   // exy
        edge_group<false>(F.e[4], F.s[4], NY, NXY, ix, qy, iz, e[4], s[4], d);   // exz
        edge_group<false>(F.e[5], F.s[5], NY, NXY, qx, iy, iz, e[5], s[5], d);   // eyz
        *dis = d;
        return;
    }
    {
        const Ax cx = ax_cent<true>(G, 0, gx, X, wn[0], x), cy = ax_cent<true>(G, 1, gy, Y, wn[1], y),
                 cz = ax_cent<true>(G, 2, gz, Z, wn[2], z);
        const int n0 = cz.i * NXY + cx.i * NY + cy.i;
#pragma unroll
        for (int k3 = 0; k3 < 2; k3++) {
            const double ddz = k3 ? cz.w1 : cz.w0;
#pragma unroll
            for (int k1 = 0; k1 < 2; k1++) {
                const double ddx = k1 ? cx.w1 : cx.w0;
#pragma unroll
                for (int k2 = 0; k2 < 2; k2++) {
                    const double ddy = k2 ? cy.w1 : cy.w0;
                    const int n = n0 + k3 * NXY + k1 * NY + k2;
                    const double w = ddx * ddy * ddz;
                    const float exx = __ldg(F.e[0] + n), eyy = __ldg(F.e[1] + n), ezz = __ldg(F.e[2] + n);
                    const float sxx = __ldg(F.s[0] + n), syy = __ldg(F.s[1] + n), szz = __ldg(F.s[2] + n);
                    e[0] += exx * w; e[1] += eyy * w; e[2] += ezz * w;
                    s[0] += sxx * w; s[1] += syy * w; s[2] += szz * w;
                    d += (double)(__fadd_rn(__fadd_rn(__fmul_rn(sxx, exx), __fmul_rn(syy, eyy)), __fmul_rn(szz, ezz))) * w;
                    e[6] += __ldg(F.pr + n) * w;
                }
            }
        }
    }
    // edge groups: node lines clamped to [1, n - 3] and the mid-point stencils, weights in [0, 1]
    const Ax ix = clamped(ax_line<true>(G, 0, gx, X, wn[0], x, 1, 3)), iy = clamped(ax_line<true>(G, 1, gy, Y, wn[1], y, 1, 3)),
             iz = clamped(ax_line<true>(G, 2, gz, Z, wn[2], z, 1, 3));
    const Ax qx = clamped(S.mx), qy = clamped(S.my), qz = clamped(S.mz);
    edge_group<true>(F.e[3], F.s[3], NY, NXY, ix, iy, qz, e[3], s[3], d);   // exy
    edge_group<true>(F.e[4], F.s[4], NY, NXY, ix, qy, iz, e[4], s[4], d);   // exz
    edge_group<true>(F.e[5], F.s[5], NY, NXY, qx, iy, iz, e[5], s[5], d);   // eyz
    *dis = d;
}

// epscalc1 with the cell given (mark3mg.c:2535-2838)
__device__ void eps_at(const Grid &G, const NodeF &F, double x, double y, double z, const int *wn, double *e,
                       double *s, double *dis)
{
    const double *gx = G.gx, *gy = G.gy, *gz = G.gz;
    const int X = G.nx, Y = G.ny, Z = G.nz;
    for (int i = 0; i < 7; i++) e[i] = 0;
    for (int i = 0; i < 6; i++) s[i] = 0;
    *dis = 0;
    if (x < 0) x = 0; if (x > G.xsize) x = G.xsize;
    if (y < 0) y = 0; if (y > G.ysize) y = G.ysize;
    if (z < 0) z = 0; if (z > G.zsize) z = G.zsize;
    const int m1 = wn[0], m2 = wn[1], m3 = wn[2];
    int a, b, c;
    double dx, dy, dz, ddx, ddy, ddz, w;
    a = m1; if (x > (gx[a] + gx[a + 1]) / 2.0) a += 1; if (a < 1) a = 1; if (a > X - 2) a = X - 2;
    b = m2; if (y > (gy[b] + gy[b + 1]) / 2.0) b += 1; if (b < 1) b = 1; if (b > Y - 2) b = Y - 2;
    c = m3; if (z > (gz[c] + gz[c + 1]) / 2.0) c += 1; if (c < 1) c = 1; if (c > Z - 2) c = Z - 2;
    dx = (gx[a + 1] - gx[a - 1]) / 2.0; dy = (gy[b + 1] - gy[b - 1]) / 2.0; dz = (gz[c + 1] - gz[c - 1]) / 2.0;
    for (int k3 = c; k3 <= c + 1; k3++) {
        ddz = ((gz[k3 - 1] + gz[k3]) / 2.0 - z) / dz; if (k3 == c) ddz = -ddz; ddz = clamp01(1.0 - ddz);
        for (int k1 = a; k1 <= a + 1; k1++) {
            ddx = ((gx[k1 - 1] + gx[k1]) / 2.0 - x) / dx; if (k1 == a) ddx = -ddx; ddx = clamp01(1.0 - ddx);
            for (int k2 = b; k2 <= b + 1; k2++) {
                ddy = ((gy[k2 - 1] + gy[k2]) / 2.0 - y) / dy; if (k2 == b) ddy = -ddy; ddy = clamp01(1.0 - ddy);
                const long n = k3 * F.NXY + (long)k1 * F.NY + k2;
                w = ddx * ddy * ddz;
                const float exx = F.e[0][n], eyy = F.e[1][n], ezz = F.e[2][n];
                const float sxx = F.s[0][n], syy = F.s[1][n], szz = F.s[2][n];
                e[0] += exx * w; e[1] += eyy * w; e[2] += ezz * w;
                s[0] += sxx * w; s[1] += syy * w; s[2] += szz * w;
                *dis += (double)(__fadd_rn(__fadd_rn(__fmul_rn(sxx, exx), __fmul_rn(syy, eyy)), __fmul_rn(szz, ezz))) * w;
                e[6] += F.pr[n] * w;
            }
        }
    }
    a = m1; if (a < 1) a = 1; if (a > X - 3) a = X - 3;
    b = m2; if (b < 1) b = 1; if (b > Y - 3) b = Y - 3;
    c = m3; if (z < (gz[c] + gz[c + 1]) / 2.0) c -= 1; if (c < 0) c = 0; if (c > Z - 3) c = Z - 3;
    dx = gx[a + 1] - gx[a]; dy = gy[b + 1] - gy[b]; dz = (gz[c + 2] - gz[c]) / 2.0;
    for (int k3 = c; k3 <= c + 1; k3++) {
        ddz = ((gz[k3] + gz[k3 + 1]) / 2.0 - z) / dz; if (k3 == c) ddz = -ddz; ddz = clamp01(1.0 - ddz);
        for (int k1 = a; k1 <= a + 1; k1++) {
            ddx = (gx[k1] - x) / dx; if (k1 == a) ddx = -ddx; ddx = clamp01(1.0 - ddx);
            for (int k2 = b; k2 <= b + 1; k2++) {
                ddy = (gy[k2] - y) / dy; if (k2 == b) ddy = -ddy; ddy = clamp01(1.0 - ddy);
                const long n = k3 * F.NXY + (long)k1 * F.NY + k2;
                w = ddx * ddy * ddz;
                e[3] += F.e[3][n] * w; s[3] += F.s[3][n] * w;
                *dis += 2.0 * F.s[3][n] * F.e[3][n] * w;
            }
        }
    }
    a = m1; if (a < 1) a = 1; if (a > X - 3) a = X - 3;
    b = m2; if (y < (gy[b] + gy[b + 1]) / 2.0) b -= 1; if (b < 0) b = 0; if (b > Y - 3) b = Y - 3;
    c = m3; if (c < 1) c = 1; if (c > Z - 3) c = Z - 3;
    dx = gx[a + 1] - gx[a]; dy = (gy[b + 2] - gy[b]) / 2.0; dz = gz[c + 1] - gz[c];
    for (int k3 = c; k3 <= c + 1; k3++) {
        ddz = (gz[k3] - z) / dz; if (k3 == c) ddz = -ddz; ddz = clamp01(1.0 - ddz);
        for (int k1 = a; k1 <= a + 1; k1++) {
            ddx = (gx[k1] - x) / dx; if (k1 == a) ddx = -ddx; ddx = clamp01(1.0 - ddx);
            for (int k2 = b; k2 <= b + 1; k2++) {
                ddy = ((gy[k2] + gy[k2 + 1]) / 2.0 - y) / dy; if (k2 == b) ddy = -ddy; ddy = clamp01(1.0 - ddy);
                const long n = k3 * F.NXY + (long)k1 * F.NY + k2;
                w = ddx * ddy * ddz;
                e[4] += F.e[4][n] * w; s[4] += F.s[4][n] * w;
                *dis += 2.0 * F.s[4][n] * F.e[4][n] * w;
            }
        }
    }
    a = m1; if (x < (gx[a] + gx[a + 1]) / 2.0) a -= 1; if (a < 0) a = 0; if (a > X - 3) a = X - 3;
    b = m2; if (b < 1) b = 1; if (b > Y - 3) b = Y - 3;
    c = m3; if (c < 1) c = 1; if (c > Z - 3) c = Z - 3;
    dx = (gx[a + 2] - gx[a]) / 2.0; dy = gy[b + 1] - gy[b]; dz = gz[c + 1] - gz[c];
    for (int k3 = c; k3 <= c + 1; k3++) {
        ddz = (gz[k3] - z) / dz; if (k3 == c) ddz = -ddz; ddz = clamp01(1.0 - ddz);
        for (int k1 = a; k1 <= a + 1; k1++) {
            ddx = ((gx[k1] + gx[k1 + 1]) / 2.0 - x) / dx; if (k1 == a) ddx = -ddx; ddx = clamp01(1.0 - ddx);
            for (int k2 = b; k2 <= b + 1; k2++) {
                ddy = (gy[k2] - y) / dy; if (k2 == b) ddy = -ddy; ddy = clamp01(1.0 - ddy);
                const long n = k3 * F.NXY + (long)k1 * F.NY + k2;
                w = ddx * ddy * ddz;
                e[5] += F.e[5][n] * w; s[5] += F.s[5][n] * w;
                *dis += 2.0 * F.s[5][n] * F.e[5][n] * w;
            }
        }
    }
}

// prcalc1 (mark3mg.c:2917-3001)
template <bool EX>
__device__ double pr_at(const Grid &G, const double *pr, long NY, long NXY, double x, double y, double z, int *wn)
{
    const double *gx = G.gx, *gy = G.gy, *gz = G.gz;
    const int X = G.nx, Y = G.ny, Z = G.nz;
    if (x < 0) x = 0; if (x > G.xsize) x = G.xsize;
    if (y < 0) y = 0; if (y > G.ysize) y = G.ysize;
    if (z < 0) z = 0; if (z > G.zsize) z = G.zsize;
    const int m1 = wn[0] = locate(gx, X, x, G.ux), m2 = wn[1] = locate(gy, Y, y, G.uy), m3 = wn[2] = locate(gz, Z, z, G.uz);
    if (!EX) {   // prcalc1's cell-centre stencil: ax_cent without the clamp of the weights
        const Ax A = ax_cent_raw(G, 0, X, m1, x), B = ax_cent_raw(G, 1, Y, m2, y), C = ax_cent_raw(G, 2, Z, m3, z);
        return tri_fact(C.i * (int)NXY + A.i * (int)NY + B.i, (int)NY, (int)NXY, A, B, C, [&](int n) { return __ldg(pr + n); });
    }
    int a = m1, b = m2, c = m3;
    if (x > (gx[a] + gx[a + 1]) / 2.0) a += 1; if (a < 1) a = 1; if (a > X - 2) a = X - 2;
    if (y > (gy[b] + gy[b + 1]) / 2.0) b += 1; if (b < 1) b = 1; if (b > Y - 2) b = Y - 2;
    if (z > (gz[c] + gz[c + 1]) / 2.0) c += 1; if (c < 1) c = 1; if (c > Z - 2) c = Z - 2;
    const double dx = (gx[a + 1] - gx[a - 1]) / 2.0, dy = (gy[b + 1] - gy[b - 1]) / 2.0, dz = (gz[c + 1] - gz[c - 1]) / 2.0;
    // prcalc1's per-corner weights, computed once per axis (1 - (-q) = 1 + q exactly)
    const double wx[2] = {1.0 + ((gx[a - 1] + gx[a]) / 2.0 - x) / dx, 1.0 - ((gx[a] + gx[a + 1]) / 2.0 - x) / dx};
    const double wy[2] = {1.0 + ((gy[b - 1] + gy[b]) / 2.0 - y) / dy, 1.0 - ((gy[b] + gy[b + 1]) / 2.0 - y) / dy};
    const double wz[2] = {1.0 + ((gz[c - 1] + gz[c]) / 2.0 - z) / dz, 1.0 - ((gz[c] + gz[c + 1]) / 2.0 - z) / dz};
    const double *p0 = pr + ((int)(c * NXY) + a * (int)NY + b);
    double p = 0;
#pragma unroll
    for (int k3 = 0; k3 < 2; k3++)
#pragma unroll
        for (int k1 = 0; k1 < 2; k1++)
#pragma unroll
            for (int k2 = 0; k2 < 2; k2++) p += p0[k3 * (int)NXY + k1 * (int)NY + k2] * (wx[k1] * wy[k2] * wz[k3]);
    return p;
}

struct Phys {
    const double *rock;   // [24 * rocknum]
    int rocknum, densimod, viscmod, outgrid, markmod;
    double nubeg, nuend, nukoef, healrate, timesum;
    double zdeep, vdeep, tdeep, nudeep, teclmin, teclmax, eroslev, sedilev, waterlev;
    int *err;
};

__device__ __forceinline__ double RK(const Phys &P, int f, int t) { return P.rock[f * P.rocknum + t]; }

// viscalc (mark3mg.c:1114-1693): rheologies A-D, F + brittle; updates the strain sign and the
// formation time like the reference.  Returns -1 for the grain-damage rheology.
__device__ double visc(const Phys &P, double mtk, double mpb, int mm2, double epsin, double markrii1, float &me, float &mft)
{
    const double rt = 8.314 * mtk;
    double e1, k1, sduct, sbrit;
    const double strain = fabs((double)me);
    const double lamb = 1.0;
    double abrit = RK(P, R_A0, mm2), bbrit = RK(P, R_B0, mm2);
    const double E0 = RK(P, R_E0, mm2), E1 = RK(P, R_E1, mm2);
    if (strain > E1) { abrit = RK(P, R_A1, mm2); bbrit = RK(P, R_B1, mm2); }
    else if (strain > E0 && E1 > E0) {
        abrit = RK(P, R_A0, mm2) + (RK(P, R_A1, mm2) - RK(P, R_A0, mm2)) * (strain - E0) / (E1 - E0);
        bbrit = RK(P, R_B0, mm2) + (RK(P, R_B1, mm2) - RK(P, R_B0, mm2)) * (strain - E0) / (E1 - E0);
    }
    const double mpf = mpb * 1e+5;
    double nubrit = 0;
    if (epsin > 0 && (bbrit > 0 || abrit * lamb > 0) && mm2 > 1) {
        sbrit = abrit + bbrit * mpf * lamb;
        if (mpf < 0) sbrit = abrit + mpf;
        if (sbrit > 0) nubrit = 1.0 / (0.5 * sbrit / epsin / markrii1);
        else nubrit = 1.0 / RK(P, R_N0, mm2);
    }
    double nunewt = 0, nupowl = 0;
    const double nu = RK(P, R_NU, mm2), dh = RK(P, R_DH, mm2), dv = RK(P, R_DV, mm2), ss = RK(P, R_SS, mm2), mm = RK(P, R_MM, mm2);
    if (nu != 0) {
        if (dh == 0 && dv == 0 && (ss == 0 || mm == 1.0)) nunewt = 1.0 / nu;
        if ((dh != 0 || dv != 0) && (ss == 0 || mm == 1.0)) {
            e1 = (dh + dv * mpb) / rt;
            if (e1 > 150.0) e1 = 150.0;
            if (dh < 0 && dv > 0) { e1 = dh * (mtk - dv); if (e1 < -150.0) e1 = -150.0; }
            if (dh < 0 && dv < 0) { e1 = (-dh) * (1.0 - (mtk - (-dv)) / (-dv)) / 8.314 / (-dv); if (e1 > 150.0) e1 = 150.0; }
            nunewt = 1.0 / (nu * exp(e1));
        }
        if ((dh == 0 && dv == 0) && ss != 0 && mm != 1.0) {
            k1 = nu / pow(ss, mm - 1.0);
            nunewt = 1.0 / (0.5 * k1);
            sduct = pow(nu * epsin, 1.0 / mm);
            if (epsin > 0) nupowl = 1.0 / (0.5 * sduct / epsin);
        }
        if (nu > 0 && dh > 0 && (dh != 0 || dv != 0) && ss != 0 && mm != 1.0) {
            e1 = (dh + dv * mpb) / rt;
            if (e1 > 150.0) e1 = 150.0;
            e1 = exp(e1);
            k1 = nu / pow(ss, mm - 1.0);
            nunewt = 1.0 / (0.5 * k1 * e1);
            sduct = pow(nu * e1 * epsin, 1.0 / mm);
            if (epsin > 0) nupowl = 1.0 / (0.5 * sduct / epsin);
        }
        if (nu < 0) {
            e1 = (ss + mpb * RK(P, R_LL, mm2)) / rt;
            if (e1 > 150.0) e1 = 150.0;
            e1 = exp(e1);
            nunewt = 1.0 / (0.5 * pow(1.0 * 1e-3 / 5e-10, 2.5) * 8e+10 / RK(P, R_S1, mm2) * e1);
            nupowl = 0;
            if (epsin > 0) {
                e1 = (dh + dv * mpb) / rt / mm;
                if (e1 > 150.0) e1 = 150.0;
                e1 = exp(e1);
                nupowl = 1.0 / (0.5 * pow(epsin, 1.0 / mm - 1.0) * 8e+10 / pow(-nu, 1.0 / mm) * e1);
            }
        }
        if (dh < 0) return -1;
    }
    double nueff = nunewt + nupowl;
    if (mm2 == 7 || mm2 == 8 || mm2 == 9 || mm2 == 10) {
        if (mtk > 1300.0) mft = 0;
        else if (mft <= 0) mft = (float)P.timesum;
    }
    if (nubrit > nueff) {
        nueff = nubrit;
        if (me == 0) me = 1e-20f;
        me = fabsf(me);
    } else {
        me = -fabsf(me);
    }
    if (nueff <= 0) nueff = 1.0 / RK(P, R_N1, mm2);
    nueff = 1.0 / nueff;
    if (nueff < RK(P, R_N0, mm2)) nueff = RK(P, R_N0, mm2);
    if (nueff > RK(P, R_N1, mm2)) nueff = RK(P, R_N1, mm2);
    if (nueff < P.nubeg) nueff = P.nubeg;
    if (nueff > P.nuend) nueff = P.nuend;
    return nueff;
}

// Grid lines to shared memory (n = nx + ny + nz doubles); with EX = false also the fast
// arithmetic's tables: mid-points, 1 / spacing and 1 / half double-spacing (3 n more doubles,
// computed from the global copy, so no barrier is needed between the two)
template <bool EX>
__device__ __forceinline__ void load_grid(const Grid &Gg, double *sh, Grid &G)
{
    const int n = Gg.nx + Gg.ny + Gg.nz;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int q = i < Gg.nx ? 0 : i < Gg.nx + Gg.ny ? 1 : 2;
        const int j = i - (q == 0 ? 0 : q == 1 ? Gg.nx : Gg.nx + Gg.ny);
        const int na = q == 0 ? Gg.nx : q == 1 ? Gg.ny : Gg.nz;
        const double *g = q == 0 ? Gg.gx : q == 1 ? Gg.gy : Gg.gz;
        sh[i] = g[j];
        if (!EX) {
            sh[n + i] = j + 1 < na ? (g[j] + g[j + 1]) / 2.0 : 0.0;
            sh[2 * n + i] = j + 1 < na ? 1.0 / (g[j + 1] - g[j]) : 0.0;
            sh[3 * n + i] = j + 2 < na ? 1.0 / ((g[j + 2] - g[j]) / 2.0) : 0.0;
        }
    }
    __syncthreads();
    G = Gg;
    G.gx = sh; G.gy = sh + Gg.nx; G.gz = sh + Gg.nx + Gg.ny;
    if (!EX) {
        const int off[3] = {0, Gg.nx, Gg.nx + Gg.ny};
        for (int q = 0; q < 3; q++) {
            G.gm[q] = sh + n + off[q];
            G.rl[q] = sh + 2 * n + off[q];
            G.rm[q] = sh + 3 * n + off[q];
        }
    }
}

// second invariant (mark3mg.c:73-74 computes it as pow(., 0.5)): the correctly rounded square
// root of the same sum, which a pow of exponent 0.5 approximates to within its own error bound
__device__ __forceinline__ double inv2(const double *e)
{
    return sqrt(0.5 * (e[0] * e[0] + e[1] * e[1] + e[2] * e[2]) + e[3] * e[3] + e[4] * e[4] + e[5] * e[5]);
}

// ------------------------------------------------------------------------------------
// movemark: rheology update + RK4 (mark3mg.c:49-310)
// ------------------------------------------------------------------------------------
// one marker of movemark (mark3mg.c:49-310)
template <bool EX>
__device__ __forceinline__ void move_one(const Marks &M, long i, const Grid &G, const NodeF &F, const Phys &P, double timestep)
{
    int t = M.t[i];
    const float fx = M.x[i], fy = M.y[i], fz = M.z[i];
    const bool inbox = fx >= 0 && fy >= 0 && fz >= 0 && (double)fx <= G.xsize && (double)fy <= G.ysize && (double)fz <= G.zsize;
    if (!(inbox || (P.outgrid != 1 && (t < 50 || t >= 100)))) return;
    if (t >= 50) { atomicOr(P.err, ERR_TYPE); return; }
    const double yold = fy;
    double v1[3], e[7], s[6], dis;
    int wn[3];
    VStencil S0;
    vxyz<EX>(G, F, fx, fy, fz, v1, wn, &S0);
    eps_from<EX>(G, F, fx, fy, fz, wn, S0, e, s, &dis);
    const double eii = inv2(e), sii = inv2(s);
    const double mpb = e[6] * 1e-5;
    float mk = M.k[i], mv = M.v[i], me = M.e[i], mft = M.ft[i], mw = M.w[i];
    const double mtk = mk;
    if (t < 50 && mtk > 0) {
        double rii = 1.0;
        if (mv > 0 && fx > G.gx[3] && fx < G.gx[G.nx - 4] && fy > G.gy[3] && fy < G.gy[G.ny - 4] && fz > G.gz[3] && fz < G.gz[G.nz - 4])
            // the power law of the stress ratio; the fast arithmetic takes it as exp(0.87 log r)
            // (relative difference ~1e-15, far below the FP32 viscosity it feeds)
            rii *= EX ? pow(0.5 * sii / eii / mv, 0.87) : exp(0.87 * log(0.5 * sii / eii / mv));
        const double mnu = visc(P, mtk, mpb, t, eii, rii, me, mft);
        if (mnu < 0) { atomicOr(P.err, ERR_GRAIN); return; }
        mv = (float)mnu;
        if (me > 0) me += timestep * eii;
        if (me > 0) { me -= timestep * P.healrate; if (me < 0) me = 0; }
        else { me += timestep * P.healrate; if (me > 0) me = 0; }
    }
    double v[3];
    if (P.markmod == 1) { v[0] = v1[0]; v[1] = v1[1]; v[2] = v1[2]; }
    else {
        double v2[3], v3[3], v4[3];
        vxyz<EX>(G, F, fx + v1[0] * timestep / 2.0, fy + v1[1] * timestep / 2.0, fz + v1[2] * timestep / 2.0, v2, wn);
        vxyz<EX>(G, F, fx + v2[0] * timestep / 2.0, fy + v2[1] * timestep / 2.0, fz + v2[2] * timestep / 2.0, v3, wn);
        vxyz<EX>(G, F, fx + v3[0] * timestep, fy + v3[1] * timestep, fz + v3[2] * timestep, v4, wn);
        for (int k = 0; k < 3; k++) v[k] = quot<EX>(v1[k] + 2.0 * v2[k] + 2.0 * v3[k] + v4[k], 6.0, 1.0 / 6.0);
    }
    if (P.outgrid == 2) {
        if (fx < 0 || (double)fx > G.xsize) v[1] = v[2] = 0;
        if (fy < 0 || (double)fy > G.ysize) v[0] = v[2] = 0;
        if (fz < 0 || (double)fz > G.zsize) v[0] = v[1] = 0;
    }
    if (fy > P.zdeep && v[1] < 0 && mk < P.tdeep && t == 10) mk = (float)P.tdeep;
    if (fy > P.zdeep && v[1] < 0 && t != 10) { t = 10; mw = 0; }
    if (fy > P.zdeep && t != 10 && t != 9) { t = 9; mw = 0; }
    const float nx_ = (float)(fx + (timestep * v[0] - 0.0));
    const float ny_ = (float)(fy + timestep * v[1]);
    const float nz_ = (float)(fz + timestep * v[2]);
    if ((yold > P.vdeep && ny_ < P.vdeep) || (yold > P.zdeep && ny_ < P.zdeep)) {
        if (mk < P.tdeep) mk = (float)P.tdeep;
        t = 10;
    }
    if (nx_ < 0 || ny_ < 0 || nz_ < 0 || (double)nx_ > G.xsize || (double)ny_ > G.ysize || (double)nz_ > G.zsize) {
        mk = 0;
        mv = 0;
    }
    M.x[i] = nx_; M.y[i] = ny_; M.z[i] = nz_;
    M.k[i] = mk; M.v[i] = mv; M.e[i] = me; M.ft[i] = mft; M.w[i] = mw; M.t[i] = (int8_t)t;
}

// Persistent grid-stride launch (a few CTAs per SM): the grid lines are staged in shared memory
// once per CTA instead of once per 256 markers.  Markers are in (tile, cell) order from the last
// sort, so a warp's interpolation corners hit the same L1 lines.
template <bool EX, int MINB>
__global__ void __launch_bounds__(256, MINB) k_move(Marks M, long n, Grid Gg, NodeF F, Phys P, double timestep)
{
    extern __shared__ double shg[];
    Grid G;
    load_grid<EX>(Gg, shg, G);
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        move_one<EX>(M, i, G, F, P, timestep);
}

// ------------------------------------------------------------------------------------
// tile sort
// ------------------------------------------------------------------------------------
struct TileGeo { int ntx, nty, ntz, ntiles; };

// markers grouped into tiles: rock markers strictly inside the box (the set both ronurecalc,
// mark3mg.c:459, and the marker temperature update, heat3mg.c:623, visit)
__device__ __forceinline__ bool r2n_active(const Grid &G, float x, float y, float z, int t, float k)
{
    (void)k;
    return x > 0 && y > 0 && z > 0 && x < G.xsize && y < G.ysize && z < G.zsize && t < 50;
}

constexpr int CPT = TX * TY * TZ;   // cells per tile

// sort key: tile, then cell inside the tile (y fastest); inactive markers sort last
__device__ __forceinline__ int cell_key(int c1, int c2, int c3, const TileGeo &T)
{
    const int tile = ((c3 / TZ) * T.ntx + (c1 / TX)) * T.nty + (c2 / TY);
    return tile * CPT + ((c3 % TZ) * TX + (c1 % TX)) * TY + (c2 % TY);
}

// persistent grid-stride launch (grid lines staged once per CTA); every thread of a CTA runs the
// same number of iterations, so the warp-wide histogram votes see whole warps
__global__ void k_tile_key(Marks M, long n, Grid Gg, TileGeo T, int *key, int *cnt)
{
    extern __shared__ double shg[];
    Grid G;
    load_grid<true>(Gg, shg, G);
    for (long base = (long)blockIdx.x * blockDim.x; base < n; base += (long)gridDim.x * blockDim.x) {
        const long i = base + threadIdx.x;
        int kk = T.ntiles * CPT;
        if (i < n) {
            const float x = M.x[i], y = M.y[i], z = M.z[i];
            if (r2n_active(G, x, y, z, M.t[i], M.k[i])) {
                double xd = x, yd = y, zd = z;
                if (xd > G.xsize) xd = G.xsize;
                if (yd > G.ysize) yd = G.ysize;
                if (zd > G.zsize) zd = G.zsize;
                kk = cell_key(locate(G.gx, G.nx, xd, G.ux), locate(G.gy, G.ny, yd, G.uy), locate(G.gz, G.nz, zd, G.uz), T);
            }
            key[i] = kk;
        }
        // warp-aggregated histogram
        const unsigned act = __ballot_sync(0xffffffffu, i < n);
        if (i < n) {
            const unsigned peers = __match_any_sync(act, kk);
            const int leader = __ffs(peers) - 1;
            if ((int)(threadIdx.x & 31) == leader) atomicAdd(&cnt[kk], __popc(peers));
        }
    }
}

// exclusive scan of n counts in three passes: chunk sums, scan of the chunk sums, chunk scans
constexpr int kScanT = 1024, kScanPer = 4, kScanChunk = kScanT * kScanPer;

__device__ __forceinline__ int block_excl_scan(int v, int *total)
{
    __shared__ int wsum[kScanT / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = v;
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wsum[w] = x;
    __syncthreads();
    if (w == 0) {
        int t = lane < (int)(blockDim.x >> 5) ? wsum[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        wsum[lane] = t;   // inclusive
    }
    __syncthreads();
    const int before = (w ? wsum[w - 1] : 0) + x - v;
    *total = wsum[(blockDim.x >> 5) - 1];
    __syncthreads();
    return before;
}

__global__ void __launch_bounds__(kScanT) k_scan_part(const int *cnt, long n, int *bsum)
{
    const long b0 = (long)blockIdx.x * kScanChunk + (long)threadIdx.x * kScanPer;
    int s = 0;
    for (int q = 0; q < kScanPer; q++) s += b0 + q < n ? cnt[b0 + q] : 0;
    int total;
    block_excl_scan(s, &total);
    if (threadIdx.x == 0) bsum[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanT) k_scan_top(int *bsum, int nb)
{
    // one block: exclusive scan of nb chunk sums in place
    const int per = (nb + kScanT - 1) / kScanT;
    const int b = threadIdx.x * per;
    int s = 0;
    for (int q = b; q < b + per && q < nb; q++) s += bsum[q];
    int total;
    int run = block_excl_scan(s, &total);
    for (int q = b; q < b + per && q < nb; q++) { const int v = bsum[q]; bsum[q] = run; run += v; }
}

__global__ void __launch_bounds__(kScanT) k_scan_apply(const int *cnt, long n, const int *bsum, int *off, int *cur)
{
    const long b0 = (long)blockIdx.x * kScanChunk + (long)threadIdx.x * kScanPer;
    int v[kScanPer], s = 0;
    for (int q = 0; q < kScanPer; q++) { v[q] = b0 + q < n ? cnt[b0 + q] : 0; s += v[q]; }
    int total;
    int run = bsum[blockIdx.x] + block_excl_scan(s, &total);
    for (int q = 0; q < kScanPer; q++)
        if (b0 + q < n) { off[b0 + q] = run; cur[b0 + q] = run; run += v[q]; }
}

// tile offsets from cell offsets
__global__ void k_tile_off(const int *coff, int ntiles, int *toff)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t <= ntiles) toff[t] = coff[(long)t * CPT];
}

__global__ void k_tile_scatter(Marks A, Marks B, long n, const int *key, int *cur)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const unsigned act = __ballot_sync(0xffffffffu, i < n);
    if (i >= n) return;
    const int kk = key[i];
    const unsigned peers = __match_any_sync(act, kk);
    const int leader = __ffs(peers) - 1;
    const int lane = threadIdx.x & 31;
    int base = 0;
    if (lane == leader) base = atomicAdd(&cur[kk], __popc(peers));
    base = __shfl_sync(peers, base, leader);
    const long d = base + __popc(peers & ((1u << lane) - 1));
    B.x[d] = A.x[i]; B.y[d] = A.y[i]; B.z[d] = A.z[i]; B.k[d] = A.k[i]; B.w[d] = A.w[i]; B.d[d] = A.d[i];
    B.v[d] = A.v[i]; B.e[d] = A.e[i]; B.ex[d] = A.ex[i]; B.ft[d] = A.ft[i]; B.rr[d] = A.rr[i]; B.rn[d] = A.rn[i];
    B.t[d] = A.t[i]; B.id[d] = A.id[i];
}

// ------------------------------------------------------------------------------------
// ronurecalc: one CTA per tile, FP64 node sums staged in shared memory
// ------------------------------------------------------------------------------------
__device__ __forceinline__ void phase_density(const Phys &P, int mm2, double mtk, double mpb, double &mro)
{
    if ((mm2 >= 7 && mm2 <= 8) || (mm2 >= 16 && mm2 <= 18)) {   // mark3mg.c:530-587
        double rokf = 1.0;
        double p_ga_in = -9222.0 + mtk * 14.0; if (p_ga_in < 2000.0) p_ga_in = 2000.0;
        double p_pl_out = -1460.0 + mtk * 20.0; if (p_pl_out < 12000.0) p_pl_out = 12000.0;
        if (mpb > p_ga_in) { if (mpb >= p_pl_out) rokf *= 1.16; else rokf *= 1.0 + 0.16 * (mpb - p_ga_in) / (p_pl_out - p_ga_in); }
        const double p_st_in = 59100.0 + mtk * 22.6;
        if (mpb > p_st_in) rokf *= 1.06;
        const double p_sp_out = 354000.0 - mtk * 40.0, p_pv_in = 352000.0 - mtk * 40.0;
        if (mpb > p_pv_in) { if (mpb >= p_sp_out) rokf *= 1.08; else rokf *= 1.0 + 0.08 * (mpb - p_pv_in) / (p_sp_out - p_pv_in); }
        if (mtk < P.teclmax) { if (mtk < P.teclmin) rokf = 1.00; else rokf = 1.0 + (rokf - 1.0) * (mtk - P.teclmin) / (P.teclmax - P.teclmin); }
        mro *= rokf;
    }
    if (mm2 >= 9 && mm2 <= 14) {   // mark3mg.c:589-641
        double rokf = 1.0;
        const double p_ol_out = 91000.0 + mtk * 27.0;
        double p_sp_in = 66000.0 + mtk * 39.0;
        if (p_sp_in > p_ol_out - 2000.0) p_sp_in = p_ol_out - 2000.0;
        if (mpb > p_sp_in) { if (mpb >= p_ol_out) rokf *= 1.06; else rokf *= 1.0 + 0.06 * (mpb - p_sp_in) / (p_ol_out - p_sp_in); }
        const double p_sp_out = 304000.0 - mtk * 40.0, p_pv_in = 302000.0 - mtk * 40.0;
        if (mpb > p_pv_in) { if (mpb >= p_sp_out) rokf *= 1.11; else rokf *= 1.0 + 0.11 * (mpb - p_pv_in) / (p_sp_out - p_pv_in); }
        if (mtk < P.teclmax) { if (mtk < P.teclmin) rokf = 1.00; else rokf = 1.0 + (rokf - 1.0) * (mtk - P.teclmin) / (P.teclmax - P.teclmin); }
        mro *= rokf;
    }
}

// Each CTA owns one tile; markers are sorted by cell inside the tile.  A warp takes one cell:
// lanes first compute the properties of up to 32 of its markers (stage 1, one marker per
// lane) into a shared staging area, then lane = 4 * node + subset accumulates all 18 sums of
// one of the cell's 8 nodes over every fourth staged marker (stage 2, the same instruction
// stream in every lane), and two shuffles combine the subsets.  Cells are visited in 8 parity
// classes; cells of one class share no node, so the per-cell sums are added to the shared node
// sums without atomics, in a fixed order.
constexpr int kR2nWarps = 16;
constexpr int kStage = 15;   // ddx0 ddx1 ddy0 ddy1 ddz0 ddz1 vnu mro mcp*mro mkt mht mbb mtk mrr wxx

template <bool EX>
__global__ void __launch_bounds__(32 * kR2nWarps) k_r2n_cells(Marks M, const int *coff, Grid Gg, NodeF F, Phys P,
                                                              TileGeo T, double timestep, double *stage)
{
    extern __shared__ double sm[];
    double *sacc = sm;                                   // [NACC][NBOX]
    double *stg = sm + NACC * NBOX;                      // [kR2nWarps][32][kStage]
    int *scode = (int *)(stg + kR2nWarps * 32 * kStage);   // [kR2nWarps][32] per-marker corner masks
    double *shg = (double *)(scode + kR2nWarps * 32);      // grid lines (and the fast tables)
    for (int q = threadIdx.x; q < NACC * NBOX; q += blockDim.x) sacc[q] = 0;
    Grid G;
    load_grid<EX>(Gg, shg, G);   // contains __syncthreads
    const int tile = blockIdx.x;
    const int ty = tile % T.nty, rest = tile / T.nty, tx = rest % T.ntx, tz = rest / T.ntx;
    const int cx0 = tx * TX, cy0 = ty * TY, cz0 = tz * TZ;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double *my = stg + warp * 32 * kStage;
    int *mycode = scode + warp * 32;
    const int nd = lane >> 2, sub = lane & 3;   // node of the cell, marker subset (m % 4)
    const int iz = nd >> 2, ix = (nd >> 1) & 1, iy = nd & 1;
    const int vm = P.viscmod;
    for (int colour = 0; colour < 8; colour++) {
        const int pz = colour >> 2, px = (colour >> 1) & 1, py = colour & 1;
        for (int q = warp; q < CPT / 8; q += kR2nWarps) {
            const int ly = 2 * (q % (TY / 2)) + py, r2 = q / (TY / 2);
            const int lx = 2 * (r2 % (TX / 2)) + px, lz = 2 * (r2 / (TX / 2)) + pz;
            const long cell = (long)tile * CPT + (lz * TX + lx) * TY + ly;
            const int beg = coff[cell], end = coff[cell + 1];
            if (beg == end) continue;   // uniform over the warp
            double a[NACC];
#pragma unroll
            for (int q = 0; q < NACC; q++) a[q] = 0;
            for (int base = beg; base < end; base += 32) {
                // stage 1: one marker per lane
                bool ok = false;
                if (base + lane < end) {
                    const int i = base + lane;
                    int mm2 = M.t[i];
                    const float fx = M.x[i], fy = M.y[i], fz = M.z[i];
                    ok = M.k[i] > 0;
                    if (ok && mm2 > 1 && fy < P.eroslev) { mm2 = 0; M.t[i] = 0; }
                    if (ok && mm2 < 2) { atomicOr(P.err, ERR_WATER); ok = false; }
                    if (ok && mm2 > 20) { atomicOr(P.err, ERR_MELT); ok = false; }
                    if (ok && P.densimod >= 2) { atomicOr(P.err, ERR_DENSI); ok = false; }
                    if (ok) {
                        int wn[3];
                        const double mpb = pr_at<EX>(G, F.pr, F.NY, F.NXY, fx, fy, fz, wn) * 1e-5;
                        const double mtk = M.k[i];
                        double mnu = M.v[i];
                        if (mnu <= 0 || timestep <= 0) {
                            double e[7], sg[6], dis;
                            eps_at(G, F, fx, fy, fz, wn, e, sg, &dis);
                            float me = M.e[i], mft = M.ft[i];
                            mnu = visc(P, mtk, mpb, mm2, inv2(e), 1.0, me, mft);
                            if (mnu < 0) { atomicOr(P.err, ERR_GRAIN); ok = false; }
                            else { M.v[i] = (float)mnu; M.e[i] = me; M.ft[i] = mft; }
                        }
                        if (ok) {
                            double mbb = 0, mro = RK(P, R_RO, mm2);
                            if (P.densimod != 0) {   // dencalc1 (mark3mg.c:3006-3024)
                                const double bb = RK(P, R_BB, mm2);
                                mbb = bb / (1.0 - bb * (mtk - 298.15));
                                mro = mro * (1.0 - bb * (mtk - 298.15)) * (1.0 + RK(P, R_AA, mm2) * (mpb - 1.0) * 1e-3);
                            }
                            phase_density(P, mm2, mtk, mpb, mro);
                            const double mcp = RK(P, R_CP, mm2);
                            const double kp = RK(P, R_KP, mm2);   // exp(0) = 1 exactly: skip it
                            const double mkt = (RK(P, R_KT, mm2) + RK(P, R_KF, mm2) / (mtk + 77.0)) * (kp != 0 ? exp(kp * mpb) : 1.0);
                            if (fy > P.vdeep && mnu > P.nudeep) mnu = P.nudeep;
                            if (fy < 5e+4 && fx > G.xsize - 1e+4 && fz > 1.5e+5 && fz < 8.7e+5 && mnu > 1e+19) mnu = 1e+19;
                            const int m10 = wn[0], m20 = wn[1], m30 = wn[2];
                            double *st = my + lane * kStage;
                            if (EX) {
                                const double dx = G.gx[m10 + 1] - G.gx[m10], dy = G.gy[m20 + 1] - G.gy[m20], dz = G.gz[m30 + 1] - G.gz[m30];
                                st[0] = 1.0 - fabs((G.gx[m10] - fx) / dx);
                                st[1] = 1.0 - fabs((G.gx[m10 + 1] - fx) / dx);
                                st[2] = 1.0 - fabs((G.gy[m20] - fy) / dy);
                                st[3] = 1.0 - fabs((G.gy[m20 + 1] - fy) / dy);
                                st[4] = 1.0 - fabs((G.gz[m30] - fz) / dz);
                                st[5] = 1.0 - fabs((G.gz[m30 + 1] - fz) / dz);
                            } else {
                                // the marker lies inside its cell: 1 - |g_i - x| / d is the
                                // distance to the other node over d (exact zeros on nodes)
                                const double rx = G.rl[0][m10], ry = G.rl[1][m20], rz = G.rl[2][m30];
                                st[0] = (G.gx[m10 + 1] - fx) * rx;
                                st[1] = (fx - G.gx[m10]) * rx;
                                st[2] = (G.gy[m20 + 1] - fy) * ry;
                                st[3] = (fy - G.gy[m20]) * ry;
                                st[4] = (G.gz[m30 + 1] - fz) * rz;
                                st[5] = (fz - G.gz[m30]) * rz;
                            }
                            st[6] = vm == 0 ? mnu : vm == 1 ? log(mnu) : 1.0 / mnu;
                            st[7] = mro;
                            st[8] = mcp * mro;
                            st[9] = mkt;
                            st[10] = RK(P, R_HT, mm2);
                            st[11] = mbb;
                            st[12] = mtk;
                            st[13] = M.rr[i];
                            // cell-centre tent weight (node 1,1,1 only) and the per-axis corner
                            // masks of the nukoef gate and of the "nearer than half a cell" tests
                            st[14] = 8.0 * (0.5 - fabs(st[1] - 0.5)) * (0.5 - fabs(st[3] - 0.5)) * (0.5 - fabs(st[5] - 0.5));
                            const double nk = P.nukoef;
                            int code = 0;
#pragma unroll
                            for (int q = 0; q < 6; q++) code |= (st[q] > nk ? 1 : 0) << q | (st[q] > 0.5 ? 1 : 0) << (8 + q);
                            mycode[lane] = code;
                        }
                    }
                }
                unsigned valid = __ballot_sync(0xffffffffu, ok);
                __syncwarp();
                // stage 2: lane (node, subset) over the staged markers m of its subset, all 18 sums
                // (the sums are compared with the oracle to FP32 rounding, so they use fused
                // multiply-adds; the weights keep the reference's expressions)
                const int bx = 1 << ix, by = 4 << iy, bz = 16 << iz;
                for (unsigned mine = valid & (0x11111111u << sub); mine; mine &= mine - 1) {
                    const int m = __ffs(mine) - 1;
                    const double *st = my + m * kStage;
                    const int code = mycode[m];
                    const double ddx = st[ix], ddy = st[2 + iy], ddz = st[4 + iz];
                    const double swt = ddx * ddy * ddz;
                    const double vnu = st[6];
                    if (swt > 0) {
                        a[A_RO] = __fma_rn(st[7], swt, a[A_RO]); a[A_CP] = __fma_rn(st[8], swt, a[A_CP]);
                        a[A_KT] = __fma_rn(st[9], swt, a[A_KT]); a[A_HT] = __fma_rn(st[10], swt, a[A_HT]);
                        a[A_ET] = __fma_rn(st[11], swt, a[A_ET]); a[A_TK] = __fma_rn(st[12], swt, a[A_TK]);
                        a[A_RR] = __fma_rn(st[13], swt, a[A_RR]); a[W_P] += swt;
                    }
                    if ((code & (bx | by | bz)) == (bx | by | bz)) { a[A_NU] = __fma_rn(vnu, swt, a[A_NU]); a[W_NU] += swt; }
                    if (ix && iy && iz) { const double w1 = st[14]; a[A_XX] = __fma_rn(vnu, w1, a[A_XX]); a[W_XX] += w1; }
                    const int hx = (code >> (8 + ix)) & 1, hy = (code >> (10 + iy)) & 1, hz = (code >> (12 + iz)) & 1;
                    if (!iz && hx && hy) {
                        const double w1 = 8.0 * (ddx - 0.5) * (ddy - 0.5) * (0.5 - fabs(ddz - 0.5));
                        a[A_XY] = __fma_rn(vnu, w1, a[A_XY]); a[W_XY] += w1;
                    }
                    if (!iy && hx && hz) {
                        const double w1 = 8.0 * (ddx - 0.5) * (0.5 - fabs(ddy - 0.5)) * (ddz - 0.5);
                        a[A_XZ] = __fma_rn(vnu, w1, a[A_XZ]); a[W_XZ] += w1;
                    }
                    if (!ix && hy && hz) {
                        const double w1 = 8.0 * (0.5 - fabs(ddx - 0.5)) * (ddy - 0.5) * (ddz - 0.5);
                        a[A_YZ] = __fma_rn(vnu, w1, a[A_YZ]); a[W_YZ] += w1;
                    }
                }
                __syncwarp();
            }
            // the four subsets of each node, then one lane per node adds the cell's sums
#pragma unroll
            for (int q = 0; q < NACC; q++) {
                a[q] += __shfl_xor_sync(0xffffffffu, a[q], 1);
                a[q] += __shfl_xor_sync(0xffffffffu, a[q], 2);
            }
            if (sub == 0) {
                double *acc_n = sacc + ((lz + iz) * NBX + (lx + ix)) * NBY + (ly + iy);
#pragma unroll
                for (int q = 0; q < NACC; q++) acc_n[q * NBOX] += a[q];
            }
        }
        __syncthreads();
    }
    // the whole node box of the tile to its staging slot; k_r2n_gather adds the boxes that share
    // a node in a fixed order (no atomics, the same sums on every run)
    double *dst = stage + (long)tile * NACC * NBOX;
    for (int q = threadIdx.x; q < NACC * NBOX; q += blockDim.x) dst[q] = sacc[q];
    (void)cx0; (void)cy0; (void)cz0;
}

// tiles whose node box holds node coordinate v along one axis (t * T <= v <= t * T + T)
__device__ __forceinline__ void box_range(int v, int TT, int nt, int &t0, int &t1)
{
    t1 = min(v / TT, nt - 1);
    t0 = v % TT == 0 && v > 0 ? v / TT - 1 : t1;
    if (t0 > t1) t0 = t1;
}

// ------------------------------------------------------------------------------------
// marker temperatures after the heat solve (heat3mg.c:592-782)
// ------------------------------------------------------------------------------------
struct TkF { const float *tk0, *tk1, *tk, *tk2, *kt, *ro, *cp; long NY, NXY; };

// tkcalc1 (mark3mg.c:2844-2910): cell, spacings, 8 weights and the 4 interpolated T arrays
// wi[0..7] corner weights; wi[8..10] the cell's spacings (EX) or their reciprocals (fast)
template <bool EX>
__device__ __forceinline__ void tk_at(const Grid &G, const TkF &T, double x, double y, double z, double *e, int *wn,
                                      long *nodes, double *wi)
{
    const int m10 = wn[0] = locate(G.gx, G.nx, x, G.ux), m20 = wn[1] = locate(G.gy, G.ny, y, G.uy), m30 = wn[2] = locate(G.gz, G.nz, z, G.uz);
    e[0] = e[1] = e[2] = e[3] = 0;
    // per-axis weights 1 - |g - x| / d of the two cell nodes (one division each, or one product
    // with the reciprocal spacing)
    double wz[2], wx[2], wy[2];
    if (EX) {
        const double dx = wi[8] = G.gx[m10 + 1] - G.gx[m10];
        const double dy = wi[9] = G.gy[m20 + 1] - G.gy[m20];
        const double dz = wi[10] = G.gz[m30 + 1] - G.gz[m30];
        wz[0] = 1.0 - fabs((G.gz[m30] - z) / dz); wz[1] = 1.0 - fabs((G.gz[m30 + 1] - z) / dz);
        wx[0] = 1.0 - fabs((G.gx[m10] - x) / dx); wx[1] = 1.0 - fabs((G.gx[m10 + 1] - x) / dx);
        wy[0] = 1.0 - fabs((G.gy[m20] - y) / dy); wy[1] = 1.0 - fabs((G.gy[m20 + 1] - y) / dy);
    } else {
        // markers inside their cell: distance to the other node over the spacing
        const double rx = wi[8] = G.rl[0][m10], ry = wi[9] = G.rl[1][m20], rz = wi[10] = G.rl[2][m30];
        wz[0] = (G.gz[m30 + 1] - z) * rz; wz[1] = (z - G.gz[m30]) * rz;
        wx[0] = (G.gx[m10 + 1] - x) * rx; wx[1] = (x - G.gx[m10]) * rx;
        wy[0] = (G.gy[m20 + 1] - y) * ry; wy[1] = (y - G.gy[m20]) * ry;
    }
    int q = 0;
#pragma unroll
    for (int k3 = 0; k3 < 2; k3++) {
#pragma unroll
        for (int k1 = 0; k1 < 2; k1++) {
#pragma unroll
            for (int k2 = 0; k2 < 2; k2++) {
                const double swt = wi[q] = wx[k1] * wy[k2] * wz[k3];
                const long m4 = nodes[q] = (long)(m30 + k3) * T.NXY + (long)(m10 + k1) * T.NY + (m20 + k2);
                e[0] += swt * __ldg(T.tk0 + m4); e[1] += swt * __ldg(T.tk1 + m4); e[2] += swt * __ldg(T.tk + m4);
                e[3] += swt * __ldg(T.tk2 + m4);
                q++;
            }
        }
    }
}

// One CTA per tile, one warp per cell (8 parity classes, as in k_r2n_cells): stage 1 updates
// up to 32 markers of the cell (one per lane) and stages their node weights and subgrid
// change; stage 2 sums them per node (lane = 2 * node + quantity) without atomics.
constexpr int kHmStage = 9;   // wi[0..7], dtk1

template <bool EX, int MINB>
__global__ void __launch_bounds__(32 * kR2nWarps, MINB) k_heat_mark_cells(Marks M, const int *coff, Grid Gg, TkF T, TileGeo TG,
                                                                    double timestep, double heatdif, double zdeep,
                                                                    double tdeep, double *stage)
{
    extern __shared__ double sm[];
    double *sw0 = sm, *sw1 = sm + NBOX;
    double *stg = sm + 2 * NBOX;
    double *shg = stg + kR2nWarps * 32 * kHmStage;
    for (int q = threadIdx.x; q < 2 * NBOX; q += blockDim.x) sm[q] = 0;
    Grid G;
    load_grid<EX>(Gg, shg, G);
    const int tile = blockIdx.x;
    const int ty = tile % TG.nty, rest = tile / TG.nty, tx = rest % TG.ntx, tz = rest / TG.ntx;
    const int cx0 = tx * TX, cy0 = ty * TY, cz0 = tz * TZ;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double *my = stg + warp * 32 * kHmStage;
    const int nd = (lane >> 1) & 7, qty = lane & 1;
    const int iz = nd >> 2, ix = (nd >> 1) & 1, iy = nd & 1;
    for (int colour = 0; colour < 8; colour++) {
        const int pz = colour >> 2, px = (colour >> 1) & 1, py = colour & 1;
        for (int q = warp; q < CPT / 8; q += kR2nWarps) {
            const int ly = 2 * (q % (TY / 2)) + py, r2 = q / (TY / 2);
            const int lx = 2 * (r2 % (TX / 2)) + px, lz = 2 * (r2 / (TX / 2)) + pz;
            const long cell = (long)tile * CPT + (lz * TX + lx) * TY + ly;
            const int beg = coff[cell], end = coff[cell + 1];
            if (beg == end) continue;   // uniform over the warp
            double acc_w = 0;
            for (int base = beg; base < end; base += 32) {
                bool staged = false;
                if (base + lane < end) {
                    const int i = base + lane;
                    const float fx = M.x[i], fy = M.y[i], fz = M.z[i];
                    double e[4], wi[11];
                    int wn[3];
                    long nodes[8];
                    tk_at<EX>(G, T, fx, fy, fz, e, wn, nodes, wi);
                    float mk = M.k[i];
                    if (mk <= 0) {
                        mk = (float)e[3];
                        if (fy > zdeep && mk < tdeep) mk = (float)tdeep;
                    }
                    if (heatdif != 0) {
                        double mkt = 0, rocp = 0, mtk = T.tk[nodes[0]];
                        for (int qq = 0; qq < 8; qq++) {
                            mkt += T.kt[nodes[qq]] * wi[qq];
                            rocp += (double)__fmul_rn(T.ro[nodes[qq]], T.cp[nodes[qq]]) * wi[qq];
                            mtk = fmax(mtk, (double)T.tk[nodes[qq]]);
                        }
                        if ((wn[0] <= 0 || wn[0] >= G.nx - 2 || wn[1] <= 0 || wn[1] >= G.ny - 2 || wn[2] <= 0 || wn[2] >= G.nz - 2) &&
                            (mk + e[2] - e[3]) > mtk)
                            mk = (float)(mtk - e[2] + e[3]);
                        const double dtk = e[3] - (double)mk;
                        const double sum_h2 = EX ? 1.0 / wi[8] / wi[8] + 1.0 / wi[9] / wi[9] + 1.0 / wi[10] / wi[10]
                                                 : wi[8] * wi[8] + wi[9] * wi[9] + wi[10] * wi[10];
                        double dtk1 = -heatdif * mkt / rocp * 2.0 * sum_h2 * timestep;
                        if (dtk1 < -150.0) dtk1 = -150.0;
                        dtk1 = dtk * (1.0 - exp(dtk1));
                        mk = __fadd_rn(mk, (float)dtk1);
                        double *st = my + lane * kHmStage;
                        for (int qq = 0; qq < 8; qq++) st[qq] = wi[qq];
                        st[8] = dtk1;
                        staged = true;
                    }
                    mk = __fadd_rn(mk, (float)(e[2] - e[3]));
                    M.k[i] = mk;
                }
                unsigned valid = __ballot_sync(0xffffffffu, staged);
                __syncwarp();
                // wi[] is ordered z, x, y (tk_at loops m3, m1, m2): node index = (iz*2 + ix)*2 + iy = nd
                for (; valid; valid &= valid - 1) {
                    const double *st = my + (__ffs(valid) - 1) * kHmStage;
                    acc_w += qty ? st[8] * st[nd] : st[nd];
                }
                __syncwarp();
            }
            if (lane < 16) {
                const int lb = ((lz + iz) * NBX + (lx + ix)) * NBY + (ly + iy);
                (qty ? sw1 : sw0)[lb] += acc_w;
            }
        }
        __syncthreads();
    }
    double *dst = stage + (long)tile * 2 * NBOX;
    for (int q = threadIdx.x; q < 2 * NBOX; q += blockDim.x) dst[q] = sm[q];
    (void)cx0; (void)cy0; (void)cz0;
}

// per node: the weight sum and the weighted temperature change over the tile boxes holding it
// (fixed tile order), then their ratio: acc[n] = sum w, acc[N + n] = sum w dT / sum w
__global__ void k_heat_mark_gather(const double *stage, TileGeo TG, int nx, int ny, int nz, double *acc, long N)
{
    const long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    const int y = (int)(n % ny), x = (int)((n / ny) % nx), z = (int)(n / ((long)nx * ny));
    int x0, x1, y0, y1, z0, z1;
    box_range(x, TX, TG.ntx, x0, x1);
    box_range(y, TY, TG.nty, y0, y1);
    box_range(z, TZ, TG.ntz, z0, z1);
    double a0 = 0, a1 = 0;
    for (int tz = z0; tz <= z1; tz++)
        for (int tx = x0; tx <= x1; tx++)
            for (int ty = y0; ty <= y1; ty++) {
                const long tile = ((long)tz * TG.ntx + tx) * TG.nty + ty;
                const int q = ((z - tz * TZ) * NBX + (x - tx * TX)) * NBY + (y - ty * TY);
                a0 += stage[tile * 2 * NBOX + q];
                a1 += stage[tile * 2 * NBOX + NBOX + q];
            }
    acc[n] = a0;
    acc[N + n] = a0 != 0.0 ? a1 / a0 : a1;
}

// antidiffusion: marker T -= interpolated mean node change (heat3mg.c:722-779)
template <bool EX>
__global__ void k_heat_mark_anti(Marks M, const int *off, int ntiles, Grid Gg, TkF T, const double *acc, long N)
{
    extern __shared__ double shg[];
    Grid G;
    load_grid<EX>(Gg, shg, G);
    const long n = off[ntiles];
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        double e[4], wi[11];
        int wn[3];
        long nodes[8];
        tk_at<EX>(G, T, M.x[i], M.y[i], M.z[i], e, wn, nodes, wi);
        double iv = 0;
        for (int q = 0; q < 8; q++) iv -= acc[N + nodes[q]] * wi[q];
        M.k[i] = __fadd_rn(M.k[i], (float)iv);
    }
}

struct NodeOut {
    float *nu, *nxx, *nxy, *nxz, *nyz, *ro, *cp, *kt, *ht, *et, *tk, *rr, *tk1;
};

// node sums over the tile boxes holding the node (fixed tile order), then the normalisation of
// mark3mg.c:938-1002
__global__ void k_r2n_gather(const double *stage, TileGeo TG, int nx, int ny, int nz, NodeOut O, int vm, double nubeg,
                             double nuend)
{
    const long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long N = (long)nx * ny * nz;
    if (n >= N) return;
    const int y = (int)(n % ny), x = (int)((n / ny) % nx), z = (int)(n / ((long)nx * ny));
    int x0, x1, y0, y1, z0, z1;
    box_range(x, TX, TG.ntx, x0, x1);
    box_range(y, TY, TG.nty, y0, y1);
    box_range(z, TZ, TG.ntz, z0, z1);
    double acc[NACC];
#pragma unroll
    for (int a = 0; a < NACC; a++) acc[a] = 0;
    for (int tz = z0; tz <= z1; tz++)
        for (int tx = x0; tx <= x1; tx++)
            for (int ty = y0; ty <= y1; ty++) {
                const long tile = ((long)tz * TG.ntx + tx) * TG.nty + ty;
                const double *b = stage + tile * NACC * NBOX + ((z - tz * TZ) * NBX + (x - tx * TX)) * NBY + (y - ty * TY);
#pragma unroll
                for (int a = 0; a < NACC; a++) acc[a] += b[a * NBOX];
            }
#define ACC(a) acc[a]
#define FIN(field, A, W) if (ACC(W) > 0.01) { double v_ = ACC(A) / ACC(W); if (vm == 1) v_ = exp(v_); if (vm == 2) v_ = 1.0 / v_; O.field[n] = (float)v_; }
    FIN(nu, A_NU, W_NU);
    FIN(nxx, A_XX, W_XX);
    FIN(nxy, A_XY, W_XY);
    FIN(nxz, A_XZ, W_XZ);
    FIN(nyz, A_YZ, W_YZ);
    if (ACC(W_P) > 0.01) {
        const double w = ACC(W_P);
        const float ro = (float)(ACC(A_RO) / w);
        O.ro[n] = ro;
        O.cp[n] = (float)(ACC(A_CP) / w / ro);
        O.kt[n] = (float)(ACC(A_KT) / w);
        O.ht[n] = (float)(ACC(A_HT) / w);
        O.et[n] = (float)(ACC(A_ET) / w);
        O.tk[n] = (float)(ACC(A_TK) / w);
        O.rr[n] = (float)(ACC(A_RR) / w);
    }
#undef FIN
#undef ACC
    float nu = O.nu[n];
    if (nu < nubeg) nu = (float)nubeg;
    if (nu > nuend) nu = (float)nuend;
    O.nu[n] = nu;
    O.tk1[n] = O.tk[n];
}

// tkrecalc (heat3mg.c:849-899): T = c + k * T_before(partner)
__global__ void k_tk_bc(float *tk, const float *tk1, int n, const int *node, const int *p, const double *c, const double *k)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    // the reference's bondv1 and tk arrays are FP32: tk = c; tk += k * tk1 in FP32
    float v = (float)c[t];
    if (p[t] >= 0) v = __fadd_rn(v, __fmul_rn((float)k[t], tk1[p[t]]));
    tk[node[t]] = v;
}

__global__ void k_iota(int *id, long n)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) id[i] = (int)i;
}

// scatter the sorted markers back to their original positions for a download
__global__ void k_unsort(Marks A, Marks B, long n)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const long d = A.id[i];
    B.x[d] = A.x[i]; B.y[d] = A.y[i]; B.z[d] = A.z[i]; B.k[d] = A.k[i]; B.w[d] = A.w[i]; B.d[d] = A.d[i];
    B.v[d] = A.v[i]; B.e[d] = A.e[i]; B.ex[d] = A.ex[i]; B.ft[d] = A.ft[i]; B.rr[d] = A.rr[i]; B.rn[d] = A.rn[i];
    B.t[d] = A.t[i];
}

// ------------------------------------------------------------------------------------
// initial markers (in3mg.c:131-797)
// ------------------------------------------------------------------------------------
// SplitMix64 (Steele, Lea & Flood 2014) of (seed, counter): the jitter's random integers.  The
// reference draws them from the C library's rand() in marker order (in3mg.c:177-186); a
// counter-based generator gives every marker its own numbers independently of the others.
__device__ __forceinline__ unsigned long long splitmix64(unsigned long long seed, unsigned long long k)
{
    unsigned long long z = seed + (k + 1) * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// one marker: the position of in3mg.c:147-175 (sub-grid per cell, built by repeated addition
// of the marker spacing), the jitter of in3mg.c:177-186 with 31-bit random integers, the rock
// bodies of in3mg.c:548-797 in file order (later bodies win) and a linear temperature in y
__global__ void k_init_markers(Marks M, long n, Grid Gg, InitDev d)
{
    const long mm1 = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (mm1 >= n) return;
    const int mpc = d.mx * d.my * d.mz;
    const long cell = mm1 / mpc;
    const int q = (int)(mm1 - cell * mpc);
    const int m5 = q / (d.mx * d.my), m6 = (q / d.my) % d.mx, m7 = q % d.my;
    const long ny1 = Gg.ny - 1, nxy1 = (long)(Gg.nx - 1) * ny1;
    const long m3 = cell / nxy1, m1 = (cell / ny1) % (Gg.nx - 1), m2 = cell % ny1;
    const double dx = d.st[0] / (double)d.mx, dy = d.st[1] / (double)d.my, dz = d.st[2] / (double)d.mz;
    double x = (double)m1 * d.st[0] + dx / 2.0, y = (double)m2 * d.st[1] + dy / 2.0, z = (double)m3 * d.st[2] + dz / 2.0;
    for (int k = 0; k < m6; k++) x += dx;
    for (int k = 0; k < m7; k++) y += dy;
    for (int k = 0; k < m5; k++) z += dz;
    float fx = (float)x, fy = (float)y, fz = (float)z;
    if (d.nonstab) {
        const int span = 2 * d.nonstab + 1;
        const float nf = (float)d.nonstab;
        const int rx = (int)(splitmix64(d.seed, 3 * (unsigned long long)mm1) >> 33);
        const int ry = (int)(splitmix64(d.seed, 3 * (unsigned long long)mm1 + 1) >> 33);
        const int rz = (int)(splitmix64(d.seed, 3 * (unsigned long long)mm1 + 2) >> 33);
        fx = __fadd_rn(fx, __fmul_rn(__fdiv_rn((float)(rx % span - d.nonstab), nf), d.jit[0]));
        fy = __fadd_rn(fy, __fmul_rn(__fdiv_rn((float)(ry % span - d.nonstab), nf), d.jit[1]));
        fz = __fadd_rn(fz, __fmul_rn(__fdiv_rn((float)(rz % span - d.nonstab), nf), d.jit[2]));
    }
    int t = d.background;
    float ex = 0.f, e = 0.f;
    const double rx = (double)fx / Gg.xsize, ry = (double)fy / Gg.ysize, rz = (double)fz / Gg.zsize;
    for (int b = 0; b < d.nbodies; b++) {
        const BodyDev &B = d.bodies[b];
        bool in;
        if (B.shape == 0) {
            const double (*k)[4] = B.k;
            in = rx >= k[0][0] + k[0][1] * ry + k[0][2] * rz + k[0][3] * ry * rz &&
                 rx <= k[1][0] + k[1][1] * ry + k[1][2] * rz + k[1][3] * ry * rz &&
                 ry >= k[2][0] + k[2][1] * rx + k[2][2] * rz + k[2][3] * rx * rz &&
                 ry <= k[3][0] + k[3][1] * rx + k[3][2] * rz + k[3][3] * rx * rz &&
                 rz >= k[4][0] + k[4][1] * ry + k[4][2] * rx + k[4][3] * ry * rx &&
                 rz <= k[5][0] + k[5][1] * ry + k[5][2] * rx + k[5][3] * ry * rx;
        } else {
            const double ux = (rx - B.c[0]) / B.s[0], uy = (ry - B.c[1]) / B.s[1], uz = (rz - B.c[2]) / B.s[2];
            const double r = B.shape == 1 ? sqrt(ux * ux + uy * uy + uz * uz) : sqrt(ux * ux + uz * uz);
            in = r >= B.r0 && r <= B.r1 && (B.shape == 1 || fabs(uy) <= 1.0);
        }
        if (in) { t = B.rock; ex = B.ex; e = B.e; }
    }
    M.x[mm1] = fx; M.y[mm1] = fy; M.z[mm1] = fz;
    M.t[mm1] = (int8_t)t;
    M.ex[mm1] = ex; M.e[mm1] = e;
    M.k[mm1] = (float)(d.ttop + (d.tbot - d.ttop) * (double)fy / Gg.ysize);
    M.w[mm1] = 0.f; M.d[mm1] = 0.f; M.v[mm1] = 0.f; M.ft[mm1] = 0.f; M.rr[mm1] = 0.f; M.rn[mm1] = 0.f;
    M.id[mm1] = (int)mm1;
}

// ------------------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------------------
static inline unsigned nb(long n, int t = 256) { return (unsigned)((n + t - 1) / t); }

#define LAUNCH(kern, grid, block, smem, ...)                                               \
    do {                                                                                   \
        kern<<<(grid), (block), (smem), c->st>>>(__VA_ARGS__);                             \
        c->launches++;                                                                     \
    } while (0)

static int alloc_marks(i3g_ctx *c, Marks &M, long n)
{
    float **f[12] = {&M.x, &M.y, &M.z, &M.k, &M.w, &M.d, &M.v, &M.e, &M.ex, &M.ft, &M.rr, &M.rn};
    for (auto p : f) I3G_CUDA(cudaMalloc((void **)p, sizeof(float) * (n > 0 ? n : 1)));
    I3G_CUDA(cudaMalloc((void **)&M.t, n > 0 ? n : 1));
    I3G_CUDA(cudaMalloc((void **)&M.id, sizeof(int) * (n > 0 ? n : 1)));
    return 0;
}

static void free_marks(Marks &M)
{
    float *f[12] = {M.x, M.y, M.z, M.k, M.w, M.d, M.v, M.e, M.ex, M.ft, M.rr, M.rn};
    for (auto p : f) cudaFree(p);
    cudaFree(M.t);
    cudaFree(M.id);
}

// 1 / spacing when the grid lines are equally spaced to 1e-6, else 0 (locate() then searches)
static double uniform_inv(const double *g, int n)
{
    if (n < 2) return 0.0;
    const double h = (g[n - 1] - g[0]) / (n - 1);
    if (!(h > 0)) return 0.0;
    for (int i = 0; i + 1 < n; i++)
        if (std::fabs((g[i + 1] - g[i]) - h) > 1e-6 * h) return 0.0;
    return 1.0 / h;
}

static Grid grid_of(i3g_ctx *c)
{
    Grid G;
    G.nx = (int)c->m.xnumx; G.ny = (int)c->m.ynumy; G.nz = (int)c->m.znumz;
    G.xsize = c->m.xsize; G.ysize = c->m.ysize; G.zsize = c->m.zsize;
    G.gx = c->gx0; G.gy = c->gy0; G.gz = c->gz0;
    G.ux = uniform_inv(c->hgx, G.nx); G.uy = uniform_inv(c->hgy, G.ny); G.uz = uniform_inv(c->hgz, G.nz);
    return G;
}

static NodeF nodes_of(i3g_ctx *c)
{
    NodeF F;
    F.vx = c->vx; F.vy = c->vy; F.vz = c->vz;
    for (int a = 0; a < 6; a++) { F.e[a] = c->eps[a]; F.s[a] = c->sig[a]; }
    F.pr = c->pr;
    F.NY = c->m.ynumy;
    F.NXY = c->m.xnumx * c->m.ynumy;
    return F;
}

static Phys phys_of(i3g_ctx *c)
{
    MarkerState *S = ms(c);
    Phys P;
    P.rock = S->rock; P.rocknum = c->m.rocknum; P.densimod = c->p.densimod; P.viscmod = c->p.viscmod;
    P.outgrid = c->p.outgrid; P.markmod = c->p.markmod;
    P.nubeg = c->p.nubeg; P.nuend = c->p.nuend; P.nukoef = c->p.nukoef; P.healrate = c->p.healrate;
    P.timesum = c->m.timesum;
    P.zdeep = c->p.zdeep; P.vdeep = c->p.vdeep; P.tdeep = c->p.tdeep; P.nudeep = c->p.nudeep;
    P.teclmin = c->p.teclmin; P.teclmax = c->p.teclmax;
    P.eroslev = c->p.eroslev; P.sedilev = c->p.sedilev; P.waterlev = c->p.waterlev;
    P.err = S->err;
    return P;
}

// grid lines plus the fast arithmetic's three tables per axis (load_grid)
static size_t grid_smem(i3g_ctx *c) { return 4 * sizeof(double) * (c->m.xnumx + c->m.ynumy + c->m.znumz); }

// the marker kernels' arithmetic: the reference's operation order (marker_exact) or the fast one
static bool mexact(i3g_ctx *c) { return c->p.marker_exact != 0; }

template <bool EX>
static void launch_move_t(i3g_ctx *c, unsigned grid, const Marks &M, long n, const Grid &G, const NodeF &F, const Phys &P,
                          double dt)
{
    switch (ms(c)->move_minb) {
    case 3: LAUNCH((k_move<EX, 3>), grid, 256, grid_smem(c), M, n, G, F, P, dt); break;
    case 4: LAUNCH((k_move<EX, 4>), grid, 256, grid_smem(c), M, n, G, F, P, dt); break;
    default: LAUNCH((k_move<EX, 2>), grid, 256, grid_smem(c), M, n, G, F, P, dt); break;
    }
}

static void launch_move(i3g_ctx *c, unsigned grid, const Marks &M, long n, const Grid &G, const NodeF &F, const Phys &P,
                        double dt)
{
    if (mexact(c)) launch_move_t<true>(c, grid, M, n, G, F, P, dt);
    else launch_move_t<false>(c, grid, M, n, G, F, P, dt);
}

// resident k_move CTAs per SM (the same for both arithmetic variants: both are capped at the
// same register count by __launch_bounds__)
static int move_occupancy(i3g_ctx *c, int *per_sm)
{
    switch (ms(c)->move_minb) {
    case 3: I3G_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, k_move<false, 3>, 256, grid_smem(c))); break;
    case 4: I3G_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, k_move<false, 4>, 256, grid_smem(c))); break;
    default: I3G_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, k_move<false, 2>, 256, grid_smem(c))); break;
    }
    return 0;
}

static void launch_r2n(i3g_ctx *c, const Marks &M, const int *coff, const TileGeo &T, double timestep, double *stage);
static void launch_heat_mark(i3g_ctx *c, const Marks &M, const int *coff, const TkF &TK, const TileGeo &T, double timestep,
                             double *stage);
static size_t r2n_smem(i3g_ctx *c) { return sizeof(double) * (NACC * NBOX + kR2nWarps * 32 * kStage) + grid_smem(c) + sizeof(int) * kR2nWarps * 32; }
static size_t heat_mark_smem(i3g_ctx *c) { return sizeof(double) * (2 * NBOX + kR2nWarps * 32 * kHmStage) + grid_smem(c); }

static void launch_r2n(i3g_ctx *c, const Marks &M, const int *coff, const TileGeo &T, double timestep, double *stage)
{
    if (mexact(c))
        LAUNCH(k_r2n_cells<true>, ms(c)->ntiles, 32 * kR2nWarps, r2n_smem(c), M, coff, grid_of(c), nodes_of(c), phys_of(c), T,
               timestep, stage);
    else
        LAUNCH(k_r2n_cells<false>, ms(c)->ntiles, 32 * kR2nWarps, r2n_smem(c), M, coff, grid_of(c), nodes_of(c), phys_of(c), T,
               timestep, stage);
}

static void launch_heat_mark(i3g_ctx *c, const Marks &M, const int *coff, const TkF &TK, const TileGeo &T, double timestep,
                             double *stage)
{
    MarkerState *S = ms(c);
    const int nt = S->ntiles;
    const size_t sm = heat_mark_smem(c);
    const Grid G = grid_of(c);
    const double hd = c->p.heatdif, zd = c->p.zdeep, td = c->p.tdeep;
    if (mexact(c)) {
        if (S->heat_minb == 2) LAUNCH((k_heat_mark_cells<true, 2>), nt, 32 * kR2nWarps, sm, M, coff, G, TK, T, timestep, hd, zd, td, stage);
        else LAUNCH((k_heat_mark_cells<true, 1>), nt, 32 * kR2nWarps, sm, M, coff, G, TK, T, timestep, hd, zd, td, stage);
    } else {
        if (S->heat_minb == 2) LAUNCH((k_heat_mark_cells<false, 2>), nt, 32 * kR2nWarps, sm, M, coff, G, TK, T, timestep, hd, zd, td, stage);
        else LAUNCH((k_heat_mark_cells<false, 1>), nt, 32 * kR2nWarps, sm, M, coff, G, TK, T, timestep, hd, zd, td, stage);
    }
}

int markers_alloc(i3g_ctx *c)
{
    MarkerState *S = new MarkerState();
    c->mk = S;
    const long n = c->marknum, N = c->nodenum;
    S->n = n;
    int rc;
    if ((rc = alloc_marks(c, S->a, n)) || (rc = alloc_marks(c, S->b, n))) return rc;
    S->ntx = (int)((c->m.xnumx - 1 + TX - 1) / TX);
    S->nty = (int)((c->m.ynumy - 1 + TY - 1) / TY);
    S->ntz = (int)((c->m.znumz - 1 + TZ - 1) / TZ);
    S->ntiles = S->ntx * S->nty * S->ntz;
    I3G_CUDA(cudaMalloc((void **)&S->key, sizeof(int) * (n > 0 ? n : 1)));
    S->nbins = (long)S->ntiles * CPT + 2;
    const long nchunks = (S->nbins + kScanChunk - 1) / kScanChunk;
    I3G_CUDA(cudaMalloc((void **)&S->cnt, sizeof(int) * S->nbins));
    I3G_CUDA(cudaMalloc((void **)&S->coff, sizeof(int) * S->nbins));
    I3G_CUDA(cudaMalloc((void **)&S->cur, sizeof(int) * S->nbins));
    I3G_CUDA(cudaMalloc((void **)&S->off, sizeof(int) * (S->ntiles + 2)));
    I3G_CUDA(cudaMalloc((void **)&S->bsum, sizeof(int) * nchunks));
    I3G_CUDA(cudaMalloc((void **)&S->acc, sizeof(double) * 2 * N));
    I3G_CUDA(cudaMalloc((void **)&S->stage, sizeof(double) * (size_t)S->ntiles * NACC * NBOX));
    I3G_CUDA(cudaMalloc((void **)&S->tk1, sizeof(float) * N));
    const int rn = c->m.rocknum;
    std::vector<double> rk(24 * (size_t)std::max(rn, 1), 0.0);
    for (int f = 0; f < 24; f++)
        for (int t = 0; t < rn; t++) rk[(size_t)f * rn + t] = c->m.rock[f] ? c->m.rock[f][t] : 0.0;
    I3G_CUDA(cudaMalloc((void **)&S->rock, sizeof(double) * rk.size()));
    I3G_CUDA(cudaMemcpyAsync(S->rock, rk.data(), sizeof(double) * rk.size(), cudaMemcpyHostToDevice, c->st));
    I3G_CUDA(cudaMalloc((void **)&S->err, sizeof(int)));
    I3G_CUDA(cudaMallocHost((void **)&S->herr, sizeof(int)));
    // temperature boundary rows of level 0 (bondm[8*nodenum + node], heat3mg.c:859-889)
    std::vector<int> tn, tp;
    std::vector<double> tc, tkk;
    for (long b = 0; b < c->m.bondnum; b++) {
        const long row = c->m.bond_row[b];
        if (row < 8 * N || row >= 9 * N) continue;
        tn.push_back((int)(row - 8 * N));
        tp.push_back(c->m.bond_partner1[b] > 0 ? (int)(c->m.bond_partner1[b] - 1) : -1);
        if (tp.back() >= N) return set_error(c, I3G_E_BC, "temperature boundary partner beyond level 0");
        tc.push_back(c->m.bond_c[b]);
        tkk.push_back(c->m.bond_k[b]);
    }
    S->tbc_n = (int)tn.size();
    I3G_CUDA(cudaMalloc((void **)&S->tbc_node, sizeof(int) * (tn.size() + 1)));
    I3G_CUDA(cudaMalloc((void **)&S->tbc_p, sizeof(int) * (tn.size() + 1)));
    I3G_CUDA(cudaMalloc((void **)&S->tbc_c, sizeof(double) * (tn.size() + 1)));
    I3G_CUDA(cudaMalloc((void **)&S->tbc_k, sizeof(double) * (tn.size() + 1)));
    if (!tn.empty()) {
        I3G_CUDA(cudaMemcpyAsync(S->tbc_node, tn.data(), sizeof(int) * tn.size(), cudaMemcpyHostToDevice, c->st));
        I3G_CUDA(cudaMemcpyAsync(S->tbc_p, tp.data(), sizeof(int) * tp.size(), cudaMemcpyHostToDevice, c->st));
        I3G_CUDA(cudaMemcpyAsync(S->tbc_c, tc.data(), sizeof(double) * tc.size(), cudaMemcpyHostToDevice, c->st));
        I3G_CUDA(cudaMemcpyAsync(S->tbc_k, tkk.data(), sizeof(double) * tkk.size(), cudaMemcpyHostToDevice, c->st));
    }
    {
        int dev = 0, sms = 0, per_sm = 0;
        I3G_CUDA(cudaGetDevice(&dev));
        I3G_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        if (const char *e = getenv("I3G_MOVE_OCC")) S->move_minb = std::min(4, std::max(2, atoi(e)));
        if (const char *e = getenv("I3G_HEAT_OCC")) S->heat_minb = std::min(2, std::max(1, atoi(e)));
        if (int rc = move_occupancy(c, &per_sm)) return rc;
        S->move_blocks = (unsigned)std::max(1, sms * std::max(per_sm, 1));
        int a = 0, b = 0;
        I3G_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_tile_key, 256, grid_smem(c)));
        I3G_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_heat_mark_anti<false>, 256, grid_smem(c)));
        S->key_blocks = (unsigned)std::max(1, sms * std::max(std::min(a, b), 1));
    }
    I3G_CUDA(cudaFuncSetAttribute(k_r2n_cells<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)r2n_smem(c)));
    I3G_CUDA(cudaFuncSetAttribute(k_r2n_cells<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)r2n_smem(c)));
    I3G_CUDA(cudaFuncSetAttribute((k_heat_mark_cells<true, 1>), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)heat_mark_smem(c)));
    I3G_CUDA(cudaFuncSetAttribute((k_heat_mark_cells<true, 2>), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)heat_mark_smem(c)));
    I3G_CUDA(cudaFuncSetAttribute((k_heat_mark_cells<false, 1>), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)heat_mark_smem(c)));
    I3G_CUDA(cudaFuncSetAttribute((k_heat_mark_cells<false, 2>), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)heat_mark_smem(c)));
    for (auto f : {k_move<true, 2>, k_move<true, 3>, k_move<true, 4>, k_move<false, 2>, k_move<false, 3>, k_move<false, 4>})
        I3G_CUDA(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)grid_smem(c)));
    for (auto f : {k_heat_mark_anti<true>, k_heat_mark_anti<false>})
        I3G_CUDA(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)grid_smem(c)));
    I3G_CUDA(cudaFuncSetAttribute(k_tile_key, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)grid_smem(c)));
    I3G_CUDA(cudaStreamSynchronize(c->st));
    // upload the host markers
    return markers_upload(c, &c->m);
}

void markers_free(i3g_ctx *c)
{
    MarkerState *S = ms(c);
    if (!S) return;
    if (c->cst) cudaStreamSynchronize(c->cst);   // no upload may still target the buffers freed here
    free_marks(S->a);
    free_marks(S->b);
    cudaFree(S->key); cudaFree(S->cnt); cudaFree(S->coff); cudaFree(S->off); cudaFree(S->cur); cudaFree(S->bsum); cudaFree(S->acc); cudaFree(S->stage); cudaFree(S->tk1);
    cudaFree(S->rock); cudaFree(S->err);
    if (S->herr) cudaFreeHost(S->herr);
    if (S->up_ev) cudaEventDestroy(S->up_ev);
    cudaFree(S->tbc_node); cudaFree(S->tbc_p); cudaFree(S->tbc_c); cudaFree(S->tbc_k);
    delete S;
    c->mk = nullptr;
}

// make the compute stream wait for an asynchronous marker upload still in flight
static int markers_wait(i3g_ctx *c)
{
    MarkerState *S = ms(c);
    if (S && S->up_pending) {
        I3G_CUDA(cudaStreamWaitEvent(c->st, S->up_ev, 0));
        S->up_pending = false;
    }
    return 0;
}

int markers_upload(i3g_ctx *c, const i3g_model *m, bool async)
{
    MarkerState *S = ms(c);
    if (!S) return 0;
    const long n = S->n;
    if (m->marknum != n) return set_error(c, I3G_E_ARG, "marker count changed (%lld != %ld)", (long long)m->marknum, n);
    int rc = markers_wait(c);
    if (rc) return rc;
    cudaStream_t st = c->st;
    if (async) {
        // the copies may only overwrite the markers once all earlier work on them is done
        if (!S->up_ev) I3G_CUDA(cudaEventCreateWithFlags(&S->up_ev, cudaEventDisableTiming));
        I3G_CUDA(cudaEventRecord(S->up_ev, c->st));
        I3G_CUDA(cudaStreamWaitEvent(c->cst, S->up_ev, 0));
        st = c->cst;
    }
    Marks &A = S->a;
    const float *src[12] = {m->markx, m->marky, m->markz, m->markk, m->markw, m->markd, m->markv, m->marke,
                            m->markex, m->markft, m->markrr, m->markrn};
    float *dst[12] = {A.x, A.y, A.z, A.k, A.w, A.d, A.v, A.e, A.ex, A.ft, A.rr, A.rn};
    for (int f = 0; f < 12; f++) {
        if (src[f]) I3G_CUDA(cudaMemcpyAsync(dst[f], src[f], sizeof(float) * n, cudaMemcpyHostToDevice, st));
        else I3G_CUDA(cudaMemsetAsync(dst[f], 0, sizeof(float) * n, st));
    }
    if (n) I3G_CUDA(cudaMemcpyAsync(A.t, m->markt, n, cudaMemcpyHostToDevice, st));
    if (n) {
        k_iota<<<nb(n), 256, 0, st>>>(A.id, n);
        c->launches++;
    }
    if (async) {
        I3G_CUDA(cudaEventRecord(S->up_ev, c->cst));
        S->up_pending = true;
    }
    S->sorted = false;
    return 0;
}

int markers_init(i3g_ctx *c, const InitDev &d)
{
    MarkerState *S = ms(c);
    if (!S || !S->n) return 0;
    if (int rc = markers_wait(c)) return rc;
    LAUNCH(k_init_markers, nb(S->n), 256, 0, S->a, S->n, grid_of(c), d);
    I3G_CUDA(cudaGetLastError());
    S->sorted = false;
    return 0;
}

int markers_download(i3g_ctx *c, i3g_model *m)
{
    MarkerState *S = ms(c);
    if (!S || !S->n) return 0;
    if (int rc = markers_wait(c)) return rc;
    const long n = S->n;
    LAUNCH(k_unsort, nb(n), 256, 0, S->a, S->b, n);
    Marks &B = S->b;
    float *dst[12] = {m->markx, m->marky, m->markz, m->markk, m->markw, m->markd, m->markv, m->marke,
                      m->markex, m->markft, m->markrr, m->markrn};
    const float *src[12] = {B.x, B.y, B.z, B.k, B.w, B.d, B.v, B.e, B.ex, B.ft, B.rr, B.rn};
    for (int f = 0; f < 12; f++)
        if (dst[f]) I3G_CUDA(cudaMemcpyAsync(dst[f], src[f], sizeof(float) * n, cudaMemcpyDeviceToHost, c->st));
    if (m->markt) I3G_CUDA(cudaMemcpyAsync(m->markt, B.t, n, cudaMemcpyDeviceToHost, c->st));
    return 0;
}

static int check_err(i3g_ctx *c, const char *what)
{
    MarkerState *S = ms(c);
    I3G_CUDA(cudaMemcpyAsync(S->herr, S->err, sizeof(int), cudaMemcpyDeviceToHost, c->st));
    I3G_CUDA(cudaStreamSynchronize(c->st));
    const int e = *S->herr;
    if (!e) return 0;
    if (e & ERR_TYPE) return set_error(c, I3G_E_UNSUPPORTED, "%s: fluid or immobile marker types (>= 50) are not supported", what);
    if (e & ERR_GRAIN) return set_error(c, I3G_E_UNSUPPORTED, "%s: grain-damage rheology (markdh < 0) is not supported", what);
    if (e & ERR_WATER) return set_error(c, I3G_E_UNSUPPORTED, "%s: air/water marker types 0-1 are not supported", what);
    if (e & ERR_MELT) return set_error(c, I3G_E_UNSUPPORTED, "%s: molten rock types > 20 are not supported", what);
    return set_error(c, I3G_E_UNSUPPORTED, "%s: densimod >= 2 (thermodynamic database) is not supported", what);
}

int markers_move(i3g_ctx *c, double timestep)
{
    MarkerState *S = ms(c);
    if (!S->n || timestep == 0) return 0;
    if (int rc = markers_wait(c)) return rc;
    EventPair ev;
    I3G_CUDA(ev.create());
    cudaEvent_t e0 = ev.a, e1 = ev.b;
    I3G_CUDA(cudaEventRecord(e0, c->st));
    I3G_CUDA(cudaMemsetAsync(S->err, 0, sizeof(int), c->st));
    launch_move(c, std::min(nb(S->n), S->move_blocks), S->a, S->n, grid_of(c), nodes_of(c), phys_of(c), timestep);
    I3G_CUDA(cudaGetLastError());
    I3G_CUDA(cudaEventRecord(e1, c->st));
    int rc = check_err(c, "movemark");
    float ms_ = 0;
    cudaEventElapsedTime(&ms_, e0, e1);
    c->st_.ms_move = ms_;
    S->sorted = false;
    return rc;
}

static int sort_markers(i3g_ctx *c)
{
    MarkerState *S = ms(c);
    const long n = S->n;
    TileGeo T{S->ntx, S->nty, S->ntz, S->ntiles};
    const long nbins = S->nbins;
    const unsigned nchunks = (unsigned)((nbins + kScanChunk - 1) / kScanChunk);
    I3G_CUDA(cudaMemsetAsync(S->cnt, 0, sizeof(int) * nbins, c->st));
    LAUNCH(k_tile_key, std::min(nb(n), S->key_blocks), 256, grid_smem(c), S->a, n, grid_of(c), T, S->key, S->cnt);
    LAUNCH(k_scan_part, nchunks, kScanT, 0, (const int *)S->cnt, nbins, S->bsum);
    LAUNCH(k_scan_top, 1, kScanT, 0, S->bsum, (int)nchunks);
    LAUNCH(k_scan_apply, nchunks, kScanT, 0, (const int *)S->cnt, nbins, (const int *)S->bsum, S->coff, S->cur);
    LAUNCH(k_tile_off, nb(S->ntiles + 1), 256, 0, (const int *)S->coff, S->ntiles, S->off);
    LAUNCH(k_tile_scatter, nb(n), 256, 0, S->a, S->b, n, (const int *)S->key, S->cur);
    std::swap(S->a, S->b);
    S->sorted = true;
    return 0;
}

int markers_to_nodes(i3g_ctx *c, double timestep)
{
    MarkerState *S = ms(c);
    const long N = c->nodenum;
    if (int rc = markers_wait(c)) return rc;
    EventPair ev;
    I3G_CUDA(ev.create());
    cudaEvent_t e0 = ev.a, e1 = ev.b;
    I3G_CUDA(cudaEventRecord(e0, c->st));
    I3G_CUDA(cudaMemsetAsync(S->err, 0, sizeof(int), c->st));
    int rc = 0;
    if (S->n) rc = sort_markers(c);
    if (rc) return rc;
    TileGeo T{S->ntx, S->nty, S->ntz, S->ntiles};
    if (S->n)
        launch_r2n(c, S->a, (const int *)S->coff, T, timestep, S->stage);
    else
        I3G_CUDA(cudaMemsetAsync(S->stage, 0, sizeof(double) * (size_t)S->ntiles * NACC * NBOX, c->st));
    NodeOut O{c->lev[0].nu, c->nxx, c->nxy, c->nxz, c->nyz, c->ro, c->cp, c->kt, c->ht, c->et, c->tk, c->rr, S->tk1};
    LAUNCH(k_r2n_gather, nb(N), 256, 0, (const double *)S->stage, T, (int)c->m.xnumx, (int)c->m.ynumy, (int)c->m.znumz, O,
           c->p.viscmod, c->p.nubeg, c->p.nuend);
    if (S->tbc_n)
        LAUNCH(k_tk_bc, nb(S->tbc_n), 256, 0, c->tk, (const float *)S->tk1, S->tbc_n, (const int *)S->tbc_node,
               (const int *)S->tbc_p, (const double *)S->tbc_c, (const double *)S->tbc_k);
    I3G_CUDA(cudaGetLastError());
    I3G_CUDA(cudaEventRecord(e1, c->st));
    rc = check_err(c, "ronurecalc");
    float ms_ = 0;
    cudaEventElapsedTime(&ms_, e0, e1);
    c->st_.ms_r2n = ms_;
    c->stokes_ready = false;
    return rc;
}

int markers_heat_update(i3g_ctx *c, double timestep, const float *tk0, const float *tk1, const float *tk2)
{
    MarkerState *S = ms(c);
    if (!S->n) return 0;
    if (int rc = markers_wait(c)) return rc;
    const long N = c->nodenum;
    if (!S->sorted) {
        int rc = sort_markers(c);
        if (rc) return rc;
    }
    TkF T{tk0, tk1, c->tk, tk2, c->kt, c->ro, c->cp, (long)c->m.ynumy, (long)(c->m.xnumx * c->m.ynumy)};
    TileGeo TG{S->ntx, S->nty, S->ntz, S->ntiles};
    launch_heat_mark(c, S->a, (const int *)S->coff, T, TG, timestep, S->stage);
    if (c->p.heatdif != 0) {
        LAUNCH(k_heat_mark_gather, nb(N), 256, 0, (const double *)S->stage, TG, (int)c->m.xnumx, (int)c->m.ynumy,
               (int)c->m.znumz, S->acc, N);
        if (mexact(c))
            LAUNCH(k_heat_mark_anti<true>, std::min(nb(S->n), S->key_blocks), 256, grid_smem(c), S->a, (const int *)S->off,
                   S->ntiles, grid_of(c), T, (const double *)S->acc, N);
        else
            LAUNCH(k_heat_mark_anti<false>, std::min(nb(S->n), S->key_blocks), 256, grid_smem(c), S->a, (const int *)S->off,
                   S->ntiles, grid_of(c), T, (const double *)S->acc, N);
    }
    I3G_CUDA(cudaGetLastError());
    return 0;
}

// Kernel timing with an empty L2 before every repetition (cold_time).  Bytes per launch are the
// algorithmic bytes per unit: 4 marker -> node sums (k_r2n_cells): 25 B per marker (x, y, z,
// type, T, viscosity, rr) + 48 B per node (12 FP32 outputs); 5 RK4 advection (k_move): 45 B per
// marker + 13 nodal FP32 fields; 9 marker temperature update (k_heat_mark_cells): 42 B per marker.
int markers_time_kernel(i3g_ctx *c, int kind, int reps, double *ms_out, double *bytes)
{
    MarkerState *S = ms(c);
    const long n = S->n, N = c->nodenum;
    if (int rc = markers_wait(c)) return rc;
    TileGeo T{S->ntx, S->nty, S->ntz, S->ntiles};
    if (!S->sorted) { int rc = sort_markers(c); if (rc) return rc; }
    TkF TK{c->tk, c->tk, c->tk, c->tk, c->kt, c->ro, c->cp, (long)c->m.ynumy, (long)(c->m.xnumx * c->m.ynumy)};
    auto launch = [&]() -> int {
        if (kind == 4)
            launch_r2n(c, S->a, (const int *)S->coff, T, 1.0, S->stage);
        else if (kind == 9)
            launch_heat_mark(c, S->a, (const int *)S->coff, TK, T, 1e10, S->stage);
        else
            launch_move(c, std::min(nb(n), S->move_blocks), S->a, n, grid_of(c), nodes_of(c), phys_of(c), 0.0);
        return 0;
    };
    launch();   // warm-up
    int rc = cold_time(c, reps, launch, ms_out);
    if (rc) return rc;
    if (kind == 4) *bytes = (double)n * 25.0 + (double)N * 48.0;
    else if (kind == 9) *bytes = (double)n * 42.0;
    else *bytes = (double)n * 45.0 + (double)N * 13.0 * 4.0;
    I3G_CUDA(cudaGetLastError());
    return 0;
}

}  // namespace i3g
