// init.cu -- initial conditions on the GPU: markers and rock bodies (in3mg.c:131-797) and the
// initial-condition passes of in3mg.c:990-1031 (nodes from markers, hydrostatic pressure,
// nodes from markers again).
//
// The reference's generator is a separate serial program that writes the first .prn file;
// here the markers of an existing context are generated in place, one thread per marker, so a
// 257x129x257 model with 226 M markers is set up in milliseconds instead of being built and
// uploaded from the host.
#include <cmath>
#include <cstring>
#include <utility>
#include <vector>
#include "heat_markers.cuh"

namespace i3g {

// in3mg.c:1010-1021: pressure integrated down each vertical column from pinit in the cell row
// below the top, with the mean density of the four nodes around each vertical cell edge (FP32
// sum, as the reference's float arrays give); one thread per (x, z) column, the reference's
// sequential order of additions
__global__ void k_hydrostatic(double *pr, const float *ro, const double *gy, int nx, int ny, int nz, double pinit,
                              double gyk)
{
    const long col = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= (long)(nx - 1) * (nz - 1)) return;
    const long m1 = 1 + col % (nx - 1), m3 = 1 + col / (nx - 1);
    const long NY = ny, NXY = (long)nx * ny;
    long m4 = NXY * m3 + m1 * NY + 1;
    pr[m4] = pinit;
    for (int m2 = 2; m2 < ny; m2++) {
        m4++;
        const float rs = __fadd_rn(__fadd_rn(__fadd_rn(ro[m4 - 1], ro[m4 - NY - 1]), ro[m4 - NXY - 1]), ro[m4 - NXY - NY - 1]);
        pr[m4] = pr[m4 - 1] + (gy[m2] - gy[m2 - 2]) / 2.0 * gyk * (double)rs / 4.0;
    }
}

}  // namespace i3g

using namespace i3g;

namespace {

// Solve the 4 x 4 system A s = r by Gaussian elimination with partial pivoting.
void solve4(double A[4][4], double r[4], double s[4])
{
    for (int col = 0; col < 4; col++) {
        int piv = col;
        for (int i = col + 1; i < 4; i++)
            if (std::fabs(A[i][col]) > std::fabs(A[piv][col])) piv = i;
        if (piv != col) {
            for (int j = 0; j < 4; j++) std::swap(A[col][j], A[piv][j]);
            std::swap(r[col], r[piv]);
        }
        for (int i = col + 1; i < 4; i++) {
            const double f = A[col][col] != 0 ? A[i][col] / A[col][col] : 0.0;
            for (int j = col; j < 4; j++) A[i][j] -= f * A[col][j];
            r[i] -= f * r[col];
        }
    }
    for (int i = 3; i >= 0; i--) {
        double v = r[i];
        for (int j = i + 1; j < 4; j++) v -= A[i][j] * s[j];
        s[i] = A[i][i] != 0 ? v / A[i][i] : 0.0;
    }
}

// Face w = a0 + a1 u + a2 v + a3 u v of a box body through four of its corners (in3mg.c:589-
// 699): the left/right faces give x(y, z), up/down y(x, z), front/back z(y, x).
void face(const double *w, const double *u, const double *v, const int *corner, double k[4])
{
    double A[4][4], r[4];
    for (int i = 0; i < 4; i++) {
        const int n = corner[i];
        A[i][0] = 1.0; A[i][1] = u[n]; A[i][2] = v[n]; A[i][3] = u[n] * v[n];
        r[i] = w[n];
    }
    solve4(A, r, k);
}

}  // namespace

extern "C" int i3g_init_markers(i3g_ctx *c, const i3g_init *s)
{
    if (!c || !s) return I3G_E_ARG;
    const i3g_model &m = c->m;
    const long mx = m.mnumx, my = m.mnumy, mz = m.mnumz;
    if (mx < 1 || my < 1 || mz < 1 || (m.xnumx - 1) * (m.ynumy - 1) * (m.znumz - 1) * mx * my * mz != c->marknum)
        return set_error(c, I3G_E_ARG, "marker count %ld is not (nx-1)(ny-1)(nz-1) x markers per cell %ldx%ldx%ld", c->marknum, mx,
                         my, mz);
    if (s->nbodies < 0 || s->nbodies > I3G_INIT_MAX_BODIES || (s->nbodies && !s->bodies))
        return set_error(c, I3G_E_ARG, "bad body list (%d bodies, at most %d)", s->nbodies, I3G_INIT_MAX_BODIES);
    if (s->nonstab < 0) return set_error(c, I3G_E_ARG, "nonstab %d < 0", s->nonstab);
    auto rock_ok = [&](int t) { return t >= 0 && t < m.rocknum && t < 50; };
    if (!rock_ok(s->background)) return set_error(c, I3G_E_UNSUPPORTED, "background rock type %d (rock types >= 50 or beyond rocknum)", s->background);
    std::vector<BodyDev> hb(s->nbodies > 0 ? s->nbodies : 1);
    // corners: bit 0 down (larger y), bit 1 right (larger x), bit 2 back (larger z)  (in3mg.c:571-576)
    static const int L[4] = {0, 1, 4, 5}, R[4] = {2, 3, 6, 7}, U[4] = {0, 2, 4, 6}, D[4] = {1, 3, 5, 7},
                     F[4] = {0, 1, 2, 3}, B[4] = {4, 5, 6, 7};
    for (int b = 0; b < s->nbodies; b++) {
        const i3g_body &q = s->bodies[b];
        BodyDev &d = hb[b];
        memset(&d, 0, sizeof d);
        if (!rock_ok(q.rock)) return set_error(c, I3G_E_UNSUPPORTED, "body %d: rock type %d (types >= 50 or beyond rocknum)", b, q.rock);
        if (q.shape < 0 || q.shape > 2) return set_error(c, I3G_E_ARG, "body %d: shape %d", b, q.shape);
        d.rock = q.rock;
        d.shape = q.shape;
        d.ex = (float)q.ex;
        d.e = (float)q.e;
        if (q.shape == 0) {
            face(q.x, q.y, q.z, L, d.k[0]); face(q.x, q.y, q.z, R, d.k[1]);
            face(q.y, q.x, q.z, U, d.k[2]); face(q.y, q.x, q.z, D, d.k[3]);
            face(q.z, q.y, q.x, F, d.k[4]); face(q.z, q.y, q.x, B, d.k[5]);
        } else {
            // ellipsoid / cylinder (in3mg.c:740-790): centre = point 0, axis scales = point 7,
            // radius range [x of point 2, x of point 5]
            d.c[0] = q.x[0]; d.c[1] = q.y[0]; d.c[2] = q.z[0];
            d.s[0] = q.x[7]; d.s[1] = q.y[7]; d.s[2] = q.z[7];
            d.r0 = q.x[2]; d.r1 = q.x[5];
            if (!(d.s[0] != 0 && d.s[1] != 0 && d.s[2] != 0)) return set_error(c, I3G_E_ARG, "body %d: zero axis scale", b);
        }
    }
    BodyDev *dbodies = nullptr;
    if (s->nbodies) {
        I3G_CUDA(cudaMalloc((void **)&dbodies, sizeof(BodyDev) * s->nbodies));
        cudaError_t e = cudaMemcpyAsync(dbodies, hb.data(), sizeof(BodyDev) * s->nbodies, cudaMemcpyHostToDevice, c->st);
        if (e != cudaSuccess) { cudaFree(dbodies); return cuda_fail(c, e, "cudaMemcpyAsync", __FILE__, __LINE__); }
    }
    InitDev d;
    memset(&d, 0, sizeof d);
    d.mx = (int)mx; d.my = (int)my; d.mz = (int)mz;
    d.st[0] = m.xsize / (double)(m.xnumx - 1);
    d.st[1] = m.ysize / (double)(m.ynumy - 1);
    d.st[2] = m.zsize / (double)(m.znumz - 1);
    // in3mg.c:87-89: jitter amplitude = fraction x marker spacing
    d.jit[0] = (float)(s->xnonstab * m.xsize / (double)(m.xnumx - 1) / (double)mx);
    d.jit[1] = (float)(s->ynonstab * m.ysize / (double)(m.ynumy - 1) / (double)my);
    d.jit[2] = (float)(s->znonstab * m.zsize / (double)(m.znumz - 1) / (double)mz);
    d.nonstab = s->nonstab;
    d.seed = s->seed;
    d.background = s->background;
    d.ttop = s->t_top;
    d.tbot = s->t_bottom;
    d.nbodies = s->nbodies;
    d.bodies = dbodies;
    int rc = markers_init(c, d);
    cudaError_t e = cudaStreamSynchronize(c->st);
    cudaFree(dbodies);
    if (rc) return rc;
    if (e != cudaSuccess) return cuda_fail(c, e, "i3g_init_markers", __FILE__, __LINE__);
    return 0;
}

extern "C" int i3g_prepare(i3g_ctx *c)
{
    if (!c) return I3G_E_ARG;
    int rc = markers_to_nodes(c, 0.0);
    if (rc) return rc;
    const int nx = (int)c->m.xnumx, ny = (int)c->m.ynumy, nz = (int)c->m.znumz;
    if (c->m.gykoef > 0) {
        const long cols = (long)(nx - 1) * (nz - 1);
        k_hydrostatic<<<(unsigned)((cols + 127) / 128), 128, 0, c->st>>>(c->pr, c->ro, c->gy0, nx, ny, nz, c->m.pinit, c->m.gykoef);
        c->launches++;
        I3G_CUDA(cudaGetLastError());
    }
    rc = markers_to_nodes(c, 0.0);
    if (rc) return rc;
    I3G_CUDA(cudaStreamSynchronize(c->st));
    c->nhist = 0;
    return 0;
}
