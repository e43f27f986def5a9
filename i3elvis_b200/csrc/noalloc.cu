// noalloc.cu -- the Stokes stopping test without any device allocation.
//
// Every other entry point works on a context whose device buffers i3g_create() allocates.
// Some host codes cannot allow that: codes that hand all device memory to their own pool
// allocator at start-up and forbid allocations afterwards, and codes that keep work queued on
// their streams, where a cudaMalloc/cudaFree may synchronise the device in the middle of it.
// They keep the Stokes solution, right-hand side and residual in their own device buffers and
// only need the library's relative-residual test on them.
//
// i3g_stokes_relres_noalloc() computes the same two numbers as i3g_stokes_relres() from
// caller-owned device arrays.  Its only scratch is the file-scope array below (one per GPU
// that loads the library, held until the process exits): one partial sum per quantity for
// every x-z grid column, which bounds the grid to I3G_NOALLOC_MAX_COLUMNS columns (nx*nz).
//
// The first call on a device looks up that device's address of the array with
// cudaGetSymbolAddress (with the device current), once; make that first call before any
// stream capture on the device.  All calls share the array: two calls whose kernels overlap
// on the GPU (different streams, no ordering between them) race on it.  Every call writes all
// the partial sums it reads, so nothing has to be cleared between calls.
#include <cmath>
#include <cstdarg>
#include <mutex>
#include "i3g_internal.cuh"

namespace {

constexpr int kQ = 6;              // sum r_mom^2, sum f_mom^2, sum r_cont^2, sum v^2, #cont rows, #vel rows
constexpr int kColWarps = 8;       // columns per 256-thread block, one warp each
constexpr int kMaxDevices = 64;

// partial sums [column][kQ]
static __device__ __align__(256) double g_relres_cols[(long)I3G_NOALLOC_MAX_COLUMNS * kQ];

__device__ __forceinline__ bool row_on_grid(int v, int i, int j, int k, int nx, int ny, int nz)
{
    switch (v) {   // rows of the staggered system (move3mg.c:1638-1667)
    case 0: return i > 0 && j > 0 && k > 0;
    case 1: return j < ny - 1 && k < nz - 1;
    case 2: return i < nx - 1 && k < nz - 1;
    default: return i < nx - 1 && j < ny - 1;
    }
}

__device__ __forceinline__ double warp_allsum(double v)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

struct Arrays {
    const double *r0, *r1, *r2, *r3;
    const double *f1, *f2, *f3;
    const double *u1, *u2, *u3;
    const uint8_t *bc;
};

// One warp per x-z column: lanes walk y (unit stride), then lane q stores quantity q.
__global__ void __launch_bounds__(32 * kColWarps) k_relres_cols(Arrays a, int nx, int ny, int nz, double *part)
{
    const long col = (long)blockIdx.x * kColWarps + (threadIdx.x >> 5);
    const int ln = threadIdx.x & 31;
    if (col >= (long)nx * nz) return;
    const int i = (int)(col % nx), k = (int)(col / nx);
    const long base = ((long)k * nx + i) * ny;
    double q[kQ] = {0, 0, 0, 0, 0, 0};
    for (int j = ln; j < ny; j += 32) {
        const long n = base + j;
        const uint8_t b = a.bc[n];
        if (row_on_grid(0, i, j, k, nx, ny, nz) && !(b & 1)) { q[2] += a.r0[n] * a.r0[n]; q[4] += 1.0; }
        if (row_on_grid(1, i, j, k, nx, ny, nz)) {
            q[3] += a.u1[n] * a.u1[n]; q[5] += 1.0;
            if (!(b & 2)) { q[0] += a.r1[n] * a.r1[n]; q[1] += a.f1[n] * a.f1[n]; }
        }
        if (row_on_grid(2, i, j, k, nx, ny, nz)) {
            q[3] += a.u2[n] * a.u2[n]; q[5] += 1.0;
            if (!(b & 4)) { q[0] += a.r2[n] * a.r2[n]; q[1] += a.f2[n] * a.f2[n]; }
        }
        if (row_on_grid(3, i, j, k, nx, ny, nz)) {
            q[3] += a.u3[n] * a.u3[n]; q[5] += 1.0;
            if (!(b & 8)) { q[0] += a.r3[n] * a.r3[n]; q[1] += a.f3[n] * a.f3[n]; }
        }
    }
    double mine = 0;
    for (int t = 0; t < kQ; t++) {
        const double s = warp_allsum(q[t]);
        if (ln == t) mine = s;
    }
    if (ln < kQ) part[col * kQ + ln] = mine;
}

// One warp per quantity sums the columns in a fixed order; thread 0 forms the two ratios
// exactly as i3g_stokes_relres() does on the host.
__global__ void __launch_bounds__(32 * kQ) k_relres_cols_final(const double *part, long ncol, double h, double *out)
{
    __shared__ double s[kQ];
    const int t = threadIdx.x >> 5, ln = threadIdx.x & 31;
    double v = 0;
    for (long c = ln; c < ncol; c += 32) v += part[c * kQ + t];
    v = warp_allsum(v);
    if (ln == 0) s[t] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        const double ncont = s[4], nvel = s[5];
        out[0] = s[1] > 0 ? sqrt(s[0] / s[1]) : sqrt(s[0]);
        out[1] = (ncont > 0 && s[3] > 0) ? sqrt(s[2] / ncont) * h / sqrt(s[3] / nvel) : sqrt(s[2]);
    }
}

std::mutex g_mu;
double *g_dev_addr[kMaxDevices] = {};   // device address of g_relres_cols, per device

int fail(int code, const char *fmt, ...)
{
    char msg[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(msg, sizeof msg, fmt, ap);
    va_end(ap);
    return set_global_error(code, "i3g_stokes_relres_noalloc: %s", msg);
}

// Address of the scratch array on the current device (looked up on the first call per device).
int scratch_address(double **out)
{
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(I3G_E_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return fail(I3G_E_ARG, "device %d beyond the %d supported", dev, kMaxDevices);
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_dev_addr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_relres_cols);
        if (e != cudaSuccess) return fail(I3G_E_CUDA, "cudaGetSymbolAddress on device %d: %s", dev, cudaGetErrorString(e));
        g_dev_addr[dev] = (double *)p;
    }
    *out = g_dev_addr[dev];
    return 0;
}

}  // namespace

extern "C" int i3g_stokes_relres_noalloc(int nx, int ny, int nz, double h, const uint8_t *bc,
                                         const double *const res[4], const double *const rhs[4],
                                         const double *const sol[4], double *out, void *stream)
{
    if (nx < 2 || ny < 2 || nz < 2) return fail(I3G_E_ARG, "grid %d x %d x %d has an axis with fewer than 2 nodes", nx, ny, nz);
    const long ncol = (long)nx * nz;
    if (ncol > I3G_NOALLOC_MAX_COLUMNS)
        return fail(I3G_E_ARG, "grid has nx*nz = %ld x-z columns; the static scratch holds at most %d", ncol,
                    I3G_NOALLOC_MAX_COLUMNS);
    if (!bc || !res || !rhs || !sol || !out) return fail(I3G_E_ARG, "null pointer argument");
    for (int v = 0; v < 4; v++)
        if (!res[v] || (v > 0 && (!rhs[v] || !sol[v]))) return fail(I3G_E_ARG, "null device array for component %d", v);
    double *part = nullptr;
    int rc = scratch_address(&part);
    if (rc) return rc;
    Arrays a{res[0], res[1], res[2], res[3], rhs[1], rhs[2], rhs[3], sol[1], sol[2], sol[3], bc};
    cudaStream_t st = (cudaStream_t)stream;
    const unsigned nb = (unsigned)((ncol + kColWarps - 1) / kColWarps);
    k_relres_cols<<<nb, 32 * kColWarps, 0, st>>>(a, nx, ny, nz, part);
    k_relres_cols_final<<<1, 32 * kQ, 0, st>>>(part, ncol, h, out);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(I3G_E_CUDA, "kernel launch: %s", cudaGetErrorString(e));
    return 0;
}
