// unet.cu -- learned warm start for the Stokes solve: a 3-D U-Net on the level-0 node grid.
//
// The reference has no learned component; its Stokes solve starts from the previous step's
// v, P (move3mg.c:1969-2019).  This network maps (log10 viscosity, density, previous velocity)
// on the node grid to a correction of that start, dv and dP, and i3g_stokes() keeps the
// corrected start only when its relative residual is below the default start's.  The solver
// still iterates to the same tolerance, so the network decides the cycle count, never the answer.
//
// Network (4 levels, 16/32/64/128 channels, 15 convolutions of 3x3x3):
//   enc0: x0 -> e0a -> e0             (16 ch, level 0)     R: e0 -> d1
//   enc1: d1 -> e1a -> e1             (32 ch, level 1)     R: e1 -> d2
//   enc2: d2 -> e2a -> e2             (64 ch, level 2)     R: e2 -> d3
//   bott: d3 -> b3a -> b3             (128 ch, level 3)    P: b3 -> u2
//   dec2: relu(conv(u2) + e2) -> g2a -> g2  (64 ch)        P: g2 -> u1
//   dec1: relu(conv(u1) + e1) -> g1a -> g1  (32 ch)        P: g1 -> u0
//   dec0: relu(conv(u0) + e0) -> g0a -> g0  (16 ch)
//   out : y = conv(g0) (linear, channels 0..3 = dP, dVx, dVy, dVz scaled)
// Level l has (n-1)/2^l + 1 nodes per axis (vertex-centred: every grid axis needs n-1
// divisible by 8).  R is full weighting (1/4,1/2,1/4 per axis), P trilinear interpolation;
// P^T = 8 R and R^T = P / 8, so the backward pass reuses the two kernels.
//
// Layout: every activation is channels-last BF16 [rows][C] over the grid padded by one zero
// node on each side (Z = nz+2, X = nx+2, Y = ny+2, row = (z*X + x)*Y + y, y fastest like the
// solver's nodes).  A 3x3x3 tap is then a constant row offset, and a convolution is an
// implicit GEMM: D[128 rows][Cout] = sum over 27 taps and Cin of A_tap[128 rows][Cin] *
// W_tap[Cin][Cout], with A_tap a contiguous block of 128 rows shifted by the tap's offset.
//
// Convolution kernels (forward and input gradient; tcgen05.mma kind::f16, BF16 x BF16 -> FP32 in
// TMEM, M = 128 rows, N = Cout, K = 16; the epilogue reads TMEM with tcgen05.ld, adds bias and
// the skip tensor, applies ReLU or the ReLU mask of the backward pass and stores BF16, or FP32
// for tests):
//   k_conv_tma   16/32 channels in and out (the fine levels, most of the time): persistent CTAs,
//                TMA boxes of a 4-D tensor map in the swizzled K-major operand layout, a ring of
//                box stages, one MMA thread, two TMEM accumulators, four epilogue warps;
//   k_conv_brick the same channel counts when no tensor-map encoder is available: producer warps
//                gather taps from a cp.async brick into no-swizzle operand stages;
//   k_conv_tc    wider layers: one CTA per 128-row tile, each tap's shifted block staged with
//                cp.async (zero fill outside the array) in a 4-deep ring.
// Weight gradients: k_wgrad_tc on the tensor cores for 16/32 channels (MN-major operands, a
// partial sum per CTA, k_wgrad_reduce), FP32 CUDA-core reductions (k_wgrad) for the rest.
// All waits on mbarriers are bounded (2 s); a timeout sets an error flag read by the host.
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>
#include <cuda.h>
#include <cuda_bf16.h>
#include "i3g_internal.cuh"

using bf16 = __nv_bfloat16;

namespace i3g {
namespace unet {

constexpr int kLevels = 4;
constexpr int kLayers = 15;
constexpr int kTileM = 128;
constexpr int kStages = 4;
constexpr int kInCh = 5;      // log10 eta, rho, vx, vy, vz
constexpr int kOutCh = 4;     // dP, dVx, dVy, dVz

// tensors of the forward pass
enum { X0, E0A, E0, D1, E1A, E1, D2, E2A, E2, D3, B3A, B3, U2, G2A, G2, U1, G1A, G1, U0, G0A, G0, Y, kTensors };
struct TensorDef { int lev, ch; };
static const TensorDef kT[kTensors] = {
    {0, 16}, {0, 16}, {0, 16}, {1, 16}, {1, 32}, {1, 32}, {2, 32}, {2, 64}, {2, 64}, {3, 64}, {3, 128}, {3, 128},
    {2, 128}, {2, 64}, {2, 64}, {1, 64}, {1, 32}, {1, 32}, {0, 32}, {0, 16}, {0, 16}, {0, 16}};
struct LayerDef { int in, out, add, relu; };
static const LayerDef kL[kLayers] = {
    {X0, E0A, -1, 1}, {E0A, E0, -1, 1}, {D1, E1A, -1, 1}, {E1A, E1, -1, 1}, {D2, E2A, -1, 1}, {E2A, E2, -1, 1},
    {D3, B3A, -1, 1}, {B3A, B3, -1, 1}, {U2, G2A, E2, 1}, {G2A, G2, -1, 1}, {U1, G1A, E1, 1}, {G1A, G1, -1, 1},
    {U0, G0A, E0, 1}, {G0A, G0, -1, 1}, {G0, Y, -1, 0}};

struct Dims {
    int nz = 0, nx = 0, ny = 0;   // nodes
    int Z = 0, X = 0, Y = 0;      // padded
    long np = 0, n = 0;           // padded rows, nodes
};

// ---------------------------------------------------------------------------------------
// device helpers
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src, int nbytes)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(nbytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ uint64_t global_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ bool mbar_try(uint32_t a, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.b32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok)
                 : "r"(a), "r"(parity)
                 : "memory");
    return ok != 0;
}
// Bounded wait: false after 2 s without the phase completing.
__device__ bool mbar_wait(uint32_t a, uint32_t parity)
{
    if (mbar_try(a, parity)) return true;
    const uint64_t t0 = global_ns();
    for (;;) {
        if (mbar_try(a, parity)) return true;
        if (global_ns() - t0 > 2000000000ull) return false;
    }
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Shared-memory matrix descriptor, no swizzle, K-major: core matrices of 8 rows x 16 B;
// lbo = byte distance between the two K halves of a K=16 step, sbo = between 8-row groups.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ void tc_mma(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc)
{
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\ttcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                 ::"r"(d), "l"(a), "l"(b), "r"(idesc), "r"(acc)
                 : "memory");
}

__device__ __forceinline__ void tc_ld16(uint32_t taddr, float (&v)[16])
{
    uint32_t r[16];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                 : "r"(taddr)
                 : "memory");
    // the registers are tied to the wait so that no use is scheduled before it
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                   "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]), "+r"(r[15])
                 :
                 : "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void unpack8(const uint4 &u, float (&f)[8])
{
    const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&u);
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const float2 t = __bfloat1622float2(h[i]);
        f[2 * i] = t.x;
        f[2 * i + 1] = t.y;
    }
}
__device__ __forceinline__ uint4 pack8(const float (&f)[8])
{
    uint4 u;
    __nv_bfloat162 *h = reinterpret_cast<__nv_bfloat162 *>(&u);
#pragma unroll
    for (int i = 0; i < 4; i++) h[i] = __floats2bfloat162_rn(f[2 * i], f[2 * i + 1]);
    return u;
}

__device__ __forceinline__ bool interior_row(long p, const Dims &d)
{
    const long xy = (long)d.X * d.Y;
    const int z = (int)(p / xy);
    const long rem = p - z * xy;
    const int x = (int)(rem / d.Y), y = (int)(rem - (long)x * d.Y);
    return z >= 1 && z <= d.nz && x >= 1 && x <= d.nx && y >= 1 && y <= d.ny;
}

// ---------------------------------------------------------------------------------------
// tcgen05 implicit-GEMM 3x3x3 convolution
// ---------------------------------------------------------------------------------------
struct ConvArgs {
    const bf16 *in;       // [np][CIN]
    const bf16 *w;        // [27][COUT][CIN]
    const float *bias;    // [COUT] or null
    const bf16 *add;      // [np][COUT] or null: added before the activation
    const bf16 *mask;     // [np][COUT] or null: result *= (mask > 0)
    bf16 *out;            // [np][COUT] (interior rows written) or null
    float *out32;         // [np][COUT] FP32 output or null
    Dims d;
    int relu;
    int off[27];          // tap row offsets, tap = (dz+1)*9 + (dx+1)*3 + (dy+1)
    int *err;
};

template <int CIN, int COUT>
struct ConvShape {
    static constexpr int KC = CIN < 64 ? CIN : 64;             // channels per stage
    static constexpr int NKC = CIN / KC;
    static constexpr int NSTEP = 27 * NKC;
    static constexpr int ABYTES = kTileM * KC * 2;
    static constexpr int BBYTES = COUT * KC * 2;
    static constexpr int SBYTES = ABYTES + BBYTES;
    static constexpr uint32_t NCOL = COUT < 32 ? 32 : COUT;     // TMEM columns (power of 2 >= 32)
    // kind::f16 instruction descriptor: D FP32, A and B BF16, both K-major, N = COUT, M = 128
    static constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(COUT >> 3) << 17) |
                                      ((uint32_t)(kTileM >> 4) << 24);
    // dynamic shared memory: the operand ring, raised so that the CTAs resident on one SM
    // never ask for more than the 512 TMEM columns (no CTA ever waits in tcgen05.alloc)
    // (plus 1 KiB: the ring starts at the next 1024-byte boundary of the dynamic buffer)
    static constexpr int SMEM_RING = kStages * SBYTES + 1024;
    static constexpr int SMEM_TMEM = (int)NCOL * 460;
    static constexpr int SMEM = SMEM_RING > SMEM_TMEM ? SMEM_RING : SMEM_TMEM;
    static_assert(CIN % 16 == 0 && COUT % 16 == 0 && COUT <= 256, "channel counts");
};

template <int CIN, int COUT>
__global__ void __launch_bounds__(128) k_conv_tc(ConvArgs a)
{
    using S = ConvShape<CIN, COUT>;
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ __align__(8) uint64_t mbar[kStages];
    __shared__ uint32_t s_tmem;
    __shared__ int s_off[27];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const long row0 = (long)blockIdx.x * kTileM;
    // The dynamic buffer follows this kernel's static shared variables and is only 16-byte
    // aligned; the tensor core reads a descriptor's matrix from a coarser-aligned start (an
    // operand at 16 mod 128 was read 16 bytes early), so the ring starts at a 1024-byte boundary.
    const uint32_t sbase = (smem_u32(smem) + 1023u) & ~1023u;
    if (tid < 27) s_off[tid] = a.off[tid];
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"(S::NCOL)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int s = 0; s < kStages; s++)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[s])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;

    auto load_stage = [&](int step) {
        const int tap = step / S::NKC, kc = step - tap * S::NKC;
        const uint32_t sA = sbase + (uint32_t)((step % kStages) * S::SBYTES);
        const uint32_t sB = sA + S::ABYTES;
        const long off = s_off[tap];
        // chunk j (channels 8j..8j+7) of row r at j*(rows*16) + r*16: 8-row core matrices
        // 128 bytes apart along M, the two K halves of a K=16 step rows*16 bytes apart
#pragma unroll
        for (int q = tid; q < kTileM * (S::KC / 8); q += 128) {
            const int r = q / (S::KC / 8), j = q - r * (S::KC / 8);
            const long src = row0 + r + off;
            const bool ok = src >= 0 && src < a.d.np;
            const bf16 *g = a.in + (ok ? src : 0) * CIN + kc * S::KC + j * 8;
            cp_async16(sA + (uint32_t)(j * (kTileM * 16) + r * 16), g, ok ? 16 : 0);
        }
#pragma unroll
        for (int q = tid; q < COUT * (S::KC / 8); q += 128) {
            const int r = q / (S::KC / 8), j = q - r * (S::KC / 8);
            const bf16 *g = a.w + ((long)tap * COUT + r) * CIN + kc * S::KC + j * 8;
            cp_async16(sB + (uint32_t)(j * (COUT * 16) + r * 16), g, 16);
        }
    };

    // prologue: stages 0 .. kStages-2 in flight
#pragma unroll
    for (int s = 0; s < kStages - 1; s++) {
        if (s < S::NSTEP) load_stage(s);
        cp_async_commit();
    }
    bool failed = false;
    int issued = 0;   // steps whose MMAs were issued
    for (int i = 0; i < S::NSTEP; i++) {
        const int j = i + kStages - 1;
        int fail = 0;
        if (j < S::NSTEP) {
            // slot j % kStages was last read by the MMAs of step i-1
            if (i >= 1 && !mbar_wait(smem_u32(&mbar[(i - 1) % kStages]), ((i - 1) / kStages) & 1)) fail = 1;
            if (!fail) load_stage(j);
        }
        cp_async_commit();
        cp_async_wait<kStages - 1>();   // the group of step i has landed
        fence_proxy_async();            // make it visible to the tensor core's (async) proxy
        if (__syncthreads_or(fail)) {
            failed = true;
            break;
        }
        if (tid == 0) {
            tc_fence_after();
            const uint32_t sA = sbase + (uint32_t)((i % kStages) * S::SBYTES);
            const uint32_t sB = sA + S::ABYTES;
#pragma unroll
            for (int k = 0; k < S::KC / 16; k++) {
                const uint64_t da = smem_desc(sA + (uint32_t)(2 * k * kTileM * 16), kTileM * 16, 128);
                const uint64_t db = smem_desc(sB + (uint32_t)(2 * k * COUT * 16), COUT * 16, 128);
                tc_mma(tmem, da, db, S::IDESC, (i > 0 || k > 0) ? 1u : 0u);
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(&mbar[i % kStages]))
                         : "memory");
        }
        issued = i + 1;
    }
    cp_async_wait<0>();
    // the commit of the last issued step arrives once every earlier MMA of this CTA completed
    int fail = 0;
    if (issued > 0 && !mbar_wait(smem_u32(&mbar[(issued - 1) % kStages]), ((issued - 1) / kStages) & 1)) fail = 1;
    failed = __syncthreads_or(fail || failed) != 0;
    if (failed) {
        // No epilogue.  MMAs committed before the timeout may still write TMEM and read the
        // ring: one more bounded wait on the last commit before the columns are released.  If
        // that also times out the device state is suspect; the host reports the error as fatal
        // for the handle (check_err).
        if (tid == 0) {
            atomicExch(a.err, 1);
            if (issued > 0) mbar_wait(smem_u32(&mbar[(issued - 1) % kStages]), ((issued - 1) / kStages) & 1);
        }
        __syncthreads();
    } else {
        tc_fence_after();
        const long p = row0 + warp * 32 + lane;
        const bool valid = p < a.d.np && interior_row(p, a.d);
#pragma unroll
        for (int c0 = 0; c0 < COUT; c0 += 16) {
            float v[16];
            tc_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);   // whole warp
            if (valid) {
                if (a.bias) {
#pragma unroll
                    for (int q = 0; q < 16; q++) v[q] += a.bias[c0 + q];
                }
                if (a.add) {
#pragma unroll
                    for (int h = 0; h < 2; h++) {
                        float f[8];
                        unpack8(*reinterpret_cast<const uint4 *>(a.add + p * COUT + c0 + 8 * h), f);
#pragma unroll
                        for (int q = 0; q < 8; q++) v[8 * h + q] += f[q];
                    }
                }
                if (a.relu) {
#pragma unroll
                    for (int q = 0; q < 16; q++) v[q] = fmaxf(v[q], 0.0f);
                }
                if (a.mask) {
#pragma unroll
                    for (int h = 0; h < 2; h++) {
                        float f[8];
                        unpack8(*reinterpret_cast<const uint4 *>(a.mask + p * COUT + c0 + 8 * h), f);
#pragma unroll
                        for (int q = 0; q < 8; q++) v[8 * h + q] = f[q] > 0.0f ? v[8 * h + q] : 0.0f;
                    }
                }
                if (a.out) {
#pragma unroll
                    for (int h = 0; h < 2; h++) {
                        float f[8];
#pragma unroll
                        for (int q = 0; q < 8; q++) f[q] = v[8 * h + q];
                        *reinterpret_cast<uint4 *>(a.out + p * COUT + c0 + 8 * h) = pack8(f);
                    }
                }
                if (a.out32) {
#pragma unroll
                    for (int q = 0; q < 16; q += 4)
                        *reinterpret_cast<float4 *>(a.out32 + p * COUT + c0 + q) = make_float4(v[q], v[q + 1], v[q + 2], v[q + 3]);
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(S::NCOL) : "memory");
}

// ---------------------------------------------------------------------------------------
// brick-staged tcgen05 convolution (CIN, COUT in {16, 32}: the layers of levels 0 and 1)
// ---------------------------------------------------------------------------------------
// k_conv_tc fetches every tap's 128-row operand from L2 (27 shifted copies of the input per
// output tile) and waits on each fetch.  Here a persistent CTA keeps all 27 taps' weights in
// shared memory and walks over output tiles of 2 x 8 x 8 nodes (z, x, y): it loads the tile's
// input brick with its one-node halo (4 x 10 x 10 rows) once, then for every tap gathers the
// shifted 128-row operands of three taps at a time from the brick into one of NST aligned
// operand stages (the canonical no-swizzle K-major layout).  The work is split by warp: four
// producer warps gather the stages and arrive on the stage's "full" mbarrier (no CTA-wide barrier
// per stage); a fifth warp, one thread, waits for "full", issues the MMAs (M = 128, N = COUT,
// K = 16) into the CTA's TMEM accumulator and commits to the stage's "empty" mbarrier, which the
// producers wait for before they reuse the stage, and after a tile's last stage to "accf".  The
// producers load the next tile's brick and then run the epilogue of the tile (k_conv_tc's: bias,
// skip add, ReLU or the backward ReLU mask, BF16 or FP32 stores of the interior rows) once
// "accf" says its MMAs completed.
constexpr int kBz = 2, kBx = 8, kBy = 8;                    // output tile (z, x, y): 128 rows
constexpr int kHz = kBz + 2, kHx = kBx + 2, kHy = kBy + 2;   // input brick with halo
constexpr int kBrickRows = kHz * kHx * kHy;
constexpr int kTapsPerStage = 3;                            // the three dy taps of one (dz, dx)

template <int CIN, int COUT>
struct BrickShape {
    static constexpr int CH = CIN / 8;                         // 16-byte channel chunks per row
    static constexpr int ABYTES = kTileM * CIN * 2;            // one tap's A operand
    static constexpr int TAPB = COUT * CIN * 2;                // one tap's B operand
    static constexpr int WBYTES = 27 * TAPB;
    static constexpr int BRICK = kBrickRows * CIN * 2;
    static constexpr int NST = CIN == 16 ? 3 : 2;              // stages (of three tap operands) in flight
    // brick rows hold their 16-byte chunks XOR-swizzled: chunk j of row r sits in slot
    // j ^ ((r >> SWS) & (CH - 1)), so that the eight consecutive rows a quarter-warp gathers fall
    // in distinct banks (rows 4 apart (CIN 16) or 2 apart (CIN 32) would otherwise collide)
    static constexpr int SWS = CIN == 16 ? 2 : 1;
    static __device__ __forceinline__ int slot(int r, int j) { return r * CH + (j ^ ((r >> SWS) & (CH - 1))); }
    static constexpr int STB = kTapsPerStage * ABYTES;
    static constexpr int SMEM = 1024 + NST * STB + WBYTES + BRICK;
    static constexpr uint32_t NCOL = COUT < 32 ? 32 : COUT;
    static constexpr uint32_t IDESC = ConvShape<CIN, COUT>::IDESC;
    static_assert((CIN == 16 || CIN == 32) && (COUT == 16 || COUT == 32), "brick kernel channel counts");
    static_assert(TAPB % 512 == 0 && ABYTES % 1024 == 0, "operand alignment");
};

// producer warps of the brick kernels (warps 0-3) and the MMA warp (warp 4)
constexpr int kProducers = 128, kBrickThreads = kProducers + 32;

// OR of a flag over the producer warps; named barrier 1, so the MMA warp does not take part
__device__ __forceinline__ bool producers_or(bool v)
{
    uint32_t r;
    asm volatile("{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\tbar.red.or.pred q, 1, %2, p;\n\tselp.u32 %0, 1, 0, q;\n\t}"
                 : "=r"(r)
                 : "r"((uint32_t)v), "n"(kProducers)
                 : "memory");
    return r != 0;
}

template <int CIN, int COUT>
__global__ void __launch_bounds__(kBrickThreads) k_conv_brick(ConvArgs a, int ntx, int nty, int ntiles)
{
    using S = BrickShape<CIN, COUT>;
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ __align__(8) uint64_t full[S::NST], empty[S::NST], accf;
    __shared__ uint32_t s_tmem;
    __shared__ int s_abort;
    const int tid = threadIdx.x, warp = tid >> 5;
    // operand stages and weights at 1024-byte boundaries (tensor-core operand alignment)
    const uint32_t sbase = (smem_u32(smem) + 1023u) & ~1023u;
    const uint32_t sA0 = sbase, sW = sbase + S::NST * S::STB, sBrick = sW + S::WBYTES;
    uint8_t *const gbase = smem + (sbase - smem_u32(smem));
    const uint8_t *const brick = gbase + S::NST * S::STB + S::WBYTES;
    uint8_t *const abuf = gbase;
    const long XY = (long)a.d.X * a.d.Y;
    auto tile_origin = [&](int tile, int &z0, int &x0, int &y0) {
        const int ty = tile % nty, r2 = tile / nty, tx = r2 % ntx, tz = r2 / ntx;
        z0 = 1 + kBz * tz; x0 = 1 + kBx * tx; y0 = 1 + kBy * ty;
    };
    // input brick of a tile, loaded by the producers: padded rows (z0-1 .. z0+2, x0-1 .. x0+8,
    // y0-1 .. y0+8), zero outside the array
    auto load_brick = [&](int tile) {
        int z0, x0, y0;
        tile_origin(tile, z0, x0, y0);
        for (int q = tid; q < kBrickRows * S::CH; q += kProducers) {
            const int br = q / S::CH, j = q - br * S::CH;
            const int bz = br / (kHx * kHy), bxy = br - bz * (kHx * kHy), bx = bxy / kHy, by = bxy - bx * kHy;
            const int zz = z0 - 1 + bz, xx = x0 - 1 + bx, yy = y0 - 1 + by;
            const bool ok = zz < a.d.Z && xx < a.d.X && yy < a.d.Y;
            const long src = ok ? (long)zz * XY + (long)xx * a.d.Y + yy : 0;
            cp_async16(sBrick + (uint32_t)(S::slot(br, j) * 16), a.in + src * CIN + j * 8, ok ? 16 : 0);
        }
    };
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"(S::NCOL)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int s = 0; s < S::NST; s++) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&full[s])), "r"(kProducers) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&empty[s])) : "memory");
        }
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&accf)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_abort = 0;
    }
    if (tid < kProducers) {
        // all taps' weights, once per CTA: tap t, output channel n, chunk j at t*TAPB + j*(COUT*16) + n*16
        for (int q = tid; q < 27 * COUT * S::CH; q += kProducers) {
            const int t = q / (COUT * S::CH), rem = q - t * (COUT * S::CH);
            const int n = rem / S::CH, j = rem - n * S::CH;
            cp_async16(sW + (uint32_t)(t * S::TAPB + j * (COUT * 16) + n * 16), a.w + ((long)t * COUT + n) * CIN + j * 8, 16);
        }
        if ((int)blockIdx.x < ntiles) load_brick(blockIdx.x);
        cp_async_commit();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;
    volatile int *abort_flag = &s_abort;
    long issued = 0;   // MMA thread: stages committed
    if (warp == kProducers / 32) {
        // ---- MMA issuer: one thread ----
        if ((tid & 31) == 0) {
            long g = 0;
            bool mfail = false;
            for (int tile = blockIdx.x; tile < ntiles && !mfail; tile += gridDim.x) {
                for (int st = 0; st < 9; st++, g++) {
                    const int b = (int)(g % S::NST);
                    if (!mbar_wait(smem_u32(&full[b]), (uint32_t)((g / S::NST) & 1))) { mfail = true; break; }
                    tc_fence_after();
#pragma unroll
                    for (int dy = 0; dy < kTapsPerStage; dy++) {
                        const int tap = st * 3 + dy;
                        const uint32_t sA = sA0 + (uint32_t)(b * S::STB + dy * S::ABYTES), sB = sW + (uint32_t)(tap * S::TAPB);
#pragma unroll
                        for (int k = 0; k < CIN / 16; k++) {
                            const uint64_t da = smem_desc(sA + (uint32_t)(2 * k * kTileM * 16), kTileM * 16, 128);
                            const uint64_t db = smem_desc(sB + (uint32_t)(2 * k * COUT * 16), COUT * 16, 128);
                            tc_mma(tmem, da, db, S::IDESC, (tap > 0 || k > 0) ? 1u : 0u);
                        }
                    }
                    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                     smem_u32(&empty[b]))
                                 : "memory");
                    issued = g + 1;
                }
                if (mfail) break;
                // arrives once every MMA of this tile completed
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                 smem_u32(&accf))
                             : "memory");
            }
            // MMAs still in flight read the stages and write TMEM: wait for the last commit
            if (issued > 0) {
                const long gl = issued - 1;
                if (!mbar_wait(smem_u32(&empty[gl % S::NST]), (uint32_t)((gl / S::NST) & 1))) mfail = true;
            }
            if (mfail) *abort_flag = 1;
        }
    } else {
        // ---- producers (warps 0-3): gathers, next brick, epilogue ----
        // A failed (timed-out) wait only sets this thread's flag: every producer still arrives on
        // every stage and reaches every producer barrier, and all stop together where the flags
        // are combined (an unbounded named barrier must never miss a participant).
        const int oz = tid >> 6, ox = (tid >> 3) & 7, oy = tid & 7;   // output row r = tid of the tile
        long g = 0;
        int q = 0;
        bool fail = false;
        for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, q++) {
            int z0, x0, y0;
            tile_origin(tile, z0, x0, y0);
            cp_async_wait<0>();                  // this thread's part of the brick (and weights)
            if (producers_or(fail)) { fail = true; break; }   // and everyone's part
            for (int st = 0; st < 9; st++, g++) {
                const int b = (int)(g % S::NST);
                // the stage's buffer was last read by the MMAs of stage g - NST
                if (!fail && g >= S::NST && !mbar_wait(smem_u32(&empty[b]), (uint32_t)((g / S::NST - 1) & 1))) fail = true;
                if (!fail) {
                    const int dz = st / 3, dx = st % 3;
                    const int br0 = ((oz + dz) * kHx + (ox + dx)) * kHy + oy;
                    uint8_t *dst = abuf + b * S::STB + tid * 16;
#pragma unroll
                    for (int dy = 0; dy < kTapsPerStage; dy++)
#pragma unroll
                        for (int j = 0; j < S::CH; j++)
                            *reinterpret_cast<uint4 *>(dst + dy * S::ABYTES + j * (kTileM * 16)) =
                                *reinterpret_cast<const uint4 *>(brick + S::slot(br0 + dy, j) * 16);
                }
                fence_proxy_async();   // the gathered operands to the tensor core's (async) proxy
                asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&full[b])) : "memory");
            }
            // every producer's gathers of this tile are done: the next tile's brick loads while the
            // epilogue runs
            if (producers_or(fail)) { fail = true; break; }
            if (tile + (int)gridDim.x < ntiles) load_brick(tile + gridDim.x);
            cp_async_commit();
            if (!mbar_wait(smem_u32(&accf), (uint32_t)(q & 1))) fail = true;
            // the TMEM load below is warp-collective: the warp decides together
            if (__any_sync(0xffffffffu, fail)) { fail = true; continue; }
            tc_fence_after();
            const int zz = z0 + oz, xx = x0 + ox, yy = y0 + oy;
            const bool valid = zz <= a.d.nz && xx <= a.d.nx && yy <= a.d.ny;
            const long p = (long)zz * XY + (long)xx * a.d.Y + yy;
            float v[COUT];
#pragma unroll
            for (int c0 = 0; c0 < COUT; c0 += 16) {
                float t16[16];
                tc_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, t16);   // whole warp
#pragma unroll
                for (int e = 0; e < 16; e++) v[c0 + e] = t16[e];
            }
            // TMEM read: the next tile's first MMA overwrites the accumulator only after the
            // gathers that follow, ordered after these reads by this fence and the mbarrier
            tc_fence_before();
            if (valid) {
#pragma unroll
                for (int c0 = 0; c0 < COUT; c0 += 8) {
                    float f[8];
#pragma unroll
                    for (int e = 0; e < 8; e++) f[e] = v[c0 + e] + (a.bias ? a.bias[c0 + e] : 0.0f);
                    if (a.add) {
                        float h[8];
                        unpack8(*reinterpret_cast<const uint4 *>(a.add + p * COUT + c0), h);
#pragma unroll
                        for (int e = 0; e < 8; e++) f[e] += h[e];
                    }
                    if (a.relu) {
#pragma unroll
                        for (int e = 0; e < 8; e++) f[e] = fmaxf(f[e], 0.0f);
                    }
                    if (a.mask) {
                        float h[8];
                        unpack8(*reinterpret_cast<const uint4 *>(a.mask + p * COUT + c0), h);
#pragma unroll
                        for (int e = 0; e < 8; e++) f[e] = h[e] > 0.0f ? f[e] : 0.0f;
                    }
                    if (a.out) *reinterpret_cast<uint4 *>(a.out + p * COUT + c0) = pack8(f);
                    if (a.out32) {
                        *reinterpret_cast<float4 *>(a.out32 + p * COUT + c0) = make_float4(f[0], f[1], f[2], f[3]);
                        *reinterpret_cast<float4 *>(a.out32 + p * COUT + c0 + 4) = make_float4(f[4], f[5], f[6], f[7]);
                    }
                }
            }
        }
        cp_async_wait<0>();
        if (fail) *abort_flag = 1;
    }
    __syncthreads();
    if (tid == 0 && *abort_flag) atomicExch(a.err, 1);
    tc_fence_after();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(S::NCOL) : "memory");
}

// ---------------------------------------------------------------------------------------
// TMA-fed tcgen05 convolution (CIN, COUT in {16, 32})
// ---------------------------------------------------------------------------------------
// Output tiles of 1 x 16 x 8 nodes (z, x, y).  For each tile one thread issues TMA loads (a 4-D
// tensor map (channels, y, x, z) over the padded activation) of the input box z0-1..z0+1,
// x0-1..x0+16 and the 8 y rows y0-1+dy.., one box per dy in {0, 1, 2}, straight into the operand
// layout of the tensor core: a node's channels land as one row of CIN * 2 bytes (32 B with the
// 32-byte swizzle, 64 B with the 64-byte one), [z 3][x 18][y 8][row], so 8 consecutive y rows are
// one swizzle atom of the K-major layout, consecutive x are 8 rows apart and the operand of tap
// (dz, dx, dy) is the dy box at (dz * 18 + dx) atoms; K steps of 16 channels advance 32 bytes inside
// the row.  Every operand start stays on its atom, no copy through registers, and one TMA row per
// node and box (16-byte rows, one per channel chunk, were half as fast).  Boxes stream through a ring of NB slots with a
// "full" (TMA bytes) and an "empty" (MMA commit) mbarrier each.  A second thread issues, per box,
// the 9 x CIN/16 MMAs (M = 128, N = COUT, K = 16) of its taps into one of two TMEM accumulators
// and commits to the slot's "empty" mbarrier, and after a tile's third box to the accumulator's
// "full" one; four warps read the accumulator (tcgen05.ld), arrive on its "empty" mbarrier and run
// k_conv_tc's epilogue.  Loads, MMAs and epilogues of consecutive boxes and tiles overlap.  Every
// wait is bounded.
constexpr int kTz = 1, kTx = 16, kTy = 8;                   // output tile: 128 rows
constexpr int kQz = kTz + 2, kQx = kTx + 2, kQy = kTy;      // one dy box
constexpr int kBoxRows = kQz * kQx * kQy;                   // 432 nodes
constexpr int kTmaThreads = 192;                           // warps 0-3 epilogue, 4 loads, 5 MMAs

template <int CIN, int COUT>
struct TmaShape {
    static constexpr int CH = CIN / 8;
    static constexpr int ROWB = CIN * 2;                    // bytes of one node in a box
    static constexpr int TXB = kBoxRows * ROWB;             // bytes one box's load delivers
    static constexpr int BOXB = (TXB + 1023) / 1024 * 1024;  // one dy box's slot
    static constexpr int TAPB = COUT * CIN * 2;
    static constexpr int WBYTES = 27 * TAPB;
    // ring of box stages: the most that keeps two CTAs on an SM (228 KiB of shared memory, 1 KiB
    // reserved per CTA) if that is at least a tile's three boxes, else the most for one CTA
    static constexpr int NB2 = (233472 / 2 - 2048 - 1024 - WBYTES) / BOXB;
    static constexpr int NB1 = (232448 - 1024 - WBYTES) / BOXB;
    static constexpr int NB = NB2 >= 3 ? (NB2 < 8 ? NB2 : 8) : (NB1 < 8 ? NB1 : 8);
    static constexpr int SMEM = 1024 + NB * BOXB + WBYTES;
    static constexpr uint32_t NCOL = 2 * COUT < 32 ? 32 : 2 * COUT;
    static constexpr uint32_t IDESC = ConvShape<CIN, COUT>::IDESC;
    // layout type of the A descriptor (bits 61-63): 6 = 32-byte swizzle, 4 = 64-byte swizzle
    static constexpr uint64_t ALAYOUT = (CIN == 16 ? 6ull : 4ull) << 61;
    static_assert((CIN == 16 || CIN == 32) && (COUT == 16 || COUT == 32), "TMA convolution channel counts");
    static_assert(BOXB % 1024 == 0, "TMA destinations on their swizzle atoms");
    static_assert(NB >= 2 && SMEM <= 232448, "shared memory of the box ring");
};

__device__ __forceinline__ void tma_load_4d(uint32_t dst, const CUtensorMap *map, int c0, int c1, int c2, int c3, uint32_t mbar)
{
    asm volatile("cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];"
                 ::"r"(dst), "l"((uint64_t)map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(mbar)
                 : "memory");
}

template <int CIN, int COUT>
__global__ void __launch_bounds__(kTmaThreads) k_conv_tma(const __grid_constant__ CUtensorMap map, ConvArgs a, int ntx, int nty,
                                                         int ntiles)
{
    using S = TmaShape<CIN, COUT>;
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ __align__(8) uint64_t bfull[S::NB], bempty[S::NB], afull[2], aempty[2];
    __shared__ uint32_t s_tmem;
    __shared__ int s_abort;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t sbase = (smem_u32(smem) + 1023u) & ~1023u;
    const uint32_t sT = sbase, sW = sbase + S::NB * S::BOXB;
    const long XY = (long)a.d.X * a.d.Y;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"(S::NCOL)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int s = 0; s < S::NB; s++) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bfull[s])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bempty[s])) : "memory");
        }
        for (int s = 0; s < 2; s++) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&afull[s])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&aempty[s])), "r"(kProducers) : "memory");
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_abort = 0;
    }
    // all taps' weights, once per CTA (B operands: tap t, output channel n, chunk j at
    // t*TAPB + j*(COUT*16) + n*16)
    if (tid < kProducers) {
        for (int q = tid; q < 27 * COUT * S::CH; q += kProducers) {
            const int t = q / (COUT * S::CH), rem = q - t * (COUT * S::CH);
            const int n = rem / S::CH, j = rem - n * S::CH;
            cp_async16(sW + (uint32_t)(t * S::TAPB + j * (COUT * 16) + n * 16), a.w + ((long)t * COUT + n) * CIN + j * 8, 16);
        }
        cp_async_commit();
        cp_async_wait<0>();
        fence_proxy_async();   // the weights to the tensor core's (async) proxy
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;
    volatile int *abort_flag = &s_abort;
    auto origin = [&](int tile, int &z0, int &x0, int &y0) {
        const int ty = tile % nty, r2 = tile / nty, tx = r2 % ntx, tz = r2 / ntx;
        z0 = 1 + kTz * tz; x0 = 1 + kTx * tx; y0 = 1 + kTy * ty;
    };
    if (warp == 4) {
        // ---- TMA loads: one thread; box g = 3 * (tile's index in this CTA) + dy in slot g % NB ----
        if (lane == 0) {
            long g = 0, last = -1;
            bool fail = false;
            for (int tile = blockIdx.x; tile < ntiles && !fail; tile += gridDim.x) {
                int z0, x0, y0;
                origin(tile, z0, x0, y0);
                for (int dy = 0; dy < 3; dy++, g++) {
                    const int sl = (int)(g % S::NB);
                    const long use = g / S::NB;
                    // the slot was last read by the MMAs of box g - NB
                    if (use >= 1 && !mbar_wait(smem_u32(&bempty[sl]), (uint32_t)((use - 1) & 1))) { fail = true; break; }
                    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(&bfull[sl])),
                                 "r"((uint32_t)S::TXB)
                                 : "memory");
                    tma_load_4d(sT + (uint32_t)(sl * S::BOXB), &map, 0, y0 - 1 + dy, x0 - 1, z0 - 1, smem_u32(&bfull[sl]));
                    last = g;
                }
            }
            // loads still in flight write shared memory: their barrier before the CTA may end
            if (last >= 0 && !mbar_wait(smem_u32(&bfull[last % S::NB]), (uint32_t)((last / S::NB) & 1))) fail = true;
            if (fail) *abort_flag = 1;
        }
    } else if (warp == 5) {
        // ---- MMA issuer: one thread ----
        if (lane == 0) {
            long g = 0, last = -1;
            int q = 0;
            bool fail = false;
            for (int tile = blockIdx.x; tile < ntiles && !fail; tile += gridDim.x, q++) {
                const int b = q & 1, u = q >> 1;
                // the accumulator was last read by the epilogue of tile q - 2
                if (u >= 1 && !mbar_wait(smem_u32(&aempty[b]), (uint32_t)((u - 1) & 1))) { fail = true; break; }
                const uint32_t acc = tmem + (uint32_t)(b * COUT);
                for (int dy = 0; dy < 3; dy++, g++) {
                    const int sl = (int)(g % S::NB);
                    if (!mbar_wait(smem_u32(&bfull[sl]), (uint32_t)((g / S::NB) & 1))) { fail = true; break; }
                    tc_fence_after();
#pragma unroll
                    for (int t9 = 0; t9 < 9; t9++) {
                        const int dz = t9 / 3, dx = t9 % 3, tap = dz * 9 + dx * 3 + dy;
                        const uint32_t sA = sT + (uint32_t)(sl * S::BOXB + (dz * kQx + dx) * 8 * S::ROWB);
                        const uint32_t sB = sW + (uint32_t)(tap * S::TAPB);
#pragma unroll
                        for (int k = 0; k < CIN / 16; k++) {
                            const uint64_t da = smem_desc(sA + (uint32_t)(32 * k), 16, 8 * S::ROWB) | S::ALAYOUT;
                            const uint64_t db = smem_desc(sB + (uint32_t)(2 * k * COUT * 16), COUT * 16, 128);
                            tc_mma(acc, da, db, S::IDESC, (dy > 0 || t9 > 0 || k > 0) ? 1u : 0u);
                        }
                    }
                    // the slot is free once these MMAs complete
                    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                     smem_u32(&bempty[sl]))
                                 : "memory");
                    last = g;
                }
                if (fail) break;
                // the accumulator is full once this tile's MMAs complete
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                 smem_u32(&afull[b]))
                             : "memory");
            }
            // MMAs still in flight read the ring and write TMEM: wait for the last commit
            if (last >= 0 && !mbar_wait(smem_u32(&bempty[last % S::NB]), (uint32_t)((last / S::NB) & 1))) fail = true;
            if (fail) *abort_flag = 1;
        }
    } else {
        // ---- epilogue warps 0-3: TMEM lane m = row (tx = m / 8, ty = m % 8) of the tile ----
        const int m = tid, ox = m >> 3, oy = m & 7;
        int q = 0;
        bool fail = false;
        for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, q++) {
            const int b = q & 1, u = q >> 1;
            if (!mbar_wait(smem_u32(&afull[b]), (uint32_t)(u & 1))) fail = true;
            if (__any_sync(0xffffffffu, fail)) { fail = true; break; }   // tcgen05.ld is warp-collective
            tc_fence_after();
            float v[COUT];
#pragma unroll
            for (int c0 = 0; c0 < COUT; c0 += 16) {
                float t16[16];
                tc_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(b * COUT + c0), t16);
#pragma unroll
                for (int e = 0; e < 16; e++) v[c0 + e] = t16[e];
            }
            tc_fence_before();
            asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&aempty[b])) : "memory");
            int z0, x0, y0;
            origin(tile, z0, x0, y0);
            const int zz = z0, xx = x0 + ox, yy = y0 + oy;
            if (zz > a.d.nz || xx > a.d.nx || yy > a.d.ny) continue;
            const long p = (long)zz * XY + (long)xx * a.d.Y + yy;
#pragma unroll
            for (int c0 = 0; c0 < COUT; c0 += 8) {
                float f[8];
#pragma unroll
                for (int e = 0; e < 8; e++) f[e] = v[c0 + e] + (a.bias ? a.bias[c0 + e] : 0.0f);
                if (a.add) {
                    float h[8];
                    unpack8(*reinterpret_cast<const uint4 *>(a.add + p * COUT + c0), h);
#pragma unroll
                    for (int e = 0; e < 8; e++) f[e] += h[e];
                }
                if (a.relu) {
#pragma unroll
                    for (int e = 0; e < 8; e++) f[e] = fmaxf(f[e], 0.0f);
                }
                if (a.mask) {
                    float h[8];
                    unpack8(*reinterpret_cast<const uint4 *>(a.mask + p * COUT + c0), h);
#pragma unroll
                    for (int e = 0; e < 8; e++) f[e] = h[e] > 0.0f ? f[e] : 0.0f;
                }
                if (a.out) *reinterpret_cast<uint4 *>(a.out + p * COUT + c0) = pack8(f);
                if (a.out32) {
                    *reinterpret_cast<float4 *>(a.out32 + p * COUT + c0) = make_float4(f[0], f[1], f[2], f[3]);
                    *reinterpret_cast<float4 *>(a.out32 + p * COUT + c0 + 4) = make_float4(f[4], f[5], f[6], f[7]);
                }
            }
        }
        if (fail) *abort_flag = 1;
    }
    __syncthreads();
    if (tid == 0 && *abort_flag) atomicExch(a.err, 1);
    tc_fence_after();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(S::NCOL) : "memory");
}

// ---------------------------------------------------------------------------------------
// weight gradients on tcgen05 (CIN, COUT in {16, 32})
// ---------------------------------------------------------------------------------------
// dW[tap][co][ci] = sum over rows of X[row + off_tap][ci] * G[row][co]: per tap a GEMM whose K
// dimension is the grid's rows.  A persistent CTA walks over the same 2 x 8 x 8 output tiles as
// k_conv_brick: it loads the tile's input brick and the tile's 128 rows of G, gathers the shifted
// tap operands from the brick into chunk planes ([channel chunk][row][16 B], as the forward
// gather does), and multiplies them with the tensor core in MN-major form: M = the 128 rows
// (tap, ci) of a group of 128 / CIN taps, N = COUT, K = 16 rows per MMA, eight MMAs per tile and
// group.  Every group accumulates in its own TMEM columns over all the CTA's tiles; at the end
// each CTA adds its sums to dW (FP32 atomics, one per weight per CTA).
template <int CIN, int COUT>
struct WgradShape {
    static constexpr int CH = CIN / 8, CHO = COUT / 8;
    static constexpr int TPG = kTileM / CIN;                        // taps per group: M = 128
    static constexpr int NG = (27 + TPG - 1) / TPG;                 // groups
    static constexpr int ABYTES = kTileM * CIN * 2;                 // one tap's operand (chunk planes)
    static constexpr int GRPB = TPG * ABYTES;                       // one group's operands = 32 KB
    static constexpr int GBYTES = kTileM * COUT * 2;                // the tile's rows of G
    static constexpr int BRICK = kBrickRows * CIN * 2;
    static constexpr int SMEM = 1024 + 2 * GRPB + GBYTES + BRICK;
    static constexpr uint32_t NCOLS = NG * COUT;                    // accumulator columns in use
    static constexpr uint32_t NCOL = NCOLS <= 32 ? 32 : NCOLS <= 64 ? 64 : NCOLS <= 128 ? 128 : 256;
    // kind::f16, D FP32, A and B BF16, both MN-major (bits 15, 16), N = COUT, M = 128
    static constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | (1u << 15) | (1u << 16) |
                                      ((uint32_t)(COUT >> 3) << 17) | ((uint32_t)(kTileM >> 4) << 24);
    static constexpr int SWS = CIN == 16 ? 2 : 1;
    static __device__ __forceinline__ int slot(int r, int j) { return r * CH + (j ^ ((r >> SWS) & (CH - 1))); }
    static_assert((CIN == 16 || CIN == 32) && (COUT == 16 || COUT == 32), "tcgen05 weight-gradient channel counts");
    static_assert(GRPB % 1024 == 0 && GBYTES % 1024 == 0, "operand alignment");
};

template <int CIN, int COUT>
__global__ void __launch_bounds__(128) k_wgrad_tc(const bf16 *X, const bf16 *G, float *part, Dims d, int ntx, int nty,
                                                  int ntiles, int *err)
{
    using S = WgradShape<CIN, COUT>;
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ __align__(8) uint64_t mbar[2];
    __shared__ uint32_t s_tmem;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t sbase = (smem_u32(smem) + 1023u) & ~1023u;
    const uint32_t sG = sbase + 2 * S::GRPB, sBrick = sG + S::GBYTES;
    uint8_t *const gbase = smem + (sbase - smem_u32(smem));
    const uint8_t *const brick = gbase + 2 * S::GRPB + S::GBYTES;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"(S::NCOL)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int s = 0; s < 2; s++)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[s])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;
    const long XY = (long)d.X * d.Y;
    const int oz = tid >> 6, ox = (tid >> 3) & 7, oy = tid & 7;   // this thread's row of the tile
    long g = 0;               // groups issued (buffer g & 1, its commit number g >> 1)
    bool failed = false, first = true;
    for (int tile = blockIdx.x; tile < ntiles && !failed; tile += gridDim.x) {
        const int ty = tile % nty, r2 = tile / nty, tx = r2 % ntx, tz = r2 / ntx;
        const int z0 = 1 + kBz * tz, x0 = 1 + kBx * tx, y0 = 1 + kBy * ty;
        // the previous tile's MMAs read G and the group buffers: all of them done before the loads
        int fail0 = 0;
        if (g > 0 && !mbar_wait(smem_u32(&mbar[(g - 1) & 1]), (uint32_t)(((g - 1) >> 1) & 1))) fail0 = 1;
        if (__syncthreads_or(fail0)) { failed = true; break; }
        for (int q = tid; q < kBrickRows * S::CH; q += 128) {
            const int br = q / S::CH, j = q - br * S::CH;
            const int bz = br / (kHx * kHy), bxy = br - bz * (kHx * kHy), bx = bxy / kHy, by = bxy - bx * kHy;
            const int zz = z0 - 1 + bz, xx = x0 - 1 + bx, yy = y0 - 1 + by;
            const bool ok = zz < d.Z && xx < d.X && yy < d.Y;
            const long src = ok ? (long)zz * XY + (long)xx * d.Y + yy : 0;
            cp_async16(sBrick + (uint32_t)(S::slot(br, j) * 16), X + src * CIN + j * 8, ok ? 16 : 0);
        }
        {
            // G rows of the tile (zero outside the interior: rows beyond the array are not loaded)
            const int zz = z0 + oz, xx = x0 + ox, yy = y0 + oy;
            const bool ok = zz <= d.nz && xx <= d.nx && yy <= d.ny;
            const long p = ok ? (long)zz * XY + (long)xx * d.Y + yy : 0;
#pragma unroll
            for (int j = 0; j < S::CHO; j++) cp_async16(sG + (uint32_t)(j * (kTileM * 16) + tid * 16), G + p * COUT + j * 8, ok ? 16 : 0);
        }
        cp_async_commit();
        cp_async_wait<0>();
        __syncthreads();
        for (int gi = 0; gi < S::NG; gi++, g++) {
            const int b = (int)(g & 1);
            int fail = 0;
            if (g >= 2 && !mbar_wait(smem_u32(&mbar[b]), (uint32_t)(((g - 2) >> 1) & 1))) fail = 1;
            if (!fail) {
                uint8_t *dst = gbase + b * S::GRPB + tid * 16;
#pragma unroll
                for (int tl = 0; tl < S::TPG; tl++) {
                    const int tap = gi * S::TPG + tl;
                    if (tap < 27) {
                        const int dz = tap / 9, dx = (tap / 3) % 3, dy = tap % 3;
                        const int br = ((oz + dz) * kHx + (ox + dx)) * kHy + (oy + dy);
#pragma unroll
                        for (int j = 0; j < S::CH; j++)
                            *reinterpret_cast<uint4 *>(dst + tl * S::ABYTES + j * (kTileM * 16)) =
                                *reinterpret_cast<const uint4 *>(brick + S::slot(br, j) * 16);
                    } else {
#pragma unroll
                        for (int j = 0; j < S::CH; j++)
                            *reinterpret_cast<uint4 *>(dst + tl * S::ABYTES + j * (kTileM * 16)) = make_uint4(0, 0, 0, 0);
                    }
                }
            }
            fence_proxy_async();
            if (__syncthreads_or(fail)) { failed = true; break; }
            if (tid == 0) {
                tc_fence_after();
                const uint32_t sA = sbase + (uint32_t)(b * S::GRPB);
                // MN-major, no swizzle: the leading byte offset is the stride between core matrices
                // along K (8-row groups, 128 B apart), the stride byte offset the one along M or N
                // (channel chunks, 2048 B apart)
#pragma unroll
                for (int kk = 0; kk < kTileM / 16; kk++) {
                    const uint64_t da = smem_desc(sA + (uint32_t)(kk * 256), 128, kTileM * 16);
                    const uint64_t db = smem_desc(sG + (uint32_t)(kk * 256), 128, kTileM * 16);
                    tc_mma(tmem + (uint32_t)(gi * COUT), da, db, S::IDESC, (first && kk == 0) ? 0u : 1u);
                }
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                 smem_u32(&mbar[b]))
                             : "memory");
            }
        }
        first = false;
    }
    int fail = 0;
    if (g > 0 && !mbar_wait(smem_u32(&mbar[(g - 1) & 1]), (uint32_t)(((g - 1) >> 1) & 1))) fail = 1;
    failed = __syncthreads_or(fail || failed) != 0;
    if (failed) {
        if (tid == 0) atomicExch(err, 1);
    } else if (g > 0) {
        // this CTA's sums to its slot of the partial buffer (k_wgrad_reduce adds the slots):
        // TMEM lane m = (tap within the group, ci); column gi * COUT + co
        float *dW = part + (long)blockIdx.x * 27 * COUT * CIN;
        tc_fence_after();
        const int m = warp * 32 + lane, tl = m / CIN, ci = m % CIN;
#pragma unroll
        for (int gi = 0; gi < S::NG; gi++) {
#pragma unroll
            for (int c0 = 0; c0 < COUT; c0 += 16) {
                float v[16];
                tc_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(gi * COUT + c0), v);   // whole warp
                const int tap = gi * S::TPG + tl;
                if (tap < 27) {
#pragma unroll
                    for (int q = 0; q < 16; q++) dW[((long)tap * COUT + c0 + q) * CIN + ci] = v[q];
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(S::NCOL) : "memory");
}

// dW[i] += sum over the CTAs' partial sums part[c][i]
__global__ void k_wgrad_reduce(const float *part, int nparts, int n, float *dW)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float s = 0.0f;
    for (int c = 0; c < nparts; c++) s += part[(long)c * n + i];
    dW[i] += s;
}

// ---------------------------------------------------------------------------------------
// weight and bias gradients (FP32, CUDA cores)
// dW[tap][co][ci] += sum_rows G[row][co] * X[row + off_tap][ci];  db[co] += sum_rows G[row][co]
// ---------------------------------------------------------------------------------------
struct Offs {
    int off[27];
};

template <int CIN, int COUT>
__global__ void __launch_bounds__(256) k_wgrad(const bf16 *X, const bf16 *G, float *dW, long np, Offs o, long rows_per_block)
{
    constexpr int TI = CIN < 32 ? CIN : 32, TO = COUT < 32 ? COUT : 32;
    constexpr int OPT = TI * TO / 256;
    constexpr int PC = 64;
    static_assert(OPT >= 1, "tile");
    __shared__ float xs[PC][TI];
    __shared__ float gs[PC][TO];
    constexpr int NTI = CIN / TI;
    int b = blockIdx.x;
    const int tap = b % 27;
    b /= 27;
    const int ti = b % NTI, to = b / NTI;
    const long off = o.off[tap];
    const long r0 = (long)blockIdx.y * rows_per_block;
    const long r1 = r0 + rows_per_block < np ? r0 + rows_per_block : np;
    float acc[OPT];
#pragma unroll
    for (int k = 0; k < OPT; k++) acc[k] = 0.0f;
    const int tid = threadIdx.x;
    for (long base = r0; base < r1; base += PC) {
        __syncthreads();
        for (int q = tid; q < PC * TI / 8; q += 256) {
            const int r = q / (TI / 8), j = q - r * (TI / 8);
            const long row = base + r, src = row + off;
            float f[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            if (row < r1 && src >= 0 && src < np) unpack8(*reinterpret_cast<const uint4 *>(X + src * CIN + ti * TI + j * 8), f);
#pragma unroll
            for (int e = 0; e < 8; e++) xs[r][j * 8 + e] = f[e];
        }
        for (int q = tid; q < PC * TO / 8; q += 256) {
            const int r = q / (TO / 8), j = q - r * (TO / 8);
            const long row = base + r;
            float f[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            if (row < r1) unpack8(*reinterpret_cast<const uint4 *>(G + row * COUT + to * TO + j * 8), f);
#pragma unroll
            for (int e = 0; e < 8; e++) gs[r][j * 8 + e] = f[e];
        }
        __syncthreads();
#pragma unroll 4
        for (int r = 0; r < PC; r++) {
#pragma unroll
            for (int k = 0; k < OPT; k++) {
                const int oi = tid + 256 * k;
                acc[k] = fmaf(gs[r][oi / TI], xs[r][oi % TI], acc[k]);
            }
        }
    }
#pragma unroll
    for (int k = 0; k < OPT; k++) {
        const int oi = tid + 256 * k;
        const int co = to * TO + oi / TI, ci = ti * TI + oi % TI;
        atomicAdd(dW + ((long)tap * COUT + co) * CIN + ci, acc[k]);
    }
}

template <int COUT>
__global__ void __launch_bounds__(256) k_bgrad(const bf16 *G, float *db, long np)
{
    constexpr int RL = 256 / COUT;   // rows handled at once
    __shared__ float red[256];
    const int ch = threadIdx.x % COUT, rl = threadIdx.x / COUT;
    float s = 0.0f;
    for (long r = (long)blockIdx.x * RL + rl; r < np; r += (long)gridDim.x * RL) s += __bfloat162float(G[r * COUT + ch]);
    red[threadIdx.x] = s;
    __syncthreads();
    if (rl == 0) {
        for (int k = 1; k < RL; k++) s += red[k * COUT + ch];
        atomicAdd(db + ch, s);
    }
}

// ---------------------------------------------------------------------------------------
// grid transfers: R (full weighting) and P (trilinear), vertex-centred, channels-last BF16
// ---------------------------------------------------------------------------------------
__global__ void k_restrict(const bf16 *in, bf16 *out, const bf16 *mask, int C, Dims f, Dims c, float scale)
{
    const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const int ng = C / 8;
    if (idx >= c.n * ng) return;
    const int g = (int)(idx % ng);
    long n = idx / ng;
    const int y = (int)(n % c.ny);
    n /= c.ny;
    const int x = (int)(n % c.nx), z = (int)(n / c.nx);
    float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int dz = -1; dz <= 1; dz++) {
        const int fz = 2 * z + dz;
        if (fz < 0 || fz >= f.nz) continue;
        const float wz = dz == 0 ? 0.5f : 0.25f;
        for (int dx = -1; dx <= 1; dx++) {
            const int fx = 2 * x + dx;
            if (fx < 0 || fx >= f.nx) continue;
            const float wzx = wz * (dx == 0 ? 0.5f : 0.25f);
            for (int dy = -1; dy <= 1; dy++) {
                const int fy = 2 * y + dy;
                if (fy < 0 || fy >= f.ny) continue;
                const float w = wzx * (dy == 0 ? 0.5f : 0.25f);
                const long row = ((long)(fz + 1) * f.X + fx + 1) * f.Y + fy + 1;
                float v[8];
                unpack8(*reinterpret_cast<const uint4 *>(in + row * C + g * 8), v);
#pragma unroll
                for (int e = 0; e < 8; e++) acc[e] = fmaf(w, v[e], acc[e]);
            }
        }
    }
    const long row = ((long)(z + 1) * c.X + x + 1) * c.Y + y + 1;
#pragma unroll
    for (int e = 0; e < 8; e++) acc[e] *= scale;
    if (mask) {
        float m[8];
        unpack8(*reinterpret_cast<const uint4 *>(mask + row * C + g * 8), m);
#pragma unroll
        for (int e = 0; e < 8; e++) acc[e] = m[e] > 0.0f ? acc[e] : 0.0f;
    }
    *reinterpret_cast<uint4 *>(out + row * C + g * 8) = pack8(acc);
}

__global__ void k_prolong(const bf16 *in, bf16 *out, const bf16 *add, const bf16 *mask, int C, Dims f, Dims c, float scale)
{
    const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const int ng = C / 8;
    if (idx >= f.n * ng) return;
    const int g = (int)(idx % ng);
    long n = idx / ng;
    const int y = (int)(n % f.ny);
    n /= f.ny;
    const int x = (int)(n % f.nx), z = (int)(n / f.nx);
    int cz[2], cx[2], cy[2];
    float wz[2], wx[2], wy[2];
    int nzc, nxc, nyc;
    auto split = [](int fi, int *ci, float *w, int &cnt) {
        if ((fi & 1) == 0) { ci[0] = fi >> 1; w[0] = 1.0f; cnt = 1; }
        else { ci[0] = fi >> 1; ci[1] = (fi >> 1) + 1; w[0] = w[1] = 0.5f; cnt = 2; }
    };
    split(z, cz, wz, nzc);
    split(x, cx, wx, nxc);
    split(y, cy, wy, nyc);
    float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int a = 0; a < nzc; a++)
        for (int b = 0; b < nxc; b++)
            for (int e = 0; e < nyc; e++) {
                const float w = wz[a] * wx[b] * wy[e];
                const long row = ((long)(cz[a] + 1) * c.X + cx[b] + 1) * c.Y + cy[e] + 1;
                float v[8];
                unpack8(*reinterpret_cast<const uint4 *>(in + row * C + g * 8), v);
#pragma unroll
                for (int q = 0; q < 8; q++) acc[q] = fmaf(w, v[q], acc[q]);
            }
    const long row = ((long)(z + 1) * f.X + x + 1) * f.Y + y + 1;
#pragma unroll
    for (int q = 0; q < 8; q++) acc[q] *= scale;
    if (add) {
        float v[8];
        unpack8(*reinterpret_cast<const uint4 *>(add + row * C + g * 8), v);
#pragma unroll
        for (int q = 0; q < 8; q++) acc[q] += v[q];
    }
    if (mask) {
        float m[8];
        unpack8(*reinterpret_cast<const uint4 *>(mask + row * C + g * 8), m);
#pragma unroll
        for (int q = 0; q < 8; q++) acc[q] = m[q] > 0.0f ? acc[q] : 0.0f;
    }
    *reinterpret_cast<uint4 *>(out + row * C + g * 8) = pack8(acc);
}

// ---------------------------------------------------------------------------------------
// input, output, loss, optimiser
// ---------------------------------------------------------------------------------------
struct Scales {
    float eta_mean, eta_inv, ro_mean, ro_inv, v_scale, p_scale;
};

__device__ __forceinline__ long node_row(long n, const Dims &d)
{
    const int y = (int)(n % d.ny);
    const long t = n / d.ny;
    const int x = (int)(t % d.nx), z = (int)(t / d.nx);
    return ((long)(z + 1) * d.X + x + 1) * d.Y + y + 1;
}

// in5 = [5][n]: log10 eta, rho, vx, vy, vz (physical units) -> x0 rows, channels 5..15 zero
__global__ void k_pack_input(const float *in5, bf16 *x0, Dims d, Scales s)
{
    const long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= d.n) return;
    const float iv = 1.0f / s.v_scale;
    float f[8] = {(in5[n] - s.eta_mean) * s.eta_inv, (in5[d.n + n] - s.ro_mean) * s.ro_inv, in5[2 * d.n + n] * iv,
                  in5[3 * d.n + n] * iv, in5[4 * d.n + n] * iv, 0.0f, 0.0f, 0.0f};
    float z[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    const long row = node_row(n, d);
    *reinterpret_cast<uint4 *>(x0 + row * 16) = pack8(f);
    *reinterpret_cast<uint4 *>(x0 + row * 16 + 8) = pack8(z);
}

// raw sample from a context's level-0 fields
__global__ void k_from_ctx(const float *nu, const float *ro, const float *vx, const float *vy, const float *vz, float *in5, long n)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    in5[i] = log10f(fmaxf(nu[i], 1e-30f));
    in5[n + i] = ro[i];
    in5[2 * n + i] = vx[i];
    in5[3 * n + i] = vy[i];
    in5[4 * n + i] = vz[i];
}

// target = converged solution - start (the previous step's values)
__global__ void k_target(const double *pr, const float *vx, const float *vy, const float *vz, const double *pr_prev,
                         const float *in5, float *tg4, long n)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    tg4[i] = (float)(pr[i] - pr_prev[i]);
    tg4[n + i] = vx[i] - in5[2 * n + i];
    tg4[2 * n + i] = vy[i] - in5[3 * n + i];
    tg4[3 * n + i] = vz[i] - in5[4 * n + i];
}

// L = mean over nodes and the 4 outputs of (y - t/scale)^2; gy = dL/dy (channels 4..15 zero)
__global__ void k_loss(const bf16 *y, const float *tg4, bf16 *gy, Dims d, Scales s, double *loss)
{
    __shared__ double red[256];
    const long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
    double l = 0.0;
    if (n < d.n) {
        const long row = node_row(n, d);
        float yv[8];
        unpack8(*reinterpret_cast<const uint4 *>(y + row * 16), yv);
        const float inv[4] = {1.0f / s.p_scale, 1.0f / s.v_scale, 1.0f / s.v_scale, 1.0f / s.v_scale};
        const float gsc = 2.0f / (4.0f * (float)d.n);
        float g[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const float diff = yv[c] - tg4[c * d.n + n] * inv[c];
            l += (double)diff * diff;
            g[c] = gsc * diff;
        }
        float z[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        if (gy) {
            *reinterpret_cast<uint4 *>(gy + row * 16) = pack8(g);
            *reinterpret_cast<uint4 *>(gy + row * 16 + 8) = pack8(z);
        }
    }
    red[threadIdx.x] = l;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) atomicAdd(loss, red[0] / (4.0 * (double)d.n));
}

// y (scaled) -> physical correction [4][n] (FP32), or guess = start + correction (FP64)
__global__ void k_unpack(const bf16 *y, Dims d, Scales s, float *out4, const double *pr, const float *vx, const float *vy,
                         const float *vz, double *g0, double *g1, double *g2, double *g3)
{
    const long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= d.n) return;
    float yv[8];
    unpack8(*reinterpret_cast<const uint4 *>(y + node_row(n, d) * 16), yv);
    const float dp = yv[0] * s.p_scale, dvx = yv[1] * s.v_scale, dvy = yv[2] * s.v_scale, dvz = yv[3] * s.v_scale;
    if (out4) {
        out4[n] = dp;
        out4[d.n + n] = dvx;
        out4[2 * d.n + n] = dvy;
        out4[3 * d.n + n] = dvz;
    }
    if (g0) {
        g0[n] = pr[n] + (double)dp;
        g1[n] = (double)vx[n] + (double)dvx;
        g2[n] = (double)vy[n] + (double)dvy;
        g3[n] = (double)vz[n] + (double)dvz;
    }
}

__global__ void k_adam(float *w, const float *g, float *m, float *v, long n, float lr, float b1, float b2, float eps,
                       float c1, float c2, float gscale)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i] * gscale;
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// FP32 master weights [27][cout][cin] -> BF16 forward copy and the flipped, transposed copy
// wt[26-tap][ci][co] used by the input-gradient convolution
__global__ void k_pack_w(const float *W, bf16 *w, bf16 *wt, int cin, int cout)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long n = 27L * cin * cout;
    if (i >= n) return;
    const int ci = (int)(i % cin);
    const long t2 = i / cin;
    const int co = (int)(t2 % cout), tap = (int)(t2 / cout);
    const bf16 b = __float2bfloat16_rn(W[i]);
    w[i] = b;
    wt[((long)(26 - tap) * cin + ci) * cout + co] = b;
}

__global__ void k_sq_norm(const float *g, long n, double *out)
{
    __shared__ double red[256];
    double s = 0.0;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) s += (double)g[i] * g[i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) atomicAdd(out, red[0]);
}

// ---------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------
inline unsigned nblk(long n, int b = 256) { return (unsigned)((n + b - 1) / b); }


Dims make_dims(int nz, int nx, int ny)
{
    Dims d;
    d.nz = nz;
    d.nx = nx;
    d.ny = ny;
    d.Z = nz + 2;
    d.X = nx + 2;
    d.Y = ny + 2;
    d.np = (long)d.Z * d.X * d.Y;
    d.n = (long)nz * nx * ny;
    return d;
}

void tap_offsets(const Dims &d, int *off)
{
    for (int dz = -1; dz <= 1; dz++)
        for (int dx = -1; dx <= 1; dx++)
            for (int dy = -1; dy <= 1; dy++)
                off[(dz + 1) * 9 + (dx + 1) * 3 + (dy + 1)] = dz * d.X * d.Y + dx * d.Y + dy;
}

// Per-device launch set-up of a persistent tensor-core kernel: its shared-memory attributes (set
// once per device: a function attribute belongs to the device it was set on) and its grid, every
// resident CTA on every SM from the shared-memory footprint (each CTA holds at most 256 of the
// 512 TMEM columns and 128 threads of fewer than 96 registers, which bind less)
struct LaunchSetup { int sms = 0, per_sm = 0; };
constexpr int kMaxDev = 64;
std::mutex g_setup_mu;   // the per-device set-up caches may be filled from several host threads

template <typename K>
cudaError_t persistent_setup(K kernel, int smem, int max_per_sm, LaunchSetup (&cache)[kMaxDev], LaunchSetup &out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDev) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_setup_mu);
    LaunchSetup &c = cache[dev];
    if (!c.per_sm) {
        if ((e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) != cudaSuccess) return e;
        // the whole unified L1 as shared memory, so that several CTAs fit on an SM
        if ((e = cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, 100)) != cudaSuccess) return e;
        int sms = 0, smem_sm = 0;
        if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
        if ((e = cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev)) != cudaSuccess) return e;
        c.sms = sms;
        c.per_sm = std::max(1, std::min(max_per_sm, smem_sm / (smem + 1024 + 64)));
    }
    out = c;
    return cudaSuccess;
}

template <int CIN, int COUT>
cudaError_t launch_conv_t(const ConvArgs &a, cudaStream_t st)
{
    using S = ConvShape<CIN, COUT>;
    static bool attr[kMaxDev] = {};
    int dev = 0;
    cudaError_t e0 = cudaGetDevice(&dev);
    if (e0 != cudaSuccess) return e0;
    if (dev < 0 || dev >= kMaxDev) return cudaErrorInvalidDevice;
    {
        std::lock_guard<std::mutex> lock(g_setup_mu);
        if (!attr[dev]) {
            cudaError_t e = cudaFuncSetAttribute(k_conv_tc<CIN, COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, S::SMEM);
            if (e != cudaSuccess) return e;
            attr[dev] = true;
        }
    }
    k_conv_tc<CIN, COUT><<<nblk(a.d.np, kTileM), 128, S::SMEM, st>>>(a);
    return cudaGetLastError();
}

// persistent grid of the brick kernel: every resident CTA on every SM, at most one per tile
template <int CIN, int COUT>
cudaError_t launch_brick_t(const ConvArgs &a, cudaStream_t st)
{
    using S = BrickShape<CIN, COUT>;
    static LaunchSetup cache[kMaxDev];
    LaunchSetup ls;
    if (cudaError_t e = persistent_setup(k_conv_brick<CIN, COUT>, S::SMEM, 8, cache, ls)) return e;
    const int sms = ls.sms, per_sm = ls.per_sm;
    const int ntx = (a.d.nx + kBx - 1) / kBx, nty = (a.d.ny + kBy - 1) / kBy, ntz = (a.d.nz + kBz - 1) / kBz;
    const int ntiles = ntx * nty * ntz;
    const int grid = std::min(ntiles, sms * per_sm);
    if (grid < 1) return cudaSuccess;
    k_conv_brick<CIN, COUT><<<grid, kBrickThreads, S::SMEM, st>>>(a, ntx, nty, ntiles);
    return cudaGetLastError();
}

// cuTensorMapEncodeTiled of the driver, looked up once through the runtime (the library links
// only the runtime); null when the driver does not offer it
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled()
{
    static const EncodeTiledFn fn = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return (EncodeTiledFn)p;
    }();
    return fn;
}

// TMA-fed kernel: a 4-D tensor map (channels, y, x, z) over the input with a 32-byte (16 channels)
// or 64-byte (32 channels) swizzle; rows past the array's ends load as zeros.  Without the driver
// entry point (or with an input that is not 16-byte aligned) the layer goes to the brick kernel.
template <int CIN, int COUT>
cudaError_t launch_tma_t(const ConvArgs &a, cudaStream_t st)
{
    using S = TmaShape<CIN, COUT>;
    const EncodeTiledFn enc = encode_tiled();
    if (!enc || (reinterpret_cast<uintptr_t>(a.in) & 15u)) return launch_brick_t<CIN, COUT>(a, st);
    static LaunchSetup cache[kMaxDev];
    LaunchSetup ls;
    if (cudaError_t e = persistent_setup(k_conv_tma<CIN, COUT>, S::SMEM, 8, cache, ls)) return e;
    CUtensorMap map;
    memset(&map, 0, sizeof(map));
    const cuuint64_t dim[4] = {(cuuint64_t)CIN, (cuuint64_t)a.d.Y, (cuuint64_t)a.d.X, (cuuint64_t)a.d.Z};
    const cuuint64_t stride[3] = {(cuuint64_t)CIN * 2, (cuuint64_t)a.d.Y * CIN * 2, (cuuint64_t)a.d.X * a.d.Y * CIN * 2};
    const cuuint32_t box[4] = {(cuuint32_t)CIN, (cuuint32_t)kQy, (cuuint32_t)kQx, (cuuint32_t)kQz}, estr[4] = {1, 1, 1, 1};
    if (enc(&map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, (void *)a.in, dim, stride, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CIN == 16 ? CU_TENSOR_MAP_SWIZZLE_32B : CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return cudaErrorInvalidValue;
    const int ntx = (a.d.nx + kTx - 1) / kTx, nty = (a.d.ny + kTy - 1) / kTy, ntz = (a.d.nz + kTz - 1) / kTz;
    const int ntiles = ntx * nty * ntz;
    const int grid = std::min(ntiles, ls.sms * ls.per_sm);
    if (grid < 1) return cudaSuccess;
    k_conv_tma<CIN, COUT><<<grid, kTmaThreads, S::SMEM, st>>>(map, a, ntx, nty, ntiles);
    return cudaGetLastError();
}

// Layers with 16 or 32 channels in and out (the fine levels, most of the network's time) go to the
// TMA-fed kernel (I3G_CONV_TMA=0: the brick kernel; with I3G_CONV_BRICK=0 as well: k_conv_tc); the
// wider ones to k_conv_tc.
cudaError_t launch_conv(int cin, int cout, const ConvArgs &a, cudaStream_t st)
{
    static const bool brick = !getenv("I3G_CONV_BRICK") || atoi(getenv("I3G_CONV_BRICK")) != 0;
    static const bool tma = !getenv("I3G_CONV_TMA") || atoi(getenv("I3G_CONV_TMA")) != 0;
    if (tma) {
#define I3G_TMA_CASE(I, O) \
        if (cin == I && cout == O) return launch_tma_t<I, O>(a, st);
        I3G_TMA_CASE(16, 16) I3G_TMA_CASE(16, 32) I3G_TMA_CASE(32, 16) I3G_TMA_CASE(32, 32)
#undef I3G_TMA_CASE
    }
    if (brick) {
#define I3G_BRICK_CASE(I, O) \
        if (cin == I && cout == O) return launch_brick_t<I, O>(a, st);
        I3G_BRICK_CASE(16, 16) I3G_BRICK_CASE(16, 32) I3G_BRICK_CASE(32, 16) I3G_BRICK_CASE(32, 32)
#undef I3G_BRICK_CASE
    }
#define I3G_CONV_CASE(I, O) \
    if (cin == I && cout == O) return launch_conv_t<I, O>(a, st);
    I3G_CONV_CASE(16, 16) I3G_CONV_CASE(16, 32) I3G_CONV_CASE(32, 16) I3G_CONV_CASE(32, 32) I3G_CONV_CASE(32, 64)
    I3G_CONV_CASE(64, 32) I3G_CONV_CASE(64, 64) I3G_CONV_CASE(64, 128) I3G_CONV_CASE(128, 64) I3G_CONV_CASE(128, 128)
#undef I3G_CONV_CASE
    return cudaErrorInvalidValue;
}

template <int CIN, int COUT>
void launch_wgrad_t(const bf16 *X, const bf16 *G, float *dW, float *db, const Dims &d, const Offs &o, cudaStream_t st)
{
    constexpr int TI = CIN < 32 ? CIN : 32, TO = COUT < 32 ? COUT : 32;
    const int gx = 27 * (CIN / TI) * (COUT / TO);
    long gy = (4L * 148 * 8 + gx - 1) / gx;
    const long maxy = (d.np + 255) / 256;
    if (gy > maxy) gy = maxy;
    if (gy < 1) gy = 1;
    long rows = (d.np + gy - 1) / gy;
    rows = (rows + 63) / 64 * 64;
    gy = (d.np + rows - 1) / rows;
    k_wgrad<CIN, COUT><<<dim3(gx, (unsigned)gy), 256, 0, st>>>(X, G, dW, d.np, o, rows);
    const long bb = (d.np + 255) / 256 < 1184 ? (d.np + 255) / 256 : 1184;
    k_bgrad<COUT><<<(unsigned)bb, 256, 0, st>>>(G, db, d.np);
}

// resident k_wgrad_tc CTAs per SM: the shared-memory footprint decides (at most 2, so that the
// TMEM columns of one SM's CTAs stay within 512)
constexpr int kWgradPerSm = 2;

template <int CIN, int COUT>
cudaError_t launch_wgrad_tc_t(const bf16 *X, const bf16 *G, float *dW, float *db, const Dims &d, float *part, int slots,
                              int *err, cudaStream_t st)
{
    using S = WgradShape<CIN, COUT>;
    static LaunchSetup cache[kMaxDev];
    LaunchSetup ls;
    if (cudaError_t e = persistent_setup(k_wgrad_tc<CIN, COUT>, S::SMEM, kWgradPerSm, cache, ls)) return e;
    const int sms = ls.sms, per_sm = ls.per_sm;
    const int ntx = (d.nx + kBx - 1) / kBx, nty = (d.ny + kBy - 1) / kBy, ntz = (d.nz + kBz - 1) / kBz;
    const int ntiles = ntx * nty * ntz;
    const int grid = std::min(std::min(ntiles, sms * per_sm), slots);
    if (grid >= 1) {
        k_wgrad_tc<CIN, COUT><<<grid, 128, S::SMEM, st>>>(X, G, part, d, ntx, nty, ntiles, err);
        const int n = 27 * COUT * CIN;
        k_wgrad_reduce<<<(n + 255) / 256, 256, 0, st>>>(part, grid, n, dW);
    }
    const long bb = (d.np + 255) / 256 < 1184 ? (d.np + 255) / 256 : 1184;
    k_bgrad<COUT><<<(unsigned)bb, 256, 0, st>>>(G, db, d.np);
    return cudaGetLastError();
}

// Weight and bias gradients of one layer.  The 16/32-channel layers (levels 0 and 1) run on the
// tensor cores (k_wgrad_tc, partial sums per CTA in part[slots][27 * 32 * 32]); the wider ones, or
// all with I3G_WGRAD_TC=0, on the CUDA cores (k_wgrad).
cudaError_t launch_wgrad(int cin, int cout, const bf16 *X, const bf16 *G, float *dW, float *db, const Dims &d, const Offs &o,
                         float *part, int slots, int *err, cudaStream_t st)
{
    static const bool tc = !getenv("I3G_WGRAD_TC") || atoi(getenv("I3G_WGRAD_TC")) != 0;
    if (tc) {
#define I3G_WT_CASE(I, O) \
        if (cin == I && cout == O) return launch_wgrad_tc_t<I, O>(X, G, dW, db, d, part, slots, err, st);
        I3G_WT_CASE(16, 16) I3G_WT_CASE(16, 32) I3G_WT_CASE(32, 16) I3G_WT_CASE(32, 32)
#undef I3G_WT_CASE
    }
#define I3G_WG_CASE(I, O) \
    if (cin == I && cout == O) { launch_wgrad_t<I, O>(X, G, dW, db, d, o, st); return cudaGetLastError(); }
    I3G_WG_CASE(16, 16) I3G_WG_CASE(16, 32) I3G_WG_CASE(32, 32) I3G_WG_CASE(32, 64) I3G_WG_CASE(64, 64)
    I3G_WG_CASE(64, 128) I3G_WG_CASE(128, 128) I3G_WG_CASE(128, 64) I3G_WG_CASE(64, 32) I3G_WG_CASE(32, 16)
#undef I3G_WG_CASE
    return cudaErrorInvalidValue;
}

}  // namespace unet
}  // namespace i3g

using namespace i3g::unet;

struct i3g_unet {
    int dev = 0;
    cudaStream_t st = nullptr;
    Dims L[kLevels];
    Offs off[kLevels];
    long nparam = 0;
    long woff[kLayers] = {}, boff[kLayers] = {};
    float *par = nullptr, *grad = nullptr, *am = nullptr, *av = nullptr;
    bf16 *w[kLayers] = {}, *wt[kLayers] = {};
    bf16 *act[kTensors] = {}, *grd[kTensors] = {};
    int cap = 0;
    float *ds_in = nullptr, *ds_tg = nullptr;   // [cap][5][n], [cap][4][n]
    float *tmp_in = nullptr, *tmp_out = nullptr;
    double *pr_prev = nullptr;                  // start pressure of the last captured input
    double *dsum = nullptr;                     // device reductions
    int *derr = nullptr;
    float *wpart = nullptr;                     // per-CTA weight-gradient sums of k_wgrad_tc
    int wpart_slots = 0;
    Scales sc = {21.0f, 0.5f, 3300.0f, 0.01f, 1e-10f, 1e6f};
    int adam_t = 0;
};

namespace {

int fail_cuda(cudaError_t e, const char *what)
{
    return set_global_error(I3G_E_CUDA, "U-Net: %s: %s", what, cudaGetErrorString(e));
}

#define UCHK(call)                                          \
    do {                                                    \
        cudaError_t e_ = (call);                            \
        if (e_ != cudaSuccess) return fail_cuda(e_, #call); \
    } while (0)

int check_err(i3g_unet *u)
{
    int h = 0;
    UCHK(cudaMemcpyAsync(&h, u->derr, sizeof(int), cudaMemcpyDeviceToHost, u->st));
    UCHK(cudaStreamSynchronize(u->st));
    // fatal: the timed-out CTA released its TMEM after a second bounded wait only, so
    // tensor-core work of that launch may have been abandoned; destroy the handle (and do not
    // reuse the CUDA context for results that must be trusted)
    if (h) return set_global_error(I3G_E_CUDA, "U-Net: a convolution timed out waiting for its tensor-core stage "
                                               "(fatal: destroy this handle)");
    return 0;
}

ConvArgs conv_args(i3g_unet *u, int lev)
{
    ConvArgs a = {};
    a.d = u->L[lev];
    memcpy(a.off, u->off[lev].off, sizeof(a.off));
    a.err = u->derr;
    return a;
}

int forward(i3g_unet *u)
{
    for (int l = 0; l < kLayers; l++) {
        const LayerDef &ld = kL[l];
        // the transfer that produces this layer's input
        const int in = ld.in;
        if (in == D1 || in == D2 || in == D3) {
            const int src = in == D1 ? E0 : in == D2 ? E1 : E2;
            const Dims &f = u->L[kT[src].lev], &c = u->L[kT[in].lev];
            k_restrict<<<nblk(c.n * kT[in].ch / 8), 256, 0, u->st>>>(u->act[src], u->act[in], nullptr, kT[in].ch, f, c, 1.0f);
        } else if (in == U2 || in == U1 || in == U0) {
            const int src = in == U2 ? B3 : in == U1 ? G2 : G1;
            const Dims &c = u->L[kT[src].lev], &f = u->L[kT[in].lev];
            k_prolong<<<nblk(f.n * kT[in].ch / 8), 256, 0, u->st>>>(u->act[src], u->act[in], nullptr, nullptr, kT[in].ch, f, c, 1.0f);
        }
        ConvArgs a = conv_args(u, kT[ld.out].lev);
        a.in = u->act[in];
        a.w = u->w[l];
        a.bias = u->par + u->boff[l];
        a.add = ld.add >= 0 ? u->act[ld.add] : nullptr;
        a.relu = ld.relu;
        a.out = u->act[ld.out];
        UCHK(launch_conv(kT[in].ch, kT[ld.out].ch, a, u->st));
    }
    return 0;
}

// Gradients of the loss for the sample in act[X0] whose dL/dy is in grd[Y]; accumulated into u->grad.
int backward(i3g_unet *u)
{
    for (int l = kLayers - 1; l >= 0; l--) {
        const LayerDef &ld = kL[l];
        const int in = ld.in, out = ld.out;
        const Dims &d = u->L[kT[out].lev];
        UCHK(launch_wgrad(kT[in].ch, kT[out].ch, u->act[in], u->grd[out], u->grad + u->woff[l], u->grad + u->boff[l], d,
                          u->off[kT[out].lev], u->wpart, u->wpart_slots, u->derr, u->st));
        if (l == 0) break;
        ConvArgs a = conv_args(u, kT[out].lev);
        a.in = u->grd[out];
        a.w = u->wt[l];
        // inputs that are ReLU outputs receive the pre-activation gradient directly
        const bool relu_in = !(in == D1 || in == D2 || in == D3 || in == U2 || in == U1 || in == U0);
        a.mask = relu_in ? u->act[in] : nullptr;
        a.out = u->grd[in];
        UCHK(launch_conv(kT[out].ch, kT[in].ch, a, u->st));
        if (in == U2 || in == U1 || in == U0) {
            // P^T = 8 R, then the ReLU mask of the decoder output it came from
            const int src = in == U2 ? B3 : in == U1 ? G2 : G1;
            const Dims &f = u->L[kT[in].lev], &c = u->L[kT[src].lev];
            k_restrict<<<nblk(c.n * kT[src].ch / 8), 256, 0, u->st>>>(u->grd[in], u->grd[src], u->act[src], kT[src].ch, f, c, 8.0f);
        } else if (in == D1 || in == D2 || in == D3) {
            // R^T = P / 8, plus the skip connection's gradient (the decoder's pre-activation
            // gradient at this level), then the encoder output's ReLU mask
            const int src = in == D1 ? E0 : in == D2 ? E1 : E2;
            const int skip = in == D1 ? G0A : in == D2 ? G1A : G2A;
            const Dims &c = u->L[kT[in].lev], &f = u->L[kT[src].lev];
            k_prolong<<<nblk(f.n * kT[src].ch / 8), 256, 0, u->st>>>(u->grd[in], u->grd[src], u->grd[skip], u->act[src],
                                                                       kT[src].ch, f, c, 0.125f);
        }
    }
    return 0;
}

int pack_weights(i3g_unet *u)
{
    for (int l = 0; l < kLayers; l++) {
        const int cin = kT[kL[l].in].ch, cout = kT[kL[l].out].ch;
        k_pack_w<<<nblk(27L * cin * cout), 256, 0, u->st>>>(u->par + u->woff[l], u->w[l], u->wt[l], cin, cout);
    }
    UCHK(cudaGetLastError());
    return 0;
}

int check_slot(i3g_unet *u, int slot)
{
    if (slot < 0 || slot >= u->cap) return set_global_error(I3G_E_ARG, "U-Net: sample slot %d outside [0, %d)", slot, u->cap);
    return 0;
}

int load_sample(i3g_unet *u, const float *in5)
{
    k_pack_input<<<nblk(u->L[0].n), 256, 0, u->st>>>(in5, u->act[X0], u->L[0], u->sc);
    UCHK(cudaGetLastError());
    return 0;
}

// forward + loss (+ backward) of one sample; loss added to dsum[0]
int sample_pass(i3g_unet *u, const float *in5, const float *tg4, bool grads)
{
    int rc;
    if ((rc = load_sample(u, in5)) || (rc = forward(u))) return rc;
    k_loss<<<nblk(u->L[0].n), 256, 0, u->st>>>(u->act[Y], tg4, grads ? u->grd[Y] : nullptr, u->L[0], u->sc, u->dsum);
    UCHK(cudaGetLastError());
    if (grads && (rc = backward(u))) return rc;
    return 0;
}

uint64_t splitmix(uint64_t &s)
{
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

}  // namespace

extern "C" {

int i3g_unet_create(int nx, int ny, int nz, int capacity, uint64_t seed, i3g_unet **out)
{
    if (!out) return set_global_error(I3G_E_ARG, "U-Net: null output pointer");
    *out = nullptr;
    const int dims[3] = {nx, ny, nz};
    for (int a = 0; a < 3; a++)
        if (dims[a] < 9 || (dims[a] - 1) % 8 != 0)
            return set_global_error(I3G_E_ARG, "U-Net: grid %d x %d x %d: every axis needs n >= 9 and n-1 divisible by 8", nx, ny, nz);
    if (capacity < 0) return set_global_error(I3G_E_ARG, "U-Net: negative capacity");
    i3g_unet *u = new i3g_unet();
    cudaGetDevice(&u->dev);
    int rc = 0;
    auto cleanup = [&](int r) {
        i3g_unet_destroy(u);
        return r;
    };
    if (cudaStreamCreateWithFlags(&u->st, cudaStreamNonBlocking) != cudaSuccess) return cleanup(fail_cuda(cudaGetLastError(), "stream"));
    for (int l = 0; l < kLevels; l++) {
        const int s = 1 << l;
        u->L[l] = make_dims((nz - 1) / s + 1, (nx - 1) / s + 1, (ny - 1) / s + 1);
        tap_offsets(u->L[l], u->off[l].off);
    }
    long np = 0;
    for (int l = 0; l < kLayers; l++) {
        const int cin = kT[kL[l].in].ch, cout = kT[kL[l].out].ch;
        u->woff[l] = np;
        np += 27L * cin * cout;
        u->boff[l] = np;
        np += cout;
    }
    u->nparam = np;
#define UALLOC(ptr, T, n)                                                                          \
    do {                                                                                           \
        cudaError_t e_ = cudaMalloc((void **)&(ptr), sizeof(T) * (size_t)(n));                     \
        if (e_ != cudaSuccess) return cleanup(set_global_error(I3G_E_NOMEM, "U-Net: cudaMalloc %s: %s", #ptr, cudaGetErrorString(e_))); \
        cudaMemset((ptr), 0, sizeof(T) * (size_t)(n));                                             \
    } while (0)
    UALLOC(u->par, float, np);
    UALLOC(u->grad, float, np);
    UALLOC(u->am, float, np);
    UALLOC(u->av, float, np);
    for (int l = 0; l < kLayers; l++) {
        const long nw = 27L * kT[kL[l].in].ch * kT[kL[l].out].ch;
        UALLOC(u->w[l], bf16, nw);
        UALLOC(u->wt[l], bf16, nw);
    }
    for (int t = 0; t < kTensors; t++) {
        const long n = u->L[kT[t].lev].np * kT[t].ch;
        UALLOC(u->act[t], bf16, n);
        if (t != X0) UALLOC(u->grd[t], bf16, n);
    }
    const long n0 = u->L[0].n;
    u->cap = capacity;
    if (capacity > 0) {
        UALLOC(u->ds_in, float, (long)capacity * kInCh * n0);
        UALLOC(u->ds_tg, float, (long)capacity * kOutCh * n0);
    }
    UALLOC(u->tmp_in, float, kInCh * n0);
    UALLOC(u->tmp_out, float, kOutCh * n0);
    UALLOC(u->pr_prev, double, n0);
    UALLOC(u->dsum, double, 4);
    UALLOC(u->derr, int, 1);
    {
        int sms = 0;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, u->dev) != cudaSuccess || sms < 1) sms = 148;
        u->wpart_slots = sms * kWgradPerSm;
        UALLOC(u->wpart, float, (long)u->wpart_slots * 27 * 32 * 32);
    }
#undef UALLOC
    // He initialisation (normal, std sqrt(2 / fan_in)); the output layer starts 100x smaller so
    // that an untrained network leaves the default start almost unchanged
    std::vector<float> h(np, 0.0f);
    uint64_t s = seed ? seed : 1;
    for (int l = 0; l < kLayers; l++) {
        const int cin = kT[kL[l].in].ch, cout = kT[kL[l].out].ch;
        const int cin_eff = l == 0 ? kInCh : cin;
        const float sd = sqrtf(2.0f / (27.0f * cin_eff)) * (l == kLayers - 1 ? 0.01f : 1.0f);
        for (int t = 0; t < 27; t++)
            for (int co = 0; co < cout; co++)
                for (int ci = 0; ci < cin; ci++) {
                    const double u1 = ((splitmix(s) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
                    const double u2 = ((splitmix(s) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
                    const double g = sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
                    h[u->woff[l] + ((long)t * cout + co) * cin + ci] = ci < cin_eff ? (float)(sd * g) : 0.0f;
                }
    }
    if (cudaMemcpy(u->par, h.data(), np * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess)
        return cleanup(fail_cuda(cudaGetLastError(), "upload parameters"));
    if ((rc = pack_weights(u))) return cleanup(rc);
    if (cudaStreamSynchronize(u->st) != cudaSuccess) return cleanup(fail_cuda(cudaGetLastError(), "init"));
    *out = u;
    return 0;
}

void i3g_unet_destroy(i3g_unet *u)
{
    if (!u) return;
    if (u->st) cudaStreamSynchronize(u->st);
    cudaFree(u->par);
    cudaFree(u->grad);
    cudaFree(u->am);
    cudaFree(u->av);
    for (int l = 0; l < kLayers; l++) {
        cudaFree(u->w[l]);
        cudaFree(u->wt[l]);
    }
    for (int t = 0; t < kTensors; t++) {
        cudaFree(u->act[t]);
        cudaFree(u->grd[t]);
    }
    cudaFree(u->ds_in);
    cudaFree(u->ds_tg);
    cudaFree(u->tmp_in);
    cudaFree(u->tmp_out);
    cudaFree(u->pr_prev);
    cudaFree(u->dsum);
    cudaFree(u->derr);
    cudaFree(u->wpart);
    if (u->st) cudaStreamDestroy(u->st);
    delete u;
}

int i3g_unet_nparams(const i3g_unet *u, int64_t *n)
{
    if (!u || !n) return set_global_error(I3G_E_ARG, "U-Net: null argument");
    *n = u->nparam;
    return 0;
}

int i3g_unet_get_params(i3g_unet *u, float *host, int64_t n)
{
    if (!u || !host || n != u->nparam) return set_global_error(I3G_E_ARG, "U-Net: parameter count %lld, expected %ld", (long long)n, u ? u->nparam : 0L);
    UCHK(cudaMemcpyAsync(host, u->par, n * sizeof(float), cudaMemcpyDeviceToHost, u->st));
    UCHK(cudaStreamSynchronize(u->st));
    return 0;
}

int i3g_unet_set_params(i3g_unet *u, const float *host, int64_t n)
{
    if (!u || !host || n != u->nparam) return set_global_error(I3G_E_ARG, "U-Net: parameter count %lld, expected %ld", (long long)n, u ? u->nparam : 0L);
    UCHK(cudaMemcpyAsync(u->par, host, n * sizeof(float), cudaMemcpyHostToDevice, u->st));
    UCHK(cudaMemsetAsync(u->am, 0, n * sizeof(float), u->st));
    UCHK(cudaMemsetAsync(u->av, 0, n * sizeof(float), u->st));
    u->adam_t = 0;
    int rc = pack_weights(u);
    if (rc) return rc;
    UCHK(cudaStreamSynchronize(u->st));
    return 0;
}

int i3g_unet_set_scales(i3g_unet *u, const float s[6])
{
    if (!u || !s) return set_global_error(I3G_E_ARG, "U-Net: null argument");
    if (!(s[1] > 0 && s[3] > 0 && s[4] > 0 && s[5] > 0)) return set_global_error(I3G_E_ARG, "U-Net: scales must be positive");
    u->sc = Scales{s[0], s[1], s[2], s[3], s[4], s[5]};
    return 0;
}

int i3g_unet_set_sample(i3g_unet *u, int slot, const float *in5, const float *tg4)
{
    if (!u) return set_global_error(I3G_E_ARG, "U-Net: null handle");
    int rc = check_slot(u, slot);
    if (rc) return rc;
    const long n = u->L[0].n;
    if (in5) UCHK(cudaMemcpyAsync(u->ds_in + (long)slot * kInCh * n, in5, kInCh * n * sizeof(float), cudaMemcpyHostToDevice, u->st));
    if (tg4) UCHK(cudaMemcpyAsync(u->ds_tg + (long)slot * kOutCh * n, tg4, kOutCh * n * sizeof(float), cudaMemcpyHostToDevice, u->st));
    UCHK(cudaStreamSynchronize(u->st));
    return 0;
}

int i3g_unet_get_sample(i3g_unet *u, int slot, float *in5, float *tg4)
{
    if (!u) return set_global_error(I3G_E_ARG, "U-Net: null handle");
    int rc = check_slot(u, slot);
    if (rc) return rc;
    const long n = u->L[0].n;
    if (in5) UCHK(cudaMemcpyAsync(in5, u->ds_in + (long)slot * kInCh * n, kInCh * n * sizeof(float), cudaMemcpyDeviceToHost, u->st));
    if (tg4) UCHK(cudaMemcpyAsync(tg4, u->ds_tg + (long)slot * kOutCh * n, kOutCh * n * sizeof(float), cudaMemcpyDeviceToHost, u->st));
    UCHK(cudaStreamSynchronize(u->st));
    return 0;
}

static int ctx_matches(i3g_unet *u, i3g_ctx *c)
{
    if (!c) return set_global_error(I3G_E_ARG, "U-Net: null context");
    const Dims &d = u->L[0];
    if (c->m.xnumx != d.nx || c->m.ynumy != d.ny || c->m.znumz != d.nz)
        return set_global_error(I3G_E_ARG, "U-Net: grid %d x %d x %d, context %lld x %lld x %lld", d.nx, d.ny, d.nz,
                                (long long)c->m.xnumx, (long long)c->m.ynumy, (long long)c->m.znumz);
    return 0;
}

// Inputs of the next Stokes solve of context c (its current fields) into sample slot.
int i3g_unet_capture_input(i3g_unet *u, i3g_ctx *c, int slot)
{
    if (!u) return set_global_error(I3G_E_ARG, "U-Net: null handle");
    int rc = check_slot(u, slot);
    if (rc || (rc = ctx_matches(u, c))) return rc;
    UCHK(cudaStreamSynchronize(c->st));
    const long n = u->L[0].n;
    float *in5 = u->ds_in + (long)slot * kInCh * n;
    k_from_ctx<<<nblk(n), 256, 0, u->st>>>(c->lev[0].nu, c->ro, c->vx, c->vy, c->vz, in5, n);
    UCHK(cudaMemcpyAsync(u->pr_prev, c->pr, n * sizeof(double), cudaMemcpyDeviceToDevice, u->st));
    UCHK(cudaStreamSynchronize(u->st));
    return 0;
}

// Converged solution of c minus the start recorded by the last capture_input into slot.
int i3g_unet_capture_target(i3g_unet *u, i3g_ctx *c, int slot)
{
    if (!u) return set_global_error(I3G_E_ARG, "U-Net: null handle");
    int rc = check_slot(u, slot);
    if (rc || (rc = ctx_matches(u, c))) return rc;
    UCHK(cudaStreamSynchronize(c->st));
    const long n = u->L[0].n;
    k_target<<<nblk(n), 256, 0, u->st>>>(c->pr, c->vx, c->vy, c->vz, u->pr_prev, u->ds_in + (long)slot * kInCh * n,
                                         u->ds_tg + (long)slot * kOutCh * n, n);
    UCHK(cudaStreamSynchronize(u->st));
    return 0;
}

int i3g_unet_train_step(i3g_unet *u, const int *slots, int nslots, float lr, double *loss)
{
    if (!u || !slots || nslots <= 0) return set_global_error(I3G_E_ARG, "U-Net: empty batch");
    int rc;
    for (int i = 0; i < nslots; i++)
        if ((rc = check_slot(u, slots[i]))) return rc;
    const long n = u->L[0].n;
    UCHK(cudaMemsetAsync(u->grad, 0, u->nparam * sizeof(float), u->st));
    UCHK(cudaMemsetAsync(u->dsum, 0, 4 * sizeof(double), u->st));
    for (int i = 0; i < nslots; i++)
        if ((rc = sample_pass(u, u->ds_in + (long)slots[i] * kInCh * n, u->ds_tg + (long)slots[i] * kOutCh * n, true))) return rc;
    u->adam_t++;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - powf(b1, (float)u->adam_t), c2 = 1.0f - powf(b2, (float)u->adam_t);
    k_adam<<<nblk(u->nparam), 256, 0, u->st>>>(u->par, u->grad, u->am, u->av, u->nparam, lr, b1, b2, 1e-8f, c1, c2, 1.0f / nslots);
    if ((rc = pack_weights(u))) return rc;
    double h[1];
    UCHK(cudaMemcpyAsync(h, u->dsum, sizeof(double), cudaMemcpyDeviceToHost, u->st));
    if ((rc = check_err(u))) return rc;
    if (loss) *loss = h[0] / nslots;
    return 0;
}

int i3g_unet_loss(i3g_unet *u, const int *slots, int nslots, double *loss)
{
    if (!u || !slots || nslots <= 0) return set_global_error(I3G_E_ARG, "U-Net: empty batch");
    int rc;
    for (int i = 0; i < nslots; i++)
        if ((rc = check_slot(u, slots[i]))) return rc;
    const long n = u->L[0].n;
    UCHK(cudaMemsetAsync(u->dsum, 0, 4 * sizeof(double), u->st));
    for (int i = 0; i < nslots; i++)
        if ((rc = sample_pass(u, u->ds_in + (long)slots[i] * kInCh * n, u->ds_tg + (long)slots[i] * kOutCh * n, false))) return rc;
    double h[1];
    UCHK(cudaMemcpyAsync(h, u->dsum, sizeof(double), cudaMemcpyDeviceToHost, u->st));
    if ((rc = check_err(u))) return rc;
    if (loss) *loss = h[0] / nslots;
    return 0;
}

// Host arrays in, host arrays out: the network's correction [4][n] (physical units) for the
// inputs in5 [5][n]; with tg4 given, also the loss and the parameter gradients of that one sample.
int i3g_unet_eval_host(i3g_unet *u, const float *in5, const float *tg4, float *out4, float *grads, double *loss)
{
    if (!u || !in5) return set_global_error(I3G_E_ARG, "U-Net: null argument");
    const long n = u->L[0].n;
    UCHK(cudaMemcpyAsync(u->tmp_in, in5, kInCh * n * sizeof(float), cudaMemcpyHostToDevice, u->st));
    UCHK(cudaMemsetAsync(u->dsum, 0, 4 * sizeof(double), u->st));
    int rc;
    if (tg4) {
        UCHK(cudaMemcpyAsync(u->tmp_out, tg4, kOutCh * n * sizeof(float), cudaMemcpyHostToDevice, u->st));
        UCHK(cudaMemsetAsync(u->grad, 0, u->nparam * sizeof(float), u->st));
        if ((rc = sample_pass(u, u->tmp_in, u->tmp_out, grads != nullptr))) return rc;
    } else {
        if ((rc = load_sample(u, u->tmp_in)) || (rc = forward(u))) return rc;
    }
    if (out4) {
        k_unpack<<<nblk(n), 256, 0, u->st>>>(u->act[Y], u->L[0], u->sc, u->tmp_out, nullptr, nullptr, nullptr, nullptr, nullptr,
                                             nullptr, nullptr, nullptr);
        UCHK(cudaMemcpyAsync(out4, u->tmp_out, kOutCh * n * sizeof(float), cudaMemcpyDeviceToHost, u->st));
    }
    if (grads && tg4) UCHK(cudaMemcpyAsync(grads, u->grad, u->nparam * sizeof(float), cudaMemcpyDeviceToHost, u->st));
    double h[1];
    UCHK(cudaMemcpyAsync(h, u->dsum, sizeof(double), cudaMemcpyDeviceToHost, u->st));
    if ((rc = check_err(u))) return rc;
    if (loss) *loss = h[0];
    return 0;
}

// Stage the network's start for the next i3g_stokes of c: previous v, P plus the correction.
int i3g_unet_predict(i3g_unet *u, i3g_ctx *c)
{
    if (!u) return set_global_error(I3G_E_ARG, "U-Net: null handle");
    int rc = ctx_matches(u, c);
    if (rc) return rc;
    const long n = u->L[0].n;
    if (!c->guess[0]) {
        // all or nothing: a partial set would be taken as complete by the next call
        bool ok = cudaMalloc((void **)&c->gdots, 2 * sizeof(double)) == cudaSuccess;
        for (int v = 0; v < 4 && ok; v++) ok = cudaMalloc((void **)&c->guess[v], n * sizeof(double)) == cudaSuccess;
        for (int v = 0; v < 8 && ok; v++) ok = cudaMalloc((void **)&c->gsave[v], n * sizeof(double)) == cudaSuccess;
        if (!ok) {
            cudaGetLastError();
            cudaFree(c->gdots);
            c->gdots = nullptr;
            for (int v = 0; v < 4; v++) { cudaFree(c->guess[v]); c->guess[v] = nullptr; }
            for (int v = 0; v < 8; v++) { cudaFree(c->gsave[v]); c->gsave[v] = nullptr; }
            return set_global_error(I3G_E_NOMEM, "U-Net: guess buffers");
        }
    }
    UCHK(cudaStreamSynchronize(c->st));
    k_from_ctx<<<nblk(n), 256, 0, u->st>>>(c->lev[0].nu, c->ro, c->vx, c->vy, c->vz, u->tmp_in, n);
    if ((rc = load_sample(u, u->tmp_in)) || (rc = forward(u))) return rc;
    k_unpack<<<nblk(n), 256, 0, u->st>>>(u->act[Y], u->L[0], u->sc, nullptr, c->pr, c->vx, c->vy, c->vz, c->guess[0],
                                         c->guess[1], c->guess[2], c->guess[3]);
    UCHK(cudaGetLastError());
    if ((rc = check_err(u))) return rc;
    c->guess_pending = 1;
    return 0;
}

// Single convolution through the tensor-core kernel on host data (BF16 bit patterns):
// in [np][cin], w [27][cout][cin], bias [cout] or null, add [np][cout] or null; out [np][cout]
// FP32 (rows outside the interior are left at zero).  Padded grid of nz+2 x nx+2 x ny+2 rows.
// Weight and bias gradients of one convolution layer on host data (BF16 bit patterns): x the
// layer's input [np][cin], g the gradient of its output [np][cout] (zero on the halo rows); dw
// [27][cout][cin] and db [cout] FP32, overwritten.  Padded grid of nz+2 x nx+2 x ny+2 rows.
int i3g_unet_wgrad_host(int cin, int cout, int nx, int ny, int nz, const uint16_t *x, const uint16_t *g, float *dw,
                        float *db)
{
    if (!x || !g || !dw || !db || nx < 1 || ny < 1 || nz < 1) return set_global_error(I3G_E_ARG, "wgrad: bad argument");
    const Dims d = make_dims(nz, nx, ny);
    Offs o;
    tap_offsets(d, o.off);
    bf16 *dx = nullptr, *dg = nullptr;
    float *ddw = nullptr, *ddb = nullptr, *part = nullptr;
    int *derr = nullptr;
    cudaStream_t st = nullptr;
    auto done = [&](int r) {
        if (st) cudaStreamSynchronize(st);
        cudaFree(dx);
        cudaFree(dg);
        cudaFree(ddw);
        cudaFree(ddb);
        cudaFree(part);
        cudaFree(derr);
        if (st) cudaStreamDestroy(st);
        return r;
    };
#define CCHK(call)                                          \
    do {                                                    \
        cudaError_t e_ = (call);                            \
        if (e_ != cudaSuccess) return done(fail_cuda(e_, #call)); \
    } while (0)
    int dev = 0, sms = 0;
    CCHK(cudaGetDevice(&dev));
    CCHK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int slots = std::max(1, sms) * kWgradPerSm;
    const long nw = 27L * cin * cout;
    CCHK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    CCHK(cudaMalloc((void **)&dx, d.np * cin * 2));
    CCHK(cudaMalloc((void **)&dg, d.np * cout * 2));
    CCHK(cudaMalloc((void **)&ddw, nw * 4));
    CCHK(cudaMalloc((void **)&ddb, cout * 4));
    CCHK(cudaMalloc((void **)&part, (long)slots * 27 * 32 * 32 * 4));
    CCHK(cudaMalloc((void **)&derr, 4));
    CCHK(cudaMemsetAsync(derr, 0, 4, st));
    CCHK(cudaMemsetAsync(ddw, 0, nw * 4, st));
    CCHK(cudaMemsetAsync(ddb, 0, cout * 4, st));
    CCHK(cudaMemcpyAsync(dx, x, d.np * cin * 2, cudaMemcpyHostToDevice, st));
    CCHK(cudaMemcpyAsync(dg, g, d.np * cout * 2, cudaMemcpyHostToDevice, st));
    CCHK(launch_wgrad(cin, cout, dx, dg, ddw, ddb, d, o, part, slots, derr, st));
    CCHK(cudaMemcpyAsync(dw, ddw, nw * 4, cudaMemcpyDeviceToHost, st));
    CCHK(cudaMemcpyAsync(db, ddb, cout * 4, cudaMemcpyDeviceToHost, st));
    int h = 0;
    CCHK(cudaMemcpyAsync(&h, derr, 4, cudaMemcpyDeviceToHost, st));
    CCHK(cudaStreamSynchronize(st));
#undef CCHK
    return done(h ? set_global_error(I3G_E_CUDA, "wgrad: tensor-core stage wait timed out") : 0);
}

int i3g_unet_conv_host(int cin, int cout, int nx, int ny, int nz, const uint16_t *in, const uint16_t *w,
                       const float *bias, const uint16_t *add, int relu, float *out)
{
    if (!in || !w || !out || nx < 1 || ny < 1 || nz < 1) return set_global_error(I3G_E_ARG, "conv: bad argument");
    const Dims d = make_dims(nz, nx, ny);
    bf16 *din = nullptr, *dw = nullptr, *dadd = nullptr;
    float *dbias = nullptr, *dout = nullptr;
    int *derr = nullptr;
    int rc = 0;
    cudaStream_t st = nullptr;
    auto done = [&](int r) {
        if (st) cudaStreamSynchronize(st);
        cudaFree(din);
        cudaFree(dw);
        cudaFree(dadd);
        cudaFree(dbias);
        cudaFree(dout);
        cudaFree(derr);
        if (st) cudaStreamDestroy(st);
        return r;
    };
#define CCHK(call)                                          \
    do {                                                    \
        cudaError_t e_ = (call);                            \
        if (e_ != cudaSuccess) return done(fail_cuda(e_, #call)); \
    } while (0)
    CCHK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    CCHK(cudaMalloc((void **)&din, d.np * cin * 2));
    CCHK(cudaMalloc((void **)&dw, 27L * cin * cout * 2));
    CCHK(cudaMalloc((void **)&dout, d.np * cout * 4));
    CCHK(cudaMalloc((void **)&derr, 4));
    CCHK(cudaMemsetAsync(derr, 0, 4, st));
    CCHK(cudaMemsetAsync(dout, 0, d.np * cout * 4, st));
    CCHK(cudaMemcpyAsync(din, in, d.np * cin * 2, cudaMemcpyHostToDevice, st));
    CCHK(cudaMemcpyAsync(dw, w, 27L * cin * cout * 2, cudaMemcpyHostToDevice, st));
    if (bias) {
        CCHK(cudaMalloc((void **)&dbias, cout * 4));
        CCHK(cudaMemcpyAsync(dbias, bias, cout * 4, cudaMemcpyHostToDevice, st));
    }
    if (add) {
        CCHK(cudaMalloc((void **)&dadd, d.np * cout * 2));
        CCHK(cudaMemcpyAsync(dadd, add, d.np * cout * 2, cudaMemcpyHostToDevice, st));
    }
    ConvArgs a = {};
    a.in = din;
    a.w = dw;
    a.bias = dbias;
    a.add = dadd;
    a.out32 = dout;
    a.relu = relu;
    a.d = d;
    tap_offsets(d, a.off);
    a.err = derr;
    CCHK(launch_conv(cin, cout, a, st));
    CCHK(cudaMemcpyAsync(out, dout, d.np * cout * 4, cudaMemcpyDeviceToHost, st));
    int h = 0;
    CCHK(cudaMemcpyAsync(&h, derr, 4, cudaMemcpyDeviceToHost, st));
    CCHK(cudaStreamSynchronize(st));
#undef CCHK
    if (h) rc = set_global_error(I3G_E_CUDA, "conv: tensor-core stage wait timed out");
    return done(rc);
}

// Time one training step (forward + backward + Adam) and one forward pass on sample slot 0.
int i3g_unet_time(i3g_unet *u, int reps, double *ms_train, double *ms_forward)
{
    if (!u || reps <= 0 || u->cap < 1) return set_global_error(I3G_E_ARG, "U-Net: timing needs one stored sample");
    i3g::EventPair ev;
    UCHK(ev.create());
    cudaEvent_t e0 = ev.a, e1 = ev.b;
    const int slot = 0;
    const long n = u->L[0].n;
    float ms = 0;
    // one untimed pass first: the first launch of each kernel loads its module and sets its attributes
    int rc = load_sample(u, u->ds_in + slot * kInCh * n);
    if (!rc) rc = forward(u);
    if (rc) return rc;
    UCHK(cudaEventRecord(e0, u->st));
    for (int r = 0; r < reps && !rc; r++) {
        if ((rc = load_sample(u, u->ds_in + slot * kInCh * n))) break;
        rc = forward(u);
    }
    UCHK(cudaEventRecord(e1, u->st));
    UCHK(cudaEventSynchronize(e1));
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms_forward) *ms_forward = ms / reps;
    if (rc) return rc;
    // parameters are restored afterwards: timing must not train the network
    std::vector<float> keep(u->nparam), km(u->nparam), kv(u->nparam);
    UCHK(cudaMemcpy(keep.data(), u->par, u->nparam * 4, cudaMemcpyDeviceToHost));
    UCHK(cudaMemcpy(km.data(), u->am, u->nparam * 4, cudaMemcpyDeviceToHost));
    UCHK(cudaMemcpy(kv.data(), u->av, u->nparam * 4, cudaMemcpyDeviceToHost));
    const int keep_t = u->adam_t;
    UCHK(cudaEventRecord(e0, u->st));
    for (int r = 0; r < reps && !rc; r++) rc = i3g_unet_train_step(u, &slot, 1, 0.0f, nullptr);
    UCHK(cudaEventRecord(e1, u->st));
    UCHK(cudaEventSynchronize(e1));
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms_train) *ms_train = ms / reps;
    UCHK(cudaMemcpy(u->par, keep.data(), u->nparam * 4, cudaMemcpyHostToDevice));
    UCHK(cudaMemcpy(u->am, km.data(), u->nparam * 4, cudaMemcpyHostToDevice));
    UCHK(cudaMemcpy(u->av, kv.data(), u->nparam * 4, cudaMemcpyHostToDevice));
    u->adam_t = keep_t;
    int r2 = pack_weights(u);
    UCHK(cudaStreamSynchronize(u->st));
    return rc ? rc : r2;
}

// Mean device time of the forward convolution of one layer (its inputs from the last forward
// pass) and the bytes it must move: interior rows of input, output and skip tensor once, weights.
int i3g_unet_time_conv(i3g_unet *u, int layer, int reps, double *ms, double *bytes)
{
    if (!u || layer < 0 || layer >= kLayers || reps <= 0) return set_global_error(I3G_E_ARG, "U-Net: bad layer or reps");
    const LayerDef &ld = kL[layer];
    const int cin = kT[ld.in].ch, cout = kT[ld.out].ch;
    ConvArgs a = conv_args(u, kT[ld.out].lev);
    a.in = u->act[ld.in];
    a.w = u->w[layer];
    a.bias = u->par + u->boff[layer];
    a.add = ld.add >= 0 ? u->act[ld.add] : nullptr;
    a.relu = ld.relu;
    a.out = u->act[ld.out];
    i3g::EventPair ev;
    UCHK(ev.create());
    cudaEvent_t e0 = ev.a, e1 = ev.b;
    UCHK(launch_conv(cin, cout, a, u->st));   // warm-up
    UCHK(cudaEventRecord(e0, u->st));
    for (int r = 0; r < reps; r++) UCHK(launch_conv(cin, cout, a, u->st));
    UCHK(cudaEventRecord(e1, u->st));
    UCHK(cudaEventSynchronize(e1));
    float t = 0;
    cudaEventElapsedTime(&t, e0, e1);
    int rc = check_err(u);
    if (rc) return rc;
    if (ms) *ms = t / reps;
    if (bytes) *bytes = (double)u->L[kT[ld.out].lev].n * 2.0 * (cin + cout + (ld.add >= 0 ? cout : 0)) + 27.0 * cin * cout * 2.0;
    return 0;
}

}  // extern "C"
