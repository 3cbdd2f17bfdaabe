// Per-particle MLP of the surrogate on the 5th-generation tensor cores.
//
// Network: 64 (48 features + zero padding) -> 128 -> 128 -> 128 -> 16 (6
// outputs + zero padding), ReLU, BF16 operands with FP32 accumulation, FP32
// master weights trained with Adam.  Everything is built from one GEMM kernel
//     D[M x N] = A[M x K] * B[N x K]^T        (both operands K-major, BF16)
// whose accumulator lives in tensor memory (TMEM):  a CTA of 4 warps owns a
// 128-row tile of D, stages K-chunks of A and B into shared memory in the
// canonical no-swizzle K-major layout (8-row x 16-byte core matrices), one
// elected thread issues tcgen05.mma (kind::f16, M = 128) and commits to an
// mbarrier, and after the last chunk every warp reads its 32 rows of D back
// with tcgen05.ld for a fused epilogue:
//   EPI_RELU      bias + ReLU, BF16 out in row-major and (optionally)
//                 transposed layout (the transposed copy is the operand of
//                 the weight-gradient GEMM of the backward pass)
//   EPI_OUT       bias, FP32 out; with targets: MSE loss and its gradient,
//                 written as BF16 row-major and transposed
//   EPI_BWD_RELU  gradient through ReLU (mask from the stored activation),
//                 BF16 row-major and transposed
//   EPI_WGRAD     split-K weight gradient, atomically added in FP32
// The forward pass of a surrogate call runs instead as one fused kernel
// (k_mlp_fwd): persistent CTAs keep all four weight matrices in shared memory,
// the feature tiles arrive by TMA (cp.async.bulk.tensor, double-buffered, the
// next tile's copy in flight while the current one is computed), and each
// layer's tcgen05 accumulator goes through TMEM into shared memory as the
// next layer's operand, so no activation touches HBM.
// No CPU fallback exists; the host side is in dmph_surrogate.cu.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include "dmph_internal.h"
#include "dmph_mlp.h"

namespace dmph {

namespace {

constexpr int kThreads = 128;
constexpr int kKC = 64;                         // K elements staged per chunk
constexpr int kStageBytes = 128 * kKC * 2;      // one 128-row operand chunk
constexpr int kSmemBytes = 2 * kStageBytes + 64;  // A, B chunks + mbarrier
constexpr long long kSpinLimit = 1ll << 22;       // bounded mbarrier waits

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

// shared-memory matrix descriptor: no swizzle, K-major canonical layout,
// LBO = byte distance between the two 8-element K halves of an MMA step,
// SBO = byte distance between 8-row groups; version 1 (sm_100)
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// instruction descriptor of kind::f16: D FP32, A and B BF16, both K-major
__host__ __device__ constexpr uint32_t instr_desc(int M, int N)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc)
{
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
        "}\n" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
}

__device__ __forceinline__ void mma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, int count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t phase)
{
    uint32_t ok;
    asm volatile(
        "{\n\t"
        ".reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t"
        "}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(phase)
        : "memory");
    return ok != 0;
}

// bounded wait: false when the limit ran out
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t phase)
{
    for (long long it = 0; it < kSpinLimit; ++it)
        if (mbar_try_wait(bar, phase)) return true;
    return false;
}

__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v)
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// stage rows [r0, r0+rows) x K-chunk [k0, k0+kc) of a row-major BF16 matrix
// (leading dimension ld, valid rows < nrows) into the canonical layout:
// offset(r, k) = (r/8)*kc*16 + (k/8)*128 + (r%8)*16 + (k%8)*2
__device__ __forceinline__ void stage_chunk(uint8_t *dst, const __nv_bfloat16 *src, long long ld, long long r0,
                                            long long nrows, int rows, long long k0, int kc, long long kend)
{
    const int vec_per_row = kc >> 3;
    const int nvec = rows * vec_per_row;
    for (int v = threadIdx.x; v < nvec; v += blockDim.x) {
        const int r = v / vec_per_row, c = v - r * vec_per_row;
        uint4 val = make_uint4(0u, 0u, 0u, 0u);
        const long long gr = r0 + r;
        if (gr < nrows && k0 + c * 8 + 8 <= kend) val = *reinterpret_cast<const uint4 *>(src + gr * ld + k0 + c * 8);
        *reinterpret_cast<uint4 *>(dst + (r >> 3) * (kc * 16) + c * 128 + (r & 7) * 16) = val;
    }
}

}  // namespace

// One 128-row tile of D = A * B^T (rows blockIdx.x), K range split over
// blockIdx.z for the weight-gradient GEMM.
__global__ void __launch_bounds__(kThreads, 1) k_gemm_tn(GemmArgs g)
{
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t *sa = smem;
    uint8_t *sb = smem + kStageBytes;
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + 2 * kStageBytes);
    __shared__ uint32_t tmem_base_s;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long m0 = (long long)blockIdx.x * 128;
    const int N = g.N;
    const uint32_t ncols = N <= 32 ? 32u : (N <= 64 ? 64u : 128u);

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_s)),
                     "r"(ncols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tmem = tmem_base_s;

    // K range of this CTA
    const long long kper = (g.K + gridDim.z - 1) / gridDim.z;
    const long long kb = (long long)blockIdx.z * kper;
    const long long ke = kb + kper < g.K ? kb + kper : g.K;
    const int kc = g.K < kKC ? (int)g.K : kKC;
    const uint32_t idesc = instr_desc(128, N);
    uint32_t phase = 0;
    bool ok = true;
    int issued = 0;
    for (long long k0 = kb; k0 < ke; k0 += kc) {
        stage_chunk(sa, g.A, g.lda, m0, g.M, 128, k0, kc, ke);
        stage_chunk(sb, g.B, g.ldb, 0, N, N, k0, kc, ke);
        fence_async_smem();
        __syncthreads();
        if (threadIdx.x == 0) {
            fence_after_sync();
            for (int ks = 0; ks < kc / 16; ++ks) {
                const uint64_t da = smem_desc(smem_u32(sa) + ks * 256, 128, kc * 16);
                const uint64_t db = smem_desc(smem_u32(sb) + ks * 256, 128, kc * 16);
                mma_bf16(tmem, da, db, idesc, issued > 0 ? 1u : 0u);
                ++issued;
            }
            mma_commit(bar);
        }
        // the chunk buffers are free again once the MMAs that read them completed;
        // every thread agrees on the outcome of the bounded wait
        ok = __syncthreads_and(mbar_wait(bar, phase)) != 0;
        if (!ok) break;
        phase ^= 1u;
    }
    if (!ok) {
        if (threadIdx.x == 0) atomicExch(g.err, 1);
        // bounded second wait for the MMAs still in flight before freeing TMEM
        mbar_wait(bar, phase);
    }
    fence_after_sync();

    const long long row = m0 + warp * 32 + lane;
    const bool have_k = ke > kb;
    if (ok && have_k) {
        float acc_loss = 0.f;
        for (int c0 = 0; c0 < N; c0 += 16) {
            float v[16];
            tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
            if (g.epi == EPI_WGRAD) {
                // D row = output feature m, column = input feature n
                if (row < g.M)
                    for (int i = 0; i < 16; ++i) {
                        const int n = c0 + i;
                        if (n >= N) break;
                        float *dst = g.transpose_out ? g.outF + (long long)n * g.ldo + row : g.outF + row * g.ldo + n;
                        atomicAdd(dst, v[i]);
                    }
                continue;
            }
            if (row >= g.M) continue;
            __align__(16) __nv_bfloat16 hb[16];
            for (int i = 0; i < 16; ++i) {
                const int n = c0 + i;
                float x = v[i];
                if (g.epi == EPI_RELU) {
                    x += g.bias[n];
                    x = fmaxf(x, 0.f);
                } else if (g.epi == EPI_OUT) {
                    x += g.bias[n];
                    if (g.outF) g.outF[row * g.ldo + n] = x;
                    if (g.target) {
                        const float d = n < g.n_valid ? x - g.target[row * g.ldt + n] : 0.f;
                        acc_loss += d * d;
                        x = d * g.grad_scale;  // dL/dy of the mean squared error
                    }
                } else if (g.epi == EPI_BWD_RELU) {
                    const float h = __bfloat162float(g.mask[row * g.ldm + n]);
                    x = h > 0.f ? x : 0.f;
                }
                hb[i] = __float2bfloat16_rn(x);
            }
            if (g.outB) {
                uint4 *dst = reinterpret_cast<uint4 *>(g.outB + row * g.ldo + c0);
                dst[0] = reinterpret_cast<const uint4 *>(hb)[0];
                dst[1] = reinterpret_cast<const uint4 *>(hb)[1];
            }
            if (g.outT)
                for (int i = 0; i < 16; ++i) g.outT[(long long)(c0 + i) * g.ldT + row] = hb[i];
        }
        if (g.epi == EPI_OUT && g.target && g.loss) {
            for (int o = 16; o > 0; o >>= 1) acc_loss += __shfl_xor_sync(0xffffffffu, acc_loss, o);
            if (lane == 0) atomicAdd(g.loss, acc_loss);
        }
    }
    fence_before_sync();
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols));
}


// ------------------------------------------------------------ fused forward
namespace {

// shared memory of k_mlp_fwd (bytes from a 1024-aligned base).  Weights in
// the canonical no-swizzle K-major layout of stage_chunk over their whole K
// (core matrices 128 B apart along K, 8-row groups K*16 B apart); the
// feature tiles and the activations in the layout the TMA box {8 columns,
// 128 rows} writes: K-slice s (8 columns) at s*2048, row r at
// (r/8)*128 + (r%8)*16 inside it (core matrices 2048 B apart along K, 8-row
// groups 128 B apart)
constexpr int kFwdThreads = 128;
constexpr int kW1 = 0;                        // 128 x 64
constexpr int kW2 = kW1 + 128 * 64 * 2;       // 128 x 128
constexpr int kW3 = kW2 + 128 * 128 * 2;      // 128 x 128
constexpr int kW4 = kW3 + 128 * 128 * 2;      // 16 x 128
constexpr int kX0 = kW4 + 16 * 128 * 2;       // two 128 x 64 feature tiles
constexpr int kXBytes = 128 * 64 * 2;
constexpr int kHa = kX0 + 2 * kXBytes;        // 128 x 128 activations
constexpr int kBias = kHa + 128 * 128 * 2;    // 3 x 128 + 16 biases
constexpr int kBiasCount = 3 * 128 + 16;
constexpr int kBarOff = kBias + kBiasCount * 4;  // full[2], mma
constexpr int kFwdSmem = kBarOff + 64;
static_assert(kX0 % 128 == 0 && kHa % 128 == 0 && kBarOff % 8 == 0, "alignment of the fused MLP's buffers");

struct FwdArgs {
    const __nv_bfloat16 *w[kMlpLayers];  // [out][in], BF16
    const float *b[kMlpLayers];
    float *Y;  // [n][kMlpOut]
    long long n;
    int *err;
};

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// one box {8 columns, 128 rows} of the feature matrix at column x (a
// multiple of 8: 16-byte aligned) and row y into shared memory
__device__ __forceinline__ void tma_box(uint32_t dst, const CUtensorMap *map, int x, int y, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
        "[%4];" ::"r"(dst),
        "l"((unsigned long long)map), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

// feature tile t (rows t*128 .. t*128+127, zero past n) into buffer b
__device__ __forceinline__ void issue_tile(uint8_t *smem, const CUtensorMap *map, long long t, int b, uint64_t *full)
{
    mbar_expect_tx(&full[b], kXBytes);
    const uint32_t dst = smem_u32(smem + kX0 + b * kXBytes);
    for (int sl = 0; sl < kMlpIn / 8; ++sl) tma_box(dst + sl * 2048, map, sl * 8, (int)(t * 128), &full[b]);
}

// hidden-layer epilogue: bias and ReLU of this thread's row of the
// accumulator, BF16 into the activation buffer (the next layer's A operand)
__device__ __forceinline__ void epi_hidden(uint32_t tmem, int warp, int lane, const float *bias, uint8_t *H)
{
    const int r = warp * 32 + lane;
    uint8_t *row = H + (r >> 3) * 128 + (r & 7) * 16;
    for (int c0 = 0; c0 < kMlpHidden; c0 += 16) {
        float v[16];
        tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
        __align__(16) __nv_bfloat16 hb[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) hb[i] = __float2bfloat16_rn(fmaxf(v[i] + bias[c0 + i], 0.f));
        *reinterpret_cast<uint4 *>(row + (c0 >> 3) * 2048) = reinterpret_cast<const uint4 *>(hb)[0];
        *reinterpret_cast<uint4 *>(row + ((c0 >> 3) + 1) * 2048) = reinterpret_cast<const uint4 *>(hb)[1];
    }
}

}  // namespace

// Y = MLP(X) for n rows: persistent CTAs over 128-row tiles.  Thread 0
// issues the TMA copies and the MMAs; all four warps run the epilogues (warp
// w reads TMEM lanes 32w..32w+31, its tile rows).  Every wait is bounded; on
// a time-out the kernel sets *err, waits (bounded) for its copies and MMAs in
// flight, frees its TMEM and returns.
__global__ void __launch_bounds__(kFwdThreads, 1) k_mlp_fwd(const __grid_constant__ CUtensorMap map, FwdArgs a)
{
    extern __shared__ __align__(1024) uint8_t smem[];
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + kBarOff);
    uint64_t *mbar = full + 2;
    float *bias = reinterpret_cast<float *>(smem + kBias);
    __shared__ uint32_t tmem_base_s;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long tiles = (a.n + 127) / 128;
    if ((long long)blockIdx.x >= tiles) return;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_s)),
                     "r"(128));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x == 0) {
        mbar_init(&full[0], 1);
        mbar_init(&full[1], 1);
        mbar_init(mbar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // weights and biases, once per CTA
    stage_chunk(smem + kW1, a.w[0], kMlpIn, 0, kMlpHidden, kMlpHidden, 0, kMlpIn, kMlpIn);
    stage_chunk(smem + kW2, a.w[1], kMlpHidden, 0, kMlpHidden, kMlpHidden, 0, kMlpHidden, kMlpHidden);
    stage_chunk(smem + kW3, a.w[2], kMlpHidden, 0, kMlpHidden, kMlpHidden, 0, kMlpHidden, kMlpHidden);
    stage_chunk(smem + kW4, a.w[3], kMlpHidden, 0, kMlpOut, kMlpOut, 0, kMlpHidden, kMlpHidden);
    for (int i = threadIdx.x; i < kBiasCount; i += blockDim.x)
        bias[i] = i < 384 ? a.b[i >> 7][i & 127] : a.b[3][i - 384];
    fence_async_smem();
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tmem = tmem_base_s;
    const uint32_t id_h = instr_desc(128, kMlpHidden), id_o = instr_desc(128, kMlpOut);
    const uint32_t w1 = smem_u32(smem + kW1), w2 = smem_u32(smem + kW2), w3 = smem_u32(smem + kW3),
                   w4 = smem_u32(smem + kW4), ha = smem_u32(smem + kHa);
    uint32_t ph_full[2] = {0u, 0u}, ph_mma = 0u;
    bool pend_full[2] = {false, false}, pend_mma = false;  // thread 0: copies / MMAs in flight
    bool ok = true;
    long long t = blockIdx.x;
    if (threadIdx.x == 0) {
        issue_tile(smem, &map, t, 0, full);
        pend_full[0] = true;
    }
    // one layer: MMAs over K (16 per instruction) from A (activation layout,
    // or the feature tile) and B (weights), then every thread waits for them
    auto layer = [&](uint32_t a_addr, uint32_t b_addr, int K, uint32_t idesc) -> bool {
        if (threadIdx.x == 0) {
            fence_after_sync();
            for (int j = 0; j < K / 16; ++j) {
                const uint64_t da = smem_desc(a_addr + j * 4096, 2048, 128);
                const uint64_t db = smem_desc(b_addr + j * 256, 128, K * 16);
                mma_bf16(tmem, da, db, idesc, j > 0 ? 1u : 0u);
            }
            mma_commit(mbar);
            pend_mma = true;
        }
        const bool done = __syncthreads_and(mbar_wait(mbar, ph_mma)) != 0;
        ph_mma ^= 1u;
        if (done && threadIdx.x == 0) pend_mma = false;
        fence_after_sync();
        return done;
    };
    for (int i = 0; t < tiles; ++i, t += gridDim.x) {
        const int b = i & 1;
        const long long tn = t + gridDim.x;
        // the other buffer was read by the previous tile's first layer, whose
        // MMAs have completed
        if (threadIdx.x == 0 && tn < tiles) {
            issue_tile(smem, &map, tn, b ^ 1, full);
            pend_full[b ^ 1] = true;
        }
        // (only thread 0 waits on the copies; its parities advance on success)
        bool got = true;
        if (threadIdx.x == 0) {
            got = mbar_wait(&full[b], ph_full[b]);
            if (got) {
                pend_full[b] = false;
                ph_full[b] ^= 1u;
            }
        }
        ok = __syncthreads_and(got) != 0;
        if (!ok) break;
        ok = layer(smem_u32(smem + kX0 + b * kXBytes), w1, kMlpIn, id_h);
        if (!ok) break;
        epi_hidden(tmem, warp, lane, bias, smem + kHa);
        fence_async_smem();
        fence_before_sync();
        __syncthreads();
        ok = layer(ha, w2, kMlpHidden, id_h);
        if (!ok) break;
        epi_hidden(tmem, warp, lane, bias + 128, smem + kHa);
        fence_async_smem();
        fence_before_sync();
        __syncthreads();
        ok = layer(ha, w3, kMlpHidden, id_h);
        if (!ok) break;
        epi_hidden(tmem, warp, lane, bias + 256, smem + kHa);
        fence_async_smem();
        fence_before_sync();
        __syncthreads();
        ok = layer(ha, w4, kMlpHidden, id_o);
        if (!ok) break;
        {
            float v[16];
            tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16), v);
            const long long row = t * 128 + warp * 32 + lane;
            if (row < a.n) {
                float4 *dst = reinterpret_cast<float4 *>(a.Y + row * kMlpOut);
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    dst[q] = make_float4(v[4 * q] + bias[384 + 4 * q], v[4 * q + 1] + bias[385 + 4 * q],
                                         v[4 * q + 2] + bias[386 + 4 * q], v[4 * q + 3] + bias[387 + 4 * q]);
            }
        }
        // the accumulator is read before the next tile's first MMA
        fence_before_sync();
        __syncthreads();
    }
    if (!ok && threadIdx.x == 0) {
        // bounded waits for the copies and MMAs still in flight (the MMA
        // parity advanced past the wait that gave up)
        atomicExch(a.err, 1);
        for (int q = 0; q < 2; ++q)
            if (pend_full[q]) mbar_wait(&full[q], ph_full[q]);
        if (pend_mma) mbar_wait(mbar, ph_mma ^ 1u);
    }
    fence_before_sync();
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(128));
}

// column sums of a transposed BF16 matrix (one row per block): bias gradients
__global__ void k_row_sums(const __nv_bfloat16 *__restrict__ T, long long ld, int cols, float *__restrict__ out)
{
    float s = 0.f;
    const __nv_bfloat16 *r = T + (long long)blockIdx.x * ld;
    for (int i = threadIdx.x; i < cols; i += blockDim.x) s += __bfloat162float(r[i]);
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    __shared__ float red[32];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
        out[blockIdx.x] += t;
    }
}

// Adam on the FP32 master parameters; refreshes the BF16 weights and their
// transposed copies
__global__ void k_adam(MlpParamsDev M, float lr, float b1, float b2, float eps, float bc1, float bc2)
{
    const int n = M.count;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float g = M.grad[i];
        const float m = b1 * M.m[i] + (1.f - b1) * g;
        const float v = b2 * M.v[i] + (1.f - b2) * g * g;
        M.m[i] = m;
        M.v[i] = v;
        M.w[i] -= lr * (m / bc1) / (sqrtf(v / bc2) + eps);
        M.grad[i] = 0.f;
    }
}

__global__ void k_weights_to_bf16(MlpParamsDev M)
{
    for (int l = 0; l < kMlpLayers; ++l) {
        const int out = M.out[l], in = M.in[l];
        const float *w = M.w + M.woff[l];
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < out * in; i += gridDim.x * blockDim.x) {
            const int o = i / in, k = i - o * in;
            const __nv_bfloat16 b = __float2bfloat16_rn(w[i]);
            M.wb[l][i] = b;
            M.wt[l][(long long)k * out + o] = b;
        }
    }
}

// ------------------------------------------------------------------ host
void launch_gemm(const GemmArgs &g, int ksplit, cudaStream_t st)
{
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_gemm_tn, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes);
        attr = true;
    }
    const long long tiles = (g.M + 127) / 128;
    dim3 grid((unsigned)tiles, 1, (unsigned)(ksplit > 0 ? ksplit : 1));
    k_gemm_tn<<<grid, kThreads, kSmemBytes, st>>>(g);
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against the driver library)
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static bool looked = false;
    if (!looked) {
        looked = true;
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &f, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
    }
    return fn;
}

int launch_mlp_forward(const MlpParamsDev &M, const __nv_bfloat16 *X, long long n, float *Y, int *err, int sms,
                       cudaStream_t st)
{
    if (n <= 0) return 0;
    if (n > (1ll << 30) || (reinterpret_cast<uintptr_t>(X) & 15) != 0) return -1;
    PFN_cuTensorMapEncodeTiled_v12000 encode = tensor_map_encoder();
    if (!encode) return -2;
    CUtensorMap map;
    const cuuint64_t dims[2] = {(cuuint64_t)kMlpIn, (cuuint64_t)n};
    const cuuint64_t strides[1] = {(cuuint64_t)kMlpIn * sizeof(__nv_bfloat16)};
    const cuuint32_t box[2] = {8u, 128u};
    const cuuint32_t estr[2] = {1u, 1u};
    if (encode(&map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<__nv_bfloat16 *>(X), dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return -3;
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_mlp_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, kFwdSmem);
        attr = true;
    }
    FwdArgs a;
    for (int l = 0; l < kMlpLayers; ++l) {
        a.w[l] = M.wb[l];
        a.b[l] = M.w + M.boff[l];
    }
    a.Y = Y;
    a.n = n;
    a.err = err;
    const long long tiles = (n + 127) / 128;
    const int grid = (int)(tiles < sms ? tiles : sms);
    k_mlp_fwd<<<grid, kFwdThreads, kFwdSmem, st>>>(map, a);
    return 0;
}

void launch_row_sums(const __nv_bfloat16 *T, long long ld, int rows, int cols, float *out, cudaStream_t st)
{
    if (rows > 0) k_row_sums<<<rows, 256, 0, st>>>(T, ld, cols, out);
}

void launch_adam(const MlpParamsDev &M, float lr, int t, cudaStream_t st)
{
    const float b1 = 0.9f, b2 = 0.999f;
    const float bc1 = 1.f - powf(b1, (float)t), bc2 = 1.f - powf(b2, (float)t);
    k_adam<<<64, 256, 0, st>>>(M, lr, b1, b2, 1e-8f, bc1, bc2);
}

void launch_weights_to_bf16(const MlpParamsDev &M, cudaStream_t st)
{
    k_weights_to_bf16<<<64, 256, 0, st>>>(M);
}

}  // namespace dmph
