// Kernels of the bipartite variable-constraint GNN that predicts an IPM warm
// start (no counterpart in the reference). Hidden width 64 throughout.
//
//   hn_gnn_spmm          out = A H or A^T H, H row-major rows x 64 (FP32),
//                        A's FP64 values rounded to FP32; each output row is a
//                        sequential sum over its row of A (deterministic)
//   hn_gnn_linear        Y = act([X1 | X2] W + b): BF16 operands on the tensor
//                        cores (mma.sync m16n8k16, FP32 accumulation)
//   hn_gnn_linear_umma   the same layer on the tcgen05 tensor cores (TMEM
//                        accumulator, bulk-copy staging)
//   hn_gnn_linear_bwd    G = dY * relu'(Y); dX = G W^T and per-CTA partials
//                        of dW = [X1 | X2]^T G on the tcgen05 tensor cores,
//                        db = sum G; partials summed in a fixed order
//                        (deterministic for a given SM count)
//   hn_gnn_adam          Adam step on FP32 master weights
//
// BF16 rounding is round-to-nearest-even of the FP32 operand
// (__float2bfloat16_rn), applied when a tile is staged into shared memory.
#include <atomic>
#include <cuda_bf16.h>

#include <algorithm>

#include "hn_internal.cuh"

namespace hn {
namespace {

constexpr int kH = 64;          // hidden width
constexpr int kGT = 128;        // threads of the GEMM kernels (4 warps)
constexpr int kRowsPerCta = 64; // GEMM rows per CTA (16 per warp)
constexpr int kMaxK = 128;      // [X1 | X2] width

__device__ __forceinline__ void mma_bf16(float* c, const uint32_t* a, const uint32_t* b) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// ---- SpMM: one warp per output row, each lane two of the 64 columns ----
__global__ void gnn_spmm_kernel(int rows, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                const double* __restrict__ val, const float* __restrict__ H, int accumulate,
                                float* __restrict__ out) {
    const int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (r >= rows) return;
    float2 acc = make_float2(0.f, 0.f);
    for (int e = rp[r]; e < rp[r + 1]; ++e) {
        const float a = static_cast<float>(val[e]);
        const float2 h = reinterpret_cast<const float2*>(H + (int64_t)ci[e] * kH)[lane];
        acc.x += a * h.x;
        acc.y += a * h.y;
    }
    float2* o = reinterpret_cast<float2*>(out + (int64_t)r * kH) + lane;
    if (accumulate) {
        const float2 p = *o;
        acc.x = p.x + acc.x;
        acc.y = p.y + acc.y;
    }
    *o = acc;
}

// dH += dX[:, :64]; dAgg = dX[:, 64:] (the two halves of a concatenated input)
__global__ void gnn_split_grad_kernel(int64_t M, const float* __restrict__ dX, float* __restrict__ dH,
                                      float* __restrict__ dAgg) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= M * kH) return;
    const int64_t r = i / kH, c = i % kH;
    dH[i] += dX[r * 2 * kH + c];
    dAgg[i] = dX[r * 2 * kH + kH + c];
}

// Squared-error head: dO[:, c] = scale * 2 (O[:, c] - T[:, c]) for c < nt, 0
// for the other columns; per-block partial sums of the squared errors.
__global__ void gnn_head_grad_kernel(int64_t M, const float* __restrict__ O, const float* __restrict__ T, int nt,
                                     float scale, float* __restrict__ dO, float* __restrict__ loss_part) {
    __shared__ double sh[32];
    double l = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < M * kH; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = i / kH;
        const int c = (int)(i % kH);
        float g = 0.f;
        if (c < nt) {
            const float e = O[i] - T[r * 2 + c];
            g = scale * 2.f * e;
            l += (double)e * (double)e;
        }
        dO[i] = g;
    }
    l = block_sum<256>(l, sh);
    if (threadIdx.x == 0) loss_part[blockIdx.x] = (float)l;
}

// ---- C[M x N] = act([X1 | X2] Bt^T + bias) ----
// X1: M x K1, X2: M x K2 (row-major FP32, K1 + K2 = K <= 128, multiples of
// 16); Bt: N x K row-major BF16 (the weight transposed, K contiguous);
// N = 64 or 128; K <= KMAX. Each warp owns 16 rows and all N columns.
template <int N, int KMAX>
__global__ void __launch_bounds__(kGT) gnn_gemm_kernel(int64_t M, int K1, int K2, const float* __restrict__ X1,
                                                       const float* __restrict__ X2,
                                                       const __nv_bfloat16* __restrict__ Bt,
                                                       const float* __restrict__ bias, int relu,
                                                       float* __restrict__ C) {
    constexpr int KP = KMAX + 8;  // padded rows: the fragment loads of a warp hit 32 banks
    __shared__ __align__(16) __nv_bfloat16 sA[kRowsPerCta][KP];
    __shared__ __align__(16) __nv_bfloat16 sB[N][KP];
    const int K = K1 + K2;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int g = lane >> 2, t = lane & 3;
    for (int idx = tid; idx < N * K; idx += kGT) {
        const int n = idx / K, k = idx % K;
        sB[n][k] = Bt[(int64_t)n * K + k];
    }
    const int64_t row0 = blockIdx.x * (int64_t)kRowsPerCta;
    for (int idx = tid; idx < kRowsPerCta * K; idx += kGT) {
        const int r = idx / K, k = idx % K;
        const int64_t gr = row0 + r;
        float v = 0.f;
        if (gr < M) v = k < K1 ? X1[gr * K1 + k] : X2[gr * K2 + (k - K1)];
        sA[r][k] = __float2bfloat16_rn(v);
    }
    __syncthreads();
    float acc[N / 8][4];
#pragma unroll
    for (int j = 0; j < N / 8; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.f;
    const int rb = warp * 16;
    for (int k0 = 0; k0 < K; k0 += 16) {
        uint32_t a[4];
        a[0] = *reinterpret_cast<const uint32_t*>(&sA[rb + g][k0 + 2 * t]);
        a[1] = *reinterpret_cast<const uint32_t*>(&sA[rb + g + 8][k0 + 2 * t]);
        a[2] = *reinterpret_cast<const uint32_t*>(&sA[rb + g][k0 + 2 * t + 8]);
        a[3] = *reinterpret_cast<const uint32_t*>(&sA[rb + g + 8][k0 + 2 * t + 8]);
#pragma unroll
        for (int j = 0; j < N / 8; ++j) {
            uint32_t b[2];
            b[0] = *reinterpret_cast<const uint32_t*>(&sB[j * 8 + g][k0 + 2 * t]);
            b[1] = *reinterpret_cast<const uint32_t*>(&sB[j * 8 + g][k0 + 2 * t + 8]);
            mma_bf16(acc[j], a, b);
        }
    }
#pragma unroll
    for (int j = 0; j < N / 8; ++j) {
        const int c = j * 8 + 2 * t;
        const float b0 = bias ? bias[c] : 0.f, b1 = bias ? bias[c + 1] : 0.f;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int64_t gr = row0 + rb + g + 8 * h;
            if (gr >= M) continue;
            float v0 = acc[j][2 * h] + b0, v1 = acc[j][2 * h + 1] + b1;
            if (relu) {
                v0 = fmaxf(v0, 0.f);
                v1 = fmaxf(v1, 0.f);
            }
            *reinterpret_cast<float2*>(C + gr * N + c) = make_float2(v0, v1);
        }
    }
}

// ---- the same layer on the 5th-generation tensor cores (tcgen05) ----
// A persistent kernel, one CTA (8 warps) per SM, walks 128-row tiles of Y
// (tile t, t + grid, ...). Per tile:
//   1. the tile's rows of X1 and of X2, contiguous in memory, arrive by one
//      bulk copy each (cp.async.bulk completing on the stage's mbarrier);
//      two stages, so tile i + 2 is in flight while tile i is processed;
//   2. the CTA rounds the staged FP32 rows to BF16 into A in the canonical
//      K-major, no-swizzle layout (core matrices of 8 rows x 16 bytes; the
//      next 8-row group 128 bytes on, the next 8-element K chunk LBO on);
//   3. one thread issues K / 16 tcgen05.mma (kind::f16, BF16 in, FP32
//      accumulated in 64 TMEM columns) and commits to an mbarrier;
//   4. each warp reads 32 rows x 32 columns back (tcgen05.ld), adds the bias,
//      applies ReLU, writes the block into its own part of an output staging
//      tile and reads it back row-wise, so that its global stores cover whole
//      128-byte lines (no wait on the stores anywhere in the loop).
// Lane mappings keep the 128-bit shared loads of step 2 and the stores of
// steps 2 and 4 free of bank conflicts when K1 and K2 are multiples of 32:
// in step 2 a half-warp converts one 8-element chunk of each of 8 rows, the
// chunk index rotating with the row; in step 4 each lane rotates its 8
// four-column groups by its lane index, and the row-wise read-back is
// contiguous per quarter-warp. Every mbarrier wait is bounded: on a timeout
// the CTA records it in *err, waits (bounded) for the copies and the MMA it
// issued, frees TMEM and returns.
constexpr int kUmmaM = 128;
constexpr int kUmmaT = 256;
constexpr uint32_t kUmmaSbo = 128;
constexpr uint32_t kUmmaLboA = (kUmmaM / 8) * 128;  // 2048
constexpr uint32_t kUmmaSpin = 1u << 24;
// Shared-memory plan of the layer kernel for N output columns and inputs of
// up to KMAX columns: two FP32 staging buffers, A (128 x KMAX BF16), B
// (N x KMAX BF16), the FP32 output staging tile. N = 64, KMAX = 128 (the
// layers): 208 KB; N = 128, KMAX = 64 (dX of a 128-wide layer): 160 KB.
template <int N, int KMAX>
struct UmmaPlan {
    static constexpr int kStage = kUmmaM * KMAX * 4;
    static constexpr int kOffA = 2 * kStage;
    static constexpr int kOffB = kOffA + kUmmaM * KMAX * 2;
    static constexpr int kOffOut = kOffB + N * KMAX * 2;
    static constexpr int kSmem = kOffOut + kUmmaM * N * 4;
    static constexpr uint32_t kLboB = (N / 8) * 128;
    // kind::f16 instruction descriptor: F32 accumulator, BF16 A and B, both K-major
    static constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) |
                                       ((uint32_t)(kUmmaM >> 4) << 24);
    static_assert(N == 64 || N == 128, "output width");
    static_assert(kSmem <= 227 * 1024, "tcgen05 layer shared memory");
};

__device__ __forceinline__ uint64_t umma_smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    // start address, leading and stride byte offsets (16-byte units), version 1, no swizzle
    return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | ((uint64_t)1 << 46);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, uint32_t limit = kUmmaSpin) {
    if (limit < kUmmaSpin) {
        // a shortened limit (the test hook) polls without suspending, so a
        // wait on copies still in flight gives up after `limit` polls
        for (uint32_t it = 0; it < limit; ++it) {
            uint32_t done;
            asm volatile(
                "{\n\t.reg .pred P1;\n\tmbarrier.test_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
                "selp.b32 %0, 1, 0, P1;\n\t}\n"
                : "=r"(done)
                : "r"(bar), "r"(parity)
                : "memory");
            if (done) return true;
        }
        return false;
    }
    for (uint32_t it = 0; it < limit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void mbar_expect(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

__device__ __forceinline__ int umma_rows(int64_t M, int64_t tile) {
    const int64_t r = M - tile * kUmmaM;
    return (int)(r < kUmmaM ? r : kUmmaM);
}

// Y (M x N, row stride N) = act([X1 | X2] Bt^T + bias), Bt: N x K BF16.
template <int N, int KMAX>
__global__ void __launch_bounds__(kUmmaT, 1) gnn_umma_kernel(int64_t M, int K1, int K2, const float* __restrict__ X1,
                                                             const float* __restrict__ X2,
                                                             const __nv_bfloat16* __restrict__ Bt,
                                                             const float* __restrict__ bias, int relu,
                                                             float* __restrict__ Y, int* err, uint32_t spin) {
    using P = UmmaPlan<N, KMAX>;
    extern __shared__ __align__(1024) uint8_t umma_smem[];
    uint8_t* sA = umma_smem + P::kOffA;
    uint8_t* sB = umma_smem + P::kOffB;
    uint8_t* sOut = umma_smem + P::kOffOut;
    __shared__ __align__(8) uint64_t full[2];
    __shared__ __align__(8) uint64_t mma_bar;
    __shared__ uint32_t s_tmem;
    __shared__ float s_bias[N];
    const int K = K1 + K2, Kc = K / 8;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int64_t ntiles = (M + kUmmaM - 1) / kUmmaM;
    const int64_t grid = gridDim.x;

    // weights: N x K BF16 into the canonical layout, bias
    for (int idx = tid; idx < N * Kc; idx += kUmmaT) {
        const int n = idx / Kc, kc = idx % Kc;
        *reinterpret_cast<uint4*>(sB + kc * P::kLboB + (n >> 3) * kUmmaSbo + (n & 7) * 16) =
            *reinterpret_cast<const uint4*>(Bt + (int64_t)n * K + kc * 8);
    }
    if (tid < N) s_bias[tid] = bias ? bias[tid] : 0.f;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"(N));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    const uint32_t bar_full0 = smem_u32(&full[0]), bar_mma = smem_u32(&mma_bar);
    const uint32_t stage0 = smem_u32(umma_smem);
    // tile t into stage s: X1 rows at the stage start, X2 rows 128 * K1 floats on
    auto issue = [&](int64_t t, int s) {
        const uint32_t rows = (uint32_t)umma_rows(M, t), bar = bar_full0 + 8 * s;
        mbar_expect(bar, rows * 4u * (uint32_t)K);
        bulk_load(stage0 + s * P::kStage, X1 + t * kUmmaM * K1, rows * 4u * (uint32_t)K1, bar);
        if (K2) bulk_load(stage0 + s * P::kStage + kUmmaM * 4 * K1, X2 + t * kUmmaM * K2, rows * 4u * (uint32_t)K2, bar);
    };
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_full0));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_full0 + 8));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_mma));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        for (int p = 0; p < 2; ++p)
            if (blockIdx.x + p * grid < ntiles) issue(blockIdx.x + p * grid, p);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // staged weights -> tensor core
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;

    const int q = warp & 3, half = warp >> 2;  // TMEM lanes 32q.., columns 32 half..
    const int orow = 32 * q + lane, rot = lane & 7;
    bool bad = false;
    int64_t i = 0, t = blockIdx.x;
    for (; t < ntiles; t += grid, ++i) {
        const int s = (int)(i & 1);
        const int rows = umma_rows(M, t);
        const bool ok = !bad && mbar_wait(bar_full0 + 8 * s, (uint32_t)((i >> 1) & 1), spin);
        if (ok) {
            const uint8_t* x1 = umma_smem + s * P::kStage;
            const uint8_t* x2 = x1 + kUmmaM * 4 * K1;
            // lane-item u: half-warp h = u / 16 converts chunk ((r / 2) + h / 16) mod Kc
            // of rows 8 (h mod 16) + r, r = l mod 8; lane l < 8 takes the half
            // (r mod 2) of it, lane l + 8 the other half
            for (int u = tid; u < 256 * Kc; u += kUmmaT) {
                const int h = u >> 4, l = u & 15;
                const int rl = l & 7, p = (l & 1) ^ (l >> 3);
                const int kc = ((rl >> 1) + (h >> 4)) % Kc;
                const int r = ((h & 15) << 3) | rl;
                const int k0 = 8 * kc + 4 * p;
                uint2 w = make_uint2(0u, 0u);
                if (r < rows) {
                    const float4 a = k0 < K1 ? *reinterpret_cast<const float4*>(x1 + 4 * (r * K1 + k0))
                                             : *reinterpret_cast<const float4*>(x2 + 4 * (r * K2 + k0 - K1));
                    w.x = (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(a.x)) |
                          ((uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(a.y)) << 16);
                    w.y = (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(a.z)) |
                          ((uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(a.w)) << 16);
                }
                *reinterpret_cast<uint2*>(sA + kc * kUmmaLboA + (h & 15) * kUmmaSbo + rl * 16 + p * 8) = w;
            }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // A -> tensor core
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        if (__syncthreads_or(!ok)) {
            bad = true;
            break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (tid == 0) {
            if (t + 2 * grid < ntiles) issue(t + 2 * grid, s);  // stage s is free again
            const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
            for (int ks = 0; ks < K / 16; ++ks) {
                const uint64_t da = umma_smem_desc(a0 + 2 * ks * kUmmaLboA, kUmmaLboA, kUmmaSbo);
                const uint64_t db = umma_smem_desc(b0 + 2 * ks * P::kLboB, P::kLboB, kUmmaSbo);
                asm volatile(
                    "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
                    "l"(da), "l"(db), "r"(P::kIdesc), "r"(ks > 0 ? 1 : 0));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar_mma)
                         : "memory");
        }
        // warp-uniform outcome: tcgen05.ld below is a .sync.aligned warp instruction
        if (!__all_sync(0xffffffffu, mbar_wait(bar_mma, (uint32_t)(i & 1), spin))) {
            bad = true;  // the next iteration's barrier takes every thread to the exit
            continue;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        // columns cb .. cb + 31 of rows 32 q .. 32 q + 31, N / 64 blocks per warp
        for (int cc = 0; cc < N / 64; ++cc) {
            const int cb = (N / 2) * half + 32 * cc;
            uint32_t v[32];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                  "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                  "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]),
                  "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]),
                  "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                : "r"(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)cb));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            // rotate the 8 four-column groups left by rot (three conditional steps)
#pragma unroll
            for (int b = 1; b < 8; b <<= 1) {
                uint32_t w[32];
#pragma unroll
                for (int e = 0; e < 32; ++e) w[e] = v[(e + 4 * b) & 31];
                if (rot & b) {
#pragma unroll
                    for (int e = 0; e < 32; ++e) v[e] = w[e];
                }
            }
            if (orow < rows) {
                uint8_t* o = sOut + orow * (N * 4) + cb * 4;
#pragma unroll
                for (int c = 0; c < 8; ++c) {
                    const int g = (c + rot) & 7;  // column group held in v[4c .. 4c + 3]
                    float w[4];
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        const float x = __uint_as_float(v[4 * c + e]) + s_bias[cb + 4 * g + e];
                        w[e] = relu ? fmaxf(x, 0.f) : x;
                    }
                    *reinterpret_cast<float4*>(o + 16 * g) = make_float4(w[0], w[1], w[2], w[3]);
                }
            }
            __syncwarp();
            // this warp's 32 x 32 block, 4 rows (4 x 128 bytes) per store instruction
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int rr = 32 * q + 4 * j + (lane >> 3);
                if (rr < rows)
                    *reinterpret_cast<float4*>(Y + (t * kUmmaM + rr) * N + cb + 4 * (lane & 7)) =
                        *reinterpret_cast<const float4*>(sOut + rr * (N * 4) + cb * 4 + 16 * (lane & 7));
            }
            __syncwarp();
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    // any warp's timeout counts (one that gave up on the last tile's MMA
    // leaves the loop without the others noticing)
    const bool any_bad = __syncthreads_or(bad);
    if (tid == 0 && any_bad) {
        // a wait timed out in iteration i: settle what is still in flight
        // (the copies of tiles i and i + 1 and the MMA of iteration i - 1)
        // with the full bound, whatever limit the loop's waits had
        atomicExch(err, 1);
        if (t < ntiles) mbar_wait(bar_full0 + 8 * (int)(i & 1), (uint32_t)((i >> 1) & 1));
        if (t + grid < ntiles) mbar_wait(bar_full0 + 8 * (int)((i + 1) & 1), (uint32_t)(((i + 1) >> 1) & 1));
        if (i > 0) mbar_wait(bar_mma, (uint32_t)((i - 1) & 1));
    }
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(N));
}

// G = dY * (Y > 0) (or dY when relu == 0)
__global__ void gnn_relu_bwd_kernel(int64_t len, const float* __restrict__ dY, const float* __restrict__ Y, int relu,
                                    float* __restrict__ G) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < len; i += (int64_t)gridDim.x * blockDim.x)
        G[i] = (!relu || Y[i] > 0.f) ? dY[i] : 0.f;
}

// ---- weight gradient on the tcgen05 tensor cores ----
// Per-CTA partial dW (K x 64) = [X1 | X2]^T G and db = column sums of G over
// the CTA's 64-row tiles (t, t + grid, ...). One MMA operand pair per tile:
// A = [X1 | X2]^T (M = 128 feature rows, the rows past K kept zero) and B =
// G^T (N = 64 outputs), both K-major over the tile's 64 rows. The tile's
// rows of X1, X2 and G arrive by bulk copies into one of three FP32 stages;
// the CTA transposes them into the BF16 operands (a thread packs 8
// consecutive rows of one column into one 16-byte core-matrix row), one
// thread issues 4 tcgen05.mma (K = 16 each) accumulating into the same 64
// TMEM columns across all of the CTA's tiles, and the next tile is staged
// once the tensor core has read the operands (an mbarrier commit per tile).
// At the end each warp reads 32 rows x 32 columns of the accumulator and
// writes its part of the CTA's partial. db is summed in FP32 by 64 threads,
// rows in order. Every wait is bounded as in the layer kernel.
constexpr int kWR = 64;                                 // rows per tile (the MMA's K extent)
constexpr int kWStages = 3;
constexpr int kWStage = kWR * (kMaxK + kH) * 4;         // 48 KB of FP32 rows
constexpr int kWOffA = kWStages * kWStage;              // 144 KB
constexpr int kWOffB = kWOffA + kUmmaM * kWR * 2;       // + 16 KB
constexpr int kWSmem = kWOffB + kH * kWR * 2;           // + 8 KB = 168 KB
constexpr uint32_t kWLboA = (kUmmaM / 8) * 128;         // 2048
constexpr uint32_t kWLboB = (kH / 8) * 128;             // 1024
constexpr uint32_t kWIdesc = UmmaPlan<kH, kMaxK>::kIdesc;  // M = 128, N = 64
static_assert(kWSmem <= 227 * 1024, "weight-gradient shared memory");

__device__ __forceinline__ int wgrad_rows(int64_t M, int64_t tile) {
    const int64_t r = M - tile * kWR;
    return (int)(r < kWR ? r : kWR);
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    return (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(lo)) |
           ((uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(hi)) << 16);
}

__global__ void __launch_bounds__(kUmmaT, 1) gnn_umma_wgrad_kernel(int64_t M, int K1, int K2,
                                                                   const float* __restrict__ X1,
                                                                   const float* __restrict__ X2,
                                                                   const float* __restrict__ G,
                                                                   float* __restrict__ part_w,
                                                                   float* __restrict__ part_b, int* err,
                                                                   uint32_t spin) {
    extern __shared__ __align__(1024) uint8_t wg_smem[];
    uint8_t* sA = wg_smem + kWOffA;
    uint8_t* sB = wg_smem + kWOffB;
    __shared__ __align__(8) uint64_t full[kWStages];
    __shared__ __align__(8) uint64_t mma_bar;
    __shared__ uint32_t s_tmem;
    const int K = K1 + K2;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int64_t ntiles = (M + kWR - 1) / kWR;
    const int64_t grid = gridDim.x;

    for (int idx = tid; idx < kUmmaM * kWR * 2 / 16; idx += kUmmaT)
        reinterpret_cast<uint4*>(sA)[idx] = make_uint4(0u, 0u, 0u, 0u);
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"(kH));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    const uint32_t bar_full0 = smem_u32(&full[0]), bar_mma = smem_u32(&mma_bar);
    const uint32_t stage0 = smem_u32(wg_smem);
    // tile t into stage s: X1 rows, then X2 rows (64 K1 floats on), then G rows (64 K floats on)
    auto issue = [&](int64_t t, int s) {
        const uint32_t rows = (uint32_t)wgrad_rows(M, t), bar = bar_full0 + 8 * s;
        const uint32_t base = stage0 + s * kWStage;
        mbar_expect(bar, rows * 4u * (uint32_t)(K + kH));
        bulk_load(base, X1 + t * kWR * K1, rows * 4u * (uint32_t)K1, bar);
        if (K2) bulk_load(base + kWR * 4 * K1, X2 + t * kWR * K2, rows * 4u * (uint32_t)K2, bar);
        bulk_load(base + kWR * 4 * K, G + t * kWR * kH, rows * 4u * (uint32_t)kH, bar);
    };
    if (tid == 0) {
        for (int p = 0; p < kWStages; ++p) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_full0 + 8 * p));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_mma));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        for (int p = 0; p < kWStages; ++p)
            if (blockIdx.x + p * grid < ntiles) issue(blockIdx.x + p * grid, p);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // zeroed A -> tensor core
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;

    float dbias = 0.f;  // column tid of db (tid < 64)
    bool bad = false;
    int64_t i = 0, t = blockIdx.x;
    for (; t < ntiles; t += grid, ++i) {
        const int s = (int)(i % kWStages);
        const int rows = wgrad_rows(M, t);
        bool ok = !bad && mbar_wait(bar_full0 + 8 * s, (uint32_t)((i / kWStages) & 1), spin);
        // the previous tile's MMAs read A and B: restage only after they completed
        if (ok && i > 0) ok = mbar_wait(bar_mma, (uint32_t)((i - 1) & 1), spin);
        if (ok) {
            const float* x1 = reinterpret_cast<const float*>(wg_smem + s * kWStage);
            const float* x2 = x1 + kWR * K1;
            const float* gs = x1 + kWR * K;
            // A[f][r] = X[r][f]: item u packs rows 8 kc .. 8 kc + 7 of column f
            for (int u = tid; u < (kWR / 8) * K; u += kUmmaT) {
                const int f = u % K, kc = u / K;
                const float* col = f < K1 ? x1 + f : x2 + (f - K1);
                const int ld = f < K1 ? K1 : K2;
                uint32_t w[4];
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int r = 8 * kc + 2 * e;
                    w[e] = pack_bf16(r < rows ? col[r * ld] : 0.f, r + 1 < rows ? col[(r + 1) * ld] : 0.f);
                }
                *reinterpret_cast<uint4*>(sA + kc * kWLboA + (f >> 3) * kUmmaSbo + (f & 7) * 16) =
                    make_uint4(w[0], w[1], w[2], w[3]);
            }
            // B[o][r] = G[r][o]
            for (int u = tid; u < (kWR / 8) * kH; u += kUmmaT) {
                const int o = u % kH, kc = u / kH;
                uint32_t w[4];
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int r = 8 * kc + 2 * e;
                    w[e] = pack_bf16(r < rows ? gs[r * kH + o] : 0.f, r + 1 < rows ? gs[(r + 1) * kH + o] : 0.f);
                }
                *reinterpret_cast<uint4*>(sB + kc * kWLboB + (o >> 3) * kUmmaSbo + (o & 7) * 16) =
                    make_uint4(w[0], w[1], w[2], w[3]);
            }
            if (tid < kH)
                for (int r = 0; r < rows; ++r) dbias += gs[r * kH + tid];
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // A, B -> tensor core
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        if (__syncthreads_or(!ok)) {
            bad = true;
            break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (tid == 0) {
            if (t + kWStages * grid < ntiles) issue(t + kWStages * grid, s);  // stage s is free again
            const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
#pragma unroll
            for (int ks = 0; ks < kWR / 16; ++ks) {
                const uint64_t da = umma_smem_desc(a0 + 2 * ks * kWLboA, kWLboA, kUmmaSbo);
                const uint64_t db = umma_smem_desc(b0 + 2 * ks * kWLboB, kWLboB, kUmmaSbo);
                asm volatile(
                    "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
                    "l"(da), "l"(db), "r"(kWIdesc), "r"((i > 0 || ks > 0) ? 1 : 0));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar_mma)
                         : "memory");
        }
    }
    // the last tile's MMAs; warp-uniform outcome (tcgen05.ld is a warp instruction)
    if (!bad && i > 0 && !__all_sync(0xffffffffu, mbar_wait(bar_mma, (uint32_t)((i - 1) & 1), spin))) bad = true;
    if (!bad) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const int q = warp & 3, half = warp >> 2;  // TMEM lanes 32q.. (rows of dW), columns 32 half..
        uint32_t v[32];
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
            "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
              "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
              "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]),
              "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]),
              "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
            : "r"(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(32 * half)));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        const int k = 32 * q + lane;
        if (k < K) {
            float* o = part_w + ((int64_t)blockIdx.x * K + k) * kH + 32 * half;
#pragma unroll
            for (int c = 0; c < 8; ++c)
                reinterpret_cast<float4*>(o)[c] = make_float4(__uint_as_float(v[4 * c]), __uint_as_float(v[4 * c + 1]),
                                                              __uint_as_float(v[4 * c + 2]),
                                                              __uint_as_float(v[4 * c + 3]));
        }
    }
    if (tid < kH) part_b[(int64_t)blockIdx.x * kH + tid] = dbias;
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    const bool any_bad = __syncthreads_or(bad);
    if (tid == 0 && any_bad) {
        // a wait timed out in iteration i (or on the last MMA): settle the
        // copies of tiles i .. i + 2 and the MMA of iteration i - 1 with the
        // full bound, whatever limit the loop's waits had
        atomicExch(err, 1);
        for (int p = 0; p < kWStages; ++p) {
            const int64_t ii = i + p;
            if (t + p * grid < ntiles)
                mbar_wait(bar_full0 + 8 * (int)(ii % kWStages), (uint32_t)((ii / kWStages) & 1));
        }
        if (i > 0) mbar_wait(bar_mma, (uint32_t)((i - 1) & 1));
    }
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kH));
}

// out[i] = sum over blocks b (in order) of part[b * len + i]
__global__ void gnn_sum_parts_kernel(int64_t nb, int64_t len, const float* __restrict__ part, float* __restrict__ out) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= len) return;
    float s = 0.f;
    for (int64_t b = 0; b < nb; ++b) s += part[b * len + i];
    out[i] = s;
}

// W (K x 64, FP32 master, row-major) -> Wt (64 x K, BF16) and Wb (K x 64, BF16)
__global__ void gnn_cast_weights_kernel(int K, const float* __restrict__ W, __nv_bfloat16* __restrict__ Wt,
                                        __nv_bfloat16* __restrict__ Wb) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= K * kH) return;
    const int k = i / kH, o = i % kH;
    const __nv_bfloat16 v = __float2bfloat16_rn(W[i]);
    Wt[o * K + k] = v;
    Wb[i] = v;
}

__global__ void gnn_adam_kernel(int64_t len, float* __restrict__ w, const float* __restrict__ g,
                                float* __restrict__ m1, float* __restrict__ m2, float lr, float b1, float b2,
                                float eps, float c1, float c2) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= len) return;
    const float gi = g[i];
    const float a = b1 * m1[i] + (1.f - b1) * gi;
    const float b = b2 * m2[i] + (1.f - b2) * gi * gi;
    m1[i] = a;
    m2[i] = b;
    w[i] -= lr * (a / c1) / (sqrtf(b / c2) + eps);
}

// Timeout flag of the tcgen05 kernels: one word of the stream's workspace
// (select word 7, which the pricing kernels do not use), read and cleared by
// hn_gnn_check.
int* umma_flag(cudaStream_t s) { return reinterpret_cast<int*>(workspace(s).select + 7); }

// Poll limit of the tcgen05 kernels' pipeline waits (hn_gnn_set_wait_limit).
std::atomic<uint32_t> g_umma_spin{kUmmaSpin};

// Raise a kernel's dynamic shared-memory limit once per device.
template <typename F>
void smem_attribute(F* kernel, int bytes, int& done_device, const char* what) {
    if (done_device != ctx().device) {
        check_cuda(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes), what);
        done_device = ctx().device;
    }
}

// The tcgen05 layer kernel, one persistent CTA per SM (at most one per tile).
template <int N, int KMAX>
void launch_umma(int64_t M, int K1, int K2, const float* X1, const float* X2, const __nv_bfloat16* Bt,
                 const float* bias, int relu, float* Y, cudaStream_t s) {
    using P = UmmaPlan<N, KMAX>;
    static int attr_device = -1;
    smem_attribute(gnn_umma_kernel<N, KMAX>, P::kSmem, attr_device, "umma smem attribute");
    const int64_t tiles = (M + kUmmaM - 1) / kUmmaM;
    gnn_umma_kernel<N, KMAX><<<(unsigned)std::min<int64_t>(tiles, ctx().sm_count), kUmmaT, P::kSmem, s>>>(
        M, K1, K2, X1, X2, Bt, bias, relu, Y, umma_flag(s), g_umma_spin.load());
    launched("gnn_umma_kernel");
}

bool misaligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) != 0; }

}  // namespace
}  // namespace hn

using namespace hn;

extern "C" {

int hn_gnn_spmm(const hn_csr* A, int trans, const float* H, float* out, int accumulate, void* stream) {
    return guard("hn_gnn_spmm", [&] {
        require_init();
        if (!A || !H || !out) fail(HN_ERR_INVALID_ARG, "null argument");
        if (trans && !A->has_t) fail(HN_ERR_INVALID_ARG, "matrix was created without its transpose");
        const int rows = (int)(trans ? A->n : A->m);
        if (rows == 0) return;
        const int32_t* rp = trans ? A->rpT : A->rp;
        const int32_t* ci = trans ? A->ciT : A->ci;
        const double* val = trans ? A->valT : A->val;
        gnn_spmm_kernel<<<(unsigned)((rows * 32LL + 255) / 256), 256, 0, as_stream(stream)>>>(rows, rp, ci, val, H,
                                                                                            accumulate, out);
        launched("gnn_spmm_kernel");
    });
}

int hn_gnn_cast_weights(int K, const float* W, void* Wt_bf16, void* Wb_bf16, void* stream) {
    return guard("hn_gnn_cast_weights", [&] {
        require_init();
        if (K <= 0 || K > kMaxK || !W || !Wt_bf16 || !Wb_bf16) fail(HN_ERR_INVALID_ARG, "bad arguments");
        gnn_cast_weights_kernel<<<(K * kH + 255) / 256, 256, 0, as_stream(stream)>>>(
            K, W, static_cast<__nv_bfloat16*>(Wt_bf16), static_cast<__nv_bfloat16*>(Wb_bf16));
        launched("gnn_cast_weights_kernel");
    });
}

int hn_gnn_linear(int64_t M, int K1, int K2, const float* X1, const float* X2, const void* Wt_bf16, int N,
                  const float* bias, int relu, float* Y, void* stream) {
    return guard("hn_gnn_linear", [&] {
        require_init();
        const int K = K1 + K2;
        if (M < 0 || K1 <= 0 || K2 < 0 || K > kMaxK || K1 % 16 || K2 % 16 || !X1 || (K2 && !X2) || !Wt_bf16 ||
            !Y || (N != 64 && N != 128))
            fail(HN_ERR_INVALID_ARG, "bad arguments (K1, K2 multiples of 16, K1 + K2 <= 128, N 64 or 128)");
        if (M == 0) return;
        const unsigned grid = (unsigned)((M + kRowsPerCta - 1) / kRowsPerCta);
        const auto* B = static_cast<const __nv_bfloat16*>(Wt_bf16);
        if (N == 64) {
            gnn_gemm_kernel<64, kMaxK><<<grid, kGT, 0, as_stream(stream)>>>(M, K1, K2, X1, X2, B, bias, relu, Y);
        } else {
            if (K > 64) fail(HN_ERR_INVALID_ARG, "N = 128 takes K1 + K2 <= 64");
            gnn_gemm_kernel<128, 64><<<grid, kGT, 0, as_stream(stream)>>>(M, K1, K2, X1, X2, B, bias, relu, Y);
        }
        launched("gnn_gemm_kernel");
    });
}

int hn_gnn_linear_umma(int64_t M, int K1, int K2, const float* X1, const float* X2, const void* Wt_bf16,
                       const float* bias, int relu, float* Y, void* stream) {
    return guard("hn_gnn_linear_umma", [&] {
        require_init();
        const int K = K1 + K2;
        if (M < 0 || K1 <= 0 || K2 < 0 || K > kMaxK || K1 % 16 || K2 % 16 || !X1 || (K2 && !X2) || !Wt_bf16 || !Y)
            fail(HN_ERR_INVALID_ARG, "bad arguments (K1, K2 multiples of 16, K1 + K2 <= 128)");
        if (misaligned16(X1) || (K2 && misaligned16(X2)) || misaligned16(Y) || misaligned16(Wt_bf16))
            fail(HN_ERR_INVALID_ARG, "X1, X2, Y and the weights must be 16-byte aligned (bulk copies)");
        if (M == 0) return;
        launch_umma<kH, kMaxK>(M, K1, K2, X1, X2, static_cast<const __nv_bfloat16*>(Wt_bf16), bias, relu, Y,
                               as_stream(stream));
    });
}

int hn_gnn_set_wait_limit(uint32_t polls) {
    g_umma_spin.store(polls == 0 ? kUmmaSpin : polls);
    return HN_OK;
}

int hn_gnn_check(void* stream) {
    return guard("hn_gnn_check", [&] {
        require_init();
        cudaStream_t s = as_stream(stream);
        int* f = umma_flag(s);
        int h = 0;
        check_cuda(cudaMemcpyAsync(&h, f, sizeof(int), cudaMemcpyDeviceToHost, s), "D2H flag");
        check_cuda(cudaMemsetAsync(f, 0, sizeof(int), s), "memset flag");
        check_cuda(cudaStreamSynchronize(s), "flag sync");
        if (h) fail(HN_ERR_CUDA, "tensor-core layer: an MMA completion wait timed out");
    });
}

int hn_gnn_linear_bwd(int64_t M, int K1, int K2, const float* X1, const float* X2, const void* Wb_bf16,
                      const float* Y, const float* dY, int relu, float* G, float* dX, float* dW, float* db,
                      float* scratch, int64_t scratch_floats, void* stream) {
    return guard("hn_gnn_linear_bwd", [&] {
        require_init();
        const int K = K1 + K2;
        if (M < 0 || K1 <= 0 || K2 < 0 || K > kMaxK || K1 % 16 || K2 % 16 || !X1 || (K2 && !X2) || !Y || !dY ||
            !G || !dW || !db || !scratch)
            fail(HN_ERR_INVALID_ARG, "bad arguments");
        if (misaligned16(X1) || (K2 && misaligned16(X2)) || misaligned16(G) || (dX && misaligned16(dX)) ||
            misaligned16(Wb_bf16) || misaligned16(scratch))
            fail(HN_ERR_INVALID_ARG, "X1, X2, G, dX, the weights and the scratch must be 16-byte aligned");
        cudaStream_t s = as_stream(stream);
        const int64_t nb = std::max<int64_t>(1, std::min<int64_t>((M + kWR - 1) / kWR, ctx().sm_count));
        if (scratch_floats < nb * (int64_t)(kH * K + kH)) fail(HN_ERR_INVALID_ARG, "scratch too small");
        const int64_t len = M * kH;
        if (len > 0) {
            gnn_relu_bwd_kernel<<<(unsigned)std::min<int64_t>((len + 255) / 256, 148 * 16), 256, 0, s>>>(len, dY, Y,
                                                                                                     relu, G);
            launched("gnn_relu_bwd_kernel");
        }
        // dX = G W^T on the tcgen05 layer kernel: input G (M x 64), N = K
        // outputs, B = W (K x 64 row-major BF16), no bias, no activation
        if (dX && M > 0) {
            if (K != 64 && K != 128) fail(HN_ERR_INVALID_ARG, "dX needs K1 + K2 of 64 or 128");
            const auto* B = static_cast<const __nv_bfloat16*>(Wb_bf16);
            if (K == 64)
                launch_umma<64, kH>(M, kH, 0, G, nullptr, B, nullptr, 0, dX, s);
            else
                launch_umma<128, kH>(M, kH, 0, G, nullptr, B, nullptr, 0, dX, s);
        }
        float* pw = scratch;
        float* pb = scratch + nb * kH * K;
        if (M > 0) {
            static int attr_device = -1;
            smem_attribute(gnn_umma_wgrad_kernel, kWSmem, attr_device, "wgrad smem attribute");
            gnn_umma_wgrad_kernel<<<(unsigned)nb, kUmmaT, kWSmem, s>>>(M, K1, K2, X1, X2, G, pw, pb, umma_flag(s),
                                                                        g_umma_spin.load());
            launched("gnn_umma_wgrad_kernel");
        } else {
            check_cuda(cudaMemsetAsync(scratch, 0, sizeof(float) * (kH * K + kH), s), "memset");
        }
        gnn_sum_parts_kernel<<<(unsigned)((kH * K + 255) / 256), 256, 0, s>>>(nb, (int64_t)kH * K, pw, dW);
        launched("gnn_sum_parts_kernel");
        gnn_sum_parts_kernel<<<1, kH, 0, s>>>(nb, kH, pb, db);
        launched("gnn_sum_parts_kernel");
    });
}

int hn_gnn_split_grad(int64_t M, const float* dX, float* dH, float* dAgg, void* stream) {
    return guard("hn_gnn_split_grad", [&] {
        require_init();
        if (M < 0 || (M && (!dX || !dH || !dAgg))) fail(HN_ERR_INVALID_ARG, "bad arguments");
        if (M == 0) return;
        gnn_split_grad_kernel<<<(unsigned)((M * kH + 255) / 256), 256, 0, as_stream(stream)>>>(M, dX, dH, dAgg);
        launched("gnn_split_grad_kernel");
    });
}

int hn_gnn_head_grad(int64_t M, const float* O, const float* T, int nt, float scale, float* dO, float* loss_part,
                     int64_t nparts, void* stream) {
    return guard("hn_gnn_head_grad", [&] {
        require_init();
        if (M < 0 || nt < 1 || nt > 2 || nparts < 1 || (M && (!O || !T || !dO)) || !loss_part)
            fail(HN_ERR_INVALID_ARG, "bad arguments");
        const int grid = (int)std::min<int64_t>(nparts, std::max<int64_t>(1, (M * kH + 255) / 256));
        gnn_head_grad_kernel<<<grid, 256, 0, as_stream(stream)>>>(M, O, T, nt, scale, dO, loss_part);
        launched("gnn_head_grad_kernel");
        if (grid < nparts)
            check_cuda(cudaMemsetAsync(loss_part + grid, 0, sizeof(float) * (nparts - grid), as_stream(stream)),
                       "memset");
    });
}

int hn_gnn_adam(int64_t len, float* w, const float* g, float* m1, float* m2, float lr, float beta1, float beta2,
                float eps, int64_t step, void* stream) {
    return guard("hn_gnn_adam", [&] {
        require_init();
        if (len < 0 || step < 1 || (len && (!w || !g || !m1 || !m2))) fail(HN_ERR_INVALID_ARG, "bad arguments");
        if (len == 0) return;
        const float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
        gnn_adam_kernel<<<(unsigned)((len + 255) / 256), 256, 0, as_stream(stream)>>>(len, w, g, m1, m2, lr, beta1,
                                                                                      beta2, eps, c1, c2);
        launched("gnn_adam_kernel");
    });
}

}  // extern "C"
