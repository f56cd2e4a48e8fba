// Kernels of the bipartite variable-constraint GNN that predicts an IPM warm
// start (no counterpart in the reference). Hidden width 64 throughout.
//
//   hn_gnn_spmm          out = A H or A^T H, H row-major rows x 64 (FP32),
//                        A's FP64 values rounded to FP32; each output row is a
//                        sequential sum over its row of A (deterministic)
//   hn_gnn_linear        Y = act([X1 | X2] W + b): BF16 operands on the tensor
//                        cores (mma.sync m16n8k16, FP32 accumulation)
//   hn_gnn_linear_bwd    G = dY * relu'(Y); dX = G W^T (tensor cores);
//                        dW = [X1 | X2]^T G and db = sum G per CTA partials,
//                        then summed in a fixed order (deterministic)
//   hn_gnn_adam          Adam step on FP32 master weights
//
// BF16 rounding is round-to-nearest-even of the FP32 operand
// (__float2bfloat16_rn), applied when a tile is staged into shared memory.
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
// One CTA (4 warps) computes a 128-row x 64-column tile of Y with K <= 128:
// both operands are staged in shared memory in the canonical K-major,
// no-swizzle layout (core matrices of 8 rows x 16 bytes; the next 8-row
// group 128 bytes on, the next 8-element K chunk LBO bytes on), one thread
// issues K / 16 tcgen05.mma (kind::f16, BF16 in, FP32 accumulated in 64
// TMEM columns), a commit signals an mbarrier, and each warp reads its 32
// rows back with tcgen05.ld for the bias/ReLU epilogue. The mbarrier wait is
// bounded: on a timeout the kernel records it in *err and still frees TMEM.
constexpr int kUmmaM = 128;
constexpr uint32_t kUmmaSbo = 128;
constexpr uint32_t kUmmaLboA = (kUmmaM / 8) * 128;  // 2048
constexpr uint32_t kUmmaLboB = (kH / 8) * 128;      // 1024
constexpr uint32_t kUmmaSpin = 1u << 24;
constexpr int kUmmaSmem = (kUmmaM + kH) * kMaxK * 2;  // 48 KB dynamic

__device__ __forceinline__ uint64_t umma_smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    // start address, leading and stride byte offsets (16-byte units), version 1, no swizzle
    return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | ((uint64_t)1 << 46);
}
// kind::f16 instruction descriptor: F32 accumulator, BF16 A and B, both K-major
constexpr uint32_t kUmmaIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kH >> 3) << 17) |
                                ((uint32_t)(kUmmaM >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__global__ void __launch_bounds__(128) gnn_umma_kernel(int64_t M, int K1, int K2, const float* __restrict__ X1,
                                                      const float* __restrict__ X2,
                                                      const __nv_bfloat16* __restrict__ Bt,
                                                      const float* __restrict__ bias, int relu,
                                                      float* __restrict__ Y, int* err) {
    extern __shared__ __align__(1024) uint8_t umma_smem[];
    uint8_t* sA = umma_smem;                        // 128 x K BF16, 32 KB at K = 128
    uint8_t* sB = umma_smem + kUmmaM * kMaxK * 2;   // 64 x K BF16, 16 KB
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t s_tmem;
    const int K = K1 + K2, tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int64_t row0 = blockIdx.x * (int64_t)kUmmaM;
    // operands: 8 consecutive K elements (16 bytes) per store
    for (int idx = tid; idx < kUmmaM * (K / 8); idx += 128) {
        const int r = idx / (K / 8), kc = idx % (K / 8);
        const int64_t gr = row0 + r;
        float v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) v[u] = 0.f;
        if (gr < M) {
            const int k = kc * 8;
            const float* src = k < K1 ? X1 + gr * K1 + k : X2 + gr * K2 + (k - K1);
#pragma unroll
            for (int u = 0; u < 8; ++u) v[u] = src[u];
        }
        uint32_t w[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const __nv_bfloat16 lo = __float2bfloat16_rn(v[2 * u]), hi = __float2bfloat16_rn(v[2 * u + 1]);
            w[u] = (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
        }
        *reinterpret_cast<uint4*>(sA + kc * kUmmaLboA + (r >> 3) * kUmmaSbo + (r & 7) * 16) =
            make_uint4(w[0], w[1], w[2], w[3]);
    }
    for (int idx = tid; idx < kH * (K / 8); idx += 128) {
        const int n = idx / (K / 8), kc = idx % (K / 8);
        *reinterpret_cast<uint4*>(sB + kc * kUmmaLboB + (n >> 3) * kUmmaSbo + (n & 7) * 16) =
            *reinterpret_cast<const uint4*>(Bt + (int64_t)n * K + kc * 8);
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"(kH));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // staged operands -> tensor core
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;
    if (tid == 0) {
        const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
        for (int ks = 0; ks < K / 16; ++ks) {
            const uint64_t da = umma_smem_desc(a0 + 2 * ks * kUmmaLboA, kUmmaLboA, kUmmaSbo);
            const uint64_t db = umma_smem_desc(b0 + 2 * ks * kUmmaLboB, kUmmaLboB, kUmmaSbo);
            asm volatile(
                "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
                "l"(da), "l"(db), "r"(kUmmaIdesc), "r"(ks > 0 ? 1 : 0));
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         smem_u32(&mbar))
                     : "memory");
    }
    uint32_t done = 0;
    for (uint32_t it = 0; it < kUmmaSpin && !done; ++it) {
        asm volatile(
            "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}\n"
            : "=r"(done)
            : "r"(smem_u32(&mbar)), "r"(0u)
            : "memory");
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (!done) {
        if (lane == 0) atomicExch(err, 1);
    } else {
        uint32_t r[64];
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x64.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
            "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32,%33,%34,%35,%36,%37,%38,%39,"
            "%40,%41,%42,%43,%44,%45,%46,%47,%48,%49,%50,%51,%52,%53,%54,%55,%56,%57,%58,%59,%60,%61,%62,%63},"
            " [%64];"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
              "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
              "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
              "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
              "=r"(r[29]), "=r"(r[30]), "=r"(r[31]), "=r"(r[32]), "=r"(r[33]), "=r"(r[34]), "=r"(r[35]),
              "=r"(r[36]), "=r"(r[37]), "=r"(r[38]), "=r"(r[39]), "=r"(r[40]), "=r"(r[41]), "=r"(r[42]),
              "=r"(r[43]), "=r"(r[44]), "=r"(r[45]), "=r"(r[46]), "=r"(r[47]), "=r"(r[48]), "=r"(r[49]),
              "=r"(r[50]), "=r"(r[51]), "=r"(r[52]), "=r"(r[53]), "=r"(r[54]), "=r"(r[55]), "=r"(r[56]),
              "=r"(r[57]), "=r"(r[58]), "=r"(r[59]), "=r"(r[60]), "=r"(r[61]), "=r"(r[62]), "=r"(r[63])
            : "r"(tmem + ((uint32_t)(warp * 32) << 16)));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        const int64_t gr = row0 + warp * 32 + lane;  // TMEM lane = row of the tile
        if (gr < M) {
            float4* out = reinterpret_cast<float4*>(Y + gr * kH);
#pragma unroll
            for (int c = 0; c < kH; c += 4) {
                float v[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    float t = __uint_as_float(r[c + u]) + (bias ? bias[c + u] : 0.f);
                    v[u] = relu ? fmaxf(t, 0.f) : t;
                }
                out[c / 4] = make_float4(v[0], v[1], v[2], v[3]);
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kH));
}

// G = dY * (Y > 0) (or dY when relu == 0)
__global__ void gnn_relu_bwd_kernel(int64_t len, const float* __restrict__ dY, const float* __restrict__ Y, int relu,
                                    float* __restrict__ G) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < len; i += (int64_t)gridDim.x * blockDim.x)
        G[i] = (!relu || Y[i] > 0.f) ? dY[i] : 0.f;
}

// Per-CTA partial dW (K x 64) = [X1 | X2]_chunk^T G_chunk over kWRows rows
// and partial db (64). Tensor cores with A = G^T (rows = the 64 outputs,
// reduction over the chunk's rows) and B = [X1 | X2] (columns = K).
constexpr int kWRows = 64;
__global__ void __launch_bounds__(kGT) gnn_wgrad_kernel(int64_t M, int K1, int K2, const float* __restrict__ X1,
                                                        const float* __restrict__ X2, const float* __restrict__ G,
                                                        float* __restrict__ part_w, float* __restrict__ part_b) {
    constexpr int RP = kWRows + 8;
    __shared__ __align__(16) __nv_bfloat16 sGt[kH][RP];     // [output o][row]
    __shared__ __align__(16) __nv_bfloat16 sXt[kMaxK][RP];  // [input k][row]
    const int K = K1 + K2;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int g = lane >> 2, t = lane & 3;
    const int64_t row0 = blockIdx.x * (int64_t)kWRows;
    for (int idx = tid; idx < kWRows * kH; idx += kGT) {
        const int r = idx / kH, o = idx % kH;
        const int64_t gr = row0 + r;
        sGt[o][r] = __float2bfloat16_rn(gr < M ? G[gr * kH + o] : 0.f);
    }
    for (int idx = tid; idx < kWRows * K; idx += kGT) {
        const int r = idx / K, k = idx % K;
        const int64_t gr = row0 + r;
        float v = 0.f;
        if (gr < M) v = k < K1 ? X1[gr * K1 + k] : X2[gr * K2 + (k - K1)];
        sXt[k][r] = __float2bfloat16_rn(v);
    }
    __syncthreads();
    // bias partial: FP32 sum of G over the chunk, rows in order
    if (tid < kH) {
        float s = 0.f;
        for (int r = 0; r < kWRows; ++r) {
            const int64_t gr = row0 + r;
            if (gr < M) s += G[gr * kH + tid];
        }
        part_b[(int64_t)blockIdx.x * kH + tid] = s;
    }
    // warp w: outputs o in [16w, 16w + 16), all K columns in 8-wide tiles
    const int ob = warp * 16;
    for (int n0 = 0; n0 < K; n0 += 8) {
        float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int k0 = 0; k0 < kWRows; k0 += 16) {
            uint32_t a[4], b[2];
            a[0] = *reinterpret_cast<const uint32_t*>(&sGt[ob + g][k0 + 2 * t]);
            a[1] = *reinterpret_cast<const uint32_t*>(&sGt[ob + g + 8][k0 + 2 * t]);
            a[2] = *reinterpret_cast<const uint32_t*>(&sGt[ob + g][k0 + 2 * t + 8]);
            a[3] = *reinterpret_cast<const uint32_t*>(&sGt[ob + g + 8][k0 + 2 * t + 8]);
            b[0] = *reinterpret_cast<const uint32_t*>(&sXt[n0 + g][k0 + 2 * t]);
            b[1] = *reinterpret_cast<const uint32_t*>(&sXt[n0 + g][k0 + 2 * t + 8]);
            mma_bf16(acc, a, b);
        }
        // dW[k][o] (the weights' K x 64 layout)
        float* pw = part_w + (int64_t)blockIdx.x * kH * K;
        const int c = n0 + 2 * t;
        pw[c * kH + ob + g] = acc[0];
        pw[(c + 1) * kH + ob + g] = acc[1];
        pw[c * kH + ob + g + 8] = acc[2];
        pw[(c + 1) * kH + ob + g + 8] = acc[3];
    }
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

// Timeout flag of the tcgen05 layer: one word of the stream's workspace
// (select word 7, which the pricing kernels do not use), read and cleared by
// hn_gnn_check.
int* umma_flag(cudaStream_t s) { return reinterpret_cast<int*>(workspace(s).select + 7); }

int hn_gnn_linear_umma(int64_t M, int K1, int K2, const float* X1, const float* X2, const void* Wt_bf16,
                       const float* bias, int relu, float* Y, void* stream) {
    return guard("hn_gnn_linear_umma", [&] {
        require_init();
        const int K = K1 + K2;
        if (M < 0 || K1 <= 0 || K2 < 0 || K > kMaxK || K1 % 16 || K2 % 16 || !X1 || (K2 && !X2) || !Wt_bf16 || !Y)
            fail(HN_ERR_INVALID_ARG, "bad arguments (K1, K2 multiples of 16, K1 + K2 <= 128)");
        if (M == 0) return;
        cudaStream_t s = as_stream(stream);
        static int attr_device = -1;
        if (attr_device != ctx().device) {
            check_cuda(cudaFuncSetAttribute(gnn_umma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kUmmaSmem),
                       "umma smem attribute");
            attr_device = ctx().device;
        }
        gnn_umma_kernel<<<(unsigned)((M + kUmmaM - 1) / kUmmaM), 128, kUmmaSmem, s>>>(
            M, K1, K2, X1, X2, static_cast<const __nv_bfloat16*>(Wt_bf16), bias, relu, Y, umma_flag(s));
        launched("gnn_umma_kernel");
    });
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
        cudaStream_t s = as_stream(stream);
        const int64_t nb = std::max<int64_t>(1, (M + kWRows - 1) / kWRows);
        if (scratch_floats < nb * (int64_t)(kH * K + kH)) fail(HN_ERR_INVALID_ARG, "scratch too small");
        const int64_t len = M * kH;
        if (len > 0) {
            gnn_relu_bwd_kernel<<<(unsigned)std::min<int64_t>((len + 255) / 256, 148 * 16), 256, 0, s>>>(len, dY, Y,
                                                                                                     relu, G);
            launched("gnn_relu_bwd_kernel");
        }
        // dX = G W^T: N = K columns, B^T = W (K x 64 row-major BF16)
        if (dX && M > 0) {
            if (K != 64 && K != 128) fail(HN_ERR_INVALID_ARG, "dX needs K1 + K2 of 64 or 128");
            const unsigned grid = (unsigned)((M + kRowsPerCta - 1) / kRowsPerCta);
            const auto* B = static_cast<const __nv_bfloat16*>(Wb_bf16);
            if (K == 64) {
                gnn_gemm_kernel<64, 64><<<grid, kGT, 0, s>>>(M, kH, 0, G, nullptr, B, nullptr, 0, dX);
            } else {
                gnn_gemm_kernel<128, 64><<<grid, kGT, 0, s>>>(M, kH, 0, G, nullptr, B, nullptr, 0, dX);
            }
            launched("gnn_gemm_kernel");
        }
        float* pw = scratch;
        float* pb = scratch + nb * kH * K;
        if (M > 0) {
            gnn_wgrad_kernel<<<(unsigned)nb, kGT, 0, s>>>(M, K1, K2, X1, X2, G, pw, pb);
            launched("gnn_wgrad_kernel");
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
