// fd2_sg_gemm.cuh -- BF16 tensor-core GEMM for the surrogate MLP.
//
// C[M x N] = sum_k A(m, k) B(k, n), BF16 operands, FP32 accumulation, with
// the epilogues the MLP needs (bias + ReLU to BF16, bias to FP32, ReLU-mask
// of an incoming gradient to BF16, FP32 split-K partials).  Operands are
// row-major matrices addressed either with the contraction index
// contiguous (A as [M][K], B as [N][K]) or with the output index contiguous
// (A as [K][M], B as [K][N]); the second form is read with ldmatrix.trans,
// so forward, input-gradient and weight-gradient products all run on the
// same kernel without transposing anything in memory.
//
// Tiles: 64 x 64 x 32 per CTA, four warps of 32 x 32, mma.sync m16n8k16.
// M and N may be ragged (zero-filled loads, guarded stores); K must be a
// multiple of 32 and every row stride a multiple of 8 elements (16-byte
// loads).  An optional device pointer caps M at run time (rows beyond it
// are skipped), for batches whose size is known only on the device.
#pragma once

#include <cuda_bf16.h>
#include <cstdint>

namespace fd2 {
namespace sg {

constexpr int kBM = 64, kBN = 64, kBK = 32;
constexpr int kGemmThreads = 128;

enum Epilogue : int {
    kEpiBiasReluBf16 = 0,  // out_bf16 = relu(acc + bias[n])
    kEpiBiasF32 = 1,       // out_f32  = acc + bias[n]
    kEpiMaskBf16 = 2,      // out_bf16 = acc * (mask_bf16[m][n] > 0)
    kEpiPartialF32 = 3     // out_f32[z][m][n] = acc (split-K partial of slice z)
};

struct GemmArgs {
    const __nv_bfloat16 *A;
    const __nv_bfloat16 *B;
    int lda, ldb;          // row strides (elements) of the stored matrices
    int M, N, K;
    const int *m_limit;    // optional: rows >= *m_limit are skipped
    int k_per_split;       // contraction length per blockIdx.z slice (multiple of kBK)
    int epi;
    const float *bias;     // [N]
    const __nv_bfloat16 *mask;  // [M][ldm]
    int ldm;
    void *C;
    int ldc;
    long long split_stride;  // elements between split-K partial planes
};

// Shared-memory tiles, padded so that the 8 row addresses of every ldmatrix
// phase fall in distinct 16-byte bank groups.
constexpr int kPadKC = kBK + 8;  // [rows][k] tiles: 40 elements (80 bytes) per row
constexpr int kPadMC = kBM + 8;  // [k][rows] tiles: 72 elements (144 bytes) per row

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void ldsm_x4(uint32_t addr, uint32_t &r0, uint32_t &r1, uint32_t &r2, uint32_t &r3)
{
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0, %1, %2, %3}, [%4];\n"
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
                 : "r"(addr));
}

__device__ __forceinline__ void ldsm_x4_t(uint32_t addr, uint32_t &r0, uint32_t &r1, uint32_t &r2, uint32_t &r3)
{
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0, %1, %2, %3}, [%4];\n"
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
                 : "r"(addr));
}

__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1)
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
        "{%0, %1, %2, %3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// kAK: A stored [M][K] (true) or [K][M] (false); kBK_: B stored [N][K]
// (true) or [K][N] (false).
template <bool kAK, bool kBKc>
__global__ void __launch_bounds__(kGemmThreads) gemm_kernel(const GemmArgs g)
{
    // A tile: [kBM][kPadKC] or [kBK][kPadMC]; B tile likewise with kBN.
    __shared__ __align__(16) __nv_bfloat16 sA[kAK ? kBM * kPadKC : kBK * kPadMC];
    __shared__ __align__(16) __nv_bfloat16 sB[kBKc ? kBN * kPadKC : kBK * kPadMC];

    const int m0 = blockIdx.y * kBM, n0 = blockIdx.x * kBN;
    const int M = g.m_limit ? min(g.M, *g.m_limit) : g.M;
    if (m0 >= M) return;
    const int N = g.N;
    const int k_begin = blockIdx.z * g.k_per_split;
    const int k_end = min(g.K, k_begin + g.k_per_split);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;

    float acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int r = 0; r < 4; ++r) acc[i][j][r] = 0.0f;

    const uint4 zero = make_uint4(0, 0, 0, 0);
    for (int k0 = k_begin; k0 < k_end; k0 += kBK) {
        // ---- global -> shared (16-byte vectors, zero-filled outside M / N)
        if (kAK) {
            // 64 rows x 32 k = 256 vectors of 8
            for (int v = tid; v < kBM * kBK / 8; v += kGemmThreads) {
                const int r = v >> 2, c = (v & 3) * 8;
                const int m = m0 + r;
                uint4 val = zero;
                if (m < M) val = *reinterpret_cast<const uint4 *>(g.A + (long long)m * g.lda + k0 + c);
                *reinterpret_cast<uint4 *>(&sA[r * kPadKC + c]) = val;
            }
        } else {
            // 32 k-rows x 64 m = 256 vectors of 8
            for (int v = tid; v < kBK * kBM / 8; v += kGemmThreads) {
                const int r = v >> 3, c = (v & 7) * 8;
                const int m = m0 + c;
                uint4 val = zero;
                if (m + 8 <= M) {
                    val = *reinterpret_cast<const uint4 *>(g.A + (long long)(k0 + r) * g.lda + m);
                } else if (m < M) {
                    __align__(16) __nv_bfloat16 tmp[8];
                    for (int e = 0; e < 8; ++e)
                        tmp[e] = (m + e < M) ? g.A[(long long)(k0 + r) * g.lda + m + e] : __float2bfloat16(0.0f);
                    val = *reinterpret_cast<const uint4 *>(tmp);
                }
                *reinterpret_cast<uint4 *>(&sA[r * kPadMC + c]) = val;
            }
        }
        if (kBKc) {
            for (int v = tid; v < kBN * kBK / 8; v += kGemmThreads) {
                const int r = v >> 2, c = (v & 3) * 8;
                const int n = n0 + r;
                uint4 val = zero;
                if (n < N) val = *reinterpret_cast<const uint4 *>(g.B + (long long)n * g.ldb + k0 + c);
                *reinterpret_cast<uint4 *>(&sB[r * kPadKC + c]) = val;
            }
        } else {
            for (int v = tid; v < kBK * kBN / 8; v += kGemmThreads) {
                const int r = v >> 3, c = (v & 7) * 8;
                const int n = n0 + c;
                uint4 val = zero;
                if (n + 8 <= N) {
                    val = *reinterpret_cast<const uint4 *>(g.B + (long long)(k0 + r) * g.ldb + n);
                } else if (n < N) {
                    __align__(16) __nv_bfloat16 tmp[8];
                    for (int e = 0; e < 8; ++e)
                        tmp[e] = (n + e < N) ? g.B[(long long)(k0 + r) * g.ldb + n + e] : __float2bfloat16(0.0f);
                    val = *reinterpret_cast<const uint4 *>(tmp);
                }
                *reinterpret_cast<uint4 *>(&sB[r * kPadMC + c]) = val;
            }
        }
        __syncthreads();

#pragma unroll
        for (int kk = 0; kk < kBK; kk += 16) {
            uint32_t af[2][4];
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                const int mb = wm + i * 16;
                if (kAK) {
                    // matrices: (m 0-7, k 0-7), (m 8-15, k 0-7), (m 0-7, k 8-15), (m 8-15, k 8-15)
                    const int row = mb + (lane & 15), col = kk + (lane >> 4) * 8;
                    ldsm_x4(smem_u32(&sA[row * kPadKC + col]), af[i][0], af[i][1], af[i][2], af[i][3]);
                } else {
                    // stored [k][m]; transposed loads of the same four matrices
                    const int krow = kk + (lane & 7) + (lane >> 4) * 8, col = mb + ((lane >> 3) & 1) * 8;
                    ldsm_x4_t(smem_u32(&sA[krow * kPadMC + col]), af[i][0], af[i][1], af[i][2], af[i][3]);
                }
            }
#pragma unroll
            for (int j2 = 0; j2 < 2; ++j2) {
                const int nb = wn + j2 * 16;
                uint32_t b0, b1, b2, b3;  // (b0, b1): n-block nb; (b2, b3): nb + 8
                if (kBKc) {
                    // matrices: (n 0-7, k 0-7), (n 0-7, k 8-15), (n 8-15, k 0-7), (n 8-15, k 8-15)
                    const int row = nb + (lane & 7) + (lane >> 4) * 8, col = kk + ((lane >> 3) & 1) * 8;
                    ldsm_x4(smem_u32(&sB[row * kPadKC + col]), b0, b1, b2, b3);
                } else {
                    // stored [k][n]: (k 0-7, n 0-7), (k 8-15, n 0-7), (k 0-7, n 8-15), (k 8-15, n 8-15)
                    const int krow = kk + (lane & 7) + ((lane >> 3) & 1) * 8, col = nb + (lane >> 4) * 8;
                    ldsm_x4_t(smem_u32(&sB[krow * kPadMC + col]), b0, b1, b2, b3);
                }
#pragma unroll
                for (int i = 0; i < 2; ++i) {
                    mma_bf16(acc[i][j2 * 2 + 0], af[i], b0, b1);
                    mma_bf16(acc[i][j2 * 2 + 1], af[i], b2, b3);
                }
            }
        }
        __syncthreads();
    }

    // ---- epilogue: fragment (i, j) covers rows wm + 16i + {g, g + 8},
    // columns wn + 8j + {2t, 2t + 1}
    const int gq = lane >> 2, tq = lane & 3;
#pragma unroll
    for (int i = 0; i < 2; ++i) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int m = m0 + wm + i * 16 + gq + h * 8;
                const int n = n0 + wn + j * 8 + tq * 2;
                if (m >= M) continue;
                float v0 = acc[i][j][h * 2 + 0], v1 = acc[i][j][h * 2 + 1];
                const bool ok0 = n < N, ok1 = n + 1 < N;
                if (g.epi == kEpiBiasReluBf16) {
                    __nv_bfloat16 *C = reinterpret_cast<__nv_bfloat16 *>(g.C) + (long long)m * g.ldc;
                    if (ok0) C[n] = __float2bfloat16(fmaxf(v0 + g.bias[n], 0.0f));
                    if (ok1) C[n + 1] = __float2bfloat16(fmaxf(v1 + g.bias[n + 1], 0.0f));
                } else if (g.epi == kEpiBiasF32) {
                    float *C = reinterpret_cast<float *>(g.C) + (long long)m * g.ldc;
                    if (ok0) C[n] = v0 + g.bias[n];
                    if (ok1) C[n + 1] = v1 + g.bias[n + 1];
                } else if (g.epi == kEpiMaskBf16) {
                    __nv_bfloat16 *C = reinterpret_cast<__nv_bfloat16 *>(g.C) + (long long)m * g.ldc;
                    const __nv_bfloat16 *Mk = g.mask + (long long)m * g.ldm;
                    if (ok0) C[n] = __float2bfloat16(__bfloat162float(Mk[n]) > 0.0f ? v0 : 0.0f);
                    if (ok1) C[n + 1] = __float2bfloat16(__bfloat162float(Mk[n + 1]) > 0.0f ? v1 : 0.0f);
                } else {
                    float *C = reinterpret_cast<float *>(g.C) + blockIdx.z * g.split_stride + (long long)m * g.ldc;
                    if (ok0) C[n] = v0;
                    if (ok1) C[n + 1] = v1;
                }
            }
        }
    }
}

}  // namespace sg
}  // namespace fd2
