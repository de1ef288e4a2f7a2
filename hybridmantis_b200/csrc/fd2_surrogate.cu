// fd2_surrogate.cu -- the learned surrogate: MLP training and inference.
//
// Network (hidden width H, 256 by default):
//   x0 [B][32]  normalised features (8 used, zero padded to the GEMM's K)
//   h1 = relu(x0 W1^T + b1), h2 = relu(h1 W2^T + b2), h3 = relu(h2 W3^T + b3)
//   out = h3 W4^T + b4       [B][64] (25 used)
// All products run on fd2_sg_gemm.cuh (BF16 operands, FP32 accumulation);
// FP32 master parameters, BF16 copies for the GEMMs, Adam in FP32.  One
// training step (batch gather, forward, loss, backward, Adam) is a CUDA
// graph replayed `steps` times; the step counter lives on the device.
//
// Loss per point with N photons, d detected and radial label counts h_j
// (j < R: quadratic bins inside radial_max_um, j = R beyond):
//   L = BCE(sigmoid(out0), d / N)
//     + lambda * sum_j y_j (-log q_j),   y_j = h_j / sum h
// with q_j the probability of bin j under the mixture of Gaussian rings
//   PRF(r) = sum_k w_k N(r; mu_k, s_k) / S_k per unit area (fd2_sg_mix.cuh),
//   w = softmax(out[1..8]), mu = 50 um * softplus(out[9..16]),
//   s = 10 um * exp(clamp(out[17..24], -6, 4)).
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "fd2.h"
#include "fd2_sg_gemm.cuh"
#include "fd2_sg_tc.cuh"
#include "fd2_sg_internal.h"
#include "fd2_sg_mix.cuh"
#include "fd2_surrogate.h"

using fd2::sg::GemmArgs;

namespace fd2 {
namespace sg {

// ------------------------------------------------------------ device math

__device__ __forceinline__ uint4 philox10(uint4 c, uint32_t k0, uint32_t k1)
{
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t lo0 = 0xD2511F53u * c.x, hi0 = __umulhi(0xD2511F53u, c.x);
        const uint32_t lo1 = 0xCD9E8D57u * c.z, hi1 = __umulhi(0xCD9E8D57u, c.z);
        c = make_uint4(hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0);
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return c;
}

// Loss of one point and (optionally) d loss / d out.  y: normalised radial
// label over bins + 1 categories (null = no radial term).  The radial term
// is the cross-entropy -sum_j y_j log q_j of the ring mixture's category
// probabilities q_j = sum_k w_k M_k(e_j, e_j+1) / S_k (fd2_sg_mix.cuh).
__device__ float point_loss(const float *o, float t, const float *y, int bins, float r_max, float lambda,
                            float *dout, float *det_loss, float *rad_loss)
{
    // detection
    const float z = o[0];
    const float p = 1.0f / (1.0f + expf(-z));
    // log p = -softplus(-z), log(1 - p) = -softplus(z)
    const float sp_neg = fmaxf(-z, 0.0f) + log1pf(expf(-fabsf(z)));
    const float sp_pos = fmaxf(z, 0.0f) + log1pf(expf(-fabsf(z)));
    const float ld = t * sp_neg + (1.0f - t) * sp_pos;
    if (dout) dout[0] = p - t;
    *det_loss = ld;
    *rad_loss = 0.0f;
    if (!y) {
        if (dout)
            for (int i = 1; i < kOutputs; ++i) dout[i] = 0.0f;
        return ld;
    }
    Mix m;
    decode_mix(o, m);
    // per component: A1 = sum_j c_j M_kj, Amu = sum_j c_j dM_kj/dmu, Asd = sum_j c_j dM_kj/dsd
    float A1[kComponents], Amu[kComponents], Asd[kComponents];
    Edge lo[kComponents];
#pragma unroll
    for (int k = 0; k < kComponents; ++k) {
        A1[k] = 0.0f;
        Amu[k] = 0.0f;
        Asd[k] = 0.0f;
        lo[k] = edge_at(0.0f, false, m.mu[k], m.sd[k]);
    }
    float lr = 0.0f;
    for (int j = 0; j <= bins; ++j) {
        const bool top = j >= bins;
        const float e_hi = top ? 0.0f : radial_edge(j + 1, bins, r_max);
        float M[kComponents], dM_mu[kComponents], dM_sd[kComponents];
        Edge hi[kComponents];
        float q = 0.0f;
#pragma unroll
        for (int k = 0; k < kComponents; ++k) {
            hi[k] = edge_at(e_hi, top, m.mu[k], m.sd[k]);
            M[k] = ring_mass(lo[k], hi[k], m.mu[k], m.sd[k], &dM_mu[k], &dM_sd[k]);
            q += m.w[k] * M[k] / m.S[k];
        }
        const float yj = y[j];
        if (yj > 0.0f) {
            const float qe = q + 1e-12f;
            lr -= yj * logf(qe);
            const float c = yj / qe;
#pragma unroll
            for (int k = 0; k < kComponents; ++k) {
                A1[k] += c * M[k];
                Amu[k] += c * dM_mu[k];
                Asd[k] += c * dM_sd[k];
            }
        }
#pragma unroll
        for (int k = 0; k < kComponents; ++k) lo[k] = hi[k];
    }
    *rad_loss = lr;
    if (dout) {
        float gw[kComponents], wg = 0.0f;
#pragma unroll
        for (int k = 0; k < kComponents; ++k) {
            gw[k] = -A1[k] / m.S[k];
            wg += m.w[k] * gw[k];
        }
#pragma unroll
        for (int k = 0; k < kComponents; ++k) {
            const float f = m.w[k] / m.S[k];
            const float gmu = -f * (Amu[k] - A1[k] * m.dS_mu[k] / m.S[k]);
            const float gsd = -f * (Asd[k] - A1[k] * m.dS_sd[k] / m.S[k]);
            dout[1 + k] = lambda * m.w[k] * (gw[k] - wg);
            dout[1 + kComponents + k] = lambda * m.dmu[k] * gmu;
            dout[1 + 2 * kComponents + k] = m.clamped[k] ? 0.0f : lambda * m.sd[k] * gsd;
        }
    }
    return ld + lambda * lr;
}

// ------------------------------------------------------------ kernels

// Normalised, zero-padded BF16 network input of one feature row.
__device__ __forceinline__ void write_input(const float *f, const float *lo, const float *inv, __nv_bfloat16 *x)
{
#pragma unroll
    for (int i = 0; i < kFeatures; ++i) x[i] = __float2bfloat16(2.0f * (f[i] - lo[i]) * inv[i] - 1.0f);
#pragma unroll
    for (int i = kFeatures; i < kInPad; ++i) x[i] = __float2bfloat16(0.0f);
}

// Training batch: rows drawn with Philox(seed, step, row) from [0, n_train),
// or the rows [first, first + b) in order when `sequential`.
__global__ void gather_kernel(const float *__restrict__ feat, const int32_t *__restrict__ photons,
                              const int32_t *__restrict__ detected, const uint32_t *__restrict__ radial, int bins,
                              int64_t n_train, int64_t first, int b, bool sequential, uint64_t seed,
                              const unsigned long long *step, NormParams norm, __nv_bfloat16 *__restrict__ x0,
                              float *__restrict__ target, float *__restrict__ ylab, float *__restrict__ has_rad)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= b) return;
    int64_t i;
    if (sequential) {
        i = first + r;
    } else {
        const uint4 h = philox10(make_uint4((uint32_t)r, (uint32_t)*step, (uint32_t)(*step >> 32), 0x5347u),
                                 (uint32_t)seed, (uint32_t)(seed >> 32));
        const unsigned long long v = ((unsigned long long)h.x << 32) | h.y;
        i = (int64_t)(v % (unsigned long long)n_train);
    }
    write_input(feat + i * kFeatures, norm.lo, norm.inv, x0 + (int64_t)r * kInPad);
    const int32_t N = photons[i];
    target[r] = N > 0 ? (float)detected[i] / (float)N : 0.0f;
    const uint32_t *h = radial + i * (int64_t)(bins + 1);
    double tot = 0.0;
    for (int j = 0; j <= bins; ++j) tot += h[j];
    const float inv = tot > 0.0 ? (float)(1.0 / tot) : 0.0f;
    for (int j = 0; j <= bins; ++j) ylab[(int64_t)r * (bins + 1) + j] = (float)h[j] * inv;
    has_rad[r] = tot > 0.0 ? 1.0f : 0.0f;
}

// Loss (summed into acc[0..2] = total, detection, radial) and, when dout is
// set, dL/dout / b as BF16 [b][64].
__global__ void loss_kernel(const float *__restrict__ out, int ldo, const float *__restrict__ target,
                            const float *__restrict__ ylab, const float *__restrict__ has_rad, int bins,
                            float r_max, float lambda, int b, float scale, __nv_bfloat16 *__restrict__ dout,
                            double *acc)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    float lt = 0.0f, ld = 0.0f, lrad = 0.0f;
    if (r < b) {
        float o[kOutputs], g[kOutputs];
        for (int i = 0; i < kOutputs; ++i) o[i] = out[(int64_t)r * ldo + i];
        const bool rad = has_rad[r] > 0.0f;
        lt = point_loss(o, target[r], rad ? ylab + (int64_t)r * (bins + 1) : nullptr, bins, r_max, lambda,
                        dout ? g : nullptr, &ld, &lrad);
        if (dout) {
            for (int i = 0; i < kOutputs; ++i) dout[(int64_t)r * kOutPad + i] = __float2bfloat16(g[i] * scale);
            for (int i = kOutputs; i < kOutPad; ++i) dout[(int64_t)r * kOutPad + i] = __float2bfloat16(0.0f);
        }
    }
    // block sums
    __shared__ float s[3][32];
    for (int off = 16; off > 0; off >>= 1) {
        lt += __shfl_down_sync(0xffffffffu, lt, off);
        ld += __shfl_down_sync(0xffffffffu, ld, off);
        lrad += __shfl_down_sync(0xffffffffu, lrad, off);
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) {
        s[0][w] = lt;
        s[1][w] = ld;
        s[2][w] = lrad;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double v = 0.0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) v += s[threadIdx.x][i];
        atomicAdd(&acc[threadIdx.x], v);
    }
}

// db[n] = sum_r dy[r][n] (BF16 rows), FP32 result; one block per 32 columns.
__global__ void colsum_kernel(const __nv_bfloat16 *__restrict__ dy, int ld, int rows, int cols, float *__restrict__ db)
{
    const int n = blockIdx.x * 32 + (threadIdx.x & 31);
    const int part = threadIdx.x >> 5, parts = blockDim.x >> 5;
    float s = 0.0f;
    if (n < cols)
        for (int r = part; r < rows; r += parts) s += __bfloat162float(dy[(int64_t)r * ld + n]);
    __shared__ float sh[32][33];
    sh[part][threadIdx.x & 31] = s;
    __syncthreads();
    if (part == 0 && n < cols) {
        float t = 0.0f;
        for (int p = 0; p < parts; ++p) t += sh[p][threadIdx.x & 31];
        db[n] = t;
    }
}

// Sum of split-K partials: out[i] = sum_z ws[z][i].
__global__ void split_sum_kernel(const float *__restrict__ ws, int splits, int64_t n, float *__restrict__ out)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        float s = 0.0f;
        for (int z = 0; z < splits; ++z) s += ws[(int64_t)z * n + i];
        out[i] = s;
    }
}

// Adam on the FP32 masters, then the BF16 copies.  `mask` zeroes the update
// of padding entries (their gradients are zero anyway).
__global__ void adam_kernel(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                            float *__restrict__ v, __nv_bfloat16 *__restrict__ pb, int64_t n, const float *lr_ptr, float b1,
                            float b2, float eps, unsigned long long *step, const uint8_t *__restrict__ live)
{
    const unsigned long long t = *step + 1;
    const float lr = *lr_ptr;
    const float c1 = 1.0f - powf(b1, (float)t), c2 = 1.0f - powf(b2, (float)t);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        if (!live[i]) continue;
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float w = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        p[i] = w;
        pb[i] = __float2bfloat16(w);
    }
}

__global__ void step_kernel(unsigned long long *step) { *step += 1; }

__global__ void to_bf16_kernel(const float *__restrict__ p, __nv_bfloat16 *__restrict__ pb, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        pb[i] = __float2bfloat16(p[i]);
}

// out[c][r] = in[r][c] for r < rows, 0 for rows <= r < rows_pad (BF16,
// 32 x 32 tiles through shared memory; in is [rows][ld_in], out
// [cols][rows_pad]).  Feeds the tcgen05 backward products, whose operands
// must be contiguous along the contraction.
__global__ void transpose_bf16_kernel(const __nv_bfloat16 *__restrict__ in, int ld_in, int rows, int cols,
                                      int rows_pad, __nv_bfloat16 *__restrict__ out)
{
    __shared__ __nv_bfloat16 t[32][33];
    const int r0 = blockIdx.x * 32, c0 = blockIdx.y * 32;
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int r = r0 + i, c = c0 + threadIdx.x;
        t[i][threadIdx.x] = (r < rows && c < cols) ? in[(int64_t)r * ld_in + c] : __float2bfloat16(0.0f);
    }
    __syncthreads();
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int c = c0 + i, r = r0 + threadIdx.x;
        if (c < cols && r < rows_pad) out[(int64_t)c * rows_pad + r] = t[threadIdx.x][i];
    }
}

// Normalised inputs of host-given feature rows.
__global__ void input_kernel(const float *__restrict__ feat, int64_t n, NormParams norm, __nv_bfloat16 *__restrict__ x0)
{
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x)
        write_input(feat + r * kFeatures, norm.lo, norm.inv, x0 + r * kInPad);
}

}  // namespace sg
}  // namespace fd2

// ================================================================ host

using namespace fd2::sg;

namespace {

unsigned grid_for(int64_t n, int block, int cap = 4096)
{
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + block - 1) / block, cap));
}

}  // namespace

fd2_status sg_fail(fd2_sg *s, fd2_status st, const std::string &msg)
{
    if (s) s->last_error = msg;
    return st;
}

fd2_status sg_cuda(fd2_sg *s, cudaError_t e, const char *what)
{
    if (e == cudaSuccess) return FD2_OK;
    return sg_fail(s, e == cudaErrorMemoryAllocation ? FD2_ERR_OUT_OF_MEMORY : FD2_ERR_CUDA,
                   std::string(what) + ": " + cudaGetErrorString(e));
}

#define SG_CUDA(s, call)                                      \
    do {                                                      \
        cudaError_t e_ = (call);                              \
        if (e_ != cudaSuccess) return sg_cuda(s, e_, #call);  \
    } while (0)

cudaError_t sg_gemm(cudaStream_t st, bool a_kc, bool b_kc, const GemmArgs &g, int splits)
{
    dim3 grid((unsigned)((g.N + kBN - 1) / kBN), (unsigned)((g.M + kBM - 1) / kBM), (unsigned)splits);
    if (a_kc && b_kc) gemm_kernel<true, true><<<grid, kGemmThreads, 0, st>>>(g);
    else if (a_kc && !b_kc) gemm_kernel<true, false><<<grid, kGemmThreads, 0, st>>>(g);
    else if (!a_kc && !b_kc) gemm_kernel<false, false><<<grid, kGemmThreads, 0, st>>>(g);
    else return cudaErrorInvalidValue;
    return cudaGetLastError();
}

namespace {

GemmArgs gemm_args(const __nv_bfloat16 *A, int lda, const __nv_bfloat16 *B, int ldb, int M, int N, int K, int epi,
                   void *C, int ldc)
{
    GemmArgs g;
    std::memset(&g, 0, sizeof g);
    g.A = A;
    g.B = B;
    g.lda = lda;
    g.ldb = ldb;
    g.M = M;
    g.N = N;
    g.K = K;
    g.k_per_split = K;
    g.epi = epi;
    g.C = C;
    g.ldc = ldc;
    return g;
}

}  // namespace

namespace {
cudaError_t launch_tc(fd2_sg *s, cudaStream_t st, const TcArgs &t0, unsigned grid_x, unsigned grid_y);
}  // namespace

// One forward product (K-contiguous operands, bias epilogue): tcgen05 when
// the shapes fit one pass of fd2_sg_tc.cuh, else the mma.sync kernel.
static cudaError_t sg_dense(fd2_sg *s, cudaStream_t st, const GemmArgs &g)
{
    const bool tc = s->use_tc && g.K % 16 == 0 && g.K <= kTcMaxK && g.N % 16 == 0 && g.N >= 16 && g.N <= kTcMaxN &&
                    g.lda % 8 == 0 && g.ldb % 8 == 0 && g.ldc % 16 == 0 && g.M > 0;
    if (!tc) {
        if ((int64_t)g.M > (int64_t)65535 * kBM) return cudaErrorInvalidValue;  // one grid row per 64 rows
        return sg_gemm(st, true, true, g, 1);
    }
    TcArgs t{};
    t.A = g.A;
    t.B = g.B;
    t.lda = g.lda;
    t.ldb = g.ldb;
    t.M = g.M;
    t.N = g.N;
    t.K = g.K;
    t.m_limit = g.m_limit;
    t.epi = g.epi;
    t.bias = g.bias;
    t.C = g.C;
    t.ldc = g.ldc;
    t.fault = s->d_tc_fault;
    const unsigned grid = (unsigned)std::min((g.M + kTcRows - 1) / kTcRows, s->sm_count);
    return launch_tc(s, st, t, grid, 1);
}

fd2_status sg_tc_check(fd2_sg *s)
{
    if (!s || !s->d_tc_fault) return FD2_OK;
    unsigned f = 0;
    SG_CUDA(s, cudaMemcpy(&f, s->d_tc_fault, sizeof f, cudaMemcpyDeviceToHost));
    if (!f) return FD2_OK;
    SG_CUDA(s, cudaMemset(s->d_tc_fault, 0, sizeof f));
    return sg_fail(s, FD2_ERR_DEVICE_ABORT, "a tensor-core GEMM tile gave up waiting for its MMAs");
}

// Forward pass over `rows` input rows in sg->x0 (row capacity >= rows):
// activations h1..h3 (BF16) and out (FP32 [rows][64]).
cudaError_t sg_forward(fd2_sg *s, cudaStream_t st, const __nv_bfloat16 *x0, int rows, const int *m_limit,
                       __nv_bfloat16 *h1, __nv_bfloat16 *h2, __nv_bfloat16 *h3, float *out)
{
    const int H = s->hidden;
    cudaError_t e;
    GemmArgs g = gemm_args(x0, kInPad, s->pb + s->off[kW1], kInPad, rows, H, kInPad, kEpiBiasReluBf16, h1, H);
    g.bias = s->p + s->off[kB1];
    g.m_limit = m_limit;
    if ((e = sg_dense(s, st, g)) != cudaSuccess) return e;
    g = gemm_args(h1, H, s->pb + s->off[kW2], H, rows, H, H, kEpiBiasReluBf16, h2, H);
    g.bias = s->p + s->off[kB2];
    g.m_limit = m_limit;
    if ((e = sg_dense(s, st, g)) != cudaSuccess) return e;
    g = gemm_args(h2, H, s->pb + s->off[kW3], H, rows, H, H, kEpiBiasReluBf16, h3, H);
    g.bias = s->p + s->off[kB3];
    g.m_limit = m_limit;
    if ((e = sg_dense(s, st, g)) != cudaSuccess) return e;
    g = gemm_args(h3, H, s->pb + s->off[kW4], H, rows, kOutPad, H, kEpiBiasF32, out, kOutPad);
    g.bias = s->p + s->off[kB4];
    g.m_limit = m_limit;
    return sg_dense(s, st, g);
}

namespace {

// Weight gradient dW [M][K] = dy^T x over `rows` batch rows, split-K.
cudaError_t weight_grad(fd2_sg *s, cudaStream_t st, const __nv_bfloat16 *dy, int ldy, int M, const __nv_bfloat16 *x,
                        int ldx, int K, int rows, float *dw)
{
    const int splits = std::max(1, std::min(kMaxSplits, rows / 512));
    const int per = ((rows + splits - 1) / splits + kBK - 1) / kBK * kBK;
    GemmArgs g = gemm_args(dy, ldy, x, ldx, M, K, rows, kEpiPartialF32, s->ws, K);
    g.k_per_split = per;
    g.split_stride = (long long)M * K;
    const int z = (rows + per - 1) / per;
    cudaError_t e = sg_gemm(st, false, false, g, z);
    if (e != cudaSuccess) return e;
    split_sum_kernel<<<grid_for((int64_t)M * K, 256), 256, 0, st>>>(s->ws, z, (int64_t)M * K, dw);
    return cudaGetLastError();
}

constexpr int kTcSlice = 256;  // batch rows per weight-gradient slice (the contraction of one tcgen05 pass)

int rows_pad(int rows) { return (rows + kTcSlice - 1) / kTcSlice * kTcSlice; }

cudaError_t launch_transpose(cudaStream_t st, const __nv_bfloat16 *in, int ld_in, int rows, int cols,
                             __nv_bfloat16 *out)
{
    const int rp = rows_pad(rows);
    transpose_bf16_kernel<<<dim3((unsigned)(rp / 32), (unsigned)((cols + 31) / 32)), dim3(32, 8), 0, st>>>(
        in, ld_in, rows, cols, rp, out);
    return cudaGetLastError();
}

// The driver's cuTensorMapEncodeTiled, through the runtime (no libcuda link).
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }();
    return fn;
}

// A 2D map of a row-major BF16 matrix (rows x cols, row stride ld elements)
// whose boxes are box_rows rows by 8 columns (16 bytes: one K column of the
// canonical no-swizzle layout) or, with sw128, by 64 columns (128 bytes,
// written with the 128-byte swizzle); rows past the matrix read as zeros.
static bool encode_map(CUtensorMap *m, const __nv_bfloat16 *base, int rows, int cols, int ld, int box_rows, bool sw128)
{
    PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    const int box_cols = sw128 ? 64 : 8;
    if (!enc || reinterpret_cast<uintptr_t>(base) % 16 != 0 || (ld * 2) % 16 != 0 || rows < 1 || cols < box_cols ||
        box_rows < 1 || box_rows > 256)
        return false;
    const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
    const cuuint32_t box[2] = {(cuuint32_t)box_cols, (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<__nv_bfloat16 *>(base), dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, sw128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE,
               CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

cudaError_t launch_tc(fd2_sg *s, cudaStream_t st, const TcArgs &t0, unsigned grid_x, unsigned grid_y)
{
    const dim3 grid(grid_x, grid_y);
    if (s->tc_pipe && t0.K % 16 == 0 && (t0.K <= kPipeChunkK || t0.K % kPipeChunkK == 0)) {
        // operands by TMA where the product has no batch slices and the maps
        // can be made (16-byte aligned bases and row strides), in 128-byte
        // swizzled rows where K is a multiple of 64 (the ring's chunks are
        // then 64 wide), else cp.async
        TcArgs t = t0;
        const bool sw = s->tc_sw128 && t.K % 64 == 0;
        t.tma = s->tc_tma && t.a_split == 0 && t.b_split == 0 &&
                encode_map(&t.tmap_a, t.A, t.M, t.K, t.lda, kTcRows, sw) &&
                encode_map(&t.tmap_b, t.B, t.N, t.K, t.ldb, t.N, sw);
        if (t.tma && sw) t.tma = 2;
        // the staged BF16 epilogues store whole 32-row blocks by TMA
        t.tma_store = s->tc_tma_store && (t.epi == kEpiBiasReluBf16 || t.epi == kEpiMaskBf16) && t.N % 64 == 0 &&
                      t.c_split == 0 && encode_map(&t.tmap_c, static_cast<const __nv_bfloat16 *>(t.C), t.M, t.N,
                                                   t.ldc, 32, true);
        const size_t smem = tc_pipe_smem_bytes(t.N, t.K);
        if (t.epi == kEpiBiasReluBf16) gemm_tc_pipe_kernel<kEpiBiasReluBf16><<<grid, kPipeThreads, smem, st>>>(t);
        else if (t.epi == kEpiBiasF32) gemm_tc_pipe_kernel<kEpiBiasF32><<<grid, kPipeThreads, smem, st>>>(t);
        else if (t.epi == kEpiMaskBf16) gemm_tc_pipe_kernel<kEpiMaskBf16><<<grid, kPipeThreads, smem, st>>>(t);
        else if (t.epi == kEpiPartialF32) gemm_tc_pipe_kernel<kEpiPartialF32><<<grid, kPipeThreads, smem, st>>>(t);
        else return cudaErrorInvalidValue;
        return cudaGetLastError();
    }
    const TcArgs &t = t0;
    const size_t smem = tc_smem_bytes(t.N, t.K);
    if (t.epi == kEpiBiasReluBf16) gemm_tc_kernel<kEpiBiasReluBf16><<<grid, kTcThreads, smem, st>>>(t);
    else if (t.epi == kEpiBiasF32) gemm_tc_kernel<kEpiBiasF32><<<grid, kTcThreads, smem, st>>>(t);
    else if (t.epi == kEpiMaskBf16) gemm_tc_kernel<kEpiMaskBf16><<<grid, kTcThreads, smem, st>>>(t);
    else if (t.epi == kEpiPartialF32) gemm_tc_kernel<kEpiPartialF32><<<grid, kTcThreads, smem, st>>>(t);
    else return cudaErrorInvalidValue;
    return cudaGetLastError();
}

// The backward products fit one tcgen05 pass per tile when every
// contraction (64 outputs, H hidden, 256-row batch slices) is <= 256 and
// every width a multiple of 16.
bool tc_backward_ok(const fd2_sg *s, int rows)
{
    const int H = s->hidden;
    return s->use_tc && s->tA && H % 16 == 0 && H >= 32 && H <= kTcMaxN && rows > 0 && rows <= s->cap_rows;
}

// Weight gradient on tcgen05: dW [M][K] = sum over 256-row slices z of
// dy_z^T x_z, with dy^T ([M][rows_pad]) and x^T ([K][rows_pad]) staged
// contiguous along the batch; one CTA per (128-row tile of dW, slice), FP32
// partial planes summed in slice order (deterministic).
cudaError_t weight_grad_tc(fd2_sg *s, cudaStream_t st, const __nv_bfloat16 *dy, int ldy, int M,
                           const __nv_bfloat16 *x, int ldx, int K, int rows, float *dw)
{
    cudaError_t e;
    const int rp = rows_pad(rows), z = rp / kTcSlice;
    if ((int64_t)z * M * K > s->ws_floats) return cudaErrorInvalidValue;
    if ((e = launch_transpose(st, dy, ldy, rows, M, s->tA)) != cudaSuccess) return e;
    if ((e = launch_transpose(st, x, ldx, rows, K, s->tB)) != cudaSuccess) return e;
    TcArgs t{};
    t.A = s->tA;
    t.B = s->tB;
    t.lda = rp;
    t.ldb = rp;
    t.M = M;
    t.N = K;
    t.K = kTcSlice;
    t.epi = kEpiPartialF32;
    t.C = s->ws;
    t.ldc = K;
    t.a_split = kTcSlice;
    t.b_split = kTcSlice;
    t.c_split = (long long)M * K;
    t.fault = s->d_tc_fault;
    if ((e = launch_tc(s, st, t, (unsigned)((M + kTcRows - 1) / kTcRows), (unsigned)z)) != cudaSuccess) return e;
    split_sum_kernel<<<grid_for((int64_t)M * K, 256), 256, 0, st>>>(s->ws, z, (int64_t)M * K, dw);
    return cudaGetLastError();
}

// Input gradient on tcgen05: d [rows][H] = (dy [rows][Nout] W [Nout][H]) *
// (h > 0), with W^T ([H][Nout]) as the K-contiguous second operand.
cudaError_t input_grad_tc(fd2_sg *s, cudaStream_t st, const __nv_bfloat16 *dy, int Nout, const __nv_bfloat16 *wT,
                          const __nv_bfloat16 *h, int rows, __nv_bfloat16 *d)
{
    const int H = s->hidden;
    TcArgs t{};
    t.A = dy;
    t.B = wT;
    t.lda = Nout;
    t.ldb = Nout;
    t.M = rows;
    t.N = H;
    t.K = Nout;
    t.epi = kEpiMaskBf16;
    t.mask = h;
    t.ldm = H;
    t.C = d;
    t.ldc = H;
    t.fault = s->d_tc_fault;
    return launch_tc(s, st, t, (unsigned)std::min((rows + kTcRows - 1) / kTcRows, s->sm_count), 1);
}

// Backward pass from dout (BF16 [rows][64], already scaled by 1/rows).
cudaError_t backward(fd2_sg *s, cudaStream_t st, int rows)
{
    const int H = s->hidden;
    cudaError_t e;
    float *G = s->g;
    if (tc_backward_ok(s, rows)) {
        // the weights' transposes (BF16 copies of this step's parameters)
        __nv_bfloat16 *w2T = s->pbT, *w3T = s->pbT + (size_t)H * H, *w4T = s->pbT + 2 * (size_t)H * H;
        const dim3 tb(32, 8), tg((unsigned)((H + 31) / 32), (unsigned)((H + 31) / 32));
        transpose_bf16_kernel<<<dim3((unsigned)((kOutPad + 31) / 32), tg.y), tb, 0, st>>>(s->pb + s->off[kW4], H,
                                                                                          kOutPad, H, kOutPad, w4T);
        transpose_bf16_kernel<<<tg, tb, 0, st>>>(s->pb + s->off[kW3], H, H, H, H, w3T);
        transpose_bf16_kernel<<<tg, tb, 0, st>>>(s->pb + s->off[kW2], H, H, H, H, w2T);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        // layer 4
        if ((e = weight_grad_tc(s, st, s->dout, kOutPad, kOutPad, s->h3, H, H, rows, G + s->off[kW4])) != cudaSuccess)
            return e;
        colsum_kernel<<<(kOutPad + 31) / 32, 1024, 0, st>>>(s->dout, kOutPad, rows, kOutPad, G + s->off[kB4]);
        if ((e = input_grad_tc(s, st, s->dout, kOutPad, w4T, s->h3, rows, s->d3)) != cudaSuccess) return e;
        // layer 3
        if ((e = weight_grad_tc(s, st, s->d3, H, H, s->h2, H, H, rows, G + s->off[kW3])) != cudaSuccess) return e;
        colsum_kernel<<<(H + 31) / 32, 1024, 0, st>>>(s->d3, H, rows, H, G + s->off[kB3]);
        if ((e = input_grad_tc(s, st, s->d3, H, w3T, s->h2, rows, s->d2)) != cudaSuccess) return e;
        // layer 2
        if ((e = weight_grad_tc(s, st, s->d2, H, H, s->h1, H, H, rows, G + s->off[kW2])) != cudaSuccess) return e;
        colsum_kernel<<<(H + 31) / 32, 1024, 0, st>>>(s->d2, H, rows, H, G + s->off[kB2]);
        if ((e = input_grad_tc(s, st, s->d2, H, w2T, s->h1, rows, s->d1)) != cudaSuccess) return e;
        // layer 1
        if ((e = weight_grad_tc(s, st, s->d1, H, H, s->x0, kInPad, kInPad, rows, G + s->off[kW1])) != cudaSuccess)
            return e;
        colsum_kernel<<<(H + 31) / 32, 1024, 0, st>>>(s->d1, H, rows, H, G + s->off[kB1]);
        return cudaGetLastError();
    }
    // layer 4
    if ((e = weight_grad(s, st, s->dout, kOutPad, kOutPad, s->h3, H, H, rows, G + s->off[kW4])) != cudaSuccess)
        return e;
    colsum_kernel<<<(kOutPad + 31) / 32, 1024, 0, st>>>(s->dout, kOutPad, rows, kOutPad, G + s->off[kB4]);
    GemmArgs g = gemm_args(s->dout, kOutPad, s->pb + s->off[kW4], H, rows, H, kOutPad, kEpiMaskBf16, s->d3, H);
    g.mask = s->h3;
    g.ldm = H;
    if ((e = sg_gemm(st, true, false, g, 1)) != cudaSuccess) return e;
    // layer 3
    if ((e = weight_grad(s, st, s->d3, H, H, s->h2, H, H, rows, G + s->off[kW3])) != cudaSuccess) return e;
    colsum_kernel<<<(H + 31) / 32, 1024, 0, st>>>(s->d3, H, rows, H, G + s->off[kB3]);
    g = gemm_args(s->d3, H, s->pb + s->off[kW3], H, rows, H, H, kEpiMaskBf16, s->d2, H);
    g.mask = s->h2;
    g.ldm = H;
    if ((e = sg_gemm(st, true, false, g, 1)) != cudaSuccess) return e;
    // layer 2
    if ((e = weight_grad(s, st, s->d2, H, H, s->h1, H, H, rows, G + s->off[kW2])) != cudaSuccess) return e;
    colsum_kernel<<<(H + 31) / 32, 1024, 0, st>>>(s->d2, H, rows, H, G + s->off[kB2]);
    g = gemm_args(s->d2, H, s->pb + s->off[kW2], H, rows, H, H, kEpiMaskBf16, s->d1, H);
    g.mask = s->h1;
    g.ldm = H;
    if ((e = sg_gemm(st, true, false, g, 1)) != cudaSuccess) return e;
    // layer 1
    if ((e = weight_grad(s, st, s->d1, H, H, s->x0, kInPad, kInPad, rows, G + s->off[kW1])) != cudaSuccess) return e;
    colsum_kernel<<<(H + 31) / 32, 1024, 0, st>>>(s->d1, H, rows, H, G + s->off[kB1]);
    return cudaGetLastError();
}

// One training step on s->batch rows (everything on the device).
cudaError_t train_step(fd2_sg *s, cudaStream_t st)
{
    const int B = s->batch, bins = s->bins;
    cudaError_t e;
    gather_kernel<<<grid_for(B, 256), 256, 0, st>>>(s->d_feat, s->d_photons, s->d_detected, s->d_radial, bins,
                                                    s->n_train, 0, B, false, s->seed, s->d_step, s->norm, s->x0,
                                                    s->target, s->ylab, s->has_rad);
    if ((e = sg_forward(s, st, s->x0, B, nullptr, s->h1, s->h2, s->h3, s->out)) != cudaSuccess) return e;
    loss_kernel<<<grid_for(B, 128), 128, 0, st>>>(s->out, kOutPad, s->target, s->ylab, s->has_rad, bins,
                                                  (float)s->radial_max, s->lambda, B, 1.0f / (float)B,
                                                  s->dout, s->d_acc);
    if ((e = backward(s, st, B)) != cudaSuccess) return e;
    adam_kernel<<<grid_for(s->n_params, 256), 256, 0, st>>>(s->p, s->g, s->m, s->v, s->pb, s->n_params, s->d_lr,
                                                            s->beta1, s->beta2, s->eps, s->d_step, s->d_live);
    step_kernel<<<1, 1, 0, st>>>(s->d_step);
    return cudaGetLastError();
}

void layout(fd2_sg *s)
{
    const int64_t H = s->hidden;
    int64_t o = 0;
    auto put = [&](int idx, int64_t n) {
        s->off[idx] = o;
        o += (n + 63) / 64 * 64;  // keep every block 128-byte aligned in BF16
    };
    put(kW1, H * kInPad);
    put(kB1, H);
    put(kW2, H * H);
    put(kB2, H);
    put(kW3, H * H);
    put(kB3, H);
    put(kW4, (int64_t)kOutPad * H);
    put(kB4, kOutPad);
    s->n_params = o;
}

// Which master entries are real parameters (not padding).
std::vector<uint8_t> live_mask(const fd2_sg *s)
{
    const int64_t H = s->hidden;
    std::vector<uint8_t> live((size_t)s->n_params, 0);
    for (int64_t r = 0; r < H; ++r)
        for (int c = 0; c < kFeatures; ++c) live[(size_t)(s->off[kW1] + r * kInPad + c)] = 1;
    for (int64_t i = 0; i < H; ++i) {
        live[(size_t)(s->off[kB1] + i)] = 1;
        live[(size_t)(s->off[kB2] + i)] = 1;
        live[(size_t)(s->off[kB3] + i)] = 1;
    }
    for (int64_t i = 0; i < H * H; ++i) {
        live[(size_t)(s->off[kW2] + i)] = 1;
        live[(size_t)(s->off[kW3] + i)] = 1;
    }
    for (int r = 0; r < kOutputs; ++r) {
        for (int64_t c = 0; c < H; ++c) live[(size_t)(s->off[kW4] + r * H + c)] = 1;
        live[(size_t)(s->off[kB4] + r)] = 1;
    }
    return live;
}

// Public parameter order (no padding) <-> master layout.
template <class F>
void for_each_public(const fd2_sg *s, F f)
{
    const int64_t H = s->hidden;
    int64_t k = 0;
    for (int64_t r = 0; r < H; ++r)
        for (int c = 0; c < kFeatures; ++c) f(k++, s->off[kW1] + r * kInPad + c);
    for (int64_t i = 0; i < H; ++i) f(k++, s->off[kB1] + i);
    for (int64_t i = 0; i < H * H; ++i) f(k++, s->off[kW2] + i);
    for (int64_t i = 0; i < H; ++i) f(k++, s->off[kB2] + i);
    for (int64_t i = 0; i < H * H; ++i) f(k++, s->off[kW3] + i);
    for (int64_t i = 0; i < H; ++i) f(k++, s->off[kB3] + i);
    for (int r = 0; r < kOutputs; ++r)
        for (int64_t c = 0; c < H; ++c) f(k++, s->off[kW4] + r * H + c);
    for (int r = 0; r < kOutputs; ++r) f(k++, s->off[kB4] + r);
}

int64_t public_count(const fd2_sg *s)
{
    const int64_t H = s->hidden;
    return H * kFeatures + H + 2 * (H * H + H) + kOutputs * H + kOutputs;
}

fd2_status upload_params(fd2_sg *s, const std::vector<float> &master)
{
    SG_CUDA(s, cudaSetDevice(s->device));
    SG_CUDA(s, cudaMemcpy(s->p, master.data(), sizeof(float) * master.size(), cudaMemcpyHostToDevice));
    to_bf16_kernel<<<grid_for(s->n_params, 256), 256>>>(s->p, s->pb, s->n_params);
    SG_CUDA(s, cudaGetLastError());
    SG_CUDA(s, cudaMemset(s->m, 0, sizeof(float) * s->n_params));
    SG_CUDA(s, cudaMemset(s->v, 0, sizeof(float) * s->n_params));
    SG_CUDA(s, cudaMemset(s->d_step, 0, sizeof(unsigned long long)));
    SG_CUDA(s, cudaDeviceSynchronize());
    return FD2_OK;
}

void set_norm(fd2_sg *s)
{
    for (int i = 0; i < kFeatures; ++i) {
        s->norm.lo[i] = s->norm_box.lo[i];
        const float span = s->norm_box.hi[i] - s->norm_box.lo[i];
        s->norm.inv[i] = span > 0.0f ? 1.0f / span : 0.5f;  // constant feature -> 0 after 2(f-lo)*inv - 1 + 1
    }
}

template <class T>
cudaError_t alloc(T **p, size_t n)
{
    if (*p) cudaFree(*p);
    *p = nullptr;
    return cudaMalloc((void **)p, sizeof(T) * std::max<size_t>(n, 1));
}

// Activation buffers for `rows` rows.
fd2_status ensure_rows(fd2_sg *s, int rows)
{
    if (rows <= s->cap_rows) return FD2_OK;
    const size_t H = (size_t)s->hidden, R = (size_t)rows;
    // tcgen05 backward: transposed operands over the rows padded to 256, and
    // one FP32 partial plane per 256-row slice
    const size_t RP = (size_t)rows_pad(rows);
    SG_CUDA(s, alloc(&s->tA, std::max<size_t>(H, kOutPad) * RP));
    SG_CUDA(s, alloc(&s->tB, std::max<size_t>(H, kInPad) * RP));
    const size_t plane = std::max<size_t>(H * H, (size_t)kOutPad * H);
    const size_t wsf = std::max<size_t>((size_t)kMaxSplits, RP / kTcSlice) * plane;
    SG_CUDA(s, alloc(&s->ws, wsf));
    s->ws_floats = (int64_t)wsf;
    SG_CUDA(s, alloc(&s->x0, R * kInPad));
    SG_CUDA(s, alloc(&s->h1, R * H));
    SG_CUDA(s, alloc(&s->h2, R * H));
    SG_CUDA(s, alloc(&s->h3, R * H));
    SG_CUDA(s, alloc(&s->d1, R * H));
    SG_CUDA(s, alloc(&s->d2, R * H));
    SG_CUDA(s, alloc(&s->d3, R * H));
    SG_CUDA(s, alloc(&s->out, R * kOutPad));
    SG_CUDA(s, alloc(&s->dout, R * kOutPad));
    SG_CUDA(s, alloc(&s->target, R));
    SG_CUDA(s, alloc(&s->has_rad, R));
    SG_CUDA(s, alloc(&s->ylab, R * (size_t)(s->bins + 1)));
    s->cap_rows = rows;
    if (s->graph) cudaGraphExecDestroy(s->graph);
    s->graph = nullptr;
    return FD2_OK;
}

}  // namespace

extern "C" {

void fd2_sg_default_config(fd2_sg_config *c)
{
    if (!c) return;
    std::memset(c, 0, sizeof *c);
    c->device = 0;
    c->hidden = 256;
    c->radial_bins = 96;
    c->radial_max_um = 400.0;
    c->batch = 8192;
    c->lr = 1e-3f;
    c->beta1 = 0.9f;
    c->beta2 = 0.999f;
    c->adam_eps = 1e-8f;
    c->radial_weight = 1.0f;
    c->lateral_um = 50.0f;
    c->seed = 0x5347fd2ull;
    c->depth_margin_um = 1.0f;
}

const char *fd2_sg_last_error(const fd2_sg *s) { return s ? s->last_error.c_str() : "no surrogate"; }

fd2_status fd2_sg_create(const fd2_sg_config *cfg, fd2_sg **out)
{
    if (!out) return FD2_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    fd2_sg_config c;
    if (cfg) c = *cfg;
    else fd2_sg_default_config(&c);
    if (c.hidden < 64 || c.hidden % 64 || c.hidden > 1024 || c.radial_bins < 1 || c.radial_bins > 1024 ||
        !(c.radial_max_um > 0) || c.batch < 64 || c.batch % 64 || c.batch > (1 << 20) || !(c.lr > 0) ||
        !(c.lateral_um >= 0) || !(c.depth_margin_um >= 0))
        return FD2_ERR_INVALID_ARGUMENT;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) return FD2_ERR_NO_DEVICE;
    if (c.device < 0 || c.device >= ndev) return FD2_ERR_INVALID_ARGUMENT;
    fd2_sg *s = new fd2_sg();
    s->device = c.device;
    s->hidden = c.hidden;
    s->bins = c.radial_bins;
    s->radial_max = c.radial_max_um;
    s->batch = c.batch;
    s->lr = c.lr;
    s->beta1 = c.beta1;
    s->beta2 = c.beta2;
    s->eps = c.adam_eps;
    s->lambda = c.radial_weight;
    s->lateral_um = c.lateral_um;
    s->depth_margin_um = c.depth_margin_um;
    s->seed = c.seed;
    for (int i = 0; i < kFeatures; ++i) {
        s->hull.lo[i] = 0.0f;
        s->hull.hi[i] = 1.0f;
        s->norm_box.lo[i] = 0.0f;
        s->norm_box.hi[i] = 1.0f;
    }
    set_norm(s);
    auto bail = [&](fd2_status st) {
        fd2_sg_destroy(s);
        return st;
    };
    if (cudaSetDevice(s->device) != cudaSuccess) return bail(FD2_ERR_CUDA);
    if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) return bail(FD2_ERR_CUDA);
    layout(s);
    const size_t P = (size_t)s->n_params;
    if (alloc(&s->p, P) || alloc(&s->g, P) || alloc(&s->m, P) || alloc(&s->v, P) || alloc(&s->pb, P) ||
        alloc(&s->d_live, P) || alloc(&s->d_step, 1) || alloc(&s->d_acc, 4) || alloc(&s->d_lr, 1) ||
        alloc(&s->pbT, 2 * (size_t)s->hidden * s->hidden + (size_t)s->hidden * kOutPad))
        return bail(FD2_ERR_OUT_OF_MEMORY);
    if (cudaMemcpy(s->d_lr, &s->lr, sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess) return bail(FD2_ERR_CUDA);
    if (alloc(&s->d_tc_fault, 1) || cudaMemset(s->d_tc_fault, 0, sizeof(unsigned)) != cudaSuccess)
        return bail(FD2_ERR_OUT_OF_MEMORY);
    {
        int sms = 0;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device) == cudaSuccess && sms > 0)
            s->sm_count = sms;
        const char *env = std::getenv("FD2_SG_GEMM");
        s->use_tc = !(env && std::strcmp(env, "mma") == 0);
        s->tc_pipe = !(env && std::strcmp(env, "tc1") == 0);
        s->tc_tma = !(env && std::strcmp(env, "cpasync") == 0);
        s->tc_sw128 = !(env && std::strcmp(env, "noswizzle") == 0);
        s->tc_tma_store = !(env && std::strcmp(env, "nostore") == 0);
        // the tcgen05 kernels' shared memory (outside any stream capture)
        const int bytes = (int)tc_smem_bytes(kTcMaxN, kTcMaxK);
        if (cudaFuncSetAttribute(gemm_tc_kernel<kEpiBiasReluBf16>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) !=
                cudaSuccess ||
            cudaFuncSetAttribute(gemm_tc_kernel<kEpiBiasF32>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) !=
                cudaSuccess ||
            cudaFuncSetAttribute(gemm_tc_kernel<kEpiMaskBf16>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) !=
                cudaSuccess ||
            cudaFuncSetAttribute(gemm_tc_kernel<kEpiPartialF32>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) !=
                cudaSuccess)
            return bail(FD2_ERR_CUDA);
        const int pbytes = (int)tc_pipe_smem_bytes(kTcMaxN, kTcMaxK);
        if (cudaFuncSetAttribute(gemm_tc_pipe_kernel<kEpiBiasReluBf16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 pbytes) != cudaSuccess ||
            cudaFuncSetAttribute(gemm_tc_pipe_kernel<kEpiBiasF32>, cudaFuncAttributeMaxDynamicSharedMemorySize, pbytes) !=
                cudaSuccess ||
            cudaFuncSetAttribute(gemm_tc_pipe_kernel<kEpiMaskBf16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 pbytes) != cudaSuccess ||
            cudaFuncSetAttribute(gemm_tc_pipe_kernel<kEpiPartialF32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 pbytes) != cudaSuccess)
            return bail(FD2_ERR_CUDA);
    }
    const std::vector<uint8_t> live = live_mask(s);
    if (cudaMemcpy(s->d_live, live.data(), P, cudaMemcpyHostToDevice) != cudaSuccess) return bail(FD2_ERR_CUDA);
    if (cudaMemset(s->g, 0, sizeof(float) * P) != cudaSuccess) return bail(FD2_ERR_CUDA);
    // He-normal weights (Box-Muller on a splitmix64 stream), small last
    // layer, zero biases; mixture biases spread the components in radius
    // and width.
    std::vector<float> master(P, 0.0f);
    uint64_t st = c.seed ^ 0x9E3779B97F4A7C15ull;
    auto next = [&]() {
        st += 0x9E3779B97F4A7C15ull;
        uint64_t z = st;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        return ((z >> 11) + 0.5) * (1.0 / 9007199254740992.0);
    };
    auto gauss = [&]() { return std::sqrt(-2.0 * std::log(next())) * std::cos(6.283185307179586 * next()); };
    const int64_t H = s->hidden;
    for (int64_t r = 0; r < H; ++r)
        for (int cc = 0; cc < kFeatures; ++cc)
            master[(size_t)(s->off[kW1] + r * kInPad + cc)] = (float)(gauss() * std::sqrt(2.0 / kFeatures));
    for (int64_t i = 0; i < H * H; ++i) {
        master[(size_t)(s->off[kW2] + i)] = (float)(gauss() * std::sqrt(2.0 / H));
        master[(size_t)(s->off[kW3] + i)] = (float)(gauss() * std::sqrt(2.0 / H));
    }
    for (int r = 0; r < kOutputs; ++r)
        for (int64_t cc = 0; cc < H; ++cc) master[(size_t)(s->off[kW4] + r * H + cc)] = (float)(gauss() * 0.01);
    for (int k = 0; k < kComponents; ++k) {
        const double mu0 = (2.5 + 7.5 * k) / kMuScale;                                          // 2.5 .. 55 um
        master[(size_t)(s->off[kB4] + 1 + kComponents + k)] = (float)std::log(std::expm1(mu0));  // softplus^-1
        master[(size_t)(s->off[kB4] + 1 + 2 * kComponents + k)] = std::log(0.2f + 0.4f * k);  // sd: 2 .. 30 um
    }
    fd2_status r = upload_params(s, master);
    if (r != FD2_OK) return bail(r);
    *out = s;
    return FD2_OK;
}

void fd2_sg_destroy(fd2_sg *s)
{
    if (!s) return;
    cudaSetDevice(s->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    if (s->graph) cudaGraphExecDestroy(s->graph);
    for (void *p : {(void *)s->p, (void *)s->g, (void *)s->m, (void *)s->v, (void *)s->pb, (void *)s->d_live,
                    (void *)s->d_step, (void *)s->d_acc, (void *)s->d_lr, (void *)s->ws, (void *)s->x0, (void *)s->h1, (void *)s->h2,
                    (void *)s->h3, (void *)s->d1, (void *)s->d2, (void *)s->d3, (void *)s->out, (void *)s->dout,
                    (void *)s->target, (void *)s->has_rad, (void *)s->ylab, (void *)s->d_feat, (void *)s->d_photons,
                    (void *)s->d_detected, (void *)s->d_radial, (void *)s->d_tc_fault, (void *)s->pbT, (void *)s->tA,
                    (void *)s->tB})
        if (p) cudaFree(p);
    sg_free_run_buffers(s);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
}

int64_t fd2_sg_num_params(const fd2_sg *s) { return s ? public_count(s) : 0; }

fd2_status fd2_sg_set_lr(fd2_sg *s, float lr)
{
    if (!s || !(lr > 0.0f) || !std::isfinite(lr)) return FD2_ERR_INVALID_ARGUMENT;
    SG_CUDA(s, cudaSetDevice(s->device));
    SG_CUDA(s, cudaStreamSynchronize(s->stream));
    s->lr = lr;
    SG_CUDA(s, cudaMemcpy(s->d_lr, &s->lr, sizeof(float), cudaMemcpyHostToDevice));
    return FD2_OK;
}

fd2_status fd2_sg_get_params(fd2_sg *s, float *params, int64_t n)
{
    if (!s || !params || n < public_count(s)) return FD2_ERR_INVALID_ARGUMENT;
    std::vector<float> master((size_t)s->n_params);
    SG_CUDA(s, cudaSetDevice(s->device));
    SG_CUDA(s, cudaStreamSynchronize(s->stream));
    SG_CUDA(s, cudaMemcpy(master.data(), s->p, sizeof(float) * master.size(), cudaMemcpyDeviceToHost));
    for_each_public(s, [&](int64_t k, int64_t i) { params[k] = master[(size_t)i]; });
    return FD2_OK;
}

fd2_status fd2_sg_set_params(fd2_sg *s, const float *params, int64_t n)
{
    if (!s || !params || n < public_count(s)) return FD2_ERR_INVALID_ARGUMENT;
    std::vector<float> master((size_t)s->n_params, 0.0f);
    for_each_public(s, [&](int64_t k, int64_t i) { master[(size_t)i] = params[k]; });
    return upload_params(s, master);
}

fd2_status fd2_sg_get_hull(fd2_sg *s, fd2_sg_hull *h)
{
    if (!s || !h) return FD2_ERR_INVALID_ARGUMENT;
    *h = s->hull;
    return FD2_OK;
}

fd2_status fd2_sg_set_edge(fd2_sg *s, float amplitude, float length_um)
{
    if (!s || !(amplitude >= 0.0f && amplitude < 1.0f) || !(length_um > 0.0f) || !std::isfinite(length_um))
        return FD2_ERR_INVALID_ARGUMENT;
    s->edge_amp = amplitude;
    s->edge_len_um = length_um;
    return FD2_OK;
}

fd2_status fd2_sg_get_edge(const fd2_sg *s, float *amplitude, float *length_um)
{
    if (!s || !amplitude || !length_um) return FD2_ERR_INVALID_ARGUMENT;
    *amplitude = s->edge_amp;
    *length_um = s->edge_len_um;
    return FD2_OK;
}

fd2_status fd2_sg_set_hull(fd2_sg *s, const fd2_sg_hull *h)
{
    if (!s || !h) return FD2_ERR_INVALID_ARGUMENT;
    for (int i = 0; i < kFeatures; ++i)
        if (!(std::isfinite(h->lo[i]) && std::isfinite(h->hi[i]) && h->hi[i] >= h->lo[i]))
            return FD2_ERR_INVALID_ARGUMENT;
    s->hull = *h;
    if (!s->norm_fixed) {
        // the network's input normalisation comes from its first hull and
        // stays with the network (later hulls only change the routing)
        s->norm_box = *h;
        s->norm_fixed = true;
        set_norm(s);
    }
    if (s->graph) cudaGraphExecDestroy(s->graph);
    s->graph = nullptr;
    return FD2_OK;
}

fd2_status fd2_sg_set_data(fd2_sg *s, const float *features, const int32_t *photons, const int32_t *detected,
                           const uint32_t *radial, int64_t n, int64_t n_val)
{
    if (!s || !features || !photons || !detected || !radial || n <= 0 || n_val < 0 || n_val >= n)
        return FD2_ERR_INVALID_ARGUMENT;
    for (int64_t i = 0; i < n; ++i) {
        if (photons[i] < 0 || detected[i] < 0 || detected[i] > photons[i])
            return sg_fail(s, FD2_ERR_INVALID_ARGUMENT, "label counts out of range");
        for (int f = 0; f < kFeatures; ++f)
            if (!std::isfinite(features[i * kFeatures + f]))
                return sg_fail(s, FD2_ERR_INVALID_ARGUMENT, "non-finite feature");
    }
    // hull = box of the training points
    fd2_sg_hull h;
    for (int f = 0; f < kFeatures; ++f) {
        h.lo[f] = features[f];
        h.hi[f] = features[f];
    }
    const int64_t n_train = n - n_val;
    for (int64_t i = 0; i < n_train; ++i)
        for (int f = 0; f < kFeatures; ++f) {
            h.lo[f] = std::min(h.lo[f], features[i * kFeatures + f]);
            h.hi[f] = std::max(h.hi[f], features[i * kFeatures + f]);
        }
    fd2_status st = fd2_sg_set_hull(s, &h);
    if (st != FD2_OK) return st;
    const size_t N = (size_t)n, nb = (size_t)(s->bins + 1);
    SG_CUDA(s, cudaSetDevice(s->device));
    SG_CUDA(s, alloc(&s->d_feat, N * kFeatures));
    SG_CUDA(s, alloc(&s->d_photons, N));
    SG_CUDA(s, alloc(&s->d_detected, N));
    SG_CUDA(s, alloc(&s->d_radial, N * nb));
    SG_CUDA(s, cudaMemcpy(s->d_feat, features, sizeof(float) * N * kFeatures, cudaMemcpyHostToDevice));
    SG_CUDA(s, cudaMemcpy(s->d_photons, photons, sizeof(int32_t) * N, cudaMemcpyHostToDevice));
    SG_CUDA(s, cudaMemcpy(s->d_detected, detected, sizeof(int32_t) * N, cudaMemcpyHostToDevice));
    SG_CUDA(s, cudaMemcpy(s->d_radial, radial, sizeof(uint32_t) * N * nb, cudaMemcpyHostToDevice));
    s->n_points = n;
    s->n_train = n_train;
    s->n_val = n_val;
    return ensure_rows(s, s->batch);
}

fd2_status fd2_sg_eval(fd2_sg *s, float *loss, float *det_loss, float *radial_loss)
{
    if (!s || s->n_points <= 0) return FD2_ERR_STATE;
    SG_CUDA(s, cudaSetDevice(s->device));
    const int64_t first = s->n_val > 0 ? s->n_train : 0;
    const int64_t count = s->n_val > 0 ? s->n_val : s->n_points;
    fd2_status st = ensure_rows(s, s->batch);
    if (st != FD2_OK) return st;
    SG_CUDA(s, cudaMemsetAsync(s->d_acc, 0, sizeof(double) * 4, s->stream));
    for (int64_t at = 0; at < count; at += s->batch) {
        const int b = (int)std::min<int64_t>(s->batch, count - at);
        gather_kernel<<<grid_for(b, 256), 256, 0, s->stream>>>(s->d_feat, s->d_photons, s->d_detected, s->d_radial,
                                                               s->bins, s->n_train, first + at, b, true, s->seed,
                                                               s->d_step, s->norm, s->x0, s->target, s->ylab,
                                                               s->has_rad);
        SG_CUDA(s, sg_forward(s, s->stream, s->x0, b, nullptr, s->h1, s->h2, s->h3, s->out));
        loss_kernel<<<grid_for(b, 128), 128, 0, s->stream>>>(s->out, kOutPad, s->target, s->ylab, s->has_rad,
                                                             s->bins, (float)s->radial_max, s->lambda, b,
                                                             1.0f, nullptr, s->d_acc);
        SG_CUDA(s, cudaGetLastError());
    }
    double acc[4];
    SG_CUDA(s, cudaMemcpyAsync(acc, s->d_acc, sizeof acc, cudaMemcpyDeviceToHost, s->stream));
    SG_CUDA(s, cudaStreamSynchronize(s->stream));
    if ((st = sg_tc_check(s)) != FD2_OK) return st;
    if (loss) *loss = (float)(acc[0] / (double)count);
    if (det_loss) *det_loss = (float)(acc[1] / (double)count);
    if (radial_loss) *radial_loss = (float)(acc[2] / (double)count);
    return FD2_OK;
}

fd2_status fd2_sg_train(fd2_sg *s, int32_t steps, float *train_loss, float *val_loss)
{
    if (!s || steps < 0) return FD2_ERR_INVALID_ARGUMENT;
    if (s->n_train <= 0) return sg_fail(s, FD2_ERR_STATE, "no training data");
    SG_CUDA(s, cudaSetDevice(s->device));
    fd2_status st = ensure_rows(s, s->batch);
    if (st != FD2_OK) return st;
    if (!s->graph) {
        cudaGraph_t gr = nullptr;
        SG_CUDA(s, cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
        cudaError_t e = train_step(s, s->stream);
        cudaError_t e2 = cudaStreamEndCapture(s->stream, &gr);
        if (e != cudaSuccess || e2 != cudaSuccess) {
            if (gr) cudaGraphDestroy(gr);
            return sg_cuda(s, e != cudaSuccess ? e : e2, "capture training step");
        }
        e = cudaGraphInstantiate(&s->graph, gr, 0);
        cudaGraphDestroy(gr);
        SG_CUDA(s, e);
    }
    // the mean loss of the last min(steps, 50) steps
    const int tail = std::min(steps, 50);
    for (int i = 0; i < steps; ++i) {
        if (i == steps - tail) SG_CUDA(s, cudaMemsetAsync(s->d_acc, 0, sizeof(double) * 4, s->stream));
        SG_CUDA(s, cudaGraphLaunch(s->graph, s->stream));
    }
    double acc[4] = {0, 0, 0, 0};
    SG_CUDA(s, cudaMemcpyAsync(acc, s->d_acc, sizeof acc, cudaMemcpyDeviceToHost, s->stream));
    SG_CUDA(s, cudaStreamSynchronize(s->stream));
    if ((st = sg_tc_check(s)) != FD2_OK) return st;
    if (train_loss) *train_loss = tail > 0 ? (float)(acc[0] / ((double)tail * s->batch)) : 0.0f;
    if (val_loss) {
        st = fd2_sg_eval(s, val_loss, nullptr, nullptr);
        if (st != FD2_OK) return st;
    }
    return FD2_OK;
}

fd2_status fd2_sg_loss_grad(fd2_sg *s, const float *features, const int32_t *photons, const int32_t *detected,
                            const uint32_t *radial, int32_t b, float *loss, float *grad)
{
    if (!s || !features || !photons || !detected || !radial || b <= 0 || b > s->batch)
        return FD2_ERR_INVALID_ARGUMENT;
    SG_CUDA(s, cudaSetDevice(s->device));
    fd2_status st = ensure_rows(s, s->batch);
    if (st != FD2_OK) return st;
    const size_t nb = (size_t)(s->bins + 1);
    float *df = nullptr;
    int32_t *dp = nullptr, *dd = nullptr;
    uint32_t *dr = nullptr;
    cudaError_t e = cudaMalloc(&df, sizeof(float) * b * kFeatures);
    if (e == cudaSuccess) e = cudaMalloc(&dp, sizeof(int32_t) * b);
    if (e == cudaSuccess) e = cudaMalloc(&dd, sizeof(int32_t) * b);
    if (e == cudaSuccess) e = cudaMalloc(&dr, sizeof(uint32_t) * b * nb);
    if (e == cudaSuccess) e = cudaMemcpy(df, features, sizeof(float) * b * kFeatures, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dp, photons, sizeof(int32_t) * b, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dd, detected, sizeof(int32_t) * b, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dr, radial, sizeof(uint32_t) * b * nb, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemsetAsync(s->d_acc, 0, sizeof(double) * 4, s->stream);
    if (e == cudaSuccess) {
        gather_kernel<<<grid_for(b, 256), 256, 0, s->stream>>>(df, dp, dd, dr, s->bins, b, 0, b, true, s->seed,
                                                               s->d_step, s->norm, s->x0, s->target, s->ylab,
                                                               s->has_rad);
        e = sg_forward(s, s->stream, s->x0, b, nullptr, s->h1, s->h2, s->h3, s->out);
    }
    if (e == cudaSuccess) {
        loss_kernel<<<grid_for(b, 128), 128, 0, s->stream>>>(s->out, kOutPad, s->target, s->ylab, s->has_rad,
                                                             s->bins, (float)s->radial_max, s->lambda, b,
                                                             1.0f / (float)b, s->dout, s->d_acc);
        e = backward(s, s->stream, b);
    }
    double acc[4] = {0, 0, 0, 0};
    std::vector<float> g((size_t)s->n_params);
    if (e == cudaSuccess) e = cudaMemcpyAsync(acc, s->d_acc, sizeof acc, cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(g.data(), s->g, sizeof(float) * g.size(), cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    cudaFree(df);
    cudaFree(dp);
    cudaFree(dd);
    cudaFree(dr);
    SG_CUDA(s, e);
    if (fd2_status t = sg_tc_check(s)) return t;
    if (loss) *loss = (float)(acc[0] / b);
    if (grad) for_each_public(s, [&](int64_t k, int64_t i) { grad[k] = g[(size_t)i]; });
    return FD2_OK;
}

fd2_status fd2_sg_predict(fd2_sg *s, const float *features, int64_t n, float *out)
{
    if (!s || !features || !out || n < 0) return FD2_ERR_INVALID_ARGUMENT;
    if (n == 0) return FD2_OK;
    SG_CUDA(s, cudaSetDevice(s->device));
    fd2_status st = ensure_rows(s, s->batch);
    if (st != FD2_OK) return st;
    float *df = nullptr;
    SG_CUDA(s, cudaMalloc(&df, sizeof(float) * (size_t)std::min<int64_t>(n, s->batch) * kFeatures));
    std::vector<float> o((size_t)s->batch * kOutPad);
    cudaError_t e = cudaSuccess;
    for (int64_t at = 0; at < n && e == cudaSuccess; at += s->batch) {
        const int b = (int)std::min<int64_t>(s->batch, n - at);
        e = cudaMemcpyAsync(df, features + at * kFeatures, sizeof(float) * b * kFeatures, cudaMemcpyHostToDevice,
                            s->stream);
        if (e != cudaSuccess) break;
        input_kernel<<<grid_for(b, 256), 256, 0, s->stream>>>(df, b, s->norm, s->x0);
        e = sg_forward(s, s->stream, s->x0, b, nullptr, s->h1, s->h2, s->h3, s->out);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(o.data(), s->out, sizeof(float) * b * kOutPad, cudaMemcpyDeviceToHost, s->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
        if (e == cudaSuccess)
            for (int r = 0; r < b; ++r)
                for (int k = 0; k < kOutputs; ++k) out[(at + r) * kOutputs + k] = o[(size_t)r * kOutPad + k];
    }
    cudaFree(df);
    SG_CUDA(s, e);
    return sg_tc_check(s);
}

// File: "FD2SG002", hidden, bins, radial_max, normalisation box, routing
// hull, public parameters; then, optionally, "EDGE" and the edge survival's
// amplitude and length (float each; a file without them loads amplitude 0).
fd2_status fd2_sg_save(fd2_sg *s, const char *path)
{
    if (!s || !path) return FD2_ERR_INVALID_ARGUMENT;
    std::vector<float> p((size_t)public_count(s));
    fd2_status st = fd2_sg_get_params(s, p.data(), (int64_t)p.size());
    if (st != FD2_OK) return st;
    FILE *f = std::fopen(path, "wb");
    if (!f) return sg_fail(s, FD2_ERR_IO, std::string("cannot write ") + path);
    const int32_t hdr[2] = {s->hidden, s->bins};
    bool ok = std::fwrite("FD2SG002", 1, 8, f) == 8 && std::fwrite(hdr, sizeof hdr, 1, f) == 1 &&
              std::fwrite(&s->radial_max, sizeof(double), 1, f) == 1 &&
              std::fwrite(&s->norm_box, sizeof s->norm_box, 1, f) == 1 &&
              std::fwrite(&s->hull, sizeof s->hull, 1, f) == 1 &&
              std::fwrite(p.data(), sizeof(float), p.size(), f) == p.size();
    if (s->edge_amp > 0.0f) {
        const float edge[2] = {s->edge_amp, s->edge_len_um};
        ok = ok && std::fwrite("EDGE", 1, 4, f) == 4 && std::fwrite(edge, sizeof edge, 1, f) == 1;
    }
    ok = (std::fclose(f) == 0) && ok;
    return ok ? FD2_OK : sg_fail(s, FD2_ERR_IO, std::string("write failed: ") + path);
}

fd2_status fd2_sg_load(fd2_sg *s, const char *path)
{
    if (!s || !path) return FD2_ERR_INVALID_ARGUMENT;
    FILE *f = std::fopen(path, "rb");
    if (!f) return sg_fail(s, FD2_ERR_IO, std::string("cannot read ") + path);
    char magic[8];
    int32_t hdr[2];
    double rmax = 0;
    fd2_sg_hull nb, h;
    std::vector<float> p((size_t)public_count(s));
    bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, "FD2SG002", 8) == 0 &&
              std::fread(hdr, sizeof hdr, 1, f) == 1 && std::fread(&rmax, sizeof rmax, 1, f) == 1 &&
              std::fread(&nb, sizeof nb, 1, f) == 1 && std::fread(&h, sizeof h, 1, f) == 1;
    ok = ok && hdr[0] == s->hidden && hdr[1] == s->bins && rmax == s->radial_max &&
         std::fread(p.data(), sizeof(float), p.size(), f) == p.size();
    float edge[2] = {0.0f, 1.0f};
    char tag[4];
    if (ok && std::fread(tag, 1, 4, f) == 4) {
        ok = std::memcmp(tag, "EDGE", 4) == 0 && std::fread(edge, sizeof edge, 1, f) == 1 && edge[0] >= 0.0f &&
             edge[0] < 1.0f && edge[1] > 0.0f;
    }
    std::fclose(f);
    if (!ok) return sg_fail(s, FD2_ERR_IO, std::string("not a matching surrogate file: ") + path);
    s->edge_amp = edge[0];
    s->edge_len_um = edge[1];
    fd2_status st = fd2_sg_set_params(s, p.data(), (int64_t)p.size());
    if (st != FD2_OK) return st;
    s->norm_box = nb;
    s->norm_fixed = true;
    set_norm(s);
    return fd2_sg_set_hull(s, &h);
}

}  // extern "C"
