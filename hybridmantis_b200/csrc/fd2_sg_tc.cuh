// fd2_sg_tc.cuh -- the surrogate's GEMMs on the 5th-generation tensor cores:
// tcgen05.mma with the accumulator in tensor memory (TMEM).
//
// C[M x N] = A[M x K] B[N x K]^T (both operands K-contiguous, BF16), FP32
// accumulation, epilogue bias + ReLU to BF16, bias to FP32, ReLU mask to
// BF16 or plain FP32 -- the four forward products of the MLP (kc x kc in
// fd2_sg_gemm.cuh) and, with the weights and the batch-major operands
// transposed first, the backward products: input gradients dY W (mask
// epilogue) and weight gradients dY^T X split over 256-row slices of the
// batch (blockIdx.y = slice, FP32 partial planes).  Two kernels: the
// pipelined one (gemm_tc_pipe_kernel, below; the default) and this simple
// one (gemm_tc_kernel), whose persistent CTAs of four warps (at most one
// per SM) walk the 128-row tiles, the whole contraction of a tile in one
// pass:
//   1. the CTA stages all of B (N x K) once and, per tile, its A tile
//      (128 x K) in shared memory (cp.async, all copies in flight together)
//      in the canonical
//      no-swizzle K-major layout of the UMMA descriptors: 8-row x 16-byte
//      core matrices, 128 bytes each, the 8-row groups of one 16-byte K
//      chunk contiguous (stride 128 B, the descriptor's SBO) and successive
//      K chunks `rows x 16` bytes apart (its LBO);
//   2. warp 0 allocates N (rounded up to a power of two >= 32) TMEM columns
//      once for the CTA;
//   3. one thread issues K/16 tcgen05.mma.cta_group::1.kind::f16 (M = 128,
//      N, K = 16 each), advancing both descriptors' start addresses by two
//      K chunks per instruction, and commits them to an mbarrier;
//   4. every warp waits on the mbarrier (bounded; one phase per tile), reads
//      its 32 TMEM lanes (rows) with tcgen05.ld 32x32b.x16 and applies the
//      epilogue;
//   5. after the last tile warp 0 frees the TMEM columns.
// Bit layouts of the shared-memory and instruction descriptors follow the
// PTX ISA's tcgen05 matrix-descriptor and instruction-descriptor formats for
// kind::f16 (as CUTLASS's cute/arch/mma_sm100_desc.hpp spells them out).
// Requirements: K % 16 == 0, K <= 256; N % 16 == 0, 16 <= N <= 256; row
// strides multiples of 8 elements.  Rows past M or past *m_limit are
// zero-filled and not stored.  The simple kernel stages its operands with
// 16-byte cp.async copies; the pipelined one uses TMA where it can (below).
// No load multicasts, and every tensor map covers this GPU's memory.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cstdint>

#include "fd2_sg_gemm.cuh"

namespace fd2 {
namespace sg {

constexpr int kTcRows = 128;
constexpr int kTcThreads = 128;
constexpr int kTcMaxK = 256, kTcMaxN = 256;
// bounded waits: the MMAs of one tile take microseconds
constexpr long long kTcWaitSpins = 1LL << 22;

struct TcArgs {
    const __nv_bfloat16 *A;
    const __nv_bfloat16 *B;
    int lda, ldb, M, N, K;
    const int *m_limit;
    int epi;  // kEpiBiasReluBf16, kEpiBiasF32, kEpiMaskBf16 or kEpiPartialF32
    const float *bias;
    const __nv_bfloat16 *mask;  // kEpiMaskBf16: out = acc * (mask[row][col] > 0)
    int ldm;
    void *C;
    int ldc;
    long long a_split, b_split, c_split;  // element offsets of slice blockIdx.y
    unsigned *fault;  // set when a wait gives up (the tile is then not stored)
    // pipelined kernel: stage A and B with TMA (no slices) through these maps
    // of A (K x M rows) and B (K x N rows).  tma == 1: boxes of 8 K-elements
    // (one 16-byte column of the no-swizzle canonical layout) by 128 rows (A)
    // or N rows (B); tma == 2 (K a multiple of 64): boxes of 64 K-elements
    // (128-byte rows) with the 128-byte swizzle, the K-major SWIZZLE_128B
    // layout of the UMMA descriptors
    int tma;
    CUtensorMap tmap_a, tmap_b;
    // pipelined kernel, BF16 epilogues staged through shared memory: store
    // each warp's 32-row x 64-column output block with one TMA store through
    // this map of C (M rows x N, boxes of 64 columns x 32 rows, 128-byte
    // swizzle: the layout of the staging tile)
    int tma_store;
    CUtensorMap tmap_c;
};

// Dynamic shared memory of one CTA: A tile + B.
__host__ __device__ inline size_t tc_smem_bytes(int N, int K)
{
    return (size_t)(kTcRows + N) * (size_t)K * sizeof(__nv_bfloat16);
}

__device__ __forceinline__ uint64_t tc_smem_desc(uint32_t addr, uint32_t lbo_bytes, uint32_t sbo_bytes)
{
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFFu);              // start address, 16-byte units, bits [0,14)
    d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;   // leading-dimension byte offset, bits [16,30)
    d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;   // stride-dimension byte offset, bits [32,46)
    d |= (uint64_t)1 << 46;                              // descriptor version for sm_100, bits [46,48)
    // base offset 0, legacy LBO mode, layout type 0 = no swizzle (bits [61,64))
    return d;
}

// K-major SWIZZLE_128B: rows of 64 BF16 K-elements (128 bytes, their 16-byte
// pieces XOR-permuted by row mod 8, as the TMA's 128-byte swizzle writes
// them), 8-row groups 1024 bytes apart (SBO); the leading offset is unused
// (1).  The groups start on 1024-byte boundaries; a K step of 16 elements
// inside the 128-byte row advances the start address by 32 bytes.
__device__ __forceinline__ uint64_t tc_smem_desc_sw128(uint32_t addr)
{
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)1 << 16;            // LBO (unused), 16-byte units
    d |= (uint64_t)(1024 >> 4) << 32;  // SBO
    d |= (uint64_t)1 << 46;            // descriptor version for sm_100
    d |= (uint64_t)2 << 61;            // layout type 2 = SWIZZLE_128B
    return d;
}

__host__ __device__ constexpr uint32_t tc_instr_desc(int M, int N)
{
    return (1u << 4)                      // D format: F32
           | (1u << 7)                    // A format: BF16
           | (1u << 10)                   // B format: BF16
           | ((uint32_t)(N >> 3) << 17)   // N / 8
           | ((uint32_t)(M >> 4) << 24);  // M / 16; A and B K-major (bits 15, 16 = 0)
}

__device__ __forceinline__ bool tc_wait(uint32_t mbar, uint32_t parity)
{
    for (long long i = 0; i < kTcWaitSpins; ++i) {
        uint32_t done = 0;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (done) return true;
        if (i > 64) __nanosleep(64);
    }
    return false;
}

// Stage rows [0, rows) of a K-contiguous matrix (row stride ld) into the
// canonical layout at `dst` with asynchronous 16-byte copies (all of a
// thread's copies in flight at once); rows >= valid are zero-filled (a copy
// of 0 source bytes).  Consecutive threads take 8 rows of one K chunk (128
// contiguous bytes of shared memory), then the next chunks of the same rows.
__device__ __forceinline__ void tc_stage(unsigned char *dst, const __nv_bfloat16 *src, int ld, int rows, int valid,
                                         int K)
{
    const int kc = K / 8;  // 16-byte chunks per row
    const int total = rows * kc;
    for (int L = threadIdx.x; L < total; L += blockDim.x) {
        const int ri = L & 7, t = L >> 3;
        const int c = t % kc, rg = t / kc;
        const int r = rg * 8 + ri;
        const bool ok = r < valid;
        const __nv_bfloat16 *g = src + (long long)(ok ? r : 0) * ld + c * 8;
        const uint32_t s = (uint32_t)__cvta_generic_to_shared(dst + (size_t)c * rows * 16 + (size_t)rg * 128 +
                                                              (size_t)ri * 16);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(s), "l"(g), "r"(ok ? 16 : 0) : "memory");
    }
}

template <int kEpi>
__global__ void __launch_bounds__(kTcThreads, 1) gemm_tc_kernel(const TcArgs g)
{
    extern __shared__ __align__(1024) unsigned char tc_smem[];
    __shared__ __align__(8) unsigned long long s_mbar;
    __shared__ uint32_t s_taddr;
    __shared__ int s_ok;

    int M = g.M;
    if (g.m_limit) M = min(M, *g.m_limit);
    const int ntiles = (M + kTcRows - 1) / kTcRows;
    if ((int)blockIdx.x >= ntiles) return;  // whole CTA, before any TMEM or barrier use
    const int N = g.N, K = g.K;
    const __nv_bfloat16 *gA = g.A + (long long)blockIdx.y * g.a_split;
    const __nv_bfloat16 *gB = g.B + (long long)blockIdx.y * g.b_split;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned char *sA = tc_smem;
    unsigned char *sB = tc_smem + (size_t)kTcRows * K * 2;
    const uint32_t cols = N <= 32 ? 32u : N <= 64 ? 64u : N <= 128 ? 128u : 256u;

    // TMEM columns (warp 0) and the completion barrier (thread 0), once
    if (warp == 0) {
        const uint32_t dst = (uint32_t)__cvta_generic_to_shared(&s_taddr);
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst), "r"(cols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    const uint32_t mbar = (uint32_t)__cvta_generic_to_shared(&s_mbar);
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
        s_ok = 1;
    }
    // B stays resident for all of the CTA's tiles
    tc_stage(sB, gB, g.ldb, N, N, K);
    const uint32_t idesc = tc_instr_desc(kTcRows, N);
    const uint32_t lbo_a = kTcRows * 16, lbo_b = (uint32_t)N * 16;
    uint32_t taddr = 0;
    int it = 0;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++it) {
        const int m0 = tile * kTcRows;
        const int valid = min(kTcRows, M - m0);
        tc_stage(sA, gA + (long long)m0 * g.lda, g.lda, kTcRows, valid, K);
        asm volatile("cp.async.wait_all;" ::: "memory");
        // the staged operands become visible to the tensor core's (async)
        // proxy; the previous tile's TMEM reads are ordered before the MMAs
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        taddr = s_taddr;
        if (threadIdx.x == 0) {
            const uint32_t a0 = (uint32_t)__cvta_generic_to_shared(sA);
            const uint32_t b0 = (uint32_t)__cvta_generic_to_shared(sB);
            for (int s = 0; s < K / 16; ++s) {
                // K step s: 16-byte K chunks 2s and 2s+1
                const uint64_t da = tc_smem_desc(a0 + 2u * s * lbo_a, lbo_a, 128);
                const uint64_t db = tc_smem_desc(b0 + 2u * s * lbo_b, lbo_b, 128);
                const uint32_t acc = s > 0 ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
                    :
                    : "r"(taddr), "l"(da), "l"(db), "r"(idesc), "r"(acc)
                    : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                         : "memory");
        }
        __syncwarp();
        // the barrier completes one phase per tile
        if (!tc_wait(mbar, (uint32_t)(it & 1))) {
            s_ok = 0;
            if (g.fault) atomicOr(g.fault, 1u);
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        __syncthreads();
        if (!s_ok) {
            // the MMAs may still be running: give them another bounded wait
            // before their accumulator columns are freed
            tc_wait(mbar, (uint32_t)(it & 1));
            break;
        }
        // epilogue: warp w owns TMEM lanes (tile rows) 32w .. 32w + 31
        const int r = warp * 32 + lane;
        const long long row = (long long)m0 + r;
        for (int c0 = 0; c0 < N; c0 += 16) {
            uint32_t v[16];
            const uint32_t src = taddr + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                "%13, %14, %15}, [%16];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                  "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                  "=r"(v[15])
                : "r"(src));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (r < valid) {
                float f[16];
#pragma unroll
                for (int j = 0; j < 16; ++j)
                    f[j] = __uint_as_float(v[j]) + ((kEpi == kEpiBiasReluBf16 || kEpi == kEpiBiasF32) ? g.bias[c0 + j] : 0.0f);
                if (kEpi == kEpiBiasReluBf16 || kEpi == kEpiMaskBf16) {
                    __align__(16) __nv_bfloat16 o[16];
                    if (kEpi == kEpiBiasReluBf16) {
#pragma unroll
                        for (int j = 0; j < 16; ++j) o[j] = __float2bfloat16(fmaxf(f[j], 0.0f));
                    } else {
                        __align__(16) __nv_bfloat16 mk[16];
                        const uint4 *ms = reinterpret_cast<const uint4 *>(g.mask + row * g.ldm + c0);
                        reinterpret_cast<uint4 *>(mk)[0] = ms[0];
                        reinterpret_cast<uint4 *>(mk)[1] = ms[1];
#pragma unroll
                        for (int j = 0; j < 16; ++j)
                            o[j] = __float2bfloat16(__bfloat162float(mk[j]) > 0.0f ? f[j] : 0.0f);
                    }
                    uint4 *dst = reinterpret_cast<uint4 *>(static_cast<__nv_bfloat16 *>(g.C) + row * g.ldc + c0);
                    dst[0] = reinterpret_cast<const uint4 *>(o)[0];
                    dst[1] = reinterpret_cast<const uint4 *>(o)[1];
                } else {
                    float4 *dst = reinterpret_cast<float4 *>(static_cast<float *>(g.C) + (long long)blockIdx.y * g.c_split +
                                                             row * g.ldc + c0);
#pragma unroll
                    for (int j = 0; j < 4; ++j) dst[j] = make_float4(f[4 * j], f[4 * j + 1], f[4 * j + 2], f[4 * j + 3]);
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols));
}


// ---------------------------------------------------------------------------
// Pipelined variant: the same products with the stages of consecutive tiles
// overlapped.  Eleven warps with fixed roles:
//   warps 4-5 (producers): stage A in 128-row x 64-K chunks (16 KB) into a ring
//     of four shared-memory stages, waiting on a stage's `empty` barrier
//     (the MMAs that read it have completed) before reuse.  With TMA (no
//     batch slices) one thread loads each chunk, arming the stage's `full`
//     barrier with its bytes: one box of 64 K-elements x 128 rows in the
//     128-byte swizzled layout where K is a multiple of 64, else one
//     16-byte column box per 8 K-elements; B likewise, once, on its own
//     barrier.  Otherwise both warps copy with cp.async, three chunks in
//     flight, and mark a chunk full (after fence.proxy.async) once its
//     copies have completed;
//   warp 6 (one elected thread): issues the tcgen05.mma of each chunk as soon
//     as its stage is full, commits each stage to its `empty` barrier and each
//     finished tile to its accumulator's `accf` barrier; two TMEM
//     accumulators alternate between tiles, and a tile starts only when the
//     epilogue has released its accumulator (`acce`);
//   warps 0-3 and 7-10 (epilogue): warp w drains TMEM lanes 32 (w mod 4) ..
//     32 (w mod 4) + 31 (the lanes its position in the warpgroup may read)
//     of a finished accumulator, warps 0-3 the even 64-column blocks and
//     warps 7-10 the odd ones (tcgen05.ld, four loads of 16 columns in flight
//     per wait), apply the epilogue (bias from shared memory), store, release
//     the accumulator: two warps per scheduler, so that one's loads and
//     stores overlap the other's arithmetic.
//     BF16 outputs (and the ReLU mask they read) pass through a 32-row x
//     128-byte tile per warp in shared memory, its 16-byte pieces XOR-swizzled
//     by row so that neither the row-per-lane side nor the coalesced side has
//     bank conflicts; that permutation is the TMA's 128-byte swizzle, so a
//     warp whose 32 rows are all valid stores the tile with one TMA store,
//     the others with coalesced 16-byte stores of whole 128-byte rows.
// So the loads of the next chunks and the epilogue of the previous tile run
// while the tensor core works.  B stays resident as before.  Every wait is
// bounded (tc_wait); a role that gives up sets the fault word and leaves its
// loop, the others' waits then run out too, and before the columns are
// freed the MMA thread waits (bounded) for everything it issued.  The
// MMAs are the simple kernel's, in the same order, so the results are
// bitwise identical to it.
constexpr int kPipeStages = 4;
constexpr int kPipeDepth = 3;  // chunks a producer lane keeps in flight (< kPipeStages)
constexpr int kPipeProducers = 2;  // producer warps
constexpr int kPipeEpiWarps = 8;  // epilogue warps: two per TMEM lane quadrant
constexpr int kPipeThreads = 32 * (kPipeEpiWarps + kPipeProducers + 1);  // epilogue, producers, 1 MMA warp
constexpr int kPipeMmaWarp = 4 + kPipeProducers;  // warps 0-3 epilogue, 4-5 producers, 6 MMA, 7-10 epilogue
constexpr int kPipeChunkK = 64;

__host__ __device__ inline int tc_pipe_chunk(int K) { return K < kPipeChunkK ? K : kPipeChunkK; }

constexpr int kPipeOutBytes = 32 * 128;  // an epilogue warp's output tile: 32 rows x 64 BF16 columns

// Dynamic shared memory of one CTA: B + the A ring + the epilogue warps'
// output tiles, from the first 1024-byte boundary (the swizzled layout's).
__host__ __device__ inline size_t tc_pipe_smem_bytes(int N, int K)
{
    return 1024 + (size_t)N * (size_t)K * sizeof(__nv_bfloat16) +
           (size_t)kPipeStages * kTcRows * (size_t)tc_pipe_chunk(K) * sizeof(__nv_bfloat16) + kPipeEpiWarps * kPipeOutBytes;
}

// 16 TMEM columns of the warp's 32 lanes (no wait).
__device__ __forceinline__ void tc_ld16(uint32_t src, uint32_t *v)
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
        "%13, %14, %15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(src));
}

// Byte offset of 16-byte piece c (0-7) of row r in a warp's output tile.
__device__ __forceinline__ uint32_t tc_out_off(int r, int c) { return (uint32_t)(r * 128 + ((c ^ (r & 7)) << 4)); }

// tc_stage for thread `tid` of `nthr` (a subset of the CTA).
__device__ __forceinline__ void tc_stage_part(unsigned char *dst, const __nv_bfloat16 *src, int ld, int rows,
                                              int valid, int K, int tid, int nthr)
{
    const int kc = K / 8;
    const int total = rows * kc;
    for (int L = tid; L < total; L += nthr) {
        const int ri = L & 7, t = L >> 3;
        const int c = t % kc, rg = t / kc;
        const int r = rg * 8 + ri;
        const bool ok = r < valid;
        const __nv_bfloat16 *g = src + (long long)(ok ? r : 0) * ld + c * 8;
        const uint32_t sa = (uint32_t)__cvta_generic_to_shared(dst + (size_t)c * rows * 16 + (size_t)rg * 128 +
                                                               (size_t)ri * 16);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(sa), "l"(g), "r"(ok ? 16 : 0) : "memory");
    }
}

__device__ __forceinline__ void tc_mbar_init(uint32_t bar, int count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void tc_mbar_arrive(uint32_t bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// TMA: one 2D box into shared memory, completing on `bar` by its bytes.
__device__ __forceinline__ void tc_tma_load(uint32_t dst, const CUtensorMap *map, int x, int y, uint32_t bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

// TMA: one 2D box from shared memory to global memory (bulk group).
__device__ __forceinline__ void tc_tma_store(const CUtensorMap *map, int x, int y, uint32_t src)
{
    asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];" ::"l"(
                     reinterpret_cast<uint64_t>(map)),
                 "r"(x), "r"(y), "r"(src)
                 : "memory");
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}

// Arrive on `bar` and add `bytes` to the transfers its phase waits for.
__device__ __forceinline__ void tc_expect_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void tc_commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

// One 128-row chunk of A (kc = CK / 8 16-byte pieces per row, a power of two)
// by the producer threads `tid` of `nthr` (a multiple of 8): the same layout
// as tc_stage, with shifts instead of divisions.
__device__ __forceinline__ void tc_stage_chunk(unsigned char *dst, const __nv_bfloat16 *src, int ld, int valid, int kc,
                                               int lg_kc, int tid, int nthr)
{
    const int ri = tid & 7;  // fixed for the thread: nthr is a multiple of 8
    const int total = kTcRows * kc;
    for (int L = tid; L < total; L += nthr) {
        const int t = L >> 3;
        const int c = t & (kc - 1), rg = t >> lg_kc;
        const int r = rg * 8 + ri;
        const bool ok = r < valid;
        const __nv_bfloat16 *gp = src + (long long)(ok ? r : 0) * ld + c * 8;
        const uint32_t sa = (uint32_t)__cvta_generic_to_shared(dst + (size_t)c * (kTcRows * 16) + (size_t)rg * 128 +
                                                               (size_t)ri * 16);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(sa), "l"(gp), "r"(ok ? 16 : 0) : "memory");
    }
}

template <int kEpi>
__global__ void __launch_bounds__(kPipeThreads, 1) gemm_tc_pipe_kernel(const __grid_constant__ TcArgs g)
{
    extern __shared__ __align__(1024) unsigned char tc_smem[];
    __shared__ __align__(8) unsigned long long s_full[kPipeStages], s_empty[kPipeStages], s_accf[2], s_acce[2],
        s_drain, s_bfull;
    __shared__ uint32_t s_taddr;
    __shared__ int s_fault;
    __shared__ __align__(16) float s_bias[kTcMaxN];
    constexpr bool kBias = kEpi == kEpiBiasReluBf16 || kEpi == kEpiBiasF32;

    int M = g.M;
    if (g.m_limit) M = min(M, *g.m_limit);
    const int ntiles = (M + kTcRows - 1) / kTcRows;
    if ((int)blockIdx.x >= ntiles) return;  // whole CTA, before any TMEM or barrier use
    const int N = g.N, K = g.K;
    const int CK = tc_pipe_chunk(K), nck = K / CK;
    const __nv_bfloat16 *gA = g.A + (long long)blockIdx.y * g.a_split;
    const __nv_bfloat16 *gB = g.B + (long long)blockIdx.y * g.b_split;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // B, then the ring, from a 1024-byte boundary: every swizzled block
    // (B's 64-element K chunks, the ring's stages) starts on one
    unsigned char *sB = tc_smem + ((1024u - ((uint32_t)__cvta_generic_to_shared(tc_smem) & 1023u)) & 1023u);
    unsigned char *sRing = sB + (size_t)N * K * 2;
    const uint32_t stage_bytes = (uint32_t)(kTcRows * CK * 2);
    unsigned char *sOut = sRing + (size_t)kPipeStages * stage_bytes;
    const uint32_t acc_cols = N <= 32 ? 32u : N <= 64 ? 64u : N <= 128 ? 128u : 256u;
    const uint32_t cols = 2u * acc_cols;

    if (warp == 0) {
        const uint32_t dst = (uint32_t)__cvta_generic_to_shared(&s_taddr);
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst), "r"(cols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    const uint32_t full0 = (uint32_t)__cvta_generic_to_shared(&s_full[0]);
    const uint32_t empty0 = (uint32_t)__cvta_generic_to_shared(&s_empty[0]);
    const uint32_t accf0 = (uint32_t)__cvta_generic_to_shared(&s_accf[0]);
    const uint32_t acce0 = (uint32_t)__cvta_generic_to_shared(&s_acce[0]);
    const uint32_t drain = (uint32_t)__cvta_generic_to_shared(&s_drain);
    const uint32_t bfull = (uint32_t)__cvta_generic_to_shared(&s_bfull);
    const bool tma = g.tma != 0;
    const bool sw = g.tma == 2;  // SWIZZLE_128B boxes and descriptors (CK == 64)
    if (threadIdx.x == 0) {
        for (int i = 0; i < kPipeStages; ++i) {
            // the producer lanes, or (TMA) one arrive with the stage's bytes
            tc_mbar_init(full0 + 8u * i, tma ? 1 : 32 * kPipeProducers);
            tc_mbar_init(empty0 + 8u * i, 1);  // one tcgen05.commit
        }
        for (int i = 0; i < 2; ++i) {
            tc_mbar_init(accf0 + 8u * i, 1);   // one tcgen05.commit
            tc_mbar_init(acce0 + 8u * i, kPipeEpiWarps);  // one arrive per epilogue warp
        }
        tc_mbar_init(drain, 1);
        tc_mbar_init(bfull, 1);
        s_fault = 0;
        if (tma) {
            // B (resident for all of the CTA's tiles) by TMA, one 16-byte K
            // column of all N rows per box; only the MMA thread waits for it
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
            tc_expect_tx(bfull, (uint32_t)(N * K * 2));
            const uint32_t b0 = (uint32_t)__cvta_generic_to_shared(sB);
            if (sw)  // one box per 64-element K chunk: N rows of 128 bytes
                for (int c = 0; c < K / 64; ++c) tc_tma_load(b0 + (uint32_t)(c * N * 128), &g.tmap_b, c * 64, 0, bfull);
            else
                for (int c = 0; c < K / 8; ++c) tc_tma_load(b0 + (uint32_t)(c * N * 16), &g.tmap_b, c * 8, 0, bfull);
        }
    }
    // B stays resident for all of the CTA's tiles
    if (!tma) tc_stage_part(sB, gB, g.ldb, N, N, K, threadIdx.x, blockDim.x);
    for (int i = threadIdx.x; i < N; i += blockDim.x) s_bias[i] = kBias ? g.bias[i] : 0.0f;
    asm volatile("cp.async.wait_all;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t taddr = s_taddr;

    if (tma && warp >= 4 && warp < kPipeMmaWarp) {
        // ---- producer (TMA): one thread; per chunk, once its stage is free,
        // the stage's byte count on its `full` barrier and one box per 16-byte
        // K column (rows past M arrive as zeros)
        if (warp == 4 && lane == 0) {
            int gc = 0;
            bool ok = true;
            const uint32_t r0 = (uint32_t)__cvta_generic_to_shared(sRing);
            for (int tile = blockIdx.x; ok && tile < ntiles; tile += gridDim.x) {
                const int m0 = tile * kTcRows;
                for (int c = 0; c < nck; ++c, ++gc) {
                    const int st = gc % kPipeStages;
                    const uint32_t ph = (uint32_t)((gc / kPipeStages) & 1);
                    if (!tc_wait(empty0 + 8u * st, ph ^ 1u)) {
                        ok = false;
                        s_fault = 1;
                        if (g.fault) atomicOr(g.fault, 1u);
                        break;
                    }
                    const uint32_t dst = r0 + (uint32_t)st * stage_bytes;
                    tc_expect_tx(full0 + 8u * st, stage_bytes);
                    if (sw)
                        tc_tma_load(dst, &g.tmap_a, c * CK, m0, full0 + 8u * st);
                    else
                        for (int j = 0; j < CK / 8; ++j)
                            tc_tma_load(dst + (uint32_t)(j * kTcRows * 16), &g.tmap_a, c * CK + j * 8, m0,
                                        full0 + 8u * st);
                }
            }
        }
        __syncwarp();
    } else if (warp >= 4 && warp < kPipeMmaWarp) {
        // ---- producers: up to kPipeDepth chunks' copies in flight per lane
        // (cp.async groups); a chunk's stage is marked full once its group
        // has completed and a proxy fence has made the writes visible to the
        // tensor core
        int gc = 0;
        bool ok = true;
        for (int tile = blockIdx.x; ok && tile < ntiles; tile += gridDim.x) {
            const int m0 = tile * kTcRows;
            const int valid = min(kTcRows, M - m0);
            for (int c = 0; c < nck; ++c, ++gc) {
                const int st = gc % kPipeStages;
                const uint32_t ph = (uint32_t)((gc / kPipeStages) & 1);
                // the warp's lanes agree on the outcome of the (bounded) wait
                ok = __all_sync(0xFFFFFFFFu, tc_wait(empty0 + 8u * st, ph ^ 1u));
                if (!ok) {
                    if (lane == 0) {
                        s_fault = 1;
                        if (g.fault) atomicOr(g.fault, 1u);
                    }
                    break;
                }
                tc_stage_chunk(sRing + (size_t)st * stage_bytes, gA + (long long)m0 * g.lda + c * CK, g.lda, valid,
                               CK / 8, __ffs(CK / 8) - 1, threadIdx.x - 128, 32 * kPipeProducers);
                asm volatile("cp.async.commit_group;" ::: "memory");
                if (gc >= kPipeDepth - 1) {
                    // chunk gc - (depth - 1) has landed
                    asm volatile("cp.async.wait_group %0;" ::"n"(kPipeDepth - 1) : "memory");
                    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                    tc_mbar_arrive(full0 + 8u * ((gc - (kPipeDepth - 1)) % kPipeStages));
                }
            }
        }
        // the chunks still in flight
        asm volatile("cp.async.wait_group 0;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        for (int j = max(gc - (kPipeDepth - 1), 0); j < gc; ++j) tc_mbar_arrive(full0 + 8u * (j % kPipeStages));
    } else if (warp == kPipeMmaWarp) {
        // ---- MMA issue (one thread)
        if (lane == 0) {
            const uint32_t idesc = tc_instr_desc(kTcRows, N);
            const uint32_t lbo_a = kTcRows * 16, lbo_b = (uint32_t)N * 16;
            const uint32_t b0 = (uint32_t)__cvta_generic_to_shared(sB);
            const uint32_t r0 = (uint32_t)__cvta_generic_to_shared(sRing);
            int gc = 0, it = 0;
            bool ok = true;
            if (tma && !tc_wait(bfull, 0u)) ok = false;  // B by TMA
            for (int tile = blockIdx.x; ok && tile < ntiles; tile += gridDim.x, ++it) {
                const int a = it & 1;
                if (!tc_wait(acce0 + 8u * a, (uint32_t)((it >> 1) & 1) ^ 1u)) {
                    ok = false;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t d = taddr + (uint32_t)a * acc_cols;
                for (int c = 0; c < nck; ++c, ++gc) {
                    const int st = gc % kPipeStages;
                    if (!tc_wait(full0 + 8u * st, (uint32_t)((gc / kPipeStages) & 1))) {
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint32_t a0 = r0 + (uint32_t)st * stage_bytes;
                    for (int kk = 0; kk < CK / 16; ++kk) {
                        const uint64_t da = sw ? tc_smem_desc_sw128(a0 + 32u * kk)
                                               : tc_smem_desc(a0 + 2u * kk * lbo_a, lbo_a, 128);
                        const uint64_t db = sw ? tc_smem_desc_sw128(b0 + (uint32_t)(c * N * 128) + 32u * kk)
                                               : tc_smem_desc(b0 + (uint32_t)(c * (CK / 8) + 2 * kk) * lbo_b, lbo_b, 128);
                        const uint32_t acc = (c > 0 || kk > 0) ? 1u : 0u;
                        asm volatile(
                            "{\n\t.reg .pred p;\n\t"
                            "setp.ne.b32 p, %4, 0;\n\t"
                            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
                            :
                            : "r"(d), "l"(da), "l"(db), "r"(idesc), "r"(acc)
                            : "memory");
                    }
                    tc_commit(empty0 + 8u * st);  // the stage is free once these MMAs have read it
                }
                if (!ok) break;
                tc_commit(accf0 + 8u * a);  // the tile's accumulator is complete
            }
            if (!ok) {
                s_fault = 1;
                if (g.fault) atomicOr(g.fault, 1u);
            }
            // everything issued has completed before the columns can be freed
            tc_commit(drain);
            if (!tc_wait(drain, 0u)) {
                s_fault = 1;
                if (g.fault) atomicOr(g.fault, 1u);
            }
        }
        __syncwarp();
    } else {
        // ---- epilogue: warp w drains TMEM lanes (tile rows) 32q .. 32q + 31,
        // q = w mod 4, columns of blocks h, h + 2, ... (h = 0 for warps 0-3,
        // 1 for warps 7-10), through output tile e of shared memory
        const int q = warp & 3, h = warp < 4 ? 0 : 1, e = warp < 4 ? warp : warp - 3;
        int it = 0;
        for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++it) {
            const int a = it & 1;
            // the warp's lanes agree on the outcome (tcgen05.ld below is warp-wide)
            if (!__all_sync(0xFFFFFFFFu, tc_wait(accf0 + 8u * a, (uint32_t)((it >> 1) & 1)))) {
                if (lane == 0) {
                    s_fault = 1;
                    if (g.fault) atomicOr(g.fault, 1u);
                }
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const int m0 = tile * kTcRows;
            const int valid = min(kTcRows, M - m0);
            const int r = q * 32 + lane;
            const long long row = (long long)m0 + r;
            const uint32_t tsrc = taddr + ((uint32_t)(q * 32) << 16) + (uint32_t)a * acc_cols;
            if ((kEpi == kEpiBiasReluBf16 || kEpi == kEpiMaskBf16) && (N & 63) == 0) {
                // 64 columns at a time through the warp's output tile; a warp
                // whose 32 rows are all valid stores it with one TMA store
                unsigned char *out = sOut + (size_t)e * kPipeOutBytes;
                const bool bulk = g.tma_store && q * 32 + 32 <= valid;
                for (int c0 = 64 * h; c0 < N; c0 += 128) {
                    // the previous block's TMA store has read the tile
                    if (lane == 0) asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
                    __syncwarp();
                    uint32_t v[64];
                    tc_ld16(tsrc + (uint32_t)c0, v);
                    tc_ld16(tsrc + (uint32_t)c0 + 16u, v + 16);
                    tc_ld16(tsrc + (uint32_t)c0 + 32u, v + 32);
                    tc_ld16(tsrc + (uint32_t)c0 + 48u, v + 48);
                    if (kEpi == kEpiMaskBf16) {
                        // the mask's 32 x 64 block, read coalesced while the TMEM loads run
#pragma unroll
                        for (int i = 0; i < 8; ++i) {
                            const int rr = 4 * i + (lane >> 3), c = lane & 7;
                            uint4 mv = make_uint4(0u, 0u, 0u, 0u);
                            if (q * 32 + rr < valid)
                                mv = *reinterpret_cast<const uint4 *>(g.mask + ((long long)m0 + q * 32 + rr) * g.ldm +
                                                                      c0 + c * 8);
                            *reinterpret_cast<uint4 *>(out + tc_out_off(rr, c)) = mv;
                        }
                        __syncwarp();
                    }
                    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                    // piece jc of the lane's own row: its mask is read from, and its
                    // output written to, the same place, by this lane only
#pragma unroll
                    for (int jc = 0; jc < 8; ++jc) {
                        const float4 b0 = *reinterpret_cast<const float4 *>(&s_bias[c0 + 8 * jc]);
                        const float4 b1 = *reinterpret_cast<const float4 *>(&s_bias[c0 + 8 * jc + 4]);
                        const float bb[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
                        __align__(16) __nv_bfloat16 o[8];
                        if (kEpi == kEpiBiasReluBf16) {
#pragma unroll
                            for (int j = 0; j < 8; ++j)
                                o[j] = __float2bfloat16(fmaxf(__uint_as_float(v[8 * jc + j]) + bb[j], 0.0f));
                        } else {
                            __align__(16) __nv_bfloat16 mk[8];
                            *reinterpret_cast<uint4 *>(mk) = *reinterpret_cast<const uint4 *>(out + tc_out_off(lane, jc));
#pragma unroll
                            for (int j = 0; j < 8; ++j) {
                                const float f = __uint_as_float(v[8 * jc + j]) + bb[j];
                                o[j] = __float2bfloat16(__bfloat162float(mk[j]) > 0.0f ? f : 0.0f);
                            }
                        }
                        *reinterpret_cast<uint4 *>(out + tc_out_off(lane, jc)) = *reinterpret_cast<const uint4 *>(o);
                    }
                    if (bulk) {
                        // the lanes' writes, visible to the async proxy, then one store
                        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                        __syncwarp();
                        if (lane == 0)
                            tc_tma_store(&g.tmap_c, c0, m0 + q * 32, (uint32_t)__cvta_generic_to_shared(out));
                        continue;
                    }
                    __syncwarp();
#pragma unroll
                    for (int i = 0; i < 8; ++i) {
                        const int rr = 4 * i + (lane >> 3), c = lane & 7;
                        const uint4 val = *reinterpret_cast<const uint4 *>(out + tc_out_off(rr, c));
                        if (q * 32 + rr < valid)
                            *reinterpret_cast<uint4 *>(static_cast<__nv_bfloat16 *>(g.C) +
                                                       ((long long)m0 + q * 32 + rr) * g.ldc + c0 + c * 8) = val;
                    }
                    __syncwarp();  // the tile is read before the next columns overwrite it
                }
            } else {
                for (int c0 = 16 * h; c0 < N; c0 += 32) {
                    uint32_t v[16];
                    tc_ld16(tsrc + (uint32_t)c0, v);
                    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                    if (r < valid) {
                        float f[16];
#pragma unroll
                        for (int j = 0; j < 16; ++j) f[j] = __uint_as_float(v[j]) + s_bias[c0 + j];
                        if (kEpi == kEpiBiasReluBf16 || kEpi == kEpiMaskBf16) {
                            __align__(16) __nv_bfloat16 o[16];
                            if (kEpi == kEpiBiasReluBf16) {
#pragma unroll
                                for (int j = 0; j < 16; ++j) o[j] = __float2bfloat16(fmaxf(f[j], 0.0f));
                            } else {
                                __align__(16) __nv_bfloat16 mk[16];
                                const uint4 *ms = reinterpret_cast<const uint4 *>(g.mask + row * g.ldm + c0);
                                reinterpret_cast<uint4 *>(mk)[0] = ms[0];
                                reinterpret_cast<uint4 *>(mk)[1] = ms[1];
#pragma unroll
                                for (int j = 0; j < 16; ++j)
                                    o[j] = __float2bfloat16(__bfloat162float(mk[j]) > 0.0f ? f[j] : 0.0f);
                            }
                            uint4 *dst = reinterpret_cast<uint4 *>(static_cast<__nv_bfloat16 *>(g.C) + row * g.ldc + c0);
                            dst[0] = reinterpret_cast<const uint4 *>(o)[0];
                            dst[1] = reinterpret_cast<const uint4 *>(o)[1];
                        } else {
                            float4 *dst = reinterpret_cast<float4 *>(static_cast<float *>(g.C) +
                                                                     (long long)blockIdx.y * g.c_split + row * g.ldc + c0);
#pragma unroll
                            for (int j = 0; j < 4; ++j)
                                dst[j] = make_float4(f[4 * j], f[4 * j + 1], f[4 * j + 2], f[4 * j + 3]);
                        }
                    }
                }
            }
            // this warp's reads of the accumulator are done: release it
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) tc_mbar_arrive(acce0 + 8u * a);
        }
        // the warp's TMA stores have completed (and read their tiles)
        if (lane == 0) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
        __syncwarp();
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols));
}

}  // namespace sg
}  // namespace fd2
