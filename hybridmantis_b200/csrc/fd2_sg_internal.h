// fd2_sg_internal.h -- state of the surrogate (fd2_surrogate.h) shared by
// its training code (fd2_surrogate.cu) and the event pipeline (fd2_sg_run.cu).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "fd2_surrogate.h"

namespace fd2 {
namespace sg {

constexpr int kFeatures = FD2_SG_FEATURES;
constexpr int kOutputs = FD2_SG_OUTPUTS;
constexpr int kComponents = FD2_SG_COMPONENTS;
constexpr int kInPad = 32;   // input width seen by the first GEMM (K multiple of 32)
constexpr int kOutPad = 64;  // output width of the last GEMM
constexpr int kMaxSplits = 16;
constexpr float kMuScale = 50.0f;  // ring radius = kMuScale * softplus(output), um (>= 0)
constexpr float kSdScale = 10.0f;  // um
constexpr float kLateralUnitUm = 50.0f;  // unit of feature 2, the deposition's distance from the detector centre
constexpr float kLogSdMin = -6.0f, kLogSdMax = 4.0f;

// Radial categories: bin j < bins covers [e_j, e_{j+1}) with quadratic edges
// e_j = r_max (j / bins)^2 (fine near the deposition, where the column wall
// shapes the profile); category `bins` is r >= r_max.
__host__ __device__ inline float radial_edge(int j, int bins, float r_max)
{
    const float t = (float)j / (float)bins;
    return r_max * t * t;
}

// parameter blocks of the FP32 master vector
enum { kW1 = 0, kB1, kW2, kB2, kW3, kB3, kW4, kB4, kNumBlocks };

// x = 2 (f - lo) inv - 1 per feature
struct NormParams {
    float lo[kFeatures];
    float inv[kFeatures];
};

}  // namespace sg
}  // namespace fd2

struct fd2_sg {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string last_error;
    int hidden = 256, bins = 64, batch = 8192;
    double radial_max = 200.0;
    float lr = 1e-3f, beta1 = 0.9f, beta2 = 0.999f, eps = 1e-8f, lambda = 1.0f;
    float lateral_um = 50.0f;
    float depth_margin_um = 1.0f;  // depths this far outside the hull take its edge
    // edge survival of the sampled azimuths (fd2_sg_set_edge): amplitude and
    // length; amplitude 0 = uniform over the directions that stay on the detector
    float edge_amp = 0.0f, edge_len_um = 1.0f;
    uint64_t seed = 0;
    fd2_sg_hull hull{};      // routing box: events outside go to the Monte Carlo
    fd2_sg_hull norm_box{};  // input normalisation box, fixed by the first hull the network gets
    bool norm_fixed = false;
    fd2::sg::NormParams norm{};

    // parameters (FP32 masters, gradients, Adam moments, BF16 copies)
    int64_t off[fd2::sg::kNumBlocks] = {};
    int64_t n_params = 0;
    float *p = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
    __nv_bfloat16 *pb = nullptr;
    uint8_t *d_live = nullptr;
    unsigned long long *d_step = nullptr;
    double *d_acc = nullptr;
    float *d_lr = nullptr;  // Adam step size (read by the captured step)
    float *ws = nullptr;  // split-K partials
    int64_t ws_floats = 0;
    // tcgen05 backward: transposed BF16 weights (W2^T, W3^T: H x H; W4^T:
    // H x 64) and batch-major operands transposed to [columns][rows padded
    // to 256] (tA: the incoming gradient, tB: the layer's input)
    __nv_bfloat16 *pbT = nullptr, *tA = nullptr, *tB = nullptr;

    // activations for up to cap_rows rows
    int cap_rows = 0;
    __nv_bfloat16 *x0 = nullptr, *h1 = nullptr, *h2 = nullptr, *h3 = nullptr;
    __nv_bfloat16 *d1 = nullptr, *d2 = nullptr, *d3 = nullptr, *dout = nullptr;
    float *out = nullptr, *target = nullptr, *ylab = nullptr, *has_rad = nullptr;
    cudaGraphExec_t graph = nullptr;

    // training data
    int64_t n_points = 0, n_train = 0, n_val = 0;
    float *d_feat = nullptr;
    int32_t *d_photons = nullptr, *d_detected = nullptr;
    uint32_t *d_radial = nullptr;

    // event-pipeline buffers (fd2_sg_run)
    struct RunBuffers *run = nullptr;

    // forward GEMMs on tcgen05 (fd2_sg_tc.cuh) unless FD2_SG_GEMM=mma; a
    // tile whose completion wait gave up sets the fault word
    bool use_tc = true;
    bool tc_pipe = true;  // the pipelined tcgen05 kernel (FD2_SG_GEMM=tc1: the one-tile-at-a-time kernel)
    bool tc_tma = true;   // its operands by TMA where possible (FD2_SG_GEMM=cpasync: cp.async)
    bool tc_sw128 = true; // TMA boxes of 128-byte swizzled rows where K % 64 == 0 (FD2_SG_GEMM=noswizzle: 16-byte columns)
    bool tc_tma_store = true;  // staged BF16 epilogues store by TMA (FD2_SG_GEMM=nostore: per-lane stores)
    unsigned *d_tc_fault = nullptr;
    int sm_count = 148;
};

fd2_status sg_fail(fd2_sg *s, fd2_status st, const std::string &msg);
fd2_status sg_cuda(fd2_sg *s, cudaError_t e, const char *what);
cudaError_t sg_forward(fd2_sg *s, cudaStream_t st, const __nv_bfloat16 *x0, int rows, const int *m_limit,
                       __nv_bfloat16 *h1, __nv_bfloat16 *h2, __nv_bfloat16 *h3, float *out);
void sg_free_run_buffers(fd2_sg *s);
// FD2_ERR_DEVICE_ABORT (and the fault word cleared) when a tensor-core tile
// gave up waiting since the last check; call after a stream synchronisation.
fd2_status sg_tc_check(fd2_sg *s);
