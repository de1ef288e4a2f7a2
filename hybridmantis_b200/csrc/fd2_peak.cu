// fd2_peak.cu -- FP32 fused multiply-add throughput of the device.
//
// The transport kernel is bound by FP32/SFU/integer issue, and its roofline
// denominator is the FP32 FMA peak: SMs x 128 FP32 lanes x 2 flops x clock.
// This kernel measures that peak on the device it runs on, so the derived
// figure can be checked against a number the chip actually delivers: every
// thread runs kChains independent FMA chains (enough instruction-level
// parallelism to cover the FMA latency at any occupancy the launch gives),
// the grid fills every SM several times over, and the timing is CUDA events
// on the launching stream.
#include <cuda_runtime.h>

#include <cstdint>

#include "fd2.h"

namespace {

constexpr int kChains = 8;
constexpr int kUnroll = 16;
constexpr int kBlock = 512;
constexpr int kBlocksPerSm = 4;

__global__ void __launch_bounds__(kBlock) fma_peak_kernel(float *out, int iters, float a, float b)
{
    float x[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = (float)(threadIdx.x + c) * 1e-7f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
#pragma unroll
            for (int c = 0; c < kChains; ++c) x[c] = fmaf(x[c], a, b);
        }
    }
    float s = 0.0f;
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += x[c];
    // never true for the arguments the host passes; keeps the chains live
    if (s == -1.0f) out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace

extern "C" fd2_status fd2_measure_fp32_peak(int32_t device, double min_seconds, double *tflops, double *seconds)
{
    if (!tflops || device < 0) return FD2_ERR_INVALID_ARGUMENT;
    int prev = 0;
    if (cudaGetDevice(&prev) != cudaSuccess) return FD2_ERR_NO_DEVICE;
    if (cudaSetDevice(device) != cudaSuccess) return FD2_ERR_NO_DEVICE;
    fd2_status st = FD2_OK;
    int sms = 0;
    cudaStream_t s = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    float *out = nullptr;
    const int iters = 4096;
    double best = 0.0, total_s = 0.0;
    do {
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
            cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
            st = FD2_ERR_CUDA;
            break;
        }
        const unsigned grid = (unsigned)(sms * kBlocksPerSm);
        if (cudaMalloc(&out, sizeof(float) * grid * kBlock) != cudaSuccess) {
            st = FD2_ERR_OUT_OF_MEMORY;
            break;
        }
        const double flops = 2.0 * kChains * kUnroll * (double)iters * grid * kBlock;
        fma_peak_kernel<<<grid, kBlock, 0, s>>>(out, iters, 0.999999f, 1e-7f);  // warm-up
        for (int rep = 0; rep < 1000 && (rep < 3 || total_s < min_seconds); ++rep) {
            cudaEventRecord(e0, s);
            fma_peak_kernel<<<grid, kBlock, 0, s>>>(out, iters, 0.999999f, 1e-7f);
            cudaEventRecord(e1, s);
            if (cudaEventSynchronize(e1) != cudaSuccess) {
                st = FD2_ERR_CUDA;
                break;
            }
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, e0, e1);
            total_s += ms * 1e-3;
            if (ms > 0.0f && flops / (ms * 1e-3) > best) best = flops / (ms * 1e-3);
        }
        if (cudaGetLastError() != cudaSuccess) st = FD2_ERR_CUDA;
    } while (false);
    if (out) cudaFree(out);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (s) cudaStreamDestroy(s);
    cudaSetDevice(prev);
    *tflops = best * 1e-12;
    if (seconds) *seconds = total_s;
    return st;
}
