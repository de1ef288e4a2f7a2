// fd2_analysis.cu -- MTF and NNPS of the transport's images (include/fd2_analysis.h).
//
// Both are discrete Fourier transforms of modest images (hundreds of pixels
// a side), taken as two passes of direct sums in FP64 with exact integer
// phase reduction: pass 1 transforms every row at the wanted column
// frequencies, pass 2 every resulting column at the wanted row frequencies.
// A pass is one thread per output value looping over the inputs, the input
// row staged in shared memory (pass 1) or read coalesced across threads
// (pass 2), twiddles exp(-2 pi i m / N) from a table.  The magnitudes are
// reduced into radial bins with FP64 atomics on the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "fd2.h"
#include "fd2_analysis.h"

namespace {

constexpr int kThreads = 128;

// tw[m] = exp(-2 pi i m / N), m < N
__global__ void twiddle_kernel(int n, double2 *tw)
{
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= n) return;
    double s, c;
    sincospi(2.0 * (double)m / (double)n, &s, &c);
    tw[m] = make_double2(c, -s);
}

// out[r * nk + k] = sum_{c < ncols} (in[(r0 + r) * ld + c0 + c] - sub) tw[(freq[k] c) mod n]
// grid (ceil(nk / kThreads), nrows); dynamic shared memory: ncols doubles.
__global__ void dft_rows_kernel(const double *__restrict__ in, int64_t ld, int r0, int c0, int ncols, double sub,
                                const int *__restrict__ freq, int nk, const double2 *__restrict__ tw, int n,
                                double2 *__restrict__ out)
{
    extern __shared__ double row[];
    const int r = blockIdx.y;
    const double *src = in + (int64_t)(r0 + r) * ld + c0;
    for (int c = threadIdx.x; c < ncols; c += blockDim.x) row[c] = src[c] - sub;
    __syncthreads();
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nk) return;
    const int f = freq[k];
    double re = 0.0, im = 0.0;
    int m = 0;
    for (int c = 0; c < ncols; ++c) {
        const double2 w = tw[m];
        re = fma(row[c], w.x, re);
        im = fma(row[c], w.y, im);
        m += f;
        if (m >= n) m -= n;
    }
    out[(int64_t)r * nk + k] = make_double2(re, im);
}

// Pass 2 at row frequency rf[u] for every column k of a (nrows x nk) matrix:
// h = sum_r a[r][k] tw[(rf[u] r) mod n].  mode 0: bin |h| / norm by the
// radius of (sf_u, sf_k); mode 1: acc[u][k] += |h|^2 (power accumulation).
// grid (ceil(nk / kThreads), nu).
__global__ void dft_cols_kernel(const double2 *__restrict__ a, int nrows, int nk, const int *__restrict__ rf,
                                const int *__restrict__ sf_row, const int *__restrict__ sf_col,
                                const double2 *__restrict__ tw, int n, int mode, double norm, int nbins,
                                double *__restrict__ bin_sum, double *__restrict__ bin_cnt, double *__restrict__ acc)
{
    const int u = blockIdx.y;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nk) return;
    const int f = rf[u];
    double re = 0.0, im = 0.0;
    int m = 0;
    for (int r = 0; r < nrows; ++r) {
        const double2 x = a[(int64_t)r * nk + k];
        const double2 w = tw[m];
        re = fma(x.x, w.x, fma(-x.y, w.y, re));
        im = fma(x.x, w.y, fma(x.y, w.x, im));
        m += f;
        if (m >= n) m -= n;
    }
    if (mode == 1) {
        acc[(int64_t)u * nk + k] += re * re + im * im;
        return;
    }
    const double su = (double)sf_row[u], sk = (double)sf_col[k];
    const int b = (int)llrint(sqrt(su * su + sk * sk));
    if (b < nbins) {
        atomicAdd(&bin_sum[b], sqrt(re * re + im * im) / norm);
        atomicAdd(&bin_cnt[b], 1.0);
    }
}

// Row and column sums of an image (the two line spread functions).
__global__ void lsf_kernel(const double *__restrict__ img, int xdim, int ydim, double *__restrict__ lsf_x,
                           double *__restrict__ lsf_y)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < xdim) {
        double s = 0.0;
        for (int j = 0; j < ydim; ++j) s += img[(int64_t)t * ydim + j];
        lsf_x[t] = s;
    }
    if (t < ydim) {
        double s = 0.0;
        for (int i = 0; i < xdim; ++i) s += img[(int64_t)i * ydim + t];
        lsf_y[t] = s;
    }
}

// |sum_i l[i] tw[(k i) mod n]| / norm for k < nk (one thread per k).
__global__ void dft_1d_mag_kernel(const double *__restrict__ l, int len, int nk, const double2 *__restrict__ tw,
                                  int n, double norm, double *__restrict__ out)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nk) return;
    double re = 0.0, im = 0.0;
    int m = 0;
    for (int i = 0; i < len; ++i) {
        const double2 w = tw[m];
        re = fma(l[i], w.x, re);
        im = fma(l[i], w.y, im);
        m += k;
        if (m >= n) m -= n;
    }
    out[k] = sqrt(re * re + im * im) / norm;
}

// Per-pixel mean over n images (x n stacked images of `count` values).
__global__ void mean_images_kernel(const double *__restrict__ imgs, int n, int64_t count, double *__restrict__ mean)
{
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < count; p += (int64_t)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int r = 0; r < n; ++r) s += imgs[(int64_t)r * count + p];
        mean[p] = s / (double)n;
    }
}

__global__ void sub_kernel(const double *__restrict__ a, const double *__restrict__ b, int64_t count,
                           double *__restrict__ out)
{
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < count; p += (int64_t)gridDim.x * blockDim.x)
        out[p] = a[p] - b[p];
}

// Sum of an roi x roi region (one block).
__global__ void region_sum_kernel(const double *__restrict__ img, int64_t ld, int x0, int y0, int roi,
                                  double *__restrict__ out)
{
    __shared__ double part[kThreads];
    double s = 0.0;
    for (int t = threadIdx.x; t < roi * roi; t += blockDim.x) s += img[(int64_t)(x0 + t / roi) * ld + y0 + t % roi];
    part[threadIdx.x] = s;
    __syncthreads();
    for (int w = kThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = part[0];
}

// Radial binning of an n x n power map in unsigned DFT order.
__global__ void bin_map_kernel(const double *__restrict__ map, int n, double scale, int nbins,
                               double *__restrict__ bin_sum, double *__restrict__ bin_cnt, double *__restrict__ out2d)
{
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= (int64_t)n * n) return;
    const int u = (int)(t / n), v = (int)(t % n);
    const double val = map[t] * scale;
    if (out2d) out2d[t] = val;
    const double su = u <= n / 2 ? u : u - n, sv = v <= n / 2 ? v : v - n;
    const int b = (int)llrint(sqrt(su * su + sv * sv));
    if (b < nbins) {
        atomicAdd(&bin_sum[b], val);
        atomicAdd(&bin_cnt[b], 1.0);
    }
}

struct Dev {
    std::vector<void *> ptrs;
    cudaError_t err = cudaSuccess;
    template <typename T>
    T *alloc(size_t n)
    {
        void *p = nullptr;
        if (err == cudaSuccess) err = cudaMalloc(&p, sizeof(T) * std::max<size_t>(n, 1));
        if (err == cudaSuccess) ptrs.push_back(p);
        return (T *)p;
    }
    ~Dev()
    {
        for (void *p : ptrs) cudaFree(p);
    }
};

fd2_status to_status(cudaError_t e)
{
    if (e == cudaSuccess) return FD2_OK;
    return e == cudaErrorMemoryAllocation ? FD2_ERR_OUT_OF_MEMORY
           : (e == cudaErrorNoDevice || e == cudaErrorInvalidDevice) ? FD2_ERR_NO_DEVICE
                                                                      : FD2_ERR_CUDA;
}

unsigned blocks_for(int64_t n) { return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + kThreads - 1) / kThreads, 1 << 20)); }

}  // namespace

extern "C" {

fd2_status fd2_mtf(int32_t device, const double *image, int32_t xdim, int32_t ydim, double pixel_um, int32_t n_freq,
                   double *freq_per_mm, double *mtf_x, double *mtf_y, double *mtf_r)
{
    if (!image || xdim < 1 || ydim < 1 || xdim > 16384 || ydim > 16384 || !(pixel_um > 0.0) || n_freq < 1)
        return FD2_ERR_INVALID_ARGUMENT;
    const int N = std::max(xdim, ydim);
    if (n_freq > N / 2 + 1) return FD2_ERR_INVALID_ARGUMENT;
    double total = 0.0;
    for (int64_t p = 0; p < (int64_t)xdim * ydim; ++p) total += image[p];
    if (!(total > 0.0) || !std::isfinite(total)) return FD2_ERR_INVALID_ARGUMENT;
    if (freq_per_mm)
        for (int k = 0; k < n_freq; ++k) freq_per_mm[k] = 1000.0 * k / (N * pixel_um);
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return to_status(e);
    Dev d;
    cudaStream_t s = nullptr;
    const int64_t npx = (int64_t)xdim * ydim;
    const int K = n_freq, V = 2 * K - 1;
    double *d_img = d.alloc<double>((size_t)npx);
    double2 *d_tw = d.alloc<double2>((size_t)N);
    double *d_lx = d.alloc<double>((size_t)xdim), *d_ly = d.alloc<double>((size_t)ydim);
    double *d_mx = d.alloc<double>((size_t)K), *d_my = d.alloc<double>((size_t)K);
    int *d_f = d.alloc<int>((size_t)V), *d_sf = d.alloc<int>((size_t)V);
    double2 *d_a = d.alloc<double2>((size_t)xdim * V);
    double *d_bs = d.alloc<double>((size_t)K), *d_bc = d.alloc<double>((size_t)K);
    if (d.err == cudaSuccess) d.err = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (d.err != cudaSuccess) return to_status(d.err);
    std::vector<int> f(V), sf(V);
    for (int t = 0; t < V; ++t) {
        sf[t] = t - (K - 1);               // signed frequency index
        f[t] = ((sf[t] % N) + N) % N;      // its phase step mod N
    }
    e = cudaMemcpyAsync(d_img, image, sizeof(double) * npx, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_f, f.data(), sizeof(int) * V, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_sf, sf.data(), sizeof(int) * V, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_bs, 0, sizeof(double) * K, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_bc, 0, sizeof(double) * K, s);
    if (e == cudaSuccess) {
        twiddle_kernel<<<blocks_for(N), kThreads, 0, s>>>(N, d_tw);
        lsf_kernel<<<blocks_for(N), kThreads, 0, s>>>(d_img, xdim, ydim, d_lx, d_ly);
        dft_1d_mag_kernel<<<blocks_for(K), kThreads, 0, s>>>(d_lx, xdim, K, d_tw, N, total, d_mx);
        dft_1d_mag_kernel<<<blocks_for(K), kThreads, 0, s>>>(d_ly, ydim, K, d_tw, N, total, d_my);
        if (mtf_r) {
            const size_t sm = sizeof(double) * (size_t)ydim;
            if (sm > 48 * 1024) e = cudaFuncSetAttribute(dft_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
            if (e == cudaSuccess) {
                dft_rows_kernel<<<dim3(blocks_for(V), (unsigned)xdim), kThreads, sm, s>>>(d_img, ydim, 0, 0, ydim, 0.0,
                                                                                          d_f, V, d_tw, N, d_a);
                dft_cols_kernel<<<dim3(blocks_for(V), (unsigned)V), kThreads, 0, s>>>(
                    d_a, xdim, V, d_f, d_sf, d_sf, d_tw, N, 0, total, K, d_bs, d_bc, nullptr);
            }
        }
        if (e == cudaSuccess) e = cudaGetLastError();
    }
    std::vector<double> bs(K), bc(K);
    if (e == cudaSuccess && mtf_x) e = cudaMemcpyAsync(mtf_x, d_mx, sizeof(double) * K, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && mtf_y) e = cudaMemcpyAsync(mtf_y, d_my, sizeof(double) * K, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && mtf_r) e = cudaMemcpyAsync(bs.data(), d_bs, sizeof(double) * K, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && mtf_r) e = cudaMemcpyAsync(bc.data(), d_bc, sizeof(double) * K, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
    if (e != cudaSuccess) return to_status(e);
    if (mtf_r)
        for (int k = 0; k < K; ++k) mtf_r[k] = bc[k] > 0.0 ? bs[k] / bc[k] : 0.0;
    return FD2_OK;
}

fd2_status fd2_nnps(int32_t device, const double *images, int32_t n_images, int32_t xdim, int32_t ydim,
                    double pixel_um, int32_t roi, int32_t x0, int32_t y0, int32_t rois_x, int32_t rois_y,
                    int32_t n_freq, double *freq_per_mm, double *nnps_r, double *nnps_2d, double *mean_signal)
{
    if (!images || n_images < 1 || xdim < 1 || ydim < 1 || !(pixel_um > 0.0) || roi < 2 || roi > 4096 ||
        rois_x < 1 || rois_y < 1 || x0 < 0 || y0 < 0 || n_freq < 1 || n_freq > roi / 2 + 1 ||
        (int64_t)x0 + (int64_t)rois_x * roi > xdim || (int64_t)y0 + (int64_t)rois_y * roi > ydim)
        return FD2_ERR_INVALID_ARGUMENT;
    if (freq_per_mm)
        for (int k = 0; k < n_freq; ++k) freq_per_mm[k] = 1000.0 * k / (roi * pixel_um);
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return to_status(e);
    Dev d;
    cudaStream_t s = nullptr;
    const int64_t npx = (int64_t)xdim * ydim;
    const int R = roi, K = n_freq, n = n_images;
    double *d_imgs = d.alloc<double>((size_t)(npx * n));
    double *d_mean = d.alloc<double>((size_t)npx);
    double *d_diff = d.alloc<double>((size_t)npx);
    double2 *d_tw = d.alloc<double2>((size_t)R);
    int *d_f = d.alloc<int>((size_t)R);
    double2 *d_a = d.alloc<double2>((size_t)R * R);
    double *d_acc = d.alloc<double>((size_t)R * R);
    double *d_sums = d.alloc<double>((size_t)rois_x * rois_y * (n + 1));
    double *d_bs = d.alloc<double>((size_t)K), *d_bc = d.alloc<double>((size_t)K);
    double *d_2d = nnps_2d ? d.alloc<double>((size_t)R * R) : nullptr;
    if (d.err == cudaSuccess) d.err = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (d.err != cudaSuccess) return to_status(d.err);
    std::vector<int> f(R);
    for (int t = 0; t < R; ++t) f[t] = t;
    e = cudaMemcpyAsync(d_imgs, images, sizeof(double) * npx * n, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_f, f.data(), sizeof(int) * R, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_acc, 0, sizeof(double) * R * R, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_bs, 0, sizeof(double) * K, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_bc, 0, sizeof(double) * K, s);
    const int nroi = rois_x * rois_y;
    const size_t sm = sizeof(double) * (size_t)R;
    if (e == cudaSuccess && sm > 48 * 1024)
        e = cudaFuncSetAttribute(dft_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e == cudaSuccess) {
        twiddle_kernel<<<blocks_for(R), kThreads, 0, s>>>(R, d_tw);
        mean_images_kernel<<<blocks_for(npx), kThreads, 0, s>>>(d_imgs, n, npx, d_mean);
        // region sums of the mean image (signal) and, with one image, of the image (its mean)
        for (int q = 0; q < nroi; ++q)
            region_sum_kernel<<<1, kThreads, 0, s>>>(d_mean, ydim, x0 + (q / rois_y) * R, y0 + (q % rois_y) * R, R,
                                                     d_sums + q);
        e = cudaGetLastError();
    }
    std::vector<double> sums((size_t)nroi);
    if (e == cudaSuccess) e = cudaMemcpyAsync(sums.data(), d_sums, sizeof(double) * nroi, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    double m = 0.0;
    for (double v : sums) m += v;
    m /= (double)nroi * R * R;
    if (e == cudaSuccess && !(m > 0.0)) e = cudaErrorInvalidValue;
    for (int r = 0; e == cudaSuccess && r < n; ++r) {
        const double *src = d_imgs + (int64_t)r * npx;
        if (n > 1) {
            sub_kernel<<<blocks_for(npx), kThreads, 0, s>>>(src, d_mean, npx, d_diff);
            src = d_diff;
        }
        for (int q = 0; q < nroi && e == cudaSuccess; ++q) {
            const int rx = x0 + (q / rois_y) * R, ry = y0 + (q % rois_y) * R;
            // one image: subtract the region's mean (the mean image is the image)
            const double sub = n > 1 ? 0.0 : sums[(size_t)q] / ((double)R * R);
            dft_rows_kernel<<<dim3(blocks_for(R), (unsigned)R), kThreads, sm, s>>>(src, ydim, rx, ry, R, sub, d_f, R,
                                                                                  d_tw, R, d_a);
            dft_cols_kernel<<<dim3(blocks_for(R), (unsigned)R), kThreads, 0, s>>>(d_a, R, R, d_f, nullptr, nullptr,
                                                                                  d_tw, R, 1, 1.0, 0, nullptr,
                                                                                  nullptr, d_acc);
            e = cudaGetLastError();
        }
    }
    // NNPS = pixel^2 (mm^2) / roi^2 * <|F|^2> * n/(n-1) / m^2
    const double px_mm = pixel_um / 1000.0;
    const double corr = n > 1 ? (double)n / (double)(n - 1) : 1.0;
    const double scale = px_mm * px_mm / ((double)R * R) * corr / ((double)n * nroi) / (m * m);
    if (e == cudaSuccess) {
        bin_map_kernel<<<blocks_for((int64_t)R * R), kThreads, 0, s>>>(d_acc, R, scale, K, d_bs, d_bc, d_2d);
        e = cudaGetLastError();
    }
    std::vector<double> bs(K), bc(K);
    if (e == cudaSuccess) e = cudaMemcpyAsync(bs.data(), d_bs, sizeof(double) * K, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(bc.data(), d_bc, sizeof(double) * K, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && nnps_2d)
        e = cudaMemcpyAsync(nnps_2d, d_2d, sizeof(double) * R * R, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
    if (e == cudaErrorInvalidValue && !(m > 0.0)) return FD2_ERR_INVALID_ARGUMENT;
    if (e != cudaSuccess) return to_status(e);
    if (nnps_r)
        for (int k = 0; k < K; ++k) nnps_r[k] = bc[k] > 0.0 ? bs[k] / bc[k] : 0.0;
    if (mean_signal) *mean_signal = m;
    return FD2_OK;
}

}  // extern "C"
