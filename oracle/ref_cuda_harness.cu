/*
 * ref_cuda_harness.cu -- launches the reference's own CUDA kernel `algo`.
 *
 * TEST/BENCHMARK INFRASTRUCTURE ONLY.  oracle/Makefile compiles this file
 * with the reference's main/kernel_cuda_c_ver1_0.cu pre-included (nvcc
 * -include, -DUSING_CUDA, -use_fast_math, as main/compile_ver1_0.sh:4-6
 * builds it), for sm_100a, into oracle/_ref/libfd2refcuda.so.  The
 * reference source is read where it lies; nothing of it is copied.  It is
 * the GPU baseline that the product's transport kernel is timed against
 * and a statistical cross-check of its tallies.
 *
 * The harness plays the role of gpuoptical_ modes 99/100/101
 * (main/hybridMANTIS_cuda_ver1_0.cu:187-446) without GSL or the Fortran
 * COMMON blocks: photon counts are given by the caller; events are packed
 * into struct start_info (positions in um, cuda:253-258); algo is launched
 * with the reference's launch shape (GRIDSIZE 18000 x BLOCKSIZE 128 covers
 * a full 2,304,000-event buffer, cuda:57-62) or the smallest grid that
 * covers the events; the device counters are zeroed before and read after.
 *
 * Memory safety: the reference kernel indexes the PRF image by
 * floor((x - lbound)/pixel) for x <= ubound, which reaches row xdim (and
 * column ydim) for photons exactly on the upper bound, and it uses the x
 * pixel as the row index although cuda:191 allocates ydim rows.  The
 * harness therefore allocates max(xdim, ydim) + 2 rows and columns; the
 * caller receives the xdim x ydim core ([ii][jj], ii = x pixel).
 */
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

/* The COMMON blocks that the reference file declares extern in its CUDA
 * branch (kernel_cuda_c_ver1_0.cu:84-236) belong to the Fortran program;
 * the kernel never references them, so they stay undefined and unused. */

namespace {

struct Deleter {
    void *p = nullptr;
    ~Deleter() { if (p) cudaFree(p); }
};

}  // namespace

extern "C" {

/* params: xdet, ydet, H, R, n_col, n_gap, top_absfrac, bulk_abs, beta,
 *         d_min, d_max, lb_x, lb_y, ub_x, ub_y, sensor_refl (16 floats) */
typedef struct {
    float v[16];
    int pixel;
} fd2refcu_geom;

/*
 * Transports n events on `device` with the reference kernel.
 * image (xdim*ydim u64, [ii][jj]) and per_primary (num_hist, index hist-1)
 * are overwritten; counters[7] = generated, detect, abs_top, abs_bulk,
 * lost, outofcol, theta1.  kernel_ms = CUDA-event time of the algo launch
 * (inputs already on the device).  grid <= 0 picks ceil(n/128) blocks;
 * otherwise the grid must cover n events.  Returns 0 or a negative code
 * (-1 bad arguments, -2 CUDA error; cuda_error receives the code).
 */
int fd2refcu_run(int device, const fd2refcu_geom *g, int64_t n, const double *x_um, const double *y_um,
                 const double *z_um, const int *hist, const int *nphot, int num_hist, int grid,
                 int xdim, int ydim, unsigned long long *image, int *per_primary,
                 unsigned long long *counters, float *kernel_ms, int *cuda_error)
{
    if (!g || n < 0 || n > 2304000 || num_hist <= 0 || xdim <= 0 || ydim <= 0 || !image || !per_primary ||
        !counters || !kernel_ms)
        return -1;
    for (int64_t i = 0; i < n; ++i)
        if (hist[i] < 1 || hist[i] > num_hist || nphot[i] < 0) return -1;
    const int block = 128;
    const int64_t need = (n + block - 1) / block;
    if (grid <= 0) grid = (int)(need > 0 ? need : 1);
    if ((int64_t)grid * block < n) return -1;

    cudaError_t err = cudaSetDevice(device);
#define RC(call)                                \
    do {                                        \
        err = (call);                           \
        if (err != cudaSuccess) {               \
            if (cuda_error) *cuda_error = err;  \
            return -2;                          \
        }                                       \
    } while (0)
    RC(err);

    const size_t n_alloc = (size_t)(n > 0 ? n : 1);
    start_info *h_info = new start_info[n_alloc];
    for (int64_t i = 0; i < n; ++i) {
        h_info[i].str_x = x_um[i];
        h_info[i].str_y = y_um[i];
        h_info[i].str_z = z_um[i];
        h_info[i].str_E = 0.0;
        h_info[i].str_histnum = hist[i];
        h_info[i].str_N = nphot[i];
    }
    const int side = (xdim > ydim ? xdim : ydim) + 2;
    Deleter d_info, d_img, d_prim;
    size_t pitch = 0;
    err = cudaMalloc(&d_info.p, n_alloc * sizeof(start_info));
    if (err == cudaSuccess) err = cudaMallocPitch(&d_img.p, &pitch, (size_t)side * sizeof(unsigned long long), side);
    if (err == cudaSuccess) err = cudaMalloc(&d_prim.p, (size_t)num_hist * sizeof(int));
    if (err == cudaSuccess) err = cudaMemcpy(d_info.p, h_info, n_alloc * sizeof(start_info), cudaMemcpyHostToDevice);
    delete[] h_info;
    RC(err);
    RC(cudaMemset2D(d_img.p, pitch, 0, (size_t)side * sizeof(unsigned long long), side));
    RC(cudaMemset(d_prim.p, 0, (size_t)num_hist * sizeof(int)));
    const unsigned long long zero = 0;
    const float fzero = 0.0f;
    RC(cudaMemcpyToSymbol(num_generated, &zero, sizeof zero));
    RC(cudaMemcpyToSymbol(num_detect, &zero, sizeof zero));
    RC(cudaMemcpyToSymbol(num_abs_top, &zero, sizeof zero));
    RC(cudaMemcpyToSymbol(num_abs_bulk, &zero, sizeof zero));
    RC(cudaMemcpyToSymbol(num_lost, &zero, sizeof zero));
    RC(cudaMemcpyToSymbol(num_outofcol, &zero, sizeof zero));
    RC(cudaMemcpyToSymbol(num_theta1, &zero, sizeof zero));
    RC(cudaMemcpyToSymbol(photon_distance, &fzero, sizeof fzero));

    const float *p = g->v;
    cudaEvent_t e0, e1;
    RC(cudaEventCreate(&e0));
    RC(cudaEventCreate(&e1));
    RC(cudaDeviceSynchronize());
    RC(cudaEventRecord(e0, 0));
    /* argument order of algo: kernel_cuda_c_ver1_0.cu:391-393 */
    algo<<<grid, block, 0, 0>>>((start_info *)d_info.p, (unsigned long long *)d_img.p, (int *)d_prim.p, pitch,
                                (int)n, p[0], p[1], p[3], p[2], p[4], p[5], p[6], p[7], p[8], p[9], g->pixel,
                                p[11], p[12], p[13], p[14], p[10], p[15]);
    RC(cudaGetLastError());
    RC(cudaEventRecord(e1, 0));
    RC(cudaEventSynchronize(e1));
    RC(cudaEventElapsedTime(kernel_ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);

    for (int ii = 0; ii < xdim; ++ii)
        RC(cudaMemcpy(image + (size_t)ii * ydim, (char *)d_img.p + (size_t)ii * pitch,
                      (size_t)ydim * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
    RC(cudaMemcpy(per_primary, d_prim.p, (size_t)num_hist * sizeof(int), cudaMemcpyDeviceToHost));
    unsigned long long c[7];
    RC(cudaMemcpyFromSymbol(&c[0], num_generated, sizeof c[0]));
    RC(cudaMemcpyFromSymbol(&c[1], num_detect, sizeof c[1]));
    RC(cudaMemcpyFromSymbol(&c[2], num_abs_top, sizeof c[2]));
    RC(cudaMemcpyFromSymbol(&c[3], num_abs_bulk, sizeof c[3]));
    RC(cudaMemcpyFromSymbol(&c[4], num_lost, sizeof c[4]));
    RC(cudaMemcpyFromSymbol(&c[5], num_outofcol, sizeof c[5]));
    RC(cudaMemcpyFromSymbol(&c[6], num_theta1, sizeof c[6]));
    memcpy(counters, c, sizeof c);
#undef RC
    return 0;
}

}  // extern "C"
