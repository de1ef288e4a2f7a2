// fd2_replay.cu -- replay of the reference's C transport on the GPU.
//
// One thread per event walks the event's photons in order, drawing from the
// reference's RANECU stream init_PRNG(event, 50000, seed_input) exactly as
// main/hybridMANTIS_c_ver1_0.c:189-340 drives main/kernel_cuda_c_ver1_0.cu
// (C branch).  Templated on the storage type T:
//   T = float   "REF"  : float variables, float operators where the
//                        reference writes float operators, double where it
//                        promotes (double literals, double libm calls);
//   T = double  "FP64" : the same walk with every quantity in double.
// Compiled with -fmad=false so no FMA changes a rounding.  The libm
// functions are CUDA's (within 1-2 ulp of glibc's), and acosf/asinf are
// evaluated as the float rounding of the double function, so a few photons
// per million may take a different branch than on the CPU: the caller
// compares per-photon records and counts divergent histories.
#include <cuda_runtime.h>

#include <cstdint>

#include "fd2_internal.h"
#include "fd2_replay_walk.cuh"

namespace fd2 {
namespace {

using replay::Walk;
using replay::ranecu_seed;
using D = double;


template <typename T>
__global__ void __launch_bounds__(64) replay_kernel(ReplayArgs a)
{
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= a.n_events) return;
    const int gi = a.ev_geom ? a.ev_geom[e] : 0;
    const DevGeom &G = a.geoms[gi];
    Walk<T> w;
    w.g = &G;
    // the reference's float parameters (cpuoptical_ copies doubles to floats)
    w.xdet = (T)G.xdet; w.ydet = (T)G.ydet; w.H = (T)G.H; w.R = (T)G.R;
    w.top = (T)G.top_absfrac; w.beta = (T)G.beta;
    w.dmin = (T)G.d_min; w.dmax = (T)G.d_max;
    w.lbx = (T)G.lb_x; w.lby = (T)G.lb_y; w.ubx = (T)G.ub_x; w.uby = (T)G.ub_y;
    w.srefl = (T)G.sensor_refl;
    w.pixel = (int)G.pixel;
    w.mu = (T)G.mu;
    w.ncol = (T)G.n_col;
    w.ngap = (T)G.n_gap;
    w.acos_tab = a.acos_tab;
    w.asin_tab = a.asin_tab;
    w.n_acos = a.n_acos;
    w.n_asin = a.n_asin;
    w.rng = ranecu_seed(a.event_index_base + e, a.seed_input);
    w.ex = a.ev_pos_d[3 * e + 0];
    w.ey = a.ev_pos_d[3 * e + 1];
    w.ez = a.ev_pos_d[3 * e + 2];
    const int prim = __float_as_int(a.ev_pos[e].w);
    w.p[0] = (T)w.ex; w.p[1] = (T)w.ey; w.p[2] = (T)w.ez;
    w.n[0] = T(0); w.n[1] = T(0); w.n[2] = T(0);
    w.xc = T(0); w.yc = T(0);
    w.emit(true);
    const int32_t N = a.ev_n[e];
    const unsigned long long first = a.ev_first[e];
    if (N > 0) atomicAdd(&a.gen_total[gi], (unsigned long long)N);
    for (int32_t k = 0; k < N; ++k) {
        w.absorbed = 0;
        w.detect = 0;
        w.bulk_abs = 0;
        w.p[0] = (T)w.ex; w.p[1] = (T)w.ey; w.p[2] = (T)w.ez;
        w.rebound = 0;
        w.fate = kAlive;
        w.pi = -1;
        w.pj = -1;
        int32_t calls = 0;
        int done = 0;
        while (!done) {
            ++calls;
            done = w.step();
            if (!done && calls >= (1 << 24)) {  // runaway guard; never reached by a physical walk
                w.set_fate(kCapped);
                done = 1;
            }
        }
        const unsigned long long rec = first + (unsigned long long)k;
        const int fate = w.fate;
        atomicAdd(&a.counters[gi * kCounterStride + fate], 1ull);
        if (fate == kDetect) {
            if (prim >= 0 && prim < a.n_prim) atomicAdd(&a.per_primary[prim], 1);
            if (w.pi >= 0 && w.pj >= 0 && w.pi < G.xdim && w.pj < G.ydim) {
                atomicAdd(&a.counters[gi * kCounterStride + kNumFates], 1ull);
                atomicAdd(&a.prf[G.prf_offset + (long long)w.pi * G.ydim + w.pj], 1ull);
            }
        }
        if (a.fate) a.fate[rec] = (int8_t)fate;
        if (a.pix) {
            a.pix[2 * rec] = fate == kDetect ? w.pi : -1;
            a.pix[2 * rec + 1] = fate == kDetect ? w.pj : -1;
        }
        if (a.seeds) {
            a.seeds[2 * rec] = w.rng.s0;
            a.seeds[2 * rec + 1] = w.rng.s1;
        }
        if (a.steps) a.steps[rec] = calls;
    }
}

}  // namespace

cudaError_t launch_replay(cudaStream_t s, int mode, const ReplayArgs &a)
{
    if (a.n_events <= 0) return cudaSuccess;
    const unsigned grid = (unsigned)((a.n_events + 63) / 64);
    if (mode == 0) replay_kernel<float><<<grid, 64, 0, s>>>(a);
    else replay_kernel<double><<<grid, 64, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace fd2
