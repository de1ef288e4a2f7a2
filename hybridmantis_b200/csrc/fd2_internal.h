// fd2_internal.h -- host/device interface between the C-ABI layer and the
// kernels.  Not installed; include/fd2.h is the public surface.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "fd2_types.h"

namespace fd2 {

// Launch configuration of the persistent transport kernel.
struct TransportConfig {
    int block = 256;     // threads per CTA (multiple of 32, <= 1024)
    int ctas_per_sm = 2; // persistent grid = SMs * ctas_per_sm
    int chunk = 32;      // photons per work-queue chunk
    int refill = 1;      // idle lanes that trigger a warp refill
    int window = 0;      // shared-memory PRF window edge (0 = off)
    int fresnel = 8;     // parked lanes that trigger the warp's Fresnel pass
    bool aggregate = false;  // single geometry: warp-aggregated, shared-memory privatised tallies
};

struct TransportArgs {
    const float4 *ev_pos;        // x, y, z (um) and the history index (hist-1) as bits
    const uint16_t *ev_geom;     // geometry of each event (null: all 0)
    const int32_t *ev_n;         // photons per event
    const uint2 *chunks;         // (event, first photon) per queue chunk
    const unsigned long long *n_chunks;
    long long chunk_capacity;    // entries allocated in `chunks`
    unsigned long long *queue_head;
    const DevGeom *geoms;
    int n_geom;
    DevGeom g0;                  // geometry 0 (read from the kernel parameters)
    unsigned long long *prf;     // all geometries' PRF images
    int32_t *per_primary;
    int32_t n_prim;
    unsigned long long *counters;  // [n_geom][kNumFates + 1]: fates, then detected-in-PRF
    double *distance;              // [n_geom]
    uint64_t seed;
    int64_t event_base;          // global index of event 0 (RNG counters)
    uint32_t round_keys[20];     // Philox key schedule of the seed
    const uint32_t *run_tag;     // device counter: runs since submission
    int chunk;
    int refill;
    int fresnel_batch;           // parked lanes before the Fresnel pass runs
    int window;                  // window edge (0 = off), applies to geometry 0
    int win_x0, win_y0;          // window origin in pixels
    const volatile int *abort_flag;
    int *status;
    // label mode: per-history radial histograms of detected photons
    unsigned int *radial;        // [n_prim][radial_bins + 1], null = off
    int radial_bins;
    float radial_inv_max;        // 1 / r_max (bin j covers r_max (j/bins)^2 .. r_max ((j+1)/bins)^2)
};

// Device status bits (the `status` word).
enum : int {
    kStatusTooManyPhotons = 1,
    kStatusBadEvent = 2,
    kStatusAborted = 4,
    kStatusChunkOverflow = 8,
    kStatusRngUnderflow = 16  // reserved (raised by no kernel since the walk draws in registers)
};

constexpr int kCounterStride = kNumFates + 1;

// Photon-count rules (values of FD2_COUNT_* in include/fd2.h).
enum : int { kCountPoisson = 0, kCountGaussian = 1, kCountGiven = 2 };

// Kernel launchers (fd2_kernels.cu).  All are stream-ordered and capture-safe.
cudaError_t launch_prep_cm(cudaStream_t s, int64_t n, const double *x_cm, const double *y_cm,
                           const double *z_cm, const double *de, const int32_t *hist, int32_t n_prim,
                           float4 *ev_pos, double *ev_e, double *ev_xyz, int *status);
cudaError_t launch_prep_um(cudaStream_t s, int64_t n, const float *x, const float *y, const float *z,
                           const float *e, const int32_t *hist, int32_t n_prim, float4 *ev_pos,
                           double *ev_e, double *ev_xyz, int *status);
cudaError_t launch_count(cudaStream_t s, int64_t n, int64_t event_base, int mode, double yield, int64_t max_per_event,
                         uint64_t seed, const uint32_t *run_tag, int chunk, const double *ev_e,
                         const int32_t *given_n, const uint16_t *ev_geom, const float4 *ev_pos,
                         int32_t *ev_n, uint32_t *ev_nchunks, unsigned long long *photons_per_geom,
                         unsigned long long *photons_total, int32_t *prim_geom, int32_t n_prim, int *status);
// Exclusive scan of per-event chunk counts; writes offsets and the total.
cudaError_t launch_scan(cudaStream_t s, int64_t n, const uint32_t *in, unsigned long long *offsets,
                        unsigned long long *block_sums, unsigned long long *total);
size_t scan_block_sums_needed(int64_t n);
// Device-submitted events (fd2_xray.cu): out[0] += sum of (float)(x_cm 1e4),
// out[1] the same for y, out[2] += sum of the positive energies.
cudaError_t launch_event_sums(cudaStream_t s, int64_t n, const double *x_cm, const double *y_cm, const double *de,
                              double *out);
cudaError_t launch_fill_chunks(cudaStream_t s, int64_t n, int chunk, const int32_t *ev_n,
                               const unsigned long long *offsets, uint2 *chunks, int64_t capacity,
                               int *status);
cudaError_t launch_transport(cudaStream_t s, const TransportConfig &cfg, int sm_count, const TransportArgs &a);
// Sets the kernel's shared-memory limit; call outside stream capture.
cudaError_t prepare_transport(const TransportConfig &cfg, int n_geom);
cudaError_t launch_bump_run_tag(cudaStream_t s, uint32_t *run_tag);
size_t transport_smem_bytes(const TransportConfig &cfg, int n_geom);
cudaError_t launch_phs(cudaStream_t s, int32_t n_prim, const int32_t *per_primary, const int32_t *prim_geom,
                       int n_geom, int32_t min_photons, int32_t max_photons, int32_t num_bins,
                       int32_t *phs, double *moments, unsigned long long *dropped);

// Replay of the reference C path (fd2_replay.cu).
struct ReplayArgs {
    int64_t n_events;
    const float4 *ev_pos;          // float positions (REF mode reads ev_pos_d when set)
    const double *ev_pos_d;        // x, y, z as double triples (positions before rounding)
    const int32_t *ev_n;
    const uint16_t *ev_geom;
    const unsigned long long *ev_first;  // photon offset of each event (exclusive scan)
    const DevGeom *geoms;
    int n_geom;
    int32_t seed_input;
    int64_t event_index_base;
    unsigned long long *prf;
    int32_t *per_primary;
    int32_t n_prim;
    unsigned long long *counters;
    unsigned long long *gen_total;   // photons per geometry, accumulated
    int8_t *fate;
    int32_t *pix;
    int32_t *seeds;
    int32_t *steps;
    const uint32_t *acos_tab, *asin_tab;  // float libm corrections (REF mode)
    uint32_t n_acos, n_asin;
};
cudaError_t launch_replay(cudaStream_t s, int mode, const ReplayArgs &a);
cudaError_t launch_photon_offsets(cudaStream_t s, int64_t n, const int32_t *ev_n, unsigned long long *first,
                                  unsigned long long *block_sums, unsigned long long *total);

}  // namespace fd2
