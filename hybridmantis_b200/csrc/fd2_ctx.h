// fd2_ctx.h -- the context behind fd2_ctx (include/fd2.h), shared by the
// C ABI (fd2_api.cpp) and the surrogate's event pipeline (fd2_sg_run.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "fd2.h"
#include "fd2_internal.h"

using fd2::DevGeom;

struct fd2_ctx {
    fd2_params params{};
    fd2_options opt{};
    int device = 0, sm_count = 0;
    std::string device_name, last_error;
    cudaStream_t stream = nullptr;

    // geometries
    std::vector<fd2_geometry> geoms;
    std::vector<DevGeom> dgeoms;
    int64_t prf_total = 0;
    DevGeom *d_geoms = nullptr;

    // events
    int64_t n_events = 0, cap_events = 0;
    float4 *d_ev_pos = nullptr;
    double *d_ev_e = nullptr, *d_ev_xyz = nullptr;
    uint16_t *d_ev_geom = nullptr;
    bool has_geom = false;
    int32_t *d_given_n = nullptr, *d_ev_n = nullptr;
    uint32_t *d_ev_nchunks = nullptr;
    unsigned long long *d_chunk_off = nullptr, *d_block_sums = nullptr;
    uint2 *d_chunks = nullptr;
    int64_t chunk_cap = 0;
    double mu_total = 0.0;
    bool counts_ready = false;
    std::vector<double> hist_per_geom;

    // staging
    void *d_stage = nullptr;
    size_t d_stage_bytes = 0;
    void *h_stage = nullptr;
    size_t h_stage_bytes = 0;

    // per-run device scalars: [0] chunks, [1] queue head, [2] photon total, [3..3+G) photons per geometry
    unsigned long long *d_scalars = nullptr;
    unsigned long long *d_gen_total = nullptr;  // photons per geometry, counted runs (transport passes)
    int *d_flags = nullptr;  // [0] status bits, [1] run counter

    // tallies
    int32_t n_prim = 0;
    unsigned long long *d_prf = nullptr, *d_counters = nullptr, *d_dropped = nullptr;
    int32_t *d_per_primary = nullptr, *d_prim_geom = nullptr, *d_phs = nullptr;
    uint32_t *d_radial = nullptr;  // label mode: [n_prim][radial_bins + 1]
    int64_t radial_len = 0;
    double *d_distance = nullptr, *d_moments = nullptr;

    // abort flag in mapped host memory
    int *h_abort = nullptr, *d_abort = nullptr;

    cudaEvent_t ev_start = nullptr, ev_t0 = nullptr, ev_t1 = nullptr, ev_end = nullptr;
    cudaGraphExec_t graph[3] = {nullptr, nullptr, nullptr};
    bool graph_valid = false;
    bool run_pending = false, ran_once = false;
    bool submitted = false;  // a submission (possibly of zero events) happened
    bool ingest_active = false;  // fd2_ingest_begin .. fd2_ingest_end
    fd2_ingest *ingest = nullptr; // the open ingest, ended by fd2_destroy
    fd2::TransportConfig cfg;
    int win_x0 = 0, win_y0 = 0;
    int win_chosen = 0, win_cx = 0, win_cy = 0;  // window and centre picked at submission
    int64_t last_photons = 0;

    // float-libm corrections of the reference-arithmetic replay
    uint32_t *d_libm = nullptr;
    uint32_t n_acos = 0, n_asin = 0;
};

namespace fd2 {
namespace api {

// Pieces of the run pipeline (fd2_api.cpp), for pipelines built around it.
cudaError_t count_pass(fd2_ctx *c, bool for_transport);   // photon counts + chunk counts
cudaError_t enqueue_segment(fd2_ctx *c, int seg);         // 0 counts+queue, 1 transport, 2 PHS + run tag
TransportArgs transport_args(fd2_ctx *c);
fd2_status ensure_chunks(fd2_ctx *c);
fd2_status ensure_events(fd2_ctx *c, int64_t n);
void choose_window(fd2_ctx *c, const float *x, const float *y, const uint16_t *geom, int64_t n);
fd2_status check_status(fd2_ctx *c);
fd2_status fail(fd2_ctx *c, fd2_status s, const std::string &msg);

}  // namespace api
}  // namespace fd2
