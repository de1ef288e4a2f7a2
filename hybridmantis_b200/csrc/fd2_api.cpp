// fd2_api.cpp -- the C ABI (include/fd2.h): contexts, event submission, the
// graph-captured run pipeline, results, output files, replay, autotuning.
//
// Ownership follows the reference's GPU driver (hybridMANTIS_cuda_ver1_0.cu
// :107-446): the caller owns host arrays, the context owns device memory
// from fd2_create to fd2_destroy, tallies accumulate across runs (the
// reference accumulates across buffers, mode 100 -> 101), and work is
// asynchronous on the context's stream until fd2_wait or a getter.  Unlike
// the reference every call returns a status instead of exiting.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <utility>
#include <vector>

#include <dlfcn.h>

#include <cuda_runtime.h>

#include "fd2.h"
#include "fd2_host.h"
#include "fd2_ctx.h"
#include "fd2_internal.h"


namespace {

fd2_status fail(fd2_ctx *c, fd2_status s, const std::string &msg)
{
    if (c) c->last_error = msg;
    return s;
}

fd2_status cuda_fail(fd2_ctx *c, cudaError_t e, const char *what)
{
    const fd2_status s = (e == cudaErrorMemoryAllocation) ? FD2_ERR_OUT_OF_MEMORY : FD2_ERR_CUDA;
    return fail(c, s, std::string(what) + ": " + cudaGetErrorString(e));
}

#define FD2_CUDA(ctx, call)                                      \
    do {                                                         \
        cudaError_t e_ = (call);                                 \
        if (e_ != cudaSuccess) return cuda_fail(ctx, e_, #call); \
    } while (0)

template <typename T>
cudaError_t dalloc(T **p, size_t n)
{
    if (*p) cudaFree(*p);
    *p = nullptr;
    return cudaMalloc((void **)p, sizeof(T) * (n ? n : 1));
}

template <typename T>
void dfree(T *&p)
{
    if (p) cudaFree(p);
    p = nullptr;
}

bool valid_geometry(const fd2_geometry &g)
{
    auto fin = [](double v) { return std::isfinite(v); };
    return fin(g.det_x) && fin(g.det_y) && fin(g.det_height) && fin(g.radius) && fin(g.n_col) && fin(g.n_gap) &&
           fin(g.top_absfrac) && fin(g.bulk_abs) && fin(g.beta) && fin(g.d_min) && fin(g.d_max) && fin(g.lb_x) &&
           fin(g.lb_y) && fin(g.ub_x) && fin(g.ub_y) && fin(g.sensor_refl) && g.det_x > 0 && g.det_y > 0 &&
           g.det_height > 0 && g.radius > 0 && g.n_col > 0 && g.n_gap > 0 && g.top_absfrac >= 0 &&
           g.top_absfrac <= 1 && g.bulk_abs >= 0 && g.beta >= 0 && g.d_min >= 0 && g.d_max >= g.d_min &&
           g.sensor_refl >= 0 && g.sensor_refl <= 1 && g.pixel > 0 && g.ub_x > g.lb_x && g.ub_y > g.lb_y;
}

// Float parameters as the reference's drivers hold them, plus the derived
// constants of the production walk.
DevGeom make_dev_geom(const fd2_geometry &g)
{
    DevGeom d;
    std::memset(&d, 0, sizeof d);
    d.xdet = (float)g.det_x;
    d.ydet = (float)g.det_y;
    d.H = (float)g.det_height;
    d.half = d.H / 2.0f;
    d.R = (float)g.radius;
    d.beta = (float)g.beta;
    d.top_absfrac = (float)g.top_absfrac;
    d.mu = (float)g.bulk_abs;
    d.neg_inv_mu = d.mu > 0.0f ? -1.0f / d.mu : 0.0f;
    d.d_min = (float)g.d_min;
    d.d_max = (float)g.d_max;
    d.d_span = d.d_max - d.d_min;
    d.lb_x = (float)g.lb_x;
    d.lb_y = (float)g.lb_y;
    d.ub_x = (float)g.ub_x;
    d.ub_y = (float)g.ub_y;
    d.sensor_refl = (float)g.sensor_refl;
    d.pixel = (float)g.pixel;
    const float band = d.H * 0.2f;
    d.cct_band_lo = d.half - band;
    d.cct_k_hi = 1.0f / (2.0f * (d.half - band));
    d.cct_k_lo = 1.0f / (2.0f * (-d.half));
    d.n_col = (float)g.n_col;
    d.n_gap = (float)g.n_gap;
    d.eta_in = d.n_col / d.n_gap;
    const double rin = (double)(d.n_gap / d.n_col);
    d.cos_tir_in = rin <= 1.0 ? (float)std::sqrt(1.0 - rin * rin) : -1.0f;
    d.eta_out = d.n_gap / d.n_col;
    d.stale_out = (d.n_col / d.n_gap) < 1.57f ? 1 : 0;
    const double rout = (double)(d.n_col / d.n_gap);
    d.cos_tir_out = rout <= 1.0 ? (float)std::sqrt(1.0 - rout * rout) : -1.0f;
    int32_t xd = 0, yd = 0;
    fd2_prf_dims(&g, &xd, &yd);
    d.xdim = xd;
    d.ydim = yd;
    return d;
}

fd2_status alloc_tallies(fd2_ctx *c)
{
    const size_t G = c->geoms.size();
    c->dgeoms.clear();
    int64_t off = 0;
    for (const auto &g : c->geoms) {
        DevGeom d = make_dev_geom(g);
        d.grid = c->opt.column_grid;
        d.pitch = (float)(2.0 * g.radius + c->opt.grid_gap_um);
        d.prf_offset = off;
        off += (int64_t)d.xdim * d.ydim;
        c->dgeoms.push_back(d);
    }
    c->prf_total = off;
    FD2_CUDA(c, dalloc(&c->d_geoms, G));
    FD2_CUDA(c, cudaMemcpy(c->d_geoms, c->dgeoms.data(), sizeof(DevGeom) * G, cudaMemcpyHostToDevice));
    FD2_CUDA(c, dalloc(&c->d_prf, (size_t)c->prf_total));
    FD2_CUDA(c, dalloc(&c->d_counters, G * fd2::kCounterStride));
    FD2_CUDA(c, dalloc(&c->d_distance, G));
    FD2_CUDA(c, dalloc(&c->d_phs, G * (size_t)std::max(c->params.num_bins, 1)));
    FD2_CUDA(c, dalloc(&c->d_moments, G * 3));
    FD2_CUDA(c, dalloc(&c->d_dropped, G));
    FD2_CUDA(c, dalloc(&c->d_scalars, 3 + G));
    FD2_CUDA(c, dalloc(&c->d_gen_total, G));
    c->hist_per_geom.assign(G, 0.0);
    c->graph_valid = false;
    return fd2_reset_tallies(c);
}

fd2_status ensure_stage(fd2_ctx *c, size_t bytes)
{
    if (bytes > c->d_stage_bytes) {
        if (c->d_stage) cudaFree(c->d_stage);
        c->d_stage = nullptr;
        FD2_CUDA(c, cudaMalloc(&c->d_stage, bytes));
        c->d_stage_bytes = bytes;
    }
    if (bytes > c->h_stage_bytes) {
        if (c->h_stage) cudaFreeHost(c->h_stage);
        c->h_stage = nullptr;
        FD2_CUDA(c, cudaHostAlloc(&c->h_stage, bytes, cudaHostAllocDefault));
        c->h_stage_bytes = bytes;
    }
    return FD2_OK;
}

fd2_status ensure_events(fd2_ctx *c, int64_t n)
{
    if (n > c->cap_events) {
        const size_t m = (size_t)n;
        FD2_CUDA(c, dalloc(&c->d_ev_pos, m));
        FD2_CUDA(c, dalloc(&c->d_ev_e, m));
        FD2_CUDA(c, dalloc(&c->d_ev_xyz, 3 * m));
        FD2_CUDA(c, dalloc(&c->d_ev_geom, m));
        FD2_CUDA(c, dalloc(&c->d_given_n, m));
        FD2_CUDA(c, dalloc(&c->d_ev_n, m));
        FD2_CUDA(c, dalloc(&c->d_ev_nchunks, m));
        FD2_CUDA(c, dalloc(&c->d_chunk_off, m));
        FD2_CUDA(c, dalloc(&c->d_block_sums, fd2::scan_block_sums_needed(n)));
        c->cap_events = n;
    }
    return FD2_OK;
}

fd2_status ensure_chunks(fd2_ctx *c)
{
    const double mu = c->mu_total;
    const double bound = mu * 1.01 + 10.0 * std::sqrt(mu) + 4096.0;
    const int64_t need = c->n_events + (int64_t)std::ceil(bound / (double)c->cfg.chunk) + 1024;
    if (need > c->chunk_cap) {
        FD2_CUDA(c, dalloc(&c->d_chunks, (size_t)need));
        c->chunk_cap = need;
        c->graph_valid = false;
    }
    return FD2_OK;
}

// Read back and clear the device status word.
fd2_status check_status(fd2_ctx *c)
{
    int st = 0;
    FD2_CUDA(c, cudaMemcpyAsync(&st, c->d_flags, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    FD2_CUDA(c, cudaStreamSynchronize(c->stream));
    if (st) FD2_CUDA(c, cudaMemsetAsync(c->d_flags, 0, sizeof(int), c->stream));
    if (st & fd2::kStatusBadEvent) return fail(c, FD2_ERR_BAD_EVENT, "event with non-finite or negative values, or history outside 1..num_hist");
    if (st & fd2::kStatusTooManyPhotons) return fail(c, FD2_ERR_TOO_MANY_PHOTONS, "an event exceeds max_photons_per_event");
    if (st & fd2::kStatusChunkOverflow) return fail(c, FD2_ERR_OUT_OF_MEMORY, "work-queue capacity exceeded");
    if (st & fd2::kStatusAborted) return fail(c, FD2_ERR_DEVICE_ABORT, "transport aborted");
    return FD2_OK;
}

void fit_window(fd2_ctx *c);

// The PRF window around the mean position (um) of geometry 0's k events,
// given as coordinate sums.
void choose_window_sums(fd2_ctx *c, double sx, double sy, int64_t k)
{
    const DevGeom &g = c->dgeoms[0];
    int w = c->opt.prf_window;
    if (w < 0) w = 128;
    if (c->d_radial) w = 0;  // label mode tallies no PRF image
    if (!(c->opt.tally_mode == 1 && c->geoms.size() == 1 && !c->opt.column_grid))
        w = 0;  // per-lane reductions go straight to the global PRF
    if (w > g.xdim) w = g.xdim;
    if (w > g.ydim) w = g.ydim;
    if (w > 176) w = 176;  // fits beside the rings in shared memory
    c->cfg.window = c->win_chosen = (k > 0 && w >= 16) ? w : 0;
    if (!c->cfg.window) return;
    c->win_cx = (int)std::floor((sx / (double)k - g.lb_x) / g.pixel);
    c->win_cy = (int)std::floor((sy / (double)k - g.lb_y) / g.pixel);
    fit_window(c);
}

void choose_window(fd2_ctx *c, const float *x, const float *y, const uint16_t *geom, int64_t n)
{
    double sx = 0, sy = 0;
    int64_t k = 0;
    for (int64_t i = 0; i < n; ++i) {
        if (geom && geom[i] != 0) continue;
        sx += x[i];
        sy += y[i];
        ++k;
    }
    choose_window_sums(c, sx, sy, k);
}

fd2::TransportArgs transport_args(fd2_ctx *c)
{
    fd2::TransportArgs a;
    a.ev_pos = c->d_ev_pos;
    a.ev_geom = c->has_geom ? c->d_ev_geom : nullptr;
    a.ev_n = c->d_ev_n;
    a.chunks = c->d_chunks;
    a.n_chunks = c->d_scalars + 0;
    a.chunk_capacity = c->chunk_cap;
    a.queue_head = c->d_scalars + 1;
    a.geoms = c->d_geoms;
    a.n_geom = (int)c->geoms.size();
    a.g0 = c->dgeoms[0];
    a.prf = c->d_prf;
    a.per_primary = c->d_per_primary;
    a.n_prim = c->n_prim;
    a.counters = c->d_counters;
    a.distance = c->d_distance;
    a.seed = c->opt.seed;
    a.event_base = c->opt.event_base;
    uint32_t k0 = (uint32_t)c->opt.seed, k1 = (uint32_t)(c->opt.seed >> 32);
    for (int r = 0; r < 10; ++r) {
        a.round_keys[2 * r] = k0;
        a.round_keys[2 * r + 1] = k1;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    a.run_tag = reinterpret_cast<const uint32_t *>(c->d_flags + 1);
    a.chunk = c->cfg.chunk;
    a.refill = c->cfg.refill;
    a.fresnel_batch = c->cfg.fresnel;
    a.window = c->cfg.window;
    a.win_x0 = c->win_x0;
    a.win_y0 = c->win_y0;
    a.abort_flag = c->d_abort;
    a.status = c->d_flags;
    a.radial = c->d_radial;
    a.radial_bins = c->d_radial ? c->opt.radial_bins : 0;
    a.radial_inv_max = c->d_radial ? (float)(1.0 / c->opt.radial_max_um) : 0.0f;
    return a;
}

cudaError_t count_pass(fd2_ctx *c, bool for_transport)
{
    const size_t G = c->geoms.size();
    cudaError_t e = cudaMemsetAsync(c->d_scalars, 0, sizeof(unsigned long long) * (3 + G), c->stream);
    if (e != cudaSuccess) return e;
    return fd2::launch_count(c->stream, c->n_events, c->opt.event_base, c->opt.count_mode, c->params.yield,
                             c->opt.max_photons_per_event, c->opt.seed, reinterpret_cast<const uint32_t *>(c->d_flags + 1), c->cfg.chunk,
                             c->d_ev_e, c->d_given_n, c->has_geom ? c->d_ev_geom : nullptr, c->d_ev_pos, c->d_ev_n,
                             c->d_ev_nchunks, c->d_scalars + 3, for_transport ? c->d_gen_total : nullptr,
                             c->d_prim_geom, c->n_prim, c->d_flags);
}

// The run pipeline in three segments on the context's stream: queue build
// (count, scan, fill), the persistent transport, and the PHS pass.  Each is
// captured as its own graph; the timing events sit between them.
cudaError_t enqueue_segment(fd2_ctx *c, int seg)
{
    const size_t G = c->geoms.size();
    cudaError_t e = cudaSuccess;
    if (seg == 0) {
        e = count_pass(c, true);
        if (e == cudaSuccess)
            e = fd2::launch_scan(c->stream, c->n_events, c->d_ev_nchunks, c->d_chunk_off, c->d_block_sums,
                                 c->d_scalars + 0);
        if (e == cudaSuccess)
            e = fd2::launch_fill_chunks(c->stream, c->n_events, c->cfg.chunk, c->d_ev_n, c->d_chunk_off, c->d_chunks,
                                        c->chunk_cap, c->d_flags);
    } else if (seg == 1) {
        e = fd2::launch_transport(c->stream, c->cfg, c->sm_count, transport_args(c));
    } else {
        e = cudaMemsetAsync(c->d_phs, 0, sizeof(int32_t) * G * (size_t)std::max(c->params.num_bins, 1), c->stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(c->d_moments, 0, sizeof(double) * G * 3, c->stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(c->d_dropped, 0, sizeof(unsigned long long) * G, c->stream);
        if (e == cudaSuccess && c->params.num_bins > 0 &&
            c->params.max_photons - c->params.min_photons >= c->params.num_bins)
            e = fd2::launch_phs(c->stream, c->n_prim, c->d_per_primary, c->has_geom ? c->d_prim_geom : nullptr, (int)G,
                                c->params.min_photons, c->params.max_photons, c->params.num_bins, c->d_phs,
                                c->d_moments, c->d_dropped);
        if (e == cudaSuccess) e = fd2::launch_bump_run_tag(c->stream, reinterpret_cast<uint32_t *>(c->d_flags + 1));
    }
    return e;
}

fd2_status build_graph(fd2_ctx *c)
{
    for (auto &g : c->graph) {
        if (g) cudaGraphExecDestroy(g);
        g = nullptr;
    }
    for (int seg = 0; seg < 3; ++seg) {
        cudaGraph_t g = nullptr;
        FD2_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        const cudaError_t e = enqueue_segment(c, seg);
        const cudaError_t e2 = cudaStreamEndCapture(c->stream, &g);
        if (e != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            return cuda_fail(c, e, "capture of the run pipeline");
        }
        FD2_CUDA(c, e2);
        const cudaError_t e3 = cudaGraphInstantiate(&c->graph[seg], g, 0);
        cudaGraphDestroy(g);
        FD2_CUDA(c, e3);
    }
    c->graph_valid = true;
    return FD2_OK;
}

// The shared-memory PRF window (a tally cache) picked at submission, shrunk
// until ctas_per_sm CTAs of the configuration fit an SM's shared memory,
// around the same centre.
void fit_window(fd2_ctx *c)
{
    fd2::TransportConfig &k = c->cfg;
    const int G = (int)c->geoms.size();
    const size_t budget = 220 * 1024;
    k.window = c->win_chosen;
    while (k.window > 0 && fd2::transport_smem_bytes(k, G) * (size_t)k.ctas_per_sm > budget)
        k.window = k.window > 16 ? k.window - 8 : 0;
    if (k.window > 0) {
        const DevGeom &g = c->dgeoms[0];
        c->win_x0 = std::min(std::max(c->win_cx - k.window / 2, 0), g.xdim - k.window);
        c->win_y0 = std::min(std::max(c->win_cy - k.window / 2, 0), g.ydim - k.window);
    }
}

// Launch shape unless the options give one, measured on a B200 (config-1
// events, 20,000 x-rays): one geometry 256 threads x 4 CTAs per SM (32 warps
// at 64 registers; 6.7e8 photons/s against 5.8e8 for 320 x 2), chunks of 16
// photons; several geometries 256 x 3 (8.5e8 against 7.9e8 for 256 x 4,
// whose variant spills); the column lattice 320 x 2 (2.2e8 against 2.0e8 for
// 256 x 2 or x 3); label mode with one geometry (the surrogate's audit) as
// one geometry, with several 256 x 2.
static void default_launch(const fd2_ctx *c, int n_geom, fd2::TransportConfig *cfg)
{
    int block = 256, ctas = 4, chunk = 16;
    if (c->opt.radial_bins > 0) {
        // label mode: one geometry (the surrogate's audit) as a production
        // run; several (training labels) 256 x 2
        if (n_geom > 1) {
            ctas = 2;
            chunk = 32;
        }
    } else if (c->opt.column_grid) {
        block = 320;
        ctas = 2;
        chunk = 32;
    } else if (n_geom > 1) {
        ctas = 3;
        chunk = 32;
    }
    cfg->block = c->opt.block_size > 0 ? c->opt.block_size : block;
    cfg->ctas_per_sm = c->opt.ctas_per_sm > 0 ? c->opt.ctas_per_sm : ctas;
    cfg->chunk = c->opt.chunk > 0 ? c->opt.chunk : chunk;
}

fd2_status set_config(fd2_ctx *c, const fd2::TransportConfig &cfg)
{
    fd2::TransportConfig k = cfg;
    k.block = std::min(std::max(k.block / 32 * 32, 32), 1024);
    k.ctas_per_sm = std::min(std::max(k.ctas_per_sm, 1), 32);
    k.chunk = std::min(std::max(k.chunk, 1), 4096);
    k.refill = std::min(std::max(k.refill, 1), 32);
    k.fresnel = std::min(std::max(k.fresnel, 1), 32);
    // warp-aggregated, shared-memory privatised tallies: single-geometry runs
    // of the reference's column model (the other kernels reduce per lane)
    k.aggregate = c->opt.tally_mode == 1 && c->geoms.size() == 1 && !c->opt.radial_bins && !c->opt.column_grid;
    c->cfg = k;
    fit_window(c);
    FD2_CUDA(c, fd2::prepare_transport(c->cfg, (int)c->geoms.size()));
    c->graph_valid = false;
    return FD2_OK;
}

// The corrections written by fd2_libm_table next to libfd2.so.
fd2_status load_libm_table(fd2_ctx *c)
{
    if (c->d_libm) return FD2_OK;
    Dl_info info;
    std::string path = "fd2_float_libm.bin";
    if (dladdr((void *)&fd2_replay, &info) && info.dli_fname) {
        std::string so(info.dli_fname);
        const size_t k = so.rfind('/');
        path = (k == std::string::npos ? std::string(".") : so.substr(0, k)) + "/fd2_float_libm.bin";
    }
    FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) return fail(c, FD2_ERR_IO, "replay table " + path + " missing (make -C hybridmantis_b200)");
    char magic[8];
    uint32_t na = 0, ns = 0;
    bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, "FD2LIBM1", 8) == 0 &&
              std::fread(&na, 4, 1, f) == 1 && std::fread(&ns, 4, 1, f) == 1 && na < (1u << 28) && ns < (1u << 28);
    std::vector<uint32_t> tab;
    if (ok) {
        tab.resize((size_t)na + ns);
        ok = std::fread(tab.data(), 4, tab.size(), f) == tab.size();
    }
    std::fclose(f);
    if (!ok) return fail(c, FD2_ERR_PARSE, "replay table " + path + " is corrupt");
    FD2_CUDA(c, dalloc(&c->d_libm, tab.size()));
    FD2_CUDA(c, cudaMemcpy(c->d_libm, tab.data(), 4 * tab.size(), cudaMemcpyHostToDevice));
    c->n_acos = na;
    c->n_asin = ns;
    return FD2_OK;
}

std::string tune_key(const fd2_ctx *c)
{
    double mean = c->n_events ? c->mu_total / (double)c->n_events : 0.0;
    char b[256];
    std::snprintf(b, sizeof b, "%s|ev%d|ph%d|g%d|m%d", c->device_name.c_str(), (int)std::log2((double)c->n_events + 1),
                  (int)std::log2(mean + 1), (int)c->geoms.size(), c->opt.count_mode);
    return b;
}

bool tune_cache_lookup(const fd2_ctx *c, fd2::TransportConfig *out)
{
    if (!c->opt.tune_cache) return false;
    FILE *f = std::fopen(c->opt.tune_cache, "r");
    if (!f) return false;
    const std::string key = tune_key(c);
    char line[1024];
    bool found = false;
    while (std::fgets(line, sizeof line, f)) {
        char k[512];
        int b, s, ch, r, fr;
        if (std::sscanf(line,
                        " \"%511[^\"]\": {\"block\": %d, \"ctas_per_sm\": %d, \"chunk\": %d, \"refill\": %d, "
                        "\"fresnel\": %d",
                        k, &b, &s, &ch, &r, &fr) == 6 &&
            key == k) {
            out->block = b;
            out->ctas_per_sm = s;
            out->chunk = ch;
            out->refill = r;
            out->fresnel = fr;
            found = true;
        }
    }
    std::fclose(f);
    return found;
}

void tune_cache_store(const fd2_ctx *c)
{
    if (!c->opt.tune_cache) return;
    // keep other keys, replace ours; one entry per line inside braces
    std::vector<std::string> keep;
    const std::string key = tune_key(c);
    if (FILE *f = std::fopen(c->opt.tune_cache, "r")) {
        char line[1024];
        while (std::fgets(line, sizeof line, f)) {
            std::string s(line);
            if (s.find("\"block\"") == std::string::npos) continue;
            if (s.find("\"" + key + "\"") != std::string::npos) continue;
            while (!s.empty() && (s.back() == '\n' || s.back() == ',')) s.pop_back();
            keep.push_back(s);
        }
        std::fclose(f);
    }
    char b[1024];
    std::snprintf(b, sizeof b,
                  "  \"%s\": {\"block\": %d, \"ctas_per_sm\": %d, \"chunk\": %d, \"refill\": %d, \"fresnel\": %d}",
                  key.c_str(), c->cfg.block, c->cfg.ctas_per_sm, c->cfg.chunk, c->cfg.refill, c->cfg.fresnel);
    keep.push_back(b);
    if (FILE *f = std::fopen(c->opt.tune_cache, "w")) {
        std::fprintf(f, "{\n");
        for (size_t i = 0; i < keep.size(); ++i) std::fprintf(f, "%s%s\n", keep[i].c_str(), i + 1 < keep.size() ? "," : "");
        std::fprintf(f, "}\n");
        std::fclose(f);
    }
}

}  // namespace

namespace fd2 {
namespace api {

cudaError_t count_pass(fd2_ctx *c, bool for_transport) { return ::count_pass(c, for_transport); }
cudaError_t enqueue_segment(fd2_ctx *c, int seg) { return ::enqueue_segment(c, seg); }
TransportArgs transport_args(fd2_ctx *c) { return ::transport_args(c); }
fd2_status ensure_chunks(fd2_ctx *c) { return ::ensure_chunks(c); }
fd2_status ensure_events(fd2_ctx *c, int64_t n) { return ::ensure_events(c, n); }
void choose_window(fd2_ctx *c, const float *x, const float *y, const uint16_t *geom, int64_t n)
{
    ::choose_window(c, x, y, geom, n);
}
fd2_status check_status(fd2_ctx *c) { return ::check_status(c); }
fd2_status fail(fd2_ctx *c, fd2_status s, const std::string &msg) { return ::fail(c, s, msg); }

}  // namespace api
}  // namespace fd2

extern "C" {

const char *fd2_status_string(fd2_status s)
{
    switch (s) {
    case FD2_OK: return "ok";
    case FD2_ERR_INVALID_ARGUMENT: return "invalid argument";
    case FD2_ERR_IO: return "i/o error";
    case FD2_ERR_PARSE: return "parse error";
    case FD2_ERR_CUDA: return "CUDA error";
    case FD2_ERR_OUT_OF_MEMORY: return "out of memory";
    case FD2_ERR_TOO_MANY_PHOTONS: return "too many photons in one event";
    case FD2_ERR_STATE: return "call out of order";
    case FD2_ERR_TIMEOUT: return "deadline expired";
    case FD2_ERR_DEVICE_ABORT: return "device abort";
    case FD2_ERR_NO_DEVICE: return "no CUDA device";
    case FD2_ERR_FILE_EXISTS: return "output file exists";
    case FD2_ERR_BAD_EVENT: return "bad event";
    }
    return "unknown status";
}

void fd2_default_options(fd2_options *o)
{
    if (!o) return;
    std::memset(o, 0, sizeof *o);
    o->device = 0;
    o->count_mode = FD2_COUNT_POISSON;
    o->seed = 0x5eed0fd2b200ull;
    o->max_photons_per_event = 900000;
    o->block_size = 0;
    o->ctas_per_sm = 0;
    o->chunk = 0;
    o->refill = 0;
    o->prf_window = -1;
    o->use_graph = 1;
    o->wait_timeout_s = 0.0;
    o->tune_cache = nullptr;
    o->event_base = 0;
    o->radial_bins = 0;
    o->radial_max_um = 200.0;
    o->column_grid = 0;
    o->grid_gap_um = 0.5;
}

const char *fd2_last_error(const fd2_ctx *c) { return c ? c->last_error.c_str() : "no context"; }

fd2_status fd2_create(const fd2_params *p, const fd2_options *opt, fd2_ctx **out)
{
    if (!p || !out) return FD2_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) return FD2_ERR_NO_DEVICE;
    fd2_ctx *c = new fd2_ctx();
    c->params = *p;
    fd2_params_fill_tags(&c->params);
    if (opt) c->opt = *opt;
    else fd2_default_options(&c->opt);
    if (c->opt.max_photons_per_event <= 0) c->opt.max_photons_per_event = 900000;
    if (c->opt.event_base < 0 || c->opt.radial_bins < 0 || c->opt.radial_bins > 4096 ||
        (c->opt.radial_bins > 0 && !(c->opt.radial_max_um > 0.0)) || c->opt.column_grid < 0 ||
        c->opt.column_grid > 2 || (c->opt.column_grid && (!(c->opt.grid_gap_um > 0.0) || c->opt.radial_bins > 0))) {
        delete c;
        return FD2_ERR_INVALID_ARGUMENT;
    }
    if (c->opt.device < 0 || c->opt.device >= ndev || p->num_hist < 0 || !(p->yield >= 0.0)) {
        delete c;
        return FD2_ERR_INVALID_ARGUMENT;
    }
    fd2_geometry g;
    fd2_params_to_geometry(p, &g);
    if (!valid_geometry(g)) {
        delete c;
        return FD2_ERR_INVALID_ARGUMENT;
    }
    c->device = c->opt.device;
    fd2_status st = FD2_OK;
    auto bail = [&](fd2_status s) {
        fd2_destroy(c);
        return s;
    };
    if (cudaSetDevice(c->device) != cudaSuccess) return bail(FD2_ERR_CUDA);
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, c->device) != cudaSuccess) return bail(FD2_ERR_CUDA);
    c->sm_count = prop.multiProcessorCount;
    c->device_name = prop.name;
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) return bail(FD2_ERR_CUDA);
    if (cudaEventCreate(&c->ev_start) != cudaSuccess || cudaEventCreate(&c->ev_t0) != cudaSuccess ||
        cudaEventCreate(&c->ev_t1) != cudaSuccess || cudaEventCreate(&c->ev_end) != cudaSuccess)
        return bail(FD2_ERR_CUDA);
    if (cudaHostAlloc((void **)&c->h_abort, sizeof(int), cudaHostAllocMapped) != cudaSuccess) return bail(FD2_ERR_CUDA);
    *c->h_abort = 0;
    if (cudaHostGetDevicePointer((void **)&c->d_abort, c->h_abort, 0) != cudaSuccess) return bail(FD2_ERR_CUDA);
    if (dalloc(&c->d_flags, 2) != cudaSuccess || cudaMemset(c->d_flags, 0, 2 * sizeof(int)) != cudaSuccess)
        return bail(FD2_ERR_OUT_OF_MEMORY);
    c->n_prim = p->num_hist;
    if (dalloc(&c->d_per_primary, (size_t)c->n_prim) != cudaSuccess || dalloc(&c->d_prim_geom, (size_t)c->n_prim) != cudaSuccess)
        return bail(FD2_ERR_OUT_OF_MEMORY);
    if (c->opt.radial_bins > 0) {
        c->radial_len = (int64_t)std::max(c->n_prim, 1) * (c->opt.radial_bins + 1);
        if (dalloc(&c->d_radial, (size_t)c->radial_len) != cudaSuccess) return bail(FD2_ERR_OUT_OF_MEMORY);
    }
    c->geoms.assign(1, g);
    if ((st = alloc_tallies(c)) != FD2_OK) return bail(st);
    fd2::TransportConfig cfg;
    default_launch(c, 1, &cfg);
    cfg.refill = c->opt.refill > 0 ? c->opt.refill : 4;
    // parked lanes before the warp's Fresnel pass (8), or with a column lattice
    // gap lanes before the warp's gap segments (12: square 1.755 / hexagonal
    // 1.333e8 photons/s on config 1, against 1.743 / 1.297 at 8)
    cfg.fresnel = c->opt.fresnel_batch > 0 ? c->opt.fresnel_batch : (c->opt.column_grid ? 12 : 8);
    if ((st = set_config(c, cfg)) != FD2_OK) return bail(st);
    *out = c;
    return FD2_OK;
}

void fd2_destroy(fd2_ctx *c)
{
    if (!c) return;
    if (c->ingest) fd2_ingest_end(c->ingest, nullptr);
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (auto g : c->graph)
        if (g) cudaGraphExecDestroy(g);
    dfree(c->d_geoms);
    dfree(c->d_ev_pos);
    dfree(c->d_ev_e);
    dfree(c->d_ev_xyz);
    dfree(c->d_ev_geom);
    dfree(c->d_given_n);
    dfree(c->d_ev_n);
    dfree(c->d_ev_nchunks);
    dfree(c->d_chunk_off);
    dfree(c->d_block_sums);
    dfree(c->d_chunks);
    dfree(c->d_scalars);
    dfree(c->d_gen_total);
    dfree(c->d_flags);
    dfree(c->d_prf);
    dfree(c->d_counters);
    dfree(c->d_dropped);
    dfree(c->d_per_primary);
    dfree(c->d_radial);
    dfree(c->d_prim_geom);
    dfree(c->d_phs);
    dfree(c->d_distance);
    dfree(c->d_moments);
    dfree(c->d_libm);
    if (c->d_stage) cudaFree(c->d_stage);
    if (c->h_stage) cudaFreeHost(c->h_stage);
    if (c->h_abort) cudaFreeHost(c->h_abort);
    for (cudaEvent_t ev : {c->ev_start, c->ev_t0, c->ev_t1, c->ev_end})
        if (ev) cudaEventDestroy(ev);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

fd2_status fd2_set_geometries(fd2_ctx *c, const fd2_geometry *g, int32_t n)
{
    if (c && c->ingest_active) return fail(c, FD2_ERR_STATE, "an event ingest is open; end it first");
    if (!c || !g || n <= 0 || n > 256) return fail(c, FD2_ERR_INVALID_ARGUMENT, "1..256 geometries");
    for (int32_t i = 0; i < n; ++i)
        if (!valid_geometry(g[i])) return fail(c, FD2_ERR_INVALID_ARGUMENT, "invalid geometry " + std::to_string(i));
    if (c->opt.column_grid && n > 1) return fail(c, FD2_ERR_STATE, "the column lattice is for one geometry");
    FD2_CUDA(c, cudaSetDevice(c->device));
    FD2_CUDA(c, cudaStreamSynchronize(c->stream));
    c->geoms.assign(g, g + n);
    c->n_events = 0;
    c->counts_ready = false;
    fd2_status st = alloc_tallies(c);
    if (st != FD2_OK) return st;
    fd2::TransportConfig k = c->cfg;
    default_launch(c, n, &k);
    return set_config(c, k);
}

// What every submission does once the events are on the device: the PRF
// window (from positions xs, ys, or from the coordinate sums when xs is
// null), the work-queue capacity and, for given counts, the count pass.
static fd2_status submit_common(fd2_ctx *c, int64_t n, const float *xs, const float *ys, const uint16_t *geom,
                                const double *sums = nullptr)
{
    c->n_events = n;
    c->submitted = true;
    c->counts_ready = false;
    c->graph_valid = false;
    c->ran_once = false;
    // history count per geometry (normalisation of per-geometry PRFs)
    const size_t G = c->geoms.size();
    c->hist_per_geom.assign(G, 0.0);
    if (G == 1) c->hist_per_geom[0] = c->params.num_hist;
    if (xs) choose_window(c, xs, ys, geom, n);
    else choose_window_sums(c, sums ? sums[0] : 0.0, sums ? sums[1] : 0.0, n);
    fd2_status st = ensure_chunks(c);
    if (st != FD2_OK) return st;
    FD2_CUDA(c, fd2::prepare_transport(c->cfg, (int)G));
    FD2_CUDA(c, cudaMemsetAsync(c->d_flags + 1, 0, sizeof(int), c->stream));  // run counter
    st = check_status(c);
    if (st != FD2_OK) {
        c->n_events = 0;
        return st;
    }
    if (c->opt.count_mode == FD2_COUNT_GIVEN) {
        FD2_CUDA(c, count_pass(c, false));
        st = check_status(c);
        if (st != FD2_OK) {
            c->n_events = 0;
            return st;
        }
        c->counts_ready = true;
    }
    return FD2_OK;
}

fd2_status fd2_submit_events(fd2_ctx *c, const double *x_cm, const double *y_cm, const double *z_cm, const double *de_ev,
                             const int32_t *hist, int64_t n)
{
    if (c && c->ingest_active) return fail(c, FD2_ERR_STATE, "an event ingest is open; end it first");
    if (!c || n < 0 || (n > 0 && (!x_cm || !y_cm || !z_cm || !de_ev || !hist)) || n >= ((int64_t)1 << 31))
        return fail(c, FD2_ERR_INVALID_ARGUMENT, "submit_events: null array or bad count");
    if (c->run_pending) {
        const fd2_status w = fd2_wait(c);
        if (w != FD2_OK) return w;
    }
    if (c->geoms.size() != 1) return fail(c, FD2_ERR_STATE, "cm submission is for a single geometry; use fd2_submit_events_um");
    if (c->opt.count_mode == FD2_COUNT_GIVEN) return fail(c, FD2_ERR_STATE, "count_mode GIVEN needs fd2_submit_events_um");
    FD2_CUDA(c, cudaSetDevice(c->device));
    fd2_status st = ensure_events(c, n);
    if (st != FD2_OK) return st;
    const size_t nb = (size_t)n;
    const size_t bytes = nb * (4 * sizeof(double) + sizeof(int32_t));
    if ((st = ensure_stage(c, bytes)) != FD2_OK) return st;
    char *h = (char *)c->h_stage;
    std::memcpy(h, x_cm, nb * 8);
    std::memcpy(h + nb * 8, y_cm, nb * 8);
    std::memcpy(h + nb * 16, z_cm, nb * 8);
    std::memcpy(h + nb * 24, de_ev, nb * 8);
    std::memcpy(h + nb * 32, hist, nb * 4);
    FD2_CUDA(c, cudaMemcpyAsync(c->d_stage, c->h_stage, bytes, cudaMemcpyHostToDevice, c->stream));
    const char *d = (const char *)c->d_stage;
    FD2_CUDA(c, fd2::launch_prep_cm(c->stream, n, (const double *)d, (const double *)(d + nb * 8),
                                    (const double *)(d + nb * 16), (const double *)(d + nb * 24),
                                    (const int32_t *)(d + nb * 32), c->n_prim, c->d_ev_pos, c->d_ev_e, c->d_ev_xyz,
                                    c->d_flags));
    c->has_geom = false;
    double mu = 0.0;
    std::vector<float> xs(nb), ys(nb);
    for (size_t i = 0; i < nb; ++i) {
        if (de_ev[i] > 0.0) mu += de_ev[i] * c->params.yield;
        xs[i] = (float)(x_cm[i] * (double)10000.0f);
        ys[i] = (float)(y_cm[i] * (double)10000.0f);
    }
    c->mu_total = mu;
    return submit_common(c, n, xs.data(), ys.data(), nullptr);
}

fd2_status fd2_submit_events_device(fd2_ctx *c, const double *x_cm, const double *y_cm, const double *z_cm,
                                    const double *de_ev, const int32_t *hist, int64_t n)
{
    if (c && c->ingest_active) return fail(c, FD2_ERR_STATE, "an event ingest is open; end it first");
    if (!c || n < 0 || (n > 0 && (!x_cm || !y_cm || !z_cm || !de_ev || !hist)) || n >= ((int64_t)1 << 31))
        return fail(c, FD2_ERR_INVALID_ARGUMENT, "submit_events_device: null array or bad count");
    if (c->run_pending) {
        const fd2_status w = fd2_wait(c);
        if (w != FD2_OK) return w;
    }
    if (c->geoms.size() != 1) return fail(c, FD2_ERR_STATE, "cm submission is for a single geometry; use fd2_submit_events_um");
    if (c->opt.count_mode == FD2_COUNT_GIVEN) return fail(c, FD2_ERR_STATE, "count_mode GIVEN needs fd2_submit_events_um");
    FD2_CUDA(c, cudaSetDevice(c->device));
    if (n > 0)
        for (const void *p : {(const void *)x_cm, (const void *)y_cm, (const void *)z_cm, (const void *)de_ev,
                              (const void *)hist}) {
            cudaPointerAttributes at{};
            if (cudaPointerGetAttributes(&at, p) != cudaSuccess ||
                (at.type != cudaMemoryTypeDevice && at.type != cudaMemoryTypeManaged) || at.device != c->device) {
                cudaGetLastError();
                return fail(c, FD2_ERR_INVALID_ARGUMENT, "submit_events_device: an array is not device memory of the context's GPU");
            }
        }
    fd2_status st = ensure_events(c, n);
    if (st != FD2_OK) return st;
    FD2_CUDA(c, fd2::launch_prep_cm(c->stream, n, x_cm, y_cm, z_cm, de_ev, hist, c->n_prim, c->d_ev_pos, c->d_ev_e,
                                    c->d_ev_xyz, c->d_flags));
    c->has_geom = false;
    // sums of x, y (um, as the host path rounds them) and of the energies
    double sums[3] = {0, 0, 0};
    if (n > 0) {
        double *d_sums = nullptr;
        FD2_CUDA(c, cudaMallocAsync((void **)&d_sums, 3 * sizeof(double), c->stream));
        FD2_CUDA(c, cudaMemsetAsync(d_sums, 0, 3 * sizeof(double), c->stream));
        FD2_CUDA(c, fd2::launch_event_sums(c->stream, n, x_cm, y_cm, de_ev, d_sums));
        FD2_CUDA(c, cudaMemcpyAsync(sums, d_sums, sizeof sums, cudaMemcpyDeviceToHost, c->stream));
        FD2_CUDA(c, cudaFreeAsync(d_sums, c->stream));
        FD2_CUDA(c, cudaStreamSynchronize(c->stream));
    }
    c->mu_total = sums[2] * c->params.yield;
    return submit_common(c, n, nullptr, nullptr, nullptr, sums);
}

fd2_status fd2_submit_events_um(fd2_ctx *c, const float *x_um, const float *y_um, const float *z_um, const float *e_ev,
                                const int32_t *hist, const int32_t *nphot, const uint16_t *geom, int64_t n)
{
    if (c && c->ingest_active) return fail(c, FD2_ERR_STATE, "an event ingest is open; end it first");
    if (!c || n < 0 || (n > 0 && (!x_um || !y_um || !z_um || !hist)) || n >= ((int64_t)1 << 31))
        return fail(c, FD2_ERR_INVALID_ARGUMENT, "submit_events_um: null array or bad count");
    if (c->run_pending) {
        const fd2_status w = fd2_wait(c);
        if (w != FD2_OK) return w;
    }
    if (c->opt.count_mode == FD2_COUNT_GIVEN && n > 0 && !nphot)
        return fail(c, FD2_ERR_INVALID_ARGUMENT, "count_mode GIVEN needs photon counts");
    if (c->opt.count_mode != FD2_COUNT_GIVEN && n > 0 && !e_ev)
        return fail(c, FD2_ERR_INVALID_ARGUMENT, "energies are needed to sample photon counts");
    const size_t G = c->geoms.size();
    if (geom)
        for (int64_t i = 0; i < n; ++i)
            if (geom[i] >= G) return fail(c, FD2_ERR_INVALID_ARGUMENT, "geometry id out of range");
    FD2_CUDA(c, cudaSetDevice(c->device));
    fd2_status st = ensure_events(c, n);
    if (st != FD2_OK) return st;
    const size_t nb = (size_t)n;
    const size_t bytes = nb * (4 * sizeof(float) + 2 * sizeof(int32_t) + sizeof(uint16_t)) + 64;
    if ((st = ensure_stage(c, bytes)) != FD2_OK) return st;
    char *h = (char *)c->h_stage;
    std::memcpy(h, x_um, nb * 4);
    std::memcpy(h + nb * 4, y_um, nb * 4);
    std::memcpy(h + nb * 8, z_um, nb * 4);
    if (e_ev) std::memcpy(h + nb * 12, e_ev, nb * 4);
    else std::memset(h + nb * 12, 0, nb * 4);
    std::memcpy(h + nb * 16, hist, nb * 4);
    if (nphot) std::memcpy(h + nb * 20, nphot, nb * 4);
    else std::memset(h + nb * 20, 0, nb * 4);
    if (geom) std::memcpy(h + nb * 24, geom, nb * 2);
    FD2_CUDA(c, cudaMemcpyAsync(c->d_stage, c->h_stage, nb * 24 + (geom ? nb * 2 : 0), cudaMemcpyHostToDevice, c->stream));
    const char *d = (const char *)c->d_stage;
    FD2_CUDA(c, fd2::launch_prep_um(c->stream, n, (const float *)d, (const float *)(d + nb * 4),
                                    (const float *)(d + nb * 8), (const float *)(d + nb * 12),
                                    (const int32_t *)(d + nb * 16), c->n_prim, c->d_ev_pos, c->d_ev_e, c->d_ev_xyz,
                                    c->d_flags));
    if (n) FD2_CUDA(c, cudaMemcpyAsync(c->d_given_n, d + nb * 20, nb * 4, cudaMemcpyDeviceToDevice, c->stream));
    c->has_geom = geom != nullptr && G > 1;
    if (geom && n) FD2_CUDA(c, cudaMemcpyAsync(c->d_ev_geom, d + nb * 24, nb * 2, cudaMemcpyDeviceToDevice, c->stream));
    double mu = 0.0;
    if (c->opt.count_mode == FD2_COUNT_GIVEN) {
        for (size_t i = 0; i < nb; ++i) mu += nphot[i] > 0 ? nphot[i] : 0;
    } else {
        for (size_t i = 0; i < nb; ++i)
            if (e_ev[i] > 0.0f) mu += (double)e_ev[i] * c->params.yield;
    }
    c->mu_total = mu;
    st = submit_common(c, n, x_um, y_um, c->has_geom ? geom : nullptr);
    if (st == FD2_OK && G > 1) {
        // histories per geometry for PRF normalisation
        std::vector<int32_t> seen((size_t)c->n_prim + 1, -1);
        for (size_t i = 0; i < nb; ++i) {
            const int32_t hh = hist[i];
            const int gg = geom ? geom[i] : 0;
            if (hh >= 1 && hh <= c->n_prim && seen[(size_t)hh] < 0) {
                seen[(size_t)hh] = gg;
                c->hist_per_geom[(size_t)gg] += 1.0;
            }
        }
    }
    return st;
}

fd2_status fd2_run(fd2_ctx *c)
{
    if (c && c->ingest_active) return fail(c, FD2_ERR_STATE, "an event ingest is open; end it first");
    if (!c) return FD2_ERR_INVALID_ARGUMENT;
    if (c->n_events <= 0 && !c->ran_once && c->cap_events == 0 && !c->submitted)
        return fail(c, FD2_ERR_STATE, "no events submitted");
    FD2_CUDA(c, cudaSetDevice(c->device));
    if (c->n_events <= 0) {
        // an empty submission: nothing to transport, tallies unchanged
        FD2_CUDA(c, cudaMemsetAsync(c->d_scalars + 3, 0, sizeof(unsigned long long) * c->geoms.size(), c->stream));
        cudaEvent_t marks[4] = {c->ev_start, c->ev_t0, c->ev_t1, c->ev_end};
        for (cudaEvent_t e : marks) FD2_CUDA(c, cudaEventRecord(e, c->stream));
        c->run_pending = true;
        c->counts_ready = true;
        c->ran_once = true;
        return FD2_OK;
    }
    fd2_status st = ensure_chunks(c);
    if (st != FD2_OK) return st;
    *c->h_abort = 0;
    if (c->opt.use_graph && !c->graph_valid && (st = build_graph(c)) != FD2_OK) return st;
    cudaEvent_t marks[4] = {c->ev_start, c->ev_t0, c->ev_t1, c->ev_end};
    for (int seg = 0; seg < 3; ++seg) {
        FD2_CUDA(c, cudaEventRecord(marks[seg], c->stream));
        if (c->opt.use_graph) FD2_CUDA(c, cudaGraphLaunch(c->graph[seg], c->stream));
        else FD2_CUDA(c, enqueue_segment(c, seg));
    }
    FD2_CUDA(c, cudaEventRecord(marks[3], c->stream));
    c->run_pending = true;
    c->counts_ready = true;
    c->ran_once = true;
    return FD2_OK;
}

fd2_status fd2_wait(fd2_ctx *c)
{
    if (!c) return FD2_ERR_INVALID_ARGUMENT;
    if (!c->run_pending) return FD2_OK;
    FD2_CUDA(c, cudaSetDevice(c->device));
    fd2_status result = FD2_OK;
    if (c->opt.wait_timeout_s > 0.0) {
        const auto t0 = std::chrono::steady_clock::now();
        for (;;) {
            const cudaError_t q = cudaEventQuery(c->ev_end);
            if (q == cudaSuccess) break;
            if (q != cudaErrorNotReady) return cuda_fail(c, q, "fd2_wait");
            const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            if (el > c->opt.wait_timeout_s) {
                // ask the persistent kernel to stop taking work; it drains what
                // its lanes hold and exits
                *(volatile int *)c->h_abort = 1;
                result = fail(c, FD2_ERR_TIMEOUT, "run exceeded wait_timeout_s; aborted, tallies are partial");
                break;
            }
            std::this_thread::sleep_for(std::chrono::microseconds(100));
        }
    }
    FD2_CUDA(c, cudaEventSynchronize(c->ev_end));
    *c->h_abort = 0;
    c->run_pending = false;
    const size_t G = c->geoms.size();
    std::vector<unsigned long long> ph(G);
    FD2_CUDA(c, cudaMemcpy(ph.data(), c->d_scalars + 3, sizeof(unsigned long long) * G, cudaMemcpyDeviceToHost));
    c->last_photons = 0;
    for (size_t g = 0; g < G; ++g) c->last_photons += (int64_t)ph[g];
    const fd2_status st = check_status(c);
    if (result != FD2_OK) return result;
    return st;
}

fd2_status fd2_reset_tallies(fd2_ctx *c)
{
    if (c && c->ingest_active) return fail(c, FD2_ERR_STATE, "an event ingest is open; end it first");
    if (!c) return FD2_ERR_INVALID_ARGUMENT;
    if (c->run_pending) return fail(c, FD2_ERR_STATE, "wait first");
    FD2_CUDA(c, cudaSetDevice(c->device));
    const size_t G = c->geoms.size();
    FD2_CUDA(c, cudaMemsetAsync(c->d_prf, 0, sizeof(unsigned long long) * (size_t)std::max<int64_t>(c->prf_total, 1), c->stream));
    FD2_CUDA(c, cudaMemsetAsync(c->d_counters, 0, sizeof(unsigned long long) * G * fd2::kCounterStride, c->stream));
    FD2_CUDA(c, cudaMemsetAsync(c->d_distance, 0, sizeof(double) * G, c->stream));
    FD2_CUDA(c, cudaMemsetAsync(c->d_per_primary, 0, sizeof(int32_t) * (size_t)std::max(c->n_prim, 1), c->stream));
    if (c->d_radial) FD2_CUDA(c, cudaMemsetAsync(c->d_radial, 0, sizeof(uint32_t) * (size_t)c->radial_len, c->stream));
    FD2_CUDA(c, cudaMemsetAsync(c->d_prim_geom, 0, sizeof(int32_t) * (size_t)std::max(c->n_prim, 1), c->stream));
    FD2_CUDA(c, cudaMemsetAsync(c->d_phs, 0, sizeof(int32_t) * G * (size_t)std::max(c->params.num_bins, 1), c->stream));
    FD2_CUDA(c, cudaMemsetAsync(c->d_moments, 0, sizeof(double) * G * 3, c->stream));
    FD2_CUDA(c, cudaMemsetAsync(c->d_dropped, 0, sizeof(unsigned long long) * G, c->stream));
    FD2_CUDA(c, cudaMemsetAsync(c->d_flags + 1, 0, sizeof(int), c->stream));
    FD2_CUDA(c, cudaMemsetAsync(c->d_gen_total, 0, sizeof(unsigned long long) * G, c->stream));
    FD2_CUDA(c, cudaStreamSynchronize(c->stream));
    return FD2_OK;
}

fd2_status fd2_get_counters(fd2_ctx *c, int32_t geom, fd2_counters *out)
{
    if (!c || !out || geom < 0 || (size_t)geom >= c->geoms.size()) return fail(c, FD2_ERR_INVALID_ARGUMENT, "geometry");
    fd2_status st = fd2_wait(c);
    if (st != FD2_OK) return st;
    unsigned long long k[fd2::kCounterStride];
    double dist = 0.0;
    FD2_CUDA(c, cudaMemcpy(k, c->d_counters + (size_t)geom * fd2::kCounterStride, sizeof k, cudaMemcpyDeviceToHost));
    FD2_CUDA(c, cudaMemcpy(&dist, c->d_distance + geom, sizeof dist, cudaMemcpyDeviceToHost));
    std::memset(out, 0, sizeof *out);
    out->detected = k[fd2::kDetect];
    out->abs_top = k[fd2::kAbsTop];
    out->abs_bulk = k[fd2::kAbsBulk];
    out->lost = k[fd2::kLost];
    out->outofcol = k[fd2::kOutOfCol];
    out->theta1 = k[fd2::kTheta1];
    out->capped = k[fd2::kCapped];
    out->detected_in_prf = k[fd2::kNumFates];
    unsigned long long gen = 0;
    FD2_CUDA(c, cudaMemcpy(&gen, c->d_gen_total + geom, sizeof gen, cudaMemcpyDeviceToHost));
    out->generated = gen;
    out->photon_distance = dist;
    return FD2_OK;
}

fd2_status fd2_get_prf_dims(fd2_ctx *c, int32_t geom, int32_t *xdim, int32_t *ydim)
{
    if (!c || !xdim || !ydim || geom < 0 || (size_t)geom >= c->geoms.size()) return FD2_ERR_INVALID_ARGUMENT;
    *xdim = c->dgeoms[(size_t)geom].xdim;
    *ydim = c->dgeoms[(size_t)geom].ydim;
    return FD2_OK;
}

fd2_status fd2_get_prf(fd2_ctx *c, int32_t geom, uint64_t *image, int64_t n)
{
    if (!c || !image || geom < 0 || (size_t)geom >= c->geoms.size()) return fail(c, FD2_ERR_INVALID_ARGUMENT, "geometry");
    const DevGeom &g = c->dgeoms[(size_t)geom];
    const int64_t m = (int64_t)g.xdim * g.ydim;
    if (n < m) return fail(c, FD2_ERR_INVALID_ARGUMENT, "image buffer too small");
    fd2_status st = fd2_wait(c);
    if (st != FD2_OK) return st;
    FD2_CUDA(c, cudaMemcpy(image, c->d_prf + g.prf_offset, sizeof(uint64_t) * (size_t)m, cudaMemcpyDeviceToHost));
    return FD2_OK;
}

fd2_status fd2_get_detected_per_primary(fd2_ctx *c, int32_t *counts, int64_t n)
{
    if (!c || !counts || n < c->n_prim) return fail(c, FD2_ERR_INVALID_ARGUMENT, "buffer too small");
    fd2_status st = fd2_wait(c);
    if (st != FD2_OK) return st;
    if (c->n_prim) FD2_CUDA(c, cudaMemcpy(counts, c->d_per_primary, sizeof(int32_t) * (size_t)c->n_prim, cudaMemcpyDeviceToHost));
    return FD2_OK;
}

fd2_status fd2_get_radial(fd2_ctx *c, uint32_t *counts, int64_t n)
{
    if (!c) return FD2_ERR_INVALID_ARGUMENT;
    if (!c->d_radial) return fail(c, FD2_ERR_STATE, "label mode is off (options.radial_bins = 0)");
    if (!counts || n < c->radial_len) return fail(c, FD2_ERR_INVALID_ARGUMENT, "buffer too small");
    fd2_status st = fd2_wait(c);
    if (st != FD2_OK) return st;
    FD2_CUDA(c, cudaMemcpy(counts, c->d_radial, sizeof(uint32_t) * (size_t)c->radial_len, cudaMemcpyDeviceToHost));
    return FD2_OK;
}

fd2_status fd2_get_photon_counts(fd2_ctx *c, int32_t *nphot, int64_t n)
{
    if (!c || !nphot || n < c->n_events) return fail(c, FD2_ERR_INVALID_ARGUMENT, "buffer too small");
    fd2_status st = fd2_wait(c);
    if (st != FD2_OK) return st;
    if (!c->counts_ready) return fail(c, FD2_ERR_STATE, "photon counts are sampled by fd2_run");
    if (c->n_events) FD2_CUDA(c, cudaMemcpy(nphot, c->d_ev_n, sizeof(int32_t) * (size_t)c->n_events, cudaMemcpyDeviceToHost));
    return FD2_OK;
}

fd2_status fd2_get_phs(fd2_ctx *c, int32_t geom, int32_t *bins, int32_t num_bins)
{
    if (!c || !bins || geom < 0 || (size_t)geom >= c->geoms.size() || num_bins != c->params.num_bins)
        return fail(c, FD2_ERR_INVALID_ARGUMENT, "geometry or bin count");
    if (c->params.num_bins <= 0 || c->params.max_photons - c->params.min_photons < c->params.num_bins)
        return fail(c, FD2_ERR_INVALID_ARGUMENT, "PHS bin width (max-min)/bins is zero");
    fd2_status st = fd2_wait(c);
    if (st != FD2_OK) return st;
    FD2_CUDA(c, cudaMemcpy(bins, c->d_phs + (size_t)geom * num_bins, sizeof(int32_t) * (size_t)num_bins, cudaMemcpyDeviceToHost));
    return FD2_OK;
}

fd2_status fd2_get_phs_stats(fd2_ctx *c, int32_t geom, fd2_phs_stats *out)
{
    if (!c || !out || geom < 0 || (size_t)geom >= c->geoms.size()) return fail(c, FD2_ERR_INVALID_ARGUMENT, "geometry");
    fd2_status st = fd2_wait(c);
    if (st != FD2_OK) return st;
    double m[3];
    unsigned long long dr = 0;
    FD2_CUDA(c, cudaMemcpy(m, c->d_moments + (size_t)geom * 3, sizeof m, cudaMemcpyDeviceToHost));
    FD2_CUDA(c, cudaMemcpy(&dr, c->d_dropped + geom, sizeof dr, cudaMemcpyDeviceToHost));
    out->primaries = m[0];
    out->sum = m[1];
    out->sum_sq = m[2];
    out->mean = m[0] > 0 ? m[1] / m[0] : 0.0;
    out->swank = (m[0] > 0 && m[2] > 0) ? (m[1] * m[1]) / (m[0] * m[2]) : 0.0;
    out->phs_dropped = (int64_t)dr;
    return FD2_OK;
}

fd2_status fd2_get_timing(fd2_ctx *c, fd2_timing *out)
{
    if (!c || !out) return FD2_ERR_INVALID_ARGUMENT;
    fd2_status st = fd2_wait(c);
    if (st != FD2_OK) return st;
    std::memset(out, 0, sizeof *out);
    if (c->ran_once) {
        FD2_CUDA(c, cudaEventElapsedTime(&out->transport_ms, c->ev_t0, c->ev_t1));
        FD2_CUDA(c, cudaEventElapsedTime(&out->pipeline_ms, c->ev_start, c->ev_end));
    }
    out->photons = c->last_photons;
    out->grid = c->sm_count * c->cfg.ctas_per_sm;
    out->block = c->cfg.block;
    out->chunk = c->cfg.chunk;
    out->refill = c->cfg.refill;
    out->prf_window = c->cfg.window;
    out->fresnel_batch = c->cfg.fresnel;
    return FD2_OK;
}

void *fd2_get_stream(fd2_ctx *c) { return c ? (void *)c->stream : nullptr; }

fd2_status fd2_write_outputs(fd2_ctx *c, const char *dir)
{
    if (!c || !dir) return FD2_ERR_INVALID_ARGUMENT;
    fd2_status st = fd2_wait(c);
    if (st != FD2_OK) return st;
    const size_t G = c->geoms.size();
    const int32_t nb = c->params.num_bins;
    if (nb <= 0 || c->params.max_photons - c->params.min_photons < nb)
        return fail(c, FD2_ERR_INVALID_ARGUMENT, "PHS bin width (max-min)/bins is zero");
    for (size_t g = 0; g < G; ++g) {
        const DevGeom &d = c->dgeoms[g];
        std::vector<uint64_t> img((size_t)d.xdim * d.ydim);
        std::vector<int32_t> phs((size_t)nb);
        if ((st = fd2_get_prf(c, (int32_t)g, img.data(), (int64_t)img.size())) != FD2_OK) return st;
        if ((st = fd2_get_phs(c, (int32_t)g, phs.data(), nb)) != FD2_OK) return st;
        const std::string suffix = G > 1 ? "_geom" + std::to_string(g) : std::string();
        const double nh = G > 1 ? std::max(c->hist_per_geom[g], 1.0) : (double)std::max(c->params.num_hist, 1);
        st = fd2_write_output_files(&c->params, &c->geoms[g], img.data(), d.xdim, d.ydim, phs.data(), nb, nh, dir,
                                    suffix.c_str());
        if (st != FD2_OK) return fail(c, st, std::string("writing the output files in ") + dir);
    }
    return FD2_OK;
}

fd2_status fd2_replay(fd2_ctx *c, int32_t mode, int32_t seed_input, int64_t event_index_base, int8_t *fate,
                      int32_t *pix, int32_t *seeds, int32_t *steps)
{
    if (c && c->ingest_active) return fail(c, FD2_ERR_STATE, "an event ingest is open; end it first");
    if (!c || (mode != FD2_REPLAY_REF && mode != FD2_REPLAY_FP64) || seed_input <= 0 || event_index_base < 0)
        return fail(c, FD2_ERR_INVALID_ARGUMENT, "replay mode / seed");
    if (c->opt.column_grid) return fail(c, FD2_ERR_STATE, "the replay follows the reference's column model only");
    fd2_status st = fd2_wait(c);
    if (st != FD2_OK) return st;
    FD2_CUDA(c, cudaSetDevice(c->device));
    if (mode == FD2_REPLAY_REF && (st = load_libm_table(c)) != FD2_OK) return st;
    if (!c->counts_ready) {
        FD2_CUDA(c, count_pass(c, false));
        if ((st = check_status(c)) != FD2_OK) return st;
        c->counts_ready = true;
    }
    // photon offsets of the events (exclusive scan of the counts)
    unsigned long long *first = nullptr;
    FD2_CUDA(c, cudaMallocAsync((void **)&first, sizeof(unsigned long long) * (size_t)std::max<int64_t>(c->n_events, 1), c->stream));
    cudaError_t e = fd2::launch_photon_offsets(c->stream, c->n_events, c->d_ev_n, first, c->d_block_sums, c->d_scalars + 2);
    unsigned long long total = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&total, c->d_scalars + 2, sizeof total, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    int8_t *d_fate = nullptr;
    int32_t *d_pix = nullptr, *d_seeds = nullptr, *d_steps = nullptr;
    const size_t T = (size_t)std::max<unsigned long long>(total, 1);
    if (e == cudaSuccess && fate) e = cudaMallocAsync((void **)&d_fate, T, c->stream);
    if (e == cudaSuccess && pix) e = cudaMallocAsync((void **)&d_pix, 8 * T, c->stream);
    if (e == cudaSuccess && seeds) e = cudaMallocAsync((void **)&d_seeds, 8 * T, c->stream);
    if (e == cudaSuccess && steps) e = cudaMallocAsync((void **)&d_steps, 4 * T, c->stream);
    if (e == cudaSuccess) {
        fd2::ReplayArgs a;
        a.n_events = c->n_events;
        a.ev_pos = c->d_ev_pos;
        a.ev_pos_d = c->d_ev_xyz;
        a.ev_n = c->d_ev_n;
        a.ev_geom = c->has_geom ? c->d_ev_geom : nullptr;
        a.ev_first = first;
        a.geoms = c->d_geoms;
        a.n_geom = (int)c->geoms.size();
        a.seed_input = seed_input;
        a.event_index_base = event_index_base;
        a.prf = c->d_prf;
        a.per_primary = c->d_per_primary;
        a.n_prim = c->n_prim;
        a.counters = c->d_counters;
        a.gen_total = c->d_gen_total;
        a.fate = d_fate;
        a.pix = d_pix;
        a.seeds = d_seeds;
        a.steps = d_steps;
        a.acos_tab = mode == FD2_REPLAY_REF ? c->d_libm : nullptr;
        a.asin_tab = mode == FD2_REPLAY_REF ? c->d_libm + c->n_acos : nullptr;
        a.n_acos = c->n_acos;
        a.n_asin = c->n_asin;
        e = fd2::launch_replay(c->stream, mode, a);
    }
    if (e == cudaSuccess && fate) e = cudaMemcpyAsync(fate, d_fate, total, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess && pix) e = cudaMemcpyAsync(pix, d_pix, 8 * total, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess && seeds) e = cudaMemcpyAsync(seeds, d_seeds, 8 * total, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess && steps) e = cudaMemcpyAsync(steps, d_steps, 4 * total, cudaMemcpyDeviceToHost, c->stream);
    for (void *p : {(void *)first, (void *)d_fate, (void *)d_pix, (void *)d_seeds, (void *)d_steps})
        if (p) cudaFreeAsync(p, c->stream);
    const cudaError_t e2 = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "replay");
    if (e2 != cudaSuccess) return cuda_fail(c, e2, "replay");
    return FD2_OK;
}

fd2_status fd2_autotune(fd2_ctx *c, int32_t budget_runs)
{
    if (c && c->ingest_active) return fail(c, FD2_ERR_STATE, "an event ingest is open; end it first");
    if (!c) return FD2_ERR_INVALID_ARGUMENT;
    if (c->n_events <= 0) return fail(c, FD2_ERR_STATE, "submit events before tuning");
    fd2_status st = fd2_wait(c);
    if (st != FD2_OK) return st;
    fd2::TransportConfig best = c->cfg;
    if (tune_cache_lookup(c, &best)) return set_config(c, best);
    auto time_cfg = [&](const fd2::TransportConfig &k, float *ms) -> fd2_status {
        fd2_status s = set_config(c, k);
        if (s != FD2_OK) return s;
        if ((s = ensure_chunks(c)) != FD2_OK) return s;
        float tot = 0.0f;
        for (int r = 0; r < 2; ++r) {
            if ((s = fd2_run(c)) != FD2_OK || (s = fd2_wait(c)) != FD2_OK) return s;
            fd2_timing t;
            if ((s = fd2_get_timing(c, &t)) != FD2_OK) return s;
            if (r) tot += t.transport_ms;
        }
        *ms = tot;
        return FD2_OK;
    };
    float best_ms = 0.0f;
    if ((st = time_cfg(best, &best_ms)) != FD2_OK) return st;
    int runs = 2;
    // launch shapes as (threads per CTA, CTAs per SM) pairs -- the register
    // budget of each compiled variant ties the two together -- then chunk,
    // refill and Fresnel batch one knob at a time, twice over
    const std::vector<std::pair<int, int>> shapes = {{256, 4}, {128, 8}, {256, 3}, {320, 2}, {256, 2}, {512, 1}};
    const std::vector<int> chunks = {8, 16, 32, 64, 128};
    const std::vector<int> refills = {1, 2, 4, 8, 16};
    const std::vector<int> fresnels = {1, 4, 8, 12, 16};
    auto try_cfg = [&](const fd2::TransportConfig &k) {
        // the CTA's shared memory must fit ctas_per_sm times (set_config
        // shrinks the PRF window to fit; without it, skip)
        fd2::TransportConfig bare = k;
        bare.window = 0;
        if (fd2::transport_smem_bytes(bare, (int)c->geoms.size()) * (size_t)k.ctas_per_sm > 220 * 1024) return;
        float ms = 0.0f;
        if (time_cfg(k, &ms) != FD2_OK) return;
        runs += 2;
        if (ms < best_ms) {
            best_ms = ms;
            best = k;
        }
    };
    for (int pass = 0; pass < 2; ++pass) {
        for (const auto &sh : shapes) {
            if (budget_runs > 0 && runs >= budget_runs) break;
            if (sh.first == best.block && sh.second == best.ctas_per_sm) continue;
            fd2::TransportConfig k = best;
            k.block = sh.first;
            k.ctas_per_sm = sh.second;
            try_cfg(k);
        }
        for (int knob = 0; knob < 3; ++knob) {
            const std::vector<int> &vals = knob == 0 ? chunks : knob == 1 ? refills : fresnels;
            for (int v : vals) {
                if (budget_runs > 0 && runs >= budget_runs) break;
                fd2::TransportConfig k = best;
                int &slot = knob == 0 ? k.chunk : knob == 1 ? k.refill : k.fresnel;
                if (slot == v) continue;
                slot = v;
                try_cfg(k);
            }
        }
    }
    if ((st = set_config(c, best)) != FD2_OK) return st;
    if ((st = ensure_chunks(c)) != FD2_OK) return st;
    tune_cache_store(c);
    return fd2_reset_tallies(c);
}

}  // extern "C"
