// fd2_noalloc.cu -- fd2_transport_noalloc: the transport without allocating.
//
// For callers that cannot allocate device memory themselves: code that runs
// inside another framework's memory pool, a process whose CUDA allocations
// are owned by an embedding application, or a hook that may not change the
// device's memory footprint while it runs.  They pass device buffers for the
// events and the tallies; the work-queue scratch (packed events, photon
// counts, chunk counts and offsets, chunk descriptors, status words) lives in
// one file-scope __device__ array of fixed size that every GPU loading the
// library holds until the process exits.
//
// Set-up: the first call on each device, with that device current, looks up
// the array's device address with cudaGetSymbolAddress (the array's name in
// host code is only a host-side stand-in, not a device address).  That first
// call should come before any stream capture on the device.
//
// Every call uses the same array and leaves its contents behind; the call
// clears what must start at zero.  Calls whose work overlaps on the GPU
// (several streams, several host threads) race on the array: serialise them.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>

#include "fd2.h"
#include "fd2_internal.h"

namespace {

// Limits of one call.
constexpr int64_t kNaMaxEvents = 262144;
constexpr int64_t kNaMaxChunks = 2097152;
constexpr int kNaChunk = 256;  // photons per queue chunk
constexpr int64_t kNaMaxPerEvent = 900000;  // photons per event (the reference's own cap)
constexpr int kNaMaxDevices = 64;

// Scratch layout (bytes, each part 256-byte aligned).
constexpr size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }
constexpr size_t kOffScalars = 0;                                   // 64 x u64: chunks, head, photons, ...
constexpr size_t kOffFlags = kOffScalars + align256(64 * 8);        // status, run counter
constexpr size_t kOffDist = kOffFlags + align256(16);               // path length (double)
constexpr size_t kOffPos = kOffDist + align256(16);                 // float4 per event
constexpr size_t kOffN = kOffPos + align256(16 * kNaMaxEvents);     // photons per event
constexpr size_t kOffNChunks = kOffN + align256(4 * kNaMaxEvents);  // chunks per event
constexpr size_t kOffOffsets = kOffNChunks + align256(4 * kNaMaxEvents);
constexpr size_t kOffBlockSums = kOffOffsets + align256(8 * kNaMaxEvents);
constexpr size_t kOffChunks = kOffBlockSums + align256(8 * (kNaMaxEvents / 4096 + 2));
constexpr size_t kScratchBytes = kOffChunks + align256(8 * kNaMaxChunks);  // ~24 MiB

static __device__ __align__(256) unsigned char fd2_noalloc_scratch[kScratchBytes];

unsigned char *g_scratch[kNaMaxDevices];
std::mutex g_setup;

// Pack the caller's event arrays (um, 1-based history) into the queue's
// float4 records, flagging invalid values.
__global__ void noalloc_pack(int64_t n, const float *__restrict__ x, const float *__restrict__ y,
                             const float *__restrict__ z, const int32_t *__restrict__ hist,
                             const int32_t *__restrict__ nphot, int32_t num_hist, float4 *__restrict__ pos, int *status)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t h = hist[i];
        if (!(isfinite(x[i]) && isfinite(y[i]) && isfinite(z[i])) || h < 1 || h > num_hist || nphot[i] < 0)
            atomicOr(status, fd2::kStatusBadEvent);
        pos[i] = make_float4(x[i], y[i], z[i], __int_as_float(h - 1));
    }
}

// Runs between the queue construction and the transport: when the call is
// going to be rejected (a flagged event, an event above the photon cap, more
// chunks than the scratch holds -- fill_chunks then leaves stale descriptors
// of an earlier call behind the ones it wrote), the queue is emptied so the
// transport tallies nothing and the caller's buffers stay as they were.
__global__ void noalloc_guard(const int *status, unsigned long long *n_chunks)
{
    constexpr int kReject = fd2::kStatusBadEvent | fd2::kStatusTooManyPhotons | fd2::kStatusChunkOverflow;
    if (threadIdx.x == 0 && (*status & kReject)) *n_chunks = 0ull;
}

fd2_status scratch_for_current_device(unsigned char **out)
{
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNaMaxDevices) return FD2_ERR_NO_DEVICE;
    std::lock_guard<std::mutex> lock(g_setup);
    if (!g_scratch[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, fd2_noalloc_scratch) != cudaSuccess || !p) return FD2_ERR_CUDA;
        g_scratch[dev] = (unsigned char *)p;
    }
    *out = g_scratch[dev];
    return FD2_OK;
}

}  // namespace

extern "C" fd2_status fd2_transport_noalloc(const fd2_geometry *geometry, const float *x_um, const float *y_um,
                                           const float *z_um, const int32_t *hist, const int32_t *nphot, int64_t n,
                                           int32_t num_hist, uint64_t seed, uint64_t *prf, int32_t *per_primary,
                                           uint64_t *counters, void *stream)
{
    if (!geometry || n < 0 || num_hist <= 0 || !prf || !per_primary || !counters ||
        (n > 0 && (!x_um || !y_um || !z_um || !hist || !nphot)))
        return FD2_ERR_INVALID_ARGUMENT;
    if (n > kNaMaxEvents) return FD2_ERR_INVALID_ARGUMENT;  // more events than the scratch holds
    int32_t xd = 0, yd = 0;
    if (fd2_prf_dims(geometry, &xd, &yd) != FD2_OK || geometry->det_height <= 0 || geometry->radius <= 0)
        return FD2_ERR_INVALID_ARGUMENT;
    unsigned char *base = nullptr;
    fd2_status st = scratch_for_current_device(&base);
    if (st != FD2_OK) return st;
    int sms = 0, dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return FD2_ERR_CUDA;
    cudaStream_t s = (cudaStream_t)stream;

    auto *scalars = reinterpret_cast<unsigned long long *>(base + kOffScalars);
    auto *flags = reinterpret_cast<int *>(base + kOffFlags);
    auto *dist = reinterpret_cast<double *>(base + kOffDist);
    auto *pos = reinterpret_cast<float4 *>(base + kOffPos);
    auto *ev_n = reinterpret_cast<int32_t *>(base + kOffN);
    auto *nchunks = reinterpret_cast<uint32_t *>(base + kOffNChunks);
    auto *offsets = reinterpret_cast<unsigned long long *>(base + kOffOffsets);
    auto *block_sums = reinterpret_cast<unsigned long long *>(base + kOffBlockSums);
    auto *chunks = reinterpret_cast<uint2 *>(base + kOffChunks);

    // geometry in the walk's float form (as fd2_create derives it)
    fd2::DevGeom g;
    std::memset(&g, 0, sizeof g);
    g.xdet = (float)geometry->det_x;
    g.ydet = (float)geometry->det_y;
    g.H = (float)geometry->det_height;
    g.half = g.H / 2.0f;
    g.R = (float)geometry->radius;
    g.beta = (float)geometry->beta;
    g.top_absfrac = (float)geometry->top_absfrac;
    g.mu = (float)geometry->bulk_abs;
    g.neg_inv_mu = g.mu > 0.0f ? -1.0f / g.mu : 0.0f;
    g.d_min = (float)geometry->d_min;
    g.d_max = (float)geometry->d_max;
    g.d_span = g.d_max - g.d_min;
    g.lb_x = (float)geometry->lb_x;
    g.lb_y = (float)geometry->lb_y;
    g.ub_x = (float)geometry->ub_x;
    g.ub_y = (float)geometry->ub_y;
    g.sensor_refl = (float)geometry->sensor_refl;
    g.pixel = (float)geometry->pixel;
    const float band = g.H * 0.2f;
    g.cct_band_lo = g.half - band;
    g.cct_k_hi = 1.0f / (2.0f * (g.half - band));
    g.cct_k_lo = 1.0f / (2.0f * (-g.half));
    g.n_col = (float)geometry->n_col;
    g.n_gap = (float)geometry->n_gap;
    g.eta_in = g.n_col / g.n_gap;
    const double rin = (double)(g.n_gap / g.n_col);
    g.cos_tir_in = rin <= 1.0 ? (float)std::sqrt(1.0 - rin * rin) : -1.0f;
    g.eta_out = g.n_gap / g.n_col;
    g.stale_out = (g.n_col / g.n_gap) < 1.57f ? 1 : 0;
    const double rout = (double)(g.n_col / g.n_gap);
    g.cos_tir_out = rout <= 1.0 ? (float)std::sqrt(1.0 - rout * rout) : -1.0f;
    g.xdim = xd;
    g.ydim = yd;
    g.prf_offset = 0;

    fd2::TransportConfig cfg;
    cfg.block = 256;
    cfg.ctas_per_sm = 2;
    cfg.chunk = kNaChunk;
    cfg.refill = 8;
    cfg.window = 0;

    // what must start at zero: queue scalars, status and run counter, path length
    cudaError_t e = cudaMemsetAsync(base, 0, kOffPos, s);
    if (e == cudaSuccess && n > 0) {
        const unsigned grid = (unsigned)std::min<int64_t>((n + 255) / 256, 4096);
        noalloc_pack<<<grid, 256, 0, s>>>(n, x_um, y_um, z_um, hist, nphot, num_hist, pos, flags);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = fd2::launch_count(s, n, 0, fd2::kCountGiven, 0.0, kNaMaxPerEvent, seed, reinterpret_cast<const uint32_t *>(flags + 1),
                              cfg.chunk, nullptr, nphot, nullptr, pos, ev_n, nchunks, scalars + 3, nullptr, nullptr,
                              num_hist, flags);
    if (e == cudaSuccess) e = fd2::launch_scan(s, n, nchunks, offsets, block_sums, scalars + 0);
    if (e == cudaSuccess) e = fd2::launch_fill_chunks(s, n, cfg.chunk, ev_n, offsets, chunks, kNaMaxChunks, flags);
    if (e == cudaSuccess) {
        noalloc_guard<<<1, 32, 0, s>>>(flags, scalars + 0);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = fd2::prepare_transport(cfg, 1);
    if (e == cudaSuccess) {
        fd2::TransportArgs a;
        std::memset(&a, 0, sizeof a);
        a.ev_pos = pos;
        a.ev_geom = nullptr;
        a.ev_n = ev_n;
        a.chunks = chunks;
        a.n_chunks = scalars + 0;
        a.chunk_capacity = kNaMaxChunks;
        a.queue_head = scalars + 1;
        a.geoms = nullptr;
        a.n_geom = 1;
        a.g0 = g;
        a.prf = reinterpret_cast<unsigned long long *>(prf);
        a.per_primary = per_primary;
        a.n_prim = num_hist;
        a.counters = reinterpret_cast<unsigned long long *>(counters);
        a.distance = dist;
        a.seed = seed;
        a.event_base = 0;
        uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
        for (int r = 0; r < 10; ++r) {
            a.round_keys[2 * r] = k0;
            a.round_keys[2 * r + 1] = k1;
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        a.run_tag = reinterpret_cast<const uint32_t *>(flags + 1);
        a.chunk = cfg.chunk;
        a.refill = cfg.refill;
        a.fresnel_batch = cfg.fresnel;
        a.window = 0;
        a.abort_flag = nullptr;
        a.status = flags;
        e = fd2::launch_transport(s, cfg, sms, a);
    }
    int status = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&status, flags, sizeof status, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return e == cudaErrorMemoryAllocation ? FD2_ERR_OUT_OF_MEMORY : FD2_ERR_CUDA;
    if (status & fd2::kStatusBadEvent) return FD2_ERR_BAD_EVENT;
    if (status & fd2::kStatusTooManyPhotons) return FD2_ERR_TOO_MANY_PHOTONS;
    if (status & fd2::kStatusChunkOverflow) return FD2_ERR_INVALID_ARGUMENT;  // more photons than the scratch holds
    if (status & fd2::kStatusAborted) return FD2_ERR_DEVICE_ABORT;
    return FD2_OK;
}
