// fd2_kernels.cu -- event preparation, photon-count sampling, work-queue
// construction, the persistent transport kernel and the PHS/Swank pass.
//
// Pipeline of one run (all on the context's stream, graph-capturable):
//   prep      events -> float4 (x, y, z um; history index) + energy     (at submit)
//   count     N ~ Poisson(E * yield) | Gaussian | given; chunks per event
//   scan      exclusive scan of chunks per event
//   fill      chunk descriptors (event, first photon)
//   transport persistent kernel: warps pull chunks, lanes regenerate photons
//   phs       per-primary counts -> PHS histogram + FP64 moments (Swank)
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "fd2_device.cuh"
#include "fd2_internal.h"

namespace fd2 {

namespace {

constexpr unsigned kFull = 0xFFFFFFFFu;

__device__ __forceinline__ unsigned lanemask_lt()
{
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// ------------------------------------------------------------------ prep

__device__ __forceinline__ bool finite_f(double v) { return isfinite(v); }

__global__ void prep_cm_kernel(int64_t n, const double *__restrict__ x, const double *__restrict__ y,
                               const double *__restrict__ z, const double *__restrict__ de,
                               const int32_t *__restrict__ hist, int32_t n_prim, float4 *__restrict__ ev_pos,
                               double *__restrict__ ev_e, double *__restrict__ ev_xyz, int *status)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        // cm -> um exactly as the reference's host driver (double * 10000.0f),
        // then the float the transport carries
        const double xu = x[i] * (double)10000.0f, yu = y[i] * (double)10000.0f, zu = z[i] * (double)10000.0f;
        const int32_t h = hist[i];
        const double e = de[i];
        if (!(finite_f(xu) && finite_f(yu) && finite_f(zu) && finite_f(e)) || e < 0.0 || h < 1 || h > n_prim)
            atomicOr(status, kStatusBadEvent);
        ev_pos[i] = make_float4((float)xu, (float)yu, (float)zu, __int_as_float(h - 1));
        ev_e[i] = e;
        ev_xyz[3 * i] = xu;
        ev_xyz[3 * i + 1] = yu;
        ev_xyz[3 * i + 2] = zu;
    }
}

__global__ void prep_um_kernel(int64_t n, const float *__restrict__ x, const float *__restrict__ y,
                               const float *__restrict__ z, const float *__restrict__ e,
                               const int32_t *__restrict__ hist, int32_t n_prim, float4 *__restrict__ ev_pos,
                               double *__restrict__ ev_e, double *__restrict__ ev_xyz, int *status)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t h = hist[i];
        const double ee = e ? (double)e[i] : 0.0;
        if (!(isfinite(x[i]) && isfinite(y[i]) && isfinite(z[i]) && isfinite(ee)) || ee < 0.0 || h < 1 || h > n_prim)
            atomicOr(status, kStatusBadEvent);
        ev_pos[i] = make_float4(x[i], y[i], z[i], __int_as_float(h - 1));
        ev_e[i] = ee;
        ev_xyz[3 * i] = (double)x[i];
        ev_xyz[3 * i + 1] = (double)y[i];
        ev_xyz[3 * i + 2] = (double)z[i];
    }
}

// ---------------------------------------------------------------- counts

// Uniform double in (0, 1) from two 32-bit words.
__device__ __forceinline__ double u01d(uint32_t a, uint32_t b)
{
    const uint64_t m = ((uint64_t)a << 21) ^ (uint64_t)(b >> 11);  // 53 bits
    return ((double)(m & ((1ull << 53) - 1)) + 0.5) * (1.0 / 9007199254740992.0);
}

struct CountRng {
    uint32_t k0, k1, event, tag, block;
    uint4 buf;
    int avail;
    __device__ double u()
    {
        if (avail == 0) {
            buf = philox4x32_10(make_uint4(block++, kCountStream, event, tag), k0, k1);
            avail = 2;
        }
        const double r = avail == 2 ? u01d(buf.x, buf.y) : u01d(buf.z, buf.w);
        --avail;
        return r;
    }
};

// Poisson(mu): inversion by multiplication for mu < 10; above, the
// transformed rejection with squeeze PTRS of W. Hormann, "The transformed
// rejection method for generating Poisson random variables", Insurance:
// Mathematics and Economics 12 (1993) 39-45.
__device__ int64_t poisson(CountRng &rng, double mu)
{
    if (!(mu > 0.0)) return 0;
    if (mu < 10.0) {
        const double limit = exp(-mu);
        double prod = rng.u();
        int64_t k = 0;
        while (prod > limit && k < 1000) {
            prod *= rng.u();
            ++k;
        }
        return k;
    }
    const double smu = sqrt(mu), logmu = log(mu);
    const double b = 0.931 + 2.53 * smu;
    const double a = -0.059 + 0.02483 * b;
    const double inv_alpha = 1.1239 + 1.1328 / (b - 3.4);
    const double vr = 0.9277 - 3.6224 / (b - 2.0);
    for (int it = 0; it < 10000; ++it) {
        const double U = rng.u() - 0.5;
        const double V = rng.u();
        const double us = 0.5 - fabs(U);
        const double k = floor((2.0 * a / us + b) * U + mu + 0.43);
        if (us >= 0.07 && V <= vr) return (int64_t)k;
        if (k < 0.0 || (us < 0.013 && V > us)) continue;
        if (log(V) + log(inv_alpha) - log(a / (us * us) + b) <= -mu + k * logmu - lgamma(k + 1.0))
            return (int64_t)k;
    }
    return (int64_t)floor(mu + 0.5);  // unreachable in practice
}

__global__ void count_kernel(int64_t n, int64_t event_base, int mode, double yield, int64_t max_per_event, uint64_t seed,
                             const uint32_t *__restrict__ run_tag_ptr, int chunk, const double *__restrict__ ev_e,
                             const int32_t *__restrict__ given_n, const uint16_t *__restrict__ ev_geom,
                             const float4 *__restrict__ ev_pos, int32_t *__restrict__ ev_n,
                             uint32_t *__restrict__ ev_nchunks, unsigned long long *photons_per_geom,
                             unsigned long long *photons_total, int32_t *__restrict__ prim_geom, int32_t n_prim,
                             int *status)
{
    const uint32_t run_tag = *run_tag_ptr;
    const int lane = threadIdx.x & 31;
    // the warp's lanes take events base + lane together, so that with one
    // geometry the warp adds its photon total with one atomic per counter
    // (every event adding its own count to the same two addresses
    // serialised the kernel at millions of events)
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;  // a multiple of 32
    for (int64_t base = blockIdx.x * (int64_t)blockDim.x + (threadIdx.x & ~31); base < n; base += stride) {
        const int64_t i = base + lane;
        const bool live = i < n;
        int64_t k = 0;
        int g = 0;
        if (live) {
            if (mode == kCountGiven) {
                k = given_n[i];
            } else {
                CountRng rng{(uint32_t)seed, (uint32_t)(seed >> 32), (uint32_t)(event_base + i), run_tag, 0u,
                             make_uint4(0, 0, 0, 0), 0};
                const double mu = ev_e[i] * yield;
                if (mode == kCountGaussian) {
                    const double u1 = rng.u(), u2 = rng.u();
                    const double zn = sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
                    k = (int64_t)llrint(mu + sqrt(fmax(mu, 0.0)) * zn);
                } else {
                    k = poisson(rng, mu);
                }
            }
            if (k < 0) k = 0;
            if (k > max_per_event) {
                atomicOr(status, kStatusTooManyPhotons);
                k = 0;
            }
            // an event the preparation flagged (non-finite, negative energy,
            // history outside 1..num_hist) gets no photons: a streamed ingest
            // queues its transport before the host sees the flag
            const float4 p = ev_pos[i];
            const int32_t prim = __float_as_int(p.w);
            const double e = ev_e ? ev_e[i] : 0.0;  // no energies with given counts (fd2_transport_noalloc)
            if (!(isfinite(p.x) && isfinite(p.y) && isfinite(p.z) && isfinite(e)) || e < 0.0 || prim < 0 || prim >= n_prim)
                k = 0;
            ev_n[i] = (int32_t)k;
            ev_nchunks[i] = (uint32_t)((k + chunk - 1) / chunk);
            g = ev_geom ? ev_geom[i] : 0;
            if (ev_geom && k) {
                atomicAdd(&photons_per_geom[g], (unsigned long long)k);
                if (photons_total) atomicAdd(&photons_total[g], (unsigned long long)k);
            }
            if (prim_geom && prim >= 0 && prim < n_prim) prim_geom[prim] = g;
        }
        if (!ev_geom) {
            unsigned long long t = (unsigned long long)k;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(kFull, t, o);
            if (lane == 0 && t) {
                atomicAdd(&photons_per_geom[0], t);
                if (photons_total) atomicAdd(&photons_total[0], t);
            }
        }
    }
}

// ------------------------------------------------------------------ scan

constexpr int kScanBlock = 1024;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanBlock * kScanItems;

template <typename T>
__device__ unsigned long long block_exclusive_scan(unsigned long long v, unsigned long long *warp_sums,
                                                   unsigned long long *total)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    unsigned long long x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(kFull, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[wid] = x;
    __syncthreads();
    if (wid == 0) {
        unsigned long long s = lane < (int)(blockDim.x >> 5) ? warp_sums[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long y = __shfl_up_sync(kFull, s, o);
            if (lane >= o) s += y;
        }
        warp_sums[lane] = s;
    }
    __syncthreads();
    const unsigned long long before = wid ? warp_sums[wid - 1] : 0;
    *total = warp_sums[(blockDim.x >> 5) - 1];
    return before + x - v;
}

// Pass 1: per-tile exclusive scan into offsets, tile totals into block_sums.
template <typename In>
__global__ void scan_tiles(int64_t n, const In *__restrict__ in, unsigned long long *__restrict__ out,
                           unsigned long long *__restrict__ block_sums)
{
    __shared__ unsigned long long warp_sums[32];
    const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
    unsigned long long v[kScanItems], sum = 0;
#pragma unroll
    for (int j = 0; j < kScanItems; ++j) {
        v[j] = (base + j < n) ? (unsigned long long)in[base + j] : 0ull;
        sum += v[j];
    }
    unsigned long long total;
    unsigned long long run = block_exclusive_scan<unsigned long long>(sum, warp_sums, &total);
#pragma unroll
    for (int j = 0; j < kScanItems; ++j) {
        if (base + j < n) out[base + j] = run;
        run += v[j];
    }
    if (threadIdx.x == 0) block_sums[blockIdx.x] = total;
}

// Pass 2: exclusive scan of the tile totals (one CTA, looping).
__global__ void scan_sums(int64_t tiles, unsigned long long *block_sums, unsigned long long *total)
{
    __shared__ unsigned long long warp_sums[32];
    unsigned long long carry = 0;
    for (int64_t b = 0; b < tiles; b += blockDim.x) {
        const int64_t i = b + threadIdx.x;
        const unsigned long long v = i < tiles ? block_sums[i] : 0ull;
        unsigned long long t;
        const unsigned long long ex = block_exclusive_scan<unsigned long long>(v, warp_sums, &t);
        if (i < tiles) block_sums[i] = carry + ex;
        carry += t;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}

// Pass 3: add tile offsets.
__global__ void scan_add(int64_t n, unsigned long long *__restrict__ out, const unsigned long long *__restrict__ block_sums)
{
    const int64_t base = (int64_t)blockIdx.x * kScanTile;
    const unsigned long long add = block_sums[blockIdx.x];
    for (int j = threadIdx.x; j < kScanTile; j += blockDim.x)
        if (base + j < n) out[base + j] += add;
}

template <typename In>
cudaError_t scan_impl(cudaStream_t s, int64_t n, const In *in, unsigned long long *offsets,
                      unsigned long long *block_sums, unsigned long long *total)
{
    const int64_t tiles = (n + kScanTile - 1) / kScanTile;
    if (n > 0) {
        scan_tiles<In><<<(unsigned)tiles, kScanBlock, 0, s>>>(n, in, offsets, block_sums);
    }
    scan_sums<<<1, kScanBlock, 0, s>>>(tiles, block_sums, total);
    if (n > 0) scan_add<<<(unsigned)tiles, 256, 0, s>>>(n, offsets, block_sums);
    return cudaGetLastError();
}

__global__ void fill_chunks_kernel(int64_t n, int chunk, const int32_t *__restrict__ ev_n,
                                   const unsigned long long *__restrict__ offsets, uint2 *__restrict__ chunks,
                                   int64_t capacity, int *status)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t k = ev_n[i];
        const unsigned long long off = offsets[i];
        const int32_t nc = (k + chunk - 1) / chunk;
        if ((int64_t)(off + nc) > capacity) {
            atomicOr(status, kStatusChunkOverflow);
            continue;
        }
        for (int32_t c = 0; c < nc; ++c) chunks[off + c] = make_uint2((uint32_t)i, (uint32_t)(c * chunk));
    }
}

// ------------------------------------------------------------- transport

struct Slot {
    float4 pos;      // event x, y, z and history index bits
    uint32_t event;  // event index
    uint32_t first;  // first photon of the chunk
    uint32_t count;  // photons in the chunk
    uint32_t geom;
};
constexpr int kRing = 32;

// Shared-memory layout of the transport kernel (dynamic).
struct SmemLayout {
    size_t geom, ring, cnt, dist, win, total;
    __host__ __device__ SmemLayout(int block, int n_geom, int window)
    {
        size_t o = 0;
        geom = o;
        o += sizeof(DevGeom) * (size_t)n_geom;
        o = (o + 15) & ~(size_t)15;
        ring = o;
        o += sizeof(Slot) * (size_t)(block / 32) * kRing;
        cnt = o;
        o += sizeof(unsigned) * (size_t)n_geom * kCounterStride;
        dist = o;
        o += sizeof(float) * (size_t)n_geom;
        o = (o + 15) & ~(size_t)15;
        win = o;
        o += sizeof(unsigned) * (size_t)window * window;
        total = o;
    }
};

// Persistent transport.  Each warp keeps a ring of up to 32 chunk slots in
// shared memory, filled with one coalesced load per lane; each lane owns one
// photon at a time and takes a new one from the ring as soon as (or, with
// refill > 1, once enough lanes of the warp are) idle, so lanes never wait
// for the longest walk in the warp.  Tallies: by default every ended photon
// adds to the global fates, per-primary counts and PRF with one L2
// reduction of its lane; with kAgg (tally_mode 1) they are aggregated across
// the warp before touching memory and the PRF core of geometry 0 is tallied
// in a shared-memory window (identical tallies, slower on a B200).  kMulti: the
// geometry of each photon comes from the table in shared memory; otherwise
// the single geometry is read from the kernel parameters.  kRadial (label
// mode): a detected photon is binned by its distance from its event into
// the history's radial histogram instead of the PRF image.
template <bool kMulti, int kMaxThreads, int kMinBlocks, bool kRadial = false, bool kGrid = false, bool kAgg = false>
__global__ void __launch_bounds__(kMaxThreads, kMinBlocks) transport_kernel(const __grid_constant__ TransportArgs a)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int nwarps = blockDim.x >> 5;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int win = a.window;
    const SmemLayout L(blockDim.x, a.n_geom, win);
    DevGeom *s_geom = reinterpret_cast<DevGeom *>(smem + L.geom);
    Slot *s_ring = reinterpret_cast<Slot *>(smem + L.ring);
    unsigned int *s_cnt = reinterpret_cast<unsigned int *>(smem + L.cnt);
    float *s_dist = reinterpret_cast<float *>(smem + L.dist);
    unsigned int *s_win = reinterpret_cast<unsigned int *>(smem + L.win);
    (void)nwarps;

    if (kMulti)
        for (int i = threadIdx.x; i < a.n_geom; i += blockDim.x) s_geom[i] = a.geoms[i];
    for (int i = threadIdx.x; i < a.n_geom * kCounterStride; i += blockDim.x) s_cnt[i] = 0;
    for (int i = threadIdx.x; i < a.n_geom; i += blockDim.x) s_dist[i] = 0.0f;
    for (int i = threadIdx.x; i < win * win; i += blockDim.x) s_win[i] = 0;
    __syncthreads();

    Slot *ring = s_ring + wid * kRing;
    // never read past the chunk buffer, whatever the scan produced
    const unsigned long long total_chunks = min(*a.n_chunks, (unsigned long long)a.chunk_capacity);
    int ring_len = 0, slot = 0, refills = 0;
    uint32_t used = 0;
    bool exhausted = false, alive = false, parked = false;
    bool xretry = false;  // the lane's crosstalk normal is retried this round
    int xtries = 0;
    const unsigned refill_min = (unsigned)a.refill;
    const unsigned fresnel_min = (unsigned)max(a.fresnel_batch, 1);
    // Philox round keys and run counter, shared by the CTA
    __shared__ uint32_t s_rk[20];
    __shared__ uint32_t s_run;
    if (threadIdx.x < 20) s_rk[threadIdx.x] = a.round_keys[threadIdx.x];
    if (threadIdx.x == 0) s_run = *a.run_tag;

    __syncthreads();
    Walker w;
    const RngKey key{s_rk, s_run};
    int geom = 0;
    // the lane's current event record (x, y, z, history index bits): read at
    // a trapped restart, a detection and in label mode, so it need not stay
    // in registers through the walk; and the lane's path-length sum
    __shared__ float4 s_lane[kMaxThreads];
    __shared__ float s_ldist[kMaxThreads];
    s_ldist[threadIdx.x] = 0.0f;

    for (;;) {
        // ---- hand out photons to idle lanes
        unsigned needy = __ballot_sync(kFull, !alive);
        if (needy && !exhausted && ((unsigned)__popc(needy) >= refill_min || needy == kFull)) {
            while (needy) {
                if (slot >= ring_len) {
                    unsigned long long base = 0;
                    int stop = 0;
                    if (lane == 0) {
                        stop = (a.abort_flag && (refills & 15) == 0 && *a.abort_flag) ? 1 : 0;
                        if (!stop) base = atomicAdd(a.queue_head, (unsigned long long)kRing);
                    }
                    ++refills;
                    stop = __shfl_sync(kFull, stop, 0);
                    base = __shfl_sync(kFull, base, 0);
                    if (stop) {
                        if (lane == 0) atomicOr(a.status, kStatusAborted);
                        exhausted = true;
                        break;
                    }
                    const unsigned long long idx = base + lane;
                    const bool ok = idx < total_chunks;
                    __syncwarp();  // every lane is done reading the old ring
                    if (ok) {
                        const uint2 c = a.chunks[idx];
                        Slot s;
                        s.pos = a.ev_pos[c.x];
                        s.event = c.x;
                        s.first = c.y;
                        const int32_t n = a.ev_n[c.x];
                        s.count = (uint32_t)min(a.chunk, n - (int32_t)c.y);
                        s.geom = (kMulti && a.ev_geom) ? a.ev_geom[c.x] : 0;
                        ring[lane] = s;
                    }
                    ring_len = __popc(__ballot_sync(kFull, ok));
                    __syncwarp();
                    slot = 0;
                    used = 0;
                    if (ring_len == 0) {
                        exhausted = true;
                        break;
                    }
                }
                const uint32_t count = ring[slot].count;
                if (used >= count) {
                    ++slot;
                    used = 0;
                    continue;
                }
                const unsigned take = min((unsigned)(count - used), (unsigned)__popc(needy));
                const unsigned rank = __popc(needy & lanemask_lt());
                const bool mine = ((needy >> lane) & 1u) && rank < take;
                if (mine) {
                    const Slot &s = ring[slot];
                    const uint32_t k = s.first + used + rank;
                    s_lane[threadIdx.x] = s.pos;
                    geom = (int)s.geom;
                    w.start(s.pos.x, s.pos.y, s.pos.z, k, (uint32_t)(a.event_base + s.event), k == 0, key);
                    if constexpr (kGrid) w.grid_place(a.g0);
                    alive = true;
                }
                needy &= ~__ballot_sync(kFull, mine);
                used += take;
            }
        }
        if (__ballot_sync(kFull, alive) == 0) {
            if (exhausted) break;
            continue;
        }

        // ---- one transport step per live lane; a lane whose photon meets a
        // column wall without crosstalk parks it there, and the warp runs the
        // Fresnel part for the parked lanes together once `fresnel_batch` of
        // them wait (or nothing else runs)
        int fate = kAlive;
        if constexpr (kGrid) {
            // explicit column lattice: one segment per round per live lane;
            // a lane in the gap waits until `fresnel_batch` lanes of the warp
            // are in the gap (or no lane is in a column), so the gap's
            // cell-by-cell search runs with more lanes at once.  Waiting only
            // delays a photon's segments: its history is unchanged.
            const unsigned gap = __ballot_sync(kFull, alive && w.in_gap);
            const unsigned col = __ballot_sync(kFull, alive && !w.in_gap);
            const bool go = alive && (!w.in_gap || (unsigned)__popc(gap) >= fresnel_min || col == 0);
            if (go) fate = w.grid_segment(a.g0);
        } else {
            if (alive && !parked && !xretry) {
                fate = kMulti ? w.step(s_geom[geom], s_lane[threadIdx.x]) : w.step(a.g0, s_lane[threadIdx.x]);
                if (fate == kNeedsFresnel) {
                    parked = true;
                    fate = kAlive;
                }
            }
            if (alive && !parked) {
                // crosstalk: one attempt at the next column's normal per round, so
                // a rejected attempt is retried beside the other lanes' first ones
                if (xretry || fate == kNeedsNormal) {
                    fate = kMulti ? w.crosstalk_normal(s_geom[geom], xtries) : w.crosstalk_normal(a.g0, xtries);
                    xretry = fate == kRetryNormal;
                    if (xretry) fate = kAlive;
                    else xtries = 0;
                }
            }
            const unsigned waiting = __ballot_sync(kFull, parked);
            if (waiting) {
                const unsigned busy = __ballot_sync(kFull, alive && !parked && fate == kAlive);
                if ((unsigned)__popc(waiting) >= fresnel_min || busy == 0) {
                    if (parked) {
                        fate = kMulti ? w.surface_fresnel(s_geom[geom]) : w.surface_fresnel(a.g0);
                        parked = false;
                    }
                }
            }
        }

        // ---- tallies of the photons that ended: one global reduction per lane
        // (the default), or (kAgg) aggregated across the warp and privatised in
        // shared memory
        const unsigned ended = __ballot_sync(kFull, fate != kAlive);
        if (ended) {
            if (fate != kAlive) {
                const unsigned key = (unsigned)(geom * kCounterStride + fate);
                if (!kAgg) {
                    atomicAdd(&a.counters[key], 1ull);
                } else {
                    const unsigned peers = __match_any_sync(ended, key);
                    if (lane == __ffs(peers) - 1) atomicAdd(&s_cnt[key], (unsigned)__popc(peers));
                }
                if (kMulti) atomicAdd(&s_dist[geom], w.dist);
                else s_ldist[threadIdx.x] += w.dist;  // lane-private: no atomic
                alive = false;
            }
            const unsigned det = __ballot_sync(kFull, fate == kDetect);
            if (fate == kDetect) {
                const float4 ev = s_lane[threadIdx.x];
                const int prim = __float_as_int(ev.w);
                if (!kAgg) {
                    if ((unsigned)prim < (unsigned)a.n_prim) atomicAdd(&a.per_primary[prim], 1);
                } else {
                    const unsigned peers = __match_any_sync(det, prim);
                    if (lane == __ffs(peers) - 1 && (unsigned)prim < (unsigned)a.n_prim)
                        atomicAdd(&a.per_primary[prim], __popc(peers));
                }
                const int xdim = kMulti ? s_geom[geom].xdim : a.g0.xdim;
                const int ydim = kMulti ? s_geom[geom].ydim : a.g0.ydim;
                if (kRadial) {
                    const float rx = w.px - ev.x, ry = w.py - ev.y;
                    // quadratic edges: bin = floor(bins sqrt(r / r_max))
                    const float rr = sqrtf(rx * rx + ry * ry) * a.radial_inv_max;
                    const int b = rr < 1.0f ? min((int)(sqrtf(rr) * (float)a.radial_bins), a.radial_bins - 1)
                                            : a.radial_bins;
                    if ((unsigned)prim < (unsigned)a.n_prim && b >= 0)
                        atomicAdd(&a.radial[(long long)prim * (a.radial_bins + 1) + b], 1u);
                } else if (w.ii >= 0 && w.jj >= 0 && w.ii < xdim && w.jj < ydim) {
                    if (!kAgg) atomicAdd(&a.counters[geom * kCounterStride + kNumFates], 1ull);
                    else atomicAdd(&s_cnt[geom * kCounterStride + kNumFates], 1u);
                    const int wx = w.ii - a.win_x0, wy = w.jj - a.win_y0;
                    if (kAgg && geom == 0 && win > 0 && (unsigned)wx < (unsigned)win && (unsigned)wy < (unsigned)win) {
                        atomicAdd(&s_win[wx * win + wy], 1u);
                    } else {
                        const long long off = kMulti ? s_geom[geom].prf_offset : a.g0.prf_offset;
                        atomicAdd(&a.prf[off + (long long)w.ii * ydim + w.jj], 1ull);
                    }
                }
            }
        }
    }

    // ---- flush the CTA's private tallies
    __syncthreads();
    for (int i = threadIdx.x; i < a.n_geom * kCounterStride; i += blockDim.x)
        if (s_cnt[i]) atomicAdd(&a.counters[i], (unsigned long long)s_cnt[i]);
    if (!kMulti) {
        // the lanes' path-length sums: summed per warp in double, then added to the CTA's
        double d = (double)s_ldist[threadIdx.x];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) d += __shfl_xor_sync(kFull, d, o);
        if (lane == 0 && d != 0.0) atomicAdd(&a.distance[0], d);
    }
    for (int i = threadIdx.x; i < a.n_geom; i += blockDim.x)
        if (s_dist[i] != 0.0f) atomicAdd(&a.distance[i], (double)s_dist[i]);
    if (win > 0) {
        const long long off = kMulti ? s_geom[0].prf_offset : a.g0.prf_offset;
        const int ydim = kMulti ? s_geom[0].ydim : a.g0.ydim;
        for (int i = threadIdx.x; i < win * win; i += blockDim.x) {
            const unsigned v = s_win[i];
            if (v) {
                const int ii = a.win_x0 + i / win, jj = a.win_y0 + i % win;
                atomicAdd(&a.prf[off + (long long)ii * ydim + jj], (unsigned long long)v);
            }
        }
    }
}

// -------------------------------------------------------------------- PHS

// PHS binning of the reference (hybridMANTIS_cuda_ver1_0.cu:376-399) per
// geometry, plus FP64 moments over histories with >= 1 detected photon.
__global__ void phs_kernel(int32_t n_prim, const int32_t *__restrict__ per_primary,
                           const int32_t *__restrict__ prim_geom, int n_geom, int32_t min_photons,
                           int32_t max_photons, int32_t num_bins, int32_t width, int32_t shift,
                           int32_t *__restrict__ phs, double *__restrict__ moments,
                           unsigned long long *dropped)
{
    const int lane = threadIdx.x & 31;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t base = (int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < n_prim; base += stride) {
        const int64_t i = base + lane;
        const int32_t c = i < n_prim ? per_primary[i] : 0;
        const int g = (i < n_prim && prim_geom) ? prim_geom[i] : 0;
        const bool has = c > 0 && g >= 0 && g < n_geom;
        if (has) {
            int32_t bin;
            if (c <= min_photons) bin = 0;
            else if (c >= max_photons) bin = num_bins - 1;
            else bin = c / width - shift;
            if (bin >= 0 && bin < num_bins) atomicAdd(&phs[(int64_t)g * num_bins + bin], 1);
            else atomicAdd(&dropped[g], 1ull);
        }
        // FP64 moments, summed over the lanes of the warp with the same geometry
        const unsigned m = __ballot_sync(kFull, has);
        if (has) {
            const unsigned peers = __match_any_sync(m, g);
            const double v1 = (double)c, v2 = (double)c * (double)c;
            double a1 = 0.0, a2 = 0.0;
            for (unsigned q = peers; q; q &= q - 1) {
                const int src = __ffs(q) - 1;
                a1 += __shfl_sync(peers, v1, src);
                a2 += __shfl_sync(peers, v2, src);
            }
            if (lane == __ffs(peers) - 1) {
                atomicAdd(&moments[g * 3 + 0], (double)__popc(peers));
                atomicAdd(&moments[g * 3 + 1], a1);
                atomicAdd(&moments[g * 3 + 2], a2);
            }
        }
    }
}

__global__ void bump_kernel(uint32_t *run_tag) { *run_tag += 1u; }

// The walk's wall root (the far intersection with the column) for given
// quadratic coefficients, compiled with the transport's flags.
__global__ void wall_root_kernel(int n, const float *__restrict__ qa, const float *__restrict__ qb,
                                 const float *__restrict__ qc, float *__restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = wall_root(qa[i], qb[i], qc[i]);
}

}  // namespace

// ------------------------------------------------------------- launchers

cudaError_t launch_bump_run_tag(cudaStream_t s, uint32_t *run_tag)
{
    bump_kernel<<<1, 1, 0, s>>>(run_tag);
    return cudaGetLastError();
}

static unsigned grid_for(int64_t n, int block, int cap = 148 * 32)
{
    int64_t g = (n + block - 1) / block;
    if (g < 1) g = 1;
    if (g > cap) g = cap;
    return (unsigned)g;
}

cudaError_t launch_prep_cm(cudaStream_t s, int64_t n, const double *x_cm, const double *y_cm, const double *z_cm,
                           const double *de, const int32_t *hist, int32_t n_prim, float4 *ev_pos, double *ev_e,
                           double *ev_xyz, int *status)
{
    if (n <= 0) return cudaSuccess;
    prep_cm_kernel<<<grid_for(n, 256), 256, 0, s>>>(n, x_cm, y_cm, z_cm, de, hist, n_prim, ev_pos, ev_e, ev_xyz,
                                                    status);
    return cudaGetLastError();
}

cudaError_t launch_prep_um(cudaStream_t s, int64_t n, const float *x, const float *y, const float *z, const float *e,
                           const int32_t *hist, int32_t n_prim, float4 *ev_pos, double *ev_e, double *ev_xyz,
                           int *status)
{
    if (n <= 0) return cudaSuccess;
    prep_um_kernel<<<grid_for(n, 256), 256, 0, s>>>(n, x, y, z, e, hist, n_prim, ev_pos, ev_e, ev_xyz, status);
    return cudaGetLastError();
}

cudaError_t launch_count(cudaStream_t s, int64_t n, int64_t event_base, int mode, double yield, int64_t max_per_event, uint64_t seed,
                         const uint32_t *run_tag, int chunk, const double *ev_e, const int32_t *given_n,
                         const uint16_t *ev_geom, const float4 *ev_pos, int32_t *ev_n, uint32_t *ev_nchunks,
                         unsigned long long *photons_per_geom, unsigned long long *photons_total,
                         int32_t *prim_geom, int32_t n_prim, int *status)
{
    if (n <= 0) return cudaSuccess;
    count_kernel<<<grid_for(n, 128), 128, 0, s>>>(n, event_base, mode, yield, max_per_event, seed, run_tag, chunk, ev_e, given_n,
                                                  ev_geom, ev_pos, ev_n, ev_nchunks, photons_per_geom, photons_total,
                                                  prim_geom, n_prim, status);
    return cudaGetLastError();
}

size_t scan_block_sums_needed(int64_t n) { return (size_t)((n + kScanTile - 1) / kScanTile) + 1; }

cudaError_t launch_scan(cudaStream_t s, int64_t n, const uint32_t *in, unsigned long long *offsets,
                        unsigned long long *block_sums, unsigned long long *total)
{
    return scan_impl<uint32_t>(s, n, in, offsets, block_sums, total);
}

cudaError_t launch_photon_offsets(cudaStream_t s, int64_t n, const int32_t *ev_n, unsigned long long *first,
                                  unsigned long long *block_sums, unsigned long long *total)
{
    return scan_impl<int32_t>(s, n, ev_n, first, block_sums, total);
}

cudaError_t launch_fill_chunks(cudaStream_t s, int64_t n, int chunk, const int32_t *ev_n,
                               const unsigned long long *offsets, uint2 *chunks, int64_t capacity, int *status)
{
    if (n <= 0) return cudaSuccess;
    fill_chunks_kernel<<<grid_for(n, 256), 256, 0, s>>>(n, chunk, ev_n, offsets, chunks, capacity, status);
    return cudaGetLastError();
}

// Register budgets: blocks of up to 256 threads are compiled for 2, 3 or 4
// resident CTAs per SM (128, 85, 64 registers), blocks of 320 threads for
// two (102 registers: 20 warps per SM; the walk fits without spills, 352
// threads would spill), other larger blocks for one.
#define FD2_TRANSPORT_VARIANTS(X)                                                          \
    X(false, 512, 1, false, false, false) X(false, 256, 2, false, false, false)            \
    X(false, 320, 2, false, false, false) X(true, 320, 2, false, false, false)             \
    X(false, 256, 2, false, true, false) X(false, 320, 2, false, true, false)              \
    X(false, 256, 3, false, false, false) X(false, 256, 4, false, false, false)            \
    X(true, 512, 1, false, false, false) X(true, 256, 2, false, false, false)              \
    X(true, 256, 3, false, false, false) X(true, 256, 2, true, false, false)               \
    X(true, 256, 4, false, false, false) X(false, 256, 3, false, true, false)              \
    X(false, 512, 1, false, false, true) X(false, 256, 2, false, false, true)              \
    X(false, 320, 2, false, false, true) X(false, 256, 3, false, false, true)              \
    X(false, 256, 4, false, false, true) X(false, 256, 4, true, false, false)

cudaError_t prepare_transport(const TransportConfig &cfg, int n_geom)
{
    // The attribute is global to each kernel, shared by every context of the
    // process, so it is set to the device's opt-in maximum (a launch only
    // reserves what it asks for): contexts with different shared-memory
    // needs cannot undo each other's setting.
    int dev = 0, max_optin = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e != cudaSuccess) return e;
    const size_t need = transport_smem_bytes(cfg, n_geom);
    // dynamic limit = opt-in maximum - the kernel's static shared memory
#define FD2_SET_ATTR(M, T, B, R, L, A)                                                                       \
    if (e == cudaSuccess) {                                                                               \
        cudaFuncAttributes fa;                                                                            \
        e = cudaFuncGetAttributes(&fa, transport_kernel<M, T, B, R, L, A>);                                  \
        const int lim = max_optin - (int)fa.sharedSizeBytes;                                              \
        if (e == cudaSuccess && need > (size_t)lim) e = cudaErrorInvalidValue;                            \
        if (e == cudaSuccess)                                                                             \
            e = cudaFuncSetAttribute(transport_kernel<M, T, B, R, L, A>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim); \
    }
    FD2_TRANSPORT_VARIANTS(FD2_SET_ATTR)
#undef FD2_SET_ATTR
    return e;
}

size_t transport_smem_bytes(const TransportConfig &cfg, int n_geom)
{
    return SmemLayout(cfg.block, n_geom, cfg.window).total;
}

cudaError_t launch_transport(cudaStream_t s, const TransportConfig &cfg, int sm_count, const TransportArgs &a)
{
    const size_t smem = transport_smem_bytes(cfg, a.n_geom);
    const unsigned grid = (unsigned)(sm_count * cfg.ctas_per_sm);
    const bool multi = a.n_geom > 1;
    const int per_sm = cfg.block > 256 ? 1 : std::min(std::max(cfg.ctas_per_sm, 2), 4);
    if (a.g0.grid) {
        // explicit column lattice: single geometry, 256 or 320 threads
        if (multi || a.radial) return cudaErrorInvalidConfiguration;
        if (cfg.block == 320) transport_kernel<false, 320, 2, false, true><<<grid, cfg.block, smem, s>>>(a);
        else if (cfg.block <= 256 && per_sm >= 3) transport_kernel<false, 256, 3, false, true><<<grid, cfg.block, smem, s>>>(a);
        else if (cfg.block <= 256) transport_kernel<false, 256, 2, false, true><<<grid, cfg.block, smem, s>>>(a);
        else return cudaErrorInvalidConfiguration;
    } else if (a.radial) {
        // label mode, 256 threads: one geometry (the surrogate's audit) as the
        // production kernel, four CTAs per SM; several geometries (training
        // labels) two CTAs per SM
        if (cfg.block > 256) return cudaErrorInvalidConfiguration;
        if (!multi && cfg.ctas_per_sm >= 4)
            transport_kernel<false, 256, 4, true><<<(unsigned)(sm_count * 4), cfg.block, smem, s>>>(a);
        else
            transport_kernel<true, 256, 2, true><<<(unsigned)(sm_count * 2), cfg.block, smem, s>>>(a);
    } else if (!multi && cfg.aggregate) {
        // warp-aggregated, shared-memory privatised tallies (tally_mode 1)
        if (cfg.block == 320) transport_kernel<false, 320, 2, false, false, true><<<grid, cfg.block, smem, s>>>(a);
        else if (per_sm == 1) transport_kernel<false, 512, 1, false, false, true><<<grid, cfg.block, smem, s>>>(a);
        else if (per_sm == 2) transport_kernel<false, 256, 2, false, false, true><<<grid, cfg.block, smem, s>>>(a);
        else if (per_sm == 3) transport_kernel<false, 256, 3, false, false, true><<<grid, cfg.block, smem, s>>>(a);
        else transport_kernel<false, 256, 4, false, false, true><<<grid, cfg.block, smem, s>>>(a);
    } else if (!multi) {
        if (cfg.block == 320) transport_kernel<false, 320, 2><<<grid, cfg.block, smem, s>>>(a);
        else if (per_sm == 1) transport_kernel<false, 512, 1><<<grid, cfg.block, smem, s>>>(a);
        else if (per_sm == 2) transport_kernel<false, 256, 2><<<grid, cfg.block, smem, s>>>(a);
        else if (per_sm == 3) transport_kernel<false, 256, 3><<<grid, cfg.block, smem, s>>>(a);
        else transport_kernel<false, 256, 4><<<grid, cfg.block, smem, s>>>(a);
    } else {
        if (cfg.block == 320) transport_kernel<true, 320, 2><<<grid, cfg.block, smem, s>>>(a);
        else if (per_sm == 1) transport_kernel<true, 512, 1><<<grid, cfg.block, smem, s>>>(a);
        else if (per_sm == 2) transport_kernel<true, 256, 2><<<grid, cfg.block, smem, s>>>(a);
        else if (per_sm == 3) transport_kernel<true, 256, 3><<<grid, cfg.block, smem, s>>>(a);
        else transport_kernel<true, 256, 4><<<grid, cfg.block, smem, s>>>(a);
    }
    return cudaGetLastError();
}

cudaError_t launch_phs(cudaStream_t s, int32_t n_prim, const int32_t *per_primary, const int32_t *prim_geom,
                       int n_geom, int32_t min_photons, int32_t max_photons, int32_t num_bins, int32_t *phs,
                       double *moments, unsigned long long *dropped)
{
    if (n_prim <= 0) return cudaSuccess;
    const int32_t width = num_bins > 0 ? (max_photons - min_photons) / num_bins : 0;
    if (width <= 0) return cudaErrorInvalidValue;
    const int32_t shift = min_photons / width;
    phs_kernel<<<grid_for(n_prim, 256, 1024), 256, 0, s>>>(n_prim, per_primary, prim_geom, n_geom, min_photons,
                                                           max_photons, num_bins, width, shift, phs, moments,
                                                           dropped);
    return cudaGetLastError();
}

}  // namespace fd2

// Diagnostic entry point (tests): evaluates the transport's wall-root routine
// on the current device for n quadratics a t^2 + b t + c = 0 given in host
// arrays, so a test can drive its FP64 fallback for a nearly cancelling
// discriminant.  Synchronous.
extern "C" __attribute__((visibility("default"))) int fd2_debug_wall_root(int32_t n, const float *qa, const float *qb,
                                                                          const float *qc, float *out)
{
    if (n < 0 || (n > 0 && (!qa || !qb || !qc || !out))) return 1;
    if (n == 0) return 0;
    float *d = nullptr;
    const size_t b = sizeof(float) * (size_t)n;
    cudaError_t e = cudaMalloc(&d, 4 * b);
    if (e != cudaSuccess) return 5;
    if (e == cudaSuccess) e = cudaMemcpy(d, qa, b, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d + n, qb, b, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d + 2 * (size_t)n, qc, b, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        fd2::wall_root_kernel<<<(unsigned)((n + 255) / 256), 256>>>(n, d, d + n, d + 2 * (size_t)n, d + 3 * (size_t)n);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(out, d + 3 * (size_t)n, b, cudaMemcpyDeviceToHost);
    cudaFree(d);
    return e == cudaSuccess ? 0 : 4;
}

