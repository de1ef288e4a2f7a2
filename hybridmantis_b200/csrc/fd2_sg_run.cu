// fd2_sg_run.cu -- the surrogate in the event pipeline (fd2_sg_run).
//
// One run over a context's resident events:
//   1. photon counts per event (the context's count pass: Poisson, Gaussian
//      or given, exactly as fd2_run samples them);
//   2. routing: every event whose features lie in the training hull becomes
//      a surrogate row (its network input is written, its photon count is
//      taken out of the Monte Carlo queue); a hash of the event index picks
//      the audit fraction among them;
//   3. the Monte Carlo transports what is left (events outside the hull);
//   4. the network runs on all surrogate rows (GEMM grid sized for every
//      event, rows beyond the device-side row count skipped);
//   5. sampling, one warp per row: detected count ~ Binomial(N, p) split over
//      the 32 lanes (geometric skipping), then each detected photon's radius
//      drawn exactly from one ring of the mixture, an azimuth uniform over
//      the directions that stay on the detector (the labels' far light is
//      what the detector's edges leave), and the PRF pixel;
//      per-history counts and counters as the Monte Carlo tallies them;
//   6. PHS and the run counter (the context's last pipeline segment);
//   7. audit: the audited rows' depositions are transported by the Monte
//      Carlo in label mode, their detected photons per radial category are
//      summed on the GPU, and the totals are compared with the predictions.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "fd2.h"
#include "fd2_ctx.h"
#include "fd2_internal.h"
#include "fd2_sg_gemm.cuh"
#include "fd2_sg_internal.h"
#include "fd2_sg_mix.cuh"
#include "fd2_surrogate.h"

using namespace fd2::sg;

struct RunBuffers {
    int64_t cap = 0;
    int *d_count = nullptr;          // [0] surrogate rows, [1] audit rows, [2] Monte Carlo events,
                                     // [3] rows the sampler has handed out
    int32_t *sg_event = nullptr;     // event of each surrogate row
    int32_t *sg_n = nullptr;         // photons of each surrogate row
    int32_t *audit_row = nullptr;    // surrogate row of each audit entry
    __nv_bfloat16 *x0 = nullptr, *ha = nullptr, *hb = nullptr;
    float *out = nullptr;
    unsigned long long *d_stat = nullptr;  // [0] surrogate photons, [1] detected
    // audit: compact copies of the audited rows, pooled predictions
    float4 *a_pos = nullptr;
    int32_t *a_n = nullptr, *a_geom = nullptr, *a_ev = nullptr;
    double *a_pool = nullptr;  // [0, bins] sum N p q_j, then sum N p, sum N p (1 - p), sum N
    unsigned long long *a_hist = nullptr;  // the audit's detected photons per radial category
    int64_t a_cap = 0;
    // label-mode Monte Carlo context of the audit, kept across runs
    fd2_ctx *audit = nullptr;
    int32_t audit_cap = 0;
    std::vector<fd2_geometry> audit_geoms;
    fd2_params audit_params{};
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
};

void sg_free_run_buffers(fd2_sg *s)
{
    RunBuffers *r = s->run;
    if (!r) return;
    for (void *p : {(void *)r->d_count, (void *)r->sg_event, (void *)r->sg_n, (void *)r->audit_row, (void *)r->x0,
                    (void *)r->ha, (void *)r->hb, (void *)r->out, (void *)r->d_stat, (void *)r->a_pos,
                    (void *)r->a_n, (void *)r->a_geom, (void *)r->a_ev, (void *)r->a_pool, (void *)r->a_hist})
        if (p) cudaFree(p);
    fd2_destroy(r->audit);
    for (cudaEvent_t e : r->ev)
        if (e) cudaEventDestroy(e);
    delete r;
    s->run = nullptr;
}

namespace {

__device__ __forceinline__ uint4 philox10(uint4 c, uint32_t k0, uint32_t k1)
{
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t lo0 = 0xD2511F53u * c.x, hi0 = __umulhi(0xD2511F53u, c.x);
        const uint32_t lo1 = 0xCD9E8D57u * c.z, hi1 = __umulhi(0xCD9E8D57u, c.z);
        c = make_uint4(hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0);
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return c;
}

// uniform in (0, 1): (k + 0.5) 2^-24
__device__ __forceinline__ float unit(uint32_t r) { return ((float)(r >> 8) + 0.5f) * 5.9604644775390625e-8f; }

constexpr uint32_t kDomainAudit = 0x41554449u;   // audit selection

struct RouteArgs {
    int64_t n;
    const float4 *ev_pos;
    const double *ev_e;
    const uint16_t *ev_geom;
    const fd2::DevGeom *geoms;
    int32_t *ev_n;
    uint32_t *ev_nchunks;
    NormParams norm;
    fd2_sg_hull hull;
    float lateral;  // largest |x - centre|, |y - centre| a surrogate row may have
    float depth_margin;  // depths this far outside the hull's range take its edge
    float audit_frac;
    uint32_t k0, k1;
    int64_t event_base;
    int *count;
    int32_t *sg_event, *sg_n, *audit_row;
    __nv_bfloat16 *x0;
};

// ctr += 1 for each lane that reaches this point together with the calling
// one (one atomic per group of converged lanes); returns the lane's slot.
__device__ __forceinline__ int group_inc(int *ctr)
{
    const unsigned m = __activemask();
    const int lane = threadIdx.x & 31, leader = __ffs(m) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(ctr, __popc(m));
    base = __shfl_sync(m, base, leader);
    return base + __popc(m & ((1u << lane) - 1u));
}

__global__ void route_kernel(const RouteArgs a)
{
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < a.n; e += (int64_t)gridDim.x * blockDim.x) {
        const int32_t N = a.ev_n[e];
        if (N <= 0) continue;
        const fd2::DevGeom &g = a.geoms[a.ev_geom ? a.ev_geom[e] : 0];
        const float4 p = a.ev_pos[e];
        float f[kFeatures];
        f[0] = g.half - p.z;                 // depth below the entrance surface
        f[1] = (float)(a.ev_e[e] * 1e-3);    // keV
        f[2] = hypotf(p.x - 0.5f * g.xdet, p.y - 0.5f * g.ydet) * (1.0f / kLateralUnitUm);  // from the centre
        f[3] = g.H;
        f[4] = g.R;
        f[5] = g.beta;
        f[6] = 1.0f - g.top_absfrac;
        f[7] = g.mu > 0.0f ? log10f(g.mu) : -INFINITY;
        // a deposition just outside the labels' depth range (they leave out
        // the layer's first and last 0.1 %) takes the range's edge depth
        if (f[0] < a.hull.lo[0] && f[0] >= a.hull.lo[0] - a.depth_margin) f[0] = a.hull.lo[0];
        if (f[0] > a.hull.hi[0] && f[0] <= a.hull.hi[0] + a.depth_margin) f[0] = a.hull.hi[0];
        bool in = fabsf(p.x - 0.5f * g.xdet) <= a.lateral && fabsf(p.y - 0.5f * g.ydet) <= a.lateral;
#pragma unroll
        for (int i = 0; i < kFeatures; ++i) in = in && f[i] >= a.hull.lo[i] && f[i] <= a.hull.hi[i];
        if (!in) {
            group_inc(&a.count[2]);
            continue;
        }
        const int row = group_inc(&a.count[0]);
        a.sg_event[row] = (int32_t)e;
        a.sg_n[row] = N;
        __nv_bfloat16 *x = a.x0 + (int64_t)row * kInPad;
#pragma unroll
        for (int i = 0; i < kFeatures; ++i)
            x[i] = __float2bfloat16(2.0f * (f[i] - a.norm.lo[i]) * a.norm.inv[i] - 1.0f);
#pragma unroll
        for (int i = kFeatures; i < kInPad; ++i) x[i] = __float2bfloat16(0.0f);
        a.ev_n[e] = 0;          // out of the Monte Carlo queue
        a.ev_nchunks[e] = 0;
        const uint64_t ge = (uint64_t)(a.event_base + e);
        const uint4 h = philox10(make_uint4((uint32_t)ge, (uint32_t)(ge >> 32), kDomainAudit, 0), a.k0, a.k1);
        if (unit(h.x) < a.audit_frac) a.audit_row[group_inc(&a.count[1])] = row;
    }
}

struct SampleArgs {
    const int *count;
    int32_t *ev_n;
    const int32_t *sg_event, *sg_n;
    const float *out;
    const float4 *ev_pos;
    const uint16_t *ev_geom;
    const fd2::DevGeom *geoms;
    unsigned long long *prf;
    int32_t *per_primary;
    int32_t n_prim;
    unsigned long long *counters;
    unsigned long long *stat;
    int *next_row;  // rows handed out so far (zero before the launch)
    uint32_t k0, k1;
    int64_t event_base;
    const uint32_t *run_tag;
    float edge_amp, edge_inv_len;  // edge survival of the azimuths (amplitude 0: off)
};

constexpr int kSampleThreads = 256;  // one warp per event
constexpr int kRowBatch = 4;         // rows a warp takes from the counter at a time
constexpr uint32_t kDomainLane = 0x4c414e45u;   // a lane's stream for one event

// A lane's random stream for one event (its detected count and its photons'
// places): xoshiro128+ (Blackman & Vigna, ACM TOMS 47(4), 2021) seeded by one
// Philox-4x32-10 block at (lane, event, domain, run), the construction of the
// transport's per-photon streams; floats from the top 24 bits (unit()).  A
// lane takes photons lane, lane + 32, ... of its event in order, so every
// draw is fixed by the event, the lane and the run.
struct LaneRng {
    uint32_t s0, s1, s2, s3;
    __device__ __forceinline__ LaneRng(uint4 k)
        : s0(k.x), s1(k.y), s2(k.z), s3(k.w | ((k.x | k.y | k.z | k.w) == 0u ? 1u : 0u))
    {
    }
    __device__ __forceinline__ float u()
    {
        const uint32_t r = s0 + s3;
        const uint32_t t = s1 << 9;
        s2 ^= s0;
        s3 ^= s1;
        s1 ^= s2;
        s0 ^= s3;
        s2 ^= t;
        s3 = __funnelshift_l(s3, s3, 11);
        return unit(r);
    }
};

// Radius from one ring component, density proportional to r N(r; mu, sd) on
// r >= 0, exactly.  In t = (r - mu) / sd the weight (mu + sd t) phi(t) splits
// into t >= 0: mu phi(t) (mass mu / 2, a half-normal) and sd t phi(t) (mass
// sd phi(0), a Rayleigh), and t0 <= t < 0, t0 = -mu / sd: a normal on
// [t0, 0) thinned with acceptance 1 + sd t / mu (mass S - mu / 2 - sd phi(0)).
// u picks the region.  All three come from one Box-Muller pair: rho =
// sqrt(-2 ln u1) is the Rayleigh, rho |cos(2 pi u2)| the half-normal, and its
// negative, kept when it is >= t0 and passes the thinning, the third region
// (retried with fresh draws otherwise), so the regions share their costly part.
__device__ __forceinline__ float ring_radius(float mu, float sd, float S, float u, LaneRng &rng)
{
    const float m1 = 0.5f * mu, m2 = sd * 0.3989422804014327f;
    const float x = u * S;
    const bool rayleigh = x >= m1 && (x < m1 + m2 || mu <= 0.0f);
    const bool upper = x < m1;
    const float t0 = -mu / sd;
    for (uint32_t k = 0; k < 64; ++k) {
        const float rho = sqrtf(-2.0f * logf(rng.u()));
        if (rayleigh) return mu + sd * rho;
        const float z = rho * fabsf(__cosf(6.283185307179586f * rng.u()));
        if (upper) return mu + sd * z;
        if (-z >= t0 && rng.u() <= 1.0f - sd * z / mu) return fmaxf(mu - sd * z, 0.0f);
    }
    return 0.5f * mu;  // not reached in practice
}

// Detected photons of one row and their PRF pixels; one warp per row, the
// warps taking rows from a counter in batches, so that rows of very
// different photon counts do not leave warps idle at the end.
__global__ void __launch_bounds__(kSampleThreads) sample_kernel(const SampleArgs a)
{
    const int lane = threadIdx.x & 31;
    __shared__ float s_mix[kSampleThreads / 32][4][kComponents];
    float(*mix)[kComponents] = s_mix[threadIdx.x >> 5];
    const int rows = *a.count;
    const uint32_t run = *a.run_tag;
    // the warp's totals over its rows (photons, detected; detected and in
    // the PRF for the current geometry), kept by lane 0 in shared memory and
    // added once per geometry run of rows and at the end: per-row atomics
    // on the same four counters serialised in the L2 at millions of rows
    __shared__ unsigned long long s_tot[kSampleThreads / 32][4];
    __shared__ int s_tgeom[kSampleThreads / 32];
    unsigned long long *tot = s_tot[threadIdx.x >> 5];
    if (lane == 0) {
        tot[0] = tot[1] = tot[2] = tot[3] = 0ull;
        s_tgeom[threadIdx.x >> 5] = -1;
    }
    int r = 0, r_end = 0;  // the warp's current batch of rows
    for (;;) {
        if (r == r_end) {
            int r0 = 0;
            if (lane == 0) r0 = atomicAdd(a.next_row, kRowBatch);
            r0 = __shfl_sync(0xffffffffu, r0, 0);
            if (r0 >= rows) break;
            r = r0;
            r_end = min(r0 + kRowBatch, rows);
        }
        const int64_t e = a.sg_event[r];
        const int32_t N = a.sg_n[r];
        const float *o = a.out + (int64_t)r * kOutPad;
        const uint16_t gi = a.ev_geom ? a.ev_geom[e] : 0;
        const fd2::DevGeom &g = a.geoms[gi];
        const float4 pos = a.ev_pos[e];
        const uint64_t ge = (uint64_t)(a.event_base + e);
        LaneRng rng(philox10(make_uint4((uint32_t)lane, (uint32_t)ge, (uint32_t)(ge >> 32) ^ kDomainLane, run), a.k0,
                             a.k1));
        // ---- detected count: lane l takes photons [lo, hi) of the N
        const float z = o[0];
        const float p = 1.0f / (1.0f + expf(-z));
        const int32_t lo = (int32_t)(((int64_t)N * lane) >> 5), hi = (int32_t)(((int64_t)N * (lane + 1)) >> 5);
        const int32_t span = hi - lo;
        int32_t k = 0;
        if (span > 0 && p > 0.0f) {
            if (p >= 1.0f) {
                k = span;
            } else {
                // count the rarer outcome by geometric skips: expected span min(p, 1 - p) + 1 draws
                const bool flip = p > 0.5f;
                const float q = flip ? 1.0f - p : p;
                const float inv_log = 1.0f / log1pf(-q);
                int32_t hits = 0, at = -1;
                for (;;) {
                    const float skip = floorf(logf(rng.u()) * inv_log);
                    const float next = (float)at + skip + 1.0f;
                    if (next >= (float)span) break;
                    at = (int32_t)next;
                    ++hits;
                }
                k = flip ? span - hits : hits;
            }
        }
        // warp total and this lane's first detected index
        int32_t before = k;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int32_t v = __shfl_up_sync(0xffffffffu, before, d);
            if (lane >= d) before += v;
        }
        const int32_t total = __shfl_sync(0xffffffffu, before, 31);
        // ---- positions of the detected photons: a ring component by weight,
        // its radius drawn exactly (ring_radius), an azimuth over the
        // directions that keep the photon on the detector, uniform or (with an
        // edge amplitude a > 0) accepted with probability
        //   W = prod over the four sides (1 - a exp(-s / len)),
        // s the point's distance to the side: the detected light thins out
        // towards the detector's sides, whose crossing loses a photon.  Only
        // the azimuth is redrawn, so the radius keeps the network's law.
        // the event's mixture in the warp's shared-memory table (every lane
        // draws from the same one; an indexed table in registers would go to
        // local memory): cumulative weight, mu, sd and normaliser per ring
        {
            Mix m;
            decode_mix(o, m);
            float acc = 0.0f;
            __syncwarp();  // the previous event's photons are placed
#pragma unroll
            for (int c = 0; c < kComponents; ++c) {
                acc += m.w[c];
                if (lane == c) {
                    mix[0][c] = c == kComponents - 1 ? 2.0f : acc;
                    mix[1][c] = m.mu[c];
                    mix[2][c] = m.sd[c];
                    mix[3][c] = m.S[c];
                }
            }
            __syncwarp();
        }
        int32_t in_prf = 0;
        // a power-of-two pixel divides exactly as a multiplication by its
        // reciprocal (the same correctly rounded quotient)
        const bool pow2 = (__float_as_uint(g.pixel) & 0x7fffffu) == 0u && g.pixel > 0.0f;
        const float inv_pixel = 1.0f / g.pixel;
        for (int32_t i = lane; i < total; i += 32) {
            // the component: the first whose cumulative weight exceeds u,
            // i.e. the number of cumulative weights <= u (they do not
            // decrease), counted without a data-dependent loop
            const float u = rng.u();
            int c = 0;
#pragma unroll
            for (int j = 0; j < kComponents - 1; ++j) c += u >= mix[0][j] ? 1 : 0;
            const float ur = rng.u();
            const float rad = ring_radius(mix[1][c], mix[2][c], mix[3][c], ur, rng);
            float sn, cs;
            sincospif(2.0f * rng.u(), &sn, &cs);
            for (uint32_t k = 0; k < 32; ++k) {
                const float tx = pos.x + rad * cs, ty = pos.y + rad * sn;
                bool ok = tx >= 0.0f && tx <= g.xdet && ty >= 0.0f && ty <= g.ydet;
                if (ok && a.edge_amp > 0.0f) {
                    const float W = (1.0f - a.edge_amp * __expf(-tx * a.edge_inv_len)) *
                                    (1.0f - a.edge_amp * __expf(-(g.xdet - tx) * a.edge_inv_len)) *
                                    (1.0f - a.edge_amp * __expf(-ty * a.edge_inv_len)) *
                                    (1.0f - a.edge_amp * __expf(-(g.ydet - ty) * a.edge_inv_len));
                    ok = rng.u() < W;
                }
                if (ok) break;
                sincospif(2.0f * rng.u(), &sn, &cs);
            }
            const float x = pos.x + rad * cs, y = pos.y + rad * sn;
            if (x <= g.ub_x && y <= g.ub_y && x >= g.lb_x && y >= g.lb_y) {
                const float qx = pow2 ? __fmul_rn(x - g.lb_x, inv_pixel) : __fdiv_rn(x - g.lb_x, g.pixel);
                const float qy = pow2 ? __fmul_rn(y - g.lb_y, inv_pixel) : __fdiv_rn(y - g.lb_y, g.pixel);
                const int ii = (int)floorf(qx);
                const int jj = (int)floorf(qy);
                if (ii >= 0 && jj >= 0 && ii < g.xdim && jj < g.ydim) {
                    atomicAdd(&a.prf[g.prf_offset + (long long)ii * g.ydim + jj], 1ull);
                    ++in_prf;
                }
            }
        }
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) in_prf += __shfl_down_sync(0xffffffffu, in_prf, d);
        if (lane == 0) {
            a.ev_n[e] = N;  // the run's photon count, as fd2_get_photon_counts reports it
            const int prim = __float_as_int(pos.w);
            if (total > 0 && prim >= 0 && prim < a.n_prim) atomicAdd(&a.per_primary[prim], total);
            int &tg = s_tgeom[threadIdx.x >> 5];
            if ((int)gi != tg) {
                if (tg >= 0) {
                    unsigned long long *cn = a.counters + (long long)tg * fd2::kCounterStride;
                    if (tot[2]) atomicAdd(&cn[fd2::kDetect], tot[2]);
                    if (tot[3]) atomicAdd(&cn[fd2::kNumFates], tot[3]);
                }
                tg = gi;
                tot[2] = tot[3] = 0ull;
            }
            tot[0] += (unsigned long long)N;
            tot[1] += (unsigned long long)total;
            tot[2] += (unsigned long long)total;
            tot[3] += (unsigned long long)in_prf;
        }
        ++r;
    }
    if (lane == 0 && s_tgeom[threadIdx.x >> 5] >= 0) {
        unsigned long long *cn = a.counters + (long long)s_tgeom[threadIdx.x >> 5] * fd2::kCounterStride;
        if (tot[2]) atomicAdd(&cn[fd2::kDetect], tot[2]);
        if (tot[3]) atomicAdd(&cn[fd2::kNumFates], tot[3]);
        atomicAdd(&a.stat[0], tot[0]);
        atomicAdd(&a.stat[1], tot[1]);
    }
}

// Compact copies of the audited rows (position, photons, geometry, event) and
// their pooled predictions: sum N p q_j over the radial categories j, sum N p,
// sum N p (1 - p) and sum N (one thread per row; each warp sums its rows'
// terms with shuffles and adds them with one FP64 atomic per term, so the
// pool's few addresses see one atomic per 32 rows).
__device__ __forceinline__ void warp_pool_add(double *dst, double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    if ((threadIdx.x & 31) == 0 && v != 0.0) atomicAdd(dst, v);
}

__global__ void audit_gather_kernel(const int *count, const int32_t *audit_row, const int32_t *sg_event,
                                    const int32_t *sg_n, const float *out, const float4 *ev_pos,
                                    const uint16_t *ev_geom, int bins, float r_max, float4 *a_pos, int32_t *a_n,
                                    int32_t *a_geom, int32_t *a_ev, double *pool)
{
    const int n = count[1];
    const int lane = threadIdx.x & 31;
    const long long warp0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    // the warp's lanes take rows base + lane together (the shuffles need all 32)
    for (long long base = warp0 * 32; base < n; base += nwarps * 32) {
        const long long i = base + lane;
        const bool live = i < n;
        double np = 0.0, q = 0.0, nn = 0.0;
        Mix m;
        if (live) {
            const int r = audit_row[i];
            const int32_t e = sg_event[r];
            const int32_t N = sg_n[r];
            a_pos[i] = ev_pos[e];
            a_n[i] = N;
            a_geom[i] = ev_geom ? ev_geom[e] : 0;
            a_ev[i] = e;
            const float *o = out + (int64_t)r * kOutPad;
            const float p = 1.0f / (1.0f + expf(-o[0]));
            decode_mix(o, m);
            np = (double)N * p;
            q = np * (1.0 - (double)p);
            nn = (double)N;
        }
        for (int j = 0; j <= bins; ++j)
            warp_pool_add(&pool[j], live ? np * (double)bin_prob(m, j, bins, r_max) : 0.0);
        warp_pool_add(&pool[bins + 1], np);
        warp_pool_add(&pool[bins + 2], q);
        warp_pool_add(&pool[bins + 3], nn);
    }
}

// Per-category totals of the audit's label-mode tally (rows [0, na) of a
// [row][nb] array of counts): partial sums per category in shared memory,
// then one 64-bit atomic per category and block.  Integer sums, so the
// totals do not depend on the order.
__global__ void radial_pool_kernel(const uint32_t *rad, int na, int nb, unsigned long long *sum)
{
    extern __shared__ unsigned long long s_sum[];
    for (int j = threadIdx.x; j < nb; j += blockDim.x) s_sum[j] = 0ull;
    __syncthreads();
    const long long total = (long long)na * nb;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const uint32_t v = rad[i];
        if (v) atomicAdd(&s_sum[(int)(i % nb)], (unsigned long long)v);
    }
    __syncthreads();
    for (int j = threadIdx.x; j < nb; j += blockDim.x)
        if (s_sum[j]) atomicAdd(&sum[j], s_sum[j]);
}

template <class T>
cudaError_t alloc(T **p, size_t n)
{
    if (*p) cudaFree(*p);
    *p = nullptr;
    return cudaMalloc((void **)p, sizeof(T) * std::max<size_t>(n, 1));
}

fd2_status ensure_run_buffers(fd2_sg *s, int64_t n)
{
    if (!s->run) {
        s->run = new RunBuffers();
        for (auto &e : s->run->ev)
            if (cudaEventCreate(&e) != cudaSuccess) return sg_fail(s, FD2_ERR_CUDA, "event create");
        if (alloc(&s->run->d_count, 4) != cudaSuccess || alloc(&s->run->d_stat, 2) != cudaSuccess)
            return sg_fail(s, FD2_ERR_OUT_OF_MEMORY, "run buffers");
    }
    RunBuffers *r = s->run;
    if (n <= r->cap) return FD2_OK;
    const size_t N = (size_t)n, H = (size_t)s->hidden;
    if (alloc(&r->sg_event, N) || alloc(&r->sg_n, N) || alloc(&r->audit_row, N) || alloc(&r->x0, N * kInPad) ||
        alloc(&r->ha, N * H) || alloc(&r->hb, N * H) || alloc(&r->out, N * kOutPad))
        return sg_fail(s, FD2_ERR_OUT_OF_MEMORY, "run buffers for " + std::to_string(n) + " events");
    r->cap = n;
    return FD2_OK;
}

}  // namespace

extern "C" fd2_status fd2_sg_run(fd2_sg *s, fd2_ctx *c, double audit_fraction, fd2_sg_stats *stats)
{
    if (!s || !c || !(audit_fraction >= 0.0 && audit_fraction <= 1.0)) return FD2_ERR_INVALID_ARGUMENT;
    if (c->device != s->device) return sg_fail(s, FD2_ERR_INVALID_ARGUMENT, "surrogate and context on different GPUs");
    if (c->d_radial) return sg_fail(s, FD2_ERR_STATE, "the context is in label mode");
    fd2_status st = fd2_wait(c);
    if (st != FD2_OK) return sg_fail(s, st, std::string("context: ") + fd2_last_error(c));
    if (c->n_events <= 0) return sg_fail(s, FD2_ERR_STATE, "no events submitted");
    if (cudaSetDevice(c->device) != cudaSuccess) return sg_fail(s, FD2_ERR_CUDA, "set device");
    if ((st = fd2::api::ensure_chunks(c)) != FD2_OK) return sg_fail(s, st, "context chunks");
    const int64_t n = c->n_events;
    // the tensor-core forward is persistent; the mma.sync one (FD2_SG_GEMM=mma) has one grid row of CTAs
    // per 64 events
    if (!s->use_tc && n > (int64_t)65535 * kBM)
        return sg_fail(s, FD2_ERR_INVALID_ARGUMENT, "more than 4,194,240 events per run on the mma.sync forward");
    if (n >= ((int64_t)1 << 31)) return sg_fail(s, FD2_ERR_INVALID_ARGUMENT, "2^31 events or more per run");
    if ((st = ensure_run_buffers(s, n)) != FD2_OK) return st;
    RunBuffers *R = s->run;
    cudaStream_t q = c->stream;
    const auto t_start = std::chrono::steady_clock::now();
    const uint32_t k0 = (uint32_t)c->opt.seed ^ 0x53475255u, k1 = (uint32_t)(c->opt.seed >> 32) ^ 0x4e5f4b31u;
    cudaError_t e = cudaEventRecord(R->ev[0], q);
    if (e == cudaSuccess) e = cudaMemsetAsync(R->d_count, 0, 4 * sizeof(int), q);
    if (e == cudaSuccess) e = cudaMemsetAsync(R->d_stat, 0, 2 * sizeof(unsigned long long), q);
    // 1-2: counts, routing
    if (e == cudaSuccess) e = fd2::api::count_pass(c, true);
    if (e == cudaSuccess) {
        RouteArgs a;
        a.n = n;
        a.ev_pos = c->d_ev_pos;
        a.ev_e = c->d_ev_e;
        a.ev_geom = c->has_geom ? c->d_ev_geom : nullptr;
        a.geoms = c->d_geoms;
        a.ev_n = c->d_ev_n;
        a.ev_nchunks = c->d_ev_nchunks;
        a.norm = s->norm;
        // the hull, widened by a few float ulps: geometry features computed
        // on the device (log10f, 1 - top_absfrac) may differ from the host's
        // by rounding
        a.hull = s->hull;
        for (int i = 0; i < kFeatures; ++i) {
            const float tol = 1e-5f * std::max(1.0f, std::max(std::fabs(a.hull.lo[i]), std::fabs(a.hull.hi[i])));
            a.hull.lo[i] -= tol;
            a.hull.hi[i] += tol;
        }
        a.lateral = s->lateral_um;
        a.depth_margin = s->depth_margin_um;
        a.audit_frac = (float)audit_fraction;
        a.k0 = k0;
        a.k1 = k1;
        a.event_base = c->opt.event_base;
        a.count = R->d_count;
        a.sg_event = R->sg_event;
        a.sg_n = R->sg_n;
        a.audit_row = R->audit_row;
        a.x0 = R->x0;
        route_kernel<<<(unsigned)std::min<int64_t>((n + 255) / 256, 8192), 256, 0, q>>>(a);
        e = cudaGetLastError();
    }
    // 3: Monte Carlo for the rest
    if (e == cudaSuccess)
        e = fd2::launch_scan(q, n, c->d_ev_nchunks, c->d_chunk_off, c->d_block_sums, c->d_scalars + 0);
    if (e == cudaSuccess)
        e = fd2::launch_fill_chunks(q, n, c->cfg.chunk, c->d_ev_n, c->d_chunk_off, c->d_chunks, c->chunk_cap,
                                    c->d_flags);
    if (e == cudaSuccess) e = cudaEventRecord(R->ev[1], q);
    if (e == cudaSuccess) e = fd2::launch_transport(q, c->cfg, c->sm_count, fd2::api::transport_args(c));
    if (e == cudaSuccess) e = cudaEventRecord(R->ev[2], q);
    // 4-5: network and sampling
    if (e == cudaSuccess) e = sg_forward(s, q, R->x0, (int)n, R->d_count, R->ha, R->hb, R->ha, R->out);
    if (e == cudaSuccess) {
        SampleArgs a;
        a.count = R->d_count;
        a.ev_n = c->d_ev_n;
        a.sg_event = R->sg_event;
        a.sg_n = R->sg_n;
        a.out = R->out;
        a.ev_pos = c->d_ev_pos;
        a.ev_geom = c->has_geom ? c->d_ev_geom : nullptr;
        a.geoms = c->d_geoms;
        a.prf = c->d_prf;
        a.per_primary = c->d_per_primary;
        a.n_prim = c->n_prim;
        a.counters = c->d_counters;
        a.stat = R->d_stat;
        a.next_row = R->d_count + 3;
        a.k0 = k0;
        a.k1 = k1;
        a.event_base = c->opt.event_base;
        a.run_tag = reinterpret_cast<const uint32_t *>(c->d_flags + 1);
        a.edge_amp = s->edge_amp;
        a.edge_inv_len = 1.0f / s->edge_len_um;
        sample_kernel<<<(unsigned)(c->sm_count * 8), kSampleThreads, 0, q>>>(a);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaEventRecord(R->ev[3], q);
    // 6: PHS and the run counter
    if (e == cudaSuccess) e = fd2::api::enqueue_segment(c, 2);
    int counts[3] = {0, 0, 0};
    unsigned long long stat[2] = {0, 0};
    if (e == cudaSuccess) e = cudaMemcpyAsync(counts, R->d_count, sizeof counts, cudaMemcpyDeviceToHost, q);
    if (e == cudaSuccess) e = cudaMemcpyAsync(stat, R->d_stat, sizeof stat, cudaMemcpyDeviceToHost, q);
    if (e == cudaSuccess) e = cudaStreamSynchronize(q);
    if (e != cudaSuccess) return sg_cuda(s, e, "surrogate run");
    if ((st = sg_tc_check(s)) != FD2_OK) return st;
    c->counts_ready = true;
    c->ran_once = true;
    c->graph_valid = false;  // the counts were rewritten outside the graph
    if ((st = fd2::api::check_status(c)) != FD2_OK) return sg_fail(s, st, std::string("context: ") + fd2_last_error(c));
    float mc_ms = 0, sg_ms = 0;
    cudaEventElapsedTime(&mc_ms, R->ev[1], R->ev[2]);
    cudaEventElapsedTime(&sg_ms, R->ev[2], R->ev[3]);
    const double run_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();

    // 7: audit
    fd2_sg_stats out;
    std::memset(&out, 0, sizeof out);
    out.events = n;
    out.surrogate_events = counts[0];
    out.audit_events = counts[1];
    out.surrogate_photons = (int64_t)stat[0];
    out.surrogate_detected = (int64_t)stat[1];
    out.sg_ms = sg_ms;
    out.mc_ms = mc_ms;
    const auto t_audit = std::chrono::steady_clock::now();
    const int na = counts[1];
    if (na > 0) {
        RunBuffers *B = R;
        const int nb = s->bins + 1;
        if (na > B->a_cap) {
            if (alloc(&B->a_pos, (size_t)na) || alloc(&B->a_n, (size_t)na) || alloc(&B->a_geom, (size_t)na) ||
                alloc(&B->a_ev, (size_t)na))
                return sg_fail(s, FD2_ERR_OUT_OF_MEMORY, "audit buffers");
            B->a_cap = na;
        }
        if ((!B->a_pool && alloc(&B->a_pool, (size_t)nb + 3)) || (!B->a_hist && alloc(&B->a_hist, (size_t)nb)))
            return sg_fail(s, FD2_ERR_OUT_OF_MEMORY, "audit buffers");
        e = cudaMemsetAsync(B->a_pool, 0, sizeof(double) * (nb + 3), q);
        if (e == cudaSuccess) {
            audit_gather_kernel<<<(unsigned)std::min((na + 127) / 128, 4096), 128, 0, q>>>(
                R->d_count, R->audit_row, R->sg_event, R->sg_n, R->out, c->d_ev_pos,
                c->has_geom ? c->d_ev_geom : nullptr, s->bins, (float)s->radial_max, B->a_pos, B->a_n, B->a_geom,
                B->a_ev, B->a_pool);
            e = cudaGetLastError();
        }
        std::vector<float4> pos((size_t)na);
        std::vector<int32_t> nph((size_t)na), geo((size_t)na), evi((size_t)na);
        std::vector<double> pool((size_t)nb + 3);
        if (e == cudaSuccess) e = cudaMemcpyAsync(pos.data(), B->a_pos, sizeof(float4) * na, cudaMemcpyDeviceToHost, q);
        if (e == cudaSuccess) e = cudaMemcpyAsync(nph.data(), B->a_n, sizeof(int32_t) * na, cudaMemcpyDeviceToHost, q);
        if (e == cudaSuccess) e = cudaMemcpyAsync(geo.data(), B->a_geom, sizeof(int32_t) * na, cudaMemcpyDeviceToHost, q);
        if (e == cudaSuccess) e = cudaMemcpyAsync(evi.data(), B->a_ev, sizeof(int32_t) * na, cudaMemcpyDeviceToHost, q);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(pool.data(), B->a_pool, sizeof(double) * (nb + 3), cudaMemcpyDeviceToHost, q);
        if (e == cudaSuccess) e = cudaStreamSynchronize(q);
        if (e != cudaSuccess) return sg_cuda(s, e, "audit gather");
        // the audited depositions through the Monte Carlo in label mode, in a
        // context kept across runs (re-made when the geometries change or the
        // audit outgrows it)
        const bool same = B->audit && B->audit_geoms.size() == c->geoms.size() &&
                          std::memcmp(B->audit_geoms.data(), c->geoms.data(),
                                      sizeof(fd2_geometry) * c->geoms.size()) == 0 &&
                          std::memcmp(&B->audit_params, &c->params, sizeof(fd2_params)) == 0;
        st = FD2_OK;
        if (!same || na > B->audit_cap) {
            fd2_destroy(B->audit);
            B->audit = nullptr;
            fd2_params ap = c->params;
            ap.num_hist = std::max(na, B->audit_cap * 2);
            fd2_options ao = c->opt;
            ao.count_mode = FD2_COUNT_GIVEN;
            ao.seed = c->opt.seed ^ 0xA0D17A0D17ull;
            ao.radial_bins = s->bins;
            ao.radial_max_um = s->radial_max;
            ao.event_base = 0;
            ao.tune_cache = nullptr;
            ao.wait_timeout_s = 0.0;
            st = fd2_create(&ap, &ao, &B->audit);
            if (st == FD2_OK && c->geoms.size() > 1)
                st = fd2_set_geometries(B->audit, c->geoms.data(), (int32_t)c->geoms.size());
            if (st != FD2_OK) {
                fd2_destroy(B->audit);
                B->audit = nullptr;
                return sg_fail(s, st, "audit context");
            }
            B->audit_cap = ap.num_hist;
            B->audit_geoms = c->geoms;
            B->audit_params = c->params;
        }
        fd2_ctx *ac = B->audit;
        // in event order: the routing kernel lists the audited rows in the
        // order its threads reach them, and an audited event's Monte Carlo
        // streams follow its place in the audit, so the order is fixed here
        std::vector<uint64_t> order((size_t)na);
        for (int i = 0; i < na; ++i) order[(size_t)i] = ((uint64_t)(uint32_t)evi[(size_t)i] << 32) | (uint32_t)i;
        std::sort(order.begin(), order.end());
        std::vector<float> xs((size_t)na), ys((size_t)na), zs((size_t)na);
        std::vector<int32_t> hist((size_t)na), nps((size_t)na);
        std::vector<uint16_t> gg((size_t)na);
        for (int k = 0; k < na; ++k) {
            const size_t i = (size_t)(order[(size_t)k] & 0xffffffffu);
            xs[(size_t)k] = pos[i].x;
            ys[(size_t)k] = pos[i].y;
            zs[(size_t)k] = pos[i].z;
            hist[(size_t)k] = k + 1;
            nps[(size_t)k] = nph[i];
            gg[(size_t)k] = (uint16_t)geo[i];
        }
        st = fd2_reset_tallies(ac);
        if (st == FD2_OK)
            st = fd2_submit_events_um(ac, xs.data(), ys.data(), zs.data(), nullptr, hist.data(), nps.data(),
                                      c->geoms.size() > 1 ? gg.data() : nullptr, na);
        if (st == FD2_OK) st = fd2_run(ac);
        if (st == FD2_OK) st = fd2_wait(ac);
        if (st != FD2_OK) return sg_fail(s, st, std::string("audit Monte Carlo: ") + fd2_last_error(ac));
        // every detected photon is in exactly one radial category: the
        // categories' totals over the audited rows, pooled on the GPU
        std::vector<unsigned long long> hsum((size_t)nb);
        e = cudaMemsetAsync(B->a_hist, 0, sizeof(unsigned long long) * nb, ac->stream);
        if (e == cudaSuccess) {
            const int blocks = (int)std::max<long long>(1, std::min<long long>(4LL * s->sm_count,
                                                                               ((long long)na * nb + 255) / 256));
            radial_pool_kernel<<<blocks, 256, sizeof(unsigned long long) * nb, ac->stream>>>(ac->d_radial, na, nb,
                                                                                           B->a_hist);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(hsum.data(), B->a_hist, sizeof(unsigned long long) * nb, cudaMemcpyDeviceToHost,
                                ac->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ac->stream);
        if (e != cudaSuccess) return sg_cuda(s, e, "audit pooling");
        std::vector<double> hmc((size_t)nb, 0.0);
        double mc = 0.0;
        for (int j = 0; j < nb; ++j) hmc[(size_t)j] = (double)hsum[(size_t)j];
        for (int j = 0; j < nb; ++j) mc += hmc[(size_t)j];
        const double expct = pool[(size_t)nb], var = pool[(size_t)nb + 1], ph = pool[(size_t)nb + 2];
        double ssg = 0.0, l1 = 0.0;
        for (int j = 0; j < nb; ++j) ssg += pool[(size_t)j];
        for (int j = 0; j < nb; ++j)
            l1 += std::fabs((mc > 0 ? hmc[(size_t)j] / mc : 0) - (ssg > 0 ? pool[(size_t)j] / ssg : 0));
        out.audit_mc_detected = mc;
        out.audit_sg_expected = expct;
        out.audit_photons = ph;
        out.audit_z = var > 0 ? (mc - expct) / std::sqrt(var) : 0.0;
        out.audit_radial_l1 = l1;
    }
    out.audit_ms = (float)std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_audit).count();
    out.total_ms = (float)(run_ms + out.audit_ms);
    out.mc_events = counts[2];
    if (stats) *stats = out;
    return FD2_OK;
}
