// fd2_device.cuh -- device-side core of the production transport.
//
// Philox-4x32-10 uniforms and the FP32 photon walker.  The walker follows
// the reference's per-photon random walk (main/kernel_cuda_c_ver1_0.cu, C
// path: algo :553, isotropic :702, dist_to_surface :966, detection :3372,
// boundary_analysis :1582, transmit :2421, refl_bottom :2985,
// trans_dir_cos :3169, RoughSurface :3261) decision for decision, with
// changes that keep the distribution and suit sm_100a:
//   * each photon draws from its own xoshiro128+ stream (Blackman & Vigna,
//     "Scrambled linear pseudorandom number generators", ACM TOMS 47(4),
//     2021) whose 128-bit state is one Philox-4x32-10 block (Salmon et al.,
//     "Parallel random numbers: as easy as 1, 2, 3", SC'11) keyed by the run
//     seed at counter (0, photon-in-event, event, run): a photon's walk does
//     not depend on which lane runs it or when, and a draw costs a handful
//     of integer operations in registers instead of a Philox block per four
//     uniforms;
//   * angle tests are made on cosines (acos(c) > 1.57 <=> c < cos 1.57) and
//     the Fresnel coefficients use the cosine forms, so the walk needs no
//     acos/asin/tan/pow; the refraction keeps the reference's formula
//     d' = -cos(t_t) n - (sin t_t / sin t_i)(d + cos(t_i) n);
//   * the wall quadratic uses the cancellation-free root, with the
//     discriminant recomputed in FP64 when it nearly cancels;
//   * the whole walk is inlined around one photon held in registers, with a
//     single site for the column change and for the new-column normal.
// Tallies are not touched here: a step returns the photon's fate (and
// pixel) and the kernel aggregates them per warp.
#pragma once

#include <cstdint>

#include "fd2_types.h"

namespace fd2 {

// ---------------------------------------------------------------- Philox

__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint32_t k0, uint32_t k1)
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

// Philox-4x32-10 with the key schedule precomputed: rk[2r], rk[2r+1] are
// the two key words of round r (the run's keys, identical for every lane).
__device__ __forceinline__ uint4 philox4x32_10_rk(uint4 c, const uint32_t *rk)
{
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t lo0 = 0xD2511F53u * c.x, hi0 = __umulhi(0xD2511F53u, c.x);
        const uint32_t lo1 = 0xCD9E8D57u * c.z, hi1 = __umulhi(0xCD9E8D57u, c.z);
        c = make_uint4(hi1 ^ c.y ^ rk[2 * r], lo1, hi0 ^ c.w ^ rk[2 * r + 1], lo0);
    }
    return c;
}

// Uniform k 2^-23 + 2^-24 in [2^-24, 1 - 2^-24] from the top 23 bits k:
// (1 + k 2^-23) - (1 - 2^-24), exact in float.
__device__ __forceinline__ float u01(uint32_t r)
{
    return __uint_as_float(0x3F800000u | (r >> 9)) - 0.99999994039535522461f;
}

// Internal step result: the photon waits at a column wall for the Fresnel
// part of its surface interaction (not a fate).
constexpr int kNeedsFresnel = 100;
// Internal step results of the crosstalk path: the photon crosses into the
// adjacent column and needs that column's normal (crosstalk_normal), or its
// attempt was rejected and is retried in the next round.
constexpr int kNeedsNormal = 101;
constexpr int kRetryNormal = 102;

// Warp-uniform part of a photon's seed: the Philox round keys of the run
// seed (the kernel keeps them in shared memory) and the run counter.
struct RngKey {
    const uint32_t *rk;
    uint32_t run;
};


// ---------------------------------------------------------------- walker

__device__ __forceinline__ void renorm(float &x, float &y, float &z)
{
    const float nrm = sqrtf(x * x + y * y + z * z);
    if (nrm < 1.0f - kEps || nrm > 1.0f + kEps) {
        const float inv = 1.0f / nrm;
        x *= inv; y *= inv; z *= inv;
    }
}

// Fresnel reflectance (unpolarised) for cos(incidence) c, cos(refraction)
// ct and relative index eta = n_incident / n_transmitted.
__device__ __forceinline__ float fresnel(float c, float ct, float eta)
{
    const float a = eta * c, b = eta * ct;
    const float rs = __fdividef(a - ct, a + ct);
    const float rp = __fdividef(c - b, c + b);
    return 0.5f * (rs * rs + rp * rp);
}

// Larger root of a t^2 + b t + c = 0 (the far wall of the column), without
// cancellation; 999 where the reference's formula yields NaN.
__device__ __forceinline__ float wall_root(float qa, float qb, float qc)
{
    float disc = qb * qb - 4.0f * qa * qc;
    if (fabsf(disc) < 2.44140625e-4f * (qb * qb)) {
        // near-cancelling discriminant: products of floats are exact in FP64
        disc = (float)((double)qb * (double)qb - 4.0 * (double)qa * (double)qc);
    }
    if (!(qa > 0.0f) || !(disc >= 0.0f)) return 999.0f;
    const float s = sqrtf(disc);
    if (qb >= 0.0f) {
        const float den = qb + s;
        return den != 0.0f ? (-2.0f * qc) / den : 0.0f;
    }
    return (s - qb) / (2.0f * qa);
}

struct Walker {
    // photon
    float px, py, pz;   // position
    float dx, dy, dz;   // direction
    float nx, ny, nz;   // current surface normal
    float xc, yc;       // centre of the current column
    float dist;         // path length
    float budget;       // absorption lengths left before bulk absorption
    uint32_t rebound;   // boundary interactions
    int ii, jj;         // detection pixel (-1: outside the PRF bounds)
    // The photon's random stream: xoshiro128+ state (never all zero; a
    // Philox block is all zero with probability 2^-128, and start() then
    // sets one bit).  The float uses the top 23 bits of each output, the
    // bits the generator's authors recommend for floating point.
    uint32_t s0, s1, s2, s3;

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
        return u01(r);
    }

    // Start photon `photon_in_event` of event `event_index` at the event's
    // position (ex, ey, ez), in the column centred on it.  The event record
    // itself stays outside the walker (the kernel keeps it in shared memory),
    // so it holds no registers through the walk.
    __device__ __forceinline__ void start(float ex, float ey, float ez, uint32_t photon_in_event,
                                          uint32_t event_index, bool first, const RngKey &key)
    {
        const uint4 k = philox4x32_10_rk(make_uint4(0u, photon_in_event, event_index, key.run), key.rk);
        s0 = k.x;
        s1 = k.y;
        s2 = k.z;
        s3 = k.w | ((k.x | k.y | k.z | k.w) == 0u ? 1u : 0u);
        px = ex; py = ey; pz = ez;
        xc = ex; yc = ey;
        nx = 0.0f; ny = 0.0f; nz = 0.0f;
        dist = 0.0f;
        rebound = 0;
        ii = -1; jj = -1;
        emit(first);
        budget = -__logf(u());  // Exp(1)
    }

    // Isotropic emission; the first photon of an event rejects |cos| <= 0.01
    // (the reference's CPU driver, hybridMANTIS_c_ver1_0.c:257-262).
    __device__ __forceinline__ void emit(bool first)
    {
        float c = 2.0f * u() - 1.0f;
        if (first) {
            for (int t = 0; t < 64 && fabsf(c) <= 0.01f; ++t) c = 2.0f * u() - 1.0f;
        }
        const float rr = sqrtf(fmaxf(0.0f, 1.0f - c * c));
        float s, co;
        __sincosf(kPi * (2.0f * u() - 1.0f), &s, &co);
        dx = rr * co;
        dy = rr * s;
        dz = c;
        renorm(dx, dy, dz);
    }

    // n <- normalize(n + beta * q), q the reference's perturbation vector:
    // z = 2u1 - 1, transverse radius sqrt(1 - u1^2), uniform azimuth, then
    // normalised (RoughSurface).
    __device__ __forceinline__ void roughen(float beta)
    {
        const float u1 = u();
        const float qz = 2.0f * u1 - 1.0f;
        const float rr = sqrtf(fmaxf(0.0f, 1.0f - u1 * u1));
        float s, c;
        __sincosf(kPi * (2.0f * u() - 1.0f), &s, &c);
        const float qx = rr * c, qy = rr * s;
        // |q|^2 = (1 - u1^2) + (2 u1 - 1)^2 = 3 u1^2 - 4 u1 + 2 for u1 in (0, 1)
        const float bq = beta * rsqrtf(fmaf(u1, fmaf(3.0f, u1, -4.0f), 2.0f));
        const float rx = fmaf(bq, qx, nx), ry = fmaf(bq, qy, ny), rz = fmaf(bq, qz, nz);
        const float ir = rsqrtf(rx * rx + ry * ry + rz * rz);
        nx = rx * ir; ny = ry * ir; nz = rz * ir;
    }

    // A new column's orientation before its own roughening: (ix, iy, iz)
    // roughened with beta = 1 and flattened to the x-y plane (the
    // reference's RoughSurface(1) followed by nz = 0 and a 2D
    // normalisation).  The 3D normalisation between the two is a positive
    // scale the 2D one removes, so the flattened direction of i + q/|q| is
    // taken directly; the draws are roughen's.
    __device__ __forceinline__ void flat_rough(float ix, float iy, float iz)
    {
        const float u1 = u();
        const float qz = 2.0f * u1 - 1.0f;
        const float rr = sqrtf(fmaxf(0.0f, 1.0f - u1 * u1));
        float s, c;
        __sincosf(kPi * (2.0f * u() - 1.0f), &s, &c);
        const float qx = rr * c, qy = rr * s;
        const float iq = rsqrtf(fmaf(u1, fmaf(3.0f, u1, -4.0f), 2.0f));  // 1 / |q|, as in roughen
        const float vx = fmaf(iq, qx, ix), vy = fmaf(iq, qy, iy);
        const float inv = rsqrtf(vx * vx + vy * vy);
        nx = vx * inv;
        ny = vy * inv;
        nz = 0.0f;
        (void)iz;
    }

    template <class G>
    __device__ __forceinline__ bool outside_xy(const G &g) const
    {
        return px < kEps || px > g.xdet || py < kEps || py > g.ydet;
    }
    template <class G>
    __device__ __forceinline__ bool outside_detector(const G &g) const
    {
        return outside_xy(g) || pz < -g.half || pz > g.half;
    }
    template <class G>
    __device__ __forceinline__ bool at_top(const G &g) const
    {
        return fabsf(pz - g.half) < kEps && dz > 0.0f;
    }

    // Wall or z plane ahead, then the reference's pull-back into the column
    // (dist_to_surface), then bulk absorption (isotropic).
    template <class G>
    __device__ __forceinline__ int flight(const G &g)
    {
        const float ddx = px - xc, ddy = py - yc;
        const float qa = dx * dx + dy * dy;
        const float qb = 2.0f * (ddx * dx + ddy * dy);
        const float qc = ddx * ddx + ddy * ddy - g.R * g.R;
        const float dcyl = wall_root(qa, qb, qc);
        float d = dcyl;
        if (dz != 0.0f) {
            const float zp = dz > 0.0f ? g.half : -g.half;
            const bool straight = fabsf(dx) < kEps && fabsf(dy) < kEps && fabsf(fabsf(dz) - 1.0f) < kEps;
            const float dplane = (zp - pz) / dz;
            if (!straight && dplane >= dcyl) {
                pz = fmaf(d, dz, pz);
            } else {
                d = dplane;
                pz = zp;
            }
        }
        px = fmaf(d, dx, px);
        py = fmaf(d, dy, py);
        if (outside_detector(g)) return kLost;
        const float thr = g.R - 1e-5f;
        float r = sqrtf((px - xc) * (px - xc) + (py - yc) * (py - yc));
        float step = 0.5f;
        int moved = 0, halved = 0;
        while (r > thr && moved < 10 && halved < 10) {
            const float sx = px, sy = py;
            px = fmaf(-step, dx, px);
            py = fmaf(-step, dy, py);
            const float rn = sqrtf((px - xc) * (px - xc) + (py - yc) * (py - yc));
            if (rn > r) {
                px = sx; py = sy;
                step *= 0.5f;
                ++halved;
            } else {
                r = rn;
                ++moved;
            }
        }
        if (r > thr) return kOutOfCol;
        if (outside_detector(g)) return kLost;
        dist += d;
        if (g.neg_inv_mu != 0.0f) {
            // bulk absorption: one Exp(1) budget of absorption lengths per
            // photon, spent flight by flight; by the exponential's lack of
            // memory the same law as the reference's fresh draw per flight
            // (absorbed when d >= -ln(u) / mu)
            const float da = d * g.mu;
            if (da >= budget && d >= 0.0f) return kAbsBulk;
            budget -= da;
        }
        return kAlive;
    }

    template <class G>
    __device__ __forceinline__ void set_pixel(const G &g)
    {
        ii = -1;
        jj = -1;
        if (px <= g.ub_x && py <= g.ub_y && px >= g.lb_x && py >= g.lb_y) {
            ii = (int)floorf(__fdiv_rn(px - g.lb_x, g.pixel));
            jj = (int)floorf(__fdiv_rn(py - g.lb_y, g.pixel));
        }
    }

    // Orientation of the next column: a random normal within 1.57 rad of
    // the reversed direction, flattened to the x-y plane, roughened.
    template <class G>
    __device__ __forceinline__ int new_column_normal(const G &g, float ix, float iy, float iz, int &tries,
                                                     bool always_rough)
    {
        for (;;) {
            flat_rough(ix, iy, iz);
            if (always_rough || g.beta > 0.0f) roughen(g.beta);
            if (!(ix * nx + iy * ny + iz * nz < kCos157)) return kAlive;
            if (tries < 100) {
                ++tries;
                continue;
            }
            return kTheta1;
        }
    }

    // Leave the current column after a transmission through its wall
    // (transmit without crosstalk; crosstalk is crosstalk_normal): hop
    // U(d_min, d_max) with the top reflector and the sensor on the way, then
    // orient the next column.  Hops after a top reflection repeat the loop.
    // A photon reflected by the sensor between columns hops again
    // (refl_bottom): up to the top, or into a new column whose normal is
    // drawn around its own reversed direction, always roughened; after a
    // sensor met at the hop's end it stays where that hop left it unless it
    // reached the top.
    // Written as a state machine so that the kernel holds one copy of each
    // part (hop, sensor, hop after the sensor, next normal, top reflector):
    // the walk's instruction fetch grows with the kernel's code size.
    template <class G>
    __device__ __forceinline__ int leave_column(const G &g)
    {
        enum { kHop, kSensor, kSensorHop, kNormal, kAfterSensor, kEnd };
        float ix = -dx, iy = -dy, iz = -dz;  // the next normal is drawn around these
        // One register for the rest: retries of the side hop's and the top
        // hops' normals (bits 0-7 and 8-15, each at most 100), top
        // reflections (bits 16-28, at most kMaxTopLoops), and three flags.
        constexpr uint32_t kSideHop = 1u << 29;     // the hop leaves a column wall (not the top)
        constexpr uint32_t kFromEnd = 1u << 30;     // the sensor was met at a hop's end, not during it
        constexpr uint32_t kAfterHop = 1u << 31;    // the pending normal follows a sensor hop
        constexpr uint32_t kTopOne = 1u << 16, kTopMask = 0x1fffu << 16;
        uint32_t counts = kSideHop;
        int st = kHop;
        for (;;) {
            if (st == kHop) {
                const float sx = px, sy = py, sz = pz;
                const float d = fmaf(u(), g.d_span, g.d_min);
                px = fmaf(dx, d, sx);
                py = fmaf(dy, d, sy);
                pz = fmaf(dz, d, sz);
                const float dtop = (g.half - sz) / dz;
                const float dbot = (-g.half - sz) / dz;
                if (outside_xy(g)) return kLost;
                counts &= ~kAfterHop;
                st = kNormal;
                if (pz < -g.half || pz > g.half) {
                    if (dtop < d && dtop > kEps) {
                        px = fmaf(dx, dtop, sx);
                        py = fmaf(dy, dtop, sy);
                        pz = g.half;
                        dist += dtop;
                    } else if (dbot < d && dbot > kEps) {
                        px = fmaf(dx, dbot, sx);
                        py = fmaf(dy, dbot, sy);
                        pz = -g.half;
                        dist += dbot;
                        counts &= ~kFromEnd;
                        st = kSensor;
                    } else {
                        return kLost;
                    }
                } else {
                    dist += d;
                }
            } else if (st == kSensor) {
                // sensor between columns: reflect with sensorRefl, else detect
                if (!(g.sensor_refl > 0.0f && u() < g.sensor_refl)) {
                    set_pixel(g);
                    return kDetect;
                }
                dz = -dz;
                renorm(dx, dy, dz);
                st = kSensorHop;
            } else if (st == kSensorHop) {
                const float sx = px, sy = py, sz = pz;
                const float hop = fmaf(u(), g.d_span, g.d_min);
                const float dtop = (g.half - sz) / dz;
                px = fmaf(dx, hop, sx);
                py = fmaf(dy, hop, sy);
                pz = fmaf(dz, hop, sz);
                if (outside_xy(g)) return kLost;
                if (pz > g.half) {
                    if (!(dtop < hop && dtop > kEps)) return kLost;
                    px = fmaf(dx, dtop, sx);
                    py = fmaf(dy, dtop, sy);
                    pz = g.half;
                    dist += dtop;
                    st = kAfterSensor;
                } else {
                    dist += hop;
                    counts |= kAfterHop;
                    st = kNormal;
                }
            } else if (st == kNormal) {
                const bool after_sensor = (counts & kAfterHop) != 0u, side_hop = (counts & kSideHop) != 0u;
                int t = after_sensor ? 0 : (int)((side_hop ? counts : counts >> 8) & 0xffu);
                // after a sensor hop: around the hop's own reversed direction
                const float ax = after_sensor ? -dx : ix, ay = after_sensor ? -dy : iy, az = after_sensor ? -dz : iz;
                const int f = new_column_normal(g, ax, ay, az, t, after_sensor);
                if (f != kAlive) return f;
                if (after_sensor) {
                    st = kAfterSensor;
                } else {
                    counts = side_hop ? (counts & ~0xffu) | (uint32_t)t : (counts & ~0xff00u) | ((uint32_t)t << 8);
                    if (side_hop && (fabsf(px) < kEps || fabsf(px - g.xdet) < kEps || fabsf(py) < kEps ||
                                     fabsf(py - g.ydet) < kEps))
                        return kLost;
                    st = kEnd;
                }
            } else if (st == kAfterSensor) {
                counts &= ~kAfterHop;
                if (!(counts & kFromEnd)) {
                    // a sensor met during the hop: the next normal follows
                    // unless the sensor hop reached the top
                    if (at_top(g)) {
                        st = kEnd;
                    } else {
                        st = kNormal;
                    }
                } else {
                    // a sensor hop that reached the top ends at the top
                    // reflector (the hop's end check finds the top at once)
                    if (!at_top(g)) return kAlive;
                    st = kEnd;
                }
            } else {
                // kEnd: top reflector / sensor at the end of the hop
                if (at_top(g)) {
                    if (g.top_absfrac > 0.0f && u() < g.top_absfrac) return kAbsTop;
                    dz = -fabsf(2.0f * u() - 1.0f);
                    const float rr = sqrtf(fmaxf(0.0f, 1.0f - dz * dz));
                    float s, c;
                    __sincosf(kPi * (2.0f * u() - 1.0f), &s, &c);
                    dx = rr * c;
                    dy = rr * s;
                    ix = -dx; iy = -dy; iz = -dz;
                    counts = (counts & ~kSideHop) + kTopOne;
                    if ((counts & kTopMask) == ((uint32_t)kMaxTopLoops << 16)) return kCapped;
                    st = kHop;
                } else {
                    if (fabsf(pz + g.half) >= kEps) return kAlive;
                    counts |= kFromEnd;
                    st = kSensor;
                }
            }
        }
    }

    // Interaction with a surface (boundary_analysis), first part: the top
    // surface and columnar crosstalk.  Returns a fate, kAlive, or
    // kNeedsFresnel when the photon meets the column wall without crosstalk;
    // the Fresnel part (surface_fresnel) can then run later, from the photon
    // state alone.
    template <class G>
    __device__ __forceinline__ int surface_entry(const G &g)
    {
        if (at_top(g)) {
            if (g.top_absfrac > 0.0f && u() < g.top_absfrac) return kAbsTop;
            dz = -fabsf(2.0f * u() - 1.0f);
            const float rr = sqrtf(fmaxf(0.0f, 1.0f - dz * dz));
            float s, c;
            __sincosf(kPi * (2.0f * u() - 1.0f), &s, &c);
            dx = rr * c;
            dy = rr * s;
            return kAlive;
        }
        // columnar crosstalk: certain in the top 20 %, linear to 0.5 at mid
        // depth, back to 1 at the sensor
        float cct = 0.0f;
        if (pz <= g.half && pz >= g.cct_band_lo) cct = 1.0f;
        else if (pz < g.cct_band_lo && pz >= 0.0f) cct = fmaf(pz, g.cct_k_hi, 0.5f);
        else if (pz < 0.0f && pz >= -g.half) cct = fmaf(pz + g.half, g.cct_k_lo, 1.0f);
        if (!(u() < cct)) return kNeedsFresnel;
        return kNeedsNormal;
    }

    // Crosstalk into the adjacent column (transmit with crosstalk): one
    // attempt at the new column's normal, a random normal within 1.57 rad of
    // the reversed direction, flattened and roughened.  Returns kAlive (the
    // photon is in the new column), kTheta1 (no normal after 100 retries) or
    // kRetryNormal (rejected: the kernel retries in its next round, beside
    // the other lanes' first attempts, instead of looping here with the few
    // rejected lanes of the warp).
    template <class G>
    __device__ __forceinline__ int crosstalk_normal(const G &g, int &tries)
    {
        const float ix = -dx, iy = -dy, iz = -dz;
        flat_rough(ix, iy, iz);
        if (g.beta > 0.0f) roughen(g.beta);
        if (!(ix * nx + iy * ny + iz * nz < kCos157)) {
            xc = fmaf(-g.R, nx, px);
            yc = fmaf(-g.R, ny, py);
            return kAlive;
        }
        if (tries < 100) {
            ++tries;
            return kRetryNormal;
        }
        return kTheta1;
    }

    // Second part: Fresnel reflection / refraction on the rough wall, with
    // hops between columns until the photon is back inside a column.
    template <class G>
    __device__ __forceinline__ int surface_fresnel(const G &g)
    {
        bool outside = false;
        int tries_theta = 0, tries_normal = 0, reperturbs = 0, smooth = 0;
        float pr = __int_as_float(0x7fc00000);  // 0/0 until a rule sets it
        float st = 0.0f, ct = 1.0f;            // sin, cos of the last refraction angle
        float kx = 0, ky = 0, kz = 0, kdx = 0, kdy = 0, kdz = 0;
        enum { kLeave, kNewSurface, kRestore, kIncidence } stage = kNewSurface;
        int fate = kAlive;
        for (int loop = 0; loop < kMaxSurfaceLoops; ++loop) {
            if (stage == kNewSurface) {
                if (!outside) {
                    const float ax = xc - px, ay = yc - py;
                    const float im = rsqrtf(ax * ax + ay * ay);
                    nx = ax * im; ny = ay * im; nz = 0.0f;
                    if (g.beta > 0.0f) roughen(g.beta);
                } else {
                    xc = fmaf(-g.R, nx, px);
                    yc = fmaf(-g.R, ny, py);
                }
                kx = nx; ky = ny; kz = nz;
                kdx = dx; kdy = dy; kdz = dz;
                stage = kRestore;
            }
            if (stage == kRestore) {
                nx = kx; ny = ky; nz = kz;
                dx = kdx; dy = kdy; dz = kdz;
                if (reperturbs != 0) {
                    if (g.beta > 0.0f) roughen(g.beta);
                    if (outside) {
                        xc = fmaf(-g.R, nx, px);
                        yc = fmaf(-g.R, ny, py);
                    }
                }
                stage = kIncidence;
            }
            if (stage == kIncidence) {
                const float c1 = -(dx * nx + dy * ny + dz * nz);
                if (c1 > 1.0f || c1 < 0.0f) {
                    if (outside) {
                        const int f = new_column_normal(g, -dx, -dy, -dz, tries_normal, false);
                        if (f != kAlive) {
                            fate = f;
                            break;
                        }
                    }
                    if (tries_theta < 100) {
                        ++tries_theta;
                        stage = kNewSurface;
                        continue;
                    }
                    fate = kTheta1;
                    break;
                }
                const float si = sqrtf(fmaxf(0.0f, 1.0f - c1 * c1));
                if (!outside) {
                    if (c1 < g.cos_tir_in) {
                        pr = 1.0f;
                    } else {
                        st = g.eta_in * si;
                        ct = sqrtf(fmaxf(0.0f, 1.0f - st * st));
                        pr = fresnel(c1, ct, g.eta_in);
                    }
                } else if (g.stale_out) {
                    if (c1 < g.cos_tir_out) pr = 1.0f;
                } else {
                    st = g.eta_out * si;
                    ct = sqrtf(fmaxf(0.0f, 1.0f - st * st));
                    pr = fresnel(c1, ct, g.eta_out);
                }
                if (u() < pr) {
                    // specular reflection
                    dx = fmaf(2.0f * c1, nx, dx);
                    dy = fmaf(2.0f * c1, ny, dy);
                    dz = fmaf(2.0f * c1, nz, dz);
                    renorm(dx, dy, dz);
                    if (kx * dx + ky * dy + kz * dz < kCos157) {
                        if (++reperturbs < 4) {
                            stage = kRestore;
                            continue;
                        }
                        nx = kx; ny = ky; nz = kz;
                        dx = kdx; dy = kdy; dz = kdz;
                        reperturbs = 0;
                        if (smooth < 25) {
                            ++smooth;
                            continue;  // stage stays kIncidence
                        }
                        fate = kTheta1;
                        break;
                    }
                    if (!outside) break;  // reflected inside the column: done
                    stage = kLeave;
                } else {
                    // refraction with the reference's formula
                    const float ratio = si > 0.0f ? __fdividef(st, si) : 0.0f;
                    const float tx = fmaf(c1, nx, dx), ty = fmaf(c1, ny, dy), tz = fmaf(c1, nz, dz);
                    dx = -ct * nx - ratio * tx;
                    dy = -ct * ny - ratio * ty;
                    dz = -ct * nz - ratio * tz;
                    renorm(dx, dy, dz);
                    if (outside) break;  // entered the next column: done
                    stage = kLeave;
                }
            }
            // kLeave: hop between columns
            const int f = leave_column(g);
            if (f != kAlive) {
                fate = f;
                break;
            }
            outside = true;
            stage = kNewSurface;
            if (loop + 1 == kMaxSurfaceLoops) fate = kCapped;
        }
        return fate;
    }

    // ---- explicit column lattice (options.column_grid = 1 or 2; no
    // counterpart in the reference, whose next column is drawn at random
    // after every crossing).  Columns are the cylinders of radius R around
    // the square lattice points ((i + 1/2) p, (j + 1/2) p), or around the
    // hexagonal lattice points ((i + 1/2) p + o_j, (j + 1/2) h), h = p sqrt(3)/2,
    // o_j = p/2 on odd rows; the photon is either inside the column centred at
    // (xc, yc) or in the gap medium between them.
    // Walls refract and reflect with the unpolarised Fresnel coefficients on
    // the roughened geometric normal (vector Snell law); in the gap the
    // photon flies straight until it meets a column (traced cell by cell),
    // the top reflector, the sensor or the detector's side.  Bulk absorption
    // acts inside the columns only.
    bool in_gap;

    template <class G>
    __device__ __forceinline__ void grid_place(const G &g)
    {
        if (g.grid == 2) {
            // the nearest of the brick's own column and its four diagonal
            // neighbours in the rows above and below
            const float h = g.pitch * 0.8660254037844386f;
            const int j = (int)floorf(py / h);
            const float o = (j & 1) ? 0.5f * g.pitch : 0.0f;
            const int i = (int)floorf((px - o) / g.pitch);
            float bx = 0.0f, by = 0.0f, bd = 3.0e38f;
#pragma unroll
            for (int q = 0; q < 5; ++q) {
                float cx, cy;
                hex_candidate(g, i, j, q, cx, cy);
                const float d2 = (px - cx) * (px - cx) + (py - cy) * (py - cy);
                if (d2 < bd) { bd = d2; bx = cx; by = cy; }
            }
            xc = bx;
            yc = by;
            in_gap = bd >= g.R * g.R;
            return;
        }
        xc = (floorf(px / g.pitch) + 0.5f) * g.pitch;
        yc = (floorf(py / g.pitch) + 0.5f) * g.pitch;
        const float rx = px - xc, ry = py - yc;
        in_gap = rx * rx + ry * ry >= g.R * g.R;
    }

    // Hexagonal lattice: the rows are strips of height h; in row j the
    // bricks [i p + o_j, (i + 1) p + o_j) each hold one column at their
    // centre.  A column reaches at most R < p/2 sideways but may reach past
    // its strip (R > h/2 when the gap is small), so the columns that
    // overlap brick (i, j) are its own (q = 0) and the four centred on its
    // corners' columns in rows j - 1 and j + 1 (q = 1..4).
    template <class G>
    __device__ __forceinline__ static void hex_candidate(const G &g, int i, int j, int q, float &cx, float &cy)
    {
        const float p = g.pitch, h = p * 0.8660254037844386f;
        const float o = (j & 1) ? 0.5f * p : 0.0f;
        cx = ((float)i + 0.5f) * p + o;
        cy = ((float)j + 0.5f) * h;
        if (q > 0) {
            cy += q <= 2 ? h : -h;
            cx += (q & 1) ? -0.5f * p : 0.5f * p;
        }
    }

    // Top reflector (absorb or diffuse reflection downwards, the reference's
    // top rule) or sensor (detect, or specular reflection with sensor_refl).
    template <class G>
    __device__ __forceinline__ int grid_plane(const G &g, bool top)
    {
        if (top) {
            if (g.top_absfrac > 0.0f && u() < g.top_absfrac) return kAbsTop;
            dz = -fabsf(2.0f * u() - 1.0f);
            const float rr = sqrtf(fmaxf(0.0f, 1.0f - dz * dz));
            float s, c;
            __sincosf(kPi * (2.0f * u() - 1.0f), &s, &c);
            dx = rr * c;
            dy = rr * s;
            return kAlive;
        }
        if (!(g.sensor_refl > 0.0f && u() < g.sensor_refl)) {
            set_pixel(g);
            return kDetect;
        }
        dz = -dz;
        return kAlive;
    }

    // A wall of the column centred at (cx, cy), met at (px, py); `inside`:
    // from within the column.  The normal toward the incident side is
    // roughened (redrawn while the photon would not meet it); reflect with
    // the Fresnel probability (total reflection included), else refract.
    template <class G>
    __device__ __forceinline__ int grid_wall(const G &g, float cx, float cy, bool inside)
    {
        float ox = px - cx, oy = py - cy;
        const float inv = rsqrtf(ox * ox + oy * oy);
        ox *= inv;
        oy *= inv;
        const float sgn = inside ? -1.0f : 1.0f;  // normal toward the incident medium
        float c1 = 0.0f;
        for (int t = 0; t < 8; ++t) {
            nx = sgn * ox; ny = sgn * oy; nz = 0.0f;
            if (g.beta > 0.0f) roughen(g.beta);
            c1 = -(dx * nx + dy * ny + dz * nz);
            if (c1 > 0.0f) break;
        }
        if (!(c1 > 0.0f)) {
            nx = sgn * ox; ny = sgn * oy; nz = 0.0f;
            c1 = fmaxf(-(dx * nx + dy * ny), 0.0f);
        }
        const float eta = inside ? g.eta_in : g.eta_out;  // n_incident / n_transmitted
        const float st2 = eta * eta * fmaxf(0.0f, 1.0f - c1 * c1);
        float pr = 1.0f, ct = 0.0f;
        if (st2 < 1.0f) {
            ct = sqrtf(1.0f - st2);
            pr = fresnel(c1, ct, eta);
        }
        if (u() < pr) {
            dx = fmaf(2.0f * c1, nx, dx);
            dy = fmaf(2.0f * c1, ny, dy);
            dz = fmaf(2.0f * c1, nz, dz);
            renorm(dx, dy, dz);
            return kAlive;
        }
        const float k = eta * c1 - ct;
        dx = fmaf(eta, dx, k * nx);
        dy = fmaf(eta, dy, k * ny);
        dz = fmaf(eta, dz, k * nz);
        renorm(dx, dy, dz);
        in_gap = inside;
        if (!inside) {
            xc = cx;
            yc = cy;
        }
        return kAlive;
    }

    // The flight of a lattice segment: to a plane (kToPlane), to the wall of
    // the column at (wx, wy) (kToWall; win: from inside it), or a fate.
    static constexpr int kToPlane = 200, kToWall = 201;
    template <class G>
    __device__ __forceinline__ int grid_flight(const G &g, float &wx, float &wy, bool &win)
    {
        const float zp = dz > 0.0f ? g.half : -g.half;
        const float dplane = dz != 0.0f ? (zp - pz) / dz : 3.0e38f;
        if (!in_gap) {
            const float ddx = px - xc, ddy = py - yc;
            const float qa = dx * dx + dy * dy;
            const float qb = 2.0f * (ddx * dx + ddy * dy);
            // a photon on the wall (rounded just outside it) is on the wall:
            // the far root then always exists
            const float qc = fminf(ddx * ddx + ddy * ddy - g.R * g.R, 0.0f);
            const float dw = wall_root(qa, qb, qc);
            const bool plane = dplane <= dw;
            const float d = fmaxf(plane ? dplane : dw, 0.0f);
            px = fmaf(d, dx, px);
            py = fmaf(d, dy, py);
            pz = plane ? zp : fmaf(d, dz, pz);
            dist += d;
            if (g.neg_inv_mu != 0.0f) {
                const float da = d * g.mu;
                if (da >= budget) return kAbsBulk;
                budget -= da;
            }
            if (outside_xy(g)) return kLost;
            if (plane) return kToPlane;
            wx = xc;
            wy = yc;
            win = true;
            return kToWall;
        }
        // in the gap: the first column along the ray, cell by cell (a column
        // lies inside its own cell, so the first hit is in the first cell
        // that holds one)
        const float p = g.pitch;
        float tx = 3.0e38f, ty = 3.0e38f;
        if (dx > 0.0f) tx = (g.xdet - px) / dx;
        else if (dx < 0.0f) tx = -px / dx;
        if (dy > 0.0f) ty = (g.ydet - py) / dy;
        else if (dy < 0.0f) ty = -py / dy;
        const float tside = fminf(tx, ty);
        const float tend = fminf(dplane, tside);
        if (g.grid == 2) {
            // brick by brick; a hit counts in the brick where it lies
            const float h = p * 0.8660254037844386f;
            int j = (int)floorf(py / h);
            int i = (int)floorf((px - ((j & 1) ? 0.5f * p : 0.0f)) / p);
            const float qa = dx * dx + dy * dy;
            float tin = 0.0f;
            for (int k = 0; k < kMaxGridCells; ++k) {
                const float o = (j & 1) ? 0.5f * p : 0.0f;
                const float xl = (float)i * p + o;
                const float tX = dx > 0.0f ? (xl + p - px) / dx : dx < 0.0f ? (xl - px) / dx : 3.0e38f;
                const float tY = dy > 0.0f ? ((float)(j + 1) * h - py) / dy : dy < 0.0f ? ((float)j * h - py) / dy : 3.0e38f;
                const float tout = fminf(tX, tY);
                float tb = 3.0e38f, bx = 0.0f, by = 0.0f;
#pragma unroll
                for (int q = 0; q < 5; ++q) {
                    float cx, cy;
                    hex_candidate(g, i, j, q, cx, cy);
                    const float fx = px - cx, fy = py - cy;
                    const float qb = 2.0f * (fx * dx + fy * dy);
                    const float qc = fx * fx + fy * fy - g.R * g.R;
                    if (qa > 0.0f && qb < 0.0f) {
                        const float disc = qb * qb - 4.0f * qa * qc;
                        if (disc >= 0.0f) {
                            const float t1 = (2.0f * qc) / (-qb + sqrtf(disc));
                            if (t1 > 1e-4f && t1 >= tin - 1e-4f && t1 <= tout + 1e-4f && t1 < tb) {
                                tb = t1;
                                bx = cx;
                                by = cy;
                            }
                        }
                    }
                }
                if (tb < tend) {
                    px = fmaf(tb, dx, px);
                    py = fmaf(tb, dy, py);
                    pz = fmaf(tb, dz, pz);
                    dist += tb;
                    wx = bx;
                    wy = by;
                    win = false;
                    return kToWall;
                }
                if (tout >= tend) break;
                if (tX < tY) {
                    i += dx > 0.0f ? 1 : -1;
                } else {
                    // the next row: the brick under the crossing point
                    j += dy > 0.0f ? 1 : -1;
                    const float xo = fmaf(tout, dx, px) - ((j & 1) ? 0.5f * p : 0.0f);
                    i = (int)floorf(xo / p);
                }
                tin = tout;
                if (k + 1 == kMaxGridCells) return kCapped;
            }
            if (dplane <= tside) {
                px = fmaf(dplane, dx, px);
                py = fmaf(dplane, dy, py);
                pz = zp;
                dist += dplane;
                return kToPlane;
            }
            return kLost;
        }
        int i = (int)floorf(px / p), j = (int)floorf(py / p);
        const int si = dx > 0.0f ? 1 : -1, sj = dy > 0.0f ? 1 : -1;
        float tmx = dx != 0.0f ? (((float)(dx > 0.0f ? i + 1 : i)) * p - px) / dx : 3.0e38f;
        float tmy = dy != 0.0f ? (((float)(dy > 0.0f ? j + 1 : j)) * p - py) / dy : 3.0e38f;
        const float tdx = dx != 0.0f ? p / fabsf(dx) : 3.0e38f;
        const float tdy = dy != 0.0f ? p / fabsf(dy) : 3.0e38f;
        const float qa = dx * dx + dy * dy;
        for (int k = 0; k < kMaxGridCells; ++k) {
            const float cx = ((float)i + 0.5f) * p, cy = ((float)j + 0.5f) * p;
            const float fx = px - cx, fy = py - cy;
            const float qb = 2.0f * (fx * dx + fy * dy);
            const float qc = fx * fx + fy * fy - g.R * g.R;
            if (qa > 0.0f && qb < 0.0f) {
                const float disc = qb * qb - 4.0f * qa * qc;
                if (disc >= 0.0f) {
                    const float t1 = (2.0f * qc) / (-qb + sqrtf(disc));  // the entry root
                    if (t1 > 1e-4f && t1 < tend) {
                        px = fmaf(t1, dx, px);
                        py = fmaf(t1, dy, py);
                        pz = fmaf(t1, dz, pz);
                        dist += t1;
                        wx = cx;
                        wy = cy;
                        win = false;
                        return kToWall;
                    }
                }
            }
            const float tn = fminf(tmx, tmy);
            if (tn >= tend) break;
            if (tmx < tmy) {
                i += si;
                tmx += tdx;
            } else {
                j += sj;
                tmy += tdy;
            }
            if (k + 1 == kMaxGridCells) return kCapped;
        }
        if (dplane <= tside) {
            px = fmaf(dplane, dx, px);
            py = fmaf(dplane, dy, py);
            pz = zp;
            dist += dplane;
            return kToPlane;
        }
        return kLost;
    }

    // One segment of the lattice walk: a flight to the next surface and what
    // happens there, the interaction in one place for lanes in either medium.
    template <class G>
    __device__ __forceinline__ int grid_segment(const G &g)
    {
        if (++rebound > kMaxBoundaryCalls) return kCapped;
        float wx = 0.0f, wy = 0.0f;
        bool win = false;
        const int f = grid_flight(g, wx, wy, win);
        if (f == kToPlane) return grid_plane(g, pz > 0.0f);
        if (f == kToWall) return grid_wall(g, wx, wy, win);
        return f;
    }

    // One transport step (the body of the reference's step function algo):
    // flight, sensor, trapped-photon restart (from `event`, the x, y, z of
    // the photon's event), or a surface interaction up to the Fresnel part.  Returns the photon's fate, kAlive while it is in
    // flight, or kNeedsFresnel (run surface_fresnel next).
    template <class G>
    __device__ __forceinline__ int step(const G &g, const float4 &event)
    {
        // one flight, and a second after a specular reflection on the sensor
        // inside a column (a loop, so that the kernel holds one flight)
        bool reflected = false;
#pragma unroll 1
        for (;;) {
            const int f = flight(g);
            if (f != kAlive) return f;
            if (reflected || !(fabsf(pz + g.half) < kEps)) break;
            // sensor plane inside a column (detection)
            if (!(g.sensor_refl > 0.0f && u() < g.sensor_refl)) {
                set_pixel(g);
                return kDetect;
            }
            dz = -dz;  // specular reflection on the flat sensor
            renorm(dx, dy, dz);
            reflected = true;
        }
        if (fabsf(dz) < kEps) {
            // trapped travelling horizontally: restart from the event position,
            // keeping the current column (the reference does not reset it)
            px = event.x; py = event.y; pz = event.z;
            emit(false);
            return kAlive;
        }
        if (++rebound > kMaxBoundaryCalls) return kCapped;
        return surface_entry(g);
    }
};

}  // namespace fd2
