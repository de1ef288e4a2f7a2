// fd2_device.cuh -- device-side core of the production transport.
//
// Geometry record, Philox-4x32-10 counter-based RNG and the FP32 photon
// walker.  The walker follows the reference's per-photon random walk
// (main/kernel_cuda_c_ver1_0.cu, C path: algo :553, isotropic :702,
// dist_to_surface :966, detection :3372, boundary_analysis :1582,
// transmit :2421, refl_bottom :2985, trans_dir_cos :3169,
// RoughSurface :3261) step for step, with three changes that keep the
// distribution and make it fast on sm_100a:
//   * every uniform comes from Philox keyed by (run seed) at counter
//     (block, photon-in-event, event, stream tag), so a photon's walk does
//     not depend on which lane runs it or when;
//   * angle tests are made on cosines (acos(c) > 1.57 <=> c < cos 1.57) and
//     the Fresnel coefficients use the cosine forms, so the walk needs no
//     acos/asin/tan/pow; the refraction keeps the reference's formula
//     d' = -cos(t_t) n - (sin t_t / sin t_i)(d + cos(t_i) n);
//   * the wall quadratic uses the cancellation-free root, with the
//     discriminant recomputed in FP64 when it nearly cancels.
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

// Uniform in [2^-24, 1 - 2^-24] from the top 23 bits.
__device__ __forceinline__ float u01(uint32_t r)
{
    return __fmaf_rn(__uint2float_rz(r >> 9), 1.1920928955078125e-7f, 5.9604644775390625e-8f);
}

// Per-photon stream: counter (block, photon, event, tag).
struct PhotonRng {
    uint32_t k0, k1, photon, event, tag, block;
    uint32_t b0, b1, b2, b3;
    int avail;

    __device__ __forceinline__ void init(uint64_t seed, uint32_t photon_in_event, uint32_t event_index,
                                         uint32_t stream_tag)
    {
        k0 = (uint32_t)seed;
        k1 = (uint32_t)(seed >> 32);
        photon = photon_in_event;
        event = event_index;
        tag = stream_tag;
        block = 0;
        avail = 0;
    }
    __device__ __forceinline__ float u()
    {
        if (avail == 0) {
            const uint4 r = philox4x32_10(make_uint4(block++, photon, event, tag), k0, k1);
            b0 = r.x; b1 = r.y; b2 = r.z; b3 = r.w;
            avail = 4;
        }
        const uint32_t r = b0;
        b0 = b1; b1 = b2; b2 = b3;
        --avail;
        return u01(r);
    }
};

// ---------------------------------------------------------------- walker

struct Photon {
    float px, py, pz;   // position
    float dx, dy, dz;   // direction
    float nx, ny, nz;   // current surface normal
    float xc, yc;       // centre of the current column
    float ex, ey, ez;   // event position (emission point)
    float dist;         // path length so far
    uint32_t rebound;   // boundary interactions so far
    int ii, jj;         // detection pixel (-1: outside the PRF bounds)
};

__device__ __forceinline__ void renorm(float &x, float &y, float &z)
{
    const float nrm = sqrtf(x * x + y * y + z * z);
    if (nrm < 1.0f - kEps || nrm > 1.0f + kEps) {
        const float inv = 1.0f / nrm;
        x *= inv; y *= inv; z *= inv;
    }
}

// Isotropic emission; the first photon of an event rejects |cos| <= 0.01
// (the reference's CPU driver, hybridMANTIS_c_ver1_0.c:257-262).
__device__ __forceinline__ void emit(Photon &p, PhotonRng &rng, bool first)
{
    float c = 2.0f * rng.u() - 1.0f;
    if (first) {
        for (int t = 0; t < 64 && fabsf(c) <= 0.01f; ++t) c = 2.0f * rng.u() - 1.0f;
    }
    const float rr = sqrtf(fmaxf(0.0f, 1.0f - c * c));
    float s, co;
    __sincosf(kPi * (2.0f * rng.u() - 1.0f), &s, &co);
    p.dx = rr * co;
    p.dy = rr * s;
    p.dz = c;
    renorm(p.dx, p.dy, p.dz);
}

// n <- normalize(n + beta * q), q the reference's perturbation vector:
// z = 2u1 - 1, transverse radius sqrt(1 - u1^2), uniform azimuth, then
// normalised (RoughSurface).
__device__ __forceinline__ void roughen(float &nx, float &ny, float &nz, PhotonRng &rng, float beta)
{
    const float u1 = rng.u();
    const float qz = 2.0f * u1 - 1.0f;
    const float rr = sqrtf(fmaxf(0.0f, 1.0f - u1 * u1));
    float s, c;
    __sincosf(kPi * (2.0f * rng.u() - 1.0f), &s, &c);
    const float qx = rr * c, qy = rr * s;
    const float iq = rsqrtf(qx * qx + qy * qy + qz * qz);
    const float rx = fmaf(beta * iq, qx, nx), ry = fmaf(beta * iq, qy, ny), rz = fmaf(beta * iq, qz, nz);
    const float ir = rsqrtf(rx * rx + ry * ry + rz * rz);
    nx = rx * ir; ny = ry * ir; nz = rz * ir;
}

__device__ __forceinline__ bool outside_detector(const Photon &p, const DevGeom &g)
{
    return p.px < kEps || p.px > g.xdet || p.py < kEps || p.py > g.ydet || p.pz < -g.half || p.pz > g.half;
}

__device__ __forceinline__ bool outside_xy(const Photon &p, const DevGeom &g)
{
    return p.px < kEps || p.px > g.xdet || p.py < kEps || p.py > g.ydet;
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

// Move to the column wall or the z plane ahead, then apply the reference's
// pull-back into the column (dist_to_surface).  Returns a fate or kAlive;
// *d receives the distance.
__device__ __forceinline__ int to_wall(Photon &p, const DevGeom &g, float *dout)
{
    if (p.rebound == 0) { p.xc = p.ex; p.yc = p.ey; }
    const float ddx = p.px - p.xc, ddy = p.py - p.yc;
    const float qa = p.dx * p.dx + p.dy * p.dy;
    const float qb = 2.0f * (ddx * p.dx + ddy * p.dy);
    const float qc = ddx * ddx + ddy * ddy - g.R * g.R;
    const float dcyl = wall_root(qa, qb, qc);
    float d;
    if (p.dz != 0.0f) {
        const float zp = p.dz > 0.0f ? g.half : -g.half;
        const float axis = p.dz > 0.0f ? 1.0f : -1.0f;
        const bool straight = fabsf(p.dx) < kEps && fabsf(p.dy) < kEps && fabsf(p.dz - axis) < kEps;
        const float dplane = (zp - p.pz) / p.dz;
        if (!straight && dplane >= dcyl) {
            d = dcyl;
            p.pz = fmaf(d, p.dz, p.pz);
        } else {
            d = dplane;
            p.pz = zp;
        }
    } else {
        d = dcyl;
    }
    p.px = fmaf(d, p.dx, p.px);
    p.py = fmaf(d, p.dy, p.py);
    if (outside_detector(p, g)) return kLost;
    const float thr = g.R - 1e-5f;
    float r = sqrtf((p.px - p.xc) * (p.px - p.xc) + (p.py - p.yc) * (p.py - p.yc));
    float step = 0.5f;
    int moved = 0, halved = 0;
    while (r > thr && moved < 10 && halved < 10) {
        const float sx = p.px, sy = p.py;
        p.px = fmaf(-step, p.dx, p.px);
        p.py = fmaf(-step, p.dy, p.py);
        const float r2 = sqrtf((p.px - p.xc) * (p.px - p.xc) + (p.py - p.yc) * (p.py - p.yc));
        if (r2 > r) {
            p.px = sx; p.py = sy;
            step *= 0.5f;
            ++halved;
        } else {
            r = r2;
            ++moved;
        }
    }
    if (r > thr) return kOutOfCol;
    if (outside_detector(p, g)) return kLost;
    *dout = d;
    return kAlive;
}

// Wall distance against exponential bulk absorption (isotropic).
__device__ __forceinline__ int flight(Photon &p, PhotonRng &rng, const DevGeom &g)
{
    float d = 0.0f;
    const int f = to_wall(p, g, &d);
    if (f != kAlive) return f;
    p.dist += d;
    if (g.neg_inv_mu != 0.0f) {
        const float dabs = g.neg_inv_mu * __logf(rng.u());
        if (d >= dabs && d >= 0.0f) return kAbsBulk;
    }
    return kAlive;
}

__device__ __forceinline__ void set_pixel(Photon &p, const DevGeom &g)
{
    p.ii = -1;
    p.jj = -1;
    if (p.px <= g.ub_x && p.py <= g.ub_y && p.px >= g.lb_x && p.py >= g.lb_y) {
        p.ii = (int)floorf(__fdiv_rn(p.px - g.lb_x, g.pixel));
        p.jj = (int)floorf(__fdiv_rn(p.py - g.lb_y, g.pixel));
    }
}

// Sensor plane inside a column (detection).
__device__ __forceinline__ int sensor(Photon &p, PhotonRng &rng, const DevGeom &g)
{
    if (fabsf(p.pz + g.half) >= kEps) return kAlive;
    if (g.sensor_refl > 0.0f && rng.u() < g.sensor_refl) {
        p.dz = -p.dz;  // specular reflection on the flat sensor, normal +z
        renorm(p.dx, p.dy, p.dz);
        return flight(p, rng, g);
    }
    set_pixel(p, g);
    return kDetect;
}

// Orientation of the next column: random normal within 1.57 rad of the
// reversed direction, flattened to the x-y plane, roughened.
__device__ __forceinline__ int next_column_normal(Photon &p, PhotonRng &rng, const DevGeom &g, float ix, float iy,
                                                  float iz, int &tries, bool always_rough)
{
    for (;;) {
        float nx = ix, ny = iy, nz = iz;
        roughen(nx, ny, nz, rng, 1.0f);
        const float inv = rsqrtf(nx * nx + ny * ny);
        nx *= inv; ny *= inv; nz = 0.0f;
        if (always_rough || g.beta > 0.0f) roughen(nx, ny, nz, rng, g.beta);
        p.nx = nx; p.ny = ny; p.nz = nz;
        if (!(ix * nx + iy * ny + iz * nz < kCos157)) return kAlive;
        if (tries < 100) { ++tries; continue; }
        return kTheta1;
    }
}

__device__ __forceinline__ bool at_top(const Photon &p, const DevGeom &g)
{
    return fabsf(p.pz - g.half) < kEps && p.dz > 0.0f;
}

// Hop after a sensor reflection between columns (refl_bottom).
__device__ __forceinline__ int hop_from_sensor(Photon &p, PhotonRng &rng, const DevGeom &g)
{
    const float sx = p.px, sy = p.py, sz = p.pz;
    const float ix = -p.dx, iy = -p.dy, iz = -p.dz;
    const float hop = fmaf(rng.u(), g.d_span, g.d_min);
    const float dtop = (g.half - sz) / p.dz;
    p.px = fmaf(p.dx, hop, sx);
    p.py = fmaf(p.dy, hop, sy);
    p.pz = fmaf(p.dz, hop, sz);
    if (outside_xy(p, g)) return kLost;
    if (p.pz > g.half) {
        if (dtop < hop && dtop > kEps) {
            p.px = fmaf(p.dx, dtop, sx);
            p.py = fmaf(p.dy, dtop, sy);
            p.pz = g.half;
            p.dist += dtop;
            return kAlive;
        }
        return kLost;
    }
    p.dist += hop;
    int tries = 0;
    return next_column_normal(p, rng, g, ix, iy, iz, tries, true);
}

// Sensor between columns: 0 alive, 1 = went back up to the top surface,
// or a fate (as -fate) when the photon ended.
__device__ __forceinline__ int sensor_between(Photon &p, PhotonRng &rng, const DevGeom &g)
{
    if (g.sensor_refl > 0.0f && rng.u() < g.sensor_refl) {
        p.dz = -p.dz;
        renorm(p.dx, p.dy, p.dz);
        const int f = hop_from_sensor(p, rng, g);
        if (f != kAlive) return -f;
        return at_top(p, g) ? 1 : 0;
    }
    set_pixel(p, g);
    return -kDetect;
}

// Leave the current column (transmit).
__device__ __noinline__ int leave_column(Photon &p, PhotonRng &rng, const DevGeom &g, bool crosstalk)
{
    float ix = -p.dx, iy = -p.dy, iz = -p.dz;
    int tries = 0, tries_top = 0;
    if (crosstalk) return next_column_normal(p, rng, g, ix, iy, iz, tries, false);

    float sx = p.px, sy = p.py, sz = p.pz;
    float hop = fmaf(rng.u(), g.d_span, g.d_min);
    p.px = fmaf(p.dx, hop, sx);
    p.py = fmaf(p.dy, hop, sy);
    p.pz = fmaf(p.dz, hop, sz);
    const float dtop = (g.half - sz) / p.dz;
    float dbot = (-g.half - sz) / p.dz;
    if (outside_xy(p, g)) return kLost;
    bool to_top = false;
    if (p.pz < -g.half || p.pz > g.half) {
        if (dtop < hop && dtop > kEps) {
            p.px = fmaf(p.dx, dtop, sx);
            p.py = fmaf(p.dy, dtop, sy);
            p.pz = g.half;
            p.dist += dtop;
        } else if (dbot < hop && dbot > kEps) {
            p.px = fmaf(p.dx, dbot, sx);
            p.py = fmaf(p.dy, dbot, sy);
            p.pz = -g.half;
            p.dist += dbot;
            const int s = sensor_between(p, rng, g);
            if (s < 0) return -s;
            to_top = (s == 1);
        } else {
            return kLost;
        }
    } else {
        p.dist += hop;
    }
    if (!to_top) {
        const int f = next_column_normal(p, rng, g, ix, iy, iz, tries, false);
        if (f != kAlive) return f;
        if (fabsf(p.px) < kEps || fabsf(p.px - g.xdet) < kEps || fabsf(p.py) < kEps || fabsf(p.py - g.ydet) < kEps)
            return kLost;
    }
    for (int loop = 0; loop < kMaxTopLoops; ++loop) {
        if (at_top(p, g)) {
            if (g.top_absfrac > 0.0f && rng.u() < g.top_absfrac) return kAbsTop;
            // isotropic reflection back down, then a hop
            p.dz = -fabsf(2.0f * rng.u() - 1.0f);
            const float rr = sqrtf(fmaxf(0.0f, 1.0f - p.dz * p.dz));
            float s, c;
            __sincosf(kPi * (2.0f * rng.u() - 1.0f), &s, &c);
            p.dx = rr * c;
            p.dy = rr * s;
            sx = p.px; sy = p.py; sz = p.pz;
            ix = -p.dx; iy = -p.dy; iz = -p.dz;
            hop = fmaf(rng.u(), g.d_span, g.d_min);
            dbot = (-g.half - sz) / p.dz;
            p.px = fmaf(p.dx, hop, sx);
            p.py = fmaf(p.dy, hop, sy);
            p.pz = fmaf(p.dz, hop, sz);
            if (outside_xy(p, g)) return kLost;
            if (p.pz < -g.half || p.pz > g.half) {
                if (dbot < hop && dbot > kEps) {
                    p.px = fmaf(p.dx, dbot, sx);
                    p.py = fmaf(p.dy, dbot, sy);
                    p.pz = -g.half;
                    p.dist += dbot;
                    const int s2 = sensor_between(p, rng, g);
                    if (s2 < 0) return -s2;
                    if (s2 == 1) continue;
                } else {
                    return kLost;
                }
            } else {
                p.dist += hop;
            }
            const int f = next_column_normal(p, rng, g, ix, iy, iz, tries_top, false);
            if (f != kAlive) return f;
        }
        if (fabsf(p.pz + g.half) < kEps) {
            const int s = sensor_between(p, rng, g);
            if (s < 0) return -s;
            if (s == 1) continue;
        }
        return kAlive;
    }
    return kCapped;
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

// Interaction with a surface (boundary_analysis).
__device__ __noinline__ int surface(Photon &p, PhotonRng &rng, const DevGeom &g)
{
    if (at_top(p, g)) {
        if (g.top_absfrac > 0.0f && rng.u() < g.top_absfrac) return kAbsTop;
        p.dz = -fabsf(2.0f * rng.u() - 1.0f);
        const float rr = sqrtf(fmaxf(0.0f, 1.0f - p.dz * p.dz));
        float s, c;
        __sincosf(kPi * (2.0f * rng.u() - 1.0f), &s, &c);
        p.dx = rr * c;
        p.dy = rr * s;
        return kAlive;
    }
    // columnar crosstalk: certain in the top 20 %, linear to 0.5 at mid depth,
    // back to 1 at the sensor
    float cct = 0.0f;
    if (p.pz <= g.half && p.pz >= g.cct_band_lo) cct = 1.0f;
    else if (p.pz < g.cct_band_lo && p.pz >= 0.0f) cct = fmaf(p.pz, g.cct_k_hi, 0.5f);
    else if (p.pz < 0.0f && p.pz >= -g.half) cct = fmaf(p.pz + g.half, g.cct_k_lo, 1.0f);
    if (rng.u() < cct) {
        const int f = leave_column(p, rng, g, true);
        if (f != kAlive) return f;
        p.xc = fmaf(-g.R, p.nx, p.px);
        p.yc = fmaf(-g.R, p.ny, p.py);
        return kAlive;
    }

    bool outside = false;
    int tries_theta = 0, tries_normal = 0, reperturbs = 0, smooth = 0;
    float pr = __int_as_float(0x7fc00000);  // 0/0 until a rule sets it
    float st = 0.0f, ct = 1.0f;            // sin, cos of the last refraction angle
    float kx = 0, ky = 0, kz = 0, kdx = 0, kdy = 0, kdz = 0;  // kept normal and direction
    enum { kNewSurface, kRestore, kIncidence } stage = kNewSurface;
    for (int loop = 0; loop < kMaxSurfaceLoops; ++loop) {
        if (stage == kNewSurface) {
            if (!outside) {
                const float ax = p.xc - p.px, ay = p.yc - p.py;
                const float im = rsqrtf(ax * ax + ay * ay);
                p.nx = ax * im; p.ny = ay * im; p.nz = 0.0f;
                if (g.beta > 0.0f) roughen(p.nx, p.ny, p.nz, rng, g.beta);
            } else {
                p.xc = fmaf(-g.R, p.nx, p.px);
                p.yc = fmaf(-g.R, p.ny, p.py);
            }
            kx = p.nx; ky = p.ny; kz = p.nz;
            kdx = p.dx; kdy = p.dy; kdz = p.dz;
            stage = kRestore;
        }
        if (stage == kRestore) {
            p.nx = kx; p.ny = ky; p.nz = kz;
            p.dx = kdx; p.dy = kdy; p.dz = kdz;
            if (reperturbs != 0) {
                if (g.beta > 0.0f) roughen(p.nx, p.ny, p.nz, rng, g.beta);
                if (outside) {
                    p.xc = fmaf(-g.R, p.nx, p.px);
                    p.yc = fmaf(-g.R, p.ny, p.py);
                }
            }
            stage = kIncidence;
        }
        const float c1 = -(p.dx * p.nx + p.dy * p.ny + p.dz * p.nz);
        if (c1 > 1.0f || c1 < 0.0f) {
            if (outside) {
                const int f = next_column_normal(p, rng, g, -p.dx, -p.dy, -p.dz, tries_normal, false);
                if (f != kAlive) return f;
            }
            if (tries_theta < 100) {
                ++tries_theta;
                stage = kNewSurface;
                continue;
            }
            return kTheta1;
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
        if (rng.u() < pr) {
            // specular reflection
            p.dx = fmaf(2.0f * c1, p.nx, p.dx);
            p.dy = fmaf(2.0f * c1, p.ny, p.dy);
            p.dz = fmaf(2.0f * c1, p.nz, p.dz);
            renorm(p.dx, p.dy, p.dz);
            if (kx * p.dx + ky * p.dy + kz * p.dz < kCos157) {
                if (++reperturbs < 4) {
                    stage = kRestore;
                    continue;
                }
                p.nx = kx; p.ny = ky; p.nz = kz;
                p.dx = kdx; p.dy = kdy; p.dz = kdz;
                reperturbs = 0;
                if (smooth < 25) {
                    ++smooth;
                    stage = kIncidence;
                    continue;
                }
                return kTheta1;
            }
            if (!outside) return kAlive;
            const int f = leave_column(p, rng, g, false);
            if (f != kAlive) return f;
            stage = kNewSurface;
            continue;
        }
        // refraction with the reference's formula
        const float ratio = si > 0.0f ? __fdividef(st, si) : 0.0f;
        const float tx = fmaf(c1, p.nx, p.dx), ty = fmaf(c1, p.ny, p.dy), tz = fmaf(c1, p.nz, p.dz);
        p.dx = -ct * p.nx - ratio * tx;
        p.dy = -ct * p.ny - ratio * ty;
        p.dz = -ct * p.nz - ratio * tz;
        renorm(p.dx, p.dy, p.dz);
        if (outside) return kAlive;
        outside = true;
        const int f = leave_column(p, rng, g, false);
        if (f != kAlive) return f;
        stage = kNewSurface;
    }
    return kCapped;
}

// Start photon k of an event at its emission point.
__device__ __forceinline__ void start_photon(Photon &p, PhotonRng &rng, bool first)
{
    p.px = p.ex; p.py = p.ey; p.pz = p.ez;
    p.xc = p.ex; p.yc = p.ey;
    p.nx = 0.0f; p.ny = 0.0f; p.nz = 0.0f;
    p.dist = 0.0f;
    p.rebound = 0;
    p.ii = -1; p.jj = -1;
    emit(p, rng, first);
}

// One transport step (the body of the reference's step function algo):
// flight, sensor, trapped-photon restart, or a surface interaction.
// Returns the photon's fate, kAlive while it is in flight.
__device__ __forceinline__ int step(Photon &p, PhotonRng &rng, const DevGeom &g)
{
    int f = flight(p, rng, g);
    if (f != kAlive) return f;
    f = sensor(p, rng, g);
    if (f != kAlive) return f;
    if (fabsf(p.dz) < kEps) {
        // trapped travelling horizontally: restart from the event position,
        // keeping the current column (the reference does not reset it)
        p.px = p.ex; p.py = p.ey; p.pz = p.ez;
        emit(p, rng, false);
        return kAlive;
    }
    if (++p.rebound > kMaxBoundaryCalls) return kCapped;
    return surface(p, rng, g);
}

}  // namespace fd2
