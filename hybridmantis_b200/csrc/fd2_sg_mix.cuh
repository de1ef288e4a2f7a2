// fd2_sg_mix.cuh -- the surrogate's radial model: a mixture of Gaussian rings.
//
// The detected photons' 2D density around their deposition is modelled as
//   PRF(r) = sum_k w_k N(r; mu_k, sd_k) / S_k        (per unit area, r >= 0)
// i.e. each component is a ring of radius mu_k >= 0 and width sd_k (mu = 0:
// an isotropic 2D Gaussian), so the radial density of component k is
//   f_k(r) = r N(r; mu, sd) / S_k,
//   S_k = int_0^inf r N(r; mu, sd) dr = mu Phi_c(t0) + sd phi(t0),  t0 = -mu / sd.
// Its mass on [a, b) has the closed form
//   M(a, b) = mu [Phi(t_b) - Phi(t_a)] + sd [phi(t_a) - phi(t_b)],  t = (r - mu) / sd,
// with derivatives
//   dM/dmu = [Phi(t_b) - Phi(t_a)] + (a phi(t_a) - b phi(t_b)) / sd
//   dM/dsd = [phi(t_a) - phi(t_b)] + (t_a a phi(t_a) - t_b b phi(t_b)) / sd.
// CDF differences use lower tails left of the mean and upper tails right of
// it, so far-tail bins keep their relative accuracy in FP32.
#pragma once

#include <cuda_runtime.h>

#include "fd2_sg_internal.h"

namespace fd2 {
namespace sg {

struct Mix {
    float w[kComponents], mu[kComponents], dmu[kComponents], sd[kComponents], S[kComponents];
    float dS_mu[kComponents], dS_sd[kComponents];
    bool clamped[kComponents];
};

__device__ __forceinline__ float norm_pdf(float a) { return 0.3989422804014327f * expf(-0.5f * a * a); }

// Values of one bin edge for one component; `inf` marks the edge at +inf.
struct Edge {
    float t, cdf, ccdf, pdf, e;
    bool inf;
};

__device__ __forceinline__ Edge edge_at(float e, bool inf, float mu, float sd)
{
    Edge x;
    x.e = e;
    x.inf = inf;
    if (inf) {
        x.t = 0.0f;
        x.cdf = 1.0f;
        x.ccdf = 0.0f;
        x.pdf = 0.0f;
    } else {
        x.t = (e - mu) / sd;
        x.cdf = normcdff(x.t);
        x.ccdf = normcdff(-x.t);
        x.pdf = norm_pdf(x.t);
    }
    return x;
}

// Mass of a ring component between two edges, and its derivatives.
__device__ __forceinline__ float ring_mass(const Edge &lo, const Edge &hi, float mu, float sd, float *dmu, float *dsd)
{
    const float dphi = fmaxf(lo.t >= 0.0f && !lo.inf ? lo.ccdf - hi.ccdf : hi.cdf - lo.cdf, 0.0f);
    const float m = fmaxf(mu * dphi + sd * (lo.pdf - hi.pdf), 0.0f);
    if (dmu) {
        const float ehi = hi.inf ? 0.0f : hi.e * hi.pdf;
        const float thi = hi.inf ? 0.0f : hi.t * hi.e * hi.pdf;
        *dmu = dphi + (lo.e * lo.pdf - ehi) / sd;
        *dsd = (lo.pdf - hi.pdf) + (lo.t * lo.e * lo.pdf - thi) / sd;
    }
    return m;
}

// Decode the network's mixture outputs (o[1..24]) and each ring's normaliser.
__device__ __forceinline__ void decode_mix(const float *o, Mix &m)
{
    float amax = o[1];
#pragma unroll
    for (int k = 1; k < kComponents; ++k) amax = fmaxf(amax, o[1 + k]);
    float s = 0.0f;
#pragma unroll
    for (int k = 0; k < kComponents; ++k) {
        m.w[k] = expf(o[1 + k] - amax);
        s += m.w[k];
    }
#pragma unroll
    for (int k = 0; k < kComponents; ++k) {
        m.w[k] /= s;
        const float om = o[1 + kComponents + k];
        m.mu[k] = kMuScale * (fmaxf(om, 0.0f) + log1pf(expf(-fabsf(om))));  // softplus
        m.dmu[k] = kMuScale / (1.0f + expf(-om));                           // d mu / d output
        const float ls = o[1 + 2 * kComponents + k];
        m.clamped[k] = ls < kLogSdMin || ls > kLogSdMax;
        m.sd[k] = kSdScale * expf(fminf(fmaxf(ls, kLogSdMin), kLogSdMax));
        const float t0 = -m.mu[k] / m.sd[k];
        const float c0 = normcdff(-t0), p0 = norm_pdf(t0);
        m.S[k] = fmaxf(m.mu[k] * c0 + m.sd[k] * p0, 1e-30f);
        m.dS_mu[k] = c0;
        m.dS_sd[k] = p0;
    }
}

// Probability of radial category j (0..bins; bins = beyond r_max).
__device__ __forceinline__ float bin_prob(const Mix &m, int j, int bins, float r_max)
{
    const float e_lo = radial_edge(j, bins, r_max);
    const bool top = j >= bins;
    const float e_hi = top ? 0.0f : radial_edge(j + 1, bins, r_max);
    float q = 0.0f;
#pragma unroll
    for (int k = 0; k < kComponents; ++k) {
        const Edge lo = edge_at(e_lo, false, m.mu[k], m.sd[k]);
        const Edge hi = edge_at(e_hi, top, m.mu[k], m.sd[k]);
        q += m.w[k] * ring_mass(lo, hi, m.mu[k], m.sd[k], nullptr, nullptr) / m.S[k];
    }
    return q;
}

}  // namespace sg
}  // namespace fd2
