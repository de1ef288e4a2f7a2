// fd2_xray.cu -- the x-ray front end on the GPU: one thread per x-ray
// history (FP64), EDEs compacted in history order, and the C ABI of
// include/fd2_xray.h.
//
// What it replaces: PENELOPE's photon and electron transport driven by
// penEasy (main/hybridMANTIS_penEasy.f, sources of PENELOPE itself not in the
// reference tree) with the BIGS source (main/sourceBoxIsotropicGaussSpectrum.f)
// and the EDE tally (main/hybridMANTIS_tallyEnergyDepositionEvents.f:155-200).
// The physics model is the one stated in include/fd2_xray.h; the oracle
// (oracle/xray_oracle.c) restates it on the CPU with the same random stream.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "fd2_internal.h"
#include "fd2_xray_internal.h"

namespace fd2x {

constexpr int kStack = 16;      // pending photons per history
constexpr int kVacancies = 16;  // pending vacancies per relaxation cascade
constexpr int kMaxTransitions = 64;
constexpr uint32_t kStreamHistory = 0x58524159u;  // counter word 3 of a history's stream
constexpr uint32_t kStreamSample = 0x534D504Cu;   // counter word 3 of fd2_xray_sample

// Device view of one material and the run's geometry and options.
struct XDev {
    int n_nodes, n_el, stride;  // stride = 3 + n_el (1 + kShells)
    const double *e;            // photon node energies
    const double *lnv;          // [node][stride]: ln mu_R, ln mu_C, ln b, per element ln mu_pe, ln mu_shell[9]
    int n_e;
    const double *ee, *lnee, *lnr, *lnl1;  // electron nodes: E, ln E, ln range, ln lambda1
    const double *binding;                 // [element][kDesignators]
    const int *toff;                       // [element][kDesignators + 1] transition offsets by vacancy shell
    const int *ts;                         // [transition]: s1 | s2 << 8
    const double *tcum, *te;               // cumulative probability within the vacancy shell, energy
    double X, Y, H2;                       // slab (cm)
    double eabs_e, eabs_ph, loss, local_e;  // local_e = max(eabs_e, electron_local_ev)
    int fluo, cap;
    uint32_t k0, k1;
};

struct XSource {
    int particle, nspec, gaussian, point;
    const double *espc, *pcum, *despc;
    double gmean, gsig, gmin, gmax;
    double ctr[3], side[3], rot[9], dir[3], cossrc;
};

struct Ede {
    double x, y, z, de;
};

struct HistInfo {
    double e0, esc_ph, esc_el, first_depth;
    int n_edes, first_kind, merged, missed;
    int n_pe, n_co, n_ra, n_fe, n_fesc, n_aug, n_steps, pad;
};

// ------------------------------------------------------------ random stream

// Philox-4x32-10 (Salmon et al., SC'11), the generator of the optical walk.
__device__ __forceinline__ uint4 philox(uint4 c, uint32_t k0, uint32_t k1)
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

struct XRng {
    uint4 ctr;
    uint32_t k0, k1;
    double buf[2];
    int left;
    __device__ XRng(uint32_t a, uint32_t b, uint64_t index, uint32_t stream)
        : ctr(make_uint4(0u, (uint32_t)index, (uint32_t)(index >> 32), stream)), k0(a), k1(b), left(0)
    {
    }
    // Uniform in (0, 1): 53 bits of a Philox word pair, (k + 1/2) 2^-53.
    __device__ double u()
    {
        if (left == 0) {
            const uint4 r = philox(ctr, k0, k1);
            ctr.x++;
            buf[0] = to_u(r.x, r.y);
            buf[1] = to_u(r.z, r.w);
            left = 2;
        }
        return buf[2 - left--];
    }
    static __device__ double to_u(uint32_t a, uint32_t b)
    {
        const unsigned long long k = ((unsigned long long)(a >> 5) << 26) | (unsigned long long)(b >> 6);
        return ((double)k + 0.5) * 1.1102230246251565404e-16;  // 2^-53
    }
};

// ------------------------------------------------------------ geometry

__device__ double dist_exit(const XDev &g, const double *p, const double *d)
{
    double t = 1e300;
    if (d[0] > 0) t = fmin(t, (g.X - p[0]) / d[0]);
    else if (d[0] < 0) t = fmin(t, -p[0] / d[0]);
    if (d[1] > 0) t = fmin(t, (g.Y - p[1]) / d[1]);
    else if (d[1] < 0) t = fmin(t, -p[1] / d[1]);
    if (d[2] > 0) t = fmin(t, (g.H2 - p[2]) / d[2]);
    else if (d[2] < 0) t = fmin(t, (-g.H2 - p[2]) / d[2]);
    return fmax(t, 0.0);
}

// Move a particle outside the slab onto it along its direction; false if
// the line misses the slab (or points away from it).
__device__ bool enter(const XDev &g, double *p, const double *d)
{
    const double lo[3] = {0.0, 0.0, -g.H2}, hi[3] = {g.X, g.Y, g.H2};
    bool in = true;
    for (int a = 0; a < 3; ++a) in = in && p[a] >= lo[a] && p[a] <= hi[a];
    if (in) return true;
    double t0 = 0.0, t1 = 1e300;
    for (int a = 0; a < 3; ++a) {
        if (d[a] == 0.0) {
            if (p[a] < lo[a] || p[a] > hi[a]) return false;
            continue;
        }
        double ta = (lo[a] - p[a]) / d[a], tb = (hi[a] - p[a]) / d[a];
        if (ta > tb) {
            const double s = ta;
            ta = tb;
            tb = s;
        }
        t0 = fmax(t0, ta);
        t1 = fmin(t1, tb);
    }
    if (!(t0 < t1)) return false;
    for (int a = 0; a < 3; ++a) p[a] += t0 * d[a];
    for (int a = 0; a < 3; ++a) p[a] = fmin(fmax(p[a], lo[a]), hi[a]);
    return true;
}

// Turn direction d by polar angle acos(c) and azimuth phi.
__device__ void rotate(double *d, double c, double phi)
{
    c = fmin(fmax(c, -1.0), 1.0);
    const double s = sqrt(fmax(0.0, 1.0 - c * c));
    double sp, cp;
    sincos(phi, &sp, &cp);
    const double k2 = d[0] * d[0] + d[1] * d[1];
    double nx, ny, nz;
    if (k2 > 1e-20) {
        const double k = sqrt(k2);
        nx = d[0] * c + s * (d[0] * d[2] * cp - d[1] * sp) / k;
        ny = d[1] * c + s * (d[1] * d[2] * cp + d[0] * sp) / k;
        nz = d[2] * c - k * s * cp;
    } else {
        const double sg = d[2] >= 0 ? 1.0 : -1.0;
        nx = s * cp;
        ny = s * sp;
        nz = sg * c;
    }
    const double n = 1.0 / sqrt(nx * nx + ny * ny + nz * nz);
    d[0] = nx * n;
    d[1] = ny * n;
    d[2] = nz * n;
}

__device__ void isotropic(XRng &r, double *d)
{
    const double c = 2.0 * r.u() - 1.0;
    const double phi = 2.0 * M_PI * r.u();
    const double s = sqrt(fmax(0.0, 1.0 - c * c));
    double sp, cp;
    sincos(phi, &sp, &cp);
    d[0] = s * cp;
    d[1] = s * sp;
    d[2] = c;
}

// ------------------------------------------------------------ tables

// Photon node interval k (e[k] <= E < e[k+1], never an edge's zero-width
// interval) and log-log weight.
__device__ void photon_interval(const XDev &g, double E, int &k, double &w)
{
    const int n = g.n_nodes;
    if (E <= g.e[0]) {
        k = 0;
        w = 0.0;
        return;
    }
    if (E >= g.e[n - 1]) {
        k = n - 2;
        w = 1.0;
        return;
    }
    int lo = 0, hi = n - 1;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (g.e[mid] <= E) lo = mid;
        else hi = mid;
    }
    k = lo;
    w = log(E / g.e[lo]) / log(g.e[lo + 1] / g.e[lo]);
}

__device__ double pval(const XDev &g, int k, double w, int col)
{
    const double a = g.lnv[k * g.stride + col], b = g.lnv[(k + 1) * g.stride + col];
    return exp(a + w * (b - a));
}

__device__ double e_range(const XDev &g, double E)
{
    if (E <= g.ee[0]) return exp(g.lnr[0]) * E / g.ee[0];
    int lo = 0, hi = g.n_e - 1;
    if (E >= g.ee[hi]) lo = hi - 1;
    else
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (g.ee[mid] <= E) lo = mid;
            else hi = mid;
        }
    const double w = (log(E) - g.lnee[lo]) / (g.lnee[lo + 1] - g.lnee[lo]);
    return exp(g.lnr[lo] + w * (g.lnr[lo + 1] - g.lnr[lo]));
}

__device__ double e_lambda1(const XDev &g, double E)
{
    if (E <= g.ee[0]) return exp(g.lnl1[0]);
    int lo = 0, hi = g.n_e - 1;
    if (E >= g.ee[hi]) lo = hi - 1;
    else
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (g.ee[mid] <= E) lo = mid;
            else hi = mid;
        }
    const double w = (log(E) - g.lnee[lo]) / (g.lnee[lo + 1] - g.lnee[lo]);
    return exp(g.lnl1[lo] + w * (g.lnl1[lo + 1] - g.lnl1[lo]));
}

// Energy whose CSDA range is R (inverse of e_range).
__device__ double e_of_range(const XDev &g, double R)
{
    const double r0 = exp(g.lnr[0]);
    if (R <= 0.0) return 0.0;
    if (R <= r0) return g.ee[0] * R / r0;
    const double lr = log(R);
    int lo = 0, hi = g.n_e - 1;
    if (lr >= g.lnr[hi]) lo = hi - 1;
    else
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (g.lnr[mid] <= lr) lo = mid;
            else hi = mid;
        }
    const double w = (lr - g.lnr[lo]) / (g.lnr[lo + 1] - g.lnr[lo]);
    return exp(g.lnee[lo] + w * (g.lnee[lo + 1] - g.lnee[lo]));
}

// ------------------------------------------------------------ samplers

// Klein-Nishina: E'/E by the two-branch composition of 1/eps and eps
// densities with rejection on the remaining factor (Butcher & Messel, 1960).
__device__ double sample_kn(XRng &r, double E)
{
    const double kappa = E / kElectronMass;
    const double e0 = 1.0 / (1.0 + 2.0 * kappa);
    const double a1 = log1p(2.0 * kappa), a2 = 0.5 * (1.0 - e0 * e0);
    for (;;) {
        double eps;
        if (r.u() * (a1 + a2) < a1) eps = exp(-a1 * r.u());
        else eps = sqrt(e0 * e0 + (1.0 - e0 * e0) * r.u());
        const double t = (1.0 - eps) / (kappa * eps);
        const double s2 = fmax(0.0, t * (2.0 - t));
        if (r.u() * (1.0 + eps * eps) <= 1.0 + eps * eps - eps * s2) return eps;
    }
}

// Rayleigh: cos(theta) from (1 + mu^2) (1 + b (1 - mu))^-4: t = 1 - mu from
// the screening factor by inversion, accepted with (1 + mu^2) / 2.
__device__ double sample_rayleigh(XRng &r, double b)
{
    for (;;) {
        const double u = r.u();
        double t;
        if (b < 1e-6) t = 2.0 * u;
        else {
            const double c = -expm1(-3.0 * log1p(2.0 * b));  // 1 - (1 + 2b)^-3
            t = expm1(-log1p(-u * c) / 3.0) / b;
        }
        t = fmin(fmax(t, 0.0), 2.0);
        const double mu = 1.0 - t;
        if (2.0 * r.u() <= 1.0 + mu * mu) return mu;
    }
}

// Sauter K-shell photoelectron: cos(theta) from
// (1 - mu^2) / nu^4 (1 + c nu), nu = 1 - beta mu, c = gamma (gamma-1) (gamma-2) / 2:
// nu from the nu^-4 density by inversion, accepted with the rest.
__device__ double sample_sauter(XRng &r, double T)
{
    const double gam = 1.0 + T / kElectronMass;
    const double beta = sqrt(fmax(0.0, 1.0 - 1.0 / (gam * gam)));
    const double c = 0.5 * gam * (gam - 1.0) * (gam - 2.0);
    if (beta < 1e-6) {
        for (;;) {
            const double mu = 2.0 * r.u() - 1.0;
            if (r.u() <= 1.0 - mu * mu) return mu;
        }
    }
    const double a = 1.0 / ((1.0 - beta) * (1.0 - beta) * (1.0 - beta));
    const double b = 1.0 / ((1.0 + beta) * (1.0 + beta) * (1.0 + beta));
    const double K = 1.0 + fmax(c, 0.0) * (1.0 + beta);
    for (;;) {
        const double nu = 1.0 / cbrt(a - r.u() * (a - b));
        const double mu = fmin(fmax((1.0 - nu) / beta, -1.0), 1.0);
        if (r.u() * K <= (1.0 - mu * mu) * (1.0 + c * nu)) return mu;
    }
}

// Condensed-step deflection: xi = (1 - cos) / 2 ~ Beta(1, 1/m - 1) with mean
// m = (1 - exp(-s / lambda1)) / 2 (the Goudsmit-Saunderson first moment).
__device__ double sample_deflection(XRng &r, double s, double lambda1)
{
    const double m = -0.5 * expm1(-s / lambda1);
    const double u = r.u();
    if (m >= 0.5 - 1e-12) return 1.0 - 2.0 * u;
    const double bb = 1.0 / m - 1.0;
    const double xi = -expm1(log(u) / bb);
    return 1.0 - 2.0 * xi;
}

// ------------------------------------------------------------ a history

struct Photon {
    double e, p[3], d[3];
    int fluo;
};

struct History {
    const XDev &g;
    XRng &r;
    Ede *slots;
    HistInfo &h;

    __device__ void deposit(double de, const double *q)
    {
        if (!(de > 0.0)) return;
        if (h.n_edes < g.cap) {
            slots[h.n_edes] = Ede{q[0], q[1], q[2], de};
            ++h.n_edes;
        } else {
            slots[g.cap - 1].de += de;
            h.merged = 1;
        }
    }

    // Continuous slowing down in condensed steps.
    __device__ void electron(double T, const double *p0, const double *d0)
    {
        double p[3] = {p0[0], p0[1], p0[2]}, d[3] = {d0[0], d0[1], d0[2]};
        for (;;) {
            if (T <= g.local_e) {
                deposit(T, p);
                return;
            }
            double Tn = T * (1.0 - g.loss);
            if (Tn < g.eabs_e) Tn = 0.0;
            const double R = e_range(g, T);
            const double Rn = Tn > 0.0 ? e_range(g, Tn) : 0.0;
            const double s = R - Rn;
            const double t = dist_exit(g, p, d);
            ++h.n_steps;
            if (s > t) {
                const double Tx = e_of_range(g, R - t);
                const double hh = r.u() * t;
                const double q[3] = {p[0] + hh * d[0], p[1] + hh * d[1], p[2] + hh * d[2]};
                deposit(T - Tx, q);
                h.esc_el += Tx;
                return;
            }
            const double hh = r.u() * s;
            const double q[3] = {p[0] + hh * d[0], p[1] + hh * d[1], p[2] + hh * d[2]};
            deposit(T - Tn, q);
            for (int a = 0; a < 3; ++a) p[a] += s * d[a];
            if (Tn == 0.0) return;
            const double c = sample_deflection(r, s, e_lambda1(g, 0.5 * (T + Tn)));
            rotate(d, c, 2.0 * M_PI * r.u());
            T = Tn;
        }
    }

    // Relaxation of a vacancy in shell `shell` of element `el` holding U.
    __device__ void relax(int el, int shell, double U, const double *p, Photon *stack, int &ns)
    {
        double local = U;
        if (g.fluo && shell > 0) {
            int v[kVacancies];
            int nv = 0, steps = 0;
            v[nv++] = shell;
            while (nv > 0 && steps < kMaxTransitions) {
                const int s0 = v[--nv];
                const int a = g.toff[el * (kDesignators + 1) + s0], b = g.toff[el * (kDesignators + 1) + s0 + 1];
                if (a == b) continue;
                const double x = r.u();
                int j = a;
                while (j < b - 1 && g.tcum[j] <= x) ++j;
                ++steps;
                const double Et = fmin(g.te[j], local);
                const int s1 = g.ts[j] & 0xFF, s2 = g.ts[j] >> 8;
                if (s2 == 0) {
                    if (Et > g.eabs_ph && ns < kStack) {
                        Photon &f = stack[ns++];
                        f.e = Et;
                        f.p[0] = p[0];
                        f.p[1] = p[1];
                        f.p[2] = p[2];
                        isotropic(r, f.d);
                        f.fluo = 1;
                        ++h.n_fe;
                        local -= Et;
                    }
                    if (nv < kVacancies) v[nv++] = s1;
                } else {
                    if (Et > g.eabs_e) {
                        double d[3];
                        isotropic(r, d);
                        ++h.n_aug;
                        local -= Et;
                        electron(Et, p, d);
                    }
                    if (nv < kVacancies - 1) {
                        v[nv++] = s1;
                        v[nv++] = s2;
                    }
                }
            }
        }
        deposit(local, p);
    }

    __device__ void photon(Photon ph, Photon *stack, int &ns)
    {
        double E = ph.e, p[3] = {ph.p[0], ph.p[1], ph.p[2]}, d[3] = {ph.d[0], ph.d[1], ph.d[2]};
        const int nel = g.n_el;
        for (;;) {
            if (E < g.eabs_ph) {
                deposit(E, p);
                return;
            }
            int k;
            double w;
            photon_interval(g, E, k, w);
            const double muR = pval(g, k, w, 0), muC = pval(g, k, w, 1);
            double mupe[FD2_XRAY_MAX_ELEMENTS];
            double mu = muR + muC;
            for (int e = 0; e < nel; ++e) {
                mupe[e] = pval(g, k, w, 3 + e * (1 + kShells));
                mu += mupe[e];
            }
            const double s = -log(r.u()) / mu;
            const double t = dist_exit(g, p, d);
            if (s >= t) {
                h.esc_ph += E;
                if (ph.fluo) ++h.n_fesc;
                return;
            }
            for (int a = 0; a < 3; ++a) p[a] += s * d[a];
            double x = r.u() * mu;
            const int kind = x < muR ? 1 : x < muR + muC ? 2 : 3;
            if (h.first_kind == 0) {
                h.first_kind = kind;
                h.first_depth = g.H2 - p[2];
            }
            if (kind == 1) {
                ++h.n_ra;
                const double c = sample_rayleigh(r, pval(g, k, w, 2));
                rotate(d, c, 2.0 * M_PI * r.u());
                continue;
            }
            if (kind == 2) {
                ++h.n_co;
                const double eps = sample_kn(r, E);
                const double c = 1.0 - (1.0 - eps) / (eps * (E / kElectronMass));
                double dn[3] = {d[0], d[1], d[2]};
                rotate(dn, c, 2.0 * M_PI * r.u());
                const double En = eps * E, Te = E - En;
                double pe[3] = {E * d[0] - En * dn[0], E * d[1] - En * dn[1], E * d[2] - En * dn[2]};
                const double nn = sqrt(pe[0] * pe[0] + pe[1] * pe[1] + pe[2] * pe[2]);
                if (nn > 0.0)
                    for (int a = 0; a < 3; ++a) pe[a] /= nn;
                else
                    for (int a = 0; a < 3; ++a) pe[a] = d[a];
                electron(Te, p, pe);
                E = En;
                for (int a = 0; a < 3; ++a) d[a] = dn[a];
                continue;
            }
            // photoelectric: element, then subshell
            ++h.n_pe;
            x -= muR + muC;
            int el = nel - 1;
            for (int e = 0; e < nel - 1; ++e) {
                if (x < mupe[e]) {
                    el = e;
                    break;
                }
                x -= mupe[e];
            }
            double y = r.u() * mupe[el];
            int shell = 0;
            for (int q = 0; q < kShells; ++q) {
                const double sq = pval(g, k, w, 3 + el * (1 + kShells) + 1 + q);
                if (y < sq) {
                    shell = q + 1;
                    break;
                }
                y -= sq;
            }
            double U = shell ? g.binding[el * kDesignators + shell] : 0.0;
            if (!(U > 0.0)) {
                shell = 0;
                U = 0.0;
            }
            U = fmin(U, E);
            const double T = E - U;
            double de[3] = {d[0], d[1], d[2]};
            const double c = sample_sauter(r, T);
            rotate(de, c, 2.0 * M_PI * r.u());
            electron(T, p, de);
            relax(el, shell, U, p, stack, ns);
            return;
        }
    }
};

__device__ void source_particle(const XSource &src, XRng &r, double *p, double *d, double &E)
{
    d[0] = src.dir[0];
    d[1] = src.dir[1];
    d[2] = src.dir[2];
    const double c = src.cossrc + (1.0 - src.cossrc) * r.u();
    rotate(d, c, 2.0 * M_PI * r.u());
    if (src.point) {
        p[0] = src.ctr[0];
        p[1] = src.ctr[1];
        p[2] = src.ctr[2];
    } else {
        const double l[3] = {src.side[0] * (r.u() - 0.5), src.side[1] * (r.u() - 0.5), src.side[2] * (r.u() - 0.5)};
        for (int a = 0; a < 3; ++a)
            p[a] = src.rot[3 * a] * l[0] + src.rot[3 * a + 1] * l[1] + src.rot[3 * a + 2] * l[2] + src.ctr[a];
    }
    if (src.gaussian) {
        for (;;) {
            const double a = sqrt(-2.0 * log(r.u()));
            E = src.gmean + src.gsig * a * sin(2.0 * M_PI * r.u());
            if (E > src.gmin && E < src.gmax) break;
        }
    } else {
        const double x = r.u();
        int lo = 0, hi = src.nspec - 1;  // pcum[0] = 0 <= x < pcum[nspec-1] = 1
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (src.pcum[mid] <= x) lo = mid;
            else hi = mid;
        }
        E = src.espc[lo] + (x - src.pcum[lo]) * src.despc[lo];
    }
}

// History i of the batch (x-ray first + i): its EDEs into its slots, its
// record into info[i].
__device__ __forceinline__ void one_history(const XDev &g, const XSource &src, int64_t first, int64_t i, Ede *slots,
                                            HistInfo *info)
{
    XRng r(g.k0, g.k1, (uint64_t)(first + i), kStreamHistory);
    HistInfo h{};
    h.first_depth = -1.0;
    double p[3], d[3], E;
    source_particle(src, r, p, d, E);
    h.e0 = E;
    History H{g, r, slots + i * (int64_t)g.cap, h};
    if (!enter(g, p, d)) {
        h.missed = 1;
        h.esc_ph = src.particle == FD2_XRAY_PHOTON ? E : 0.0;
        h.esc_el = src.particle == FD2_XRAY_PHOTON ? 0.0 : E;
        info[i] = h;
        return;
    }
    if (src.particle == FD2_XRAY_ELECTRON) {
        H.electron(E, p, d);
    } else {
        Photon stack[kStack];
        int ns = 0;
        Photon first_ph;
        first_ph.e = E;
        for (int a = 0; a < 3; ++a) {
            first_ph.p[a] = p[a];
            first_ph.d[a] = d[a];
        }
        first_ph.fluo = 0;
        H.photon(first_ph, stack, ns);
        while (ns > 0) {
            const Photon f = stack[--ns];
            H.photon(f, stack, ns);
        }
    }
    info[i] = h;
}

// Each thread takes histories from a counter (*next, zero at launch) until
// the batch is done: histories differ in length by orders of magnitude
// (fluorescence, electrons), and one history per thread kept blocks
// resident for their longest history while most of their threads idled.
// A history's random numbers and outputs depend only on its index.
__global__ void __launch_bounds__(128) history_kernel(XDev g, XSource src, int64_t first, int64_t n, Ede *slots,
                                                      HistInfo *info, unsigned long long *next)
{
    for (;;) {
        const int64_t i = (int64_t)atomicAdd(next, 1ull);
        if (i >= n) return;
        one_history(g, src, first, i, slots, info);
    }
}

// EDE counts of a batch for the scan.
__global__ void count_kernel(const HistInfo *info, int64_t n, uint32_t *counts)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) counts[i] = (uint32_t)info[i].n_edes;
}

struct Totals {
    unsigned long long missed, edes, merged, pe, co, ra, fe, fesc, aug, steps;
    double e0, dep, esc_ph, esc_el;
};

__global__ void scatter_kernel(const HistInfo *info, const Ede *slots, int cap, int64_t n, int64_t first,
                               const unsigned long long *offsets, int64_t base, double *ox, double *oy, double *oz,
                               double *ode, int32_t *ohist, Totals *tot)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    double dep = 0.0;
    HistInfo h{};
    if (i < n) {
        h = info[i];
        const int64_t o = base + (int64_t)offsets[i];
        const Ede *s = slots + i * (int64_t)cap;
        for (int k = 0; k < h.n_edes; ++k) {
            const Ede e = s[k];
            ox[o + k] = e.x;
            oy[o + k] = e.y;
            oz[o + k] = e.z;
            ode[o + k] = e.de;
            ohist[o + k] = (int32_t)(first + i + 1);
            dep += e.de;
        }
    }
    // warp sums, one atomic per warp and field
    unsigned long long v[10] = {(unsigned long long)h.missed, (unsigned long long)h.n_edes,
                                (unsigned long long)h.merged, (unsigned long long)h.n_pe,
                                (unsigned long long)h.n_co,   (unsigned long long)h.n_ra,
                                (unsigned long long)h.n_fe,   (unsigned long long)h.n_fesc,
                                (unsigned long long)h.n_aug,  (unsigned long long)h.n_steps};
    double f[4] = {h.e0, dep, h.esc_ph, h.esc_el};
    for (int off = 16; off > 0; off >>= 1) {
        for (int q = 0; q < 10; ++q) v[q] += __shfl_down_sync(0xFFFFFFFFu, v[q], off);
        for (int q = 0; q < 4; ++q) f[q] += __shfl_down_sync(0xFFFFFFFFu, f[q], off);
    }
    if ((threadIdx.x & 31) == 0) {
        unsigned long long *tv = &tot->missed;
        for (int q = 0; q < 10; ++q)
            if (v[q]) atomicAdd(tv + q, v[q]);
        double *tf = &tot->e0;
        for (int q = 0; q < 4; ++q)
            if (f[q] != 0.0) atomicAdd(tf + q, f[q]);
    }
}

__global__ void sample_kernel(XDev g, int which, double E, double param, int64_t n, uint32_t k0, uint32_t k1,
                              double *out)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    XRng r(k0, k1, (uint64_t)i, kStreamSample);
    double v = 0.0;
    if (which == 0) v = sample_kn(r, E);
    else if (which == 1) {
        int k;
        double w;
        photon_interval(g, E, k, w);
        v = sample_rayleigh(r, pval(g, k, w, 2));
    } else if (which == 2) v = sample_sauter(r, E);
    else v = sample_deflection(r, param, e_lambda1(g, E));
    out[i] = v;
}

}  // namespace fd2x

namespace fd2 {

__global__ void event_sums_kernel(int64_t n, const double *x, const double *y, const double *de, double *out)
{
    double a = 0, b = 0, c = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        a += (double)(float)(x[i] * (double)10000.0f);
        b += (double)(float)(y[i] * (double)10000.0f);
        if (de[i] > 0.0) c += de[i];
    }
    for (int off = 16; off > 0; off >>= 1) {
        a += __shfl_down_sync(0xFFFFFFFFu, a, off);
        b += __shfl_down_sync(0xFFFFFFFFu, b, off);
        c += __shfl_down_sync(0xFFFFFFFFu, c, off);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(out, a);
        atomicAdd(out + 1, b);
        atomicAdd(out + 2, c);
    }
}

cudaError_t launch_event_sums(cudaStream_t s, int64_t n, const double *x_cm, const double *y_cm, const double *de,
                              double *out)
{
    if (n <= 0) return cudaSuccess;
    const int blocks = (int)std::min<int64_t>((n + 255) / 256, 1184);
    event_sums_kernel<<<blocks, 256, 0, s>>>(n, x_cm, y_cm, de, out);
    return cudaGetLastError();
}

}  // namespace fd2

// ============================================================ C ABI

using namespace fd2x;

struct fd2_xray {
    Material m;
    fd2_xray_options opt{};
    std::string err;
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[4] = {};
    // device tables
    double *d_e = nullptr, *d_lnv = nullptr, *d_ee = nullptr, *d_lnee = nullptr, *d_lnr = nullptr,
           *d_lnl1 = nullptr, *d_bind = nullptr, *d_tcum = nullptr, *d_te = nullptr;
    int *d_toff = nullptr, *d_ts = nullptr;
    XDev dev{};
    // batch buffers
    Ede *d_slots = nullptr;
    HistInfo *d_info = nullptr;  // the run's per-history records (device; copied out on request)
    int64_t info_cap = 0, n_info = 0;
    uint32_t *d_counts = nullptr;
    unsigned long long *d_offsets = nullptr, *d_block_sums = nullptr, *d_total = nullptr;
    int64_t batch_cap = 0;
    // run outputs
    double *d_x = nullptr, *d_y = nullptr, *d_z = nullptr, *d_de = nullptr;
    int32_t *d_hist = nullptr;
    int64_t out_cap = 0, n_out = 0;
    Totals *d_tot = nullptr;
    fd2_xray_stats stats{};
    float t_transport = 0, t_compact = 0;
    // source buffers
    double *d_spec = nullptr;
    int spec_cap = 0;
};

namespace {

fd2_status xfail(fd2_xray *x, fd2_status s, const std::string &m)
{
    if (x) x->err = m;
    return s;
}

#define XCUDA(x, call)                                                                  \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess) return xfail(x, FD2_ERR_CUDA, cudaGetErrorString(e_)); \
    } while (0)

template <class T>
cudaError_t upload(T **d, const std::vector<T> &h)
{
    if (*d) cudaFree(*d);
    *d = nullptr;
    cudaError_t e = cudaMalloc((void **)d, sizeof(T) * std::max<size_t>(h.size(), 1));
    if (e != cudaSuccess) return e;
    return h.empty() ? cudaSuccess : cudaMemcpy(*d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice);
}

double lnz(double v) { return std::log(std::max(v, 1e-300)); }

fd2_status upload_tables(fd2_xray *x)
{
    const Material &m = x->m;
    const int nel = m.n_el(), stride = 3 + nel * (1 + kShells);
    const size_t n = m.e.size();
    std::vector<double> lnv(n * stride);
    for (size_t i = 0; i < n; ++i) {
        double *r = &lnv[i * stride];
        r[0] = lnz(m.mu_r[i]);
        r[1] = lnz(m.mu_c[i]);
        r[2] = lnz(m.ray_b[i]);
        for (int k = 0; k < nel; ++k) {
            r[3 + k * (1 + kShells)] = lnz(m.mu_pe[i * nel + k]);
            for (int q = 0; q < kShells; ++q) r[3 + k * (1 + kShells) + 1 + q] = lnz(m.mu_sh[(i * nel + k) * kShells + q]);
        }
    }
    std::vector<double> lnee(m.ee.size()), lnr(m.ee.size()), lnl1(m.ee.size());
    for (size_t i = 0; i < m.ee.size(); ++i) {
        lnee[i] = std::log(m.ee[i]);
        lnr[i] = std::log(m.range[i]);
        lnl1[i] = std::log(m.lambda1[i]);
    }
    std::vector<double> bind(nel * kDesignators);
    std::vector<int> toff(nel * (kDesignators + 1)), ts;
    std::vector<double> tcum, te;
    for (int k = 0; k < nel; ++k) {
        for (int d = 0; d < kDesignators; ++d) bind[k * kDesignators + d] = m.binding[k][d];
        for (int s0 = 0; s0 < kDesignators; ++s0) {
            toff[k * (kDesignators + 1) + s0] = (int)ts.size();
            double sum = 0;
            for (const auto &t : m.trans[k])
                if (t.s0 == s0) sum += t.p;
            double acc = 0;
            for (const auto &t : m.trans[k])
                if (t.s0 == s0) {
                    acc += t.p;
                    ts.push_back(t.s1 | (t.s2 << 8));
                    tcum.push_back(acc / sum);
                    te.push_back(t.e);
                }
        }
        toff[k * (kDesignators + 1) + kDesignators] = (int)ts.size();
    }
    XCUDA(x, upload(&x->d_e, m.e));
    XCUDA(x, upload(&x->d_lnv, lnv));
    XCUDA(x, upload(&x->d_ee, m.ee));
    XCUDA(x, upload(&x->d_lnee, lnee));
    XCUDA(x, upload(&x->d_lnr, lnr));
    XCUDA(x, upload(&x->d_lnl1, lnl1));
    XCUDA(x, upload(&x->d_bind, bind));
    XCUDA(x, upload(&x->d_toff, toff));
    XCUDA(x, upload(&x->d_ts, ts));
    XCUDA(x, upload(&x->d_tcum, tcum));
    XCUDA(x, upload(&x->d_te, te));
    XDev &g = x->dev;
    g.n_nodes = (int)n;
    g.n_el = nel;
    g.stride = stride;
    g.e = x->d_e;
    g.lnv = x->d_lnv;
    g.n_e = (int)m.ee.size();
    g.ee = x->d_ee;
    g.lnee = x->d_lnee;
    g.lnr = x->d_lnr;
    g.lnl1 = x->d_lnl1;
    g.binding = x->d_bind;
    g.toff = x->d_toff;
    g.ts = x->d_ts;
    g.tcum = x->d_tcum;
    g.te = x->d_te;
    const fd2_xray_options &o = x->opt;
    g.X = o.det_x_um * 1e-4;
    g.Y = o.det_y_um * 1e-4;
    g.H2 = 0.5 * o.det_height_um * 1e-4;
    g.eabs_e = o.eabs_electron_ev;
    g.eabs_ph = o.eabs_photon_ev;
    g.loss = o.electron_step_loss;
    g.local_e = std::max(o.eabs_electron_ev, o.electron_local_ev);
    g.fluo = o.fluorescence;
    g.cap = o.max_edes_per_history;
    g.k0 = (uint32_t)o.seed;
    g.k1 = (uint32_t)(o.seed >> 32);
    return FD2_OK;
}

template <class T>
void dfree(T *&p)
{
    if (p) cudaFree(p);
    p = nullptr;
}

fd2_status ensure_batch(fd2_xray *x, int64_t b)
{
    if (b <= x->batch_cap) return FD2_OK;
    dfree(x->d_slots);
    dfree(x->d_counts);
    dfree(x->d_offsets);
    dfree(x->d_block_sums);
    x->batch_cap = 0;
    XCUDA(x, cudaMalloc(&x->d_slots, sizeof(Ede) * (size_t)b * x->opt.max_edes_per_history));
    XCUDA(x, cudaMalloc(&x->d_counts, sizeof(uint32_t) * (size_t)b));
    XCUDA(x, cudaMalloc(&x->d_offsets, sizeof(unsigned long long) * (size_t)b));
    XCUDA(x, cudaMalloc(&x->d_block_sums, sizeof(unsigned long long) * std::max<size_t>(fd2::scan_block_sums_needed(b), 1)));
    x->batch_cap = b;
    return FD2_OK;
}

fd2_status ensure_out(fd2_xray *x, int64_t need)
{
    if (need <= x->out_cap) return FD2_OK;
    const int64_t cap = std::max<int64_t>(need, x->out_cap + x->out_cap / 2);
    double *nx, *ny, *nz, *nd;
    int32_t *nh;
    XCUDA(x, cudaMalloc(&nx, sizeof(double) * cap));
    XCUDA(x, cudaMalloc(&ny, sizeof(double) * cap));
    XCUDA(x, cudaMalloc(&nz, sizeof(double) * cap));
    XCUDA(x, cudaMalloc(&nd, sizeof(double) * cap));
    XCUDA(x, cudaMalloc(&nh, sizeof(int32_t) * cap));
    if (x->n_out) {
        XCUDA(x, cudaMemcpyAsync(nx, x->d_x, sizeof(double) * x->n_out, cudaMemcpyDeviceToDevice, x->stream));
        XCUDA(x, cudaMemcpyAsync(ny, x->d_y, sizeof(double) * x->n_out, cudaMemcpyDeviceToDevice, x->stream));
        XCUDA(x, cudaMemcpyAsync(nz, x->d_z, sizeof(double) * x->n_out, cudaMemcpyDeviceToDevice, x->stream));
        XCUDA(x, cudaMemcpyAsync(nd, x->d_de, sizeof(double) * x->n_out, cudaMemcpyDeviceToDevice, x->stream));
        XCUDA(x, cudaMemcpyAsync(nh, x->d_hist, sizeof(int32_t) * x->n_out, cudaMemcpyDeviceToDevice, x->stream));
        XCUDA(x, cudaStreamSynchronize(x->stream));
    }
    dfree(x->d_x);
    dfree(x->d_y);
    dfree(x->d_z);
    dfree(x->d_de);
    dfree(x->d_hist);
    x->d_x = nx;
    x->d_y = ny;
    x->d_z = nz;
    x->d_de = nd;
    x->d_hist = nh;
    x->out_cap = cap;
    return FD2_OK;
}

// Validate a source and build its device form (spectrum in d_spec).
fd2_status make_source(fd2_xray *x, const fd2_xray_source *s, XSource &o)
{
    if (!s || (s->particle != FD2_XRAY_PHOTON && s->particle != FD2_XRAY_ELECTRON) || s->n_spectrum < 2 ||
        s->n_spectrum > 100000 || !s->e_ev || !s->prob)
        return xfail(x, FD2_ERR_INVALID_ARGUMENT, "source: particle, spectrum lines or arrays");
    if (!(s->semiaperture_deg >= 0.0 && s->semiaperture_deg <= 180.0))
        return xfail(x, FD2_ERR_INVALID_ARGUMENT, "source: semiaperture outside [0, 180]");
    const int n = s->n_spectrum;
    for (int i = 0; i < n; ++i)
        if (!(s->e_ev[i] >= 0.0) || (i && s->e_ev[i] < s->e_ev[i - 1]))
            return xfail(x, FD2_ERR_INVALID_ARGUMENT, "source: spectrum energies negative or decreasing");
    std::memset(&o, 0, sizeof o);
    o.particle = s->particle;
    std::vector<double> buf;
    double psum = 0;
    for (int i = 0; i < n - 1; ++i) {
        if (!(s->prob[i] >= 0.0)) return xfail(x, FD2_ERR_INVALID_ARGUMENT, "source: negative bin probability");
        psum += s->prob[i];
    }
    if (psum > 0.0) {
        std::vector<double> pc(n), de(n, 0.0);
        pc[0] = 0;
        for (int i = 0; i < n - 1; ++i) pc[i + 1] = pc[i] + s->prob[i];
        for (int i = 0; i < n; ++i) pc[i] /= pc[n - 1];
        for (int i = 0; i < n - 1; ++i)
            if (pc[i + 1] > pc[i]) de[i] = (s->e_ev[i + 1] - s->e_ev[i]) / (pc[i + 1] - pc[i]);
        buf.insert(buf.end(), s->e_ev, s->e_ev + n);
        buf.insert(buf.end(), pc.begin(), pc.end());
        buf.insert(buf.end(), de.begin(), de.end());
        o.nspec = n;
    } else {
        if (n != 2) return xfail(x, FD2_ERR_INVALID_ARGUMENT, "source: a Gaussian spectrum has exactly 2 lines");
        o.gaussian = 1;
        o.gmean = 0.5 * (s->e_ev[0] + s->e_ev[1]);
        o.gsig = 0.42466090014400952 * (s->e_ev[1] - s->e_ev[0]);  // FWHM to sigma
        o.gmin = std::max(0.0, o.gmean - 6.0 * o.gsig);
        o.gmax = o.gmean + 6.0 * o.gsig;
        if (!(o.gsig > 0.0)) return xfail(x, FD2_ERR_INVALID_ARGUMENT, "source: Gaussian FWHM must be positive");
        buf.assign(3, 0.0);
    }
    if ((int)buf.size() > x->spec_cap) {
        dfree(x->d_spec);
        XCUDA(x, cudaMalloc(&x->d_spec, sizeof(double) * buf.size()));
        x->spec_cap = (int)buf.size();
    }
    XCUDA(x, cudaMemcpy(x->d_spec, buf.data(), sizeof(double) * buf.size(), cudaMemcpyHostToDevice));
    o.espc = x->d_spec;
    o.pcum = x->d_spec + n;
    o.despc = x->d_spec + 2 * n;
    for (int a = 0; a < 3; ++a) {
        o.ctr[a] = s->center_cm[a];
        o.side[a] = s->sides_cm[a];
    }
    o.point = s->sides_cm[0] == 0.0 && s->sides_cm[1] == 0.0 && s->sides_cm[2] == 0.0;
    // box rotation by the Euler angles (omega about z, theta about y, phi
    // about z), the matrix of sourceBoxIsotropicGaussSpectrum.f:333-348
    const double dr = M_PI / 180.0;
    const double so = std::sin(s->euler_deg[0] * dr), co = std::cos(s->euler_deg[0] * dr);
    const double st = std::sin(s->euler_deg[1] * dr), ct = std::cos(s->euler_deg[1] * dr);
    const double sp = std::sin(s->euler_deg[2] * dr), cp = std::cos(s->euler_deg[2] * dr);
    const double R[9] = {cp * ct * co - sp * so, -cp * ct * so - sp * co, cp * st,
                         sp * ct * co + cp * so, -sp * ct * so + cp * co, sp * st,
                         -st * co,               st * so,                 ct};
    std::memcpy(o.rot, R, sizeof R);
    const double nrm = std::sqrt(s->direction[0] * s->direction[0] + s->direction[1] * s->direction[1] +
                                 s->direction[2] * s->direction[2]);
    if (nrm < 1e-30) {
        if (s->semiaperture_deg != 180.0)
            return xfail(x, FD2_ERR_INVALID_ARGUMENT, "source: a null direction needs a 180 degree aperture");
        o.dir[0] = 0;
        o.dir[1] = 0;
        o.dir[2] = 1;
    } else
        for (int a = 0; a < 3; ++a) o.dir[a] = s->direction[a] / nrm;
    o.cossrc = std::cos(s->semiaperture_deg * M_PI / 180.0);
    return FD2_OK;
}

}  // namespace

extern "C" {

FD2_API fd2_status fd2_xray_load_material(const char *path, fd2_xray_material **out)
{
    if (!path || !out) return FD2_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    auto *m = new fd2_xray_material();
    std::string err;
    FILE *f = std::fopen(path, "r");
    if (!f) {
        delete m;
        return FD2_ERR_IO;
    }
    char head[64] = {0};
    const size_t got = std::fread(head, 1, sizeof head - 1, f);
    std::fclose(f);
    const bool table = got >= 17 && std::strncmp(head, "fd2-xray-material", 17) == 0;
    const bool ok = table ? load_table(path, m->m, err) : load_penelope(path, m->m, err);
    if (!ok) {
        delete m;
        return FD2_ERR_PARSE;
    }
    *out = m;
    return FD2_OK;
}

FD2_API fd2_status fd2_xray_save_material(const fd2_xray_material *m, const char *path)
{
    if (!m || !path) return FD2_ERR_INVALID_ARGUMENT;
    std::string err;
    return save_table(m->m, path, err) ? FD2_OK : FD2_ERR_IO;
}

FD2_API void fd2_xray_free_material(fd2_xray_material *m) { delete m; }

FD2_API fd2_status fd2_xray_material_get_info(const fd2_xray_material *mm, fd2_xray_material_info *o)
{
    if (!mm || !o) return FD2_ERR_INVALID_ARGUMENT;
    const Material &m = mm->m;
    std::memset(o, 0, sizeof *o);
    o->density_g_cm3 = m.density;
    o->molar_mass_g_mol = m.molar_mass;
    o->molecules_per_cm3 = m.molecules_per_cm3;
    o->n_elements = m.n_el();
    for (int k = 0; k < m.n_el(); ++k) {
        o->z[k] = m.z[k];
        o->atoms_per_molecule[k] = m.atoms[k];
        o->k_edge_ev[k] = m.binding[k][1];
    }
    o->e_min_ev = m.e.front();
    o->e_max_ev = m.e.back();
    o->n_photon_nodes = (int32_t)m.e.size();
    int nt = 0;
    for (const auto &t : m.trans) nt += (int)t.size();
    o->n_transitions = nt;
    o->rayleigh_screening_cm = m.rayleigh_a;
    return FD2_OK;
}

FD2_API fd2_status fd2_xray_attenuation(const fd2_xray_material *m, const double *e, int64_t n, double *out)
{
    if (!m || n < 0 || (n && (!e || !out))) return FD2_ERR_INVALID_ARGUMENT;
    for (int64_t i = 0; i < n; ++i) attenuation(m->m, e[i], out + 4 * i);
    return FD2_OK;
}

FD2_API fd2_status fd2_xray_electron_tables(const fd2_xray_material *m, const double *e, int64_t n, double *range,
                                            double *lambda1)
{
    if (!m || n < 0 || (n && (!e || !range || !lambda1))) return FD2_ERR_INVALID_ARGUMENT;
    for (int64_t i = 0; i < n; ++i) electron_at(m->m, e[i], range + i, lambda1 + i);
    return FD2_OK;
}

FD2_API void fd2_xray_default_options(fd2_xray_options *o)
{
    if (!o) return;
    std::memset(o, 0, sizeof *o);
    o->device = 0;
    o->det_x_um = 909.0;  // example/CsI.geo: 0.0909 cm square, 150 um thick
    o->det_y_um = 909.0;
    o->det_height_um = 150.0;
    o->eabs_electron_ev = 50.0;
    o->eabs_photon_ev = 50.0;
    o->electron_step_loss = 0.25;
    o->electron_local_ev = 1000.0;
    o->fluorescence = 1;
    o->max_edes_per_history = 256;
    o->batch_histories = 65536;
    o->seed = 12345;
}

FD2_API fd2_status fd2_xray_create(const fd2_xray_material *m, const fd2_xray_options *o, fd2_xray **out)
{
    if (!m || !o || !out) return FD2_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    if (!(o->det_x_um > 0 && o->det_y_um > 0 && o->det_height_um > 0) || !(o->eabs_electron_ev > 0) ||
        !(o->eabs_photon_ev > 0) || !(o->electron_step_loss > 0.01 && o->electron_step_loss < 1.0) || !(o->electron_local_ev >= 0.0) ||
        o->max_edes_per_history < 64 || o->max_edes_per_history > 4096 || o->batch_histories < 1 ||
        o->batch_histories > (1 << 22) || (o->fluorescence != 0 && o->fluorescence != 1))
        return FD2_ERR_INVALID_ARGUMENT;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return FD2_ERR_NO_DEVICE;
    if (o->device < 0 || o->device >= ndev) return FD2_ERR_INVALID_ARGUMENT;
    auto *x = new fd2_xray();
    x->m = m->m;
    x->opt = *o;
    x->device = o->device;
    fd2_status st = FD2_OK;
    if (cudaSetDevice(x->device) != cudaSuccess || cudaStreamCreateWithFlags(&x->stream, cudaStreamNonBlocking) != cudaSuccess)
        st = FD2_ERR_CUDA;
    for (int i = 0; st == FD2_OK && i < 4; ++i)
        if (cudaEventCreate(&x->ev[i]) != cudaSuccess) st = FD2_ERR_CUDA;
    if (st == FD2_OK) st = upload_tables(x);
    if (st == FD2_OK && cudaMalloc(&x->d_tot, sizeof(Totals)) != cudaSuccess) st = FD2_ERR_OUT_OF_MEMORY;
    // [0] a batch's EDE total, [1] the history kernel's counter
    if (st == FD2_OK && cudaMalloc(&x->d_total, 2 * sizeof(unsigned long long)) != cudaSuccess)
        st = FD2_ERR_OUT_OF_MEMORY;
    if (st == FD2_OK && cudaMemset(x->d_tot, 0, sizeof(Totals)) != cudaSuccess) st = FD2_ERR_CUDA;
    if (st != FD2_OK) {
        fd2_xray_destroy(x);
        return st;
    }
    *out = x;
    return FD2_OK;
}

FD2_API void fd2_xray_destroy(fd2_xray *x)
{
    if (!x) return;
    cudaSetDevice(x->device);
    if (x->stream) cudaStreamSynchronize(x->stream);
    for (double *p : {x->d_e, x->d_lnv, x->d_ee, x->d_lnee, x->d_lnr, x->d_lnl1, x->d_bind, x->d_tcum, x->d_te, x->d_x,
                      x->d_y, x->d_z, x->d_de, x->d_spec})
        if (p) cudaFree(p);
    for (void *p : {(void *)x->d_toff, (void *)x->d_ts, (void *)x->d_slots, (void *)x->d_info,
                    (void *)x->d_counts, (void *)x->d_offsets, (void *)x->d_block_sums, (void *)x->d_total,
                    (void *)x->d_hist, (void *)x->d_tot})
        if (p) cudaFree(p);
    for (auto &e : x->ev)
        if (e) cudaEventDestroy(e);
    if (x->stream) cudaStreamDestroy(x->stream);
    delete x;
}

FD2_API const char *fd2_xray_last_error(const fd2_xray *x) { return x ? x->err.c_str() : ""; }

FD2_API fd2_status fd2_xray_run(fd2_xray *x, const fd2_xray_source *src, int64_t first, int64_t n)
{
    if (!x) return FD2_ERR_INVALID_ARGUMENT;
    if (n < 0 || first < 0 || first + n >= ((int64_t)1 << 31))
        return xfail(x, FD2_ERR_INVALID_ARGUMENT, "run: histories must lie in [0, 2^31 - 1)");
    XCUDA(x, cudaSetDevice(x->device));
    XSource s;
    fd2_status st = make_source(x, src, s);
    if (st != FD2_OK) return st;
    const int64_t B = std::min<int64_t>(x->opt.batch_histories, std::max<int64_t>(n, 1));
    if ((st = ensure_batch(x, B)) != FD2_OK) return st;
    if (n > x->info_cap) {
        dfree(x->d_info);
        x->info_cap = 0;
        XCUDA(x, cudaMalloc(&x->d_info, sizeof(HistInfo) * (size_t)std::max<int64_t>(n, 1)));
        x->info_cap = n;
    }
    x->n_info = n;
    x->n_out = 0;
    x->t_transport = x->t_compact = 0;
    for (int64_t b0 = 0; b0 < n; b0 += B) {
        const int64_t nb = std::min(B, n - b0);
        const unsigned grid = (unsigned)((nb + 127) / 128);
        XCUDA(x, cudaEventRecord(x->ev[0], x->stream));
        HistInfo *info = x->d_info + b0;
        XCUDA(x, cudaMemsetAsync(x->d_total + 1, 0, sizeof(unsigned long long), x->stream));
        history_kernel<<<grid, 128, 0, x->stream>>>(x->dev, s, first + b0, nb, x->d_slots, info, x->d_total + 1);
        XCUDA(x, cudaGetLastError());
        XCUDA(x, cudaEventRecord(x->ev[1], x->stream));
        count_kernel<<<grid, 128, 0, x->stream>>>(info, nb, x->d_counts);
        XCUDA(x, cudaGetLastError());
        XCUDA(x, fd2::launch_scan(x->stream, nb, x->d_counts, x->d_offsets, x->d_block_sums, x->d_total));
        unsigned long long tot = 0;
        XCUDA(x, cudaMemcpyAsync(&tot, x->d_total, sizeof tot, cudaMemcpyDeviceToHost, x->stream));
        XCUDA(x, cudaStreamSynchronize(x->stream));
        if ((st = ensure_out(x, x->n_out + (int64_t)tot)) != FD2_OK) return st;
        XCUDA(x, cudaEventRecord(x->ev[2], x->stream));
        scatter_kernel<<<grid, 128, 0, x->stream>>>(info, x->d_slots, x->opt.max_edes_per_history, nb,
                                                   first + b0, x->d_offsets, x->n_out, x->d_x, x->d_y, x->d_z,
                                                   x->d_de, x->d_hist, x->d_tot);
        XCUDA(x, cudaGetLastError());
        XCUDA(x, cudaEventRecord(x->ev[3], x->stream));
        XCUDA(x, cudaStreamSynchronize(x->stream));
        float a = 0, c = 0, d = 0;
        cudaEventElapsedTime(&a, x->ev[0], x->ev[1]);
        cudaEventElapsedTime(&c, x->ev[1], x->ev[2]);
        cudaEventElapsedTime(&d, x->ev[2], x->ev[3]);
        x->t_transport += a;
        x->t_compact += c + d;
        x->n_out += (int64_t)tot;
    }
    x->stats.histories += n;
    return FD2_OK;
}

FD2_API fd2_status fd2_xray_num_edes(fd2_xray *x, int64_t *n)
{
    if (!x || !n) return FD2_ERR_INVALID_ARGUMENT;
    *n = x->n_out;
    return FD2_OK;
}

FD2_API fd2_status fd2_xray_get_edes(fd2_xray *x, double *xs, double *ys, double *zs, double *des, int32_t *hs,
                                     int64_t cap)
{
    if (!x) return FD2_ERR_INVALID_ARGUMENT;
    if (cap < x->n_out) return xfail(x, FD2_ERR_INVALID_ARGUMENT, "get_edes: arrays shorter than the EDE count");
    const size_t n = (size_t)x->n_out;
    if (!n) return FD2_OK;
    XCUDA(x, cudaSetDevice(x->device));
    if (xs) XCUDA(x, cudaMemcpy(xs, x->d_x, 8 * n, cudaMemcpyDeviceToHost));
    if (ys) XCUDA(x, cudaMemcpy(ys, x->d_y, 8 * n, cudaMemcpyDeviceToHost));
    if (zs) XCUDA(x, cudaMemcpy(zs, x->d_z, 8 * n, cudaMemcpyDeviceToHost));
    if (des) XCUDA(x, cudaMemcpy(des, x->d_de, 8 * n, cudaMemcpyDeviceToHost));
    if (hs) XCUDA(x, cudaMemcpy(hs, x->d_hist, 4 * n, cudaMemcpyDeviceToHost));
    return FD2_OK;
}

FD2_API fd2_status fd2_xray_get_history_info(fd2_xray *x, double *e0, double *esc_ph, double *esc_el, double *depth,
                                             int32_t *kind, int32_t *nedes, int64_t n)
{
    if (!x || n < 0) return FD2_ERR_INVALID_ARGUMENT;
    if (n > x->n_info) return xfail(x, FD2_ERR_INVALID_ARGUMENT, "history_info: n above the run's histories");
    std::vector<HistInfo> info((size_t)n);
    if (n) {
        XCUDA(x, cudaSetDevice(x->device));
        XCUDA(x, cudaMemcpy(info.data(), x->d_info, sizeof(HistInfo) * (size_t)n, cudaMemcpyDeviceToHost));
    }
    for (int64_t i = 0; i < n; ++i) {
        const HistInfo &h = info[(size_t)i];
        if (e0) e0[i] = h.e0;
        if (esc_ph) esc_ph[i] = h.esc_ph;
        if (esc_el) esc_el[i] = h.esc_el;
        if (depth) depth[i] = h.first_kind ? h.first_depth : -1.0;
        if (kind) kind[i] = h.first_kind;
        if (nedes) nedes[i] = h.n_edes;
    }
    return FD2_OK;
}

FD2_API fd2_status fd2_xray_get_stats(fd2_xray *x, fd2_xray_stats *o)
{
    if (!x || !o) return FD2_ERR_INVALID_ARGUMENT;
    Totals t{};
    XCUDA(x, cudaSetDevice(x->device));
    XCUDA(x, cudaMemcpy(&t, x->d_tot, sizeof t, cudaMemcpyDeviceToHost));
    *o = fd2_xray_stats{};
    o->histories = x->stats.histories;
    o->missed = (int64_t)t.missed;
    o->edes = (int64_t)t.edes;
    o->merged_histories = (int64_t)t.merged;
    o->photoelectric = (int64_t)t.pe;
    o->compton = (int64_t)t.co;
    o->rayleigh = (int64_t)t.ra;
    o->fluorescence_emitted = (int64_t)t.fe;
    o->fluorescence_escaped = (int64_t)t.fesc;
    o->auger_emitted = (int64_t)t.aug;
    o->electron_steps = (int64_t)t.steps;
    o->e_source_ev = t.e0;
    o->e_deposited_ev = t.dep;
    o->e_escaped_photon_ev = t.esc_ph;
    o->e_escaped_electron_ev = t.esc_el;
    return FD2_OK;
}

FD2_API fd2_status fd2_xray_clear_stats(fd2_xray *x)
{
    if (!x) return FD2_ERR_INVALID_ARGUMENT;
    XCUDA(x, cudaSetDevice(x->device));
    XCUDA(x, cudaMemset(x->d_tot, 0, sizeof(Totals)));
    x->stats = fd2_xray_stats{};
    return FD2_OK;
}

FD2_API fd2_status fd2_xray_get_timing(fd2_xray *x, double *transport_ms, double *compact_ms)
{
    if (!x) return FD2_ERR_INVALID_ARGUMENT;
    if (transport_ms) *transport_ms = x->t_transport;
    if (compact_ms) *compact_ms = x->t_compact;
    return FD2_OK;
}

FD2_API fd2_status fd2_xray_device_edes(fd2_xray *x, const double **xs, const double **ys, const double **zs,
                                        const double **des, const int32_t **hs, int64_t *n)
{
    if (!x) return FD2_ERR_INVALID_ARGUMENT;
    if (xs) *xs = x->d_x;
    if (ys) *ys = x->d_y;
    if (zs) *zs = x->d_z;
    if (des) *des = x->d_de;
    if (hs) *hs = x->d_hist;
    if (n) *n = x->n_out;
    return FD2_OK;
}

FD2_API fd2_status fd2_xray_submit(fd2_xray *x, fd2_ctx *optical)
{
    if (!x || !optical) return FD2_ERR_INVALID_ARGUMENT;
    return fd2_submit_events_device(optical, x->d_x, x->d_y, x->d_z, x->d_de, x->d_hist, x->n_out);
}

FD2_API fd2_status fd2_xray_sample(fd2_xray *x, int32_t which, double e, double param, int64_t n, uint64_t seed,
                                   double *out)
{
    if (!x || which < 0 || which > 3 || n < 0 || (n && !out) || !(e > 0) || (which == 3 && !(param > 0)))
        return xfail(x, FD2_ERR_INVALID_ARGUMENT, "sample: bad arguments");
    if (!n) return FD2_OK;
    XCUDA(x, cudaSetDevice(x->device));
    double *d = nullptr;
    XCUDA(x, cudaMalloc(&d, sizeof(double) * n));
    sample_kernel<<<(unsigned)((n + 127) / 128), 128, 0, x->stream>>>(x->dev, which, e, param, n, (uint32_t)seed,
                                                                      (uint32_t)(seed >> 32), d);
    cudaError_t err = cudaGetLastError();
    if (err == cudaSuccess) err = cudaMemcpyAsync(out, d, sizeof(double) * n, cudaMemcpyDeviceToHost, x->stream);
    if (err == cudaSuccess) err = cudaStreamSynchronize(x->stream);
    cudaFree(d);
    if (err != cudaSuccess) return xfail(x, FD2_ERR_CUDA, cudaGetErrorString(err));
    return FD2_OK;
}

}  // extern "C"
