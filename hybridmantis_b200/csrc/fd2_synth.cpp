// fd2_synth.cpp -- seeded synthetic energy-deposition streams.
//
// PENELOPE (the reference's x-ray/electron transport) is not part of this
// path and its sources are not shipped, so the benchmark configurations are
// driven by these generators, with the shapes and distributions the
// configurations state.  Positions in micrometres with the reference's
// coordinates: x, y in (0, det), z in (-H/2, H/2), x-rays entering at
// z = +H/2, so a deposition at depth d has z = H/2 - d.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "fd2.h"
#include "fd2_host.h"

namespace fd2host {

static uint64_t splitmix64(uint64_t &x)
{
    uint64_t z = (x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

HostRng::HostRng(uint64_t seed)
{
    uint64_t x = seed;
    for (auto &v : s) v = splitmix64(x);
}

uint64_t HostRng::next()
{
    const uint64_t r = rotl(s[1] * 5, 7) * 9;
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return r;
}

double HostRng::uniform() { return ((double)(next() >> 11) + 0.5) * (1.0 / 9007199254740992.0); }

double HostRng::normal()
{
    for (;;) {
        const double a = 2.0 * uniform() - 1.0, b = 2.0 * uniform() - 1.0;
        const double r = a * a + b * b;
        if (r > 0.0 && r < 1.0) return a * std::sqrt(-2.0 * std::log(r) / r);
    }
}

// Exponential with the given mean, conditioned on [0, upper] (inverse CDF).
double HostRng::trunc_exp(double mean, double upper)
{
    const double f = 1.0 - std::exp(-upper / mean);
    return -mean * std::log1p(-uniform() * f);
}

double HostRng::triangular(double a, double c, double b)
{
    const double u = uniform(), fc = (c - a) / (b - a);
    return u < fc ? a + std::sqrt(u * (b - a) * (c - a)) : b - std::sqrt((1.0 - u) * (b - a) * (b - c));
}

int HostRng::poisson_small(double mu)
{
    const double lim = std::exp(-mu);
    double p = uniform();
    int k = 0;
    while (p > lim && k < 1000) {
        p *= uniform();
        ++k;
    }
    return k;
}

}  // namespace fd2host

namespace {

struct Builder {
    std::vector<float> x, y, z, e;
    std::vector<int32_t> h;
    std::vector<uint16_t> g;
    void add(float xx, float yy, float zz, float ee, int32_t hh, uint16_t gg)
    {
        x.push_back(xx);
        y.push_back(yy);
        z.push_back(zz);
        e.push_back(ee);
        h.push_back(hh);
        g.push_back(gg);
    }
};

fd2_params base_params(int32_t num_hist, double H, double R)
{
    fd2_params p;
    std::memset(&p, 0, sizeof p);
    p.num_hist = num_hist;
    p.min_photons = 0;
    p.max_photons = 2000;
    p.num_bins = 1000;
    p.det_x = 501.0;
    p.det_y = 501.0;
    p.det_height = H;
    p.radius = R;
    p.n_col = 1.8;
    p.n_gap = 1.0;
    p.top_absfrac = 0.1;  // top reflectivity 0.9
    p.bulk_abs = 1e-4;
    p.beta = 0.2;
    p.d_min = 0.5;        // the configurations' 0.5 um column gap
    p.d_max = 280.0;      // the reference example's maximum hop
    p.lb_x = 0.0;
    p.lb_y = 0.0;
    p.ub_x = 501.0;
    p.ub_y = 501.0;
    p.yield = 0.054;      // 54 photons / keV
    p.pixel = 1;
    p.sensor_refl = 0.0;  // ideal sensor
    p.run_gpu = 1;
    p.machine = 1;
    return p;
}

// Deposition clusters of one x-ray: 1 + Poisson(1.5) clusters sharing the
// absorbed energy by a flat Dirichlet, depths ~ Exp(90 um) truncated to the
// layer, lateral offsets N(0, 5 um) around the beam.
void add_clusters(Builder &b, fd2host::HostRng &rng, double energy_ev, double H, int32_t hist, uint16_t geom)
{
    const int k = 1 + rng.poisson_small(1.5);
    double w[64], sum = 0.0;
    const int kk = k < 64 ? k : 64;
    for (int j = 0; j < kk; ++j) {
        w[j] = -std::log(rng.uniform());
        sum += w[j];
    }
    for (int j = 0; j < kk; ++j) {
        const double d = rng.trunc_exp(90.0, H);
        const double xx = 250.5 + 5.0 * rng.normal(), yy = 250.5 + 5.0 * rng.normal();
        b.add((float)xx, (float)yy, (float)(H / 2.0 - d), (float)(energy_ev * w[j] / sum), hist, geom);
    }
}

fd2_status finish(Builder &b, int32_t num_hist, const fd2_params &p, const std::vector<fd2_geometry> &geoms,
                  bool keep_geom, fd2_events *out)
{
    fd2_status st = fd2host::events_from_vectors(b.x, b.y, b.z, b.e, b.h, num_hist, out);
    if (st != FD2_OK) return st;
    out->params = p;
    fd2_params_fill_tags(&out->params);
    out->num_geom = (int32_t)geoms.size();
    out->geometries = (fd2_geometry *)std::malloc(sizeof(fd2_geometry) * geoms.size());
    if (!out->geometries) {
        fd2_free_events(out);
        return FD2_ERR_OUT_OF_MEMORY;
    }
    std::memcpy(out->geometries, geoms.data(), sizeof(fd2_geometry) * geoms.size());
    if (keep_geom) {
        const size_t n = b.g.size() ? b.g.size() : 1;
        out->geom = (uint16_t *)std::malloc(2 * n);
        if (!out->geom) {
            fd2_free_events(out);
            return FD2_ERR_OUT_OF_MEMORY;
        }
        if (!b.g.empty()) std::memcpy(out->geom, b.g.data(), 2 * b.g.size());
    }
    return FD2_OK;
}

}  // namespace

extern "C" fd2_status fd2_synth_events(int32_t config, int32_t num_xrays, uint64_t seed, fd2_events *out)
{
    if (!out || num_xrays < 0) return FD2_ERR_INVALID_ARGUMENT;
    std::memset(out, 0, sizeof *out);
    fd2host::HostRng rng(seed * 0x9E3779B97F4A7C15ull + (uint64_t)config);
    Builder b;
    switch (config) {
    case 0: {
        // 25 keV pencil beam, one deposition at depth ~ Exp(60 um) in 150 um,
        // lateral N(0, 2 um); ~1350 photons per event at 54 / keV
        const int32_t nx = num_xrays ? num_xrays : 1000;
        const double H = 150.0;
        fd2_params p = base_params(nx, H, 5.0);
        for (int32_t i = 0; i < nx; ++i) {
            const double d = rng.trunc_exp(60.0, H);
            const double xx = 250.5 + 2.0 * rng.normal(), yy = 250.5 + 2.0 * rng.normal();
            b.add((float)xx, (float)yy, (float)(H / 2.0 - d), 25000.0f, i + 1, 0);
        }
        fd2_geometry g;
        fd2_params_to_geometry(&p, &g);
        return finish(b, nx, p, {g}, false, out);
    }
    case 1:
    case 4: {
        // triangular spectrum on [20, 70] keV (mode 40), clustered depositions;
        // config 1: 300 um layer, R = 4; config 4: 500 um layer, R = 5
        const int32_t nx = num_xrays ? num_xrays : (config == 1 ? 100000 : 1000000);
        const double H = config == 1 ? 300.0 : 500.0;
        fd2_params p = base_params(nx, H, config == 1 ? 4.0 : 5.0);
        p.max_photons = 4000;
        for (int32_t i = 0; i < nx; ++i) add_clusters(b, rng, 1000.0 * rng.triangular(20.0, 40.0, 70.0), H, i + 1, 0);
        fd2_geometry g;
        fd2_params_to_geometry(&p, &g);
        return finish(b, nx, p, {g}, false, out);
    }
    case 2: {
        // 64 geometries x 2000 x-rays, energies U(15, 80) keV
        const int32_t per = num_xrays ? num_xrays : 2000;
        const int ng = 64;
        std::vector<fd2_geometry> geoms((size_t)ng);
        fd2_params p = base_params(per * ng, 300.0, 5.0);
        p.max_photons = 4400;
        for (int gi = 0; gi < ng; ++gi) {
            fd2_params q = p;
            q.det_height = 100.0 + 500.0 * rng.uniform();
            q.radius = 2.5 + 5.0 * rng.uniform();
            q.beta = 0.5 * rng.uniform();
            q.top_absfrac = 1.0 - rng.uniform();
            q.bulk_abs = std::exp(std::log(1e-5) + (std::log(1e-3) - std::log(1e-5)) * rng.uniform());
            fd2_params_to_geometry(&q, &geoms[(size_t)gi]);
        }
        int32_t hist = 0;
        for (int gi = 0; gi < ng; ++gi)
            for (int32_t i = 0; i < per; ++i)
                add_clusters(b, rng, 1000.0 * (15.0 + 65.0 * rng.uniform()), geoms[(size_t)gi].det_height, ++hist,
                             (uint16_t)gi);
        return finish(b, hist, p, geoms, true, out);
    }
    default:
        return FD2_ERR_INVALID_ARGUMENT;
    }
}
