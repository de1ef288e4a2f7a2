// fd2_host.h -- host-only helpers shared by the C-ABI translation units.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "fd2.h"

namespace fd2host {

fd2_status events_from_vectors(const std::vector<float> &x, const std::vector<float> &y, const std::vector<float> &z,
                               const std::vector<float> &e, const std::vector<int32_t> &h, int32_t num_hist,
                               fd2_events *out);

// detected_/myimage_ + the ten raw tags joined with '_' + ".dat"
std::string output_name(const fd2_params &p, const char *prefix);
std::string format_prf(const uint64_t *image, int32_t xdim, int32_t ydim, const fd2_geometry &g, double num_hist);
std::string format_phs(const int32_t *bins, int32_t num_bins);
fd2_status write_new_file(const std::string &path, const std::string &data);

// xoshiro256** (Blackman & Vigna, 2018) seeded through splitmix64.
struct HostRng {
    uint64_t s[4];
    explicit HostRng(uint64_t seed);
    uint64_t next();
    double uniform();                   // (0, 1)
    double normal();                    // N(0, 1), polar Box-Muller
    double trunc_exp(double mean, double upper);
    double triangular(double a, double c, double b);
    int poisson_small(double mu);       // Knuth's product method, small mu
};

}  // namespace fd2host
