// fd2_host.h -- host-only helpers shared by the C-ABI translation units.
#pragma once

#include <cstdint>
#include <functional>
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

// Streaming EDE readers (fd2_io.cpp).  The sink gets consecutive pieces of at
// most `batch` events; a non-OK return stops the read and is returned.
// Text rows "x y z de hist" in cm / eV, as written by the EDE tally; '#'
// lines and blank lines skipped.
using TextSink = std::function<fd2_status(const double *x_cm, const double *y_cm, const double *z_cm,
                                          const double *de_ev, const int32_t *hist, int64_t n)>;
fd2_status stream_events_text(const char *path, int64_t batch, const TextSink &sink);
// Binary planar form of fd2_write_events_binary (um / eV).
struct BinHeader {
    int64_t n;
    int32_t num_hist, has_geom;
};
using BinHeaderSink = std::function<fd2_status(const BinHeader &)>;
using BinSink = std::function<fd2_status(const float *x_um, const float *y_um, const float *z_um, const float *e_ev,
                                         const int32_t *hist, const uint16_t *geom, int64_t n)>;
fd2_status stream_events_binary(const char *path, int64_t batch, const BinHeaderSink &on_header, const BinSink &sink);

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
