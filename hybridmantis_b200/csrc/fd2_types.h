// fd2_types.h -- types and constants shared by host and device code.
#pragma once

#include <cstdint>

namespace fd2 {

constexpr float kEps = 8.1929093e-6f;      // the reference's float-comparison epsilon
constexpr float kCos157 = 7.9632671e-4f;   // cos(1.57): acos(c) > 1.57  <=>  c < kCos157
constexpr float kPi = 3.14159265358979f;
constexpr uint32_t kCountStream = 0xFFFFFFFFu; // Philox counter word for photon-count draws

enum Fate : int {
    kAlive = 0,
    kDetect = 1,
    kAbsTop = 2,
    kAbsBulk = 3,
    kLost = 4,
    kOutOfCol = 5,
    kTheta1 = 6,
    kCapped = 7,
    kNumFates = 8
};

// Safety caps: the reference loops are unbounded in principle; these are
// far beyond anything a physical walk reaches and turn a runaway photon
// into the `capped` fate instead of a hung kernel.
constexpr uint32_t kMaxBoundaryCalls = 1u << 20;  // boundary interactions per photon
constexpr int kMaxSurfaceLoops = 1 << 16;         // Fresnel/hop cycles per interaction
constexpr int kMaxTopLoops = 1 << 12;             // top/sensor ping-pong per hop
constexpr int kMaxGridCells = 1 << 14;            // lattice cells one gap flight may cross

// One detector geometry, in the float form the walk uses.
struct DevGeom {
    float xdet, ydet, H, half, R, beta, top_absfrac, neg_inv_mu, d_min, d_span;
    float lb_x, lb_y, ub_x, ub_y, sensor_refl, pixel;
    float cct_band_lo;  // H/2 - 0.2 H: crosstalk is certain above it
    float cct_k_hi;     // 1 / (2 (H/2 - 0.2 H)) for 0 <= z < band
    float cct_k_lo;     // 1 / (2 (-H/2))        for -H/2 <= z < 0
    float eta_in;       // n_col / n_gap (leaving a column)
    float cos_tir_in;   // inside: total internal reflection iff cos(t_i) < this
    float eta_out;      // n_gap / n_col (entering a column)
    float cos_tir_out;  // outside, low-contrast rule: TIR iff cos(t_i) < this
    int stale_out;      // n_col/n_gap < 1.57: outside Fresnel decides only TIR
    int xdim, ydim;
    long long prf_offset;  // first PRF element of this geometry
    // the reference's float parameters, as given (used by the replay)
    float mu, n_col, n_gap, d_max;
    // explicit column lattice (options.column_grid; no counterpart in the
    // reference): 0 = off, 1 = square lattice of columns centred at
    // ((i + 1/2) pitch, (j + 1/2) pitch), pitch = 2 R + gap
    int grid;
    float pitch;
};

}  // namespace fd2
