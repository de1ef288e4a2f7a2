// fd2_xray_internal.h -- the x-ray front end's material tables (host) and
// the flat views its kernels read.  Not installed; include/fd2_xray.h is the
// public surface.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "fd2_xray.h"

namespace fd2x {

constexpr int kShells = 9;        // photoelectric subshells K, L1-L3, M1-M5 (PENELOPE designators 1..9)
constexpr int kDesignators = 31;  // relaxation shell designators 1..30 (30: outer shells)
constexpr double kElectronMass = 510998.918;        // m c^2, eV
constexpr double kClassicalRadius = 2.8179403262e-13;  // r_e, cm
constexpr double kHbarC = 1.973269804e-5;           // hbar c, eV cm
constexpr double kAvogadro = 6.02214076e23;

// The tables one material contributes (all energies in eV, lengths in cm).
struct Material {
    double density = 0;
    double molar_mass = 0;
    double molecules_per_cm3 = 0;
    std::vector<int> z;
    std::vector<double> atoms;  // per molecule

    // photon nodes: energies ascending; an absorption edge appears as two
    // nodes at the same energy (values below, then above the edge)
    std::vector<double> e;
    std::vector<double> mu_r, mu_c;     // 1/cm
    std::vector<double> ray_b;          // Rayleigh screening: b = 2 (a k)^2 at each node
    std::vector<double> mu_pe;          // [node][element]: total photoelectric, 1/cm
    std::vector<double> mu_sh;          // [node][element][kShells]: per subshell, 1/cm

    // electron nodes (ascending energies): CSDA range, first transport mfp
    std::vector<double> ee, range, lambda1;

    // relaxation, per element: binding energies of designators 1..30 (0:
    // unknown) and the transitions (s0, s1, s2, probability, energy)
    struct Transition {
        int s0, s1, s2;
        double p, e;
    };
    std::vector<std::vector<double>> binding;       // [element][kDesignators]
    std::vector<std::vector<Transition>> trans;     // [element]

    double rayleigh_a = 0;   // equivalent screening radius at the fitted energies (info only)

    int n_el() const { return (int)z.size(); }
};

// Molar mass of element Z (standard atomic weight, g/mol); 0 if unknown.
double atomic_weight(int Z);
// Build the derived tables (Rayleigh screening) once the raw ones are set.
void finalize(Material &m);
// Parsers / writer.
bool load_penelope(const std::string &path, Material &m, std::string &err);
bool load_table(const std::string &path, Material &m, std::string &err);
bool save_table(const Material &m, const std::string &path, std::string &err);
// Host evaluation (the same interpolation the kernels use).
void attenuation(const Material &m, double e, double out[4]);
void electron_at(const Material &m, double e, double *range, double *lambda1);

}  // namespace fd2x

struct fd2_xray_material {
    fd2x::Material m;
};
