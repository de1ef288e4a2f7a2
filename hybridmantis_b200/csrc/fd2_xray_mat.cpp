// fd2_xray_mat.cpp -- material tables of the x-ray front end: the PENELOPE
// material data file reader, the library's own table format, the derived
// tables (electron CSDA range, Rayleigh screening) and the host copies of
// the kernels' interpolation.
//
// PENELOPE (2006) material files (example/CsI.mat) hold, besides the header
// (mass density, elements and atoms per molecule):
//   *** RELAX: Z, shells (designator, name, occupation, binding energy eV),
//       transitions (vacancy shell s0, filling shell s1, emitted-electron
//       shell s2 -- 0 for a radiative transition --, probability, energy eV);
//   *** Stopping powers for electrons and positrons: E, collision and
//       radiative mass stopping powers of electrons (MeV cm^2/g), then
//       positrons;
//   *** Electron and positron elastic cross sections: E, sigma0, sigma1
//       (first transport), sigma2 of electrons (cm^2 per molecule), then
//       positrons;
//   *** Rayleigh, Compton and pair-production cross sections: E, sigma
//       (cm^2 per molecule);
//   *** Photoelectric cross sections, IZ, NSHELL: E, total and per-subshell
//       sigma (cm^2 per atom); an absorption edge is a repeated energy.
// Everything else in the file (electron inelastic models, bremsstrahlung,
// elastic differential cross sections, positrons) is not used here.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>

#include "fd2_xray_internal.h"

namespace fd2x {

double atomic_weight(int Z)
{
    // standard atomic weights (g/mol), Z = 1..100
    static const double w[101] = {
        0,       1.008,   4.0026,  6.94,    9.0122,  10.81,   12.011,  14.007,  15.999,  18.998,  20.180,
        22.990,  24.305,  26.982,  28.085,  30.974,  32.06,   35.45,   39.948,  39.098,  40.078,  44.956,
        47.867,  50.942,  51.996,  54.938,  55.845,  58.933,  58.693,  63.546,  65.38,   69.723,  72.630,
        74.922,  78.971,  79.904,  83.798,  85.468,  87.62,   88.906,  91.224,  92.906,  95.95,   98.0,
        101.07,  102.91,  106.42,  107.87,  112.41,  114.82,  118.71,  121.76,  127.60,  126.90,  131.29,
        132.91,  137.33,  138.91,  140.12,  140.91,  144.24,  145.0,   150.36,  151.96,  157.25,  158.93,
        162.50,  164.93,  167.26,  168.93,  173.05,  174.97,  178.49,  180.95,  183.84,  186.21,  190.23,
        192.22,  195.08,  196.97,  200.59,  204.38,  207.2,   208.98,  209.0,   210.0,   222.0,   223.0,
        226.0,   227.0,   232.04,  231.04,  238.03,  237.0,   244.0,   243.0,   247.0,   247.0,   251.0,
        252.0,   257.0};
    return (Z >= 1 && Z <= 100) ? w[Z] : 0.0;
}

namespace {

// A piecewise log-log function with jumps at repeated abscissae.
struct Curve {
    std::vector<double> x, y;
};

// Value of a curve at u from the left (side 0) or the right (side 1) of a
// jump; log-log interpolation between nodes (linear where a value is 0).
double eval(const Curve &c, double u, int side)
{
    const auto &x = c.x;
    const size_t n = x.size();
    if (n == 0) return 0.0;
    if (u <= x[0]) return c.y[0];
    if (u >= x[n - 1]) return c.y[n - 1];
    // first node with x > u
    size_t hi = std::upper_bound(x.begin(), x.end(), u) - x.begin();
    size_t lo = hi - 1;
    if (x[lo] == u) {
        // u is a node: left limit = first node at u, right = last node at u
        size_t first = lo;
        while (first > 0 && x[first - 1] == u) --first;
        return side ? c.y[lo] : c.y[first];
    }
    const double y0 = c.y[lo], y1 = c.y[hi];
    const double t = std::log(u / x[lo]) / std::log(x[hi] / x[lo]);
    if (y0 > 0 && y1 > 0) return std::exp(std::log(y0) + t * (std::log(y1) - std::log(y0)));
    return y0 + t * (y1 - y0);
}

bool is_jump(const Curve &c, double u)
{
    auto it = std::lower_bound(c.x.begin(), c.x.end(), u);
    return it != c.x.end() && *it == u && (it + 1) != c.x.end() && *(it + 1) == u;
}

// I(b) = integral over mu in [-1, 1] of (1 + mu^2) / (1 + b (1 - mu))^4,
// by Simpson's rule in w = ln(1 + b t), t = 1 - mu.
double rayleigh_integral(double b)
{
    if (b < 1e-12) return 8.0 / 3.0;
    const int n = 2000;  // even
    const double W = std::log1p(2.0 * b), h = W / n;
    double s = 0.0;
    for (int i = 0; i <= n; ++i) {
        const double w = i * h;
        const double t = std::expm1(w) / b;
        const double f = (2.0 - 2.0 * t + t * t) * std::exp(-3.0 * w) / b;
        s += f * (i == 0 || i == n ? 1.0 : (i & 1) ? 4.0 : 2.0);
    }
    return s * h / 3.0;
}

bool read_lines(const std::string &path, std::vector<std::string> &lines, std::string &err)
{
    std::ifstream f(path);
    if (!f) {
        err = "cannot open " + path;
        return false;
    }
    std::string s;
    while (std::getline(f, s)) lines.push_back(s);
    return true;
}

bool starts_with_token(const std::string &s, const char *tok)
{
    return s.find(tok) != std::string::npos;
}

int int_after(const std::string &s, const char *key)
{
    const size_t p = s.find(key);
    if (p == std::string::npos) return -1;
    return std::atoi(s.c_str() + p + std::strlen(key));
}

}  // namespace

void finalize(Material &m)
{
    // Rayleigh screening per node: the b that makes the Thomson distribution
    // times (1 + b (1 - mu))^-4 give the node's cross section.
    double fz2 = 0.0;
    for (int k = 0; k < m.n_el(); ++k) fz2 += m.atoms[k] * (double)m.z[k] * (double)m.z[k];
    const double s0 = M_PI * kClassicalRadius * kClassicalRadius * fz2;
    const size_t n = m.e.size();
    m.ray_b.assign(n, 0.0);
    for (size_t i = 0; i < n; ++i) {
        const double sig = m.mu_r[i] / m.molecules_per_cm3;
        if (!(sig > 0.0) || sig >= s0 * (8.0 / 3.0)) continue;
        double lo = -40.0, hi = 40.0;  // ln b
        for (int it = 0; it < 200; ++it) {
            const double mid = 0.5 * (lo + hi);
            if (s0 * rayleigh_integral(std::exp(mid)) > sig) lo = mid;
            else hi = mid;
        }
        m.ray_b[i] = std::exp(0.5 * (lo + hi));
    }
    // equivalent screening radius at the node nearest 50 keV: b = 2 (a k)^2
    size_t best = 0;
    for (size_t i = 0; i < n; ++i)
        if (std::fabs(m.e[i] - 5e4) < std::fabs(m.e[best] - 5e4)) best = i;
    if (n) {
        const double k = m.e[best] / kHbarC;
        m.rayleigh_a = std::sqrt(m.ray_b[best] / 2.0) / k;
    }
}

bool load_penelope(const std::string &path, Material &m, std::string &err)
{
    std::vector<std::string> L;
    if (!read_lines(path, L, err)) return false;
    if (L.empty() || L[0].find("PENELOPE") == std::string::npos) {
        err = "not a PENELOPE material file: " + path;
        return false;
    }
    m = Material();
    Curve ray, com;
    std::vector<Curve> pe_tot, pe_sh;  // per element; pe_sh[el * kShells + s]
    std::vector<double> se, stot, el_e, el_s1;
    std::vector<int> relax_z;
    std::vector<std::vector<double>> relax_b;
    std::vector<std::vector<Material::Transition>> relax_t;
    std::vector<int> pe_z;
    size_t i = 0;
    int nel = -1;
    for (; i < L.size(); ++i) {
        const std::string &s = L[i];
        if (starts_with_token(s, "Mass density")) {
            const size_t p = s.find('=');
            m.density = std::atof(s.c_str() + p + 1);
        } else if (starts_with_token(s, "Number of elements in the molecule")) {
            const size_t p = s.find('=');
            nel = std::atoi(s.c_str() + p + 1);
            if (nel < 1 || nel > FD2_XRAY_MAX_ELEMENTS) {
                err = "unsupported number of elements";
                return false;
            }
            for (int k = 0; k < nel; ++k) {
                const std::string &t = L.at(++i);
                const int Z = int_after(t, "atomic number =");
                const size_t p2 = t.find("atoms/molecule =");
                if (Z < 1 || p2 == std::string::npos) {
                    err = "bad element line: " + t;
                    return false;
                }
                m.z.push_back(Z);
                m.atoms.push_back(std::atof(t.c_str() + p2 + 16));
            }
        } else if (starts_with_token(s, "*** RELAX:")) {
            const int Z = int_after(s, "Z =");
            const int nsh = int_after(s, "NO. OF SHELLS =");
            const int ntr = int_after(s, "NO. OF TRANSITIONS =");
            std::vector<double> b(kDesignators, 0.0);
            for (int k = 0; k < nsh; ++k) {
                int d = 0, occ = 0;
                char name[32];
                double e = 0;
                if (std::sscanf(L.at(++i).c_str(), "%d %31s %d %lf", &d, name, &occ, &e) != 4 || d < 1 ||
                    d >= kDesignators) {
                    err = "bad RELAX shell line";
                    return false;
                }
                b[d] = e;
            }
            std::vector<Material::Transition> tr;
            for (int k = 0; k < ntr; ++k) {
                Material::Transition t{};
                if (std::sscanf(L.at(++i).c_str(), "%d %d %d %lf %lf", &t.s0, &t.s1, &t.s2, &t.p, &t.e) != 5 ||
                    t.s0 < 1 || t.s0 >= kDesignators || t.s1 < 1 || t.s1 >= kDesignators || t.s2 < 0 ||
                    t.s2 >= kDesignators) {
                    err = "bad RELAX transition line";
                    return false;
                }
                tr.push_back(t);
            }
            relax_z.push_back(Z);
            relax_b.push_back(b);
            relax_t.push_back(tr);
        } else if (starts_with_token(s, "*** Stopping powers for electrons")) {
            const int nd = int_after(s, "NDATA =");
            for (int k = 0; k < nd; ++k) {
                double e, c, r, cp, rp;
                if (std::sscanf(L.at(++i).c_str(), "%lf %lf %lf %lf %lf", &e, &c, &r, &cp, &rp) != 5) {
                    err = "bad stopping-power line";
                    return false;
                }
                se.push_back(e);
                stot.push_back((c + r) * 1e6 * m.density);  // eV/cm
            }
        } else if (starts_with_token(s, "Electron and positron elastic cross sections")) {
            const int nd = int_after(s, "NDATA =");
            for (int k = 0; k < nd; ++k) {
                double e, s0, s1;
                if (std::sscanf(L.at(++i).c_str(), "%lf %lf %lf", &e, &s0, &s1) != 3) {
                    err = "bad elastic line";
                    return false;
                }
                el_e.push_back(e);
                el_s1.push_back(s1);
            }
        } else if (starts_with_token(s, "*** Rayleigh, Compton and pair-production")) {
            const int nd = int_after(s, "NDATA =");
            for (int k = 0; k < nd; ++k) {
                double e, r, c;
                if (std::sscanf(L.at(++i).c_str(), "%lf %lf %lf", &e, &r, &c) != 3) {
                    err = "bad Rayleigh/Compton line";
                    return false;
                }
                ray.x.push_back(e);
                ray.y.push_back(r);
                com.x.push_back(e);
                com.y.push_back(c);
            }
        } else if (starts_with_token(s, "Photoelectric cross sections")) {
            const int Z = int_after(s, "IZ =");
            const int nsh = int_after(s, "NSHELL =");
            const int nd = int_after(s, "NDATA =");
            if (nsh < 0 || nsh > 16 || nd < 2) {
                err = "bad photoelectric header";
                return false;
            }
            Curve tot;
            std::vector<Curve> sh(kShells);
            for (int k = 0; k < nd; ++k) {
                std::istringstream is(L.at(++i));
                double e, t;
                if (!(is >> e >> t)) {
                    err = "bad photoelectric line";
                    return false;
                }
                tot.x.push_back(e);
                tot.y.push_back(t);
                for (int q = 0; q < nsh; ++q) {
                    double v = 0;
                    is >> v;
                    if (q < kShells) {
                        sh[q].x.push_back(e);
                        sh[q].y.push_back(v);
                    }
                }
                for (int q = nsh; q < kShells; ++q) {
                    sh[q].x.push_back(e);
                    sh[q].y.push_back(0.0);
                }
            }
            pe_z.push_back(Z);
            pe_tot.push_back(tot);
            for (auto &c : sh) pe_sh.push_back(c);
        }
    }
    if (nel < 1 || !(m.density > 0) || ray.x.empty() || se.empty() || el_e.empty()) {
        err = "material file lacks a section this front end needs";
        return false;
    }
    // molecular weight and number density
    double M = 0;
    for (int k = 0; k < nel; ++k) {
        const double w = atomic_weight(m.z[k]);
        if (w <= 0) {
            err = "no atomic weight for Z = " + std::to_string(m.z[k]);
            return false;
        }
        M += m.atoms[k] * w;
    }
    m.molar_mass = M;
    m.molecules_per_cm3 = m.density * kAvogadro / M;
    const double N = m.molecules_per_cm3;
    // photoelectric tables in element order
    std::vector<int> pe_of(nel, -1), rx_of(nel, -1);
    for (int k = 0; k < nel; ++k) {
        for (size_t q = 0; q < pe_z.size(); ++q)
            if (pe_z[q] == m.z[k]) pe_of[k] = (int)q;
        for (size_t q = 0; q < relax_z.size(); ++q)
            if (relax_z[q] == m.z[k]) rx_of[k] = (int)q;
        if (pe_of[k] < 0 || rx_of[k] < 0) {
            err = "missing photoelectric or relaxation data for Z = " + std::to_string(m.z[k]);
            return false;
        }
    }
    // union photon grid over the common range, two nodes at every edge
    double lo = ray.x.front(), hi = ray.x.back();
    std::vector<double> u(ray.x.begin(), ray.x.end());
    for (int k = 0; k < nel; ++k) {
        const Curve &c = pe_tot[pe_of[k]];
        lo = std::max(lo, c.x.front());
        hi = std::min(hi, c.x.back());
        u.insert(u.end(), c.x.begin(), c.x.end());
    }
    std::sort(u.begin(), u.end());
    u.erase(std::unique(u.begin(), u.end()), u.end());
    for (double x : u) {
        if (x < lo || x > hi) continue;
        bool jump = false;
        for (int k = 0; k < nel; ++k) jump = jump || is_jump(pe_tot[pe_of[k]], x);
        for (int side = 0; side < (jump ? 2 : 1); ++side) {
            const int sd = jump ? side : 1;
            m.e.push_back(x);
            m.mu_r.push_back(N * eval(ray, x, sd));
            m.mu_c.push_back(N * eval(com, x, sd));
            for (int k = 0; k < nel; ++k) {
                const double na = N * m.atoms[k];
                m.mu_pe.push_back(na * eval(pe_tot[pe_of[k]], x, sd));
                for (int q = 0; q < kShells; ++q)
                    m.mu_sh.push_back(na * eval(pe_sh[pe_of[k] * kShells + q], x, sd));
            }
        }
    }
    // electron tables on the stopping-power nodes
    Curve S{se, stot}, s1{el_e, el_s1};
    m.ee = se;
    m.range.assign(se.size(), 0.0);
    m.lambda1.assign(se.size(), 0.0);
    m.range[0] = se[0] / stot[0];  // below the table: range proportional to energy
    for (size_t k = 1; k < se.size(); ++k) {
        // integral of dE / S over [e_{k-1}, e_k], Simpson in ln E
        const int n = 32;
        const double a = std::log(se[k - 1]), b = std::log(se[k]), h = (b - a) / n;
        double acc = 0;
        for (int j = 0; j <= n; ++j) {
            const double e = std::exp(a + j * h);
            const double f = e / eval(S, e, 1);
            acc += f * (j == 0 || j == n ? 1.0 : (j & 1) ? 4.0 : 2.0);
        }
        m.range[k] = m.range[k - 1] + acc * h / 3.0;
    }
    for (size_t k = 0; k < se.size(); ++k) m.lambda1[k] = 1.0 / (N * eval(s1, se[k], 1));
    // relaxation
    for (int k = 0; k < nel; ++k) {
        m.binding.push_back(relax_b[rx_of[k]]);
        m.trans.push_back(relax_t[rx_of[k]]);
    }
    finalize(m);
    return true;
}

bool save_table(const Material &m, const std::string &path, std::string &err)
{
    FILE *f = std::fopen(path.c_str(), "w");
    if (!f) {
        err = "cannot write " + path;
        return false;
    }
    const int nel = m.n_el();
    std::fprintf(f, "fd2-xray-material 1\n");
    std::fprintf(f, "density %.17g\nmolar_mass %.17g\nelements %d\n", m.density, m.molar_mass, nel);
    for (int k = 0; k < nel; ++k) std::fprintf(f, "%d %.17g\n", m.z[k], m.atoms[k]);
    std::fprintf(f, "photon_nodes %zu\n", m.e.size());
    for (size_t i = 0; i < m.e.size(); ++i) {
        std::fprintf(f, "%.17g %.17g %.17g", m.e[i], m.mu_r[i], m.mu_c[i]);
        for (int k = 0; k < nel; ++k) {
            std::fprintf(f, " %.17g", m.mu_pe[i * nel + k]);
            for (int q = 0; q < kShells; ++q) std::fprintf(f, " %.17g", m.mu_sh[(i * nel + k) * kShells + q]);
        }
        std::fprintf(f, "\n");
    }
    std::fprintf(f, "electron_nodes %zu\n", m.ee.size());
    for (size_t i = 0; i < m.ee.size(); ++i)
        std::fprintf(f, "%.17g %.17g %.17g\n", m.ee[i], m.range[i], m.lambda1[i]);
    for (int k = 0; k < nel; ++k) {
        int nb = 0;
        for (int d = 1; d < kDesignators; ++d) nb += m.binding[k][d] > 0;
        std::fprintf(f, "shells %d %d\n", m.z[k], nb);
        for (int d = 1; d < kDesignators; ++d)
            if (m.binding[k][d] > 0) std::fprintf(f, "%d %.17g\n", d, m.binding[k][d]);
        std::fprintf(f, "transitions %d %zu\n", m.z[k], m.trans[k].size());
        for (const auto &t : m.trans[k]) std::fprintf(f, "%d %d %d %.17g %.17g\n", t.s0, t.s1, t.s2, t.p, t.e);
    }
    std::fprintf(f, "end\n");
    const bool ok = std::fclose(f) == 0;
    if (!ok) err = "write failed: " + path;
    return ok;
}

bool load_table(const std::string &path, Material &m, std::string &err)
{
    std::ifstream f(path);
    if (!f) {
        err = "cannot open " + path;
        return false;
    }
    m = Material();
    std::string key;
    int ver = 0, nel = 0;
    if (!(f >> key >> ver) || key != "fd2-xray-material" || ver != 1) {
        err = "not an fd2 x-ray material table: " + path;
        return false;
    }
    auto bad = [&](const char *what) {
        err = std::string("bad material table (") + what + "): " + path;
        return false;
    };
    if (!(f >> key >> m.density) || key != "density") return bad("density");
    if (!(f >> key >> m.molar_mass) || key != "molar_mass") return bad("molar_mass");
    if (!(f >> key >> nel) || key != "elements" || nel < 1 || nel > FD2_XRAY_MAX_ELEMENTS) return bad("elements");
    m.z.resize(nel);
    m.atoms.resize(nel);
    for (int k = 0; k < nel; ++k)
        if (!(f >> m.z[k] >> m.atoms[k])) return bad("element");
    m.molecules_per_cm3 = m.density * kAvogadro / m.molar_mass;
    size_t n = 0;
    if (!(f >> key >> n) || key != "photon_nodes" || n < 2) return bad("photon_nodes");
    m.e.resize(n);
    m.mu_r.resize(n);
    m.mu_c.resize(n);
    m.mu_pe.resize(n * nel);
    m.mu_sh.resize(n * nel * kShells);
    for (size_t i = 0; i < n; ++i) {
        if (!(f >> m.e[i] >> m.mu_r[i] >> m.mu_c[i])) return bad("photon node");
        for (int k = 0; k < nel; ++k) {
            if (!(f >> m.mu_pe[i * nel + k])) return bad("photon node");
            for (int q = 0; q < kShells; ++q)
                if (!(f >> m.mu_sh[(i * nel + k) * kShells + q])) return bad("photon node");
        }
        if (i && m.e[i] < m.e[i - 1]) return bad("photon energies not ascending");
    }
    if (!(f >> key >> n) || key != "electron_nodes" || n < 2) return bad("electron_nodes");
    m.ee.resize(n);
    m.range.resize(n);
    m.lambda1.resize(n);
    for (size_t i = 0; i < n; ++i)
        if (!(f >> m.ee[i] >> m.range[i] >> m.lambda1[i])) return bad("electron node");
    m.binding.assign(nel, std::vector<double>(kDesignators, 0.0));
    m.trans.assign(nel, {});
    for (int k = 0; k < nel; ++k) {
        int Z = 0, nb = 0;
        if (!(f >> key >> Z >> nb) || key != "shells" || Z != m.z[k]) return bad("shells");
        for (int j = 0; j < nb; ++j) {
            int d = 0;
            double e = 0;
            if (!(f >> d >> e) || d < 1 || d >= kDesignators) return bad("shell");
            m.binding[k][d] = e;
        }
        size_t nt = 0;
        if (!(f >> key >> Z >> nt) || key != "transitions" || Z != m.z[k]) return bad("transitions");
        for (size_t j = 0; j < nt; ++j) {
            Material::Transition t{};
            if (!(f >> t.s0 >> t.s1 >> t.s2 >> t.p >> t.e) || t.s0 < 1 || t.s0 >= kDesignators || t.s1 < 1 ||
                t.s1 >= kDesignators || t.s2 < 0 || t.s2 >= kDesignators)
                return bad("transition");
            m.trans[k].push_back(t);
        }
    }
    if (!(f >> key) || key != "end") return bad("end");
    finalize(m);
    return true;
}

namespace {

// Node interval of a photon energy: k with e[k] <= E < e[k+1] (never a
// zero-width edge interval), and the log-log weight.
void photon_interval(const Material &m, double E, size_t *k, double *w)
{
    const size_t n = m.e.size();
    if (E <= m.e[0]) {
        *k = 0;
        *w = 0;
        return;
    }
    if (E >= m.e[n - 1]) {
        *k = n - 2;
        *w = 1;
        return;
    }
    const size_t hi = std::upper_bound(m.e.begin(), m.e.end(), E) - m.e.begin();
    *k = hi - 1;
    *w = std::log(E / m.e[*k]) / std::log(m.e[hi] / m.e[*k]);
}

double loglog(double y0, double y1, double w)
{
    const double a = std::log(std::max(y0, 1e-300)), b = std::log(std::max(y1, 1e-300));
    return std::exp(a + w * (b - a));
}

}  // namespace

void attenuation(const Material &m, double E, double out[4])
{
    size_t k;
    double w;
    photon_interval(m, E, &k, &w);
    const int nel = m.n_el();
    out[0] = loglog(m.mu_r[k], m.mu_r[k + 1], w);
    out[1] = loglog(m.mu_c[k], m.mu_c[k + 1], w);
    double pe = 0;
    for (int q = 0; q < nel; ++q) pe += loglog(m.mu_pe[k * nel + q], m.mu_pe[(k + 1) * nel + q], w);
    out[2] = pe;
    out[3] = out[0] + out[1] + out[2];
}

void electron_at(const Material &m, double E, double *range, double *lambda1)
{
    const size_t n = m.ee.size();
    if (E <= m.ee[0]) {
        *range = m.range[0] * E / m.ee[0];
        *lambda1 = m.lambda1[0];
        return;
    }
    size_t hi = std::upper_bound(m.ee.begin(), m.ee.end(), E) - m.ee.begin();
    if (hi >= n) hi = n - 1;
    const size_t k = hi - 1;
    const double w = std::log(E / m.ee[k]) / std::log(m.ee[hi] / m.ee[k]);
    *range = loglog(m.range[k], m.range[hi], w);
    *lambda1 = loglog(m.lambda1[k], m.lambda1[hi], w);
}

}  // namespace fd2x

extern "C" FD2_API fd2_status fd2_xray_read_penEasy_source(const char *path, fd2_xray_source *src, double *e_ev,
                                                           double *prob, int32_t cap)
{
    if (!path || !src || !e_ev || !prob || cap < 2) return FD2_ERR_INVALID_ARGUMENT;
    std::ifstream f(path);
    if (!f) return FD2_ERR_IO;
    std::string line;
    bool found = false;
    while (std::getline(f, line))
        if (line.find("[SECTION SOURCE BOX ISOTROPIC GAUSS SPECTRUM") != std::string::npos) {
            found = true;
            break;
        }
    if (!found || !std::getline(f, line)) return FD2_ERR_PARSE;
    // status field "(ON )": the three characters after the first
    const std::string st = line.size() >= 4 ? line.substr(1, 3) : "";
    if (st.find("ON") == std::string::npos) return FD2_ERR_PARSE;
    auto nums = [&](int k, double *v) {
        if (!std::getline(f, line)) return false;
        std::istringstream is(line);
        for (int i = 0; i < k; ++i)
            if (!(is >> v[i])) return false;
        return true;
    };
    double v[3];
    if (!nums(1, v)) return FD2_ERR_PARSE;
    fd2_xray_source s{};
    s.particle = (int32_t)v[0];
    if (!std::getline(f, line)) return FD2_ERR_PARSE;  // the spectrum's title line
    int n = 0;
    for (;;) {
        if (!nums(2, v) || n >= cap) return FD2_ERR_PARSE;
        e_ev[n] = v[0];
        prob[n] = v[1];
        ++n;
        if (v[1] < 0.0) break;
    }
    s.n_spectrum = n;
    s.e_ev = e_ev;
    s.prob = prob;
    if (!nums(3, s.center_cm) || !nums(3, s.sides_cm) || !nums(3, s.euler_deg)) return FD2_ERR_PARSE;
    if (!nums(1, v) || v[0] != 0.0) return FD2_ERR_PARSE;  // source material: only 0 (any) is supported
    if (!nums(3, s.direction) || !nums(1, v)) return FD2_ERR_PARSE;
    s.semiaperture_deg = v[0];
    *src = s;
    return FD2_OK;
}

