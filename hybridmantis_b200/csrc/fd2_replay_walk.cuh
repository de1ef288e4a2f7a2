// fd2_replay_walk.cuh -- the reference-arithmetic walker of the replay
// (see fd2_replay.cu).  Host-compilable so that tests can run the same code
// on the CPU; the product runs it only on the GPU.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>

#include "fd2_types.h"

#if defined(__CUDACC__)
#define FD2_HD __host__ __device__
#else
#define FD2_HD
#endif

namespace fd2 {
namespace replay {

using std::acos;
using std::asin;
using std::cos;
using std::fabs;
using std::floor;
using std::log;
using std::sin;
using std::sqrt;
using std::tan;

using D = double;
constexpr D kRefEps = 8.1929093e-6;  // a double literal in the reference
constexpr D kRefTwoPi = 6.283185308;
constexpr D kRefPi = 3.14159265;

struct Ranecu {
    int32_t s0, s1;
    FD2_HD float u()
    {
        int32_t k = s0 / 53668;
        s0 = 40014 * (s0 - k * 53668) - k * 12211;
        k = s1 / 52774;
        s1 = 40692 * (s1 - k * 52774) - k * 3791;
        if (s0 < 0) s0 += 2147483563;
        if (s1 < 0) s1 += 2147483399;
        int32_t z = s0 - s1;
        if (z < 1) z += 2147483562;
        return (float)z * (float)(1.0 / 2147483563.0);
    }
};

FD2_HD int64_t powmod(int64_t b, uint64_t e, int64_t m)
{
    int64_t r = 1;
    b %= m;
    while (e) {
        if (e & 1) r = (r * b) % m;
        b = (b * b) % m;
        e >>= 1;
    }
    return r;
}

FD2_HD Ranecu ranecu_seed(int64_t index, int32_t seed_input)
{
    const uint64_t leap = (uint64_t)(index + 1) * 50000ull * 1000ull;
    Ranecu r;
    r.s0 = (int32_t)(((int64_t)seed_input * powmod(40014, leap, 2147483563)) % 2147483563);
    r.s1 = (int32_t)(((int64_t)seed_input * powmod(40692, leap, 2147483399)) % 2147483399);
    return r;
}

template <typename T>
struct Walk {
    const DevGeom *g;
    Ranecu rng;
    T p[3], d[3], n[3];
    T xc, yc;
    uint64_t rebound;
    int absorbed, detect, bulk_abs;
    D ex, ey, ez;  // event position (double, as struct start_info)
    int fate, pi, pj;
    // geometry in T
    T xdet, ydet, H, R, ncol, ngap, top, mu, beta, dmin, dmax, lbx, lby, ubx, uby, srefl;
    int pixel;

    FD2_HD T u() { return (T)rng.u(); }
    // Float acosf/asinf of the reference C: the float rounding of the double
    // function, moved by one ulp where the C library's float function
    // differs (tables of fd2_libm_table.c, inputs in [0, 1]).
    const uint32_t *acos_tab = nullptr, *asin_tab = nullptr;
    uint32_t n_acos = 0, n_asin = 0;

    FD2_HD static uint32_t bits(float f)
    {
        uint32_t u;
        memcpy(&u, &f, 4);
        return u;
    }
    FD2_HD static float from_bits(uint32_t u)
    {
        float f;
        memcpy(&f, &u, 4);
        return f;
    }
    FD2_HD static float corrected(float r, float x, const uint32_t *tab, uint32_t n)
    {
        if (!tab || !(x >= 0.0f && x <= 1.0f)) return r;
        const uint32_t key = bits(x);
        uint32_t lo = 0, hi = n;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if ((tab[mid] & 0x7FFFFFFFu) < key) lo = mid + 1;
            else hi = mid;
        }
        if (lo < n && (tab[lo] & 0x7FFFFFFFu) == key) r = from_bits(bits(r) + ((tab[lo] >> 31) ? 0xFFFFFFFFu : 1u));
        return r;
    }
    FD2_HD T acos_t(T x) const
    {
        const T r = (T)acos((D)x);
        return sizeof(T) == 4 ? (T)corrected((float)r, (float)x, acos_tab, n_acos) : r;
    }
    FD2_HD T asin_t(T x) const
    {
        const T r = (T)asin((D)x);
        return sizeof(T) == 4 ? (T)corrected((float)r, (float)x, asin_tab, n_asin) : r;
    }

    FD2_HD void renorm(T *v)
    {
        const T nrm = (T)sqrt((D)(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]));
        if ((D)nrm < 1.0 - kRefEps || (D)nrm > 1.0 + kRefEps) {
            v[0] = v[0] / nrm;
            v[1] = v[1] / nrm;
            v[2] = v[2] / nrm;
        }
    }

    FD2_HD void emit(bool first)
    {
        T c = (u() * T(2)) - T(1);
        T rr;
        if (first) {
            for (int t = 0; t < 4096 && fabs((D)c) <= (D)T(0.01f); ++t) c = (u() * T(2)) - T(1);
            rr = (T)sqrt((D)(T(1) - c * c));
        } else {
            rr = (T)sqrt(1.0 - (D)(c * c));
        }
        const T phi = (T)((D)u() * kRefTwoPi);
        d[2] = c;
        d[0] = (T)((D)rr * cos((D)phi));
        d[1] = (T)((D)rr * sin((D)phi));
        renorm(d);
    }

    FD2_HD void rough(T b)
    {
        T uu = u();
        T qz = T(2) * uu - T(1);
        const T rr = (T)sqrt((D)(T(1) - uu * uu));
        uu = u();
        const T phi = (T)((D)(uu * T(2)) * kRefPi);
        T qx = (T)((D)rr * cos((D)phi));
        T qy = (T)((D)rr * sin((D)phi));
        T len = (T)sqrt((D)qx * (D)qx + (D)qy * (D)qy + (D)qz * (D)qz);
        qx = qx / len;
        qy = qy / len;
        qz = qz / len;
        const T r0 = b * qx + n[0], r1 = b * qy + n[1], r2 = b * qz + n[2];
        len = (T)sqrt((D)r0 * (D)r0 + (D)r1 * (D)r1 + (D)r2 * (D)r2);
        n[0] = r0 / len;
        n[1] = r1 / len;
        n[2] = r2 / len;
    }

    FD2_HD static T dot(const T *a, const T *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

    FD2_HD void redirect(T ti, T tt, int refract)
    {
        const T inv[3] = {-d[0], -d[1], -d[2]};
        const T ci = dot(inv, n);
        if (!refract) {
            for (int k = 0; k < 3; ++k) d[k] = T(2) * ci * n[k] + d[k];
        } else {
            const D ct = cos((D)tt), ratio = sin((D)tt) / sin((D)ti);
            for (int k = 0; k < 3; ++k) d[k] = (T)((D)(-n[k]) * ct - ratio * (D)(d[k] + (ci * n[k])));
        }
        renorm(d);
    }

    FD2_HD void set_fate(int f) { fate = f; }

    FD2_HD void detected()
    {
        fate = kDetect;
        const int ii = (int)floor((D)((p[0] - lbx) / (T)pixel));
        const int jj = (int)floor((D)((p[1] - lby) / (T)pixel));
        pi = -1;
        pj = -1;
        if (p[0] <= ubx && p[1] <= uby && p[0] >= lbx && p[1] >= lby) {
            pi = ii;
            pj = jj;
        }
    }

    FD2_HD bool outside_detector() const
    {
        return ((D)p[0] < kRefEps) || (p[0] > xdet) || ((D)p[1] < kRefEps) || (p[1] > ydet) ||
               (p[2] < -H / T(2)) || (p[2] > H / T(2));
    }
    FD2_HD bool outside_xy() const
    {
        return (D)p[0] < kRefEps || p[0] > xdet || (D)p[1] < kRefEps || p[1] > ydet;
    }
    FD2_HD T radius() const
    {
        return (T)sqrt((D)((p[0] - xc) * (p[0] - xc) + (p[1] - yc) * (p[1] - yc)));
    }

    FD2_HD T to_wall()
    {
        const T s0 = p[0], s1 = p[1], s2 = p[2];
        if (rebound == 0) {
            xc = (T)ex;
            yc = (T)ey;
        }
        const T qa = d[0] * d[0] + d[1] * d[1];
        const T qb = T(2) * (((p[0] - xc) * d[0]) + ((p[1] - yc) * d[1]));
        const T qc = (p[0] - xc) * (p[0] - xc) + (p[1] - yc) * (p[1] - yc) - (R * R);
        const D root = sqrt((D)((qb * qb) - (T(4) * qa * qc)));
        const T r1 = (T)(((D)(-qb) + root) / (D)(T(2) * qa));
        const T r2 = (T)(((D)(-qb) - root) / (D)(T(2) * qa));
        T dcyl = T(999);
        if (r1 >= r2) dcyl = r1;
        else if (r2 > r1) dcyl = r2;
        T dist;
        if (d[2] != T(0)) {
            const T zp = d[2] > T(0) ? H / T(2) : -H / T(2);
            const T axis = d[2] > T(0) ? T(1) : T(-1);
            const bool straight = fabs((D)d[0]) < kRefEps && fabs((D)d[1]) < kRefEps && fabs((D)(d[2] - axis)) < kRefEps;
            const T dplane = (zp - p[2]) / d[2];
            if (!straight && dplane >= dcyl) {
                dist = dcyl;
                p[2] = s2 + dist * d[2];
            } else {
                dist = dplane;
                p[2] = zp;
            }
        } else {
            dist = dcyl;
            p[2] = s2 + dist * d[2];
        }
        p[0] = s0 + dist * d[0];
        p[1] = s1 + dist * d[1];
        if (outside_detector()) {
            set_fate(kLost);
            return T(-99);
        }
        T r = radius();
        T step = T(0.5f);
        int moved = 0, halved = 0;
        while ((D)r > (D)R - 1e-5 && moved < 10 && halved < 10) {
            const T sx = p[0], sy = p[1];
            p[0] = p[0] + step * (-d[0]);
            p[1] = p[1] + step * (-d[1]);
            const T r2n = radius();
            if (r2n > r) {
                p[0] = sx;
                p[1] = sy;
                step = step / T(2);
                halved++;
            } else {
                r = r2n;
                moved++;
            }
        }
        if ((D)r > (D)R - 1e-5) {
            set_fate(kOutOfCol);
            return T(-99);
        }
        if (outside_detector()) {
            set_fate(kLost);
            return T(-99);
        }
        return dist;
    }

    FD2_HD int flight()
    {
        const T dsurf = to_wall();
        T dabs = T(999999);
        if (mu > T(0)) dabs = (T)((D)(T(-1) / mu) * log((D)u()));
        if (fabs((D)(dsurf - T(-99))) < kRefEps) return 1;
        if (dsurf < dabs && dsurf >= T(0)) return 0;
        if (dsurf >= dabs && dsurf >= T(0)) {
            set_fate(kAbsBulk);
            return 1;
        }
        return 0;
    }

    FD2_HD int sensor()
    {
        if (fabs((D)(p[2] - (T)(-H / T(2)))) >= kRefEps) return 0;
        if (u() < srefl) {
            n[0] = T(0); n[1] = T(0); n[2] = T(1);
            redirect(T(0), T(0), 0);
            return flight() == 1;
        }
        detected();
        return 1;
    }

    FD2_HD int next_column_normal(const T *inv, int *tries, bool always_rough)
    {
        for (;;) {
            n[0] = inv[0]; n[1] = inv[1]; n[2] = inv[2];
            rough(T(1));
            const T den = (T)sqrt((D)(n[0] * n[0] + n[1] * n[1]));
            n[2] = T(0);
            n[0] = n[0] / den;
            n[1] = n[1] / den;
            if (always_rough || beta > T(0)) rough(beta);
            const T ang = acos_t(dot(inv, n));
            if (!(ang < T(0) || ang > T(1.57f))) return 0;
            if (*tries < 100) {
                (*tries)++;
                continue;
            }
            set_fate(kTheta1);
            return 1;
        }
    }

    FD2_HD int hop_from_sensor()
    {
        const T s[3] = {p[0], p[1], p[2]};
        const T inv[3] = {-d[0], -d[1], -d[2]};
        const T hop = u() * (dmax - dmin) + dmin;
        const T dtop = ((H / T(2)) - s[2]) / d[2];
        for (int k = 0; k < 3; ++k) p[k] = s[k] + d[k] * hop;
        if (outside_xy()) {
            set_fate(kLost);
            return 1;
        }
        if (p[2] > H / T(2)) {
            if (dtop < hop && (D)dtop > kRefEps) {
                p[0] = s[0] + d[0] * dtop;
                p[1] = s[1] + d[1] * dtop;
                p[2] = H / T(2);
                return 0;
            }
            set_fate(kLost);
            return 1;
        }
        int tries = 0;
        return next_column_normal(inv, &tries, true);
    }

    FD2_HD bool at_top() const { return fabs((D)(p[2] - (H / T(2)))) < kRefEps && d[2] > T(0); }

    FD2_HD int sensor_between()
    {
        if (u() < srefl) {
            n[0] = T(0); n[1] = T(0); n[2] = T(1);
            redirect(T(0), T(0), 0);
            if (hop_from_sensor()) return 1;
            return at_top() ? 2 : 0;
        }
        detected();
        return 1;
    }

    FD2_HD void top_reflect()
    {
        d[2] = (T)(-fabs((D)((u() * T(2)) - T(1))));
        const T rr = (T)sqrt((D)(T(1) - d[2] * d[2]));
        const T phi = (T)((D)u() * kRefTwoPi);
        d[0] = (T)((D)rr * cos((D)phi));
        d[1] = (T)((D)rr * sin((D)phi));
    }

    FD2_HD int leave_column(int crosstalk)
    {
        T s[3] = {p[0], p[1], p[2]};
        T inv[3] = {-d[0], -d[1], -d[2]};
        int tries = 0, tries_top = 0;
        if (crosstalk) return next_column_normal(inv, &tries, false);
        const T half = H / T(2);
        T hop = u() * (dmax - dmin) + dmin;
        for (int k = 0; k < 3; ++k) p[k] = s[k] + d[k] * hop;
        const T dtop = (half - s[2]) / d[2];
        T dbot = ((-H / T(2)) - s[2]) / d[2];
        if (outside_xy()) {
            set_fate(kLost);
            return 1;
        }
        int to_top = 0;
        if (p[2] < -H / T(2) || p[2] > half) {
            if (dtop < hop && (D)dtop > kRefEps) {
                p[0] = s[0] + d[0] * dtop;
                p[1] = s[1] + d[1] * dtop;
                p[2] = half;
            } else if (dbot < hop && (D)dbot > kRefEps) {
                p[0] = s[0] + d[0] * dbot;
                p[1] = s[1] + d[1] * dbot;
                p[2] = -H / T(2);
                const int r = sensor_between();
                if (r == 1) return 1;
                to_top = (r == 2);
            } else {
                set_fate(kLost);
                return 1;
            }
        }
        if (!to_top) {
            if (next_column_normal(inv, &tries, false)) return 1;
            if (fabs((D)(p[0] - T(0))) < kRefEps || fabs((D)(p[0] - xdet)) < kRefEps ||
                fabs((D)(p[1] - T(0))) < kRefEps || fabs((D)(p[1] - ydet)) < kRefEps) {
                set_fate(kLost);
                return 1;
            }
        }
        for (int loop = 0; loop < kMaxTopLoops; ++loop) {
            if (at_top()) {
                n[0] = T(0); n[1] = T(0); n[2] = T(-1);
                if (top > T(0) && u() < top) {
                    set_fate(kAbsTop);
                    return 1;
                }
                top_reflect();
                for (int k = 0; k < 3; ++k) {
                    s[k] = p[k];
                    inv[k] = -d[k];
                }
                hop = u() * (dmax - dmin) + dmin;
                dbot = ((-H / T(2)) - s[2]) / d[2];
                for (int k = 0; k < 3; ++k) p[k] = s[k] + d[k] * hop;
                if (outside_xy()) {
                    set_fate(kLost);
                    return 1;
                }
                if (p[2] < -H / T(2) || p[2] > half) {
                    if (dbot < hop && (D)dbot > kRefEps) {
                        p[0] = s[0] + d[0] * dbot;
                        p[1] = s[1] + d[1] * dbot;
                        p[2] = -H / T(2);
                        const int r = sensor_between();
                        if (r == 1) return 1;
                        if (r == 2) continue;
                    } else {
                        set_fate(kLost);
                        return 1;
                    }
                }
                if (next_column_normal(inv, &tries_top, false)) return 1;
            }
            if (fabs((D)(p[2] - (-H / T(2)))) < kRefEps) {
                const int r = sensor_between();
                if (r == 1) return 1;
                if (r == 2) continue;
            }
            return 0;
        }
        set_fate(kCapped);
        return 1;
    }

    FD2_HD static void fresnel(T t1, T t2, T *pr, T *pt)
    {
        const D dm = (D)(t1 - t2), dp = (D)(t1 + t2);
        const D s2 = sin((D)(T(2) * t1)) * sin((D)(T(2) * t2));
        const D tm = tan(dm), tp = tan(dp), sm = sin(dm), sp = sin(dp), cm = cos(dm);
        *pr = (T)((D)T(0.5f) * (((tm * tm) / (tp * tp)) + ((sm * sm) / (sp * sp))));
        *pt = (T)((D)T(0.5f) * ((s2 / ((sp * sp) * (cm * cm))) + (s2 / (sp * sp))));
    }

    FD2_HD int surface()
    {
        const T half = H / T(2);
        if (fabs((D)(p[2] - (T)(H / T(2)))) < kRefEps && d[2] > T(0)) {
            if (top > T(0) && u() < top) {
                set_fate(kAbsTop);
                return 1;
            }
            n[0] = T(0); n[1] = T(0); n[2] = T(-1);
            top_reflect();
            return 0;
        }
        const T band = H * T(0.2f);
        T cct = T(0);
        if (p[2] <= half && p[2] >= (half - band)) cct = T(1);
        else if (p[2] < (half - band) && p[2] >= T(0)) cct = (T)((D)(p[2] / (T(2) * (half - band))) + 0.5);
        else if (p[2] < T(0) && p[2] >= (-H / T(2)))
            cct = (T)((D)((p[2] - (-H / T(2))) / (T(2) * (-H / T(2)))) + 1.0);
        if (u() < cct) {
            if (leave_column(1)) return 1;
            xc = (T)(p[0] + R * (-n[0]));
            yc = (T)(p[1] + R * (-n[1]));
            return 0;
        }
        int outside = 0, tries_theta = 0, tries_normal = 0, reperturbs = 0, smooth = 0;
        T pr = T(0), pt = T(0), t1 = T(0), t2 = T(0);
        T kn[3], kd[3], inv[3];
        int stage = 0;  // 0 new surface, 1 restore, 2 incidence
        for (int loop = 0; loop < kMaxSurfaceLoops; ++loop) {
            if (stage == 0) {
                if (!outside) {
                    const T mag = (T)sqrt((D)(((xc - p[0]) * (xc - p[0])) + ((yc - p[1]) * (yc - p[1]))));
                    n[0] = (xc - p[0]) / mag;
                    n[1] = (yc - p[1]) / mag;
                    n[2] = T(0);
                    if (beta > T(0)) rough(beta);
                } else {
                    xc = (T)(p[0] + R * (-n[0]));
                    yc = (T)(p[1] + R * (-n[1]));
                }
                for (int k = 0; k < 3; ++k) {
                    kn[k] = n[k];
                    kd[k] = d[k];
                }
                stage = 1;
            }
            if (stage == 1) {
                for (int k = 0; k < 3; ++k) {
                    n[k] = kn[k];
                    d[k] = kd[k];
                }
                if (reperturbs != 0 && beta > T(0)) rough(beta);
                if (reperturbs != 0 && outside) {
                    xc = (T)(p[0] + R * (-n[0]));
                    yc = (T)(p[1] + R * (-n[1]));
                }
                stage = 2;
            }
            for (int k = 0; k < 3; ++k) inv[k] = -d[k];
            t1 = dot(inv, n);
            if (t1 > T(1) || t1 < T(0)) {
                if (outside && next_column_normal(inv, &tries_normal, false)) return 1;
                if (tries_theta < 100) {
                    tries_theta++;
                    stage = 0;
                    continue;
                }
                set_fate(kTheta1);
                return 1;
            }
            t1 = acos_t(t1);
            if (!outside) {
                if ((D)t1 > asin((D)(ngap / ncol))) {
                    pr = T(1);
                    pt = T(0);
                } else {
                    if ((D)t1 < kRefEps) t1 = (T)0.00042;
                    t2 = asin_t((T)((D)(T)(ncol / ngap) * sin((D)t1)));
                    fresnel(t1, t2, &pr, &pt);
                }
            } else if ((ncol / ngap) < T(1.57f)) {
                if ((D)t1 > asin((D)(ncol / ngap))) {
                    pr = T(1);
                    pt = T(0);
                }
            } else if ((D)t1 < kRefEps) {
                t1 = (T)0.00042;
                t2 = asin_t((T)((D)(T)(ncol / ngap) * sin((D)t1)));
                fresnel(t1, t2, &pr, &pt);
            } else {
                t2 = asin_t((T)((D)(T)(ngap / ncol) * sin((D)t1)));
                fresnel(t1, t2, &pr, &pt);
            }
            const T total = pr + pt;
            pr = pr / total;
            pt = pt / total;
            if (u() < pr) {
                redirect(t1, t2, 0);
                if (acos_t(dot(kn, d)) > T(1.57f)) {
                    reperturbs++;
                    if (reperturbs < 4) {
                        stage = 1;
                        continue;
                    }
                    for (int k = 0; k < 3; ++k) {
                        n[k] = kn[k];
                        d[k] = kd[k];
                    }
                    reperturbs = 0;
                    if (smooth < 25) {
                        smooth++;
                        stage = 2;
                        continue;
                    }
                    set_fate(kTheta1);
                    return 1;
                }
                if (!outside) return 0;
                if (leave_column(0)) return 1;
                stage = 0;
                continue;
            }
            redirect(t1, t2, 1);
            if (outside) return 0;
            outside = 1;
            if (leave_column(0)) return 1;
            stage = 0;
        }
        set_fate(kCapped);
        return 1;
    }

    FD2_HD void restart()
    {
        emit(false);
        p[0] = (T)ex;
        p[1] = (T)ey;
        p[2] = (T)ez;
        n[0] = T(0); n[1] = T(0); n[2] = T(0);
        if (beta > T(0)) rough(beta);
        absorbed = 0;
        detect = 0;
        bulk_abs = 0;
    }

    FD2_HD int step()
    {
        if (absorbed == 0) {
            bulk_abs = flight();
            if (bulk_abs == 0) detect = sensor();
        }
        if (detect == 1 || absorbed == 1 || bulk_abs == 1) {
            restart();
            return 1;
        }
        if (fabs((D)(d[2] - T(0))) < kRefEps) {
            restart();
            return 0;
        }
        rebound++;
        if (rebound > kMaxBoundaryCalls) {
            set_fate(kCapped);
            absorbed = 1;
            return 0;
        }
        absorbed = surface();
        return 0;
    }
};

}  // namespace replay
}  // namespace fd2
