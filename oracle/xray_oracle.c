/*
 * xray_oracle.c -- CPU restatement of the x-ray front end
 * (hybridmantis_b200/csrc/fd2_xray.cu), TEST INFRASTRUCTURE ONLY: tests use
 * it as the checker of the GPU front end; nothing in the library links it.
 *
 * It reads the front end's table file (the library's own text format, made
 * from the reference's PENELOPE material file example/CsI.mat) and runs each
 * history in double precision with the C library's math functions and the
 * same Philox-4x32-10 stream as the GPU (key = seed, counter = draw block,
 * history index, stream id), so that GPU and oracle histories can be
 * compared one by one: they agree unless a draw falls within rounding of a
 * decision threshold.
 *
 * The source follows penEasy's BIGS source
 * (main/sourceBoxIsotropicGaussSpectrum.f:59-178: direction in a cone, point
 * in a rotated box, energy from the binned spectrum or a truncated
 * Gaussian); EDEs follow the EDE tally
 * (main/hybridMANTIS_tallyEnergyDepositionEvents.f:155-200: every energy
 * loss in the detector, minus the secondaries' energy).  The transport model
 * (no counterpart in the reference tree, whose PENELOPE sources are absent)
 * is the front end's: photoelectric absorption with relaxation cascades,
 * Klein-Nishina Compton, screened-Thomson Rayleigh, condensed-history
 * electrons.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define NSH 9
#define NDES 31
#define MAXEL 8
#define STACK 16
#define VAC 16
#define MAXTR 64
#define ME 510998.918

static int n_nodes, n_el, stride, n_e;
static double *E_, *lnv;
static double *ee, *lnee, *lnr, *lnl1;
static double bind[MAXEL][NDES];
static int toff[MAXEL][NDES + 1];
static int *ts;
static double *tcum, *te;

static double lnz(double v) { return log(v > 1e-300 ? v : 1e-300); }

/* ------------------------------------------------------------ tables */

typedef struct {
    int s0, s1, s2;
    double p, e;
} tr_t;

int xo_load(const char *path)
{
    FILE *f = fopen(path, "r");
    if (!f) return 1;
    char key[64];
    int ver;
    double dens, molar;
    if (fscanf(f, "%63s %d", key, &ver) != 2 || strcmp(key, "fd2-xray-material")) return 2;
    if (fscanf(f, "%63s %lf %63s %lf %63s %d", key, &dens, key, &molar, key, &n_el) != 6 || n_el < 1 || n_el > MAXEL)
        return 3;
    int z[MAXEL];
    double at[MAXEL];
    for (int k = 0; k < n_el; ++k)
        if (fscanf(f, "%d %lf", &z[k], &at[k]) != 2) return 4;
    if (fscanf(f, "%63s %d", key, &n_nodes) != 2) return 5;
    stride = 3 + n_el * (1 + NSH);
    E_ = malloc(sizeof(double) * n_nodes);
    lnv = malloc(sizeof(double) * n_nodes * stride);
    double *mur = malloc(sizeof(double) * n_nodes);
    for (int i = 0; i < n_nodes; ++i) {
        double r, c;
        if (fscanf(f, "%lf %lf %lf", &E_[i], &r, &c) != 3) return 6;
        mur[i] = r;
        lnv[i * stride + 0] = lnz(r);
        lnv[i * stride + 1] = lnz(c);
        for (int k = 0; k < n_el; ++k)
            for (int q = 0; q <= NSH; ++q) {
                double v;
                if (fscanf(f, "%lf", &v) != 1) return 7;
                lnv[i * stride + 3 + k * (1 + NSH) + q] = lnz(v);
            }
    }
    if (fscanf(f, "%63s %d", key, &n_e) != 2) return 8;
    ee = malloc(sizeof(double) * n_e);
    lnee = malloc(sizeof(double) * n_e);
    lnr = malloc(sizeof(double) * n_e);
    lnl1 = malloc(sizeof(double) * n_e);
    for (int i = 0; i < n_e; ++i) {
        double r, l;
        if (fscanf(f, "%lf %lf %lf", &ee[i], &r, &l) != 3) return 9;
        lnee[i] = log(ee[i]);
        lnr[i] = log(r);
        lnl1[i] = log(l);
    }
    tr_t *all[MAXEL];
    int ntr[MAXEL], total = 0;
    memset(bind, 0, sizeof bind);
    for (int k = 0; k < n_el; ++k) {
        int Z, nb;
        if (fscanf(f, "%63s %d %d", key, &Z, &nb) != 3) return 10;
        for (int j = 0; j < nb; ++j) {
            int d;
            double e;
            if (fscanf(f, "%d %lf", &d, &e) != 2 || d < 1 || d >= NDES) return 11;
            bind[k][d] = e;
        }
        if (fscanf(f, "%63s %d %d", key, &Z, &ntr[k]) != 3) return 12;
        all[k] = malloc(sizeof(tr_t) * (ntr[k] + 1));
        for (int j = 0; j < ntr[k]; ++j)
            if (fscanf(f, "%d %d %d %lf %lf", &all[k][j].s0, &all[k][j].s1, &all[k][j].s2, &all[k][j].p,
                       &all[k][j].e) != 5)
                return 13;
        total += ntr[k];
    }
    fclose(f);
    ts = malloc(sizeof(int) * (total + 1));
    tcum = malloc(sizeof(double) * (total + 1));
    te = malloc(sizeof(double) * (total + 1));
    int pos = 0;
    for (int k = 0; k < n_el; ++k) {
        for (int s0 = 0; s0 < NDES; ++s0) {
            toff[k][s0] = pos;
            double sum = 0, acc = 0;
            for (int j = 0; j < ntr[k]; ++j)
                if (all[k][j].s0 == s0) sum += all[k][j].p;
            for (int j = 0; j < ntr[k]; ++j)
                if (all[k][j].s0 == s0) {
                    acc += all[k][j].p;
                    ts[pos] = all[k][j].s1 | (all[k][j].s2 << 8);
                    tcum[pos] = acc / sum;
                    te[pos] = all[k][j].e;
                    ++pos;
                }
        }
        toff[k][NDES] = pos;
        free(all[k]);
    }
    /* Rayleigh screening b per node: the oracle's own solution of
     * sigma_R(E) = pi r_e^2 sum(n Z^2) I(b), I(b) the integral over mu of
     * (1 + mu^2) (1 + b (1 - mu))^-4 (closed form below). */
    double fz2 = 0;
    for (int k = 0; k < n_el; ++k) fz2 += at[k] * (double)z[k] * z[k];
    const double re = 2.8179403262e-13, NA = 6.02214076e23;
    const double N = dens * NA / molar, s0 = M_PI * re * re * fz2;
    for (int i = 0; i < n_nodes; ++i) {
        const double sig = mur[i] / N;
        double b = 0;
        if (sig > 0 && sig < s0 * 8.0 / 3.0) {
            double lo = -40, hi = 40;
            for (int it = 0; it < 200; ++it) {
                const double mid = 0.5 * (lo + hi), bb = exp(mid);
                /* I(b) = int_0^2 (2 - 2t + t^2) (1 + b t)^-4 dt */
                double I;
                if (bb < 0.05) {
                    /* (1 + b t)^-4 = sum_n (n+1)(n+2)(n+3)/6 (-b t)^n; moments of the quadratic */
                    I = 0;
                    double bn = 1;
                    for (int q = 0; q < 60; ++q) {
                        const double p2 = pow(2.0, q + 1);
                        const double M = 2 * p2 / (q + 1) - 2 * 2 * p2 / (q + 2) + 4 * p2 / (q + 3);
                        I += (q + 1.0) * (q + 2.0) * (q + 3.0) / 6.0 * bn * M;
                        bn *= -bb;
                    }
                } else {
                    /* with v = 1 + b t: 2 - 2t + t^2 = A + Bc v + C v^2 */
                    const double v = 1 + 2 * bb;
                    const double A = 2 + 2 / bb + 1 / (bb * bb), Bc = -(2 / bb + 2 / (bb * bb)), C = 1 / (bb * bb);
                    I = (A * (1 - pow(v, -3)) / 3 + Bc * (1 - pow(v, -2)) / 2 + C * (1 - 1 / v)) / bb;
                }
                if (s0 * I > sig) lo = mid;
                else hi = mid;
            }
            b = exp(0.5 * (lo + hi));
        }
        lnv[i * stride + 2] = lnz(b);
    }
    free(mur);
    return 0;
}

/* ------------------------------------------------------------ random stream */

typedef struct {
    uint32_t c[4], k0, k1;
    double buf[2];
    int left;
} rng_t;

static void philox(uint32_t c[4], uint32_t k0, uint32_t k1, uint32_t out[4])
{
    uint32_t x = c[0], y = c[1], z = c[2], w = c[3];
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * x, p1 = (uint64_t)0xCD9E8D57u * z;
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0, hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        const uint32_t nx = hi1 ^ y ^ k0, ny = lo1, nz = hi0 ^ w ^ k1, nw = lo0;
        x = nx;
        y = ny;
        z = nz;
        w = nw;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = x;
    out[1] = y;
    out[2] = z;
    out[3] = w;
}

static double to_u(uint32_t a, uint32_t b)
{
    const uint64_t k = ((uint64_t)(a >> 5) << 26) | (uint64_t)(b >> 6);
    return ((double)k + 0.5) * 1.1102230246251565404e-16;
}

static double U(rng_t *r)
{
    if (r->left == 0) {
        uint32_t o[4];
        philox(r->c, r->k0, r->k1, o);
        r->c[0]++;
        r->buf[0] = to_u(o[0], o[1]);
        r->buf[1] = to_u(o[2], o[3]);
        r->left = 2;
    }
    return r->buf[2 - r->left--];
}

/* ------------------------------------------------------------ geometry */

static double X_, Y_, H2, EABS_E, EABS_PH, LOSS, LOCAL_E;
static int FLUO, CAP;

static double dist_exit(const double *p, const double *d)
{
    double t = 1e300;
    if (d[0] > 0) t = fmin(t, (X_ - p[0]) / d[0]);
    else if (d[0] < 0) t = fmin(t, -p[0] / d[0]);
    if (d[1] > 0) t = fmin(t, (Y_ - p[1]) / d[1]);
    else if (d[1] < 0) t = fmin(t, -p[1] / d[1]);
    if (d[2] > 0) t = fmin(t, (H2 - p[2]) / d[2]);
    else if (d[2] < 0) t = fmin(t, (-H2 - p[2]) / d[2]);
    return fmax(t, 0.0);
}

static int enter(double *p, const double *d)
{
    const double lo[3] = {0, 0, -H2}, hi[3] = {X_, Y_, H2};
    int in = 1;
    for (int a = 0; a < 3; ++a) in = in && p[a] >= lo[a] && p[a] <= hi[a];
    if (in) return 1;
    double t0 = 0, t1 = 1e300;
    for (int a = 0; a < 3; ++a) {
        if (d[a] == 0) {
            if (p[a] < lo[a] || p[a] > hi[a]) return 0;
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
    if (!(t0 < t1)) return 0;
    for (int a = 0; a < 3; ++a) p[a] += t0 * d[a];
    for (int a = 0; a < 3; ++a) p[a] = fmin(fmax(p[a], lo[a]), hi[a]);
    return 1;
}

static void rotate(double *d, double c, double phi)
{
    c = fmin(fmax(c, -1.0), 1.0);
    const double s = sqrt(fmax(0.0, 1.0 - c * c));
    const double sp = sin(phi), cp = cos(phi);
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

static void isotropic(rng_t *r, double *d)
{
    const double c = 2.0 * U(r) - 1.0, phi = 2.0 * M_PI * U(r);
    const double s = sqrt(fmax(0.0, 1.0 - c * c));
    d[0] = s * cos(phi);
    d[1] = s * sin(phi);
    d[2] = c;
}

/* ------------------------------------------------------------ tables */

static void interval(double E, int *k, double *w)
{
    if (E <= E_[0]) {
        *k = 0;
        *w = 0;
        return;
    }
    if (E >= E_[n_nodes - 1]) {
        *k = n_nodes - 2;
        *w = 1;
        return;
    }
    int lo = 0, hi = n_nodes - 1;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (E_[mid] <= E) lo = mid;
        else hi = mid;
    }
    *k = lo;
    *w = log(E / E_[lo]) / log(E_[lo + 1] / E_[lo]);
}

static double pval(int k, double w, int col)
{
    const double a = lnv[k * stride + col], b = lnv[(k + 1) * stride + col];
    return exp(a + w * (b - a));
}

static int e_node(double E)
{
    int lo = 0, hi = n_e - 1;
    if (E >= ee[hi]) return hi - 1;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (ee[mid] <= E) lo = mid;
        else hi = mid;
    }
    return lo;
}

static double e_range(double E)
{
    if (E <= ee[0]) return exp(lnr[0]) * E / ee[0];
    const int lo = e_node(E);
    const double w = (log(E) - lnee[lo]) / (lnee[lo + 1] - lnee[lo]);
    return exp(lnr[lo] + w * (lnr[lo + 1] - lnr[lo]));
}

static double e_lambda1(double E)
{
    if (E <= ee[0]) return exp(lnl1[0]);
    const int lo = e_node(E);
    const double w = (log(E) - lnee[lo]) / (lnee[lo + 1] - lnee[lo]);
    return exp(lnl1[lo] + w * (lnl1[lo + 1] - lnl1[lo]));
}

static double e_of_range(double R)
{
    const double r0 = exp(lnr[0]);
    if (R <= 0) return 0;
    if (R <= r0) return ee[0] * R / r0;
    const double lr = log(R);
    int lo = 0, hi = n_e - 1;
    if (lr >= lnr[hi]) lo = hi - 1;
    else
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (lnr[mid] <= lr) lo = mid;
            else hi = mid;
        }
    const double w = (lr - lnr[lo]) / (lnr[lo + 1] - lnr[lo]);
    return exp(lnee[lo] + w * (lnee[lo + 1] - lnee[lo]));
}

/* ------------------------------------------------------------ samplers */

static double sample_kn(rng_t *r, double E)
{
    const double kappa = E / ME, e0 = 1.0 / (1.0 + 2.0 * kappa);
    const double a1 = log1p(2.0 * kappa), a2 = 0.5 * (1.0 - e0 * e0);
    for (;;) {
        double eps;
        if (U(r) * (a1 + a2) < a1) eps = exp(-a1 * U(r));
        else eps = sqrt(e0 * e0 + (1.0 - e0 * e0) * U(r));
        const double t = (1.0 - eps) / (kappa * eps);
        const double s2 = fmax(0.0, t * (2.0 - t));
        if (U(r) * (1.0 + eps * eps) <= 1.0 + eps * eps - eps * s2) return eps;
    }
}

static double sample_rayleigh(rng_t *r, double b)
{
    for (;;) {
        const double u = U(r);
        double t;
        if (b < 1e-6) t = 2.0 * u;
        else {
            const double c = -expm1(-3.0 * log1p(2.0 * b));
            t = expm1(-log1p(-u * c) / 3.0) / b;
        }
        t = fmin(fmax(t, 0.0), 2.0);
        const double mu = 1.0 - t;
        if (2.0 * U(r) <= 1.0 + mu * mu) return mu;
    }
}

static double sample_sauter(rng_t *r, double T)
{
    const double gam = 1.0 + T / ME;
    const double beta = sqrt(fmax(0.0, 1.0 - 1.0 / (gam * gam)));
    const double c = 0.5 * gam * (gam - 1.0) * (gam - 2.0);
    if (beta < 1e-6) {
        for (;;) {
            const double mu = 2.0 * U(r) - 1.0;
            if (U(r) <= 1.0 - mu * mu) return mu;
        }
    }
    const double a = 1.0 / ((1.0 - beta) * (1.0 - beta) * (1.0 - beta));
    const double b = 1.0 / ((1.0 + beta) * (1.0 + beta) * (1.0 + beta));
    const double K = 1.0 + fmax(c, 0.0) * (1.0 + beta);
    for (;;) {
        const double nu = 1.0 / cbrt(a - U(r) * (a - b));
        const double mu = fmin(fmax((1.0 - nu) / beta, -1.0), 1.0);
        if (U(r) * K <= (1.0 - mu * mu) * (1.0 + c * nu)) return mu;
    }
}

static double sample_deflection(rng_t *r, double s, double l1)
{
    const double m = -0.5 * expm1(-s / l1);
    const double u = U(r);
    if (m >= 0.5 - 1e-12) return 1.0 - 2.0 * u;
    const double bb = 1.0 / m - 1.0;
    return 1.0 - 2.0 * (-expm1(log(u) / bb));
}

/* ------------------------------------------------------------ a history */

typedef struct {
    double e0, esc_ph, esc_el, first_depth;
    int n_edes, first_kind, merged, missed;
    int n_pe, n_co, n_ra, n_fe, n_fesc, n_aug, n_steps;
} hinfo_t;

typedef struct {
    double e, p[3], d[3];
    int fluo;
} photon_t;

typedef struct {
    rng_t *r;
    double *slots; /* CAP x 4 */
    hinfo_t *h;
} hist_t;

static void deposit(hist_t *H, double de, const double *q)
{
    if (!(de > 0.0)) return;
    if (H->h->n_edes < CAP) {
        double *s = H->slots + 4 * H->h->n_edes;
        s[0] = q[0];
        s[1] = q[1];
        s[2] = q[2];
        s[3] = de;
        H->h->n_edes++;
    } else {
        H->slots[4 * (CAP - 1) + 3] += de;
        H->h->merged = 1;
    }
}

static void electron(hist_t *H, double T, const double *p0, const double *d0)
{
    double p[3] = {p0[0], p0[1], p0[2]}, d[3] = {d0[0], d0[1], d0[2]};
    for (;;) {
        if (T <= LOCAL_E) {
            deposit(H, T, p);
            return;
        }
        double Tn = T * (1.0 - LOSS);
        if (Tn < EABS_E) Tn = 0.0;
        const double R = e_range(T), Rn = Tn > 0.0 ? e_range(Tn) : 0.0;
        const double s = R - Rn, t = dist_exit(p, d);
        H->h->n_steps++;
        if (s > t) {
            const double Tx = e_of_range(R - t);
            const double hh = U(H->r) * t;
            const double q[3] = {p[0] + hh * d[0], p[1] + hh * d[1], p[2] + hh * d[2]};
            deposit(H, T - Tx, q);
            H->h->esc_el += Tx;
            return;
        }
        const double hh = U(H->r) * s;
        const double q[3] = {p[0] + hh * d[0], p[1] + hh * d[1], p[2] + hh * d[2]};
        deposit(H, T - Tn, q);
        for (int a = 0; a < 3; ++a) p[a] += s * d[a];
        if (Tn == 0.0) return;
        const double c = sample_deflection(H->r, s, e_lambda1(0.5 * (T + Tn)));
        rotate(d, c, 2.0 * M_PI * U(H->r));
        T = Tn;
    }
}

static void relax(hist_t *H, int el, int shell, double Ub, const double *p, photon_t *stack, int *ns)
{
    double local = Ub;
    if (FLUO && shell > 0) {
        int v[VAC], nv = 0, steps = 0;
        v[nv++] = shell;
        while (nv > 0 && steps < MAXTR) {
            const int s0 = v[--nv];
            const int a = toff[el][s0], b = toff[el][s0 + 1];
            if (a == b) continue;
            const double x = U(H->r);
            int j = a;
            while (j < b - 1 && tcum[j] <= x) ++j;
            ++steps;
            const double Et = fmin(te[j], local);
            const int s1 = ts[j] & 0xFF, s2 = ts[j] >> 8;
            if (s2 == 0) {
                if (Et > EABS_PH && *ns < STACK) {
                    photon_t *f = &stack[(*ns)++];
                    f->e = Et;
                    f->p[0] = p[0];
                    f->p[1] = p[1];
                    f->p[2] = p[2];
                    isotropic(H->r, f->d);
                    f->fluo = 1;
                    H->h->n_fe++;
                    local -= Et;
                }
                if (nv < VAC) v[nv++] = s1;
            } else {
                if (Et > EABS_E) {
                    double d[3];
                    isotropic(H->r, d);
                    H->h->n_aug++;
                    local -= Et;
                    electron(H, Et, p, d);
                }
                if (nv < VAC - 1) {
                    v[nv++] = s1;
                    v[nv++] = s2;
                }
            }
        }
    }
    deposit(H, local, p);
}

static void photon(hist_t *H, photon_t ph, photon_t *stack, int *ns)
{
    double E = ph.e, p[3] = {ph.p[0], ph.p[1], ph.p[2]}, d[3] = {ph.d[0], ph.d[1], ph.d[2]};
    for (;;) {
        if (E < EABS_PH) {
            deposit(H, E, p);
            return;
        }
        int k;
        double w;
        interval(E, &k, &w);
        const double muR = pval(k, w, 0), muC = pval(k, w, 1);
        double mupe[MAXEL], mu = muR + muC;
        for (int e = 0; e < n_el; ++e) {
            mupe[e] = pval(k, w, 3 + e * (1 + NSH));
            mu += mupe[e];
        }
        const double s = -log(U(H->r)) / mu, t = dist_exit(p, d);
        if (s >= t) {
            H->h->esc_ph += E;
            if (ph.fluo) H->h->n_fesc++;
            return;
        }
        for (int a = 0; a < 3; ++a) p[a] += s * d[a];
        double x = U(H->r) * mu;
        const int kind = x < muR ? 1 : x < muR + muC ? 2 : 3;
        if (H->h->first_kind == 0) {
            H->h->first_kind = kind;
            H->h->first_depth = H2 - p[2];
        }
        if (kind == 1) {
            H->h->n_ra++;
            const double c = sample_rayleigh(H->r, pval(k, w, 2));
            rotate(d, c, 2.0 * M_PI * U(H->r));
            continue;
        }
        if (kind == 2) {
            H->h->n_co++;
            const double eps = sample_kn(H->r, E);
            const double c = 1.0 - (1.0 - eps) / (eps * (E / ME));
            double dn[3] = {d[0], d[1], d[2]};
            rotate(dn, c, 2.0 * M_PI * U(H->r));
            const double En = eps * E, Te = E - En;
            double pe[3] = {E * d[0] - En * dn[0], E * d[1] - En * dn[1], E * d[2] - En * dn[2]};
            const double nn = sqrt(pe[0] * pe[0] + pe[1] * pe[1] + pe[2] * pe[2]);
            for (int a = 0; a < 3; ++a) pe[a] = nn > 0 ? pe[a] / nn : d[a];
            electron(H, Te, p, pe);
            E = En;
            for (int a = 0; a < 3; ++a) d[a] = dn[a];
            continue;
        }
        H->h->n_pe++;
        x -= muR + muC;
        int el = n_el - 1;
        for (int e = 0; e < n_el - 1; ++e) {
            if (x < mupe[e]) {
                el = e;
                break;
            }
            x -= mupe[e];
        }
        double y = U(H->r) * mupe[el];
        int shell = 0;
        for (int q = 0; q < NSH; ++q) {
            const double sq = pval(k, w, 3 + el * (1 + NSH) + 1 + q);
            if (y < sq) {
                shell = q + 1;
                break;
            }
            y -= sq;
        }
        double Ub = shell ? bind[el][shell] : 0.0;
        if (!(Ub > 0.0)) {
            shell = 0;
            Ub = 0.0;
        }
        Ub = fmin(Ub, E);
        const double T = E - Ub;
        double de[3] = {d[0], d[1], d[2]};
        const double c = sample_sauter(H->r, T);
        rotate(de, c, 2.0 * M_PI * U(H->r));
        electron(H, T, p, de);
        relax(H, el, shell, Ub, p, stack, ns);
        return;
    }
}

/* Source as prepared by the caller (oracle/xray_oracle.py restates the
 * BIGS initialisation, sourceBoxIsotropicGaussSpectrum.f:263-400). */
typedef struct {
    int particle, nspec, gaussian, point;
    const double *espc, *pcum, *despc;
    double gmean, gsig, gmin, gmax;
    double ctr[3], side[3], rot[9], dir[3], cossrc;
} xo_source;

typedef struct {
    double X, Y, H2, eabs_e, eabs_ph, loss, local_e;
    int fluo, cap;
    uint64_t seed;
} xo_opts;

/* Run histories first .. first + n - 1.  info: n x 15 doubles (e0, esc_ph,
 * esc_el, first_depth, n_edes, first_kind, merged, missed, n_pe, n_co, n_ra,
 * n_fe, n_fesc, n_aug, n_steps); slots: n x cap x 4 (x, y, z, de). */
int xo_run(const xo_opts *o, const xo_source *src, int64_t first, int64_t n, double *info, double *slots)
{
    X_ = o->X;
    Y_ = o->Y;
    H2 = o->H2;
    EABS_E = o->eabs_e;
    EABS_PH = o->eabs_ph;
    LOSS = o->loss;
    LOCAL_E = fmax(o->eabs_e, o->local_e);
    FLUO = o->fluo;
    CAP = o->cap;
    for (int64_t i = 0; i < n; ++i) {
        const uint64_t g = (uint64_t)(first + i);
        rng_t r = {{0u, (uint32_t)g, (uint32_t)(g >> 32), 0x58524159u}, (uint32_t)o->seed, (uint32_t)(o->seed >> 32),
                   {0, 0}, 0};
        hinfo_t h;
        memset(&h, 0, sizeof h);
        h.first_depth = -1.0;
        double p[3], d[3] = {src->dir[0], src->dir[1], src->dir[2]}, E;
        const double c = src->cossrc + (1.0 - src->cossrc) * U(&r);
        rotate(d, c, 2.0 * M_PI * U(&r));
        if (src->point) {
            for (int a = 0; a < 3; ++a) p[a] = src->ctr[a];
        } else {
            const double l[3] = {src->side[0] * (U(&r) - 0.5), src->side[1] * (U(&r) - 0.5),
                                 src->side[2] * (U(&r) - 0.5)};
            for (int a = 0; a < 3; ++a)
                p[a] = src->rot[3 * a] * l[0] + src->rot[3 * a + 1] * l[1] + src->rot[3 * a + 2] * l[2] + src->ctr[a];
        }
        if (src->gaussian) {
            for (;;) {
                const double a = sqrt(-2.0 * log(U(&r)));
                E = src->gmean + src->gsig * a * sin(2.0 * M_PI * U(&r));
                if (E > src->gmin && E < src->gmax) break;
            }
        } else {
            const double x = U(&r);
            int lo = 0, hi = src->nspec - 1;
            while (hi - lo > 1) {
                const int mid = (lo + hi) >> 1;
                if (src->pcum[mid] <= x) lo = mid;
                else hi = mid;
            }
            E = src->espc[lo] + (x - src->pcum[lo]) * src->despc[lo];
        }
        h.e0 = E;
        hist_t H = {&r, slots + (size_t)i * CAP * 4, &h};
        if (!enter(p, d)) {
            h.missed = 1;
            if (src->particle == 2) h.esc_ph = E;
            else h.esc_el = E;
        } else if (src->particle == 1) {
            electron(&H, E, p, d);
        } else {
            photon_t stack[STACK];
            int ns = 0;
            photon_t f0 = {E, {p[0], p[1], p[2]}, {d[0], d[1], d[2]}, 0};
            photon(&H, f0, stack, &ns);
            while (ns > 0) {
                const photon_t f = stack[--ns];
                photon(&H, f, stack, &ns);
            }
        }
        double *q = info + 15 * i;
        const double v[15] = {h.e0,    h.esc_ph, h.esc_el, h.first_depth, h.n_edes, h.first_kind, h.merged, h.missed,
                              h.n_pe, h.n_co,   h.n_ra,   h.n_fe,        h.n_fesc, h.n_aug,      h.n_steps};
        memcpy(q, v, sizeof v);
    }
    return 0;
}

/* The samplers alone, on the stream of fd2_xray_sample (counter word 3 =
 * 'SMPL', word 1..2 = draw index). */
int xo_sample(int which, double E, double param, int64_t n, uint64_t seed, double *out)
{
    for (int64_t i = 0; i < n; ++i) {
        rng_t r = {{0u, (uint32_t)i, (uint32_t)((uint64_t)i >> 32), 0x534D504Cu}, (uint32_t)seed,
                   (uint32_t)(seed >> 32), {0, 0}, 0};
        double v;
        if (which == 0) v = sample_kn(&r, E);
        else if (which == 1) {
            int k;
            double w;
            interval(E, &k, &w);
            v = sample_rayleigh(&r, pval(k, w, 2));
        } else if (which == 2) v = sample_sauter(&r, E);
        else v = sample_deflection(&r, param, e_lambda1(E));
        out[i] = v;
    }
    return 0;
}

/* Rayleigh screening b at energy E (the oracle's own closed-form solution). */
double xo_rayleigh_b(double E)
{
    int k;
    double w;
    interval(E, &k, &w);
    return pval(k, w, 2);
}
