/*
 * grid_oracle.c -- CPU oracle of the explicit column lattice
 * (fd2_options.column_grid = 1).  TEST INFRASTRUCTURE ONLY: tests/ load it
 * to check the GPU lattice walk (hybridmantis_b200/csrc/fd2_device.cuh,
 * Walker::grid_*).  The lattice has no counterpart in the reference, whose
 * next column is drawn at random after every crossing; this file restates
 * the lattice walk itself, in double precision, with its own random stream
 * (xoshiro256** per photon, seeded through splitmix64), so GPU and oracle
 * agree in distribution, not photon by photon.  The building blocks it
 * shares with the reference walk keep the reference's rules: isotropic
 * emission with the first photon's |cos| > 0.01 rejection
 * (main/hybridMANTIS_c_ver1_0.c:257-262), RoughSurface's perturbation built
 * from sqrt(1 - u^2) of the uniform itself (main/kernel_cuda_c_ver1_0.cu,
 * RoughSurface), the top reflector's diffuse downward reflection and the
 * sensor rule (boundary_analysis / detection), and the PRF pixel rule.
 *
 * Lattice: columns of radius R around ((i + 1/2) p, (j + 1/2) p), pitch p
 * (square), or around ((i + 1/2) p + o_j, (j + 1/2) h), h = p sqrt(3)/2,
 * o_j = p/2 on odd rows (hexagonal).
 * Inside a column: flight to the wall or to the top / sensor plane, bulk
 * absorption against an Exp(1) budget of absorption lengths.  At a wall:
 * the normal toward the incident medium, roughened (up to 8 draws until the
 * photon meets it), Fresnel reflection probability (unpolarised; total
 * reflection inside beyond the critical angle), else vector-Snell
 * refraction.  In the gap: straight flight, cell by cell, to the first
 * column met, the top or sensor plane, or the detector's side (lost).
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

typedef struct {
    double xdet, ydet, H, R, pitch, n_col, n_gap, top_absfrac, mu, beta, sensor_refl;
    double lb_x, lb_y, ub_x, ub_y;
    int32_t pixel, xdim, ydim;
    int32_t lattice; /* 1 square, 2 hexagonal */
} go_geom;

enum { DETECT = 0, ABS_TOP = 1, ABS_BULK = 2, LOST = 3, CAPPED = 6, ALIVE = -1 };

static const double kEps = 8.1929093e-6;
static const double kPi = 3.14159265358979323846;

typedef struct {
    uint64_t s[4];
} rng_t;

static uint64_t splitmix(uint64_t *x)
{
    uint64_t z = (*x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

static double unif(rng_t *r)
{
    uint64_t *s = r->s;
    const uint64_t out = rotl(s[1] * 5, 7) * 9;
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return ((double)(out >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}

typedef struct {
    double px, py, pz, dx, dy, dz, nx, ny, nz, xc, yc, budget;
    int in_gap;
    uint32_t rebound;
    int ii, jj;
    rng_t rng;
} photon_t;

static void renorm(double *x, double *y, double *z)
{
    const double n = sqrt(*x * *x + *y * *y + *z * *z);
    if (n > 0.0) {
        *x /= n;
        *y /= n;
        *z /= n;
    }
}

static double fresnel(double c, double ct, double eta)
{
    const double a = eta * c, b = eta * ct;
    const double rs = (a - ct) / (a + ct), rp = (c - b) / (c + b);
    return 0.5 * (rs * rs + rp * rp);
}

static void roughen(photon_t *ph, double beta)
{
    const double u1 = unif(&ph->rng);
    const double qz = 2.0 * u1 - 1.0;
    const double rr = sqrt(fmax(0.0, 1.0 - u1 * u1));
    const double phi = kPi * (2.0 * unif(&ph->rng) - 1.0);
    const double qx = rr * cos(phi), qy = rr * sin(phi);
    const double bq = beta / sqrt(qx * qx + qy * qy + qz * qz);
    double rx = ph->nx + bq * qx, ry = ph->ny + bq * qy, rz = ph->nz + bq * qz;
    renorm(&rx, &ry, &rz);
    ph->nx = rx;
    ph->ny = ry;
    ph->nz = rz;
}

static void set_pixel(photon_t *ph, const go_geom *g)
{
    ph->ii = ph->jj = -1;
    if (ph->px <= g->ub_x && ph->py <= g->ub_y && ph->px >= g->lb_x && ph->py >= g->lb_y) {
        ph->ii = (int)floor((ph->px - g->lb_x) / g->pixel);
        ph->jj = (int)floor((ph->py - g->lb_y) / g->pixel);
    }
}

static int plane(photon_t *ph, const go_geom *g, int top)
{
    if (top) {
        if (g->top_absfrac > 0.0 && unif(&ph->rng) < g->top_absfrac) return ABS_TOP;
        ph->dz = -fabs(2.0 * unif(&ph->rng) - 1.0);
        const double rr = sqrt(fmax(0.0, 1.0 - ph->dz * ph->dz));
        const double phi = kPi * (2.0 * unif(&ph->rng) - 1.0);
        ph->dx = rr * cos(phi);
        ph->dy = rr * sin(phi);
        return ALIVE;
    }
    if (!(g->sensor_refl > 0.0 && unif(&ph->rng) < g->sensor_refl)) {
        set_pixel(ph, g);
        return DETECT;
    }
    ph->dz = -ph->dz;
    return ALIVE;
}

static int wall(photon_t *ph, const go_geom *g, double cx, double cy, int inside)
{
    double ox = ph->px - cx, oy = ph->py - cy;
    const double on = sqrt(ox * ox + oy * oy);
    ox /= on;
    oy /= on;
    const double sgn = inside ? -1.0 : 1.0;
    double c1 = 0.0;
    for (int t = 0; t < 8; ++t) {
        ph->nx = sgn * ox;
        ph->ny = sgn * oy;
        ph->nz = 0.0;
        if (g->beta > 0.0) roughen(ph, g->beta);
        c1 = -(ph->dx * ph->nx + ph->dy * ph->ny + ph->dz * ph->nz);
        if (c1 > 0.0) break;
    }
    if (!(c1 > 0.0)) {
        ph->nx = sgn * ox;
        ph->ny = sgn * oy;
        ph->nz = 0.0;
        c1 = fmax(-(ph->dx * ph->nx + ph->dy * ph->ny), 0.0);
    }
    const double eta = inside ? g->n_col / g->n_gap : g->n_gap / g->n_col;
    const double st2 = eta * eta * fmax(0.0, 1.0 - c1 * c1);
    double pr = 1.0, ct = 0.0;
    if (st2 < 1.0) {
        ct = sqrt(1.0 - st2);
        pr = fresnel(c1, ct, eta);
    }
    if (unif(&ph->rng) < pr) {
        ph->dx += 2.0 * c1 * ph->nx;
        ph->dy += 2.0 * c1 * ph->ny;
        ph->dz += 2.0 * c1 * ph->nz;
        renorm(&ph->dx, &ph->dy, &ph->dz);
        return ALIVE;
    }
    const double k = eta * c1 - ct;
    ph->dx = eta * ph->dx + k * ph->nx;
    ph->dy = eta * ph->dy + k * ph->ny;
    ph->dz = eta * ph->dz + k * ph->nz;
    renorm(&ph->dx, &ph->dy, &ph->dz);
    ph->in_gap = inside;
    if (!inside) {
        ph->xc = cx;
        ph->yc = cy;
    }
    return ALIVE;
}

/* Hexagonal lattice: brick (i, j) of row j holds the column at its centre;
 * q = 0 is that column, q = 1..4 the columns of rows j +- 1 centred on its
 * corners' x (the only other columns that reach into the brick). */
static void hex_candidate(const go_geom *g, int i, int j, int q, double *cx, double *cy)
{
    const double p = g->pitch, h = p * sqrt(3.0) / 2.0;
    const double o = (j & 1) ? 0.5 * p : 0.0;
    *cx = (i + 0.5) * p + o;
    *cy = (j + 0.5) * h;
    if (q > 0) {
        *cy += q <= 2 ? h : -h;
        *cx += (q & 1) ? -0.5 * p : 0.5 * p;
    }
}

static int hex_first_hit(const go_geom *g, double px, double py, double dx, double dy, double tend, double *t_out,
                         double *cx_out, double *cy_out)
{
    const double p = g->pitch, h = p * sqrt(3.0) / 2.0;
    int j = (int)floor(py / h);
    int i = (int)floor((px - ((j & 1) ? 0.5 * p : 0.0)) / p);
    const double qa = dx * dx + dy * dy;
    double tin = 0.0;
    for (int k = 0; k < (1 << 14); ++k) {
        const double o = (j & 1) ? 0.5 * p : 0.0;
        const double xl = i * p + o;
        const double tX = dx > 0.0 ? (xl + p - px) / dx : dx < 0.0 ? (xl - px) / dx : INFINITY;
        const double tY = dy > 0.0 ? ((j + 1) * h - py) / dy : dy < 0.0 ? (j * h - py) / dy : INFINITY;
        const double tout = fmin(tX, tY);
        double tb = INFINITY, bx = 0.0, by = 0.0;
        for (int q = 0; q < 5; ++q) {
            double cx, cy;
            hex_candidate(g, i, j, q, &cx, &cy);
            const double fx = px - cx, fy = py - cy;
            const double qb = 2.0 * (fx * dx + fy * dy);
            const double qc = fx * fx + fy * fy - g->R * g->R;
            if (qa > 0.0 && qb < 0.0) {
                const double disc = qb * qb - 4.0 * qa * qc;
                if (disc >= 0.0) {
                    const double t1 = (2.0 * qc) / (-qb + sqrt(disc));
                    if (t1 > 1e-4 && t1 >= tin - 1e-4 && t1 <= tout + 1e-4 && t1 < tb) {
                        tb = t1;
                        bx = cx;
                        by = cy;
                    }
                }
            }
        }
        if (tb < tend) {
            *t_out = tb;
            *cx_out = bx;
            *cy_out = by;
            return 1;
        }
        if (tout >= tend) return 0;
        if (tX < tY) {
            i += dx > 0.0 ? 1 : -1;
        } else {
            j += dy > 0.0 ? 1 : -1;
            i = (int)floor((px + tout * dx - ((j & 1) ? 0.5 * p : 0.0)) / p);
        }
        tin = tout;
    }
    return -1;
}

/* The first column met by a gap flight from (px, py) along (dx, dy) before
 * path length tend; 1 and (t, cx, cy) when there is one. */
int go_first_hit(const go_geom *g, double px, double py, double dx, double dy, double tend, double *t_out,
                 double *cx_out, double *cy_out)
{
    if (g->lattice == 2) return hex_first_hit(g, px, py, dx, dy, tend, t_out, cx_out, cy_out);
    const double p = g->pitch;
    int i = (int)floor(px / p), j = (int)floor(py / p);
    const int si = dx > 0.0 ? 1 : -1, sj = dy > 0.0 ? 1 : -1;
    double tmx = dx != 0.0 ? ((double)(dx > 0.0 ? i + 1 : i) * p - px) / dx : INFINITY;
    double tmy = dy != 0.0 ? ((double)(dy > 0.0 ? j + 1 : j) * p - py) / dy : INFINITY;
    const double tdx = dx != 0.0 ? p / fabs(dx) : INFINITY;
    const double tdy = dy != 0.0 ? p / fabs(dy) : INFINITY;
    const double qa = dx * dx + dy * dy;
    for (int k = 0; k < (1 << 14); ++k) {
        const double cx = (i + 0.5) * p, cy = (j + 0.5) * p;
        const double fx = px - cx, fy = py - cy;
        const double qb = 2.0 * (fx * dx + fy * dy);
        const double qc = fx * fx + fy * fy - g->R * g->R;
        if (qa > 0.0 && qb < 0.0) {
            const double disc = qb * qb - 4.0 * qa * qc;
            if (disc >= 0.0) {
                const double t1 = (2.0 * qc) / (-qb + sqrt(disc));
                if (t1 > 1e-4 && t1 < tend) {
                    *t_out = t1;
                    *cx_out = cx;
                    *cy_out = cy;
                    return 1;
                }
            }
        }
        const double tn = fmin(tmx, tmy);
        if (tn >= tend) return 0;
        if (tmx < tmy) {
            i += si;
            tmx += tdx;
        } else {
            j += sj;
            tmy += tdy;
        }
    }
    return -1; /* capped */
}

static int segment(photon_t *ph, const go_geom *g)
{
    if (++ph->rebound > (1u << 20)) return CAPPED;
    const double half = g->H / 2.0;
    const double zp = ph->dz > 0.0 ? half : -half;
    const double dplane = ph->dz != 0.0 ? (zp - ph->pz) / ph->dz : INFINITY;
    if (!ph->in_gap) {
        const double ddx = ph->px - ph->xc, ddy = ph->py - ph->yc;
        const double qa = ph->dx * ph->dx + ph->dy * ph->dy;
        const double qb = 2.0 * (ddx * ph->dx + ddy * ph->dy);
        const double qc = fmin(ddx * ddx + ddy * ddy - g->R * g->R, 0.0); /* on the wall, not outside */
        double dw = INFINITY;
        const double disc = qb * qb - 4.0 * qa * qc;
        if (qa > 0.0 && disc >= 0.0) {
            const double s = sqrt(disc);
            dw = qb >= 0.0 ? (qb + s != 0.0 ? (-2.0 * qc) / (qb + s) : 0.0) : (s - qb) / (2.0 * qa);
        }
        const int pl = dplane <= dw;
        const double d = fmax(pl ? dplane : dw, 0.0);
        ph->px += d * ph->dx;
        ph->py += d * ph->dy;
        ph->pz = pl ? zp : ph->pz + d * ph->dz;
        if (g->mu > 0.0) {
            const double da = d * g->mu;
            if (da >= ph->budget) return ABS_BULK;
            ph->budget -= da;
        }
        if (ph->px < kEps || ph->px > g->xdet || ph->py < kEps || ph->py > g->ydet) return LOST;
        if (pl) return plane(ph, g, zp > 0.0);
        return wall(ph, g, ph->xc, ph->yc, 1);
    }
    double tx = INFINITY, ty = INFINITY;
    if (ph->dx > 0.0) tx = (g->xdet - ph->px) / ph->dx;
    else if (ph->dx < 0.0) tx = -ph->px / ph->dx;
    if (ph->dy > 0.0) ty = (g->ydet - ph->py) / ph->dy;
    else if (ph->dy < 0.0) ty = -ph->py / ph->dy;
    const double tside = fmin(tx, ty);
    const double tend = fmin(dplane, tside);
    double t, cx, cy;
    const int hit = go_first_hit(g, ph->px, ph->py, ph->dx, ph->dy, tend, &t, &cx, &cy);
    if (hit < 0) return CAPPED;
    if (hit) {
        ph->px += t * ph->dx;
        ph->py += t * ph->dy;
        ph->pz += t * ph->dz;
        return wall(ph, g, cx, cy, 0);
    }
    if (dplane <= tside) {
        ph->px += dplane * ph->dx;
        ph->py += dplane * ph->dy;
        ph->pz = zp;
        return plane(ph, g, zp > 0.0);
    }
    return LOST;
}

/* Transport every photon of every event.  counters[8]: generated, detected,
 * abs_top, abs_bulk, lost, outofcol, theta1, capped; prf [xdim][ydim];
 * per_primary[num_hist] by history (1-based hist). */
int go_run(const go_geom *g, int64_t n, const double *x, const double *y, const double *z, const int32_t *hist,
           const int32_t *nphot, int32_t num_hist, uint64_t seed, uint64_t *counters, uint64_t *prf,
           int32_t *per_primary)
{
    if (!g || n < 0 || g->pitch < 2.0 * g->R) return 1;
    for (int64_t e = 0; e < n; ++e) {
        for (int32_t k = 0; k < nphot[e]; ++k) {
            photon_t ph;
            memset(&ph, 0, sizeof ph);
            uint64_t sm = seed ^ ((uint64_t)e * 0x9E3779B97F4A7C15ull) ^ ((uint64_t)k << 40) ^ (uint64_t)k;
            for (int q = 0; q < 4; ++q) ph.rng.s[q] = splitmix(&sm);
            ph.px = x[e];
            ph.py = y[e];
            ph.pz = z[e];
            double c = 2.0 * unif(&ph.rng) - 1.0;
            if (k == 0)
                for (int t = 0; t < 64 && fabs(c) <= 0.01; ++t) c = 2.0 * unif(&ph.rng) - 1.0;
            const double rr = sqrt(fmax(0.0, 1.0 - c * c));
            const double phi = kPi * (2.0 * unif(&ph.rng) - 1.0);
            ph.dx = rr * cos(phi);
            ph.dy = rr * sin(phi);
            ph.dz = c;
            renorm(&ph.dx, &ph.dy, &ph.dz);
            ph.budget = -log(unif(&ph.rng));
            if (g->lattice == 2) {
                const double h = g->pitch * sqrt(3.0) / 2.0;
                const int j = (int)floor(ph.py / h);
                const int i = (int)floor((ph.px - ((j & 1) ? 0.5 * g->pitch : 0.0)) / g->pitch);
                double bd = INFINITY;
                for (int q = 0; q < 5; ++q) {
                    double cx, cy;
                    hex_candidate(g, i, j, q, &cx, &cy);
                    const double d2 = (ph.px - cx) * (ph.px - cx) + (ph.py - cy) * (ph.py - cy);
                    if (d2 < bd) {
                        bd = d2;
                        ph.xc = cx;
                        ph.yc = cy;
                    }
                }
                ph.in_gap = bd >= g->R * g->R;
            } else {
                ph.xc = (floor(ph.px / g->pitch) + 0.5) * g->pitch;
                ph.yc = (floor(ph.py / g->pitch) + 0.5) * g->pitch;
                const double rx = ph.px - ph.xc, ry = ph.py - ph.yc;
                ph.in_gap = rx * rx + ry * ry >= g->R * g->R;
            }
            int fate = ALIVE;
            while (fate == ALIVE) fate = segment(&ph, g);
            counters[0] += 1;
            counters[1 + fate] += 1;
            if (fate == DETECT) {
                const int32_t h = hist[e];
                if (h >= 1 && h <= num_hist) per_primary[h - 1] += 1;
                if (ph.ii >= 0 && ph.jj >= 0 && ph.ii < g->xdim && ph.jj < g->ydim)
                    prf[(int64_t)ph.ii * g->ydim + ph.jj] += 1;
            }
        }
    }
    return 0;
}
