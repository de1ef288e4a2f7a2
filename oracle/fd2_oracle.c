/*
 * fd2_oracle.c -- CPU oracle for the fastDETECT2 optical transport.
 *
 * TEST INFRASTRUCTURE ONLY (the checker).  Loaded by tests/, the smoke
 * entry point and bench.py's cpu_baseline leg; never part of the product.
 *
 * A plain-C restatement of the reference's CPU path,
 * main/kernel_cuda_c_ver1_0.cu (C branches) driven the way
 * main/hybridMANTIS_c_ver1_0.c:189-340 drives it.  The control flow is
 * re-expressed (state machines instead of labels), but every arithmetic
 * expression keeps the reference's operand types: float storage, float
 * arithmetic where the reference writes float operators, double where a
 * double literal or a double libm call promotes the expression, and the
 * same libm functions (sqrt, log, sin, cos, tan, pow, asin, asinf, acosf,
 * floor).  Built with -ffp-contract=off so no FMA is formed.  With that,
 * photon fates, pixels and RANECU states match the reference's own C
 * functions bit for bit (pinned by tests against oracle/_ref).
 */
#include "fd2_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* Constants of kernel_cuda_c_ver1_0.cu:56-58 (double literals there). */
#define O_TWOPI 6.283185308
#define O_PI 3.14159265
#define O_EPS 8.1929093e-6

/* RANECU parameters, kernel_cuda_c_ver1_0.cu:3453-3458. */
#define O_M1 2147483563
#define O_M2 2147483399
#define O_A1 40014
#define O_A2 40692
#define O_LEAP 1000

enum { C_GEN, C_DETECT, C_ABS_TOP, C_ABS_BULK, C_LOST, C_OUTOFCOL, C_THETA1 };

/* Call counts of the transport's building blocks (reset by
 * fd2o_reset_call_counts); used to express the work per photon.  One set
 * per host thread: callers that run event slices on several threads do not
 * share (or fight over) the counters, and a reset / read sees the calling
 * thread's calls only. */
static _Thread_local uint64_t o_calls[FD2O_NCALLS];
#define O_CALL(k) (o_calls[(k)]++)

void fd2o_reset_call_counts(void) { memset(o_calls, 0, sizeof o_calls); }
void fd2o_get_call_counts(uint64_t out[FD2O_NCALLS]) { memcpy(out, o_calls, sizeof o_calls); }

typedef struct {
    const fd2o_geom *g;
    int32_t seed[2];
    float pos[3], dcos[3], normal[3];
    float xc, yc;             /* centre of the current column */
    uint64_t rebound;         /* boundary_analysis calls of this photon */
    int absorbed, detect, bulk_abs;
    double ex, ey, ez;        /* event position (double, struct start_info) */
    int32_t hist;
    int32_t xdim, ydim, prim_size;
    uint64_t *image;
    int32_t *per_primary;
    uint64_t *cnt;
    int fate, pix_i, pix_j;
} o_walk;

/* ------------------------------------------------------------------ RNG */

/* One RANECU draw: two Schrage-factored MLCG steps combined, scaled by the
 * float constant 1/m1 (ranecu, kernel_cuda_c_ver1_0.cu:3694-3710). */
static float o_u(o_walk *w)
{
    O_CALL(FD2O_CALL_UNIFORM);
    int32_t *s = w->seed;
    int32_t k = s[0] / 53668;
    s[0] = O_A1 * (s[0] - k * 53668) - k * 12211;
    k = s[1] / 52774;
    s[1] = O_A2 * (s[1] - k * 52774) - k * 3791;
    if (s[0] < 0) s[0] += O_M1;
    if (s[1] < 0) s[1] += O_M2;
    int32_t z = s[0] - s[1];
    if (z < 1) z += O_M1 - 1;
    const float scale = (float)(1.0 / 2147483563.0);
    return (float)z * scale;
}

/* (base^e) mod m by binary exponentiation in 64-bit integers. */
static int64_t o_powmod(int64_t base, uint64_t e, int64_t m)
{
    int64_t r = 1;
    base %= m;
    while (e) {
        if (e & 1) r = (r * base) % m;
        base = (base * base) % m;
        e >>= 1;
    }
    return r;
}

/* Jump both MLCGs (history_batch+1)*histories_per_thread*1000 steps ahead
 * of seed_input (init_PRNG, kernel_cuda_c_ver1_0.cu:3516-3584; L'Ecuyer,
 * Commun. ACM 31 (1988) 742). */
void fd2o_init_prng(int64_t history_batch, int32_t histories_per_thread,
                    int32_t seed_input, int32_t seed[2])
{
    uint64_t leap = (uint64_t)(history_batch + 1) *
                    (uint64_t)(int32_t)(histories_per_thread * O_LEAP);
    seed[0] = (int32_t)(((int64_t)seed_input * o_powmod(O_A1, leap, O_M1)) % O_M1);
    seed[1] = (int32_t)(((int64_t)seed_input * o_powmod(O_A2, leap, O_M2)) % O_M2);
}

void fd2o_ranecu(int32_t seed[2], int32_t n, float *out)
{
    o_walk w;
    w.seed[0] = seed[0];
    w.seed[1] = seed[1];
    for (int32_t i = 0; i < n; ++i) out[i] = o_u(&w);
    seed[0] = w.seed[0];
    seed[1] = w.seed[1];
}

/* ------------------------------------------------------------- helpers */

static float o_dot(const float *a, const float *b)
{
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

/* Renormalise when |v| leaves [1-eps, 1+eps] (the check repeated after
 * every direction update in the reference). */
static void o_renorm(float *v)
{
    float norm = (float)sqrt((double)(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]));
    if ((double)norm < 1.0 - O_EPS || (double)norm > 1.0 + O_EPS) {
        v[0] = v[0] / norm;
        v[1] = v[1] / norm;
        v[2] = v[2] / norm;
    }
}

/* Isotropic direction from the uniforms cos(theta) = 2u-1 and phi = 2*pi*u.
 * first != 0: the driver's first photon of an event, which rejects
 * |cos(theta)| <= 0.01 and takes sqrt of a float argument
 * (hybridMANTIS_c_ver1_0.c:257-277); otherwise the re-emission of the C
 * step, whose sqrt argument is double (kernel_cuda_c_ver1_0.cu:577-589). */
static void o_emit(o_walk *w, int first)
{
    float c = (o_u(w) * 2.0f) - 1.0f;
    float rr;
    if (first) {
        while (fabsf(c) <= 0.01f) c = (o_u(w) * 2.0f) - 1.0f;
        rr = (float)sqrt((double)(1.0f - c * c));
    } else {
        rr = (float)sqrt(1.0 - (double)(c * c));
    }
    float phi = (float)((double)o_u(w) * O_TWOPI);
    w->dcos[2] = c;
    w->dcos[0] = (float)((double)rr * cos((double)phi));
    w->dcos[1] = (float)((double)rr * sin((double)phi));
    o_renorm(w->dcos);
}

/* Perturb the surface normal: n' = normalize(n + beta * p), p a random
 * unit vector built from u1 (z = 2u1-1, transverse radius sqrt(1-u1^2))
 * and u2 (azimuth) (RoughSurface, kernel_cuda_c_ver1_0.cu:3261-3300). */
static void o_rough(o_walk *w, float beta)
{
    O_CALL(FD2O_CALL_ROUGH);
    float *n = w->normal;
    float u = o_u(w);
    float pz = 2.0f * u - 1.0f;
    float rr = (float)sqrt((double)(1.0f - u * u));
    u = o_u(w);
    float phi = (float)((double)(u * 2.0f) * O_PI);
    float px = (float)((double)rr * cos((double)phi));
    float py = (float)((double)rr * sin((double)phi));
    float len = (float)sqrt(pow((double)px, 2) + pow((double)py, 2) + pow((double)pz, 2));
    px = px / len;
    py = py / len;
    pz = pz / len;
    float r0 = beta * px + n[0], r1 = beta * py + n[1], r2 = beta * pz + n[2];
    len = (float)sqrt(pow((double)r0, 2) + pow((double)r1, 2) + pow((double)r2, 2));
    n[0] = r0 / len;
    n[1] = r1 / len;
    n[2] = r2 / len;
}

/* Specular reflection (refract == 0) or the reference's refraction formula
 * d' = -n cos(tt) - (sin(tt)/sin(ti)) (d + cos_i n), then renormalise
 * (trans_dir_cos, kernel_cuda_c_ver1_0.cu:3169-3205). */
static void o_redirect(o_walk *w, float ti, float tt, int refract)
{
    O_CALL(refract ? FD2O_CALL_REFRACT : FD2O_CALL_REFLECT);
    float *d = w->dcos, *n = w->normal;
    float inv[3] = {-d[0], -d[1], -d[2]};
    float ci = o_dot(inv, n);
    if (!refract) {
        d[0] = 2.0f * ci * n[0] + d[0];
        d[1] = 2.0f * ci * n[1] + d[1];
        d[2] = 2.0f * ci * n[2] + d[2];
    } else {
        for (int k = 0; k < 3; ++k) {
            double a = (double)(-n[k]) * cos((double)tt);
            double b = (sin((double)tt) / sin((double)ti)) * (double)(d[k] + (ci * n[k]));
            d[k] = (float)(a - b);
        }
    }
    o_renorm(d);
}

static void o_count(o_walk *w, int which, int fate)
{
    w->cnt[which]++;
    w->fate = fate;
}

/* Detection at the sensor plane: PRF pixel floor((x-lb)/pixel) inside the
 * closed bounds, per-primary count (detection, kernel_cuda_c_ver1_0.cu:
 * 3408-3420; transmit :2517-2528).  Pixels outside the caller's image are
 * skipped instead of written out of bounds. */
static void o_detected(o_walk *w)
{
    const fd2o_geom *g = w->g;
    float *p = w->pos;
    o_count(w, C_DETECT, FD2O_FATE_DETECT);
    int ii = (int)floor((double)((p[0] - g->lb_x) / (float)g->pixel));
    int jj = (int)floor((double)((p[1] - g->lb_y) / (float)g->pixel));
    w->pix_i = -1;
    w->pix_j = -1;
    if (p[0] <= g->ub_x && p[1] <= g->ub_y && p[0] >= g->lb_x && p[1] >= g->lb_y) {
        w->pix_i = ii;
        w->pix_j = jj;
        if (ii >= 0 && jj >= 0 && ii < w->xdim && jj < w->ydim)
            w->image[(int64_t)ii * w->ydim + jj]++;
    }
    if (w->hist >= 1 && w->hist <= w->prim_size) w->per_primary[w->hist - 1]++;
}

/* -------------------------------------------------------- column walls */

static int o_outside_detector(const o_walk *w)
{
    const fd2o_geom *g = w->g;
    const float *p = w->pos;
    return ((double)p[0] < O_EPS) || (p[0] > g->xdet) || ((double)p[1] < O_EPS) ||
           (p[1] > g->ydet) || (p[2] < -g->H / 2.0f) || (p[2] > g->H / 2.0f);
}

static float o_radius(const o_walk *w)
{
    const float *p = w->pos;
    return (float)sqrt((double)((p[0] - w->xc) * (p[0] - w->xc) + (p[1] - w->yc) * (p[1] - w->yc)));
}

/* Move the photon to the first of: the wall of the current cylinder, or
 * the plane z = +-H/2 it is heading to; then pull it back inside the
 * column if rounding left it at r > R - 1e-5 (dist_to_surface,
 * kernel_cuda_c_ver1_0.cu:966-1186).  Returns the distance, or -99 when
 * the photon is lost or killed out of column. */
static float o_to_wall(o_walk *w)
{
    O_CALL(FD2O_CALL_TO_WALL);
    const fd2o_geom *g = w->g;
    float *p = w->pos, *d = w->dcos;
    const float start[3] = {p[0], p[1], p[2]};
    if (w->rebound == 0) {
        w->xc = (float)w->ex;
        w->yc = (float)w->ey;
    }
    float qa = d[0] * d[0] + d[1] * d[1];
    float qb = 2.0f * (((p[0] - w->xc) * d[0]) + ((p[1] - w->yc) * d[1]));
    float qc = (p[0] - w->xc) * (p[0] - w->xc) + (p[1] - w->yc) * (p[1] - w->yc) - (g->R * g->R);
    double root = sqrt((double)((qb * qb) - (4.0f * qa * qc)));
    float r1 = (float)(((double)(-qb) + root) / (double)(2.0f * qa));
    float r2 = (float)(((double)(-qb) - root) / (double)(2.0f * qa));
    float dcyl = 999.0f;
    if (r1 >= r2) dcyl = r1;
    else if (r2 > r1) dcyl = r2;

    float dist;
    if (d[2] != 0.0f) {
        float zp = d[2] > 0.0f ? g->H / 2.0f : -g->H / 2.0f;
        float axis = d[2] > 0.0f ? 1.0f : -1.0f;
        int straight = fabs((double)d[0]) < O_EPS && fabs((double)d[1]) < O_EPS &&
                       fabs((double)(d[2] - axis)) < O_EPS;
        float dplane = (zp - p[2]) / d[2];
        if (!straight && dplane >= dcyl) {
            dist = dcyl;
            p[2] = start[2] + dist * d[2];
        } else {
            dist = dplane;
            p[2] = zp;
        }
    } else {
        dist = dcyl;
        p[2] = start[2] + dist * d[2];
    }
    p[0] = start[0] + dist * d[0];
    p[1] = start[1] + dist * d[1];

    if (o_outside_detector(w)) {
        o_count(w, C_LOST, FD2O_FATE_LOST);
        return -99.0f;
    }
    float r = o_radius(w);
    float step = 0.5f;
    int moved = 0, halved = 0;
    while ((double)r > (double)g->R - 1e-5 && moved < 10 && halved < 10) {
        O_CALL(FD2O_CALL_PULLBACK);
        float sx = p[0], sy = p[1];
        p[0] = p[0] + step * (-d[0]);
        p[1] = p[1] + step * (-d[1]);
        float r_new = o_radius(w);
        if (r_new > r) {
            p[0] = sx;
            p[1] = sy;
            step = step / 2.0f;
            halved++;
        } else {
            r = r_new;
            moved++;
        }
    }
    if ((double)r > (double)g->R - 1e-5) {
        o_count(w, C_OUTOFCOL, FD2O_FATE_OUTOFCOL);
        return -99.0f;
    }
    if (o_outside_detector(w)) {
        o_count(w, C_LOST, FD2O_FATE_LOST);
        return -99.0f;
    }
    return dist;
}

/* Wall distance against exponential bulk-absorption distance
 * (isotropic, kernel_cuda_c_ver1_0.cu:702-740).  1 = photon ended. */
static int o_flight(o_walk *w)
{
    const fd2o_geom *g = w->g;
    float dsurf = o_to_wall(w);
    float dabs = 999999.0f;
    if (g->bulk_abs > 0.0f) dabs = (float)((double)(-1.0f / g->bulk_abs) * log((double)o_u(w)));
    if (fabs((double)(dsurf - (-99.0f))) < O_EPS) return 1;
    if (dsurf < dabs && dsurf >= 0.0f) return 0;
    if (dsurf >= dabs && dsurf >= 0.0f) {
        o_count(w, C_ABS_BULK, FD2O_FATE_ABS_BULK);
        return 1;
    }
    return 0;
}

/* At z = -H/2 inside a column: specular reflection with probability
 * sensorRefl followed by a new flight, else detection
 * (detection, kernel_cuda_c_ver1_0.cu:3372-3427).  1 = photon ended. */
static int o_sensor(o_walk *w)
{
    const fd2o_geom *g = w->g;
    if (fabs((double)(w->pos[2] - (float)(-g->H / 2.0f))) >= O_EPS) return 0;
    if (o_u(w) < g->sensor_refl) {
        w->normal[0] = 0.0f;
        w->normal[1] = 0.0f;
        w->normal[2] = 1.0f;
        o_redirect(w, 0.0f, 0.0f, 0);
        return o_flight(w) == 1;
    }
    o_detected(w);
    return 1;
}

/* Orientation of the next column: a random normal within 1.57 rad of the
 * reversed travel direction inv, flattened to the x-y plane and roughened
 * (the newnormal loops of transmit/refl_bottom/boundary_analysis).  Each
 * retry increments *tries; after 100 the photon is killed (return 1). */
static int o_next_column_normal(o_walk *w, const float inv[3], int *tries, int always_rough)
{
    const fd2o_geom *g = w->g;
    float *n = w->normal;
    for (;;) {
        O_CALL(FD2O_CALL_NEW_NORMAL);
        n[0] = inv[0];
        n[1] = inv[1];
        n[2] = inv[2];
        o_rough(w, 1.0f);
        float den = (float)sqrt((double)(n[0] * n[0] + n[1] * n[1]));
        n[2] = 0.0f;
        n[0] = n[0] / den;
        n[1] = n[1] / den;
        if (always_rough || g->beta > 0.0f) o_rough(w, g->beta);
        float ang = acosf(o_dot(inv, n));
        if (!(ang < 0.0f || ang > 1.57f)) return 0;
        if (*tries < 100) {
            (*tries)++;
            continue;
        }
        o_count(w, C_THETA1, FD2O_FATE_THETA1);
        return 1;
    }
}

static void o_set_normal(o_walk *w, float x, float y, float z)
{
    w->normal[0] = x;
    w->normal[1] = y;
    w->normal[2] = z;
}

/* Hop of U(d_min, d_max) after the sensor reflected the photon between
 * columns; lands on a new column or the top (refl_bottom,
 * kernel_cuda_c_ver1_0.cu:2985-3087).  1 = photon ended. */
static int o_hop_from_sensor(o_walk *w)
{
    const fd2o_geom *g = w->g;
    float *p = w->pos, *d = w->dcos;
    const float start[3] = {p[0], p[1], p[2]};
    const float inv[3] = {-d[0], -d[1], -d[2]};
    float hop = o_u(w) * (g->d_max - g->d_min) + g->d_min;
    float dtop = ((g->H / 2.0f) - start[2]) / d[2];
    p[0] = start[0] + d[0] * hop;
    p[1] = start[1] + d[1] * hop;
    p[2] = start[2] + d[2] * hop;
    if ((double)p[0] < O_EPS || p[0] > g->xdet || (double)p[1] < O_EPS || p[1] > g->ydet) {
        o_count(w, C_LOST, FD2O_FATE_LOST);
        return 1;
    }
    if (p[2] > g->H / 2.0f) {
        if (dtop < hop && (double)dtop > O_EPS) {
            p[0] = start[0] + d[0] * dtop;
            p[1] = start[1] + d[1] * dtop;
            p[2] = g->H / 2.0f;
            return 0;
        }
        o_count(w, C_LOST, FD2O_FATE_LOST);
        return 1;
    }
    int tries = 0;
    return o_next_column_normal(w, inv, &tries, 1);
}

static int o_at_top(const o_walk *w)
{
    return fabs((double)(w->pos[2] - (w->g->H / 2.0f))) < O_EPS && w->dcos[2] > 0.0f;
}

/* Sensor reached between columns: reflect with probability sensorRefl and
 * hop (returns 0, or 2 when the hop ended on the top surface heading up),
 * else detect (returns 1). */
static int o_sensor_between(o_walk *w)
{
    if (o_u(w) < w->g->sensor_refl) {
        o_set_normal(w, 0.0f, 0.0f, 1.0f);
        o_redirect(w, 0.0f, 0.0f, 0);
        if (o_hop_from_sensor(w)) return 1;
        return o_at_top(w) ? 2 : 0;
    }
    o_detected(w);
    return 1;
}

/* Leave the current column (transmit, kernel_cuda_c_ver1_0.cu:2421-2865).
 * crosstalk != 0: cross straight into an adjacent column of random
 * orientation.  Otherwise travel U(d_min, d_max), handling the top
 * reflector and the sensor on the way, then orient the next column.
 * 1 = photon ended. */
static int o_leave_column(o_walk *w, int crosstalk)
{
    O_CALL(crosstalk ? FD2O_CALL_CROSSTALK : FD2O_CALL_HOP);
    const fd2o_geom *g = w->g;
    float *p = w->pos, *d = w->dcos;
    float start[3] = {p[0], p[1], p[2]};
    float inv[3] = {-d[0], -d[1], -d[2]};
    int tries = 0, tries_top = 0;
    if (crosstalk) return o_next_column_normal(w, inv, &tries, 0);

    const float half = g->H / 2.0f;
    float hop = o_u(w) * (g->d_max - g->d_min) + g->d_min;
    p[0] = start[0] + d[0] * hop;
    p[1] = start[1] + d[1] * hop;
    p[2] = start[2] + d[2] * hop;
    float dtop = (half - start[2]) / d[2];
    float dbot = ((-g->H / 2.0f) - start[2]) / d[2];
    if ((double)p[0] < O_EPS || p[0] > g->xdet || (double)p[1] < O_EPS || p[1] > g->ydet) {
        o_count(w, C_LOST, FD2O_FATE_LOST);
        return 1;
    }
    int to_top = 0;
    if (p[2] < -g->H / 2.0f || p[2] > half) {
        if (dtop < hop && (double)dtop > O_EPS) {
            p[0] = start[0] + d[0] * dtop;
            p[1] = start[1] + d[1] * dtop;
            p[2] = half;
        } else if (dbot < hop && (double)dbot > O_EPS) {
            p[0] = start[0] + d[0] * dbot;
            p[1] = start[1] + d[1] * dbot;
            p[2] = -g->H / 2.0f;
            int s = o_sensor_between(w);
            if (s == 1) return 1;
            to_top = (s == 2);
        } else {
            o_count(w, C_LOST, FD2O_FATE_LOST);
            return 1;
        }
    }
    if (!to_top) {
        if (o_next_column_normal(w, inv, &tries, 0)) return 1;
        if (fabs((double)(p[0] - 0.0f)) < O_EPS || fabs((double)(p[0] - g->xdet)) < O_EPS ||
            fabs((double)(p[1] - 0.0f)) < O_EPS || fabs((double)(p[1] - g->ydet)) < O_EPS) {
            o_count(w, C_LOST, FD2O_FATE_LOST);
            return 1;
        }
    }
    for (;;) {
        if (o_at_top(w)) {
            o_set_normal(w, 0.0f, 0.0f, -1.0f);
            if (g->top_absfrac > 0.0f && o_u(w) < g->top_absfrac) {
                o_count(w, C_ABS_TOP, FD2O_FATE_ABS_TOP);
                return 1;
            }
            /* isotropic reflection back down, then another hop */
            d[2] = (float)(-fabs((double)((o_u(w) * 2.0f) - 1.0f)));
            float rr = (float)sqrt((double)(1.0f - d[2] * d[2]));
            float phi = (float)((double)o_u(w) * O_TWOPI);
            d[0] = (float)((double)rr * cos((double)phi));
            d[1] = (float)((double)rr * sin((double)phi));
            for (int k = 0; k < 3; ++k) {
                start[k] = p[k];
                inv[k] = -d[k];
            }
            hop = o_u(w) * (g->d_max - g->d_min) + g->d_min;
            dbot = ((-g->H / 2.0f) - start[2]) / d[2];
            p[0] = start[0] + d[0] * hop;
            p[1] = start[1] + d[1] * hop;
            p[2] = start[2] + d[2] * hop;
            if ((double)p[0] < O_EPS || p[0] > g->xdet || (double)p[1] < O_EPS || p[1] > g->ydet) {
                o_count(w, C_LOST, FD2O_FATE_LOST);
                return 1;
            }
            if (p[2] < -g->H / 2.0f || p[2] > half) {
                if (dbot < hop && (double)dbot > O_EPS) {
                    p[0] = start[0] + d[0] * dbot;
                    p[1] = start[1] + d[1] * dbot;
                    p[2] = -g->H / 2.0f;
                    int s = o_sensor_between(w);
                    if (s == 1) return 1;
                    if (s == 2) continue;
                } else {
                    o_count(w, C_LOST, FD2O_FATE_LOST);
                    return 1;
                }
            }
            if (o_next_column_normal(w, inv, &tries_top, 0)) return 1;
        }
        if (fabs((double)(p[2] - (-g->H / 2.0f))) < O_EPS) {
            int s = o_sensor_between(w);
            if (s == 1) return 1;
            if (s == 2) continue;
        }
        return 0;
    }
}

/* Fresnel probabilities from the angles (boundary_analysis,
 * kernel_cuda_c_ver1_0.cu:1818-1819 and repeats). */
static void o_fresnel(float t1, float t2, float *pr, float *pt)
{
    O_CALL(FD2O_CALL_FRESNEL);
    double dm = (double)(t1 - t2), dp = (double)(t1 + t2);
    double s2 = sin((double)(2.0f * t1)) * sin((double)(2.0f * t2));
    *pr = (float)(0.5f * ((pow(tan(dm), 2) / pow(tan(dp), 2)) + (pow(sin(dm), 2) / pow(sin(dp), 2))));
    *pt = (float)(0.5f * ((s2 / (pow(sin(dp), 2) * pow(cos(dm), 2))) + (s2 / pow(sin(dp), 2))));
}

enum { BA_NEW_SURFACE, BA_RESTORE, BA_INCIDENCE };

/* Interaction with a surface (boundary_analysis,
 * kernel_cuda_c_ver1_0.cu:1582-1958): top absorber/reflector, columnar
 * crosstalk, or Fresnel reflection/refraction on a rough wall with the
 * reference's resampling rules.  Returns 1 when the photon ended. */
static int o_surface(o_walk *w)
{
    O_CALL(FD2O_CALL_SURFACE);
    const fd2o_geom *g = w->g;
    float *p = w->pos, *d = w->dcos, *n = w->normal;
    const float half = g->H / 2.0f;

    if (fabs((double)(p[2] - (float)(g->H / 2.0f))) < O_EPS && d[2] > 0.0f) {
        if (g->top_absfrac > 0.0f && o_u(w) < g->top_absfrac) {
            o_count(w, C_ABS_TOP, FD2O_FATE_ABS_TOP);
            return 1;
        }
        o_set_normal(w, 0.0f, 0.0f, -1.0f);
        d[2] = (float)(-fabs((double)((o_u(w) * 2.0f) - 1.0f)));
        float rr = (float)sqrt((double)(1.0f - d[2] * d[2]));
        float phi = (float)((double)o_u(w) * O_TWOPI);
        d[0] = (float)((double)rr * cos((double)phi));
        d[1] = (float)((double)rr * sin((double)phi));
        return 0;
    }

    /* columnar crosstalk probability: 1 in the top 20 %, linear to 0.5 at
     * mid depth, back to 1 at the sensor */
    float top_band = g->H * 0.2f;
    float cct = 0.0f;
    if (p[2] <= half && p[2] >= (half - top_band)) cct = 1.0f;
    else if (p[2] < (half - top_band) && p[2] >= 0.0f)
        cct = (float)((double)(p[2] / (2.0f * (half - top_band))) + 0.5);
    else if (p[2] < 0.0f && p[2] >= (-g->H / 2.0f))
        cct = (float)((double)((p[2] - (-g->H / 2.0f)) / (2.0f * (-g->H / 2.0f))) + 1.0);
    if (o_u(w) < cct) {
        if (o_leave_column(w, 1)) return 1;
        w->xc = (float)(p[0] + g->R * (-n[0]));
        w->yc = (float)(p[1] + g->R * (-n[1]));
        return 0;
    }

    int outside = 0; /* between columns after a refraction out of the column */
    int tries_theta = 0, tries_normal = 0, reperturbs = 0, smooth_retries = 0;
    float pr = 0.0f, pt = 0.0f, t1 = 0.0f, t2 = 0.0f;
    float keep_n[3], keep_d[3], inv[3];
    int stage = BA_NEW_SURFACE;
    for (;;) {
        if (stage == BA_NEW_SURFACE) {
            if (!outside) {
                float mag = (float)sqrt((double)(((w->xc - p[0]) * (w->xc - p[0])) +
                                                 ((w->yc - p[1]) * (w->yc - p[1]))));
                n[0] = (w->xc - p[0]) / mag;
                n[1] = (w->yc - p[1]) / mag;
                n[2] = 0.0f;
                if (g->beta > 0.0f) o_rough(w, g->beta);
            } else {
                w->xc = (float)(p[0] + g->R * (-n[0]));
                w->yc = (float)(p[1] + g->R * (-n[1]));
            }
            for (int k = 0; k < 3; ++k) {
                keep_n[k] = n[k];
                keep_d[k] = d[k];
            }
            stage = BA_RESTORE;
        }
        if (stage == BA_RESTORE) {
            for (int k = 0; k < 3; ++k) {
                n[k] = keep_n[k];
                d[k] = keep_d[k];
            }
            if (reperturbs != 0 && g->beta > 0.0f) o_rough(w, g->beta);
            if (reperturbs != 0 && outside) {
                w->xc = (float)(p[0] + g->R * (-n[0]));
                w->yc = (float)(p[1] + g->R * (-n[1]));
            }
            stage = BA_INCIDENCE;
        }
        /* BA_INCIDENCE */
        O_CALL(FD2O_CALL_INCIDENCE);
        for (int k = 0; k < 3; ++k) inv[k] = -d[k];
        t1 = o_dot(inv, n);
        if (t1 > 1.0f || t1 < 0.0f) {
            if (outside && o_next_column_normal(w, inv, &tries_normal, 0)) return 1;
            if (tries_theta < 100) {
                tries_theta++;
                stage = BA_NEW_SURFACE;
                continue;
            }
            o_count(w, C_THETA1, FD2O_FATE_THETA1);
            return 1;
        }
        t1 = acosf(t1);
        if (!outside) {
            if ((double)t1 > asin((double)(g->n_gap / g->n_col))) {
                pr = 1.0f;
                pt = 0.0f;
            } else {
                if ((double)t1 < O_EPS) t1 = (float)0.00042;
                t2 = asinf((float)((double)(float)(g->n_col / g->n_gap) * sin((double)t1)));
                o_fresnel(t1, t2, &pr, &pt);
            }
        } else if ((g->n_col / g->n_gap) < 1.57f) {
            /* only TIR is decided here; otherwise pr, pt keep their values */
            if ((double)t1 > asin((double)(g->n_col / g->n_gap))) {
                pr = 1.0f;
                pt = 0.0f;
            }
        } else if ((double)t1 < O_EPS) {
            t1 = (float)0.00042;
            t2 = asinf((float)((double)(float)(g->n_col / g->n_gap) * sin((double)t1)));
            o_fresnel(t1, t2, &pr, &pt);
        } else {
            t2 = asinf((float)((double)(float)(g->n_gap / g->n_col) * sin((double)t1)));
            o_fresnel(t1, t2, &pr, &pt);
        }
        float total = pr + pt;
        pr = pr / total;
        pt = pt / total;

        if (o_u(w) < pr) {
            o_redirect(w, t1, t2, 0);
            if (acosf(o_dot(keep_n, d)) > 1.57f) {
                reperturbs++;
                if (reperturbs < 4) {
                    stage = BA_RESTORE;
                    continue;
                }
                for (int k = 0; k < 3; ++k) {
                    n[k] = keep_n[k];
                    d[k] = keep_d[k];
                }
                reperturbs = 0;
                if (smooth_retries < 25) {
                    smooth_retries++;
                    stage = BA_INCIDENCE;
                    continue;
                }
                o_count(w, C_THETA1, FD2O_FATE_THETA1);
                return 1;
            }
            if (!outside) return 0;
            if (o_leave_column(w, 0)) return 1;
            stage = BA_NEW_SURFACE;
            continue;
        }
        o_redirect(w, t1, t2, 1);
        if (outside) return 0;
        outside = 1;
        if (o_leave_column(w, 0)) return 1;
        stage = BA_NEW_SURFACE;
    }
}

/* Restart the current photon from the event position with a new
 * direction (after termination, or when trapped with dcos_z ~ 0). */
static void o_restart(o_walk *w)
{
    o_emit(w, 0);
    w->pos[0] = (float)w->ex;
    w->pos[1] = (float)w->ey;
    w->pos[2] = (float)w->ez;
    o_set_normal(w, 0.0f, 0.0f, 0.0f);
    if (w->g->beta > 0.0f) o_rough(w, w->g->beta);
    w->absorbed = 0;
    w->detect = 0;
    w->bulk_abs = 0;
}

/* One call of the C transport step (algo, kernel_cuda_c_ver1_0.cu:553-658).
 * Returns 1 when the photon terminated in this call. */
static int o_step(o_walk *w)
{
    O_CALL(FD2O_CALL_STEP);
    if (w->absorbed == 0) {
        w->bulk_abs = o_flight(w);
        if (w->bulk_abs == 0) w->detect = o_sensor(w);
    }
    if (w->detect == 1 || w->absorbed == 1 || w->bulk_abs == 1) {
        o_restart(w);
        return 1;
    }
    if (fabs((double)(w->dcos[2] - 0.0f)) < O_EPS) {
        o_restart(w);
        return 0;
    }
    w->rebound++;
    w->absorbed = o_surface(w);
    return 0;
}

int fd2o_run(const fd2o_geom *g, int n_events,
             const double *x_um, const double *y_um, const double *z_um,
             const int32_t *hist, const int32_t *nphot,
             int32_t seed_input, int64_t event_index_base,
             int32_t prim_size, int32_t xdim, int32_t ydim,
             uint64_t *image, int32_t *per_primary, uint64_t *counters,
             int8_t *fate, int32_t *pix, int32_t *seeds, int32_t *steps)
{
    if (!g || n_events < 0 || !x_um || !y_um || !z_um || !hist || !nphot || !image ||
        !per_primary || !counters || xdim < 0 || ydim < 0 || prim_size < 0)
        return -1;
    o_walk w;
    memset(&w, 0, sizeof w);
    w.g = g;
    w.xdim = xdim;
    w.ydim = ydim;
    w.prim_size = prim_size;
    w.image = image;
    w.per_primary = per_primary;
    w.cnt = counters;
    int64_t rec = 0;
    for (int e = 0; e < n_events; ++e) {
        if (nphot[e] < 0) return -1;
        fd2o_init_prng(event_index_base + e, 50000, seed_input, w.seed);
        w.ex = x_um[e];
        w.ey = y_um[e];
        w.ez = z_um[e];
        w.hist = hist[e];
        w.pos[0] = (float)w.ex;
        w.pos[1] = (float)w.ey;
        w.pos[2] = (float)w.ez;
        o_set_normal(&w, 0.0f, 0.0f, 0.0f);
        o_emit(&w, 1);
        for (int32_t k = 0; k < nphot[e]; ++k, ++rec) {
            w.absorbed = 0;
            w.detect = 0;
            w.bulk_abs = 0;
            w.pos[0] = (float)w.ex;
            w.pos[1] = (float)w.ey;
            w.pos[2] = (float)w.ez;
            w.rebound = 0;
            w.fate = FD2O_FATE_NONE;
            w.pix_i = -1;
            w.pix_j = -1;
            counters[C_GEN]++;
            int32_t calls = 0;
            do {
                calls++;
            } while (o_step(&w) == 0);
            if (fate) fate[rec] = (int8_t)w.fate;
            if (pix) {
                pix[2 * rec] = w.fate == FD2O_FATE_DETECT ? w.pix_i : -1;
                pix[2 * rec + 1] = w.fate == FD2O_FATE_DETECT ? w.pix_j : -1;
            }
            if (seeds) {
                seeds[2 * rec] = w.seed[0];
                seeds[2 * rec + 1] = w.seed[1];
            }
            if (steps) steps[rec] = calls;
        }
    }
    return 0;
}

int fd2o_phs(const int32_t *per_primary, int32_t num_primary,
             int32_t min_photons, int32_t max_photons, int32_t num_bins,
             int32_t *histogram)
{
    if (num_bins <= 0) return -1;
    int32_t width = (max_photons - min_photons) / num_bins;
    if (width <= 0) return -1;
    int32_t shift = min_photons / width;
    for (int32_t i = 0; i < num_primary; ++i) {
        int32_t c = per_primary[i];
        if (c <= 0) continue;
        int32_t bin;
        if (c <= min_photons) bin = 0;
        else if (c >= max_photons) bin = num_bins - 1;
        else bin = c / width - shift;
        if (bin >= 0 && bin < num_bins) histogram[bin]++;
    }
    return 0;
}
