/*
 * ref_harness.c -- drives the reference's own C transport functions.
 *
 * TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles the reference file
 * main/kernel_cuda_c_ver1_0.cu as C, unmodified and where it lies, and
 * links it with this harness into oracle/_ref/libfd2ref_O{0,2}.so.  Tests
 * use it to pin the oracle restatement (fd2_oracle.c); bench.py may time
 * it as the reference CPU baseline.  Nothing of it ships in the product.
 *
 * The harness plays the role of cpuoptical_ (main/hybridMANTIS_c_ver1_0.c:
 * 189-340), which cannot be built here (GSL and the Fortran COMMON blocks
 * are absent): per event it seeds RANECU with init_PRNG(event, 50000,
 * seed_input), draws the first direction with the |cos| > 0.01 rejection,
 * and calls the reference's C step `algo` until each photon terminates.
 * Photon counts are given by the caller instead of gsl_ran_poisson.  The
 * fate of each photon is read from the reference's global counters.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* Same layout as struct start_info, kernel_cuda_c_ver1_0.cu:67-75. */
struct start_info {
    double str_x, str_y, str_z, str_E;
    int str_histnum;
    int str_N;
};

/* Symbols defined by the reference file (C branch). */
int algo(float *normal, float *old_pos, float *pos, float *dcos, unsigned long long *num_rebound,
         int *seed, struct start_info info, unsigned long long *myimage, float xdetector,
         float ydetector, float R, float H, float n1, float n2, float top_absfrac,
         float bulk_abscoeff, float beta, float d_min, int pixelsize, float lbound_x,
         float lbound_y, float ubound_x, float ubound_y, float sensorRefl, float d_max,
         int ydim, int *h_num_detected_prim);
void init_PRNG(int history_batch, int histories_per_thread, int seed_input, int *seed);
float ranecu(int *seed);
extern unsigned long long num_generated, num_detect, num_abs_top, num_abs_bulk, num_lost,
    num_outofcol, local_counter, num_theta1;
extern int absorbed, detect, bulk_abs;

/* The one Fortran COMMON block the C transport writes (the PRF image,
 * kernel_cuda_c_ver1_0.cu:151-163); here a plain C object. */
struct {
    unsigned long long newimageopt[501][501];
    unsigned long long tempimageopt[501][501];
} outputimage_;

#define RH_TWOPI 6.283185308
#define RH_EPS 8.1929093e-6

/* params: xdet, ydet, H, R, n_col, n_gap, top_absfrac, bulk_abs, beta,
 *         d_min, d_max, lb_x, lb_y, ub_x, ub_y, sensor_refl (16 floats) */
typedef struct {
    float v[16];
    int pixel;
} fd2ref_geom;

void fd2ref_init_prng(int history_batch, int histories_per_thread, int seed_input, int seed[2])
{
    init_PRNG(history_batch, histories_per_thread, seed_input, seed);
}

void fd2ref_ranecu(int seed[2], int n, float *out)
{
    for (int i = 0; i < n; ++i) out[i] = ranecu(seed);
}

/*
 * Transport n_events events (stream index event_index_base + e).
 * image501 receives the reference's 501x501 PRF of this call (zeroed
 * first, [ii][jj]); per_primary (prim_size, indexed hist-1) and counters
 * (generated, detect, abs_top, abs_bulk, lost, outofcol, theta1) are
 * accumulated.  Optional per-photon fate / RANECU state / step count.
 * Returns 0, -1 on bad arguments, -2 when a photon's fate could not be
 * attributed to exactly one counter.
 */
int fd2ref_run(const fd2ref_geom *g, int n_events, const double *x_um, const double *y_um,
               const double *z_um, const int *hist, const int *nphot, int seed_input,
               int event_index_base, int prim_size, unsigned long long *image501,
               int *per_primary, unsigned long long *counters, signed char *fate, int *seeds,
               int *steps)
{
    if (!g || n_events < 0 || !image501 || !per_primary || !counters) return -1;
    const float *p = g->v;
    float xdet = p[0], ydet = p[1], H = p[2], R = p[3], n_col = p[4], n_gap = p[5];
    float top = p[6], mu = p[7], beta = p[8], dmin = p[9], dmax = p[10];
    float lbx = p[11], lby = p[12], ubx = p[13], uby = p[14], srefl = p[15];
    int status = 0;

    memset(&outputimage_, 0, sizeof outputimage_);
    /* the reference C indexes per-primary counts by the 1-based history
     * number itself, so one extra slot is needed */
    int *prim = (int *)calloc((size_t)prim_size + 2, sizeof(int));
    if (!prim) return -1;

    long long rec = 0;
    for (int e = 0; e < n_events; ++e) {
        struct start_info info;
        info.str_x = x_um[e];
        info.str_y = y_um[e];
        info.str_z = z_um[e];
        info.str_E = 0.0;
        info.str_histnum = hist[e];
        info.str_N = nphot[e];
        if (info.str_histnum < 0 || info.str_histnum > prim_size) {
            free(prim);
            return -1;
        }
        num_generated = num_detect = num_abs_top = num_abs_bulk = 0;
        num_lost = num_outofcol = num_theta1 = 0;

        unsigned long long *rebound =
            (unsigned long long *)calloc((size_t)(info.str_N > 0 ? info.str_N : 1) + 1,
                                         sizeof(unsigned long long));
        int seed[2];
        init_PRNG(event_index_base + e, 50000, seed_input, seed);

        float dcos[3] = {0, 0, 0}, normal[3] = {0, 0, 0}, pos[3], old_pos[3];
        pos[0] = old_pos[0] = (float)info.str_x;
        pos[1] = old_pos[1] = (float)info.str_y;
        pos[2] = old_pos[2] = (float)info.str_z;

        /* first direction of the event, as cpuoptical_ draws it */
        float r = (ranecu(seed) * 2.0f) - 1.0f;
        while (fabs(r) <= 0.01f) r = (ranecu(seed) * 2.0f) - 1.0f;
        dcos[2] = r;
        float rr = sqrt(1.0f - r * r);
        float theta = ranecu(seed) * RH_TWOPI;
        dcos[0] = rr * cos(theta);
        dcos[1] = rr * sin(theta);
        float norm = sqrt(dcos[0] * dcos[0] + dcos[1] * dcos[1] + dcos[2] * dcos[2]);
        if ((norm < (1.0f - RH_EPS)) || (norm > (1.0f + RH_EPS))) {
            dcos[0] = dcos[0] / norm;
            dcos[1] = dcos[1] / norm;
            dcos[2] = dcos[2] / norm;
        }

        local_counter = 0;
        while (local_counter < (unsigned long long)info.str_N) {
            absorbed = 0;
            detect = 0;
            bulk_abs = 0;
            pos[0] = old_pos[0] = (float)info.str_x;
            pos[1] = old_pos[1] = (float)info.str_y;
            pos[2] = old_pos[2] = (float)info.str_z;
            num_generated++;
            unsigned long long before[6] = {num_detect, num_abs_top, num_abs_bulk,
                                            num_lost, num_outofcol, num_theta1};
            int calls = 0, done = 0;
            while (done == 0) {
                calls++;
                done = algo(normal, old_pos, pos, dcos, rebound, seed, info,
                            &outputimage_.newimageopt[0][0], xdet, ydet, R, H, n_col, n_gap, top,
                            mu, beta, dmin, 1 * g->pixel, lbx, lby, ubx, uby, srefl, dmax, 501,
                            prim);
            }
            unsigned long long after[6] = {num_detect, num_abs_top, num_abs_bulk,
                                           num_lost, num_outofcol, num_theta1};
            int which = -1, changed = 0;
            for (int k = 0; k < 6; ++k)
                if (after[k] != before[k]) {
                    changed += (int)(after[k] - before[k]);
                    which = k;
                }
            if (changed != 1) status = -2;
            if (fate) fate[rec] = (signed char)(changed == 1 ? which + 1 : -1);
            if (seeds) {
                seeds[2 * rec] = seed[0];
                seeds[2 * rec + 1] = seed[1];
            }
            if (steps) steps[rec] = calls;
            rec++;
        }
        free(rebound);
        counters[0] += num_generated;
        counters[1] += num_detect;
        counters[2] += num_abs_top;
        counters[3] += num_abs_bulk;
        counters[4] += num_lost;
        counters[5] += num_outofcol;
        counters[6] += num_theta1;
    }
    for (int h = 1; h <= prim_size; ++h) per_primary[h - 1] += prim[h];
    memcpy(image501, &outputimage_.newimageopt[0][0], sizeof outputimage_.newimageopt);
    free(prim);
    return status;
}
