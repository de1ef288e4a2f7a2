/*
 * fd2_oracle.h -- CPU oracle for the fastDETECT2 optical transport.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker: tests/, the smoke entry
 * point and bench.py's cpu_baseline leg load it; the product library
 * (hybridmantis_b200/) never links, loads or calls it.
 *
 * It restates, in plain C, the reference's CPU path for one buffer of
 * energy-deposition events (EDEs):
 *   - driver loop        main/hybridMANTIS_c_ver1_0.c:189-340 (cpuoptical_)
 *   - transport step     main/kernel_cuda_c_ver1_0.cu:553-658  (C algo)
 *   - helpers            main/kernel_cuda_c_ver1_0.cu (C branches of
 *                        isotropic, dist_to_surface, boundary_analysis,
 *                        transmit, refl_bottom, trans_dir_cos,
 *                        RoughSurface, detection, init_PRNG, ranecu)
 *   - PHS binning        main/hybridMANTIS_c_ver1_0.c:342-366
 * with the float/double mix of the reference C expressions kept exactly,
 * so that photon fates, pixels and RANECU states are bit-identical to the
 * reference's own C functions for the same seeds.  Parity is pinned by
 * tests against the reference compiled in place (oracle/_ref, built by
 * oracle/Makefile from the reference sources).
 *
 * Differences from cpuoptical_ (all deliberate, all in the driver):
 *   - seed_input is a parameter (the reference uses wall-clock time);
 *   - photon counts are given per event (the reference samples them with
 *     GSL's Poisson generator, which is not vendored);
 *   - the PRF image has caller-chosen dimensions, row-major [ii][jj]
 *     (ii = x pixel), and pixels outside it are skipped instead of
 *     written past the end of the array;
 *   - per-photon records (fate, pixel, RNG state, step count) are kept.
 */
#ifndef FD2_ORACLE_H
#define FD2_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Photon fates, shared numbering with the product's replay records. */
enum {
    FD2O_FATE_NONE = 0,
    FD2O_FATE_DETECT = 1,     /* reached the sensor plane and was detected */
    FD2O_FATE_ABS_TOP = 2,    /* absorbed at the top surface */
    FD2O_FATE_ABS_BULK = 3,   /* absorbed in the bulk */
    FD2O_FATE_LOST = 4,       /* left the detector laterally / vertically */
    FD2O_FATE_OUTOFCOL = 5,   /* killed by the out-of-column repair loop */
    FD2O_FATE_THETA1 = 6      /* killed after exhausting normal resampling */
};

/* Detector parameters in the reference's float form (cpuoptical_ copies the
 * double inputargs_ values into these floats, hybridMANTIS_c_ver1_0.c:146-168). */
typedef struct {
    float xdet, ydet, H, R, n_col, n_gap, top_absfrac, bulk_abs, beta;
    float d_min, d_max, lb_x, lb_y, ub_x, ub_y, sensor_refl;
    int pixel;
} fd2o_geom;

/* Counters, in the order generated, detect, abs_top, abs_bulk, lost,
 * outofcol, theta1. */
#define FD2O_NCOUNTERS 7

/*
 * Transport n_events events.  Event e uses the RANECU stream
 * init_PRNG(event_index_base + e, 50000, seed_input).
 *   x_um, y_um, z_um : event position in micrometres (double, as the
 *                      reference's struct start_info holds them)
 *   hist             : 1-based x-ray history number
 *   nphot            : optical photons to transport for the event
 *   image            : xdim*ydim counts, index ii*ydim + jj, accumulated
 *   per_primary      : detected photons per history, indexed hist-1,
 *                      prim_size entries, accumulated
 *   counters         : FD2O_NCOUNTERS entries, accumulated
 *   Optional per-photon outputs (NULL to skip), photon p of event e at
 *   offset sum(nphot[0..e-1]) + p:
 *   fate   (int8) , pix (2 ints: ii, jj; -1,-1 when not in the image),
 *   seeds  (2 ints: RANECU state after the photon terminated, before the
 *           re-emission draws of the next photon),
 *   steps  (int: calls of the transport step for the photon)
 * Returns 0, or -1 on invalid arguments.
 */
int fd2o_run(const fd2o_geom *g, int n_events,
             const double *x_um, const double *y_um, const double *z_um,
             const int32_t *hist, const int32_t *nphot,
             int32_t seed_input, int64_t event_index_base,
             int32_t prim_size, int32_t xdim, int32_t ydim,
             uint64_t *image, int32_t *per_primary, uint64_t *counters,
             int8_t *fate, int32_t *pix, int32_t *seeds, int32_t *steps);

/* Call counts of the transport's building blocks since the last reset,
 * FD2O_NCALLS entries indexed by FD2O_CALL_*; counted per host thread (a
 * reset and a read see the calling thread's transport calls). */
enum {
    FD2O_CALL_STEP, FD2O_CALL_TO_WALL, FD2O_CALL_PULLBACK, FD2O_CALL_SURFACE, FD2O_CALL_INCIDENCE,
    FD2O_CALL_FRESNEL, FD2O_CALL_REFLECT, FD2O_CALL_REFRACT, FD2O_CALL_CROSSTALK, FD2O_CALL_HOP,
    FD2O_CALL_NEW_NORMAL, FD2O_CALL_ROUGH, FD2O_CALL_UNIFORM, FD2O_NCALLS
};
void fd2o_reset_call_counts(void);
void fd2o_get_call_counts(uint64_t out[FD2O_NCALLS]);

/* RANECU seeds for one stream (init_PRNG, kernel_cuda_c_ver1_0.cu:3516). */
void fd2o_init_prng(int64_t history_batch, int32_t histories_per_thread,
                    int32_t seed_input, int32_t seed[2]);

/* n uniforms from a RANECU stream (ranecu, kernel_cuda_c_ver1_0.cu:3694). */
void fd2o_ranecu(int32_t seed[2], int32_t n, float *out);

/* PHS binning of per-primary counts (hybridMANTIS_c_ver1_0.c:342-366);
 * histogram is num_bins entries, accumulated.  Returns -1 when the
 * reference's integer bin size would be zero. */
int fd2o_phs(const int32_t *per_primary, int32_t num_primary,
             int32_t min_photons, int32_t max_photons, int32_t num_bins,
             int32_t *histogram);

#ifdef __cplusplus
}
#endif
#endif
