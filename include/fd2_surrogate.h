/*
 * fd2_surrogate.h -- learned surrogate of the optical transport.
 *
 * No counterpart in the reference: hybridMANTIS always runs the full
 * optical Monte Carlo.  This is a small MLP that maps one energy
 * deposition (depth below the entrance surface, deposited energy, lateral
 * distance from the detector centre) and the detector geometry (thickness, column radius,
 * roughness, top reflectivity, bulk absorption) to
 *   - the probability that one optical photon from it is detected, and
 *   - the radial distribution of the detected photons around the deposition
 *     (an 8-component Gaussian mixture in r, truncated to r >= 0),
 * trained only on labels produced by this library's own Monte Carlo
 * (fd2_options.radial_bins label mode), with hand-written BF16 tensor-core
 * GEMMs (FP32 accumulation) for the forward and backward passes and Adam.
 *
 * In the event pipeline (fd2_sg_run) each event inside the training hull
 * draws its detected photon count from Binomial(N, p) and the detected
 * photons' positions from the mixture; events outside the hull are
 * transported by the Monte Carlo; a random audit fraction of the in-hull
 * events is also transported by the Monte Carlo (label mode) to measure the
 * surrogate's error on this very run.
 *
 * Feature vector (FD2_SG_FEATURES floats), in physical units:
 *   0 depth below the entrance (top) surface, um   (z = H/2 - depth)
 *   1 deposited energy, keV
 *   2 lateral distance of the deposition from the detector centre, in units
 *     of 50 um (photons that reach the detector's sides are lost, so the
 *     detected fraction falls with it: about -5e-6 per um^2 of r^2 on the
 *     500 um detector, -0.07 % at 10 um and -1.2 % at 50 um)
 *   3 thickness H, um     4 column radius R, um    5 roughness beta
 *   6 top reflectivity (1 - top_absfrac)           7 log10(bulk absorption, 1/um)
 * Network outputs (FD2_SG_OUTPUTS per point): [0] detection logit,
 * [1..8] weight logits of an 8-component mixture of Gaussian rings
 * (PRF(r) = sum_k w_k N(r; mu_k, sd_k) / S_k per unit area), [9..16] ring
 * radii (mu = 50 um * softplus(.)), [17..24] log widths (sd = 10 um *
 * exp(.), clamped to [-6, 4]).  Radial label categories: bin j <
 * radial_bins covers r_max (j/bins)^2 .. r_max ((j+1)/bins)^2, the last is
 * r >= r_max.
 */
#ifndef FD2_SURROGATE_H
#define FD2_SURROGATE_H

#include "fd2.h"

#ifdef __cplusplus
extern "C" {
#endif

#define FD2_SG_FEATURES 8
#define FD2_SG_OUTPUTS 25
#define FD2_SG_COMPONENTS 8

typedef struct fd2_sg fd2_sg;

typedef struct fd2_sg_config {
    int32_t device;
    int32_t hidden;          /* width of the three hidden layers (multiple of 64; 256) */
    int32_t radial_bins;     /* label histogram bins up to radial_max_um (+1 beyond); 96 */
    double radial_max_um;    /* 400 */
    int32_t batch;           /* training batch (multiple of 64; 8192) */
    float lr, beta1, beta2, adam_eps;
    float radial_weight;     /* weight of the radial loss beside the detection loss */
    float lateral_um;        /* fd2_sg_run: depositions farther than this from the
                                detector centre (in x or y) go to the Monte Carlo;
                                the labels sit at the centre, so their far light is
                                what the detector's edges leave from there; 50 */
    uint64_t seed;           /* initialisation and batch sampling */
    float depth_margin_um;   /* fd2_sg_run: a deposition at most this far outside the
                                hull's depth range (the labels leave out the first and
                                last 0.1 % of the layer) is given the range's edge
                                depth and goes to the network; 1 */
} fd2_sg_config;

/* Box of the training data: events whose features lie outside it go to the
 * Monte Carlo.  The first hull a new network gets (fd2_sg_set_data or
 * fd2_sg_set_hull) also fixes its input normalisation, which then stays with
 * the network (saved, loaded); later hulls only change the routing, e.g.
 * narrowed to the data of a continued training. */
typedef struct fd2_sg_hull {
    float lo[FD2_SG_FEATURES];
    float hi[FD2_SG_FEATURES];
} fd2_sg_hull;

/* Surrogate-in-the-loop run statistics. */
typedef struct fd2_sg_stats {
    int64_t events, surrogate_events, mc_events, audit_events;
    int64_t surrogate_photons;       /* photons generated in surrogate events */
    int64_t surrogate_detected;      /* photons the surrogate detected        */
    double audit_mc_detected;        /* audited events: MC detected photons   */
    double audit_sg_expected;        /* audited events: sum of N p            */
    double audit_photons;            /* audited events: photons generated     */
    double audit_z;                  /* (MC - expected) / binomial SE         */
    double audit_radial_l1;          /* L1 between pooled MC and predicted radial bin probabilities */
    float sg_ms, mc_ms, audit_ms, total_ms;
} fd2_sg_stats;

FD2_API void fd2_sg_default_config(fd2_sg_config *cfg);
FD2_API fd2_status fd2_sg_create(const fd2_sg_config *cfg, fd2_sg **out);
FD2_API void fd2_sg_destroy(fd2_sg *sg);
FD2_API const char *fd2_sg_last_error(const fd2_sg *sg);

/* Training data (host arrays): n points of features [n][8], photons per
 * point, detected photons per point and the radial label histogram
 * [n][radial_bins + 1].  The last n_val points are held out.  The hull is
 * set from the training points. */
FD2_API fd2_status fd2_sg_set_data(fd2_sg *sg, const float *features, const int32_t *photons,
                                   const int32_t *detected, const uint32_t *radial, int64_t n, int64_t n_val);
/* `steps` Adam steps on batches drawn uniformly from the training points;
 * returns the mean training loss of the last steps and the held-out loss. */
FD2_API fd2_status fd2_sg_train(fd2_sg *sg, int32_t steps, float *train_loss, float *val_loss);
/* Adam step size of the following training steps (schedules). */
FD2_API fd2_status fd2_sg_set_lr(fd2_sg *sg, float lr);
/* Loss on the held-out points (or all points when n_val = 0). */
FD2_API fd2_status fd2_sg_eval(fd2_sg *sg, float *loss, float *det_loss, float *radial_loss);

/* Parameters: FP32 masters, in the order W1 [hidden][8], b1, W2, b2, W3, b3,
 * W4 [25][hidden], b4 (n_params floats; the GEMMs use their BF16 copies). */
FD2_API int64_t fd2_sg_num_params(const fd2_sg *sg);
FD2_API fd2_status fd2_sg_get_params(fd2_sg *sg, float *params, int64_t n);
FD2_API fd2_status fd2_sg_set_params(fd2_sg *sg, const float *params, int64_t n);
FD2_API fd2_status fd2_sg_get_hull(fd2_sg *sg, fd2_sg_hull *hull);
FD2_API fd2_status fd2_sg_set_hull(fd2_sg *sg, const fd2_sg_hull *hull);
FD2_API fd2_status fd2_sg_save(fd2_sg *sg, const char *path);
FD2_API fd2_status fd2_sg_load(fd2_sg *sg, const char *path);
/* Edge survival of the sampled azimuths in fd2_sg_run: a detected photon's
 * azimuth (its radius drawn from the network) is accepted with probability
 * prod over the detector's four sides (1 - amplitude exp(-s / length_um)),
 * s its distance to the side, redrawn otherwise; amplitude 0 (the default)
 * = uniform over the directions that stay on the detector.  Fitted per model
 * from a Monte Carlo PRF image of its geometry (surrogate.fit_edge) and
 * saved with the network.  0 <= amplitude < 1, length_um > 0. */
FD2_API fd2_status fd2_sg_set_edge(fd2_sg *sg, float amplitude, float length_um);
FD2_API fd2_status fd2_sg_get_edge(const fd2_sg *sg, float *amplitude, float *length_um);

/* One forward and backward pass on the given batch (host arrays, b rows,
 * b <= batch): loss and the gradient of every parameter (same order as
 * fd2_sg_get_params).  For gradient checks. */
FD2_API fd2_status fd2_sg_loss_grad(fd2_sg *sg, const float *features, const int32_t *photons,
                                    const int32_t *detected, const uint32_t *radial, int32_t b, float *loss,
                                    float *grad);
/* Network outputs for n feature rows (host arrays): out [n][25]. */
FD2_API fd2_status fd2_sg_predict(fd2_sg *sg, const float *features, int64_t n, float *out);

/* Surrogate in the loop: one run of ctx's resident events (single geometry
 * or batched) in which in-hull events are handled by the surrogate and the
 * rest by the Monte Carlo; a fraction `audit_fraction` of the in-hull
 * events (chosen by a hash of the event index and the seed) is also
 * transported by the Monte Carlo to fill `stats`.  Tallies (PRF, detected
 * per primary, PHS, counters) accumulate in ctx as for fd2_run; counters
 * of surrogate photons count them generated and detected only. */
FD2_API fd2_status fd2_sg_run(fd2_sg *sg, fd2_ctx *ctx, double audit_fraction, fd2_sg_stats *stats);

#ifdef __cplusplus
}
#endif
#endif
