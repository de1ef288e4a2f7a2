/*
 * fd2_xray.h -- GPU x-ray front end: the energy-deposition events (EDEs)
 * that feed the optical transport, produced on the device.
 *
 * In hybridMANTIS the EDEs come from PENELOPE driven by penEasy: a photon
 * source (penEasy's SOURCE BOX ISOTROPIC GAUSS SPECTRUM,
 * main/sourceBoxIsotropicGaussSpectrum.f:25-178 sampling, :181-400 input),
 * the CsI slab of example/CsI.geo, and the EDE tally
 * (main/hybridMANTIS_tallyEnergyDepositionEvents.f:155-200), which records
 * every energy loss in the detector material as (x, y, z in cm, deposited
 * energy in eV minus the energy of the secondaries it created, history
 * number starting at 1).  PENELOPE's own sources are not in the reference
 * tree; its material data file is (example/CsI.mat), and this front end
 * reads it.
 *
 * Physics (FP64 throughout, one GPU thread per x-ray history):
 *   photons   total attenuation from the material file's Rayleigh, Compton
 *             and per-element, per-shell photoelectric cross sections
 *             (log-log interpolation; absorption edges kept exact);
 *             photoelectric absorption picks the element and the shell
 *             (K, L1-L3, M1-M5, or the outer shells) by their partial cross
 *             sections, the photoelectron leaves with E - U(shell) in a
 *             Sauter direction, and the vacancy relaxes through the file's
 *             transition table: fluorescence x-rays are transported,
 *             Auger electrons are transported, binding energy left in
 *             unfilled vacancies is deposited on the spot;
 *             Compton scattering follows Klein-Nishina on free electrons
 *             (no binding or Doppler broadening); Rayleigh scattering uses
 *             the Thomson distribution times a screened form factor whose
 *             radius reproduces the file's Rayleigh cross section;
 *   electrons continuous slowing down with the file's collision + radiative
 *             stopping power, in condensed steps that each lose a fixed
 *             fraction of the energy; each step deposits its loss at a
 *             random point along the step (one EDE) and is then deflected
 *             with the Goudsmit-Saunderson mean <1 - cos> = 1 -
 *             exp(-s / lambda1), lambda1 from the file's first transport
 *             cross section; an electron at or below
 *             max(eabs_electron_ev, electron_local_ev) deposits what it has
 *             left on the spot.
 * Particles that leave the slab take their energy with them; histories
 * whose source particle misses the slab leave no EDE.  Every history
 * conserves energy: its EDEs plus the energy that escaped equal its source
 * energy (fd2_xray_get_history_info).
 *
 * Output order is deterministic: EDEs in history order, within a history in
 * the order they were made; the random stream is Philox-4x32-10 keyed by the
 * seed, counter (draw block, history index, stream id).
 */
#ifndef FD2_XRAY_H
#define FD2_XRAY_H

#include "fd2.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fd2_xray_material fd2_xray_material;
typedef struct fd2_xray fd2_xray;

/* Read a material: a PENELOPE (2006) material data file such as
 * example/CsI.mat, or a table file written by fd2_xray_save_material. */
FD2_API fd2_status fd2_xray_load_material(const char *path, fd2_xray_material **out);
/* Write the tables this front end uses (text, the library's own format). */
FD2_API fd2_status fd2_xray_save_material(const fd2_xray_material *m, const char *path);
FD2_API void fd2_xray_free_material(fd2_xray_material *m);

#define FD2_XRAY_MAX_ELEMENTS 8
typedef struct fd2_xray_material_info {
    double density_g_cm3;
    double molar_mass_g_mol;           /* of one molecule (stoichiometric unit) */
    double molecules_per_cm3;
    int32_t n_elements;
    int32_t z[FD2_XRAY_MAX_ELEMENTS];
    double atoms_per_molecule[FD2_XRAY_MAX_ELEMENTS];
    double k_edge_ev[FD2_XRAY_MAX_ELEMENTS];
    double e_min_ev, e_max_ev;         /* photon table range */
    int32_t n_photon_nodes, n_transitions;
    double rayleigh_screening_cm;      /* form-factor radius fitted to the Rayleigh cross section */
} fd2_xray_material_info;
FD2_API fd2_status fd2_xray_material_get_info(const fd2_xray_material *m, fd2_xray_material_info *out);

/* Linear attenuation coefficients (1/cm) at n energies: out[4 i + k] with
 * k = 0 Rayleigh, 1 Compton, 2 photoelectric, 3 total. */
FD2_API fd2_status fd2_xray_attenuation(const fd2_xray_material *m, const double *e_ev, int64_t n, double *out);
/* Electron CSDA range (cm) and first transport mean free path (cm). */
FD2_API fd2_status fd2_xray_electron_tables(const fd2_xray_material *m, const double *e_ev, int64_t n,
                                            double *range_cm, double *lambda1_cm);

#define FD2_XRAY_PHOTON 2
#define FD2_XRAY_ELECTRON 1

/* penEasy's SOURCE BOX ISOTROPIC GAUSS SPECTRUM section, field for field
 * (sourceBoxIsotropicGaussSpectrum.f:254-400).  The spectrum is the section's
 * (energy, relative probability) lines: bin i covers [e_ev[i], e_ev[i+1])
 * with probability prob[i], sampled uniformly inside the bin; the last
 * line's probability is not used (the file marks it with -1).  Two lines
 * with prob[0] == 0 mean a Gaussian of mean (e0 + e1) / 2 and FWHM e1 - e0,
 * truncated to 6 sigma (:307-330).  Positions in cm. */
typedef struct fd2_xray_source {
    int32_t particle;               /* FD2_XRAY_PHOTON or FD2_XRAY_ELECTRON */
    int32_t n_spectrum;             /* lines, >= 2 */
    const double *e_ev;
    const double *prob;
    double center_cm[3];            /* box centre */
    double sides_cm[3];             /* box sides (all 0: point source) */
    double euler_deg[3];            /* box rotation [Rz, Ry, Rz] */
    double direction[3];            /* beam axis (need not be normalised) */
    double semiaperture_deg;        /* cone half-angle, [0, 180] */
} fd2_xray_source;

/* Read the SOURCE BOX ISOTROPIC GAUSS SPECTRUM section of a penEasy input
 * file (read in the order of sourceBoxIsotropicGaussSpectrum.f:218-400):
 * fills *src and copies the spectrum lines into e_ev / prob (cap lines at
 * most; src->e_ev / src->prob point at them).  FD2_ERR_PARSE if the section
 * is missing or OFF, or names a source material other than 0. */
FD2_API fd2_status fd2_xray_read_penEasy_source(const char *path, fd2_xray_source *src, double *e_ev, double *prob,
                                                int32_t cap);

typedef struct fd2_xray_options {
    int32_t device;
    double det_x_um, det_y_um;      /* slab: x in (0, det_x), y in (0, det_y) */
    double det_height_um;           /*       z in (-H/2, H/2) (um; EDEs in cm) */
    double eabs_electron_ev;        /* EABS(e-) of the penEasy input: 50 */
    double eabs_photon_ev;          /* EABS(ph): 50 */
    double electron_step_loss;      /* energy fraction lost per condensed step: 0.25 */
    double electron_local_ev;       /* an electron at or below this deposits all it has on the
                                       spot (range 0.04 um at 1 keV in CsI, far below a pixel):
                                       1000; eabs_electron_ev tracks every electron to the end */
    int32_t fluorescence;           /* 1: relax vacancies (x-rays, Auger); 0: deposit U on the spot */
    int32_t max_edes_per_history;   /* EDE slots per history (64..4096; 256); a history that
                                       needs more adds the rest to its last EDE and is counted */
    int64_t batch_histories;        /* histories per kernel batch (default 65536) */
    uint64_t seed;
} fd2_xray_options;

typedef struct fd2_xray_stats {
    int64_t histories;              /* run so far (since create or the last clear) */
    int64_t missed;                 /* source particle never reached the slab */
    int64_t edes;
    int64_t merged_histories;       /* ran out of EDE slots (rest added to the last EDE) */
    int64_t photoelectric, compton, rayleigh;
    int64_t fluorescence_emitted, fluorescence_escaped;
    int64_t auger_emitted;
    int64_t electron_steps;
    double e_source_ev, e_deposited_ev, e_escaped_photon_ev, e_escaped_electron_ev;
} fd2_xray_stats;

FD2_API void fd2_xray_default_options(fd2_xray_options *o);
FD2_API fd2_status fd2_xray_create(const fd2_xray_material *m, const fd2_xray_options *o, fd2_xray **out);
FD2_API void fd2_xray_destroy(fd2_xray *x);
FD2_API const char *fd2_xray_last_error(const fd2_xray *x);

/* Run histories [first_history, first_history + n) (0-based; EDEs carry
 * first_history + i + 1).  Replaces the EDEs of the previous run; statistics
 * accumulate.  Synchronous. */
FD2_API fd2_status fd2_xray_run(fd2_xray *x, const fd2_xray_source *src, int64_t first_history, int64_t n);
FD2_API fd2_status fd2_xray_num_edes(fd2_xray *x, int64_t *n);
/* Copy the last run's EDEs to host arrays of at least fd2_xray_num_edes. */
FD2_API fd2_status fd2_xray_get_edes(fd2_xray *x, double *x_cm, double *y_cm, double *z_cm, double *de_ev,
                                     int32_t *hist, int64_t cap);
/* Per history of the last run (arrays of n, any may be null): source energy,
 * energy that left the slab as photons / electrons, depth below the entrance
 * plane z = +H/2 of the first interaction (cm; -1 if none), EDE count. */
FD2_API fd2_status fd2_xray_get_history_info(fd2_xray *x, double *e_source_ev, double *e_escaped_photon_ev,
                                             double *e_escaped_electron_ev, double *first_depth_cm,
                                             int32_t *first_kind, int32_t *n_edes, int64_t n);
FD2_API fd2_status fd2_xray_get_stats(fd2_xray *x, fd2_xray_stats *out);
FD2_API fd2_status fd2_xray_clear_stats(fd2_xray *x);
/* GPU time of the last run (ms): transport kernel, compaction. */
FD2_API fd2_status fd2_xray_get_timing(fd2_xray *x, double *transport_ms, double *compact_ms);

/* Hand the last run's EDEs to an optical context on the device
 * (fd2_submit_events_device): no host copy of the events.  Both must be on
 * the same device. */
FD2_API fd2_status fd2_xray_submit(fd2_xray *x, fd2_ctx *optical);

/* Device pointers to the last run's EDE arrays (valid until the next run). */
FD2_API fd2_status fd2_xray_device_edes(fd2_xray *x, const double **x_cm, const double **y_cm, const double **z_cm,
                                        const double **de_ev, const int32_t **hist, int64_t *n);

/* Sampler check: n draws on the GPU of one of the front end's angular and
 * energy distributions at energy e_ev (out[i]):
 *   0 Klein-Nishina: scattered photon energy fraction E'/E
 *   1 Rayleigh: cos(theta)
 *   2 Sauter photoelectron: cos(theta) to the photon direction
 *   3 electron step deflection for a step of s = param cm: cos(theta)
 */
FD2_API fd2_status fd2_xray_sample(fd2_xray *x, int32_t which, double e_ev, double param, int64_t n, uint64_t seed,
                                   double *out);

#ifdef __cplusplus
}
#endif
#endif
