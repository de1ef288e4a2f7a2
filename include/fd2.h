/*
 * fd2.h -- C ABI of fd2-b200, a B200-native fastDETECT2 (optical-photon
 * transport in columnar CsI, the hot path of hybridMANTIS).
 *
 * Plain C types only: host pointers, sizes and opaque handles.  Every call
 * returns an fd2_status and never exits the process.  One context per host
 * thread; a context owns its device memory, its CUDA stream and its tallies.
 *
 * Reference interfaces replaced (paths inside the hybridMANTIS tree):
 *   fd2_parse_input_file   main/hybridMANTIS_penEasy.f:190-229 (the 24-value
 *                          hybridMANTIS_input.in reader) and :290-299 (tags)
 *   fd2_submit_events      main/hybridMANTIS_cuda_ver1_0.cu:250-268 (copy of
 *                          the EDE buffer, cm -> um, Poisson photon counts)
 *   fd2_run / fd2_wait     main/hybridMANTIS_cuda_ver1_0.cu:229-279 (mode 100:
 *                          async H2D + algo<<<18000,128>>>) and :287-358
 *                          (mode 101: last launch + D2H)
 *   fd2_get_prf            main/hybridMANTIS_cuda_ver1_0.cu:352,371-374
 *   fd2_get_phs            main/hybridMANTIS_cuda_ver1_0.cu:376-399
 *   fd2_get_counters       main/hybridMANTIS_cuda_ver1_0.cu:362-368,402-430
 *   fd2_write_outputs      main/hybridMANTIS_tallyEnergyDepositionEvents.f:
 *                          418-458 (myimage_*.dat / detected_*.dat)
 *   fd2_replay             main/hybridMANTIS_c_ver1_0.c:81-375 (cpuoptical_,
 *                          the CPU path whose RANECU sequence it replays)
 * The Fortran-callable shims gpuoptical_ / cpuoptical_ are in fd2_compat.h.
 */
#ifndef FD2_H
#define FD2_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define FD2_API __attribute__((visibility("default")))
#else
#define FD2_API
#endif

typedef enum fd2_status {
    FD2_OK = 0,
    FD2_ERR_INVALID_ARGUMENT = 1,
    FD2_ERR_IO = 2,
    FD2_ERR_PARSE = 3,
    FD2_ERR_CUDA = 4,
    FD2_ERR_OUT_OF_MEMORY = 5,
    FD2_ERR_TOO_MANY_PHOTONS = 6, /* an event exceeds max_photons_per_event */
    FD2_ERR_STATE = 7,            /* call out of order (e.g. run before submit) */
    FD2_ERR_TIMEOUT = 8,          /* fd2_wait deadline expired; run aborted */
    FD2_ERR_DEVICE_ABORT = 9,     /* the device raised its abort flag */
    FD2_ERR_NO_DEVICE = 10,
    FD2_ERR_FILE_EXISTS = 11,     /* output file exists (reference opens NEW) */
    FD2_ERR_BAD_EVENT = 12        /* NaN/negative energy, hist out of range */
} fd2_status;

/* hybridMANTIS_input.in: the 24 values in file order
 * (hybridMANTIS_penEasy.f:206-229).  Lengths in micrometres. */
typedef struct fd2_params {
    int32_t num_hist;     /*  1 x-ray histories (normalises the PRF)        */
    int32_t min_photons;  /*  2 PHS lower bound                             */
    int32_t max_photons;  /*  3 PHS upper bound                             */
    int32_t num_bins;     /*  4 PHS bins (the reference allows <= 1000)     */
    double det_x;         /*  5 detector size in x, x in (0, det_x)         */
    double det_y;         /*  6 detector size in y                          */
    double det_height;    /*  7 thickness H, z in (-H/2, H/2)               */
    double radius;        /*  8 column radius R                             */
    double n_col;         /*  9 refractive index of the columns             */
    double n_gap;         /* 10 refractive index between columns            */
    double top_absfrac;   /* 11 top-surface absorption fraction             */
    double bulk_abs;      /* 12 bulk absorption coefficient (1/um)          */
    double beta;          /* 13 wall roughness                              */
    double d_min;         /* 14 min distance to the next column             */
    double d_max;         /* 15 max distance to the next column             */
    double lb_x, lb_y;    /* 16,17 PRF lower bounds                         */
    double ub_x, ub_y;    /* 18,19 PRF upper bounds                         */
    double yield;         /* 20 light yield (photons / eV)                  */
    int32_t pixel;        /* 21 PRF pixel pitch (um, integer)               */
    double sensor_refl;   /* 22 sensor reflectivity (fraction)              */
    int32_t run_gpu;      /* 23 kept for file compatibility (always GPU)    */
    int32_t machine;      /* 24 machine number (output file tag)            */
    /* Raw strings (first 10 characters) of values 7, 8, 11, 12, 13, 15, 22,
     * 20, 21, 24, joined with '_' into the output file names exactly as
     * hybridMANTIS_penEasy.f:290-299 and the EDE tally do.  Empty strings
     * are filled from the numbers by fd2_params_fill_tags. */
    char tag[10][11];
} fd2_params;

/* One detector geometry of a batched run (fd2_set_geometries). */
typedef struct fd2_geometry {
    double det_x, det_y, det_height, radius, n_col, n_gap;
    double top_absfrac, bulk_abs, beta, d_min, d_max;
    double lb_x, lb_y, ub_x, ub_y, sensor_refl;
    int32_t pixel;
    int32_t reserved;
} fd2_geometry;

enum {
    FD2_COUNT_POISSON = 0,  /* N ~ Poisson(E * yield), the reference's rule  */
    FD2_COUNT_GAUSSIAN = 1, /* N = max(0, round(mu + sqrt(mu) z))            */
    FD2_COUNT_GIVEN = 2     /* counts supplied with the events               */
};

enum {
    FD2_REPLAY_REF = 0, /* float storage, double libm intermediates (as the reference C) */
    FD2_REPLAY_FP64 = 1 /* every quantity in double precision                            */
};

typedef struct fd2_options {
    int32_t device;                /* CUDA device ordinal                        */
    int32_t count_mode;            /* FD2_COUNT_*                                */
    uint64_t seed;                 /* production RNG key (Philox-4x32-10)        */
    int64_t max_photons_per_event; /* reference limit 900000                     */
    int32_t block_size;            /* transport CTA size; 0 = tuned default      */
    int32_t ctas_per_sm;           /* persistent grid = SMs * this; 0 = default  */
    int32_t chunk;                 /* photons per work-queue chunk; 0 = default  */
    int32_t refill;                /* idle lanes before a warp refills; 0 = def. */
    int32_t prf_window;            /* shared-memory PRF window edge; 0 = off, -1 = auto */
    int32_t use_graph;             /* replay the pipeline as one CUDA graph      */
    double wait_timeout_s;         /* fd2_wait deadline; <= 0 = none             */
    const char *tune_cache;        /* autotuner cache file (JSON), may be NULL   */
    int64_t event_base;            /* global index of the first submitted event: a
                                      shard of a larger stream draws the same
                                      random numbers as in the unsharded run     */
    int32_t fresnel_batch;         /* lanes parked at a column wall before the warp
                                      runs their Fresnel interaction (with a
                                      column lattice: lanes in the gap before the
                                      warp runs their gap segments); 0 = tuned    */
    int32_t radial_bins;           /* > 0: label mode -- each history's detected
                                      photons are binned by distance r from their
                                      event instead of the PRF image: bin j <
                                      radial_bins covers r_max (j/bins)^2 ..
                                      r_max ((j+1)/bins)^2, bin radial_bins is
                                      r >= r_max = radial_max_um (fd2_get_radial) */
    double radial_max_um;
    int32_t column_grid;           /* 0: the reference's column model (after each
                                      crossing the next column's orientation is
                                      drawn at random, hops U(d_min, d_max));
                                      1 / 2: an explicit square / hexagonal
                                      lattice of columns of pitch (nearest-
                                      neighbour distance) 2 radius +
                                      grid_gap_um, with
                                      Fresnel refraction at every wall and
                                      straight flights through the gap (no
                                      counterpart in the reference; single
                                      geometry, production transport only)  */
    double grid_gap_um;            /* lattice: gap between neighbouring columns */
    int32_t tally_mode;            /* 0 (default): each ended photon adds to the
                                      global tallies with one L2 reduction of its
                                      lane; 1 (single-geometry runs of the
                                      reference's column model): fates and
                                      per-history counts are aggregated across the
                                      warp (__match_any_sync) and privatised in
                                      shared memory, the PRF core in a
                                      shared-memory window (prf_window).  The
                                      tallies are identical; 0 is faster on a B200
                                      (the tally rate is far below the L2's atomic
                                      throughput, so aggregation only costs issue) */
} fd2_options;

typedef struct fd2_counters {
    uint64_t generated, detected, abs_top, abs_bulk, lost, outofcol, theta1, capped;
    uint64_t detected_in_prf; /* detections that landed inside the PRF image */
    double photon_distance;   /* total path length (um)                      */
} fd2_counters;

typedef struct fd2_phs_stats {
    double primaries;      /* histories with >= 1 detected photon (M0) */
    double sum, sum_sq;    /* M1, M2 over those histories (FP64)       */
    double mean;           /* M1 / M0                                  */
    double swank;          /* M1^2 / (M0 M2)                           */
    int64_t phs_dropped;   /* counts the reference would bin past the last bin */
} fd2_phs_stats;

typedef struct fd2_timing {
    float transport_ms; /* persistent transport kernel, last run        */
    float pipeline_ms;  /* count + queue + transport + PHS, last run     */
    int64_t photons;    /* photons transported in the last run          */
    int32_t grid, block, chunk, refill, prf_window, fresnel_batch;
} fd2_timing;

typedef struct fd2_ctx fd2_ctx;

FD2_API const char *fd2_status_string(fd2_status s);
FD2_API void fd2_default_options(fd2_options *opt);

/* Input file (hybridMANTIS_input.in).  '#' lines and blank lines are
 * skipped; the first blank-delimited token of each other line is a value. */
FD2_API fd2_status fd2_parse_input_file(const char *path, fd2_params *out);
FD2_API fd2_status fd2_params_fill_tags(fd2_params *p);
FD2_API fd2_status fd2_params_to_geometry(const fd2_params *p, fd2_geometry *g);
/* PRF image size used for tallies: ceil((ub - lb) / pixel) per axis. */
FD2_API fd2_status fd2_prf_dims(const fd2_geometry *g, int32_t *xdim, int32_t *ydim);

FD2_API fd2_status fd2_create(const fd2_params *p, const fd2_options *opt, fd2_ctx **out);
FD2_API void fd2_destroy(fd2_ctx *ctx);
FD2_API const char *fd2_last_error(const fd2_ctx *ctx);

/* Batched runs: geometry g of events tagged g (default one geometry from
 * the params).  At most 256 geometries. */
FD2_API fd2_status fd2_set_geometries(fd2_ctx *ctx, const fd2_geometry *g, int32_t n);

/* Events in the reference's units: x, y, z in cm, deposited energy in eV,
 * 1-based history number.  Photon counts are sampled on the GPU.  Replaces
 * the previous submission; the events stay resident for repeated runs. */
FD2_API fd2_status fd2_submit_events(fd2_ctx *ctx, const double *x_cm, const double *y_cm,
                                     const double *z_cm, const double *de_ev,
                                     const int32_t *hist, int64_t n);
/* Events in micrometres (float), optional per-event photon counts
 * (count_mode FD2_COUNT_GIVEN) and geometry ids (NULL = geometry 0). */
FD2_API fd2_status fd2_submit_events_um(fd2_ctx *ctx, const float *x_um, const float *y_um,
                                        const float *z_um, const float *e_ev,
                                        const int32_t *hist, const int32_t *nphot,
                                        const uint16_t *geom, int64_t n);
/* fd2_submit_events with the arrays in device memory of the context's
 * device (a GPU producer such as the x-ray front end, fd2_xray.h): the
 * events never pass through the host, and the transport is identical to a
 * host submission of the same arrays.  The arrays must be complete when
 * this is called (their producer synchronised); they are not kept. */
FD2_API fd2_status fd2_submit_events_device(fd2_ctx *ctx, const double *x_cm, const double *y_cm,
                                            const double *z_cm, const double *de_ev,
                                            const int32_t *hist, int64_t n);

/* Transport the resident events; tallies accumulate across runs.  Returns
 * once the work is queued on the context's stream. */
FD2_API fd2_status fd2_run(fd2_ctx *ctx);
/* Block until the queued work is done (deadline: options.wait_timeout_s). */
FD2_API fd2_status fd2_wait(fd2_ctx *ctx);
FD2_API fd2_status fd2_reset_tallies(fd2_ctx *ctx);

FD2_API fd2_status fd2_get_counters(fd2_ctx *ctx, int32_t geom, fd2_counters *out);
FD2_API fd2_status fd2_get_prf_dims(fd2_ctx *ctx, int32_t geom, int32_t *xdim, int32_t *ydim);
/* PRF counts, index ii * ydim + jj (ii = x pixel). */
FD2_API fd2_status fd2_get_prf(fd2_ctx *ctx, int32_t geom, uint64_t *image, int64_t n);
/* Detected photons per history, index hist - 1. */
FD2_API fd2_status fd2_get_detected_per_primary(fd2_ctx *ctx, int32_t *counts, int64_t n);
/* Label mode (options.radial_bins > 0): counts[h * (radial_bins + 1) + b]
 * for history h (0-based) and radial bin b (the last is the overflow);
 * n >= num_hist * (radial_bins + 1).  Surrogate training labels. */
FD2_API fd2_status fd2_get_radial(fd2_ctx *ctx, uint32_t *counts, int64_t n);
FD2_API fd2_status fd2_get_photon_counts(fd2_ctx *ctx, int32_t *nphot, int64_t n);
FD2_API fd2_status fd2_get_phs(fd2_ctx *ctx, int32_t geom, int32_t *bins, int32_t num_bins);
FD2_API fd2_status fd2_get_phs_stats(fd2_ctx *ctx, int32_t geom, fd2_phs_stats *out);
FD2_API fd2_status fd2_get_timing(fd2_ctx *ctx, fd2_timing *out);
/* The context's cudaStream_t (as void*), for event timing by the caller. */
FD2_API void *fd2_get_stream(fd2_ctx *ctx);

/* detected_<tags>.dat and myimage_<tags>.dat in dir, in the reference's
 * formats; fails with FD2_ERR_FILE_EXISTS if either file exists. */
FD2_API fd2_status fd2_write_outputs(fd2_ctx *ctx, const char *dir);

/* The same two files from host arrays (e.g. tallies merged across GPUs):
 * image is xdim*ydim counts [ii*ydim + jj], phs num_bins rows, PRF values
 * divided by num_hist.  suffix (may be NULL) is inserted before ".dat". */
FD2_API fd2_status fd2_write_output_files(const fd2_params *p, const fd2_geometry *g, const uint64_t *image,
                                          int32_t xdim, int32_t ydim, const int32_t *phs, int32_t num_bins,
                                          double num_hist, const char *dir, const char *suffix);

/* FP64/reference-arithmetic replay of the reference C path: RANECU stream
 * init_PRNG(event_index_base + e, 50000, seed_input) per event, photon counts
 * as submitted.  Per-photon records (NULL to skip) in event order:
 * fate (1 detect, 2 top, 3 bulk, 4 lost, 5 out-of-column, 6 theta1,
 * 7 capped), pix (ii, jj or -1), seeds (RANECU state after the photon's
 * last step), steps (step calls).  Tallies go to the context as usual. */
FD2_API fd2_status fd2_replay(fd2_ctx *ctx, int32_t mode, int32_t seed_input,
                              int64_t event_index_base, int8_t *fate, int32_t *pix,
                              int32_t *seeds, int32_t *steps);

/* Transport without allocating, for callers that cannot allocate device
 * memory (code running inside another framework's memory pool, or that may
 * not change the device's memory footprint).  No counterpart in the
 * reference.  All pointers are device pointers; events in micrometres with
 * 1-based histories (<= num_hist) and given photon counts; tallies are added
 * into prf (xdim*ydim u64, [ii*ydim + jj]), per_primary (num_hist int32,
 * index hist-1) and counters (9 u64: unused, detected, abs_top, abs_bulk,
 * lost, outofcol, theta1, capped, detected in the PRF).  At most 262144
 * events, 900000 photons per event and 2097152 work-queue chunks of 256
 * photons per call.  More events return FD2_ERR_INVALID_ARGUMENT at once;
 * more chunks return FD2_ERR_INVALID_ARGUMENT, an event above 900000
 * photons FD2_ERR_TOO_MANY_PHOTONS and an invalid event (non-finite
 * position, history outside 1..num_hist, negative count) FD2_ERR_BAD_EVENT
 * after the device has checked them; a call that fails in any of these
 * ways transports nothing and leaves prf, per_primary and counters as they
 * were.  The work queue lives in one
 * fixed ~24 MiB __device__ array that every GPU loading the library holds
 * until exit; the first call on a device looks up its address (make it
 * before any stream capture on that device).  Calls share that array:
 * calls that overlap on the GPU race, so serialise them.  Synchronises
 * `stream` (a cudaStream_t, NULL = legacy default stream) before returning.
 * Same random streams as fd2_run's first run with seed `seed`, so the
 * tallies equal the context API's for the same events. */
FD2_API fd2_status fd2_transport_noalloc(const fd2_geometry *geometry, const float *x_um, const float *y_um,
                                         const float *z_um, const int32_t *hist, const int32_t *nphot, int64_t n,
                                         int32_t num_hist, uint64_t seed, uint64_t *prf, int32_t *per_primary,
                                         uint64_t *counters, void *stream);

/* FP32 fused multiply-add throughput of `device`, the transport's roofline
 * denominator measured instead of derived: a kernel of independent FMA
 * chains over every SM, launched repeatedly for at least `min_seconds`
 * (CUDA events); *tflops is the best launch (2 flops per FMA), *seconds the
 * time spent (may be NULL).  No counterpart in the reference. */
FD2_API fd2_status fd2_measure_fp32_peak(int32_t device, double min_seconds, double *tflops, double *seconds);

/* Diagnostic (tests): the transport's column-wall root routine on the
 * current device for n quadratics a t^2 + b t + c = 0 (host arrays in and
 * out; the larger root, 999 where there is none).  Its FP64 fallback for a
 * nearly cancelling discriminant is the compensated quadratic of the walk
 * (dist_to_surface, main/kernel_cuda_c_ver1_0.cu:966-1186, has none).
 * Returns an fd2_status value. */
FD2_API int fd2_debug_wall_root(int32_t n, const float *qa, const float *qb, const float *qc, float *out);

/* Autotuner: times transport configurations on the resident events and
 * keeps the fastest (cached in options.tune_cache when set). */
FD2_API fd2_status fd2_autotune(fd2_ctx *ctx, int32_t budget_runs);

/* Synthetic energy-deposition streams standing in for PENELOPE, seeded:
 * config 0..4 of the benchmark suite (0 = 25 keV pencil beam on 150 um,
 * 1 = triangular 20-70 keV with clusters on 300 um, 2 = 64 geometries,
 * 4 = triangular on 500 um).  Outputs are allocated by the library and
 * released with fd2_free_events. */
typedef struct fd2_events {
    int64_t n;
    int32_t num_hist;
    float *x_um, *y_um, *z_um, *e_ev;
    int32_t *hist;
    uint16_t *geom;
    int32_t num_geom;
    fd2_geometry *geometries;
    fd2_params params;
} fd2_events;
FD2_API fd2_status fd2_synth_events(int32_t config, int32_t num_xrays, uint64_t seed,
                                    fd2_events *out);
FD2_API void fd2_free_events(fd2_events *ev);

/* EDE stream files: text rows "x y z de hist" (cm, eV, 1-based), the
 * format of the EDE tally's event write, or the binary form written by
 * fd2_write_events_binary. */
FD2_API fd2_status fd2_read_events_text(const char *path, fd2_events *out);
FD2_API fd2_status fd2_write_events_text(const char *path, const fd2_events *ev);
FD2_API fd2_status fd2_read_events_binary(const char *path, fd2_events *out);
FD2_API fd2_status fd2_write_events_binary(const char *path, const fd2_events *ev);

/* Streaming event ingest: the EDE tally's fill-and-flush loop
 * (main/hybridMANTIS_tallyEnergyDepositionEvents.f:171-310, one blocking
 * gpuoptical_ call per full buffer, main/hybridMANTIS_cuda_ver1_0.cu:107)
 * without the block.  Pushed events fill one of two pinned staging batches
 * of batch_events; a full batch is copied to the GPU on a copy stream and
 * transported while the caller fills the other one, and a push waits only
 * when both batches are still in flight.  Event indices run on across
 * batches and the whole stream shares one run counter, so the tallies equal
 * those of one fd2_submit_events (or _um) + fd2_run over the concatenated
 * stream, bit for bit, for every batch size.  The PHS is built once, at
 * fd2_ingest_end, from the per-history counts of the whole stream, so a
 * history split across batches is one PHS entry.  Single-geometry
 * contexts.  Between begin and end the context takes no submit, run,
 * reset, autotune or replay (FD2_ERR_STATE); getters see partial tallies.
 * Bad events and oversized photon counts are reported by fd2_ingest_end.
 * units: FD2_UNITS_CM (x, y, z in cm and deposited energy in eV as doubles,
 * the tally's buffer) or FD2_UNITS_UM (floats in um and eV). */
typedef struct fd2_ingest fd2_ingest;
enum { FD2_UNITS_CM = 0, FD2_UNITS_UM = 1 };
typedef struct fd2_ingest_stats {
    int64_t events;          /* events transported                         */
    int64_t batches;         /* batches launched                           */
    int64_t photons;         /* optical photons transported                */
    double host_seconds;     /* fd2_ingest_begin to the end of fd2_ingest_end */
    double push_wait_seconds;/* time pushes waited for a free staging batch */
    float device_ms;         /* first copy to the PHS pass, CUDA events    */
} fd2_ingest_stats;
FD2_API fd2_status fd2_ingest_begin(fd2_ctx *ctx, int64_t batch_events, int32_t units, fd2_ingest **out);
FD2_API fd2_status fd2_ingest_push(fd2_ingest *in, const double *x_cm, const double *y_cm, const double *z_cm,
                                   const double *de_ev, const int32_t *hist, int64_t n);
FD2_API fd2_status fd2_ingest_push_um(fd2_ingest *in, const float *x_um, const float *y_um, const float *z_um,
                                      const float *e_ev, const int32_t *hist, int64_t n);
/* Stream an EDE file through the ingest, reading it in batch-sized pieces:
 * text rows "x y z de hist" (cm, eV, 1-based; '#' lines skipped) into a
 * FD2_UNITS_CM ingest, or the binary form of fd2_write_events_binary
 * (without geometry ids) into a FD2_UNITS_UM ingest. */
FD2_API fd2_status fd2_ingest_file(fd2_ingest *in, const char *path);
/* Transport what is left, build the PHS, wait, report the stream's status;
 * releases `in` whatever the result.  stats may be NULL. */
FD2_API fd2_status fd2_ingest_end(fd2_ingest *in, fd2_ingest_stats *stats);

#ifdef __cplusplus
}
#endif
#endif
