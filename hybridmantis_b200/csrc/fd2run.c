/*
 * fd2run -- command-line driver: hybridMANTIS_input.in + an EDE stream in,
 * detected_*.dat and myimage_*.dat out (the files EDEreport writes,
 * main/hybridMANTIS_tallyEnergyDepositionEvents.f:336-502), plus the
 * optical transport statistics block it prints.
 *
 *   fd2run [--seed N] [--gaussian] [--autotune] [--device D] [--out DIR]
 *          hybridMANTIS_input.in events.{txt,bin}
 *   fd2run [options] --xray penEasy_input.in --material CsI.mat hybridMANTIS_input.in
 *
 * Text event files hold rows "x y z de hist" in cm / eV (the EDE tally's
 * event format); any other extension is read as fd2's binary format.  With
 * --xray the events come from the GPU x-ray front end (fd2_xray.h) instead:
 * the penEasy input's BIGS source section, the PENELOPE material file and
 * the detector of hybridMANTIS_input.in, num_hist histories -- the whole
 * hybridMANTIS run without PENELOPE.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "fd2.h"
#include "fd2_xray.h"

static int ends_with(const char *s, const char *suf)
{
    size_t n = strlen(s), m = strlen(suf);
    return n >= m && strcmp(s + n - m, suf) == 0;
}

int main(int argc, char **argv)
{
    fd2_options opt;
    fd2_default_options(&opt);
    const char *out = ".", *input = NULL, *events = NULL, *penEasy = NULL, *material = NULL;
    int tune = 0;
    for (int i = 1; i < argc; ++i) {
        if (!strcmp(argv[i], "--seed") && i + 1 < argc) opt.seed = strtoull(argv[++i], NULL, 0);
        else if (!strcmp(argv[i], "--xray") && i + 1 < argc) penEasy = argv[++i];
        else if (!strcmp(argv[i], "--material") && i + 1 < argc) material = argv[++i];
        else if (!strcmp(argv[i], "--gaussian")) opt.count_mode = FD2_COUNT_GAUSSIAN;
        else if (!strcmp(argv[i], "--autotune")) tune = 1;
        else if (!strcmp(argv[i], "--device") && i + 1 < argc) opt.device = atoi(argv[++i]);
        else if (!strcmp(argv[i], "--out") && i + 1 < argc) out = argv[++i];
        else if (!input) input = argv[i];
        else if (!events) events = argv[i];
        else {
            fprintf(stderr, "unexpected argument %s\n", argv[i]);
            return 2;
        }
    }
    if (!input || (!events && !(penEasy && material)) || (events && penEasy)) {
        fprintf(stderr, "usage: fd2run [--seed N] [--gaussian] [--autotune] [--device D] [--out DIR] input.in events\n"
                        "       fd2run [options] --xray penEasy_input.in --material file.mat input.in\n");
        return 2;
    }
    fd2_params p;
    fd2_status s = fd2_parse_input_file(input, &p);
    if (s != FD2_OK) {
        fprintf(stderr, "fd2run: %s: %s\n", input, fd2_status_string(s));
        return 1;
    }
    fd2_events ev;
    memset(&ev, 0, sizeof ev);
    fd2_xray_material *mat = NULL;
    fd2_xray *xr = NULL;
    static double spec_e[100000], spec_p[100000];
    if (events) {
        s = (ends_with(events, ".txt") || ends_with(events, ".dat")) ? fd2_read_events_text(events, &ev)
                                                                      : fd2_read_events_binary(events, &ev);
        if (s != FD2_OK) {
            fprintf(stderr, "fd2run: %s: %s\n", events, fd2_status_string(s));
            return 1;
        }
    } else {
        fd2_xray_source src;
        fd2_xray_options xo;
        fd2_xray_default_options(&xo);
        xo.device = opt.device;
        xo.seed = opt.seed;
        xo.det_x_um = p.det_x;
        xo.det_y_um = p.det_y;
        xo.det_height_um = p.det_height;
        s = fd2_xray_read_penEasy_source(penEasy, &src, spec_e, spec_p, 100000);
        if (s != FD2_OK) {
            fprintf(stderr, "fd2run: %s: %s (no usable BIGS source section)\n", penEasy, fd2_status_string(s));
            return 1;
        }
        s = fd2_xray_load_material(material, &mat);
        if (s == FD2_OK) s = fd2_xray_create(mat, &xo, &xr);
        if (s == FD2_OK) s = fd2_xray_run(xr, &src, 0, p.num_hist);
        if (s == FD2_OK) {
            int64_t n = 0;
            fd2_xray_num_edes(xr, &n);
            ev.n = n;
        }
        if (s != FD2_OK) {
            fprintf(stderr, "fd2run: x-ray front end: %s (%s)\n", fd2_status_string(s), xr ? fd2_xray_last_error(xr) : "");
            fd2_xray_destroy(xr);
            fd2_xray_free_material(mat);
            return 1;
        }
    }
    fd2_ctx *ctx = NULL;
    s = fd2_create(&p, &opt, &ctx);
    if (s == FD2_OK)
        s = xr ? fd2_xray_submit(xr, ctx)
               : fd2_submit_events_um(ctx, ev.x_um, ev.y_um, ev.z_um, ev.e_ev, ev.hist, NULL, NULL, ev.n);
    if (s == FD2_OK && tune) s = fd2_autotune(ctx, 0);
    if (s == FD2_OK) s = fd2_run(ctx);
    if (s == FD2_OK) s = fd2_wait(ctx);
    fd2_counters k;
    fd2_phs_stats ps;
    fd2_timing t;
    if (s == FD2_OK) s = fd2_get_counters(ctx, 0, &k);
    if (s == FD2_OK) s = fd2_get_phs_stats(ctx, 0, &ps);
    if (s == FD2_OK) s = fd2_get_timing(ctx, &t);
    if (s == FD2_OK) s = fd2_write_outputs(ctx, out);
    if (s != FD2_OK) {
        fprintf(stderr, "fd2run: %s (%s)\n", fd2_status_string(s), ctx ? fd2_last_error(ctx) : "");
        fd2_destroy(ctx);
        if (!xr) fd2_free_events(&ev);
        fd2_xray_destroy(xr);
        fd2_xray_free_material(mat);
        return 1;
    }
    printf(">>>>>>>>> EDEreport >>>>>>>>>\n");
    printf("    Number of energy deposition events: %lld\n", (long long)ev.n);
    if (xr) {
        fd2_xray_stats xs;
        fd2_xray_get_stats(xr, &xs);
        printf("    Depositions per primary = %12.5E\n", (double)xs.edes / (double)(p.num_hist > 0 ? p.num_hist : 1));
        printf("    x-ray front end: photoelectric %lld, Compton %lld, Rayleigh %lld, fluorescence %lld (%lld escaped)\n",
               (long long)xs.photoelectric, (long long)xs.compton, (long long)xs.rayleigh,
               (long long)xs.fluorescence_emitted, (long long)xs.fluorescence_escaped);
    }
    printf("\n    OPTICAL TRANSPORT STATISTICS\n\n");
    printf("Generated\n %12.2f\nDetected\n %12.2f\nAbsorbed at top\n %12.2f\n", (double)k.generated, (double)k.detected,
           (double)k.abs_top);
    printf("Absorbed in bulk\n %12.2f\nLost\n %12.2f\nOut of Column\n %12.2f\n", (double)k.abs_bulk, (double)k.lost,
           (double)k.outofcol);
    printf("Theta1 kills\n %12.2f\nCapped\n %12.2f\n", (double)k.theta1, (double)k.capped);
    printf("PHS mean (detected / history with >= 1)\n %12.4f\nSwank factor\n %12.6f\n", ps.mean, ps.swank);
    printf("Transport time (ms)\n %12.3f\nPhotons / s\n %12.4e\n", t.transport_ms,
           t.transport_ms > 0 ? (double)t.photons / (t.transport_ms * 1e-3) : 0.0);
    fd2_destroy(ctx);
    if (!xr) fd2_free_events(&ev);
    fd2_xray_destroy(xr);
    fd2_xray_free_material(mat);
    return 0;
}
