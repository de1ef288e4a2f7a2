/*
 * compat_driver.c -- stands in for the Fortran program around the
 * gpuoptical_ / cpuoptical_ / gpuoptlb_ / cpuoptlb_ shims (tests only).
 *
 * It defines the COMMON blocks the way gfortran lays them out
 * (kernel_cuda_c_ver1_0.cu:84-236), fills /inputargs/ and /optical/ from a
 * seeded synthetic config-0 stream (positions in cm, energies in eV,
 * 1-based histories, as the EDE tally buffers them), makes the calls the
 * EDE tally makes (hybridMANTIS_tallyEnergyDepositionEvents.f:198-310) and
 * prints the COMMON-block results as one JSON line.
 *
 *   compat_driver gpu  N_XRAYS SEED   modes 99, 100 (first half), 101 (rest)
 *   compat_driver cpu  N_XRAYS SEED   cpuoptical_(0) over the whole buffer
 *   compat_driver lb   N_XRAYS SEED   gpuoptlb_ over the whole buffer
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "fd2_compat.h"

struct fd2_common_optical optical_;
struct fd2_common_inputargs inputargs_;
struct fd2_common_optstats optstats_;
struct fd2_common_outputdetprim outputdetprim_;
struct fd2_common_outputimage outputimage_;

int main(int argc, char **argv)
{
    if (argc != 4) {
        fprintf(stderr, "usage: compat_driver gpu|cpu|lb N_XRAYS SEED\n");
        return 2;
    }
    const char *mode = argv[1];
    fd2_events ev;
    if (fd2_synth_events(0, atoi(argv[2]), strtoull(argv[3], NULL, 0), &ev) != FD2_OK) return 3;
    if (ev.n > FD2_GPUBUFSIZE) return 4;
    const fd2_params *p = &ev.params;
    struct fd2_common_inputargs *a = &inputargs_;
    a->detx = p->det_x;
    a->dety = p->det_y;
    a->detheight = p->det_height;
    a->detradius = p->radius;
    a->detnC = p->n_col;
    a->detnIC = p->n_gap;
    a->dettop = p->top_absfrac;
    a->detbulk = p->bulk_abs;
    a->detbeta = p->beta;
    a->detdmin = p->d_min;
    a->detdmax = p->d_max;
    a->detlboundx = p->lb_x;
    a->detlboundy = p->lb_y;
    a->detuboundx = p->ub_x;
    a->detuboundy = p->ub_y;
    a->detyield = p->yield;
    a->detsensorRefl = p->sensor_refl;
    a->detpixel = p->pixel;
    a->rungpu = 1;
    a->machinenum = p->machine;
    a->mynumhist = p->num_hist;
    a->minphotons = p->min_photons;
    a->maxphotons = p->max_photons;
    a->mynumbins = p->num_bins;
    for (int64_t i = 0; i < ev.n; ++i) {
        optical_.xbufopt[i] = ev.x_um[i] / 1e4;
        optical_.ybufopt[i] = ev.y_um[i] / 1e4;
        optical_.zbufopt[i] = ev.z_um[i] / 1e4;
        optical_.debufopt[i] = ev.e_ev[i];
        optical_.nbufopt[i] = ev.hist[i];
    }
    optical_.myctropt = (int)ev.n;
    int n = (int)ev.n;
    double seconds = -1.0;
    if (!strcmp(mode, "gpu")) {
        int ctr = 99, half = n / 2, rest = n - half;
        gpuoptical_(&ctr, &half);
        if (fd2_compat_status() != FD2_OK) return 10;
        /* the second buffer starts at the beginning of /optical/, as the
         * EDE tally refills it after each call (the library has copied the
         * first buffer before gpuoptical_ returns) */
        ctr = 100;
        gpuoptical_(&ctr, &half);
        if (fd2_compat_status() != FD2_OK) return 11;
        ctr = 101;
        memmove(optical_.xbufopt, optical_.xbufopt + half, sizeof(double) * (size_t)rest);
        memmove(optical_.ybufopt, optical_.ybufopt + half, sizeof(double) * (size_t)rest);
        memmove(optical_.zbufopt, optical_.zbufopt + half, sizeof(double) * (size_t)rest);
        memmove(optical_.debufopt, optical_.debufopt + half, sizeof(double) * (size_t)rest);
        memmove(optical_.nbufopt, optical_.nbufopt + half, sizeof(int) * (size_t)rest);
        gpuoptical_(&ctr, &rest);
        if (fd2_compat_status() != FD2_OK) return 12;
    } else if (!strcmp(mode, "cpu")) {
        int zero = 0;
        cpuoptical_(&zero);
        if (fd2_compat_status() != FD2_OK) return 13;
    } else if (!strcmp(mode, "lb")) {
        gpuoptlb_(&seconds, &n);
        if (fd2_compat_status() != FD2_OK) return 14;
    } else {
        return 2;
    }
    unsigned long long img = 0, center = 0;
    for (int i = 0; i < 501; ++i)
        for (int j = 0; j < 501; ++j) {
            img += outputimage_.newimageopt[i][j];
            center = center * 1000003ull + outputimage_.newimageopt[i][j];
        }
    unsigned long long phs = 0, phs_hash = 0;
    for (int k = 0; k < 1000; ++k) {
        phs += outputdetprim_.gldetprimary[k];
        phs_hash = phs_hash * 31ull + (unsigned long long)outputdetprim_.gldetprimary[k];
    }
    printf("{\"events\": %d, \"glgen\": %.0f, \"gldetect\": %.0f, \"glabstop\": %.0f, \"glabsbulk\": %.0f, "
           "\"gllost\": %.0f, \"gloutofcol\": %.0f, \"gltheta1\": %.0f, \"glgputime\": %.6f, "
           "\"image_sum\": %llu, \"image_hash\": %llu, \"phs_sum\": %llu, \"phs_hash\": %llu, \"seconds\": %.6f}\n",
           n, optstats_.glgen, optstats_.gldetect, optstats_.glabstop, optstats_.glabsbulk, optstats_.gllost,
           optstats_.gloutofcol, optstats_.gltheta1, optstats_.glgputime, img, center, phs, phs_hash, seconds);
    fd2_free_events(&ev);
    return 0;
}
