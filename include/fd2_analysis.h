/*
 * fd2_analysis.h -- image-quality metrics of the transport's outputs, on the
 * GPU in FP64: the modulation transfer function (MTF) of a point response
 * (PRF) image, the normalised noise power spectrum (NNPS) of flat-field
 * images, and the detective quantum efficiency (DQE) that combines them.
 *
 * No counterpart in the reference: its PRF and PHS files
 * (myimage_*.dat / detected_*.dat, written by
 * main/hybridMANTIS_tallyEnergyDepositionEvents.f:418-458) are only plotted
 * (GNUPLOT_scripts/PRF.gnu, PHS.gnu).  These entry points consume exactly
 * those images: fd2_get_prf's counts, or the values of a myimage file.
 *
 * Images are [xdim][ydim] row-major with the x pixel index first (the PRF
 * layout of fd2_get_prf), pixel pitch `pixel_um` micrometres, host memory.
 * Frequencies are in cycles/mm.  All functions allocate device memory on
 * `device` for the call and free it before returning.
 */
#ifndef FD2_ANALYSIS_H
#define FD2_ANALYSIS_H

#include "fd2.h"

#ifdef __cplusplus
extern "C" {
#endif

/* MTF of a point response image I (no background), at f_k = k / (N pixel),
 * k = 0 .. n_freq-1, N = max(xdim, ydim):
 *   mtf_x(f) = |sum_i LSF_x[i] exp(-2 pi i f x_i)| / sum I,  LSF_x[i] = sum_j I[i][j]
 *   mtf_y(f)   likewise along y
 *   mtf_r(f_k) = mean of |H(u, v)| / sum I over the integer grid points
 *                (u, v), |u|, |v| < n_freq, with round(sqrt(u^2 + v^2)) = k,
 *                H(u, v) = sum_ij I[i][j] exp(-2 pi i (u i + v j) / N)
 * n_freq <= N/2 + 1.  Any output pointer may be NULL. */
FD2_API fd2_status fd2_mtf(int32_t device, const double *image, int32_t xdim, int32_t ydim, double pixel_um,
                           int32_t n_freq, double *freq_per_mm, double *mtf_x, double *mtf_y, double *mtf_r);

/* NNPS of n_images flat-field images over a grid of rois_x * rois_y
 * non-overlapping square regions of `roi` pixels whose first corner is
 * (x0, y0).  With n_images >= 2 the per-pixel mean over the images is
 * subtracted (and the power scaled by n/(n-1)); with one image each region's
 * mean.  For each image and region, F(u, v) = DFT of the difference over the
 * region, and
 *   NPS(u, v)  = pixel^2 / roi^2 * <|F(u, v)|^2>     (mm^2 x signal^2)
 *   NNPS(u, v) = NPS(u, v) / m^2,  m = mean signal over the regions
 * nnps_r[k] averages NNPS over (u, v) with round(|f| / df) = k, df = 1/(roi
 * pixel), signed frequencies; f_k = k df, k < n_freq <= roi/2 + 1.
 * nnps_2d (roi * roi values, u-major, unsigned DFT order) and mean_signal may
 * be NULL. */
FD2_API fd2_status fd2_nnps(int32_t device, const double *images, int32_t n_images, int32_t xdim, int32_t ydim,
                            double pixel_um, int32_t roi, int32_t x0, int32_t y0, int32_t rois_x, int32_t rois_y,
                            int32_t n_freq, double *freq_per_mm, double *nnps_r, double *nnps_2d,
                            double *mean_signal);

#ifdef __cplusplus
}
#endif
#endif
