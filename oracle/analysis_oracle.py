"""CPU oracle of the image-quality metrics: MTF, NNPS, DQE.

TEST INFRASTRUCTURE ONLY (tests/ import it to check fd2_mtf and fd2_nnps).
The metrics have no counterpart in the reference (its myimage_*.dat point
response images, main/hybridMANTIS_tallyEnergyDepositionEvents.f:418-458,
are only plotted by GNUPLOT_scripts/PRF.gnu).  This restates, with numpy's
FFT in FP64, the definitions that include/fd2_analysis.h documents:

  MTF   mtf_x[k] = |DFT_N(LSF_x)[k]| / sum(I),  LSF_x[i] = sum_j I[i][j],
        N = max(xdim, ydim) (the image zero-padded to N), f_k = k / (N pixel);
        mtf_r[k] = mean |H(u, v)| / sum(I) over |u|, |v| < n_freq with
        round(sqrt(u^2 + v^2)) = k, H the N x N DFT of the padded image.
  NNPS  per image and region: D = image - mean image (n >= 2 images) or
        D = region - its mean (one image); F = DFT_roi(D);
        NNPS(u, v) = pixel_mm^2 / roi^2 * <|F|^2> * n/(n-1) / m^2,
        m = the mean image's mean over the regions; nnps_r radial average by
        round(|signed (u, v)|), f_k = k / (roi pixel).
  DQE   DQE(f) = MTF(f)^2 / (q NNPS(f)), q = x-rays per mm^2.
"""
from __future__ import annotations

import numpy as np


def mtf(image, pixel_um: float, n_freq: int):
    img = np.asarray(image, np.float64)
    X, Y = img.shape
    N = max(X, Y)
    S = img.sum()
    pad = np.zeros((N, N))
    pad[:X, :Y] = img
    lx = np.zeros(N)
    ly = np.zeros(N)
    lx[:X] = img.sum(axis=1)
    ly[:Y] = img.sum(axis=0)
    mtf_x = np.abs(np.fft.fft(lx))[:n_freq] / S
    mtf_y = np.abs(np.fft.fft(ly))[:n_freq] / S
    H = np.abs(np.fft.fft2(pad)) / S
    K = n_freq
    s = np.arange(-(K - 1), K)
    u, v = np.meshgrid(s, s, indexing="ij")
    b = np.rint(np.sqrt(u * u + v * v)).astype(int)
    vals = H[u % N, v % N]
    sums = np.bincount(b.ravel(), weights=vals.ravel(), minlength=2 * K)[:K]
    cnts = np.bincount(b.ravel(), minlength=2 * K)[:K]
    mtf_r = np.where(cnts > 0, sums / np.maximum(cnts, 1), 0.0)
    freq = 1000.0 * np.arange(K) / (N * pixel_um)
    return freq, mtf_x, mtf_y, mtf_r


def nnps(images, pixel_um: float, roi: int, x0: int, y0: int, rois_x: int, rois_y: int, n_freq: int):
    imgs = np.asarray(images, np.float64)
    if imgs.ndim == 2:
        imgs = imgs[None]
    n = imgs.shape[0]
    R = roi
    mean_img = imgs.mean(axis=0)
    regions = [(x0 + a * R, y0 + b * R) for a in range(rois_x) for b in range(rois_y)]
    m = np.mean([mean_img[rx:rx + R, ry:ry + R].mean() for rx, ry in regions])
    acc = np.zeros((R, R))
    for r in range(n):
        for rx, ry in regions:
            if n > 1:
                d = imgs[r, rx:rx + R, ry:ry + R] - mean_img[rx:rx + R, ry:ry + R]
            else:
                blk = imgs[r, rx:rx + R, ry:ry + R]
                d = blk - blk.mean()
            acc += np.abs(np.fft.fft2(d)) ** 2
    corr = n / (n - 1) if n > 1 else 1.0
    px = pixel_um / 1000.0
    nnps2d = acc * (px * px / (R * R)) * corr / (n * len(regions)) / (m * m)
    k = np.arange(R)
    s = np.where(k <= R // 2, k, k - R)
    u, v = np.meshgrid(s, s, indexing="ij")
    b = np.rint(np.sqrt(u * u + v * v)).astype(int)
    sums = np.bincount(b.ravel(), weights=nnps2d.ravel(), minlength=R)[:n_freq]
    cnts = np.bincount(b.ravel(), minlength=R)[:n_freq]
    nnps_r = np.where(cnts > 0, sums / np.maximum(cnts, 1), 0.0)
    freq = 1000.0 * np.arange(n_freq) / (R * pixel_um)
    return freq, nnps_r, nnps2d, m


def dqe(mtf_vals, nnps_vals, fluence_per_mm2: float):
    return np.asarray(mtf_vals) ** 2 / (fluence_per_mm2 * np.asarray(nnps_vals))
