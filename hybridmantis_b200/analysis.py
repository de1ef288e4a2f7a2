"""Image-quality metrics of the transport's outputs (include/fd2_analysis.h).

MTF from a point response image, NNPS from flat-field images, DQE from both,
computed by libfd2.so on the GPU.  The reference only plots its PRF output
(myimage_*.dat; GNUPLOT_scripts/PRF.gnu); `read_prf_file` reads that file so
the metrics apply to the reference's own results as well.

    python -m hybridmantis_b200.analysis myimage_<tags>.dat [--pixel 1] [--n-freq 64]
"""
from __future__ import annotations

import argparse
import ctypes

import numpy as np

from . import _lib
from ._lib import check, ptr


def _img(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def mtf(image, pixel_um: float, n_freq: int | None = None, device: int = 0) -> dict:
    """MTF of a point response image ([x][y], the fd2_get_prf layout)."""
    img = _img(image)
    X, Y = img.shape
    N = max(X, Y)
    K = N // 2 + 1 if n_freq is None else int(n_freq)
    out = {k: np.zeros(K) for k in ("freq", "mtf_x", "mtf_y", "mtf_r")}
    st = _lib.load().fd2_mtf(device, ptr(img), X, Y, float(pixel_um), K, ptr(out["freq"]), ptr(out["mtf_x"]),
                             ptr(out["mtf_y"]), ptr(out["mtf_r"]))
    check(st, "mtf")
    return out


def nnps(images, pixel_um: float, roi: int, x0: int | None = None, y0: int | None = None, rois_x: int = 1,
         rois_y: int = 1, n_freq: int | None = None, device: int = 0) -> dict:
    """NNPS of flat-field images (one [x][y] image or a stack [n][x][y])."""
    imgs = _img(images)
    if imgs.ndim == 2:
        imgs = imgs[None]
    n, X, Y = imgs.shape
    if x0 is None:
        x0 = (X - rois_x * roi) // 2
    if y0 is None:
        y0 = (Y - rois_y * roi) // 2
    K = roi // 2 + 1 if n_freq is None else int(n_freq)
    freq, nr = np.zeros(K), np.zeros(K)
    n2 = np.zeros((roi, roi))
    m = ctypes.c_double()
    st = _lib.load().fd2_nnps(device, ptr(imgs), n, X, Y, float(pixel_um), int(roi), int(x0), int(y0), int(rois_x),
                              int(rois_y), K, ptr(freq), ptr(nr), ptr(n2), ctypes.byref(m))
    check(st, "nnps")
    return {"freq": freq, "nnps_r": nr, "nnps_2d": n2, "mean_signal": m.value}


def flat_field(es, width_um: float, pixel_um: int, seed: int):
    """A pencil-beam stream (each history's depositions around the detector's
    centre, as the synthetic configurations make them) turned into a flat
    field: every history's depositions shifted together to an entry point
    uniform over a width_um x width_um detector, whose PRF bounds and pixel
    are set to image all of it.  Returns (EventSet, x-rays per mm^2)."""
    from .fastdetect2 import EventSet, Params
    rng = np.random.default_rng(seed)
    nh = int(es.num_hist)
    sx = rng.uniform(0.0, width_um, nh) - es.params.det_x / 2.0
    sy = rng.uniform(0.0, width_um, nh) - es.params.det_y / 2.0
    h = es.hist.astype(np.int64) - 1
    p = Params.from_buffer_copy(es.params)
    p.det_x = p.det_y = p.ub_x = p.ub_y = float(width_um)
    p.lb_x = p.lb_y = 0.0
    p.pixel = int(pixel_um)
    out = EventSet((es.x_um + sx[h]).astype(np.float32), (es.y_um + sy[h]).astype(np.float32), es.z_um.copy(),
                   es.e_ev.copy(), es.hist.copy(), None, p, [], es.num_hist)
    return out, nh / (width_um * width_um * 1e-6)


def dqe(mtf_vals, nnps_vals, fluence_per_mm2: float):
    """DQE(f) = MTF(f)^2 / (q NNPS(f)), q in x-rays per mm^2."""
    return np.asarray(mtf_vals) ** 2 / (float(fluence_per_mm2) * np.asarray(nnps_vals))


def read_prf_file(path: str) -> np.ndarray:
    """A myimage_*.dat file (one value per line, a blank line after each
    block of one y pixel index) as an [x][y] array."""
    blocks, cur = [], []
    with open(path) as f:
        for line in f:
            t = line.strip()
            if not t:
                if cur:
                    blocks.append(cur)
                    cur = []
                continue
            cur.append(float(t))
    if cur:
        blocks.append(cur)
    return np.array(blocks, dtype=np.float64).T


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("prf_file")
    ap.add_argument("--pixel", type=float, default=1.0, help="pixel pitch (um)")
    ap.add_argument("--n-freq", type=int, default=64)
    a = ap.parse_args(argv)
    r = mtf(read_prf_file(a.prf_file), a.pixel, a.n_freq)
    print("# f (cycles/mm)   MTF_x   MTF_y   MTF_radial")
    for k in range(a.n_freq):
        print(f"{r['freq'][k]:12.4f} {r['mtf_x'][k]:9.6f} {r['mtf_y'][k]:9.6f} {r['mtf_r'][k]:9.6f}")


if __name__ == "__main__":
    main()
