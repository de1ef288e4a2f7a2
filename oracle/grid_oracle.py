"""ctypes wrapper of the lattice walk's CPU oracle (grid_oracle.c).

TEST INFRASTRUCTURE ONLY: tests/ use it to check the GPU lattice walk
(fd2_options.column_grid = 1), which has no counterpart in the reference.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SO = os.path.join(HERE, "_build", "libfd2grid.so")
_lib = None


class GoGeom(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in ("xdet", "ydet", "H", "R", "pitch", "n_col", "n_gap", "top_absfrac",
                                               "mu", "beta", "sensor_refl", "lb_x", "lb_y", "ub_x", "ub_y")] + \
               [("pixel", ctypes.c_int32), ("xdim", ctypes.c_int32), ("ydim", ctypes.c_int32),
                ("lattice", ctypes.c_int32)]


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(SO):
            subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
        _lib = ctypes.CDLL(SO)
        vp = ctypes.c_void_p
        _lib.go_run.argtypes = [ctypes.POINTER(GoGeom), ctypes.c_int64, vp, vp, vp, vp, vp, ctypes.c_int32,
                                ctypes.c_uint64, vp, vp, vp]
        _lib.go_first_hit.argtypes = [ctypes.POINTER(GoGeom)] + [ctypes.c_double] * 5 + \
                                     [ctypes.POINTER(ctypes.c_double)] * 3
    return _lib


def geometry(p, gap_um: float, xdim: int, ydim: int, lattice: int = 1) -> GoGeom:
    """The lattice geometry of fd2 params `p` (hybridmantis_b200 Params);
    lattice 1 square, 2 hexagonal."""
    return GoGeom(xdet=p.det_x, ydet=p.det_y, H=p.det_height, R=p.radius, pitch=2 * p.radius + gap_um,
                  n_col=p.n_col, n_gap=p.n_gap, top_absfrac=p.top_absfrac, mu=p.bulk_abs, beta=p.beta,
                  sensor_refl=p.sensor_refl, lb_x=p.lb_x, lb_y=p.lb_y, ub_x=p.ub_x, ub_y=p.ub_y, pixel=p.pixel,
                  xdim=xdim, ydim=ydim, lattice=lattice)


def first_hit(g: GoGeom, px, py, dx, dy, tend):
    t, cx, cy = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    r = load().go_first_hit(ctypes.byref(g), px, py, dx, dy, tend, ctypes.byref(t), ctypes.byref(cx), ctypes.byref(cy))
    return (t.value, cx.value, cy.value) if r == 1 else None


def run(g: GoGeom, x_um, y_um, z_um, hist, nphot, num_hist: int, seed: int = 1):
    x, y, z = (np.ascontiguousarray(v, np.float64) for v in (x_um, y_um, z_um))
    h = np.ascontiguousarray(hist, np.int32)
    n = np.ascontiguousarray(nphot, np.int32)
    cnt = np.zeros(8, np.uint64)
    prf = np.zeros(g.xdim * g.ydim, np.uint64)
    prim = np.zeros(max(num_hist, 1), np.int32)
    p = lambda a: ctypes.c_void_p(a.ctypes.data)  # noqa: E731
    rc = load().go_run(ctypes.byref(g), len(x), p(x), p(y), p(z), p(h), p(n), num_hist, ctypes.c_uint64(seed), p(cnt),
                       p(prf), p(prim))
    assert rc == 0
    names = ["generated", "detected", "abs_top", "abs_bulk", "lost", "outofcol", "theta1", "capped"]
    return dict(zip(names, cnt.tolist())), prf.reshape(g.xdim, g.ydim), prim[:num_hist]
