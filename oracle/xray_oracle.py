"""ctypes wrapper of the x-ray front end's CPU oracle (xray_oracle.c).

TEST INFRASTRUCTURE ONLY: tests/ use it to check the GPU front end
(include/fd2_xray.h).  The source preparation below restates penEasy's BIGS
initialisation (main/sourceBoxIsotropicGaussSpectrum.f:263-400): the binned
spectrum normalised to a cumulative with per-bin slopes (:294-305), the
two-line Gaussian (:306-330, FWHM to sigma, 6 sigma cut), the Euler-angle box
rotation (:333-348) and the cone direction (:362-385).
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SO = os.path.join(HERE, "_build", "libfd2xray.so")
INFO_FIELDS = ["e0", "esc_ph", "esc_el", "first_depth", "n_edes", "first_kind", "merged", "missed", "n_pe", "n_co",
               "n_ra", "n_fe", "n_fesc", "n_aug", "n_steps"]
_lib = None
_loaded = None


class XoSource(ctypes.Structure):
    _fields_ = [("particle", ctypes.c_int), ("nspec", ctypes.c_int), ("gaussian", ctypes.c_int),
                ("point", ctypes.c_int), ("espc", ctypes.c_void_p), ("pcum", ctypes.c_void_p),
                ("despc", ctypes.c_void_p), ("gmean", ctypes.c_double), ("gsig", ctypes.c_double),
                ("gmin", ctypes.c_double), ("gmax", ctypes.c_double), ("ctr", ctypes.c_double * 3),
                ("side", ctypes.c_double * 3), ("rot", ctypes.c_double * 9), ("dir", ctypes.c_double * 3),
                ("cossrc", ctypes.c_double)]


class XoOpts(ctypes.Structure):
    _fields_ = [("X", ctypes.c_double), ("Y", ctypes.c_double), ("H2", ctypes.c_double),
                ("eabs_e", ctypes.c_double), ("eabs_ph", ctypes.c_double), ("loss", ctypes.c_double),
                ("local_e", ctypes.c_double), ("fluo", ctypes.c_int), ("cap", ctypes.c_int), ("seed", ctypes.c_uint64)]


def load(table: str):
    global _lib, _loaded
    if _lib is None:
        if not os.path.exists(SO):
            subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
        _lib = ctypes.CDLL(SO)
        vp = ctypes.c_void_p
        _lib.xo_load.argtypes = [ctypes.c_char_p]
        _lib.xo_run.argtypes = [ctypes.POINTER(XoOpts), ctypes.POINTER(XoSource), ctypes.c_int64, ctypes.c_int64,
                                vp, vp]
        _lib.xo_sample.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int64, ctypes.c_uint64,
                                   vp]
        _lib.xo_rayleigh_b.argtypes = [ctypes.c_double]
        _lib.xo_rayleigh_b.restype = ctypes.c_double
    if _loaded != table:
        r = _lib.xo_load(table.encode())
        if r != 0:
            raise RuntimeError(f"xo_load({table}) = {r}")
        _loaded = table
    return _lib


def prepare_source(src):
    """An XoSource from a hybridmantis_b200.xray.Source (BIGS initialisation)."""
    e = np.asarray(src.e_ev, np.float64)
    p = np.asarray(src.prob, np.float64)
    n = len(e)
    s = XoSource()
    s.particle = src.particle
    keep = []
    if p[:n - 1].sum() > 0:
        pc = np.zeros(n)
        for i in range(n - 1):
            pc[i + 1] = pc[i] + p[i]
        pc /= pc[n - 1]
        de = np.zeros(n)
        for i in range(n - 1):
            if pc[i + 1] > pc[i]:
                de[i] = (e[i + 1] - e[i]) / (pc[i + 1] - pc[i])
        keep = [np.ascontiguousarray(e), pc, de]
        s.nspec = n
        s.espc, s.pcum, s.despc = (a.ctypes.data for a in keep)
    else:
        s.gaussian = 1
        s.gmean = 0.5 * (e[0] + e[1])
        s.gsig = 0.42466090014400952 * (e[1] - e[0])
        s.gmin = max(0.0, s.gmean - 6 * s.gsig)
        s.gmax = s.gmean + 6 * s.gsig
    for a in range(3):
        s.ctr[a] = src.center_cm[a]
        s.side[a] = src.sides_cm[a]
    s.point = int(all(v == 0.0 for v in src.sides_cm))
    om, th, ph = (math.radians(v) for v in src.euler_deg)
    so, co, st, ct, sp, cp = math.sin(om), math.cos(om), math.sin(th), math.cos(th), math.sin(ph), math.cos(ph)
    rot = [cp * ct * co - sp * so, -cp * ct * so - sp * co, cp * st,
           sp * ct * co + cp * so, -sp * ct * so + cp * co, sp * st,
           -st * co, st * so, ct]
    for k in range(9):
        s.rot[k] = rot[k]
    nrm = math.sqrt(sum(v * v for v in src.direction))
    d = (0.0, 0.0, 1.0) if nrm < 1e-30 else tuple(v / nrm for v in src.direction)
    for a in range(3):
        s.dir[a] = d[a]
    s.cossrc = math.cos(math.radians(src.semiaperture_deg))
    return s, keep


def run(table: str, src, n: int, *, first: int = 0, det_x_um=909.0, det_y_um=909.0, det_height_um=150.0,
        eabs_e=50.0, eabs_ph=50.0, loss=0.25, local_e=1000.0, fluo=True, cap=256, seed=12345):
    """Histories first..first+n-1: (per-history dict, list of EDE arrays (k x 4: x, y, z cm, de eV))."""
    lib = load(table)
    s, keep = prepare_source(src)
    o = XoOpts(X=det_x_um * 1e-4, Y=det_y_um * 1e-4, H2=0.5 * det_height_um * 1e-4, eabs_e=eabs_e, eabs_ph=eabs_ph,
               loss=loss, local_e=local_e, fluo=int(fluo), cap=cap, seed=seed)
    info = np.zeros((n, 15))
    slots = np.zeros((n, cap, 4))
    lib.xo_run(ctypes.byref(o), ctypes.byref(s), int(first), int(n), info.ctypes.data, slots.ctypes.data)
    del keep
    h = {k: info[:, i] for i, k in enumerate(INFO_FIELDS)}
    counts = h["n_edes"].astype(int)
    edes = [slots[i, :counts[i]] for i in range(n)]
    return h, edes


def sample(table: str, which: int, e_ev: float, n: int, seed: int = 1, param: float = 0.0):
    lib = load(table)
    out = np.zeros(n)
    lib.xo_sample(int(which), float(e_ev), float(param), int(n), int(seed), out.ctypes.data)
    return out


def rayleigh_b(table: str, e_ev: float) -> float:
    return load(table).xo_rayleigh_b(float(e_ev))
