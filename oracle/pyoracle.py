"""ctypes bindings for the CPU oracle and the reference harness.

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke`` and
bench.py's CPU-baseline leg.  The product package never imports this.

``run_oracle`` calls the C restatement (oracle/fd2_oracle.c); ``run_ref``
calls the reference's own C transport compiled in place (oracle/_ref, built
by oracle/Makefile from main/kernel_cuda_c_ver1_0.cu); ``run_ref_cuda``
launches the reference's own CUDA kernel from the same file, compiled for
sm_100a (the GPU baseline; needs a GPU).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libfd2oracle.so")
REF_SO = {"O0": os.path.join(HERE, "_ref", "libfd2ref_O0.so"),
          "O2": os.path.join(HERE, "_ref", "libfd2ref_O2.so")}
REF_CUDA_SO = os.path.join(HERE, "_ref", "libfd2refcuda.so")
SYNTH_SO = os.path.join(HERE, "_build", "libfd2synth.so")

FATE_NAMES = {0: "none", 1: "detect", 2: "abs_top", 3: "abs_bulk", 4: "lost",
              5: "outofcol", 6: "theta1"}
COUNTER_NAMES = ["generated", "detect", "abs_top", "abs_bulk", "lost", "outofcol", "theta1"]


def build() -> None:
    """Build the oracle (and the reference harness when the sources exist)."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)


_libs: dict = {}


def _load(path: str):
    if path not in _libs:
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle`")
        _libs[path] = ctypes.CDLL(path)
    return _libs[path]


def ref_available(opt: str = "O2") -> bool:
    return os.path.exists(REF_SO[opt])


@dataclass
class Geometry:
    """Detector parameters in the reference's units (micrometres)."""
    xdet: float = 501.0
    ydet: float = 501.0
    H: float = 150.0
    R: float = 5.0
    n_col: float = 1.8
    n_gap: float = 1.0
    top_absfrac: float = 0.1
    bulk_abs: float = 1e-4
    beta: float = 0.2
    d_min: float = 0.5
    d_max: float = 280.0
    lb_x: float = 0.0
    lb_y: float = 0.0
    ub_x: float = 501.0
    ub_y: float = 501.0
    sensor_refl: float = 0.0
    pixel: int = 1

    def floats(self):
        return [self.xdet, self.ydet, self.H, self.R, self.n_col, self.n_gap,
                self.top_absfrac, self.bulk_abs, self.beta, self.d_min, self.d_max,
                self.lb_x, self.lb_y, self.ub_x, self.ub_y, self.sensor_refl]

    @property
    def xdim(self) -> int:
        return int(np.ceil(np.float32((np.float32(self.ub_x) - np.float32(self.lb_x)) / np.float32(self.pixel))))

    @property
    def ydim(self) -> int:
        return int(np.ceil(np.float32((np.float32(self.ub_y) - np.float32(self.lb_y)) / np.float32(self.pixel))))


class _OGeom(ctypes.Structure):
    _fields_ = [(n, ctypes.c_float) for n in
                ["xdet", "ydet", "H", "R", "n_col", "n_gap", "top_absfrac", "bulk_abs", "beta",
                 "d_min", "d_max", "lb_x", "lb_y", "ub_x", "ub_y", "sensor_refl"]] + \
              [("pixel", ctypes.c_int)]


class _RGeom(ctypes.Structure):
    _fields_ = [("v", ctypes.c_float * 16), ("pixel", ctypes.c_int)]


def _ptr(a, ct):
    return a.ctypes.data_as(ctypes.POINTER(ct)) if a is not None else None


@dataclass
class RunResult:
    image: np.ndarray
    per_primary: np.ndarray
    counters: np.ndarray
    fate: np.ndarray | None = None
    pix: np.ndarray | None = None
    seeds: np.ndarray | None = None
    steps: np.ndarray | None = None
    status: int = 0
    extra: dict = field(default_factory=dict)


def _events(x, y, z, hist, nphot):
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    z = np.ascontiguousarray(z, dtype=np.float64)
    hist = np.ascontiguousarray(hist, dtype=np.int32)
    nphot = np.ascontiguousarray(nphot, dtype=np.int32)
    return x, y, z, hist, nphot


def run_oracle(g: Geometry, x, y, z, hist, nphot, seed_input=271828182, base=0,
               prim_size=None, records=True, xdim=None, ydim=None) -> RunResult:
    lib = _load(ORACLE_SO)
    x, y, z, hist, nphot = _events(x, y, z, hist, nphot)
    n = len(x)
    prim_size = int(hist.max()) if prim_size is None and n else (prim_size or 0)
    xdim = g.xdim if xdim is None else xdim
    ydim = g.ydim if ydim is None else ydim
    image = np.zeros(xdim * ydim, np.uint64)
    prim = np.zeros(max(prim_size, 1), np.int32)
    cnt = np.zeros(7, np.uint64)
    tot = int(nphot.sum())
    fate = np.zeros(tot, np.int8) if records else None
    pix = np.zeros(2 * tot, np.int32) if records else None
    seeds = np.zeros(2 * tot, np.int32) if records else None
    steps = np.zeros(tot, np.int32) if records else None
    og = _OGeom(*[ctypes.c_float(v) for v in g.floats()], ctypes.c_int(g.pixel))
    lib.fd2o_run.restype = ctypes.c_int
    rc = lib.fd2o_run(ctypes.byref(og), ctypes.c_int(n),
                      _ptr(x, ctypes.c_double), _ptr(y, ctypes.c_double), _ptr(z, ctypes.c_double),
                      _ptr(hist, ctypes.c_int32), _ptr(nphot, ctypes.c_int32),
                      ctypes.c_int32(seed_input), ctypes.c_int64(base), ctypes.c_int32(prim_size),
                      ctypes.c_int32(xdim), ctypes.c_int32(ydim),
                      _ptr(image, ctypes.c_uint64), _ptr(prim, ctypes.c_int32), _ptr(cnt, ctypes.c_uint64),
                      _ptr(fate, ctypes.c_int8), _ptr(pix, ctypes.c_int32), _ptr(seeds, ctypes.c_int32),
                      _ptr(steps, ctypes.c_int32))
    if rc != 0:
        raise ValueError(f"fd2o_run returned {rc}")
    return RunResult(image.reshape(xdim, ydim), prim[:prim_size], cnt, fate,
                     None if pix is None else pix.reshape(-1, 2),
                     None if seeds is None else seeds.reshape(-1, 2), steps)


def run_ref(g: Geometry, x, y, z, hist, nphot, seed_input=271828182, base=0,
            prim_size=None, records=True, opt="O2") -> RunResult:
    lib = _load(REF_SO[opt])
    x, y, z, hist, nphot = _events(x, y, z, hist, nphot)
    n = len(x)
    prim_size = int(hist.max()) if prim_size is None and n else (prim_size or 0)
    image = np.zeros(501 * 501, np.uint64)
    prim = np.zeros(max(prim_size, 1), np.int32)
    cnt = np.zeros(7, np.uint64)
    tot = int(nphot.sum())
    fate = np.zeros(tot, np.int8) if records else None
    seeds = np.zeros(2 * tot, np.int32) if records else None
    steps = np.zeros(tot, np.int32) if records else None
    rg = _RGeom((ctypes.c_float * 16)(*g.floats()), ctypes.c_int(g.pixel))
    lib.fd2ref_run.restype = ctypes.c_int
    rc = lib.fd2ref_run(ctypes.byref(rg), ctypes.c_int(n),
                        _ptr(x, ctypes.c_double), _ptr(y, ctypes.c_double), _ptr(z, ctypes.c_double),
                        _ptr(hist, ctypes.c_int32), _ptr(nphot, ctypes.c_int32),
                        ctypes.c_int(seed_input), ctypes.c_int(base), ctypes.c_int(prim_size),
                        _ptr(image, ctypes.c_uint64), _ptr(prim, ctypes.c_int32), _ptr(cnt, ctypes.c_uint64),
                        _ptr(fate, ctypes.c_int8), _ptr(seeds, ctypes.c_int32), _ptr(steps, ctypes.c_int32))
    if rc == -1:
        raise ValueError("fd2ref_run rejected its arguments")
    return RunResult(image.reshape(501, 501), prim[:prim_size], cnt, fate, None,
                     None if seeds is None else seeds.reshape(-1, 2), steps, status=rc)


def init_prng(index: int, seed_input: int = 271828182, per_thread: int = 50000, ref=False):
    seed = np.zeros(2, np.int32)
    if ref:
        _load(REF_SO["O2"]).fd2ref_init_prng(ctypes.c_int(index), ctypes.c_int(per_thread),
                                             ctypes.c_int(seed_input), _ptr(seed, ctypes.c_int32))
    else:
        _load(ORACLE_SO).fd2o_init_prng(ctypes.c_int64(index), ctypes.c_int32(per_thread),
                                        ctypes.c_int32(seed_input), _ptr(seed, ctypes.c_int32))
    return seed


def ranecu(seed, n: int, ref=False):
    seed = np.ascontiguousarray(seed, dtype=np.int32).copy()
    out = np.zeros(n, np.float32)
    if ref:
        _load(REF_SO["O2"]).fd2ref_ranecu(_ptr(seed, ctypes.c_int32), ctypes.c_int(n), _ptr(out, ctypes.c_float))
    else:
        _load(ORACLE_SO).fd2o_ranecu(_ptr(seed, ctypes.c_int32), ctypes.c_int32(n), _ptr(out, ctypes.c_float))
    return out, seed


CALL_NAMES = ["step", "to_wall", "pullback", "surface", "incidence", "fresnel", "reflect", "refract",
              "crosstalk", "hop", "new_normal", "rough", "uniform"]


def reset_call_counts():
    _load(ORACLE_SO).fd2o_reset_call_counts()


def call_counts() -> dict:
    out = np.zeros(len(CALL_NAMES), np.uint64)
    _load(ORACLE_SO).fd2o_get_call_counts(_ptr(out, ctypes.c_uint64))
    return dict(zip(CALL_NAMES, [int(v) for v in out]))


def phs(per_primary, min_photons, max_photons, num_bins):
    pp = np.ascontiguousarray(per_primary, dtype=np.int32)
    h = np.zeros(num_bins, np.int32)
    rc = _load(ORACLE_SO).fd2o_phs(_ptr(pp, ctypes.c_int32), ctypes.c_int32(len(pp)),
                                   ctypes.c_int32(min_photons), ctypes.c_int32(max_photons),
                                   ctypes.c_int32(num_bins), _ptr(h, ctypes.c_int32))
    if rc != 0:
        raise ValueError("PHS bin width is zero")
    return h


def ref_cuda_available() -> bool:
    return os.path.exists(REF_CUDA_SO)


def run_ref_cuda(g: Geometry, x, y, z, hist, nphot, num_hist: int, grid: int = 18000,
                 device: int = 0) -> RunResult:
    """Launch the reference's CUDA kernel once over the events (inputs in um).

    ``grid`` = 18000 is the reference's fixed launch (cuda:82); 0 = just enough
    blocks of 128 threads.  ``extra["kernel_ms"]`` is the CUDA-event time of
    the launch.  Counters: generated, detect, abs_top, abs_bulk, lost,
    outofcol, theta1.
    """
    lib = _load(REF_CUDA_SO)
    x, y, z, hist, nphot = _events(x, y, z, hist, nphot)
    n = len(x)
    xdim, ydim = g.xdim, g.ydim
    image = np.zeros(xdim * ydim, np.uint64)
    prim = np.zeros(num_hist, np.int32)
    cnt = np.zeros(7, np.uint64)
    ms = ctypes.c_float(0.0)
    err = ctypes.c_int(0)
    rg = _RGeom((ctypes.c_float * 16)(*g.floats()), ctypes.c_int(g.pixel))
    lib.fd2refcu_run.restype = ctypes.c_int
    rc = lib.fd2refcu_run(ctypes.c_int(device), ctypes.byref(rg), ctypes.c_int64(n),
                          _ptr(x, ctypes.c_double), _ptr(y, ctypes.c_double), _ptr(z, ctypes.c_double),
                          _ptr(hist, ctypes.c_int32), _ptr(nphot, ctypes.c_int32), ctypes.c_int(num_hist),
                          ctypes.c_int(grid), ctypes.c_int(xdim), ctypes.c_int(ydim),
                          _ptr(image, ctypes.c_uint64), _ptr(prim, ctypes.c_int32), _ptr(cnt, ctypes.c_uint64),
                          ctypes.byref(ms), ctypes.byref(err))
    if rc != 0:
        raise RuntimeError(f"fd2refcu_run returned {rc} (CUDA error {err.value})")
    return RunResult(image.reshape(xdim, ydim), prim, cnt, extra={"kernel_ms": float(ms.value)})


@dataclass
class HostEvents:
    """A synthetic EDE stream built on the host (micrometres, eV, 1-based
    histories) with the benchmark configuration's parameters."""
    x_um: np.ndarray
    y_um: np.ndarray
    z_um: np.ndarray
    e_ev: np.ndarray
    hist: np.ndarray
    params: object
    num_hist: int

    @property
    def n(self) -> int:
        return len(self.x_um)


def synth_events_host(config: int, num_xrays: int = 0, seed: int = 12345) -> HostEvents:
    """The seeded synthetic EDE stream of benchmark configuration ``config``
    from the host-only build of the product's generator (_build/libfd2synth.so):
    the same events as ``hybridmantis_b200.synth_events`` with the same
    arguments, without loading the product library (bench.py's reference arm
    runs in a process that maps no product code)."""
    from hybridmantis_b200._lib import Events  # ctypes layouts only; loads no library

    lib = _load(SYNTH_SO)
    ev = Events()
    lib.fd2_synth_events.restype = ctypes.c_int
    rc = lib.fd2_synth_events(ctypes.c_int32(config), ctypes.c_int32(num_xrays), ctypes.c_uint64(seed),
                              ctypes.byref(ev))
    if rc != 0:
        raise ValueError(f"fd2_synth_events returned {rc}")
    n = int(ev.n)

    def arr(p, dt):
        return np.ctypeslib.as_array(p, shape=(n,)).astype(dt, copy=True) if n and p else np.zeros(0, dt)

    out = HostEvents(arr(ev.x_um, np.float32), arr(ev.y_um, np.float32), arr(ev.z_um, np.float32),
                     arr(ev.e_ev, np.float32), arr(ev.hist, np.int32), type(ev.params).from_buffer_copy(ev.params),
                     int(ev.num_hist))
    lib.fd2_free_events(ctypes.byref(ev))
    return out
