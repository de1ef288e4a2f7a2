"""Python host layer over the fd2 C ABI.

Mirrors the reference's interface for the fastDETECT2 path: the 24-value
``hybridMANTIS_input.in`` (main/hybridMANTIS_penEasy.f:190-229), EDE buffers
in cm / eV / 1-based histories (main/hybridMANTIS_tallyEnergyDepositionEvents.f
:176-180), one transport per buffer (gpuoptical_ mode 100, main/
hybridMANTIS_cuda_ver1_0.cu:229-279), and the PRF / PHS / counter results
that EDEreport writes (tally.f:418-493).  All work runs in libfd2.so on the
GPU; this module only moves numpy arrays across the C boundary.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import (COUNT_GAUSSIAN, COUNT_GIVEN, COUNT_POISSON, REPLAY_FP64, REPLAY_REF, UNITS_CM, UNITS_UM,
                   Counters, Fd2Error, Geometry, IngestStats, Options, Params, PhsStats, Timing, check, load, ptr)

__all__ = ["read_input_file", "default_params", "params_to_geometry", "prf_dims", "EventSet", "synth_events",
           "OpticalTransport", "Fd2Error", "COUNT_POISSON", "COUNT_GAUSSIAN", "COUNT_GIVEN",
           "REPLAY_REF", "REPLAY_FP64", "UNITS_CM", "UNITS_UM", "Ingest", "write_output_files", "read_events_text", "write_events_text", "read_events_binary",
           "write_events_binary"]


def read_input_file(path: str) -> Params:
    p = Params()
    check(load().fd2_parse_input_file(str(path).encode(), ctypes.byref(p)), f"parse {path}")
    return p


def default_params(**kw) -> Params:
    """Parameters of the 25 keV / 150 um benchmark case, overridable by keyword."""
    p = Params()
    vals = dict(num_hist=1000, min_photons=0, max_photons=2000, num_bins=1000, det_x=501.0, det_y=501.0,
                det_height=150.0, radius=5.0, n_col=1.8, n_gap=1.0, top_absfrac=0.1, bulk_abs=1e-4, beta=0.2,
                d_min=0.5, d_max=280.0, lb_x=0.0, lb_y=0.0, ub_x=501.0, ub_y=501.0, yield_=0.054, pixel=1,
                sensor_refl=0.0, run_gpu=1, machine=1)
    vals.update(kw)
    for k, v in vals.items():
        setattr(p, k, v)
    load().fd2_params_fill_tags(ctypes.byref(p))
    return p


def params_to_geometry(p: Params) -> Geometry:
    g = Geometry()
    check(load().fd2_params_to_geometry(ctypes.byref(p), ctypes.byref(g)), "params_to_geometry")
    return g


def prf_dims(g: Geometry) -> tuple[int, int]:
    x, y = ctypes.c_int32(), ctypes.c_int32()
    check(load().fd2_prf_dims(ctypes.byref(g), ctypes.byref(x), ctypes.byref(y)), "prf_dims")
    return x.value, y.value


@dataclass
class EventSet:
    """Energy-deposition events in micrometres and eV."""
    x_um: np.ndarray
    y_um: np.ndarray
    z_um: np.ndarray
    e_ev: np.ndarray
    hist: np.ndarray
    geom: np.ndarray | None
    params: Params
    geometries: list
    num_hist: int

    @property
    def n(self) -> int:
        return len(self.x_um)

    def to_cm(self):
        return (self.x_um.astype(np.float64) / 1e4, self.y_um.astype(np.float64) / 1e4,
                self.z_um.astype(np.float64) / 1e4)

    def subset(self, idx) -> "EventSet":
        return EventSet(self.x_um[idx], self.y_um[idx], self.z_um[idx], self.e_ev[idx], self.hist[idx],
                        None if self.geom is None else self.geom[idx], self.params, self.geometries, self.num_hist)


def _events_from_struct(ev: _lib.Events) -> EventSet:
    n = ev.n

    def arr(p, dt):
        if n == 0 or not p:
            return np.zeros(0, dt)
        return np.ctypeslib.as_array(p, shape=(n,)).astype(dt, copy=True)

    geoms = [ev.geometries[i] for i in range(ev.num_geom)] if ev.geometries else []
    geoms = [Geometry.from_buffer_copy(g) for g in geoms]
    out = EventSet(arr(ev.x_um, np.float32), arr(ev.y_um, np.float32), arr(ev.z_um, np.float32),
                   arr(ev.e_ev, np.float32), arr(ev.hist, np.int32),
                   arr(ev.geom, np.uint16) if ev.geom else None, Params.from_buffer_copy(ev.params), geoms,
                   ev.num_hist)
    load().fd2_free_events(ctypes.byref(ev))
    return out


def synth_events(config: int, num_xrays: int = 0, seed: int = 12345) -> EventSet:
    """Seeded synthetic EDE stream of benchmark configuration ``config``."""
    ev = _lib.Events()
    check(load().fd2_synth_events(int(config), int(num_xrays), ctypes.c_uint64(seed), ctypes.byref(ev)), "synth_events")
    return _events_from_struct(ev)


def read_events_text(path: str) -> EventSet:
    ev = _lib.Events()
    check(load().fd2_read_events_text(str(path).encode(), ctypes.byref(ev)), f"read {path}")
    return _events_from_struct(ev)


def read_events_binary(path: str) -> EventSet:
    ev = _lib.Events()
    check(load().fd2_read_events_binary(str(path).encode(), ctypes.byref(ev)), f"read {path}")
    return _events_from_struct(ev)


def write_output_files(params: Params, geometry: Geometry, image, phs, num_hist: float, directory: str,
                       suffix: str = "") -> None:
    """detected_*.dat and myimage_*.dat from host arrays (reference formats)."""
    img = np.ascontiguousarray(image, dtype=np.uint64)
    ph = np.ascontiguousarray(phs, dtype=np.int32)
    check(load().fd2_write_output_files(ctypes.byref(params), ctypes.byref(geometry), ptr(img), img.shape[0],
                                        img.shape[1], ptr(ph), len(ph), float(num_hist), str(directory).encode(),
                                        suffix.encode()), "write_output_files")


def _as_struct(es: EventSet):
    keep = [np.ascontiguousarray(a) for a in (es.x_um, es.y_um, es.z_um, es.e_ev)]
    h = np.ascontiguousarray(es.hist, dtype=np.int32)
    ev = _lib.Events()
    ev.n = es.n
    ev.num_hist = es.num_hist
    ev.x_um, ev.y_um, ev.z_um, ev.e_ev = [a.ctypes.data_as(ctypes.POINTER(ctypes.c_float)) for a in keep]
    ev.hist = h.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
    g = None
    if es.geom is not None:
        g = np.ascontiguousarray(es.geom, dtype=np.uint16)
        ev.geom = g.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16))
    return ev, (keep, h, g)


def write_events_text(path: str, es: EventSet) -> None:
    ev, _keep = _as_struct(es)
    check(load().fd2_write_events_text(str(path).encode(), ctypes.byref(ev)), f"write {path}")


def write_events_binary(path: str, es: EventSet) -> None:
    ev, _keep = _as_struct(es)
    check(load().fd2_write_events_binary(str(path).encode(), ctypes.byref(ev)), f"write {path}")


class OpticalTransport:
    """One fd2 context: a GPU, a stream, resident events and tallies."""

    def __init__(self, params: Params, *, device: int = 0, count_mode: int = COUNT_POISSON, seed: int | None = None,
                 block_size: int = 0, ctas_per_sm: int = 0, chunk: int = 0, refill: int = 0, prf_window: int = -1,
                 use_graph: bool = True, wait_timeout_s: float = 0.0, max_photons_per_event: int = 900000,
                 tune_cache: str | None = None, event_base: int = 0, fresnel_batch: int = 0,
                 radial_bins: int = 0, radial_max_um: float = 200.0, column_grid: int = 0,
                 grid_gap_um: float = 0.5, tally_mode: int = 0):
        lib = load()
        self._lib = lib
        opt = Options()
        lib.fd2_default_options(ctypes.byref(opt))
        opt.device = device
        opt.count_mode = count_mode
        if seed is not None:
            opt.seed = seed
        opt.block_size, opt.ctas_per_sm, opt.chunk, opt.refill = block_size, ctas_per_sm, chunk, refill
        opt.prf_window = prf_window
        opt.use_graph = 1 if use_graph else 0
        opt.wait_timeout_s = wait_timeout_s
        opt.max_photons_per_event = max_photons_per_event
        opt.event_base = event_base
        opt.fresnel_batch = fresnel_batch
        opt.radial_bins = radial_bins
        opt.radial_max_um = radial_max_um
        opt.column_grid = column_grid
        opt.grid_gap_um = grid_gap_um
        opt.tally_mode = tally_mode
        self.radial_bins = radial_bins
        self._tune_cache = tune_cache.encode() if tune_cache else None
        opt.tune_cache = self._tune_cache
        self.params = params
        self._h = ctypes.c_void_p()
        check(lib.fd2_create(ctypes.byref(params), ctypes.byref(opt), ctypes.byref(self._h)), "fd2_create")
        self.num_bins = params.num_bins
        self.n_geom = 1

    # -- lifecycle
    def close(self):
        if self._h:
            self._lib.fd2_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def _check(self, st, where):
        check(st, where, self._h)

    # -- configuration and input
    def set_geometries(self, geoms):
        arr = (Geometry * len(geoms))(*geoms)
        self._check(self._lib.fd2_set_geometries(self._h, arr, len(geoms)), "set_geometries")
        self.n_geom = len(geoms)

    def submit_events(self, x_cm, y_cm, z_cm, de_ev, hist):
        """EDE buffer in the reference's units (cm, eV, 1-based history)."""
        a = [np.ascontiguousarray(v, dtype=np.float64) for v in (x_cm, y_cm, z_cm, de_ev)]
        h = np.ascontiguousarray(hist, dtype=np.int32)
        self._check(self._lib.fd2_submit_events(self._h, *[ptr(v) for v in a], ptr(h), len(h)), "submit_events")

    def submit_events_um(self, x_um, y_um, z_um, e_ev, hist, nphot=None, geom=None):
        a = [np.ascontiguousarray(v, dtype=np.float32) for v in (x_um, y_um, z_um)]
        e = None if e_ev is None else np.ascontiguousarray(e_ev, dtype=np.float32)
        h = np.ascontiguousarray(hist, dtype=np.int32)
        n = None if nphot is None else np.ascontiguousarray(nphot, dtype=np.int32)
        g = None if geom is None else np.ascontiguousarray(geom, dtype=np.uint16)
        self._check(self._lib.fd2_submit_events_um(self._h, *[ptr(v) for v in a], ptr(e), ptr(h), ptr(n), ptr(g),
                                                   len(h)), "submit_events_um")

    def submit(self, es: EventSet, nphot=None):
        self.submit_events_um(es.x_um, es.y_um, es.z_um, es.e_ev, es.hist, nphot, es.geom)

    def ingest(self, batch_events: int = 1 << 18, units: int = UNITS_CM) -> "Ingest":
        """Open a streaming ingest (fd2_ingest_begin): pushed events are
        transported batch by batch while the caller goes on pushing."""
        h = ctypes.c_void_p()
        self._check(self._lib.fd2_ingest_begin(self._h, int(batch_events), int(units), ctypes.byref(h)),
                    "ingest_begin")
        return Ingest(self, h)

    # -- execution
    def run(self):
        self._check(self._lib.fd2_run(self._h), "run")

    def wait(self):
        self._check(self._lib.fd2_wait(self._h), "wait")

    def run_sync(self):
        self.run()
        self.wait()

    def reset_tallies(self):
        self._check(self._lib.fd2_reset_tallies(self._h), "reset_tallies")

    def autotune(self, budget_runs: int = 0):
        self._check(self._lib.fd2_autotune(self._h, budget_runs), "autotune")

    # -- results
    def counters(self, geom: int = 0) -> dict:
        c = Counters()
        self._check(self._lib.fd2_get_counters(self._h, geom, ctypes.byref(c)), "get_counters")
        return c.as_dict()

    def prf_dims(self, geom: int = 0):
        x, y = ctypes.c_int32(), ctypes.c_int32()
        self._check(self._lib.fd2_get_prf_dims(self._h, geom, ctypes.byref(x), ctypes.byref(y)), "get_prf_dims")
        return x.value, y.value

    def prf(self, geom: int = 0) -> np.ndarray:
        """PRF counts, shape (xdim, ydim), [ii, jj] with ii the x pixel."""
        xd, yd = self.prf_dims(geom)
        img = np.zeros(xd * yd, np.uint64)
        self._check(self._lib.fd2_get_prf(self._h, geom, ptr(img), img.size), "get_prf")
        return img.reshape(xd, yd)

    def detected_per_primary(self) -> np.ndarray:
        out = np.zeros(max(self.params.num_hist, 1), np.int32)
        self._check(self._lib.fd2_get_detected_per_primary(self._h, ptr(out), out.size), "get_detected_per_primary")
        return out[:self.params.num_hist]

    def radial(self) -> np.ndarray:
        """Label mode: [num_hist, radial_bins + 1] detected photons by distance
        from their event (last column: beyond radial_max_um)."""
        nb = self.radial_bins + 1
        out = np.zeros(max(self.params.num_hist, 1) * nb, np.uint32)
        self._check(self._lib.fd2_get_radial(self._h, ptr(out), out.size), "get_radial")
        return out.reshape(-1, nb)[:self.params.num_hist]

    def photon_counts(self, n_events: int) -> np.ndarray:
        out = np.zeros(max(n_events, 1), np.int32)
        self._check(self._lib.fd2_get_photon_counts(self._h, ptr(out), out.size), "get_photon_counts")
        return out[:n_events]

    def phs(self, geom: int = 0) -> np.ndarray:
        out = np.zeros(self.num_bins, np.int32)
        self._check(self._lib.fd2_get_phs(self._h, geom, ptr(out), self.num_bins), "get_phs")
        return out

    def phs_stats(self, geom: int = 0) -> dict:
        s = PhsStats()
        self._check(self._lib.fd2_get_phs_stats(self._h, geom, ctypes.byref(s)), "get_phs_stats")
        return {n: getattr(s, n) for n, _ in s._fields_}

    def timing(self) -> dict:
        t = Timing()
        self._check(self._lib.fd2_get_timing(self._h, ctypes.byref(t)), "get_timing")
        return {n: getattr(t, n) for n, _ in t._fields_}

    def stream_ptr(self) -> int:
        return self._lib.fd2_get_stream(self._h) or 0

    def write_outputs(self, directory: str):
        self._check(self._lib.fd2_write_outputs(self._h, str(directory).encode()), "write_outputs")

    def replay(self, total_photons: int, mode: int = REPLAY_REF, seed_input: int = 271828182, base: int = 0,
               records: bool = True):
        """Replay of the reference C path; per-photon records when asked."""
        fate = np.zeros(max(total_photons, 1), np.int8) if records else None
        pix = np.zeros(2 * max(total_photons, 1), np.int32) if records else None
        seeds = np.zeros(2 * max(total_photons, 1), np.int32) if records else None
        steps = np.zeros(max(total_photons, 1), np.int32) if records else None
        self._check(self._lib.fd2_replay(self._h, mode, seed_input, base, ptr(fate), ptr(pix), ptr(seeds), ptr(steps)),
                    "replay")
        if not records:
            return None
        return {"fate": fate[:total_photons], "pix": pix[:2 * total_photons].reshape(-1, 2),
                "seeds": seeds[:2 * total_photons].reshape(-1, 2), "steps": steps[:total_photons]}


class Ingest:
    """An open event stream of an OpticalTransport (include/fd2.h,
    fd2_ingest_*).  The tallies after end() equal one submission and run of
    the concatenated stream."""

    def __init__(self, transport: OpticalTransport, handle):
        self._t = transport
        self._h = handle

    def _check(self, st, where):
        if st == 0:
            return
        try:
            self._t._check(st, where)
        finally:  # the stream is unusable after an error: release it
            h, self._h = self._h, None
            if h:
                self._t._lib.fd2_ingest_end(h, None)

    def push(self, x_cm, y_cm, z_cm, de_ev, hist):
        """Events in the reference's units (cm, eV, 1-based history)."""
        a = [np.ascontiguousarray(v, dtype=np.float64) for v in (x_cm, y_cm, z_cm, de_ev)]
        h = np.ascontiguousarray(hist, dtype=np.int32)
        self._check(self._t._lib.fd2_ingest_push(self._h, *[ptr(v) for v in a], ptr(h), len(h)), "ingest_push")

    def push_um(self, x_um, y_um, z_um, e_ev, hist):
        a = [np.ascontiguousarray(v, dtype=np.float32) for v in (x_um, y_um, z_um, e_ev)]
        h = np.ascontiguousarray(hist, dtype=np.int32)
        self._check(self._t._lib.fd2_ingest_push_um(self._h, *[ptr(v) for v in a], ptr(h), len(h)), "ingest_push_um")

    def push_file(self, path: str):
        self._check(self._t._lib.fd2_ingest_file(self._h, path.encode()), "ingest_file")

    def end(self) -> dict:
        st = IngestStats()
        h, self._h = self._h, None
        if h is None:
            raise Fd2Error(7, "ingest_end", "the stream is closed")
        self._t._check(self._t._lib.fd2_ingest_end(h, ctypes.byref(st)), "ingest_end")
        return st.as_dict()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        if self._h is not None:
            if exc[0] is None:
                self.end()
            else:
                h, self._h = self._h, None
                self._t._lib.fd2_ingest_end(h, None)
