"""ctypes bindings of the fd2 C ABI (include/fd2.h).

The shared library is built in-tree (``hybridmantis_b200/lib/libfd2.so``,
``make -C hybridmantis_b200``).  Loading fails loudly when it is missing:
there is no Python or CPU fallback for the transport.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, "lib", "libfd2.so")

# fd2_status
OK = 0
STATUS_NAMES = {
    0: "FD2_OK", 1: "FD2_ERR_INVALID_ARGUMENT", 2: "FD2_ERR_IO", 3: "FD2_ERR_PARSE",
    4: "FD2_ERR_CUDA", 5: "FD2_ERR_OUT_OF_MEMORY", 6: "FD2_ERR_TOO_MANY_PHOTONS",
    7: "FD2_ERR_STATE", 8: "FD2_ERR_TIMEOUT", 9: "FD2_ERR_DEVICE_ABORT", 10: "FD2_ERR_NO_DEVICE",
    11: "FD2_ERR_FILE_EXISTS", 12: "FD2_ERR_BAD_EVENT",
}
COUNT_POISSON, COUNT_GAUSSIAN, COUNT_GIVEN = 0, 1, 2
REPLAY_REF, REPLAY_FP64 = 0, 1
UNITS_CM, UNITS_UM = 0, 1


class Fd2Error(RuntimeError):
    def __init__(self, status: int, where: str, detail: str = ""):
        self.status = status
        super().__init__(f"{where}: {STATUS_NAMES.get(status, status)} {detail}".strip())


class Params(ctypes.Structure):
    """hybridMANTIS_input.in, the 24 values in file order."""
    _fields_ = [
        ("num_hist", ctypes.c_int32), ("min_photons", ctypes.c_int32), ("max_photons", ctypes.c_int32),
        ("num_bins", ctypes.c_int32), ("det_x", ctypes.c_double), ("det_y", ctypes.c_double),
        ("det_height", ctypes.c_double), ("radius", ctypes.c_double), ("n_col", ctypes.c_double),
        ("n_gap", ctypes.c_double), ("top_absfrac", ctypes.c_double), ("bulk_abs", ctypes.c_double),
        ("beta", ctypes.c_double), ("d_min", ctypes.c_double), ("d_max", ctypes.c_double),
        ("lb_x", ctypes.c_double), ("lb_y", ctypes.c_double), ("ub_x", ctypes.c_double),
        ("ub_y", ctypes.c_double), ("yield_", ctypes.c_double), ("pixel", ctypes.c_int32),
        ("sensor_refl", ctypes.c_double), ("run_gpu", ctypes.c_int32), ("machine", ctypes.c_int32),
        ("tag", (ctypes.c_char * 11) * 10),
    ]

    def tags(self):
        return [bytes(t).split(b"\0")[0].decode() for t in self.tag]


class Geometry(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in
                ["det_x", "det_y", "det_height", "radius", "n_col", "n_gap", "top_absfrac", "bulk_abs",
                 "beta", "d_min", "d_max", "lb_x", "lb_y", "ub_x", "ub_y", "sensor_refl"]] + \
              [("pixel", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class Options(ctypes.Structure):
    _fields_ = [
        ("device", ctypes.c_int32), ("count_mode", ctypes.c_int32), ("seed", ctypes.c_uint64),
        ("max_photons_per_event", ctypes.c_int64), ("block_size", ctypes.c_int32),
        ("ctas_per_sm", ctypes.c_int32), ("chunk", ctypes.c_int32), ("refill", ctypes.c_int32),
        ("prf_window", ctypes.c_int32), ("use_graph", ctypes.c_int32), ("wait_timeout_s", ctypes.c_double),
        ("tune_cache", ctypes.c_char_p), ("event_base", ctypes.c_int64), ("fresnel_batch", ctypes.c_int32),
        ("radial_bins", ctypes.c_int32), ("radial_max_um", ctypes.c_double),
        ("column_grid", ctypes.c_int32), ("grid_gap_um", ctypes.c_double), ("tally_mode", ctypes.c_int32),
    ]


class Counters(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in
                ["generated", "detected", "abs_top", "abs_bulk", "lost", "outofcol", "theta1", "capped",
                 "detected_in_prf"]] + [("photon_distance", ctypes.c_double)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class PhsStats(ctypes.Structure):
    _fields_ = [("primaries", ctypes.c_double), ("sum", ctypes.c_double), ("sum_sq", ctypes.c_double),
                ("mean", ctypes.c_double), ("swank", ctypes.c_double), ("phs_dropped", ctypes.c_int64)]


class Timing(ctypes.Structure):
    _fields_ = [("transport_ms", ctypes.c_float), ("pipeline_ms", ctypes.c_float), ("photons", ctypes.c_int64),
                ("grid", ctypes.c_int32), ("block", ctypes.c_int32), ("chunk", ctypes.c_int32),
                ("refill", ctypes.c_int32), ("prf_window", ctypes.c_int32), ("fresnel_batch", ctypes.c_int32)]


class IngestStats(ctypes.Structure):
    _fields_ = [("events", ctypes.c_int64), ("batches", ctypes.c_int64), ("photons", ctypes.c_int64),
                ("host_seconds", ctypes.c_double), ("push_wait_seconds", ctypes.c_double),
                ("device_ms", ctypes.c_float)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class Events(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int64), ("num_hist", ctypes.c_int32),
        ("x_um", ctypes.POINTER(ctypes.c_float)), ("y_um", ctypes.POINTER(ctypes.c_float)),
        ("z_um", ctypes.POINTER(ctypes.c_float)), ("e_ev", ctypes.POINTER(ctypes.c_float)),
        ("hist", ctypes.POINTER(ctypes.c_int32)), ("geom", ctypes.POINTER(ctypes.c_uint16)),
        ("num_geom", ctypes.c_int32), ("geometries", ctypes.POINTER(Geometry)), ("params", Params),
    ]


class SgConfig(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int32), ("hidden", ctypes.c_int32), ("radial_bins", ctypes.c_int32),
                ("radial_max_um", ctypes.c_double), ("batch", ctypes.c_int32), ("lr", ctypes.c_float),
                ("beta1", ctypes.c_float), ("beta2", ctypes.c_float), ("adam_eps", ctypes.c_float),
                ("radial_weight", ctypes.c_float), ("lateral_um", ctypes.c_float), ("seed", ctypes.c_uint64),
                ("depth_margin_um", ctypes.c_float)]


class SgHull(ctypes.Structure):
    _fields_ = [("lo", ctypes.c_float * 8), ("hi", ctypes.c_float * 8)]


class SgStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int64) for n in ["events", "surrogate_events", "mc_events", "audit_events",
                                              "surrogate_photons", "surrogate_detected"]] + \
               [(n, ctypes.c_double) for n in ["audit_mc_detected", "audit_sg_expected", "audit_photons",
                                               "audit_z", "audit_radial_l1"]] + \
               [(n, ctypes.c_float) for n in ["sg_ms", "mc_ms", "audit_ms", "total_ms"]]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class XrayMaterialInfo(ctypes.Structure):
    _fields_ = [("density_g_cm3", ctypes.c_double), ("molar_mass_g_mol", ctypes.c_double),
                ("molecules_per_cm3", ctypes.c_double), ("n_elements", ctypes.c_int32),
                ("z", ctypes.c_int32 * 8), ("atoms_per_molecule", ctypes.c_double * 8),
                ("k_edge_ev", ctypes.c_double * 8), ("e_min_ev", ctypes.c_double), ("e_max_ev", ctypes.c_double),
                ("n_photon_nodes", ctypes.c_int32), ("n_transitions", ctypes.c_int32),
                ("rayleigh_screening_cm", ctypes.c_double)]


class XraySource(ctypes.Structure):
    _fields_ = [("particle", ctypes.c_int32), ("n_spectrum", ctypes.c_int32), ("e_ev", ctypes.c_void_p),
                ("prob", ctypes.c_void_p), ("center_cm", ctypes.c_double * 3), ("sides_cm", ctypes.c_double * 3),
                ("euler_deg", ctypes.c_double * 3), ("direction", ctypes.c_double * 3),
                ("semiaperture_deg", ctypes.c_double)]


class XrayOptions(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int32), ("det_x_um", ctypes.c_double), ("det_y_um", ctypes.c_double),
                ("det_height_um", ctypes.c_double), ("eabs_electron_ev", ctypes.c_double),
                ("eabs_photon_ev", ctypes.c_double), ("electron_step_loss", ctypes.c_double),
                ("electron_local_ev", ctypes.c_double), ("fluorescence", ctypes.c_int32), ("max_edes_per_history", ctypes.c_int32),
                ("batch_histories", ctypes.c_int64), ("seed", ctypes.c_uint64)]


class XrayStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int64) for n in ["histories", "missed", "edes", "merged_histories", "photoelectric",
                                              "compton", "rayleigh", "fluorescence_emitted",
                                              "fluorescence_escaped", "auger_emitted", "electron_steps"]] + \
               [(n, ctypes.c_double) for n in ["e_source_ev", "e_deposited_ev", "e_escaped_photon_ev",
                                               "e_escaped_electron_ev"]]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


_lib = None

# Every symbol include/*.h declare.
EXPORTED = [
    "fd2_status_string", "fd2_default_options", "fd2_parse_input_file", "fd2_params_fill_tags",
    "fd2_params_to_geometry", "fd2_prf_dims", "fd2_create", "fd2_destroy", "fd2_last_error",
    "fd2_set_geometries", "fd2_submit_events", "fd2_submit_events_um", "fd2_run", "fd2_wait",
    "fd2_reset_tallies", "fd2_get_counters", "fd2_get_prf_dims", "fd2_get_prf",
    "fd2_get_detected_per_primary", "fd2_get_radial", "fd2_get_photon_counts", "fd2_get_phs", "fd2_get_phs_stats",
    "fd2_get_timing", "fd2_get_stream", "fd2_write_outputs", "fd2_write_output_files", "fd2_replay",
    "fd2_autotune", "fd2_transport_noalloc", "fd2_measure_fp32_peak", "fd2_debug_wall_root",
    "fd2_synth_events", "fd2_free_events", "fd2_read_events_text", "fd2_write_events_text",
    "fd2_read_events_binary", "fd2_write_events_binary",
    "fd2_ingest_begin", "fd2_ingest_push", "fd2_ingest_push_um", "fd2_ingest_file", "fd2_ingest_end",
    "gpuoptical_", "cpuoptical_", "gpuoptlb_", "cpuoptlb_", "fd2_compat_status",
    "fd2_sg_default_config", "fd2_sg_create", "fd2_sg_destroy", "fd2_sg_last_error", "fd2_sg_set_data",
    "fd2_sg_train", "fd2_sg_set_lr", "fd2_sg_eval", "fd2_sg_num_params", "fd2_sg_get_params", "fd2_sg_set_params",
    "fd2_sg_get_hull", "fd2_sg_set_hull", "fd2_sg_save", "fd2_sg_load", "fd2_sg_loss_grad", "fd2_sg_predict",
    "fd2_sg_set_edge", "fd2_sg_get_edge",
    "fd2_sg_run",
    "fd2_mtf", "fd2_nnps",
    "fd2_submit_events_device",
    "fd2_xray_load_material", "fd2_xray_save_material", "fd2_xray_free_material", "fd2_xray_material_get_info",
    "fd2_xray_attenuation", "fd2_xray_electron_tables", "fd2_xray_default_options", "fd2_xray_create",
    "fd2_xray_destroy", "fd2_xray_last_error", "fd2_xray_run", "fd2_xray_num_edes", "fd2_xray_get_edes",
    "fd2_xray_get_history_info", "fd2_xray_get_stats", "fd2_xray_clear_stats", "fd2_xray_get_timing",
    "fd2_xray_submit", "fd2_xray_device_edes", "fd2_xray_sample", "fd2_xray_read_penEasy_source",
]


def load():
    """Load libfd2.so (raises when the extension has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `make -C {PKG_DIR}` "
                          "(or __graft_entry__.build()); there is no fallback path")
    lib = ctypes.CDLL(LIB_PATH)
    P = ctypes.POINTER
    vp = ctypes.c_void_p
    sig = {
        "fd2_status_string": (ctypes.c_char_p, [ctypes.c_int]),
        "fd2_default_options": (None, [P(Options)]),
        "fd2_parse_input_file": (ctypes.c_int, [ctypes.c_char_p, P(Params)]),
        "fd2_params_fill_tags": (ctypes.c_int, [P(Params)]),
        "fd2_params_to_geometry": (ctypes.c_int, [P(Params), P(Geometry)]),
        "fd2_prf_dims": (ctypes.c_int, [P(Geometry), P(ctypes.c_int32), P(ctypes.c_int32)]),
        "fd2_create": (ctypes.c_int, [P(Params), P(Options), P(vp)]),
        "fd2_debug_wall_root": (ctypes.c_int, [ctypes.c_int32, vp, vp, vp, vp]),
        "fd2_measure_fp32_peak": (ctypes.c_int, [ctypes.c_int32, ctypes.c_double, P(ctypes.c_double),
                                                 P(ctypes.c_double)]),
        "fd2_destroy": (None, [vp]),
        "fd2_last_error": (ctypes.c_char_p, [vp]),
        "fd2_set_geometries": (ctypes.c_int, [vp, P(Geometry), ctypes.c_int32]),
        "fd2_submit_events": (ctypes.c_int, [vp, vp, vp, vp, vp, vp, ctypes.c_int64]),
        "fd2_submit_events_um": (ctypes.c_int, [vp, vp, vp, vp, vp, vp, vp, vp, ctypes.c_int64]),
        "fd2_run": (ctypes.c_int, [vp]),
        "fd2_wait": (ctypes.c_int, [vp]),
        "fd2_reset_tallies": (ctypes.c_int, [vp]),
        "fd2_get_counters": (ctypes.c_int, [vp, ctypes.c_int32, P(Counters)]),
        "fd2_get_prf_dims": (ctypes.c_int, [vp, ctypes.c_int32, P(ctypes.c_int32), P(ctypes.c_int32)]),
        "fd2_get_prf": (ctypes.c_int, [vp, ctypes.c_int32, vp, ctypes.c_int64]),
        "fd2_get_detected_per_primary": (ctypes.c_int, [vp, vp, ctypes.c_int64]),
        "fd2_get_radial": (ctypes.c_int, [vp, vp, ctypes.c_int64]),
        "fd2_get_photon_counts": (ctypes.c_int, [vp, vp, ctypes.c_int64]),
        "fd2_get_phs": (ctypes.c_int, [vp, ctypes.c_int32, vp, ctypes.c_int32]),
        "fd2_get_phs_stats": (ctypes.c_int, [vp, ctypes.c_int32, P(PhsStats)]),
        "fd2_get_timing": (ctypes.c_int, [vp, P(Timing)]),
        "fd2_get_stream": (vp, [vp]),
        "fd2_write_outputs": (ctypes.c_int, [vp, ctypes.c_char_p]),
        "fd2_write_output_files": (ctypes.c_int, [P(Params), P(Geometry), vp, ctypes.c_int32, ctypes.c_int32, vp,
                                                  ctypes.c_int32, ctypes.c_double, ctypes.c_char_p, ctypes.c_char_p]),
        "fd2_replay": (ctypes.c_int, [vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_int64, vp, vp, vp, vp]),
        "fd2_autotune": (ctypes.c_int, [vp, ctypes.c_int32]),
        "fd2_transport_noalloc": (ctypes.c_int, [P(Geometry), vp, vp, vp, vp, vp, ctypes.c_int64, ctypes.c_int32,
                                                 ctypes.c_uint64, vp, vp, vp, vp]),
        "fd2_synth_events": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, ctypes.c_uint64, P(Events)]),
        "fd2_free_events": (None, [P(Events)]),
        "fd2_read_events_text": (ctypes.c_int, [ctypes.c_char_p, P(Events)]),
        "fd2_write_events_text": (ctypes.c_int, [ctypes.c_char_p, P(Events)]),
        "fd2_read_events_binary": (ctypes.c_int, [ctypes.c_char_p, P(Events)]),
        "fd2_write_events_binary": (ctypes.c_int, [ctypes.c_char_p, P(Events)]),
        "fd2_ingest_begin": (ctypes.c_int, [vp, ctypes.c_int64, ctypes.c_int32, P(vp)]),
        "fd2_ingest_push": (ctypes.c_int, [vp, vp, vp, vp, vp, vp, ctypes.c_int64]),
        "fd2_ingest_push_um": (ctypes.c_int, [vp, vp, vp, vp, vp, vp, ctypes.c_int64]),
        "fd2_ingest_file": (ctypes.c_int, [vp, ctypes.c_char_p]),
        "fd2_ingest_end": (ctypes.c_int, [vp, P(IngestStats)]),
        "fd2_compat_status": (ctypes.c_int, []),
        "fd2_sg_default_config": (None, [P(SgConfig)]),
        "fd2_sg_create": (ctypes.c_int, [P(SgConfig), P(vp)]),
        "fd2_sg_destroy": (None, [vp]),
        "fd2_sg_last_error": (ctypes.c_char_p, [vp]),
        "fd2_sg_set_data": (ctypes.c_int, [vp, vp, vp, vp, vp, ctypes.c_int64, ctypes.c_int64]),
        "fd2_sg_train": (ctypes.c_int, [vp, ctypes.c_int32, P(ctypes.c_float), P(ctypes.c_float)]),
        "fd2_sg_eval": (ctypes.c_int, [vp, P(ctypes.c_float), P(ctypes.c_float), P(ctypes.c_float)]),
        "fd2_sg_set_lr": (ctypes.c_int, [vp, ctypes.c_float]),
        "fd2_sg_num_params": (ctypes.c_int64, [vp]),
        "fd2_sg_get_params": (ctypes.c_int, [vp, vp, ctypes.c_int64]),
        "fd2_sg_set_params": (ctypes.c_int, [vp, vp, ctypes.c_int64]),
        "fd2_sg_get_hull": (ctypes.c_int, [vp, P(SgHull)]),
        "fd2_sg_set_hull": (ctypes.c_int, [vp, P(SgHull)]),
        "fd2_sg_save": (ctypes.c_int, [vp, ctypes.c_char_p]),
        "fd2_sg_load": (ctypes.c_int, [vp, ctypes.c_char_p]),
        "fd2_sg_set_edge": (ctypes.c_int, [vp, ctypes.c_float, ctypes.c_float]),
        "fd2_sg_get_edge": (ctypes.c_int, [vp, P(ctypes.c_float), P(ctypes.c_float)]),
        "fd2_sg_loss_grad": (ctypes.c_int, [vp, vp, vp, vp, vp, ctypes.c_int32, P(ctypes.c_float), vp]),
        "fd2_sg_predict": (ctypes.c_int, [vp, vp, ctypes.c_int64, vp]),
        "fd2_sg_run": (ctypes.c_int, [vp, vp, ctypes.c_double, P(SgStats)]),
        "fd2_mtf": (ctypes.c_int, [ctypes.c_int32, vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_double, ctypes.c_int32,
                                   vp, vp, vp, vp]),
        "fd2_nnps": (ctypes.c_int, [ctypes.c_int32, vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_double,
                                    ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                    ctypes.c_int32, vp, vp, vp, P(ctypes.c_double)]),
        "fd2_submit_events_device": (ctypes.c_int, [vp, vp, vp, vp, vp, vp, ctypes.c_int64]),
        "fd2_xray_load_material": (ctypes.c_int, [ctypes.c_char_p, P(vp)]),
        "fd2_xray_save_material": (ctypes.c_int, [vp, ctypes.c_char_p]),
        "fd2_xray_free_material": (None, [vp]),
        "fd2_xray_material_get_info": (ctypes.c_int, [vp, P(XrayMaterialInfo)]),
        "fd2_xray_attenuation": (ctypes.c_int, [vp, vp, ctypes.c_int64, vp]),
        "fd2_xray_electron_tables": (ctypes.c_int, [vp, vp, ctypes.c_int64, vp, vp]),
        "fd2_xray_default_options": (None, [P(XrayOptions)]),
        "fd2_xray_create": (ctypes.c_int, [vp, P(XrayOptions), P(vp)]),
        "fd2_xray_destroy": (None, [vp]),
        "fd2_xray_last_error": (ctypes.c_char_p, [vp]),
        "fd2_xray_run": (ctypes.c_int, [vp, P(XraySource), ctypes.c_int64, ctypes.c_int64]),
        "fd2_xray_num_edes": (ctypes.c_int, [vp, P(ctypes.c_int64)]),
        "fd2_xray_get_edes": (ctypes.c_int, [vp, vp, vp, vp, vp, vp, ctypes.c_int64]),
        "fd2_xray_get_history_info": (ctypes.c_int, [vp, vp, vp, vp, vp, vp, vp, ctypes.c_int64]),
        "fd2_xray_get_stats": (ctypes.c_int, [vp, P(XrayStats)]),
        "fd2_xray_clear_stats": (ctypes.c_int, [vp]),
        "fd2_xray_get_timing": (ctypes.c_int, [vp, P(ctypes.c_double), P(ctypes.c_double)]),
        "fd2_xray_submit": (ctypes.c_int, [vp, vp]),
        "fd2_xray_device_edes": (ctypes.c_int, [vp, P(vp), P(vp), P(vp), P(vp), P(vp), P(ctypes.c_int64)]),
        "fd2_xray_sample": (ctypes.c_int, [vp, ctypes.c_int32, ctypes.c_double, ctypes.c_double, ctypes.c_int64,
                                           ctypes.c_uint64, vp]),
        "fd2_xray_read_penEasy_source": (ctypes.c_int, [ctypes.c_char_p, P(XraySource), vp, vp, ctypes.c_int32]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def check(status: int, where: str, ctx=None):
    if status != OK:
        detail = ""
        if ctx is not None:
            detail = load().fd2_last_error(ctx).decode(errors="replace")
        raise Fd2Error(status, where, detail)


def ptr(a: np.ndarray | None):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)
