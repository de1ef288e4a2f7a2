"""GPU x-ray front end (``include/fd2_xray.h``): energy-deposition events
for the optical transport, produced on the device.

In hybridMANTIS the EDEs come from PENELOPE run by penEasy with the BIGS
source (main/sourceBoxIsotropicGaussSpectrum.f) and the EDE tally
(main/hybridMANTIS_tallyEnergyDepositionEvents.f:155-200).  This module
reads the same inputs -- the PENELOPE material file (example/CsI.mat) and
the penEasy input's SOURCE BOX ISOTROPIC GAUSS SPECTRUM section -- and runs
the front end's own photon/electron transport on the GPU.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field

import numpy as np

from ._lib import XrayMaterialInfo, XrayOptions, XraySource, XrayStats, check, load, ptr

PHOTON = 2
ELECTRON = 1
DATA_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")
CSI_TABLE = os.path.join(DATA_DIR, "csi_xray.tab")


class Material:
    """Tables of one detector material (PENELOPE .mat file or a table file)."""

    def __init__(self, path: str = CSI_TABLE):
        self._lib = load()
        self._h = ctypes.c_void_p()
        check(self._lib.fd2_xray_load_material(path.encode(), ctypes.byref(self._h)), f"load_material({path})")

    def close(self):
        if self._h:
            self._lib.fd2_xray_free_material(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def save(self, path: str):
        check(self._lib.fd2_xray_save_material(self._h, path.encode()), "save_material")

    def info(self) -> dict:
        i = XrayMaterialInfo()
        check(self._lib.fd2_xray_material_get_info(self._h, ctypes.byref(i)), "material_get_info")
        n = i.n_elements
        return {"density": i.density_g_cm3, "molar_mass": i.molar_mass_g_mol,
                "molecules_per_cm3": i.molecules_per_cm3, "z": list(i.z[:n]),
                "atoms": list(i.atoms_per_molecule[:n]), "k_edge_ev": list(i.k_edge_ev[:n]),
                "e_min": i.e_min_ev, "e_max": i.e_max_ev, "photon_nodes": i.n_photon_nodes,
                "transitions": i.n_transitions, "rayleigh_screening_cm": i.rayleigh_screening_cm}

    def attenuation(self, e_ev) -> np.ndarray:
        """Linear attenuation (1/cm): columns Rayleigh, Compton, photoelectric, total."""
        e = np.ascontiguousarray(np.atleast_1d(e_ev), dtype=np.float64)
        out = np.zeros((len(e), 4))
        check(self._lib.fd2_xray_attenuation(self._h, ptr(e), len(e), ptr(out)), "attenuation")
        return out

    def electron(self, e_ev):
        """CSDA range (cm) and first transport mean free path (cm)."""
        e = np.ascontiguousarray(np.atleast_1d(e_ev), dtype=np.float64)
        r = np.zeros(len(e))
        l1 = np.zeros(len(e))
        check(self._lib.fd2_xray_electron_tables(self._h, ptr(e), len(e), ptr(r), ptr(l1)), "electron_tables")
        return r, l1


@dataclass
class Source:
    """penEasy's SOURCE BOX ISOTROPIC GAUSS SPECTRUM section (cm, eV, deg)."""
    e_ev: np.ndarray
    prob: np.ndarray
    particle: int = PHOTON
    center_cm: tuple = (0.04545, 0.04545, 1.0)
    sides_cm: tuple = (0.0, 0.0, 0.0)
    euler_deg: tuple = (0.0, 0.0, 0.0)
    direction: tuple = (0.0, 0.0, -1.0)
    semiaperture_deg: float = 0.0
    _keep: list = field(default_factory=list, repr=False)

    def as_struct(self) -> XraySource:
        e = np.ascontiguousarray(self.e_ev, dtype=np.float64)
        p = np.ascontiguousarray(self.prob, dtype=np.float64)
        self._keep = [e, p]
        s = XraySource()
        s.particle = self.particle
        s.n_spectrum = len(e)
        s.e_ev = e.ctypes.data
        s.prob = p.ctypes.data
        for a in range(3):
            s.center_cm[a] = self.center_cm[a]
            s.sides_cm[a] = self.sides_cm[a]
            s.euler_deg[a] = self.euler_deg[a]
            s.direction[a] = self.direction[a]
        s.semiaperture_deg = self.semiaperture_deg
        return s


def monoenergetic(e_ev: float, **kw) -> Source:
    """A line source: one bin of zero width (the reference example's form)."""
    return Source(np.array([e_ev, e_ev]), np.array([1.0, -1.0]), **kw)


def triangular_spectrum(lo_ev: float, mode_ev: float, hi_ev: float, bins: int = 200, **kw) -> Source:
    """Triangular(lo, mode, hi) as a binned penEasy spectrum (config 1's x-rays)."""
    e = np.linspace(lo_ev, hi_ev, bins + 1)
    mid = 0.5 * (e[:-1] + e[1:])
    pdf = np.where(mid < mode_ev, (mid - lo_ev) / (mode_ev - lo_ev), (hi_ev - mid) / (hi_ev - mode_ev))
    return Source(e, np.append(pdf, -1.0), **kw)


def read_penEasy_source(path: str) -> Source:
    """The BIGS section of a penEasy input file (fd2_xray_read_penEasy_source)."""
    cap = 100000
    e = np.zeros(cap)
    pr = np.zeros(cap)
    s = XraySource()
    check(load().fd2_xray_read_penEasy_source(path.encode(), ctypes.byref(s), ptr(e), ptr(pr), cap),
          f"read_penEasy_source({path})")
    n = s.n_spectrum
    return Source(e[:n].copy(), pr[:n].copy(), particle=s.particle, center_cm=tuple(s.center_cm),
                  sides_cm=tuple(s.sides_cm), euler_deg=tuple(s.euler_deg), direction=tuple(s.direction),
                  semiaperture_deg=s.semiaperture_deg)


class XrayFrontEnd:
    """One front-end context on a GPU (fd2_xray_create)."""

    def __init__(self, material: Material | str = CSI_TABLE, *, det_x_um: float = 909.0, det_y_um: float = 909.0,
                 det_height_um: float = 150.0, eabs_electron_ev: float = 50.0, eabs_photon_ev: float = 50.0,
                 electron_step_loss: float = 0.25, electron_local_ev: float = 1000.0, fluorescence: bool = True,
                 max_edes_per_history: int = 256,
                 batch_histories: int = 65536, seed: int = 12345, device: int = 0):
        self._lib = load()
        self.material = material if isinstance(material, Material) else Material(material)
        o = XrayOptions()
        self._lib.fd2_xray_default_options(ctypes.byref(o))
        o.device = device
        o.det_x_um, o.det_y_um, o.det_height_um = det_x_um, det_y_um, det_height_um
        o.eabs_electron_ev, o.eabs_photon_ev = eabs_electron_ev, eabs_photon_ev
        o.electron_step_loss = electron_step_loss
        o.electron_local_ev = electron_local_ev
        o.fluorescence = 1 if fluorescence else 0
        o.max_edes_per_history = max_edes_per_history
        o.batch_histories = batch_histories
        o.seed = seed
        self.options = o
        self._h = ctypes.c_void_p()
        check(self._lib.fd2_xray_create(self.material._h, ctypes.byref(o), ctypes.byref(self._h)), "xray_create")
        self.n_histories = 0

    def close(self):
        if self._h:
            self._lib.fd2_xray_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st, where):
        if st != 0:
            from ._lib import Fd2Error
            raise Fd2Error(st, where, self._lib.fd2_xray_last_error(self._h).decode(errors="replace"))

    def run(self, source: Source, n: int, first: int = 0):
        s = source.as_struct()
        self._check(self._lib.fd2_xray_run(self._h, ctypes.byref(s), int(first), int(n)), "xray_run")
        self.n_histories = n

    def num_edes(self) -> int:
        v = ctypes.c_int64()
        self._check(self._lib.fd2_xray_num_edes(self._h, ctypes.byref(v)), "num_edes")
        return v.value

    def edes(self) -> dict:
        n = self.num_edes()
        out = {k: np.zeros(n) for k in ("x_cm", "y_cm", "z_cm", "de_ev")}
        out["hist"] = np.zeros(n, np.int32)
        self._check(self._lib.fd2_xray_get_edes(self._h, ptr(out["x_cm"]), ptr(out["y_cm"]), ptr(out["z_cm"]),
                                                ptr(out["de_ev"]), ptr(out["hist"]), n), "get_edes")
        return out

    def history_info(self) -> dict:
        n = self.n_histories
        out = {k: np.zeros(n) for k in ("e_source_ev", "e_escaped_photon_ev", "e_escaped_electron_ev",
                                        "first_depth_cm")}
        out["first_kind"] = np.zeros(n, np.int32)
        out["n_edes"] = np.zeros(n, np.int32)
        self._check(self._lib.fd2_xray_get_history_info(
            self._h, ptr(out["e_source_ev"]), ptr(out["e_escaped_photon_ev"]), ptr(out["e_escaped_electron_ev"]),
            ptr(out["first_depth_cm"]), ptr(out["first_kind"]), ptr(out["n_edes"]), n), "history_info")
        return out

    def stats(self) -> dict:
        s = XrayStats()
        self._check(self._lib.fd2_xray_get_stats(self._h, ctypes.byref(s)), "get_stats")
        return s.as_dict()

    def clear_stats(self):
        self._check(self._lib.fd2_xray_clear_stats(self._h), "clear_stats")

    def timing(self) -> dict:
        a, b = ctypes.c_double(), ctypes.c_double()
        self._check(self._lib.fd2_xray_get_timing(self._h, ctypes.byref(a), ctypes.byref(b)), "get_timing")
        return {"transport_ms": a.value, "compact_ms": b.value}

    def submit(self, optical):
        """Hand the last run's EDEs to an OpticalTransport on the device."""
        self._check(self._lib.fd2_xray_submit(self._h, optical._h), "xray_submit")

    def sample(self, which: int, e_ev: float, n: int, seed: int = 1, param: float = 0.0) -> np.ndarray:
        out = np.zeros(n)
        self._check(self._lib.fd2_xray_sample(self._h, int(which), float(e_ev), float(param), int(n), int(seed),
                                              ptr(out)), "xray_sample")
        return out
