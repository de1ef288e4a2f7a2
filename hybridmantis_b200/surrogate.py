"""Learned surrogate of the optical transport (include/fd2_surrogate.h).

``label_points`` produces training data with this library's own Monte Carlo
in label mode: every point is one deposition transported with a fixed number
of photons, and its label is the detected count and the radial histogram of
the detected photons around it.  ``Surrogate`` wraps the C ABI: BF16
tensor-core training on the GPU, prediction, and the surrogate-in-the-loop
event pipeline (``run``).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import Geometry, SgConfig, SgHull, SgStats, check, load, ptr
from .fastdetect2 import COUNT_GIVEN, OpticalTransport, default_params

FEATURES = ["depth_um", "energy_kev", "lateral_r", "thickness_um", "radius_um", "beta", "top_reflectivity",
            "log10_mu"]
N_FEATURES = 8
N_OUTPUTS = 25
N_COMPONENTS = 8
MU_SCALE, SD_SCALE = 50.0, 10.0
LATERAL_UNIT_UM = 50.0  # unit of feature 2: the deposition's distance from the detector centre


def geometry_features(g: Geometry) -> np.ndarray:
    """Features 3..7 of a geometry."""
    return np.array([g.det_height, g.radius, g.beta, 1.0 - g.top_absfrac, np.log10(max(g.bulk_abs, 1e-30))],
                    np.float32)


def features(depth_um, energy_kev, lateral_um, g: Geometry) -> np.ndarray:
    """Network inputs of depositions at depth `depth_um` below the entrance
    surface, energy `energy_kev`, `lateral_um` from the detector centre."""
    depth_um = np.asarray(depth_um, np.float32)
    n = depth_um.size
    f = np.empty((n, N_FEATURES), np.float32)
    f[:, 0] = depth_um
    f[:, 1] = energy_kev
    f[:, 2] = np.asarray(lateral_um, np.float32) / LATERAL_UNIT_UM
    f[:, 3:] = geometry_features(g)
    return f


def sample_geometries(n: int, seed: int, base: Geometry | None = None) -> list:
    """Detector geometries over the batched-workload ranges: thickness
    U(100, 600) um, column radius U(2.5, 7.5) um, roughness U(0, 0.5), top
    reflectivity U(0, 1), bulk absorption log-uniform on [1e-5, 1e-3] /um;
    the other parameters from `base` (default: the benchmark detector)."""
    rng = np.random.default_rng(seed)
    if base is None:
        base = _lib.Geometry()
        load().fd2_params_to_geometry(ctypes.byref(default_params()), ctypes.byref(base))
    out = []
    for _ in range(n):
        g = Geometry.from_buffer_copy(base)
        g.det_height = rng.uniform(100.0, 600.0)
        g.radius = rng.uniform(2.5, 7.5)
        g.beta = rng.uniform(0.0, 0.5)
        g.top_absfrac = 1.0 - rng.uniform(0.0, 1.0)
        g.bulk_abs = float(np.exp(rng.uniform(np.log(1e-5), np.log(1e-3))))
        out.append(g)
    return out


def label_points(geoms, points_per_geom: int, photons: int, seed: int, device: int = 0, radial_bins: int = 96,
                 radial_max_um: float = 400.0, energy_kev=(1.0, 80.0), lateral_um: float = 60.0):
    """Monte Carlo labels: for each geometry, `points_per_geom` depositions
    with depth H u (half of them) or H u^2 (the other half: denser near the
    entrance surface, where x-rays deposit most and the PRF is widest),
    u ~ U(0, 1), energy U(energy_kev), at a distance r from the detector
    centre (uniform azimuth) with r = lateral_um sqrt(v) for half of them
    (uniform over the disc) and lateral_um v^2 for the other half (dense near
    the centre, where the events of a pencil beam lie), v ~ U(0, 1) -- the
    detected fraction falls with r as photons reach the detector's sides --
    each transported with `photons` photons.  Returns
    (features [n, 8], photons [n], detected [n], radial [n, radial_bins + 1])."""
    rng = np.random.default_rng(seed)
    feats, phot, det, rad = [], [], [], []
    for g0 in range(0, len(geoms), 256):
        gs = list(geoms[g0:g0 + 256])
        n = len(gs) * points_per_geom
        p = default_params(num_hist=n)
        with OpticalTransport(p, device=device, count_mode=COUNT_GIVEN, seed=seed + 7919 * g0,
                              radial_bins=radial_bins, radial_max_um=radial_max_um) as t:
            t.set_geometries(gs)
            gi = np.repeat(np.arange(len(gs)), points_per_geom).astype(np.uint16)
            H = np.array([g.det_height for g in gs])[gi]
            u = rng.uniform(0.001, 0.999, n)
            u = np.where(rng.random(n) < 0.5, u, np.maximum(u * u, 0.001))
            depth = (H * u).astype(np.float32).astype(np.float64)
            # half uniform over the disc, half with density ~ r^-1/2 (r = R u^2):
            # in-loop events sit mostly within ~10 um of the beam, where a
            # uniform disc would put few labels
            ul = rng.uniform(0.0, 1.0, n)
            lat = lateral_um * np.where(rng.random(n) < 0.5, np.sqrt(ul), ul * ul)
            phi = rng.uniform(0.0, 2.0 * np.pi, n)
            cx = (np.array([g.det_x / 2.0 for g in gs])[gi] + lat * np.cos(phi)).astype(np.float32)
            cy = (np.array([g.det_y / 2.0 for g in gs])[gi] + lat * np.sin(phi)).astype(np.float32)
            # the feature is the distance of the float positions the walk starts from
            lat = np.hypot(cx.astype(np.float64) - np.array([g.det_x / 2.0 for g in gs])[gi],
                           cy.astype(np.float64) - np.array([g.det_y / 2.0 for g in gs])[gi])
            z = H / 2.0 - depth
            energy = rng.uniform(energy_kev[0], energy_kev[1], n)
            nph = np.full(n, photons, np.int32)
            t.submit_events_um(cx, cy, z, energy * 1000.0, np.arange(1, n + 1), nphot=nph, geom=gi)
            t.run_sync()
            d = t.detected_per_primary()
            r = t.radial()
        f = np.empty((n, N_FEATURES), np.float32)
        f[:, 0] = depth
        f[:, 1] = energy
        f[:, 2] = lat / LATERAL_UNIT_UM
        f[:, 3:] = np.stack([geometry_features(g) for g in gs])[gi]
        feats.append(f)
        phot.append(nph)
        det.append(d.astype(np.int32))
        rad.append(r.astype(np.uint32))
    return np.concatenate(feats), np.concatenate(phot), np.concatenate(det), np.concatenate(rad)


def radial_edges(bins: int = 96, radial_max_um: float = 400.0) -> np.ndarray:
    """Edges of the radial label bins: r_max (j / bins)^2, j = 0..bins."""
    return radial_max_um * (np.arange(bins + 1) / bins) ** 2


def mixture(out: np.ndarray):
    """Decode network outputs [n, 25] into (p_detect [n], w [n, 8], ring radii mu [n, 8], widths sd [n, 8]) in um."""
    out = np.asarray(out, np.float64)
    p = 1.0 / (1.0 + np.exp(-out[:, 0]))
    a = out[:, 1:1 + N_COMPONENTS]
    w = np.exp(a - a.max(1, keepdims=True))
    w /= w.sum(1, keepdims=True)
    om = out[:, 1 + N_COMPONENTS:1 + 2 * N_COMPONENTS]
    mu = MU_SCALE * (np.maximum(om, 0) + np.log1p(np.exp(-np.abs(om))))
    sd = SD_SCALE * np.exp(np.clip(out[:, 1 + 2 * N_COMPONENTS:], -6.0, 4.0))
    return p, w, mu, sd


def radial_bin_probs(out: np.ndarray, bins: int = 96, radial_max_um: float = 400.0) -> np.ndarray:
    """Category probabilities [n, bins + 1] of the mixture of Gaussian rings
    (last: beyond radial_max_um): component k has radial density
    r N(r; mu_k, sd_k) / S_k, mass mu [Phi(t_b) - Phi(t_a)] + sd [phi(t_a) - phi(t_b)]."""
    from scipy.special import ndtr
    _, w, mu, sd = mixture(out)
    e = np.concatenate([radial_edges(bins, radial_max_um), [np.inf]])
    t = (e[None, None, :] - mu[:, :, None]) / sd[:, :, None]
    c, cc = ndtr(t), ndtr(-t)
    ph = np.where(np.isinf(t), 0.0, np.exp(-0.5 * np.where(np.isinf(t), 0.0, t) ** 2) / np.sqrt(2 * np.pi))
    lo = t[:, :, :-1]
    dphi = np.maximum(np.where(lo >= 0, cc[:, :, :-1] - cc[:, :, 1:], c[:, :, 1:] - c[:, :, :-1]), 0.0)
    M = np.maximum(mu[:, :, None] * dphi + sd[:, :, None] * (ph[:, :, :-1] - ph[:, :, 1:]), 0.0)
    t0 = -mu / sd
    S = mu * ndtr(-t0) + sd * np.exp(-0.5 * t0 ** 2) / np.sqrt(2 * np.pi)
    return (w[:, :, None] * M / S[:, :, None]).sum(1)


def edge_weights(amplitude: float, length_um: float, x, y, det_x: float, det_y: float) -> np.ndarray:
    """The sampler's azimuth acceptance at points (x, y) of a det_x x det_y
    detector: prod over its four sides of (1 - amplitude exp(-s / length))."""
    w = np.ones(np.broadcast(x, y).shape)
    for s in (x, det_x - x, y, det_y - y):
        w = w * (1.0 - amplitude * np.exp(-np.asarray(s, np.float64) / length_um))
    return w


def fit_edge(image, cx_um: float, cy_um: float, det_x: float, det_y: float, lb_x: float = 0.0, lb_y: float = 0.0,
             pixel: float = 1.0):
    """Fit the edge survival (amplitude, length) to a Monte Carlo PRF image
    of depositions around (cx, cy): the image's own ring marginal (rings one
    pixel wide around the centre), spread over each ring with the weights
    edge_weights, is compared with the image on the rings at least half the
    distance from the centre to the nearest side out (nearer in, the weights
    are 1 and only the rings' discretisation would count); the pair with the
    smallest L1 wins (amplitude 0 -- uniform rings -- included).  Returns
    (amplitude, length_um, l1_uniform, l1_fitted) over those rings."""
    img = np.asarray(image, np.float64)
    img = img / img.sum()
    nx, ny = img.shape
    x = lb_x + (np.arange(nx) + 0.5) * pixel
    y = lb_y + (np.arange(ny) + 0.5) * pixel
    X, Y = np.meshgrid(x, y, indexing="ij")
    r = np.hypot(X - cx_um, Y - cy_um).ravel()
    rb = np.floor(r / pixel).astype(np.int64)
    ring = np.bincount(rb, img.ravel())
    flat = img.ravel()
    far = r >= 0.5 * min(cx_um, det_x - cx_um, cy_um, det_y - cy_um)

    def l1(a, l):
        w = edge_weights(a, l, X, Y, det_x, det_y).ravel() if a > 0 else np.ones_like(flat)
        pred = ring[rb] * w / np.maximum(np.bincount(rb, w)[rb], 1e-300)
        return float(np.abs(pred - flat)[far].sum())

    base = l1(0.0, 1.0)
    best = (base, 0.0, 1.0)
    for a in np.arange(0.05, 0.95, 0.05):
        for l in (5, 8, 12, 16, 20, 25, 30, 36, 43, 50, 60, 75, 90):
            v = l1(a, l)
            if v < best[0]:
                best = (v, float(a), float(l))
    if best[1] > 0:
        # local refinement around the grid's best point
        _, a0, l0 = best
        for a in np.linspace(max(a0 - 0.05, 0.01), min(a0 + 0.05, 0.95), 11):
            for l in np.linspace(0.8 * l0, 1.2 * l0, 9):
                v = l1(a, l)
                if v < best[0]:
                    best = (v, float(a), float(l))
    return best[1], best[2], base, best[0]


class Surrogate:
    """One surrogate network with its optimizer state on a GPU."""

    def __init__(self, device: int = 0, hidden: int = 256, radial_bins: int = 96, radial_max_um: float = 400.0,
                 batch: int = 8192, lr: float = 1e-3, radial_weight: float = 1.0, seed: int = 0x5347fd2,
                 lateral_um: float = 50.0, depth_margin_um: float = 1.0):
        lib = load()
        self._lib = lib
        c = SgConfig()
        lib.fd2_sg_default_config(ctypes.byref(c))
        c.device, c.hidden, c.radial_bins, c.radial_max_um = device, hidden, radial_bins, radial_max_um
        c.batch, c.lr, c.radial_weight, c.seed, c.lateral_um = batch, lr, radial_weight, seed, lateral_um
        c.depth_margin_um = depth_margin_um
        self.config = c
        self.radial_bins = radial_bins
        self.radial_max_um = radial_max_um
        self._h = ctypes.c_void_p()
        check(lib.fd2_sg_create(ctypes.byref(c), ctypes.byref(self._h)), "fd2_sg_create")

    def close(self):
        if self._h:
            self._lib.fd2_sg_destroy(self._h)
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

    def _check(self, st, where):
        if st != _lib.OK:
            raise _lib.Fd2Error(st, where, self._lib.fd2_sg_last_error(self._h).decode(errors="replace"))

    def set_data(self, feats, photons, detected, radial, n_val: int = 0):
        f = np.ascontiguousarray(feats, np.float32)
        p = np.ascontiguousarray(photons, np.int32)
        d = np.ascontiguousarray(detected, np.int32)
        r = np.ascontiguousarray(radial, np.uint32)
        self._check(self._lib.fd2_sg_set_data(self._h, ptr(f), ptr(p), ptr(d), ptr(r), len(p), n_val), "set_data")

    def train(self, steps: int):
        tl, vl = ctypes.c_float(), ctypes.c_float()
        self._check(self._lib.fd2_sg_train(self._h, steps, ctypes.byref(tl), ctypes.byref(vl)), "train")
        return float(tl.value), float(vl.value)

    def set_lr(self, lr: float):
        self._check(self._lib.fd2_sg_set_lr(self._h, lr), "set_lr")

    def eval(self) -> dict:
        a, b, c = ctypes.c_float(), ctypes.c_float(), ctypes.c_float()
        self._check(self._lib.fd2_sg_eval(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)), "eval")
        return {"loss": a.value, "det_loss": b.value, "radial_loss": c.value}

    def num_params(self) -> int:
        return int(self._lib.fd2_sg_num_params(self._h))

    def params(self) -> np.ndarray:
        out = np.zeros(self.num_params(), np.float32)
        self._check(self._lib.fd2_sg_get_params(self._h, ptr(out), out.size), "get_params")
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        self._check(self._lib.fd2_sg_set_params(self._h, ptr(p), p.size), "set_params")

    def hull(self):
        h = SgHull()
        self._check(self._lib.fd2_sg_get_hull(self._h, ctypes.byref(h)), "get_hull")
        return np.array(h.lo[:], np.float32), np.array(h.hi[:], np.float32)

    def set_hull(self, lo, hi):
        h = SgHull()
        h.lo[:] = [float(v) for v in lo]
        h.hi[:] = [float(v) for v in hi]
        self._check(self._lib.fd2_sg_set_hull(self._h, ctypes.byref(h)), "set_hull")

    def set_edge(self, amplitude: float, length_um: float):
        """Edge survival of the in-loop sampler's azimuths (see fit_edge)."""
        self._check(self._lib.fd2_sg_set_edge(self._h, float(amplitude), float(length_um)), "set_edge")

    def edge(self):
        a, l = ctypes.c_float(), ctypes.c_float()
        self._check(self._lib.fd2_sg_get_edge(self._h, ctypes.byref(a), ctypes.byref(l)), "get_edge")
        return float(a.value), float(l.value)

    def save(self, path: str):
        self._check(self._lib.fd2_sg_save(self._h, path.encode()), "save")

    def load(self, path: str):
        self._check(self._lib.fd2_sg_load(self._h, path.encode()), "load")

    def loss_grad(self, feats, photons, detected, radial):
        f = np.ascontiguousarray(feats, np.float32)
        p = np.ascontiguousarray(photons, np.int32)
        d = np.ascontiguousarray(detected, np.int32)
        r = np.ascontiguousarray(radial, np.uint32)
        loss = ctypes.c_float()
        g = np.zeros(self.num_params(), np.float32)
        self._check(self._lib.fd2_sg_loss_grad(self._h, ptr(f), ptr(p), ptr(d), ptr(r), len(p), ctypes.byref(loss),
                                               ptr(g)), "loss_grad")
        return float(loss.value), g

    def predict(self, feats) -> np.ndarray:
        f = np.ascontiguousarray(feats, np.float32)
        out = np.zeros((len(f), N_OUTPUTS), np.float32)
        self._check(self._lib.fd2_sg_predict(self._h, ptr(f), len(f), ptr(out)), "predict")
        return out

    def run(self, transport: OpticalTransport, audit_fraction: float = 0.01) -> dict:
        st = SgStats()
        self._check(self._lib.fd2_sg_run(self._h, transport.handle, audit_fraction, ctypes.byref(st)), "run")
        return st.as_dict()
