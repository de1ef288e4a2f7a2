"""Surrogate in the loop against the plain Monte Carlo on the same events:
``python -m hybridmantis_b200.eval_surrogate --model FILE``.

Transports one seeded synthetic stream twice through the same context
settings -- once with fd2_run (Monte Carlo), once with fd2_sg_run -- and
prints one JSON line: x-rays/s of both, PHS mean and Swank factor of both,
the L1 distance of their normalised radial PRF profiles and of their
normalised PRF images, and the audit statistics.  Default stream: 1,000,000
x-rays, triangular 20-70 keV, 500 um CsI, R = 5 um, clusters as the
benchmark workload (the surrogate-in-the-loop configuration).
"""
import argparse
import json
import time

import numpy as np

from . import fastdetect2 as fd
from . import surrogate as sgm


def _moments(prim):
    c = np.asarray(prim, np.float64)
    c = c[c > 0]
    m1, m2 = c.mean(), (c * c).mean()
    return float(m1), float(m1 * m1 / m2)


def _radial(img, cx, cy, edges):
    img = np.asarray(img, np.float64)
    ii, jj = np.meshgrid(np.arange(img.shape[0]) + 0.5, np.arange(img.shape[1]) + 0.5, indexing="ij")
    r = np.hypot(ii - cx, jj - cy)
    h = np.histogram(r.ravel(), bins=edges, weights=img.ravel())[0]
    return h / max(h.sum(), 1.0)


def _l1_by_radius(a, b, cx, cy, bands):
    """Contributions to the L1 distance of two normalised images from pixels
    in radial bands around (cx, cy) (pixel centres)."""
    a = np.asarray(a, np.float64) / max(np.sum(a), 1.0)
    b = np.asarray(b, np.float64) / max(np.sum(b), 1.0)
    ii, jj = np.meshgrid(np.arange(a.shape[0]) + 0.5, np.arange(a.shape[1]) + 0.5, indexing="ij")
    r = np.hypot(ii - cx, jj - cy)
    d = np.abs(a - b)
    return [float(d[(r >= lo) & (r < hi)].sum()) for lo, hi in zip(bands[:-1], bands[1:])]


def evaluate(model: str, config: int = 4, xrays: int = 1_000_000, seed: int = 4242, audit: float = 0.01,
             device: int = 0, repeats: int = 2, noise_floor: bool = False, frontend: bool = False,
             lateral_um: float = 50.0) -> dict:
    """With ``frontend`` the events come from the GPU x-ray front end (the
    configuration's detector and Triangular(20, 40, 70) keV pencil beam at its
    centre) instead of the synthetic cluster generator, handed to each
    context on the device."""
    fe = None
    if frontend:
        from . import xray
        es = fd.synth_events(config, 1, seed)
        p = es.params
        p.num_hist = xrays
        fe = xray.XrayFrontEnd(det_x_um=p.det_x, det_y_um=p.det_y, det_height_um=p.det_height, seed=seed,
                               device=device)
        fe.run(xray.triangular_spectrum(20e3, 40e3, 70e3, center_cm=(p.det_x * 0.5e-4, p.det_y * 0.5e-4, 1.0)),
               xrays)
        out = {"config": config, "xrays": xrays, "events": fe.num_edes(), "events_from": "x-ray front end"}
    else:
        es = fd.synth_events(config, xrays, seed)
        out = {"config": config, "xrays": es.params.num_hist, "events": es.n}
    res = {}
    out["lateral_um"] = lateral_um
    with sgm.Surrogate(device=device, lateral_um=lateral_um) as s:
        s.load(model)
        for mode in ("mc", "mc2", "sg"):
            if mode == "mc2" and not noise_floor:
                continue
            # mc2: the Monte Carlo again with other random streams (the
            # noise floor of the comparison)
            with fd.OpticalTransport(es.params, device=device, seed=seed + (2 if mode == "mc2" else 1)) as t:
                if fe is not None:
                    fe.submit(t)
                else:
                    t.submit(es)
                # warm-up run, then timed runs on reset tallies
                if mode != "sg":
                    t.run_sync()
                else:
                    s.run(t, audit)
                times = []
                stats = None
                for _ in range(repeats):
                    t.reset_tallies()
                    t0 = time.perf_counter()
                    if mode != "sg":
                        t.run_sync()
                    else:
                        stats = s.run(t, audit)
                    times.append(time.perf_counter() - t0)
                prim = t.detected_per_primary()
                img = t.prf().astype(np.float64)
                c = t.counters()
            mean, swank = _moments(prim)
            res[mode] = {"seconds": min(times), "xrays_per_s": out["xrays"] / min(times), "phs_mean": mean,
                         "swank": swank, "detected": c["detected"], "image": img, "stats": stats}
    edges = np.array([0, 1, 2, 3, 4, 6, 8, 11, 15, 20, 30, 45, 70, 110, 170, 260, 400])
    if fe is not None:
        cx, cy = 0.5 * es.params.det_x - es.params.lb_x, 0.5 * es.params.det_y - es.params.lb_y
        fe.close()
    else:
        cx = float(np.mean(es.x_um)) - es.params.lb_x
        cy = float(np.mean(es.y_um)) - es.params.lb_y
    rm, rs = _radial(res["mc"]["image"], cx, cy, edges), _radial(res["sg"]["image"], cx, cy, edges)
    im, isg = res["mc"]["image"], res["sg"]["image"]
    out.update({
        "mc_xrays_per_s": res["mc"]["xrays_per_s"], "sg_xrays_per_s": res["sg"]["xrays_per_s"],
        "speedup": res["sg"]["xrays_per_s"] / res["mc"]["xrays_per_s"],
        "mc_seconds": res["mc"]["seconds"], "sg_seconds": res["sg"]["seconds"],
        "phs_mean": [res["mc"]["phs_mean"], res["sg"]["phs_mean"]],
        "swank": [res["mc"]["swank"], res["sg"]["swank"]],
        "swank_diff": res["sg"]["swank"] - res["mc"]["swank"],
        "radial_prf_l1": float(np.abs(rm - rs).sum()),
        "radial_profile": {"edges_um": edges.tolist(), "mc": rm.tolist(), "sg": rs.tolist()},
        "prf_image_l1": float(np.abs(im / im.sum() - isg / isg.sum()).sum()),
        "prf_image_l1_by_radius": {"bands_um": [0, 3, 6, 10, 20, 50, 100, 1000],
                                   "sg_vs_mc": _l1_by_radius(isg, im, cx, cy, [0, 3, 6, 10, 20, 50, 100, 1000])},
        "detected": [res["mc"]["detected"], res["sg"]["detected"]],
        "sg_stats": res["sg"]["stats"],
    })
    if noise_floor:
        # the same two comparisons between two Monte Carlo runs of the same
        # events with different random streams
        i2 = res["mc2"]["image"]
        r2 = _radial(i2, cx, cy, edges)
        out["mc_vs_mc"] = {"radial_prf_l1": float(np.abs(rm - r2).sum()),
                           "prf_image_l1": float(np.abs(im / im.sum() - i2 / i2.sum()).sum()),
                           "prf_image_l1_by_radius": _l1_by_radius(i2, im, cx, cy, [0, 3, 6, 10, 20, 50, 100, 1000]),
                           "phs_mean": res["mc2"]["phs_mean"], "swank": res["mc2"]["swank"]}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--model", required=True)
    ap.add_argument("--config", type=int, default=4)
    ap.add_argument("--xrays", type=int, default=1_000_000)
    ap.add_argument("--seed", type=int, default=4242)
    ap.add_argument("--audit", type=float, default=0.01)
    ap.add_argument("--noise-floor", action="store_true")
    ap.add_argument("--xray-frontend", action="store_true", help="events from the GPU x-ray front end")
    ap.add_argument("--lateral", type=float, default=50.0,
                    help="depositions within this distance (um) of the detector centre go to the network")
    a = ap.parse_args()
    print(json.dumps(evaluate(a.model, a.config, a.xrays, a.seed, a.audit, noise_floor=a.noise_floor,
                              frontend=a.xray_frontend, lateral_um=a.lateral)))


if __name__ == "__main__":
    main()
