"""Train the surrogate on Monte Carlo labels: ``python -m hybridmantis_b200.train_surrogate``.

Defaults follow the surrogate-training workload: 2,000,000 points over
detector geometries drawn from the batched workload's ranges (thickness
100-600 um, column radius 2.5-7.5 um, roughness 0-0.5, top reflectivity 0-1,
bulk absorption 1e-5..1e-3 /um), each point a deposition at depth U(0, H)
with energy U(0.05, 80) keV labelled by 10,000 Monte Carlo photons
(detected fraction and a 96-bin radial histogram to 400 um, quadratic bin
edges); MLP 8-256-256-256-25, BF16 GEMMs with FP32 accumulation, Adam with
a cosine step-size decay, batch 8,192, 5 % held out.

``--focus CONFIG`` continues the training of ``--init`` on depositions in the
detector of one benchmark configuration only (the detector a simulation
campaign uses), with the routing hull narrowed to it.

``--edge-config CONFIG`` fits the in-loop sampler's edge survival
(surrogate.fit_edge) to a Monte Carlo PRF image of ``--edge-xrays`` x-rays of
that configuration and saves it with the network; with ``--steps 0`` and
``--init`` only that fit is made.

Prints one JSON line with the losses and timings; writes the network with
``--out``.
"""
import math
import argparse
import json
import time

import numpy as np

from . import fastdetect2 as fd
from . import surrogate as sgm


def fit_edge_from_mc(s, config: int, xrays: int, seed: int, device: int):
    """Fit and set the surrogate's edge survival from a Monte Carlo PRF image
    of `xrays` x-rays of `config` (no fit for config < 0)."""
    if config < 0:
        return None
    es = fd.synth_events(config, xrays, seed + 7)
    with fd.OpticalTransport(es.params, device=device, seed=seed + 8) as t:
        t.submit(es)
        t.run_sync()
        img = t.prf()
    p = es.params
    amp, length, l1_uniform, l1_fit = sgm.fit_edge(img, float(np.mean(es.x_um)), float(np.mean(es.y_um)), p.det_x,
                                                   p.det_y, p.lb_x, p.lb_y, p.pixel)
    if amp > 0:
        s.set_edge(amp, length)
    return {"config": config, "xrays": xrays, "amplitude": amp, "length_um": length, "ring_l1_uniform": l1_uniform,
            "ring_l1_fitted": l1_fit}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--geometries", type=int, default=1024)
    ap.add_argument("--points", type=int, default=2_000_000)
    ap.add_argument("--photons", type=int, default=10_000)
    ap.add_argument("--steps", type=int, default=6000)
    ap.add_argument("--batch", type=int, default=8192)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--val", type=float, default=0.05)
    ap.add_argument("--seed", type=int, default=20240)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--lr-min", type=float, default=1e-5)
    ap.add_argument("--init", default="")
    ap.add_argument("--focus", type=int, default=-1)
    ap.add_argument("--radial-weight", type=float, default=1.0,
                    help="weight of the radial cross-entropy against the detection BCE in the loss")
    ap.add_argument("--out", default="")
    ap.add_argument("--edge-config", type=int, default=-1)
    ap.add_argument("--edge-xrays", type=int, default=200_000)
    a = ap.parse_args()
    if a.steps == 0 and a.init:
        with sgm.Surrogate(device=a.device) as s:
            s.load(a.init)
            edge = fit_edge_from_mc(s, a.edge_config, a.edge_xrays, a.seed, a.device)
            if a.out:
                s.save(a.out)
        print(json.dumps({"edge": edge}))
        return
    t0 = time.perf_counter()
    if a.focus >= 0:
        geoms = [fd.params_to_geometry(fd.synth_events(a.focus, 1, 1).params)]
    else:
        geoms = sgm.sample_geometries(a.geometries, seed=a.seed)
    per = max(1, a.points // len(geoms))
    f, ph, det, rad = sgm.label_points(geoms, per, a.photons, seed=a.seed + 1, device=a.device,
                                       energy_kev=(0.05, 80.0))
    t_label = time.perf_counter() - t0
    perm = np.random.default_rng(a.seed + 2).permutation(len(f))
    f, ph, det, rad = f[perm], ph[perm], det[perm], rad[perm]
    n_val = int(a.val * len(f))
    with sgm.Surrogate(device=a.device, batch=a.batch, lr=a.lr, seed=a.seed + 3, radial_weight=a.radial_weight) as s:
        if a.init:
            s.load(a.init)
        s.set_data(f, ph, det, rad, n_val=n_val)
        before = s.eval()
        t1 = time.perf_counter()
        curve = []
        done = 0
        while done < a.steps:
            k = min(250, a.steps - done)
            frac = (done + 0.5 * k) / a.steps
            s.set_lr(a.lr_min + 0.5 * (a.lr - a.lr_min) * (1.0 + math.cos(math.pi * frac)))
            tl, vl = s.train(k)
            done += k
            curve.append({"step": done, "train": tl, "val": vl})
        t_train = time.perf_counter() - t1
        after = s.eval()
        edge = fit_edge_from_mc(s, a.edge_config, a.edge_xrays, a.seed, a.device)
        if a.out:
            s.save(a.out)
    print(json.dumps({"points": len(f), "photons_per_point": a.photons, "geometries": a.geometries,
                      "label_s": t_label, "label_photons_per_s": float(np.sum(ph)) / t_label,
                      "train_s": t_train, "steps": a.steps, "batch": a.batch,
                      "val_before": before, "val_after": after, "curve": curve, "edge": edge}))


if __name__ == "__main__":
    main()
