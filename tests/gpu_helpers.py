"""Shared setup of the GPU parity tests (events, oracle geometry, reports)."""
import json
import os

import numpy as np

import hybridmantis_b200 as hb
from oracle import pyoracle as po


def c0_events(n, seed=3):
    """Config-0 events (25 keV pencil beam on 150 um) with Gaussian photon
    counts N ~ round(Normal(1350, sqrt(1350))) fixed on the host, so the
    oracle and the GPU transport the same photons."""
    es = hb.synth_events(0, n, seed)
    rng = np.random.default_rng(seed)
    N = np.maximum(0, np.rint(rng.normal(1350.0, np.sqrt(1350.0), n))).astype(np.int32)
    return es, N


def oracle_geometry(p) -> po.Geometry:
    return po.Geometry(xdet=p.det_x, ydet=p.det_y, H=p.det_height, R=p.radius, n_col=p.n_col, n_gap=p.n_gap,
                       top_absfrac=p.top_absfrac, bulk_abs=p.bulk_abs, beta=p.beta, d_min=p.d_min, d_max=p.d_max,
                       lb_x=p.lb_x, lb_y=p.lb_y, ub_x=p.ub_x, ub_y=p.ub_y, sensor_refl=p.sensor_refl,
                       pixel=p.pixel)


def run_oracle_on(es, N, params=None, seed_input=271828182, records=False):
    p = params or es.params
    return po.run_oracle(oracle_geometry(p), es.x_um.astype(np.float64), es.y_um.astype(np.float64),
                         es.z_um.astype(np.float64), es.hist, N, seed_input=seed_input,
                         prim_size=p.num_hist, records=records)


def compare_replay(N, gpu, orc):
    """Per-event comparison of per-photon records.  An event is divergent
    from its first photon whose fate, pixel, RANECU state or step count
    differs (its RNG stream is shared by the later photons)."""
    first = np.concatenate([[0], np.cumsum(N)])
    same = ((gpu["fate"] == orc.fate) & (gpu["pix"] == orc.pix).all(1) & (gpu["seeds"] == orc.seeds).all(1)
            & (gpu["steps"] == orc.steps))
    fate_same = (gpu["fate"] == orc.fate) & (gpu["pix"] == orc.pix).all(1)
    div_events = 0
    photons_before = 0
    first_div = []
    for e in range(len(N)):
        s = same[first[e]:first[e + 1]]
        if s.all():
            photons_before += len(s)
        else:
            div_events += 1
            k = int(np.argmin(s))
            photons_before += k
            first_div.append((e, k))
    return {"events": int(len(N)), "divergent_events": int(div_events), "photons": int(N.sum()),
            "photons_matched_before_divergence": int(photons_before),
            "photon_fate_pixel_agreement": float(fate_same.mean()) if len(fate_same) else 1.0,
            "first_divergences": first_div[:10]}


def report(name, payload):
    d = os.environ.get("FD2_REPORT_DIR")
    if not d:
        return
    os.makedirs(d, exist_ok=True)
    with open(os.path.join(d, f"{name}.json"), "w") as f:
        json.dump(payload, f, indent=1, default=lambda o: o.tolist() if hasattr(o, "tolist") else str(o))
