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


def run_oracle_parallel(es, N, params=None, seed_input=271828182, workers=None):
    """The oracle over contiguous event slices on host threads (ctypes
    releases the GIL during the call).  Event e keeps its own RANECU stream
    init_PRNG(base + e), so the summed tallies equal one call over all events
    (tests/test_oracle_cpu.py checks this)."""
    from concurrent.futures import ThreadPoolExecutor

    p = params or es.params
    g = oracle_geometry(p)
    n = es.n
    workers = workers or max(1, min(len(os.sched_getaffinity(0)), 32))
    N = np.asarray(N, np.int32)
    # equal photon shares per slice
    cum = np.concatenate([[0], np.cumsum(N, dtype=np.int64)])
    cuts = np.searchsorted(cum, np.linspace(0, cum[-1], workers + 1)).clip(0, n)
    cuts[0], cuts[-1] = 0, n
    cuts = np.unique(cuts)

    def one(a, b):
        return po.run_oracle(g, es.x_um[a:b].astype(np.float64), es.y_um[a:b].astype(np.float64),
                             es.z_um[a:b].astype(np.float64), es.hist[a:b], N[a:b], seed_input=seed_input, base=int(a),
                             prim_size=p.num_hist, records=False)

    with ThreadPoolExecutor(len(cuts) - 1) as ex:
        parts = list(ex.map(lambda ab: one(*ab), zip(cuts[:-1], cuts[1:])))
    out = parts[0]
    for r in parts[1:]:
        out.image += r.image
        out.per_primary += r.per_primary
        out.counters += r.counters
    return out


def given_counts(es, seed):
    """Poisson(E * yield) photon counts fixed on the host."""
    rng = np.random.default_rng(seed)
    return rng.poisson(es.e_ev.astype(np.float64) * es.params.yield_).astype(np.int32)


def geometry_params(es, g):
    """Params of geometry g of a batched stream (the base params with the
    geometry's fields)."""
    p = hb.default_params()
    for f, _ in p._fields_:
        setattr(p, f, getattr(es.params, f))
    geo = es.geometries[g]
    for f, _ in geo._fields_:
        if f != "reserved" and hasattr(p, f):
            setattr(p, f, getattr(geo, f))
    return p
