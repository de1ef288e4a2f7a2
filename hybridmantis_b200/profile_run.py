"""Small transport run for profilers (ncu): ``python -m hybridmantis_b200.profile_run``.

Transports a seeded synthetic EDE stream ``--runs`` times through the C ABI
and prints the per-run transport time and photon rate.
"""
import argparse
import json

import numpy as np

from . import fastdetect2 as fd


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", type=int, default=1)
    ap.add_argument("--xrays", type=int, default=2000)
    ap.add_argument("--runs", type=int, default=2)
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--block", type=int, default=0)
    ap.add_argument("--ctas", type=int, default=0)
    ap.add_argument("--chunk", type=int, default=0)
    ap.add_argument("--refill", type=int, default=0)
    ap.add_argument("--window", type=int, default=-1)
    ap.add_argument("--fresnel", type=int, default=0)
    ap.add_argument("--grid", type=int, default=0, help="1 / 2: explicit square / hexagonal column lattice")
    ap.add_argument("--gap", type=float, default=0.5, help="lattice gap between columns (um)")
    ap.add_argument("--tally-mode", type=int, default=0,
                    help="0: per-lane L2 reductions; 1: warp-aggregated, shared-memory privatised tallies")
    a = ap.parse_args()
    es = fd.synth_events(a.config, a.xrays, a.seed)
    x, y, z = es.to_cm()
    with fd.OpticalTransport(es.params, block_size=a.block, ctas_per_sm=a.ctas, chunk=a.chunk, refill=a.refill,
                             prf_window=a.window, fresnel_batch=a.fresnel, column_grid=a.grid,
                             grid_gap_um=a.gap, tally_mode=a.tally_mode) as t:
        t.submit_events(x, y, z, es.e_ev.astype(np.float64), es.hist)
        out = []
        for _ in range(a.runs):
            t.run_sync()
            tm = t.timing()
            out.append({"transport_ms": tm["transport_ms"], "photons": tm["photons"],
                        "photons_per_s": tm["photons"] / (tm["transport_ms"] * 1e-3)})
        c = t.counters()
        st = t.phs_stats()
        n = max(c["generated"], 1)
        fates = {k: c[k] / n for k in ("detected", "abs_top", "abs_bulk", "lost", "capped")}
        print(json.dumps({"events": es.n, "runs": out, "fates": fates, "phs_mean": st["mean"], "swank": st["swank"],
                          "launch": {k: tm[k] for k in
                                                                 ("grid", "block", "chunk", "refill", "prf_window",
                                                                                  "fresnel_batch")}}))


if __name__ == "__main__":
    main()
