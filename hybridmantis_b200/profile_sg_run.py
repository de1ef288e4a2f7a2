"""Surrogate-in-the-loop run for profilers (ncu): ``python -m hybridmantis_b200.profile_sg_run``.

Loads a surrogate network, submits a seeded synthetic EDE stream of one
configuration to a transport context and runs ``fd2_sg_run`` on it
``--runs`` times (reset tallies between runs), printing the last run's
statistics (time of the network and sampling, of the Monte Carlo of the
events outside the hull, and of the audit).
"""
import argparse
import json
import os

from . import fastdetect2 as fd
from . import surrogate as sgm


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--model", default=os.path.join(os.path.dirname(__file__), "data", "surrogate_c4.fd2sg"))
    ap.add_argument("--config", type=int, default=4)
    ap.add_argument("--xrays", type=int, default=200_000)
    ap.add_argument("--seed", type=int, default=4242)
    ap.add_argument("--runs", type=int, default=2)
    ap.add_argument("--audit", type=float, default=0.01)
    a = ap.parse_args()
    es = fd.synth_events(a.config, a.xrays, a.seed)
    with sgm.Surrogate() as s:
        s.load(a.model)
        with fd.OpticalTransport(es.params, seed=a.seed + 1) as t:
            t.submit(es)
            st = None
            for _ in range(a.runs):
                t.reset_tallies()
                st = s.run(t, a.audit)
    print(json.dumps({k: st[k] for k in ("events", "surrogate_events", "mc_events", "audit_events", "sg_ms", "mc_ms",
                                         "audit_ms", "total_ms")}))


if __name__ == "__main__":
    main()
