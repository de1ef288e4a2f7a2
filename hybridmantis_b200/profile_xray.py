"""Small x-ray front-end run for profilers (ncu): ``python -m hybridmantis_b200.profile_xray``.

Runs ``--xrays`` histories of config 1's spectrum (Triangular(20, 40, 70)
keV pencil beam) through the GPU x-ray front end on config 1's detector,
``--runs`` times, and prints the per-run kernel times and statistics.
"""
import argparse
import json

from . import fastdetect2 as fd
from . import xray


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--xrays", type=int, default=100000)
    ap.add_argument("--runs", type=int, default=2)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--local", type=float, default=1000.0, help="electron_local_ev")
    a = ap.parse_args()
    p = fd.synth_events(1, 1, a.seed).params
    src = xray.triangular_spectrum(20e3, 40e3, 70e3, center_cm=(p.det_x * 0.5e-4, p.det_y * 0.5e-4, 1.0))
    with xray.XrayFrontEnd(det_x_um=p.det_x, det_y_um=p.det_y, det_height_um=p.det_height, seed=a.seed,
                           electron_local_ev=a.local) as fe:
        runs = []
        for _ in range(a.runs):
            fe.run(src, a.xrays)
            t = fe.timing()
            t["xrays_per_s"] = a.xrays / ((t["transport_ms"] + t["compact_ms"]) * 1e-3)
            runs.append(t)
        st = fe.stats()
    print(json.dumps({"xrays": a.xrays, "runs": runs, "edes_per_xray": st["edes"] / (a.xrays * a.runs),
                      "electron_steps_per_xray": st["electron_steps"] / (a.xrays * a.runs)}))


if __name__ == "__main__":
    main()
