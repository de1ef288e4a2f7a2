"""Generates the golden fixtures of tests/golden from the reference.

Run in a tree where the reference is present (default /root/reference) and
oracle/_ref has been built (make -C oracle):

    python tests/golden/make_golden.py [REFERENCE_ROOT]

Writes
  example_hybridMANTIS_input.in   the reference example's 24-value input file
  example_detected.txt            its PHS output (detected_*.dat, 140 rows)
  example_myimage.npz             its PRF output (myimage_*.dat) as integers
                                  value * 1e4 in file order, plus the name
  ranecu_kat.json                 init_PRNG seeds and first uniforms of several
                                  RANECU streams, from the reference's C code
  ref_small_runs.npz              per-photon fates, RANECU states and step
                                  counts of the reference's C transport on
                                  small seeded cases (three geometries)
"""
import json
import os
import shutil
import sys
import zlib

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import pyoracle as po  # noqa: E402

SMALL_CASES = {
    "c0": dict(),
    "sensor": dict(sensor_refl=0.3, beta=0.35, top_absfrac=0.0),
    "pix9": dict(pixel=9, ub_x=450.0, ub_y=450.0, xdet=909.0, ydet=909.0, H=300.0, R=4.0, bulk_abs=1e-3),
}


def small_case(name, kw):
    g = po.Geometry(**kw)
    rng = np.random.default_rng(zlib.crc32(name.encode()))
    n = 6
    x = g.xdet / 2 + rng.normal(0, 3, n)
    y = g.ydet / 2 + rng.normal(0, 3, n)
    z = g.H / 2 - np.minimum(rng.exponential(60, n), 0.99 * g.H)
    hist = np.arange(1, n + 1, dtype=np.int32)
    N = rng.integers(50, 250, n).astype(np.int32)
    return g, x, y, z, hist, N


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    ex = os.path.join(ref, "example")
    shutil.copyfile(os.path.join(ex, "hybridMANTIS_input.in"), os.path.join(HERE, "example_hybridMANTIS_input.in"))
    outs = os.path.join(ex, "output_files")
    det = [f for f in os.listdir(outs) if f.startswith("detected_")][0]
    img = [f for f in os.listdir(outs) if f.startswith("myimage_")][0]
    shutil.copyfile(os.path.join(outs, det), os.path.join(HERE, "example_detected.txt"))
    vals = [line.strip() for line in open(os.path.join(outs, img))]
    nums = np.array([int(round(float(v) * 1e4)) for v in vals if v], dtype=np.int64)
    blank = np.array([i for i, v in enumerate(vals) if not v], dtype=np.int64)
    np.savez_compressed(os.path.join(HERE, "example_myimage.npz"), values_e4=nums, blank_lines=blank,
                        n_lines=len(vals), name=img, detected_name=det)

    kat = {"seed_input": 271828182, "streams": []}
    for idx in [0, 1, 2, 17, 12345, 2303999]:
        s = po.init_prng(idx, ref=True)
        u, after = po.ranecu(s, 10, ref=True)
        kat["streams"].append({"index": idx, "seeds": [int(v) for v in s], "uniforms": [float(v) for v in u],
                               "seeds_after_10": [int(v) for v in after]})
    with open(os.path.join(HERE, "ranecu_kat.json"), "w") as f:
        json.dump(kat, f, indent=1)

    arrays = {}
    for name, kw in SMALL_CASES.items():
        g, x, y, z, hist, N = small_case(name, kw)
        r = po.run_ref(g, x, y, z, hist, N, seed_input=12345, base=7)
        assert r.status == 0
        arrays.update({f"{name}_geom": np.array(g.floats() + [g.pixel], np.float64), f"{name}_x": x,
                       f"{name}_y": y, f"{name}_z": z, f"{name}_hist": hist, f"{name}_N": N,
                       f"{name}_fate": r.fate, f"{name}_seeds": r.seeds, f"{name}_steps": r.steps,
                       f"{name}_counters": r.counters, f"{name}_per_primary": r.per_primary,
                       f"{name}_image_nz": np.argwhere(r.image > 0).astype(np.int32),
                       f"{name}_image_vals": r.image[r.image > 0]})
    np.savez_compressed(os.path.join(HERE, "ref_small_runs.npz"), **arrays)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
