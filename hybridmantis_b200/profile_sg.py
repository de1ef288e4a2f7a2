"""Surrogate forward pass for profilers (ncu): ``python -m hybridmantis_b200.profile_sg``.

Runs the network's forward pass (fd2_sg_predict: input normalisation and the
four GEMMs) on ``--rows`` seeded random inputs ``--runs`` times, with random
weights of the full-size network, and prints the host time per pass.
FD2_SG_GEMM in the environment selects an earlier form of the GEMMs: ``mma``
(mma.sync), ``tc1`` (one tcgen05 tile at a time), ``cpasync`` (pipelined,
operands by cp.async), ``noswizzle`` (TMA boxes of 16-byte columns instead of
128-byte swizzled rows), ``nostore`` (per-lane output stores instead of TMA
stores).
"""
import argparse
import json
import os
import time

import numpy as np

from . import surrogate as sgm


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--rows", type=int, default=65536)
    ap.add_argument("--runs", type=int, default=6)
    ap.add_argument("--hidden", type=int, default=256)
    ap.add_argument("--train", type=int, default=0,
                    help="instead of forward passes: this many training steps (forward, loss, the backward "
                         "GEMMs, Adam) on --rows random labelled points, batch 8192")
    a = ap.parse_args()
    if a.train:
        rng = np.random.default_rng(2)
        n = a.rows
        f = rng.uniform(0, 1, (n, 8)).astype(np.float32)
        ph = rng.integers(500, 3000, n).astype(np.int32)
        det = (ph * rng.uniform(0.1, 0.6, n)).astype(np.int32)
        rad = rng.integers(0, 40, (n, 97)).astype(np.uint32)
        with sgm.Surrogate(hidden=a.hidden, batch=8192) as s:
            s.set_data(f, ph, det, rad, n_val=0)
            ms = []
            for _ in range(a.runs):
                t0 = time.perf_counter()
                tl, _ = s.train(a.train)
                ms.append((time.perf_counter() - t0) * 1e3 / a.train)
        print(json.dumps({"gemm": os.environ.get("FD2_SG_GEMM", "tc"), "train_step_ms": ms, "loss": tl}))
        return
    rng = np.random.default_rng(1)
    with sgm.Surrogate(hidden=a.hidden, batch=a.rows) as s:
        s.set_params(rng.normal(0, 0.05, s.num_params()).astype(np.float32))
        s.set_hull(np.zeros(8, np.float32), np.ones(8, np.float32))
        f = rng.uniform(0, 1, (a.rows, 8)).astype(np.float32)
        ms = []
        for _ in range(a.runs):
            t0 = time.perf_counter()
            out = s.predict(f)
            ms.append((time.perf_counter() - t0) * 1e3)
    print(json.dumps({"gemm": os.environ.get("FD2_SG_GEMM", "tc"), "rows": a.rows, "predict_ms": ms,
                      "mean_abs_output": float(np.abs(out).mean())}))


if __name__ == "__main__":
    main()
