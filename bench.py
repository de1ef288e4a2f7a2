#!/usr/bin/env python
"""Benchmark: optical photons/s of the fastDETECT2 transport on B200.

One step = one transport pass over the synthetic energy-deposition stream of
benchmark configuration 1 (100,000 x-rays, triangular 20-70 keV spectrum,
1 + Poisson(1.5) clusters, 300 um CsI, R = 4 um; ~2.3e8 optical photons),
photon counts ~ Poisson(E * 54/keV) sampled on the GPU each step.

  value   photons/s with the events resident in HBM (CUDA events on the
          library's stream around K steps, L2 flushed between steps)
  e2e     photons/s through the C ABI with host buffers: H2D of the EDE
          buffer (cm / eV / history), transport, D2H of PRF + PHS + stats
  roofline  the transport kernel against the FP32 issue roofline
  cpu_baseline  the reference's own C transport (oracle/_ref) on a bounded
          sample of the same stream and photon counts: all host cores at
          gcc -O2 (the value), one core at -O2 and one core at -O0 (the
          reference's own flags), with the CPU model
  results.parity  the GPU's FP32 tallies on the cpu_baseline sample's
          events and photon counts against the reference C's: fate z-scores,
          PHS mean and Swank z-scores and relative errors, per-bin PRF
          chi-square
  reference_gpu the reference's own CUDA kernel `algo` (oracle/_ref,
          compiled for sm_100a with its own flags) on the same events and
          photon counts, one launch of its 18000 x 128 grid
  surrogate  x-rays/s of the surrogate in the loop (fd2_sg_run, trained
          network in hybridmantis_b200/data) against the plain Monte Carlo on
          the same 1,000,000-x-ray, 500 um stream, with the PHS/Swank and PRF
          errors between the two and the same errors between two Monte Carlo
          runs (the noise floor)
  xray_frontend  x-rays/s of the GPU x-ray front end (EDEs from x-rays by
          FP64 photon + electron transport) on config 1's detector and
          spectrum, alone and chained with the optical transport through the
          device handoff

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
Multi-GPU: one rank per GPU (torchrun); each rank transports its own x-ray
stream (weak scaling), timing is the max over ranks, tallies are merged once
after the timed region with an all-reduce.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "optical photons/s (MC) & x-rays/s (surrogate) at matched PRF/Swank error"
WORKLOAD = ("config 1: 100000 x-rays, triangular 20-70 keV (mode 40), 1+Poisson(1.5) clusters, Dirichlet(1) "
            "energy split, depth Exp(90 um) in 300 um CsI, offsets N(0,5 um), R=4 um, n 1.8/1.0, top refl 0.9, "
            "mu 1e-4/um, beta 0.2, d 0.5-280 um, ideal sensor, PRF 501x501 of 1 um, PHS 1000 bins, 54 photons/keV")

# FP32 operations per call of the reference's building blocks, counted once
# from main/kernel_cuda_c_ver1_0.cu (C branch): each +, -, *, /, sqrt,
# comparison and libm call (sin, cos, tan, log, pow, acos, asin) is one
# operation.  Multiplied by the call frequencies the oracle measures for the
# workload, they give the algorithmic FP32 work per photon.
OPS_PER_CALL = {
    "step": 4,         # algo: termination / trapped tests
    "to_wall": 68,     # dist_to_surface quadratic, plane, bounds, radius + isotropic absorption
    "pullback": 12,    # one iteration of the out-of-column repair loop
    "surface": 10,     # boundary_analysis: top test, crosstalk probability and draw
    "incidence": 18,   # wall normal, cos(theta1), acos, TIR test
    "fresnel": 34,     # asinf refraction angle, Pr and Pt from tan/sin/cos/pow, normalisation
    "reflect": 32,     # trans_dir_cos reflection + renormalisation + 1.57 rad check
    "refract": 38,     # trans_dir_cos refraction + renormalisation
    "crosstalk": 7,    # transmit entry and the new column centre
    "hop": 32,         # transmit hop: distance, position, top/bottom/side tests
    "new_normal": 14,  # one new-column-normal attempt (besides its two RoughSurface calls)
    "rough": 35,       # RoughSurface
    "uniform": 2,      # RANECU int->float scaling (the MLCG steps are integer work)
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", type=int, default=1)
    ap.add_argument("--xrays", type=int, default=0)
    ap.add_argument("--seed", type=int, default=20240)
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-ref-gpu", action="store_true")
    ap.add_argument("--surrogate-model", default=os.path.join(ROOT, "hybridmantis_b200", "data", "surrogate_c4.fd2sg"))
    ap.add_argument("--surrogate-xrays", type=int, default=1_000_000)
    ap.add_argument("--no-surrogate", action="store_true")
    ap.add_argument("--no-frontend", action="store_true")
    return ap.parse_args()


# --------------------------------------------------------------- host CPU

def _cpu_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def _ref_worker(args):
    sys.path.insert(0, ROOT)
    from oracle import pyoracle as po
    geom, x, y, z, hist, nphot, base, prim_size, opt, keep = args
    t0 = time.perf_counter()
    r = po.run_ref(geom, x, y, z, hist, nphot, seed_input=271828182, base=base, prim_size=prim_size,
                   records=False, opt=opt)
    dt = time.perf_counter() - t0
    tallies = (r.image, r.per_primary, r.counters) if keep else None
    return dt, int(r.counters[0]), tallies


def _oracle_geometry(p):
    from oracle import pyoracle as po
    return po.Geometry(xdet=p.det_x, ydet=p.det_y, H=p.det_height, R=p.radius, n_col=p.n_col, n_gap=p.n_gap,
                       top_absfrac=p.top_absfrac, bulk_abs=p.bulk_abs, beta=p.beta, d_min=p.d_min, d_max=p.d_max,
                       lb_x=p.lb_x, lb_y=p.lb_y, ub_x=p.ub_x, ub_y=p.ub_y, sensor_refl=p.sensor_refl, pixel=p.pixel)


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or "unknown"


class CpuReference:
    """The reference's C transport (oracle/_ref) on the host cores; one
    process per core over contiguous event slices (each event keeps its own
    RANECU stream, so the split does not change results)."""

    def __init__(self, es, nphot):
        import multiprocessing as mp
        from concurrent.futures import ProcessPoolExecutor
        self.es, self.N = es, np.asarray(nphot, np.int32)
        self.g = _oracle_geometry(es.params)
        self.cores = _cpu_cores()
        self.pool = ProcessPoolExecutor(self.cores, mp_context=mp.get_context("spawn"))
        # pilot on one core to size samples
        k = self._events_for(20000, 0)
        dt, ph, _ = self.pool.submit(_ref_worker, self._args(0, k, "O2", False)).result()
        self.rate1 = ph / max(dt, 1e-6)

    def _events_for(self, photons, start):
        c = np.cumsum(self.N[start:])
        return int(min(len(c), np.searchsorted(c, photons) + 1))

    def _args(self, start, count, opt, keep):
        es = self.es
        sl = slice(start, start + count)
        return (self.g, es.x_um[sl].astype(np.float64), es.y_um[sl].astype(np.float64),
                es.z_um[sl].astype(np.float64), es.hist[sl], self.N[sl], start, int(es.params.num_hist), opt, keep)

    def timed_sample(self, seconds, start=0, cores=None, opt="O2", keep=False, rate=None):
        """Transport about `seconds` of work from event `start` on `cores`
        processes; returns photons/s, photons, events, seconds and (keep) the
        summed tallies (image, per-primary counts, counters)."""
        cores = cores or self.cores
        photons = (rate or self.rate1) * cores * seconds
        count = self._events_for(photons, start)
        bounds = np.linspace(start, start + count, cores + 1).astype(int)
        t0 = time.perf_counter()
        futs = [self.pool.submit(_ref_worker, self._args(a, b - a, opt, keep))
                for a, b in zip(bounds[:-1], bounds[1:]) if b > a]
        res = [f.result() for f in futs]
        dt = time.perf_counter() - t0
        ph = sum(r[1] for r in res)
        tallies = None
        if keep:
            img = sum(r[2][0] for r in res)
            prim = sum(r[2][1] for r in res)
            cnt = sum(r[2][2] for r in res)
            tallies = (img, prim, cnt)
        return ph / dt, ph, count, dt, tallies

    def close(self):
        self.pool.shutdown()


def cpu_variants(ref, seconds_one_core=6.0):
    """One core at -O2 and at -O0 (the reference's own compile flags,
    main/compile_ver1_0.sh:10) on the first events of the stream."""
    out = {}
    for opt in ("O2", "O0"):
        rate = ref.rate1 if opt == "O2" else ref.rate1 / 2.5
        r, ph, nev, dt, _ = ref.timed_sample(seconds_one_core, cores=1, opt=opt, rate=rate)
        out[f"1core_{opt}"] = {"value": r, "unit": "photons/s", "cores": 1, "flags": f"gcc -{opt}",
                               "sample": f"first {nev} events ({ph} photons), {dt:.1f} s"}
    return out


# ---------------------------------------------------------- parity stats

def _phs_moments(per_primary):
    c = np.asarray(per_primary, np.float64)
    c = c[c > 0]
    n = len(c)
    m1, m2 = c.mean(), (c * c).mean()
    g = np.array([2 * m1 / m2, -m1 * m1 / (m2 * m2)])
    cov = np.cov(np.vstack([c, c * c]), ddof=1) / n
    return {"n": n, "mean": m1, "se_mean": c.std(ddof=1) / np.sqrt(n), "swank": m1 * m1 / m2,
            "se_swank": float(np.sqrt(g @ cov @ g))}


def _z_binomial(k1, n1, k2, n2):
    p = (k1 + k2) / (n1 + n2)
    return (k1 / n1 - k2 / n2) / np.sqrt(max(p * (1 - p) * (1 / n1 + 1 / n2), 1e-300))


def _chi2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    m = (a + b) > 0
    return float((((a - b) ** 2) / (a + b))[m].sum()), int(m.sum())


def parity_vs_reference(es, nphot, nev, ref_tallies, device, seed):
    """The GPU's FP32 production transport against the reference C on the
    same events (the first `nev` of the stream) and the same photon counts:
    z-scores of the fate fractions, the PHS mean and the Swank factor, and a
    per-bin Poisson chi-square of the PRF (central 41 x 41 one-micron pixels
    around the beam plus ring totals outside them)."""
    import hybridmantis_b200 as hb
    img_r, prim_r, cnt_r = ref_tallies
    N = np.asarray(nphot[:nev], np.int32)
    sub = es.subset(slice(0, nev))
    with hb.OpticalTransport(es.params, device=device, count_mode=hb.COUNT_GIVEN, seed=seed) as t:
        t.submit(sub, nphot=N)
        t.run_sync()
        c = t.counters()
        prim = t.detected_per_primary()
        img = t.prf()
    n = int(N.sum())
    names = ["detected", "abs_top", "abs_bulk", "lost", "outofcol", "theta1"]
    ref = dict(zip(names, [int(v) for v in cnt_r[1:7]]))
    z_f = {k: float(_z_binomial(c[k], n, ref[k], n)) for k in names[:4]}
    g, o = _phs_moments(prim), _phs_moments(prim_r)
    z_mean = (g["mean"] - o["mean"]) / np.hypot(g["se_mean"], o["se_mean"])
    z_swank = (g["swank"] - o["swank"]) / np.hypot(g["se_swank"], o["se_swank"])
    p = es.params
    cx = int(np.floor((np.median(sub.x_um) - p.lb_x) / p.pixel))
    cy = int(np.floor((np.median(sub.y_um) - p.lb_y) / p.pixel))
    a = np.asarray(img, np.float64)
    b = np.asarray(img_r, np.float64)[:a.shape[0], :a.shape[1]]
    box = (slice(cx - 20, cx + 21), slice(cy - 20, cy + 21))
    chi_core, dof_core = _chi2(a[box].ravel(), b[box].ravel())
    a[box] = 0.0
    b[box] = 0.0
    ii, jj = np.meshgrid(np.arange(a.shape[0]) + 0.5, np.arange(a.shape[1]) + 0.5, indexing="ij")
    r = np.hypot(ii - (cx + 0.5), jj - (cy + 0.5)).ravel()
    edges = np.array([20.5, 25, 30, 40, 55, 75, 100, 140, 200, 300, 400])
    chi_ring, dof_ring = _chi2(np.histogram(r, edges, weights=a.ravel())[0], np.histogram(r, edges, weights=b.ravel())[0])
    chi2, dof = chi_core + chi_ring, dof_core + dof_ring
    return {"sample": f"first {nev} events of the step's stream, {n} photons, the step's photon counts",
            "against": "reference C transport (oracle/_ref, main/kernel_cuda_c_ver1_0.cu C path)",
            "z_fates": z_f, "z_phs_mean": float(z_mean), "z_swank": float(z_swank),
            "phs_mean": {"gpu": g["mean"], "reference": o["mean"], "rel_err": g["mean"] / o["mean"] - 1.0,
                         "se": float(np.hypot(g["se_mean"], o["se_mean"]))},
            "swank": {"gpu": g["swank"], "reference": o["swank"], "rel_err": g["swank"] / o["swank"] - 1.0,
                      "se": float(np.hypot(g["se_swank"], o["se_swank"]))},
            "prf_chi2": chi2, "prf_dof": dof, "prf_chi2_per_dof": chi2 / max(dof, 1),
            "prf_z": float((chi2 - dof) / np.sqrt(2.0 * max(dof, 1)))}


# DRAM bytes per photon of the transport kernel: dram__bytes_read.sum +
# dram__bytes_write.sum of one ncu capture (26,748,000 B for 46,784,158
# photons of the config-1 stream, 20,000 x-rays, steady state); the traffic is
# one event record per chunk and grows in proportion to the photons.
TRANSPORT_DRAM_BYTES_PER_PHOTON = 0.57
# ncu counters of the transport kernel in steady state (one capture of this
# build on 20,000 config-1 x-rays, where the launch's tail is small): issue
# slots used (smsp__issue_active), FP32 FMA pipe busy (sm__pipe_fma_cycles_
# active), active lanes per warp instruction (smsp__thread_inst_executed_per_
# inst_executed), warp instructions per photon (smsp__inst_executed.sum /
# photons) and the tallies' L2 reductions against their peak
# (lts__t_sectors_op_red.avg.pct_of_peak_sustained_elapsed).
TRANSPORT_NCU = {"issue_slot_utilisation": 0.851, "fp32_pipe_utilisation": 0.334,
                 "lanes_per_instruction": 16.03, "warp_instructions_per_photon": 1233.4,
                 "l2_reduction_pct_of_peak": 0.66,
                 "source": "ncu --clock-control none on 20,000 config-1 x-rays "
                           "(transport_kernel<false,256,4,false,false,false>, default launch)"}


def bench_config(es, world):
    """The workload description both arms print (identical keys and values)."""
    return {"workload": WORKLOAD, "events_per_step": int(es.n), "xrays_per_step": int(es.params.num_hist),
            "photon_counts": "N ~ Poisson(E x 54/keV) per event",
            "l2": "GPU arm: 256 MiB buffer written between timed steps (inside the timed region)",
            "parallelism": f"weak-scaling x{world}" if world > 1 else "single GPU"}


def measure_fp32_peak(device, seconds=2.0):
    """FP32 FMA throughput measured by the library's microbenchmark kernel,
    with the SM clock sampled while it runs."""
    import ctypes
    import hybridmantis_b200 as hb
    tf, dt = ctypes.c_double(0.0), ctypes.c_double(0.0)
    with ClockSampler(device) as clk:
        st = hb.load().fd2_measure_fp32_peak(device, seconds, ctypes.byref(tf), ctypes.byref(dt))
    if st != 0:
        return None
    c = clk.summary()
    out = {"tflops": tf.value, "seconds": dt.value, "sm_mhz": c["sm_mhz"], "sm_max_mhz": c["sm_max_mhz"],
           "reasons": c["reasons"]}
    if c["sm_mhz"] and c["sm_max_mhz"]:
        out["tflops_at_max_clock"] = tf.value * c["sm_max_mhz"] / c["sm_mhz"]
    return out


def reference_gpu(es, nphot, device):
    """One launch of the reference's CUDA kernel over the step's events."""
    from oracle import pyoracle as po
    if not po.ref_cuda_available():
        return None
    r = po.run_ref_cuda(_oracle_geometry(es.params), es.x_um.astype(np.float64), es.y_um.astype(np.float64),
                        es.z_um.astype(np.float64), es.hist, nphot, num_hist=int(es.params.num_hist), grid=18000,
                        device=device)
    ms = r.extra["kernel_ms"]
    photons = int(np.sum(nphot))
    return {"value": photons / (ms / 1e3), "unit": "photons/s", "kernel_ms": ms, "photons": photons,
            "kind": "reference CUDA kernel algo (main/kernel_cuda_c_ver1_0.cu, -DUSING_CUDA -use_fast_math -O3) "
                    "compiled for sm_100a, GRIDSIZE 18000 x BLOCKSIZE 128, events resident, CUDA-event timed"}


def work_per_photon(es, nphot, n_events=300):
    """Algorithmic FP32 operations per photon from the oracle's call counts."""
    from oracle import pyoracle as po
    g = _oracle_geometry(es.params)
    k = min(n_events, es.n)
    po.reset_call_counts()
    po.run_oracle(g, es.x_um[:k].astype(np.float64), es.y_um[:k].astype(np.float64), es.z_um[:k].astype(np.float64),
                  es.hist[:k], np.asarray(nphot[:k], np.int32), prim_size=int(es.params.num_hist), records=False)
    calls = po.call_counts()
    photons = float(np.sum(nphot[:k]))
    per = {n: calls[n] / photons for n in OPS_PER_CALL}
    return sum(per[n] * OPS_PER_CALL[n] for n in OPS_PER_CALL), per


# --------------------------------------------------------------- clocks

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-i", str(self.idx), "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [v.strip() for v in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# --------------------------------------------------------------- our arm

def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except Exception:
        return {}


def frontend_leg(params, device, seed, runs=3):
    """The GPU x-ray front end on config 1's detector and spectrum: x-rays/s of
    the front end alone (its kernels' CUDA-event times) and of the chain
    x-ray -> EDEs -> device handoff -> optical transport -> tallies."""
    import copy
    import hybridmantis_b200 as hb
    from hybridmantis_b200 import xray
    p = copy.copy(params)
    n = int(p.num_hist)
    src = xray.triangular_spectrum(20e3, 40e3, 70e3, center_cm=(p.det_x * 0.5e-4, p.det_y * 0.5e-4, 1.0))
    with xray.XrayFrontEnd(det_x_um=p.det_x, det_y_um=p.det_y, det_height_um=p.det_height, seed=seed,
                           device=device) as fe, hb.OpticalTransport(p, device=device, seed=seed + 1) as t:
        fe.run(src, n)  # warm-up (allocations)
        fe.submit(t)
        t.run_sync()
        fe_ms, chain_ms, walls = [], [], []
        for _ in range(runs):
            t.reset_tallies()
            w0 = time.perf_counter()
            fe.run(src, n)
            fe.submit(t)
            t.run_sync()
            walls.append(time.perf_counter() - w0)
            ft = fe.timing()
            fe_ms.append(ft["transport_ms"] + ft["compact_ms"])
            chain_ms.append(fe_ms[-1] + t.timing()["pipeline_ms"])
        st = fe.stats()
        ps = t.phs_stats()
        edes = fe.num_edes()
        photons = t.timing()["photons"]
    # CPU baseline: the same model restated in C (the front end's oracle), one core, a bounded sample
    from oracle import xray_oracle as xo
    m = 20000
    w0 = time.perf_counter()
    xo.run(xray.CSI_TABLE, src, m, det_x_um=p.det_x, det_y_um=p.det_y, det_height_um=p.det_height, seed=seed)
    cpu_dt = time.perf_counter() - w0
    return {"metric": "x-rays/s", "value": n / (np.median(fe_ms) * 1e-3),
            "cpu_baseline": {"value": m / cpu_dt, "unit": "x-rays/s", "cores": 1, "kind": "port",
                             "sample": f"{m} histories of the same source, oracle/xray_oracle.c (gcc -O2, FP64), "
                                       f"{cpu_dt:.1f} s"},
            "chain_xrays_per_s": n / (np.median(chain_ms) * 1e-3),
            "chain_wall_xrays_per_s": n / np.median(walls),
            "workload": f"config-1 detector {p.det_x:g} x {p.det_y:g} x {p.det_height:g} um, {n} x-rays, "
                        f"Triangular(20, 40, 70) keV pencil beam, FP64 photon + electron transport",
            "frontend_ms": float(np.median(fe_ms)), "chain_ms": float(np.median(chain_ms)),
            "edes_per_xray": edes / n, "photons_per_xray": photons / n,
            "fluorescence_escape": st["fluorescence_escaped"] / max(st["fluorescence_emitted"], 1),
            "phs_mean": ps["mean"], "swank": ps["swank"]}


def run_ours(a, rank, world, local_rank):
    import torch
    import hybridmantis_b200 as hb

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    es = hb.synth_events(a.config, a.xrays, a.seed + 7919 * rank)  # rank 0: the reference arm's stream
    x, y, z = es.to_cm()
    de = es.e_ev.astype(np.float64)
    t = hb.OpticalTransport(es.params, device=local_rank, seed=0x5eed + rank,
                            tune_cache=os.path.expanduser("~/.cache/fd2_tune.json"))
    t.submit_events(x, y, z, de, es.hist)
    if not a.no_autotune:
        t.autotune(48)
    for _ in range(a.warmup):
        t.run_sync()
    t.reset_tallies()
    ext = torch.cuda.ExternalStream(t.stream_ptr(), device=local_rank)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local_rank}")
    with torch.cuda.stream(ext):
        flush.zero_()  # first touch of the buffer (page mapping) stays out of the timed region
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    kern_ms = []
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clk:
        start.record(ext)
        for _ in range(a.steps):
            with torch.cuda.stream(ext):
                flush.zero_()  # evict the previous step's working set from L2
            t.run()
            t.wait()
            kern_ms.append(t.timing()["transport_ms"])
        end.record(ext)
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ms = start.elapsed_time(end)
    cnt = t.counters()
    photons = cnt["generated"]
    stats = t.phs_stats()
    tm = t.timing()
    # whole-job numbers: max time, summed photons
    if dist:
        v = torch.tensor([ms], dtype=torch.float64, device=f"cuda:{local_rank}")
        dist.all_reduce(v, op=dist.ReduceOp.MAX)
        ms = float(v.item())
        p = torch.tensor([photons], dtype=torch.float64, device=f"cuda:{local_rank}")
        dist.all_reduce(p)
        photons = float(p.item())
    value = photons / (ms / 1e3)

    # merge the tallies of all ranks once (the path's only exchange step)
    merge_ms = None
    if dist:
        t0 = time.perf_counter()
        prf = torch.from_numpy(t.prf().astype(np.int64)).to(f"cuda:{local_rank}")
        phs = torch.from_numpy(t.phs().astype(np.int64)).to(f"cuda:{local_rank}")
        dist.all_reduce(prf)
        dist.all_reduce(phs)
        torch.cuda.synchronize()
        merge_ms = (time.perf_counter() - t0) * 1e3

    # end to end through the C ABI with host buffers
    t.reset_tallies()
    e2e_steps = max(2, a.steps)
    h2d = es.n * (4 * 8 + 4)
    xd, yd = t.prf_dims()
    d2h = xd * yd * 8 + es.params.num_bins * 4 + 48
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        t.submit_events(x, y, z, de, es.hist)
        t.run()
        t.wait()
        t.prf()
        t.phs()
        t.phs_stats()
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    e2e_photons = t.counters()["generated"]
    if dist:
        v = torch.tensor([e2e_s], dtype=torch.float64, device=f"cuda:{local_rank}")
        dist.all_reduce(v, op=dist.ReduceOp.MAX)
        e2e_s = float(v.item())
        p = torch.tensor([e2e_photons], dtype=torch.float64, device=f"cuda:{local_rank}")
        dist.all_reduce(p)
        e2e_photons = float(p.item())

    out = None
    if rank == 0:
        nphot = t.photon_counts(es.n)
        wpp, calls = work_per_photon(es, nphot)
        peaks = _peaks()
        import torch as _t
        sms = _t.cuda.get_device_properties(local_rank).multi_processor_count
        sm_max = float(peaks.get("sm_max_mhz", 1965.0))
        peak_tflops = sms * 128 * 2 * sm_max * 1e6 / 1e12
        photons_per_launch = tm["photons"]
        avg_kern_s = float(np.mean(kern_ms)) / 1e3
        achieved = photons_per_launch * wpp / avg_kern_s / 1e12
        fma = measure_fp32_peak(local_rank) if world == 1 else None
        roofline = {"bound": "fp32-issue", "achieved": achieved, "peak": peak_tflops, "unit": "TFLOP/s",
                    "frac": achieved / peak_tflops,
                    "traffic": TRANSPORT_DRAM_BYTES_PER_PHOTON * photons_per_launch,
                    "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of a 20,000-x-ray capture, "
                                      "scaled by photons",
                    "peak_source": f"derived: {sms} SMs x 128 FP32 lanes x 2 (FMA) x {sm_max:.0f} MHz "
                                   f"(sm_max_mhz of MEASURED_PEAKS.json; the file has no FP32 entry)",
                    "peak_measured_fma": fma,
                    "work_per_photon_fp32_ops": wpp, "kernel_ms_per_launch": avg_kern_s * 1e3,
                    "photons_per_launch": photons_per_launch,
                    "ncu": TRANSPORT_NCU}
        cpu = None
        parity = None
        if not a.no_cpu_baseline and world == 1:
            ref = CpuReference(es, nphot)
            rate, ph, nev, dt, tallies = ref.timed_sample(a.cpu_seconds, keep=True)
            variants = cpu_variants(ref)
            ref.close()
            cpu = {"value": rate, "unit": "photons/s", "cores": ref.cores, "kind": "reference",
                   "cpu_model": cpu_model(),
                   "sample": f"first {nev} events ({ph} photons) of the same stream and the same photon counts, "
                             f"reference C transport (gcc -O2), {ref.cores} processes, {dt:.1f} s",
                   "variants": dict(variants, **{f"{ref.cores}core_O2": {
                       "value": rate, "unit": "photons/s", "cores": ref.cores, "flags": "gcc -O2",
                       "sample": f"first {nev} events ({ph} photons), {dt:.1f} s"}})}
            parity = parity_vs_reference(es, nphot, nev, tallies, local_rank, seed=0xa11ce)
        ref_gpu = None
        if not a.no_ref_gpu and world == 1:
            ref_gpu = reference_gpu(es, nphot, local_rank)
        surrogate = None
        if not a.no_surrogate and world == 1 and os.path.exists(a.surrogate_model):
            from hybridmantis_b200 import eval_surrogate
            ev = eval_surrogate.evaluate(a.surrogate_model, config=4, xrays=a.surrogate_xrays, seed=a.seed,
                                         audit=0.01, device=local_rank, repeats=2, noise_floor=True)
            st = ev.pop("sg_stats")
            surrogate = {"metric": "x-rays/s", "value": ev["sg_xrays_per_s"], "mc_value": ev["mc_xrays_per_s"],
                         "speedup_vs_mc": ev["speedup"],
                         "workload": f"config 4: {ev['xrays']} x-rays, triangular 20-70 keV, 500 um CsI, R=5 um, "
                                     f"clusters as config 1 ({ev['events']} events); same seeded stream for both",
                         "phs_mean": ev["phs_mean"], "swank": ev["swank"], "swank_diff": ev["swank_diff"],
                         "radial_prf_l1": ev["radial_prf_l1"], "prf_image_l1": ev["prf_image_l1"],
                         "mc_vs_mc": ev.get("mc_vs_mc"),
                         "audit": {k: st[k] for k in ("audit_events", "audit_z", "audit_radial_l1", "audit_ms")},
                         "mc_fallback_events": st["mc_events"], "surrogate_events": st["surrogate_events"],
                         "ms": {"network_and_sampling": st["sg_ms"], "monte_carlo_outside_hull": st["mc_ms"],
                                "audit": st["audit_ms"], "total": st["total_ms"]},
                         "model": os.path.relpath(a.surrogate_model, ROOT)}
        frontend = None
        if not a.no_frontend and world == 1:
            frontend = frontend_leg(es.params, local_rank, a.seed)
        clocks = clk.summary()
        out = {
            "metric": METRIC, "value": value, "unit": "photons/s", "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms / a.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded EDE generator; PENELOPE not shipped)",
            "config": bench_config(es, world),
            "launch": {k: tm[k] for k in ("grid", "block", "chunk", "refill", "prf_window", "fresnel_batch")},
            "e2e": {"value": e2e_photons / e2e_s, "unit": "photons/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            # per step: count, scan_tiles, scan_sums, scan_add, fill_chunks, transport, phs, bump
            "gpu_launches": a.steps * 8,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "reference_gpu": ref_gpu,
            "surrogate": surrogate,
            "xray_frontend": frontend,
            "clocks": clocks,
            "results": {"phs_mean": stats["mean"], "swank": stats["swank"],
                        "fates_per_photon": {k: cnt[k] / max(cnt["generated"], 1) for k in
                                             ("detected", "abs_top", "abs_bulk", "lost", "outofcol", "theta1",
                                              "capped")},
                        "xrays_per_s": es.params.num_hist * a.steps * world / (ms / 1e3),
                        "photons_per_step": photons / max(a.steps, 1) / world,
                        "merge_ms": merge_ms, "calls_per_photon": calls, "parity": parity},
        }
    t.close()
    if dist:
        dist.destroy_process_group()
    return out


# --------------------------------------------------------- reference arm

def run_reference(a, rank, world):
    """The reference's own C transport (oracle/_ref, gcc -O2) on every host
    core, over the same event stream as the product arm (the generator's
    host-only build in oracle/, so this process maps no product library) with
    photon counts N ~ Poisson(E * yield) drawn on the host, as the reference's
    driver does with GSL (numpy stands in for GSL)."""
    if rank != 0:
        return None
    from oracle import pyoracle as po
    es = po.synth_events_host(a.config, a.xrays, a.seed)
    rng = np.random.default_rng(a.seed)
    nphot = rng.poisson(es.e_ev.astype(np.float64) * es.params.yield_).astype(np.int32)
    ref = CpuReference(es, nphot)
    per_step_s = max(1.0, min(6.0, 150.0 / max(a.steps + a.warmup, 1)))
    start = 0
    for _ in range(a.warmup):
        ref.timed_sample(per_step_s / 2, start)
    total_ph, total_t, nev_tot = 0, 0.0, 0
    for _ in range(a.steps):
        rate, ph, nev, dt, _ = ref.timed_sample(per_step_s, start)
        total_ph += ph
        total_t += dt
        nev_tot += nev
        start = (start + nev) % max(es.n - nev - 1, 1)
    ref.close()
    value = total_ph / total_t
    return {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "photons/s", "n_gpus": a.gpus,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": total_t / a.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded EDE generator; PENELOPE not shipped)",
        "config": bench_config(es, world),
        "cpu_baseline": {"value": value, "unit": "photons/s", "cores": ref.cores, "kind": "reference",
                         "cpu_model": cpu_model(),
                         "sample": f"{a.steps} samples of ~{per_step_s:.1f} s ({nev_tot} events, {total_ph} photons) "
                                   f"of the config-1 stream, reference C transport compiled in place (gcc -O2, "
                                   f"float walk with double libm intermediates), one process per core"},
        "e2e": {"value": value, "unit": "photons/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    a = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if a.impl == "reference":
        out = run_reference(a, rank, world)
    else:
        out = run_ours(a, rank, world, local_rank)
    if rank == 0 and out is not None:
        print(json.dumps(out))


if __name__ == "__main__":
    main()
