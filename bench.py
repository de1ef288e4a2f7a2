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
  cpu_baseline  the reference's own C transport (oracle/_ref, gcc -O2,
          all host cores) on a bounded sample of the same stream
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
    geom, x, y, z, hist, nphot, base, prim_size = args
    t0 = time.perf_counter()
    r = po.run_ref(geom, x, y, z, hist, nphot, seed_input=271828182, base=base, prim_size=prim_size,
                   records=False, opt="O2")
    return time.perf_counter() - t0, int(r.counters[0])


def _oracle_geometry(p):
    from oracle import pyoracle as po
    return po.Geometry(xdet=p.det_x, ydet=p.det_y, H=p.det_height, R=p.radius, n_col=p.n_col, n_gap=p.n_gap,
                       top_absfrac=p.top_absfrac, bulk_abs=p.bulk_abs, beta=p.beta, d_min=p.d_min, d_max=p.d_max,
                       lb_x=p.lb_x, lb_y=p.lb_y, ub_x=p.ub_x, ub_y=p.ub_y, sensor_refl=p.sensor_refl, pixel=p.pixel)


class CpuReference:
    """The reference's C transport (oracle/_ref, -O2) on all host cores; one
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
        dt, ph = _ref_worker(self._args(0, k))
        self.rate1 = ph / max(dt, 1e-6)

    def _events_for(self, photons, start):
        c = np.cumsum(self.N[start:])
        return int(min(len(c), np.searchsorted(c, photons) + 1))

    def _args(self, start, count):
        es = self.es
        sl = slice(start, start + count)
        return (self.g, es.x_um[sl].astype(np.float64), es.y_um[sl].astype(np.float64),
                es.z_um[sl].astype(np.float64), es.hist[sl], self.N[sl], start, int(es.params.num_hist))

    def timed_sample(self, seconds, start=0):
        photons = self.rate1 * self.cores * seconds
        count = self._events_for(photons, start)
        bounds = np.linspace(start, start + count, self.cores + 1).astype(int)
        t0 = time.perf_counter()
        futs = [self.pool.submit(_ref_worker, self._args(a, b - a)) for a, b in zip(bounds[:-1], bounds[1:]) if b > a]
        ph = sum(f.result()[1] for f in futs)
        dt = time.perf_counter() - t0
        return ph / dt, ph, count, dt

    def close(self):
        self.pool.shutdown()


# DRAM bytes per photon of the transport kernel: dram__bytes_read.sum +
# dram__bytes_write.sum of one ncu capture (3,338,240 B for 4,690,971 photons
# of the config-1 stream, 2,000 x-rays); the traffic is one event record per
# chunk and grows in proportion to the photons.
TRANSPORT_DRAM_BYTES_PER_PHOTON = 3338240.0 / 4690971.0
# Issue slots the transport kernel uses in steady state (ncu
# smsp__issue_active of 20,000 config-1 x-rays, where its tail is small).
TRANSPORT_ISSUE_ACTIVE = 0.554


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
    es = hb.synth_events(a.config, a.xrays, a.seed + 7919 * rank)
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
        roofline = {"bound": "fp32-issue", "achieved": achieved, "peak": peak_tflops, "unit": "TFLOP/s",
                    "frac": achieved / peak_tflops,
                    "traffic": TRANSPORT_DRAM_BYTES_PER_PHOTON * photons_per_launch,
                    "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of a 2,000-x-ray capture, "
                                      "scaled by photons",
                    "peak_source": f"derived: {sms} SMs x 128 FP32 lanes x 2 (FMA) x {sm_max:.0f} MHz "
                                   f"(sm_max_mhz of MEASURED_PEAKS.json; the file has no FP32 entry)",
                    "work_per_photon_fp32_ops": wpp, "kernel_ms_per_launch": avg_kern_s * 1e3,
                    "photons_per_launch": photons_per_launch,
                    # the north-star criterion for this issue-bound kernel: scheduler issue slots used
                    "issue_slot_utilisation": TRANSPORT_ISSUE_ACTIVE,
                    "issue_slot_source": "ncu smsp__issue_active.avg.pct_of_peak_sustained_active of the same "
                                         "kernel on 20,000 config-1 x-rays (steady state, "
                                         "profiles/transport_kernel_config1_20k.md)"}
        cpu = None
        if not a.no_cpu_baseline and world == 1:
            ref = CpuReference(es, nphot)
            rate, ph, nev, dt = ref.timed_sample(a.cpu_seconds)
            ref.close()
            cpu = {"value": rate, "unit": "photons/s", "cores": ref.cores, "kind": "reference",
                   "sample": f"first {nev} events ({ph} photons) of the same stream and the same photon counts, "
                             f"reference C transport (gcc -O2), {ref.cores} processes, {dt:.1f} s"}
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
                         "model": os.path.relpath(a.surrogate_model, ROOT)}
        frontend = None
        if not a.no_frontend and world == 1:
            frontend = frontend_leg(es.params, local_rank, a.seed)
        clocks = clk.summary()
        out = {
            "metric": METRIC, "value": value, "unit": "photons/s", "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms / a.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded EDE generator; PENELOPE not shipped)",
            "config": {"workload": WORKLOAD, "events_per_step": es.n, "xrays_per_step": es.params.num_hist,
                       "photons_per_step": photons / max(a.steps, 1) / world,
                       "l2": "256 MiB buffer written between timed steps (inside the timed region)",
                       "parallelism": f"weak-scaling x{world}" if world > 1 else "single GPU",
                       "launch": {k: tm[k] for k in ("grid", "block", "chunk", "refill", "prf_window",
                                                           "fresnel_batch")}},
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
                        "merge_ms": merge_ms, "calls_per_photon": calls},
        }
    t.close()
    if dist:
        dist.destroy_process_group()
    return out


# --------------------------------------------------------- reference arm

def run_reference(a, rank):
    if rank != 0:
        return None
    import hybridmantis_b200 as hb
    es = hb.synth_events(a.config, a.xrays, a.seed)
    rng = np.random.default_rng(a.seed)
    # the reference samples N ~ Poisson(E * yield) on the host (GSL); numpy here
    nphot = rng.poisson(es.e_ev.astype(np.float64) * es.params.yield_).astype(np.int32)
    ref = CpuReference(es, nphot)
    per_step_s = max(1.0, min(6.0, 150.0 / max(a.steps + a.warmup, 1)))
    start = 0
    for _ in range(a.warmup):
        ref.timed_sample(per_step_s / 2, start)
    rates, total_ph, total_t, nev_tot = [], 0, 0.0, 0
    for _ in range(a.steps):
        rate, ph, nev, dt = ref.timed_sample(per_step_s, start)
        rates.append(rate)
        total_ph += ph
        total_t += dt
        nev_tot += nev
        start = (start + nev) % max(es.n - nev - 1, 1)
    ref.close()
    value = total_ph / total_t
    return {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "photons/s", "n_gpus": a.gpus,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": total_t / a.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 (double libm intermediates)",
        "data": "synthetic (seeded EDE generator; PENELOPE not shipped)",
        "config": {"workload": WORKLOAD, "events_per_step": es.n, "sample_per_step_s": per_step_s},
        "cpu_baseline": {"value": value, "unit": "photons/s", "cores": ref.cores, "kind": "reference",
                         "sample": f"{a.steps} samples of ~{per_step_s:.1f} s ({nev_tot} events, {total_ph} photons) "
                                   f"of the config-1 stream, reference C transport compiled in place (gcc -O2), "
                                   f"one process per core"},
        "e2e": {"value": value, "unit": "photons/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    a = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if a.impl == "reference":
        out = run_reference(a, rank)
    else:
        out = run_ours(a, rank, world, local_rank)
    if rank == 0 and out is not None:
        print(json.dumps(out))


if __name__ == "__main__":
    main()
