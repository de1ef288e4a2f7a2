"""GPU parity of the FP32 production path on the benchmarked workload.

The bench's workload is the config-1 stream: triangular 20-70 keV x-rays
with 1 + Poisson(1.5) deposition clusters in 300 um CsI, R = 4 um.  Here
1,000 of its x-rays (about 2.3e6 optical photons) go through the production
kernel and through the oracle (the reference's C path restated,
oracle/fd2_oracle.c, main/kernel_cuda_c_ver1_0.cu:553-658 driven as
main/hybridMANTIS_c_ver1_0.c:189-340) with the same events and the same
photon counts.  Asserted, each within 5 standard errors:

* fate fractions (detected, top, bulk, lost), two-sample binomial z;
* PHS mean and Swank factor over histories with a detection (delta-method
  standard errors);
* the PRF per bin: a Poisson chi-square over the central 41 x 41 one-micron
  pixels around the beam plus the totals of rings outside them
  (main/kernel_cuda_c_ver1_0.cu:3405-3416 is the reference's tally).

The same test runs with sensorRefl = 0.25, the reference example's value,
which drives the sensor reflection (refl_bottom, main/kernel_cuda_c_ver1_0.cu
:2985-3087, and the reflect branch of detection, :3372-3400).

The PHS binning on the GPU (phs_kernel) is checked bin for bin against the
oracle's rule (main/hybridMANTIS_cuda_ver1_0.cu:376-399) on the very same
per-history counts, with min > 0, counts at or above max, and a bin width
that does not divide the range.
"""
import numpy as np
import pytest

import hybridmantis_b200 as hb
from oracle import pyoracle as po
from tests.gpu_helpers import report, run_oracle_parallel
from tests.mcstats import phs_moments, poisson_chi2, radial_profile, z_binomial

pytestmark = pytest.mark.gpu

Z_MAX = 5.0


def _copy_params(p):
    return type(p).from_buffer_copy(p)


def c1_events(xrays, seed):
    """Config-1 events with Poisson(E * yield) photon counts fixed on the host."""
    es = hb.synth_events(1, xrays, seed)
    rng = np.random.default_rng(seed)
    N = rng.poisson(es.e_ev.astype(np.float64) * es.params.yield_).astype(np.int32)
    return es, N


def prf_chi2(img_a, img_b, cx, cy, half=20):
    """Per-bin Poisson chi-square of two PRF images over the (2 half + 1)^2
    pixels around pixel (cx, cy), plus the totals of rings outside that box."""
    a = np.asarray(img_a, np.float64)
    b = np.asarray(img_b, np.float64)
    box = (slice(cx - half, cx + half + 1), slice(cy - half, cy + half + 1))
    chi_core, dof_core = poisson_chi2(a[box].ravel(), b[box].ravel())
    ma, mb = a.copy(), b.copy()
    ma[box] = 0.0
    mb[box] = 0.0
    edges = np.array([half + 0.5, 25, 30, 40, 55, 75, 100, 140, 200, 300, 400])
    ra = radial_profile(ma, cx + 0.5, cy + 0.5, edges)
    rb = radial_profile(mb, cx + 0.5, cy + 0.5, edges)
    chi_ring, dof_ring = poisson_chi2(ra, rb)
    return chi_core + chi_ring, dof_core + dof_ring, {"core": (chi_core, dof_core), "rings": (chi_ring, dof_ring)}


def compare_with_oracle(es, N, params, seed, name):
    with hb.OpticalTransport(params, count_mode=hb.COUNT_GIVEN, seed=seed) as t:
        t.submit(es, nphot=N)
        t.run_sync()
        c = t.counters()
        prim = t.detected_per_primary()
        img = t.prf()
        stats_dev = t.phs_stats()
    orc = run_oracle_parallel(es, N, params=params)
    n = int(N.sum())
    oc = dict(zip(po.COUNTER_NAMES, [int(v) for v in orc.counters]))
    oc["detected"] = oc.pop("detect")
    assert oc["generated"] == n == c["generated"]
    zs = {k: float(z_binomial(c[k], n, oc[k], n)) for k in ["detected", "abs_top", "abs_bulk", "lost"]}
    g = phs_moments(prim)
    o = phs_moments(orc.per_primary)
    z_mean = (g["mean"] - o["mean"]) / np.hypot(g["se_mean"], o["se_mean"])
    z_swank = (g["swank"] - o["swank"]) / np.hypot(g["se_swank"], o["se_swank"])
    cx = int(np.floor((np.median(es.x_um) - params.lb_x) / params.pixel))
    cy = int(np.floor((np.median(es.y_um) - params.lb_y) / params.pixel))
    chi2, dof, parts = prf_chi2(img, orc.image, cx, cy)
    z_chi2 = (chi2 - dof) / np.sqrt(2.0 * dof)
    rep = {"photons": n, "z_fates": zs, "gpu": g, "oracle": o, "z_mean": float(z_mean), "z_swank": float(z_swank),
           "prf_chi2": chi2, "prf_dof": dof, "prf_z": float(z_chi2), "prf_parts": parts, "gpu_counters": c,
           "oracle_counters": oc, "rel_err": {"phs_mean": g["mean"] / o["mean"] - 1.0,
                                              "swank": g["swank"] / o["swank"] - 1.0}}
    report(name, rep)
    assert c["capped"] == 0, rep
    for k, z in zs.items():
        assert abs(z) < Z_MAX, (k, rep)
    assert abs(z_mean) < Z_MAX, rep
    assert abs(z_swank) < Z_MAX, rep
    assert z_chi2 < Z_MAX, rep
    # device FP64 moments equal the host's on the same counts
    assert stats_dev["primaries"] == g["n"]
    assert abs(stats_dev["mean"] - g["mean"]) < 1e-9 * g["mean"]
    assert abs(stats_dev["swank"] - g["swank"]) < 1e-12
    return rep


@pytest.mark.parametrize("sensor_refl", [0.0, 0.25])
def test_production_matches_oracle_config1(require_gpu, sensor_refl):
    es, N = c1_events(1000, seed=41 if sensor_refl == 0.0 else 43)
    p = _copy_params(es.params)
    p.sensor_refl = sensor_refl
    rep = compare_with_oracle(es, N, p, seed=0x1234 + int(sensor_refl * 100), name=f"production_vs_oracle_c1_sr{sensor_refl}")
    if sensor_refl > 0.0:
        # the sensor reflection is exercised: fewer detections per photon
        # than the ideal sensor's on the same stream
        assert rep["oracle_counters"]["detected"] > 0


@pytest.mark.parametrize("lo,hi,bins", [(600, 1500, 90), (449, 1368, 20), (0, 4000, 1000)])
def test_gpu_phs_binning_matches_reference_rule(require_gpu, lo, hi, bins):
    # no oracle transport here (only its binning rule), so 2,000 x-rays: the
    # middle case then has ~10 histories in its past-the-end range
    es, N = c1_events(2000, seed=47)
    p = _copy_params(es.params)
    p.min_photons, p.max_photons, p.num_bins = lo, hi, bins
    with hb.OpticalTransport(p, count_mode=hb.COUNT_GIVEN, seed=99) as t:
        t.submit(es, nphot=N)
        t.run_sync()
        prim = t.detected_per_primary()
        phs = t.phs()
        st = t.phs_stats()
    want = po.phs(prim, lo, hi, bins)
    pos = prim[prim > 0]
    width = (hi - lo) // bins
    # the cases reach the rule's edges: counts <= min, counts >= max
    if lo > 0:
        assert (pos <= lo).any() and (pos >= hi).any()
    assert np.array_equal(phs, want)
    # histories the reference would bin past the last bin are dropped and counted
    shift = lo // width
    mid = pos[(pos > lo) & (pos < hi)]
    past = int(((mid // width - shift) >= bins).sum())
    if (lo, hi, bins) == (449, 1368, 20):
        assert past > 0  # width 45 leaves counts 1305..1367 past the last bin
    assert st["phs_dropped"] == past
    assert phs.sum() + past == len(pos)
