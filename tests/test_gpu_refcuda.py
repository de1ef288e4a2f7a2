"""The reference's own CUDA kernel (compiled for sm_100a) against this library.

oracle/_ref/libfd2refcuda.so launches `algo` from the reference's
main/kernel_cuda_c_ver1_0.cu, built with its own flags (-use_fast_math).
Both transport the same events with the same photon counts; with different
random streams the tallies agree within Monte Carlo error: fate fractions,
PHS mean and Swank factor, and the radial PRF.
"""
import numpy as np
import pytest

import hybridmantis_b200 as hb
from oracle import pyoracle as po

from gpu_helpers import c0_events, oracle_geometry, report
from mcstats import phs_moments, poisson_chi2, radial_profile, z_binomial

pytestmark = pytest.mark.gpu

FATES = ["detect", "abs_top", "abs_bulk", "lost"]


@pytest.fixture(scope="module")
def ref_cuda():
    if not po.ref_cuda_available():
        pytest.skip("oracle/_ref/libfd2refcuda.so not built (reference sources absent when it was built)")
    return po


def test_reference_cuda_kernel_statistics(require_gpu, ref_cuda):
    es, N = c0_events(400, seed=5)
    p = es.params
    ref = ref_cuda.run_ref_cuda(oracle_geometry(p), es.x_um.astype(np.float64), es.y_um.astype(np.float64),
                                es.z_um.astype(np.float64), es.hist, N, num_hist=p.num_hist)
    rc = dict(zip(po.COUNTER_NAMES, [int(v) for v in ref.counters]))
    n = int(N.sum())
    assert rc["generated"] == n
    with hb.OpticalTransport(p, count_mode=hb.COUNT_GIVEN, seed=77) as t:
        t.submit(es, nphot=N)
        t.run_sync()
        c = t.counters()
        prim = t.detected_per_primary()
        img = t.prf()
    ours = {"detect": c["detected"], "abs_top": c["abs_top"], "abs_bulk": c["abs_bulk"], "lost": c["lost"]}
    zs = {k: float(z_binomial(ours[k], n, rc[k], n)) for k in FATES}
    g = phs_moments(prim)
    o = phs_moments(ref.per_primary)
    z_mean = (g["mean"] - o["mean"]) / np.hypot(g["se_mean"], o["se_mean"])
    z_swank = (g["swank"] - o["swank"]) / np.hypot(g["se_swank"], o["se_swank"])
    edges = np.array([0, 1, 2, 3, 4, 6, 8, 11, 15, 20, 30, 45, 70, 110, 170, 260, 400])
    chi2, dof = poisson_chi2(radial_profile(img, 250.5, 250.5, edges), radial_profile(ref.image, 250.5, 250.5, edges))
    rep = {"z_fates": zs, "ours": g, "reference_cuda": o, "z_mean": z_mean, "z_swank": z_swank,
           "radial_chi2": chi2, "radial_dof": dof, "ref_counters": rc, "our_counters": c,
           "ref_kernel_ms": ref.extra["kernel_ms"]}
    report("production_vs_reference_cuda_c0", rep)
    # the reference's detected-per-primary array is indexed hist-1 on the GPU path
    assert int(ref.per_primary.sum()) == rc["detect"]
    for k, z in zs.items():
        assert abs(z) < 5.0, rep
    assert abs(z_mean) < 5.0, rep
    assert abs(z_swank) < 5.0, rep
    assert chi2 < dof + 6 * np.sqrt(2 * dof), rep


def test_reference_generated_counter_counts_zero_photon_events(require_gpu, ref_cuda):
    """The reference kernel counts the first photon of every event before its loop
    (main/kernel_cuda_c_ver1_0.cu:443), so each event with N = 0 adds one "generated" photon
    that is never transported: its console's generated total exceeds the sum of its fate
    counters by the number of zero-photon EDEs (12.0 M of the example run's 95.2 M).  This
    library counts the photons it transports."""
    es, N = c0_events(300, seed=8)
    N = N.copy()
    N[::3] = 0
    p = es.params
    ref = ref_cuda.run_ref_cuda(oracle_geometry(p), es.x_um.astype(np.float64), es.y_um.astype(np.float64),
                                es.z_um.astype(np.float64), es.hist, N, num_hist=p.num_hist)
    rc = dict(zip(po.COUNTER_NAMES, [int(v) for v in ref.counters]))
    n, zeros = int(N.sum()), int((N == 0).sum())
    fates = rc["detect"] + rc["abs_top"] + rc["abs_bulk"] + rc["lost"] + rc["outofcol"] + rc["theta1"]
    report("reference_generated_counter", {"ref": rc, "photons": n, "zero_events": zeros, "ref_fate_sum": fates})
    assert rc["generated"] == n + zeros
    assert abs(fates - n) <= 1e-3 * n
    with hb.OpticalTransport(p, count_mode=hb.COUNT_GIVEN, seed=3) as t:
        t.submit(es, nphot=N)
        t.run_sync()
        c = t.counters()
    assert c["generated"] == n
    assert sum(c[k] for k in ("detected", "abs_top", "abs_bulk", "lost", "outofcol", "theta1", "capped")) == n
