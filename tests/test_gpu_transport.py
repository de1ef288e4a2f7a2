"""GPU parity tests of the transport, through the C ABI.

* replay (REF and FP64) against the CPU oracle, photon by photon, with
  divergent histories counted;
* the FP32 production path against the oracle within Monte Carlo
  standard errors (PHS mean, Swank factor, fate fractions, PRF);
* bookkeeping invariants, determinism across launch shapes, tallies.
"""
import numpy as np
import pytest

import hybridmantis_b200 as hb
from tests.gpu_helpers import c0_events, compare_replay, oracle_geometry, report, run_oracle_on
from tests.mcstats import phs_moments, poisson_chi2, radial_profile, z_binomial

pytestmark = pytest.mark.gpu

FATES = ["detected", "abs_top", "abs_bulk", "lost", "outofcol", "theta1", "capped"]


def _run_given(es, N, **kw):
    t = hb.OpticalTransport(es.params, count_mode=hb.COUNT_GIVEN, **kw)
    t.submit(es, nphot=N)
    t.run_sync()
    return t


def test_bookkeeping(require_gpu):
    es, N = c0_events(64)
    with _run_given(es, N) as t:
        c = t.counters()
        assert c["generated"] == N.sum()
        assert sum(c[k] for k in FATES) == N.sum()
        assert c["capped"] == 0
        prim = t.detected_per_primary()
        assert prim.sum() == c["detected"]
        assert t.prf().sum() == c["detected_in_prf"] <= c["detected"]
        tm = t.timing()
        assert tm["photons"] == N.sum() and tm["transport_ms"] > 0


@pytest.mark.parametrize("mode,min_identical", [(hb.REPLAY_REF, 0.95), (hb.REPLAY_FP64, 0.0)])
def test_replay_matches_oracle(require_gpu, mode, min_identical):
    """REF: float storage with the reference's double promotions and the C
    library's float acosf/asinf -> the oracle's photon histories exactly,
    up to rare 1-ulp differences of CUDA's double libm.  FP64: the same walk
    in double; the column billiard amplifies the precision difference, so
    histories diverge after a few photons -- counted, not asserted."""
    es, N = c0_events(40, seed=11)
    with hb.OpticalTransport(es.params, count_mode=hb.COUNT_GIVEN) as t:
        t.submit(es, nphot=N)
        gpu = t.replay(int(N.sum()), mode=mode, seed_input=271828182)
        c = t.counters()
    orc = run_oracle_on(es, N, records=True)
    stats = compare_replay(N, gpu, orc)
    report(f"replay_{'ref' if mode == hb.REPLAY_REF else 'fp64'}", stats)
    assert c["generated"] == N.sum()
    assert 1.0 - stats["divergent_events"] / stats["events"] >= min_identical, stats
    if mode == hb.REPLAY_REF:
        assert stats["photons_matched_before_divergence"] >= 0.95 * stats["photons"], stats


def test_production_matches_oracle_statistics(require_gpu):
    es, N = c0_events(400, seed=5)
    with _run_given(es, N) as t:
        c = t.counters()
        prim = t.detected_per_primary()
        img = t.prf()
        stats_dev = t.phs_stats()
    orc = run_oracle_on(es, N)
    n = int(N.sum())
    oc = dict(zip(["generated", "detected", "abs_top", "abs_bulk", "lost", "outofcol", "theta1"],
                  [int(v) for v in orc.counters]))
    zs = {k: float(z_binomial(c[k], n, oc[k], n)) for k in ["detected", "abs_top", "abs_bulk", "lost"]}
    g = phs_moments(prim)
    o = phs_moments(orc.per_primary)
    z_mean = (g["mean"] - o["mean"]) / np.hypot(g["se_mean"], o["se_mean"])
    z_swank = (g["swank"] - o["swank"]) / np.hypot(g["se_swank"], o["se_swank"])
    edges = np.array([0, 1, 2, 3, 4, 6, 8, 11, 15, 20, 30, 45, 70, 110, 170, 260, 400])
    rg = radial_profile(img, 250.5, 250.5, edges)
    ro = radial_profile(orc.image, 250.5, 250.5, edges)
    chi2, dof = poisson_chi2(rg, ro)
    rep = {"z_fates": zs, "gpu": g, "oracle": o, "z_mean": z_mean, "z_swank": z_swank,
           "radial_chi2": chi2, "radial_dof": dof, "gpu_counters": c, "oracle_counters": oc,
           "device_phs_stats": stats_dev}
    report("production_vs_oracle_c0", rep)
    assert c["capped"] == 0
    for k, z in zs.items():
        assert abs(z) < 5.0, rep
    assert abs(z_mean) < 5.0, rep
    assert abs(z_swank) < 5.0, rep
    assert chi2 < dof + 6 * np.sqrt(2 * dof), rep
    # device FP64 moments equal the host's on the same counts
    assert stats_dev["primaries"] == g["n"]
    assert abs(stats_dev["mean"] - g["mean"]) < 1e-9 * g["mean"]
    assert abs(stats_dev["swank"] - g["swank"]) < 1e-12


def test_results_independent_of_launch_shape(require_gpu):
    es, N = c0_events(48, seed=9)
    outs = []
    for kw in [dict(), dict(block_size=128, chunk=8, refill=4, prf_window=0),
               dict(block_size=256, ctas_per_sm=3, refill=8, fresnel_batch=4),
               dict(block_size=512, ctas_per_sm=1, chunk=64, use_graph=False),
               dict(tally_mode=1), dict(tally_mode=1, block_size=320, ctas_per_sm=2, prf_window=48)]:
        with _run_given(es, N, seed=77, **kw) as t:
            c = t.counters()
            c.pop("photon_distance")
            outs.append((c, t.detected_per_primary().copy(), t.prf().copy()))
    for c, prim, img in outs[1:]:
        assert c == outs[0][0]
        assert np.array_equal(prim, outs[0][1])
        assert np.array_equal(img, outs[0][2])


def test_runs_accumulate_and_reset(require_gpu):
    es, N = c0_events(16, seed=2)
    with hb.OpticalTransport(es.params, count_mode=hb.COUNT_GIVEN) as t:
        t.submit(es, nphot=N)
        t.run_sync()
        a = t.counters()
        t.run()
        t.run()
        t.wait()
        b = t.counters()
        assert b["generated"] == 3 * N.sum()
        t.reset_tallies()
        t.run_sync()
        c = t.counters()
        assert c["generated"] == N.sum()
        assert c["detected"] == a["detected"]  # run counter restarts: same realisation


def test_poisson_counts(require_gpu):
    from scipy import stats
    rng = np.random.default_rng(0)
    for mu in [0.7, 4.0, 9.9, 30.0, 1350.0]:
        n = 20000
        p = hb.default_params(num_hist=n, yield_=0.054)
        x = np.full(n, 250.5, np.float32)
        z = np.full(n, 70.0, np.float32)
        e = np.full(n, mu / 0.054, np.float32)
        with hb.OpticalTransport(p, count_mode=hb.COUNT_POISSON, seed=int(rng.integers(1 << 40))) as t:
            t.submit_events_um(x, x, z, e, np.arange(1, n + 1))
            t.run_sync()
            k = t.photon_counts(n)
        mu_f = float(np.float64(np.float32(mu / 0.054)) * 0.054)
        assert abs(k.mean() - mu_f) < 5 * np.sqrt(mu_f / n)
        assert abs(k.var() / mu_f - 1.0) < 5 * np.sqrt(2.0 / n)
        lo, hi = stats.poisson.ppf([1e-4, 1 - 1e-4], mu_f).astype(int)
        obs = np.array([(k == v).sum() for v in range(lo, hi + 1)])
        exp = stats.poisson.pmf(np.arange(lo, hi + 1), mu_f) * n
        m = exp > 5
        chi2 = (((obs - exp) ** 2) / exp)[m].sum()
        assert chi2 < m.sum() + 6 * np.sqrt(2 * m.sum())


def test_gaussian_counts(require_gpu):
    n, mu = 20000, 1350.0
    p = hb.default_params(num_hist=n)
    x = np.full(n, 250.5, np.float32)
    with hb.OpticalTransport(p, count_mode=hb.COUNT_GAUSSIAN) as t:
        t.submit_events_um(x, x, np.full(n, 70.0, np.float32), np.full(n, 25000.0, np.float32), np.arange(1, n + 1))
        t.run_sync()
        k = t.photon_counts(n)
    assert abs(k.mean() - mu) < 5 * np.sqrt(mu / n)
    assert abs(k.var() / mu - 1.0) < 0.05


def test_cm_submission_matches_um(require_gpu):
    es = hb.synth_events(0, 32, 4)
    x, y, z = es.to_cm()
    with hb.OpticalTransport(es.params, seed=5) as a, hb.OpticalTransport(es.params, seed=5) as b:
        a.submit_events(x, y, z, es.e_ev.astype(np.float64), es.hist)
        a.run_sync()
        # the same floats reach the device either way
        xu = (x * np.float64(np.float32(10000.0))).astype(np.float32)
        yu = (y * np.float64(np.float32(10000.0))).astype(np.float32)
        zu = (z * np.float64(np.float32(10000.0))).astype(np.float32)
        b.submit_events_um(xu, yu, zu, es.e_ev, es.hist)
        b.run_sync()
        assert np.array_equal(a.photon_counts(es.n), b.photon_counts(es.n))
        assert np.array_equal(a.prf(), b.prf())


def test_bad_events_rejected(require_gpu):
    p = hb.default_params(num_hist=4)
    with hb.OpticalTransport(p) as t:
        ok = np.array([250.0] * 3, np.float32)
        with pytest.raises(hb.Fd2Error) as ei:
            t.submit_events_um(ok, ok, np.zeros(3, np.float32), np.array([1e4, np.nan, 1e4], np.float32), [1, 2, 3])
        assert ei.value.status == 12
        with pytest.raises(hb.Fd2Error) as ei:
            t.submit_events_um(ok, ok, np.zeros(3, np.float32), np.array([1e4, -5, 1e4], np.float32), [1, 2, 3])
        assert ei.value.status == 12
        with pytest.raises(hb.Fd2Error) as ei:
            t.submit_events_um(ok, ok, np.zeros(3, np.float32), np.array([1e4] * 3, np.float32), [1, 2, 9])
        assert ei.value.status == 12
        # still usable
        t.submit_events_um(ok, ok, np.zeros(3, np.float32), np.array([1e4] * 3, np.float32), [1, 2, 3])
        t.run_sync()
        assert t.counters()["generated"] > 0


def test_too_many_photons(require_gpu):
    p = hb.default_params(num_hist=2)
    with hb.OpticalTransport(p, count_mode=hb.COUNT_GIVEN, max_photons_per_event=1000) as t:
        v = np.array([250.0, 250.0], np.float32)
        with pytest.raises(hb.Fd2Error) as ei:
            t.submit_events_um(v, v, np.zeros(2, np.float32), None, [1, 2], nphot=[10, 5000])
        assert ei.value.status == 6


def test_empty_submission(require_gpu):
    # an empty EDE buffer is a valid submission: the run transports nothing and leaves the tallies alone
    p = hb.default_params(num_hist=4)
    with hb.OpticalTransport(p) as t:
        e = np.zeros(0)
        t.submit_events(e, e, e, e, np.zeros(0, np.int32))
        t.run_sync()
        c = t.counters()
        assert c["generated"] == 0 and c["detected"] == 0
        assert t.phs().sum() == 0 and t.prf().sum() == 0 and t.timing()["photons"] == 0
        v = np.full(3, 0.025)
        t.submit_events(v, v, np.zeros(3), np.full(3, 1e4), np.array([1, 2, 3], np.int32))
        t.run_sync()
        assert t.counters()["generated"] > 0


def test_deadline_aborts_and_context_recovers(require_gpu):
    es = hb.synth_events(1, 4000, 3)
    with hb.OpticalTransport(es.params, wait_timeout_s=1e-6) as t:
        t.submit(es)
        t.run()
        with pytest.raises(hb.Fd2Error) as ei:
            t.wait()
        assert ei.value.status in (8, 9)
    with hb.OpticalTransport(es.params) as t:
        t.submit(es)
        t.run_sync()
        c = t.counters()
        assert sum(c[k] for k in FATES) == c["generated"] > 0


def test_write_outputs(require_gpu, tmp_path):
    es, N = c0_events(20)
    with _run_given(es, N) as t:
        t.write_outputs(str(tmp_path))
        names = sorted(p.name for p in tmp_path.iterdir())
        assert names == ["detected_150_5_0.1_0.0001_0.2_280_0_0.054_1_1.dat",
                         "myimage_150_5_0.1_0.0001_0.2_280_0_0.054_1_1.dat"]
        det = (tmp_path / names[0]).read_text().splitlines()
        assert len(det) == es.params.num_bins and all(len(l) == 9 for l in det)
        phs = np.array([int(l) for l in det])
        assert np.array_equal(phs, t.phs())
        img = (tmp_path / names[1]).read_text().split("\n")
        assert len(img) == 501 * 502 + 1
        vals = np.array([float(v) for v in img if v.strip()]).reshape(501, 501)  # [jj, ii]
        prf = t.prf() / es.params.num_hist
        assert np.allclose(vals.T, np.round(prf, 4), atol=1e-9)
        with pytest.raises(hb.Fd2Error) as ei:
            t.write_outputs(str(tmp_path))
        assert ei.value.status == 11


def test_wall_root_fp64_fallback(require_gpu):
    """The column-wall quadratic near tangency: the discriminant b^2 - 4ac
    nearly cancels, and in float its sign -- root or no root -- is noise.
    The walk recomputes it from the float coefficients in FP64 (products of
    floats are exact there); compare with an FP64 root of the same float
    coefficients."""
    import ctypes

    rng = np.random.default_rng(12)
    n = 20000
    qa = rng.uniform(0.2, 1.0, n).astype(np.float32)
    qb = (rng.uniform(0.5, 10.0, n) * rng.choice([-1.0, 1.0], n)).astype(np.float32)
    delta = 10.0 ** rng.uniform(-9.5, -5.0, n) * rng.choice([-1.0, 1.0], n)
    qc = (qb.astype(np.float64) ** 2 / (4.0 * qa.astype(np.float64)) * (1.0 - delta)).astype(np.float32)
    out = np.zeros(n, np.float32)
    lib = hb.load()
    st = lib.fd2_debug_wall_root(n, qa.ctypes.data_as(ctypes.c_void_p), qb.ctypes.data_as(ctypes.c_void_p),
                                 qc.ctypes.data_as(ctypes.c_void_p), out.ctypes.data_as(ctypes.c_void_p))
    assert st == 0
    a, b, c = qa.astype(np.float64), qb.astype(np.float64), qc.astype(np.float64)
    disc = b * b - 4.0 * a * c
    s = np.sqrt(np.maximum(disc, 0.0))
    root = np.where(b >= 0.0, -2.0 * c / (b + s), (s - b) / (2.0 * a))
    naive = qb * qb - np.float32(4.0) * qa * qc  # the float discriminant without the fallback
    flipped = np.sign(naive) != np.sign(disc)
    assert flipped.mean() > 0.1  # the cases do reach the cancellation
    has = disc >= 0.0
    assert np.array_equal(out == 999.0, ~has)
    rel = np.abs(out[has] - root[has]) / np.abs(root[has])
    assert rel.max() < 1e-5, rel.max()
