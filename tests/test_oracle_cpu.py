"""CPU tests pinning the oracle to the reference.

* RANECU / init_PRNG known answers generated from the reference's own C
  code (tests/golden/ranecu_kat.json);
* per-photon fates, RANECU states and step counts of the reference's C
  transport on small seeded cases (tests/golden/ref_small_runs.npz);
* when the reference compiled in place is available (oracle/_ref), a wider
  bit-exact comparison across parameter regimes, at -O0 and -O2;
* the PHS binning rules.
"""
import json
import os

import numpy as np
import pytest

from oracle import pyoracle as po

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_ranecu_known_answers():
    kat = json.load(open(os.path.join(GOLDEN, "ranecu_kat.json")))
    for st in kat["streams"]:
        s = po.init_prng(st["index"], kat["seed_input"])
        assert list(s) == st["seeds"], st["index"]
        u, after = po.ranecu(s, 10)
        assert np.array_equal(u, np.array(st["uniforms"], np.float32))
        assert list(after) == st["seeds_after_10"]
    # the first stream of the default seed: seeds after one draw and the draw
    s0 = po.init_prng(0)
    u, after = po.ranecu(s0, 1)
    assert list(after) == [573276812, 397012565]
    assert abs(float(u[0]) - 0.0820794329) < 1e-9


def _golden_case(z, name):
    gv = z[f"{name}_geom"]
    g = po.Geometry(*[float(v) for v in gv[:16]], pixel=int(gv[16]))
    return g, z[f"{name}_x"], z[f"{name}_y"], z[f"{name}_z"], z[f"{name}_hist"], z[f"{name}_N"]


@pytest.mark.parametrize("name", ["c0", "sensor", "pix9"])
def test_oracle_matches_reference_golden(name):
    z = np.load(os.path.join(GOLDEN, "ref_small_runs.npz"))
    g, x, y, zz, hist, N = _golden_case(z, name)
    o = po.run_oracle(g, x, y, zz, hist, N, seed_input=12345, base=7, prim_size=int(hist.max()),
                      xdim=501, ydim=501)
    assert np.array_equal(o.fate, z[f"{name}_fate"])
    assert np.array_equal(o.seeds, z[f"{name}_seeds"])
    assert np.array_equal(o.steps, z[f"{name}_steps"])
    assert np.array_equal(o.counters, z[f"{name}_counters"])
    assert np.array_equal(o.per_primary, z[f"{name}_per_primary"])
    nz = z[f"{name}_image_nz"]
    assert np.array_equal(np.argwhere(o.image > 0), nz)
    assert np.array_equal(o.image[o.image > 0], z[f"{name}_image_vals"])
    # every detected photon's pixel lands in the image
    det = o.fate == 1
    pix = o.pix[det]
    inside = (pix[:, 0] >= 0) & (pix[:, 1] >= 0)
    assert int(o.image.sum()) == int(inside.sum())


REGIMES = {
    "c0": dict(),
    "beta0": dict(beta=0.0),
    "no_absorption": dict(top_absfrac=0.0, bulk_abs=0.0),
    "low_contrast": dict(n_col=1.4, n_gap=1.0),
    "matched_index": dict(n_col=1.0, n_gap=1.0),
    "narrow_detector": dict(xdet=60.0, ydet=60.0, ub_x=60.0, ub_y=60.0, H=500.0, R=2.5, beta=0.5),
    "thick_absorbing": dict(H=600.0, R=7.5, beta=0.45, top_absfrac=0.95, bulk_abs=1e-3, sensor_refl=0.5),
    "example": dict(xdet=909, ydet=909, H=150, R=5.1, d_min=1.0, ub_x=909, ub_y=909, pixel=9, sensor_refl=0.25),
}


@pytest.mark.skipif(not po.ref_available("O2"), reason="reference not compiled in place (oracle/_ref)")
@pytest.mark.parametrize("regime", sorted(REGIMES))
def test_oracle_matches_reference_inplace(regime):
    g = po.Geometry(**REGIMES[regime])
    rng = np.random.default_rng(len(regime) * 7919)
    n = 12
    x = g.xdet / 2 + rng.normal(0, 3, n)
    y = g.ydet / 2 + rng.normal(0, 3, n)
    z = g.H / 2 - np.minimum(rng.exponential(60, n), 0.999 * g.H)
    hist = np.arange(1, n + 1)
    N = rng.integers(0, 400, n)
    o = po.run_oracle(g, x, y, z, hist, N, seed_input=12345, base=17, xdim=501, ydim=501)
    r = po.run_ref(g, x, y, z, hist, N, seed_input=12345, base=17)
    assert r.status == 0
    assert np.array_equal(o.counters, r.counters)
    assert np.array_equal(o.fate, r.fate)
    assert np.array_equal(o.seeds, r.seeds)
    assert np.array_equal(o.steps, r.steps)
    assert np.array_equal(o.per_primary, r.per_primary)
    xd, yd = min(501, g.xdim), min(501, g.ydim)
    assert np.array_equal(o.image[:xd, :yd], r.image[:xd, :yd])


@pytest.mark.skipif(not po.ref_available("O0"), reason="reference not compiled in place (oracle/_ref)")
def test_reference_optimisation_levels_agree():
    g = po.Geometry()
    x = np.array([250.5, 251.0]); z = np.array([10.0, -40.0])
    a = po.run_ref(g, x, x, z, [1, 2], [300, 300], opt="O0")
    b = po.run_ref(g, x, x, z, [1, 2], [300, 300], opt="O2")
    assert np.array_equal(a.fate, b.fate) and np.array_equal(a.seeds, b.seeds)


def test_event_streams_are_independent_of_grouping():
    """Event e always uses stream init_PRNG(base + e): splitting a buffer
    into pieces with the matching bases gives identical results."""
    g = po.Geometry()
    rng = np.random.default_rng(3)
    n = 10
    x = 250.5 + rng.normal(0, 2, n)
    z = 75.0 - np.minimum(rng.exponential(60, n), 149.0)
    hist = np.arange(1, n + 1)
    N = rng.integers(20, 120, n)
    whole = po.run_oracle(g, x, x, z, hist, N, prim_size=n)
    a = po.run_oracle(g, x[:4], x[:4], z[:4], hist[:4], N[:4], base=0, prim_size=n)
    b = po.run_oracle(g, x[4:], x[4:], z[4:], hist[4:], N[4:], base=4, prim_size=n)
    assert np.array_equal(whole.fate, np.concatenate([a.fate, b.fate]))
    assert np.array_equal(whole.image, a.image + b.image)
    assert np.array_equal(whole.per_primary, a.per_primary + b.per_primary)


def test_phs_binning_rules():
    # width (max-min)/bins = 10, min 0: c<=0 excluded, c>=max -> last bin
    prim = np.array([0, 1, 9, 10, 55, 1399, 1400, 5000, -3], np.int32)
    h = po.phs(prim, 0, 1400, 140)
    expect = np.zeros(140, np.int32)
    for c in [1, 9, 10, 55, 1399]:
        expect[c // 10] += 1
    expect[139] += 2
    assert np.array_equal(h, expect)
    # min > 0: counts <= min go to bin 0, bins shift by min/width
    h = po.phs(np.array([3, 20, 25, 40], np.int32), 20, 60, 4)
    assert list(h) == [3, 0, 1, 0]
    with pytest.raises(ValueError):
        po.phs(np.array([1], np.int32), 0, 5, 10)


def test_threaded_oracle_equals_one_call():
    """The GPU parity tests run the oracle over event slices on host threads
    (tests/gpu_helpers.run_oracle_parallel); the sums equal one call, and the
    per-thread call counters of the calling thread are untouched by the
    workers."""
    import hybridmantis_b200 as hb
    from tests.gpu_helpers import run_oracle_on, run_oracle_parallel

    es = hb.synth_events(1, 40, 5)
    rng = np.random.default_rng(1)
    N = rng.poisson(es.e_ev.astype(np.float64) * 0.01).astype(np.int32)
    po.reset_call_counts()
    a = run_oracle_parallel(es, N, workers=4)
    assert sum(po.call_counts().values()) == 0
    b = run_oracle_on(es, N)
    assert sum(po.call_counts().values()) > 0
    assert np.array_equal(a.image, b.image)
    assert np.array_equal(a.per_primary, b.per_primary)
    assert np.array_equal(a.counters, b.counters)
