"""The surrogate in the event pipeline (fd2_sg_run) against the plain Monte Carlo.

A surrogate trained on Monte Carlo labels of the benchmark's 150 um detector
replaces the transport of the same seeded 25 keV pencil-beam events: the
per-x-ray detected counts (PHS mean, Swank factor) and the radial PRF must
agree with a full Monte Carlo run of the same events within the accuracy a
short training reaches, the bookkeeping must be consistent, and the audit
must report its comparison.
"""
import numpy as np
import pytest

import hybridmantis_b200 as hb
from hybridmantis_b200 import surrogate as sgm

from gpu_helpers import report
from mcstats import phs_moments, radial_profile

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def trained(require_gpu):
    es = hb.synth_events(0, 600, 41)
    g = hb.params_to_geometry(es.params)
    f, ph, det, rad = sgm.label_points([g], 6144, 2000, seed=42, energy_kev=(0.5, 30.0))
    s = sgm.Surrogate(hidden=256, batch=2048, lr=2e-3, seed=43)
    s.set_data(f, ph, det, rad, n_val=512)
    s.train(1500)
    yield s, es
    s.close()


def _run(es, sg=None, audit=0.0):
    with hb.OpticalTransport(es.params, count_mode=hb.COUNT_GAUSSIAN, seed=99) as t:
        t.submit(es)
        stats = None
        if sg is None:
            t.run_sync()
        else:
            stats = sg.run(t, audit)
        return {"counters": t.counters(), "prim": t.detected_per_primary(), "prf": t.prf(), "stats": stats,
                "counts": t.photon_counts(es.n)}


def test_surrogate_run_matches_monte_carlo(trained):
    sg, es = trained
    mc = _run(es)
    sr = _run(es, sg, audit=0.1)
    st = sr["stats"]
    # every event with photons went one way or the other; same photon counts
    n_with = int(np.count_nonzero(mc["counts"]))
    assert st["surrogate_events"] + st["mc_events"] == n_with
    assert np.array_equal(sr["counts"], mc["counts"])
    assert st["surrogate_events"] >= 0.9 * n_with
    assert st["audit_events"] > 0
    # bookkeeping: the detected counter equals the per-history counts
    assert sr["counters"]["detected"] == int(sr["prim"].sum())
    assert sr["counters"]["generated"] == mc["counters"]["generated"]
    # PHS statistics
    a, b = phs_moments(sr["prim"]), phs_moments(mc["prim"])
    rep = {"sg": a, "mc": b, "stats": st}
    assert abs(a["mean"] - b["mean"]) <= 0.03 * b["mean"], rep
    assert abs(a["swank"] - b["swank"]) <= 0.01, rep
    # radial PRF profile (normalised), L1 distance
    edges = np.array([0, 1, 2, 3, 4, 6, 8, 11, 15, 20, 30, 45, 70, 110, 170, 260, 400])
    rs = radial_profile(sr["prf"], 250.5, 250.5, edges).astype(np.float64)
    rm = radial_profile(mc["prf"], 250.5, 250.5, edges).astype(np.float64)
    l1 = np.abs(rs / rs.sum() - rm / rm.sum()).sum()
    rep["radial_l1"] = l1
    report("surrogate_loop_c0", rep)
    assert l1 < 0.06, rep
    # audit: the Monte Carlo of the audited events agrees with the prediction
    assert abs(st["audit_z"]) < 6.0 or abs(st["audit_mc_detected"] - st["audit_sg_expected"]) \
        <= 0.03 * st["audit_mc_detected"], rep
    assert st["audit_radial_l1"] < 0.1, rep


def test_out_of_hull_events_use_monte_carlo(trained):
    sg, es = trained
    lo, hi = sg.hull()
    # a hull no event's energy reaches: all Monte Carlo, identical to fd2_run
    lo2, hi2 = lo.copy(), hi.copy()
    lo2[1], hi2[1] = 1e6, 2e6
    sg.set_hull(lo2, hi2)
    try:
        sr = _run(es, sg, audit=0.0)
    finally:
        sg.set_hull(lo, hi)
    mc = _run(es)
    assert sr["stats"]["surrogate_events"] == 0
    assert np.array_equal(sr["prim"], mc["prim"])
    assert np.array_equal(sr["prf"], mc["prf"])


def test_edge_survival_moves_positions_only(trained, tmp_path):
    """The sampler's edge survival redraws azimuths only: per-history counts,
    counters and the radial profile's first rings are those of the run
    without it, while light near the detector's sides thins out; the
    setting travels with the saved network."""
    sg, es = trained
    assert sg.edge() == (0.0, 1.0)
    plain = _run(es, sg, audit=0.0)
    sg.set_edge(0.5, 40.0)
    try:
        edged = _run(es, sg, audit=0.0)
        path = str(tmp_path / "edge.fd2sg")
        sg.save(path)
        with sgm.Surrogate(hidden=256, batch=2048) as s2:
            s2.load(path)
            assert s2.edge() == (0.5, 40.0)
    finally:
        sg.set_edge(0.0, 1.0)
    assert np.array_equal(plain["prim"], edged["prim"])
    assert plain["counters"]["detected"] == edged["counters"]["detected"]
    assert not np.array_equal(plain["prf"], edged["prf"])
    # the same light within the image, less of it along the sides
    a, b = plain["prf"].astype(np.float64), edged["prf"].astype(np.float64)
    assert abs(a.sum() - b.sum()) <= 1e-3 * a.sum()
    side = np.zeros(a.shape, bool)
    side[:20, :] = side[-20:, :] = side[:, :20] = side[:, -20:] = True
    assert b[side].sum() < a[side].sum()
    for bad in ((1.0, 10.0), (-0.1, 10.0), (0.5, 0.0)):
        with pytest.raises(Exception):
            sg.set_edge(*bad)


def test_depth_margin_routes_depositions_just_outside_the_labels(trained, tmp_path):
    """Depositions a fraction of a micrometre shallower than the hull's depth
    range go to the network with the default 1-um margin (at the range's
    edge depth) and to the Monte Carlo without it."""
    sg, es = trained
    lo, _ = sg.hull()
    assert 0.0 < lo[0] < 1.0
    moved = es.subset(np.arange(es.n))
    moved.z_um = np.full(es.n, es.params.det_height / 2 - 0.5 * lo[0], np.float32)
    with_margin = _run(moved, sg, audit=0.0)["stats"]
    path = str(tmp_path / "net.fd2sg")
    sg.save(path)
    with sgm.Surrogate(hidden=256, batch=2048, depth_margin_um=0.0) as s0:
        s0.load(path)
        without = _run(moved, s0, audit=0.0)["stats"]
    n_with = with_margin["surrogate_events"] + with_margin["mc_events"]
    assert with_margin["surrogate_events"] >= 0.9 * n_with
    assert without["surrogate_events"] == 0 and without["mc_events"] == n_with


def test_audit_is_reproducible(trained, tmp_path):
    """The audit's Monte Carlo takes the audited events in event order, so two
    fresh surrogates (each with its own audit context) report the same audited
    detections on the same events, although the routing kernel lists the
    audited rows in whatever order its threads reach them."""
    sg, es = trained
    path = str(tmp_path / "net.fd2sg")
    sg.save(path)
    res = []
    for _ in range(2):
        with sgm.Surrogate(hidden=256, batch=2048) as s2:
            s2.load(path)
            res.append(_run(es, s2, audit=0.2)["stats"])
    a, b = res
    assert a["audit_events"] == b["audit_events"] > 0
    assert a["audit_mc_detected"] == b["audit_mc_detected"]
    assert a["audit_photons"] == b["audit_photons"]
    assert abs(a["audit_sg_expected"] - b["audit_sg_expected"]) <= 1e-9 * a["audit_sg_expected"]
