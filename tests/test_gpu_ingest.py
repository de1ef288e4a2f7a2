"""Streaming event ingest (fd2_ingest_*) against one submission of the stream.

The EDE tally flushes its buffer to fastDETECT2 whenever it is full
(main/hybridMANTIS_tallyEnergyDepositionEvents.f:171-310); the ingest keeps
that stream-of-buffers shape but transports batch k while batch k+1 is being
filled and copied.  Event indices run on across batches and the run counter
is fixed for the stream, so every tally must equal, bit for bit, the tallies
of fd2_submit_events + fd2_run over the concatenated stream, whatever the
batch size and however the pushes are cut.
"""
import numpy as np
import pytest

import hybridmantis_b200 as hb

pytestmark = pytest.mark.gpu


def tallies(t):
    return {"prf": t.prf(), "per_primary": t.detected_per_primary(), "phs": t.phs(), "counters": t.counters(),
            "phs_stats": t.phs_stats()}


def assert_same(a, b):
    assert np.array_equal(a["prf"], b["prf"])
    assert np.array_equal(a["per_primary"], b["per_primary"])
    assert np.array_equal(a["phs"], b["phs"])
    for k, v in a["counters"].items():
        if k == "photon_distance":  # FP32 path lengths summed in a different order
            assert v == pytest.approx(b["counters"][k], rel=1e-6)
        else:
            assert v == b["counters"][k], k
    assert a["phs_stats"]["mean"] == b["phs_stats"]["mean"]
    assert a["phs_stats"]["swank"] == b["phs_stats"]["swank"]


@pytest.fixture(scope="module")
def stream():
    es = hb.synth_events(1, 3000, 77)
    return es, es.to_cm()


def whole(es, cm, seed=11):
    x, y, z = cm
    with hb.OpticalTransport(es.params, seed=seed) as t:
        t.submit_events(x, y, z, es.e_ev.astype(np.float64), es.hist)
        t.run_sync()
        return tallies(t)


@pytest.mark.parametrize("batch", [1000, 4096, 1 << 20])
def test_ingest_equals_one_submission(require_gpu, stream, batch):
    es, (x, y, z) = stream
    assert es.n > 5000
    ref = whole(es, (x, y, z))
    de = es.e_ev.astype(np.float64)
    with hb.OpticalTransport(es.params, seed=11) as t:
        ing = t.ingest(batch_events=batch)
        cuts = [0, 1, 17, 999, 2500, 2501, 5000, es.n]
        for a, b in zip(cuts[:-1], cuts[1:]):
            ing.push(x[a:b], y[a:b], z[a:b], de[a:b], es.hist[a:b])
        st = ing.end()
        got = tallies(t)
        tm = t.timing()
    assert st["events"] == es.n
    assert st["batches"] == -(-es.n // batch)
    assert st["photons"] == got["counters"]["generated"]
    assert tm["photons"] == st["photons"]
    assert_same(got, ref)


def test_ingest_files_equal_submissions(require_gpu, stream, tmp_path):
    es, _ = stream
    # text rows in cm / eV: the same doubles through fd2_submit_events
    hb.write_events_text(str(tmp_path / "ev.txt"), es)
    rows = np.loadtxt(tmp_path / "ev.txt")
    with hb.OpticalTransport(es.params, seed=5) as t:
        t.submit_events(rows[:, 0], rows[:, 1], rows[:, 2], rows[:, 3], rows[:, 4].astype(np.int32))
        t.run_sync()
        ref_txt = tallies(t)
    with hb.OpticalTransport(es.params, seed=5) as t:
        ing = t.ingest(batch_events=1500)
        ing.push_file(str(tmp_path / "ev.txt"))
        ing.end()
        assert_same(tallies(t), ref_txt)
    # binary planar file in um through fd2_submit_events_um
    hb.write_events_binary(str(tmp_path / "ev.bin"), es)
    with hb.OpticalTransport(es.params, seed=5) as t:
        t.submit(es)
        t.run_sync()
        ref_bin = tallies(t)
    with hb.OpticalTransport(es.params, seed=5) as t:
        ing = t.ingest(batch_events=2048, units=hb.UNITS_UM)
        ing.push_file(str(tmp_path / "ev.bin"))
        ing.end()
        assert_same(tallies(t), ref_bin)


def test_ingest_state_rules_and_bad_events(require_gpu, stream):
    es, (x, y, z) = stream
    de = es.e_ev.astype(np.float64)
    with hb.OpticalTransport(es.params, seed=3) as t:
        ing = t.ingest(batch_events=512)
        ing.push(x[:100], y[:100], z[:100], de[:100], es.hist[:100])
        for call in (t.run, t.reset_tallies, lambda: t.submit_events(x, y, z, de, es.hist)):
            with pytest.raises(hb.Fd2Error) as err:
                call()
            assert err.value.status == 7  # FD2_ERR_STATE
        with pytest.raises(hb.Fd2Error):
            t.ingest()  # one open stream per context
        with pytest.raises(hb.Fd2Error):
            ing.push_um(es.x_um[:4], es.y_um[:4], es.z_um[:4], es.e_ev[:4], es.hist[:4])  # wrong units
        # the failed push closed the stream; the context takes work again
        t.reset_tallies()
        # a history outside 1..num_hist and a negative energy: flagged, no photons
        h = es.hist[:1000].copy()
        e = de[:1000].copy()
        h[10] = 0
        e[20] = -1.0
        ing = t.ingest(batch_events=256)
        ing.push(x[:1000], y[:1000], z[:1000], e, h)
        with pytest.raises(hb.Fd2Error) as err:
            ing.end()
        assert err.value.status == 12  # FD2_ERR_BAD_EVENT
        # the context is usable after the failed stream
        t.reset_tallies()
        t.submit_events(x[:500], y[:500], z[:500], de[:500], es.hist[:500])
        t.run_sync()
        assert t.counters()["generated"] > 0


def test_ingest_overlaps_copies_with_transport(require_gpu):
    """A producer pushing a large stream in small pieces: pushes wait only
    for staging batches still in flight, and the device time is the
    transport's (copies hidden behind it)."""
    es = hb.synth_events(1, 20000, 9)
    x, y, z = es.to_cm()
    de = es.e_ev.astype(np.float64)
    with hb.OpticalTransport(es.params, seed=2) as t:
        t.submit_events(x, y, z, de, es.hist)
        t.run_sync()
        one_ms = t.timing()["pipeline_ms"]
        t.reset_tallies()
        ing = t.ingest(batch_events=8192)
        for a in range(0, es.n, 3000):
            ing.push(x[a:a + 3000], y[a:a + 3000], z[a:a + 3000], de[a:a + 3000], es.hist[a:a + 3000])
        st = ing.end()
    assert st["events"] == es.n and st["batches"] == -(-es.n // 8192)
    # the whole stream's device span stays close to one submission's run
    assert st["device_ms"] < 1.5 * one_ms + 20.0, (st, one_ms)
