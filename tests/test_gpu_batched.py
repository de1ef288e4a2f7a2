"""Batched geometries (configuration 2: 64 detector geometries, each with its
own x-rays, transported in one launch of the multi-geometry kernel) on the GPU:
- batching does not change a geometry's results: its tallies equal, bit for
  bit, a run of that geometry's events alone through the same kernel (the same
  photons: random streams keyed by the global event index, `event_base`
  aligning the two); against the single-geometry kernel, a separate
  compilation of the same walk, they differ only where FP rounding differs
  (observed: up to 2 photons in 10^4);
- each geometry against the CPU oracle within Monte Carlo error (fate
  fractions, PHS mean and Swank factor over its own histories).
"""
import numpy as np
import pytest

import hybridmantis_b200 as hb
from oracle import pyoracle as po

from gpu_helpers import geometry_params, given_counts, oracle_geometry, report
from mcstats import phs_moments, z_binomial

pytestmark = pytest.mark.gpu
FATES = ["detected", "abs_top", "abs_bulk", "lost"]
ORACLE_FATES = {"detected": 1, "abs_top": 2, "abs_bulk": 3, "lost": 4}


@pytest.fixture(scope="module")
def batch(require_gpu):
    es = hb.synth_events(2, 40, 17)
    N = given_counts(es, 5)
    with hb.OpticalTransport(es.params, count_mode=hb.COUNT_GIVEN, seed=99) as t:
        t.set_geometries(es.geometries)
        t.submit(es, nphot=N)
        t.run_sync()
        out = {"counters": [t.counters(g) for g in range(len(es.geometries))],
               "prf": [t.prf(g).copy() for g in range(len(es.geometries))],
               "prim": t.detected_per_primary().copy()}
    return es, N, out


@pytest.mark.parametrize("g", [0, 17, 40, 63])
def test_batched_geometry_equals_its_single_run(batch, g):
    es, N, out = batch
    idx = np.nonzero(es.geom == g)[0]
    a, b = int(idx[0]), int(idx[-1]) + 1
    assert np.all(es.geom[a:b] == g)
    cb = dict(out["counters"][g])
    cb.pop("photon_distance")
    h = np.unique(es.hist[a:b]) - 1
    # alone, through the multi-geometry kernel (a second geometry without events selects it)
    other = es.geometries[(g + 1) % len(es.geometries)]
    for geoms in ([es.geometries[g], other], [es.geometries[g]]):
        with hb.OpticalTransport(es.params, count_mode=hb.COUNT_GIVEN, seed=99, event_base=a) as t:
            t.set_geometries(geoms)
            t.submit_events_um(es.x_um[a:b], es.y_um[a:b], es.z_um[a:b], es.e_ev[a:b], es.hist[a:b], nphot=N[a:b],
                               geom=np.zeros(b - a, np.uint16))
            t.run_sync()
            c = dict(t.counters(0))
            c.pop("photon_distance")
            prf = t.prf(0)
            prim = t.detected_per_primary()
        if len(geoms) == 2:
            assert c == cb
            assert np.array_equal(prf, out["prf"][g])
            assert np.array_equal(prim[h], out["prim"][h])
        else:
            # the single-geometry kernel: the same photons, FP rounding of another compilation
            n = c["generated"]
            assert n == cb["generated"]
            for k in FATES:
                assert abs(c[k] - cb[k]) <= max(10, 1e-3 * n), (k, c, cb)


@pytest.mark.parametrize("g", [5, 50])
def test_batched_geometry_matches_the_oracle(batch, g):
    es, N, out = batch
    idx = np.nonzero(es.geom == g)[0]
    a, b = int(idx[0]), int(idx[-1]) + 1
    p = geometry_params(es, g)
    orc = po.run_oracle(oracle_geometry(p), es.x_um[a:b].astype(np.float64), es.y_um[a:b].astype(np.float64),
                        es.z_um[a:b].astype(np.float64), es.hist[a:b], N[a:b], prim_size=p.num_hist)
    n = int(N[a:b].sum())
    c = out["counters"][g]
    assert c["generated"] == n == int(orc.counters[0])
    zs = {k: float(z_binomial(c[k], n, int(orc.counters[i]), n)) for k, i in ORACLE_FATES.items()}
    h = np.unique(es.hist[a:b]) - 1
    gm, om = phs_moments(out["prim"][h]), phs_moments(orc.per_primary[h])
    z_mean = (gm["mean"] - om["mean"]) / np.hypot(gm["se_mean"], om["se_mean"])
    z_swank = (gm["swank"] - om["swank"]) / np.hypot(gm["se_swank"], om["se_swank"])
    rep = {"geometry": g, "photons": n, "z_fates": zs, "z_mean": z_mean, "z_swank": z_swank,
           "H": p.det_height, "R": p.radius, "beta": p.beta, "top_absfrac": p.top_absfrac, "mu": p.bulk_abs}
    report(f"batched_vs_oracle_g{g}", rep)
    for z in zs.values():
        assert abs(z) < 5, rep
    assert abs(z_mean) < 5 and abs(z_swank) < 5, rep
