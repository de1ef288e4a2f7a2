"""The explicit column lattices (fd2_options.column_grid = 1 square, 2
hexagonal) on the GPU.

The lattice has no counterpart in the reference (whose next column is drawn
at random after each crossing), so it is checked against its own CPU oracle
(oracle/grid_oracle.c, double precision, another random stream) in
distribution, and against a closed form:
- fate fractions, PHS mean and Swank factor, and the radial PRF agree with
  the oracle on the same events and photon counts within Monte Carlo error;
- with equal column and gap indices the walls vanish: with a black top and
  no absorption the detected fraction is the straight-line solid-angle
  integral;
- results are bitwise independent of the launch shape;
- the lattice refuses what it does not support (several geometries, the
  reference-arithmetic replay, label mode).
"""
import numpy as np
import pytest

import hybridmantis_b200 as hb
from oracle import grid_oracle as go

from gpu_helpers import c0_events, report
from mcstats import phs_moments, poisson_chi2, radial_profile, z_binomial
from test_grid_cpu import straight_line_detected_fraction

pytestmark = pytest.mark.gpu

FATES = ["detected", "abs_top", "abs_bulk", "lost", "capped"]


def run_grid(es, N, gap=0.5, kind=1, **kw):
    t = hb.OpticalTransport(es.params, count_mode=hb.COUNT_GIVEN, column_grid=kind, grid_gap_um=gap, **kw)
    t.submit(es, nphot=N)
    t.run_sync()
    return t


@pytest.mark.parametrize("kind", [1, 2])
def test_lattice_matches_its_oracle(require_gpu, kind):
    es, N = c0_events(80, seed=12)
    p = es.params
    n = int(N.sum())
    with run_grid(es, N, seed=21, kind=kind) as t:
        c = t.counters()
        prim = t.detected_per_primary()
        img = t.prf()
    xd, yd = img.shape
    oc, oimg, oprim = go.run(go.geometry(p, 0.5, xd, yd, kind), es.x_um, es.y_um, es.z_um, es.hist, N, p.num_hist,
                             seed=5)
    assert c["generated"] == oc["generated"] == n
    zs = {k: float(z_binomial(c[k], n, oc[k], n)) for k in FATES}
    g, o = phs_moments(prim), phs_moments(oprim)
    z_mean = (g["mean"] - o["mean"]) / np.hypot(g["se_mean"], o["se_mean"])
    z_swank = (g["swank"] - o["swank"]) / np.hypot(g["se_swank"], o["se_swank"])
    edges = np.array([0, 2, 4, 6, 8, 11, 15, 20, 30, 45, 70, 110, 170, 260, 400])
    chi2, dof = poisson_chi2(radial_profile(img, 250.5, 250.5, edges), radial_profile(oimg, 250.5, 250.5, edges))
    rep = {"z_fates": zs, "gpu": {k: c[k] / n for k in FATES}, "oracle": {k: oc[k] / n for k in FATES},
           "z_mean": z_mean, "z_swank": z_swank, "radial_chi2": chi2, "dof": dof}
    report(f"grid_vs_oracle_c0_lattice{kind}", rep)
    for k, z in zs.items():
        assert abs(z) < 5.0, rep
    assert abs(z_mean) < 5.0 and abs(z_swank) < 5.0, rep
    assert chi2 < dof + 6 * np.sqrt(2 * dof), rep


@pytest.mark.parametrize("kind", [1, 2])
def test_index_matched_lattice_is_invisible(require_gpu, kind):
    p = hb.default_params()
    p.radius, p.n_col, p.n_gap, p.top_absfrac, p.bulk_abs, p.beta = 5.0, 1.8, 1.8, 1.0, 0.0, 0.3
    es = hb.synth_events(0, 1, 1)
    es.params = p
    x0, y0, z0 = 250.5, 250.5, 30.0
    es.x_um[:] = x0
    es.y_um[:] = y0
    es.z_um[:] = z0
    n = 600_000
    with run_grid(es, np.array([n], np.int32), kind=kind) as t:
        c = t.counters()
    expect = straight_line_detected_fraction(x0, y0, z0 + p.det_height / 2, p.det_x)
    got = c["detected"] / n
    assert got == pytest.approx(expect, abs=4 * np.sqrt(expect * (1 - expect) / n)), (got, expect)
    assert c["abs_bulk"] == 0 and c["capped"] == 0


@pytest.mark.parametrize("kind", [1, 2])
def test_lattice_results_independent_of_launch_shape(require_gpu, kind):
    es, N = c0_events(32, seed=3)
    outs = []
    for kw in (dict(), dict(block_size=256, chunk=8, refill=8, prf_window=0), dict(block_size=128, use_graph=False)):
        with run_grid(es, N, seed=4, kind=kind, **kw) as t:
            c = t.counters()
            c.pop("photon_distance")
            outs.append((c, t.detected_per_primary().copy(), t.prf().copy()))
    for c, prim, img in outs[1:]:
        assert c == outs[0][0]
        assert np.array_equal(prim, outs[0][1]) and np.array_equal(img, outs[0][2])


def test_lattice_refuses_what_it_does_not_support(require_gpu):
    es, N = c0_events(4, seed=1)
    with run_grid(es, N) as t:
        g = hb.params_to_geometry(es.params)
        with pytest.raises(hb.Fd2Error) as err:
            t.set_geometries([g, g])
        assert err.value.status == 7
        with pytest.raises(hb.Fd2Error) as err:
            t.replay(int(N.sum()))
        assert err.value.status == 7
    with pytest.raises(hb.Fd2Error) as err:
        hb.OpticalTransport(es.params, column_grid=1, radial_bins=16)
    assert err.value.status == 1
