"""CPU tests of the explicit column lattice's oracle (oracle/grid_oracle.c).

The lattice (fd2_options.column_grid = 1) has no counterpart in the
reference; its oracle restates the lattice walk in double precision and is
pinned here to geometry and to a closed form:
- the gap flight's first column, traced cell by cell, equals a brute-force
  search over every column near the ray;
- with the column and gap indices equal the walls vanish (no reflection, no
  bending), so with a black top and no absorption a photon is detected
  exactly when its straight downward line reaches the sensor inside the
  detector: the detected fraction equals that solid-angle integral;
- every photon ends in exactly one fate.
"""
import numpy as np
import pytest

import hybridmantis_b200 as hb
from oracle import grid_oracle as go


def lattice(R=5.0, gap=0.5, **kw):
    p = hb.default_params()
    p.radius = R
    for k, v in kw.items():
        setattr(p, k, v)
    return p, go.geometry(p, gap, 501, 501)


def brute_first_hit(g, px, py, dx, dy, tend):
    p, R = g.pitch, g.R
    reach = tend * np.hypot(dx, dy) + p
    i0, i1 = int(np.floor((px - reach) / p)) - 1, int(np.floor((px + reach) / p)) + 1
    j0, j1 = int(np.floor((py - reach) / p)) - 1, int(np.floor((py + reach) / p)) + 1
    best = None
    qa = dx * dx + dy * dy
    for i in range(i0, i1 + 1):
        for j in range(j0, j1 + 1):
            cx, cy = (i + 0.5) * p, (j + 0.5) * p
            fx, fy = px - cx, py - cy
            qb = 2 * (fx * dx + fy * dy)
            qc = fx * fx + fy * fy - R * R
            disc = qb * qb - 4 * qa * qc
            if qa <= 0 or disc < 0 or qb >= 0:
                continue
            t = (-qb - np.sqrt(disc)) / (2 * qa)
            if 1e-4 < t < tend and (best is None or t < best[0]):
                best = (t, cx, cy)
    return best


def test_gap_flight_meets_the_nearest_column():
    _, g = lattice(R=4.0, gap=0.5)
    rng = np.random.default_rng(3)
    hits = 0
    for _ in range(3000):
        # a start in the gap
        while True:
            px, py = rng.uniform(100, 400, 2)
            cx = (np.floor(px / g.pitch) + 0.5) * g.pitch
            cy = (np.floor(py / g.pitch) + 0.5) * g.pitch
            if np.hypot(px - cx, py - cy) > g.R + 1e-3:
                break
        c = rng.uniform(-1, 1)
        phi = rng.uniform(-np.pi, np.pi)
        s = np.sqrt(1 - c * c)
        dx, dy = s * np.cos(phi), s * np.sin(phi)
        tend = rng.uniform(1, 300)
        a = go.first_hit(g, px, py, dx, dy, tend)
        b = brute_first_hit(g, px, py, dx, dy, tend)
        assert (a is None) == (b is None), (px, py, dx, dy, tend, a, b)
        if a:
            hits += 1
            assert a[0] == pytest.approx(b[0], rel=1e-9, abs=1e-9)
            assert a[1:] == pytest.approx(b[1:])
    assert hits > 1500


def straight_line_detected_fraction(x0, y0, h, W, n=4_000_000, seed=0):
    """P(an isotropic photon at height h above the sensor lands on the
    W x W sensor going straight down), by sampling directions."""
    rng = np.random.default_rng(seed)
    c = rng.uniform(-1, 1, n)
    phi = rng.uniform(-np.pi, np.pi, n)
    down = c < 0
    s = np.sqrt(1 - c * c)
    t = np.where(down, h / np.maximum(-c, 1e-300), 0.0)
    x = x0 + t * s * np.cos(phi)
    y = y0 + t * s * np.sin(phi)
    eps = 8.1929093e-6
    ok = down & (x >= eps) & (x <= W) & (y >= eps) & (y <= W)
    return ok.mean()


def test_index_matched_lattice_is_invisible():
    p, g = lattice(R=5.0, gap=0.5, n_col=1.8, n_gap=1.8, top_absfrac=1.0, bulk_abs=0.0, beta=0.3)
    g.n_gap = 1.8
    x0, y0, z0 = 250.5, 250.5, 30.0  # 30 um above the layer's mid-plane
    n = 40000
    c, prf, prim = go.run(g, [x0], [y0], [z0], [1], [n], 1, seed=9)
    assert sum(v for k, v in c.items() if k != "generated") == c["generated"] == n
    expect = straight_line_detected_fraction(x0, y0, z0 + p.det_height / 2, p.det_x)
    got = c["detected"] / n
    assert got == pytest.approx(expect, abs=4 * np.sqrt(expect * (1 - expect) / n)), (got, expect)
    assert c["abs_bulk"] == 0 and c["capped"] == 0


def test_every_photon_has_one_fate():
    p, g = lattice(R=4.0, gap=0.5, det_height=300.0)
    es = hb.synth_events(1, 40, 5)
    N = np.full(es.n, 300, np.int32)
    c, prf, prim = go.run(g, es.x_um, es.y_um, es.z_um, es.hist, N, es.params.num_hist, seed=2)
    assert c["generated"] == N.sum()
    assert sum(v for k, v in c.items() if k != "generated") == N.sum()
    assert prim.sum() == c["detected"] >= prf.sum()
    assert 0.3 < c["detected"] / N.sum() < 0.99
