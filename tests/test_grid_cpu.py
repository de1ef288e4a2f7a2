"""CPU tests of the explicit column lattice's oracle (oracle/grid_oracle.c).

The lattices (fd2_options.column_grid = 1 square, 2 hexagonal) have no
counterpart in the reference; the oracle restates the lattice walk in double
precision and is pinned here, for both lattices, to geometry and to a closed
form:
- the gap flight's first column, traced cell by cell (brick by brick on the
  hexagonal lattice), equals a brute-force search over every column near
  the ray;
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


def lattice(R=5.0, gap=0.5, kind=1, **kw):
    p = hb.default_params()
    p.radius = R
    for k, v in kw.items():
        setattr(p, k, v)
    return p, go.geometry(p, gap, 501, 501, kind)


def centres(g, x0, x1, y0, y1):
    """Every column centre of the lattice in a window (brute force)."""
    p = g.pitch
    if g.lattice == 2:
        h = p * np.sqrt(3) / 2
        out = []
        for j in range(int(np.floor(y0 / h)) - 2, int(np.floor(y1 / h)) + 3):
            o = p / 2 if j % 2 else 0.0
            for i in range(int(np.floor((x0 - o) / p)) - 2, int(np.floor((x1 - o) / p)) + 3):
                out.append(((i + 0.5) * p + o, (j + 0.5) * h))
        return out
    return [((i + 0.5) * p, (j + 0.5) * p) for i in range(int(np.floor(x0 / p)) - 2, int(np.floor(x1 / p)) + 3)
            for j in range(int(np.floor(y0 / p)) - 2, int(np.floor(y1 / p)) + 3)]


def brute_first_hit(g, px, py, dx, dy, tend):
    R = g.R
    reach = tend * np.hypot(dx, dy) + g.pitch
    best = None
    qa = dx * dx + dy * dy
    for cx, cy in centres(g, px - reach, px + reach, py - reach, py + reach):
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


@pytest.mark.parametrize("kind", [1, 2])
def test_gap_flight_meets_the_nearest_column(kind):
    _, g = lattice(R=4.0, gap=0.5, kind=kind)
    rng = np.random.default_rng(3)
    hits = 0
    for _ in range(2000):
        # a start in the gap
        while True:
            px, py = rng.uniform(100, 400, 2)
            near = centres(g, px - g.pitch, px + g.pitch, py - g.pitch, py + g.pitch)
            if min(np.hypot(px - cx, py - cy) for cx, cy in near) > g.R + 1e-3:
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
    assert hits > 1000


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


@pytest.mark.parametrize("kind", [1, 2])
def test_index_matched_lattice_is_invisible(kind):
    p, g = lattice(R=5.0, gap=0.5, kind=kind, n_col=1.8, n_gap=1.8, top_absfrac=1.0, bulk_abs=0.0, beta=0.3)
    g.n_gap = 1.8
    x0, y0, z0 = 250.5, 250.5, 30.0  # 30 um above the layer's mid-plane
    n = 40000
    c, prf, prim = go.run(g, [x0], [y0], [z0], [1], [n], 1, seed=9)
    assert sum(v for k, v in c.items() if k != "generated") == c["generated"] == n
    expect = straight_line_detected_fraction(x0, y0, z0 + p.det_height / 2, p.det_x)
    got = c["detected"] / n
    assert got == pytest.approx(expect, abs=4 * np.sqrt(expect * (1 - expect) / n)), (got, expect)
    assert c["abs_bulk"] == 0 and c["capped"] == 0


@pytest.mark.parametrize("kind", [1, 2])
def test_every_photon_has_one_fate(kind):
    p, g = lattice(R=4.0, gap=0.5, kind=kind, det_height=300.0)
    es = hb.synth_events(1, 40, 5)
    N = np.full(es.n, 300, np.int32)
    c, prf, prim = go.run(g, es.x_um, es.y_um, es.z_um, es.hist, N, es.params.num_hist, seed=2)
    assert c["generated"] == N.sum()
    assert sum(v for k, v in c.items() if k != "generated") == N.sum()
    assert prim.sum() == c["detected"] >= prf.sum()
    assert 0.3 < c["detected"] / N.sum() < 0.99
