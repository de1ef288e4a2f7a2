"""CPU checks of the surrogate's oracle (oracle/sg_oracle.py) and host helpers.

The analytic gradient of the FP64 oracle is checked against central finite
differences of its loss, so the GPU gradient test (test_gpu_surrogate.py)
compares against formulas that are themselves verified.
"""
import numpy as np

from oracle import sg_oracle as so
from hybridmantis_b200 import surrogate as sgm


def _problem(seed, n=24, hidden=64):
    rng = np.random.default_rng(seed)
    f = rng.uniform(0, 1, (n, 8)).astype(np.float32)
    f[:, 0] *= 300.0
    f[:, 1] *= 80.0
    lo, hi = f.min(0), f.max(0)
    npar = hidden * 8 + hidden + 2 * (hidden * hidden + hidden) + 25 * hidden + 25
    p = rng.normal(0, 0.3, npar)
    W1, b1, W2, b2, W3, b3, W4, b4 = so.unpack(p, hidden)
    W1 *= np.sqrt(2 / 8) / 0.3
    W2 *= np.sqrt(2 / hidden) / 0.3
    W3 *= np.sqrt(2 / hidden) / 0.3
    W4 *= 0.1
    b4[9:17] = np.linspace(0.05, 1.1, 8)
    b4[17:25] = np.log(np.linspace(0.2, 3.0, 8))
    p = so.pack([W1, b1, W2, b2, W3, b3, W4, b4])
    photons = rng.integers(500, 3000, n).astype(np.int32)
    detected = (photons * rng.uniform(0.1, 0.6, n)).astype(np.int32)
    radial = rng.integers(0, 40, (n, 65)).astype(np.uint32)
    radial[0] = 0  # a point without detected photons in the label
    return p, hidden, f, lo, hi, photons, detected, radial


def test_oracle_gradient_matches_finite_differences():
    p, H, f, lo, hi, ph, de, ra = _problem(1)
    L, g = so.loss_grad(p, H, f, lo, hi, ph, de, ra, bf=False)
    assert np.isclose(L, so.loss_only(p, H, f, lo, hi, ph, de, ra))
    rng = np.random.default_rng(2)
    # every output-layer parameter block and a sample of the hidden ones
    sizes = [H * 8, H, H * H, H, H * H, H, 25 * H, 25]
    starts = np.concatenate([[0], np.cumsum(sizes)])
    idx = np.concatenate([rng.choice(np.arange(starts[b], starts[b + 1]), size=min(12, sizes[b]), replace=False)
                          for b in range(8)])
    # The loss's own rounding noise (ndtr differences near 1) is ~1e-9, so
    # the steps are large.  Where the two steps disagree a ReLU kink lies
    # within them and the point is skipped; nearly all points are checked.
    checked = 0
    for i in idx:
        fds = []
        for h in (3e-3, 1e-3):
            pp, pm = p.copy(), p.copy()
            pp[i] += h
            pm[i] -= h
            fds.append((so.loss_only(pp, H, f, lo, hi, ph, de, ra) - so.loss_only(pm, H, f, lo, hi, ph, de, ra)) / (2 * h))
        if abs(fds[0] - fds[1]) > 2e-6 + 2e-3 * abs(fds[1]):
            continue
        checked += 1
        assert abs(fds[1] - g[i]) <= 2e-6 + 1e-3 * abs(fds[1]), (i, fds, g[i])
    assert checked >= 0.8 * len(idx), (checked, len(idx))


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 2 ** -9, 1.0 + 3 * 2 ** -9, -2.5, 3.0e-20], np.float32)
    r = so.bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0 + 2 ** -7 or r[1] == 1.0  # tie: to even
    assert r[2] == 1.0                             # below half an ulp
    assert r[3] == 1.0 + 2 ** -7                   # above half an ulp
    assert r[4] == -2.5
    assert abs(r[5] - 3.0e-20) / 3.0e-20 < 2 ** -8


def test_fit_edge_recovers_the_edge_survival():
    """fit_edge explains an image whose rings are spread with the sampler's
    edge weights as well as the true weights do (amplitude and length trade
    off against each other in part, so the pair itself is not unique), and
    finds nothing to explain in uniform rings."""
    n, c = 301, 150.5
    x = np.arange(n) + 0.5
    X, Y = np.meshgrid(x, x, indexing="ij")
    profile = np.exp(-np.hypot(X - c, Y - c) / 60.0)
    for amp, length in ((0.5, 30.0), (0.3, 12.0)):
        img = profile * sgm.edge_weights(amp, length, X, Y, float(n), float(n))
        fa, fl, l1u, l1f = sgm.fit_edge(img, c, c, float(n), float(n))
        assert fa > 0.0, (fa, fl)
        # the true pair's residual: the rings' own discretisation
        w = sgm.edge_weights(fa, fl, X, Y, float(n), float(n))
        assert l1f < 0.25 * l1u, (fa, fl, l1u, l1f)
        # the fitted weights reproduce the side-to-corner contrast of the image
        r = np.hypot(X - c, Y - c)
        band = (r > 120) & (r < 145)
        towards_side = band & (np.minimum(np.abs(X - c), np.abs(Y - c)) < 20)
        towards_corner = band & (np.abs(np.abs(X - c) - np.abs(Y - c)) < 20)
        truth = img[towards_side].mean() / img[towards_corner].mean()
        fitted = (profile * w)[towards_side].mean() / (profile * w)[towards_corner].mean()
        assert abs(fitted - truth) <= 0.02 * truth, (fa, fl, truth, fitted)
    fa, fl, l1u, l1f = sgm.fit_edge(profile, c, c, float(n), float(n))
    assert fa == 0.0 or l1f > 0.8 * l1u, (fa, fl, l1u, l1f)
