"""A simulated imaging detector for the DQE tests (numpy, no GPU)."""
import numpy as np


def simulate_detector(rng, n_xrays, W, sigma, pencil=False):
    """x-rays at the field's centre or uniform over W x W pixels; each gives
    g ~ Poisson(Gamma(4, 50/4)) quanta, each displaced by N(0, sigma^2)
    pixels, counted in unit pixels.  Returns (image, gains)."""
    g = rng.poisson(rng.gamma(4.0, 12.5, n_xrays))
    if pencil:
        pos = np.full((n_xrays, 2), W / 2.0)
    else:
        pos = rng.uniform(0, W, (n_xrays, 2))
    p = np.repeat(pos, g, axis=0) + rng.normal(0.0, sigma, (int(g.sum()), 2))
    img, _, _ = np.histogram2d(p[:, 0], p[:, 1], bins=W, range=[[0, W], [0, W]])
    return img, g
