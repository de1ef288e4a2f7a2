"""Monte Carlo statistics used by the parity tests (FP64, numpy)."""
import numpy as np


def phs_moments(per_primary):
    """PHS mean and Swank factor over histories with >= 1 detected photon,
    with standard errors from the delta method."""
    c = np.asarray(per_primary, dtype=np.float64)
    c = c[c > 0]
    n = len(c)
    m1, m2 = c.mean(), (c * c).mean()
    swank = m1 * m1 / m2
    se_mean = c.std(ddof=1) / np.sqrt(n)
    # Swank = m1^2 / m2: gradient (2 m1 / m2, -m1^2 / m2^2) on the sample means
    g = np.array([2 * m1 / m2, -m1 * m1 / (m2 * m2)])
    cov = np.cov(np.vstack([c, c * c]), ddof=1) / n
    se_swank = float(np.sqrt(g @ cov @ g))
    return {"n": n, "mean": m1, "se_mean": se_mean, "swank": swank, "se_swank": se_swank}


def z_binomial(k1, n1, k2, n2):
    p1, p2 = k1 / n1, k2 / n2
    p = (k1 + k2) / (n1 + n2)
    se = np.sqrt(max(p * (1 - p) * (1 / n1 + 1 / n2), 1e-300))
    return (p1 - p2) / se


def radial_profile(image, cx, cy, edges):
    """Counts of a PRF image in radial rings (pixel centres) around (cx, cy)."""
    img = np.asarray(image, dtype=np.float64)
    ii, jj = np.meshgrid(np.arange(img.shape[0]) + 0.5, np.arange(img.shape[1]) + 0.5, indexing="ij")
    r = np.hypot(ii - cx, jj - cy)
    return np.histogram(r.ravel(), bins=edges, weights=img.ravel())[0]


def poisson_chi2(a, b):
    """Chi-square of two independent count vectors (same expected totals),
    over bins where either is non-zero; returns (chi2, dof)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    m = (a + b) > 0
    chi2 = float((((a - b) ** 2) / (a + b))[m].sum())
    return chi2, int(m.sum())
