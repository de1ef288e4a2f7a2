"""CPU oracle of the surrogate network: forward pass, loss and gradients.

TEST INFRASTRUCTURE ONLY (tests/ import it to check the GPU training kernels).
The surrogate has no counterpart in the reference; this restates, in numpy
FP64, the network and loss that include/fd2_surrogate.h documents:

  x   = 2 (f - lo) / (hi - lo) - 1          (8 features; constant features -> 0)
  h1  = relu(x W1^T + b1), h2 = relu(h1 W2^T + b2), h3 = relu(h2 W3^T + b3)
  out = h3 W4^T + b4                         (25 outputs)
  mixture of Gaussian rings: PRF(r) = sum_k w_k N(r; mu_k, sd_k) / S_k per
           unit area, w = softmax(out[1..8]), mu = 50 um softplus(out[9..16]),
           sd = 10 um exp(clamp(out[17..24], -6, 4));
  radial categories: quadratic edges r_max (j/bins)^2, then r >= r_max
  L   = mean_i [ BCE(sigmoid(out0), d/N) + lambda * CE(y, q(out)) ]

With ``bf16=True`` it rounds to BF16 exactly where the GPU stores BF16 (the
network input, weights, hidden activations, the output gradient and the
hidden-layer gradients), so GPU and oracle differ only by FP32 summation
order.  With ``bf16=False`` it is plain FP64, for finite-difference checks
of the gradient formulas themselves.
"""
from __future__ import annotations

import numpy as np
from scipy.special import ndtr

K = 8
MU_SCALE, SD_SCALE = 50.0, 10.0
LOG_SD_MIN, LOG_SD_MAX = -6.0, 4.0


def bf16(a):
    """Round to the nearest BF16 (ties to even), returned as float64."""
    f = np.asarray(a, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p, hidden):
    """Public parameter vector -> (W1 [H,8], b1, W2, b2, W3, b3, W4 [25,H], b4)."""
    H = hidden
    sizes = [H * 8, H, H * H, H, H * H, H, 25 * H, 25]
    shapes = [(H, 8), (H,), (H, H), (H,), (H, H), (H,), (25, H), (25,)]
    out, o = [], 0
    for n, s in zip(sizes, shapes):
        out.append(np.asarray(p[o:o + n], np.float64).reshape(s))
        o += n
    return out


def pack(parts):
    return np.concatenate([np.asarray(a, np.float64).ravel() for a in parts])


def normalise(f, lo, hi):
    f = np.asarray(f, np.float32)
    lo = np.asarray(lo, np.float32)
    span = np.asarray(hi, np.float32) - lo
    inv = np.where(span > 0, np.float32(1.0) / np.where(span > 0, span, np.float32(1.0)), np.float32(0.5))
    return (np.float32(2.0) * (f - lo) * inv.astype(np.float32) - np.float32(1.0)).astype(np.float64)


def forward(p, hidden, f, lo, hi, bf=True):
    W1, b1, W2, b2, W3, b3, W4, b4 = unpack(p, hidden)
    r = bf16 if bf else (lambda a: np.asarray(a, np.float64))
    x = r(normalise(f, lo, hi))
    Ws = [r(W1), r(W2), r(W3), r(W4)]
    h1 = r(np.maximum(x @ Ws[0].T + b1, 0.0))
    h2 = r(np.maximum(h1 @ Ws[1].T + b2, 0.0))
    h3 = r(np.maximum(h2 @ Ws[2].T + b3, 0.0))
    out = h3 @ Ws[3].T + b4
    return out, (x, h1, h2, h3, Ws)


def _ring(mu, sd, e, inf):
    """Edge values of ring components: t, Phi, Phi_c, phi, e (arrays [..., E])."""
    t = np.where(inf, 0.0, (e - mu) / sd)
    cdf = np.where(inf, 1.0, ndtr(t))
    ccdf = np.where(inf, 0.0, ndtr(-t))
    pdf = np.where(inf, 0.0, np.exp(-0.5 * t * t) / np.sqrt(2 * np.pi))
    return t, cdf, ccdf, pdf, np.where(inf, 0.0, e)


def point_loss(out, t, y, bins, r_max, lam):
    """Loss of every row and dL/dout (rows of 25); rows whose y is all zero
    have no radial term.  Radial model: mixture of Gaussian rings, component
    k's radial density r N(r; mu_k, sd_k) / S_k on r >= 0; bin masses
    M(a, b) = mu [Phi(t_b) - Phi(t_a)] + sd [phi(t_a) - phi(t_b)]; quadratic
    bin edges r_max (j / bins)^2 and a last category beyond r_max."""
    n = out.shape[0]
    z = out[:, 0]
    p = 1.0 / (1.0 + np.exp(-z))
    sp_neg = np.maximum(-z, 0) + np.log1p(np.exp(-np.abs(z)))
    sp_pos = np.maximum(z, 0) + np.log1p(np.exp(-np.abs(z)))
    ld = t * sp_neg + (1 - t) * sp_pos
    g = np.zeros_like(out)
    g[:, 0] = p - t
    a = out[:, 1:1 + K]
    w = np.exp(a - a.max(1, keepdims=True))
    w /= w.sum(1, keepdims=True)
    om = out[:, 1 + K:1 + 2 * K]
    mu = MU_SCALE * (np.maximum(om, 0) + np.log1p(np.exp(-np.abs(om))))
    dmu = MU_SCALE / (1.0 + np.exp(-om))
    ls = out[:, 1 + 2 * K:1 + 3 * K]
    clamped = (ls < LOG_SD_MIN) | (ls > LOG_SD_MAX)
    sd = SD_SCALE * np.exp(np.clip(ls, LOG_SD_MIN, LOG_SD_MAX))
    edges = r_max * (np.arange(bins + 1) / bins) ** 2
    E = np.concatenate([edges, [0.0]])                       # bins + 2 edges, the last is +inf
    inf = np.zeros(bins + 2, bool)
    inf[-1] = True
    mu3, sd3 = mu[:, :, None], sd[:, :, None]
    tt, cdf, ccdf, pdf, ee = _ring(mu3, sd3, E[None, None, :], inf[None, None, :])
    tlo, thi = tt[:, :, :-1], tt[:, :, 1:]
    dphi = np.maximum(np.where((tlo >= 0) & ~inf[None, None, :-1], ccdf[:, :, :-1] - ccdf[:, :, 1:],
                               cdf[:, :, 1:] - cdf[:, :, :-1]), 0.0)
    plo, phi_ = pdf[:, :, :-1], pdf[:, :, 1:]
    elo, ehi = ee[:, :, :-1], ee[:, :, 1:]
    M = np.maximum(mu3 * dphi + sd3 * (plo - phi_), 0.0)       # [n, K, bins+1]
    dM_mu = dphi + (elo * plo - ehi * phi_) / sd3
    dM_sd = (plo - phi_) + (tlo * elo * plo - thi * ehi * phi_) / sd3
    t0 = -mu / sd
    c0 = ndtr(-t0)
    p0 = np.exp(-0.5 * t0 * t0) / np.sqrt(2 * np.pi)
    S = np.maximum(mu * c0 + sd * p0, 1e-30)
    q = (w[:, :, None] * M / S[:, :, None]).sum(1)             # [n, bins+1]
    qe = q + 1e-12
    has = y.sum(1) > 0
    lr = -(y * np.log(qe)).sum(1)
    c = y / qe
    A1 = (c[:, None, :] * M).sum(2)
    Amu = (c[:, None, :] * dM_mu).sum(2)
    Asd = (c[:, None, :] * dM_sd).sum(2)
    gw = -A1 / S
    f = w / S
    gmu = -f * (Amu - A1 * c0 / S)
    gsd = -f * (Asd - A1 * p0 / S)
    wg = (w * gw).sum(1, keepdims=True)
    g[:, 1:1 + K] = lam * w * (gw - wg)
    g[:, 1 + K:1 + 2 * K] = lam * dmu * gmu
    g[:, 1 + 2 * K:] = np.where(clamped, 0.0, lam * sd * gsd)
    g[~has, 1:] = 0.0
    lr = np.where(has, lr, 0.0)
    return ld + lam * lr, g, ld, lr


def labels(photons, detected, radial):
    photons = np.asarray(photons, np.float64)
    t = np.where(photons > 0, np.asarray(detected, np.float64) / np.maximum(photons, 1), 0.0)
    r = np.asarray(radial, np.float64)
    tot = r.sum(1, keepdims=True)
    y = np.where(tot > 0, r / np.maximum(tot, 1), 0.0)
    return t.astype(np.float32).astype(np.float64), y.astype(np.float32).astype(np.float64)


def loss_grad(p, hidden, f, lo, hi, photons, detected, radial, bins=64, radial_max=200.0, lam=1.0, bf=True):
    """Mean loss and its gradient (public parameter order)."""
    W1, b1, W2, b2, W3, b3, W4, b4 = unpack(p, hidden)
    r = bf16 if bf else (lambda a: np.asarray(a, np.float64))
    out, (x, h1, h2, h3, Ws) = forward(p, hidden, f, lo, hi, bf)
    if bf:
        out = out.astype(np.float32).astype(np.float64)
    t, y = labels(photons, detected, radial)
    L, g, _, _ = point_loss(out, t, y, bins, radial_max, lam)
    n = out.shape[0]
    dout = r(g / n)
    dW4 = dout.T @ h3
    db4 = dout.sum(0)
    d3 = r((dout @ Ws[3]) * (h3 > 0))
    dW3 = d3.T @ h2
    db3 = d3.sum(0)
    d2 = r((d3 @ Ws[2]) * (h2 > 0))
    dW2 = d2.T @ h1
    db2 = d2.sum(0)
    d1 = r((d2 @ Ws[1]) * (h1 > 0))
    dW1 = d1.T @ x
    db1 = d1.sum(0)
    return float(L.mean()), pack([dW1, db1, dW2, db2, dW3, db3, dW4, db4])


def loss_only(p, hidden, f, lo, hi, photons, detected, radial, bins=64, radial_max=200.0, lam=1.0):
    out, _ = forward(p, hidden, f, lo, hi, bf=False)
    t, y = labels(photons, detected, radial)
    L, _, _, _ = point_loss(out, t, y, bins, radial_max, lam)
    return float(L.mean())
