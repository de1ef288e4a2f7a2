"""CPU tests of the image-quality oracle (MTF, NNPS, DQE) and of the analysis
entry points' argument checks (no GPU calls).

The oracle is pinned to closed forms: a sampled Gaussian point response has
MTF exp(-2 pi^2 sigma^2 f^2); uncorrelated Poisson pixels have a flat
NNPS = pixel^2 / mean; a blurred white field has NNPS = pixel^2 / mean times
the squared transfer function of the blur; and a simulated detector whose
x-rays give a random number g of light quanta, each displaced by the same
Gaussian blur T, has DQE(f) = m1^2 T^2 / (m1 + (m2 - m1) T^2), m1 and m2
the moments of g (the Swank factor m1^2/m2 as f -> 0).
"""
import ctypes

import numpy as np
import pytest

import hybridmantis_b200 as hb
from hybridmantis_b200 import analysis
from oracle import analysis_oracle as ao

from imaging_helpers import simulate_detector


def gaussian_image(n, sigma, cx, cy):
    i = np.arange(n)[:, None]
    j = np.arange(n)[None, :]
    return np.exp(-((i - cx) ** 2 + (j - cy) ** 2) / (2 * sigma * sigma))


def test_oracle_mtf_of_gaussian_matches_closed_form():
    n, sigma, pix = 257, 3.0, 2.0
    img = gaussian_image(n, sigma, 128.3, 127.6)
    freq, mx, my, mr = ao.mtf(img, pix, 60)
    f_px = np.arange(60) / n  # cycles per pixel
    expect = np.exp(-2 * np.pi ** 2 * sigma ** 2 * f_px ** 2)
    assert np.allclose(mx, expect, atol=1e-9)
    assert np.allclose(my, expect, atol=1e-9)
    assert freq[1] == pytest.approx(1000.0 / (n * pix))
    # the radial average sits between the ring's inner and outer values
    k = np.arange(1, 40)
    lo = np.exp(-2 * np.pi ** 2 * sigma ** 2 * ((k + 0.5) / n) ** 2)
    hi = np.exp(-2 * np.pi ** 2 * sigma ** 2 * ((k - 0.5) / n) ** 2)
    assert np.all(mr[k] >= lo - 1e-9) and np.all(mr[k] <= hi + 1e-9)
    assert mr[0] == pytest.approx(1.0)


def test_oracle_nnps_of_poisson_pixels_is_flat():
    rng = np.random.default_rng(5)
    mean, pix = 400.0, 1.5
    imgs = rng.poisson(mean, (6, 96, 80)).astype(np.float64)
    expect = (pix / 1000.0) ** 2 / mean
    for stack in (imgs, imgs[:1]):
        freq, nr, n2, m = ao.nnps(stack, pix, 32, 8, 4, 2, 2, 17)
        assert m == pytest.approx(mean, rel=0.01)
        assert np.mean(nr[1:]) == pytest.approx(expect, rel=0.05)
        assert freq[1] == pytest.approx(1000.0 / (32 * pix))


def test_oracle_nnps_of_blurred_noise_follows_the_blur():
    rng = np.random.default_rng(9)
    n, R, mean = 128, 64, 1000.0
    k = np.fft.fftfreq(n)
    T = np.exp(-2 * np.pi ** 2 * 1.5 ** 2 * (k[:, None] ** 2 + k[None, :] ** 2))
    imgs = []
    for _ in range(8):
        w = rng.normal(0.0, np.sqrt(mean), (n, n))
        imgs.append(mean + np.real(np.fft.ifft2(np.fft.fft2(w) * T)))
    freq, nr, n2, m = ao.nnps(np.array(imgs), 1.0, R, 0, 0, 2, 2, 20)
    f = np.arange(20) / R
    expect = 1e-6 / mean * np.exp(-4 * np.pi ** 2 * 1.5 ** 2 * f ** 2)
    assert np.allclose(nr[2:12], expect[2:12], rtol=0.15)


def test_dqe_of_an_ideal_counter_is_one():
    # Poisson x-rays, one count each, no blur: MTF = 1, NNPS = 1/q
    q = 2.5e5
    assert np.allclose(ao.dqe(np.ones(5), np.full(5, 1.0 / q), q), 1.0)
    assert np.allclose(analysis.dqe(np.ones(5), np.full(5, 1.0 / q), q), 1.0)


def test_prf_file_reader_round_trips_the_writer(tmp_path):
    p = hb.default_params()
    g = hb.params_to_geometry(p)
    xd, yd = hb.prf_dims(g)
    rng = np.random.default_rng(2)
    img = rng.integers(0, 50, (xd, yd)).astype(np.uint64)
    phs = np.zeros(p.num_bins, np.int32)
    hb.write_output_files(p, g, img, phs, 10.0, str(tmp_path))
    name = [f for f in tmp_path.iterdir() if f.name.startswith("myimage_")][0]
    back = analysis.read_prf_file(str(name))
    assert back.shape == (xd, yd)
    assert np.allclose(back, img / 10.0, atol=5e-5)


def test_analysis_entry_points_check_arguments():
    lib = hb.load()
    img = np.ones((8, 8))
    out = np.zeros(8)
    vp = lambda a: ctypes.c_void_p(a.ctypes.data)  # noqa: E731
    assert lib.fd2_mtf(0, None, 8, 8, 1.0, 4, None, None, None, None) == 1
    assert lib.fd2_mtf(0, vp(img), 8, 8, 1.0, 6, None, None, None, None) == 1      # n_freq > N/2 + 1
    assert lib.fd2_mtf(0, vp(img), 8, 8, 0.0, 4, None, None, None, None) == 1      # pixel
    zero = np.zeros((8, 8))
    assert lib.fd2_mtf(0, vp(zero), 8, 8, 1.0, 4, None, None, None, None) == 1     # no signal
    assert lib.fd2_nnps(0, vp(img), 1, 8, 8, 1.0, 4, 0, 0, 3, 1, 3, vp(out), vp(out), None, None) == 1  # off image
    assert lib.fd2_nnps(0, vp(img), 1, 8, 8, 1.0, 4, 0, 0, 2, 2, 4, vp(out), vp(out), None, None) == 1  # n_freq
    assert lib.fd2_nnps(0, vp(img), 0, 8, 8, 1.0, 4, 0, 0, 2, 2, 3, vp(out), vp(out), None, None) == 1  # no images


def test_oracle_dqe_of_a_simulated_detector_matches_theory():
    rng = np.random.default_rng(1)
    # sigma small against the 128-pixel regions: the regions' rectangular
    # window blurs the spectrum over ~1 frequency bin (leakage), which biases
    # a spectrum only a few bins wide
    W, R, px, sigma = 384, 128, 3.0, 1.5
    pen, _ = simulate_detector(rng, 3000, W, sigma, pencil=True)
    pad = np.zeros((2 * R, 2 * R))
    pad[:, :] = pen[W // 2 - R:W // 2 + R, W // 2 - R:W // 2 + R]
    _, mx, my, _ = ao.mtf(pad, px, R // 2 + 1)
    mtf = 0.5 * (mx + my)
    n_x, imgs, gs = 4000, [], []
    for _ in range(48):
        img, g = simulate_detector(rng, n_x, W, sigma)
        imgs.append(img)
        gs.append(g)
    _, nr, _, m = ao.nnps(np.array(imgs), px, R, (W - R) // 2, (W - R) // 2, 1, 1, R // 4)
    q = n_x / (W * px / 1000.0) ** 2
    k = np.arange(1, 24)
    d = ao.dqe(mtf[2 * k], nr[k], q)
    g = np.concatenate(gs).astype(float)
    m1, m2 = g.mean(), (g * g).mean()
    T = np.exp(-2 * np.pi ** 2 * sigma ** 2 * (k / R) ** 2)
    theory = m1 * m1 * T * T / (m1 + (m2 - m1) * T * T)
    assert m == pytest.approx(q * m1 * (px / 1000.0) ** 2, rel=0.02)
    # each ring holds ~8 k frequency points x 48 images
    assert np.allclose(d[:20], theory[:20], rtol=0.15), (d, theory)
    assert np.mean(d[:6]) == pytest.approx(np.mean(theory[:6]), rel=0.08)
    assert theory[0] == pytest.approx(m1 * m1 / m2, rel=0.01)  # the Swank factor
