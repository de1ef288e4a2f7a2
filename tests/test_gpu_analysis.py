"""fd2_mtf / fd2_nnps on the GPU against the numpy oracle, and DQE.

Parity: FP64 direct DFTs on the GPU against numpy's FFT on the same images,
to 1e-9 relative: random images, a transported PRF, and flat-field images
of the transport.  Physics: (1) a simulated detector whose x-rays give
Poisson-Gamma numbers of quanta, each blurred by the same Gaussian, has
DQE(f) = m1^2 T^2 / (m1 + (m2 - m1) T^2), the Swank factor as f -> 0, and
the GPU pipeline (fd2_mtf, fd2_nnps) recovers it; (2) for the config-1
detector (made 1.5 mm wide) the DQE from a pencil-beam MTF and 64 flat
fields is reported beside the Swank factor of its PHS.  Its PRF has a halo
of inter-column hops (up to 280 um each) that reaches the field's edges, so
the images are not shift-invariant at the lowest frequencies and the DQE
there is not a test of DQE(0) = Swank; it must fall with frequency.
"""
import numpy as np
import pytest

import hybridmantis_b200 as hb
from hybridmantis_b200 import analysis
from oracle import analysis_oracle as ao

from gpu_helpers import report
from imaging_helpers import simulate_detector

pytestmark = pytest.mark.gpu


def test_mtf_matches_oracle(require_gpu):
    rng = np.random.default_rng(4)
    for shape, k in (((101, 73), 40), ((64, 64), 33)):
        img = rng.gamma(2.0, 3.0, shape)
        img[shape[0] // 2, shape[1] // 3] += 500.0
        got = analysis.mtf(img, 1.5, k)
        freq, mx, my, mr = ao.mtf(img, 1.5, k)
        assert np.allclose(got["freq"], freq, rtol=1e-12)
        for a, b in ((got["mtf_x"], mx), (got["mtf_y"], my), (got["mtf_r"], mr)):
            assert np.allclose(a, b, rtol=1e-9, atol=1e-12)


def test_nnps_matches_oracle(require_gpu):
    rng = np.random.default_rng(8)
    imgs = rng.poisson(300.0, (3, 128, 96)).astype(np.float64)
    for stack in (imgs, imgs[:1]):
        got = analysis.nnps(stack, 2.0, 32, 5, 7, 3, 2, 17)
        freq, nr, n2, m = ao.nnps(stack, 2.0, 32, 5, 7, 3, 2, 17)
        assert got["mean_signal"] == pytest.approx(m, rel=1e-12)
        assert np.allclose(got["nnps_r"], nr, rtol=1e-9, atol=0)
        assert np.allclose(got["nnps_2d"], n2, rtol=1e-9, atol=1e-20)


def test_mtf_of_a_transported_point_response(require_gpu):
    es = hb.synth_events(1, 3000, 21)
    x, y, z = es.to_cm()
    with hb.OpticalTransport(es.params, seed=3) as t:
        t.submit_events(x, y, z, es.e_ev.astype(np.float64), es.hist)
        t.run_sync()
        img = t.prf().astype(np.float64)
    got = analysis.mtf(img, 1.0, 100)
    freq, mx, my, mr = ao.mtf(img, 1.0, 100)
    assert np.allclose(got["mtf_x"], mx, rtol=1e-9, atol=1e-12)
    assert np.allclose(got["mtf_r"], mr, rtol=1e-9, atol=1e-12)
    assert got["mtf_x"][0] == pytest.approx(1.0)
    assert np.all(np.diff(got["mtf_r"][:40]) < 0.02)  # falls with frequency


def test_dqe_of_a_simulated_detector(require_gpu):
    rng = np.random.default_rng(1)
    W, R, px, sigma = 384, 128, 3.0, 1.5
    pen, _ = simulate_detector(rng, 3000, W, sigma, pencil=True)
    m = analysis.mtf(pen[W // 2 - R:W // 2 + R, W // 2 - R:W // 2 + R], px, R // 2 + 1)
    mtf = 0.5 * (m["mtf_x"] + m["mtf_y"])
    n_x, imgs, gs = 4000, [], []
    for _ in range(48):
        img, g = simulate_detector(rng, n_x, W, sigma)
        imgs.append(img)
        gs.append(g)
    nn = analysis.nnps(np.array(imgs), px, R, n_freq=R // 4)
    q = n_x / (W * px / 1000.0) ** 2
    k = np.arange(1, 24)
    d = analysis.dqe(mtf[2 * k], nn["nnps_r"][k], q)
    g = np.concatenate(gs).astype(float)
    m1, m2 = g.mean(), (g * g).mean()
    T = np.exp(-2 * np.pi ** 2 * sigma ** 2 * (k / R) ** 2)
    theory = m1 * m1 * T * T / (m1 + (m2 - m1) * T * T)
    assert np.allclose(d[:20], theory[:20], rtol=0.15), (d, theory)
    assert np.mean(d[:6]) == pytest.approx(np.mean(theory[:6]), rel=0.08)


def test_dqe_of_the_config1_detector(require_gpu):
    W, px, R = 1503.0, 3, 256
    es = hb.synth_events(1, 20000, 31)
    pencil, _ = analysis.flat_field(es, W, px, 0)
    sh = np.float32(W / 2.0 - es.params.det_x / 2.0)
    pencil.x_um[:] = es.x_um + sh  # the pencil beam at the wide detector's centre
    pencil.y_um[:] = es.y_um + sh
    x, y, z = pencil.to_cm()
    with hb.OpticalTransport(pencil.params, seed=5) as t:
        t.submit_events(x, y, z, pencil.e_ev.astype(np.float64), pencil.hist)
        t.run_sync()
        prf = t.prf().astype(np.float64)
    # zero-padded to 2 R: every second MTF frequency is an NNPS frequency
    pad = np.zeros((2 * R, 2 * R))
    pad[:prf.shape[0], :prf.shape[1]] = prf
    m = analysis.mtf(pad, float(px), R // 2 + 1)
    mtf = 0.5 * (m["mtf_x"] + m["mtf_y"])
    imgs, swank, qs = [], [], []
    for r in range(64):
        ff, q = analysis.flat_field(hb.synth_events(1, 5000, 100 + r), W, px, 7 + r)
        fx, fy, fz = ff.to_cm()
        with hb.OpticalTransport(ff.params, seed=50 + r) as t:
            t.submit_events(fx, fy, fz, ff.e_ev.astype(np.float64), ff.hist)
            t.run_sync()
            imgs.append(t.prf().astype(np.float64))
            swank.append(t.phs_stats()["swank"])
        qs.append(q)
    imgs = np.array(imgs)
    nn = analysis.nnps(imgs, float(px), R, rois_x=1, rois_y=1, n_freq=R // 4)
    x0 = (imgs.shape[1] - R) // 2
    _, nr, _, mean = ao.nnps(imgs, float(px), R, x0, x0, 1, 1, R // 4)
    assert np.allclose(nn["nnps_r"], nr, rtol=1e-9)
    assert nn["mean_signal"] == pytest.approx(mean, rel=1e-12)
    k = np.arange(1, R // 4)
    dqe = analysis.dqe(mtf[2 * k], nn["nnps_r"][k], float(np.mean(qs)))
    rep = {"swank": float(np.mean(swank)), "freq_per_mm": nn["freq"][k][:16].tolist(), "dqe": dqe[:16].tolist(),
           "mtf": mtf[2 * k][:16].tolist(), "mean_signal": nn["mean_signal"], "fluence_per_mm2": float(np.mean(qs))}
    report("dqe_config1", rep)
    assert np.all(np.isfinite(dqe)) and np.all(dqe > 0), rep
    assert np.mean(dqe[40:60]) < 0.2 * np.mean(dqe[:3]), rep
