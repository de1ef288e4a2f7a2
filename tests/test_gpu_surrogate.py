"""The learned surrogate on the GPU: gradients, label mode, training.

- The GPU forward/backward (BF16 tensor-core GEMMs, FP32 accumulation) is
  checked against the CPU oracle (oracle/sg_oracle.py), which rounds to BF16
  at the same points; the oracle's own gradient formulas are checked
  against finite differences in test_surrogate_cpu.py.
- Label mode bins every detected photon: per-point detected counts equal the
  radial histograms' totals and the ordinary run's per-history counts.
- A short training run on Monte Carlo labels beats the best constant
  predictor (mean detection fraction and pooled radial profile), which is
  the estimate available without the network.
"""
import numpy as np
import pytest

import hybridmantis_b200 as hb
from hybridmantis_b200 import surrogate as sgm
from oracle import sg_oracle as so

pytestmark = pytest.mark.gpu

BLOCKS = ["W1", "b1", "W2", "b2", "W3", "b3", "W4", "b4"]


def _random_problem(seed, n, hidden):
    rng = np.random.default_rng(seed)
    f = np.stack([rng.uniform(0, 300, n), rng.uniform(1, 80, n), rng.uniform(0, 1, n), rng.uniform(100, 600, n),
                  rng.uniform(2.5, 7.5, n), rng.uniform(0, 0.5, n), rng.uniform(0, 1, n), rng.uniform(-5, -3, n)],
                 1).astype(np.float32)
    lo, hi = f.min(0), f.max(0)
    sizes = [hidden * 8, hidden, hidden * hidden, hidden, hidden * hidden, hidden, 25 * hidden, 25]
    p = np.concatenate([rng.normal(0, s, k) for s, k in
                        zip([np.sqrt(2 / 8), 0.05, np.sqrt(2 / hidden), 0.05, np.sqrt(2 / hidden), 0.05, 0.05, 0.0],
                            sizes)]).astype(np.float32)
    b4 = p[-25:]
    b4[9:17] = np.linspace(0.05, 1.1, 8)
    b4[17:25] = np.log(np.linspace(0.2, 3.0, 8))
    photons = rng.integers(500, 3000, n).astype(np.int32)
    detected = (photons * rng.uniform(0.1, 0.6, n)).astype(np.int32)
    radial = rng.integers(0, 40, (n, 65)).astype(np.uint32)
    radial[3] = 0
    return p, f, lo, hi, photons, detected, radial


def test_gradients_match_oracle(require_gpu):
    H, n = 64, 192
    p, f, lo, hi, ph, de, ra = _random_problem(11, n, H)
    with sgm.Surrogate(hidden=H, batch=256, radial_bins=64, radial_max_um=200.0) as s:
        s.set_params(p)
        s.set_hull(lo, hi)
        assert np.array_equal(s.params(), p)
        loss, g = s.loss_grad(f, ph, de, ra)
    lo_ref, g_ref = so.loss_grad(p.astype(np.float64), H, f, lo, hi, ph, de, ra, bf=True)
    assert abs(loss - lo_ref) <= 1e-3 * abs(lo_ref), (loss, lo_ref)
    sizes = [H * 8, H, H * H, H, H * H, H, 25 * H, 25]
    o = 0
    for name, k in zip(BLOCKS, sizes):
        a, b = g[o:o + k].astype(np.float64), g_ref[o:o + k]
        o += k
        rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-12)
        cos = a @ b / max(np.linalg.norm(a) * np.linalg.norm(b), 1e-30)
        assert rel < 2e-2 and cos > 0.9995, (name, rel, cos)


def test_label_mode_counts_every_detected_photon(require_gpu):
    geoms = sgm.sample_geometries(3, seed=5)
    # depositions at the detector centre (lateral_um=0), so the comparison run
    # below can place the same photons
    f, ph, det, rad = sgm.label_points(geoms, 40, 1500, seed=9, lateral_um=0.0)
    assert f.shape == (120, 8) and rad.shape == (120, 97)
    assert np.array_equal(det, rad.sum(1).astype(np.int32))
    assert np.all(det <= ph) and 0.02 < det.sum() / ph.sum() < 0.98
    # the same photons without label mode: identical per-history counts
    p = hb.default_params(num_hist=120)
    gi = np.repeat(np.arange(3), 40).astype(np.uint16)
    cx = np.array([g.det_x / 2 for g in geoms])[gi]
    cy = np.array([g.det_y / 2 for g in geoms])[gi]
    H = np.array([g.det_height for g in geoms])[gi]
    with hb.OpticalTransport(p, count_mode=hb.COUNT_GIVEN, seed=9) as t:
        t.set_geometries(geoms)
        t.submit_events_um(cx, cy, H / 2 - f[:, 0], f[:, 1] * 1000, np.arange(1, 121), nphot=ph, geom=gi)
        t.run_sync()
        assert np.array_equal(t.detected_per_primary(), det)


def test_label_mode_single_geometry_counts_every_detected_photon(require_gpu):
    """Label mode with one geometry (the surrogate's audit runs it) uses the
    single-geometry kernel shape: its per-history counts equal a production
    run of the same photons, and its radial bins hold every detection."""
    g = sgm.sample_geometries(1, seed=15)[0]
    f, ph, det, rad = sgm.label_points([g], 96, 1500, seed=19, lateral_um=0.0)
    assert np.array_equal(det, rad.sum(1).astype(np.int32))
    p = hb.default_params(num_hist=96)
    with hb.OpticalTransport(p, count_mode=hb.COUNT_GIVEN, seed=19) as t:
        t.set_geometries([g])
        n = len(f)
        t.submit_events_um(np.full(n, g.det_x / 2), np.full(n, g.det_y / 2), g.det_height / 2 - f[:, 0],
                           f[:, 1] * 1000, np.arange(1, n + 1), nphot=ph, geom=np.zeros(n, np.uint16))
        t.run_sync()
        assert np.array_equal(t.detected_per_primary(), det)


def _constant_predictor_losses(t_tr, y_tr, t_va, y_va):
    pc = np.clip(t_tr.mean(), 1e-6, 1 - 1e-6)
    det = -(t_va * np.log(pc) + (1 - t_va) * np.log(1 - pc)).mean()
    has_tr = y_tr.sum(1) > 0
    q = y_tr[has_tr].mean(0)
    has_va = y_va.sum(1) > 0
    rad = -(y_va[has_va] * np.log(q + 1e-12)).sum(1).sum() / len(y_va)
    return det, rad


def test_training_beats_constant_predictor(require_gpu, tmp_path):
    geoms = sgm.sample_geometries(16, seed=21)
    f, ph, det, rad = sgm.label_points(geoms, 192, 1000, seed=22)
    rng = np.random.default_rng(3)
    perm = rng.permutation(len(f))
    f, ph, det, rad = f[perm], ph[perm], det[perm], rad[perm]
    n_val = 512
    with sgm.Surrogate(hidden=128, batch=512, lr=2e-3, seed=7) as s:
        s.set_data(f, ph, det, rad, n_val=n_val)
        before = s.eval()
        s.train(600)
        after = s.eval()
        path = str(tmp_path / "sg.bin")
        s.save(path)
        params = s.params()
        out = s.predict(f[-n_val:])
    t, y = so.labels(ph, det, rad)
    c_det, c_rad = _constant_predictor_losses(t[:-n_val], y[:-n_val], t[-n_val:], y[-n_val:])
    sgm_report = {"before": before, "after": after, "constant_det": c_det, "constant_rad": c_rad}
    assert after["loss"] < before["loss"], sgm_report
    assert after["det_loss"] < c_det, sgm_report
    assert after["radial_loss"] < c_rad, sgm_report
    # predicted detection fractions track the Monte Carlo's
    p_hat = 1 / (1 + np.exp(-out[:, 0].astype(np.float64)))
    assert np.corrcoef(p_hat, t[-n_val:])[0, 1] > 0.8, sgm_report
    with sgm.Surrogate(hidden=128, batch=512) as s2:
        s2.load(path)
        assert np.array_equal(s2.params(), params)
        assert np.allclose(s2.predict(f[-n_val:]), out, atol=1e-5)


def test_contexts_with_different_shared_memory_alternate(require_gpu):
    """A label-mode context (no PRF window) created between two runs of an
    ordinary one (a shared-memory PRF window) must not break the latter:
    the kernels' shared-memory limit is process-wide."""
    es = hb.synth_events(0, 40, 3)
    with hb.OpticalTransport(es.params, seed=1) as t:
        t.submit(es)
        t.run_sync()
        first = t.counters()["generated"]
        geoms = sgm.sample_geometries(1, seed=2)
        sgm.label_points(geoms, 16, 500, seed=3)
        t.run_sync()
        assert t.counters()["generated"] > first


def test_tensor_core_forward_matches_mma_sync(require_gpu, monkeypatch):
    """The forward GEMMs run on tcgen05 (TMEM accumulators); the mma.sync
    kernel (FD2_SG_GEMM=mma) computes the same BF16 x BF16 -> FP32 products
    in another summation order.  Ragged batch (1,000 rows: 7 full 128-row
    tiles and a partial one), full-size network."""
    H = 256
    p, f, lo, hi, ph, de, ra = _random_problem(5, 1000, H)
    outs = []
    for mode in ("tc", "mma"):
        if mode == "mma":
            monkeypatch.setenv("FD2_SG_GEMM", "mma")
        else:
            monkeypatch.delenv("FD2_SG_GEMM", raising=False)
        with sgm.Surrogate(hidden=H, batch=512) as s:
            s.set_params(p)
            s.set_hull(lo, hi)
            outs.append(s.predict(f))
    a, b = outs
    assert a.shape == (1000, 25) and np.all(np.isfinite(a))
    scale = np.abs(b).max()
    # BF16 hidden activations: a different FP32 summation order can move an
    # activation by one BF16 step now and then
    assert np.abs(a - b).max() <= 2e-2 * scale, np.abs(a - b).max()
    assert np.abs(a - b).mean() <= 1e-3 * scale, np.abs(a - b).mean()


def test_tensor_core_backward_matches_mma_sync(require_gpu, monkeypatch):
    """The backward products run on tcgen05 too: input gradients dY W with
    the weights transposed once per step, weight gradients dY^T X over
    256-row slices of the batch with both operands transposed to be
    contiguous along the batch (FP32 partial planes summed in slice order).
    Against the mma.sync kernels (FD2_SG_GEMM=mma) on a full-size network and
    a ragged batch of 3,000 rows (12 slices, the last one partly padding):
    every parameter block's gradient agrees to BF16 accuracy."""
    H, n = 256, 3000
    p, f, lo, hi, ph, de, ra = _random_problem(17, n, H)
    grads = []
    for mode in ("tc", "mma"):
        if mode == "mma":
            monkeypatch.setenv("FD2_SG_GEMM", "mma")
        else:
            monkeypatch.delenv("FD2_SG_GEMM", raising=False)
        with sgm.Surrogate(hidden=H, batch=4096, radial_bins=64, radial_max_um=200.0) as s:
            s.set_params(p)
            s.set_hull(lo, hi)
            loss, g = s.loss_grad(f, ph, de, ra)
            grads.append((loss, g.astype(np.float64)))
    (la, ga), (lb, gb) = grads
    assert abs(la - lb) <= 1e-5 * abs(lb)
    sizes = [H * 8, H, H * H, H, H * H, H, 25 * H, 25]
    o = 0
    for name, k in zip(BLOCKS, sizes):
        a, b = ga[o:o + k], gb[o:o + k]
        o += k
        rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-12)
        cos = a @ b / max(np.linalg.norm(a) * np.linalg.norm(b), 1e-30)
        assert np.all(np.isfinite(a)) and rel < 1e-2 and cos > 0.9999, (name, rel, cos)


def test_pipelined_tensor_core_kernel_equals_simple(require_gpu, monkeypatch):
    """The default tcgen05 kernel overlaps the loads of the next chunks and
    the epilogue of the previous tile with the MMAs (producer warp, MMA
    thread, four epilogue warps, mbarrier ring, two TMEM accumulators); the
    one-tile-at-a-time kernel (FD2_SG_GEMM=tc1) issues the same MMAs in the
    same order, so forward outputs and gradients are bitwise equal.  Ragged
    sizes: 9,000 prediction rows (70 full tiles and a partial one), 3,000
    training rows (12 batch slices)."""
    H = 256
    p, f, lo, hi, ph, de, ra = _random_problem(23, 9000, H)
    res = []
    for mode in ("pipe", "tc1"):
        if mode == "tc1":
            monkeypatch.setenv("FD2_SG_GEMM", "tc1")
        else:
            monkeypatch.delenv("FD2_SG_GEMM", raising=False)
        with sgm.Surrogate(hidden=H, batch=4096, radial_bins=64, radial_max_um=200.0) as s:
            s.set_params(p)
            s.set_hull(lo, hi)
            out = s.predict(f)
            loss, g = s.loss_grad(f[:3000], ph[:3000], de[:3000], ra[:3000])
        res.append((out, loss, g))
    (oa, la, ga), (ob, lb, gb) = res
    assert np.all(np.isfinite(oa)) and np.array_equal(oa, ob)
    assert la == lb and np.array_equal(ga, gb)
