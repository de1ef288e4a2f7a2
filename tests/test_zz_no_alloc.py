"""fd2_transport_noalloc against the context API (GPU).

fd2_transport_noalloc is for callers that cannot allocate device memory
(code inside another framework's memory pool, or that may not change the
device's memory footprint): they pass device buffers for events and tallies,
and the work queue lives in the library's fixed __device__ scratch array.
Its tallies must equal the context API's (fd2_submit_events_um + fd2_run
with the same seed and photon counts) exactly -- both draw the same Philox
streams -- on two calls in a row, the second reusing the scratch the first
left behind.  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

import hybridmantis_b200 as hb

pytestmark = pytest.mark.gpu


def test_noalloc_matches_context_api(require_gpu):
    import torch

    es = hb.synth_events(0, 120, 31)
    rng = np.random.default_rng(31)
    N = np.maximum(0, np.rint(rng.normal(1350.0, np.sqrt(1350.0), es.n))).astype(np.int32)
    seed = 0xC0FFEE
    p = es.params
    with hb.OpticalTransport(p, count_mode=hb.COUNT_GIVEN, seed=seed) as t:
        t.submit(es, nphot=N)
        t.run_sync()
        ref_prf = t.prf()
        ref_prim = t.detected_per_primary()
        ref = t.counters()

    lib = hb.load()
    geom = hb.params_to_geometry(p)
    xd, yd = hb.prf_dims(geom)
    dev = torch.device("cuda", 0)
    x = torch.from_numpy(es.x_um).to(dev)
    y = torch.from_numpy(es.y_um).to(dev)
    z = torch.from_numpy(es.z_um).to(dev)
    h = torch.from_numpy(es.hist.astype(np.int32)).to(dev)
    n = torch.from_numpy(N).to(dev)
    prf = torch.zeros(xd * yd, dtype=torch.int64, device=dev)
    prim = torch.zeros(p.num_hist, dtype=torch.int32, device=dev)
    cnt = torch.zeros(9, dtype=torch.int64, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    names = ["detected", "abs_top", "abs_bulk", "lost", "outofcol", "theta1", "capped", "detected_in_prf"]
    for call in range(2):
        prf.zero_()
        prim.zero_()
        cnt.zero_()
        torch.cuda.synchronize()
        st = lib.fd2_transport_noalloc(ctypes.byref(geom), ctypes.c_void_p(x.data_ptr()),
                                       ctypes.c_void_p(y.data_ptr()), ctypes.c_void_p(z.data_ptr()),
                                       ctypes.c_void_p(h.data_ptr()), ctypes.c_void_p(n.data_ptr()), es.n,
                                       p.num_hist, ctypes.c_uint64(seed), ctypes.c_void_p(prf.data_ptr()),
                                       ctypes.c_void_p(prim.data_ptr()), ctypes.c_void_p(cnt.data_ptr()),
                                       ctypes.c_void_p(stream))
        assert st == 0, f"call {call}: status {st}"
        got = cnt.cpu().numpy().astype(np.uint64)
        assert dict(zip(names, [int(v) for v in got[1:]])) == {k: ref[k] for k in names}, f"call {call}"
        assert int(got[1:8].sum()) == int(N.sum())
        assert np.array_equal(prf.cpu().numpy().astype(np.uint64).reshape(xd, yd), ref_prf), f"call {call}"
        assert np.array_equal(prim.cpu().numpy(), ref_prim), f"call {call}"


def test_noalloc_rejects_oversized_inputs(require_gpu):
    lib = hb.load()
    geom = hb.params_to_geometry(hb.default_params())
    dummy = ctypes.c_void_p(16)
    st = lib.fd2_transport_noalloc(ctypes.byref(geom), dummy, dummy, dummy, dummy, dummy, 262145, 10,
                                   ctypes.c_uint64(1), dummy, dummy, dummy, None)
    assert st == 1


@pytest.mark.parametrize("case", ["chunk_overflow", "too_many_photons", "bad_history"])
def test_noalloc_rejected_call_leaves_tallies(require_gpu, case):
    """A call the device rejects (more queue chunks than the scratch holds,
    an event above the 900,000-photon cap, a history outside 1..num_hist)
    returns its status and adds nothing to the caller's tallies."""
    import torch

    lib = hb.load()
    p = hb.default_params(num_hist=1000)
    geom = hb.params_to_geometry(p)
    xd, yd = hb.prf_dims(geom)
    dev = torch.device("cuda", 0)
    if case == "chunk_overflow":
        # 600 events x 900,000 photons = 600 x 3,516 chunks of 256 > 2,097,152
        n, nph, hist, want = 600, np.full(600, 900000, np.int32), np.arange(1, 601, dtype=np.int32), 1
    elif case == "too_many_photons":
        n, nph, hist, want = 4, np.array([1000, 900001, 1000, 1000], np.int32), np.arange(1, 5, dtype=np.int32), 6
    else:
        n, nph, hist, want = 4, np.full(4, 1000, np.int32), np.array([1, 2, 1001, 3], np.int32), 12
    pos = torch.full((n,), 250.5, dtype=torch.float32, device=dev)
    z = torch.full((n,), 10.0, dtype=torch.float32, device=dev)
    h = torch.from_numpy(hist).to(dev)
    k = torch.from_numpy(nph).to(dev)
    prf = torch.zeros(xd * yd, dtype=torch.int64, device=dev)
    prim = torch.zeros(p.num_hist, dtype=torch.int32, device=dev)
    cnt = torch.zeros(9, dtype=torch.int64, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    torch.cuda.synchronize()
    st = lib.fd2_transport_noalloc(ctypes.byref(geom), ctypes.c_void_p(pos.data_ptr()),
                                   ctypes.c_void_p(pos.data_ptr()), ctypes.c_void_p(z.data_ptr()),
                                   ctypes.c_void_p(h.data_ptr()), ctypes.c_void_p(k.data_ptr()), n, p.num_hist,
                                   ctypes.c_uint64(7), ctypes.c_void_p(prf.data_ptr()),
                                   ctypes.c_void_p(prim.data_ptr()), ctypes.c_void_p(cnt.data_ptr()),
                                   ctypes.c_void_p(stream))
    assert st == want
    assert int(cnt.abs().sum()) == 0 and int(prf.abs().sum()) == 0 and int(prim.abs().sum()) == 0
