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
