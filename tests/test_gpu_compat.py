"""The Fortran-facing shims (gpuoptical_, cpuoptical_, gpuoptlb_) on the GPU.

tests/compat_driver.c plays the Fortran program: it defines the COMMON
blocks, buffers a seeded synthetic stream in /optical/ (cm, eV, 1-based
histories) and makes the EDE tally's calls.  The COMMON-block results must
equal, bit for bit, those of the same calls made through the context API
with the library's default options (same seed, same runs).
"""
import json
import os
import subprocess

import numpy as np
import pytest

import hybridmantis_b200 as hb

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
N_XRAYS, SEED = 60, 4242


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("compat") / "compat_driver")
    lib = os.path.join(ROOT, "hybridmantis_b200", "lib")
    subprocess.run(["gcc", "-O2", "-Wall", "-I", os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "compat_driver.c"),
                    "-L", lib, "-lfd2", f"-Wl,-rpath,{lib}", "-o", exe], check=True)
    return exe


def _run(driver, mode):
    out = subprocess.run([driver, mode, str(N_XRAYS), str(SEED)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, (out.returncode, out.stderr)
    return json.loads(out.stdout.strip().splitlines()[-1])


def _expected(buffers):
    es = hb.synth_events(0, N_XRAYS, SEED)
    with hb.OpticalTransport(es.params) as t:
        for sl in buffers(es.n):
            sub = es.subset(sl)
            x, y, z = sub.to_cm()
            t.submit_events(x, y, z, sub.e_ev.astype(np.float64), sub.hist)
            t.run_sync()
        c = t.counters()
        img = t.prf()
        phs = t.phs()
    m = 2 ** 64
    ih = 0
    for v in img[:501, :501].ravel().tolist():
        ih = (ih * 1000003 + v) % m
    ph = 0
    for v in list(phs) + [0] * (1000 - len(phs)):
        ph = (ph * 31 + int(v)) % m
    return {"glgen": c["generated"], "gldetect": c["detected"], "glabstop": c["abs_top"], "glabsbulk": c["abs_bulk"],
            "gllost": c["lost"], "gloutofcol": c["outofcol"], "gltheta1": c["theta1"],
            "image_sum": int(img[:501, :501].sum()), "image_hash": ih, "phs_sum": int(phs.sum()), "phs_hash": ph}


def _check(got, want):
    for k, v in want.items():
        assert int(got[k]) == int(v), (k, got, want)


def test_gpuoptical_modes(require_gpu, driver):
    got = _run(driver, "gpu")
    want = _expected(lambda n: [slice(0, n // 2), slice(n // 2, n)])
    _check(got, want)
    assert got["glgputime"] > 0


def test_cpuoptical(require_gpu, driver):
    _check(_run(driver, "cpu"), _expected(lambda n: [slice(0, n)]))


def test_gpuoptlb_probe(require_gpu, driver):
    got = _run(driver, "lb")
    _check(got, _expected(lambda n: [slice(0, n)]))
    assert got["seconds"] > 0
