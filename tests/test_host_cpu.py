"""CPU tests of the host side of the C ABI (no GPU calls).

* the library loads and exports every symbol include/*.h declares;
* the input-file reader on the reference example (24 values, raw tags);
* the output writers reproduce the reference example's files byte for byte;
* EDE stream files round-trip (text in the tally's format, binary);
* the synthetic EDE generators have the configured distributions.
"""
import ctypes
import os
import re

import numpy as np
import pytest

import hybridmantis_b200 as hb
from hybridmantis_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def declared_symbols():
    names = set()
    for h in sorted(f for f in os.listdir(os.path.join(ROOT, "include")) if f.endswith(".h")):
        text = open(os.path.join(ROOT, "include", h)).read()
        for m in re.finditer(r"FD2_API\s+[\w\s\*]+?\b(\w+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    lib = hb.load()
    names = declared_symbols()
    assert len(names) >= 35
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing
    assert names == set(_lib.EXPORTED)


def test_status_strings():
    lib = hb.load()
    for s in range(13):
        assert lib.fd2_status_string(s).decode() != "unknown status"


def test_parse_reference_example_input():
    p = hb.read_input_file(os.path.join(GOLDEN, "example_hybridMANTIS_input.in"))
    assert (p.num_hist, p.min_photons, p.max_photons, p.num_bins) == (100000, 0, 1400, 140)
    assert (p.det_x, p.det_y, p.det_height, p.radius) == (909.0, 909.0, 150.0, 5.1)
    assert (p.n_col, p.n_gap, p.top_absfrac, p.bulk_abs, p.beta) == (1.8, 1.0, 0.1, 1e-4, 0.2)
    assert (p.d_min, p.d_max, p.lb_x, p.lb_y, p.ub_x, p.ub_y) == (1.0, 280.0, 0.0, 0.0, 909.0, 909.0)
    assert (p.yield_, p.pixel, p.sensor_refl, p.run_gpu, p.machine) == (0.055, 9, 0.25, 1, 1)
    z = np.load(os.path.join(GOLDEN, "example_myimage.npz"))
    assert "myimage_" + "_".join(p.tags()) + ".dat" == str(z["name"])
    assert "detected_" + "_".join(p.tags()) + ".dat" == str(z["detected_name"])


def test_parse_errors(tmp_path):
    f = tmp_path / "short.in"
    f.write_text("# comment\n100 # hist\n0\n")
    with pytest.raises(hb.Fd2Error) as e:
        hb.read_input_file(str(f))
    assert e.value.status == 3
    with pytest.raises(hb.Fd2Error) as e:
        hb.read_input_file(str(tmp_path / "missing.in"))
    assert e.value.status == 2
    lines = open(os.path.join(GOLDEN, "example_hybridMANTIS_input.in")).read().replace("140 ", "1.5e2 ")
    f.write_text(lines)
    with pytest.raises(hb.Fd2Error):
        hb.read_input_file(str(f))  # an integer field given as a real
    f.write_text(open(os.path.join(GOLDEN, "example_hybridMANTIS_input.in")).read().replace("1e-4", "1d-4"))
    assert hb.read_input_file(str(f)).bulk_abs == 1e-4  # Fortran exponent letter


def test_writers_reproduce_reference_example_files(tmp_path):
    p = hb.read_input_file(os.path.join(GOLDEN, "example_hybridMANTIS_input.in"))
    g = hb.params_to_geometry(p)
    assert hb.prf_dims(g) == (101, 101)
    z = np.load(os.path.join(GOLDEN, "example_myimage.npz"))
    vals = z["values_e4"].reshape(101, 101)  # file order: [jj (block), ii (row)]
    # counts whose normalised value prints as the example's 4-decimal value
    counts = (vals.T.astype(np.float64) * 1e-4 * p.num_hist).round().astype(np.uint64)
    phs = np.array([int(v) for v in open(os.path.join(GOLDEN, "example_detected.txt"))], np.int32)
    hb.write_output_files(p, g, counts, phs, p.num_hist, str(tmp_path))
    ours_img = (tmp_path / str(z["name"])).read_bytes()
    ours_det = (tmp_path / str(z["detected_name"])).read_bytes()
    assert ours_det == open(os.path.join(GOLDEN, "example_detected.txt"), "rb").read()
    # rebuild the example's PRF text from the fixture and compare bytes
    lines = []
    k = 0
    blanks = set(int(b) for b in z["blank_lines"])
    for i in range(int(z["n_lines"])):
        if i in blanks:
            lines.append("")
        else:
            lines.append(" %12.4f" % (z["values_e4"][k] * 1e-4))
            k += 1
    assert ours_img == ("\n".join(lines) + "\n").encode()
    with pytest.raises(hb.Fd2Error) as e:
        hb.write_output_files(p, g, counts, phs, p.num_hist, str(tmp_path))
    assert e.value.status == 11  # STATUS='NEW'


def test_example_phs_statistics():
    """Sanity values of the reference example (bin width 10)."""
    phs = np.array([int(v) for v in open(os.path.join(GOLDEN, "example_detected.txt"))], np.float64)
    centres = np.arange(len(phs)) * 10.0 + 5.0
    m0, m1, m2 = phs.sum(), (phs * centres).sum(), (phs * centres ** 2).sum()
    assert m0 == 60965
    assert abs(m1 / m0 - 848.8) < 0.1
    assert abs(m1 * m1 / (m0 * m2) - 0.9799) < 1e-4


def test_event_files_round_trip(tmp_path):
    es = hb.synth_events(1, 50, 9)
    hb.write_events_binary(str(tmp_path / "ev.bin"), es)
    back = hb.read_events_binary(str(tmp_path / "ev.bin"))
    for a in ("x_um", "y_um", "z_um", "e_ev", "hist"):
        assert np.array_equal(getattr(es, a), getattr(back, a))
    hb.write_events_text(str(tmp_path / "ev.txt"), es)
    txt = hb.read_events_text(str(tmp_path / "ev.txt"))
    assert np.array_equal(txt.hist, es.hist)
    assert np.allclose(txt.x_um, es.x_um, rtol=1e-7, atol=1e-4)
    assert np.allclose(txt.e_ev, es.e_ev, rtol=1e-4)
    line = open(tmp_path / "ev.txt").readline()
    assert re.fullmatch(r"( [ -]\d\.\d{9}E[+-]\d\d){3}   ?[ -]\d\.\d{4}E[+-]\d\d {0,7}\d+\n", line)
    # comment lines (the tally's history separators) are skipped
    with open(tmp_path / "ev2.txt", "w") as f:
        f.write("#  Past hist =        1 ; Total edep =       2.5000E+04\n\n")
        f.write(open(tmp_path / "ev.txt").read())
    assert hb.read_events_text(str(tmp_path / "ev2.txt")).n == es.n


def test_synthetic_config0():
    es = hb.synth_events(0, 4000, 1)
    assert es.n == 4000 and es.params.num_hist == 4000
    assert np.all(es.e_ev == 25000.0)
    d = es.params.det_height / 2 - es.z_um
    assert d.min() >= 0 and d.max() <= 150.0
    # truncated exponential mean: 60 - 150 e^-2.5 / (1 - e^-2.5)
    mean = 60 - 150 * np.exp(-2.5) / (1 - np.exp(-2.5))
    assert abs(d.mean() - mean) < 4 * 55 / np.sqrt(es.n)
    assert abs(np.std(es.x_um - 250.5) - 2.0) < 0.1
    assert np.array_equal(es.hist, np.arange(1, 4001))


def test_synthetic_config1():
    es = hb.synth_events(1, 20000, 2)
    nx = es.params.num_hist
    per = np.bincount(es.hist, minlength=nx + 1)[1:]
    assert abs(per.mean() - 2.5) < 0.05  # 1 + Poisson(1.5) clusters
    e_xray = np.bincount(es.hist, weights=es.e_ev.astype(np.float64), minlength=nx + 1)[1:] / 1e3
    assert abs(e_xray.mean() - 130 / 3) < 0.3  # triangular(20, 40, 70) mean
    assert e_xray.min() >= 20 and e_xray.max() <= 70
    d = es.params.det_height / 2 - es.z_um
    assert d.min() >= 0 and d.max() <= 300.0 and es.params.radius == 4.0


def test_synthetic_config2_geometries():
    es = hb.synth_events(2, 20, 3)
    assert len(es.geometries) == 64 and es.geom is not None
    H = np.array([g.det_height for g in es.geometries])
    R = np.array([g.radius for g in es.geometries])
    mu = np.array([g.bulk_abs for g in es.geometries])
    assert H.min() >= 100 and H.max() <= 600 and R.min() >= 2.5 and R.max() <= 7.5
    assert mu.min() >= 1e-5 and mu.max() <= 1e-3
    for gi in range(64):
        sel = es.geom == gi
        assert np.all(es.params.det_height >= 0)
        dz = es.geometries[gi].det_height / 2 - es.z_um[sel]
        assert dz.min() >= 0 and dz.max() <= es.geometries[gi].det_height


def test_create_without_gpu_reports_no_device():
    from tests.conftest import gpu_available
    if gpu_available():
        pytest.skip("a GPU is visible")
    with pytest.raises(hb.Fd2Error) as e:
        hb.OpticalTransport(hb.default_params())
    assert e.value.status == 10


def test_invalid_arguments_are_rejected():
    lib = hb.load()
    g = hb.params_to_geometry(hb.default_params())
    x, y = ctypes.c_int32(), ctypes.c_int32()
    g.pixel = 0
    assert lib.fd2_prf_dims(ctypes.byref(g), ctypes.byref(x), ctypes.byref(y)) == 1
    assert lib.fd2_parse_input_file(None, None) == 1


def test_streaming_text_reader_edge_cases(tmp_path):
    """The text reader streams the file through a 4 MiB window: rows that
    straddle window ends, Fortran 'D' exponents, tabs and CR-LF endings, a
    last row without a newline, extra columns (ignored) and malformed rows."""
    rng = np.random.default_rng(3)
    n = 120_000  # about 9 MB of text: the window slides twice
    x, y, z = rng.uniform(0, 0.1, (3, n))
    e = rng.uniform(1.0, 3.0e4, n)
    h = np.sort(rng.integers(1, 5000, n)).astype(np.int32)
    rows = []
    for i in range(n):
        s = f" {x[i]:16.9E} {y[i]:16.9E} {z[i]:16.9E} {e[i]:12.4E}{h[i]:8d}"
        if i % 7 == 0:
            s = s.replace("E", "D")
        if i % 11 == 0:
            s = s.replace(" ", "\t", 2)
        if i % 13 == 0:
            s += "  extra"
        rows.append(s + ("\r\n" if i % 5 == 0 else "\n"))
        if i % 1000 == 0:
            rows.append("#  Past hist = 1\n\n")
    text = "".join(rows).rstrip("\n")  # last row without its newline
    (tmp_path / "big.txt").write_text(text)
    es = hb.read_events_text(str(tmp_path / "big.txt"))
    assert es.n == n
    assert np.array_equal(es.hist, h)
    # the reader's conversion: float(x_cm * (double)10000.0f) of the parsed value
    xp = np.array([float(r.split()[0].replace("D", "E")) for r in rows if not r.startswith(("#", "\n"))])
    assert np.array_equal(es.x_um, (xp * np.float64(np.float32(10000.0))).astype(np.float32))
    for bad in ("1.0 2.0 3.0 4.0\n", "1.0 2.0 3.0 4.0 x\n", "1.0 2.0 zz 4.0 5\n", "1 2 3 4 99999999999\n"):
        (tmp_path / "bad.txt").write_text(" 1.0 2.0 3.0 4.0 1\n" + bad)
        with pytest.raises(hb.Fd2Error) as err:
            hb.read_events_text(str(tmp_path / "bad.txt"))
        assert err.value.status == 3  # FD2_ERR_PARSE


def test_streaming_binary_reader_pieces(tmp_path):
    """The binary reader reads each plane piece by piece (1 Mi events per
    piece); a file larger than one piece and a truncated file."""
    es = hb.synth_events(1, 500_000, 4)
    assert es.n > (1 << 20)
    hb.write_events_binary(str(tmp_path / "ev.bin"), es)
    back = hb.read_events_binary(str(tmp_path / "ev.bin"))
    for a in ("x_um", "y_um", "z_um", "e_ev", "hist"):
        assert np.array_equal(getattr(es, a), getattr(back, a))
    data = open(tmp_path / "ev.bin", "rb").read()
    (tmp_path / "cut.bin").write_bytes(data[:-10])
    with pytest.raises(hb.Fd2Error) as err:
        hb.read_events_binary(str(tmp_path / "cut.bin"))
    assert err.value.status == 3


def test_ingest_entry_points_reject_null_handles():
    lib = hb.load()
    out = ctypes.c_void_p()
    assert lib.fd2_ingest_begin(None, 1024, 0, ctypes.byref(out)) == 1
    assert lib.fd2_ingest_push(None, None, None, None, None, None, 0) == 1
    assert lib.fd2_ingest_push_um(None, None, None, None, None, None, 0) == 1
    assert lib.fd2_ingest_file(None, b"x") == 1
    assert lib.fd2_ingest_end(None, None) == 1


def test_fd2run_usage():
    """The command-line driver refuses incomplete or conflicting arguments before touching a GPU."""
    import subprocess
    exe = os.path.join(ROOT, "hybridmantis_b200", "bin", "fd2run")
    inp = os.path.join(GOLDEN, "example_hybridMANTIS_input.in")
    for args in ([], [inp], ["--xray", "pe.in", inp], ["--material", "m.mat", inp],
                 ["--xray", "pe.in", "--material", "m.mat", inp, "events.txt"]):
        r = subprocess.run([exe] + args, capture_output=True, text=True, timeout=60)
        assert r.returncode == 2, (args, r.stderr)
        assert "usage" in r.stderr
    # a source section that cannot be read is reported, not run
    r = subprocess.run([exe, "--xray", os.path.join(GOLDEN, "example_detected.txt"), "--material", "m.mat", inp],
                       capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "BIGS" in r.stderr


def test_host_generator_build_equals_product_generator():
    """bench.py's reference arm builds its event stream with the host-only
    build of the generator (oracle/_build/libfd2synth.so), so its process maps
    no product library; the events are the product generator's."""
    from oracle import pyoracle as po

    for cfg, n in [(0, 50), (1, 200), (4, 100)]:
        a = po.synth_events_host(cfg, n, 99)
        b = hb.synth_events(cfg, n, 99)
        assert a.n == b.n > 0
        for k in ("x_um", "y_um", "z_um", "e_ev", "hist"):
            assert np.array_equal(getattr(a, k), getattr(b, k)), (cfg, k)
        assert bytes(a.params) == bytes(b.params)
