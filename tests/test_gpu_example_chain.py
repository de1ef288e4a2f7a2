"""The reference's own example, end to end on the GPU: its penEasy source
(main/penEasy_CsI_input.in BIGS section: a 25 keV line from a 30 x 30 um box
at z = 1 cm aimed down the z axis) through the x-ray front end, then its
detector input (example/hybridMANTIS_input.in: 909 x 909 x 150 um, R = 5.1 um,
sensor reflectivity 0.25, yield 0.055/eV, 9 um PRF pixels) through the optical
transport, compared with the outputs the reference ships for that run
(example/output_files): the pulse-height spectrum (detected_*.dat), the PRF
image (myimage_*.dat) and the fate counts of 1e5xrays_console.out:281-293.

The reference's EDEs came from PENELOPE (463 per x-ray); ours come from the
front end's own transport (12 per x-ray), so agreement here checks the chain
as a whole against the reference's published numbers, not EDE by EDE.  The
console's "Generated" count is not compared: the reference kernel counts one
photon for every event before its loop (main/kernel_cuda_c_ver1_0.cu:443),
so its zero-photon events (most of PENELOPE's tens-of-eV depositions) add
photons that are never transported; its fate counters sum to the photons
actually transported, and that sum is compared.
"""
import os

import numpy as np
import pytest

import hybridmantis_b200 as hb
from hybridmantis_b200 import xray

from gpu_helpers import report

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

# 1e5xrays_console.out:281-293 (the reference's GPU run of the example)
REF_FATES = {"detected": 51718347, "abs_top": 8184844, "abs_bulk": 3175019, "lost": 20111907, "outofcol": 29389}


def phs_stats(d):
    x = (np.arange(len(d)) + 0.5) * 10.0  # 140 bins of 10 photons (input: max 1400, 140 bins)
    m0, m1, m2 = d.sum(), (d * x).sum(), (d * x * x).sum()
    return m0, m1 / m0, m1 * m1 / (m0 * m2)


def test_reference_example_end_to_end(require_gpu):
    p = hb.read_input_file(os.path.join(GOLDEN, "example_hybridMANTIS_input.in"))
    ref_phs = np.array([float(v) for v in open(os.path.join(GOLDEN, "example_detected.txt"))])
    ref_img = np.load(os.path.join(GOLDEN, "example_myimage.npz"))["values_e4"].reshape(101, 101) * 1e-4
    src = xray.Source(np.array([25e3, 25e3]), np.array([1.0, -1.0]), center_cm=(0.0454, 0.0454, 1.0),
                      sides_cm=(0.003, 0.003, 0.0), direction=(0.0, 0.0, -1.0))
    n = p.num_hist
    with xray.XrayFrontEnd(det_x_um=p.det_x, det_y_um=p.det_y, det_height_um=p.det_height, seed=3) as fe, \
            hb.OpticalTransport(p, seed=5) as t:
        fe.run(src, n)
        fe.submit(t)
        t.run_sync()
        c = t.counters()
        phs = t.phs().astype(np.float64)
        img = t.prf().astype(np.float64) / n
    r0, rmean, rswank = phs_stats(ref_phs)
    g0, gmean, gswank = phs_stats(phs)
    ref_total = sum(REF_FATES.values())
    gen = c["generated"]
    chi2 = float((((phs / g0 - ref_phs / r0) ** 2) / np.maximum(ref_phs / r0 ** 2 + phs / g0 ** 2, 1e-30)).sum())
    rep = {"phs_primaries": [g0, r0], "phs_mean": [gmean, rmean], "swank": [gswank, rswank],
           "prf_per_xray": [img.sum(), ref_img.sum()], "photons_per_xray": [gen / n, ref_total / n],
           "fates": {k: [c[k] / gen, v / ref_total] for k, v in REF_FATES.items()}, "phs_shape_chi2": chi2,
           "prf_l1": float(np.abs(img / img.sum() - ref_img / ref_img.sum()).sum())}
    report("example_end_to_end", rep)
    # x-rays that deposit anything: binomial
    z = (g0 - r0) / np.sqrt(2 * n * (r0 / n) * (1 - r0 / n))
    assert abs(z) < 5, rep
    assert gmean == pytest.approx(rmean, rel=0.01), rep
    assert gswank == pytest.approx(rswank, abs=0.003), rep
    assert img.sum() == pytest.approx(ref_img.sum(), rel=0.01), rep
    assert gen / n == pytest.approx(ref_total / n, rel=0.01), rep
    for k, v in REF_FATES.items():
        assert c[k] / gen == pytest.approx(v / ref_total, abs=0.003), (k, rep)
    dof = int((ref_phs + phs > 0).sum()) - 1
    assert chi2 < dof + 6 * np.sqrt(2 * dof), rep
    assert rep["prf_l1"] < 0.03, rep


BIGS = """[SECTION SOURCE BOX ISOTROPIC GAUSS SPECTRUM v.2006-08-01]
(ON )                            STATUS (ON or OFF)
 2                               PARTICLE TYPE (1=electron, 2=photon, 3=positron)
 Energy(eV)  Probability         ENERGY SPECTRUM
 25.0e3       1.0
 25.0e3       0.000000010
  1.e6        -1
 4.540e-2  4.540e-2  1.000e0     CENTER COORDINATES OF THE BOX ENCLOSURE (cm)
 3.000e-3  3.000e-3  0.000e0     BOX SIDES (cm)
 0.000e0  0.000e0  0.000e0       EULER ANGLES [Rz,Ry,Rz](deg) TO ROTATE BOX
 0                               MATERIAL (0=DO NOT CARE)
 0.000e0  0.000e0  -1.000        DIRECTION VECTOR, NO NEED TO NORMALIZE
 0.000e0                         ANGLE OF SEMIAPERTURE [0,180] (deg)
[END OF BIGS SECTION]
"""


def test_fd2run_runs_the_example_from_its_input_files(require_gpu, tmp_path):
    """The command-line driver, x-ray mode: a penEasy source section (the example's, with its 1e-8
    tail bin up to 1 MeV), the CsI tables and hybridMANTIS_input.in in; the reference's two output
    files out, under the reference's own file names."""
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    exe = os.path.join(root, "hybridmantis_b200", "bin", "fd2run")
    pe = tmp_path / "penEasy.in"
    pe.write_text("# penEasy input (source section only)\n" + BIGS)
    out = tmp_path / "out"
    out.mkdir()
    r = subprocess.run([exe, "--seed", "11", "--xray", str(pe), "--material", xray.CSI_TABLE, "--out", str(out),
                        os.path.join(GOLDEN, "example_hybridMANTIS_input.in")], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr
    z = np.load(os.path.join(GOLDEN, "example_myimage.npz"))
    names = sorted(os.listdir(out))
    assert names == sorted([str(z["detected_name"]), str(z["name"])]), names
    phs = np.array([float(v) for v in open(out / str(z["detected_name"]))])
    ref_phs = np.array([float(v) for v in open(os.path.join(GOLDEN, "example_detected.txt"))])
    _, gmean, gswank = phs_stats(phs)
    _, rmean, rswank = phs_stats(ref_phs)
    assert gmean == pytest.approx(rmean, rel=0.01) and gswank == pytest.approx(rswank, abs=0.003), r.stdout
    assert "Depositions per primary" in r.stdout
