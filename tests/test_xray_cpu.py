"""CPU tests of the x-ray front end's tables (library host code) and of its
oracle (oracle/xray_oracle.c).

The front end replaces PENELOPE + penEasy, whose sources are not in the
reference tree; what the reference does hold is the material file
(example/CsI.mat) and the source and tally semantics.  Pinned here:
- the library's tables (hybridmantis_b200/data/csi_xray.tab, made from
  example/CsI.mat) reproduce the file's numbers, read by an independent
  parser into tests/golden/csi_mat_raw.npz: cross sections at the file's
  nodes, the absorption edges, the electron CSDA range as the integral of
  1 / S, the transport mean free paths, the relaxation transitions;
- the library's PENELOPE reader, run on a file in that format holding the
  fixture's numbers, gives the committed tables;
- the oracle's Rayleigh screening reproduces the file's Rayleigh cross
  section through its angular integral;
- the oracle against closed forms: energy is conserved history by history;
  the first-interaction depth is exponential with the table's attenuation;
  the first-interaction kinds follow the partial attenuations; the
  deposited-energy spectrum of a 50 keV beam has the K-escape lines of the
  file's transitions; an electron far from the surfaces deposits exactly
  its energy in a known number of steps.
"""
import os

import numpy as np
import pytest
from scipy import integrate, stats

import hybridmantis_b200 as hb
from hybridmantis_b200 import xray
from oracle import xray_oracle as xo

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
RAW = np.load(os.path.join(GOLDEN, "csi_mat_raw.npz"))
NA = 6.02214076e23
WEIGHT = {53: 126.90, 55: 132.91}


@pytest.fixture(scope="module")
def mat():
    return xray.Material()


def loglog(x, xs, ys):
    """Log-log interpolation inside a table (no edges in the interval)."""
    i = np.searchsorted(xs, x, side="right") - 1
    i = np.clip(i, 0, len(xs) - 2)
    w = np.log(x / xs[i]) / np.log(xs[i + 1] / xs[i])
    return np.exp(np.log(ys[i]) + w * (np.log(ys[i + 1]) - np.log(ys[i])))


def molecules(info):
    return RAW["density"] * NA / sum(a * WEIGHT[z] for z, a in zip(RAW["z"], RAW["atoms"]))


def test_material_header(mat):
    info = mat.info()
    assert info["density"] == pytest.approx(float(RAW["density"]))
    assert info["z"] == list(RAW["z"]) and info["atoms"] == list(RAW["atoms"])
    assert info["molecules_per_cm3"] == pytest.approx(molecules(info), rel=1e-12)
    assert info["k_edge_ev"] == pytest.approx([33170.0, 35985.0])
    assert info["transitions"] == len(RAW["relax_trans_53"]) + len(RAW["relax_trans_55"])


def test_rayleigh_compton_at_the_file_nodes(mat):
    N = mat.info()["molecules_per_cm3"]
    e = RAW["rc_e"]
    e = e[(e >= 1e3)]
    mu = mat.attenuation(e)
    np.testing.assert_allclose(mu[:, 0] / N, RAW["rc_r"][-len(e):], rtol=1e-12)
    np.testing.assert_allclose(mu[:, 1] / N, RAW["rc_c"][-len(e):], rtol=1e-12)


def test_photoelectric_at_the_file_nodes_and_edges(mat):
    N = mat.info()["molecules_per_cm3"]
    a53, a55 = RAW["pe_53"], RAW["pe_55"]
    for own, other in ((a53, a55), (a55, a53)):
        e = own[:, 0]
        dup = np.r_[e[1:] == e[:-1], False] | np.r_[False, e[1:] == e[:-1]]
        sel = (e >= 1e3) & ~dup & ~np.isin(e, other[:, 0])
        ee = e[sel]
        # the other element's value, log-log between its nodes (away from its edges)
        oth = loglog(ee, other[:, 0], other[:, 1])
        expect = N * (own[sel, 1] + oth)
        np.testing.assert_allclose(mat.attenuation(ee)[:, 2], expect, rtol=1e-9)
    # the K edges: just below and above, the jump of the file's K-shell column
    for z, arr in ((53, a53), (55, a55)):
        ek = arr[np.r_[arr[1:, 0] == arr[:-1, 0], False] & (arr[:, 0] > 3e4), 0][0]
        lo, hi = mat.attenuation([ek * (1 - 1e-12), ek * (1 + 1e-12)])[:, 2]
        i = np.where(arr[:, 0] == ek)[0]
        jump = N * (arr[i[1], 1] - arr[i[0], 1])
        assert hi - lo == pytest.approx(jump, rel=1e-6)


def test_electron_range_and_transport_mfp(mat):
    e, S = RAW["sp_e"], (RAW["sp_col"] + RAW["sp_rad"]) * 1e6 * float(RAW["density"])  # eV/cm
    E = np.array([100.0, 1e3, 1e4, 3e4, 6e4, 1e5])
    R, L1 = mat.electron(E)

    def csda(x):
        f = lambda q: 1.0 / loglog(np.array([q]), e, S)[0]  # noqa: E731
        r0 = e[0] / S[0]
        val, _ = integrate.quad(f, e[0], x, limit=400, points=e[(e > e[0]) & (e < x)][:300])
        return r0 + val

    np.testing.assert_allclose(R, [csda(x) for x in E], rtol=2e-4)
    N = mat.info()["molecules_per_cm3"]
    nodes = RAW["el_e"][(RAW["el_e"] >= 100) & (RAW["el_e"] <= 1e5)]
    s1 = RAW["el_s1"][(RAW["el_e"] >= 100) & (RAW["el_e"] <= 1e5)]
    _, l1n = mat.electron(nodes)
    np.testing.assert_allclose(l1n, 1.0 / (N * s1), rtol=1e-12)
    # physical scale: a 30 keV electron's CSDA range in CsI is several micrometres
    assert 5e-4 < mat.electron([3e4])[0][0] < 1.2e-3


def test_rayleigh_screening_reproduces_the_cross_section(mat):
    N = mat.info()["molecules_per_cm3"]
    re2 = 2.8179403262e-13 ** 2
    fz2 = sum(a * z * z for z, a in zip(RAW["z"], RAW["atoms"]))
    for E in (5e3, 2e4, 3e4, 5e4, 1e5, 3e5):
        b = xo.rayleigh_b(xray.CSI_TABLE, E)
        I, _ = integrate.quad(lambda mu: (1 + mu * mu) / (1 + b * (1 - mu)) ** 4, -1, 1, epsabs=0, epsrel=1e-12,
                              limit=400)
        sig = np.pi * re2 * fz2 * I
        assert sig == pytest.approx(mat.attenuation([E])[0, 0] / N, rel=1e-7)


def test_table_file_round_trip(tmp_path, mat):
    p1 = str(tmp_path / "a.tab")
    mat.save(p1)
    m2 = xray.Material(p1)
    p2 = str(tmp_path / "b.tab")
    m2.save(p2)
    assert open(p1).read() == open(p2).read() == open(xray.CSI_TABLE).read()


def test_front_end_needs_a_gpu_here(mat):
    with pytest.raises(hb.Fd2Error) as e:
        xray.XrayFrontEnd(mat)
    assert e.value.status == 10  # FD2_ERR_NO_DEVICE


def test_penEasy_source_section(tmp_path):
    txt = """# a penEasy input
[SECTION SOURCE BOX ISOTROPIC GAUSS SPECTRUM v.2006-08-01]
(ON )                            STATUS (ON or OFF)
 2                               PARTICLE TYPE (1=electron, 2=photon, 3=positron)
 Energy(eV)  Probability         ENERGY SPECTRUM
 20.0e3       1.0
 30.0e3       3.0
 40.0e3       -1
 4.5e-2  4.4e-2  1.0e0           CENTER COORDINATES OF THE BOX ENCLOSURE (cm)
 3.0e-3  2.0e-3  0.0e0           BOX SIDES (cm)
 0.0e0  10.0e0  0.0e0            EULER ANGLES [Rz,Ry,Rz](deg) TO ROTATE BOX
 0                               MATERIAL (0=DO NOT CARE)
 0.0e0  0.0e0  -1.0              DIRECTION VECTOR, NO NEED TO NORMALIZE
 2.5e0                           ANGLE OF SEMIAPERTURE [0,180] (deg)
[END OF BIGS SECTION]
"""
    p = tmp_path / "pe.in"
    p.write_text(txt)
    s = xray.read_penEasy_source(str(p))
    assert s.particle == 2 and list(s.e_ev) == [20e3, 30e3, 40e3] and list(s.prob) == [1.0, 3.0, -1.0]
    assert s.center_cm == (0.045, 0.044, 1.0) and s.sides_cm == (0.003, 0.002, 0.0)
    assert s.euler_deg == (0.0, 10.0, 0.0) and s.direction == (0.0, 0.0, -1.0) and s.semiaperture_deg == 2.5


def test_penEasy_source_section_refusals(tmp_path):
    good = (tmp_path / "g.in")
    base = [" 2   PARTICLE", " Energy(eV)  Probability", " 30.0e3 1.0", " 30.0e3 -1", " 0.04 0.04 1.0", " 0 0 0",
            " 0 0 0", " 0", " 0 0 -1", " 0.0"]
    head = "[SECTION SOURCE BOX ISOTROPIC GAUSS SPECTRUM v.2006-08-01]"
    good.write_text("\n".join([head, "(ON )"] + base) + "\n")
    assert xray.read_penEasy_source(str(good)).e_ev.tolist() == [30e3, 30e3]
    for name, lines in (("off", [head, "(OFF)"] + base), ("mat", [head, "(ON )"] + base[:7] + [" 1"] + base[8:]),
                        ("none", ["[SECTION SOURCE PHASE SPACE FILE v.2008-06-01]", "(ON )"])):
        f = tmp_path / f"{name}.in"
        f.write_text("\n".join(lines) + "\n")
        with pytest.raises(hb.Fd2Error) as e:
            xray.read_penEasy_source(str(f))
        assert e.value.status == 3


# ------------------------------------------------------------------ oracle

def run(src, n, **kw):
    return xo.run(xray.CSI_TABLE, src, n, **kw)


def balance(h, edes):
    dep = np.array([e[:, 3].sum() for e in edes])
    return dep + h["esc_ph"] + h["esc_el"] - h["e0"]


@pytest.mark.parametrize("kind", ["mono50", "tri", "gauss", "box_cone", "electron", "merged"])
def test_oracle_conserves_energy(kind):
    kw = {}
    if kind == "mono50":
        src = xray.monoenergetic(50e3)
    elif kind == "tri":
        src = xray.triangular_spectrum(20e3, 40e3, 70e3)
    elif kind == "gauss":
        src = xray.Source(np.array([55e3, 60e3]), np.array([0.0, -1.0]))
    elif kind == "box_cone":
        src = xray.Source(np.array([30e3, 80e3]), np.array([1.0, -1.0]), sides_cm=(0.05, 0.05, 0.0),
                          euler_deg=(20.0, 5.0, 0.0), semiaperture_deg=30.0)
    elif kind == "electron":
        src = xray.monoenergetic(40e3, particle=xray.ELECTRON, center_cm=(0.04545, 0.04545, 0.0),
                                 direction=(0, 0, 0), semiaperture_deg=180.0)
    else:
        src = xray.monoenergetic(70e3)
        kw = dict(local_e=50.0, cap=64)
    h, edes = run(src, 1500, seed=3, **kw)
    assert np.abs(balance(h, edes)).max() < 1e-6
    for e in edes:
        assert np.all(e[:, 3] > 0)
        assert np.all((e[:, 0] >= 0) & (e[:, 0] <= 0.0909) & (e[:, 1] >= 0) & (e[:, 1] <= 0.0909))
        assert np.all(np.abs(e[:, 2]) <= 0.0075)
    if kind == "merged":
        assert h["merged"].sum() > 0
    if kind == "gauss":
        assert 50e3 < h["e0"].mean() < 65e3


@pytest.mark.parametrize("E", [30e3, 50e3])
def test_oracle_first_interaction_depth_and_kind(mat, E):
    n = 20000
    h, _ = run(xray.monoenergetic(E), n, seed=11)
    mu = mat.attenuation([E])[0]
    H = 0.015
    hit = h["first_kind"] > 0
    p = 1 - np.exp(-mu[3] * H)
    z = (hit.sum() - n * p) / np.sqrt(n * p * (1 - p))
    assert abs(z) < 4.5
    d = h["first_depth"][hit]
    cdf = lambda x: (1 - np.exp(-mu[3] * x)) / (1 - np.exp(-mu[3] * H))  # noqa: E731
    assert stats.kstest(d, cdf).pvalue > 1e-4
    k = h["first_kind"][hit].astype(int)
    for kind, frac in ((1, mu[0] / mu[3]), (2, mu[1] / mu[3]), (3, mu[2] / mu[3])):
        m = hit.sum()
        zk = ((k == kind).sum() - m * frac) / np.sqrt(m * frac * (1 - frac))
        assert abs(zk) < 4.5, (kind, zk)


def test_oracle_k_escape_lines():
    E0 = 50e3
    h, edes = run(xray.monoenergetic(E0), 20000, seed=5)
    dep = np.array([e[:, 3].sum() for e in edes])
    vals, cnt = np.unique(np.round(dep, 3), return_counts=True)
    frequent = set(vals[cnt >= 40])
    for Z in (53, 55):
        tr = RAW[f"relax_trans_{Z}"]
        rad = tr[(tr[:, 0] == 1) & (tr[:, 2] == 0)]
        for line in rad[np.argsort(-rad[:, 3])][:2]:   # the two strongest K lines (K-L3, K-L2)
            assert round(E0 - line[4], 3) in frequent, (Z, line)
    assert E0 in frequent  # the full-energy peak


def test_oracle_electron_steps_in_bulk():
    T0, loss, local = 30e3, 0.25, 1000.0
    src = xray.monoenergetic(T0, particle=xray.ELECTRON, center_cm=(0.04545, 0.04545, 0.0), direction=(0, 0, 1),
                             semiaperture_deg=180.0)
    h, edes = run(src, 500, seed=2, loss=loss, local_e=local)
    steps = 0
    T = T0
    while T > local:
        T *= 1 - loss
        steps += 1
    assert np.all(h["n_steps"] == steps)
    assert np.all(h["n_edes"] == steps + 1)
    dep = np.array([e[:, 3].sum() for e in edes])
    np.testing.assert_allclose(dep, T0, rtol=1e-12)
    assert np.all(h["esc_el"] == 0)


def test_oracle_without_fluorescence():
    h, edes = run(xray.monoenergetic(50e3), 3000, seed=4, fluo=False)
    assert h["n_fe"].sum() == 0 and h["n_aug"].sum() == 0
    assert np.abs(balance(h, edes)).max() < 1e-6


def write_penelope_file(path):
    """A PENELOPE-format material file holding the fixture's numbers (energies up to 1 MeV)."""
    L = [" PENELOPE (v. 2006)  Material data file ...............",
         " Material: CESIUM IODIDE  (141)",
         f" Mass density = {float(RAW['density']):.8E} g/cm**3",
         f" Number of elements in the molecule =  {len(RAW['z'])}"]
    for z, a in zip(RAW["z"], RAW["atoms"]):
        L.append(f"   atomic number = {int(z)},  atoms/molecule = {a:.8E}")
    for z in RAW["z"]:
        sh, tr = RAW[f"relax_shells_{z}"], RAW[f"relax_trans_{z}"]
        L.append(f" *** RELAX:  Z = {int(z)},  NO. OF SHELLS = {len(sh)},  NO. OF TRANSITIONS = {len(tr)}")
        L += [f"  {int(d):2d} X 2  {e:.8E}" for d, e in sh]
        L += [f"  {int(t[0]):2d} {int(t[1]):2d} {int(t[2]):2d}  {t[3]:.6E}  {t[4]:.6E}" for t in tr]
    L.append(f" *** Stopping powers for electrons and positrons,  NDATA = {len(RAW['sp_e'])}")
    L += [f" {e:.3E} {c:.5E} {r:.5E} {c:.5E} {r:.5E}" for e, c, r in zip(RAW["sp_e"], RAW["sp_col"], RAW["sp_rad"])]
    L.append(f" ***  Electron and positron elastic cross sections,  NDATA = {len(RAW['el_e'])}")
    L += [f" {e:.3E} {30 * s:.5E} {s:.5E} {2 * s:.5E} {30 * s:.5E} {s:.5E} {2 * s:.5E}"
          for e, s in zip(RAW["el_e"], RAW["el_s1"])]
    L.append(f" *** Rayleigh, Compton and pair-production cross sections,  NDATA = {len(RAW['rc_e'])}")
    L += [f" {e:.3E} {r:.5E} {c:.5E} 0.00000E+00" for e, r, c in zip(RAW["rc_e"], RAW["rc_r"], RAW["rc_c"])]
    for z in RAW["z"]:
        a = RAW[f"pe_{z}"]
        L.append(f" ***  Photoelectric cross sections,  IZ = {int(z)},  NSHELL =  {a.shape[1] - 2},  NDATA = {len(a)}")
        L += [" " + " ".join(f"{v:.5E}" for v in row) for row in a]
    L.append(" PENELOPE (v. 2006)  End of material data file ........")
    path.write_text("\n".join(L) + "\n")


def test_penelope_reader_on_a_material_file(tmp_path, mat):
    """The library's PENELOPE reader on a file in that format (the fixture's numbers, to 1 MeV): the
    same tables as the committed ones, which were read from the reference's own file."""
    f = tmp_path / "CsI_1MeV.mat"
    write_penelope_file(f)
    m2 = xray.Material(str(f))
    i1, i2 = mat.info(), m2.info()
    for k in ("density", "molar_mass", "molecules_per_cm3", "z", "atoms", "k_edge_ev", "transitions"):
        assert i1[k] == i2[k], k
    E = np.geomspace(1.2e3, 9e5, 400)
    np.testing.assert_allclose(m2.attenuation(E), mat.attenuation(E), rtol=1e-5)
    r1, l1 = mat.electron(E)
    r2, l2 = m2.electron(E)
    np.testing.assert_allclose(r2, r1, rtol=1e-5)
    np.testing.assert_allclose(l2, l1, rtol=1e-5)
    # the Rayleigh screening solved from the parsed cross sections: same samples as the oracle's
    assert i2["rayleigh_screening_cm"] == pytest.approx(i1["rayleigh_screening_cm"], rel=1e-5)
