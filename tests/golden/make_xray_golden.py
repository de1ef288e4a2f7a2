"""Generates tests/golden/csi_mat_raw.npz from the reference's PENELOPE
material file (example/CsI.mat), parsed here independently of the library's
reader, so that the x-ray front end's tables (hybridmantis_b200/data/
csi_xray.tab) can be checked against the file's own numbers on any machine.

    python tests/golden/make_xray_golden.py [/root/reference/example/CsI.mat]

Kept (energies up to 1 MeV): density and elements; the Rayleigh / Compton
cross sections per molecule; the photoelectric cross sections per atom
(total and per subshell) of each element; the electron collision +
radiative mass stopping powers; the electron first transport cross
sections; the relaxation shells and transitions of each element.
"""
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def parse(path):
    L = open(path).read().splitlines()
    out = {}
    i = 0
    pe = {}
    relax = {}
    while i < len(L):
        s = L[i]
        if "Mass density" in s:
            out["density"] = float(s.split("=")[1].split()[0])
        elif "Number of elements in the molecule" in s:
            n = int(s.split("=")[1])
            zs, at = [], []
            for k in range(n):
                m = re.search(r"atomic number =\s*(\d+),\s*atoms/molecule =\s*(\S+)", L[i + 1 + k])
                zs.append(int(m.group(1)))
                at.append(float(m.group(2)))
            out["z"] = np.array(zs)
            out["atoms"] = np.array(at)
        elif "*** RELAX:" in s:
            m = re.search(r"Z =\s*(\d+),\s*NO. OF SHELLS =\s*(\d+),\s*NO. OF TRANSITIONS =\s*(\d+)", s)
            Z, ns, nt = (int(v) for v in m.groups())
            sh = np.array([[float(L[i + 1 + k].split()[0]), float(L[i + 1 + k].split()[3])] for k in range(ns)])
            tr = np.array([[float(v) for v in L[i + 1 + ns + k].split()[:5]] for k in range(nt)])
            relax[Z] = (sh, tr)
            i += ns + nt
        elif "Stopping powers for electrons and positrons" in s:
            nd = int(s.split("NDATA =")[1])
            a = np.array([[float(v) for v in L[i + 1 + k].split()[:5]] for k in range(nd)])
            out["sp_e"], out["sp_col"], out["sp_rad"] = a[:, 0], a[:, 1], a[:, 2]
            i += nd
        elif "Electron and positron elastic cross sections" in s:
            nd = int(s.split("NDATA =")[1])
            a = np.array([[float(v) for v in L[i + 1 + k].split()[:3]] for k in range(nd)])
            out["el_e"], out["el_s1"] = a[:, 0], a[:, 2]
            i += nd
        elif "Rayleigh, Compton and pair-production" in s:
            nd = int(s.split("NDATA =")[1])
            a = np.array([[float(v) for v in L[i + 1 + k].split()[:3]] for k in range(nd)])
            out["rc_e"], out["rc_r"], out["rc_c"] = a[:, 0], a[:, 1], a[:, 2]
            i += nd
        elif "Photoelectric cross sections" in s:
            Z = int(re.search(r"IZ =\s*(\d+)", s).group(1))
            nsh = int(re.search(r"NSHELL =\s*(\d+)", s).group(1))
            nd = int(s.split("NDATA =")[1])
            a = np.array([[float(v) for v in L[i + 1 + k].split()[:nsh + 2]] for k in range(nd)])
            pe[Z] = a
            i += nd
        i += 1
    keep = lambda e: e <= 1e6  # noqa: E731
    res = {"density": out["density"], "z": out["z"], "atoms": out["atoms"]}
    k = keep(out["rc_e"])
    res.update(rc_e=out["rc_e"][k], rc_r=out["rc_r"][k], rc_c=out["rc_c"][k])
    k = keep(out["sp_e"])
    res.update(sp_e=out["sp_e"][k], sp_col=out["sp_col"][k], sp_rad=out["sp_rad"][k])
    k = keep(out["el_e"])
    res.update(el_e=out["el_e"][k], el_s1=out["el_s1"][k])
    for Z, a in pe.items():
        res[f"pe_{Z}"] = a[a[:, 0] <= 1e6]
    for Z, (sh, tr) in relax.items():
        res[f"relax_shells_{Z}"] = sh
        res[f"relax_trans_{Z}"] = tr
    return res


def main():
    src = sys.argv[1] if len(sys.argv) > 1 else "/root/reference/example/CsI.mat"
    res = parse(src)
    np.savez_compressed(os.path.join(HERE, "csi_mat_raw.npz"), **res)
    print({k: np.shape(v) for k, v in res.items()})


if __name__ == "__main__":
    main()
