"""Write csi_xray.tab, the x-ray front end's CsI tables, from the PENELOPE
material file of the reference's example (example/CsI.mat).

    python hybridmantis_b200/data/make_xray_tables.py /path/to/reference/example/CsI.mat

The table file holds what the front end reads from the material file
(photon cross sections on the union energy grid, relaxation transitions,
electron CSDA ranges and transport mean free paths) in the library's own
text format, so that runs without the reference tree have the same data.
"""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from hybridmantis_b200.xray import Material  # noqa: E402


def main():
    src = sys.argv[1]
    out = sys.argv[2] if len(sys.argv) > 2 else os.path.join(HERE, "csi_xray.tab")
    m = Material(src)
    m.save(out)
    print(out, m.info())


if __name__ == "__main__":
    main()
