"""Writes tests/golden/kerr_qnm.txt: Kerr quasinormal frequencies from the
reference's table files QNM_Extraction/Tables/kerr/n<n+1>l<l>m<m>.dat
(columns a, Re omega, Im omega, Re A, Im A), the (l, m) = (2, 2) and (2, -2)
fundamental (n = 0) and first overtone (n = 1), and (3, 2) n = 0, sampled
every 0.01 in a.  The reference's loadqnmtable
(QNM_Extraction/Library/ringdownlib.py:149-161) reads the same files and
interpolates linearly in a.

  BHR_REFERENCE_ROOT=<reference checkout> python tests/golden/make_kerr_qnm.py
"""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))
from oracle.build_ref import default_reference_root  # noqa: E402

ROOT = default_reference_root()
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "kerr_qnm.txt")
FILES = [(2, 2, 0, "n1l2m2.dat"), (2, -2, 0, "n1l2mm2.dat"), (2, 2, 1, "n2l2m2.dat"), (2, -2, 1, "n2l2mm2.dat"),
         (3, 2, 0, "n1l3m2.dat")]


def main():
    lines = ["# l m n a Re(omega) Im(omega)  (from QNM_Extraction/Tables/kerr, every 0.01 in a)"]
    for l, m, n, name in FILES:
        d = np.loadtxt(os.path.join(ROOT, "QNM_Extraction", "Tables", "kerr", name), usecols=(0, 1, 2))
        keep = np.isclose(np.round(d[:, 0] * 100), d[:, 0] * 100, atol=1e-6)
        for a, wr, wi in d[keep]:
            lines.append(f"{l} {m} {n} {a:.4f} {wr:.10e} {wi:.10e}")
    with open(OUT, "w") as f:
        f.write("\n".join(lines) + "\n")


if __name__ == "__main__":
    main()
