"""Writes tests/golden/qnm_tables_a0.6/{kerr,swsh}/: the rows of the
reference's QNM_Extraction/Tables files that the ringdown pipeline reads
at spin a = 0.6 for m = +-2 and l, l' = 2..6 (mmax = 4) -- the table row at
a = 0.6 and its neighbours, under the reference's own file names, so
bh_ringdown_b200.ringdown.Tables reads them unchanged and interpolates to
the same values as from the full tables.

  BHR_REFERENCE_ROOT=<reference checkout> python tests/golden/make_qnm_tables.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle.build_ref import default_reference_root  # noqa: E402

A = 0.6
LS = range(2, 7)
OUT = os.path.join(HERE, "qnm_tables_a0.6")


def excerpt(src, dst):
    lines = [ln for ln in open(src).read().splitlines() if ln.strip()]
    a = np.array([float(ln.split()[0]) for ln in lines])
    k = int(np.argmin(np.abs(a - A)))
    keep = lines[max(0, k - 1):k + 2]
    with open(dst, "w") as f:
        f.write("\n".join(keep) + "\n")


def main():
    tabs = os.path.join(default_reference_root(), "QNM_Extraction", "Tables")
    for sub in ("kerr", "swsh"):
        os.makedirs(os.path.join(OUT, sub), exist_ok=True)
    for l in LS:
        for name in (f"n1l{l}m2.dat", f"n1l{l}mm2.dat"):
            excerpt(os.path.join(tabs, "kerr", name), os.path.join(OUT, "kerr", name))
        for lp in LS:
            for name in (f"l{l}m2lp{lp}np0.dat", f"l{l}mm2lp{lp}np0.dat"):
                excerpt(os.path.join(tabs, "swsh", name), os.path.join(OUT, "swsh", name))


if __name__ == "__main__":
    main()
