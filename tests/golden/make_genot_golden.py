"""Generate tests/golden/genot_cases.npz: the reference's trajectory
generator run on synthetic inputs.

GenOT/ParamWLMino.cc and GenOT/WL_BL.cc, compiled from where they lie into
oracle/_ref/genot/ (oracle/build_ref.py, tag "genot"), are run for three
cases (equatorial, inclined, inclined beyond 90 degrees; both transition
models).  Their inputs are written by this script: the stand-in inspiral
table (bh_ringdown_b200.genot.synthetic_inspiral) and the Ori-Thorne table
X(T) (bh_ringdown_b200.genot.ot_table) as OT_X_vs_L.dat in the programs'
working directory, where ParamWLMino reads it.  WL_BL keeps eleven
200000-row arrays on its stack, so it runs with a 64 MB stack limit.
Recorded: the inspiral table, a subsample of the Mino-time rows and of the
.traj rows (every row of both is compared when the programs are present,
by tests/test_genot.py), the .traj file name, and every 1000th row of the
reference's own OT_X_vs_L.dat (the table genot.ot_table replaces).
Nothing of the generator is restated here: this script only writes inputs
and reads the reference's outputs.

    python oracle/build_ref.py genot
    python tests/golden/make_genot_golden.py --out <dir>
    cp <dir>/genot_cases.npz tests/golden/
"""
from __future__ import annotations

import argparse
import glob
import os
import resource
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

BIN = os.path.join(ROOT, "oracle", "_ref", "genot")
INSP_ROWS = 400
MINO_STRIDE, BL_STRIDE = 17, 997
# name: (a, inclination, insp r_start, eta, LTi, LTf, r_start, model, lambda_start, t_stop, chi0, phi0)
CASES = {
    "eq_a07": (0.7, 0.0, 4.5, 1e-4, -3.0, 2.35, 4.4, 2, -100.0, 150.0, 30.0, 10.0),
    "inc30_a03": (0.3, 30.0, 7.0, 1e-4, -3.0, 2.35, 6.9, 1, -200.0, 120.0, 40.0, 0.0),
    "inc120_a05": (0.5, 120.0, 6.0, 1e-4, -3.0, 2.35, 5.9, 2, -200.0, 120.0, 40.0, 0.0),
}


def _big_stack():
    resource.setrlimit(resource.RLIMIT_STACK, (64 << 20, resource.getrlimit(resource.RLIMIT_STACK)[1]))


def run_reference(work: str, case) -> dict:
    """Run ParamWLMino and WL_BL in `work` on one case; their outputs."""
    from bh_ringdown_b200 import genot
    a, inc, r_insp, eta, LTi, LTf, r_start, model, lam0, t_stop, chi0, phi0 = case
    insp = genot.synthetic_inspiral(a, r_insp, rows=INSP_ROWS, inclination_deg=inc)
    np.savetxt(os.path.join(work, "insp"), insp, fmt="%.17g")
    np.savetxt(os.path.join(work, "OT_X_vs_L.dat"), genot.ot_table(), fmt="%.17g", delimiter="\t")
    args = [os.path.join(BIN, "ParamWLMino"), repr(a), repr(eta), "insp", repr(LTi), repr(LTf), repr(r_start),
            str(model)]
    out = subprocess.run(args, cwd=work, capture_output=True, text=True, check=True)
    with open(os.path.join(work, "mino"), "w") as f:
        f.write(out.stdout)
    mino = np.loadtxt(os.path.join(work, "mino"))
    for old in glob.glob(os.path.join(work, "*.traj")):
        os.remove(old)
    args = [os.path.join(BIN, "WL_BL"), repr(a), "mino", repr(lam0), repr(t_stop), repr(chi0), repr(phi0)]
    subprocess.run(args, cwd=work, capture_output=True, text=True, check=True, preexec_fn=_big_stack)
    (traj,) = glob.glob(os.path.join(work, "*.traj"))
    return {"insp": insp, "mino": mino, "traj": np.loadtxt(traj), "name": os.path.basename(traj)}


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--ref", default=None, help="reference root (for its OT_X_vs_L.dat)")
    args = ap.parse_args()
    from oracle.build_ref import default_reference_root
    ref_root = args.ref or default_reference_root()
    rec = {}
    for name, case in CASES.items():
        with tempfile.TemporaryDirectory() as work:
            r = run_reference(work, case)
        nm, nt = len(r["mino"]), len(r["traj"])
        km = np.unique(np.concatenate([np.arange(0, nm, MINO_STRIDE), np.arange(max(0, nm - 40), nm)]))
        kt = np.unique(np.concatenate([np.arange(0, nt, BL_STRIDE), [nt - 1]]))
        rec[f"{name}/case"] = np.array(case, dtype=np.float64)
        rec[f"{name}/insp"] = r["insp"]
        rec[f"{name}/mino_n"] = np.array(nm)
        rec[f"{name}/mino_k"] = km
        rec[f"{name}/mino"] = r["mino"][km]
        rec[f"{name}/traj_n"] = np.array(nt)
        rec[f"{name}/traj_k"] = kt
        rec[f"{name}/traj"] = r["traj"][kt]
        rec[f"{name}/name"] = np.array(r["name"])
        print(name, nm, nt, r["name"])
    ot = np.loadtxt(os.path.join(ref_root, "GenOT", "OT_X_vs_L.dat"))
    rec["ot_ref_every1000"] = ot[::1000]
    os.makedirs(args.out, exist_ok=True)
    path = os.path.join(args.out, "genot_cases.npz")
    np.savez_compressed(path, **rec)
    print("wrote", path, os.path.getsize(path), "bytes")
    return 0


if __name__ == "__main__":
    sys.exit(main())
