"""Generate tests/golden/hostloop_gpin_a06_m2.npz: the reference's whole
host loop, run by the reference itself.

HighOrder/body.cu (the trajectory cursor of :97-124, the double time
integration and dE/dt of :168-187, the projections and the output rows of
:189-212) and HighOrder/kern.cu, compiled unchanged by nvcc for sm_100a
into oracle/_ref/refgpu_gpin (oracle/build_ref.py, grid 256 x 32 on
[-50, 50], T = 300, Fr = 50), are run on a GPU for one mode.  The inputs
are a synthetic prograde equatorial plunge (bh_ringdown_b200.trajectory,
rows every dt/2) written where body() reads it; the outputs recorded are
the hm02 waveform file (rows from t = Xmax + 200, six significant digits,
HighOrder/body.cu:208) and the dE/dt lines body() prints every Fr steps
(HighOrder/body.cu:210).  Nothing of the host loop is restated here: this
script only writes the trajectory file and reads the reference's outputs.

Needs a GPU and the built oracle/_ref/refgpu_gpin (made where the
reference tree is present):

    python tests/golden/make_hostloop_golden.py --out <dir>
    cp <dir>/hostloop_gpin_a06_m2.npz tests/golden/
"""
from __future__ import annotations

import argparse
import glob
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

N, M, XMIN, XMAX, T, FR = 256, 32, -50.0, 50.0, 300.0, 50
A, MM = 0.6, 2.0
DT = 0.25 * (XMAX - XMIN) / N
TRAJ_DURATION = 300.0


def trajectory():
    from bh_ringdown_b200.trajectory import synthetic_plunge
    return synthetic_plunge(A, DT / 2.0, duration=TRAJ_DURATION)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    args = ap.parse_args()
    exe = os.path.join(ROOT, "oracle", "_ref", "refgpu_gpin")
    if not os.path.exists(exe):
        raise SystemExit(f"{exe} not built (oracle/build_ref.py gpin, where the reference tree is present)")
    rows = trajectory()
    with tempfile.TemporaryDirectory() as work:
        os.makedirs(os.path.join(work, "Trajectories"))
        os.makedirs(os.path.join(work, "run"))
        np.savetxt(os.path.join(work, "Trajectories", "a0.0_thi000_thf090.0_n.traj"), rows, fmt="%.17g")
        out = subprocess.run([exe, work, "%.17g" % A, "%.17g" % MM, "%.17g" % DT], capture_output=True, text=True,
                             timeout=600)
        if out.returncode != 0:
            raise SystemExit(f"refgpu_gpin failed ({out.returncode}):\n{out.stdout[-2000:]}\n{out.stderr[-2000:]}")
        lines = out.stdout.strip().splitlines()
        info = json.loads(lines[-1])
        dedt = []
        for ln in lines[:-1]:
            parts = ln.split()
            if len(parts) == 2:
                try:
                    dedt.append((float(parts[0]), float(parts[1])))
                except ValueError:
                    pass
        files = glob.glob(os.path.join(work, "run", "*.dat"))
        if len(files) != 1:
            raise SystemExit(f"expected one waveform file, found {files}")
        text = open(files[0]).read()
    wave = np.array([[float(v) for v in ln.split()] for ln in text.strip().splitlines()])
    np.savez_compressed(os.path.join(args.out, "hostloop_gpin_a06_m2.npz"), N=N, M=M, Xmin=XMIN, Xmax=XMAX, T=T, Fr=FR,
                        a=A, m=MM, dt=DT, traj_duration=TRAJ_DURATION, traj=rows, nt=info["nt"], wave=wave,
                        wave_file=os.path.basename(files[0]), dedt=np.array(dedt), seconds=info["seconds"])
    print(json.dumps({"rows": len(wave), "dedt_lines": len(dedt), **info}))


if __name__ == "__main__":
    main()
