"""The drop-in, run for real: the reference's own main.c (its m = -5..5
loop over body(), aa = 1e-8, dt = 0.002; HighOrder/main.c:25-55) and
proj.c, built as HighOrder/build.sh builds them, with
bh_ringdown_b200/integration/body_bhr.c in place of body.cu and kern.cu,
linked to libbhr.so (oracle/build_ref.py, tag "dropin": 256 x 32 on
[-50, 50], T = 270, Fr = 50).

It reads its trajectory where body() does, ../Trajectories/
a0.0_thi000_thf090.0_n.traj (HighOrder/body.cu:77), here written as the
reference's workflow writes it: GenOT's transition-to-plunge worldline
(bh_ringdown_b200.genot, a = 1e-8, mass ratio 1e-3) sampled at dt/2; it
writes one waveform file per m.
The test checks the eleven files' names and row format (the columns
QNM_Extraction's loadwaveforms reads: time, then h+ and hx for
l = |m|..|m|+6, QNM_Extraction/Library/ringdownlib.py:102-109), that the
rows start at t = Xmax + 200 every Fr steps, and that the m = 2 file is
byte-identical to the same solve run through the Python binding.  Both runs
fix the stage tiling (BHR_STAGE_TILING): the autotuner times the tilings in
each process, and different tilings agree to rounding, not bit for bit."""
import os
import subprocess

import numpy as np
import pytest

import bh_ringdown_b200 as bhr
from bh_ringdown_b200.genot import transition_plunge

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "oracle", "_ref", "dropin_run")
NAME = "a0.0_thi000_thf090.0_n"
N, M, XMIN, XMAX, T, FR = 256, 32, -50.0, 50.0, 270.0, 50
AA, DT = 1e-8, 0.002  # HighOrder/main.c:41,46
TILING = "block8n"


@pytest.fixture(scope="module")
def dropin_run(tmp_path_factory):
    if not os.path.exists(EXE):
        pytest.skip("oracle/_ref/dropin_run is built only where the reference tree is present")
    work = tmp_path_factory.mktemp("dropin")
    (work / "Trajectories").mkdir()
    (work / "run").mkdir()
    traj = work / "Trajectories" / f"{NAME}.traj"
    # from the start of the transition near the ISCO through the plunge
    np.savetxt(traj, transition_plunge(AA, 1e-3, DT / 2.0, T), fmt="%.17g")
    env = dict(os.environ, BHR_STAGE_TILING=TILING)
    out = subprocess.run([EXE], cwd=work / "run", capture_output=True, text=True, timeout=900, env=env)
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr[-2000:]
    assert "bhr:" not in out.stderr, out.stderr[-2000:]
    return work


def test_dropin_writes_one_reference_format_file_per_mode(dropin_run):
    for m in range(-5, 6):
        fn = dropin_run / "run" / (f"hm{m}_{NAME}.dat" if m >= 0 else f"hmm{-m}_{NAME}.dat")
        assert fn.exists(), fn
        rows = [ln.split() for ln in fn.read_text().strip().splitlines()]
        assert len(rows) >= 190 and all(len(r) == 15 for r in rows)
        t = np.array([float(r[0]) for r in rows])
        # body.cu:204-208: t - Xmax on steps k % Fr == 0 once k dt >= Xmax + 200
        assert t[0] >= 200.0 - 1e-9 and np.allclose(np.diff(t), FR * DT, rtol=0, atol=1e-6)
        # what loadwaveforms takes: the header line dropped, h+ of l=|m| in column 1
        data = np.loadtxt(fn, skiprows=1)
        assert data.shape[1] == 15 and np.all(np.isfinite(data))
        assert np.max(np.abs(data[:, 1:])) > 0


def test_dropin_m2_file_equals_the_python_binding_run(dropin_run, tmp_path, monkeypatch):
    monkeypatch.setenv("BHR_STAGE_TILING", TILING)
    prm = bhr.Params(N=N, M=M, Xmin=XMIN, Xmax=XMAX, T=T, Fr=FR, PTSX=128, PTSY=128, out_start=XMAX + 200.0,
                     mass=1.0, a=AA, m=2.0, dt=DT, device=0)
    with bhr.Solver(prm) as s:
        assert s.info()["tiling"] == TILING
        s.load_trajectory(str(dropin_run / "Trajectories" / f"{NAME}.traj"))
        s.run(str(tmp_path), NAME)
    for suffix in (".dat", ".dat.full"):
        a = (dropin_run / "run" / f"hm2_{NAME}{suffix}").read_bytes()
        b = (tmp_path / f"hm2_{NAME}{suffix}").read_bytes()
        assert a == b, suffix
