"""The trajectory generator (bh_ringdown_b200.genot, bhr_genot_* in libbhr)
against the reference's own programs.

tests/golden/genot_cases.npz holds what GenOT/ParamWLMino.cc and
GenOT/WL_BL.cc, compiled unchanged, wrote for three cases (equatorial,
inclined, inclined past 90 degrees; both transition models), with this
package's stand-in inspiral table and Ori-Thorne table as their inputs
(tests/golden/make_genot_golden.py), and every 1000th row of the
reference's own Ori-Thorne table.  Where oracle/_ref/genot is built (the
reference tree present), one more case is run through the programs live
and compared row by row.  The programs print 12 decimals (Mino-time rows)
and 13 significant digits (.traj rows): the tolerances are those."""
import glob
import os
import resource
import subprocess

import numpy as np
import pytest

import bh_ringdown_b200 as bhr
from bh_ringdown_b200 import genot
from bh_ringdown_b200.trajectory import read_traj

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
G = np.load(os.path.join(HERE, "golden", "genot_cases.npz"))
CASES = sorted({k.split("/")[0] for k in G.files if "/" in k})
BIN = os.path.join(ROOT, "oracle", "_ref", "genot")


def _as_printed(rows: np.ndarray) -> np.ndarray:
    """Rows as the reference's Mino-time file carries them ("%.12lf")."""
    return np.array([[float("%.12f" % v) for v in r] for r in rows])


def test_ot_table_solves_the_ori_thorne_equation_and_matches_the_reference_table():
    ot = genot.ot_table()
    T, X = ot[:, 0], ot[:, 1]
    assert len(ot) == 43411 and T[0] == -40.0 and abs(T[-1] - 3.41) < 1e-12
    # the reference's table, every 1000th row: same grid, X to its own accuracy
    ref = G["ot_ref_every1000"]
    mine = ot[::1000]
    assert np.allclose(mine[:, 0], ref[:, 0], rtol=0, atol=1e-12)
    lo = ref[:, 0] <= 2.5
    assert np.max(np.abs(mine[lo, 1] - ref[lo, 1])) < 1e-6
    # X'' = -X^2 - T on the grid (second differences: their O(h^2 X'''') truncation
    # grows as X turns over toward its blow-up past T = 3.41)
    h = T[1] - T[0]
    resid = np.abs((X[2:] - 2 * X[1:-1] + X[:-2]) / h ** 2 + X[1:-1] ** 2 + T[1:-1])
    assert np.max(resid[T[1:-1] <= 0.0]) < 1e-7 and np.max(resid[T[1:-1] <= 2.0]) < 2e-5
    # X -> sqrt(-T) + 1/(8 T^2) as T -> -infinity, and the start point does not matter
    assert abs(X[0] - (40.0 ** 0.5 + 1 / (8 * 1600.0))) < 1e-7
    other = genot.ot_table(T_start=-100.0)
    assert np.max(np.abs(other[T <= 2.5, 1] - X[T <= 2.5])) < 1e-9
    # an independent integration (8th-order Dormand-Prince, scipy) of the same equation
    from scipy.integrate import solve_ivp
    u = 400.0
    X0 = u ** 0.5 + u ** -2 / 8 - 49 / 128 * u ** -4.5
    V0 = -(0.5 * u ** -0.5 - 0.25 * u ** -3 + 49 / 128 * 4.5 * u ** -5.5)
    sol = solve_ivp(lambda t, y: [y[1], -y[0] ** 2 - t], (-u, T[-1]), [X0, V0], method="DOP853", rtol=1e-13,
                    atol=1e-14, dense_output=True)
    Xd = sol.sol(T)[0]
    m = T <= 3.3
    assert np.max(np.abs(Xd[m] - X[m]) / np.maximum(1.0, np.abs(X[m]))) < 1e-10


@pytest.mark.parametrize("name", CASES)
def test_stand_in_inspiral_is_the_recorded_input(name):
    a, inc, r_insp = G[f"{name}/case"][:3]
    insp = genot.synthetic_inspiral(a, r_insp, rows=len(G[f"{name}/insp"]), inclination_deg=inc)
    np.testing.assert_allclose(insp, G[f"{name}/insp"], rtol=1e-12, atol=1e-14)
    # Mino time increases, r decreases to the ISCO, fluxes positive
    assert np.all(np.diff(insp[:, 1]) > 0) and np.all(np.diff(insp[:, 2]) < 0) and np.all(insp[:, 8] > 0)


def _mino(name):
    a, inc, r_insp, eta, LTi, LTf, r_start, model = G[f"{name}/case"][:8]
    return genot.mino_worldline(a, eta, G[f"{name}/insp"], LTi, LTf, r_start, model=int(model))


@pytest.mark.parametrize("name", CASES)
def test_mino_worldline_matches_the_reference(name):
    mino = _mino(name)
    assert len(mino) == int(G[f"{name}/mino_n"])
    k = G[f"{name}/mino_k"]
    np.testing.assert_allclose(mino[k], G[f"{name}/mino"], rtol=1e-11, atol=1e-11)


@pytest.mark.parametrize("name", CASES)
def test_bl_worldline_matches_the_reference(name):
    a = G[f"{name}/case"][0]
    lam0, t_stop, chi0, phi0 = G[f"{name}/case"][8:12]
    mino = _as_printed(_mino(name))
    rows, thf, pos = genot.bl_worldline(mino, a, lam0, t_stop, chi0, phi0)
    assert len(rows) == int(G[f"{name}/traj_n"])
    k = G[f"{name}/traj_k"]
    np.testing.assert_allclose(rows[k], G[f"{name}/traj"], rtol=1e-9, atol=1e-10)
    assert genot.traj_name(a, mino[0, 2], thf, pos) == str(G[f"{name}/name"])
    # every stride-th row is the same row
    sub, thf2, _ = genot.bl_worldline(mino, a, lam0, t_stop, chi0, phi0, stride=997)
    assert thf2 == thf and np.array_equal(sub, rows[::997])


def _big_stack():
    resource.setrlimit(resource.RLIMIT_STACK, (64 << 20, resource.getrlimit(resource.RLIMIT_STACK)[1]))


@pytest.mark.skipif(not os.path.exists(os.path.join(BIN, "WL_BL")),
                    reason="oracle/_ref/genot is built only where the reference tree is present")
def test_live_against_the_reference_programs(tmp_path):
    """a = 0.9, inclined 15 degrees, model 1, another mass ratio and
    transition window: every row of both programs' outputs."""
    a, inc, eta, LTi, LTf, r_start, model = 0.9, 15.0, 3e-4, -4.0, 2.6, 3.9, 1
    insp = genot.synthetic_inspiral(a, 4.0, rows=600, inclination_deg=inc)
    np.savetxt(tmp_path / "insp", insp, fmt="%.17g")
    np.savetxt(tmp_path / "OT_X_vs_L.dat", genot.ot_table(), fmt="%.17g", delimiter="\t")
    out = subprocess.run([os.path.join(BIN, "ParamWLMino"), repr(a), repr(eta), "insp", repr(LTi), repr(LTf),
                          repr(r_start), str(model)], cwd=tmp_path, capture_output=True, text=True, check=True)
    (tmp_path / "mino").write_text(out.stdout)
    ref_mino = np.loadtxt(tmp_path / "mino")
    mino = genot.mino_worldline(a, eta, np.loadtxt(tmp_path / "insp"), LTi, LTf, r_start, model=model)
    assert mino.shape == ref_mino.shape
    np.testing.assert_allclose(mino, ref_mino, rtol=1e-11, atol=1e-11)
    subprocess.run([os.path.join(BIN, "WL_BL"), repr(a), "mino", "-50.0", "60.0", "75.0", "5.0"], cwd=tmp_path,
                   capture_output=True, text=True, check=True, preexec_fn=_big_stack)
    (traj,) = glob.glob(str(tmp_path / "*.traj"))
    ref = np.loadtxt(traj)
    (tmp_path / "mine").mkdir()
    path = genot.write_traj(str(tmp_path / "mine"), ref_mino, a, -50.0, 60.0, 75.0, 5.0)
    assert os.path.basename(path) == os.path.basename(traj)
    mine = read_traj(path)
    assert mine.shape == ref.shape
    np.testing.assert_allclose(mine, ref, rtol=1e-9, atol=1e-10)


def test_traj_name_follows_the_reference_format():
    assert genot.traj_name(0.7, 0.0, 90.0, False) == "a0.7_thi000_thf090.0_n.traj"
    assert genot.traj_name(0.5, 5.7, 4.25, True) == "a0.5_thi005_thf004.2_p.traj"
    assert genot.traj_name(0.9, 45.0, 123.45, True) == "a0.9_thi045_thf123.5_p.traj"
    assert genot.traj_name(0.3, 135.2, 170.0, False) == "a0.3_thi135_thf170.0_n.traj"
    # the zero padding is chosen from the value before rounding, as the reference's is
    assert genot.traj_name(0.5, 10.0, 9.96, True) == "a0.5_thi010_thf0010.0_p.traj"


def test_write_traj_makes_a_solver_trajectory(tmp_path):
    name = CASES[0]
    a = G[f"{name}/case"][0]
    mino = _as_printed(_mino(name))
    path = genot.write_traj(str(tmp_path), mino, a, -100.0, 2.0, 30.0, 10.0)
    rows = read_traj(path)
    assert rows.shape == (2001, 10) and os.path.dirname(path) == str(tmp_path)
    np.testing.assert_allclose(rows[:, 0], np.arange(2001) * 0.001, atol=1e-9)


def test_bad_inputs_are_rejected():
    name = CASES[0]
    a, inc, r_insp, eta, LTi, LTf, r_start, model = G[f"{name}/case"][:8]
    insp = G[f"{name}/insp"]
    with pytest.raises(bhr.BhrError, match="model"):
        genot.mino_worldline(a, eta, insp, LTi, LTf, r_start, model=3)
    with pytest.raises(bhr.BhrError, match="LTf"):
        genot.mino_worldline(a, eta, insp, LTi, 3.5, r_start)
    with pytest.raises(bhr.BhrError, match="r_start"):
        genot.mino_worldline(a, eta, insp, LTi, LTf, insp[0, 2] + 1.0)
    with pytest.raises(ValueError):
        genot.synthetic_inspiral(0.7, 3.0)
    twice = np.array(insp)
    twice[5, 1] = twice[4, 1]  # a repeated Mino time
    with pytest.raises(bhr.BhrError, match="increase"):
        genot.mino_worldline(a, eta, twice, LTi, LTf, r_start)
    mino = _mino(name)
    back = np.array(mino[:50])
    back[10, 0] = back[9, 0]
    with pytest.raises(bhr.BhrError, match="increase"):
        genot.bl_worldline(back, a, float(back[2, 0]), 1.0)


@pytest.mark.gpu
def test_inclined_genot_worldline_drives_the_solver_as_the_oracle():
    """The inclined case's worldline (theta oscillating, dtheta/dt != 0),
    sampled at dt/2 of a 256 x 32 solve, as the particle source: the CUDA
    path against the oracle, fields and waveform."""
    from oracle import pyoracle
    from tests.test_gpu_parity import FIELD_TOL, WAVE_TOL, rel_field_err
    from tests.test_source import product_coef_fn
    name = "inc30_a03"
    a = G[f"{name}/case"][0]
    N, M, Xmin, Xmax, m, n = 256, 32, -50.0, 50.0, 2.0, 300
    dt = 0.25 * (Xmax - Xmin) / N
    rows, _, _ = genot.bl_worldline(_as_printed(_mino(name)), a, -200.0, (n + 2) * dt, 40.0, 0.0, dt=dt / 2.0)
    assert np.ptp(rows[:, 2]) > 0.05 and np.max(np.abs(rows[:, 4])) > 1e-3  # theta moves
    prm = bhr.Params(N=N, M=M, Xmin=Xmin, Xmax=Xmax, a=a, m=m, dt=dt, Fr=5, T=100.0, out_start=0.0, ext_col=154)
    with bhr.Solver(prm) as s:
        s.set_trajectory(rows)
        s.step(n)
        ts, hs, _ = s.waveform()
        gs = s.get_state()
    o = pyoracle.Oracle(N, M, Xmin, Xmax, a, m, dt, T=100.0, Fr=5, out_start=0.0, ext_col=154)
    t, h, _, _, _, _ = o.run(traj=rows, coef_fn=product_coef_fn(), nsteps=n)
    assert np.array_equal(ts, t) and np.max(np.abs(h)) > 0
    assert rel_field_err(gs, o.get_state()) <= FIELD_TOL
    assert np.linalg.norm(hs - h) <= WAVE_TOL * np.linalg.norm(h)
