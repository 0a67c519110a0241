"""CUDA path (through the C ABI) against the FP64 CPU oracle.

Tolerances: field planes within 1e-12 of the field scale after tens of
steps; waveform rows (h+, hx for l = |m|..|m|+6) within relative L2 1e-10,
the FP64 bar of the solver; times bit-identical.
"""
import numpy as np
import pytest

import bh_ringdown_b200 as bhr
from oracle import pyoracle

pytestmark = pytest.mark.gpu

WAVE_TOL = 1e-10
FIELD_TOL = 1e-12


def pair(N, M, Xmin, Xmax, a, m, dt=None, center=5.0, width=2.0, ell=2.0, Fr=1, T=100.0, ext_col=-1,
         courant=0.25, out_every=0.0):
    prm = bhr.Params(N=N, M=M, Xmin=Xmin, Xmax=Xmax, a=a, m=m, dt=dt if dt else 0.0, courant=courant,
                     out_every=out_every, Fr=Fr, T=T, out_start=0.0, ext_col=ext_col,
                     init_kind=bhr.BHR_INIT_GAUSSIAN, init_center=center, init_width=width, init_ell=ell)
    s = bhr.Solver(prm)
    info = s.info()
    o = pyoracle.Oracle(N, M, Xmin, Xmax, a, m, info["dt"], T=T, Fr=info["Fr"], out_start=0.0, ext_col=ext_col)
    o.init_gaussian(center, width, ell)
    return s, o, info


def rel_field_err(a_planes, b_planes):
    scale = max(np.max(np.abs(b)) for b in b_planes)
    return max(np.max(np.abs(a - b)) for a, b in zip(a_planes, b_planes)) / scale


@pytest.mark.parametrize("a,m,center", [(0.6, 2.0, 5.0), (0.3, 3.0, 40.0), (0.9, -1.0, 0.0), (0.5, 0.0, 10.0)])
def test_initial_state_and_steps_match_oracle(a, m, center):
    N, M, Xmin, Xmax = 256, 32, -50.0, 50.0
    s, o, info = pair(N, M, Xmin, Xmax, a, m, dt=0.25 * (Xmax - Xmin) / N, center=center,
                      ell=max(2.0, abs(m)))
    assert rel_field_err(s.get_state(), o.get_state()) <= 1e-15
    for k in (1, 9, 30):
        s.step(k)
        o.step(k)
        assert rel_field_err(s.get_state(), o.get_state()) <= FIELD_TOL, k
    er, ei = o.ext()
    pr, pi, *_ = s.get_extraction()
    scale = max(np.max(np.abs(x)) for x in o.get_state()[:2])
    assert max(np.max(np.abs(pr - er)), np.max(np.abs(pi - ei))) <= FIELD_TOL * scale


@pytest.mark.parametrize("m", [2.0, -3.0])
def test_waveform_rows_match_oracle(m):
    """Extraction at column N-1, rectangle-rule double time integral and
    Boole/swsh projection every Fr steps (HighOrder/body.cu:174-212)."""
    N, M, Xmin, Xmax = 512, 64, -50.0, 50.0
    s, o, info = pair(N, M, Xmin, Xmax, 0.7, m, dt=0.3 * (Xmax - Xmin) / N, center=30.0, ell=max(2.0, abs(m)),
                      Fr=5)
    nsteps = 600
    s.step(nsteps)
    t, h, dedt, steps, er, ei = o.run(nsteps=nsteps, ext_every=5, max_ext=nsteps // 5)
    ts, hs, es = s.waveform()
    assert len(ts) == len(t) == nsteps // 5
    assert np.array_equal(ts, t)
    assert np.linalg.norm(hs - h) <= WAVE_TOL * np.linalg.norm(h)
    assert np.linalg.norm(es - dedt) <= WAVE_TOL * np.linalg.norm(dedt)
    # the raw psi(theta) samples behind the rows (kern.cu:750-751 column copy)
    pr, pi = s.psi_samples()
    assert pr.shape == er.shape == (nsteps // 5, M)
    scale = max(np.max(np.abs(er)), np.max(np.abs(ei)))
    assert scale > 1e-8
    assert max(np.max(np.abs(pr - er)), np.max(np.abs(pi - ei))) <= FIELD_TOL * scale


def test_config1_full_length_waveform():
    """Config 1 at full size and length: 1024 x 64 on [-100, 300], a=0.5,
    m=2, dt from the Courant rule rounded so 0.5M outputs are whole steps,
    psi0 = exp(-(x-20)^2/8) swsh(2,2), extraction at the column nearest
    x=250, T=300."""
    N, M, Xmin, Xmax = 1024, 64, -100.0, 300.0
    x = Xmin + np.arange(N) * (Xmax - Xmin) / N
    col = int(np.argmin(np.abs(x - 250.0)))
    s, o, info = pair(N, M, Xmin, Xmax, 0.5, 2.0, center=20.0, width=2.0, ell=2.0, T=300.0, ext_col=col,
                      courant=0.25, out_every=0.5)
    nsteps = info["nt"]
    s.step(nsteps)
    t, h, dedt, steps, _, _ = o.run(nsteps=nsteps)
    ts, hs, es = s.waveform()
    assert np.array_equal(ts, t)
    assert np.linalg.norm(hs - h) <= WAVE_TOL * np.linalg.norm(h)
    # 13200 steps: rounding differences (fused multiply-adds on the GPU) grow
    # to ~1e-9 of the field scale; the waveform bar above is the parity bar.
    gs, os_ = s.get_state(), o.get_state()
    err = rel_field_err(gs, os_)
    where = np.unravel_index(np.argmax(np.abs(gs[0] - os_[0])), gs[0].shape)
    assert err <= 1e-8, (err, where)


def traj_pair(N, M, Xmin, Xmax, a, m, Fr=5, T=100.0, PTSX=128, PTSY=128, ext_col=-1):
    from bh_ringdown_b200.trajectory import synthetic_plunge
    from tests.test_source import product_coef_fn
    dt = 0.25 * (Xmax - Xmin) / N
    prm = bhr.Params(N=N, M=M, Xmin=Xmin, Xmax=Xmax, a=a, m=m, dt=dt, Fr=Fr, T=T, out_start=0.0,
                     PTSX=PTSX, PTSY=PTSY, ext_col=ext_col)
    rows = synthetic_plunge(a, dt / 2.0, duration=T)
    s = bhr.Solver(prm)
    s.set_trajectory(rows)
    o = pyoracle.Oracle(N, M, Xmin, Xmax, a, m, dt, T=T, Fr=Fr, out_start=0.0, PTSX=PTSX, PTSY=PTSY,
                        ext_col=ext_col)
    return s, o, rows, product_coef_fn()


@pytest.mark.parametrize("a,m", [(0.6, 2.0), (0.9, -3.0)])
def test_plunge_sourced_run_matches_oracle(a, m):
    """Source from a plunge worldline: trajectory cursor (two rows per step,
    rp + 1e-6, backward-difference accelerations), patch placement, Gaussian
    approximants, tilde-phi phase, turn-on, and the evolution it drives."""
    s, o, rows, coef = traj_pair(256, 32, -50.0, 50.0, a, m)
    n = 300
    # the turn-on window (1 - exp(-t/25))^4 is zero at step 0; compare the
    # deposit of step 20
    s.step(21)
    o.run(traj=rows, coef_fn=coef, nsteps=21, max_rows=10)
    gt, gi = s.get_source()
    ot, oi = o.get_source()
    scale = np.max(np.abs(ot + 1j * oi))
    assert scale > 0
    assert np.max(np.abs((gt + 1j * gi) - (ot + 1j * oi))) <= 1e-12 * scale
    # full run from scratch, extracting at x = 10 where the driven field is
    s2, o2, rows, coef = traj_pair(256, 32, -50.0, 50.0, a, m, ext_col=154)
    s2.step(n)
    t, h, dedt, steps, _, _ = o2.run(traj=rows, coef_fn=coef, nsteps=n)
    ts, hs, es = s2.waveform()
    assert np.array_equal(ts, t)
    assert rel_field_err(s2.get_state(), o2.get_state()) <= FIELD_TOL
    assert np.linalg.norm(hs - h) <= WAVE_TOL * np.linalg.norm(h)


def test_source_patch_clipped_at_the_grid_edge():
    """Patch columns at or past N are dropped (the reference writes past the
    row end there); the grid is narrow enough that the 128-wide patch of a
    particle near r=3.5 reaches past column N-1."""
    s, o, rows, coef = traj_pair(128, 16, -50.0, 50.0, 0.6, 2.0)
    s.step(5)
    o.run(traj=rows, coef_fn=coef, nsteps=5, max_rows=10)
    assert rel_field_err(s.get_state(), o.get_state()) <= FIELD_TOL


def test_headline_workload_grid_matches_oracle():
    """The benchmark workload at full size: 8192 x 128 on [-200, 600],
    a=0.9, m=2, plunge source; 40 steps on both paths."""
    from bh_ringdown_b200.trajectory import synthetic_plunge
    from tests.test_source import product_coef_fn
    N, M, Xmin, Xmax, a, m = 8192, 128, -200.0, 600.0, 0.9, 2.0
    x, r, th = bhr.grid(bhr.Params(N=N, M=M, Xmin=Xmin, Xmax=Xmax, a=a))
    dt = 0.25 * min((Xmax - Xmin) / N, r[0] * np.pi / M)
    prm = bhr.Params(N=N, M=M, Xmin=Xmin, Xmax=Xmax, a=a, m=m, dt=dt, Fr=10, T=1000.0, out_start=0.0)
    rows = synthetic_plunge(a, dt / 2.0, duration=5.0)
    s = bhr.Solver(prm)
    s.set_trajectory(rows)
    o = pyoracle.Oracle(N, M, Xmin, Xmax, a, m, dt, T=1000.0, Fr=10, out_start=0.0)
    s.step(40)
    o.run(traj=rows, coef_fn=product_coef_fn(), nsteps=40, max_rows=10)
    assert rel_field_err(s.get_state(), o.get_state()) <= FIELD_TOL


@pytest.mark.parametrize("tiling", ["block8", "block16", "persistent", "block8n", "ring", "strip12"])
def test_every_stage_tiling_matches_oracle(tiling, monkeypatch):
    """Each stage tiling (8- and 16-row tiles one per block, persistent
    blocks walking 16-row tiles, or 8-row tiles two blocks per SM, through
    two buffers) on a sourced plunge whose grid has several tiles per
    persistent block and a patch that crosses tile edges."""
    monkeypatch.setenv("BHR_STAGE_TILING", tiling)
    s, o, rows, coef = traj_pair(1024, 64, -50.0, 50.0, 0.7, 2.0, ext_col=640)
    info = s.info()
    assert info["tiling"] == tiling
    assert info["persistent"] == (tiling in ("persistent", "ring"))
    assert info["tile_rows"] == (8 if tiling in ("block8", "block8n", "ring", "strip12") else 16)
    n = 120
    s.step(n)
    t, h, dedt, steps, _, _ = o.run(traj=rows, coef_fn=coef, nsteps=n)
    ts, hs, es = s.waveform()
    assert np.array_equal(ts, t)
    assert rel_field_err(s.get_state(), o.get_state()) <= FIELD_TOL
    assert np.linalg.norm(hs - h) <= WAVE_TOL * np.linalg.norm(h)


@pytest.mark.parametrize("tiling", ["block16", "persistent", "ring", "strip12"])
def test_trajectory_set_after_stepping(tiling, monkeypatch):
    """A step taken before the trajectory is set captures the step graph
    without a source; setting the trajectory must rebuild what was captured.
    The turn-on window (1 - exp(-t/25))^4 is zero at t = 0, so one step
    without the source equals the oracle's first sourced step."""
    monkeypatch.setenv("BHR_STAGE_TILING", tiling)
    s, o, rows, coef = traj_pair(256, 32, -50.0, 50.0, 0.6, 2.0, ext_col=154)
    s2 = bhr.Solver(s.params)
    s2.step(1)
    s2.set_trajectory(rows)
    n = 80
    s2.step(n - 1)
    o.run(traj=rows, coef_fn=coef, nsteps=n)
    assert rel_field_err(s2.get_state(), o.get_state()) <= FIELD_TOL
    s2.close()
    s.close()


def test_long_trajectory_records_built_while_stepping():
    """A trajectory longer than the source records built up front (8192
    steps): the rest are built on a host thread while the solver steps.  The
    waveform over 12000 steps, past the first chunk boundary, matches the
    oracle, which forms every step's source itself."""
    from bh_ringdown_b200.trajectory import synthetic_plunge
    from tests.test_source import product_coef_fn
    N, M, Xmin, Xmax, a = 256, 32, -50.0, 50.0, 0.6
    dt = 0.25 * (Xmax - Xmin) / N
    prm = bhr.Params(N=N, M=M, Xmin=Xmin, Xmax=Xmax, a=a, m=2.0, dt=dt, Fr=50, T=1500.0, out_start=0.0,
                     ext_col=154)
    rows = synthetic_plunge(a, dt / 2.0, duration=200.0)
    n = 12000
    with bhr.Solver(prm) as s:
        s.set_trajectory(rows)
        s.step(n)                            # races the record thread
        ts, hs, _ = s.waveform()
        gs = s.get_state()
    o = pyoracle.Oracle(N, M, Xmin, Xmax, a, 2.0, dt, T=1500.0, Fr=50, out_start=0.0, ext_col=154)
    t, h, _, _, _, _ = o.run(traj=rows, coef_fn=product_coef_fn(), nsteps=n)
    assert len(ts) == n // 50 and np.array_equal(ts, t) and np.max(np.abs(h)) > 0
    assert np.linalg.norm(hs - h) <= WAVE_TOL * np.linalg.norm(h)
    assert rel_field_err(gs, o.get_state()) <= 1e-9  # 12000 steps of rounding


@pytest.mark.parametrize("tiling", ["block8", "block16", "persistent", "block8n", "ring", "strip12"])
@pytest.mark.parametrize("N,M", [(64, 16), (128, 16), (192, 32)])
def test_tiny_grids_every_tiling(tiling, N, M, monkeypatch):
    """Grids of one to a dozen tiles, every tile at an edge, persistent
    kernels with more block slots than tiles: each tiling against the
    oracle."""
    monkeypatch.setenv("BHR_STAGE_TILING", tiling)
    Xmin, Xmax = -20.0, 20.0
    s, o, info = pair(N, M, Xmin, Xmax, 0.7, 2.0, dt=0.2 * (Xmax - Xmin) / N, center=0.0, width=2.0)
    assert info["tiling"] == tiling
    s.step(20)
    o.step(20)
    assert rel_field_err(s.get_state(), o.get_state()) <= FIELD_TOL
    s.close()


_PREFETCH_RUN = """
import sys
import numpy as np
import bh_ringdown_b200 as bhr
from bh_ringdown_b200.trajectory import synthetic_plunge
N, M, Xmin, Xmax, a = 1024, 64, -50.0, 50.0, 0.7
dt = 0.25 * (Xmax - Xmin) / N
prm = bhr.Params(N=N, M=M, Xmin=Xmin, Xmax=Xmax, a=a, m=2.0, dt=dt, Fr=5, T=100.0, out_start=0.0, ext_col=640)
with bhr.Solver(prm) as s:
    assert s.info()["tiling"] == "block8n", s.info()
    s.set_trajectory(synthetic_plunge(a, dt / 2.0, duration=100.0))
    s.step(60)
    t, h, _ = s.waveform()
    np.savez(sys.argv[1], state=np.array(s.get_state()), h=h, ahead=s.info()["prefetch_ahead"])
"""


def test_l2_prefetch_distance_does_not_change_results(tmp_path):
    """The L2 prefetch is only a hint: a sourced block8n solve with it off,
    at the default distance and past the end of the grid gives bit-identical
    fields and waveform (each in its own process: the distance override is
    read once per process)."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    runs = {}
    for ahead in ("0", "296", "100000"):
        env = dict(os.environ, BHR_STAGE_TILING="block8n", BHR_PREFETCH_AHEAD=ahead)
        f = tmp_path / f"run{ahead}.npz"
        subprocess.run([sys.executable, "-c", _PREFETCH_RUN, str(f)], env=env, cwd=root, check=True, timeout=600)
        runs[ahead] = np.load(f)
        assert int(runs[ahead]["ahead"]) == int(ahead)
    for ahead in ("296", "100000"):
        assert np.array_equal(runs[ahead]["state"], runs["0"]["state"])
        assert np.array_equal(runs[ahead]["h"], runs["0"]["h"])


@pytest.mark.parametrize("tiling", ["block8n", "block16", "block8"])
@pytest.mark.parametrize("N,M,a,m", [(320, 48, 0.3, 1.0), (448, 80, 0.95, -2.0), (1088, 112, 0.6, 3.0)])
def test_odd_tile_counts_with_a_source(tiling, N, M, a, m, monkeypatch):
    """Grids whose tile counts are odd and not multiples of the SM count
    (5, 7 or 17 column tiles, 3, 5 or 7 of 16 rows; a partial last wave,
    the L2 prefetch reaching past the end and into the next stage's tiles),
    with a plunge source crossing tile edges: each tiling against the
    oracle."""
    monkeypatch.setenv("BHR_STAGE_TILING", tiling)
    s, o, rows, coef = traj_pair(N, M, -50.0, 50.0, a, m, ext_col=N * 6 // 10)
    assert s.info()["tiling"] == tiling
    n = 60
    s.step(n)
    t, h, _, _, _, _ = o.run(traj=rows, coef_fn=coef, nsteps=n)
    ts, hs, _ = s.waveform()
    assert np.array_equal(ts, t)
    assert rel_field_err(s.get_state(), o.get_state()) <= FIELD_TOL
    assert np.linalg.norm(hs - h) <= WAVE_TOL * np.linalg.norm(h)
    s.close()
