"""The CUDA path against the FP64 oracle at the benchmarked and configured
sizes: the 16384 x 256 grid of the default benchmark (the size the HBM
target is quoted at), the 8192 x 128 plunge configuration over 2000 steps
with waveform rows at the outer column and at x = 500, and a batch-engine
request of 16384 x 256 beside a small one.

Tolerances as in the other parity tests: fields within 1e-12 of the field
scale, waveform rows within relative L2 1e-10, times bit-identical.  Each
case starts from a Gaussian pulse placed where the extraction column sees
it within the run (a zero start under the source's (1 - e^{-t/25})^4
turn-on stays at rounding level for the first thousands of steps), and the
sourced cases also carry the plunge source.
"""
import numpy as np
import pytest

import bh_ringdown_b200 as bhr
from bh_ringdown_b200.trajectory import synthetic_plunge
from oracle import pyoracle
from tests.test_source import product_coef_fn

pytestmark = pytest.mark.gpu

WAVE_TOL = 1e-10
FIELD_TOL = 1e-12
XMIN, XMAX, A, MM = -200.0, 600.0, 0.9, 2.0


def rel_field_err(a_planes, b_planes):
    scale = max(np.max(np.abs(b)) for b in b_planes)
    return max(np.max(np.abs(a - b)) for a, b in zip(a_planes, b_planes)) / scale


def col_of(x, N):
    return int(round((x - XMIN) / (XMAX - XMIN) * N))


def setup(N, M, center, ext_col, Fr, T=1000.0, sourced=True, nsteps=30):
    x, r, th = bhr.grid(bhr.Params(N=N, M=M, Xmin=XMIN, Xmax=XMAX, a=A))
    dt = 0.25 * min((XMAX - XMIN) / N, r[0] * np.pi / M)
    prm = bhr.Params(N=N, M=M, Xmin=XMIN, Xmax=XMAX, a=A, m=MM, dt=dt, Fr=Fr, T=T, out_start=0.0, ext_col=ext_col,
                     init_kind=bhr.BHR_INIT_GAUSSIAN, init_center=center, init_width=2.0, init_ell=2.0)
    rows = synthetic_plunge(A, dt / 2.0, duration=max(5.0, 1.2 * nsteps * dt)) if sourced else None
    o = pyoracle.Oracle(N, M, XMIN, XMAX, A, MM, dt, T=T, Fr=Fr, out_start=0.0, ext_col=ext_col)
    o.init_gaussian(center, 2.0, 2.0)
    return prm, rows, o


def test_benchmark_grid_16384x256_matches_oracle():
    """The default benchmark's grid and physics: 16384 x 256 on [-200, 600],
    a=0.9, m=2, plunge source; 30 steps, a waveform row every step at x=10,
    where the pulse sits."""
    N, M, n = 16384, 256, 30
    prm, rows, o = setup(N, M, center=10.0, ext_col=col_of(10.0, N), Fr=1, nsteps=n)
    with bhr.Solver(prm) as s:
        s.set_trajectory(rows)
        s.step(n)
        ts, hs, es = s.waveform()
        gs = s.get_state()
        gt, gi = s.get_source()
    t, h, dedt, steps, _, _ = o.run(traj=rows, coef_fn=product_coef_fn(), nsteps=n)
    assert len(ts) == n and np.array_equal(ts, t)
    assert np.max(np.abs(h)) > 1e-6
    assert rel_field_err(gs, o.get_state()) <= FIELD_TOL
    assert np.linalg.norm(hs - h) <= WAVE_TOL * np.linalg.norm(h)
    assert np.linalg.norm(es - dedt) <= WAVE_TOL * np.linalg.norm(dedt)
    # the deposit of the last step (the oracle holds the source it stepped with)
    ot, oi = o.get_source()
    scale = np.max(np.abs(ot + 1j * oi))
    assert scale > 0
    assert np.max(np.abs((gt + 1j * gi) - (ot + 1j * oi))) <= 1e-12 * scale


@pytest.mark.parametrize("where", ["outer", "x500"])
def test_plunge_8192x128_2000_steps_waveform(where):
    """The plunge configuration's grid, 2000 steps with the plunge source;
    rows every 10 steps at the outer column N-1 (the hyperboloidal layer's
    last point, where the reference extracts) with the pulse started inside
    the layer, or at x = 500 with the pulse started at x = 490."""
    N, M, n = 8192, 128, 2000
    center, ext = (590.0, N - 1) if where == "outer" else (490.0, col_of(500.0, N))
    prm, rows, o = setup(N, M, center=center, ext_col=ext, Fr=10, nsteps=n)
    with bhr.Solver(prm) as s:
        s.set_trajectory(rows)
        s.step(n)
        ts, hs, es = s.waveform()
        gs = s.get_state()
    t, h, dedt, steps, _, _ = o.run(traj=rows, coef_fn=product_coef_fn(), nsteps=n)
    assert len(ts) == n // 10 and np.array_equal(ts, t)
    assert np.max(np.abs(h)) > 1e-6
    assert np.linalg.norm(hs - h) <= WAVE_TOL * np.linalg.norm(h)
    # 2000 steps of rounding differences (fused multiply-adds on the GPU)
    assert rel_field_err(gs, o.get_state()) <= 1e-10


def test_engine_batch_with_a_16384x256_member_matches_oracle():
    """A batch-engine request of the default benchmark's grid (16384 x 256,
    source-free, 30 steps), run beside a small request, against the
    oracle."""
    N, M, n = 16384, 256, 30
    prm, _, o = setup(N, M, center=10.0, ext_col=col_of(10.0, N), Fr=1, sourced=False, nsteps=n)
    prm.T = n * prm.dt * 1.0000001 + 0.0  # a request runs to its final time: n steps
    small = bhr.Params(N=256, M=32, Xmin=-50.0, Xmax=50.0, a=0.5, m=2.0, dt=0.1, Fr=5, T=2.0, out_start=0.0,
                       init_kind=bhr.BHR_INIT_GAUSSIAN, init_center=5.0)
    with bhr.Engine() as e:
        rid = e.submit(prm)
        e.submit(small)
        e.run_all()
        info = e.poll(rid)
        assert info["state"] == bhr.Engine.DONE, info
        tg, hg, dg = e.result(rid)
    nt = info["steps_total"]
    t, h, dedt, steps, _, _ = o.run(nsteps=nt)
    assert nt >= n and len(tg) == nt and np.array_equal(tg, t)
    assert np.max(np.abs(h)) > 1e-6
    assert np.linalg.norm(hg - h) <= WAVE_TOL * np.linalg.norm(h)


@pytest.mark.parametrize("N,M", [(16384, 256), (8192, 128), (1024, 64)])
def test_fused_strip_stages_agree_with_separate_stages(N, M, monkeypatch):
    """The strip12 tiling computes stages 1 and 2 in one launch with u1 kept
    on chip; every point goes through the same row work as the separate
    stage kernels (up to the compiler's fused multiply-add choices, which
    differ between the row work's instantiations for interior and edge
    segments, and the strip cuts the grid into segments differently), so
    after sourced steps the fields and waveform rows agree with the block8n
    tiling's to rounding, and match the oracle."""
    n = 24
    prm, rows, o = setup(N, M, center=10.0, ext_col=col_of(10.0, N), Fr=1, nsteps=n)
    out = {}
    for tiling in ("block8n", "strip12"):
        monkeypatch.setenv("BHR_STAGE_TILING", tiling)
        with bhr.Solver(prm) as s:
            assert s.info()["tiling"] == tiling
            s.set_trajectory(rows)
            s.step(n)
            out[tiling] = (s.get_state(), s.waveform())
    (sa, (ta, ha, _)), (sb, (tb, hb, _)) = out["block8n"], out["strip12"]
    assert rel_field_err(sb, sa) <= 1e-13
    assert np.array_equal(ta, tb) and np.linalg.norm(hb - ha) <= 1e-13 * np.linalg.norm(ha)
    t, h, dedt, steps, _, _ = o.run(traj=rows, coef_fn=product_coef_fn(), nsteps=n)
    assert rel_field_err(sb, o.get_state()) <= FIELD_TOL
    assert np.linalg.norm(hb - h) <= WAVE_TOL * np.linalg.norm(h)
