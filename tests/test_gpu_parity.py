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
    t, h, dedt, steps, _, _ = o.run(nsteps=nsteps)
    ts, hs, es = s.waveform()
    assert len(ts) == len(t) == nsteps // 5
    assert np.array_equal(ts, t)
    assert np.linalg.norm(hs - h) <= WAVE_TOL * np.linalg.norm(h)
    assert np.linalg.norm(es - dedt) <= WAVE_TOL * np.linalg.norm(dedt)


def test_config1_domain_reduced_length_waveform():
    """Config-1 grid (1024 x 64 on [-100, 300], a=0.5, m=2, dt from the
    Courant rule rounded to 0.5M outputs) with extraction at the column
    nearest x=250, for the first 20M."""
    N, M, Xmin, Xmax = 1024, 64, -100.0, 300.0
    x = Xmin + np.arange(N) * (Xmax - Xmin) / N
    col = int(np.argmin(np.abs(x - 250.0)))
    s, o, info = pair(N, M, Xmin, Xmax, 0.5, 2.0, center=20.0, width=2.0, ell=2.0, T=300.0, ext_col=col,
                      courant=0.25, out_every=0.5)
    nsteps = int(round(20.0 / info["dt"]))
    s.step(nsteps)
    t, h, dedt, steps, _, _ = o.run(nsteps=nsteps)
    ts, hs, es = s.waveform()
    assert np.array_equal(ts, t)
    assert np.linalg.norm(hs - h) <= WAVE_TOL * np.linalg.norm(h)
    assert rel_field_err(s.get_state(), o.get_state()) <= FIELD_TOL * 10
