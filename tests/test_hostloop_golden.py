"""The host loop of HighOrder/body.cu against the reference itself.

tests/golden/hostloop_gpin_a06_m2.npz holds what the reference's own body()
and kern.cu, compiled unchanged for sm_100a and run on a GPU
(tests/golden/make_hostloop_golden.py), produced for one sourced mode on a
256 x 32 grid over 3072 steps: the waveform file (rows from
t = Xmax + 200, HighOrder/body.cu:204-208) and the dE/dt lines it prints
every Fr steps (HighOrder/body.cu:209-210), with the trajectory it read.
That pins, through the reference's outputs, what the kernel fixtures do
not: the trajectory cursor (two rows per step, rp + 1e-6, backward
differences; HighOrder/body.cu:97-124), the rectangle-rule integrals
int and dint and dE/dt (:174-187), the projections (:189-202) and the
output cadence (:204-212).

The reference prints six significant digits (%g) and the time with %lf,
so values are compared to that: within 6e-6 of the printed value's
magnitude (a cursor one row off, or a missing factor, changes them by
orders of magnitude more).  The CPU test holds the oracle to the fixture;
the GPU test holds the CUDA path to it.
"""
import os

import numpy as np
import pytest

import bh_ringdown_b200 as bhr
from oracle import pyoracle
from tests.test_source import product_coef_fn

GOLD = os.path.join(os.path.dirname(__file__), "golden", "hostloop_gpin_a06_m2.npz")
REL = 6e-6


def fixture():
    if not os.path.exists(GOLD):
        pytest.skip("hostloop fixture not generated")
    return np.load(GOLD)


def check_against_reference(g, t, h, dedt):
    """t, h (rows x 14), dedt: rows every Fr steps from k = 0 (out_start 0)."""
    Xmax, Fr, dt = float(g["Xmax"]), int(g["Fr"]), float(g["dt"])
    # dE/dt lines: timer and dE/dt on every step k % Fr == 0 (HighOrder/body.cu:210)
    ref_d = g["dedt"]
    n = len(ref_d)
    assert n > 10 and len(t) >= n
    assert np.allclose(t[:n] + Xmax, ref_d[:, 0], rtol=0, atol=1e-6)
    assert np.max(np.abs(dedt[:n] - ref_d[:, 1]) / np.maximum(np.abs(ref_d[:, 1]), 1e-300)) <= REL
    assert np.max(np.abs(ref_d[:, 1])) > 0
    # the waveform file: rows from k dt >= Xmax + 200
    wave = g["wave"]
    first = next(i for i in range(len(t)) if i * Fr * dt >= Xmax + 200.0)
    assert len(wave) > 5 and len(t) >= first + len(wave)
    sel = slice(first, first + len(wave))
    assert np.allclose(t[sel], wave[:, 0], rtol=0, atol=1e-6)
    ref_h = wave[:, 1:]
    got = h[sel]
    scale = np.maximum(np.abs(ref_h), 1e-300)
    assert np.max(np.abs(got - ref_h) / scale) <= REL
    assert np.max(np.abs(ref_h)) > 0


def test_oracle_host_loop_matches_reference_body():
    g = fixture()
    N, M, a, m, dt = int(g["N"]), int(g["M"]), float(g["a"]), float(g["m"]), float(g["dt"])
    o = pyoracle.Oracle(N, M, float(g["Xmin"]), float(g["Xmax"]), a, m, dt, T=float(g["T"]), Fr=int(g["Fr"]),
                        out_start=0.0)
    t, h, dedt, steps, _, _ = o.run(traj=g["traj"], coef_fn=product_coef_fn(), nsteps=int(g["nt"]))
    check_against_reference(g, t, h, dedt)


@pytest.mark.gpu
def test_cuda_host_loop_matches_reference_body():
    g = fixture()
    prm = bhr.Params(N=int(g["N"]), M=int(g["M"]), Xmin=float(g["Xmin"]), Xmax=float(g["Xmax"]), a=float(g["a"]),
                     m=float(g["m"]), dt=float(g["dt"]), T=float(g["T"]), Fr=int(g["Fr"]), out_start=0.0)
    with bhr.Solver(prm) as s:
        s.set_trajectory(g["traj"])
        assert s.info()["nt"] == int(g["nt"])
        s.run()
        t, h, dedt = s.waveform()
    check_against_reference(g, t, h, dedt)
