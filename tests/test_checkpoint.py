"""Checkpoint and resume: a solve checkpointed part-way and restored into a
fresh solve with the same parameters (and trajectory) continues
bit-identically to an uninterrupted run -- fields, waveform rows and the
source patch."""
import numpy as np
import pytest

import bh_ringdown_b200 as bhr

pytestmark = pytest.mark.gpu


def params(sourced):
    dt = 0.25 * 100.0 / 256
    kw = dict(N=256, M=32, Xmin=-50.0, Xmax=50.0, a=0.6, m=2.0, dt=dt, Fr=5, T=100.0, out_start=0.0, ext_col=154)
    if not sourced:
        kw.update(init_kind=bhr.BHR_INIT_GAUSSIAN, init_center=5.0, init_width=2.0, init_ell=2.0)
    return bhr.Params(**kw)


@pytest.mark.parametrize("sourced", [False, True])
def test_resume_is_bit_identical(sourced):
    from bh_ringdown_b200.trajectory import synthetic_plunge
    prm = params(sourced)
    rows = synthetic_plunge(0.6, prm.dt / 2.0, duration=prm.T) if sourced else None

    def make():
        s = bhr.Solver(prm)
        if sourced:
            s.set_trajectory(rows)
        return s
    with make() as ref:
        ref.step(300)
        t0, h0, e0 = ref.waveform()
        st0 = ref.get_state()
    with make() as a:
        a.step(137)
        ck = a.checkpoint()
    with make() as b:
        b.step(11)  # whatever it did before is replaced
        b.restore(ck)
        assert b.info()["steps_done"] == 137
        b.step(163)
        t1, h1, e1 = b.waveform()
        st1 = b.get_state()
    assert len(t0) == 60 and np.array_equal(t0, t1) and np.array_equal(h0, h1) and np.array_equal(e0, e1)
    assert all(np.array_equal(x, y) for x, y in zip(st0, st1))


def test_checkpoint_of_another_solve_is_rejected():
    with bhr.Solver(params(False)) as a:
        a.step(3)
        ck = a.checkpoint()
    other = params(False)
    other.m = 3.0
    with bhr.Solver(other) as b:
        with pytest.raises(bhr.BhrError) as e:
            b.restore(ck)
        assert e.value.status == 1
        with pytest.raises(bhr.BhrError):
            b.restore(ck[:100])
