"""Failure detection, all without a GPU fault: errors are made on the host
(bad files, bad values, a rank that exits), or by a bounded device wait that
runs out and reports BHR_TIMEOUT to the host.
"""
import os
import socket
import time

import numpy as np
import pytest
import torch.multiprocessing as mp

import bh_ringdown_b200 as bhr
from bh_ringdown_b200 import replicas


def small_params(**kw):
    prm = bhr.Params(N=256, M=32, Xmin=-50.0, Xmax=50.0, a=0.5, m=2.0, dt=0.04, T=20.0, Fr=1, out_start=0.0,
                     init_kind=bhr.BHR_INIT_GAUSSIAN, init_center=5.0, init_width=2.0, init_ell=2.0)
    for k, v in kw.items():
        setattr(prm, k, v)
    return prm


# ---- multi-process layer (gloo on CPU) -----------------------------------

def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_that_may_exit(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=10))
    if rank == 1:
        os._exit(3)  # leaves between steps, before the timing all-reduce
    t0 = time.time()
    try:
        replicas.max_over_ranks(1.0, dist)
        out.put((rank, "completed", time.time() - t0))
    except Exception as e:  # the surviving rank learns of it from the collective
        out.put((rank, type(e).__name__, time.time() - t0))
    os._exit(0)


def test_a_rank_that_exits_is_reported_not_waited_for():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_that_may_exit, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    rank, what, waited = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
    assert rank == 0 and what != "completed", what
    assert waited < 60.0
    assert procs[1].exitcode == 3 and procs[0].exitcode == 0


# ---- host-side input errors (need a device for the solve object) ----------

@pytest.mark.gpu
def test_trajectory_files_that_cannot_be_read(tmp_path):
    with bhr.Solver(small_params()) as s:
        with pytest.raises(bhr.BhrError) as e:
            s.load_trajectory(str(tmp_path / "missing.traj"))
        assert e.value.status == 6  # BHR_IO_ERROR
        bad = tmp_path / "bad.traj"
        bad.write_text("0 10 1.5 0 0 0.1 0 0.9 3.0 0\n0.1 10 1.5 0 0 0.1 0.01 0.9 3.0\n")  # a 9-column row
        with pytest.raises(bhr.BhrError) as e:
            s.load_trajectory(str(bad))
        assert e.value.status == 6
        short = tmp_path / "short.traj"
        short.write_text("0 10 1.5 0 0 0.1 0 0.9 3.0 0\n")
        with pytest.raises(bhr.BhrError):
            s.load_trajectory(str(short))  # one row: the cursor needs two
        s.step(3)  # the solve is still usable
        assert s.info()["steps_done"] == 3


@pytest.mark.gpu
def test_particle_inside_the_horizon_is_rejected():
    from bh_ringdown_b200.trajectory import synthetic_plunge
    prm = small_params(dt=0.05, T=10.0)
    rows = synthetic_plunge(0.5, 0.025, duration=10.0).copy()
    rows[:, 1] = 1.0  # r below r+ = 1.87 on every row
    with bhr.Solver(prm) as s:
        with pytest.raises(bhr.BhrError) as e:
            s.set_trajectory(rows)
        assert e.value.status == 1


@pytest.mark.gpu
def test_source_at_zero_spin_is_rejected():
    """a = 0 exactly: the source's Kerr tortoise formula takes 0 ln(inf)
    (HighOrder/kern.cu:1198-1199; the reference runs with aa = 1e-8), so the
    trajectory is refused instead of depositing NaN; a = 1e-8 runs."""
    from bh_ringdown_b200.trajectory import synthetic_plunge
    rows = synthetic_plunge(1e-8, 0.025, duration=10.0)
    with bhr.Solver(small_params(dt=0.05, T=10.0, a=0.0)) as s:
        with pytest.raises(bhr.BhrError) as e:
            s.set_trajectory(rows)
        assert e.value.status == 1
    with bhr.Solver(small_params(dt=0.05, T=10.0, a=1e-8)) as s:
        s.set_trajectory(rows)
        s.step(5)
        t, h, _ = s.waveform()
        assert np.all(np.isfinite(h))


@pytest.mark.gpu
def test_non_finite_state_is_detected_at_the_extraction():
    """A NaN planted in the state where the extraction column's closure reads
    it: the extraction flags BHR_NAN_DETECTED, which the step call that runs
    that extraction reports (a step's extraction runs beside the next
    step)."""
    prm = small_params()
    with bhr.Solver(prm) as s:
        st = s.get_state()
        st[0][10, prm.N - 4] = np.nan  # an interior point the extraction column's closure reads
        s.set_state(*st)
        with pytest.raises(bhr.BhrError) as e:
            s.step(2)
        assert e.value.status == 4  # BHR_NAN_DETECTED


@pytest.mark.gpu
def test_bounded_wait_gives_up_and_the_device_stays_usable():
    t0 = time.time()
    status = bhr.selftest_bounded_wait(0)
    waited = time.time() - t0
    assert status == 5  # BHR_TIMEOUT, reported by the kernel, not a fault
    assert waited < 30.0
    with bhr.Solver(small_params()) as s:  # the context still works
        s.step(5)
        t, h, _ = s.waveform()
        assert len(t) == 5 and np.all(np.isfinite(h))


@pytest.mark.gpu
@pytest.mark.timeout(300)
def test_failed_trajectory_change_is_reported_at_the_next_step():
    """A sourced solve whose second trajectory fails after the first one's
    record thread was stopped: its next step reports that, instead of
    stepping on the old records or waiting for records no thread publishes;
    a good trajectory makes it usable again."""
    from bh_ringdown_b200.trajectory import synthetic_plunge
    prm = small_params(dt=0.05, T=500.0)  # 10000 steps: past the first 8192 records come from the thread
    rows = synthetic_plunge(0.5, 0.025, duration=60.0)
    with bhr.Solver(prm) as s:
        s.set_trajectory(rows)
        s.step(5)
        bad = rows.copy()
        bad[:, 1] = 1.0  # inside the horizon on every row
        with pytest.raises(bhr.BhrError) as e:
            s.set_trajectory(bad)
        assert e.value.status == 1
        with pytest.raises(bhr.BhrError) as e:
            s.step(3)
        assert e.value.status == 1 and "set one before stepping" in str(e.value)
        s.set_trajectory(rows)
        s.step(3)
        assert s.info()["steps_done"] == 8
