"""Batch engine (bhr_engine_*): many solves advanced by one launch per RK
stage (per group of up to 112 solves) over a (solve, tile) work-list.

A request's waveform must not depend on what it shares the GPU with: the
same request run alone in an engine and in a mixed batch (other grids,
spins, m, sourced and source-free, different lengths, joining mid-run)
gives bit-identical rows.  Against a lone bhr_solver the rows agree to the
FP64 bar (relative L2 1e-12; times bit-identical), and one engine request is
checked against the CPU oracle directly.
"""
import numpy as np
import pytest

import bh_ringdown_b200 as bhr
from bh_ringdown_b200.trajectory import synthetic_plunge
from oracle import pyoracle

pytestmark = pytest.mark.gpu

WAVE_TOL = 1e-12


def gauss(N, M, Xmin, Xmax, a, m, T, center=5.0):
    # extraction at x = Xmin + 0.65 (Xmax - Xmin), inside the region the
    # pulse crosses within T
    return bhr.Params(N=N, M=M, Xmin=Xmin, Xmax=Xmax, a=a, m=m, dt=0.25 * (Xmax - Xmin) / N, Fr=5, T=T,
                      out_start=0.0, ext_col=N * 65 // 100, init_kind=bhr.BHR_INIT_GAUSSIAN,
                      init_center=center, init_width=2.0, init_ell=max(2.0, abs(m)))


def plunge(N, M, Xmin, Xmax, a, m, T):
    dt = 0.25 * (Xmax - Xmin) / N
    prm = bhr.Params(N=N, M=M, Xmin=Xmin, Xmax=Xmax, a=a, m=m, dt=dt, Fr=5, T=T, out_start=0.0,
                     ext_col=N * 6 // 10)
    return prm, synthetic_plunge(a, dt / 2.0, duration=T)


def requests():
    p1, tr1 = plunge(256, 32, -50.0, 50.0, 0.6, 2.0, 30.0)
    return [
        (gauss(256, 32, -50.0, 50.0, 0.5, 2.0, 20.0), None),
        (gauss(512, 64, -50.0, 50.0, 0.9, -3.0, 25.0, center=3.0), None),
        (p1, tr1),
        (gauss(128, 16, -40.0, 40.0, 0.0, 1.0, 12.0), None),
    ]


def run_alone(prm, traj):
    with bhr.Engine() as e:
        rid = e.submit(prm, traj)
        e.run_all()
        info = e.poll(rid)
        assert info["state"] == bhr.Engine.DONE, info
        return e.result(rid)


def test_mixed_batch_is_bit_identical_to_alone():
    reqs = requests()
    alone = [run_alone(p, t) for p, t in reqs]
    with bhr.Engine() as e:
        ids = [e.submit(p, t) for p, t in reqs]
        chunks = 0
        while True:
            running = e.step(7)  # small chunks: membership changes as solves finish
            chunks += 1
            if running == 0 and e.stats()["queued"] == 0:
                break
        assert chunks > 4
        for rid, (t0, h0, d0) in zip(ids, alone):
            t, h, d = e.result(rid)
            assert len(t) > 0 and np.max(np.abs(h0)) > 1e-8
            assert np.array_equal(t, t0) and np.array_equal(h, h0) and np.array_equal(d, d0)
        st = e.stats()
        assert st["finished"] == len(reqs) and st["running"] == 0 and st["bytes_in_use"] == 0


def test_request_joining_mid_run_is_bit_identical():
    reqs = requests()
    alone = run_alone(*reqs[2])
    with bhr.Engine() as e:
        first = e.submit(*reqs[1])
        e.step(40)
        assert e.poll(first)["state"] == bhr.Engine.RUNNING
        late = e.submit(*reqs[2])
        assert e.poll(late)["state"] in (bhr.Engine.QUEUED, bhr.Engine.RUNNING)
        while e.poll(late)["state"] != bhr.Engine.RUNNING:  # prepared off the stepping thread
            e.step(0)
        e.step(10)
        info = e.poll(late)
        assert info["state"] == bhr.Engine.RUNNING and info["steps_done"] == 10
        e.run_all()
        t, h, d = e.result(late)
        assert np.array_equal(t, alone[0]) and np.array_equal(h, alone[1]) and np.array_equal(d, alone[2])
        info = e.poll(late)
        assert info["submit_s"] <= info["start_s"] <= info["finish_s"]


def test_membership_growing_one_by_one():
    """Requests joining one per call (the device tables regrow as the batch
    grows) and leaving at different steps."""
    reqs = [(gauss(128, 16, -40.0, 40.0, 0.1 * i, 1.0 + i % 3, 6.0 + i), None) for i in range(7)]
    alone = [run_alone(p, t) for p, t in reqs]
    with bhr.Engine() as e:
        ids = []
        for p, t in reqs:
            ids.append(e.submit(p, t))
            e.step(3)
        e.run_all()
        for rid, (t0, h0, d0) in zip(ids, alone):
            t, h, d = e.result(rid)
            assert np.array_equal(t, t0) and np.array_equal(h, h0) and np.array_equal(d, d0)


@pytest.mark.parametrize("tiling", ["block8n", "ring"])
def test_more_solves_than_one_launch_group(tiling, monkeypatch):
    """232 running solves: a stage launch takes at most 112 solves' arguments
    in its parameters, so every stage runs as several launch groups (stage 1:
    three; FP64 stages 2 and 3: two; the FP32 stages of the mixed requests:
    two).  Four kinds of request (grids, spins, m, FP64 and mixed precision)
    alternate, and every 29th request is a sourced plunge (its source patch
    and step records are arguments too), so a block that took a neighbouring
    solve's arguments would change a result: each must be bit-identical to
    its kind run alone."""
    monkeypatch.setenv("BHR_ENGINE_TILING", tiling)
    kinds = [(gauss(128, 16, -40.0, 40.0, 0.0, 1.0, 6.0), None),
             (gauss(192, 32, -40.0, 40.0, 0.5, 2.0, 6.0, center=4.0), None),
             (gauss(128, 16, -40.0, 40.0, 0.3, -2.0, 6.0), None),
             (gauss(192, 32, -40.0, 40.0, 0.8, 3.0, 6.0, center=4.0), None),
             plunge(256, 32, -50.0, 50.0, 0.6, 2.0, 8.0)]
    kinds[2][0].precision = bhr.BHR_MIXED
    kinds[3][0].precision = bhr.BHR_MIXED
    alone = [run_alone(p, t) for p, t in kinds]
    for (_, h0, _), (_, h1, _) in zip(alone, alone[1:]):
        assert not np.array_equal(h0, h1)
    n = 232
    kind = [4 if i % 29 == 7 else i % 4 for i in range(n)]
    # stage-1 tiles (8 rows) of every solve plus the mixed solves' 16-row FP32 tiles
    tiles = {0: 2 * 2, 1: 3 * 4, 2: 2 * 2 + 2 * 1, 3: 3 * 4 + 3 * 2, 4: 4 * 4}
    with bhr.Engine() as e:
        ids = [e.submit(*kinds[k]) for k in kind]
        while e.stats()["queued"] > 0:  # every request prepared, so all join the first batch step
            e.step(0)
        e.step(1)
        st = e.stats()
        assert st["running"] == n and st["tiles"] == sum(tiles[k] for k in kind)
        e.run_all()
        for i, rid in enumerate(ids):
            t, h, d = e.result(rid)
            t0, h0, d0 = alone[kind[i]]
            assert np.array_equal(t, t0) and np.array_equal(h, h0) and np.array_equal(d, d0), i


def test_mixed_precision_requests_in_a_mixed_batch():
    """FP32-corrected (BHR_MIXED) and FP64 requests side by side: each
    result bit-identical to the same request alone in an engine, and the
    mixed ones within the FP64 bar of a lone mixed-precision solver."""
    reqs = requests()
    for k in (1, 2):
        reqs[k][0].precision = bhr.BHR_MIXED
    alone = [run_alone(p, t) for p, t in reqs]
    with bhr.Engine() as e:
        ids = [e.submit(p, t) for p, t in reqs]
        e.run_all()
        for rid, (t0, h0, d0) in zip(ids, alone):
            t, h, d = e.result(rid)
            assert np.array_equal(t, t0) and np.array_equal(h, h0) and np.array_equal(d, d0)
    for k in (1, 2):
        prm, traj = reqs[k]
        with bhr.Solver(prm) as s:
            if traj is not None:
                s.set_trajectory(traj)
            s.run()
            ts, hs, _ = s.waveform()
        t, h, _ = alone[k]
        assert np.array_equal(t, ts)
        assert np.linalg.norm(h - hs) <= WAVE_TOL * np.linalg.norm(hs)


@pytest.mark.parametrize("tiling", ["block8", "block16", "persistent", "block8n", "ring"])
def test_every_engine_tiling(tiling, monkeypatch):
    """Each FP64 stage tiling over the work-list, with FP64 and mixed-precision
    requests in one batch (mixed solves run their FP64 stage 1 on the
    tiling's tiles and the FP32 stages on 16-row tiles): every result within
    the FP64 bar of a lone solver on the same request."""
    monkeypatch.setenv("BHR_ENGINE_TILING", tiling)
    reqs = requests()
    reqs[1][0].precision = bhr.BHR_MIXED
    with bhr.Engine() as e:
        ids = [e.submit(p, t) for p, t in reqs]
        e.run_all()
        got = [e.result(i) for i in ids]
    for (prm, traj), (t, h, _) in zip(reqs, got):
        with bhr.Solver(prm) as s:
            if traj is not None:
                s.set_trajectory(traj)
            s.run()
            ts, hs, _ = s.waveform()
        assert np.array_equal(t, ts) and np.max(np.abs(hs)) > 1e-8
        assert np.linalg.norm(h - hs) <= WAVE_TOL * np.linalg.norm(hs)


def test_engine_matches_lone_solver():
    for prm, traj in requests():
        s = bhr.Solver(prm)
        if traj is not None:
            s.set_trajectory(traj)
        s.run()
        ts, hs, ds = s.waveform()
        s.close()
        t, h, d = run_alone(prm, traj)
        assert np.array_equal(t, ts)
        assert np.linalg.norm(h - hs) <= WAVE_TOL * np.linalg.norm(hs)


def test_engine_request_matches_oracle():
    prm = gauss(256, 32, -50.0, 50.0, 0.7, 2.0, 15.0)
    t, h, d = run_alone(prm, None)
    o = pyoracle.Oracle(prm.N, prm.M, prm.Xmin, prm.Xmax, prm.a, prm.m, prm.dt, T=prm.T, Fr=prm.Fr, out_start=0.0,
                        ext_col=prm.ext_col)
    o.init_gaussian(prm.init_center, prm.init_width, prm.init_ell)
    with bhr.Solver(prm) as s:
        nt = s.info()["nt"]
    to, ho, do, steps, _, _ = o.run(nsteps=nt)
    assert np.array_equal(t, to)
    assert np.max(np.abs(ho)) > 1e-6  # the pulse has reached the extraction column
    assert np.linalg.norm(h - ho) <= 1e-10 * np.linalg.norm(ho)


def test_genot_worldline_request_matches_the_oracle():
    """A served plunge request with a GenOT transition-to-plunge worldline
    (inclined, so theta moves), in a batch with a source-free request, is
    bit-identical to the same request alone and matches the oracle."""
    from bh_ringdown_b200 import genot
    from tests.test_source import product_coef_fn
    N, M, Xmin, Xmax, a = 256, 32, -50.0, 50.0, 0.3
    dt = 0.25 * (Xmax - Xmin) / N
    prm = bhr.Params(N=N, M=M, Xmin=Xmin, Xmax=Xmax, a=a, m=2.0, dt=dt, Fr=5, T=25.0, out_start=0.0,
                     ext_col=N * 6 // 10)
    rows = genot.transition_plunge(a, 1e-3, dt / 2.0, 30.0, inclination_deg=30.0, chi0_deg=40.0)
    assert np.ptp(rows[:, 2]) > 0.05
    alone = run_alone(prm, rows)
    with bhr.Engine() as e:
        rid = e.submit(prm, rows)
        other = e.submit(gauss(512, 64, -50.0, 50.0, 0.9, -3.0, 25.0, center=3.0))
        e.run_all()
        t, h, d = e.result(rid)
        assert e.poll(other)["state"] == bhr.Engine.DONE
    assert np.array_equal(t, alone[0]) and np.array_equal(h, alone[1])
    o = pyoracle.Oracle(N, M, Xmin, Xmax, a, 2.0, dt, T=prm.T, Fr=prm.Fr, out_start=0.0, ext_col=prm.ext_col)
    with bhr.Solver(prm) as s:
        nt = s.info()["nt"]
    to, ho, _, _, _, _ = o.run(traj=rows, coef_fn=product_coef_fn(), nsteps=nt)
    assert np.array_equal(t, to) and np.max(np.abs(ho)) > 0
    assert np.linalg.norm(h - ho) <= 1e-10 * np.linalg.norm(ho)


def test_budget_admits_one_at_a_time_when_tight():
    reqs = requests()[:2]
    alone = [run_alone(p, t) for p, t in reqs]
    with bhr.Engine(hbm_budget_bytes=1) as e:
        ids = [e.submit(p, t) for p, t in reqs]
        e.step(1)
        st = e.stats()
        assert st["running"] == 1 and st["queued"] == 1
        e.run_all()
        for rid, (t0, h0, d0) in zip(ids, alone):
            t, h, d = e.result(rid)
            assert np.array_equal(h, h0)


def test_requests_that_fit_go_ahead_of_one_that_does_not():
    """Budget for one large solve and some small ones: with a large one
    running, a second large request waits while the small requests behind
    it are admitted (no head-of-line blocking), and all finish as alone."""
    big = [gauss(2048, 256, -50.0, 50.0, 0.5, 2.0, 15.0, center=4.0 + k) for k in range(2)]
    small = [gauss(256, 32, -50.0, 50.0, 0.7, 2.0, 5.0, center=5.0 + k) for k in range(2)]
    with bhr.Engine(hbm_budget_bytes=80 << 20) as e:
        ids = [e.submit(p) for p in big + small]
        e.run_all(chunk=8)
        info = [e.poll(i) for i in ids]
        assert all(x["state"] == bhr.Engine.DONE for x in info), info
        # the second large solve starts after the first finished; the small ones before that
        assert info[1]["start_s"] >= info[0]["finish_s"]
        assert info[2]["start_s"] < info[0]["finish_s"] and info[3]["start_s"] < info[0]["finish_s"]
        res = [e.result(i) for i in ids]
    for p, (t, h, d) in zip(big + small, res):
        t0, h0, d0 = run_alone(p, None)
        assert np.array_equal(t, t0) and np.array_equal(h, h0)


def test_invalid_request_fails_alone():
    good = requests()[0]
    bad = gauss(200, 32, -50.0, 50.0, 0.5, 2.0, 10.0)  # N not a multiple of 64
    with bhr.Engine() as e:
        rb = e.submit(bad)
        rg = e.submit(*good)
        e.run_all()
        assert e.poll(rb)["state"] == bhr.Engine.FAILED
        assert e.poll(rb)["status"] == 1  # BHR_INVALID_ARG
        with pytest.raises(bhr.BhrError):
            e.result(rb)
        assert e.poll(rg)["state"] == bhr.Engine.DONE
