"""Classical RK4 (BHR_RK4), the integrator option for runs specified with
RK4 (the reference itself integrates with SSP-RK3).

CPU: the oracle's RK4 step is held to the textbook RK4 written here in
numpy over the oracle's own right-hand side, and RK4 and SSP-RK3 are held
to the same solution.  GPU: the CUDA RK4 path (stage 1 with dt/2, two
y = u^n + h L(y') stages, the second of which also forms
z = (y1 + 2 y2 - u^n)/3, and u^{n+1} = z + y3/3 + dt/6 L(y3)) against the
oracle's textbook form, at the FP64 bars of the SSP-RK3 path: fields within
1e-12 of scale after tens of steps, waveforms within relative L2 1e-10.
"""
import numpy as np
import pytest

import bh_ringdown_b200 as bhr
from oracle import pyoracle

WAVE_TOL = 1e-10
FIELD_TOL = 1e-12


def rel_field_err(a_planes, b_planes):
    scale = max(np.max(np.abs(b)) for b in b_planes)
    return max(np.max(np.abs(a - b)) for a, b in zip(a_planes, b_planes)) / scale


def oracle_gauss(N, M, Xmin, Xmax, a, m, dt, integrator, center=5.0, ell=2.0, T=100.0, Fr=1, ext_col=-1):
    o = pyoracle.Oracle(N, M, Xmin, Xmax, a, m, dt, T=T, Fr=Fr, out_start=0.0, ext_col=ext_col,
                        integrator=integrator)
    o.init_gaussian(center, 2.0, ell)
    return o


@pytest.mark.parametrize("m", [2.0, -3.0])
def test_oracle_rk4_is_the_textbook_scheme(m):
    """Two oracle RK4 steps against u + dt/6 (k1 + 2 k2 + 2 k3 + k4) built
    from the oracle's right-hand side, with a source plane switched on."""
    N, M, Xmin, Xmax, a = 128, 16, -40.0, 40.0, 0.7
    dt = 0.25 * (Xmax - Xmin) / N
    o = oracle_gauss(N, M, Xmin, Xmax, a, m, dt, 1, ell=max(2.0, abs(m)))
    rng = np.random.default_rng(5)
    tre, tim = rng.standard_normal((M, N)) * 1e-3, rng.standard_normal((M, N)) * 1e-3
    o.set_source(tre, tim)
    inner = np.zeros((M, N), dtype=bool)
    inner[3:M - 3, 3:N - 3] = True
    u = np.stack(o.get_state())
    for _ in range(2):
        k1 = o.eval_rhs(u)
        y = u.copy(); y[:, inner] = (u + 0.5 * dt * k1)[:, inner]
        k2 = o.eval_rhs(y)
        y = u.copy(); y[:, inner] = (u + 0.5 * dt * k2)[:, inner]
        k3 = o.eval_rhs(y)
        y = u.copy(); y[:, inner] = (u + dt * k3)[:, inner]
        k4 = o.eval_rhs(y)
        nxt = u.copy()
        nxt[:, inner] = (u + dt / 6.0 * (k1 + 2.0 * k2 + 2.0 * k3 + k4))[:, inner]
        o.step(1)
        # the closure of the result, through the oracle
        ref = pyoracle.Oracle(N, M, Xmin, Xmax, a, m, dt)
        ref.set_state(list(nxt))
        ref.apply_closure()
        u = np.stack(ref.get_state())
        assert rel_field_err(o.get_state(), list(u)) <= 1e-14


def test_rk4_and_ssprk3_integrate_the_same_equation():
    """Config 1's grid for 40 M at the config's dt = 0.5/22 and at half of
    it: the two integrators' waveforms (column nearest x = 60) differ by
    SSP-RK3's third-order truncation error -- 3.4e-6 relative, then 8x less
    (measured 3.42e-6 and 4.36e-7)."""
    N, M, Xmin, Xmax = 1024, 64, -100.0, 300.0
    x = Xmin + np.arange(N) * (Xmax - Xmin) / N
    col = int(np.argmin(np.abs(x - 60.0)))
    rel = []
    for nsub in (22, 44):
        runs = []
        for integ in (0, 1):
            o = oracle_gauss(N, M, Xmin, Xmax, 0.5, 2.0, 0.5 / nsub, integ, center=20.0, T=40.0, Fr=nsub,
                             ext_col=col)
            t, h, _, _, _, _ = o.run(nsteps=80 * nsub)
            runs.append((t, h))
        (t0, h0), (t1, h1) = runs
        assert np.array_equal(t0, t1) and np.max(np.abs(h0)) > 0.1
        rel.append(np.linalg.norm(h1 - h0) / np.linalg.norm(h0))
    assert rel[0] <= 1e-5
    assert 6.0 <= rel[0] / rel[1] <= 10.0, rel


def test_rk4_option_is_validated_without_a_device():
    with pytest.raises(bhr.BhrError) as e:
        bhr.grid(bhr.Params(N=256, M=32, integrator=bhr.BHR_RK4, precision=bhr.BHR_MIXED))
    assert e.value.status == 1
    with pytest.raises(bhr.BhrError):
        bhr.grid(bhr.Params(N=256, M=32, integrator=7))
    bhr.grid(bhr.Params(N=256, M=32, integrator=bhr.BHR_RK4))


# ---- the CUDA path ---------------------------------------------------------

def gpu_pair(N, M, Xmin, Xmax, a, m, dt, center=5.0, Fr=1, T=100.0, ext_col=-1):
    ell = max(2.0, abs(m))
    prm = bhr.Params(N=N, M=M, Xmin=Xmin, Xmax=Xmax, a=a, m=m, dt=dt, Fr=Fr, T=T, out_start=0.0, ext_col=ext_col,
                     init_kind=bhr.BHR_INIT_GAUSSIAN, init_center=center, init_width=2.0, init_ell=ell,
                     integrator=bhr.BHR_RK4)
    s = bhr.Solver(prm)
    o = oracle_gauss(N, M, Xmin, Xmax, a, m, dt, 1, center=center, ell=ell, T=T, Fr=s.info()["Fr"],
                     ext_col=ext_col)
    return s, o


@pytest.mark.gpu
@pytest.mark.parametrize("tiling", ["block8", "block16", "persistent", "block8n", "ring"])
def test_rk4_every_stage_tiling_matches_oracle(tiling, monkeypatch):
    """1024 x 64 (several tiles per persistent block), a=0.6, m=2."""
    monkeypatch.setenv("BHR_STAGE_TILING", tiling)
    N, M, Xmin, Xmax = 1024, 64, -50.0, 50.0
    s, o = gpu_pair(N, M, Xmin, Xmax, 0.6, 2.0, 0.25 * (Xmax - Xmin) / N, Fr=5, ext_col=700)
    info = s.info()
    assert info["tiling"] == tiling and info["persistent"] == (tiling in ("persistent", "ring"))
    for k in (1, 9, 30):
        s.step(k)
        o.step(k)
        assert rel_field_err(s.get_state(), o.get_state()) <= FIELD_TOL, k
    s2, o2 = gpu_pair(N, M, Xmin, Xmax, 0.6, 2.0, 0.25 * (Xmax - Xmin) / N, Fr=5, ext_col=700)
    s2.step(200)
    t, h, dedt, _, _, _ = o2.run(nsteps=200)
    ts, hs, es = s2.waveform()
    assert np.array_equal(ts, t) and np.max(np.abs(h)) > 1e-6
    assert np.linalg.norm(hs - h) <= WAVE_TOL * np.linalg.norm(h)


@pytest.mark.gpu
@pytest.mark.parametrize("a,m", [(0.3, -3.0), (0.9, 1.0), (0.5, 0.0)])
def test_rk4_odd_negative_and_zero_m(a, m):
    N, M, Xmin, Xmax = 256, 32, -50.0, 50.0
    s, o = gpu_pair(N, M, Xmin, Xmax, a, m, 0.25 * (Xmax - Xmin) / N, center=10.0)
    s.step(40)
    o.step(40)
    assert rel_field_err(s.get_state(), o.get_state()) <= FIELD_TOL


@pytest.mark.gpu
@pytest.mark.parametrize("a,m", [(0.6, 2.0), (0.9, -3.0)])
def test_rk4_plunge_matches_oracle(a, m):
    """Sourced plunge: the step's patch enters all four stages."""
    from bh_ringdown_b200.trajectory import synthetic_plunge
    from tests.test_source import product_coef_fn
    N, M, Xmin, Xmax, T = 256, 32, -50.0, 50.0, 100.0
    dt = 0.25 * (Xmax - Xmin) / N
    prm = bhr.Params(N=N, M=M, Xmin=Xmin, Xmax=Xmax, a=a, m=m, dt=dt, Fr=5, T=T, out_start=0.0, ext_col=154,
                     integrator=bhr.BHR_RK4)
    rows = synthetic_plunge(a, dt / 2.0, duration=T)
    with bhr.Solver(prm) as s:
        s.set_trajectory(rows)
        o = pyoracle.Oracle(N, M, Xmin, Xmax, a, m, dt, T=T, Fr=5, out_start=0.0, ext_col=154, integrator=1)
        s.step(300)
        t, h, _, _, _, _ = o.run(traj=rows, coef_fn=product_coef_fn(), nsteps=300)
        ts, hs, _ = s.waveform()
        assert np.array_equal(ts, t) and np.max(np.abs(h)) > 0
        assert rel_field_err(s.get_state(), o.get_state()) <= FIELD_TOL
        assert np.linalg.norm(hs - h) <= WAVE_TOL * np.linalg.norm(h)


@pytest.mark.gpu
def test_rk4_config1_full_length_waveform():
    """Config 1 as specified, RK4 included: 1024 x 64 on [-100, 300],
    a=0.5, m=2, Courant 0.25 rounded to whole 0.5M outputs, T=300, the
    column nearest x=250."""
    N, M, Xmin, Xmax = 1024, 64, -100.0, 300.0
    x = Xmin + np.arange(N) * (Xmax - Xmin) / N
    col = int(np.argmin(np.abs(x - 250.0)))
    prm = bhr.Params(N=N, M=M, Xmin=Xmin, Xmax=Xmax, a=0.5, m=2.0, dt=0.0, courant=0.25, out_every=0.5, Fr=0,
                     T=300.0, out_start=0.0, ext_col=col, init_kind=bhr.BHR_INIT_GAUSSIAN, init_center=20.0,
                     init_width=2.0, init_ell=2.0, integrator=bhr.BHR_RK4)
    with bhr.Solver(prm) as s:
        info = s.info()
        s.step(info["nt"])
        ts, hs, _ = s.waveform()
    o = oracle_gauss(N, M, Xmin, Xmax, 0.5, 2.0, info["dt"], 1, center=20.0, T=300.0, Fr=info["Fr"], ext_col=col)
    t, h, _, _, _, _ = o.run(nsteps=info["nt"])
    assert np.array_equal(ts, t) and np.max(np.abs(h)) > 1.0
    assert np.linalg.norm(hs - h) <= WAVE_TOL * np.linalg.norm(h)


@pytest.mark.gpu
def test_rk4_is_rejected_where_unsupported():
    with bhr.Engine() as e:
        with pytest.raises(bhr.BhrError) as err:
            e.submit(bhr.Params(N=256, M=32, Xmin=-50.0, Xmax=50.0, a=0.5, dt=0.1, T=5.0,
                                integrator=bhr.BHR_RK4))
        assert err.value.status == 1
