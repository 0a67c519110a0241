"""bhr_step_noalloc: SSP-RK3 steps for callers that cannot call cudaMalloc.

Those callers (a framework that owns the device memory and hands out
pieces of it; a latency-critical loop that may not take cudaMalloc's
device synchronisation) pass a state they already hold in device memory;
the intermediate stages live in the library's fixed device array.  This
file runs last (pytest collects it after the others) and checks the entry
point through the C ABI against the normal solver path, bhr_solver_step,
on two calls in a row, at the field tolerance of the other parity tests.
"""
import numpy as np
import pytest

import bh_ringdown_b200 as bhr

pytestmark = pytest.mark.gpu

FIELD_TOL = 1e-12


def params(m, a):
    N, M, Xmin, Xmax = 512, 64, -50.0, 50.0
    return bhr.Params(N=N, M=M, Xmin=Xmin, Xmax=Xmax, a=a, m=m, dt=0.25 * (Xmax - Xmin) / N, T=100.0,
                      out_start=0.0, init_kind=bhr.BHR_INIT_GAUSSIAN, init_center=8.0, init_width=2.0,
                      init_ell=max(2.0, abs(m)))


@pytest.mark.parametrize("m,a", [(2.0, 0.7), (-3.0, 0.4)])
def test_noalloc_steps_match_the_solver_on_two_calls(m, a):
    import torch
    prm = params(m, a)
    ref = bhr.Solver(prm)
    start = np.stack(ref.get_state())                  # closed initial state, 4 x M x N
    state = torch.from_numpy(start.copy()).to("cuda")  # device memory the caller owns
    torch.cuda.synchronize()
    for nsteps in (7, 13):
        bhr.step_noalloc(prm, state.data_ptr(), nsteps)
        ref.step(nsteps)
        got = state.cpu().numpy()
        want = np.stack(ref.get_state())
        scale = np.max(np.abs(want))
        assert np.max(np.abs(got - want)) <= FIELD_TOL * scale
    ref.close()


def test_noalloc_calls_with_different_spin_and_m_back_to_back():
    """The scratch's coefficient tables follow the parameters of each call:
    alternating (a, m) on one grid, each call checked against its own solver."""
    import torch
    cases = [params(2.0, 0.7), params(-3.0, 0.4), params(2.0, 0.7)]
    refs = [bhr.Solver(prm) for prm in cases[:2]]
    states = [torch.from_numpy(np.stack(r.get_state()).copy()).to("cuda") for r in refs]
    torch.cuda.synchronize()
    for i, prm in enumerate(cases):
        j = i % 2
        bhr.step_noalloc(prm, states[j].data_ptr(), 5)
        refs[j].step(5)
        want = np.stack(refs[j].get_state())
        got = states[j].cpu().numpy()
        assert np.max(np.abs(got - want)) <= FIELD_TOL * np.max(np.abs(want)), i
    for r in refs:
        r.close()


def test_noalloc_rejects_grids_beyond_its_scratch():
    import torch
    prm = bhr.Params(N=1024, M=256, Xmin=-50.0, Xmax=50.0, a=0.5, m=2.0, dt=0.01)
    state = torch.zeros(16, dtype=torch.float64, device="cuda")
    with pytest.raises(bhr.BhrError) as e:
        bhr.step_noalloc(prm, state.data_ptr(), 1)
    assert e.value.status == 1 and "scratch" in str(e.value)
