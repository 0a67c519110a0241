"""Convergence under grid refinement (a physics check of the discretisation).

Grids nest under doubling (x_l = Xmin + l dx, theta_m = m pi / M), so the
solution on N (or M) points is compared with the one on 2N (2M) at the
coarse points, with dt fixed.  Measured on the oracle, which follows the
reference's scheme (HighOrder/kern.cu:171-299, 320-449):

* radially the error falls at 6th order or faster (the 6th-order stencils,
  and the Kreiss-Oliger term, whose dx^8 / dt scaling takes over on fine
  grids): observed orders 6.0 and 7.7 for N = 256 -> 512 -> 1024 -> 2048;
* in theta the reference's pole closure -- rows 0..2 extrapolated as
  (4 f1 - f2)/3 for even m, set to zero for odd m -- limits the global
  convergence to between first and second order (observed 1.0-1.4 for
  odd m, 1.5-1.9 for even m at t = 1), while mid-latitudes converge at high
  order until the pole error reaches them (orders > 8 there at t = 1;
  2.5-3.5 by t = 4).
The CUDA path is held to the oracle elsewhere; the GPU test repeats the
radial check through it on larger grids.
"""
import numpy as np
import pytest

import bh_ringdown_b200 as bhr
from oracle import pyoracle


def oracle_state(N, M, dt, T, m=2.0, ell=2.0, width=1.0, a=0.5, Xmin=-50.0, Xmax=50.0):
    o = pyoracle.Oracle(N, M, Xmin, Xmax, a, m, dt, T=T, Fr=1, out_start=0.0)
    o.init_gaussian(-5.0, width, ell)
    o.step(int(round(T / dt)))
    return np.stack(o.get_state())


def orders(errs):
    return [float(np.log2(errs[i] / errs[i + 1])) for i in range(len(errs) - 1)]


def test_radial_convergence_is_sixth_order_or_better():
    M, dt, T = 32, 0.01, 4.0
    sols = {N: oracle_state(N, M, dt, T) for N in (256, 512, 1024, 2048)}
    errs = [np.max(np.abs(sols[N] - sols[2 * N][:, :, ::2])[:, 3:M - 3, 8:-8]) for N in (256, 512, 1024)]
    assert errs[0] > 1e-4  # resolved differences, well above rounding
    assert min(orders(errs)) >= 5.5, (errs, orders(errs))


@pytest.mark.parametrize("m,ell,lo,hi", [(2.0, 2.0, 1.2, 2.1), (3.0, 3.0, 0.8, 1.6)])
def test_theta_convergence_is_limited_by_the_pole_closure(m, ell, lo, hi):
    N, dt, T = 512, 0.004, 1.0
    sols = {M: oracle_state(N, M, dt, T, m=m, ell=ell, width=2.0) for M in (16, 32, 64, 128)}
    glob, mid = [], []
    for M in (16, 32, 64):
        d = np.abs(sols[M] - sols[2 * M][:, ::2, :])[:, :, 8:-8]
        glob.append(np.max(d))
        mid.append(np.max(d[:, M // 4:3 * M // 4]))
    assert all(lo <= o <= hi for o in orders(glob)), orders(glob)
    assert min(orders(mid)) >= 6.0, orders(mid)


@pytest.mark.gpu
def test_cuda_path_radial_convergence():
    """The same radial check through the C ABI on 1024..8192 x 64."""
    M, dt, T = 64, 0.0025, 2.0

    def state(N):
        prm = bhr.Params(N=N, M=M, Xmin=-50.0, Xmax=50.0, a=0.5, m=2.0, dt=dt, T=T, Fr=1, out_start=0.0,
                         init_kind=bhr.BHR_INIT_GAUSSIAN, init_center=-5.0, init_width=0.5, init_ell=2.0)
        with bhr.Solver(prm) as s:
            s.step(int(round(T / dt)))
            return np.stack(s.get_state())
    sols = {N: state(N) for N in (1024, 2048, 4096, 8192)}
    errs = [np.max(np.abs(sols[N] - sols[2 * N][:, :, ::2])[:, 3:M - 3, 8:-8]) for N in (1024, 2048, 4096)]
    assert errs[0] > 1e-5
    assert min(orders(errs)) >= 5.5, (errs, orders(errs))
