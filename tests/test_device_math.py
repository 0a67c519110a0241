"""The hand-written FP64 reciprocal and square root of the stage kernels
(bhr_device.cuh: Newton-Raphson from the hardware's rcp.approx / rsqrt.approx,
a named method) against CUDA's own correctly rounded 1.0 / x and sqrt(x),
both evaluated on the device, over a sweep of magnitudes.  Stated bound:
at most 1 ulp apart everywhere on the sweep."""
import numpy as np
import pytest

import bh_ringdown_b200 as bhr

pytestmark = pytest.mark.gpu

MAX_ULP = 1


def ulp_distance(a, b):
    """Distance in units in the last place between doubles of equal sign."""
    ia = a.view(np.int64).astype(object)
    ib = b.view(np.int64).astype(object)
    return np.array([abs(x - y) for x, y in zip(ia, ib)], dtype=np.int64)


def sweep():
    rng = np.random.default_rng(20261203)
    exps = np.arange(-300, 301, 3)
    mant = rng.uniform(1.0, 10.0, size=(len(exps), 40))
    x = (mant * 10.0 ** exps[:, None]).reshape(-1)
    # the ranges the kernels meet: bir = B0 + B1 sin^2 (order 1e-3 .. 1e4),
    # the discriminant of bb, and values next to powers of two
    special = np.concatenate([rng.uniform(1e-3, 1e4, 4000), np.ldexp(1.0, np.arange(-900, 900, 7)),
                              np.nextafter(np.ldexp(1.0, np.arange(-900, 900, 7)), 0.0), [1.0, 2.0, 3.0, 0.1]])
    return np.concatenate([x, special])


def test_reciprocal_within_one_ulp_of_cuda_division():
    x = sweep()
    x = np.concatenate([x, -x[::5]])
    rcp, ref, _, _ = bhr.selftest_math(x)
    assert np.all(np.isfinite(rcp))
    d = ulp_distance(rcp, ref)
    assert d.max() <= MAX_ULP, (d.max(), x[np.argmax(d)])


def test_square_root_within_one_ulp_of_cuda_sqrt():
    x = sweep()
    _, _, sq, ref = bhr.selftest_math(x)
    d = ulp_distance(sq, ref)
    assert d.max() <= MAX_ULP, (d.max(), x[np.argmax(d)])
    _, _, z, _ = bhr.selftest_math(np.array([0.0]))
    assert z[0] == 0.0
