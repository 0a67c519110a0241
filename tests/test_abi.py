"""The C ABI library loads on a machine without a GPU, exports every entry
point include/bhr.h declares, and its host-side pieces match the oracle."""
import os
import re

import numpy as np
import pytest

import bh_ringdown_b200 as bhr
from oracle import pyoracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for hdr in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if hdr.endswith(".h"):
            text = open(os.path.join(ROOT, "include", hdr)).read()
            names += re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*(bhr_[a-z_0-9]+)\s*\(", text, re.M)
    return sorted(set(names))


def test_library_loads_and_exports_every_declared_symbol():
    lib = bhr.load_library()
    names = declared_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    assert lib.bhr_abi_version() == 3


def test_params_default_are_the_reference_values():
    lib = bhr.load_library()
    p = bhr._Params()
    assert lib.bhr_params_default(p) == 0
    assert (p.N, p.M, p.Xmin, p.Xmax, p.a, p.dt, p.T, p.Fr, p.PTSX, p.PTSY) == \
        (16000, 256, -50.0, 50.0, 1e-8, 0.002, 1500.0, 50, 128, 128)
    assert p.out_start == 250.0


@pytest.mark.parametrize("N,M,Xmin,Xmax,a", [(256, 32, -50.0, 50.0, 0.6), (1024, 64, -100.0, 300.0, 0.5),
                                             (8192, 128, -200.0, 600.0, 0.9), (512, 16, -50.0, 50.0, 0.0)])
def test_grid_matches_oracle_bit_for_bit(N, M, Xmin, Xmax, a):
    x, r, t = bhr.grid(bhr.Params(N=N, M=M, Xmin=Xmin, Xmax=Xmax, a=a))
    o = pyoracle.Oracle(N, M, Xmin, Xmax, a, 2.0, 0.01)
    xo, ro, to = o.grid()
    assert np.array_equal(x, xo) and np.array_equal(r, ro) and np.array_equal(t, to)
    assert np.all(np.isfinite(r))


def test_swsh_matches_oracle():
    for ell in range(0, 9):
        for m in range(-4, 5):
            for th in np.linspace(0, np.pi, 9):
                assert bhr.swsh(ell, m, th) == pyoracle.swsh(ell, m, th)


def test_invalid_parameters_are_rejected_without_a_device():
    with pytest.raises(bhr.BhrError) as e:
        bhr.grid(bhr.Params(N=100, M=32))
    assert e.value.status == 1
    with pytest.raises(bhr.BhrError):
        bhr.grid(bhr.Params(N=256, M=20))
    with pytest.raises(bhr.BhrError):
        bhr.grid(bhr.Params(N=256, M=32, a=1.5))
