"""The particle source: this project's derivation of the s=-2 point-particle
Teukolsky source (bh_ringdown_b200/csrc/gen_source.py) against the
reference's own deposit (fixtures from HighOrder/kern.cu sourced(), run on
CPU by tests/golden/make_golden.py)."""
import ctypes
import os

import numpy as np
import pytest

import bh_ringdown_b200 as bhr
from oracle import pyoracle

GOLD = os.path.join(os.path.dirname(__file__), "golden")
NAMES = [n for n, _ in pyoracle.OrcParticle._fields_]


def product_coef_fn():
    lib = bhr.load_library()

    def fn(pt, a, mass, m, cr, ci):
        p = bhr.Particle(*[getattr(pt.contents, n) for n in NAMES])
        st = lib.bhr_source_coefficients(ctypes.byref(p), a, mass, m, cr, ci)
        assert st == 0
    return pyoracle.COEF_FN(fn)


@pytest.mark.parametrize("name", ["source_pin_a06_m2", "source_pin_a09_mneg3", "source_pin_a03_m1_inclined",
                                  "source_pin_a095_m4_inclined"])
def test_deposit_matches_reference(name):
    g = np.load(os.path.join(GOLD, name + ".npz"))
    N, M, a, m = int(g["N"]), int(g["M"]), float(g["a"]), float(g["m"])
    o = pyoracle.Oracle(N, M, float(g["Xmin"]), float(g["Xmax"]), a, m, 0.1)
    for k, st in enumerate(g["states"]):
        pt = bhr.Particle(*st)
        C = bhr.source_coefficients(pt, a, 1.0, m)
        o.deposit_source(pyoracle.OrcParticle(*st), C, float(g["timer"]), 0.0)
        tre, tim = o.get_source()
        ref = g["tred"][k] + 1j * g["timd"][k]
        got = tre + 1j * tim
        scale = np.max(np.abs(ref))
        assert scale > 0
        assert np.max(np.abs(got - ref)) <= 1e-12 * scale, (name, k, np.max(np.abs(got - ref)) / scale)


def test_coefficients_reject_bad_particles():
    with pytest.raises(bhr.BhrError):
        bhr.source_coefficients(bhr.Particle(rp=1.2, tp=1.0, E=0.9, lz=3.0), 0.6, 1.0, 2.0)  # inside r+
    with pytest.raises(bhr.BhrError):
        bhr.source_coefficients(bhr.Particle(rp=6.0, tp=0.0, E=0.9, lz=3.0), 0.6, 1.0, 2.0)  # on the pole


def test_coefficients_are_linear_in_the_particle_mass_and_mode_phase():
    """Size-independent properties: phase exp(-i m phip) and the complex
    conjugate symmetry m -> -m of an equatorial circular orbit's static part."""
    st = dict(rp=7.0, tp=np.pi / 2, E=0.93, lz=3.0, dphidt=0.05)
    c0 = bhr.source_coefficients(bhr.Particle(phip=0.0, **st), 0.5, 1.0, 2.0)
    c1 = bhr.source_coefficients(bhr.Particle(phip=0.7, **st), 0.5, 1.0, 2.0)
    assert np.allclose(c1, c0 * np.exp(-2j * 0.7), rtol=1e-13, atol=0)
