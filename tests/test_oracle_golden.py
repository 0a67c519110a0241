"""The C oracle against fixtures produced by the reference's own HighOrder
code (tests/golden/make_golden.py runs the reference kernels on CPU)."""
import os

import numpy as np
import pytest

from oracle import pyoracle

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def load(name):
    return np.load(os.path.join(GOLD, name))


@pytest.mark.parametrize("case", ["evolve_pin_m2", "evolve_pin_m3", "evolve_pin_mneg1"])
def test_grid_coefficients_and_evolution_match_reference(case):
    g = load(case + ".npz")
    N, M = int(g["N"]), int(g["M"])
    o = pyoracle.Oracle(N, M, float(g["Xmin"]), float(g["Xmax"]), float(g["a"]), float(g["m"]), float(g["dt"]))
    x, r, t = o.grid()
    # grid(): same arithmetic, bit for bit (HighOrder/main.c:64-183)
    assert np.array_equal(x, g["x_c"]) and np.array_equal(r, g["r_c"]) and np.array_equal(t, g["theta"])
    if "coeffs_every4" in g:
        for k in range(9):
            c = o.coeff(k)[:, ::4]
            ref = g["coeffs_every4"][k]
            assert np.max(np.abs(c - ref)) <= 1e-14 * np.max(np.abs(ref)), k
    # initial data: oracle's pulse + closure equals the reference-closed pulse
    o.init_gaussian(float(g["center"]), float(g["width"]), float(g["ell"]))
    st0 = o.get_state()
    assert np.max(np.abs(st0[0] - g["init_qre"])) <= 1e-15 * np.max(np.abs(g["init_qre"]))
    o.set_state([g["init_qre"], np.zeros((M, N)), np.zeros((M, N)), np.zeros((M, N))])
    ext = np.zeros_like(g["ext"])
    for k in range(int(g["nsteps"])):
        o.step()
        ext[k] = np.array(o.ext())
    st = o.get_state()
    for f in range(4):
        ref = g["final"][f]
        scale = max(np.max(np.abs(ref)), 1e-300)
        assert np.max(np.abs(st[f] - ref)) <= 1e-12 * scale, (case, f, np.max(np.abs(st[f] - ref)) / scale)
    # psi at column N-1 every step (d_qre_buff/d_qim_buff), compared on the
    # scale of the field: far from the pulse the column holds rounding noise.
    scale = np.max(np.abs(g["final"][:2]))
    assert np.max(np.abs(ext - g["ext"])) <= 1e-12 * scale


def test_swsh_and_projection_match_reference():
    g = load("proj_pin.npz")
    for ell, m, th, v in zip(g["ell"], g["m"], g["theta"], g["swsh"]):
        assert pyoracle.swsh(ell, m, th) == pytest.approx(v, rel=1e-13, abs=1e-300)
    L = pyoracle.lib()
    M = int(g["M"])
    for i in range(4):
        for l in range(7):
            buf = np.ascontiguousarray(g["qq"][i].copy())
            val = L.orc_project(buf.ctypes.data_as(pyoracle.C.POINTER(pyoracle.D)), M, float(2 + l), 2.0)
            assert val == pytest.approx(g["proj"][i, l], rel=1e-13, abs=1e-14)


def test_reference_grid_is_nan_on_config1_domain_and_oracle_floors_it():
    """On [-100, 300] the reference grid() loses r - r+ below FP64
    resolution and returns NaN radii; the oracle (and the product) put
    those points on the next double above r+ and agree elsewhere."""
    g = load("grid_c1s_a05.npz")
    N, M = int(g["N"]), int(g["M"])
    ref_r = g["r_c"]
    rp = 1.0 + np.sqrt(1.0 - 0.25)
    bad = ~np.isfinite(ref_r)
    assert bad.any() and bad[:5].all()
    bad |= ~(ref_r > rp)  # the last finite reference point sits exactly on r+
    o = pyoracle.Oracle(N, M, float(g["Xmin"]), float(g["Xmax"]), float(g["a"]), 2.0, 0.01)
    _, r, _ = o.grid()
    assert np.all(np.isfinite(r))
    assert np.array_equal(r[~bad], ref_r[~bad])
    assert np.all(r[bad] == np.nextafter(rp, np.inf))
