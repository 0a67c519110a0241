"""Generate tests/golden/*.npz from the reference's own HighOrder code.

Runs the reference kernels, grid() and proj.c on CPU cores through
oracle/_ref/libref_<tag>.so (built by oracle/build_ref.py from the sources
under the reference tree) and stores small input/output fixtures.  The CPU
tests check the C oracle against these; the oracle in turn checks the CUDA
path on the GPU.  Needs the reference tree, so it runs only where the
reference is mounted:

    python oracle/build_ref.py pin c1s && python tests/golden/make_golden.py
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import pyoracle  # noqa: E402

D = C.c_double
from oracle.build_ref import default_reference_root  # noqa: E402

REF = default_reference_root()


def ref_lib(tag):
    L = C.CDLL(os.path.join(ROOT, "oracle", "_ref", f"libref_{tag}.so"))
    for f in ("ref_Xmin", "ref_Xmax", "ref_project", "ref_swsh"):
        getattr(L, f).restype = D
    L.ref_project.argtypes = [C.c_void_p, D, D]
    L.ref_swsh.argtypes = [D, D, D]
    L.ref_source.argtypes = [D] * 16
    for f in ("ref_grid", "ref_init"):
        getattr(L, f).restype = None
    return L


def p(a):
    return a.ctypes.data_as(C.c_void_p)


def grid_and_init(L, mass, a, m, dt):
    N, M = L.ref_N(), L.ref_M()
    x, r, t = np.zeros(N), np.zeros(N), np.zeros(M)
    L.ref_grid(D(mass), D(a), p(x), p(r), p(t))
    L.ref_init(D(mass), D(a), D(m), D(dt), p(t), p(r))
    return x, r, t


def evolution_case(L, a, m, center, width, ell, nsteps, dt_fac=0.25, with_coeffs=False):
    """Gaussian pulse closed by the reference's own boundary kernels, then
    nsteps reference steps.  Returns inputs and outputs."""
    N, M = L.ref_N(), L.ref_M()
    Xmin, Xmax = L.ref_Xmin(), L.ref_Xmax()
    dx = (Xmax - Xmin) / N
    dt = dt_fac * dx
    x, r, t = grid_and_init(L, 1.0, a, m, dt)
    psi = np.exp(-((x[None, :] - center) ** 2) / (2 * width * width)) * \
        np.array([pyoracle.swsh(ell, m, th) for th in t])[:, None]
    zero = np.zeros((M, N))
    planes = [np.ascontiguousarray(v.reshape(-1)) for v in (psi, zero, zero, zero)]
    L.ref_set_state(*[p(v) for v in planes])
    L.ref_apply_closure()
    st0 = [np.zeros(N * M) for _ in range(4)]
    L.ref_get_state(*[p(v) for v in st0])
    ext = np.zeros((nsteps, 2, M))
    er, ei = np.zeros(M), np.zeros(M)
    for k in range(nsteps):
        L.ref_step(p(er), p(ei))
        ext[k, 0], ext[k, 1] = er, ei
    st = [np.zeros(N * M) for _ in range(4)]
    L.ref_get_state(*[p(v) for v in st])
    coeffs = []
    for k in range(9):
        c = np.zeros(N * M)
        L.ref_get_coeff(k, p(c))
        coeffs.append(c.reshape(M, N))
    out = dict(N=N, M=M, Xmin=Xmin, Xmax=Xmax, a=a, m=m, dt=dt, nsteps=nsteps, center=center, width=width,
               ell=ell, x_c=x, r_c=r, theta=t, init_qre=st0[0].reshape(M, N),
               final=np.stack([v.reshape(M, N) for v in st]), ext=ext)
    if with_coeffs:  # every 4th column keeps the fixture small
        out["coeffs_every4"] = np.stack(coeffs)[:, :, ::4]
    return out


# Particle states for the source fixtures: (rp, tp, phip, E, lz, Q, drdt,
# d2rdt2, d3rdt3, dthdt, d2thdt2, d3thdt3, dphidt, d2phidt2).
def particle_states(a):
    out = []
    # circular equatorial prograde orbits (Bardeen-Press-Teukolsky E, Lz)
    for r0 in (6.0, 8.0, 11.0):
        v = 1.0 / np.sqrt(r0)
        den = np.sqrt(1 - 3 * v * v + 2 * a * v ** 3)
        E = (1 - 2 * v * v + a * v ** 3) / den
        Lz = np.sqrt(r0) * (1 - 2 * a * v ** 3 + a * a * v ** 4) / den
        Om = 1.0 / (r0 ** 1.5 + a)
        out.append((r0, np.pi / 2, 0.3 * r0, E, Lz, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, Om, 0.0))
    # plunging / inclined states with non-zero velocities and accelerations
    out.append((7.3, 1.35, 2.1, 0.93, 2.9, 1.5, -0.021, -0.0013, 0.0, 0.004, -0.0002, 0.0, 0.051, 0.0007))
    out.append((5.1, 1.7, 5.9, 0.91, 2.4, 0.7, -0.08, -0.006, 0.0, -0.011, 0.0009, 0.0, 0.09, 0.002))
    return out


# Inclined states (theta-dot and its derivative non-zero, theta off the
# equator on both hemispheres, retrograde phi-dot) for the later fixtures.
def inclined_states():
    return [
        (6.5, 1.1, 0.4, 0.95, 2.2, 4.1, -0.01, -0.0005, 0.0, 0.03, -0.001, 0.0, 0.06, 0.0004),
        (9.0, 2.0, 1.0, 0.96, -1.5, 6.0, 0.0, 0.0, 0.0, -0.02, 0.0005, 0.0, -0.03, 0.0),
        (4.2, 0.8, 3.3, 0.9, 1.1, 8.5, -0.15, -0.02, 0.0, 0.05, 0.004, 0.0, 0.12, 0.003),
        (12.0, 2.5, 5.5, 0.97, 0.9, 9.0, 0.02, 0.0001, 0.0, -0.008, -0.0002, 0.0, 0.01, -0.0001),
    ]


def source_case(L, a, m, timer, states=None):
    N, M = L.ref_N(), L.ref_M()
    Xmin, Xmax = L.ref_Xmin(), L.ref_Xmax()
    dx = (Xmax - Xmin) / N
    x, r, t = grid_and_init(L, 1.0, a, m, 0.25 * dx)
    states = np.array(particle_states(a))[:4] if states is None else np.array(states)
    tre_all, tim_all = [], []
    for s in states:
        rp, tp, phip, E, lz, Q, drdt, d2r, d3r, dth, d2th, d3th, dph, d2ph = s
        L.ref_source(D(0.0), D(timer), D(rp), D(phip), D(tp), D(E), D(lz), D(Q), D(drdt), D(d2r), D(d3r), D(dth),
                     D(d2th), D(d3th), D(dph), D(d2ph))
        tre, tim = np.zeros(N * M), np.zeros(N * M)
        L.ref_get_source(p(tre), p(tim))
        tre_all.append(tre.reshape(M, N))
        tim_all.append(tim.reshape(M, N))
    return dict(N=N, M=M, Xmin=Xmin, Xmax=Xmax, a=a, m=m, timer=timer, states=states, tred=np.stack(tre_all),
                timd=np.stack(tim_all))


def swsh_case(L, M):
    ells, ms, ths, vals = [], [], [], []
    for ell in range(0, 9):
        for m in range(-4, 5):
            for th in np.linspace(0.0, np.pi, 7):
                ells.append(ell)
                ms.append(m)
                ths.append(th)
                vals.append(L.ref_swsh(ell, m, th))
    rng = np.random.default_rng(20261203)
    qq = rng.standard_normal((4, M + 1))
    proj = np.zeros((4, 7))
    for i in range(4):
        for l in range(7):
            buf = qq[i].copy()
            proj[i, l] = L.ref_project(p(buf), float(2 + l), 2.0)
    return dict(ell=np.array(ells, float), m=np.array(ms, float), theta=np.array(ths), swsh=np.array(vals), qq=qq,
                proj=proj, M=M)


def main():
    L = ref_lib("pin")
    cases = {
        "evolve_pin_m2": evolution_case(L, 0.6, 2.0, 5.0, 2.0, 2.0, 30, with_coeffs=True),
        "evolve_pin_m3": evolution_case(L, 0.3, 3.0, 40.0, 1.5, 3.0, 30),
        "evolve_pin_mneg1": evolution_case(L, 0.9, -1.0, 0.0, 2.5, 2.0, 30),
    }
    for name, d in cases.items():
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **d)
    np.savez_compressed(os.path.join(HERE, "source_pin_a06_m2.npz"), **source_case(L, 0.6, 2.0, 37.0))
    np.savez_compressed(os.path.join(HERE, "source_pin_a09_mneg3.npz"), **source_case(L, 0.9, -3.0, 12.5))
    # a third and fourth (a, m): the inclined states, and the remaining
    # equatorial/plunging ones
    np.savez_compressed(os.path.join(HERE, "source_pin_a03_m1_inclined.npz"),
                        **source_case(L, 0.3, 1.0, 41.0, inclined_states()))
    np.savez_compressed(os.path.join(HERE, "source_pin_a095_m4_inclined.npz"),
                        **source_case(L, 0.95, 4.0, 80.0, inclined_states() + particle_states(0.95)[3:]))
    np.savez_compressed(os.path.join(HERE, "proj_pin.npz"), **swsh_case(L, L.ref_M()))
    # The config-1 domain [-100, 300]: the reference's grid() returns NaN
    # radii near the inner edge (r - r+ below FP64 resolution).
    L2 = ref_lib("c1s")
    N2, M2 = L2.ref_N(), L2.ref_M()
    x, r, t = np.zeros(N2), np.zeros(N2), np.zeros(M2)
    L2.ref_grid(D(1.0), D(0.5), p(x), p(r), p(t))
    np.savez_compressed(os.path.join(HERE, "grid_c1s_a05.npz"), x_c=x, r_c=r, theta=t, N=N2, M=M2,
                        Xmin=L2.ref_Xmin(), Xmax=L2.ref_Xmax(), a=0.5)
    # The head of two of the reference's example waveform files
    # (QNM_Extraction/Examples, written by HighOrder/body.cu:208) for the
    # byte-level writer test.
    ex = os.path.join(REF, "QNM_Extraction", "Examples")
    for fn in ("hm2_a0.7_thi000_thf090.0_n.dat", "hmm1_a0.7_thi000_thf090.0_n.dat"):
        with open(os.path.join(ex, fn)) as f:
            head = [next(f) for _ in range(40)]
        with open(os.path.join(HERE, "example_head_" + fn.replace(".dat", ".txt")), "w") as f:
            f.writelines(head)
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))


if __name__ == "__main__":
    main()
