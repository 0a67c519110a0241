"""ctypes binding of the FP64 CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the
cpu_baseline leg of bench.py as the oracle.  The product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
D, I = C.c_double, C.c_int


class OrcParams(C.Structure):
    _fields_ = [("N", I), ("M", I), ("Xmin", D), ("Xmax", D), ("mass", D), ("a", D), ("m", D), ("dt", D),
                ("T", D), ("Fr", I), ("PTSX", I), ("PTSY", I), ("wr_fac", D), ("wt_fac", D), ("out_start", D),
                ("ext_col", I)]


class OrcParticle(C.Structure):
    _fields_ = [(n, D) for n in ("rp", "tp", "phip", "E", "lz", "Q", "drdt", "d2rdt2", "d3rdt3", "dthdt",
                                 "d2thdt2", "d3thdt3", "dphidt", "d2phidt2")]


COEF_FN = C.CFUNCTYPE(None, C.POINTER(OrcParticle), D, D, D, C.POINTER(D), C.POINTER(D))

_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        vp, dp = C.c_void_p, C.POINTER(D)
        sig = {
            "orc_create": (vp, [C.POINTER(OrcParams)]),
            "orc_destroy": (None, [vp]),
            "orc_get_grid": (None, [vp, dp, dp, dp]),
            "orc_get_coeff": (None, [vp, I, dp]),
            "orc_set_state": (None, [vp, dp, dp, dp, dp]),
            "orc_get_state": (None, [vp, dp, dp, dp, dp]),
            "orc_apply_closure": (None, [vp]),
            "orc_init_gaussian": (None, [vp, D, D, D]),
            "orc_set_source": (None, [vp, dp, dp]),
            "orc_get_source": (None, [vp, dp, dp]),
            "orc_deposit_source": (None, [vp, C.POINTER(OrcParticle), dp, dp, D, D]),
            "orc_step": (None, [vp]),
            "orc_set_integrator": (None, [vp, I]),
            "orc_eval_rhs": (None, [vp, dp, dp]),
            "orc_get_ext": (None, [vp, dp, dp]),
            "orc_swsh": (D, [D, D, D]),
            "orc_project": (D, [dp, I, D, D]),
            "orc_run": (I, [vp, dp, I, COEF_FN, I, dp, dp, dp, I, C.POINTER(I), I, dp, dp, I, C.POINTER(I)]),
            "orc_num_threads": (I, []),
            "orc_set_num_threads": (None, [I]),
        }
        for n, (r, a) in sig.items():
            f = getattr(L, n)
            f.restype, f.argtypes = r, a
        _lib = L
    return _lib


def _p(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(D))


class Oracle:
    """FP64 CPU restatement of the reference HighOrder step (see teuk_oracle.h)."""

    def __init__(self, N, M, Xmin, Xmax, a, m, dt, mass=1.0, T=100.0, Fr=1, PTSX=128, PTSY=128, wr_fac=2.0,
                 wt_fac=6.0, out_start=0.0, ext_col=-1, integrator=0):
        """integrator: 0 SSP-RK3 (the reference's), 1 classical RK4."""
        self.L = lib()
        self.N, self.M = N, M
        self.params = OrcParams(N, M, Xmin, Xmax, mass, a, m, dt, T, Fr, PTSX, PTSY, wr_fac, wt_fac, out_start,
                                N - 1 if ext_col < 0 else ext_col)
        self.h = self.L.orc_create(C.byref(self.params))
        if not self.h:
            raise ValueError("orc_create rejected the parameters")
        self.h = C.c_void_p(self.h)
        self.L.orc_set_integrator(self.h, integrator)

    def close(self):
        if self.h:
            self.L.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def grid(self):
        x, r, t = np.zeros(self.N), np.zeros(self.N), np.zeros(self.M)
        self.L.orc_get_grid(self.h, _p(x), _p(r), _p(t))
        return x, r, t

    def coeff(self, k):
        out = np.zeros(self.N * self.M)
        self.L.orc_get_coeff(self.h, k, _p(out))
        return out.reshape(self.M, self.N)

    def set_state(self, planes):
        arrs = [np.ascontiguousarray(x, dtype=np.float64).reshape(-1) for x in planes]
        self.L.orc_set_state(self.h, *[_p(x) for x in arrs])

    def get_state(self):
        out = [np.zeros(self.N * self.M) for _ in range(4)]
        self.L.orc_get_state(self.h, *[_p(x) for x in out])
        return [x.reshape(self.M, self.N) for x in out]

    def init_gaussian(self, center, width, ell):
        self.L.orc_init_gaussian(self.h, center, width, ell)

    def apply_closure(self):
        self.L.orc_apply_closure(self.h)

    def set_source(self, tre=None, tim=None):
        a = None if tre is None else np.ascontiguousarray(tre, dtype=np.float64).reshape(-1)
        b = None if tim is None else np.ascontiguousarray(tim, dtype=np.float64).reshape(-1)
        self.L.orc_set_source(self.h, _p(a), _p(b))

    def get_source(self):
        a, b = np.zeros(self.N * self.M), np.zeros(self.N * self.M)
        self.L.orc_get_source(self.h, _p(a), _p(b))
        return a.reshape(self.M, self.N), b.reshape(self.M, self.N)

    def deposit_source(self, pt: OrcParticle, coef6: np.ndarray, timer: float, start: float = 0.0):
        cr = np.ascontiguousarray(coef6.real, dtype=np.float64)
        ci = np.ascontiguousarray(coef6.imag, dtype=np.float64)
        self.L.orc_deposit_source(self.h, C.byref(pt), _p(cr), _p(ci), timer, start)

    def eval_rhs(self, planes):
        """kernel_rhs of the closure of `planes` (4 x M x N), interior points."""
        x = np.ascontiguousarray(np.stack([np.asarray(p, dtype=np.float64) for p in planes]))
        out = np.zeros_like(x)
        self.L.orc_eval_rhs(self.h, _p(x.reshape(-1)), _p(out.reshape(-1)))
        return out

    def step(self, n=1):
        for _ in range(n):
            self.L.orc_step(self.h)

    def ext(self):
        a, b = np.zeros(self.M), np.zeros(self.M)
        self.L.orc_get_ext(self.h, _p(a), _p(b))
        return a, b

    def run(self, traj=None, coef_fn=None, nsteps=-1, max_rows=100000, ext_every=0, max_ext=0):
        t, h, e = np.zeros(max_rows), np.zeros(max_rows * 14), np.zeros(max_rows)
        steps = np.zeros(max_rows, dtype=np.int32)
        er, ei = np.zeros(max(1, max_ext) * self.M), np.zeros(max(1, max_ext) * self.M)
        next_ = I(0)
        tr = None if traj is None else np.ascontiguousarray(traj, dtype=np.float64)
        cb = coef_fn if coef_fn is not None else COEF_FN()
        n = self.L.orc_run(self.h, _p(tr), 0 if tr is None else tr.shape[0], cb, nsteps, _p(t), _p(h), _p(e),
                           max_rows, steps.ctypes.data_as(C.POINTER(I)), ext_every, _p(er), _p(ei), max_ext,
                           C.byref(next_))
        if n < 0:
            raise ValueError("orc_run failed")
        k = next_.value
        return (t[:n], h[: 14 * n].reshape(n, 14), e[:n], steps[:n],
                er[: k * self.M].reshape(k, self.M), ei[: k * self.M].reshape(k, self.M))


def swsh(ell, m, th):
    return lib().orc_swsh(ell, m, th)


def set_threads(n):
    lib().orc_set_num_threads(n)


def num_threads():
    return lib().orc_num_threads()
