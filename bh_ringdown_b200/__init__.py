"""bh_ringdown_b200: B200-native time-domain Teukolsky solver (Python host mirror).

The compute path is the C ABI of ``include/bhr.h`` implemented in
``bh_ringdown_b200/libbhr.so`` (sm_100a CUDA kernels plus C++ host code).
This module binds that library with ctypes and mirrors the reference
driver surface: the run knobs of TD_GPU_code/HighOrder/parm.h and main.c,
the .traj trajectory input and the hm*.dat waveform output of body.cu.

There is no fallback: if the library is missing or fails to load, every
call raises.  Build it with ``python __graft_entry__.py`` or
``make -C bh_ringdown_b200/csrc``.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field, fields
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libbhr.so")

D = C.c_double
I = C.c_int

BHR_OK = 0
STATUS_NAMES = {0: "OK", 1: "INVALID_ARG", 2: "OUT_OF_MEMORY", 3: "CUDA_ERROR", 4: "NAN_DETECTED",
                5: "TIMEOUT", 6: "IO_ERROR", 7: "NO_DEVICE"}

BHR_SSPRK3, BHR_RK4 = 0, 1
BHR_FP64, BHR_MIXED = 0, 1
BHR_INIT_ZERO, BHR_INIT_GAUSSIAN = 0, 1


class BhrError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


class _Params(C.Structure):
    _fields_ = [("N", I), ("M", I), ("Xmin", D), ("Xmax", D), ("mass", D), ("a", D), ("m", D), ("dt", D),
                ("courant", D), ("out_every", D), ("T", D), ("Fr", I), ("out_start", D), ("ext_col", I),
                ("PTSX", I), ("PTSY", I), ("wr_fac", D), ("wt_fac", D), ("integrator", I), ("precision", I),
                ("init_kind", I), ("init_center", D), ("init_width", D), ("init_ell", D), ("device", I)]


class Particle(C.Structure):
    """One particle state as HighOrder/body.cu:112-124 hands it to sourced()."""
    _fields_ = [(n, D) for n in ("rp", "tp", "phip", "E", "lz", "Q", "drdt", "d2rdt2", "d3rdt3", "dthdt",
                                 "d2thdt2", "d3thdt3", "dphidt", "d2phidt2")]


class _Info(C.Structure):
    _fields_ = [("N", I), ("M", I), ("dx", D), ("dtheta", D), ("dt", D), ("nt", I), ("Fr", I),
                ("steps_done", I), ("rows_done", I), ("has_source", I), ("r_plus", D), ("device_bytes", C.c_size_t),
                ("tile_rows", I), ("persistent", I), ("tiling", I), ("prefetch_ahead", I)]

TILINGS = ("block8", "block16", "persistent", "block8n", "ring", "strip12")  # bhr_tiling, by value


class _RequestInfo(C.Structure):
    _fields_ = [("state", I), ("status", I), ("steps_total", I), ("steps_done", I), ("nrows", I),
                ("submit_s", D), ("start_s", D), ("finish_s", D)]


class _EngineStats(C.Structure):
    _fields_ = [("queued", I), ("running", I), ("finished", I), ("tiles", I), ("batch_steps", C.c_longlong),
                ("point_updates", D), ("device_ms", D), ("bytes_in_use", C.c_size_t), ("budget", C.c_size_t)]


@dataclass
class Params:
    """Run parameters; defaults are the reference's (HighOrder/parm.h, main.c)."""
    N: int = 16000
    M: int = 256
    Xmin: float = -50.0
    Xmax: float = 50.0
    mass: float = 1.0
    a: float = 1e-8
    m: float = 2.0
    dt: float = 0.002
    courant: float = 0.25
    out_every: float = 0.0
    T: float = 1500.0
    Fr: int = 50
    out_start: Optional[float] = None  # None -> Xmax + 200 (HighOrder/body.cu:207)
    ext_col: int = -1
    PTSX: int = 128
    PTSY: int = 128
    wr_fac: float = 2.0
    wt_fac: float = 6.0
    integrator: int = BHR_SSPRK3
    precision: int = BHR_FP64
    init_kind: int = BHR_INIT_ZERO
    init_center: float = 20.0
    init_width: float = 2.0
    init_ell: float = 2.0
    device: int = 0

    def to_c(self) -> _Params:
        p = _Params()
        for f in fields(self):
            v = getattr(self, f.name)
            if f.name == "out_start" and v is None:
                v = self.Xmax + 200.0
            setattr(p, f.name, v)
        return p


_lib = None


def load_library(path: str = LIB_PATH) -> C.CDLL:
    """Load libbhr.so (raises if it is missing: there is no CPU fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"{path} not built; run `python __graft_entry__.py` or `make -C bh_ringdown_b200/csrc`")
    lib = C.CDLL(path)
    P = C.POINTER
    vp = C.c_void_p
    dp = P(D)
    sigs = {
        "bhr_abi_version": (I, []),
        "bhr_selftest_bounded_wait": (I, [I, C.POINTER(I)]),
        "bhr_selftest_math": (I, [I, dp, I, dp]),
        "bhr_last_error_string": (C.c_char_p, []),
        "bhr_params_default": (I, [P(_Params)]),
        "bhr_grid": (I, [P(_Params), dp, dp, dp]),
        "bhr_solver_create": (I, [P(_Params), P(vp)]),
        "bhr_solver_destroy": (None, [vp]),
        "bhr_solver_info": (I, [vp, P(_Info)]),
        "bhr_solver_set_trajectory": (I, [vp, dp, I]),
        "bhr_solver_load_trajectory": (I, [vp, C.c_char_p]),
        "bhr_solver_step": (I, [vp, I]),
        "bhr_solver_run": (I, [vp, C.c_char_p, C.c_char_p]),
        "bhr_solver_waveform": (I, [vp, dp, dp, dp, I, P(I)]),
        "bhr_solver_get_state": (I, [vp, dp, dp, dp, dp]),
        "bhr_solver_set_state": (I, [vp, dp, dp, dp, dp]),
        "bhr_solver_get_extraction": (I, [vp, dp, dp, dp, dp, dp, dp]),
        "bhr_solver_get_source": (I, [vp, dp, dp]),
        "bhr_solver_psi_samples": (I, [vp, dp, dp, I, C.POINTER(I)]),
        "bhr_solver_checkpoint_size": (C.c_size_t, [vp]),
        "bhr_solver_checkpoint": (I, [vp, vp, C.c_size_t]),
        "bhr_solver_restore": (I, [vp, vp, C.c_size_t]),
        "bhr_solver_stream": (vp, [vp]),
        "bhr_solver_profile": (I, [vp, I, dp, dp]),
        "bhr_solver_time_steps": (I, [vp, I, dp]),
        "bhr_source_coefficients": (I, [P(Particle), D, D, D, dp, dp]),
        "bhr_swsh": (D, [D, D, D]),
        "bhr_write_waveform": (I, [C.c_char_p, C.c_char_p, D, dp, dp, dp, I]),
        "bhr_step_noalloc": (I, [P(_Params), vp, I, vp]),
        "bhr_engine_create": (I, [I, C.c_size_t, P(vp)]),
        "bhr_engine_destroy": (None, [vp]),
        "bhr_engine_submit": (I, [vp, P(_Params), dp, I, P(C.c_int64)]),
        "bhr_engine_step": (I, [vp, I, P(I)]),
        "bhr_engine_poll": (I, [vp, C.c_int64, P(_RequestInfo)]),
        "bhr_engine_result": (I, [vp, C.c_int64, dp, dp, dp, I, P(I)]),
        "bhr_engine_stats": (I, [vp, P(_EngineStats)]),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _ptr(a: Optional[np.ndarray]):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(D))


def _check(st: int):
    if st != BHR_OK:
        raise BhrError(st, load_library().bhr_last_error_string().decode(errors="replace"))


def selftest_bounded_wait(device: int = 0) -> int:
    """Runs the device self-check of the bounded waits; returns the status
    the kernel reported (BHR_TIMEOUT when the wait gave up as designed)."""
    st = I(0)
    _check(load_library().bhr_selftest_bounded_wait(device, C.byref(st)))
    return st.value


def selftest_math(x: np.ndarray, device: int = 0):
    """(rcp, 1/x, sqrt, sqrt(x)) computed on the device: the library's
    Newton-refined reciprocal and square root beside CUDA's own."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.zeros(4 * len(x))
    _check(load_library().bhr_selftest_math(device, _ptr(x), len(x), _ptr(out)))
    return out.reshape(4, len(x))


def grid(params: Params):
    """x_c[N], r_c[N], theta[M] of HighOrder/main.c:64-183."""
    lib = load_library()
    x, r, t = np.zeros(params.N), np.zeros(params.N), np.zeros(params.M)
    p = params.to_c()
    _check(lib.bhr_grid(C.byref(p), _ptr(x), _ptr(r), _ptr(t)))
    return x, r, t


def swsh(ell: float, m: float, theta: float) -> float:
    return load_library().bhr_swsh(ell, m, theta)


def source_coefficients(pt: Particle, a: float, mass: float, m: float):
    """Six complex coefficients of DelR^(i) DelTH^(j), (i,j) in
    (0,0) (0,1) (0,2) (1,0) (1,1) (2,0)."""
    lib = load_library()
    cr, ci = np.zeros(6), np.zeros(6)
    _check(lib.bhr_source_coefficients(C.byref(pt), a, mass, m, _ptr(cr), _ptr(ci)))
    return cr + 1j * ci


def write_waveform(out_dir: str, name: str, m: float, t: np.ndarray, h: np.ndarray, dedt=None):
    """hm<m>_<name>.dat in the reference format (plus a full-precision .full)."""
    t = np.ascontiguousarray(t, dtype=np.float64)
    h = np.ascontiguousarray(h, dtype=np.float64).reshape(len(t), 14)
    e = None if dedt is None else np.ascontiguousarray(dedt, dtype=np.float64)
    _check(load_library().bhr_write_waveform(out_dir.encode(), name.encode(), m, _ptr(t), _ptr(h), _ptr(e), len(t)))


def step_noalloc(params: Params, state_ptr: int, nsteps: int, stream: int = 0):
    """bhr_step_noalloc on device memory the caller owns (state_ptr: address
    of four contiguous closed M x N FP64 planes)."""
    p = params.to_c()
    _check(load_library().bhr_step_noalloc(C.byref(p), C.c_void_p(state_ptr), int(nsteps),
                                           C.c_void_p(stream) if stream else None))


class Solver:
    """One solve on one device (replaces HighOrder/body.cu:body())."""

    def __init__(self, params: Params):
        self.lib = load_library()
        self.params = params
        self._p = params.to_c()
        h = C.c_void_p()
        _check(self.lib.bhr_solver_create(C.byref(self._p), C.byref(h)))
        self._h = h
        self.N, self.M = params.N, params.M

    def close(self):
        if getattr(self, "_h", None):
            self.lib.bhr_solver_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def info(self) -> dict:
        inf = _Info()
        _check(self.lib.bhr_solver_info(self._h, C.byref(inf)))
        d = {f[0]: getattr(inf, f[0]) for f in _Info._fields_}
        d["tiling"] = TILINGS[d["tiling"]]
        return d

    def set_trajectory(self, rows: np.ndarray):
        rows = np.ascontiguousarray(rows, dtype=np.float64)
        assert rows.ndim == 2 and rows.shape[1] == 10
        _check(self.lib.bhr_solver_set_trajectory(self._h, _ptr(rows), rows.shape[0]))

    def load_trajectory(self, path: str):
        _check(self.lib.bhr_solver_load_trajectory(self._h, path.encode()))

    def step(self, nsteps: int = 1):
        _check(self.lib.bhr_solver_step(self._h, int(nsteps)))

    def run(self, out_dir: Optional[str] = None, name: Optional[str] = None):
        _check(self.lib.bhr_solver_run(self._h, out_dir.encode() if out_dir else None,
                                       name.encode() if name else None))

    def waveform(self):
        n_max = self.info()["rows_done"]
        t, h, e = np.zeros(n_max), np.zeros(n_max * 14), np.zeros(n_max)
        n = I(0)
        _check(self.lib.bhr_solver_waveform(self._h, _ptr(t), _ptr(h), _ptr(e), n_max, C.byref(n)))
        n = n.value
        return t[:n], h[: n * 14].reshape(n, 14), e[:n]

    def get_state(self):
        NM = self.N * self.M
        out = [np.zeros(NM) for _ in range(4)]
        _check(self.lib.bhr_solver_get_state(self._h, *[_ptr(x) for x in out]))
        return [x.reshape(self.M, self.N) for x in out]

    def set_state(self, qre, qim, pre, pim):
        arrs = [np.ascontiguousarray(x, dtype=np.float64).reshape(-1) for x in (qre, qim, pre, pim)]
        _check(self.lib.bhr_solver_set_state(self._h, *[_ptr(x) for x in arrs]))

    def get_extraction(self):
        out = [np.zeros(self.M) for _ in range(6)]
        _check(self.lib.bhr_solver_get_extraction(self._h, *[_ptr(x) for x in out]))
        return out

    def get_source(self):
        tre, tim = np.zeros(self.N * self.M), np.zeros(self.N * self.M)
        _check(self.lib.bhr_solver_get_source(self._h, _ptr(tre), _ptr(tim)))
        return tre.reshape(self.M, self.N), tim.reshape(self.M, self.N)

    def psi_samples(self):
        """psi(theta) at the extraction column on each waveform row's step:
        (re, im), each rows x M."""
        n = self.info()["rows_done"]
        re, im = np.zeros(max(1, n) * self.M), np.zeros(max(1, n) * self.M)
        got = I(0)
        _check(self.lib.bhr_solver_psi_samples(self._h, _ptr(re), _ptr(im), n, C.byref(got)))
        k = got.value
        return re[:k * self.M].reshape(k, self.M), im[:k * self.M].reshape(k, self.M)

    def checkpoint(self) -> bytes:
        """The solve's resumable state (fields, extraction integrals, counters,
        waveform rows so far) as bytes; see restore()."""
        n = self.lib.bhr_solver_checkpoint_size(self._h)
        if n == 0:
            raise BhrError(3, "checkpoint size unavailable: " + self.lib.bhr_last_error_string().decode(errors="replace"))
        buf = C.create_string_buffer(n)
        _check(self.lib.bhr_solver_checkpoint(self._h, buf, n))
        return buf.raw

    def restore(self, data: bytes):
        """Continues from a checkpoint of a solve with the same parameters
        (and the same trajectory, when sourced)."""
        buf = C.create_string_buffer(bytes(data), len(data))
        _check(self.lib.bhr_solver_restore(self._h, buf, len(data)))

    def stream(self) -> int:
        return int(self.lib.bhr_solver_stream(self._h) or 0)

    def time_steps(self, nsteps: int) -> float:
        """Advance nsteps (captured CUDA graphs) and return their device time in ms."""
        ms = np.zeros(1)
        _check(self.lib.bhr_solver_time_steps(self._h, int(nsteps), _ptr(ms)))
        return float(ms[0])

    def profile(self, nsteps: int):
        avg, tot = np.zeros(5), np.zeros(1)
        _check(self.lib.bhr_solver_profile(self._h, int(nsteps), _ptr(avg), _ptr(tot)))
        return avg, float(tot[0])


class Engine:
    """Many solves on one device advanced together (bhr_engine_*): submit
    requests at any time, call step() to advance everything running, and
    collect each finished request's waveform with result()."""

    QUEUED, RUNNING, DONE, FAILED = 1, 2, 3, 4

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 64 << 30):
        self.lib = load_library()
        h = C.c_void_p()
        _check(self.lib.bhr_engine_create(int(device), int(hbm_budget_bytes), C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self.lib.bhr_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def submit(self, params: Params, traj: Optional[np.ndarray] = None) -> int:
        p = params.to_c()
        rid = C.c_int64(0)
        if traj is None:
            _check(self.lib.bhr_engine_submit(self._h, C.byref(p), None, 0, C.byref(rid)))
        else:
            rows = np.ascontiguousarray(traj, dtype=np.float64)
            assert rows.ndim == 2 and rows.shape[1] == 10
            _check(self.lib.bhr_engine_submit(self._h, C.byref(p), _ptr(rows), rows.shape[0], C.byref(rid)))
        return rid.value

    def step(self, max_steps: int) -> int:
        running = I(0)
        _check(self.lib.bhr_engine_step(self._h, int(max_steps), C.byref(running)))
        return running.value

    def poll(self, rid: int) -> dict:
        inf = _RequestInfo()
        _check(self.lib.bhr_engine_poll(self._h, int(rid), C.byref(inf)))
        return {f[0]: getattr(inf, f[0]) for f in _RequestInfo._fields_}

    def result(self, rid: int):
        n_max = self.poll(rid)["nrows"]
        t, h, e = np.zeros(n_max), np.zeros(n_max * 14), np.zeros(n_max)
        n = I(0)
        _check(self.lib.bhr_engine_result(self._h, int(rid), _ptr(t), _ptr(h), _ptr(e), n_max, C.byref(n)))
        n = n.value
        return t[:n], h[: n * 14].reshape(n, 14), e[:n]

    def stats(self) -> dict:
        st = _EngineStats()
        _check(self.lib.bhr_engine_stats(self._h, C.byref(st)))
        return {f[0]: getattr(st, f[0]) for f in _EngineStats._fields_}

    def run_all(self, chunk: int = 1 << 30) -> None:
        """Steps until nothing is queued, running or being released."""
        while True:
            running = self.step(chunk)
            st = self.stats()
            if running == 0 and st["queued"] == 0 and st["running"] == 0:
                return


__all__ = ["Params", "Particle", "Solver", "Engine", "BhrError", "grid", "swsh", "source_coefficients", "load_library",
           "BHR_INIT_ZERO", "BHR_INIT_GAUSSIAN", "BHR_FP64", "BHR_MIXED", "BHR_SSPRK3", "BHR_RK4"]
