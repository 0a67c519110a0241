"""Trajectory generation: GenOT restated (GenOT/ParamWLMino.cc, GenOT/WL_BL.cc).

The reference makes the worldlines its solver reads in two programs: one
stitches an adiabatic inspiral (a table made from frequency-domain fluxes
by GREMLIN), the generalised Ori-Thorne transition and a geodesic plunge
into a worldline sampled in Mino time; the other integrates that worldline
in Boyer-Lindquist time and writes the 10-column .traj file
(GenOT/README:39-123).  Both steps are host C++ in libbhr
(`bhr_genot_mino`, `bhr_genot_bl`, bhr_genot.cpp); this module holds what
feeds them:

* `ot_table` -- the universal Ori-Thorne function X(T), the solution of
  X'' = -X^2 - T that approaches sqrt(-T) as T -> -infinity, integrated
  from its asymptotic series (`bhr_genot_ot_table`; the reference ships it
  as a table, GenOT/OT_X_vs_L.dat, on the same grid T = -40 + 0.001 k up
  to 3.41);
* `synthetic_inspiral` -- a stand-in for the GREMLIN inspiral tables, which
  are not part of the reference tree: circular prograde Kerr orbits from
  r_start down to the ISCO (equatorial, or tilted as in Schwarzschild),
  with the leading-order quadrupole flux dE/dt = -(32/5) (M Omega)^(10/3)
  (mass ratio scaled out), in the 11-column layout ParamWLMino reads
  (GenOT/ParamWLMino.cc:24-36);
* `mino_worldline`, `bl_worldline`, `write_traj` -- the two programs as
  calls (their arguments in the reference's order and meaning).
"""
from __future__ import annotations

import ctypes as C
import functools
import os
from typing import Optional

import numpy as np

from . import BhrError, _check, _ptr, load_library

D = C.c_double
I = C.c_int


class GenotParams(C.Structure):
    _fields_ = [("a", D), ("eta", D), ("LTi", D), ("LTf", D), ("r_start", D), ("dl", D), ("model", I)]


class GenotBLParams(C.Structure):
    _fields_ = [("a", D), ("lambda_start", D), ("t_stop", D), ("chi0_deg", D), ("phi0_deg", D), ("dt", D)]


def _lib():
    lib = load_library()
    if getattr(lib, "_genot_sigs", False):
        return lib
    dp = C.POINTER(D)
    lib.bhr_genot_mino.restype = I
    lib.bhr_genot_mino.argtypes = [C.POINTER(GenotParams), dp, I, dp, I, dp, I, C.POINTER(I), dp]
    lib.bhr_genot_bl.restype = I
    lib.bhr_genot_bl.argtypes = [C.POINTER(GenotBLParams), dp, I, I, dp, I, C.POINTER(I), dp, C.POINTER(I),
                                 C.c_char_p]
    lib.bhr_genot_traj_name.restype = I
    lib.bhr_genot_traj_name.argtypes = [D, D, D, I, C.c_char_p, I]
    lib.bhr_genot_ot_table.restype = I
    lib.bhr_genot_ot_table.argtypes = [D, D, I, D, dp]
    lib._genot_sigs = True
    return lib


# ---- the Ori-Thorne function ------------------------------------------------
OT_T0, OT_DT, OT_ROWS = -40.0, 0.001, 43411  # the reference table's grid: T = -40 .. 3.41


@functools.lru_cache(maxsize=4)
def ot_table(T0: float = OT_T0, dT: float = OT_DT, rows: int = OT_ROWS, T_start: float = -400.0) -> np.ndarray:
    """Rows (T, X(T)) of the Ori-Thorne function on T = T0 + k dT.

    X'' = -X^2 - T is integrated from its asymptotic series at T_start
    (bhr_genot_ot_table: adaptive classical RK4 with step doubling, relative
    tolerance 1e-13); the result does not change with T_start.  Returned
    read-only."""
    T = T0 + dT * np.arange(rows, dtype=np.float64)
    X = np.zeros(rows)
    _check(_lib().bhr_genot_ot_table(T0, dT, rows, T_start, _ptr(X)))
    out = np.ascontiguousarray(np.column_stack([T, X]))
    out.setflags(write=False)
    return out


# ---- the stand-in adiabatic inspiral ----------------------------------------
def _circular_eq(r: np.ndarray, a: float):
    """E, L and Omega of circular prograde equatorial Kerr orbits (M = 1)."""
    v = 1.0 / np.sqrt(r)
    den = np.sqrt(1.0 - v * v * (3.0 - 2.0 * a * v))
    E = (1.0 - v * v * (2.0 - a * v)) / den
    L = r * v * (1.0 - a * v ** 3 * (2.0 - a * v)) / den
    Om = 1.0 / (r ** 1.5 + a)
    return E, L, Om


def _isco(a: float) -> float:
    z1 = 1.0 + (1.0 - a * a) ** (1.0 / 3.0) * ((1.0 + a) ** (1.0 / 3.0) + (1.0 - a) ** (1.0 / 3.0))
    z2 = np.sqrt(3.0 * a * a + z1 * z1)
    return float(3.0 + z2 - np.sqrt((3.0 - z1) * (3.0 + z1 + 2.0 * z2)))


def synthetic_inspiral(a: float, r_start: float, rows: int = 2000, fine: int = 40,
                       inclination_deg: float = 0.0) -> np.ndarray:
    """An adiabatic inspiral table (rows x 11) from r_start to the ISCO.

    Columns as ParamWLMino reads them: time, Mino time, r, eccentricity,
    theta_inc (degrees), E, L, Q, then the E, L, Q fluxes per unit Mino
    time; time, Mino time and fluxes have the mass ratio scaled out.  The
    orbits are circular and prograde, E and the total angular momentum L
    those of the equatorial orbit; the energy flux per unit (scaled) time is
    (32/5) Omega^(10/3), the angular-momentum flux that over Omega, and
    Mino time follows from dlambda = -(dE/dr) dr / (dE/dlambda) with
    dt/dlambda of the circular orbit.  The last row is the ISCO, where dE/dr
    vanishes.  inclination_deg = i tilts the orbit as in Schwarzschild
    (exact there, a stand-in for a != 0): theta_inc = i, L_z = L cos i,
    Q = L^2 sin^2 i."""
    r_isco = _isco(a)
    if not r_start > r_isco:
        raise ValueError(f"r_start must lie outside the ISCO ({r_isco:.6f})")
    # radii from r_start to the ISCO, dense near the ISCO (r - r_isco ~ s^2)
    s = np.linspace(1.0, 0.0, (rows - 1) * fine + 1)
    r = r_isco + (r_start - r_isco) * s * s
    E, L, Om = _circular_eq(r, a)
    D_ = r * r - 2.0 * r + a * a
    r2a2 = r * r + a * a
    dtdl = E * r2a2 * r2a2 / D_ - a * L * r2a2 / D_ - a * a * E + a * L
    fE = 32.0 / 5.0 * Om ** (10.0 / 3.0) * dtdl       # -dE/dlambda
    # dE/dr of circular orbits, analytically through dE/dv (v = r^(-1/2))
    v = 1.0 / np.sqrt(r)
    g = 1.0 - v * v * (3.0 - 2.0 * a * v)
    num = 1.0 - v * v * (2.0 - a * v)
    dnum = -4.0 * v + 3.0 * a * v * v
    dg = -6.0 * v + 6.0 * a * v * v
    dEdv = (dnum * np.sqrt(g) - num * 0.5 * dg / np.sqrt(g)) / g
    dEdr = dEdv * (-0.5 * r ** -1.5)
    # lambda and t along decreasing r (trapezoid on the fine grid)
    dldr = -dEdr / fE
    lam = np.concatenate([[0.0], np.cumsum(0.5 * (dldr[1:] + dldr[:-1]) * np.diff(r))])
    t = np.concatenate([[0.0], np.cumsum(0.5 * (dtdl[1:] + dtdl[:-1]) * np.diff(lam))])
    k = np.arange(0, len(r), fine)
    ci, si = np.cos(np.radians(inclination_deg)), np.sin(np.radians(inclination_deg))
    fL = fE[k] / Om[k]
    out = np.zeros((len(k), 11))
    out[:, 0] = t[k]
    out[:, 1] = lam[k]
    out[:, 2] = r[k]
    out[:, 4] = inclination_deg
    out[:, 5] = E[k]
    out[:, 6] = L[k] * ci
    out[:, 7] = (L[k] * si) ** 2
    out[:, 8] = fE[k]
    out[:, 9] = fL * ci
    out[:, 10] = 2.0 * L[k] * fL * si * si
    return out


# ---- the two steps ----------------------------------------------------------
def mino_worldline(a: float, eta: float, insp: np.ndarray, LTi: float, LTf: float, r_start: float,
                   model: int = 2, dl: float = 0.1, ot: Optional[np.ndarray] = None,
                   transition: Optional[np.ndarray] = None) -> np.ndarray:
    """Rows (lambda, r, theta_inc, E, L, Q): ParamWLMino's output for
    arguments a, eta, the inspiral table, LTi, LTf, r_start and model.
    transition (4 floats, optional) receives lambda and r where the
    transition begins and ends."""
    lib = _lib()
    insp = np.ascontiguousarray(insp, dtype=np.float64)
    ot = np.ascontiguousarray(ot_table() if ot is None else ot, dtype=np.float64)
    if insp.ndim != 2 or insp.shape[1] != 11 or ot.ndim != 2 or ot.shape[1] != 2:
        raise ValueError("inspiral table needs 11 columns, the Ori-Thorne table 2")
    p = GenotParams(a, eta, LTi, LTf, r_start, dl, model)
    n = I(0)
    tr = np.zeros(4)
    _check(lib.bhr_genot_mino(C.byref(p), _ptr(insp), len(insp), _ptr(ot), len(ot), None, 0, C.byref(n), None))
    out = np.zeros((n.value, 6))
    _check(lib.bhr_genot_mino(C.byref(p), _ptr(insp), len(insp), _ptr(ot), len(ot), _ptr(out), n.value,
                              C.byref(n), _ptr(tr)))
    if transition is not None:
        transition[:] = (tr[0], tr[2], tr[1], tr[3])
    return out[: n.value]


def bl_worldline(mino: np.ndarray, a: float, lambda_start: float, t_stop: float, chi0_deg: float = 0.0,
                 phi0_deg: float = 0.0, dt: float = 0.001, stride: int = 1, path: Optional[str] = None,
                 rows: bool = True):
    """WL_BL's worldline: (rows, theta_f in degrees, dtheta/dlambda > 0 at the end).

    rows: every stride-th .traj row (None with rows=False); path: every row
    written there in the reference's text format."""
    lib = _lib()
    mino = np.ascontiguousarray(mino, dtype=np.float64)
    if mino.ndim != 2 or mino.shape[1] != 6:
        raise ValueError("the Mino-time worldline needs 6 columns")
    p = GenotBLParams(a, lambda_start, t_stop, chi0_deg, phi0_deg, dt)
    n = I(0)
    out = None
    if rows:
        _check(lib.bhr_genot_bl(C.byref(p), _ptr(mino), len(mino), stride, None, 0, C.byref(n), None, None, None))
        out = np.zeros((n.value, 10))
    thf, pos = D(0.0), I(0)
    _check(lib.bhr_genot_bl(C.byref(p), _ptr(mino), len(mino), stride, _ptr(out), 0 if out is None else len(out),
                            C.byref(n), C.byref(thf), C.byref(pos), None if path is None else path.encode()))
    return out, thf.value, bool(pos.value)


def traj_name(a: float, thi0_deg: float, thf_deg: float, thdot_pos: bool) -> str:
    """The reference's .traj file name for these values (GenOT/WL_BL.cc:101-153)."""
    buf = C.create_string_buffer(128)
    _check(_lib().bhr_genot_traj_name(a, thi0_deg, thf_deg, 1 if thdot_pos else 0, buf, len(buf)))
    return buf.value.decode()


def write_traj(directory: str, mino: np.ndarray, a: float, lambda_start: float, t_stop: float,
               chi0_deg: float = 0.0, phi0_deg: float = 0.0, dt: float = 0.001) -> str:
    """WL_BL as the reference runs it: a first pass finds theta_f and the
    sign of dtheta/dlambda at t_stop, which name the file; the second writes
    every row there.  Returns the path."""
    _, thf, pos = bl_worldline(mino, a, lambda_start, t_stop, chi0_deg, phi0_deg, dt, rows=False)
    path = os.path.join(directory, traj_name(a, float(mino[0, 2]), thf, pos))
    _, thf2, _ = bl_worldline(mino, a, lambda_start, t_stop, chi0_deg, phi0_deg, dt, rows=False, path=path)
    if thf2 != thf:
        raise BhrError(1, "bl_worldline: the two passes disagree")
    return path


def transition_plunge(a: float, eta: float, dt_row: float, duration: float, inclination_deg: float = 0.0,
                      LTi: float = -3.0, LTf: float = 2.35, model: int = 2, chi0_deg: float = 0.0) -> np.ndarray:
    """A transition-to-plunge source worldline as .traj rows every dt_row
    in BL time for `duration`: the stand-in inspiral of spin a (from 1 M
    outside the ISCO), GenOT's Mino-time worldline for mass ratio eta
    (LTi = -3, LTf = 2.35, the values GenOT/README:159-166 recommends;
    model 2), and its BL-time worldline from the Mino time at which the
    transition begins, near the ISCO.  After the plunge the particle
    approaches the horizon for the rest of the duration, as the reference's
    files do."""
    r_isco = _isco(a)
    insp = synthetic_inspiral(a, r_isco + 1.0, inclination_deg=inclination_deg)
    tr = np.zeros(4)
    mino = mino_worldline(a, eta, insp, LTi, LTf, r_isco + 0.5, model=model, transition=tr)
    rows, _, _ = bl_worldline(mino, a, tr[0], duration, chi0_deg, 0.0, dt=dt_row)
    return rows


def read_insp(path: str) -> np.ndarray:
    """An adiabatic inspiral table file (11 whitespace-separated columns)."""
    rows = np.loadtxt(path, dtype=np.float64, ndmin=2)
    if rows.shape[1] < 11:
        raise ValueError(f"{path}: expected 11 columns, found {rows.shape[1]}")
    return np.ascontiguousarray(rows[:, :11])


def read_mino(path: str) -> np.ndarray:
    """A Mino-time worldline file (lambda r theta_inc E L Q)."""
    rows = np.loadtxt(path, dtype=np.float64, ndmin=2)
    if rows.shape[1] != 6:
        raise ValueError(f"{path}: expected 6 columns, found {rows.shape[1]}")
    return rows
