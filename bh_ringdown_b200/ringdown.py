"""Spheroidal QNM excitation coefficients of waveform files: the analysis the
reference runs on its solver output (QNM_Extraction/Scripts/
Extract_Ringdown_MoreModes.py, Scripts/Postprocess.py and
Library/ringdownlib.py), restated so it runs here on this solver's files.

The inputs are the reference's: the .traj file (only its light-ring
crossing time is used), the hm<m>_/hmm<|m|>_ waveform files (t, then h+ and
hx for l = |m|..|m|+6), the Kerr QNM tables Tables/kerr/n<n+1>l<l>m<m>.dat
(a, Re omega, Im omega, ...) and the spherical-spheroidal overlap tables
Tables/swsh/l<l>m<m>lp<l'>np<n'>.dat (a, Re mu, Im mu).

Step 1 (spheroidal_coefficients, Extract_Ringdown_MoreModes.py:94-211):
for one m and l = max(2,|m|)..|m|+mmax, the waveform columns are put on
the file's uniform time grid and then on a 0.1 M grid by linear
interpolation; from 50 M before the light-ring crossing on, the spherical
multipoles h_l = h+ - i hx and their time derivatives (second-order
central differences) are, at every time, the right-hand side of a square
linear system whose unknowns are the co- and counter-rotating spheroidal
(l', n'=0) amplitudes at the crossing time:
    h_l(t)  = sum_l' mu_{l l'} e^{w_l' (t - t_lr)} C_l'
    h_l'(t) = sum_l' w_l' mu_{l l'} e^{w_l' (t - t_lr)} C_l'
with w = -i omega_R - omega_I for co-rotating modes and i omega_R - omega_I
for counter-rotating ones, and mu the conjugated overlap (co-rotating) or
(-1)^l times the overlap (counter-rotating) (Extract_Ringdown_MoreModes.py:
13-83).  Step 2 (excitation_coefficients, Postprocess.py:19-167): the
50 M window, among those starting in the first 250 M of the solution, over
which the amplitudes |C| vary least (sum of std/mean) gives the excitation
amplitudes and phases (mean over the window, phases unwrapped, mod 2 pi).

The writers reproduce the reference's file names and number formats, so
its example outputs (QNM_Extraction/Examples) can be compared as text.
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np


def light_ring_radius(a: float) -> float:
    """Prograde equatorial light ring of a Kerr hole of spin a (M = 1)
    (Extract_Ringdown_MoreModes.py:234)."""
    return 2.0 * (1.0 + np.cos((2.0 / 3.0) * np.arccos(-abs(a))))


def light_ring_crossing(traj_rows: np.ndarray, a: float) -> float:
    """Time of the trajectory row whose radius is nearest the light ring
    (ringdownlib.py:42-47)."""
    r_lr = light_ring_radius(a)
    return float(traj_rows[np.argmin(np.abs(traj_rows[:, 1] - r_lr)), 0])


def m_label(m: int) -> str:
    return f"mm{abs(m)}" if m < 0 else f"m{m}"


@dataclass
class Tables:
    """The reference's table folders; files are read once and cached."""
    kerr_dir: str
    swsh_dir: str
    _cache: Dict[str, np.ndarray] = field(default_factory=dict, repr=False)

    def _load(self, path: str, **kw) -> np.ndarray:
        if path not in self._cache:
            self._cache[path] = np.loadtxt(path, **kw)
        return self._cache[path]

    def qnm(self, l: int, m: int, n: int, a: float) -> complex:
        """omega_{lmn}(a), Im < 0, linear in a between rows; negative m
        reads the table of |m| at -a, and negative spin the mm table
        (ringdownlib.py:144-157)."""
        if m < 0:
            m, a = -m, -a
        name = f"n{n + 1}l{l}m{m}.dat" if a >= 0 else f"n{n + 1}l{l}mm{m}.dat"
        d = self._load(os.path.join(self.kerr_dir, name), usecols=(0, 1, 2))
        x = abs(a)
        return complex(np.interp(x, d[:, 0], d[:, 1]), np.interp(x, d[:, 0], d[:, 2]))

    def overlap(self, m: int, l: int, lp: int, npr: int, a: float) -> Tuple[float, float]:
        """(Re, Im) of the spherical (l, m) - spheroidal (l', m, n') overlap
        at spin a (ringdownlib.py:125-142): linear in a between rows, or
        the single row of a one-row file when its spin is a."""
        name = f"l{l}m{m}lp{lp}np{npr}.dat" if m >= 0 else f"l{l}mm{abs(m)}lp{lp}np{npr}.dat"
        d = self._load(os.path.join(self.swsh_dir, name))
        if d.ndim == 1:
            if a != d[0]:
                raise ValueError(f"{name} holds spin {d[0]} only")
            return float(d[1]), float(d[2])
        return float(np.interp(a, d[:, 0], d[:, 1])), float(np.interp(a, d[:, 0], d[:, 2]))


def mode_files(paths: Sequence[str], m: int, mmax: int) -> Dict[int, Tuple[str, int]]:
    """{l: (file, column of h+)} for l = max(2,|m|)..|m|+mmax: the file whose
    name says it holds m (hm<k>_ for m = k >= 0, hmm<k>_ for m = -k), the
    column 1 + 2 (l - |m|) (ringdownlib.py:61-113)."""
    want: Dict[int, Tuple[str, int]] = {}
    for p in paths:
        b = os.path.basename(p)
        fm = -int(b[3]) if b[3] != "_" else int(b[2])
        if fm != m:
            continue
        for l in range(max(2, abs(m)), abs(m) + mmax + 1):
            want[l] = (p, 1 + 2 * (l - abs(m)))
    missing = [l for l in range(max(2, abs(m)), abs(m) + mmax + 1) if l not in want]
    if missing:
        raise ValueError(f"no waveform file for m={m}, l={missing}")
    return want


def _read_waveform(path: str) -> np.ndarray:
    # the first line of a waveform file is taken as a header (ringdownlib.py:102)
    return np.loadtxt(path, skiprows=1, ndmin=2)


def _uniform(d: np.ndarray, col: int) -> Tuple[np.ndarray, np.ndarray]:
    """The column on the file's own uniform grid t0 + k (t1 - t0) (ringdownlib.py:103-113)."""
    step = d[1, 0] - d[0, 0]
    t = np.arange(d[0, 0], d[-1, 0], step)
    return t, np.interp(t, d[:, 0], d[:, col])


def system_matrix(tables: Tables, m: int, mmax: int, a: float) -> Tuple[np.ndarray, np.ndarray]:
    """(mu, w): the time-independent factors of the linear system, rows
    [h_l for l..., dh_l/dt for l...], columns [(l', +|m|), (l', -|m|) for
    l'...] ((l', 0), (-l', 0) for m = 0), Extract_Ringdown_MoreModes.py:13-78."""
    am = abs(m)
    ls = list(range(max(2, am), am + mmax + 1))
    rows = [(l, d) for d in (0, 1) for l in ls]
    cols = [(l, s) for l in ls for s in (am, -am)]
    if m == 0:
        cols = [(l * (-1) ** i, s) for i, (l, s) in enumerate(cols)]
    n = len(rows)
    mu = np.zeros((n, n), dtype=complex)
    w = np.zeros((n, n), dtype=complex)
    for j, (lp, mp) in enumerate(cols):
        co = mp * m > 0 or (m == 0 and lp > 0)
        om = tables.qnm(abs(lp), mp, 0, a)
        wr, wi = (om.real if (m != 0 or lp > 0) else -om.real), abs(om.imag)
        w_j = (-1j * wr - wi) if (mp * m > 0 or m == 0) else (1j * wr - wi)
        for i, (lv, der) in enumerate(rows):
            re, im = tables.overlap(mp, lv, abs(lp), 0, a)
            v = complex(re, -im) if co else (-1) ** lv * complex(re, im)
            if der:
                v *= w_j
            mu[i, j] = v
            w[i, j] = w_j
    return mu, w


@dataclass
class SpheroidalFit:
    m: int
    modes: List[int]          # l = max(2,|m|)..|m|+mmax
    time: np.ndarray          # solution times
    coeffs: np.ndarray        # [time, 2 * len(modes)]: (l', +|m|), (l', -|m|) pairs
    t_lr: float


def spheroidal_coefficients(tables: Tables, wave_paths: Sequence[str], traj_rows: np.ndarray, a: float, m: int,
                            mmax: int) -> SpheroidalFit:
    """Spheroidal amplitudes of mode m at every 0.1 M from 50 M before the
    light-ring crossing (Extract_Ringdown_MoreModes.py:94-181)."""
    t_lr = light_ring_crossing(traj_rows, a)
    files = mode_files(wave_paths, m, mmax)
    ls = sorted(files)
    cache: Dict[str, np.ndarray] = {}
    series = []
    for l in ls:
        path, col = files[l]
        if path not in cache:
            cache[path] = _read_waveform(path)
        d = cache[path]
        t, hp = _uniform(d, col)
        _, hc = _uniform(d, col + 1)
        series.append((t, hp, hc))
    t_file = series[0][0]
    for t, _, _ in series[1:]:
        if abs(np.sum(t_file - t)) >= 1e-10:
            raise ValueError("waveform files are on different time grids")
    tg = np.arange(t_file[0], t_file[-1], 0.1)
    step = tg[1] - tg[0]
    start = int(np.searchsorted(tg, t_lr - 50.0, side="left"))
    h = np.stack([np.interp(tg, t_file, hp)[start:-1] - 1j * np.interp(tg, t_file, hc)[start:-1]
                  for _, hp, hc in series])
    dh = np.stack([np.gradient(x, step) for x in h])
    rhs = np.concatenate([h, dh]).T                     # [time, 2 nmodes]
    ts = tg[start:-1]
    mu, w = system_matrix(tables, m, mmax, a)
    A = mu[None, :, :] * np.exp(w[None, :, :] * (ts[:, None, None] - t_lr))
    coeffs = np.stack([np.linalg.solve(A[k], rhs[k]) for k in range(len(ts))])
    return SpheroidalFit(m=m, modes=ls, time=ts, coeffs=coeffs, t_lr=t_lr)


def spheroidal_file_name(m: int, a: float, thinc: int, thf: str) -> str:
    return f"spheroidal_coefficients_{m_label(m)}_a{('%.2f' % a)[-2:]}_thinc{thinc:03d}_thf{thf}.out"


def write_spheroidal(fit: SpheroidalFit, out_dir: str, a: float, thinc: int, thf: str) -> str:
    """The reference's .out file (Extract_Ringdown_MoreModes.py:183-209)."""
    path = os.path.join(out_dir, spheroidal_file_name(fit.m, a, thinc, thf))
    lines = ["#[0] time"]
    for i, l in enumerate(fit.modes):
        lines += [f"#[{4 * i + 1}] realamp_l{l}{m_label(fit.m)}", f"#[{4 * i + 2}] imagamp_l{l}{m_label(fit.m)}",
                  f"#[{4 * i + 3}] realamp_l{l}{m_label(-fit.m)}", f"#[{4 * i + 4}] imagamp_l{l}{m_label(-fit.m)}"]
    body = []
    for t, row in zip(fit.time, fit.coeffs):
        body.append("%.2f" % t + "".join("\t%.5e\t%.5e" % (float(c.real), float(c.imag)) for c in row))
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n" + "\n".join(body) + ("\n" if body else ""))
    return path


@dataclass
class Excitation:
    thf: float
    sign: str                 # "n" or "p": the sign of theta-dot at the end of the trajectory
    amp: np.ndarray           # [2 nmodes]
    phase: np.ndarray         # [2 nmodes], in [0, 2 pi)
    window: Tuple[float, float]


def excitation_coefficients(time: np.ndarray, coeffs_reim: np.ndarray, thf: float, sign: str,
                            window: float = 50.0, search: float = 250.0) -> Excitation:
    """Amplitudes and phases over the steadiest window (Postprocess.py:45-119).
    coeffs_reim: [time, 2 * nunknowns] as the .out file holds them (re, im)."""
    re, im = coeffs_reim[:, 0::2].T, coeffs_reim[:, 1::2].T
    amp = np.sqrt(re ** 2 + im ** 2)
    ang = np.unwrap(np.angle(re + 1j * im))
    best = (np.inf, None)
    i = 0
    t_hi = 0.0
    while t_hi < min(time[-1], time[0] + search):
        t_lo = time[i]
        t_hi = t_lo + window
        hit = np.nonzero(np.abs(time - t_hi) < 1e-10)[0]
        if len(hit) != 1:
            raise ValueError(f"no single sample at t = {t_hi}")
        j = int(hit[0])
        mean = np.mean(amp[:, i:j], axis=1)
        score = np.sum(np.std(amp[:, i:j], axis=1) / mean)
        if score < best[0]:
            best = (score, (mean, np.mean(ang[:, i:j], axis=1) % (2 * np.pi), (t_lo, t_hi)))
        i += 1
    mean, phase, win = best[1]
    return Excitation(thf=thf, sign=sign, amp=mean, phase=phase, window=win)


def parse_spheroidal_name(name: str) -> Tuple[float, str]:
    """(theta_f, sign) from ..._thf<deg>_<n|p>.out (Postprocess.py:51-53)."""
    parts = name.split("_")
    return float(parts[-2][3:]), parts[-1][0]


def write_excitation(results: Sequence[Excitation], m: int, nmodes: int, out_dir: str, a: float, thinc: int,
                     modes: Sequence[int]) -> str:
    """The reference's excitation_coefficients file (Postprocess.py:121-164):
    the negative-sign rows, then the positive-sign ones; an equatorial start
    (thinc 0 or 180) puts each result in both."""
    neg = [r for r in results if r.sign == "n" or (r.sign == "p" and thinc in (0, 180))]
    pos = [r for r in results if r.sign == "p" or (r.sign == "n" and thinc in (0, 180))]
    pos_sfx, neg_sfx = ("", "prime") if m >= 0 else ("prime", "")
    head = ["#[0] thetafin", "#[1] sign_thetafindot"]
    for i, l in enumerate(modes):
        head += [f"#[{4 * i + 2}] l{l}{m_label(abs(m))}{pos_sfx}_amp", f"#[{4 * i + 3}] l{l}{m_label(abs(m))}{pos_sfx}_phase",
                 f"#[{4 * i + 4}] l{l}{m_label(-abs(m))}{neg_sfx}_amp",
                 f"#[{4 * i + 5}] l{l}{m_label(-abs(m))}{neg_sfx}_phase"]
    rows = []
    for sgn, group in ((-1, neg), (1, pos)):
        for r in group:
            rows.append("%.2f\t%d" % (r.thf, sgn) + "".join("\t%.4e\t%.4e" % (x, y) for x, y in zip(r.amp, r.phase)))
    path = os.path.join(out_dir, f"excitation_coefficients_a{('%.2f' % a)[-2:]}_thinc{thinc:03d}_h{m_label(m)}.dat")
    with open(path, "w") as f:
        f.write("\n".join(head) + "\n" + "".join(row + "\n" for row in rows))
    return path
