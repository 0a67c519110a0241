"""Quasinormal-mode checks of solver waveforms.

* Kerr frequency tables in the reference's format (QNM_Extraction/Tables/
  kerr/n<n+1>l<l>m<m>.dat: a, Re omega, Im omega, ...), read and linearly
  interpolated in a as QNM_Extraction/Library/ringdownlib.py:149-161
  (loadqnmtable) does; a committed excerpt of them serves the tests.
* A least-squares ringdown fit: the complex waveform h = h_plus - i h_cross
  of one (l, m) column is modelled over [t0, t1] as
      h(t) = sum_k A_k exp(-i omega_k (t - t0)) + c_0 + c_1 (t - t0),
  the polynomial absorbing the integration constants of the twice
  time-integrated field the solver projects.  The model is linear in A_k
  and c_j, so for given frequencies they come from a linear least-squares
  solve (variable projection) and only the omega_k are iterated.
"""
from __future__ import annotations

import os
from typing import Dict, Iterable, Optional, Sequence, Tuple

import numpy as np

FIXTURE = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "tests", "golden",
                       "kerr_qnm.txt")


def load_table(path: str = FIXTURE) -> Dict[Tuple[int, int, int], np.ndarray]:
    """{(l, m, n): array of rows (a, Re omega, Im omega)} from the excerpt
    file (columns l m n a Re Im)."""
    d = np.loadtxt(path, comments="#")
    out: Dict[Tuple[int, int, int], list] = {}
    for l, m, n, a, wr, wi in d:
        out.setdefault((int(l), int(m), int(n)), []).append((a, wr, wi))
    return {k: np.array(v) for k, v in out.items()}


def load_reference_table(qnm_dir: str, l: int, m: int, n: int) -> np.ndarray:
    """Rows (a, Re omega, Im omega) of one reference table file."""
    name = f"n{n + 1}l{l}m{m}.dat" if m >= 0 else f"n{n + 1}l{l}mm{-m}.dat"
    return np.loadtxt(os.path.join(qnm_dir, name), usecols=(0, 1, 2))


def frequency(table: Dict[Tuple[int, int, int], np.ndarray], l: int, m: int, n: int, a: float) -> complex:
    """Kerr omega_{lmn}(a), linear in a between table rows; for a < 0 the
    (l, -m) table at -a (the reference's sign convention)."""
    if a < 0:
        m, a = -m, -a
    rows = table[(l, m, n)]
    return complex(np.interp(a, rows[:, 0], rows[:, 1]), np.interp(a, rows[:, 0], rows[:, 2]))


def _basis(tau: np.ndarray, omegas: Sequence[complex], npoly: int) -> np.ndarray:
    cols = [np.exp(-1j * w * tau) for w in omegas] + [tau.astype(complex) ** j for j in range(npoly)]
    return np.stack(cols, axis=1)


def fit(t: np.ndarray, h: np.ndarray, guess: Iterable[complex], t0: float, t1: float, npoly: int = 2,
        fix: Optional[Sequence[bool]] = None):
    """Fits h over [t0, t1] (h complex, sampled at t).  Returns
    (omegas, amplitudes at t0, polynomial coefficients, relative residual).
    `fix[k]` keeps omega_k at its guess."""
    from scipy.optimize import least_squares

    sel = (t >= t0) & (t <= t1)
    tau, y = t[sel] - t0, h[sel]
    guess = [complex(w) for w in guess]
    fix = [False] * len(guess) if fix is None else list(fix)
    free = [k for k in range(len(guess)) if not fix[k]]
    scale = np.linalg.norm(y)

    def omegas_of(x):
        w = list(guess)
        for i, k in enumerate(free):
            w[k] = complex(x[2 * i], x[2 * i + 1])
        return w

    def resid(x):
        B = _basis(tau, omegas_of(x), npoly)
        c, *_ = np.linalg.lstsq(B, y, rcond=None)
        r = (B @ c - y) / scale
        return np.concatenate([r.real, r.imag])

    x0 = np.array([v for k in free for v in (guess[k].real, guess[k].imag)])
    sol = least_squares(resid, x0, method="lm", xtol=1e-15, ftol=1e-15, gtol=1e-15, max_nfev=20000)
    w = omegas_of(sol.x)
    B = _basis(tau, w, npoly)
    c, *_ = np.linalg.lstsq(B, y, rcond=None)
    rel = np.linalg.norm(B @ c - y) / scale
    K = len(guess)
    return np.array(w), c[:K], c[K:], float(rel)


def complex_waveform(h14: np.ndarray, l_index: int = 0) -> np.ndarray:
    """h_plus - i h_cross of column pair l_index (l = |m| + l_index) of the
    solver's 14 waveform columns."""
    return h14[:, 2 * l_index] - 1j * h14[:, 2 * l_index + 1]
