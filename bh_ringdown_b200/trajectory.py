"""Trajectory files: the 10-column .traj format and a geodesic plunge.

The reference takes its source worldline from GenOT
(GenOT/README:113-123: columns t r theta dr/dt dtheta/dt dphi/dt phi E Lz
Q); bh_ringdown_b200.genot restates GenOT and makes the workloads'
worldlines.  `synthetic_plunge` here is a simpler worldline for tests: a
prograde equatorial Kerr geodesic that starts just inside the ISCO with the
ISCO energy and angular momentum and plunges; it is integrated in
Boyer-Lindquist time with the 8th-order Dormand-Prince method (scipy's
DOP853, dense output) and sampled on a uniform time grid (body.cu consumes
two rows per step, so a run with step dt wants rows every dt/2).
"""
from __future__ import annotations

import numpy as np


def read_traj(path: str) -> np.ndarray:
    rows = np.loadtxt(path, dtype=np.float64, ndmin=2)
    if rows.shape[1] != 10:
        raise ValueError(f"{path}: expected 10 columns, found {rows.shape[1]}")
    return rows


def write_traj(path: str, rows: np.ndarray) -> None:
    np.savetxt(path, rows, fmt="%.18e")


def isco_prograde(a: float, mass: float = 1.0):
    """ISCO radius, specific energy and angular momentum (Bardeen, Press,
    Teukolsky 1972) for prograde equatorial orbits."""
    a = a / mass
    z1 = 1 + (1 - a * a) ** (1 / 3) * ((1 + a) ** (1 / 3) + (1 - a) ** (1 / 3))
    z2 = np.sqrt(3 * a * a + z1 * z1)
    r = 3 + z2 - np.sqrt((3 - z1) * (3 + z1 + 2 * z2))
    v = 1 / np.sqrt(r)
    den = np.sqrt(1 - 3 * v * v + 2 * a * v ** 3)
    E = (1 - 2 * v * v + a * v ** 3) / den
    L = np.sqrt(r) * (1 - 2 * a * v ** 3 + a * a * v ** 4) / den
    return r * mass, E, L * mass


def _rhs(y, a, E, L):
    """d/dt of (r, phi) on an equatorial plunge (M = 1), r decreasing."""
    r = y[0]
    D = r * r - 2 * r + a * a
    P = E * (r * r + a * a) - a * L
    R = P * P - D * (r * r + (L - a * E) ** 2)
    tdot = ((r * r + a * a) / D * P - a * (a * E - L)) / (r * r)
    phidot = (a / D * P - (a * E - L)) / (r * r)
    rdot = -np.sqrt(max(R, 0.0)) / (r * r)
    return np.array([rdot / tdot, phidot / tdot])


def synthetic_plunge(a: float, dt_row: float, duration: float, r_offset: float = 0.05,
                     r_stop_above_horizon: float = 0.02) -> np.ndarray:
    """Rows of a prograde equatorial plunge starting at r_isco - r_offset.

    Sampled every dt_row in BL time for `duration`, or until r comes within
    r_stop_above_horizon of r+; after that the file simply ends (a reader
    past the end keeps the last row, as the reference's fscanf loop does).
    """
    from scipy.integrate import solve_ivp

    r_isco, E, L = isco_prograde(a)
    r_plus = 1 + np.sqrt(1 - a * a)
    n = int(np.floor(duration / dt_row)) + 1
    t_rows = np.arange(n) * dt_row
    # Dense output of an 8th-order Dormand-Prince integration (relative
    # tolerance 1e-13), sampled at the row times.
    # The integration ends where r reaches r+ + r_stop_above_horizon / 2,
    # past the last row kept.
    def near_horizon(t, y):
        return y[0] - (r_plus + 0.5 * r_stop_above_horizon)

    near_horizon.terminal = True
    sol = solve_ivp(lambda t, y: _rhs(y, a, E, L), (0.0, t_rows[-1] if n > 1 else dt_row),
                    np.array([r_isco - r_offset, 0.0]), method="DOP853", rtol=1e-13, atol=1e-13,
                    dense_output=True, events=near_horizon)
    t_rows = t_rows[t_rows <= sol.t[-1]]
    n = len(t_rows)
    y = sol.sol(t_rows)
    rows = []
    for i in range(n):
        r, phi = y[0, i], y[1, i]
        if r < r_plus + r_stop_above_horizon:
            break
        rdot, phidot = _rhs((r, phi), a, E, L)
        rows.append((t_rows[i], r, np.pi / 2, rdot, 0.0, phidot, phi, E, L, 0.0))
    return np.array(rows, dtype=np.float64)
