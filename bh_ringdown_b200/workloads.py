"""Seeded request sets for the batched and served forms of the solver.

* ``batch_requests``: source-free solves of mixed size and physics (spin a
  uniform in [0, 0.99], m in {1..4}, N_r in {2048, 4096, 8192, 16384},
  N_theta in {64, 128, 256}, Gaussian pulse centre uniform in [10, 40] and
  width in [1, 4] times the s=-2 harmonic with l = max(2, |m|); x in
  [-100, 300], T = 500, waveform every 0.5 at the column nearest x = 250).
* ``serve_requests``: a Poisson request stream, 70 % source-free solves
  (N_r in {2048, 4096}, N_theta in {64, ..., 128}, a in [0, 0.99]) and 30 %
  plunge-driven solves (a in [0, 0.95], 8192 x 128 on [-200, 600], T = 1000,
  source from GenOT's transition-to-plunge worldline, prograde equatorial,
  mass ratio 1e-3, from the ISCO).

There is no public request log for this solver: these are synthetic
stand-ins with the sizes and value ranges above.  ``time_scale`` shortens
every request's final time T (and with it its step count) so that a
bounded sample of the stream runs in minutes; callers state the scale they
used.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List, Optional

import numpy as np

from . import BHR_FP64, BHR_INIT_GAUSSIAN, Params
from .genot import transition_plunge

SEED = 20261203


@dataclass
class Request:
    params: Params
    traj: Optional[np.ndarray]
    arrival_s: float = 0.0
    kind: str = "free"

    def points(self) -> int:
        return self.params.N * self.params.M


def _free(rng, N, M, a, m, T, Xmin=-100.0, Xmax=300.0, x_ext=250.0, precision=BHR_FP64):
    c, w = rng.uniform(10.0, 40.0), rng.uniform(1.0, 4.0)
    dx = (Xmax - Xmin) / N
    return Params(N=int(N), M=int(M), Xmin=Xmin, Xmax=Xmax, a=float(a), m=float(m), dt=0.0, courant=0.25,
                  out_every=0.5, Fr=0, T=T, out_start=0.0, ext_col=int(round((x_ext - Xmin) / dx)),
                  init_kind=BHR_INIT_GAUSSIAN, init_center=c, init_width=w, init_ell=float(max(2, abs(m))),
                  precision=precision)


def batch_requests(n: int = 64, seed: int = SEED, T: float = 500.0, precision: int = BHR_FP64) -> List[Request]:
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        a = rng.uniform(0.0, 0.99)
        m = int(rng.integers(1, 5))
        N = int(rng.choice([2048, 4096, 8192, 16384]))
        M = int(rng.choice([64, 128, 256]))
        out.append(Request(_free(rng, N, M, a, m, T, precision=precision), None))
    return out


def plunge_params(a: float, T: float, N: int = 8192, M: int = 128, Xmin: float = -200.0, Xmax: float = 600.0,
                  x_ext: float = 500.0, precision: int = BHR_FP64) -> Params:
    """Plunge-driven solve; dt = 0.25 min(dx, r_min dtheta) as the waveform
    rows are every Fr = 50 steps."""
    from . import grid
    prm = Params(N=N, M=M, Xmin=Xmin, Xmax=Xmax, a=a, m=2.0, dt=0.0, courant=0.25, Fr=50, T=T, out_start=0.0,
                 precision=precision)
    _, r, _ = grid(prm)
    dx = (Xmax - Xmin) / N
    prm.dt = 0.25 * min(dx, r[0] * np.pi / M)
    prm.ext_col = int(round((x_ext - Xmin) / dx))
    return prm


def serve_requests(n: int = 2000, rate_per_s: float = 1.0, seed: int = SEED, time_scale: float = 1.0,
                   plunge_fraction: float = 0.3, precision: int = BHR_FP64) -> List[Request]:
    """n requests with exponential inter-arrival times of mean 1/rate_per_s."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    trajs = {}
    for _ in range(n):
        t += rng.exponential(1.0 / rate_per_s)
        if rng.uniform() < plunge_fraction:
            a = max(1e-8, round(float(rng.uniform(0.0, 0.95)), 2))  # trajectories shared per 0.01 in a
            prm = plunge_params(a, 1000.0 * time_scale, precision=precision)
            key = (a, prm.dt)
            if key not in trajs:
                trajs[key] = transition_plunge(a, 1e-3, prm.dt / 2.0, prm.T)
            out.append(Request(prm, trajs[key], t, "plunge"))
        else:
            a = rng.uniform(0.0, 0.99)
            m = int(rng.integers(1, 5))
            N = int(rng.choice([2048, 4096]))
            M = int(rng.choice([64, 80, 96, 112, 128]))
            out.append(Request(_free(rng, N, M, a, m, 500.0 * time_scale, precision=precision), None, t, "free"))
    return out


def with_arrivals(reqs: List[Request], rate_per_s: float, seed: int = SEED + 1) -> List[Request]:
    """Re-times a request list as a Poisson stream of the given rate."""
    rng = np.random.default_rng(seed)
    t = 0.0
    for r in reqs:
        t += rng.exponential(1.0 / rate_per_s)
        r.arrival_s = t
    return reqs
