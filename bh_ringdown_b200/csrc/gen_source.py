"""Generate bhr_source_gen.inc: the particle-only coefficients of the
point-particle source of the s=-2 Teukolsky equation, mode m.

Derivation (sympy, run once; the output is committed):

* Source term of the Teukolsky master equation (Teukolsky 1973, ApJ 185,
  635, eqs. 2.15 and 4.7): 4 pi Sigma T with T = 2 rho^-4 T_4 and
    T_4 = (D_n + 3g - g* + 4u + u*) [ (D_m* - 2t* + 2al) T_nm* - (D_n + g - g* + u) T_m*m* ]
        + (D_m* - t* + b* + 3al + 4pi) [ (D_n + 2g + 2u*) T_nm* - (D_m* - t* + 2b* + 2al) T_nn ]
  in the Kinnersley tetrad (D_n = n^mu d_mu, D_m* = mbar^mu d_mu; g, u,
  t, al, b, pi the spin coefficients gamma, mu, tau, alpha, beta, pi;
  * = complex conjugate).  The factor in front of T_m*m* carries mu, not
  mu*: that is the form whose output the reference's source has
  (HighOrder/kern.cu:1229-2664), and the one this solver must reproduce.
* Point particle: T^{ab} = mu_p u^a u^b / (Sigma sin(theta) u^t)
  delta(r - rp(t)) delta(theta - thp(t)) delta(phi - php(t)), with
  u_t = -E, u_phi = Lz, Sigma u^t from E and Lz, u^r = u^t dr/dt and
  u^theta = u^t dtheta/dt.  Mode m of delta(phi - php) is
  exp(-i m php)/(2 pi); d/dphi acts as i m.
* The operators act on the distribution; time derivatives of the
  worldline enter through the chain rule (rp, thp, php as cubic Taylor
  polynomials in t around the current time, so their first three
  derivatives are the inputs drdt..d3thdt3).  Every grid-point function is
  then moved onto the particle with
    f(r) delta^(n)(r - rp) = sum_k C(n,k) (-1)^k f^(k)(rp) delta^(n-k)(r - rp),
  leaving T_4 = sum C_ij delta^(i)(r - rp) delta^(j)(theta - thp) with
  particle-only C_ij for (i,j) in (0,0) (0,1) (0,2) (1,0) (1,1) (2,0).

Usage: python bh_ringdown_b200/csrc/gen_source.py  (writes bhr_source_gen.inc)
"""
from __future__ import annotations

import os
import sys
import time

import sympy as sp
from sympy.printing.c import C99CodePrinter

HERE = os.path.dirname(os.path.abspath(__file__))
ORDER = [(0, 0), (0, 1), (0, 2), (1, 0), (1, 1), (2, 0)]


def derive():
    t, r, th = sp.symbols("t r theta", real=True)
    a, Mm, m, mu = sp.symbols("a mass m nmu", real=True)
    E, L = sp.symbols("E lz", real=True)
    rp0, tp0 = sp.symbols("rp tp", positive=True)
    drdt, d2rdt2, d3rdt3, dthdt, d2thdt2, d3thdt3, dphidt, d2phidt2 = sp.symbols(
        "drdt d2rdt2 d3rdt3 dthdt d2thdt2 d3thdt3 dphidt d2phidt2", real=True)
    I = sp.I
    sq2 = sp.sqrt(2)

    def conj(e):
        return e.subs(I, -I)

    rp = rp0 + drdt * t + d2rdt2 * t ** 2 / 2 + d3rdt3 * t ** 3 / 6
    thp = tp0 + dthdt * t + d2thdt2 * t ** 2 / 2 + d3thdt3 * t ** 3 / 6
    phdot = dphidt + d2phidt2 * t
    rdot, thdot = sp.diff(rp, t), sp.diff(thp, t)

    cth, sth = sp.cos(th), sp.sin(th)
    Sig = r ** 2 + a ** 2 * cth ** 2
    Del = r ** 2 - 2 * Mm * r + a ** 2
    rho = -1 / (r - I * a * cth)
    rhob = -1 / (r + I * a * cth)
    beta = -rhob * sp.cot(th) / (2 * sq2)
    betab = conj(beta)
    piS = I * a * rho ** 2 * sth / sq2
    tau = -I * a * rho * rhob * sth / sq2
    taub = conj(tau)
    muS = rho ** 2 * rhob * Del / 2
    mub = conj(muS)
    gam = muS + rho * rhob * (r - Mm) / 2
    gamb = conj(gam)
    alpha = piS - betab
    n_t, n_r, n_ph = (r ** 2 + a ** 2) / (2 * Sig), -Del / (2 * Sig), a / (2 * Sig)
    mb_t = -I * a * sth / (sq2 * (r - I * a * cth))
    mb_th = 1 / (sq2 * (r - I * a * cth))
    mb_ph = -I / (sth * sq2 * (r - I * a * cth))

    def add(d, k, v):
        d[k] = d.get(k, 0) + v

    def dT(X):
        out = {}
        for (i, j), c in X.items():
            add(out, (i, j), sp.diff(c, t) + c * (-I * m * phdot))
            add(out, (i + 1, j), -c * rdot)
            add(out, (i, j + 1), -c * thdot)
        return out

    def dR(X):
        out = {}
        for (i, j), c in X.items():
            add(out, (i, j), sp.diff(c, r))
            add(out, (i + 1, j), c)
        return out

    def dTH(X):
        out = {}
        for (i, j), c in X.items():
            add(out, (i, j), sp.diff(c, th))
            add(out, (i, j + 1), c)
        return out

    def lin(*terms):
        out = {}
        for f, X in terms:
            for k, v in X.items():
                add(out, k, f * v)
        return out

    def Dn(X):
        return lin((n_t, dT(X)), (n_r, dR(X)), (n_ph * I * m, X))

    def Dmb(X):
        return lin((mb_t, dT(X)), (mb_th, dTH(X)), (mb_ph * I * m, X))

    def op(D, f):
        return lambda X: lin((1, D(X)), (f, X))

    cthp, sthp = sp.cos(thp), sp.sin(thp)
    Sigp = rp ** 2 + a ** 2 * cthp ** 2
    Delp = rp ** 2 - 2 * Mm * rp + a ** 2
    tS = E * ((rp ** 2 + a ** 2) ** 2 / Delp - a ** 2 * sthp ** 2) + a * L * (1 - (rp ** 2 + a ** 2) / Delp)
    Pn = E * (rp ** 2 + a ** 2) + rdot * tS - a * L
    Pm = I * sthp * (a * E - L / sthp ** 2) + thdot * tS
    un = -Pn / (2 * Sigp)
    umb = Pm / (sq2 * (rp - I * a * cthp))
    den = sthp * tS
    Tnn = {(0, 0): mu * un * un / den}
    Tnmb = {(0, 0): mu * un * umb / den}
    Tmbmb = {(0, 0): mu * umb * umb / den}

    A1 = op(Dn, 3 * gam - gamb + 4 * muS + mub)
    B1 = op(Dmb, -2 * taub + 2 * alpha)
    B2 = op(Dn, gam - gamb + muS)
    A2 = op(Dmb, -taub + betab + 3 * alpha + 4 * piS)
    B3 = op(Dn, 2 * gam + 2 * mub)
    B4 = op(Dmb, -taub + 2 * betab + 2 * alpha)
    T4 = lin((1, A1(lin((1, B1(Tnmb)), (-1, B2(Tmbmb))))), (1, A2(lin((1, B3(Tnmb)), (-1, B4(Tnn))))))

    coefs = []
    for key in ORDER:
        tot = 0
        for (i, j), c in T4.items():
            for k in range(i + 1):
                for l in range(j + 1):
                    if (i - k, j - l) != key:
                        continue
                    dc = c
                    if k:
                        dc = sp.diff(dc, r, k)
                    if l:
                        dc = sp.diff(dc, th, l)
                    v = sp.binomial(i, k) * sp.binomial(j, l) * (-1) ** (k + l) * dc
                    tot += v.subs({r: rp, th: thp}).subs(t, 0)
        coefs.append(tot)
    return coefs


class _Printer(C99CodePrinter):
    """C++ with std::complex<double>: integer literals printed as doubles,
    integer powers as ipow(), the imaginary unit as I_."""

    def _print_ImaginaryUnit(self, expr):
        return "I_"

    def _print_Integer(self, expr):
        return f"{int(expr)}.0"

    def _print_Pow(self, expr):
        b, e = expr.as_base_exp()
        if e.is_Integer:
            return f"ipow({self._print(b)}, {int(e)})"
        if e == sp.Rational(1, 2):
            return f"std::sqrt({self._print(b)})"
        if e == sp.Rational(-1, 2):
            return f"(1.0/std::sqrt({self._print(b)}))"
        return f"std::pow({self._print(b)}, {self._print(e)})"


def main():
    t0 = time.time()
    coefs = derive()
    print(f"derived in {time.time() - t0:.1f}s", file=sys.stderr)
    repl, red = sp.cse(coefs, symbols=sp.numbered_symbols("x"), optimizations="basic")
    print(f"cse: {len(repl)} subexpressions in {time.time() - t0:.1f}s", file=sys.stderr)
    pr = _Printer()
    lines = [
        "// Generated by bh_ringdown_b200/csrc/gen_source.py -- do not edit.",
        "// Particle-only coefficients of the s=-2 point-particle Teukolsky source",
        "// T_4 = sum_k C[k] delta^(i_k)(r - rp) delta^(j_k)(theta - tp),",
        "// (i,j) = (0,0) (0,1) (0,2) (1,0) (1,1) (2,0); without the exp(-i m phip)/(2 pi)",
        "// mode factor, which the caller applies.",
        "// Inputs: rp tp E lz drdt d2rdt2 d3rdt3 dthdt d2thdt2 d3thdt3 dphidt d2phidt2 a mass m nmu.",
    ]
    for s, e in repl:
        lines.append(f"const cplx {s} = {pr.doprint(e)};")
    for k, e in enumerate(red):
        lines.append(f"C[{k}] = {pr.doprint(e)};")
    with open(os.path.join(HERE, "bhr_source_gen.inc"), "w") as f:
        f.write("\n".join(lines) + "\n")
    print(f"wrote bhr_source_gen.inc in {time.time() - t0:.1f}s", file=sys.stderr)


if __name__ == "__main__":
    main()
