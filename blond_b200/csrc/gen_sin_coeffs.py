"""Coefficients of the FP64 RF sine's and cosine's polynomials (rf_sin and
rf_sincos in common.cuh).

sin(r) on [-pi/2, pi/2] is written r + r^3 P(r^2).  P is the degree-7
Chebyshev approximation (mpmath.chebyfit: interpolation at Chebyshev
nodes, near-minimax; J. C. Mason and D. C. Handscomb, "Chebyshev
Polynomials", 2003, ch. 6) of g(u) = (sin(sqrt u) - sqrt u) / u^(3/2) on
u in [0, (pi/2)^2], computed at 60 significant digits and rounded to
double.  Its approximation error in sin is below 1.3e-18; evaluated in
double by Horner's rule with fused multiply-adds, the result is within 2
units in the last place of sin(r) (checked here with exact fma
emulation), as the Taylor polynomial through r^21 it replaces was, with two
fewer terms.  The cosine (for the adjoint's derivatives) is 1 + r^2 Q(r^2),
Q the degree-8 Chebyshev approximation of (cos(sqrt u) - 1) / u (error
below 3e-20; 1.6e-16 absolute in double).  Run with mpmath installed;
prints the coefficients, highest degree first.
"""
import math
import random
from fractions import Fraction

import mpmath as mp


def coefficients(degree: int = 7):
    mp.mp.dps = 60

    def g(u):
        if u == 0:
            return mp.mpf(-1) / 6
        s = mp.sqrt(u)
        return (mp.sin(s) - s) / (u * s)

    poly, err = mp.chebyfit(g, [0, (mp.pi / 2) ** 2], degree + 1, error=True)
    return [float(c) for c in poly], float(err * (mp.pi / 2) ** 3)


def _fma(a, b, c):
    return float(Fraction(a) * Fraction(b) + Fraction(c))


def evaluate(r: float, co) -> float:
    r2 = float(Fraction(r) * Fraction(r))
    p = co[0]
    for c in co[1:]:
        p = _fma(p, r2, c)
    return _fma(float(Fraction(r) * Fraction(r2)), p, r)


def cos_coefficients(degree: int = 7):
    """cos(r) = 1 + r^2 Q(r^2) on [-pi/2, pi/2]: Q the degree-`degree`
    Chebyshev approximation of (cos(sqrt u) - 1) / u on [0, (pi/2)^2]."""
    mp.mp.dps = 60

    def h(u):
        if u == 0:
            return mp.mpf(-1) / 2
        return (mp.cos(mp.sqrt(u)) - 1) / u

    poly, err = mp.chebyfit(h, [0, (mp.pi / 2) ** 2], degree + 1, error=True)
    return [float(c) for c in poly], float(err * (mp.pi / 2) ** 2)


def evaluate_cos(r: float, co) -> float:
    r2 = float(Fraction(r) * Fraction(r))
    p = co[0]
    for c in co[1:]:
        p = _fma(p, r2, c)
    return _fma(r2, p, 1.0)


if __name__ == "__main__":
    co, bound = coefficients()
    print("approximation error bound:", bound)
    for c in co:
        print(repr(c))
    random.seed(7)
    pts = [random.uniform(-math.pi / 2, math.pi / 2) for _ in range(20000)]
    worst = max(abs(evaluate(r, co) - float(mp.sin(r))) / math.ulp(float(mp.sin(r)))
                for r in pts if r != 0.0)
    print("max error over 20000 points (ulps):", worst)
    fco, fbound = coefficients(4)
    print("float sine (degree 4 in r^2): approximation error bound:", fbound)
    for c in fco:
        print(repr(float(__import__("numpy").float32(c))))
    cco, cbound = cos_coefficients(8)
    print("cosine: approximation error bound:", cbound)
    for c in cco:
        print(repr(c))
    worst = max(abs(evaluate_cos(r, cco) - float(mp.cos(r))) for r in pts)
    print("max absolute error over 20000 points:", worst)
