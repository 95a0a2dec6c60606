"""SU(2) recoupling coefficients for the host planner, exact rational arithmetic.

The reference obtains these from the ``racah`` crate (racah-py 0.1.1) at Dynkin label
``(two_j,)`` (``symmetry/_sun_coeff.py:75-112``, ``symmetry/su2.py:174-252``).  The
planner needs them once per structure, on the host, so they are computed here from the
published closed forms and cached:

* 6j symbols by Racah's single-sum formula, summed exactly over integers;
* ``[F^{abc}_d]_{e,f} = (-1)^(a+b+c+d) sqrt((2e+1)(2f+1)) {a b e; c d f}`` -- the
  TensorKitSectors ``SU2Irrep`` gauge the reference's fixtures pin;
* ``R^{ab}_c = (-1)^(ja+jb-jc)``;
* ``B^{ab}_c = sqrt(d_a d_b / d_c) [F^{a b b}_a]_{c,0}``;
* ``chi_a = (-1)^(2j)`` (the sign of ``[F^{a a a}_a]_{0,0}``).

Spins are doubled (``two_j``) so every label is an int.  Values are correctly rounded
up to the single final square root.
"""

from __future__ import annotations

from fractions import Fraction
from functools import cache
from math import sqrt

_FACT = [1]


def _fact(n: int) -> int:
    while len(_FACT) <= n:
        _FACT.append(_FACT[-1] * len(_FACT))
    return _FACT[n]


def triangle(a: int, b: int, c: int) -> bool:
    return abs(a - b) <= c <= a + b and not (a + b + c) & 1


def _tri2(a: int, b: int, c: int) -> Fraction:
    """Delta(abc)^2 = (a+b-c)!(a-b+c)!(-a+b+c)! / (a+b+c+1)!, doubled spins."""
    return Fraction(_fact((a + b - c) >> 1) * _fact((a - b + c) >> 1) * _fact((b + c - a) >> 1),
                    _fact(((a + b + c) >> 1) + 1))


@cache
def wigner_6j(a: int, b: int, c: int, d: int, e: int, f: int) -> float:
    if not (triangle(a, b, c) and triangle(a, e, f) and triangle(d, b, f) and triangle(d, e, c)):
        return 0.0
    alphas = ((a + b + c) >> 1, (a + e + f) >> 1, (d + b + f) >> 1, (d + e + c) >> 1)
    betas = ((a + b + d + e) >> 1, (b + c + e + f) >> 1, (a + c + d + f) >> 1)
    s = Fraction(0)
    for z in range(max(alphas), min(betas) + 1):
        den = 1
        for x in alphas:
            den *= _fact(z - x)
        for y in betas:
            den *= _fact(y - z)
        s += Fraction(-_fact(z + 1) if z & 1 else _fact(z + 1), den)
    if s == 0:
        return 0.0
    mag = sqrt(float(s * s * _tri2(a, b, c) * _tri2(a, e, f) * _tri2(d, b, f) * _tri2(d, e, c)))
    return mag if s > 0 else -mag


@cache
def f_symbol(a: int, b: int, c: int, d: int, e: int, f: int) -> float:
    if not (triangle(a, b, e) and triangle(e, c, d) and triangle(b, c, f) and triangle(a, f, d)):
        return 0.0
    v = sqrt((e + 1) * (f + 1)) * wigner_6j(a, b, e, c, d, f)
    return -v if ((a + b + c + d) >> 1) & 1 else v


def r_symbol(a: int, b: int, c: int) -> int:
    if not triangle(a, b, c):
        return 0
    return -1 if ((a + b - c) >> 1) & 1 else 1


@cache
def b_symbol(a: int, b: int, c: int) -> float:
    if not triangle(a, b, c):
        return 0.0
    return sqrt((a + 1) * (b + 1) / (c + 1)) * f_symbol(a, b, b, a, c, 0)


def frobenius_schur(a: int) -> int:
    return -1 if a & 1 else 1
