"""Oracle (test infrastructure only): SU(2) recoupling coefficients, exact arithmetic.

The reference takes its SU(2) F/R/B/Frobenius-Schur symbols and Clebsch-Gordan tensors
from the third-party Rust crate ``racah`` through its PyO3 wheel ``racah-py``, pinned at
0.1.1 (``uv.lock:1155-1156``).  That crate is not vendored in the reference tree, so this
module restates the published closed forms it implements at Dynkin label ``(two_j,)``:

* Wigner 6j symbol by Racah's single-sum formula (G. Racah, Phys. Rev. 62, 438 (1942));
* Clebsch-Gordan coefficients by Racah's formula in the Condon-Shortley phase, magnetic
  index descending (index ``k`` of ``V_j`` carries ``m = j - k``), the convention the
  reference states at ``symmetry/su2.py:57-68`` and ``su2.py:164-172``;
* the F-symbol in the TensorKitSectors ``SU2Irrep`` gauge,
  ``[F^{abc}_d]_{e,f} = (-1)^(a+b+c+d) sqrt((2e+1)(2f+1)) {a b e; c d f}``, pinned against
  the reference's vendored fixture ``tests/fixtures/su2_f.txt`` (109,900 rows, 2j <= 12,
  checked at 1e-13 by ``tests/symmetry/test_su2_recoupling.py:84-109``);
* ``R^{ab}_c = (-1)^(ja + jb - jc)`` (``symmetry/su2.py:206-218``), pinned against
  ``tests/fixtures/su2_r.txt``;
* ``B^{ab}_c = sqrt(d_a d_b / d_c) [F^{a b b}_a]_{c,0}`` (``symmetry/_sun_coeff.py:94-106``)
  and ``chi_a = sign([F^{a a a}_a]_{0,0})`` (``_sun_coeff.py:109-112``).

All sums are evaluated in exact rational arithmetic (Python integers and ``Fraction``) and
rounded to float once at the end, so every value is correctly rounded up to the final
square root.  Spins are doubled throughout (``two_j``), so every label is an int.

This module is imported only by the test suite, the golden-vector generator and the
CPU baseline; the shipped package computes its own coefficients.
"""

from __future__ import annotations

from fractions import Fraction
from functools import cache
from math import factorial, sqrt

__all__ = ["b_symbol", "cg", "cg_tensor", "f_symbol", "frobenius_schur", "r_symbol",
           "six_j", "triangle"]


def triangle(a: int, b: int, c: int) -> bool:
    """Doubled-spin triangle rule (``symmetry/su2.py:47-49``)."""
    return abs(a - b) <= c <= a + b and (a + b + c) % 2 == 0


def _delta2(a: int, b: int, c: int) -> Fraction:
    """Squared triangle coefficient Delta(abc)^2 for doubled spins."""
    return Fraction(
        factorial((a + b - c) // 2) * factorial((a - b + c) // 2) * factorial((-a + b + c) // 2),
        factorial((a + b + c) // 2 + 1),
    )


@cache
def six_j(a: int, b: int, c: int, d: int, e: int, f: int) -> float:
    """Wigner 6j symbol {a b c; d e f} (doubled spins), Racah's formula, exact sum."""
    if not (triangle(a, b, c) and triangle(a, e, f) and triangle(d, b, f) and triangle(d, e, c)):
        return 0.0
    t1, t2, t3, t4 = (a + b + c) // 2, (a + e + f) // 2, (d + b + f) // 2, (d + e + c) // 2
    p1, p2, p3 = (a + b + d + e) // 2, (b + c + e + f) // 2, (c + a + f + d) // 2
    total = Fraction(0)
    for z in range(max(t1, t2, t3, t4), min(p1, p2, p3) + 1):
        num = (-1) ** z * factorial(z + 1)
        den = (factorial(z - t1) * factorial(z - t2) * factorial(z - t3) * factorial(z - t4)
               * factorial(p1 - z) * factorial(p2 - z) * factorial(p3 - z))
        total += Fraction(num, den)
    if total == 0:
        return 0.0
    sq = total * total * _delta2(a, b, c) * _delta2(a, e, f) * _delta2(d, b, f) * _delta2(d, e, c)
    # float(Fraction) is correctly rounded, so only the final sqrt rounds again
    mag = sqrt(float(sq))
    return mag if total > 0 else -mag


@cache
def f_symbol(a: int, b: int, c: int, d: int, e: int, f: int) -> float:
    """``[F^{abc}_d]_{e,f}``; ``e`` inner line of ((ab)c), ``f`` of (a(bc)).  Zero if any
    vertex is forbidden (the guard of ``symmetry/su2.py:174-204``)."""
    if not (triangle(a, b, e) and triangle(e, c, d) and triangle(b, c, f) and triangle(a, f, d)):
        return 0.0
    sign = -1.0 if ((a + b + c + d) // 2) % 2 else 1.0
    return sign * sqrt((e + 1) * (f + 1)) * six_j(a, b, e, c, d, f)


def r_symbol(a: int, b: int, c: int) -> int:
    """``R^{ab}_c = (-1)^(ja + jb - jc)``, exactly +-1; 0 off the triangle."""
    if not triangle(a, b, c):
        return 0
    return -1 if ((a + b - c) // 2) % 2 else 1


def b_symbol(a: int, b: int, c: int) -> float:
    """``B^{ab}_c = sqrt(d_a d_b / d_c) [F^{a b b}_a]_{c, 0}``; SU(2) is self-dual."""
    if not triangle(a, b, c):
        return 0.0
    return sqrt((a + 1) * (b + 1) / (c + 1)) * f_symbol(a, b, b, a, c, 0)


def frobenius_schur(a: int) -> int:
    """``chi_a = sign([F^{a a a}_a]_{0,0})`` = ``(-1)^(2j)``."""
    return 1 if f_symbol(a, a, a, a, 0, 0) > 0 else -1


@cache
def cg(j1: int, m1: int, j2: int, m2: int, j: int, m: int) -> float:
    """<j1 m1; j2 m2 | j m> in the Condon-Shortley phase; all arguments doubled."""
    if m1 + m2 != m or not triangle(j1, j2, j):
        return 0.0
    if abs(m1) > j1 or abs(m2) > j2 or abs(m) > j:
        return 0.0
    k_lo = max(0, (j2 - j - m1) // 2, (j1 + m2 - j) // 2)
    k_hi = min((j1 + j2 - j) // 2, (j1 - m1) // 2, (j2 + m2) // 2)
    total = Fraction(0)
    for k in range(k_lo, k_hi + 1):
        den = (factorial(k) * factorial((j1 + j2 - j) // 2 - k) * factorial((j1 - m1) // 2 - k)
               * factorial((j2 + m2) // 2 - k) * factorial((j - j2 + m1) // 2 + k)
               * factorial((j - j1 - m2) // 2 + k))
        total += Fraction((-1) ** k, den)
    if total == 0:
        return 0.0
    pre = (Fraction(j + 1) * _delta2(j1, j2, j)
           * factorial((j1 + m1) // 2) * factorial((j1 - m1) // 2)
           * factorial((j2 + m2) // 2) * factorial((j2 - m2) // 2)
           * factorial((j + m) // 2) * factorial((j - m) // 2))
    mag = sqrt(float(pre * total * total))
    return mag if total > 0 else -mag


@cache
def cg_tensor(a: int, b: int, c: int):
    """Clebsch-Gordan tensor ``(d_a, d_b, d_c, 1)``, magnetic index descending
    (``symmetry/su2.py:164-172``)."""
    import numpy as np

    out = np.zeros((a + 1, b + 1, c + 1, 1))
    for i in range(a + 1):
        for k in range(b + 1):
            ma, mb = a - 2 * i, b - 2 * k
            mc = ma + mb
            if abs(mc) > c:
                continue
            out[i, k, (c - mc) // 2, 0] = cg(a, ma, b, mb, c, mc)
    out.flags.writeable = False
    return out
