"""Test-only stand-in for the ``racah`` PyO3 wheel (racah-py 0.1.1), SU(2) only.

Used exclusively by ``tests/golden/make_golden.py`` so that the unmodified reference can be
imported in the build container to produce golden vectors.  It exposes the surface the
reference calls at ``symmetry/_sun_coeff.py:45-117`` and ``symmetry/su2.py:55``, with the
numbers computed by ``oracle/racah_su2.py`` (Racah's closed forms, TensorKitSectors gauge).
"""

import numpy as np

from oracle import racah_su2 as _c


def sun_authority_fingerprint() -> str:
    return "racah-shim-su2-exact-racah-formula"


class Irrep:
    def __init__(self, dynkin):
        dynkin = tuple(int(x) for x in dynkin)
        if len(dynkin) != 1:
            raise NotImplementedError("racah shim: SU(2) only")
        self.dynkin = list(dynkin)
        self._j = dynkin[0]

    def dim(self) -> int:
        return self._j + 1

    def dual(self) -> "Irrep":
        return Irrep((self._j,))

    def __repr__(self) -> str:
        return f"Irrep({self.dynkin})"


def fusion(a: Irrep, b: Irrep):
    lo, hi = abs(a._j - b._j), a._j + b._j
    return [(Irrep((c,)), 1) for c in range(lo, hi + 1, 2)]


def fusion_multiplicity(a: Irrep, b: Irrep, c: Irrep) -> int:
    return int(_c.triangle(a._j, b._j, c._j))


def clebsch_gordan(a: Irrep, b: Irrep, c: Irrep) -> np.ndarray:
    if not _c.triangle(a._j, b._j, c._j):
        raise ValueError("racah shim: forbidden vertex")
    return np.array(_c.cg_tensor(a._j, b._j, c._j))


def f_symbol(a, b, c, d, e, f) -> np.ndarray:
    js = [x._j for x in (a, b, c, d, e, f)]
    for x, y, z in ((0, 1, 4), (4, 2, 3), (1, 2, 5), (0, 5, 3)):
        if not _c.triangle(js[x], js[y], js[z]):
            raise ValueError("racah shim: N = 0 vertex")
    return np.full((1, 1, 1, 1), _c.f_symbol(*js))


def r_symbol(a, b, c) -> np.ndarray:
    return np.full((1, 1), float(_c.r_symbol(a._j, b._j, c._j)))
