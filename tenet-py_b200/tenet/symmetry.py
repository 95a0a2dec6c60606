"""Symmetry providers on the hot path: U(1), Z2, fermion parity fZ2, and SU(2).

Public names and semantics follow the reference's ``tenet.symmetry``
(``symmetry/u1.py``, ``z2.py``, ``fz2.py``, ``su2.py``, ``base.py``): sectors are frozen,
ordered value types (``U1Sector(charge)``, ``Z2Sector(parity)``, ``FZ2Sector(parity)``,
``SU2Sector(two_j)``) and providers are singletons (``U1``, ``Z2``, ``fZ2``, ``SU2``).

The planner underneath works on the integer *label* of a sector (the charge, parity or
``two_j``), which sorts exactly like the sector itself; every provider therefore exposes
a label-level core (``_fuse``, ``_dual``, ``_qdim``, ``_fs``, ``_twist``) next to the
sector-level API.
"""

from __future__ import annotations

from dataclasses import dataclass

from tenet import _su2

__all__ = [
    "SU2", "U1", "U1xU1xfZ2", "Z2", "CapabilityError", "FZ2Sector", "ProductProvider",
    "ProductSector", "Provider", "SU2Sector", "Sector", "StructureChangingError", "U1Sector",
    "Z2Sector", "fZ2",
]


class CapabilityError(TypeError):
    """A provider lacks a capability the operation needs (``symmetry/base.py:700-701``)."""


class StructureChangingError(TypeError):
    """An operation whose output structure depends on block values ran under a trace."""


class Sector:
    """Marker base of sector labels."""

    __slots__ = ()


@dataclass(frozen=True, slots=True, order=True)
class U1Sector(Sector):
    charge: int


@dataclass(frozen=True, slots=True, order=True)
class Z2Sector(Sector):
    parity: int

    def __post_init__(self) -> None:
        if not isinstance(self.parity, int) or isinstance(self.parity, bool):
            raise TypeError(f"parity must be an int, got {self.parity!r}")
        if self.parity not in (0, 1):
            raise ValueError(f"parity must be 0 or 1, got {self.parity}")


@dataclass(frozen=True, slots=True, order=True)
class FZ2Sector(Sector):
    parity: int

    def __post_init__(self) -> None:
        if not isinstance(self.parity, int) or isinstance(self.parity, bool):
            raise TypeError(f"parity must be an int, got {self.parity!r}")
        if self.parity not in (0, 1):
            raise ValueError(f"parity must be 0 or 1, got {self.parity}")


@dataclass(frozen=True, slots=True, order=True)
class SU2Sector(Sector):
    two_j: int

    def __post_init__(self) -> None:
        if not isinstance(self.two_j, int) or isinstance(self.two_j, bool):
            raise TypeError(f"two_j must be an int, got {type(self.two_j).__name__}")
        if self.two_j < 0:
            raise ValueError(f"two_j must be non-negative, got {self.two_j}")


@dataclass(frozen=True, slots=True, order=True)
class ProductSector(Sector):
    """A sector of U(1) x U(1) x fZ2: particle number ``n``, ``two_sz`` and fermion parity
    (the grading of a spinful fermion chain such as the Hubbard chain).  Ordered
    lexicographically by ``(n, two_sz, parity)``."""

    n: int
    two_sz: int
    parity: int

    def __post_init__(self) -> None:
        for v in (self.n, self.two_sz, self.parity):
            if not isinstance(v, int) or isinstance(v, bool):
                raise TypeError(f"product sector components must be ints, got {v!r}")
        if self.parity not in (0, 1):
            raise ValueError(f"parity must be 0 or 1, got {self.parity}")
        if not (-_PROD_OFF < self.n < _PROD_OFF and -_PROD_OFF < self.two_sz < _PROD_OFF):
            raise ValueError("product sector charge out of range")


# integer labels of product sectors: ((n + OFF) * 2^21 + (two_sz + OFF)) * 2 + parity, so the
# parity is the lowest bit (the Koszul sign reads it there) and labels sort like sectors
_PROD_OFF = 1 << 20
_PROD_SPAN = 1 << 21


def _prod_encode(n: int, sz: int, p: int) -> int:
    return ((n + _PROD_OFF) * _PROD_SPAN + (sz + _PROD_OFF)) * 2 + p


def _prod_decode(label: int) -> tuple[int, int, int]:
    q = label >> 1
    return (q // _PROD_SPAN) - _PROD_OFF, (q % _PROD_SPAN) - _PROD_OFF, label & 1


@dataclass(frozen=True, slots=True)
class Provider:
    """One symmetry.  ``kind`` selects the label arithmetic; ``name`` is the display name."""

    name: str

    # ---- label level (ints) ------------------------------------------------------------
    @property
    def abelian(self) -> bool:
        return self.name != "SU2"

    @property
    def fermionic(self) -> bool:
        return self.name == "fZ2"

    def _fuse(self, a: int, b: int) -> tuple[int, ...]:
        if self.name == "U1":
            return (a + b,)
        if self.name == "SU2":
            return tuple(range(abs(a - b), a + b + 1, 2))
        return (a ^ b,)

    def _dual(self, a: int) -> int:
        return -a if self.name == "U1" else a

    def _qdim(self, a: int) -> float:
        return float(a + 1) if self.name == "SU2" else 1.0

    def _fs(self, a: int) -> int:
        return _su2.frobenius_schur(a) if self.name == "SU2" else 1

    def _twist(self, a: int) -> int:
        return -1 if (self.name == "fZ2" and a) else 1

    def label(self, s: Sector) -> int:
        if self.name == "U1":
            return s.charge
        if self.name == "SU2":
            return s.two_j
        return s.parity

    def sector(self, label: int) -> Sector:
        if self.name == "U1":
            return U1Sector(label)
        if self.name == "SU2":
            return SU2Sector(label)
        if self.name == "Z2":
            return Z2Sector(label)
        return FZ2Sector(label)

    @property
    def sector_type(self) -> type:
        return {"U1": U1Sector, "Z2": Z2Sector, "fZ2": FZ2Sector, "SU2": SU2Sector}[self.name]

    # ---- sector level (the reference's provider protocol) -------------------------------
    @property
    def unit(self) -> Sector:
        return self.sector(self._unit_label())

    def _unit_label(self) -> int:
        return 0

    def dual(self, a: Sector) -> Sector:
        return self.sector(self._dual(self.label(a)))

    def fusion(self, a: Sector, b: Sector) -> tuple[Sector, ...]:
        return tuple(self.sector(c) for c in self._fuse(self.label(a), self.label(b)))

    def n_symbol(self, a: Sector, b: Sector, c: Sector) -> int:
        return int(self.label(c) in self._fuse(self.label(a), self.label(b)))

    def qdim(self, a: Sector) -> float:
        return self._qdim(self.label(a))

    def irrep_dim(self, a: Sector) -> int:
        return int(self._qdim(self.label(a)))

    def frobenius_schur(self, a: Sector) -> int:
        return self._fs(self.label(a))

    def twist(self, a: Sector) -> int:
        return self._twist(self.label(a))

    def f_symbol(self, a, b, c, d, e, f) -> float:
        if self.name != "SU2":
            ls = [self.label(x) for x in (a, b, c, d, e, f)]
            ok = (ls[4] in self._fuse(ls[0], ls[1]) and ls[3] in self._fuse(ls[4], ls[2])
                  and ls[5] in self._fuse(ls[1], ls[2]) and ls[3] in self._fuse(ls[0], ls[5]))
            return 1.0 if ok else 0.0
        return _su2.f_symbol(*(self.label(x) for x in (a, b, c, d, e, f)))

    def r_symbol(self, a, b, c) -> float:
        la, lb, lc = self.label(a), self.label(b), self.label(c)
        if lc not in self._fuse(la, lb):
            return 0
        if self.name == "SU2":
            return _su2.r_symbol(la, lb, lc)
        if self.name == "fZ2":
            return -1 if (la and lb) else 1
        return 1

    def b_symbol(self, a, b, c) -> float:
        if self.name == "SU2":
            return _su2.b_symbol(self.label(a), self.label(b), self.label(c))
        return float(self.n_symbol(a, b, c))

    def __repr__(self) -> str:
        return f"{self.name}Provider()"


@dataclass(frozen=True, slots=True)
class ProductProvider(Provider):
    """U(1) x U(1) x fZ2: charges add, parities add mod 2, the braiding sign is the fZ2
    one (``-1`` when both lines are odd), every quantum dimension is 1.  The reference
    composes such groups with ``ProductProvider`` (``symmetry/product.py``); its labels
    here are single integers (``_prod_encode``) so the planner's integer core applies
    unchanged."""

    @property
    def fermionic(self) -> bool:
        return True

    def _unit_label(self) -> int:
        return _prod_encode(0, 0, 0)

    def _fuse(self, a: int, b: int) -> tuple[int, ...]:
        n1, s1, p1 = _prod_decode(a)
        n2, s2, p2 = _prod_decode(b)
        return (_prod_encode(n1 + n2, s1 + s2, p1 ^ p2),)

    def _dual(self, a: int) -> int:
        n, sz, p = _prod_decode(a)
        return _prod_encode(-n, -sz, p)

    def _qdim(self, a: int) -> float:
        return 1.0

    def _fs(self, a: int) -> int:
        return 1

    def _twist(self, a: int) -> int:
        return -1 if a & 1 else 1

    def label(self, s: Sector) -> int:
        return _prod_encode(s.n, s.two_sz, s.parity)

    def sector(self, label: int) -> Sector:
        return ProductSector(*_prod_decode(label))

    @property
    def sector_type(self) -> type:
        return ProductSector

    def r_symbol(self, a, b, c) -> float:
        la, lb, lc = self.label(a), self.label(b), self.label(c)
        if lc not in self._fuse(la, lb):
            return 0
        return -1 if (la & 1 and lb & 1) else 1


U1 = Provider("U1")
Z2 = Provider("Z2")
fZ2 = Provider("fZ2")
SU2 = Provider("SU2")
U1xU1xfZ2 = ProductProvider("U1xU1xfZ2")
