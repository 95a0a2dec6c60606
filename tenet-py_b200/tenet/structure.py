"""Categorical metadata: graded spaces, legs, fusion trees, block keys, tensor structures.

The public types mirror the reference's (``space.py``, ``leg.py``, ``fusion_tree.py``,
``structure.py``): frozen, hashable, array-free values, with the block order as the
storage contract (``structure.py:166-176``).  Underneath, the planner works on a
degeneracy-free *pattern* of integer labels -- two structures that differ only in
degeneracies share every block key, tree and coefficient, exactly the split the
reference makes with ``_pattern`` (``structure.py:330-338``) -- and on integer tree
tuples ``(uncoupled, inner, coupled)`` whose sort order is the reference's
``FusionTree`` order (multiplicity labels are always zero on this path's providers).
"""

from __future__ import annotations

import enum
from collections.abc import Hashable, Iterable, Mapping
from dataclasses import dataclass, field
from functools import cache
from itertools import product
from math import prod

import numpy as np

from tenet.symmetry import Provider, Sector

__all__ = ["IN", "OUT", "FusionBlockKey", "FusionTree", "GradedSpace", "Leg", "Side",
           "TensorStructure"]


class Side(enum.Enum):
    OUT = "out"
    IN = "in"


OUT = Side.OUT
IN = Side.IN


@dataclass(frozen=True, slots=True)
class GradedSpace:
    """``V = (+)_a C^{m_a} (x) V_a``; sectors sorted, all ``m >= 1`` (``space.py:27-140``)."""

    provider: Provider
    sectors: tuple

    @classmethod
    def new(cls, provider: Provider, sectors: Mapping | Iterable) -> GradedSpace:
        pairs = list(sectors.items() if isinstance(sectors, Mapping) else sectors)
        seen = set()
        for a, m in pairs:
            if type(a) is not provider.sector_type:
                raise TypeError(f"sector {a!r} does not belong to provider {provider.name}")
            if m <= 0:
                raise ValueError(f"degeneracy of {a!r} must be positive, got {m}")
            if a in seen:
                raise ValueError(f"duplicate sector {a!r}")
            seen.add(a)
        return cls(provider, tuple(sorted(((a, int(m)) for a, m in pairs), key=lambda p: p[0])))

    @property
    def labels(self) -> tuple[int, ...]:
        return _space_labels(self)

    def degeneracy(self, a: Sector) -> int:
        for b, m in self.sectors:
            if b == a:
                return m
        return 0

    def __iter__(self):
        return (a for a, _ in self.sectors)

    def __len__(self) -> int:
        return len(self.sectors)

    def __contains__(self, a) -> bool:
        return self.degeneracy(a) > 0

    @property
    def reduced_dim(self) -> int:
        return sum(m for _, m in self.sectors)

    @property
    def dim(self) -> int:
        return sum(m * self.provider.irrep_dim(a) for a, m in self.sectors)


@cache
def _space_labels(space: GradedSpace) -> tuple[int, ...]:
    return tuple(space.provider.label(a) for a, _ in space.sectors)


@cache
def _space_degs(space: GradedSpace) -> dict[int, int]:
    return {space.provider.label(a): m for a, m in space.sectors}


@dataclass(frozen=True, slots=True)
class Leg:
    """One axis: a space, a side, a dual flag, a name (``leg.py:34-187``)."""

    space: GradedSpace
    side: Side
    dual: bool = False
    name: Hashable | None = None

    @property
    def provider(self) -> Provider:
        return self.space.provider

    @property
    def sectors(self) -> tuple:
        return tuple(self.space)

    def degeneracy(self, a: Sector) -> int:
        return self.space.degeneracy(a)

    def fused_sector(self, a: Sector) -> Sector:
        return self.provider.dual(a) if self.dual else a

    def space_sector(self, u: Sector) -> Sector:
        return self.provider.dual(u) if self.dual else u

    def dualized(self) -> Leg:
        return Leg(self.space, self.side, not self.dual, self.name)

    def renamed(self, name) -> Leg:
        return Leg(self.space, self.side, self.dual, name)


@dataclass(frozen=True, slots=True, order=True)
class FusionTree:
    """A left-associated fusion tree (``fusion_tree.py:33-163``); public view only."""

    uncoupled: tuple
    inner: tuple
    multiplicities: tuple
    coupled: Sector

    @property
    def rank(self) -> int:
        return len(self.uncoupled)


@dataclass(frozen=True, slots=True, order=True)
class FusionBlockKey:
    """An (output tree, input tree) pair sharing one coupled sector (``structure.py:44-78``)."""

    output_tree: FusionTree
    input_tree: FusionTree

    @property
    def coupled(self) -> Sector:
        return self.output_tree.coupled


# ---------------------------------------------------------------------------------------
# the integer pattern


@dataclass(frozen=True, slots=True)
class Pattern:
    """A structure with degeneracies dropped: provider + per leg (labels, is_out, dual)."""

    provider: Provider
    legs: tuple  # ((labels, is_out, dual), ...)

    @property
    def out_axes(self) -> tuple[int, ...]:
        return tuple(i for i, leg in enumerate(self.legs) if leg[1])

    @property
    def in_axes(self) -> tuple[int, ...]:
        return tuple(i for i, leg in enumerate(self.legs) if not leg[1])


@cache
def all_trees(p: Provider, uncoupled: tuple[int, ...]) -> tuple:
    """All left-associated trees over ``uncoupled``, sorted (``fusion_tree.py:251-267``)."""
    if not uncoupled:
        return (((), (), p._unit_label()),)
    if len(uncoupled) == 1:
        return ((uncoupled, (), uncoupled[0]),)
    last = uncoupled[-1]
    out = []
    for u, inner, e in all_trees(p, uncoupled[:-1]):
        nin = (*inner, e) if len(u) >= 2 else ()
        for c in p._fuse(e, last):
            out.append((uncoupled, nin, c))
    out.sort()
    return tuple(out)


@cache
def trees_to(p: Provider, uncoupled: tuple[int, ...], coupled: int) -> tuple:
    return tuple(t for t in all_trees(p, uncoupled) if t[2] == coupled)


@cache
def coupled_of(p: Provider, uncoupled: tuple[int, ...]) -> tuple[int, ...]:
    return tuple(sorted({t[2] for t in all_trees(p, uncoupled)}))


@cache
def block_keys(pat: Pattern) -> tuple:
    """Every allowed key of a pattern, sorted (``structure.py:349-371``): every OUT tree
    over the OUT legs' labels paired with every IN tree over the IN legs' labels that
    ends in the same coupled sector."""
    p = pat.provider
    fused = [tuple(p._dual(a) if dual else a for a in labels) for labels, _, dual in pat.legs]

    def trees_by_coupled(axes):
        by_c: dict = {}
        for u in product(*(fused[i] for i in axes)):
            for t in all_trees(p, u):
                by_c.setdefault(t[2], []).append(t)
        return by_c

    outs, ins = trees_by_coupled(pat.out_axes), trees_by_coupled(pat.in_axes)
    keys = [(ot, it) for c, ots in outs.items() if c in ins for ot in ots for it in ins[c]]
    keys.sort()
    return tuple(keys)


@cache
def key_index(pat: Pattern) -> dict:
    return {k: i for i, k in enumerate(block_keys(pat))}


# ---------------------------------------------------------------------------------------


class TensorStructure:
    """Ordered legs plus everything derived from them; immutable and hashable
    (``structure.py:81-331``).  ``block_order`` is the storage contract."""

    __slots__ = ("legs", "_hash", "_pattern")

    def __init__(self, legs) -> None:
        legs = tuple(legs)
        if not legs:
            raise ValueError("TensorStructure needs at least one leg")
        object.__setattr__(self, "legs", legs)
        object.__setattr__(self, "_hash", hash(legs))
        p = legs[0].provider
        for i, leg in enumerate(legs):
            if leg.provider != p:
                raise ValueError(f"leg {i} has provider {leg.provider.name}, leg 0 has {p.name}")
        object.__setattr__(self, "_pattern", Pattern(
            p, tuple((leg.space.labels, leg.side is OUT, bool(leg.dual)) for leg in legs)))

    def __setattr__(self, *_):
        raise AttributeError("TensorStructure is immutable")

    def __hash__(self) -> int:
        return self._hash

    def __eq__(self, other) -> bool:
        return isinstance(other, TensorStructure) and self.legs == other.legs

    def __repr__(self) -> str:
        return f"TensorStructure({self.legs!r})"

    @property
    def pattern(self) -> Pattern:
        return self._pattern

    @property
    def provider(self) -> Provider:
        return self.legs[0].provider

    @property
    def ndim(self) -> int:
        return len(self.legs)

    @property
    def out_axes(self) -> tuple[int, ...]:
        return self._pattern.out_axes

    @property
    def in_axes(self) -> tuple[int, ...]:
        return self._pattern.in_axes

    @property
    def codomain(self) -> tuple:
        return tuple(self.legs[i] for i in self.out_axes)

    @property
    def domain(self) -> tuple:
        return tuple(self.legs[i] for i in self.in_axes)

    @property
    def keys(self) -> tuple:
        """Block keys as integer tree tuples, in block order."""
        return block_keys(self._pattern)

    @property
    def num_blocks(self) -> int:
        return len(block_keys(self._pattern))

    @property
    def block_order(self) -> tuple:
        return _public_keys(self._pattern)

    def index_of(self, key: FusionBlockKey) -> int:
        return _public_index(self._pattern)[key]

    def block_shape(self, key: FusionBlockKey) -> tuple[int, ...]:
        return tuple(int(x) for x in layout(self).shapes[self.index_of(key)])

    @property
    def size(self) -> int:
        return layout(self).size


@cache
def _public_keys(pat: Pattern) -> tuple:
    p = pat.provider

    def tree(t):
        u, inner, c = t
        return FusionTree(tuple(p.sector(x) for x in u), tuple(p.sector(x) for x in inner),
                          (0,) * max(len(u) - 1, 0), p.sector(c))

    return tuple(FusionBlockKey(tree(o), tree(i)) for o, i in block_keys(pat))


@cache
def _public_index(pat: Pattern) -> dict:
    return {k: i for i, k in enumerate(_public_keys(pat))}


# ---------------------------------------------------------------------------------------
# arena layout: blocks concatenated in block order, each C-contiguous in public axis order


@dataclass(frozen=True)
class ArenaLayout:
    shapes: np.ndarray   # (n_blocks, ndim) int64, public axis order
    sizes: np.ndarray    # (n_blocks,) int64
    offsets: np.ndarray  # (n_blocks,) int64
    strides: np.ndarray  # (n_blocks, ndim) int64, C-contiguous
    size: int
    coupled: np.ndarray = field(repr=False)  # (n_blocks,) int64 coupled-sector label


@cache
def layout(s: TensorStructure) -> ArenaLayout:
    p = s.provider
    keys = s.keys
    n, nd = len(keys), s.ndim
    oa, ia = s.out_axes, s.in_axes
    # per axis: label -> degeneracy, the dual already applied
    degs = []
    for leg in s.legs:
        d = _space_degs(leg.space)
        degs.append({p._dual(u): m for u, m in d.items()} if leg.dual else d)
    rows = [[0] * nd for _ in range(n)]
    coupled = np.zeros(n, dtype=np.int64)
    for b, (ot, it) in enumerate(keys):
        row = rows[b]
        for ax, u in zip(oa, ot[0]):
            row[ax] = degs[ax][u]
        for ax, u in zip(ia, it[0]):
            row[ax] = degs[ax][u]
        coupled[b] = ot[2]
    shapes = np.array(rows, dtype=np.int64).reshape(n, nd)
    sizes = shapes.prod(axis=1) if n else np.zeros(0, dtype=np.int64)
    offsets = np.zeros(n, dtype=np.int64)
    if n:
        offsets[1:] = np.cumsum(sizes)[:-1]
    strides = np.ones((n, nd), dtype=np.int64)
    for ax in range(nd - 2, -1, -1):
        strides[:, ax] = strides[:, ax + 1] * shapes[:, ax + 1]
    return ArenaLayout(shapes, sizes, offsets, strides, int(sizes.sum()) if n else 0, coupled)


# ---------------------------------------------------------------------------------------
# coupled-sector matrix layout (map_view.py:69-219): rows = OUT trees, cols = IN trees


@dataclass(frozen=True)
class MatrixLayout:
    sectors: tuple            # coupled labels, sorted
    shape: dict               # label -> (rows, cols)
    base: dict                # label -> element offset of B_c in the packed buffer
    size: int
    block_sector: np.ndarray  # (n_blocks,) coupled label of each block
    block_off: np.ndarray     # (n_blocks,) element offset of the block's window
    block_ld: np.ndarray      # (n_blocks,) leading dimension (cols of its B_c)
    rstride: np.ndarray       # (n_blocks, ndim) stride in units of ld (OUT axes)
    cstride: np.ndarray       # (n_blocks, ndim) stride in elements (IN axes)


@cache
def matrix_layout(s: TensorStructure) -> MatrixLayout:
    lay = layout(s)
    keys = s.keys
    oa, ia = s.out_axes, s.in_axes
    n, nd = len(keys), s.ndim
    shapes = lay.shapes
    rsz = shapes[:, list(oa)].prod(axis=1) if oa else np.ones(n, dtype=np.int64)
    csz = shapes[:, list(ia)].prod(axis=1) if ia else np.ones(n, dtype=np.int64)
    rows: dict = {}
    cols: dict = {}
    for b, (ot, it) in enumerate(keys):
        rows.setdefault(ot[2], {}).setdefault(ot, int(rsz[b]))
        cols.setdefault(ot[2], {}).setdefault(it, int(csz[b]))
    sectors = tuple(sorted(rows))
    shape, base, roff, coff = {}, {}, {}, {}
    off = 0
    for c in sectors:
        r = 0
        for t in sorted(rows[c]):
            roff[t] = r
            r += rows[c][t]
        q = 0
        for t in sorted(cols[c]):
            coff[t] = q
            q += cols[c][t]
        shape[c] = (r, q)
        base[c] = off
        off += r * q
    block_sector = np.zeros(n, dtype=np.int64)
    block_off = np.zeros(n, dtype=np.int64)
    block_ld = np.zeros(n, dtype=np.int64)
    for b, (ot, it) in enumerate(keys):
        c = ot[2]
        ld = shape[c][1]
        block_sector[b] = c
        block_ld[b] = ld
        block_off[b] = base[c] + roff[ot] * ld + coff[it]
    rstride = np.zeros((n, nd), dtype=np.int64)
    cstride = np.zeros((n, nd), dtype=np.int64)
    acc = np.ones(n, dtype=np.int64)
    for ax in reversed(oa):
        rstride[:, ax] = acc
        acc = acc * shapes[:, ax]
    acc = np.ones(n, dtype=np.int64)
    for ax in reversed(ia):
        cstride[:, ax] = acc
        acc = acc * shapes[:, ax]
    return MatrixLayout(sectors, shape, base, off, block_sector, block_off, block_ld, rstride,
                        cstride)


def structure_size(s: TensorStructure) -> int:
    return layout(s).size


def numel(shape) -> int:
    return prod(shape)
