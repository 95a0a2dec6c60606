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
    """``V = (+)_a C^{m_a} (x) V_a``; sectors sorted, all ``m >= 1`` (``space.py:27-140``).
    The hash is computed once (spaces key the planner's caches)."""

    provider: Provider
    sectors: tuple
    _hash: int = field(default=0, init=False, repr=False, compare=False)

    def __post_init__(self) -> None:
        object.__setattr__(self, "_hash", hash((self.provider, self.sectors)))

    def __hash__(self) -> int:
        return self._hash

    def __reduce__(self):  # rebuilt where it lands: hashes differ between processes
        return (GradedSpace, (self.provider, self.sectors))

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
    """A structure with degeneracies dropped: provider + per leg (labels, is_out, dual).
    The hash is computed once (patterns key the planner's caches)."""

    provider: Provider
    legs: tuple  # ((labels, is_out, dual), ...)
    _hash: int = field(default=0, init=False, repr=False, compare=False)

    def __post_init__(self) -> None:
        object.__setattr__(self, "_hash", hash((self.provider, self.legs)))

    def __hash__(self) -> int:
        return self._hash

    def __reduce__(self):  # rebuilt where it lands: hashes differ between processes
        return (Pattern, (self.provider, self.legs))

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


@dataclass(frozen=True)
class _LayoutPlan:
    """The degeneracy-free part of a layout, per pattern: for every axis the distinct space
    labels its blocks use and each block's index into them (the dual already undone, so
    the label is the leg space's own), and every block's coupled label."""

    labels: tuple            # per axis, the distinct space labels (sorted)
    index: np.ndarray        # (n_blocks, ndim) int64 index into labels[axis]
    coupled: np.ndarray      # (n_blocks,) int64


@cache
def _layout_plan(pat: Pattern) -> _LayoutPlan:
    p = pat.provider
    keys = block_keys(pat)
    n, nd = len(keys), len(pat.legs)
    oa, ia = pat.out_axes, pat.in_axes
    lab = np.zeros((n, nd), dtype=np.int64)
    coupled = np.zeros(n, dtype=np.int64)
    dual = [bool(leg[2]) for leg in pat.legs]
    for b, (ot, it) in enumerate(keys):
        for ax, u in zip(oa, ot[0]):
            lab[b, ax] = p._dual(u) if dual[ax] else u
        for ax, u in zip(ia, it[0]):
            lab[b, ax] = p._dual(u) if dual[ax] else u
        coupled[b] = ot[2]
    labels, index = [], np.zeros((n, nd), dtype=np.int64)
    for ax in range(nd):
        uniq, inv = np.unique(lab[:, ax], return_inverse=True)
        labels.append(tuple(int(x) for x in uniq))
        index[:, ax] = inv.reshape(-1)
    index.flags.writeable = coupled.flags.writeable = False  # shared by every structure
    return _LayoutPlan(tuple(labels), index, coupled)


@cache
def layout(s: TensorStructure) -> ArenaLayout:
    """Block shapes, sizes, offsets and C-contiguous strides of ``s``'s arena: the pattern's
    plan (``_layout_plan``) filled with this structure's degeneracies."""
    plan = _layout_plan(s.pattern)
    n, nd = plan.index.shape
    shapes = np.empty((n, nd), dtype=np.int64)
    for ax, leg in enumerate(s.legs):
        d = _space_degs(leg.space)
        vals = np.array([d[u] for u in plan.labels[ax]], dtype=np.int64)
        shapes[:, ax] = vals[plan.index[:, ax]] if n else 0
    sizes = shapes.prod(axis=1) if n else np.zeros(0, dtype=np.int64)
    offsets = np.zeros(n, dtype=np.int64)
    if n:
        offsets[1:] = np.cumsum(sizes)[:-1]
    strides = np.ones((n, nd), dtype=np.int64)
    for ax in range(nd - 2, -1, -1):
        strides[:, ax] = strides[:, ax + 1] * shapes[:, ax + 1]
    return ArenaLayout(shapes, sizes, offsets, strides, int(sizes.sum()) if n else 0,
                       plan.coupled)


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


@dataclass(frozen=True)
class _MatrixPlan:
    """The degeneracy-free part of a matrix layout, per pattern.  OUT trees (rows) and IN
    trees (columns) are numbered sector by sector, sectors and trees in sorted order; each
    block has its sector's and its trees' numbers, each tree its sector's number and a
    block that carries it (all such blocks share the tree's row or column count)."""

    sectors: tuple           # coupled labels, sorted
    block_sec: np.ndarray    # (n_blocks,) sector number
    block_row: np.ndarray    # (n_blocks,) OUT tree number
    block_col: np.ndarray    # (n_blocks,) IN tree number
    row_sec: np.ndarray      # (n_rows,) sector number of each OUT tree
    row_rep: np.ndarray      # (n_rows,) a block with that OUT tree
    col_sec: np.ndarray
    col_rep: np.ndarray


@cache
def _matrix_plan(pat: Pattern) -> _MatrixPlan:
    keys = block_keys(pat)
    rows: dict = {}
    cols: dict = {}
    for b, (ot, it) in enumerate(keys):
        rows.setdefault(ot[2], {}).setdefault(ot, b)
        cols.setdefault(ot[2], {}).setdefault(it, b)
    sectors = tuple(sorted(rows))
    sec_no = {c: k for k, c in enumerate(sectors)}

    def number(trees_of):
        no, sec, rep = {}, [], []
        for c in sectors:
            for t in sorted(trees_of[c]):
                no[(c, t)] = len(sec)
                sec.append(sec_no[c])
                rep.append(trees_of[c][t])
        return no, np.array(sec, dtype=np.int64), np.array(rep, dtype=np.int64)

    row_no, row_sec, row_rep = number(rows)
    col_no, col_sec, col_rep = number(cols)
    n = len(keys)
    block_sec = np.fromiter((sec_no[ot[2]] for ot, _ in keys), dtype=np.int64, count=n)
    block_row = np.fromiter((row_no[(ot[2], ot)] for ot, _ in keys), dtype=np.int64, count=n)
    block_col = np.fromiter((col_no[(ot[2], it)] for ot, it in keys), dtype=np.int64, count=n)
    for a in (block_sec, block_row, block_col, row_sec, row_rep, col_sec, col_rep):
        a.flags.writeable = False  # shared by every structure of the pattern
    return _MatrixPlan(sectors, block_sec, block_row, block_col, row_sec, row_rep, col_sec,
                       col_rep)


def _starts(sizes: np.ndarray, group: np.ndarray, n_groups: int) -> tuple:
    """Per group the total of ``sizes`` and per item its offset inside its group, for
    items grouped consecutively (``group`` nondecreasing, no group empty); exact integer
    sums."""
    if not len(sizes):
        return np.zeros(n_groups, dtype=np.int64), sizes
    starts = np.searchsorted(group, np.arange(n_groups))
    tot = np.add.reduceat(sizes, starts)
    first = np.zeros(n_groups, dtype=np.int64)
    first[1:] = np.cumsum(tot)[:-1]
    return tot, (np.cumsum(sizes) - sizes) - first[group]


@cache
def matrix_layout(s: TensorStructure) -> MatrixLayout:
    """The coupled-sector matrices of ``s`` (``map_view.py:69-219``): the pattern's plan
    (``_matrix_plan``) filled with this structure's row and column counts."""
    lay = layout(s)
    plan = _matrix_plan(s.pattern)
    oa, ia = s.out_axes, s.in_axes
    n, nd = lay.shapes.shape
    shapes = lay.shapes
    rsz = shapes[:, list(oa)].prod(axis=1) if oa else np.ones(n, dtype=np.int64)
    csz = shapes[:, list(ia)].prod(axis=1) if ia else np.ones(n, dtype=np.int64)
    ns = len(plan.sectors)
    R, roff = _starts(rsz[plan.row_rep], plan.row_sec, ns)
    Q, coff = _starts(csz[plan.col_rep], plan.col_sec, ns)
    area = R * Q
    base = np.zeros(ns, dtype=np.int64)
    if ns:
        base[1:] = np.cumsum(area)[:-1]
    sec = plan.block_sec
    block_ld = Q[sec]
    block_off = base[sec] + roff[plan.block_row] * block_ld + coff[plan.block_col]
    block_sector = np.array(plan.sectors, dtype=np.int64)[sec] if n else np.zeros(0, np.int64)
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
    shape = {c: (int(R[k]), int(Q[k])) for k, c in enumerate(plan.sectors)}
    bases = {c: int(base[k]) for k, c in enumerate(plan.sectors)}
    return MatrixLayout(plan.sectors, shape, bases, int(area.sum()), block_sector, block_off,
                        block_ld, rstride, cstride)


def structure_size(s: TensorStructure) -> int:
    return layout(s).size


def numel(shape) -> int:
    return prod(shape)
