"""Oracle (test infrastructure only): a CPU restatement of TeNeT-py's block-sparse path.

This is the checker the CUDA path is compared against.  It restates, in plain NumPy
FP64, the algorithm of the reference for the hot path: block enumeration, fusion-tree
permutation and bending coefficients, the transpose -> bend -> transpose repartition
sandwich, the coupled-sector matrix lowering, ``compose``/``tensordot``/``einsum``, the
qdim-weighted vector space, the truncated blockwise SVD with its greedy dense-budget keep
rule, Lanczos, and the two-site effective-Hamiltonian matvec with its environment folds.
Every function cites the reference file (paths relative to ``src/tenet``) it follows.

It is pinned by the golden vectors in ``tests/golden`` (outputs of the reference itself,
run under test-only shims) and by the reference's own SU(2) F/R fixtures.  Only the test
suite, ``__graft_entry__.smoke`` and ``bench.py``'s CPU-baseline leg import it; the
shipped package never does.

Data model: a sector is a plain ``int`` (U(1) charge, Z2/fZ2 parity, SU(2) ``two_j``); a
fusion tree is ``(uncoupled, inner, coupled)`` (multiplicity labels are all zero for the
multiplicity-free providers on this path, so they are omitted without changing the sort
order of ``fusion_tree.py:33-163``); a block key is ``(output_tree, input_tree)``; a leg is
``Leg(sectors, side, dual)`` with ``sectors`` the sorted ``((sector, degeneracy), ...)``.
"""

from __future__ import annotations

from dataclasses import dataclass, replace
from functools import cache
from itertools import product
from math import sqrt

import numpy as np

from oracle import racah_su2

OUT, IN = "out", "in"


# ---------------------------------------------------------------------------------------
# providers  (symmetry/u1.py, z2.py, fz2.py, su2.py, base.py)


@dataclass(frozen=True)
class Provider:
    name: str

    # -- fusion rules -----------------------------------------------------------------
    def unit(self) -> int:
        return 0

    def dual(self, a: int) -> int:
        return -a if self.name == "U1" else a

    def fusion(self, a: int, b: int) -> tuple[int, ...]:
        if self.name == "U1":
            return (a + b,)
        if self.name in ("Z2", "fZ2"):
            return (a ^ b,)
        return tuple(range(abs(a - b), a + b + 1, 2))  # su2.py fusion: ascending two_j

    def n_symbol(self, a: int, b: int, c: int) -> int:
        return int(c in self.fusion(a, b))

    def qdim(self, a: int) -> float:
        return float(a + 1) if self.name == "SU2" else 1.0

    def frobenius_schur(self, a: int) -> float:
        return float(racah_su2.frobenius_schur(a)) if self.name == "SU2" else 1.0

    def twist(self, a: int) -> float:
        return -1.0 if (self.name == "fZ2" and a) else 1.0

    @property
    def abelian(self) -> bool:
        return self.name != "SU2"


U1, Z2, FZ2, SU2 = Provider("U1"), Provider("Z2"), Provider("fZ2"), Provider("SU2")
PROVIDERS = {"U1": U1, "Z2": Z2, "fZ2": FZ2, "SU2": SU2}


@cache
def all_trees(p: Provider, uncoupled: tuple[int, ...]) -> tuple:
    """Every left-associated tree over ``uncoupled``, sorted (``fusion_tree.py:251-267``)."""
    if not uncoupled:
        return (((), (), p.unit()),)
    if len(uncoupled) == 1:
        return ((uncoupled, (), uncoupled[0]),)
    out = []
    for tree in all_trees(p, uncoupled[:-1]):
        e = tree[2]
        inner = (*tree[1], e) if len(tree[0]) >= 2 else ()
        for c in p.fusion(e, uncoupled[-1]):
            out.append((uncoupled, inner, c))
    return tuple(sorted(out))


@cache
def fusion_trees(p: Provider, uncoupled: tuple[int, ...], coupled: int) -> tuple:
    return tuple(t for t in all_trees(p, uncoupled) if t[2] == coupled)


def lines(tree) -> tuple[int, ...]:
    """The left spine ``(e_0 .. e_{N-1})`` (``fusion_tree.py:99-114``)."""
    u, inner, c = tree
    if len(u) == 0:
        return ()
    if len(u) == 1:
        return (c,)
    return (u[0], *inner, c)


def _unique_tree(p: Provider, uncoupled, coupled):
    trees = fusion_trees(p, tuple(uncoupled), coupled)
    assert len(trees) == 1, (uncoupled, coupled, trees)
    return trees[0]


def koszul_sign(uncoupled, perm) -> float:
    """``(-1)^(odd-odd inversions of perm)`` (``symmetry/fz2.py:91-130``)."""
    odd = [i for i in perm if uncoupled[i]]
    inv = sum(1 for j in range(len(odd)) for k in range(j + 1, len(odd)) if odd[j] > odd[k])
    return -1.0 if inv % 2 else 1.0


@cache
def _artin_braid(p: Provider, tree, i: int):
    """Swap uncoupled lines i, i+1 of a left-associated tree (``symmetry/base.py:898-996``),
    scalar (multiplicity-free) branch."""
    u, inner, c = tree
    spine = lines(tree)
    new_u = (*u[:i], u[i + 1], u[i], *u[i + 2:])
    if i == 0:
        return (((new_u, inner, c), float(racah_su2.r_symbol(u[0], u[1], spine[1]))),)
    a, b, cc, e, f = spine[i - 1], u[i], u[i + 1], spine[i], spine[i + 1]
    out = []
    for new_e in p.fusion(a, cc):
        if not p.n_symbol(new_e, b, f):
            continue
        coeff = sum(
            racah_su2.f_symbol(a, b, cc, f, e, d) * racah_su2.r_symbol(b, cc, d)
            * racah_su2.f_symbol(a, cc, b, f, new_e, d)
            for d in p.fusion(b, cc)
        )
        new_inner = (*inner[: i - 1], new_e, *inner[i:])
        out.append(((new_u, new_inner, c), coeff))
    return tuple(out)


@cache
def permute_tree(p: Provider, tree, perm: tuple[int, ...]):
    """``permute_tree`` per provider: unique-tree recompute for U(1)/Z2
    (``base.py:778-825``), plus the Koszul sign for fZ2 (``fz2.py:185-200``), and the
    Artin-generator expansion for SU(2) (``base.py:828-895``)."""
    u, _, c = tree
    if p.abelian:
        new = _unique_tree(p, tuple(u[i] for i in perm), c)
        return ((new, koszul_sign(u, perm) if p.name == "fZ2" else 1.0),)
    terms = {tree: 1.0}
    current = list(range(len(u)))
    for j, target in enumerate(perm):
        for i in range(current.index(target) - 1, j - 1, -1):
            current[i], current[i + 1] = current[i + 1], current[i]
            nxt: dict = {}
            for t, cf in terms.items():
                for braided, cb in _artin_braid(p, t, i):
                    nxt[braided] = nxt.get(braided, 0.0) + cf * cb
            terms = nxt
    return tuple(terms.items())


def bend_key(p: Provider, key, *, right: bool, dual: bool):
    """``bend_right``/``bend_left``: ``bend_unique`` (``base.py:999-1074``) for the abelian
    providers, ``bend_braided`` (``base.py:1077-1190``) for SU(2)."""
    ot, it = key
    src, dst = (ot, it) if right else (it, ot)
    assert len(src[0]) > 0
    b = src[0][-1]
    if p.abelian:
        remaining = src[0][:-1]
        cs = sorted({t[2] for t in all_trees(p, remaining)})
        assert len(cs) == 1
        new_src = _unique_tree(p, remaining, cs[0])
        new_dst = _unique_tree(p, (*dst[0], p.dual(b)), cs[0])
        coeff = 1.0
    else:
        c = src[2]
        a = lines(src)[-2] if len(src[0]) >= 2 else p.unit()
        new_src = (src[0][:-1], src[1][:-1], a)
        scale = sqrt(p.qdim(c) / p.qdim(a))
        if dual:
            scale *= p.frobenius_schur(p.dual(b))
        new_dst = ((*dst[0], p.dual(b)), lines(dst)[1:], a)
        coeff = scale * racah_su2.b_symbol(a, b, c)
    new_key = (new_src, new_dst) if right else (new_dst, new_src)
    return ((new_key, coeff),)


# ---------------------------------------------------------------------------------------
# structure  (leg.py, structure.py)


@dataclass(frozen=True)
class Leg:
    sectors: tuple  # ((sector, degeneracy), ...) sorted by sector
    side: str
    dual: bool = False

    def degeneracy(self, a: int) -> int:
        for s, m in self.sectors:
            if s == a:
                return m
        return 0


@dataclass(frozen=True)
class Structure:
    provider: Provider
    legs: tuple

    @property
    def out_axes(self):
        return tuple(i for i, leg in enumerate(self.legs) if leg.side == OUT)

    @property
    def in_axes(self):
        return tuple(i for i, leg in enumerate(self.legs) if leg.side == IN)

    @property
    def codomain(self):
        return tuple(self.legs[i] for i in self.out_axes)

    @property
    def domain(self):
        return tuple(self.legs[i] for i in self.in_axes)


def fused(p: Provider, leg: Leg, a: int) -> int:
    return p.dual(a) if leg.dual else a


@cache
def block_order(s: Structure) -> tuple:
    """Every allowed key, sorted (``structure.py:349-371``)."""
    p = s.provider
    oa, ia = s.out_axes, s.in_axes
    keys = set()
    for assignment in product(*([a for a, _ in leg.sectors] for leg in s.legs)):
        u = tuple(fused(p, leg, a) for leg, a in zip(s.legs, assignment))
        out_u = tuple(u[i] for i in oa)
        in_u = tuple(u[i] for i in ia)
        for c in sorted({t[2] for t in all_trees(p, out_u)}):
            keys.update((ot, it) for ot in fusion_trees(p, out_u, c)
                        for it in fusion_trees(p, in_u, c))
    return tuple(sorted(keys))


@cache
def index_map(s: Structure) -> dict:
    return {k: i for i, k in enumerate(block_order(s))}


def block_shape(s: Structure, key) -> tuple[int, ...]:
    """Degeneracies in public axis order (``structure.py:374-405``)."""
    p = s.provider
    by_axis = dict(zip(s.out_axes, key[0][0])) | dict(zip(s.in_axes, key[1][0]))
    return tuple(leg.degeneracy(fused(p, leg, by_axis[ax])) for ax, leg in enumerate(s.legs))


@dataclass
class Tensor:
    structure: Structure
    blocks: list

    @property
    def legs(self):
        return self.structure.legs

    @property
    def ndim(self):
        return len(self.structure.legs)

    def arena(self) -> np.ndarray:
        if not self.blocks:
            return np.zeros(0)
        return np.concatenate([np.asarray(b, dtype=np.float64).ravel() for b in self.blocks])


def from_arena(s: Structure, arena: np.ndarray) -> Tensor:
    blocks, off = [], 0
    for k in block_order(s):
        shape = block_shape(s, k)
        n = int(np.prod(shape))
        blocks.append(np.asarray(arena[off:off + n], dtype=np.float64).reshape(shape))
        off += n
    assert off == arena.size
    return Tensor(s, blocks)


def random(s: Structure, seed: int) -> Tensor:
    """``SymmetricTensor.random``: one ``standard_normal`` draw per block in block order
    from ``np.random.default_rng(seed)`` (``tensor.py:232-262``)."""
    rng = np.random.default_rng(seed)
    return Tensor(s, [rng.standard_normal(block_shape(s, k)) for k in block_order(s)])


def zeros(s: Structure) -> Tensor:
    return Tensor(s, [np.zeros(block_shape(s, k)) for k in block_order(s)])


# ---------------------------------------------------------------------------------------
# permutation and bending plans  (ops/permutation.py, ops/repartition.py)


def _side_perm(axes, old_side_axes, new_side_axes):
    pos = {old: j for j, old in enumerate(old_side_axes)}
    return tuple(pos[axes[i]] for i in new_side_axes)


@cache
def permutation_plan(s: Structure, axes: tuple[int, ...]):
    """(new structure, terms) of a public transpose (``ops/permutation.py:159-197``)."""
    new = Structure(s.provider, tuple(s.legs[i] for i in axes))
    op = _side_perm(axes, s.out_axes, new.out_axes)
    ip = _side_perm(axes, s.in_axes, new.in_axes)
    order = block_order(s)
    if op == tuple(range(len(op))) and ip == tuple(range(len(ip))):
        return new, tuple((i, i, 1.0) for i in range(len(order)))
    idx = index_map(new)
    terms = []
    for src, (ot, it) in enumerate(order):
        for ot2, c1 in permute_tree(s.provider, ot, op):
            for it2, c2 in permute_tree(s.provider, it, ip):
                c = c1 * c2
                if c == 0:
                    continue
                terms.append((src, idx[(ot2, it2)], c))
    return new, tuple(terms)


@cache
def bend_plan(s: Structure, axis: int):
    """Bend the last leg of its side (``ops/repartition.py:134-183``)."""
    leg = s.legs[axis]
    right = leg.side == OUT
    moved = replace(leg, side=IN if right else OUT, dual=not leg.dual)
    new = Structure(s.provider, (*(x for i, x in enumerate(s.legs) if i != axis), moved))
    idx = index_map(new)
    terms = []
    for src, key in enumerate(block_order(s)):
        for nk, c in bend_key(s.provider, key, right=right, dual=leg.dual):
            if c != 0:
                terms.append((src, idx[nk], c))
    return new, tuple(terms)


def _compose_terms(terms, following):
    """Sparse product of two block maps (``ops/repartition.py:298-316``)."""
    by_src: dict = {}
    for src, dst, c in following:
        by_src.setdefault(src, []).append((dst, c))
    merged: dict = {}
    for src, mid, c in terms:
        for dst, o in by_src.get(mid, ()):
            merged[(src, dst)] = merged.get((src, dst), 0.0) + c * o
    return tuple((s, d, c) for (s, d), c in merged.items())


@cache
def repartition_plan(s: Structure, outputs: tuple, inputs: tuple):
    """The composed transpose/bend/transpose chain (``ops/repartition.py:341-385``)."""
    ndim = len(s.legs)
    want = {ax: OUT for ax in outputs} | {ax: IN for ax in inputs}
    crossing = [ax for ax in range(ndim) if s.legs[ax].side != want[ax]]
    perm = tuple(range(ndim))
    terms = tuple((i, i, 1.0) for i in range(len(block_order(s))))
    labels = list(range(ndim))
    cur = s
    for ax in crossing:
        p = labels.index(ax)
        axes = tuple(i for i in range(ndim) if i != p) + (p,)
        cur, t = permutation_plan(cur, axes)
        perm = tuple(perm[i] for i in axes)
        terms = _compose_terms(terms, t)
        labels.append(labels.pop(p))
        cur, t = bend_plan(cur, ndim - 1)
        terms = _compose_terms(terms, t)
    position = {a: q for q, a in enumerate(labels)}
    axes = tuple(position[ax] for ax in (*outputs, *inputs))
    cur, t = permutation_plan(cur, axes)
    return cur, tuple(perm[i] for i in axes), _compose_terms(terms, t)


def _execute(t: Tensor, new: Structure, perm, terms) -> Tensor:
    """``out[dst] += coeff * transpose(in[src], perm)`` (``ops/repartition.py:458-476``)."""
    moved = {src: np.transpose(t.blocks[src], perm) for src in {s for s, _, _ in terms}}
    blocks: dict = {}
    for src, dst, c in terms:
        contrib = moved[src] if c == 1 else moved[src] * c
        blocks[dst] = contrib if dst not in blocks else blocks[dst] + contrib
    n = len(block_order(new))
    assert len(blocks) == n, "plan does not fill every target block"
    return Tensor(new, [np.ascontiguousarray(blocks[i]) for i in range(n)])


def transpose(t: Tensor, axes) -> Tensor:
    axes = tuple(axes)
    new, terms = permutation_plan(t.structure, axes)
    return _execute(t, new, axes, terms)


def repartition(t: Tensor, outputs, inputs) -> Tensor:
    outputs, inputs = tuple(outputs), tuple(inputs)
    want = {ax: OUT for ax in outputs} | {ax: IN for ax in inputs}
    if not any(t.legs[ax].side != want[ax] for ax in range(t.ndim)):
        return transpose(t, (*outputs, *inputs))
    new, perm, terms = repartition_plan(t.structure, outputs, inputs)
    return _execute(t, new, perm, terms)


def adjoint(t: Tensor) -> Tensor:
    """Legs flip side, block ``(ot, it)`` <- conj of ``(it, ot)`` (``ops/map.py:418-493``)."""
    s = t.structure
    new = Structure(s.provider, tuple(replace(leg, side=IN if leg.side == OUT else OUT)
                                      for leg in s.legs))
    idx = index_map(s)
    return Tensor(new, [np.conj(t.blocks[idx[(it, ot)]]) for ot, it in block_order(new)])


# ---------------------------------------------------------------------------------------
# coupled-sector lowering and composition  (map_view.py, ops/map.py)


@cache
def map_layout(s: Structure):
    """Per coupled sector: sorted row trees and column trees with offsets/extents
    (``map_view.py:154-219``)."""
    p = s.provider
    rows: dict = {}
    cols: dict = {}
    for ot, it in block_order(s):
        rows.setdefault(ot[2], {})[ot] = None
        cols.setdefault(ot[2], {})[it] = None

    def bands(axes, trees):
        out, off = [], 0
        for tr in trees:
            ext = 1
            for ax, u in zip(axes, tr[0]):
                ext *= s.legs[ax].degeneracy(fused(p, s.legs[ax], u))
            out.append((tr, off, ext))
            off += ext
        return out, off

    layout = {}
    for c in sorted(rows):
        rb, nr = bands(s.out_axes, rows[c])
        cb, nc = bands(s.in_axes, cols[c])
        layout[c] = (rb, cb, nr, nc)
    return layout


def to_matrices(t: Tensor) -> dict:
    s = t.structure
    order = (*s.out_axes, *s.in_axes)
    idx = index_map(s)
    mats = {}
    for c, (rb, cb, nr, nc) in map_layout(s).items():
        m = np.zeros((nr, nc))
        for ot, ro, dr in rb:
            for it, co, dc in cb:
                m[ro:ro + dr, co:co + dc] = np.transpose(t.blocks[idx[(ot, it)]], order).reshape(dr, dc)
        mats[c] = m
    return mats


def from_matrices(s: Structure, mats: dict) -> Tensor:
    order = (*s.out_axes, *s.in_axes)
    inverse = tuple(sorted(range(len(order)), key=order.__getitem__))
    idx = index_map(s)
    blocks = [None] * len(block_order(s))
    for c, (rb, cb, nr, nc) in map_layout(s).items():
        for ot, ro, dr in rb:
            for it, co, dc in cb:
                i = idx[(ot, it)]
                shape = block_shape(s, (ot, it))
                piece = mats[c][ro:ro + dr, co:co + dc].reshape(tuple(shape[a] for a in order))
                blocks[i] = np.ascontiguousarray(np.transpose(piece, inverse))
    return Tensor(s, blocks)


#: Running total of the sector products' flops (2 M K N each) that ``compose`` performed:
#: the algorithmic work of a contraction, read by the benchmark's CPU legs.
FLOPS = [0]


def compose(a: Tensor, b: Tensor) -> Tensor:
    """One matmul per shared coupled sector, zero elsewhere (``ops/map.py:155-172``)."""
    s = Structure(a.structure.provider, (*a.structure.codomain, *b.structure.domain))
    ma, mb = to_matrices(a), to_matrices(b)
    mats = {}
    for c, (_, _, nr, nc) in map_layout(s).items():
        if c in ma and c in mb:
            mats[c] = ma[c] @ mb[c]
            FLOPS[0] += 2 * nr * nc * ma[c].shape[1]
        else:
            mats[c] = np.zeros((nr, nc))
    return from_matrices(s, mats)


# ---------------------------------------------------------------------------------------
# contraction  (ops/contraction.py)


def outward_dual(leg: Leg) -> bool:
    return leg.dual != (leg.side == IN)


def contraction_plan(a: Structure, b: Structure, axes):
    """``ops/contraction.py:247-306``: free legs return unchanged."""
    ca, cb = tuple(axes[0]), tuple(axes[1])
    for i, j in zip(ca, cb):
        x, y = a.legs[i], b.legs[j]
        if x.sectors != y.sectors or outward_dual(x) == outward_dual(y):
            raise ValueError(f"tensordot: axis {i} of a and axis {j} of b do not contract")
    fa = tuple(i for i in range(len(a.legs)) if i not in ca)
    fb = tuple(j for j in range(len(b.legs)) if j not in cb)
    free = (*(a.legs[i] for i in fa), *(b.legs[j] for j in fb))
    outputs = tuple(k for k, leg in enumerate(free) if leg.side == OUT)
    inputs = tuple(k for k, leg in enumerate(free) if leg.side == IN)
    position = {k: q for q, k in enumerate((*outputs, *inputs))}
    return fa, ca, cb, fb, outputs, inputs, tuple(position[k] for k in range(len(free)))


def tensordot(a: Tensor, b: Tensor, axes) -> Tensor:
    """``repartition -> compose -> repartition -> transpose`` (``ops/contraction.py:309-376``)."""
    fa, ca, cb, fb, ro, ri, ft = contraction_plan(a.structure, b.structure, axes)
    c = compose(repartition(a, fa, ca), repartition(b, cb, fb))
    return transpose(repartition(c, ro, ri), ft)


def einsum(equation: str, *ops: Tensor) -> Tensor:
    """One- and two-operand ``einsum`` (``ops/contraction.py:695-794``)."""
    lhs, out = equation.replace(" ", "").split("->")
    terms = lhs.split(",")
    if len(ops) == 1:
        return transpose(ops[0], tuple(terms[0].index(x) for x in out))
    if len(ops) > 2:
        # three or more operands: pairwise, left to right (a valid contraction path; the
        # reference's order comes from opt_einsum and differs only in rounding here)
        acc, at = ops[0], terms[0]
        for k in range(1, len(ops)):
            later = set(out).union(*map(set, terms[k + 1:]))
            mid = "".join([x for x in at if x in later] + [x for x in terms[k] if x in later])
            acc = einsum(f"{at},{terms[k]}->{mid}", acc, ops[k])
            at = mid
        return transpose(acc, tuple(at.index(x) for x in out))
    shared = [x for x in terms[0] if x in terms[1]]
    axes = (tuple(terms[0].index(x) for x in shared), tuple(terms[1].index(x) for x in shared))
    free = [x for x in terms[0] if x not in shared] + [x for x in terms[1] if x not in shared]
    return transpose(tensordot(ops[0], ops[1], axes), tuple(free.index(x) for x in out))


def composed(equation: str, a: Tensor, b: Tensor, bend: str = "") -> Tensor:
    """Two-operand einsum with named wires bent first (``network/env.py:60-90``)."""
    if bend:
        lhs, out = equation.split("->")
        ta, tb = lhs.split(",")

        def bent(t, term):
            flip = set(bend)
            outs = tuple(i for i, ch in enumerate(term) if (t.legs[i].side == OUT) != (ch in flip))
            ins = tuple(i for i in range(len(term)) if i not in outs)
            return repartition(t, outs, ins), "".join(term[i] for i in (*outs, *ins))

        a, ta = bent(a, ta)
        b, tb = bent(b, tb)
        equation = f"{ta},{tb}->{out}"
    return einsum(equation, a, b)


# ---------------------------------------------------------------------------------------
# vector space  (ops/basic.py, ops/contraction.py:517-589)


def inner(a: Tensor, b: Tensor) -> float:
    p = a.structure.provider
    return float(sum(p.qdim(k[0][2]) * np.sum(np.conj(x) * y)
                     for k, x, y in zip(block_order(a.structure), a.blocks, b.blocks)))


def norm(t: Tensor) -> float:
    p = t.structure.provider
    return float(np.sqrt(sum(p.qdim(k[0][2]) * np.sum(np.abs(x) ** 2)
                             for k, x in zip(block_order(t.structure), t.blocks))))


def axpby(alpha: float, x: Tensor, beta: float, y: Tensor) -> Tensor:
    return Tensor(x.structure, [alpha * a + beta * b for a, b in zip(x.blocks, y.blocks)])


def scale(t: Tensor, s: float) -> Tensor:
    return Tensor(t.structure, [b * s for b in t.blocks])


# ---------------------------------------------------------------------------------------
# truncated blockwise SVD  (ops/linalg.py)


def _admissible(spectrum, qdim, cutoff, mode) -> int:
    """``ops/linalg.py:1100-1129``."""
    if cutoff is None:
        return len(spectrum)
    if mode == "abs":
        return sum(1 for sg, _, _ in spectrum if sg > cutoff)
    if mode == "rel":
        th = cutoff * spectrum[0][0]
        return sum(1 for sg, _, _ in spectrum if sg > th)
    power = 2 if mode in ("sum2", "rsum2") else 1
    weights = [qdim(c) * sg ** power for sg, c, _ in spectrum]
    th = cutoff * sum(weights) if mode.startswith("r") else cutoff
    kept, dropped = len(spectrum), 0.0
    for w in reversed(weights):
        if dropped + w >= th:
            break
        dropped += w
        kept -= 1
    return kept


def decide(spectrum, p: Provider, max_bond, cutoff, mode="rsum2"):
    """The keep rule (``ops/linalg.py:1274-1324``): returns ``{sector: kept count}``."""
    adm = _admissible(spectrum, p.qdim, cutoff, mode)
    keep: dict = {}
    dense = 0.0
    for sg, c, _ in spectrum[:adm]:
        if max_bond is not None and dense + p.qdim(c) > max_bond:
            break
        dense += p.qdim(c)
        keep[c] = keep.get(c, 0) + 1
    return keep


def svd_truncated(t: Tensor, axes, *, max_bond=None, cutoff=None, cutoff_mode="rsum2"):
    """``ops/linalg.py:1441-1612``; returns ``(U, S, Vh)``."""
    m = repartition(t, tuple(axes[0]), tuple(axes[1]))
    p = m.structure.provider
    mats = to_matrices(m)
    parts = {c: np.linalg.svd(b, full_matrices=False) for c, b in mats.items()}
    spectrum = [(float(sg), c, i) for c, pr in parts.items() for i, sg in enumerate(pr[1])]
    spectrum.sort(key=lambda e: (-e[0], e[1], e[2]))
    keep = decide(spectrum, p, max_bond, cutoff, cutoff_mode)
    bond = tuple(sorted(keep.items()))
    su = Structure(p, (*m.structure.codomain, Leg(bond, IN)))
    ss = Structure(p, (Leg(bond, OUT), Leg(bond, IN)))
    sv = Structure(p, (Leg(bond, OUT), *m.structure.domain))
    return (from_matrices(su, {c: parts[c][0][:, :k] for c, k in keep.items()}),
            from_matrices(ss, {c: np.diag(parts[c][1][:k]) for c, k in keep.items()}),
            from_matrices(sv, {c: parts[c][2][:k, :] for c, k in keep.items()}))


# ---------------------------------------------------------------------------------------
# two-site effective Hamiltonian and Lanczos  (network/env.py, network/dmrg.py)


def heff2(fl: Tensor, w1: Tensor, w2: Tensor, fr: Tensor, aa: Tensor) -> Tensor:
    """Site-tensor matvec, four pairwise contractions (``network/env.py:416-432``)."""
    t = einsum("apqr,rys->apqys", aa, fr)
    t = composed("apqys,mQqy->apQms", t, w2, bend="q")
    t = composed("apQms,xPpm->aPQxs", t, w1, bend="p")
    return composed("aPQxs,axB->BPQs", t, fl, bend="a")


def env_update_last(f: Tensor, a: Tensor, w: Tensor) -> Tensor:
    """``F[(n, n+1)]`` from ``F[(n-1, n)]`` (``network/env.py:620-625``), bra = ket."""
    bra = adjoint(a)
    t = einsum("axB,apr->xBpr", f, a)
    t = einsum("xPpm,xBpr->BrPm", w, t)
    return einsum("BPs,BrPm->rms", bra, t)


def env_update_first(f: Tensor, a: Tensor, w: Tensor) -> Tensor:
    """``F[(n, n-1)]`` from ``F[(n+1, n)]`` (``network/env.py:626-629``), bra = ket."""
    bra = adjoint(a)
    t = einsum("apr,rys->apys", a, f)
    t = composed("apys,xPpy->axPs", t, w, bend="p")
    return composed("axPs,BPs->axB", t, bra, bend="P")


def lanczos(matvec, v: Tensor, *, ncv: int = 3, tol: float = 1e-13):
    """Three-term recurrence, no reorthogonalisation (``network/dmrg.py:106-227``)."""
    vecs = [scale(v, 1.0 / norm(v))]
    alphas, betas = [], []
    for j in range(ncv):
        w = matvec(vecs[j])
        alphas.append(inner(vecs[j], w))
        w = axpby(1.0, w, -alphas[j], vecs[j])
        if j:
            w = axpby(1.0, w, -betas[j - 1], vecs[j - 1])
        beta = norm(w)
        if j + 1 == ncv or beta < tol:
            break
        betas.append(beta)
        vecs.append(scale(w, 1.0 / beta))
    tri = np.diag(alphas) + np.diag(betas, 1) + np.diag(betas, -1)
    values, states = np.linalg.eigh(tri)
    g = states[:, 0]
    out = scale(vecs[0], float(g[0]))
    for k in range(1, len(vecs)):
        out = axpby(1.0, out, float(g[k]), vecs[k])
    return float(values[0]), scale(out, 1.0 / norm(out))


# ---------------------------------------------------------------------------------------
# the two-site DMRG driver  (network/mps.py:312-352, network/env.py:506-633,
# network/dmrg.py:321-843, noiseless flat-chi branch)


def heisenberg_mpo_su2(n_sites: int, j: float = 1.0) -> list:
    """The site tensors of ``MPO.from_terms(L, [(j, [(S.S, (i, i + 1))])]).materialize()``
    on spin-1/2 SU(2) sites (``network/mps.py:3135-3341``, ``models/sites.py:121-195``): MPO
    bond channels "start" (2j = 0), "open" (2j = 2, the split ``S.S``'s first factor) and
    "done" (2j = 0); in the fusion-tree basis the reduced coefficients are 1 on the
    identity channels, ``sqrt(3/2)`` to open and ``-sqrt(3/8) j`` to close (their
    product ``-3/4 j`` is the reduced ``S.S``).  Legs ``(x IN*, P OUT, p IN, m OUT*)``."""
    phys = ((1, 1),)

    def states(b):
        if b == 0:
            return [("start", 0)]
        if b == n_sites:
            return [("done", 0)]
        if b == 1:
            return [("start", 0), ("open", 2)]
        if b == n_sites - 1:
            return [("done", 0), ("open", 2)]
        return [("start", 0), ("done", 0), ("open", 2)]

    def leg(st, side):
        count: dict = {}
        for _, a in st:
            count[a] = count.get(a, 0) + 1
        return Leg(tuple(sorted(count.items())), side, True)

    def index(st, label):
        a = dict(st)[label]
        return a, [x for x, b in st if b == a].index(label)

    rules = [("start", "start", 1.0), ("done", "done", 1.0), ("start", "open", np.sqrt(1.5)),
             ("open", "done", -np.sqrt(3.0 / 8.0) * j)]
    out = []
    for n in range(n_sites):
        sl, sr = states(n), states(n + 1)
        s = Structure(SU2, (leg(sl, IN), Leg(phys, OUT), Leg(phys, IN), leg(sr, OUT)))
        blocks = []
        for key in block_order(s):
            (ps, ms), _, c = key[0]
            (xs, _), _, _ = key[1]
            blk = np.zeros(block_shape(s, key))
            if c == 1:
                for a, b, v in rules:
                    if a in dict(sl) and b in dict(sr):
                        (xa, xi), (mb, mi) = index(sl, a), index(sr, b)
                        if xa == xs and mb == ms:
                            blk[xi, 0, 0, mi] = v
            blocks.append(blk)
        out.append(Tensor(s, blocks))
    return out


def lq(t: Tensor, outputs, inputs):
    """Reduced LQ per coupled sector (``ops/linalg.py:549-620``): ``(L, Q)`` with the new
    bond IN on ``L`` and OUT on ``Q``, of degeneracy ``min(rows, cols)``."""
    m = repartition(t, tuple(outputs), tuple(inputs))
    p = m.structure.provider
    mats = to_matrices(m)
    parts = {}
    for c, b in mats.items():
        q, r = np.linalg.qr(b.T)
        parts[c] = (r.T, q.T)
    bond = tuple(sorted((c, min(b.shape)) for c, b in mats.items()))
    sl = Structure(p, (*m.structure.codomain, Leg(bond, IN)))
    sq = Structure(p, (Leg(bond, OUT), *m.structure.domain))
    return (from_matrices(sl, {c: v[0] for c, v in parts.items()}),
            from_matrices(sq, {c: v[1] for c, v in parts.items()}))


def _site(t: Tensor) -> Tensor:
    """The MPS write barrier: a site tensor on ``(l, p | r)`` (``network/mps.py:126-143``)."""
    return repartition(t, (0, 1), (2,))


def canonize(psi: list) -> list:
    """Right-canonical form by one LQ per site from the right (``network/mps.py:312-352``)."""
    psi = list(psi)
    for n in range(len(psi) - 1, 0, -1):
        left, q = lq(psi[n], (0,), (1, 2))
        psi[n] = _site(q)
        psi[n - 1] = _site(einsum("apx,xy->apy", psi[n - 1], left))
    psi[0] = scale(psi[0], 1.0 / norm(psi[0]))
    return psi


def dmrg(psi: list, h: list, *, chi: int, cutoff: float, ncv: int, max_sweeps: int,
         energy_tol: float = 1e-12, schmidt_tol: float = 1e-8, on_sweep=None):
    """Two-site DMRG (``network/dmrg.py:321-843``, no noise, flat ``chi`` / ``cutoff``):
    canonise, build the environments towards site 0, sweep right then left solving each
    bond by ``lanczos`` and splitting by ``svd_truncated``, stop when both the energy and
    the worst Schmidt change fall under their tolerances.  ``psi`` and ``h`` are lists of
    site tensors; returns ``(energy per sweep, final psi)``.  ``on_sweep(k, psi, energy)``
    is called after each sweep."""
    n_sites = len(psi)
    psi = canonize(psi)
    kl, kr = psi[0].structure.legs[0], psi[-1].structure.legs[2]
    wl, wr = h[0].structure.legs[0], h[-1].structure.legs[3]
    p = psi[0].structure.provider
    F = {(-1, 0): ones(Structure(p, (Leg(kl.sectors, IN, kl.dual), Leg(wl.sectors, OUT, wl.dual),
                                     Leg(kl.sectors, OUT, kl.dual)))),
         (n_sites, n_sites - 1): ones(Structure(p, (Leg(kr.sectors, OUT, kr.dual),
                                                    Leg(wr.sectors, IN, wr.dual),
                                                    Leg(kr.sectors, IN, kr.dual))))}
    for n in range(n_sites - 1, 0, -1):
        F[n, n - 1] = env_update_first(F[n + 1, n], psi[n], h[n])
    energies, schmidt, energy = [], {}, float("inf")
    for it in range(1, max_sweeps + 1):
        old_e, old_s = energy, dict(schmidt)
        for forward in (True, False):
            for n in (range(n_sites - 1) if forward else range(n_sites - 2, -1, -1)):
                aa = einsum("apx,xqr->apqr", psi[n], psi[n + 1])
                fl, fr = F[n - 1, n], F[n + 2, n + 1]
                energy, aa = lanczos(lambda v: heff2(fl, h[n], h[n + 1], fr, v), aa, ncv=ncv)
                u, s, vh = svd_truncated(aa, ((0, 1), (2, 3)), max_bond=chi, cutoff=cutoff)
                s = scale(s, 1.0 / norm(s))
                if forward:
                    psi[n], psi[n + 1] = _site(u), _site(einsum("xy,yqr->xqr", s, vh))
                else:
                    psi[n], psi[n + 1] = _site(einsum("apx,xy->apy", u, s)), _site(vh)
                schmidt[n] = corner_spectrum(s)
                F.pop((n, n - 1), None), F.pop((n, n + 1), None)
                F.pop((n + 1, n), None), F.pop((n + 1, n + 2), None)
                if forward:
                    F[n, n + 1] = env_update_last(F[n - 1, n], psi[n], h[n])
                else:
                    F[n + 1, n] = env_update_first(F[n + 2, n + 1], psi[n + 1], h[n + 1])
        energies.append(energy)
        if on_sweep is not None:
            on_sweep(it, psi, energy)
        if abs(old_e - energy) < energy_tol and _schmidt_change(old_s, schmidt) < schmidt_tol:
            break
    return energies, psi


def _schmidt_change(old: dict, new: dict) -> float:
    """Worst bond's zero-padded Schmidt-spectrum distance, infinite before any history
    (``network/dmrg.py:545-561``)."""
    if not old:
        return float("inf")
    worst = 0.0
    for n, cur in new.items():
        prev = old.get(n, [])
        m = max(len(prev), len(cur))
        a, b = prev + [0.0] * (m - len(prev)), cur + [0.0] * (m - len(cur))
        worst = max(worst, sum((x - y) ** 2 for x, y in zip(a, b)) ** 0.5)
    return worst


# ---------------------------------------------------------------------------------------
# JSON helpers for the golden vectors (tests/golden/make_golden.py writes this format)


def structure_from_json(legs_json) -> Structure:
    p = PROVIDERS[legs_json[0]["provider"]]
    legs = tuple(Leg(tuple((int(a), int(m)) for a, m in leg["sectors"]), leg["side"],
                     bool(leg["dual"])) for leg in legs_json)
    return Structure(p, legs)


def keys_from_json(keys_json) -> tuple:
    def tree(t):
        return (tuple(t[0]), tuple(t[1]), t[2])
    return tuple((tree(o), tree(i)) for o, i in keys_json)


# ---------------------------------------------------------------------------------------
# C4v CTMRG, single layer  (network/ctmrg.py:166-660, examples/toy_codes/ctmrg.py:547-592)


def identity_tensor(p: Provider, leg: Leg) -> Tensor:
    """``identity((leg,))``: legs ``(leg OUT, leg IN)``, eye per coupled sector
    (``ops/map.py:175-234``)."""
    s = Structure(p, (replace(leg, side=OUT), replace(leg, side=IN)))
    return from_matrices(s, {c: np.eye(nr) for c, (_, _, nr, nc) in map_layout(s).items()})


def ones(s: Structure) -> Tensor:
    return Tensor(s, [np.ones(block_shape(s, k)) for k in block_order(s)])


def ctm_seed(bulk: Tensor):
    """``init_env(bulk, Leg(bulk.legs[0].space, IN))`` (``network/ctmrg.py:337-385``)."""
    p = bulk.structure.provider
    unit = Leg(((p.unit(), 1),), OUT)
    c = identity_tensor(p, unit)
    e = ones(Structure(p, (Leg(unit.sectors, IN), Leg(unit.sectors, OUT),
                           Leg(bulk.legs[0].sectors, IN))))
    return c, e


def ctm_corner(c: Tensor, e: Tensor, bulk: Tensor) -> Tensor:
    """``einsum("ab,ace,fbg,gehi->chfi", c, e, e, bulk)`` (``network/ctmrg.py:238-244``),
    contracted left to right."""
    t = einsum("ab,ace->bce", c, e)
    t = einsum("bce,fbg->cefg", t, e)
    return einsum("cefg,gehi->chfi", t, bulk)


def ctm_edge(e: Tensor, p: Tensor, bulk: Tensor) -> Tensor:
    """``network/ctmrg.py:246-253``."""
    big = einsum("abe,gehi->abghi", e, bulk)
    t = einsum("abghi,agx->bhix", big, p)
    return einsum("bhix,bhy->xyi", t, adjoint(p))


def ctm_move(c: Tensor, e: Tensor, bulk: Tensor, chi: int):
    """One C4v move (``network/ctmrg.py:451-526``): new corner = the singular values."""
    big = ctm_corner(c, e, bulk)
    p, s, _ = svd_truncated(big, ((0, 1), (2, 3)), max_bond=chi)
    new_e = ctm_edge(e, p, bulk)
    return scale(s, 1.0 / norm(s)), scale(new_e, 1.0 / norm(new_e)), p.structure.legs[-1].sectors


def corner_spectrum(s: Tensor) -> list:
    """Diagonal values times sqrt(qdim), descending (``network/common.py:147-194``)."""
    p = s.structure.provider
    out = []
    for c, m in to_matrices(s).items():
        out.extend(float(v) * p.qdim(c) ** 0.5 for v in np.diag(m))
    return sorted(out, reverse=True)


def _spectrum_change(old, new) -> float:
    n = max(len(old), len(new))
    a = np.array(list(old) + [0.0] * (n - len(old)))
    b = np.array(list(new) + [0.0] * (n - len(new)))
    return float(np.abs(a - b).max()) if n else 0.0


def ctmrg(bulk: Tensor, *, chi: int, tol: float, max_sweeps: int):
    """The move loop to a corner-spectrum tolerance (``network/ctmrg.py:572-660``)."""
    c, e = ctm_seed(bulk)
    prev, history, bond = corner_spectrum(c), [], None
    for _ in range(max_sweeps):
        c, e, bond = ctm_move(c, e, bulk, chi)
        cur = corner_spectrum(c)
        history.append(_spectrum_change(prev, cur))
        prev = cur
        if history[-1] < tol:
            break
    return c, e, bond, history


def full_trace(t: Tensor) -> float:
    """``sum_c qdim(c) tr(M_c)`` (``ops/contraction.py:440-514``)."""
    p = t.structure.provider
    return float(sum(p.qdim(c) * np.trace(m) for c, m in to_matrices(t).items()))


def beta_free_energy(c: Tensor, e: Tensor, bulk: Tensor) -> float:
    """``beta f = -ln kappa``, Baxter's corner-transfer ratio on the converged environment
    (``examples/toy_codes/ctmrg.py:547-592`` with no unrolled moves)."""
    cc, ca, ec, ea = c, adjoint(c), e, adjoint(e)
    z_c = full_trace(einsum("ab,ac,dc,eb->de", cc, ca, cc, ca))
    z_h = full_trace(einsum("ab,ac,dcf,ed,eg,ghf->hb", cc, ca, ea, cc, ca, ec))
    z_a = full_trace(einsum("ab,acp,cd,edq,fe,gfr,gh,hks,spqr->kb",
                            cc, ec, ca, ea, cc, ea, ca, ec, bulk))
    return -float(np.log(z_a * z_c / z_h ** 2))


def onsager_beta_f(beta: float, n: int = 20001) -> float:
    """Onsager's exact ``beta f`` of the square-lattice Ising model (J = 1, no field), the
    value ``examples/toy_codes/ctmrg.py``'s ``onsager`` quotes:
    ``-beta f = ln(2 cosh 2b) + (1/2pi) int_0^pi ln[(1 + sqrt(1 - k^2 sin^2 t)) / 2] dt``
    with ``k = 2 sinh 2b / cosh^2 2b``, the integral by Simpson's rule on ``n`` points."""
    k = 2.0 * np.sinh(2.0 * beta) / np.cosh(2.0 * beta) ** 2
    t = np.linspace(0.0, np.pi, n)
    f = np.log((1.0 + np.sqrt(np.maximum(0.0, 1.0 - (k * np.sin(t)) ** 2))) / 2.0)
    h = t[1] - t[0]
    integral = h / 3.0 * (f[0] + f[-1] + 4.0 * f[1:-1:2].sum() + 2.0 * f[2:-1:2].sum())
    return -float(np.log(2.0 * np.cosh(2.0 * beta)) + integral / (2.0 * np.pi))
