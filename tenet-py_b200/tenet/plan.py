"""Array-free plans: the block maps of transpose, bend, repartition and adjoint.

A block map is ``(perm, terms)``: every destination block ``dst`` equals
``sum coeff * transpose(src_block, perm)`` over its terms ``(src, dst, coeff)``.  The
maps are computed once per degeneracy-free pattern and cached, as the reference does
(``ops/permutation.py:137-197``, ``ops/repartition.py:117-385``).  Coefficients are
exact FP64 scalars: 1 for U(1)/Z2, the Koszul sign for fZ2, and for SU(2) sums of
F * R * F products over Artin generators and ``sqrt(d_c/d_a) * B`` bends.
"""

from __future__ import annotations

from functools import cache
from math import sqrt

import numpy as np

from tenet import _su2
from tenet.structure import IN, OUT, Leg, Pattern, TensorStructure, all_trees, block_keys, \
    coupled_of, key_index, trees_to
from tenet.symmetry import CapabilityError, Provider

# ---------------------------------------------------------------------------------------
# tree moves


def _spine(tree) -> tuple[int, ...]:
    u, inner, c = tree
    if not u:
        return ()
    if len(u) == 1:
        return (c,)
    return (u[0], *inner, c)


def _unique(p: Provider, uncoupled: tuple, coupled: int):
    ts = trees_to(p, uncoupled, coupled)
    if len(ts) != 1:
        raise CapabilityError(f"{p.name}: {uncoupled} -> {coupled} has {len(ts)} trees")
    return ts[0]


def _koszul(uncoupled, perm) -> float:
    """``(-1)^(odd-odd inversions)`` (``symmetry/fz2.py:91-130``)."""
    odd = [i for i in perm if uncoupled[i] & 1]
    inv = 0
    for j in range(len(odd)):
        for k in range(j + 1, len(odd)):
            inv += odd[j] > odd[k]
    return -1.0 if inv & 1 else 1.0


@cache
def _swap(p: Provider, tree, i: int) -> tuple:
    """Artin generator on lines i, i+1 of an SU(2) tree (``symmetry/base.py:898-996``)."""
    u, inner, c = tree
    sp = _spine(tree)
    nu = (*u[:i], u[i + 1], u[i], *u[i + 2:])
    if i == 0:
        return (((nu, inner, c), float(_su2.r_symbol(u[0], u[1], sp[1]))),)
    a, b, cc, e, f = sp[i - 1], u[i], u[i + 1], sp[i], sp[i + 1]
    out = []
    for ne in p._fuse(a, cc):
        if f not in p._fuse(ne, b):
            continue
        coeff = 0.0
        for d in p._fuse(b, cc):
            coeff += (_su2.f_symbol(a, b, cc, f, e, d) * _su2.r_symbol(b, cc, d)
                      * _su2.f_symbol(a, cc, b, f, ne, d))
        out.append(((nu, (*inner[: i - 1], ne, *inner[i:]), c), coeff))
    return tuple(out)


@cache
def permute_tree(p: Provider, tree, perm: tuple[int, ...]) -> tuple:
    """Expansion of a tree with permuted uncoupled lines over canonical trees."""
    u, _, c = tree
    if p.abelian:
        nt = _unique(p, tuple(u[i] for i in perm), c)
        return ((nt, _koszul(u, perm) if p.fermionic else 1.0),)
    terms = {tree: 1.0}
    cur = list(range(len(u)))
    for j, target in enumerate(perm):
        for i in range(cur.index(target) - 1, j - 1, -1):
            cur[i], cur[i + 1] = cur[i + 1], cur[i]
            nxt: dict = {}
            for t, cf in terms.items():
                for bt, cb in _swap(p, t, i):
                    nxt[bt] = nxt.get(bt, 0.0) + cf * cb
            terms = nxt
    return tuple(terms.items())


def _bend_key(p: Provider, key, right: bool, dual: bool) -> tuple:
    """Move the last line of one tree onto the end of the other
    (``symmetry/base.py:999-1190``)."""
    ot, it = key
    src, dst = (ot, it) if right else (it, ot)
    if not src[0]:
        raise ValueError("cannot bend from an empty tree")
    b = src[0][-1]
    if p.abelian:
        rem = src[0][:-1]
        cs = coupled_of(p, rem)
        if len(cs) != 1:
            raise CapabilityError(f"{p.name}: non-unique coupled sector after a bend")
        nsrc = _unique(p, rem, cs[0])
        ndst = _unique(p, (*dst[0], p._dual(b)), cs[0])
        coeff = 1.0
    else:
        c = src[2]
        a = _spine(src)[-2] if len(src[0]) >= 2 else 0
        nsrc = (src[0][:-1], src[1][:-1], a)
        scale = sqrt(p._qdim(c) / p._qdim(a))
        if dual:
            scale *= p._fs(p._dual(b))
        ndst = ((*dst[0], p._dual(b)), _spine(dst)[1:], a)
        coeff = scale * _su2.b_symbol(a, b, c)
    return (((nsrc, ndst) if right else (ndst, nsrc), coeff),)


# ---------------------------------------------------------------------------------------
# pattern-level block maps


def _legs_pattern(p: Provider, legs) -> Pattern:
    return Pattern(p, tuple(legs))


def _side_perm(axes, old_side, new_side) -> tuple[int, ...]:
    pos = {old: j for j, old in enumerate(old_side)}
    return tuple(pos[axes[i]] for i in new_side)


@cache
def permutation_map(pat: Pattern, axes: tuple[int, ...]):
    """``(new pattern, terms)`` of a public transpose (``ops/permutation.py:159-197``)."""
    new = _legs_pattern(pat.provider, tuple(pat.legs[i] for i in axes))
    op = _side_perm(axes, pat.out_axes, new.out_axes)
    ip = _side_perm(axes, pat.in_axes, new.in_axes)
    keys = block_keys(pat)
    if op == tuple(range(len(op))) and ip == tuple(range(len(ip))):
        return new, tuple((i, i, 1.0) for i in range(len(keys)))
    p = pat.provider
    idx = key_index(new)
    terms = []
    for src, (ot, it) in enumerate(keys):
        for ot2, c1 in permute_tree(p, ot, op):
            for it2, c2 in permute_tree(p, it, ip):
                cf = c1 * c2
                if cf != 0:
                    terms.append((src, idx[(ot2, it2)], cf))
    return new, tuple(terms)


@cache
def bend_map(pat: Pattern, axis: int):
    """Bend the last leg of its side (``ops/repartition.py:134-183``)."""
    labels, is_out, dual = pat.legs[axis]
    moved = (labels, not is_out, not dual)
    new = _legs_pattern(pat.provider, (*(x for i, x in enumerate(pat.legs) if i != axis), moved))
    idx = key_index(new)
    terms = []
    for src, key in enumerate(block_keys(pat)):
        for nk, cf in _bend_key(pat.provider, key, is_out, dual):
            if cf != 0:
                terms.append((src, idx[nk], cf))
    return new, tuple(terms)


def compose_terms(terms, following) -> np.ndarray:
    """Sparse product of two block maps, duplicates summed (``ops/repartition.py:298-316``).

    Terms are ``(src, dst, coeff)`` rows.  The result lists each ``(src, dst)`` pair once,
    in order of its first occurrence when the terms of ``terms`` are walked in order and
    each is followed through the terms of ``following`` in their order; each coefficient
    is summed in that same order, starting from zero (the library's host planner,
    ``tnb_plan_compose``)."""
    from tenet import _lib

    a = np.ascontiguousarray(terms, dtype=np.float64).reshape(-1, 3)
    b = np.ascontiguousarray(following, dtype=np.float64).reshape(-1, 3)
    if not len(a) or not len(b):
        return np.zeros((0, 3))
    per_mid = np.bincount(b[:, 0].astype(np.int64))
    mid = a[:, 1].astype(np.int64)
    cap = int(per_mid[mid[mid < len(per_mid)]].sum())
    out = np.empty((max(cap, 1), 3))
    n = _lib.load().tnb_plan_compose(len(a), a.ctypes.data, len(b), b.ctypes.data,
                                     out.ctypes.data, cap)
    if n < 0:
        raise RuntimeError(f"tnb_plan_compose failed ({n})")
    return out[:n]


@cache
def repartition_map(pat: Pattern, outputs: tuple, inputs: tuple):
    """``(new pattern, perm, terms)`` of the transpose/bend/transpose chain
    (``ops/repartition.py:341-385``)."""
    nd = len(pat.legs)
    want = {ax: True for ax in outputs} | {ax: False for ax in inputs}
    crossing = [ax for ax in range(nd) if pat.legs[ax][1] != want[ax]]
    perm = tuple(range(nd))
    n = len(block_keys(pat))
    terms = np.stack([np.arange(n), np.arange(n), np.ones(n)], axis=1).astype(np.float64)
    labels = list(range(nd))
    cur = pat
    for ax in crossing:
        q = labels.index(ax)
        axes = tuple(i for i in range(nd) if i != q) + (q,)
        cur, t = permutation_map(cur, axes)
        perm = tuple(perm[i] for i in axes)
        terms = compose_terms(terms, t)
        labels.append(labels.pop(q))
        cur, t = bend_map(cur, nd - 1)
        terms = compose_terms(terms, t)
    pos = {a: q for q, a in enumerate(labels)}
    axes = tuple(pos[ax] for ax in (*outputs, *inputs))
    cur, t = permutation_map(cur, axes)
    return cur, tuple(perm[i] for i in axes), compose_terms(terms, t)


@cache
def adjoint_map(pat: Pattern):
    """Block ``(ot, it)`` of the adjoint is block ``(it, ot)`` (``ops/map.py:418-443``)."""
    new = _legs_pattern(pat.provider, tuple((lab, not o, d) for lab, o, d in pat.legs))
    idx = key_index(pat)
    return new, tuple((idx[(it, ot)], j, 1.0) for j, (ot, it) in enumerate(block_keys(new)))


# ---------------------------------------------------------------------------------------
# structure-level wrappers: new legs carry spaces/names; maps come from the pattern


def _on_side(leg: Leg, side) -> Leg:
    return leg if leg.side is side else Leg(leg.space, side, not leg.dual, leg.name)


@cache
def transpose_plan(s: TensorStructure, axes: tuple):
    _, terms = permutation_map(s.pattern, axes)
    return TensorStructure(tuple(s.legs[i] for i in axes)), axes, terms


@cache
def repartition_plan(s: TensorStructure, outputs: tuple, inputs: tuple):
    want = {ax: OUT for ax in outputs} | {ax: IN for ax in inputs}
    if not any(s.legs[ax].side is not want[ax] for ax in range(s.ndim)):
        return transpose_plan(s, (*outputs, *inputs))
    _, perm, terms = repartition_map(s.pattern, outputs, inputs)
    legs = tuple(_on_side(s.legs[ax], want[ax]) for ax in (*outputs, *inputs))
    return TensorStructure(legs), perm, terms


@cache
def adjoint_plan(s: TensorStructure):
    _, terms = adjoint_map(s.pattern)
    legs = tuple(Leg(l.space, IN if l.side is OUT else OUT, l.dual, l.name) for l in s.legs)
    return TensorStructure(legs), tuple(range(s.ndim)), terms


def chain(first, second):
    """Compose two structure-level plans: apply ``first`` then ``second``."""
    s1, p1, t1 = first
    s2, p2, t2 = second
    return s2, tuple(p1[i] for i in p2), compose_terms(t1, t2)


def validate_axes(ndim: int, axes) -> tuple[int, ...]:
    axes = tuple(int(a) for a in axes)
    if sorted(axes) != list(range(ndim)):
        raise ValueError(f"transpose: axes {axes} is not a permutation of range({ndim})")
    return axes


def validate_partition(ndim: int, outputs, inputs) -> tuple[tuple, tuple]:
    outputs, inputs = tuple(int(a) for a in outputs), tuple(int(a) for a in inputs)
    if sorted(outputs + inputs) != list(range(ndim)):
        raise ValueError(f"repartition: {outputs} + {inputs} is not a permutation of range({ndim})")
    return outputs, inputs


__all__ = ["adjoint_plan", "all_trees", "bend_map", "chain", "compose_terms", "permutation_map",
           "permute_tree", "repartition_map", "repartition_plan", "transpose_plan"]
