"""Tensor operations on the hot path, executed by the CUDA library.

Public names, argument meaning and refusals follow the reference's ``tenet.ops``:
``transpose`` (``ops/permutation.py:200-272``), ``repartition``
(``ops/repartition.py:388-476``), ``adjoint``/``compose`` (``ops/map.py``),
``tensordot``/``einsum``/``inner`` (``ops/contraction.py``), ``add``/``subtract``/
``multiply``/``divide``/``norm`` (``ops/basic.py``).  Every refusal is raised on the host
before any kernel is launched.

A pairwise contraction is three launches: one gather packs both operands straight into
their coupled-sector matrices (the reference's repartition + ``to_matrices``, fused), one
grouped GEMM multiplies every shared sector, and one gather scatters the product into
the output blocks (``from_matrices`` + the restoring repartition + the final transpose,
composed into a single block map).
"""

from __future__ import annotations

import operator
import threading
from collections import Counter
from contextlib import contextmanager
from dataclasses import dataclass
from functools import cache

import numpy as np
import torch

from tenet import _exec, _lib
from tenet.plan import adjoint_plan, chain, repartition_plan, transpose_plan, validate_axes, \
    validate_partition
from tenet.structure import IN, OUT, TensorStructure, layout, matrix_layout
from tenet.symmetry import CapabilityError
from tenet.tensor import SymmetricTensor

__all__ = ["add", "adjoint", "compose", "contractible", "divide", "einsum", "full_trace",
           "identity", "inner", "multiply", "norm", "outward_dual", "repartition", "subtract",
           "tensordot", "transpose"]


# ---------------------------------------------------------------------------------------
# unary block maps


@cache
def _map_exec(src: TensorStructure, kind: str, a=None, b=None):
    """``(destination structure, gather or None)`` of a cached unary block map: a
    transpose (``kind`` "t", axes ``a``), a repartition ("r", outputs ``a``, inputs ``b``)
    or the adjoint ("a").  ``None`` marks an identity map, whose result shares the arena."""
    plan = (transpose_plan(src, a) if kind == "t" else
            repartition_plan(src, a, b) if kind == "r" else adjoint_plan(src))
    dst, perm, terms = plan
    t = np.asarray(terms, dtype=np.float64).reshape(-1, 3)
    if perm == tuple(range(src.ndim)) and len(t) == dst.num_blocks \
            and (t[:, 0] == t[:, 1]).all() and (t[:, 2] == 1.0).all():
        return dst, None
    return dst, _exec.make_gather(_exec.gather_rows(src, "arena", dst, "arena", perm, terms))


def _apply_map(t: SymmetricTensor, kind: str, a=None, b=None) -> SymmetricTensor:
    dst, table = _map_exec(t.structure, kind, a, b)
    if table is None:
        return SymmetricTensor(dst, arena=t.arena)  # identity block map: share the arena
    out = SymmetricTensor.empty(dst)
    table.run(t.arena, out.arena)
    return out


def transpose(t: SymmetricTensor, axes=None) -> SymmetricTensor:
    """Public-axis permutation; within-side reorders are braids (``ops/permutation.py``)."""
    axes = tuple(reversed(range(t.ndim))) if axes is None else validate_axes(t.ndim, axes)
    return _apply_map(t, "t", axes)


def repartition(t: SymmetricTensor, outputs, inputs) -> SymmetricTensor:
    """``outputs`` become OUT, ``inputs`` IN, in that public order (``ops/repartition.py``)."""
    outputs, inputs = validate_partition(t.ndim, outputs, inputs)
    return _apply_map(t, "r", outputs, inputs)


def adjoint(t: SymmetricTensor) -> SymmetricTensor:
    """Every leg flips side; block ``(ot, it)`` <- block ``(it, ot)`` (``ops/map.py:446-493``)."""
    return _apply_map(t, "a")


# ---------------------------------------------------------------------------------------
# contraction


def outward_dual(leg) -> bool:
    return leg.dual != (leg.side is IN)


def contractible(x, y) -> bool:
    return x.space == y.space and outward_dual(x) != outward_dual(y)


def _validated_axes(a: TensorStructure, b: TensorStructure, axes):
    if hasattr(axes, "__index__"):
        n = operator.index(axes)
        if n < 0 or n > a.ndim or n > b.ndim:
            raise ValueError(f"tensordot: axes={n} is out of range")
        return tuple(range(a.ndim - n, a.ndim)), tuple(range(n))
    try:
        raw_a, raw_b = axes
    except (TypeError, ValueError) as exc:
        raise ValueError(f"tensordot: axes {axes!r} must be an integer or a pair") from exc
    parts = []
    for name, t, raw in (("a", a, raw_a), ("b", b, raw_b)):
        raw = (raw,) if hasattr(raw, "__index__") else raw
        got = tuple(operator.index(x) for x in raw)
        if len(set(got)) != len(got) or any(not 0 <= x < t.ndim for x in got):
            raise ValueError(f"tensordot: bad axes {got} for {name}")
        parts.append(got)
    if len(parts[0]) != len(parts[1]):
        raise ValueError("tensordot: contracted axes are paired in order; lengths differ")
    return tuple(parts)


@dataclass
class ContractionExec:
    """Cached device program of one pairwise contraction (``ops/contraction.py:247-376``)."""

    out: TensorStructure
    a_mat: int
    b_mat: int
    c_mat: int
    pack: _exec.GatherTable
    gemm: _exec.GemmTable
    unpack: _exec.GatherTable

    def run(self, a: torch.Tensor, b: torch.Tensor, out: torch.Tensor | None = None,
            scratch: tuple | None = None) -> torch.Tensor:
        dev = a.device
        if scratch is None:
            ap = torch.empty(self.a_mat, dtype=torch.float64, device=dev)
            bp = torch.empty(self.b_mat, dtype=torch.float64, device=dev)
            cp = torch.empty(self.c_mat, dtype=torch.float64, device=dev)
        else:
            ap, bp, cp = scratch
        if out is None:
            out = torch.empty(layout(self.out).size, dtype=torch.float64, device=dev)
        if self.pack._dev is None:  # first run: every table of this contraction at once
            _exec.upload_together((self.pack, *getattr(self.gemm, "parts", (self.gemm,)),
                                   self.unpack))
        self.pack.run(a, ap, b, bp)
        self.gemm.run(ap, bp, cp)
        self.unpack.run(cp, out)
        return out

    @property
    def flops(self) -> int:
        return self.gemm.flops


# per host thread: the arithmetic of the coupled-sector products of eager contractions,
# ("f64", None) or a tensor-core precision ("tf32" / "3xbf16") with its size rule
_PREC = threading.local()


def current_precision() -> tuple:
    """``(precision, tc_min_flops)`` of eager contractions on this thread."""
    return getattr(_PREC, "value", ("f64", None))


@contextmanager
def precision(kind: str = "f64", tc_min_flops: int | None = None):
    """Run the coupled-sector products of eager contractions (``tensordot``, ``einsum``)
    inside the block in ``kind``: "f64" (the plain form), or "tf32" / "3xbf16" on the
    tcgen05 tensor cores for the products of at least ``tc_min_flops`` (default
    ``_exec.TC_MIN_FLOPS``), FP64 in and out.  Gathers, SVDs and norms stay FP64."""
    if kind != "f64" and kind not in _exec.TC_KINDS:
        raise ValueError(f"unknown precision {kind!r}")
    prev = current_precision()
    _PREC.value = (kind, tc_min_flops)
    try:
        yield
    finally:
        _PREC.value = prev


@cache
def contraction_exec(sa: TensorStructure, sb: TensorStructure, axes, precision: str = "f64",
                     tc_min_flops: int | None = None, out_axes=None) -> ContractionExec:
    """Planned pairwise contraction.  ``out_axes`` (a permutation of the free legs) folds a
    final transpose into the unpack gather: the result comes out already permuted, the
    composed block map applied in one pass (as ``einsum`` needs)."""
    ca, cb = axes
    if sa.provider != sb.provider:
        raise ValueError("tensordot: operands have different providers")
    for k, (i, j) in enumerate(zip(ca, cb)):
        if not contractible(sa.legs[i], sb.legs[j]):
            raise ValueError(f"tensordot: pair {k}, axis {i} of a and axis {j} of b do not "
                             "contract (same space and opposite `dual xor (side is IN)` needed)")
    fa = tuple(i for i in range(sa.ndim) if i not in ca)
    fb = tuple(j for j in range(sb.ndim) if j not in cb)
    if not fa and not fb:
        raise ValueError("tensordot: this contraction leaves no free leg")
    free = (*(sa.legs[i] for i in fa), *(sb.legs[j] for j in fb))
    ro = tuple(k for k, leg in enumerate(free) if leg.side is OUT)
    ri = tuple(k for k, leg in enumerate(free) if leg.side is IN)
    pos = {k: q for q, k in enumerate((*ro, *ri))}
    ft = tuple(pos[k] for k in range(len(free)))

    sa2, perm_a, terms_a = repartition_plan(sa, fa, ca)
    sb2, perm_b, terms_b = repartition_plan(sb, cb, fb)
    sc = TensorStructure((*sa2.codomain, *sb2.domain))
    so, perm_u, terms_u = chain(repartition_plan(sc, ro, ri), transpose_plan(
        repartition_plan(sc, ro, ri)[0], ft))
    assert so.legs == free, "the restoring repartition must return the free legs unchanged"
    if out_axes is not None and tuple(out_axes) != tuple(range(len(free))):
        so, perm_u, terms_u = chain((so, perm_u, terms_u), transpose_plan(so, tuple(out_axes)))

    ma, mb, mc = matrix_layout(sa2), matrix_layout(sb2), matrix_layout(sc)
    products, used = [], set()
    for c in mc.sectors:
        M, N = mc.shape[c]
        if c in ma.shape and c in mb.shape:
            K = ma.shape[c][1]
            assert K == mb.shape[c][0] and ma.shape[c][0] == M and mb.shape[c][1] == N
            products.append((M, N, K, ma.base[c], K, mb.base[c], N, mc.base[c], N))
            used.add(c)
        else:
            products.append((M, N, 0, 0, 0, 0, N, mc.base[c], N))
    keep_a = [int(x) in used for x in ma.block_sector]
    keep_b = [int(x) in used for x in mb.block_sector]
    pack = _exec.make_gather(
        _exec.gather_rows(sa, "arena", sa2, "matrix", perm_a, terms_a, 0, keep_a),
        _exec.gather_rows(sb, "arena", sb2, "matrix", perm_b, terms_b, 1, keep_b))
    unpack = _exec.make_gather(_exec.gather_rows(sc, "matrix", so, "arena", perm_u, terms_u))
    return ContractionExec(so, ma.size, mb.size, mc.size, pack,
                           _exec.GemmGroup(products, precision, tc_min_flops), unpack)


def tensordot(a: SymmetricTensor, b: SymmetricTensor, axes, out_axes=None) -> SymmetricTensor:
    """Contract ``axes[0]`` of ``a`` with ``axes[1]`` of ``b``; free legs come back unchanged
    (or transposed by ``out_axes``, in the same pass)."""
    ex = contraction_exec(a.structure, b.structure, _validated_axes(a.structure, b.structure, axes),
                          *current_precision(), None if out_axes is None else tuple(out_axes))
    return SymmetricTensor(ex.out, arena=ex.run(a.arena, b.arena))


def compose(a: SymmetricTensor, b: SymmetricTensor) -> SymmetricTensor:
    """``a o b``: ``a``'s domain consumes ``b``'s codomain (``ops/map.py:105-172``)."""
    ia, ob = a.structure.in_axes, b.structure.out_axes
    if len(ia) != len(ob):
        raise ValueError("compose: a's domain and b's codomain have different lengths")
    for i, j in zip(ia, ob):
        x, y = a.legs[i], b.legs[j]
        if x.space != y.space or x.dual != y.dual:
            raise ValueError(f"compose: a's domain and b's codomain differ at axis {i} / {j}")
    return tensordot(a, b, (ia, ob))


def _parse(equation: str, n: int):
    if "." in equation:
        raise ValueError("einsum: ellipsis is not supported for symmetric tensors")
    lhs, arrow, rhs = equation.replace(" ", "").partition("->")
    terms = lhs.split(",")
    if len(terms) != n:
        raise ValueError(f"einsum: {len(terms)} terms for {n} operands")
    counts = Counter(lhs.replace(",", ""))
    for label, k in counts.items():
        if not label.isalpha() or not label.isascii():
            raise ValueError(f"einsum: label {label!r} is not an ASCII letter")
        if k > 2:
            raise ValueError(f"einsum: label {label!r} occurs {k} times")
    for term in terms:
        if len(set(term)) != len(term):
            raise ValueError(f"einsum: a label is repeated inside term {term!r}")
    out = rhs if arrow else "".join(sorted(x for x, k in counts.items() if k == 1))
    for x, k in counts.items():
        if k == 1 and x not in out:
            raise ValueError(f"einsum: input label {x!r} is missing from the output")
    return terms, out


@cache
def _pair_plan(equation: str, na: int, nb: int):
    """``(axes, perm)`` of a two-operand equation on operands of ``na`` and ``nb`` axes,
    validated once (a sweep repeats a handful of equations thousands of times)."""
    terms, out = _parse(equation, 2)
    for term, n in zip(terms, (na, nb)):
        if len(term) != n:
            raise ValueError(f"einsum: term {term!r} labels {len(term)} axes of a {n}-axis tensor")
    shared = [x for x in terms[0] if x in terms[1]]
    axes = (tuple(terms[0].index(x) for x in shared), tuple(terms[1].index(x) for x in shared))
    free = [x for x in terms[0] if x not in shared] + [x for x in terms[1] if x not in shared]
    return axes, tuple(free.index(x) for x in out)


def einsum(equation: str, *operands: SymmetricTensor, optimize=None) -> SymmetricTensor:
    """Label-equation contraction (``ops/contraction.py:695-794``).  Three or more operands
    are contracted left to right in the caller's order."""
    if len(operands) == 2:
        a, b = operands
        axes, perm = _pair_plan(equation, a.ndim, b.ndim)
        prec = current_precision()
        if a.provider.abelian:
            # one +-1 term per block: the transpose folds into the unpack exactly
            ex = contraction_exec(a.structure, b.structure, axes, *prec, perm)
            return SymmetricTensor(ex.out, arena=ex.run(a.arena, b.arena))
        # SU(2): the unpack and the transpose stay two passes, the reference's order of
        # roundings (composing their multi-term maps would round the sums differently)
        ex = contraction_exec(a.structure, b.structure, axes, *prec, None)
        return transpose(SymmetricTensor(ex.out, arena=ex.run(a.arena, b.arena)), perm)
    terms, out = _parse(equation, len(operands))
    for term, t in zip(terms, operands):
        if len(term) != t.ndim:
            raise ValueError(f"einsum: term {term!r} labels {len(term)} axes of a {t.ndim}-axis tensor")
    if len(operands) == 1:
        return transpose(operands[0], tuple(terms[0].index(x) for x in out))
    # three or more operands
    keep = set(out)
    acc, at = operands[0], terms[0]
    for k in range(1, len(operands)):
        later = keep.union(*map(set, terms[k + 1:]))
        mid = "".join([x for x in at if x in later] + [x for x in terms[k] if x in later])
        acc = einsum(f"{at},{terms[k]}->{mid}", acc, operands[k])
        at = mid
    return transpose(acc, tuple(at.index(x) for x in out))


# ---------------------------------------------------------------------------------------
# vector space


@cache
def _runs(s: TensorStructure) -> _exec.DotRuns:
    return _exec.make_runs(s)


def _check_same(a: SymmetricTensor, b: SymmetricTensor, op: str) -> None:
    if a.structure != b.structure:
        raise ValueError(f"{op}: the two tensors have different structures")


def inner_device(a: SymmetricTensor, b: SymmetricTensor, out: torch.Tensor) -> None:
    """``<a|b>`` written into the device scalar ``out`` (no host sync)."""
    _check_same(a, b, "inner")
    r = _runs(a.structure)
    n = a.arena.numel()
    work = _exec.dot_workspace(n)
    _lib.call("tnb_weighted_dot", _exec.ptr(a.arena), _exec.ptr(b.arena), n, _exec.ptr(r.start),
              _exec.ptr(r.weight), r.n_runs, _exec.ptr(work), _exec.ptr(out), _exec.stream_ptr())


def inner(a: SymmetricTensor, b: SymmetricTensor) -> float:
    """``sum_tau qdim(c_tau) <A_tau, B_tau>`` (``ops/contraction.py:517-589``)."""
    out = torch.empty(1, dtype=torch.float64, device=a.arena.device)
    inner_device(a, b, out)
    return float(out.item())


def norm(t: SymmetricTensor) -> float:
    """qdim-weighted Frobenius norm (``ops/basic.py:309``)."""
    return max(inner(t, t), 0.0) ** 0.5


def _axpby(alpha, x: SymmetricTensor, beta, y: SymmetricTensor) -> SymmetricTensor:
    out = SymmetricTensor.empty(x.structure)
    _lib.call("tnb_axpby", x.arena.numel(), float(alpha), _exec.ptr(x.arena), float(beta),
              _exec.ptr(y.arena), _exec.ptr(out.arena), _exec.stream_ptr())
    return out


def axpby_into(alpha, x: torch.Tensor, beta, y: torch.Tensor, out: torch.Tensor) -> None:
    """``out = alpha x + beta y`` on raw arenas (``out`` may alias ``x`` or ``y``)."""
    _lib.call("tnb_axpby", x.numel(), float(alpha), _exec.ptr(x), float(beta), _exec.ptr(y),
              _exec.ptr(out), _exec.stream_ptr())


def add(a: SymmetricTensor, b: SymmetricTensor) -> SymmetricTensor:
    _check_same(a, b, "add")
    return _axpby(1.0, a, 1.0, b)


def subtract(a: SymmetricTensor, b: SymmetricTensor) -> SymmetricTensor:
    _check_same(a, b, "subtract")
    return _axpby(1.0, a, -1.0, b)


def multiply(t: SymmetricTensor, s) -> SymmetricTensor:
    if isinstance(s, SymmetricTensor):
        raise CapabilityError("multiply: blockwise products of two tensors are not on this path")
    return _axpby(float(s), t, 0.0, t)


def divide(t: SymmetricTensor, s) -> SymmetricTensor:
    return _axpby(1.0 / float(s), t, 0.0, t)


def block_sqrt(t: SymmetricTensor) -> SymmetricTensor:
    """Entry-by-entry square root of every block (``ops/blocks.py:95-135``): the square
    root of a singular-value tensor."""
    out = SymmetricTensor.empty(t.structure)
    torch.sqrt(t.arena, out=out.arena)
    return out


# ---------------------------------------------------------------------------------------
# identity and trace


def identity(legs) -> SymmetricTensor:
    """``id`` on the legs: ``(*legs OUT, *legs IN)``, one eye per coupled sector
    (``ops/map.py:175-234``)."""
    import numpy as np

    from tenet.linalg import _raise_exec
    from tenet.structure import Leg

    legs = tuple(legs)
    s = TensorStructure((*(Leg(l.space, OUT, l.dual, l.name) for l in legs),
                         *(Leg(l.space, IN, l.dual, l.name) for l in legs)))
    ml = matrix_layout(s)
    host = np.zeros(ml.size)
    for c in ml.sectors:
        r, q = ml.shape[c]
        host[ml.base[c]:ml.base[c] + r * q] = np.eye(r, q).ravel()
    out = SymmetricTensor.empty(s)
    _raise_exec(s).run(torch.from_numpy(host).to(out.arena.device), out.arena)
    return out


def full_trace(t: SymmetricTensor) -> float:
    """``sum_c qdim(c) tr(M_c)`` of an endomorphism (``ops/contraction.py:440-514``)."""
    from tenet.linalg import _lower_exec

    s = t.structure
    m, lower = _lower_exec(s, s.out_axes, s.in_axes)
    ml = matrix_layout(m)
    buf = torch.empty(ml.size, dtype=torch.float64, device=t.arena.device)
    lower.run(t.arena, buf)
    p = t.provider
    total = 0.0
    for c in ml.sectors:
        r, q = ml.shape[c]
        if r != q:
            raise ValueError("full_trace: the tensor is not an endomorphism (non-square sector)")
        total += p._qdim(c) * float(torch.diagonal(buf[ml.base[c]:ml.base[c] + r * q].view(r, q)).sum())
    return total
