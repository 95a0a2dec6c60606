"""Batched block-sparse operations: one operation on ``n`` independent operand sets of
identical structures, every stage of it one launch for the whole batch.

A ``TensorBatch`` holds ``n`` tensors of one structure as an ``(n, size)`` arena (row k is
tensor k's arena in block order), or one shared tensor broadcast to every member.  The
descriptor tables of a single operation are replicated across the batch with each
member's offsets shifted by its row of the batched arenas: gather rows and their terms
are copied per member, and the coupled-sector products are re-planned over the whole
batch (so the tile kind, split-K and, in the precision form, the tensor-core choice see
the batch's total work).  A broadcast operand is read by every member at the same
offsets.  The arithmetic of each member is exactly that of the unbatched operation.

There is no reference counterpart; the reference contracts one tensor pair per call
(``ops/contraction.py:592-866``).  This is the batched form of the same lowering, for
workloads such as many independent environment updates of one shape.
"""

from __future__ import annotations

from functools import cache

import numpy as np
import torch

from tenet import _exec, ops
from tenet.structure import OUT, TensorStructure, layout
from tenet.tensor import SymmetricTensor

__all__ = ["BatchedHeff2", "TensorBatch", "adjoint", "composed", "einsum", "env_update_last",
           "heff2", "repartition", "tensordot", "transpose"]

#: pick the FP64 tile kind of batched products by measurement (``_exec.autotune``), keyed
#: on the block-size histogram; False uses the size heuristic
AUTOTUNE = True


class TensorBatch:
    """``n`` tensors of one structure, or one tensor shared by every member of a batch."""

    def __init__(self, structure: TensorStructure, arena: torch.Tensor, n: int,
                 shared: bool = False) -> None:
        size = layout(structure).size
        want = (size,) if shared else (n, size)
        if tuple(arena.shape) != want:
            raise ValueError(f"TensorBatch: arena of shape {tuple(arena.shape)}, expected {want}")
        self.structure, self.arena, self.n, self.shared = structure, arena, n, shared

    @classmethod
    def stack(cls, tensors) -> TensorBatch:
        tensors = list(tensors)
        s = tensors[0].structure
        if any(t.structure != s for t in tensors):
            raise ValueError("TensorBatch.stack: the tensors' structures differ")
        return cls(s, torch.stack([t.arena for t in tensors]), len(tensors))

    @classmethod
    def broadcast(cls, t: SymmetricTensor, n: int) -> TensorBatch:
        return cls(t.structure, t.arena, n, shared=True)

    @property
    def legs(self):
        return self.structure.legs

    @property
    def ndim(self) -> int:
        return self.structure.ndim

    @property
    def provider(self):
        return self.structure.provider

    def __getitem__(self, k: int) -> SymmetricTensor:
        return SymmetricTensor(self.structure, arena=self.arena if self.shared else self.arena[k])

    def stride(self) -> int:
        """Elements between consecutive members' arenas (0 when shared)."""
        return 0 if self.shared else layout(self.structure).size


def _batch_rows(table: _exec.GatherTable, n: int, src_strides, dst_strides):
    """Gather rows and terms of ``table`` replicated for ``n`` members: member k's rows
    write ``k * dst_strides[buf]`` further and its terms read ``k * src_strides[buf]``
    further, ``buf`` being the row's buffer pair."""
    seg = table.seg
    if not len(seg):
        return np.zeros((0, _exec.SEG_W), np.int64), np.zeros(0, np.int64), np.zeros(0), \
            np.zeros(0, np.int64)
    bufs = seg[:, 5].astype(np.int64)
    order = np.argsort(seg[:, 3], kind="stable")  # rows in term order: each term's buffer
    term_buf = np.repeat(bufs[order], (seg[:, 4] - seg[:, 3])[order])
    dst_stride = np.asarray(dst_strides, np.int64)[bufs]
    src_stride = np.asarray(src_strides, np.int64)[term_buf]
    nt = table.n_term
    rows, tsrc = [], []
    for k in range(n):
        r = seg.copy()
        r[:, 0] += k * dst_stride
        r[:, 3:5] += k * nt
        rows.append(r)
        tsrc.append(table.tsrc + k * src_stride)
    return (np.concatenate(rows), np.concatenate(tsrc), np.tile(table.tcf, n),
            np.tile(table.tld, n))


def _batch_gather(table, n, src_strides, dst_strides):
    if table is None:
        return None
    return _exec.make_gather(_batch_rows(table, n, src_strides, dst_strides))


def _batch_products(products, n, a_stride, b_stride, c_stride):
    out = []
    for k in range(n):
        for M, N, K, ao, lda, bo, ldb, co, ldc in products:
            out.append((M, N, K, ao + k * a_stride, lda, bo + k * b_stride, ldb, co + k * c_stride,
                        ldc))
    return out


class _BatchedContraction:
    """One contraction for ``n`` members.  A shared operand is packed once into its
    coupled-sector matrices and every member's products read that one copy."""

    def __init__(self, ex: ops.ContractionExec, n: int, sa_stride: int, sb_stride: int,
                 precision: str, tc_min_flops, tuned: bool = False) -> None:
        self.out, self.n = ex.out, n
        self.a_mat, self.b_mat, self.c_mat = ex.a_mat, ex.b_mat, ex.c_mat
        self.a_shared, self.b_shared = sa_stride == 0, sb_stride == 0
        parts = []
        for buf, stride, mat in ((0, sa_stride, ex.a_mat), (1, sb_stride, ex.b_mat)):
            sub = _exec.make_gather(_rows_of_buf(ex.pack, buf))
            parts.append(_batch_rows(sub, 1 if stride == 0 else n, (stride, stride), (mat, mat)))
        self.pack = _exec.make_gather(*parts)
        self.gemm = _exec.GemmGroup(
            _batch_products(ex.gemm.products, n, 0 if self.a_shared else ex.a_mat,
                            0 if self.b_shared else ex.b_mat, ex.c_mat),
            precision, tc_min_flops, tuned=tuned)
        self.out_size = layout(ex.out).size
        self.unpack = _batch_gather(ex.unpack, n, (ex.c_mat, 0), (self.out_size, 0))

    def run(self, a: torch.Tensor, b: torch.Tensor) -> torch.Tensor:
        f64 = dict(dtype=torch.float64, device=a.device)
        ap = torch.empty(max(1, (1 if self.a_shared else self.n) * self.a_mat), **f64)
        bp = torch.empty(max(1, (1 if self.b_shared else self.n) * self.b_mat), **f64)
        cp = torch.empty(max(1, self.n * self.c_mat), **f64)
        out = torch.empty((self.n, self.out_size), **f64)
        self.pack.run(a.reshape(-1), ap, b.reshape(-1), bp)
        self.gemm.run(ap, bp, cp)
        self.unpack.run(cp, out.reshape(-1))
        return out


def _rows_of_buf(table: _exec.GatherTable, buf: int):
    """The rows (and their terms) of one buffer pair of a gather table."""
    seg = table.seg
    keep = seg[:, 5] == buf
    rows, tsrc, tcf, tld = [], [], [], []
    for r in seg[keep]:
        r = r.copy()
        t0, t1 = int(r[3]), int(r[4])
        r[3], r[4] = len(tsrc), len(tsrc) + (t1 - t0)
        rows.append(r)
        tsrc.extend(table.tsrc[t0:t1])
        tcf.extend(table.tcf[t0:t1])
        tld.extend(table.tld[t0:t1])
    rows = np.stack(rows) if rows else np.zeros((0, _exec.SEG_W), np.int64)
    return rows, np.asarray(tsrc, np.int64), np.asarray(tcf), np.asarray(tld, np.int64)


@cache
def _contraction(sa, sb, axes, n, a_shared, b_shared, precision, tc_min_flops, out_axes=None,
                 tuned=None):
    ex = ops.contraction_exec(sa, sb, axes, precision, tc_min_flops, out_axes)
    return _BatchedContraction(ex, n, 0 if a_shared else layout(sa).size,
                               0 if b_shared else layout(sb).size, precision, tc_min_flops,
                               bool(tuned))


def tensordot(a: TensorBatch, b: TensorBatch, axes, out_axes=None) -> TensorBatch:
    """Member-wise ``ops.tensordot`` in one launch per stage (precision: ``ops.precision``)."""
    if a.n != b.n:
        raise ValueError("batch: operands of different batch sizes")
    ax = ops._validated_axes(a.structure, b.structure, axes)
    bc = _contraction(a.structure, b.structure, ax, a.n, a.shared, b.shared, *ops.current_precision(),
                      None if out_axes is None else tuple(out_axes), AUTOTUNE)
    return TensorBatch(bc.out, bc.run(a.arena, b.arena), a.n)


@cache
def _unary(s: TensorStructure, kind: str, x, y, n: int):
    dst, table = ops._map_exec(s, kind, x, y)
    size = layout(dst).size
    return dst, _batch_gather(table, n, (layout(s).size, 0), (size, 0))


def _apply(t: TensorBatch, kind: str, x=None, y=None) -> TensorBatch:
    if t.shared:
        src = t[0]
        one = (ops.transpose(src, x) if kind == "t" else
               ops.repartition(src, x, y) if kind == "r" else ops.adjoint(src))
        return TensorBatch.broadcast(one, t.n)
    dst, table = _unary(t.structure, kind, x, y, t.n)
    if table is None:
        return TensorBatch(dst, t.arena, t.n)
    out = torch.empty((t.n, layout(dst).size), dtype=torch.float64, device=t.arena.device)
    table.run(t.arena.reshape(-1), out.reshape(-1))
    return TensorBatch(dst, out, t.n)


def transpose(t: TensorBatch, axes) -> TensorBatch:
    return _apply(t, "t", tuple(axes))


def adjoint(t: TensorBatch) -> TensorBatch:
    return _apply(t, "a")


def repartition(t: TensorBatch, outputs, inputs) -> TensorBatch:
    return _apply(t, "r", tuple(outputs), tuple(inputs))


def einsum(equation: str, a: TensorBatch, b: TensorBatch) -> TensorBatch:
    """Two-operand member-wise ``ops.einsum``."""
    terms, out = ops._parse(equation, 2)
    ta, tb = terms
    for term, t in zip(terms, (a, b)):
        if len(term) != t.ndim:
            raise ValueError(f"einsum: term {term!r} labels {len(term)} axes of a {t.ndim}-axis tensor")
    shared = [x for x in ta if x in tb]
    axes = (tuple(ta.index(x) for x in shared), tuple(tb.index(x) for x in shared))
    free = [x for x in ta if x not in shared] + [x for x in tb if x not in shared]
    perm = tuple(free.index(x) for x in out)
    if a.provider.abelian:  # exact fold of the output transpose (see ops.einsum)
        return tensordot(a, b, axes, perm)
    return transpose(tensordot(a, b, axes), perm)


def env_update_last(f: TensorBatch, a: TensorBatch, w: TensorBatch) -> TensorBatch:
    """Member-wise ``network.env_update_last``: ``L' = A^dagger . L . W . A``."""
    bra = adjoint(a)
    t = einsum("axB,apr->xBpr", f, a)
    t = einsum("xPpm,xBpr->BrPm", w, t)
    return einsum("BPs,BrPm->rms", bra, t)


def composed(equation: str, a: TensorBatch, b: TensorBatch, bend: str = "") -> TensorBatch:
    """Member-wise ``network.composed``: the wires named in ``bend`` bent first."""
    if bend:
        lhs, out = equation.split("->")
        ta, tb = lhs.split(",")

        def bent(t: TensorBatch, term: str):
            flip = set(bend)
            outs = tuple(i for i, ch in enumerate(term)
                         if (t.legs[i].side is OUT) != (ch in flip))
            ins = tuple(i for i in range(len(term)) if i not in outs)
            return repartition(t, outs, ins), "".join(term[i] for i in (*outs, *ins))

        a, ta = bent(a, ta)
        b, tb = bent(b, tb)
        equation = f"{ta},{tb}->{out}"
    return einsum(equation, a, b)


def heff2(fl: TensorBatch, w1: TensorBatch, w2: TensorBatch, fr: TensorBatch,
          aa: TensorBatch) -> TensorBatch:
    """Member-wise ``network.heff2``: ``n`` two-site matvecs, every stage one launch."""
    t = einsum("apqr,rys->apqys", aa, fr)
    t = composed("apqys,mQqy->apQms", t, w2, bend="q")
    t = composed("apQms,xPpm->aPQxs", t, w1, bend="p")
    return composed("aPQxs,axB->BPQs", t, fl, bend="a")


class _BLink:
    """One link of ``BatchedHeff2``: its replicated A gather (None when the products read
    the source in place), GEMM group, buffers, fixed operand, and whether the next gather
    computes its product (``deferred``)."""

    __slots__ = ("a_g", "gemm", "bufs", "op", "direct", "c_elems", "deferred")

    def __init__(self, a_g, gemm, bufs, op, direct, c_elems) -> None:
        self.a_g, self.gemm, self.bufs, self.op = a_g, gemm, bufs, op
        self.direct, self.c_elems, self.deferred = direct, c_elems, False


class BatchedHeff2:
    """The compiled two-site matvec (``program.heff2_program``: six launches in the FP64
    form) for ``n`` members at once: every table of the single-member chain replicated
    across the batch, every fixed operand packed once (per member, or once for a shared
    operand), so one ``run`` is the same few launches for all ``n`` matvecs.  ``defer`` as
    in ``ChainProgram``.  ``precision`` / ``tc_min_flops`` as in ``ChainProgram``; the FP64 tile kinds
    of the batched products are autotuned when ``tuned``."""

    def __init__(self, fl: TensorBatch, w1: TensorBatch, w2: TensorBatch, fr: TensorBatch,
                 in_struct: TensorStructure, precision: str = "f64", tc_min_flops=None,
                 tuned: bool = True, defer: bool = False) -> None:
        from tenet import program

        class _S:
            def __init__(self, s):
                self.structure = s

        n = fl.n
        tmpl = program.heff2_program(*(_S(t.structure) for t in (fl, w1, w2, fr)), in_struct,
                                     allocate=False, precision=precision,
                                     tc_min_flops=tc_min_flops, defer=defer)
        operands = {"fr": fr, "w2": w2, "w1": w1, "fl": fl}
        dev = _exec.device()
        f64 = dict(dtype=torch.float64, device=dev)
        self.n, self.in_struct, self.out_struct = n, in_struct, tmpl.out_struct
        self.in_size, self.out_size = layout(in_struct).size, layout(tmpl.out_struct).size
        def plain(g):  # the replicated table starts from the materialised-product form
            return g.base if isinstance(g, _exec.ProductGather) else g

        self.links = []
        src_stride = self.in_size
        for lk, name in zip(tmpl.links, tmpl.operand_names):
            op = operands[name]
            m = 1 if op.shared else n
            # a link whose products read their source in place reads each member's source
            a_g = None if lk.a_direct else _batch_gather(plain(lk.a_gather), n,
                                                         (src_stride, 0), (lk.a_size, 0))
            b_g = _batch_gather(lk.b_gather, m, (layout(op.structure).size, 0), (lk.b_size, 0))
            gemm = _exec.GemmGroup(
                _batch_products(lk.gemm.products, n, src_stride if lk.a_direct else lk.a_size,
                                0 if op.shared else lk.b_size, lk.c_size),
                precision, tc_min_flops, tuned=tuned)
            bufs = (torch.empty(max(1, n * lk.a_size), **f64),
                    torch.empty(max(1, m * lk.b_size), **f64),
                    torch.empty(max(1, n * lk.c_size), **f64))
            if b_g is not None:
                b_g.run(op.arena.reshape(-1), bufs[1])
            self.links.append(_BLink(a_g, gemm, bufs, op, lk.a_direct, n * lk.c_size))
            src_stride = lk.c_size
        self.out_gather = _batch_gather(plain(tmpl.out_gather), n, (src_stride, 0),
                                        (self.out_size, 0))
        # the links the single-member chain folds into their consumer gathers, replicated
        for i, lk in enumerate(tmpl.links):
            bl = self.links[i]
            if not lk.deferred or len(bl.gemm.parts) != 1:
                continue
            last = i + 1 == len(self.links)
            consumer = self.out_gather if last else self.links[i + 1].a_g
            pg = _exec.product_gather(consumer, bl.gemm.parts[0])
            if pg is None:
                continue
            bl.deferred = True
            if last:
                self.out_gather = pg
            else:
                self.links[i + 1].a_g = pg
        self.flops = sum(bl.gemm.flops for bl in self.links)

    @property
    def launches(self) -> int:
        return (sum((0 if bl.deferred else bl.gemm.launches)
                    + (bl.a_g is not None and bl.a_g.n_seg > 0) for bl in self.links)
                + (self.out_gather is not None))

    def run(self, x: torch.Tensor, out: torch.Tensor) -> torch.Tensor:
        """``out[k] = H_k x[k]`` for the ``(n, size)`` arenas ``x`` and ``out``."""
        src, pending = x.reshape(-1), None
        for bl in self.links:
            ab, bb, cb = bl.bufs
            a = src if bl.direct else ab
            if isinstance(bl.a_g, _exec.ProductGather):
                bl.a_g.run(*pending, ab)
            elif bl.a_g is not None:
                bl.a_g.run(src, ab)
            if bl.deferred:
                pending = (a, bb)
            else:
                bl.gemm.run(a, bb, cb)
            src = cb
        if isinstance(self.out_gather, _exec.ProductGather):
            self.out_gather.run(*pending, out.reshape(-1))
        elif self.out_gather is not None:
            self.out_gather.run(src, out.reshape(-1))
        return out

    def __call__(self, aa: TensorBatch) -> TensorBatch:
        if aa.structure != self.in_struct or aa.n != self.n:
            raise ValueError("BatchedHeff2: the batch's structure or size differs")
        out = torch.empty((self.n, self.out_size), dtype=torch.float64, device=aa.arena.device)
        return TensorBatch(self.out_struct, self.run(aa.arena, out), self.n)
