"""Blockwise truncated SVD (``ops/linalg.py:1441-1612``) on the device.

The tensor is lowered to its coupled-sector matrices by one gather, each sector is
factorised on the GPU (sectors of equal shape are batched into one call), the singular
values -- and only they -- come to the host, where the keep rule runs exactly as the
reference's ``_spectrum``/``_admissible``/``_decide`` (``ops/linalg.py:1079-1324``): one
global spectrum sorted by (-sigma, sector, index), a qdim-weighted cutoff, then a greedy
walk under the dense budget ``sum_c qdim(c) m_c <= max_bond`` that stops at the first
overflow.  The kept prefixes are scattered back into U, S, Vh by gathers.
"""

from __future__ import annotations

from dataclasses import dataclass
from functools import cache

import numpy as np
import torch

from tenet import _exec
from tenet.plan import repartition_plan, validate_partition
from tenet.structure import IN, OUT, GradedSpace, Leg, TensorStructure, layout, matrix_layout
from tenet.tensor import SymmetricTensor

__all__ = ["BondSelection", "lq", "svd_truncated", "svd_truncated_selected"]

_CUTOFF_MODES = ("abs", "rel", "sum2", "rsum2", "sum1", "rsum1")


def _admissible(spectrum, qdim, cutoff, mode) -> int:
    if cutoff is None:
        return len(spectrum)
    if mode == "abs":
        return sum(1 for s, _, _ in spectrum if s > cutoff)
    if mode == "rel":
        th = cutoff * spectrum[0][0]
        return sum(1 for s, _, _ in spectrum if s > th)
    power = 2 if mode in ("sum2", "rsum2") else 1
    weights = [qdim(c) * s ** power for s, c, _ in spectrum]
    th = cutoff * sum(weights) if mode.startswith("r") else cutoff
    kept, dropped = len(spectrum), 0.0
    for w in reversed(weights):
        if dropped + w >= th:
            break
        dropped += w
        kept -= 1
    return kept


@dataclass(frozen=True)
class BondSelection:
    """The truncation decision (``ops/linalg.py:1159-1271``), sector labels as ints."""

    keep: dict
    dense_dim: float
    reduced_dim: int
    discarded_weight: float
    scale: float


def decide(spectrum, provider, max_bond, cutoff, cutoff_mode="rsum2", renorm=False,
           budget="dense"):
    """The keep rule (``ops/linalg.py:1274-1324``).  ``budget="reduced"`` counts each
    kept multiplet as 1 against ``max_bond`` instead of its dimension (a build-side
    mode; the reference's budget is the dense one)."""
    qdim = provider._qdim
    cost = qdim if budget == "dense" else (lambda c: 1)
    if not spectrum:
        raise ValueError("svd_truncated: this tensor has no singular values at all")
    adm = _admissible(spectrum, qdim, cutoff, cutoff_mode)
    keep: dict = {}
    dense = 0.0
    kept_w = 0.0
    n = 0
    used = 0
    for s, c, _ in spectrum[:adm]:
        if max_bond is not None and used + cost(c) > max_bond:
            break
        used += cost(c)
        dense += qdim(c)
        keep[c] = keep.get(c, 0) + 1
        kept_w += qdim(c) * s * s
        n += 1
    if not keep:
        raise ValueError("svd_truncated: the truncation keeps no singular value at all")
    total = sum(qdim(c) * s * s for s, c, _ in spectrum)
    disc = sum(qdim(c) * s * s for s, c, _ in spectrum[n:])
    return BondSelection(keep, dense, n, disc, (total / kept_w) ** 0.5 if renorm else 1.0)


@cache
def _lower_exec(s: TensorStructure, outputs: tuple, inputs: tuple):
    m, perm, terms = repartition_plan(s, outputs, inputs)
    table = _exec.make_gather(_exec.gather_rows(s, "arena", m, "matrix", perm, terms))
    return m, table


@cache
def _raise_exec(s: TensorStructure):
    """Matrix buffer -> arena for structure ``s`` (``from_matrices``, ``map_view.py:282-335``)."""
    terms = tuple((j, j, 1.0) for j in range(s.num_blocks))
    return _exec.make_gather(_exec.gather_rows(s, "matrix", s, "arena", tuple(range(s.ndim)),
                                               terms))


class _SvdPlan:
    """Device tables of one lowered structure's blockwise SVD: per coupled sector (in label
    order) its shape and the offsets of its full factors, the decision's sector table,
    and pinned host buffers for the one read-back of a truncation."""

    def __init__(self, m: TensorStructure) -> None:
        from tenet import _lib

        ml = matrix_layout(m)
        p = m.provider
        self.ml = ml
        self.sectors = tuple(sorted(ml.sectors))
        smem_max = int(_lib.load().tnb_block_svd_smem_doubles())
        rows, sec_rows, qd = [], [], []
        self.kfull = {}
        uo = so = vo = wo = 0
        smem = 0
        for c in self.sectors:
            r, q = ml.shape[c]
            k = min(r, q)
            need = max(r, q) * k + k * k + 2 * k
            if need <= smem_max:
                w = -1
                smem = max(smem, need)
            else:
                w = wo
                wo += need
            rows.append((r, q, ml.base[c], uo, so, vo, w, 0))
            sec_rows.append((k, so, c, 0))
            qd.append(float(p._qdim(c)))
            self.kfull[c] = (k, uo, so, vo)
            uo, so, vo = uo + r * k, so + k, vo + k * q
        self.n_u, self.n_s, self.n_v, self.n_w, self.smem = uo, so, vo, wo, smem
        self.total = so
        dev = _exec.device()
        i64 = dict(dtype=torch.int64, device=dev)
        self.rows = torch.tensor(rows or [(0,) * 8], **i64)
        self.sec_rows = torch.tensor(sec_rows or [(0,) * 4], **i64)
        self.qdim = torch.tensor(qd or [1.0], dtype=torch.float64, device=dev)
        # everything the decision reads back, in one device buffer and one pinned copy:
        # stats (8 f64), keep (ns i64), sorted values (T f64), info (ns i32), sorted sectors
        # (T i32)
        n, T = max(1, len(self.sectors)), max(1, self.total)
        self.o_keep = 64
        self.o_sorted = self.o_keep + 8 * n
        self.o_info = self.o_sorted + 8 * T
        self.o_csec = self.o_info + 4 * n
        self.nbytes = -(-(self.o_csec + 4 * T) // 8) * 8
        self.T = T
        self._readbacks: dict = {}  # stream -> _Readback
        self.post: dict = {}  # kept counts -> truncated structures and compaction table

    def readback(self, stream: int) -> "_Readback":
        """This stream's read-back buffers: a decision in flight on one stream (between
        ``svd_truncated_launch`` and ``svd_truncated_finish``) never shares them with a
        decision of the same structure on another."""
        rb = self._readbacks.get(stream)
        if rb is None:
            rb = self._readbacks[stream] = _Readback(self)
        return rb


class _Readback:
    """One device buffer and its pinned copy holding what a decision reads back: stats (8
    f64), keep (ns i64), sorted values (T f64), info (ns i32), sorted sectors (T i32)."""

    def __init__(self, plan: _SvdPlan) -> None:
        self.dev = torch.zeros(plan.nbytes, dtype=torch.uint8, device=_exec.device())
        self.host = torch.zeros(plan.nbytes, dtype=torch.uint8).pin_memory()
        h = self.host.numpy()
        self.h_stats = h[:64].view(np.float64)
        self.h_keep = h[plan.o_keep:plan.o_sorted].view(np.int64)
        self.h_sorted = h[plan.o_sorted:plan.o_info].view(np.float64)
        self.h_info = h[plan.o_info:plan.o_csec].view(np.int32)
        self.h_csec = h[plan.o_csec:plan.o_csec + 4 * plan.T].view(np.int32)
        self.event = torch.cuda.Event()


@cache
def _svd_plan(m: TensorStructure) -> _SvdPlan:
    return _SvdPlan(m)


_MODES = {"abs": 0, "rel": 1, "sum2": 2, "rsum2": 3, "sum1": 4, "rsum1": 5}


def svd_truncated(t: SymmetricTensor, axes=None, *, max_bond=None, cutoff=None,
                  cutoff_mode: str = "rsum2", renorm: bool = False, budget: str = "dense"):
    """``U, S, Vh`` on the truncated bond.  Same legs, keep rule and refusals as the
    reference; returns ``(U, S, Vh)``.  ``budget`` as in ``decide``.

    All on the device: the lowering gather, one blockwise SVD launch (a CTA per coupled
    sector), the decision launch (global order, cutoff prefix, budget walk), one read-back
    of the decision, and one launch that packs the kept prefixes before the three raising
    gathers."""
    return svd_truncated_selected(t, axes, max_bond=max_bond, cutoff=cutoff,
                                  cutoff_mode=cutoff_mode, renorm=renorm, budget=budget)[:3]


def svd_truncated_selected(t: SymmetricTensor, axes=None, *, max_bond=None, cutoff=None,
                           cutoff_mode: str = "rsum2", renorm: bool = False,
                           budget: str = "dense"):
    """``svd_truncated`` plus what its decision read back: ``(U, S, Vh, selection,
    kept)``, ``selection`` the ``BondSelection`` and ``kept`` the kept singular values in
    the global order as ``(sigma * scale, sector label)`` pairs."""
    return svd_truncated_finish(svd_truncated_launch(
        t, axes, max_bond=max_bond, cutoff=cutoff, cutoff_mode=cutoff_mode, renorm=renorm,
        budget=budget))


class _SvdPending:
    """A truncation between its launch and its read-back."""

    __slots__ = ("plan", "m", "rb", "U", "Sv", "V", "keep_alive", "renorm", "dev", "ns")


def svd_truncated_launch(t: SymmetricTensor, axes=None, *, max_bond=None, cutoff=None,
                         cutoff_mode: str = "rsum2", renorm: bool = False,
                         budget: str = "dense") -> _SvdPending:
    """The first half of ``svd_truncated_selected``: the argument checks (the reference's
    refusals), the lowering, the blockwise SVD, the decision and the copy of the decision to
    pinned host memory, all enqueued on the current stream; nothing waits.  A caller with
    other work (a serving loop) does it before ``svd_truncated_finish``."""
    from tenet import _lib

    if budget not in ("dense", "reduced"):
        raise ValueError(f"unknown budget {budget!r}")
    if max_bond is None and cutoff is None:
        raise ValueError("svd_truncated needs at least one of max_bond or cutoff")
    if max_bond is not None and max_bond <= 0:
        raise ValueError(f"max_bond must be positive, got {max_bond!r}")
    if cutoff is not None and cutoff < 0:
        raise ValueError(f"cutoff must be non-negative, got {cutoff!r}")
    if cutoff_mode not in _CUTOFF_MODES:
        raise ValueError(f"unknown cutoff_mode {cutoff_mode!r}")
    if axes is None:
        axes = (t.structure.out_axes, t.structure.in_axes)
    outputs, inputs = validate_partition(t.ndim, axes[0], axes[1])
    m, lower = _lower_exec(t.structure, outputs, inputs)
    plan = _svd_plan(m)
    if plan.total == 0:
        raise ValueError("svd_truncated: this tensor has no singular values at all")
    ml = plan.ml
    dev = t.arena.device
    f64 = dict(dtype=torch.float64, device=dev)
    buf = torch.empty(max(1, ml.size), **f64)
    lower.run(t.arena, buf)
    U = torch.empty(max(1, plan.n_u), **f64)
    Sv = torch.empty(max(1, plan.n_s), **f64)
    V = torch.empty(max(1, plan.n_v), **f64)
    W = torch.empty(max(1, plan.n_w), **f64)
    P, st = _exec.ptr, _exec.stream_ptr()
    ns = len(plan.sectors)
    rb = plan.readback(st)
    base = rb.dev.data_ptr()
    _lib.call("tnb_block_svd", P(plan.rows), ns, P(buf), buf.numel(), P(U), U.numel(), P(Sv),
              Sv.numel(), P(V), V.numel(), P(W), plan.n_w, base + plan.o_info, plan.smem, st)
    _lib.call("tnb_truncate_decide", P(plan.sec_rows), P(plan.qdim), ns, P(Sv), Sv.numel(),
              -1.0 if cutoff is None else float(cutoff), _MODES[cutoff_mode],
              -1.0 if max_bond is None else float(max_bond), 0 if budget == "dense" else 1,
              base + plan.o_keep, base + plan.o_sorted, base + plan.o_csec, base, st)
    rb.host.copy_(rb.dev, non_blocking=True)
    rb.event.record()
    p = _SvdPending()
    p.plan, p.m, p.rb, p.U, p.Sv, p.V = plan, m, rb, U, Sv, V
    p.keep_alive, p.renorm, p.dev, p.ns = (buf, W), renorm, dev, ns
    return p


def svd_truncated_finish(p: _SvdPending):
    """The second half: wait for the decision's read-back, build the truncated structures
    and pack the kept factors (on the current stream, which must be the launch's)."""
    from tenet import _lib

    plan, m, rb, ns = p.plan, p.m, p.rb, p.ns
    ml = plan.ml
    f64 = dict(dtype=torch.float64, device=p.dev)
    P, st = _exec.ptr, _exec.stream_ptr()
    rb.event.synchronize()
    info = rb.h_info[:ns]
    if np.any(info != 0):
        raise RuntimeError(f"svd_truncated: the blockwise SVD did not converge (info "
                           f"{info.tolist()})")
    keep_h = rb.h_keep[:ns]
    n_kept, dense, disc, total, kept_w = (float(x) for x in rb.h_stats[:5])
    if n_kept == 0:
        raise ValueError("svd_truncated: the truncation keeps no singular value at all")
    keep = {c: int(k) for c, k in zip(plan.sectors, keep_h) if k > 0}
    scale = (total / kept_w) ** 0.5 if p.renorm else 1.0
    prov = m.provider
    sel = BondSelection(keep, dense, int(n_kept), disc, scale)
    nk = int(n_kept)
    kept = [(float(x) * scale, plan.sectors[int(k)])
            for x, k in zip(rb.h_sorted[:nk], rb.h_csec[:nk])]
    # the truncated structures and the compaction table depend on the kept counts only:
    # a bond that keeps what it kept before (every converged sweep) reuses them
    post = plan.post.get(tuple(keep.items()))
    if post is None:
        bond = GradedSpace.new(prov, {prov.sector(c): k for c, k in keep.items()})
        su = TensorStructure((*m.codomain, Leg(bond, IN)))
        ss = TensorStructure((Leg(bond, OUT), Leg(bond, IN)))
        sv = TensorStructure((Leg(bond, OUT), *m.domain))
        lu, ls, lv = matrix_layout(su), matrix_layout(ss), matrix_layout(sv)
        rows = []
        for c, k in keep.items():
            kf, uo, so, vo = plan.kfull[c]
            r, q = ml.shape[c]
            rows.append((r, q, kf, k, uo, so, vo, lu.base[c], ls.base[c], lv.base[c], 0, 0))
        crows = torch.tensor(rows, dtype=torch.int64, device=p.dev)
        post = (su, ss, sv, lu.size, ls.size, lv.size, crows, len(rows))
        if len(plan.post) >= 64:
            plan.post.pop(next(iter(plan.post)))
        plan.post[tuple(keep.items())] = post
    su, ss, sv, nu, nsz, nv, crows, n_rows = post
    PU, PS, PV = (torch.empty(max(1, x), **f64) for x in (nu, nsz, nv))
    U, Sv, V = p.U, p.Sv, p.V
    _lib.call("tnb_svd_compact", P(crows), n_rows, P(U), U.numel(), P(Sv), Sv.numel(), P(V),
              V.numel(), float(scale), P(PU), PU.numel(), P(PS), PS.numel(), P(PV), PV.numel(),
              st)
    out = []
    for structure, packed in ((su, PU), (ss, PS), (sv, PV)):
        o = SymmetricTensor.empty(structure)
        _raise_exec(structure).run(packed, o.arena)
        out.append(o)
    return (*out, sel, kept)


def singular_values(s: SymmetricTensor) -> dict:
    """``{sector label: diagonal}`` of an ``S`` returned by ``svd_truncated`` (host)."""
    lay = layout(s.structure)
    host = s.numpy_arena()
    out = {}
    for b, (ot, _) in enumerate(s.structure.keys):
        n = int(lay.shapes[b, 0])
        blk = host[int(lay.offsets[b]):int(lay.offsets[b]) + n * n].reshape(n, n)
        out[ot[2]] = np.diag(blk).copy()
    return out


class _LqPlan:
    """Device table of one lowered structure's blockwise LQ: per coupled sector its shape,
    the sector's offset in the lowered buffer and in the matrix layouts of ``L`` and
    ``Q`` (which the kernel writes directly), and its work area (shared memory when it
    fits)."""

    def __init__(self, m: TensorStructure) -> None:
        from tenet import _lib

        ml = matrix_layout(m)
        p = m.provider
        self.ml = ml
        bond = GradedSpace.new(p, {p.sector(c): min(ml.shape[c]) for c in ml.sectors})
        self.sl = TensorStructure((*m.codomain, Leg(bond, IN)))
        self.sq = TensorStructure((Leg(bond, OUT), *m.domain))
        ll, lq_ = matrix_layout(self.sl), matrix_layout(self.sq)
        self.n_l, self.n_q = ll.size, lq_.size
        smem_max = int(_lib.load().tnb_block_svd_smem_doubles())
        rows, wo, smem = [], 0, 0
        for c in sorted(ml.sectors):
            r, q = ml.shape[c]
            k = min(r, q)
            assert ll.shape[c] == (r, k) and lq_.shape[c] == (k, q)
            need = q * r + q * k + 2 * k
            if need <= smem_max:
                w = -1
                smem = max(smem, need)
            else:
                w, wo = wo, wo + need
            rows.append((r, q, ml.base[c], ll.base[c], lq_.base[c], w, 0, 0))
        self.n_rows, self.n_w, self.smem = len(rows), wo, smem
        self.rows = torch.tensor(rows or [(0,) * 8], dtype=torch.int64, device=_exec.device())


@cache
def _lq_plan(m: TensorStructure) -> _LqPlan:
    return _LqPlan(m)


def lq(t: SymmetricTensor, axes=None):
    """``T = L o Q``, the reduced LQ per coupled sector (``ops/linalg.py:549-620``): per
    sector ``B^T = q r``, ``L = r^T`` with legs ``(*left, bond IN)`` and ``Q = q^T`` with
    legs ``(bond OUT, *right)``, bond degeneracy ``min(rows, cols)``.

    One launch factors every sector (a CTA each) by Householder reflections in LAPACK's
    convention, so ``L`` and ``Q`` carry the gauge of the reference's QR; the lowering and
    the two raising gathers are the only other launches."""
    from tenet import _lib

    if axes is None:
        axes = (t.structure.out_axes, t.structure.in_axes)
    outputs, inputs = validate_partition(t.ndim, axes[0], axes[1])
    m, lower = _lower_exec(t.structure, outputs, inputs)
    plan = _lq_plan(m)
    dev = t.arena.device
    f64 = dict(dtype=torch.float64, device=dev)
    buf = torch.empty(max(1, plan.ml.size), **f64)
    lower.run(t.arena, buf)
    lbuf = torch.empty(max(1, plan.n_l), **f64)
    qbuf = torch.empty(max(1, plan.n_q), **f64)
    work = torch.empty(max(1, plan.n_w), **f64)
    P = _exec.ptr
    _lib.call("tnb_block_lq", P(plan.rows), plan.n_rows, P(buf), buf.numel(), P(lbuf),
              lbuf.numel(), P(qbuf), qbuf.numel(), P(work), plan.n_w, plan.smem,
              _exec.stream_ptr())
    out_l, out_q = SymmetricTensor.empty(plan.sl), SymmetricTensor.empty(plan.sq)
    _raise_exec(plan.sl).run(lbuf, out_l.arena)
    _raise_exec(plan.sq).run(qbuf, out_q.arena)
    return out_l, out_q
