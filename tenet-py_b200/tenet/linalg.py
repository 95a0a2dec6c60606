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

__all__ = ["BondSelection", "lq", "svd_truncated"]

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


def svd_truncated(t: SymmetricTensor, axes=None, *, max_bond=None, cutoff=None,
                  cutoff_mode: str = "rsum2", renorm: bool = False, budget: str = "dense"):
    """``U, S, Vh`` on the truncated bond.  Same legs, keep rule and refusals as the
    reference; returns ``(U, S, Vh)``.  ``budget`` as in ``decide``."""
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
    ml = matrix_layout(m)
    buf = torch.empty(ml.size, dtype=torch.float64, device=t.arena.device)
    lower.run(t.arena, buf)

    # factorise: batch sectors of equal shape into one cuSOLVER call
    by_shape: dict = {}
    for c in ml.sectors:
        by_shape.setdefault(ml.shape[c], []).append(c)
    parts = {}
    for (r, q), cs in by_shape.items():
        stack = torch.stack([buf[ml.base[c]:ml.base[c] + r * q].view(r, q) for c in cs])
        u, s, vh = torch.linalg.svd(stack, full_matrices=False)
        for i, c in enumerate(cs):
            parts[c] = (u[i], s[i], vh[i])

    # the decision on the host, bit-exact to the reference's keep rule
    host_s = {c: parts[c][1].cpu().numpy() for c in ml.sectors}
    spectrum = [(float(sg), c, i) for c in ml.sectors for i, sg in enumerate(host_s[c])]
    spectrum.sort(key=lambda e: (-e[0], e[1], e[2]))
    p = t.provider
    sel = decide(spectrum, p, max_bond, cutoff, cutoff_mode, renorm, budget)
    bond = GradedSpace.new(p, {p.sector(c): k for c, k in sel.keep.items()})
    su = TensorStructure((*m.codomain, Leg(bond, IN)))
    ss = TensorStructure((Leg(bond, OUT), Leg(bond, IN)))
    sv = TensorStructure((Leg(bond, OUT), *m.domain))
    dev = t.arena.device

    def assemble(structure, piece):
        lay = matrix_layout(structure)
        mbuf = torch.empty(lay.size, dtype=torch.float64, device=dev)
        for c in lay.sectors:
            r, q = lay.shape[c]
            mbuf[lay.base[c]:lay.base[c] + r * q].view(r, q).copy_(piece(c))
        out = SymmetricTensor.empty(structure)
        _raise_exec(structure).run(mbuf, out.arena)
        return out

    U = assemble(su, lambda c: parts[c][0][:, :sel.keep[c]])
    S = assemble(ss, lambda c: torch.diag(parts[c][1][:sel.keep[c]] * sel.scale))
    V = assemble(sv, lambda c: parts[c][2][:sel.keep[c], :])
    return U, S, V


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


def lq(t: SymmetricTensor, axes=None):
    """``T = L o Q``, the reduced LQ per coupled sector (``ops/linalg.py:549-620``): per
    sector ``B^T = q r`` on the device, ``L = r^T`` with legs ``(*left, bond IN)`` and
    ``Q = q^T`` with legs ``(bond OUT, *right)``, bond degeneracy ``min(rows, cols)``."""
    if axes is None:
        axes = (t.structure.out_axes, t.structure.in_axes)
    outputs, inputs = validate_partition(t.ndim, axes[0], axes[1])
    m, lower = _lower_exec(t.structure, outputs, inputs)
    ml = matrix_layout(m)
    buf = torch.empty(ml.size, dtype=torch.float64, device=t.arena.device)
    lower.run(t.arena, buf)
    p = t.provider
    parts = {}
    for c in ml.sectors:
        r, q = ml.shape[c]
        qq, rr = torch.linalg.qr(buf[ml.base[c]:ml.base[c] + r * q].view(r, q).T)
        parts[c] = (rr.T, qq.T)
    bond = GradedSpace.new(p, {p.sector(c): min(ml.shape[c]) for c in ml.sectors})
    sl = TensorStructure((*m.codomain, Leg(bond, IN)))
    sq = TensorStructure((Leg(bond, OUT), *m.domain))
    dev = t.arena.device

    def assemble(structure, piece):
        lay = matrix_layout(structure)
        mbuf = torch.empty(lay.size, dtype=torch.float64, device=dev)
        for c in lay.sectors:
            r, q = lay.shape[c]
            mbuf[lay.base[c]:lay.base[c] + r * q].view(r, q).copy_(piece(c))
        out = SymmetricTensor.empty(structure)
        _raise_exec(structure).run(mbuf, out.arena)
        return out

    return assemble(sl, lambda c: parts[c][0]), assemble(sq, lambda c: parts[c][1])
