"""Two-site DMRG pieces on the hot path: the effective-Hamiltonian matvec, the
environment folds and Lanczos.

``heff2`` is the reference's site-tensor matvec ``_heff2_full`` (``network/env.py:416-432``):
right environment, then ``W[n+1]``, then ``W[n]``, then the left environment, each step a
pairwise contraction whose bent wires are named (``_composed``, ``network/env.py:60-90``).
``lanczos`` is the reference's three-term recurrence without reorthogonalisation
(``network/dmrg.py:106-227``); the vector operations run on the device, and the
``alpha``/``beta`` scalars come to the host once per step exactly as the reference's
``float()`` calls do.
"""

from __future__ import annotations

from collections.abc import Callable

import numpy as np
import torch

from tenet import ops
from tenet.structure import OUT
from tenet.tensor import SymmetricTensor

__all__ = ["composed", "env_update_first", "env_update_last", "heff2", "lanczos"]


def composed(equation: str, a: SymmetricTensor, b: SymmetricTensor, bend: str = "") -> SymmetricTensor:
    """A two-operand einsum with the wires named in ``bend`` bent first."""
    if bend:
        lhs, out = equation.split("->")
        ta, tb = lhs.split(",")

        def bent(t: SymmetricTensor, term: str):
            flip = set(bend)
            outs = tuple(i for i, ch in enumerate(term) if (t.legs[i].side is OUT) != (ch in flip))
            ins = tuple(i for i in range(len(term)) if i not in outs)
            return ops.repartition(t, outs, ins), "".join(term[i] for i in (*outs, *ins))

        a, ta = bent(a, ta)
        b, tb = bent(b, tb)
        equation = f"{ta},{tb}->{out}"
    return ops.einsum(equation, a, b)


def heff2(fl: SymmetricTensor, w1: SymmetricTensor, w2: SymmetricTensor, fr: SymmetricTensor,
          aa: SymmetricTensor) -> SymmetricTensor:
    """``H_eff @ aa`` on the bond (n, n+1): ``fl = F[(n-1, n)]``, ``w1 = W[n]``,
    ``w2 = W[n+1]``, ``fr = F[(n+2, n+1)]``."""
    t = ops.einsum("apqr,rys->apqys", aa, fr)
    t = composed("apqys,mQqy->apQms", t, w2, bend="q")
    t = composed("apQms,xPpm->aPQxs", t, w1, bend="p")
    return composed("aPQxs,axB->BPQs", t, fl, bend="a")


def env_update_last(f: SymmetricTensor, a: SymmetricTensor, w: SymmetricTensor) -> SymmetricTensor:
    """``F[(n, n+1)]`` from ``F[(n-1, n)]``, bra = ket (``network/env.py:620-625``)."""
    bra = ops.adjoint(a)
    t = ops.einsum("axB,apr->xBpr", f, a)
    t = ops.einsum("xPpm,xBpr->BrPm", w, t)
    return ops.einsum("BPs,BrPm->rms", bra, t)


def env_update_first(f: SymmetricTensor, a: SymmetricTensor, w: SymmetricTensor) -> SymmetricTensor:
    """``F[(n, n-1)]`` from ``F[(n+1, n)]``, bra = ket (``network/env.py:626-629``)."""
    bra = ops.adjoint(a)
    t = ops.einsum("apr,rys->apys", a, f)
    t = composed("apys,xPpy->axPs", t, w, bend="p")
    return composed("axPs,BPs->axB", t, bra, bend="P")


def lanczos(matvec: Callable[[SymmetricTensor], SymmetricTensor], v: SymmetricTensor, *,
            ncv: int = 3, tol: float = 1e-13) -> tuple[float, SymmetricTensor]:
    """Ground Ritz pair of a Hermitian ``matvec`` (``network/dmrg.py:106-227``)."""
    vecs = [v / ops.norm(v)]
    alphas: list[float] = []
    betas: list[float] = []
    for j in range(ncv):
        w = matvec(vecs[j])
        alphas.append(ops.inner(vecs[j], w))
        w = ops._axpby(1.0, w, -alphas[j], vecs[j])
        if j:
            w = ops._axpby(1.0, w, -betas[j - 1], vecs[j - 1])
        beta = ops.norm(w)
        if j + 1 == ncv or beta < tol:
            break
        betas.append(beta)
        vecs.append(w / beta)
    tri = np.diag(alphas) + np.diag(betas, 1) + np.diag(betas, -1)
    values, states = np.linalg.eigh(tri)
    g = states[:, 0]
    out = SymmetricTensor.empty(v.structure)
    coeffs = torch.tensor([float(x) for x in g[: len(vecs)]], dtype=torch.float64,
                          device=v.arena.device)
    ptrs = torch.tensor([x.arena.data_ptr() for x in vecs], dtype=torch.int64,
                        device=v.arena.device)
    from tenet import _exec, _lib

    _lib.call("tnb_lincomb", v.arena.numel(), len(vecs), _exec.ptr(coeffs), _exec.ptr(ptrs),
              _exec.ptr(out.arena), _exec.stream_ptr())
    return float(values[0]), out / ops.norm(out)
