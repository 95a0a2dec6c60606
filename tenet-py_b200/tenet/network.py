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

from collections.abc import Callable, Sequence
from typing import NamedTuple

import numpy as np
import torch

from tenet import ops
from tenet.structure import OUT
from tenet.tensor import SymmetricTensor

__all__ = ["DMRG_out", "Env", "MPO", "MPS", "Sweep", "composed", "ctmrg", "dmrg_", "local_op",
           "env_update_first", "env_update_last", "heff2", "lanczos", "spectrum", "sweep_"]


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


def fold_left(fl: SymmetricTensor, w1: SymmetricTensor) -> SymmetricTensor:
    """``F[(n-1, n)] . W[n]`` on ``(a, B, P, p, m)``: the left environment with the left
    site's MPO tensor folded in (the reference's prepared path folds its environments the
    same way once per solve, ``network/env.py:234-264``)."""
    return ops.einsum("axB,xPpm->aBPpm", fl, w1)


def fold_right(w2: SymmetricTensor, fr: SymmetricTensor) -> SymmetricTensor:
    """``W[n+1] . F[(n+2, n+1)]`` on ``(m, Q, q, r, s)``."""
    return ops.einsum("mQqy,rys->mQqrs", w2, fr)


def env_update_last_folded(lf: SymmetricTensor, a: SymmetricTensor,
                           bra_site: SymmetricTensor | None = None) -> SymmetricTensor:
    """``F[(n, n+1)]`` from ``lf = fold_left(F[(n-1, n)], W[n])``: the ket contracted into
    the folded environment, then the bra -- two contractions instead of three, the same
    operator as ``env_update_last`` (``network/env.py:618-626``)."""
    bra = ops.adjoint(a if bra_site is None else bra_site)
    t = ops.einsum("aBPpm,apr->BrPm", lf, a)
    return ops.einsum("BPs,BrPm->rms", bra, t)


def env_update_first_folded(rf: SymmetricTensor, a: SymmetricTensor,
                            bra_site: SymmetricTensor | None = None) -> SymmetricTensor:
    """``F[(n, n-1)]`` from ``rf = fold_right(W[n], F[(n+1, n)])``: the counterpart of
    ``env_update_last_folded`` for ``env_update_first`` (``network/env.py:627-633``)."""
    bra = ops.adjoint(a if bra_site is None else bra_site)
    t = composed("apr,xPprs->axPs", a, rf, bend="p")
    return composed("axPs,BPs->axB", t, bra, bend="P")


def heff2_folded(lf: SymmetricTensor, rf: SymmetricTensor, aa: SymmetricTensor) -> SymmetricTensor:
    """``H_eff @ aa`` from the folded environments: ``(aa . rf) . lf``."""
    t = ops.einsum("apqr,mQqrs->apmQs", aa, rf)
    return ops.einsum("apmQs,aBPpm->BPQs", t, lf)


def env_update_last(f: SymmetricTensor, a: SymmetricTensor, w: SymmetricTensor,
                    bra_site: SymmetricTensor | None = None) -> SymmetricTensor:
    """``F[(n, n+1)]`` from ``F[(n-1, n)]`` (``network/env.py:618-626``); the bra site is
    ``a`` unless ``bra_site`` is given."""
    bra = ops.adjoint(a if bra_site is None else bra_site)
    t = ops.einsum("axB,apr->xBpr", f, a)
    t = ops.einsum("xPpm,xBpr->BrPm", w, t)
    return ops.einsum("BPs,BrPm->rms", bra, t)


def env_update_first(f: SymmetricTensor, a: SymmetricTensor, w: SymmetricTensor,
                     bra_site: SymmetricTensor | None = None) -> SymmetricTensor:
    """``F[(n, n-1)]`` from ``F[(n+1, n)]`` (``network/env.py:627-633``); the bra site is
    ``a`` unless ``bra_site`` is given."""
    bra = ops.adjoint(a if bra_site is None else bra_site)
    t = ops.einsum("apr,rys->apys", a, f)
    t = composed("apys,xPpy->axPs", t, w, bend="p")
    return composed("axPs,BPs->axB", t, bra, bend="P")


def _orthonormal(vectors) -> tuple:
    """Gram-Schmidt of ``vectors`` against each other, null ones dropped
    (``network/dmrg.py:70-87``): ``(vector, <vector, vector>)`` pairs."""
    basis: list = []
    for t in vectors:
        t = _project_out(t, basis)
        gram = float(ops.inner(t, t))
        if abs(gram) > 1e-24 and float(ops.norm(t)) > 1e-12:
            basis.append((t, gram))
    return tuple(basis)


def _project_out(t: SymmetricTensor, basis) -> SymmetricTensor:
    """``t - sum_k b_k <b_k, t> / <b_k, b_k>`` (``network/dmrg.py:90-103``)."""
    for b, gram in basis:
        t = ops.subtract(t, b * (float(ops.inner(b, t)) / gram))
    return t


def lanczos(matvec: Callable[[SymmetricTensor], SymmetricTensor], v: SymmetricTensor, *,
            ncv: int = 3, tol: float = 1e-13, orthogonal_to: Sequence[SymmetricTensor] = (),
            correct: Callable[[SymmetricTensor], SymmetricTensor] | None = None
            ) -> tuple[float, SymmetricTensor]:
    """Ground Ritz pair of a Hermitian ``matvec`` (``network/dmrg.py:106-227``).

    ``orthogonal_to`` holds the solve orthogonal to the given vectors by hard projection
    of the start vector and of every matvec result (the reference's rule; ``ValueError``
    when the projected start vector vanishes).  ``correct`` is the FP64 correction of the
    precision form: when ``matvec`` runs its products in reduced precision, the returned
    energy is the Rayleigh quotient ``<v|H v>`` of the Ritz vector under the FP64
    operator ``correct`` -- one FP64 matvec per solve -- whose error is quadratic in the
    Ritz vector's."""
    basis = _orthonormal(orthogonal_to)
    if basis:
        v = _project_out(v, basis)
        if float(ops.norm(v)) < 1e-12:
            raise ValueError("the start vector lies in the span of orthogonal_to, so there is "
                             "no vector left to iterate on at this bond")
        full = matvec

        def matvec(x: SymmetricTensor) -> SymmetricTensor:
            return _project_out(full(x), basis)

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
    out = out / ops.norm(out)
    if correct is not None:
        return ops.inner(out, correct(out)), out
    return float(values[0]), out


class DeviceLanczos:
    """The reference's Lanczos (``network/dmrg.py:106-227``) with the whole recurrence on
    the device: one library call (``tnb_lanczos_solve``) launches the ``ncv`` matvecs --
    the program's recorded launch sequence replayed on each Krylov vector -- every
    ``alpha``/``beta``, the three-term update and the happy-breakdown stop, with
    device-resident scalars.  The host then makes one synchronising read of the
    tridiagonal, solves it with ``np.linalg.eigh`` exactly as the reference does, and a
    second call (``tnb_lanczos_ritz``) forms and normalises the Ritz vector (and, in the
    precision form, applies the FP64 correction program for the Rayleigh-quotient
    energy)."""

    def __init__(self, program, ncv: int, tol: float = 1e-13, correct=None,
                 reorthogonalize: bool | None = None, residual: bool = True) -> None:
        """``reorthogonalize`` (default: on exactly when ``correct`` is given, i.e. in the
        precision form) adds classical Gram-Schmidt, applied twice, of every new Krylov
        vector against all earlier ones in FP64.  A reduced-precision matvec never drives
        ``beta`` below an absolute breakdown tolerance, so without it the recurrence runs
        on past an exhausted Krylov space and produces spurious Ritz values; the FP64
        form keeps the reference's unreorthogonalised recurrence."""
        from tenet import _exec, _lib
        from tenet.structure import layout

        self.program, self.ncv, self.tol, self.correct = program, ncv, tol, correct
        # the precision form's FP64 residual correction of the Ritz vector (``finish``)
        self.residual = residual and correct is not None
        self.reorth = (correct is not None) if reorthogonalize is None else reorthogonalize
        s = program.in_struct
        n = layout(s).size
        dev = _exec.device()
        f64 = dict(dtype=torch.float64, device=dev)
        self.n = n
        self.V = torch.zeros((ncv + 1, max(n, 1)), **f64)
        self.W = torch.zeros(max(n, 1), **f64)
        self.W2 = torch.zeros(max(n, 1), **f64)
        self.state = torch.zeros(3 * ncv + 2, **f64)
        self.scal = torch.zeros(2, **f64)  # [0] a squared norm, [1] the corrected energy
        self.coef = torch.zeros(ncv, **f64)
        # the rows' addresses, computed on the device (no host -> device copy, no sync)
        self.ptrs = self.V.data_ptr() + torch.arange(ncv, dtype=torch.int64, device=dev) \
            * (self.V.stride(0) * self.V.element_size())
        lib = _lib.load()
        self.work = torch.zeros(int(lib.tnb_dot_work_bytes(n)), dtype=torch.uint8, device=dev)
        self.mwork = torch.zeros(int(lib.tnb_multi_dot_work_bytes(n, ncv)) if self.reorth
                                 else 1, dtype=torch.uint8, device=dev)
        self.gs = torch.zeros(ncv, **f64)
        self.runs = ops._runs(s)
        self._host_state = torch.zeros(3 * ncv + 2, dtype=torch.float64).pin_memory()
        self._host_coef = torch.zeros(ncv, dtype=torch.float64).pin_memory()
        self._uses, self._graph, self._x0 = 0, None, None
        if self.residual:
            # residual r, its image Hr, the previous direction p and Hp, and a scratch
            self.R, self.W3, self.Pd, self.HP, self.T = (
                torch.zeros(max(n, 1), **f64) for _ in range(5))
            self.dots = torch.zeros(12, **f64)
            self._host_dots = torch.zeros(12, dtype=torch.float64).pin_memory()

    #: replay a solve from a CUDA graph once the same solver runs a second time (a bond
    #: whose structure came back in the next sweep); a solver used once runs eagerly.
    #: Off by default: capturing and instantiating a solve's graph took ~6 ms on B200
    #: against ~0.6 ms of launches saved per replay, and a DMRG solve reuses a bond's
    #: solver about six times (L = 64 warm solve 1.65 s with it, 1.53 s without)
    GRAPH = False

    def _solve_call(self, x: torch.Tensor) -> None:
        from tenet import _exec, _lib

        P, p, r = _exec.ptr, self.program, self.runs
        _lib.call("tnb_lanczos_solve", p.exec_seq.handle, P(p.x_slot), P(p.y_slot), self.n,
                  self.ncv, float(self.tol), int(self.reorth), P(x), P(self.V),
                  self.V.stride(0), P(self.W), P(self.state), P(self.scal),
                  P(self.ptrs), P(self.gs), P(r.start), P(r.weight), r.n_runs, P(self.work),
                  P(self.mwork), _exec.stream_ptr())

    def launch(self, x: torch.Tensor) -> None:
        """Enqueue the recurrence from start vector ``x`` (an arena of ``n`` doubles).  The
        first call launches its ~9 ncv kernels one by one; from the second on, the whole
        solve -- every buffer it touches is this solver's own and fixed -- is one graph
        launch after a copy of ``x`` into the solver's start buffer."""
        if not (self.GRAPH and self._uses) or self._graph is False:
            self._uses += 1
            self._solve_call(x)
            return
        if self._graph is None:
            self._x0 = torch.empty_like(self.W)
            g = torch.cuda.CUDAGraph()
            side = torch.cuda.Stream()
            try:
                with torch.cuda.stream(side):
                    g.capture_begin(capture_error_mode="thread_local")
                    try:
                        self._solve_call(self._x0)
                    finally:
                        g.capture_end()
            except RuntimeError:  # a stream that cannot be captured: stay eager
                self._graph = False
                return self.launch(x)
            self._graph = g
        self._x0[:self.n].copy_(x.reshape(-1)[:self.n])
        self._graph.replay()
        self._uses += 1

    def tridiagonal(self) -> tuple[np.ndarray, np.ndarray]:
        """Ground eigenpair of the recorded tridiagonal (one synchronising read)."""
        self._host_state.copy_(self.state)
        st = self._host_state.numpy()
        ncv = self.ncv
        m = int(st[3 * ncv])
        alphas, betas = st[:m], st[ncv:ncv + m - 1]
        tri = np.diag(alphas) + np.diag(betas, 1) + np.diag(betas, -1)
        values, states = np.linalg.eigh(tri)
        coef = np.zeros(ncv)
        coef[:m] = states[:, 0]
        return values, coef

    def ritz(self, coef: np.ndarray, out: torch.Tensor) -> None:
        """Enqueue the normalised Ritz vector ``sum_j coef[j] v_j`` into ``out`` (and the
        corrected energy into ``scal[1]`` in the precision form)."""
        from tenet import _exec, _lib

        P, c, r = _exec.ptr, self.correct, self.runs
        self._host_coef.numpy()[:] = coef
        self.coef.copy_(self._host_coef, non_blocking=True)
        _lib.call("tnb_lanczos_ritz", c.exec_seq.handle if c is not None else None,
                  P(c.x_slot) if c is not None else None, P(c.y_slot) if c is not None else None,
                  self.n, self.ncv, P(self.coef), P(self.ptrs), P(out), P(self.W2),
                  P(self.scal), P(r.start), P(r.weight), r.n_runs, P(self.work),
                  _exec.stream_ptr())

    def finish(self) -> tuple[float, SymmetricTensor]:
        """After ``launch``: read the tridiagonal, form the Ritz vector, return the pair.
        In the precision form the pair is then corrected in FP64 (``_residual_step``)."""
        values, coef = self.tridiagonal()
        out = SymmetricTensor.empty(self.program.in_struct)
        self.ritz(coef, out.arena)
        if self.correct is not None:
            if self.residual:
                return self._residual_step(out)
            return float(self.scal[1].item()), out
        return float(values[0]), out

    def _dot(self, x: torch.Tensor, y: torch.Tensor, k: int) -> None:
        from tenet import _exec, _lib

        P, r = _exec.ptr, self.runs
        _lib.call("tnb_weighted_dot", P(x), P(y), self.n, P(r.start), P(r.weight), r.n_runs,
                  P(self.work), P(self.dots) + 8 * k, _exec.stream_ptr())

    #: FP64 refinement steps after a reduced-precision solve, and the relative residual
    #: ``|Hx - theta x| / |theta|`` at which they stop early
    REFINE_STEPS = 4
    REFINE_TOL = 1e-12

    def _residual_step(self, out: SymmetricTensor) -> tuple[float, SymmetricTensor]:
        """The FP64 residual correction of the reduced-precision Ritz vector: locally
        optimal block-free steps (Knyazev's LOBPCG with one vector) in FP64.  With ``x`` the
        normalised Ritz vector, ``Hx`` its FP64 image (formed by the Ritz call) and ``r =
        Hx - theta x`` the FP64 residual, each step takes the lowest Ritz pair of the FP64
        operator on span{x, r, p} (``p`` the previous step's direction; span{x, r} on the
        first step): one FP64 matvec (``H r``; ``H x`` and ``H p`` follow by linearity) and
        a 3 x 3 generalised eigenproblem on the host.  Up to ``REFINE_STEPS`` steps, ending
        once the relative residual is below ``REFINE_TOL``; a basis that has become
        numerically dependent drops ``p``, then stops."""
        from tenet import ops

        x, hx, r, hr, p, hp, t = out.arena, self.W2, self.R, self.W3, self.Pd, self.HP, self.T
        theta = float(self.scal[1].item())
        have_p = False
        for _ in range(self.REFINE_STEPS):
            ops.axpby_into(1.0, hx, -theta, x, r)
            self.correct.run(r, hr)
            pairs = [(x, x), (x, hx), (x, r), (r, r), (r, hx), (r, hr)]
            if have_p:
                pairs += [(x, p), (r, p), (p, p), (x, hp), (r, hp), (p, hp)]
            for k, (a, b) in enumerate(pairs):
                self._dot(a, b, k)
            self._host_dots.copy_(self.dots)
            d = self._host_dots.numpy()
            sxx, hxx, sxr, srr, hrx, hrr = (float(v) for v in d[:6])
            if not srr > 0.0 or srr ** 0.5 <= self.REFINE_TOL * abs(theta) * sxx ** 0.5:
                break
            A = [[hxx, hrx], [hrx, hrr]]
            B = [[sxx, sxr], [sxr, srr]]
            if have_p:
                sxp, srp, spp, hxp, hrp, hpp = (float(v) for v in d[6:12])
                A = [[hxx, hrx, hxp], [hrx, hrr, hrp], [hxp, hrp, hpp]]
                B = [[sxx, sxr, sxp], [sxr, srr, srp], [sxp, srp, spp]]
            lam = c = None
            try:
                import scipy.linalg

                lam, vec = scipy.linalg.eigh(np.array(A), np.array(B))
                c = vec[:, 0]
            except Exception:  # numerically dependent: retry without p, else stop
                if not have_p:
                    break
                have_p = False
                continue
            if not np.isfinite(lam[0]) or lam[0] > theta + 1e-14 * abs(theta):
                break  # the span holds x, so a larger value is rounding: keep the pair
            c1, c2 = float(c[1]), float(c[2]) if have_p else 0.0
            # p <- c1 r + c2 p and Hp likewise; x <- c0 x + p and Hx likewise
            if have_p:
                ops.axpby_into(c1, r, c2, p, t)
                ops.axpby_into(c1, hr, c2, hp, hp)
                p, t = t, p
            else:
                ops.axpby_into(c1, r, 0.0, r, p)
                ops.axpby_into(c1, hr, 0.0, hr, hp)
            self.Pd, self.T = p, t
            c0 = float(c[0])
            ops.axpby_into(c0, x, 1.0, p, x)
            ops.axpby_into(c0, hx, 1.0, hp, hx)
            nrm = float(ops.norm(out))
            ops.axpby_into(1.0 / nrm, x, 0.0, x, x)
            ops.axpby_into(1.0 / nrm, hx, 0.0, hx, hx)
            theta = float(lam[0])
            have_p = True
        return theta, out

    def solve(self, v: SymmetricTensor) -> tuple[float, SymmetricTensor]:
        if v.structure != self.program.in_struct:
            raise ValueError("DeviceLanczos: the start vector's structure differs")
        if self.n == 0:
            return 0.0, v
        self.launch(v.arena)
        return self.finish()


# ---------------------------------------------------------------------------------------
# MPS / MPO / environments / sweeps  (network/mps.py, network/env.py, network/dmrg.py)


def ones(legs) -> SymmetricTensor:
    """A tensor with every structurally allowed entry 1 (``network/common.py:323-346``)."""
    t = SymmetricTensor.zeros(legs)
    t.arena.fill_(1.0)
    return t


class MPS:
    """Site tensors on the partition ``(bond OUT, phys OUT | bond IN)`` (``network/mps.py``)."""

    def __init__(self, sites, center=None) -> None:
        from tenet import ops

        self.sites = [ops.repartition(t, (0, 1), (2,)) for t in sites]
        self.center = center

    def __len__(self) -> int:
        return len(self.sites)

    def __getitem__(self, n: int) -> SymmetricTensor:
        return self.sites[n]

    def __setitem__(self, n: int, t: SymmetricTensor) -> None:
        """The write barrier: every factor is put back on ``(l, p | r)``
        (``network/mps.py:126-143``)."""
        from tenet import ops

        if t.ndim != 3:
            raise ValueError(f"an MPS site tensor is rank 3, got rank {t.ndim}")
        self.sites[n] = ops.repartition(t, (0, 1), (2,))

    @classmethod
    def random(cls, phys, bonds, *, seed: int = 0) -> "MPS":
        """Site ``i`` draws with ``seed + i`` (``network/mps.py:161-191``), so a seeded state
        here holds the reference's numbers."""
        from tenet.structure import IN, Leg

        return cls(SymmetricTensor.random((Leg(bonds[i], OUT), Leg(phys, OUT),
                                           Leg(bonds[i + 1], IN)), seed=seed + i)
                   for i in range(len(bonds) - 1))

    def save(self, path) -> None:
        """Write a directory: one ``NNN.npz`` per site plus ``mps.json``
        (``network/mps.py:567-607``; ``tenet.serialize``)."""
        from tenet import serialize

        serialize.save_mps(self, path)

    @classmethod
    def load(cls, path) -> "MPS":
        """Read a directory written by ``save`` (``network/mps.py:609-676``)."""
        from tenet import serialize

        return serialize.load_mps(path)

    def canonize_(self, to: int = 0) -> "MPS":
        """Right-canonicalise by one LQ per site from the right (``network/mps.py:312-352``).
        The LQ's gauge is the reference's (Householder QR of the transpose, LAPACK's sign
        convention), which the sweeps that follow depend on at the level of their
        unreorthogonalised Lanczos: an SVD split in another gauge of the same bonds moved
        the L = 64 run's first-sweep energy by 3e-6 per site."""
        from tenet import linalg, ops

        if to != 0:
            raise NotImplementedError("only to=0 (right-canonical) is implemented")
        for n in range(len(self) - 1, 0, -1):
            left, q = linalg.lq(self[n], ((0,), (1, 2)))
            self[n] = q
            self[n - 1] = ops.einsum("apx,xy->apy", self[n - 1], left)
        self[0] = self[0] / ops.norm(self[0])
        self.center = to
        return self


class MPO:
    """Site operators ``W = (x IN, P OUT, p IN, m OUT)`` (the materialised site-tensor form
    of ``network/mps.py:2551-2729``)."""

    def __init__(self, sites) -> None:
        self.sites = list(sites)

    @classmethod
    def identity(cls, n_sites: int, phys) -> "MPO":
        """The identity operator on ``n_sites`` sites of ``phys`` with a unit MPO bond
        (``network/mps.py:2745-2777``): the overlap operator of a two-state ``Env``."""
        from tenet.structure import GradedSpace, Leg

        sym = phys.provider
        unit = GradedSpace.new(sym, {sym.unit: 1})
        eye = ops.identity((Leg(unit, OUT), Leg(phys, OUT)))  # (u OUT, p OUT, u IN, p IN)
        return cls([ops.transpose(eye, (2, 1, 3, 0))] * n_sites)

    def materialize(self) -> "MPO":
        """The site-tensor form: this MPO already is one."""
        return self

    @classmethod
    def from_terms(cls, n_sites: int, terms) -> "MPO":
        """An MPO from a term list (``network/mps.py:3135-3341``), for the SU(2) spin-1/2
        chains of this build: every term ``(coef, [(op, (i, j))])`` with ``op`` an
        invariant two-site operator (``spin_half(SU2).ops["S.S"]`` or any combination of
        it and the identity) on sites ``i < j`` with ``j - i`` 1 or 2.  The MPO is the
        finite-state machine of ``su2_chain_mpo``; other term shapes are refused."""
        j1 = [0.0] * (n_sites - 1)
        j2 = [0.0] * max(n_sites - 2, 0)
        onsite = [0.0] * n_sites
        for term in terms:
            try:
                coef, factors = term
                ((op, where),) = factors
                i, j = where
            except (TypeError, ValueError):
                raise ValueError("from_terms: each term must be (coef, [(op, (i, j))]) with one "
                                 "invariant two-site operator") from None
            if not (0 <= i < j < n_sites) or j - i not in (1, 2):
                raise ValueError(f"from_terms: sites {(i, j)} are not neighbours or next "
                                 f"neighbours on a chain of {n_sites}")
            a, b = su2_invariant_coefficients(op.structure, op.numpy_arena())
            (j1 if j - i == 1 else j2)[i] += float(coef) * a
            onsite[i] += float(coef) * b
        return su2_chain_mpo(n_sites, j1, j2, onsite)

    def __len__(self) -> int:
        return len(self.sites)

    def __getitem__(self, n: int) -> SymmetricTensor:
        return self.sites[n]


def identity_w(aux, phys) -> SymmetricTensor:
    """A spectator MPO site: ``id(aux) (x) id(phys)`` on ``(wl IN, p OUT, p IN, wr OUT)``
    (``network/mps.py:1170-1182``), the identity that carries an open channel of a
    non-adjacent term through a site it does not touch.  Built as the reference does:
    the outer product of the two identities, then put on the MPO partition
    (``_as_w``, ``network/mps.py:1044-1056``)."""
    from tenet import ops
    from tenet.structure import IN, Leg

    t = ops.einsum("ba,pq->apqb", ops.identity((aux,)), ops.identity((Leg(phys, IN),)))
    return ops.transpose(ops.repartition(t, (1, 3), (0, 2)), (2, 0, 3, 1))


def heisenberg_mpo_su2(n_sites: int, j: float = 1.0, j2: float = 0.0) -> MPO:
    """``H = J sum_i S_i . S_{i+1} + J2 sum_i S_i . S_{i+2}`` on spin-1/2 SU(2) sites, as
    site tensors (uniform couplings; see ``su2_chain_mpo``)."""
    if n_sites < 2:
        raise ValueError("a Heisenberg chain needs at least two sites")
    return su2_chain_mpo(n_sites, [j] * (n_sites - 1), [j2] * max(n_sites - 2, 0))


def su2_chain_mpo(n_sites: int, j1, j2=(), onsite=()) -> MPO:
    """``H = sum_i j1[i] S_i . S_{i+1} + sum_i j2[i] S_i . S_{i+2} + sum_i onsite[i]`` on
    spin-1/2 SU(2) sites, as site tensors.

    The MPO bond carries the finite-state machine of the invariant terms: a spin-0 "not
    started" channel, a spin-1 channel carrying the first ``S``, and a spin-0 "finished"
    channel -- multiplets ``{0: 2, 2: 1}`` in the bulk, as the reference's
    ``MPO.from_terms(...).materialize()`` builds for ``spin_half(SU2).ops["S.S"]``.  In the
    fusion-tree basis of the blocks ``(P, m | x, p)`` the reduced coefficients are 1 for
    the identity channels, ``sqrt(3/2)`` for opening the spin-1 channel and
    ``-sqrt(3/8) J`` for closing it (their product is ``-3/4 J``, the reduced S.S).  With
    any ``j2`` nonzero a second spin-1 channel carries the opened ``S`` one site further:
    the open channel passes a site through the spectator identity (``identity_w``) and
    closes with ``-sqrt(3/8) J2`` -- the reference's reading of a non-adjacent invariant
    S.S term in ``from_terms`` (bulk multiplets ``{0: 2, 2: 2}``).  ``onsite[i]`` is a
    constant on site ``i`` (the identity part of an invariant two-site term), carried by
    the start -> finished channel.
    """
    import math

    from tenet.structure import IN, GradedSpace, Leg, TensorStructure, layout
    from tenet.symmetry import SU2

    if n_sites < 2:
        raise ValueError("a chain MPO needs at least two sites")
    j1 = [float(x) for x in j1]
    j2 = [float(x) for x in j2] + [0.0] * (max(n_sites - 2, 0) - len(j2))
    onsite = [float(x) for x in onsite] + [0.0] * (n_sites - len(onsite))
    if len(j1) != n_sites - 1 or len(j2) != max(n_sites - 2, 0) or len(onsite) != n_sites:
        raise ValueError("su2_chain_mpo: j1 needs n - 1 couplings, j2 at most n - 2, "
                         "onsite at most n")
    has_j2 = any(j2)
    phys = GradedSpace.new(SU2, {SU2.sector(1): 1})

    # states per bond: list of (label, sector two_j) in degeneracy order within a sector
    def states(b):
        if b == 0:
            st = [("start", 0)]
        elif b == n_sites:
            st = [("done", 0)]
        elif b == 1:
            st = [("start", 0), ("open", 2)]
        elif b == n_sites - 1:
            st = [("done", 0), ("open", 2)]
        else:
            st = [("start", 0), ("done", 0), ("open", 2)]
        if has_j2 and 2 <= b <= n_sites - 1:
            st.append(("open2", 2))
        return st

    def space(st):
        count: dict = {}
        for _, sec in st:
            count[sec] = count.get(sec, 0) + 1
        return GradedSpace.new(SU2, {SU2.sector(sec): m for sec, m in count.items()})

    def index(st, label):
        sec = dict(st)[label]
        return sec, [lab for lab, x in st if x == sec].index(label)

    opn, cls = math.sqrt(1.5), -math.sqrt(3.0 / 8.0)
    spec = None
    if has_j2:
        # the spectator's reduced blocks, keyed like the site tensor's own block keys
        v1 = GradedSpace.new(SU2, {SU2.sector(2): 1})
        t = identity_w(Leg(v1, IN, True), phys)
        tl, th = layout(t.structure), t.numpy_arena()
        spec = {key: th[int(tl.offsets[b]):int(tl.offsets[b]) + int(tl.sizes[b])]
                for b, key in enumerate(t.structure.keys)}
    sites = []
    for n in range(n_sites):
        sl, sr = states(n), states(n + 1)
        rules = [("start", "start", 1.0), ("done", "done", 1.0), ("start", "open", opn),
                 ("open", "done", cls * (j1[n - 1] if n >= 1 else 0.0)),
                 ("open2", "done", cls * (j2[n - 2] if n >= 2 else 0.0))]
        if onsite[n]:
            rules.append(("start", "done", onsite[n]))
        legs = (Leg(space(sl), IN, True), Leg(phys, OUT), Leg(phys, IN), Leg(space(sr), OUT, True))
        s = TensorStructure(legs)
        lay = layout(s)
        host = np.zeros(lay.size)
        for b, key in enumerate(s.keys):
            ot, it = key
            (ps, ms), _, c = ot
            (xs, pps), _, _ = it
            shape = tuple(int(x) for x in lay.shapes[b])
            blk = np.zeros(shape)
            if c == 1:  # the spin-1/2 coupled channel carries the single-site operators
                for a, bb, v in rules:
                    if a not in dict(sl) or bb not in dict(sr):
                        continue
                    xsec, xi = index(sl, a)
                    msec, mi = index(sr, bb)
                    if xsec == xs and msec == ms:
                        blk[xi, 0, 0, mi] = v
            if spec is not None and key in spec and "open" in dict(sl) \
                    and "open2" in dict(sr):
                _, xi = index(sl, "open")
                _, mi = index(sr, "open2")
                blk[xi, 0, 0, mi] = spec[key][0]
            o = int(lay.offsets[b])
            host[o:o + blk.size] = blk.ravel()
        sites.append(SymmetricTensor.from_numpy_arena(s, host))
    return MPO(sites)


def local_op(matrix, *, phys, charge=None) -> SymmetricTensor:
    """A dense two-site operator on spin-1/2 SU(2) sites as the invariant rank-4 tensor on
    ``(p OUT, p OUT, p IN, p IN)`` (``network/mps.py:960-1041``, the ``charge=None`` form).
    The dense basis is the reference's: magnetic index descending (``m = j - k``).  On two
    spin-1/2 sites an invariant operator is ``t0`` on the singlet and ``t2`` on the
    triplet; those are its two blocks.  A matrix that is not invariant is refused."""
    from tenet.structure import IN, Leg, TensorStructure

    m = np.asarray(matrix, dtype=np.float64)
    if charge is not None or phys.provider.name != "SU2" \
            or dict((a.two_j, k) for a, k in phys.sectors) != {1: 1} or m.size != 16:
        raise ValueError("local_op: this build constructs invariant two-site operators on "
                         "spin-1/2 SU(2) sites only")
    m = m.reshape(4, 4)
    singlet = np.array([0.0, 1.0, -1.0, 0.0]) / np.sqrt(2.0)
    t0 = float(singlet @ m @ singlet)
    t2 = float(m[0, 0])
    want = t2 * np.eye(4) + (t0 - t2) * np.outer(singlet, singlet)
    if np.abs(m - want).max() > 1e-12 * max(1.0, np.abs(m).max()):
        raise ValueError("local_op: the matrix is not SU(2)-invariant")
    s = TensorStructure((Leg(phys, OUT), Leg(phys, OUT), Leg(phys, IN), Leg(phys, IN)))
    host = np.array([t0 if key[0][2] == 0 else t2 for key in s.keys])
    return SymmetricTensor.from_numpy_arena(s, host)


def su2_invariant_coefficients(structure, host: np.ndarray) -> tuple[float, float]:
    """``(a, b)`` with ``T = a S.S + b 1`` for an SU(2)-invariant two-site operator ``T``
    on spin-1/2 legs ``(p OUT, p OUT, p IN, p IN)`` given by its structure and block arena.
    On two spin-1/2 sites the invariant operators are spanned by the identity and ``S.S``
    (one reduced value per total spin: ``-3/4`` and ``1/4`` for ``S.S``)."""
    from tenet.structure import IN

    legs = structure.legs
    ok = len(legs) == 4 and all(leg.space.provider.name == "SU2" for leg in legs) \
        and [leg.side is IN for leg in legs] == [False, False, True, True] \
        and all(dict((a.two_j, m) for a, m in leg.space.sectors) == {1: 1} for leg in legs)
    if not ok:
        raise ValueError("from_terms: a two-site SU(2) term must be an invariant operator on "
                         "spin-1/2 legs (p OUT, p OUT, p IN, p IN), as spin_half(SU2).ops['S.S']")
    vals = {}
    for key, v in zip(structure.keys, host):
        vals[key[0][2]] = float(v)
    t0, t2 = vals.get(0, 0.0), vals.get(2, 0.0)
    a = t2 - t0
    return a, t2 - a / 4.0
class Env:
    """``<bra|H|psi>`` environments keyed by directed bond (``network/env.py:435-645``):
    ``F[(n, n+1)] = (ket IN, mpo OUT, bra OUT)`` from sites ``<= n``, ``F[(n, n-1)] =
    (ket OUT, mpo IN, bra IN)`` from sites ``>= n``; ``bra`` defaults to ``psi``.

    ``compile`` is the reference's injection seam (``network/env.py:448-453,750-769``): a
    callable that wraps the bond's two-site matvec once per structure key, and whose result
    then serves every ``heff2`` call with that key.  Without it the matvec runs as this
    build's compiled form (``compiled=True``): a recorded, graph-captured chain program
    rebuilt whenever the bond's structures change, and a device-resident Lanczos."""

    def __init__(self, psi: MPS, h: MPO, *, bra: MPS | None = None, compile=None,
                 compiled: bool = True, precision: str = "f64",
                 tc_min_flops: int | None = None, fold: bool = True) -> None:
        from tenet.structure import IN, Leg

        self.psi, self.h, self.compiled, self.precision = psi, h, compiled, precision
        self.fold = fold
        self.bra = psi if bra is None else bra
        self.compile = compile
        self.tc_min_flops = tc_min_flops
        n = len(psi)
        kl, kr = psi[0].legs[0], psi[n - 1].legs[2]
        bl, br = self.bra[0].legs[0], self.bra[len(self.bra) - 1].legs[2]
        wl, wr = h[0].legs[0], h[n - 1].legs[3]
        self.F = {
            (-1, 0): ones((Leg(kl.space, IN, kl.dual), Leg(wl.space, OUT, wl.dual),
                           Leg(bl.space, OUT, bl.dual))),
            (n, n - 1): ones((Leg(kr.space, OUT, kr.dual), Leg(wr.space, IN, wr.dual),
                              Leg(br.space, IN, br.dual))),
        }
        self._prog: dict = {}
        self._wrapped: dict = {}
        self._lf: dict = {}  # bond n -> (F[(n-1, n)] it was folded from, fold_left)
        self._rf: dict = {}  # bond n -> (F[(n+2, n+1)] it was folded from, fold_right)

    def fold_l(self, n: int) -> SymmetricTensor:
        """``fold_left(F[(n-1, n)], W[n])``, kept while that environment is unchanged."""
        f = self.F[n - 1, n]
        hit = self._lf.get(n)
        if hit is None or hit[0] is not f:
            hit = (f, fold_left(f, self.h[n]))
            self._lf[n] = hit
        return hit[1]

    def fold_r(self, n: int) -> SymmetricTensor:
        """``fold_right(W[n+1], F[(n+2, n+1)])``, kept while that environment is unchanged."""
        f = self.F[n + 2, n + 1]
        hit = self._rf.get(n)
        if hit is None or hit[0] is not f:
            hit = (f, fold_right(self.h[n + 1], f))
            self._rf[n] = hit
        return hit[1]

    @property
    def device_solves(self) -> bool:
        """Whether a sweep solves this env's bonds by the device-resident Lanczos."""
        return self.compiled and self.compile is None and self.bra is self.psi

    def setup_(self, to: int = 0) -> "Env":
        if to != 0:
            raise NotImplementedError("only to=0 is implemented; canonize_ has the same note")
        for n in range(len(self.psi) - 1, 0, -1):
            self.update_(n, to="first")
        return self

    def update_(self, n: int, *, to: str) -> None:
        """With ``fold``, an environment whose MPO site is already folded into the old one
        (the bond's matvec folded it) grows through that fold: two contractions."""
        bra = None if self.bra is self.psi else self.bra[n]
        if to == "last":
            hit = self._lf.get(n)
            if self.fold and hit is not None and hit[0] is self.F.get((n - 1, n)):
                self.F[n, n + 1] = env_update_last_folded(hit[1], self.psi[n], bra)
            else:
                self.F[n, n + 1] = env_update_last(self.F[n - 1, n], self.psi[n], self.h[n], bra)
        else:
            hit = self._rf.get(n - 1)
            if self.fold and hit is not None and hit[0] is self.F.get((n + 1, n)):
                self.F[n, n - 1] = env_update_first_folded(hit[1], self.psi[n], bra)
            else:
                self.F[n, n - 1] = env_update_first(self.F[n + 1, n], self.psi[n], self.h[n],
                                                    bra)

    def clear_(self, *sites: int) -> None:
        for n in sites:
            self.F.pop((n, n - 1), None)
            self.F.pop((n, n + 1), None)

    def heff2(self, n: int, aa: SymmetricTensor) -> SymmetricTensor:
        fl, fr = self.F[n - 1, n], self.F[n + 2, n + 1]
        if self.compile is not None:
            key = (n, fl.structure, fr.structure, aa.structure)
            fn = self._wrapped.get(n)
            if fn is None or fn[0] != key:
                w1, w2 = self.h[n], self.h[n + 1]
                fn = (key, self.compile(lambda v: heff2(fl, w1, w2, fr, v)))
                self._wrapped[n] = fn
            return fn[1](aa)
        if not self.compiled:
            return heff2(fl, self.h[n], self.h[n + 1], fr, aa)
        return self.matvec(n, aa.structure)(aa)

    def heff2_families(self, n: int, aa: SymmetricTensor) -> tuple:
        """``heff2``'s term families, unsummed (``network/env.py:772-840``).  A site-tensor
        MPO carries no term symbols, so -- as in the reference's site-tensor path -- the
        single family is the operator's own action, ``(heff2(n, aa),)``."""
        return (self.heff2(n, aa),)

    def project2(self, n: int, aa: SymmetricTensor) -> SymmetricTensor:
        """``aa`` on the ket's bonds carried to the bra's (``network/env.py:843-920``):
        ``<bra env| H_n H_{n+1} |aa, ket env>`` by the four site-tensor contractions; with
        ``h`` the identity MPO it is the ket state's two-site reduced form in the bra's
        environment gauge."""
        return heff2(self.F[n - 1, n], self.h[n], self.h[n + 1], self.F[n + 2, n + 1], aa)

    def _bond(self, n: int, structure, precision: str) -> dict:
        """The bond's cached programs: one allocated heff2 program per precision (plus what
        was captured around it), re-packed when only the environment values changed.  With
        ``fold`` (the default) the program is the two-contraction folded form
        (``heff2_folded_program``), its operands ``fold_left`` / ``fold_right`` of the
        current environments; otherwise the reference's four-contraction order."""
        from tenet.program import heff2_folded_program, heff2_program

        fl, fr = self.F[n - 1, n], self.F[n + 2, n + 1]
        w1, w2 = self.h[n], self.h[n + 1]
        skey = (fl.structure, fr.structure, structure, self.fold)
        hit = self._prog.get((n, precision))

        def operands():
            if self.fold:
                return {"lf": self.fold_l(n), "rf": self.fold_r(n)}
            return {"fr": fr, "w2": w2, "w1": w1, "fl": fl}

        if hit is None or hit["skey"] != skey:
            # one program per bond and precision; a new structure replaces it
            ops_ = operands()
            if self.fold:
                prog = heff2_folded_program(ops_["lf"], ops_["rf"], structure,
                                            precision=precision, tc_min_flops=self.tc_min_flops)
            else:
                prog = heff2_program(fl, w1, w2, fr, structure, precision=precision,
                                     tc_min_flops=self.tc_min_flops)
            hit = {"skey": skey, "bound": (fl, fr), "captured": {}, "program": prog}
            self._prog[(n, precision)] = hit
        elif hit["bound"][0] is not fl or hit["bound"][1] is not fr:
            # same structures, new environment values: re-pack the fixed operands into the
            # program's buffers; everything captured around them stays valid
            bound = operands()
            prog = hit["program"]
            for lk, name in zip(prog.links, prog.operand_names):
                lk.b_tensor = bound[name]
            prog.refresh()
            hit["bound"] = (fl, fr)
        return hit

    def matvec(self, n: int, structure, precision: str | None = None):
        """The graph-captured matvec of bond n for the current environments, in the
        env's precision (or ``precision``)."""
        from tenet.program import GraphMatvec

        hit = self._bond(n, structure, precision or self.precision)
        if "matvec" not in hit["captured"]:
            hit["captured"]["matvec"] = GraphMatvec(hit["program"])
        return hit["captured"]["matvec"]

    def lanczos(self, n: int, structure, ncv: int) -> DeviceLanczos:
        """The bond's device Lanczos.  In the precision form its matvec is the tensor-core
        program, corrected by the FP64 one; when no product of the bond is big enough for
        the tensor cores, the precision program is all FP64 and the FP64 program serves
        alone, uncorrected."""
        correct = None
        hit = self._bond(n, structure, "f64")
        if self.precision != "f64" and \
                hit["program"].tensor_core_candidates(self.tc_min_flops):
            correct = hit["program"]
            hit = self._bond(n, structure, self.precision)
        key = ("lanczos", ncv)
        lg = hit["captured"].get(key)
        if lg is None or lg.correct is not correct:
            lg = DeviceLanczos(hit["program"], ncv, correct=correct)
            hit["captured"][key] = lg
        return lg

    def solve(self, n: int, aa: SymmetricTensor, ncv: int) -> tuple[float, SymmetricTensor]:
        """Ground Ritz pair at bond n by the device-resident Lanczos (``DeviceLanczos``)."""
        return self.lanczos(n, aa.structure, ncv).solve(aa)

    def correction(self, n: int):
        """The FP64 matvec that corrects a reduced-precision solve at bond n (None in FP64)."""
        if self.precision == "f64" or not self.compiled:
            return None
        return lambda v, n=n: self.matvec(n, v.structure, "f64")(v)


def _pair(left: SymmetricTensor, right: SymmetricTensor) -> SymmetricTensor:
    from tenet import ops

    return ops.einsum("apx,xqr->apqr", left, right)


def drain(gen):
    """Run a step generator (``sweep_steps``, ``dmrg_steps``) to its return value."""
    while True:
        try:
            next(gen)
        except StopIteration as stop:
            return stop.value


class Sweep(NamedTuple):
    """One schedule entry (``network/dmrg.py:32-67``): the SVD's ``chi`` cap and
    ``cutoff``, and the noise mixed in at each split."""

    chi: int = 64
    cutoff: float = 1e-14
    noise: float = 0.0
    noise_type: str = "wavefunction"


#: The two spellings of ``noise``; each also decides the decimation (``dmrg.py:229-231``).
_NOISE_TYPES = ("wavefunction", "perturbative")


class DMRG_out(NamedTuple):
    """The record ``dmrg_`` returns and hands its ``callback`` (``network/dmrg.py:564-617``):
    ``history`` holds one ``(energy, denergy, dSchmidt, discarded)`` per sweep and
    ``schedule`` the realised ``Sweep`` entries."""

    sweeps: int
    energy: float
    denergy: float
    max_dSchmidt: float
    max_discarded_weight: float
    history: list
    schedule: list
    psi: MPS


def _schmidt_change(old: dict, new: dict) -> float:
    """``max_k ||S_k - S_k^old||`` over bonds, zero-padded; infinite before any history
    (``network/dmrg.py:545-561``)."""
    if not old:
        return float("inf")
    worst = 0.0
    for n, current in new.items():
        previous = old.get(n, [])
        m = max(len(previous), len(current))
        a = previous + [0.0] * (m - len(previous))
        b = current + [0.0] * (m - len(current))
        worst = max(worst, sum((x - y) ** 2 for x, y in zip(a, b, strict=True)) ** 0.5)
    return worst


def _rho(m: SymmetricTensor, forward: bool) -> SymmetricTensor:
    from tenet import ops

    return ops.compose(m, ops.adjoint(m)) if forward else ops.compose(ops.adjoint(m), m)


def _perturbations(env: Env, n: int, aa: SymmetricTensor, noise: float) -> tuple:
    """The operator's families on ``aa``, each normalised, scaled to total squared norm
    ``noise`` (``network/dmrg.py:251-272``)."""
    from tenet import ops

    parts = [(q, float(ops.norm(q))) for q in env.heff2_families(n, aa)]
    live = [(q, w) for q, w in parts if w > 0.0]
    if not live:
        return ()
    scale = (noise / len(live)) ** 0.5
    return tuple(q * (scale / w) for q, w in live)


def _split_dm(aa, forward, *, chi, cutoff, perturbations=(), budget="dense"):
    """The density-matrix split of perturbative noise (``network/dmrg.py:275-318``):
    ``svd_truncated`` of ``rho = tr aa aa^dag`` plus the perturbations' ``rho``, with
    ``cutoff_mode="rsum1"``; returns ``(left, right, s)``."""
    from tenet import linalg, ops

    m = ops.repartition(aa, (0, 1), (2, 3))
    rho = _rho(m, forward)
    for q in perturbations:
        rho = ops.add(rho, _rho(ops.repartition(q, (0, 1), (2, 3)), forward))
    v, w, _ = linalg.svd_truncated(rho, max_bond=chi, cutoff=cutoff, cutoff_mode="rsum1",
                                   budget=budget)
    s = ops.block_sqrt(w)
    if forward:
        return v, ops.compose(ops.adjoint(v), m), s
    return ops.compose(m, v), ops.transpose(ops.adjoint(v), (2, 0, 1)), s


def sweep_steps(psi: MPS, h: MPO, env: Env, schmidt: dict | None = None, *, chi: int,
                cutoff: float, ncv: int = 3, noise: float = 0.0,
                noise_type: str = "wavefunction", orthogonal_to=(), seed: int = 0,
                budget: str = "dense"):
    """One left-to-right then right-to-left two-site sweep (``network/dmrg.py:321-542``)
    as a generator: with the device Lanczos it yields right after each bond's solve is
    enqueued on the current stream and again after its truncation is (so a scheduler can
    run other work while the device computes); it returns ``(energy, max discarded
    weight)``.  ``schmidt`` (bond ->
    spectrum) is updated in place.  ``budget="reduced"`` caps the number of kept
    multiplets at ``chi`` instead of the reference's dense dimension (a build-side mode
    with no reference counterpart)."""
    from tenet import linalg, ops

    if noise_type not in _NOISE_TYPES:
        raise ValueError(f"noise_type={noise_type!r} is not one of {_NOISE_TYPES}; it decides "
                         "the decimation as well as the perturbation")
    n_sites = len(psi)
    energy, max_dw = 0.0, 0.0
    for direction in ("right", "left"):
        forward = direction == "right"
        bonds = range(n_sites - 1) if forward else range(n_sites - 2, -1, -1)
        for n in bonds:
            aa = _pair(psi[n], psi[n + 1])
            if orthogonal_to:
                proj = [o.project2(n, _pair(o.psi[n], o.psi[n + 1])) for o in orthogonal_to]
                energy, aa = lanczos(lambda v, n=n: env.heff2(n, v), aa, ncv=ncv,
                                     orthogonal_to=proj)
            elif env.device_solves:
                lz = env.lanczos(n, aa.structure, ncv)
                if lz.n:
                    lz.launch(aa.arena)
                    yield n
                    energy, aa = lz.finish()
                else:
                    energy = 0.0
            else:
                energy, aa = lanczos(lambda v, n=n: env.heff2(n, v), aa, ncv=ncv)
            if noise and noise_type == "perturbative":
                left, right, s = _split_dm(aa, forward, chi=chi, cutoff=cutoff, budget=budget,
                                           perturbations=_perturbations(env, n, aa, noise))
                carrier = right if forward else left
                norm_c = ops.norm(carrier)
                max_dw = max(max_dw, 1.0 - float(norm_c / ops.norm(aa)) ** 2)
                psi[n] = left if forward else left / norm_c
                psi[n + 1] = right / norm_c if forward else right
                if schmidt is not None:
                    schmidt[n] = spectrum(s / ops.norm(s))
            else:
                if noise:
                    r = SymmetricTensor.random(aa.legs, seed=seed + n)
                    aa = ops.add(aa, r * float(noise * ops.norm(aa) / ops.norm(r)))
                    aa = aa / ops.norm(aa)
                pending = linalg.svd_truncated_launch(
                    aa, ((0, 1), (2, 3)), max_bond=chi, cutoff=cutoff, budget=budget)
                if env.device_solves:
                    yield n  # the decision is on its way back: a scheduler runs others
                u, s, vh, sel, kept = linalg.svd_truncated_finish(pending)
                # Pythagoras from the decision's read-back: |S|^2 is the kept qdim-weighted
                # sum of sigma^2 and |aa|^2 the whole one (the reference takes both norms
                # numerically, network/dmrg.py:514-517)
                qd = aa.provider._qdim
                norm_s = sum(qd(c) * x * x for x, c in kept) ** 0.5
                norm_aa = (sel.discarded_weight + norm_s * norm_s) ** 0.5
                max_dw = max(max_dw, 1.0 - float(norm_s / norm_aa) ** 2)
                s = s / norm_s
                psi[n + 1] = vh
                if forward:
                    psi[n] = u
                    psi[n + 1] = ops.einsum("xy,yqr->xqr", s, psi[n + 1])
                else:
                    psi[n] = ops.einsum("apx,xy->apy", u, s)
                if schmidt is not None:
                    schmidt[n] = sorted((x * qd(c) ** 0.5 / norm_s for x, c in kept),
                                        reverse=True)
            psi.center = n + 1 if forward else n
            for e in (env, *orthogonal_to):
                e.clear_(n, n + 1)
                if forward:
                    e.update_(n, to="last")
                else:
                    e.update_(n + 1, to="first")
    return energy, max_dw


def sweep_(psi: MPS, h: MPO, env: Env, schmidt: dict | None = None, *, chi: int,
           cutoff: float, ncv: int = 3, noise: float = 0.0, noise_type: str = "wavefunction",
           orthogonal_to=(), seed: int = 0, budget: str = "dense"):
    """One two-site sweep; returns ``(energy, max discarded weight)``."""
    return drain(sweep_steps(psi, h, env, schmidt, chi=chi, cutoff=cutoff, ncv=ncv,
                             noise=noise, noise_type=noise_type, orthogonal_to=orthogonal_to,
                             seed=seed, budget=budget))


def dmrg_steps(psi: MPS, h: MPO, *, schedule=None, chi: int | None = None,
               cutoff: float | None = None, energy_tol: float = 1e-12,
               schmidt_tol: float = 1e-8, max_sweeps: int = 40, ncv: int = 3,
               orthogonal_to=None, seed: int = 0, callback=None, compile=None,
               compiled: bool = True, precision: str = "f64",
               tc_min_flops: int | None = None, budget: str = "dense", fold: bool = True):
    """``dmrg_`` as a step generator (see ``sweep_steps``); returns the ``DMRG_out``."""
    if schedule is not None:
        if chi is not None or cutoff is not None:
            raise ValueError("pass either schedule=[Sweep(chi=..., cutoff=...), ...] or the "
                             "flat chi= / cutoff= kwargs, not both")
        plan = list(schedule)
        if not plan:
            raise ValueError("schedule is empty; a run needs at least one Sweep entry")
    else:
        plan = [Sweep(64 if chi is None else chi, 1e-14 if cutoff is None else cutoff)]
    psi.canonize_(0)
    env = Env(psi, h, compile=compile, compiled=compiled, precision=precision,
              tc_min_flops=tc_min_flops, fold=fold).setup_(0)
    orthos: tuple = ()
    if orthogonal_to:
        ident = MPO.identity(len(psi), psi[0].legs[1].space)
        ends = (psi[0].legs[0], psi[len(psi) - 1].legs[2])
        orthos = tuple(
            Env(phi, ident, bra=psi).setup_(0) for phi in orthogonal_to
            # a state whose boundary legs put it in another sector is orthogonal already
            if (phi[0].legs[0].space, phi[0].legs[0].dual) == (ends[0].space, ends[0].dual)
            and (phi[len(phi) - 1].legs[2].space, phi[len(phi) - 1].legs[2].dual)
            == (ends[1].space, ends[1].dual))
    schmidt: dict = {}
    energy = float("inf")
    history: list = []
    realized: list = []
    out = None
    for it in range(1, max_sweeps + 1):
        entry = plan[it - 1] if it <= len(plan) else plan[-1]
        old_energy, old_schmidt = energy, dict(schmidt)
        energy, max_dw = yield from sweep_steps(
            psi, h, env, schmidt, chi=entry.chi, cutoff=entry.cutoff, ncv=ncv,
            noise=entry.noise, noise_type=entry.noise_type, orthogonal_to=orthos,
            seed=seed + 977 * it, budget=budget)
        denergy = abs(old_energy - energy)
        d_schmidt = _schmidt_change(old_schmidt, schmidt)
        history.append((energy, denergy, d_schmidt, max_dw))
        realized.append(entry)
        out = DMRG_out(it, energy, denergy, d_schmidt, max_dw, history, realized, psi)
        if callback:
            callback(out)
        if denergy < energy_tol and d_schmidt < schmidt_tol and it >= len(plan) \
                and entry.noise == 0.0:
            break
    return out


def dmrg_(psi: MPS, h: MPO, *, schedule=None, chi: int | None = None,
          cutoff: float | None = None, energy_tol: float = 1e-12, schmidt_tol: float = 1e-8,
          max_sweeps: int = 40, ncv: int = 3, orthogonal_to=None, seed: int = 0,
          callback=None, compile=None, compiled: bool = True, precision: str = "f64",
          tc_min_flops: int | None = None, budget: str = "dense",
          fold: bool = True) -> DMRG_out:
    """Sweep ``psi`` to the ground state of ``h`` in place and return a ``DMRG_out``
    (``network/dmrg.py:620-843``): the same arguments, defaults, refusals, schedule rule
    (the last entry repeats), noise forms, excited-state projection and the two
    convergence criteria (``|dE| < energy_tol`` and Schmidt change ``< schmidt_tol`` in one
    noiseless sweep at the schedule's last entry).

    Beyond the reference's arguments: ``compiled`` (default) solves each bond by the
    device-resident Lanczos on a graph-captured matvec; ``precision`` "tf32" or "3xbf16"
    runs the matvec products big enough for the tensor cores there (``tc_min_flops``),
    with FP64 reorthogonalisation and the FP64 correction of every such solve, while the
    SVD and truncation stay FP64; ``budget="reduced"`` caps kept multiplets instead of
    the dense dimension; ``fold`` (default) runs the matvec as two contractions of the
    MPO-folded environments, ``fold=False`` in the reference's four-contraction order."""
    return drain(dmrg_steps(psi, h, schedule=schedule, chi=chi, cutoff=cutoff,
                            energy_tol=energy_tol, schmidt_tol=schmidt_tol,
                            max_sweeps=max_sweeps, ncv=ncv, orthogonal_to=orthogonal_to,
                            seed=seed, callback=callback, compile=compile, compiled=compiled,
                            precision=precision, tc_min_flops=tc_min_flops, budget=budget,
                            fold=fold))


# ---------------------------------------------------------------------------------------
# C4v CTMRG, single layer  (network/ctmrg.py:166-660)


def ising_bulk(beta: float) -> SymmetricTensor:
    """Classical 2D Ising transfer tensor on Z2 legs ``(l OUT, u OUT, r IN, d IN)``: the
    weights ``sum_s W[s,l] W[s,u] W[s,r] W[s,d]`` with ``W = [[sqrt cosh b, sqrt sinh b],
    [sqrt cosh b, -sqrt sinh b]]`` (the splitting of ``examples/toy_codes/ctmrg.py:162-187``),
    which is already the parity basis, so each Z2 block is one dense entry."""
    import math

    from tenet.structure import IN, GradedSpace, Leg, TensorStructure, layout
    from tenet.symmetry import Z2

    c, s = math.sqrt(math.cosh(beta)), math.sqrt(math.sinh(beta))
    w = np.array([[c, s], [c, -s]])
    dense = np.einsum("sl,su,sr,sd->lurd", w, w, w, w)
    space = GradedSpace.new(Z2, {Z2.sector(0): 1, Z2.sector(1): 1})
    st = TensorStructure((Leg(space, OUT), Leg(space, OUT), Leg(space, IN), Leg(space, IN)))
    lay = layout(st)
    host = np.zeros(lay.size)
    for b, (ot, it) in enumerate(st.keys):
        (lu, _, _), (rd, _, _) = ot, it
        host[int(lay.offsets[b])] = dense[lu[0], lu[1], rd[0], rd[1]]
    return SymmetricTensor.from_numpy_arena(st, host)


class Absorb:
    """The single-layer absorption pair over one bulk tensor (``network/ctmrg.py:217-253``)."""

    def __init__(self, bulk: SymmetricTensor) -> None:
        self.bulk = bulk

    def corner(self, c: SymmetricTensor, e: SymmetricTensor) -> SymmetricTensor:
        return ops.einsum("ab,ace,fbg,gehi->chfi", c, e, e, self.bulk)

    def edge(self, e: SymmetricTensor, p: SymmetricTensor) -> SymmetricTensor:
        big = ops.einsum("abe,gehi->abghi", e, self.bulk)
        return ops.einsum("abghi,agx,bhy->xyi", big, p, ops.adjoint(p))


def single_layer_ctm(bulk: SymmetricTensor):
    """``(absorber, c, e)``: the seed corner is the identity on the unit sector and the seed
    edge ones on ``(unit IN, unit OUT, bulk bond IN)`` (``network/ctmrg.py:337-410``)."""
    from tenet.structure import IN, GradedSpace, Leg

    p = bulk.provider
    unit = GradedSpace.new(p, {p.unit: 1})
    c = ops.identity((Leg(unit, OUT),))
    e = ones((Leg(unit, IN), Leg(unit, OUT), Leg(bulk.legs[0].space, IN)))
    return Absorb(bulk), c, e


def spectrum(s: SymmetricTensor) -> list[float]:
    """Diagonal of a singular-value tensor times sqrt(qdim), descending
    (``network/common.py:147-194``)."""
    from tenet.linalg import singular_values

    p = s.provider
    out = []
    for c, vals in singular_values(s).items():
        out.extend(float(v) * p._qdim(c) ** 0.5 for v in vals)
    return sorted(out, reverse=True)


def move(c: SymmetricTensor, e: SymmetricTensor, absorb: Absorb, *, chi: int,
         precision: str = "f64", tc_min_flops: int | None = None):
    """One C4v move (``network/ctmrg.py:451-526``): the enlarged corner's truncated SVD;
    the new corner is the singular-value tensor, the new edge is projected with ``u``.
    ``precision`` "tf32" / "3xbf16" runs the corner and edge contractions' sector
    products on the tensor cores (``ops.precision``); the SVD and truncation stay FP64."""
    from tenet import linalg

    with ops.precision(precision, tc_min_flops):
        big = absorb.corner(c, e)
    n = big.ndim // 2
    p, s, _ = linalg.svd_truncated(big, (tuple(range(n)), tuple(range(n, 2 * n))), max_bond=chi)
    with ops.precision(precision, tc_min_flops):
        e2 = absorb.edge(e, p)
    return s / ops.norm(s), e2 / ops.norm(e2), p.legs[-1].space


def ctmrg(absorb: Absorb, c: SymmetricTensor, e: SymmetricTensor, *, chi: int,
          tol: float = 1e-10, max_sweeps: int = 100, precision: str = "f64",
          tc_min_flops: int | None = None):
    """Moves until the corner spectrum changes by less than ``tol`` (``network/ctmrg.py:572-660``).
    Returns ``(c, e, bond, history)``.  ``precision``: see ``move``."""
    prev, history, bond = spectrum(c), [], None
    for _ in range(max_sweeps):
        c, e, bond = move(c, e, absorb, chi=chi, precision=precision, tc_min_flops=tc_min_flops)
        cur = spectrum(c)
        n = max(len(prev), len(cur))
        a = np.array(prev + [0.0] * (n - len(prev)))
        b = np.array(cur + [0.0] * (n - len(cur)))
        history.append(float(np.abs(a - b).max()))
        prev = cur
        if history[-1] < tol:
            break
    return c, e, bond, history


def beta_free_energy(c: SymmetricTensor, e: SymmetricTensor, bulk: SymmetricTensor) -> float:
    """``beta f = -ln kappa`` from the environment, Baxter's corner-transfer ratio
    (``examples/toy_codes/ctmrg.py:547-592`` with no unrolled moves)."""
    cc, ca, ec, ea = c, ops.adjoint(c), e, ops.adjoint(e)
    z_c = ops.full_trace(ops.einsum("ab,ac,dc,eb->de", cc, ca, cc, ca))
    z_h = ops.full_trace(ops.einsum("ab,ac,dcf,ed,eg,ghf->hb", cc, ca, ea, cc, ca, ec))
    z_a = ops.full_trace(ops.einsum("ab,acp,cd,edq,fe,gfr,gh,hks,spqr->kb",
                                    cc, ec, ca, ea, cc, ea, ca, ec, bulk))
    return -float(np.log(z_a * z_c / z_h ** 2))
