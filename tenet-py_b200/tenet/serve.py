"""Served DMRG solves: a continuous-batching request loop on one GPU.

Independent ground-state solves (SU(2) J1-J2 Heisenberg chains of different lengths,
bond dimensions and couplings) are admitted as they arrive, as long as a slot is free
and their HBM footprint estimate fits the budget.  Every admitted solve keeps its MPS,
environments, compiled matvec programs and Lanczos buffers on the device, on a CUDA
stream of its own.  The loop advances each active solve by one bond step per round:
a step ends right after its Lanczos solve (one library call launching the whole
recurrence) is enqueued, so while one solve's recurrence runs on the device the host
finishes the previous step of the others (tridiagonal read, SVD truncation decision,
environment update) and enqueues their work, and the device interleaves the streams.
A solve that finishes frees its slot and its share of the budget at once, and the next
arrival is admitted in the same round (continuous batching, not a queue of whole jobs).

Every request's arithmetic is its own -- its own buffers, private split-K scratch,
deterministic kernels -- so a solve gives the same result alone and in the mix.

There is no reference counterpart: the reference runs one solve per process
(``network/dmrg.py:620-843``); this is the serving form of that driver.
"""

from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np
import torch

from tenet import network
from tenet.structure import GradedSpace
from tenet.symmetry import SU2

__all__ = ["ProcessServer", "SolveRequest", "SolveResult", "Server", "clear_plan_caches",
           "footprint_bytes", "request_stream", "solve_alone"]


@dataclass(frozen=True)
class SolveRequest:
    """One ground-state solve: ``L`` sites, ``J1 = 1``, ``J2 = j2``, dense ``chi``."""

    rid: int
    L: int
    j2: float
    chi: int
    sweeps: int = 8
    arrival: float = 0.0  # seconds after the stream starts
    seed: int = 0


@dataclass
class SolveResult:
    rid: int
    energy: float
    history: list
    arrival: float
    admitted: float
    finished: float
    footprint: int
    request: SolveRequest = field(repr=False, default=None)

    @property
    def time_to_solution(self) -> float:
        """Arrival to finish, queueing included."""
        return self.finished - self.arrival


def _phys():
    return GradedSpace.new(SU2, {SU2.sector(1): 1})


def _start_bonds(L: int):
    """The seeded start's bond spaces: every spin allowed by the distance to an end."""
    return [GradedSpace.new(SU2, {SU2.sector(j): 1 for j in range(i % 2, min(i, L - i) + 1, 2)})
            for i in range(L + 1)]


def footprint_bytes(req: SolveRequest, ncv: int = 20) -> int:
    """HBM estimate of one solve, an upper bound by dense counting: ``L + 1``
    environments of ``chi^2 D_w`` doubles (``D_w = 8`` dense for J1-J2), ``L`` site
    tensors of ``2 chi^2``, per cached bond program about ``24 chi^2`` doubles of
    intermediates and ``(ncv + 5) 4 chi^2`` doubles of Krylov vectors for the bond in
    flight, plus a fixed 32 MiB of plan tables and scratch."""
    c2 = req.chi * req.chi
    per_site = 8 * (8 * c2 + 2 * c2)
    bond = 8 * (24 * c2 + (ncv + 5) * 4 * c2)
    return int(req.L * per_site + 4 * bond + (32 << 20))


def request_stream(n: int, rate: float, *, seed: int = 0, lengths=(16, 32, 64, 128),
                   chis=(32, 64, 128, 256), j2_max: float = 0.4, sweeps: int = 8):
    """``n`` requests with Poisson arrivals at ``rate`` per second (``inf``: all at once),
    parameters drawn from ``np.random.default_rng(seed)``."""
    rng = np.random.default_rng(seed)
    gaps = np.zeros(n) if np.isinf(rate) else rng.exponential(1.0 / rate, size=n)
    t = np.cumsum(gaps)
    out = []
    for i in range(n):
        out.append(SolveRequest(rid=i, L=int(rng.choice(lengths)),
                                j2=float(rng.uniform(0.0, j2_max)), chi=int(rng.choice(chis)),
                                sweeps=sweeps, arrival=float(t[i]), seed=int(rng.integers(1 << 30))))
    return out


def _solve_steps(req: SolveRequest, *, precision: str, ncv: int, cutoff: float,
                 compiled: bool = True, tc_min_flops=None):
    h = network.heisenberg_mpo_su2(req.L, 1.0, req.j2)
    psi = network.MPS.random(_phys(), _start_bonds(req.L), seed=req.seed)
    return (yield from network.dmrg_steps(psi, h, chi=req.chi, cutoff=cutoff, ncv=ncv,
                                          max_sweeps=req.sweeps, energy_tol=0.0,
                                          schmidt_tol=0.0,
                                          compiled=compiled, precision=precision,
                                          tc_min_flops=tc_min_flops))


def solve_alone(req: SolveRequest, *, precision: str = "f64", ncv: int = 20,
                cutoff: float = 1e-10, compiled: bool = True, tc_min_flops=None):
    """The same solve outside the server: ``(energy, history)``."""
    out = network.drain(_solve_steps(req, precision=precision, ncv=ncv, cutoff=cutoff,
                                            compiled=compiled, tc_min_flops=tc_min_flops))
    return out.energy, [h[0] for h in out.history]


@dataclass
class _Slot:
    req: SolveRequest
    stream: torch.cuda.Stream
    gen: object
    admitted: float
    footprint: int


class Server:
    """The request loop.  ``max_active`` bounds the solves in flight, ``hbm_budget`` (bytes;
    default 80 % of the device's free memory at construction) bounds the sum of their
    footprint estimates.  Admission is in arrival order."""

    def __init__(self, *, max_active: int = 8, hbm_budget: int | None = None,
                 precision: str = "3xbf16", ncv: int = 20, cutoff: float = 1e-10,
                 tc_min_flops=None) -> None:
        if max_active < 1:
            raise ValueError("max_active must be at least 1")
        if hbm_budget is None:
            free, _ = torch.cuda.mem_get_info()
            hbm_budget = int(0.8 * free)
        self.max_active, self.hbm_budget = max_active, hbm_budget
        self.precision, self.ncv, self.cutoff = precision, ncv, cutoff
        self.tc_min_flops = tc_min_flops
        self._streams: list = []
        self.peak_active = 0
        self.rounds = 0

    def _stream(self) -> torch.cuda.Stream:
        return self._streams.pop() if self._streams else torch.cuda.Stream()

    def run(self, requests, clock=time.perf_counter) -> list[SolveResult]:
        """Serve ``requests`` (arrival times relative to the call) to completion; results in
        completion order."""
        pending = sorted(requests, key=lambda r: (r.arrival, r.rid))
        for r in pending:
            if footprint_bytes(r, self.ncv) > self.hbm_budget:
                raise ValueError(f"request {r.rid} needs more HBM than the whole budget")
        active: list[_Slot] = []
        results: list[SolveResult] = []
        used = 0
        torch.cuda.synchronize()
        t0 = clock()
        while pending or active:
            now = clock() - t0
            while pending and pending[0].arrival <= now and len(active) < self.max_active:
                fp = footprint_bytes(pending[0], self.ncv)
                if used + fp > self.hbm_budget:
                    break
                req = pending.pop(0)
                used += fp
                stream = self._stream()
                stream.wait_stream(torch.cuda.current_stream())
                gen = _solve_steps(req, precision=self.precision, ncv=self.ncv,
                                   cutoff=self.cutoff, tc_min_flops=self.tc_min_flops)
                active.append(_Slot(req, stream, gen, now, fp))
            self.peak_active = max(self.peak_active, len(active))
            if not active:
                time.sleep(max(0.0, min(pending[0].arrival - (clock() - t0), 0.01)))
                continue
            self.rounds += 1
            for slot in list(active):
                with torch.cuda.stream(slot.stream):
                    try:
                        next(slot.gen)
                        continue
                    except StopIteration as stop:
                        energy, history = stop.value.energy, [h[0] for h in stop.value.history]
                    slot.stream.synchronize()
                active.remove(slot)
                used -= slot.footprint
                self._streams.append(slot.stream)
                results.append(SolveResult(slot.req.rid, energy, history, slot.req.arrival,
                                           slot.admitted, clock() - t0, slot.footprint, slot.req))
        torch.cuda.synchronize()
        return results


# ---------------------------------------------------------------------------------------
# host-parallel serving: worker processes on one GPU

_WORKER: dict = {}


def _worker_init(precision: str, ncv: int, cutoff: float, tc_min_flops) -> None:
    torch.cuda.set_device(0)
    _WORKER.update(precision=precision, ncv=ncv, cutoff=cutoff, tc_min_flops=tc_min_flops)
    # load the library and the CUDA context now, not inside the first timed request
    solve_alone(SolveRequest(-1, 8, 0.1, 16, sweeps=1), precision=precision, ncv=ncv,
                cutoff=cutoff, tc_min_flops=tc_min_flops)
    torch.cuda.synchronize()


def _worker_ready(_: int) -> int:
    import os

    time.sleep(0.2)  # long enough that every worker of the pool takes one
    return os.getpid()


def _worker_solve(req: SolveRequest):
    w = _WORKER
    e, hist = solve_alone(req, precision=w["precision"], ncv=w["ncv"], cutoff=w["cutoff"],
                          tc_min_flops=w["tc_min_flops"])
    torch.cuda.synchronize()
    return e, hist


class ProcessServer:
    """Continuous batching over host-parallel workers: ``workers`` processes (spawned,
    each with its own CUDA context on the same GPU) solve the admitted requests, so the
    per-bond host work of one solve -- planning, the SVD decision, launches -- runs beside
    the others' instead of after it.  Admission is the same as ``Server``'s: arrival
    order, a free worker, and the summed footprint estimates within ``hbm_budget``.  The
    workers start and warm up (library, CUDA context) when the server is built; a
    long-running server keeps them.  Kernels of different workers share the GPU by time
    slicing."""

    def __init__(self, *, workers: int = 4, hbm_budget: int | None = None,
                 precision: str = "3xbf16", ncv: int = 20, cutoff: float = 1e-10,
                 tc_min_flops=None) -> None:
        import multiprocessing
        from concurrent.futures import ProcessPoolExecutor

        if workers < 1:
            raise ValueError("workers must be at least 1")
        if hbm_budget is None:
            free, _ = torch.cuda.mem_get_info()
            hbm_budget = int(0.6 * free)
        self.workers, self.hbm_budget, self.ncv = workers, hbm_budget, ncv
        self.pool = ProcessPoolExecutor(
            max_workers=workers, mp_context=multiprocessing.get_context("spawn"),
            initializer=_worker_init, initargs=(precision, ncv, cutoff, tc_min_flops))
        self.pids = set(self.pool.map(_worker_ready, range(2 * workers)))
        self.peak_active = 0

    def close(self) -> None:
        self.pool.shutdown()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def run(self, requests, clock=time.perf_counter) -> list[SolveResult]:
        from concurrent.futures import FIRST_COMPLETED, wait

        pending = sorted(requests, key=lambda r: (r.arrival, r.rid))
        for r in pending:
            if footprint_bytes(r, self.ncv) > self.hbm_budget:
                raise ValueError(f"request {r.rid} needs more HBM than the whole budget")
        results: list[SolveResult] = []
        active: dict = {}
        used = 0
        t0 = clock()
        while pending or active:
            now = clock() - t0
            while pending and pending[0].arrival <= now and len(active) < self.workers:
                fp = footprint_bytes(pending[0], self.ncv)
                if used + fp > self.hbm_budget:
                    break
                req = pending.pop(0)
                used += fp
                active[self.pool.submit(_worker_solve, req)] = (req, now, fp)
            self.peak_active = max(self.peak_active, len(active))
            if not active:
                time.sleep(max(0.0, min(pending[0].arrival - (clock() - t0), 0.01)))
                continue
            timeout = max(0.0, pending[0].arrival - now) if pending else None
            done, _ = wait(list(active), timeout=timeout, return_when=FIRST_COMPLETED)
            for f in done:
                req, admitted, fp = active.pop(f)
                energy, history = f.result()
                used -= fp
                results.append(SolveResult(req.rid, energy, history, req.arrival, admitted,
                                           clock() - t0, fp, req))
        return results


def clear_plan_caches() -> None:
    """Empty every host plan cache (structures, block maps, descriptor tables, SU(2)
    coefficients), so that a measurement starts cold."""
    import sys

    for name, mod in list(sys.modules.items()):
        if not name.startswith("tenet.") or mod is None:
            continue
        for attr in list(vars(mod).values()):
            if callable(getattr(attr, "cache_clear", None)):
                attr.cache_clear()
    from tenet import program

    program._HEFF_TABLES.clear()


def summarize(results, wall: float) -> dict:
    """solves/s and the p50/p99 time to solution of a served run."""
    tts = np.array([r.time_to_solution for r in results])
    return {"solves": len(results), "wall_s": wall,
            "solves_per_s": len(results) / wall if wall > 0 else float("nan"),
            "p50_s": float(np.percentile(tts, 50)) if len(tts) else None,
            "p99_s": float(np.percentile(tts, 99)) if len(tts) else None}
