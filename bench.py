"""Benchmark: the two-site effective-Hamiltonian matvec of the SU(2) Heisenberg chain.

Workload (the configuration the headline metric is quoted on): the Heff matvec that
Lanczos applies at a mid-chain bond of the spin-1/2 SU(2) Heisenberg chain (L = 64) with
a maximum multiplet bond dimension of 256 -- 256 multiplets per bond over half-integer
bond spins 2j = 1..17 -- and the S.S MPO bond of three multiplets (2j = 0, 0, 2).  The
inputs are seeded synthetic tensors of exactly those structures (random FP64 blocks;
the cost of a matvec depends on the structure only).  A step is one ``heff2``
application: four pairwise contractions, each a pack gather, a grouped FP64 GEMM and an
unpack gather, plus the three named-wire bends.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl tenet|reference]

``value`` is matvec TFLOP/s (algorithmic GEMM flops of the lowering, sum of 2 M K N over
every coupled-sector product, divided by device time), inputs resident in HBM, L2
flushed between timed steps.  ``e2e`` is the same metric through the public API with the
two-site tensor copied from pinned host memory and the result copied back inside the
timed region.  ``--impl reference`` times the oracle port of the reference's NumPy path
on the host cores instead.  With ``--gpus N`` under torchrun every rank runs an
independent replica (the path does not shard), and the job value is the sum of all
ranks' matvecs over the slowest rank's time.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
for _p in (ROOT, ROOT / "tenet-py_b200"):
    if str(_p) not in sys.path:
        sys.path.insert(0, str(_p))

METRIC = "Heff matvec TFLOP/s (SU(2) Heisenberg two-site, FP64)"
# dram__bytes_read.sum + dram__bytes_write.sum per launch of each kernel class on the
# headline matvec, mean over the launches of one matvec in one ncu --set full capture of
# this build (bench.py --profile-heff2 10; cold cache, so the tables and operands count)
NCU_TRAFFIC: dict = {"block_gather": (65_024 + 98_560 + 65_024) // 3,
                     "grouped_gemm_f64": (87_808 + 113_152) // 2}
# multiplets per spin of the mid-chain bond (sites 31 | 32) of the reference's own
# converged state of this chain: L = 64, chi = 256 (dense), cutoff 1e-10, ncv = 20, from
# the seeded start, 6 sweeps (tests/golden/dmrg64.json, bond 32; 85 states dense)
BOND = {0: 8, 2: 14, 4: 7}
MPO = {0: 2, 2: 1}
PHYS = {1: 1}
WORKLOAD = "su2-heisenberg-L64-chi256-cutoff1e-10-mid-bond-heff2"
# further matvec workloads, reported beside the headline: the mid bond of the same chain
# grown under a cap of 256 multiplets at cutoff 1e-14 (bench.py --derive-bond: the cap never
# binds; 67 multiplets, 207 states dense), and a synthetic stress bond of 256 multiplets
# over half-integer spins 2j = 1..17 (no state of this chain needs it)
WORKLOADS = {
    "L64_cutoff1e-14_mid_bond": {0: 17, 2: 32, 4: 16, 6: 2},
    "synthetic_256_multiplets": {1: 60, 3: 56, 5: 46, 7: 36, 9: 25, 11: 16, 13: 10, 15: 5,
                                 17: 2},
}
# the reference's energy for this chain and its sweep count (same run as BOND)
REF_DMRG = {"energy": -28.175424844464963, "sweeps": 6}


def build_workload(seed: int = 0, bond: dict | None = None):
    """(fl, w1, w2, fr, aa) as tenet tensors with the golden-vector leg conventions of the
    reference's ``Env`` (``network/env.py``): F[(n-1,n)] = (ket IN, mpo OUT*, bra OUT),
    F[(n+2,n+1)] = (ket OUT, mpo IN*, bra IN), W = (x IN*, P OUT, p IN, m OUT*)."""
    import tenet
    from tenet.structure import IN, OUT, GradedSpace, Leg
    from tenet.symmetry import SU2

    def sp(d):
        return GradedSpace.new(SU2, {SU2.sector(a): m for a, m in d.items()})

    B, M, P = sp(bond or BOND), sp(MPO), sp(PHYS)
    rnd = tenet.SymmetricTensor.random
    fl = rnd((Leg(B, IN), Leg(M, OUT, True), Leg(B, OUT)), seed=seed)
    fr = rnd((Leg(B, OUT), Leg(M, IN, True), Leg(B, IN)), seed=seed + 1)
    w = (Leg(M, IN, True), Leg(P, OUT), Leg(P, IN), Leg(M, OUT, True))
    w1, w2 = rnd(w, seed=seed + 2), rnd(w, seed=seed + 3)
    aa = rnd((Leg(B, OUT), Leg(P, OUT), Leg(P, OUT), Leg(B, IN)), seed=seed + 4)
    return fl, w1, w2, fr, aa


def workload_structures(bond: dict | None = None):
    """The five structures of ``build_workload`` (host only, no device needed)."""
    from tenet.structure import IN, OUT, GradedSpace, Leg, TensorStructure
    from tenet.symmetry import SU2

    def sp(d):
        return GradedSpace.new(SU2, {SU2.sector(a): m for a, m in d.items()})

    B, M, P = sp(bond or BOND), sp(MPO), sp(PHYS)
    w = TensorStructure((Leg(M, IN, True), Leg(P, OUT), Leg(P, IN), Leg(M, OUT, True)))
    return (TensorStructure((Leg(B, IN), Leg(M, OUT, True), Leg(B, OUT))), w, w,
            TensorStructure((Leg(B, OUT), Leg(M, IN, True), Leg(B, IN))),
            TensorStructure((Leg(B, OUT), Leg(P, OUT), Leg(P, OUT), Leg(B, IN))))


def oracle_workload(seed: int = 0):
    """The same tensors for the oracle, built from the oracle's own types (nothing of the
    tenet package is imported): same structures, same seeded draws."""
    import oracle.tenet_oracle as O

    def leg(d, side, dual=False):
        return O.Leg(tuple(sorted(d.items())), side, dual)

    w = (leg(MPO, O.IN, True), leg(PHYS, O.OUT), leg(PHYS, O.IN), leg(MPO, O.OUT, True))
    legs = {"fl": (leg(BOND, O.IN), leg(MPO, O.OUT, True), leg(BOND, O.OUT)),
            "w1": w, "w2": w,
            "fr": (leg(BOND, O.OUT), leg(MPO, O.IN, True), leg(BOND, O.IN)),
            "aa": (leg(BOND, O.OUT), leg(PHYS, O.OUT), leg(PHYS, O.OUT), leg(BOND, O.IN))}
    seeds = {"fl": 0, "fr": 1, "w1": 2, "w2": 3, "aa": 4}
    return [O.random(O.Structure(O.SU2, legs[k]), seed + seeds[k])
            for k in ("fl", "w1", "w2", "fr", "aa")]


def bench_config(world: int = 1) -> dict:
    """The workload description both arms print (identical by construction)."""
    return {"workload": WORKLOAD, "bond_multiplets": {str(k): v for k, v in BOND.items()},
            "mpo_multiplets": {str(k): v for k, v in MPO.items()},
            "l2": "flushed between timed steps (256 MiB write)",
            "parallelism": f"replicas{world}"}


def host_cores() -> int:
    try:
        from threadpoolctl import threadpool_info

        return int(max((i.get("num_threads", 1) for i in threadpool_info()), default=1))
    except Exception:
        return os.cpu_count() or 1


def heff2_flops(bond: dict | None = None) -> int:
    """Algorithmic flops of one heff2 from the plans alone (host, no device): the sum of
    2 M K N over every coupled-sector product of the four contractions."""
    from tenet import ops
    from tenet.plan import repartition_plan, transpose_plan
    from tenet.structure import OUT

    def einsum_s(eq, sa, sb):
        lhs, out = eq.split("->")
        ta, tb = lhs.split(",")
        shared = [x for x in ta if x in tb]
        axes = (tuple(ta.index(x) for x in shared), tuple(tb.index(x) for x in shared))
        ex = ops.contraction_exec(sa, sb, axes)
        free = [x for x in ta if x not in shared] + [x for x in tb if x not in shared]
        return transpose_plan(ex.out, tuple(free.index(x) for x in out))[0], ex.flops

    def composed_s(eq, sa, sb, bend):
        lhs, out = eq.split("->")
        ta, tb = lhs.split(",")

        def bent(s, term):
            outs = tuple(i for i, ch in enumerate(term) if (s.legs[i].side is OUT) != (ch in bend))
            ins = tuple(i for i in range(len(term)) if i not in outs)
            return repartition_plan(s, outs, ins)[0], "".join(term[i] for i in (*outs, *ins))

        sa, ta = bent(sa, ta)
        sb, tb = bent(sb, tb)
        return einsum_s(f"{ta},{tb}->{out}", sa, sb)

    fl, w1, w2, fr, aa = workload_structures(bond)
    t, f0 = einsum_s("apqr,rys->apqys", aa, fr)
    t, f1 = composed_s("apqys,mQqy->apQms", t, w2, "q")
    t, f2 = composed_s("apQms,xPpm->aPQxs", t, w1, "p")
    _, f3 = composed_s("aPQxs,axB->BPQs", t, fl, "a")
    return f0 + f1 + f2 + f3


def launches_per_matvec(tensors) -> int:
    from tenet import _exec, network

    log = _exec.LaunchLog(timed=False)
    with log:
        network.heff2(*tensors)
    return log.count


class Clocks:
    """Samples nvidia-smi during the timed region (SM clock, throttle reasons)."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int) -> None:
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [x for x in out.splitlines() if x.strip()]

    def summary(self) -> dict:
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in getattr(self, "lines", []):
            f = [x.strip() for x in line.split(",")]
            try:
                sm.append(float(f[0]))
                mx = float(f[1])
            except (ValueError, IndexError):
                continue
            for name, val in zip(names, f[3:7]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "samples": len(sm), "reasons": sorted(reasons),
                "window": "timed steps plus 1 s of the same graph replay loop"}


def peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": d.get("hbm_gbs"), "src": "measured"}
    return {"hbm_gbs": 6650.0, "src": "fallback"}


def gemm_probe(n: int, dgemm: float | None, reps: int = 5) -> dict:
    """The grouped GEMM's tile kinds on one n x n x n product (each operand n^2 doubles,
    128 MiB at n = 4096, so nothing stays in L2 between repetitions): FP64 64 x 64 tiles
    against cuBLAS DGEMM, the tensor-core kinds against the measured dense BF16 peak
    (3xBF16 issues three BF16 products per product, TF32 runs at half the BF16 rate).
    The tensor-core times include packing the operands (the first of two launches)."""
    import torch

    from tenet import _exec

    p = ROOT / "MEASURED_PEAKS.json"
    bf16 = json.loads(p.read_text()).get("bf16_tflops") if p.exists() else None
    src = "MEASURED_PEAKS.json bf16_tflops (measured)" if bf16 else "fallback 1590"
    bf16 = bf16 or 1590.0
    g = torch.Generator(device="cuda").manual_seed(5)
    a = torch.randn(n * n, dtype=torch.float64, device="cuda", generator=g)
    b = torch.randn(n * n, dtype=torch.float64, device="cuda", generator=g)
    prod = [(n, n, n, 0, n, 0, n, 0, n)]
    out = {"workload": f"one {n}^3 FP64-in/FP64-out product", "flops": 2 * n ** 3,
           "peak_bf16_tflops": bf16, "peak_source": src, "dgemm_tflops": dgemm}
    ref = None
    for name, kind in (("f64_64x64", _exec.TILE_64), ("tf32", _exec.TILE_TC_TF32),
                       ("3xbf16", _exec.TILE_TC_3XBF16)):
        t = _exec.make_gemm(prod, kind, split_k=False)
        c = torch.empty(n * n, dtype=torch.float64, device="cuda")
        t.run(a, b, c)
        torch.cuda.synchronize()
        times = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            t.run(a, b, c)
            e1.record()
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        ms = float(np.median(times))
        tf = 2 * n ** 3 / (ms * 1e-3) / 1e12
        d = {"ms": ms, "tflops": tf, "launches": t.launches}
        if ref is None:
            ref = c.clone()
            d["frac_of_cublas_dgemm"] = tf / dgemm if dgemm else None
        else:
            d["rel_error_vs_f64"] = float((c - ref).norm() / ref.norm())
            mult = 3 if name == "3xbf16" else 2
            d["bf16_equivalent_tflops"] = tf * mult
            d["frac_of_bf16_peak"] = tf * mult / bf16
        out[name] = d
    return out


def measure_dgemm_peak(torch) -> float:
    """cuBLAS DGEMM throughput on this GPU (TFLOP/s), the FP64 roofline denominator."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e9
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    return 2 * n ** 3 / (best * 1e-3) / 1e12


def cpu_baseline(flops: int, budget_s: float = 20.0) -> dict:
    """The oracle's NumPy path (the reference's algorithm) on this host's cores."""
    import oracle.tenet_oracle as O

    fl, w1, w2, fr, aa = oracle_workload()
    O.FLOPS[0] = 0
    O.heff2(fl, w1, w2, fr, aa)  # warm the plan caches, as the reference's own bench does
    assert O.FLOPS[0] == flops, "the oracle's work differs from the planner's"
    times = []
    t_end = time.perf_counter() + budget_s
    while time.perf_counter() < t_end and len(times) < 5:
        t0 = time.perf_counter()
        O.heff2(fl, w1, w2, fr, aa)
        times.append(time.perf_counter() - t0)
    med = float(np.median(times))
    return {"value": flops / med / 1e12, "unit": "TFLOP/s", "cores": host_cores(), "kind": "port",
            "sample": f"{len(times)} oracle heff2 matvecs on the same structures (median "
                      f"{med * 1e3:.1f} ms each), plan caches warm",
            "ms_per_matvec": med * 1e3}


def config3_spaces(seed: int = 1000, lam: float = 24.0, max_deg: int = 256):
    """The U(1) x U(1) x fZ2 spaces of the batched environment update: a bond leg with
    sectors (N, 2Sz) in [-4, 4]^2 on the allowed grid (2Sz = N mod 2, parity N mod 2; 41
    sectors) and degeneracies Poisson(lam) clipped to 1..max_deg from
    ``np.random.default_rng(seed)``; an MPO leg of width 6 with the Hubbard chain's
    sectors (two identity channels and the four single-fermion channels c+up, c+dn,
    c up, c dn); the Hubbard site's four states."""
    from tenet.structure import GradedSpace
    from tenet.symmetry import ProductSector as PS
    from tenet.symmetry import U1xU1xfZ2 as P

    rng = np.random.default_rng(seed)
    bond = {}
    for n in range(-4, 5):
        for sz in range(-4, 5):
            if (sz - n) % 2 == 0:
                bond[PS(n, sz, n % 2)] = int(np.clip(rng.poisson(lam), 1, max_deg))
    mpo = {PS(0, 0, 0): 2, PS(1, 1, 1): 1, PS(1, -1, 1): 1, PS(-1, -1, 1): 1, PS(-1, 1, 1): 1}
    phys = {PS(0, 0, 0): 1, PS(1, 1, 1): 1, PS(1, -1, 1): 1, PS(2, 0, 0): 1}
    return (GradedSpace.new(P, bond), GradedSpace.new(P, mpo), GradedSpace.new(P, phys))


def config3_batch(n: int, seed: int = 1000, lam: float = 24.0, max_deg: int = 256):
    """``(F, A, W)`` for ``n`` independent environment updates ``L' = A^dagger L W A``:
    ``F = (ket IN, mpo OUT*, bra OUT)`` and ``A = (l OUT, p OUT, r IN)`` per member, ``W =
    (x IN*, P OUT, p IN, m OUT*)`` shared, N(0, 1) values rounded to FP32 (member k's F
    and A draw with seeds 2k and 2k + 1 after ``seed``)."""
    import torch

    from tenet import batch
    from tenet.structure import IN, OUT, Leg, TensorStructure, layout
    from tenet.tensor import SymmetricTensor

    V, M, Pp = config3_spaces(seed, lam, max_deg)
    sf = TensorStructure((Leg(V, IN), Leg(M, OUT, True), Leg(V, OUT)))
    sa = TensorStructure((Leg(V, OUT), Leg(Pp, OUT), Leg(V, IN)))
    sw = TensorStructure((Leg(M, IN, True), Leg(Pp, OUT), Leg(Pp, IN), Leg(M, OUT, True)))

    def values(s, sd, rows):
        rng = np.random.default_rng(sd)
        host = rng.standard_normal((rows, layout(s).size), dtype=np.float32).astype(np.float64)
        return torch.from_numpy(host).cuda()

    F = batch.TensorBatch(sf, values(sf, seed + 1, n), n)
    A = batch.TensorBatch(sa, values(sa, seed + 2, n), n)
    W = batch.TensorBatch.broadcast(SymmetricTensor(sw, arena=values(sw, seed + 3, 1)[0]), n)
    return F, A, W


def batched_matvecs(args, plain_ms: float, graph_ms: float) -> dict:
    """``n`` independent two-site matvecs of the bench workload's structures (own
    environments and Krylov vectors, shared MPO sites) as one batch, every stage one
    launch for all members: FP64 (autotuned tile kinds), and the precision forms with the
    default tensor-core size rule and with every product on the tensor cores.  Reported
    per matvec against the plain FP64 form (one eager op-by-op matvec) and the compiled
    single matvec of the same run; errors are relative Frobenius norms against the FP64
    batch, worst member."""
    import torch

    from tenet import _exec, batch, ops

    n = args.batch_n
    members = [build_workload(seed=10 * k) for k in range(n)]
    fl, fr, aa = (batch.TensorBatch.stack([m[i] for m in members]) for i in (0, 3, 4))
    w1 = batch.TensorBatch.broadcast(members[0][1], n)
    w2 = batch.TensorBatch.broadcast(members[0][2], n)
    flops = heff2_flops() * n
    flush = torch.empty(256 * 1024 * 1024 // 8, dtype=torch.float64, device="cuda")

    def timed(fn, steps):
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(steps)]
        for k in range(steps):
            flush.fill_(float(k))
            ev[k][0].record()
            fn()
            ev[k][1].record()
        torch.cuda.synchronize()
        return sum(a.elapsed_time(b) for a, b in ev) / steps

    out = {"workload": f"{n} SU(2) heff2 matvecs on the headline bond (seeds 0, 10, ...), "
                       "shared MPO sites; compiled batched chain (BatchedHeff2) unless named "
                       "eager", "flops_per_batch": flops,
           "l2": "flushed between timed steps (256 MiB write)"}
    exact = batch.heff2(fl, w1, w2, fr, aa).arena.cpu().numpy()
    for name, prec in (("f64", ("f64", None)), ("3xbf16", ("3xbf16", None)),
                       ("3xbf16_all_products", ("3xbf16", 0)), ("tf32_all_products", ("tf32", 0)),
                       ("f64_eager_batch", None)):
        if prec is None:  # the same batch through the eager batched ops (no compiled chain)
            fn = lambda: batch.heff2(fl, w1, w2, fr, aa)  # noqa: E731
        else:
            prog = batch.BatchedHeff2(fl, w1, w2, fr, aa.structure, precision=prec[0],
                                      tc_min_flops=prec[1])
            y = torch.empty((n, prog.out_size), dtype=torch.float64, device="cuda")
            fn = lambda: prog.run(aa.arena, y)  # noqa: E731
        for _ in range(args.warmup):
            fn()
        ms = timed(fn, args.steps)
        if prec is None:
            got = fn().arena.cpu().numpy()
        else:
            fn()
            got = y.cpu().numpy()
        err = max(float(np.linalg.norm(got[k] - exact[k]) / np.linalg.norm(exact[k]))
                  for k in range(n))
        per = ms / n
        out[name] = {"ms_per_batch": ms, "us_per_matvec": per * 1e3,
                     "tflops": flops / (ms * 1e-3) / 1e12, "max_rel_error_vs_f64": err,
                     "matvec_throughput_vs_plain_f64": plain_ms / per,
                     "matvec_throughput_vs_compiled_single": graph_ms / per}
    return out


def batched_env_updates(args) -> dict:
    """``n`` independent U(1) x U(1) x fZ2 environment updates ``L' = A^dagger L W A`` as one
    batch (every stage one launch for all members), in FP64 and with every sector product
    on the tensor cores (3xBF16, TF32), against the same updates run one by one in FP64.
    Errors are relative Frobenius norms against the FP64 batch, worst member."""
    import torch

    from tenet import _exec, batch, network, ops

    n = args.config3_n
    F, A, W = config3_batch(n)
    flush = torch.empty(256 * 1024 * 1024 // 8, dtype=torch.float64, device="cuda")

    def timed(fn, steps):
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(steps)]
        for k in range(steps):
            flush.fill_(float(k))
            ev[k][0].record()
            fn()
            ev[k][1].record()
        torch.cuda.synchronize()
        return sum(a.elapsed_time(b) for a, b in ev) / steps

    out = {"workload": f"{n} U1xU1xfZ2 env updates, bond 41 sectors Poisson(24) clipped 1..256 "
                       "(seed 1000), MPO width 6 (Hubbard sectors), values N(0,1) rounded to FP32",
           "l2": "flushed between timed steps (256 MiB write)"}
    exact = batch.env_update_last(F, A, W)
    log = _exec.LaunchLog(timed=True)
    with log:
        batch.env_update_last(F, A, W)
    kinds = log.summary()
    flops = sum(v["work"] for k, v in kinds.items() if k.startswith("grouped_gemm"))
    out["flops_per_batch"] = int(flops)
    out["launches_per_batch"] = int(sum(v["launches"] for v in kinds.values()))
    ex = exact.arena.cpu().numpy()
    for name, prec in (("f64", ("f64", None)), ("3xbf16", ("3xbf16", 0)), ("tf32", ("tf32", 0))):
        with ops.precision(*prec):
            fn = lambda: batch.env_update_last(F, A, W)  # noqa: E731
            for _ in range(args.warmup):
                fn()
            ms = timed(fn, args.steps)
            got = fn().arena.cpu().numpy()
        err = max(float(np.linalg.norm(got[k] - ex[k]) / np.linalg.norm(ex[k])) for k in range(n))
        out[name] = {"ms_per_batch": ms, "tflops": flops / (ms * 1e-3) / 1e12,
                     "max_rel_error_vs_f64": err}
    # the same FP64 batch with the size heuristic instead of the autotuned tile kinds
    batch.AUTOTUNE = False
    try:
        fn = lambda: batch.env_update_last(F, A, W)  # noqa: E731
        for _ in range(args.warmup):
            fn()
        out["f64_heuristic_tiles"] = {"ms_per_batch": timed(fn, args.steps)}
    finally:
        batch.AUTOTUNE = True
    out["autotuned_kinds"] = {str(k): list(v) for k, v in _exec.AUTOTUNE_CACHE.items()}
    members = [(F[k], A[k], W[k]) for k in range(n)]
    one = lambda: [network.env_update_last(*m) for m in members]  # noqa: E731
    for _ in range(args.warmup):
        one()
    ms1 = timed(one, max(1, args.steps // 4))
    out["f64_one_by_one"] = {"ms_per_batch": ms1, "tflops": flops / (ms1 * 1e-3) / 1e12}
    out["batched_f64_speedup_over_one_by_one"] = ms1 / out["f64"]["ms_per_batch"]
    return out


def serving(args) -> dict:
    """Served DMRG solves against the plain FP64 form on the same seeded request sample
    (SU(2) J1-J2 chains, 8 sweeps, ncv = 20, cutoff 1e-10).  Arms, each from empty plan
    caches: the plain FP64 form (eager op-by-op matvec, host-driven Lanczos), the
    compiled FP64 form one solve at a time, the single-process serving loop in FP64 and
    in the precision form, the same with host-parallel worker processes (started and
    warmed before the timed run), every request arriving at once, and the worker form
    again at a Poisson arrival rate of 0.7 x its burst throughput for the latency point;
    then the single-process loop and the compiled sequential solves again with the plan
    caches warm, as in a long-running server."""
    import torch

    from tenet import serve

    kw = {} if args.serve_full else {"lengths": (16, 32), "chis": (32, 64)}
    reqs = serve.request_stream(args.serve_requests, float("inf"), seed=0, **kw)
    out = {"sample": (f"{len(reqs)} requests of the seeded config-5 stream (seed 0), "
                      + ("full distribution" if args.serve_full else
                         "L in {16, 32}, chi in {32, 64}") + ", J2/J1 in [0, 0.4], 8 sweeps"),
           "requests": [{"rid": r.rid, "L": r.L, "chi": r.chi, "j2": round(r.j2, 4)}
                        for r in reqs],
           "timing": "wall clock from the first arrival to the last result; every arm starts "
                     "with empty host plan caches except the two *_warm_caches arms, which "
                     "run after the arms before them have planned every structure"}
    energies = {}

    def sequential(name, warm=False, **kw):
        if not warm:
            serve.clear_plan_caches()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        done, en = [], {}
        for r in reqs:
            e, _ = serve.solve_alone(r, **kw)
            torch.cuda.synchronize()
            done.append(time.perf_counter() - t0)
            en[r.rid] = e
        wall = time.perf_counter() - t0
        energies[name] = en
        out[name] = {"solves_per_s": len(reqs) / wall, "wall_s": wall,
                     "p50_s": float(np.percentile(done, 50)), "p99_s": float(np.percentile(done, 99))}

    def served(name, requests, workers=0, warm=False, **kw):
        if not warm:
            serve.clear_plan_caches()
        if workers:  # worker processes, started and warmed before the timed run
            srv = serve.ProcessServer(workers=workers, **kw)
        else:
            srv = serve.Server(max_active=args.serve_slots, **kw)
        t0 = time.perf_counter()
        res = srv.run(requests)
        wall = time.perf_counter() - t0
        if workers:
            srv.close()
        energies[name] = {r.rid: r.energy for r in res}
        out[name] = serve.summarize(res, wall) | {"peak_active": srv.peak_active}

    sequential("plain_f64_sequential", precision="f64", compiled=False)
    sequential("compiled_f64_sequential", precision="f64")
    served("served_f64", reqs, precision="f64")
    # a long-running server keeps its host plan caches: the same two arms again, warm
    served("served_f64_warm_caches", reqs, warm=True, precision="f64")
    sequential("compiled_f64_sequential_warm_caches", warm=True, precision="f64")
    served("served_3xbf16", reqs, precision="3xbf16")
    w = args.serve_workers
    served(f"served_f64_{w}workers", reqs, workers=w, precision="f64")
    served(f"served_3xbf16_{w}workers", reqs, workers=w, precision="3xbf16")
    rate = 0.7 * out[f"served_3xbf16_{w}workers"]["solves_per_s"]
    poisson = serve.request_stream(len(reqs), rate, seed=0, **kw)
    served(f"served_3xbf16_{w}workers_poisson", poisson, workers=w, precision="3xbf16")
    out[f"served_3xbf16_{w}workers_poisson"]["arrival_rate_per_s"] = rate
    ref = energies["plain_f64_sequential"]
    out["max_abs_dE_per_site_vs_plain_f64"] = {
        k: max(abs(v[r.rid] - ref[r.rid]) / r.L for r in reqs) for k, v in energies.items()
        if k != "plain_f64_sequential" and not k.endswith("poisson")}
    base = out["plain_f64_sequential"]["solves_per_s"]
    out["solves_per_s_vs_plain_f64"] = {
        k: out[k]["solves_per_s"] / base for k in
        ("compiled_f64_sequential", "served_f64", "served_3xbf16", f"served_f64_{w}workers",
         f"served_3xbf16_{w}workers", "served_f64_warm_caches",
         "compiled_f64_sequential_warm_caches")}
    return out


def serve_stream(args) -> None:
    """The config-5 stream at full distribution (L in {16, 32, 64, 128}, chi in {32, 64,
    128, 256}, J2/J1 in [0, 0.4], 8 sweeps, ncv = 20, cutoff 1e-10), ``--serve-requests``
    requests served by ``--serve-workers`` worker processes in the 3xBF16 precision form:
    first all at once (the burst throughput), then as Poisson streams at 0.5x and 0.85x
    that rate (the first ``--serve-rate-requests`` of the same seeded stream); p50 / p99
    time-to-solution per arm.  The workers keep their plan caches across the arms, as a
    long-running server does.  The plain FP64 form (eager matvecs,
    host-driven Lanczos) solves a seeded sample of the same requests one by one for the
    baseline solves/s and the per-request |dE/L| of the served energies.  Prints one JSON
    line and exits."""
    import torch

    from tenet import serve

    n, w = args.serve_requests, args.serve_workers
    reqs = serve.request_stream(n, float("inf"), seed=0)
    out = {"requests": n, "workers": w, "precision": "3xbf16",
           "distribution": {str(L): sum(r.L == L for r in reqs) for L in (16, 32, 64, 128)}}
    energies = {}
    serve.clear_plan_caches()
    srv = serve.ProcessServer(workers=w, precision="3xbf16")
    try:
        t0 = time.perf_counter()
        res = srv.run(reqs)
        out["burst"] = serve.summarize(res, time.perf_counter() - t0)
        energies.update({r.rid: r.energy for r in res})
        burst = out["burst"]["solves_per_s"]
        # each arm's line as soon as it is done (a long stream may outlast its time limit)
        print(json.dumps({"serve_stream_arm": "burst", **out["burst"]}), flush=True)
        nr = min(n, args.serve_rate_requests or n)
        for frac in (0.5, 0.85):
            stream = serve.request_stream(nr, frac * burst, seed=0)
            t0 = time.perf_counter()
            res = srv.run(stream)
            out[f"poisson_{frac}x"] = serve.summarize(res, time.perf_counter() - t0) | {
                "arrival_rate_per_s": frac * burst, "requests": nr}
            print(json.dumps({"serve_stream_arm": f"poisson_{frac}x",
                              **out[f"poisson_{frac}x"]}), flush=True)
    finally:
        srv.close()
    k = min(args.serve_plain_sample, n)
    sample = [reqs[i] for i in np.random.default_rng(1).choice(n, size=k, replace=False)]
    serve.clear_plan_caches()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    plain = {}
    for r in sample:
        plain[r.rid], _ = serve.solve_alone(r, precision="f64", compiled=False)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    out["plain_f64_sample"] = {"requests": k, "wall_s": wall, "solves_per_s": k / wall,
                               "max_abs_dE_per_site_served_vs_plain": max(
                                   abs(energies[r.rid] - plain[r.rid]) / r.L for r in sample)}
    out["burst_solves_per_s_vs_plain_f64"] = burst / (k / wall)
    print(json.dumps({"serve_stream": out}))


def chain64_start(L: int = 64, max_2j: int = 16, seed: int = 0):
    """The seeded start of the L = 64 SU(2) Heisenberg runs: bond spins 2j <= min(i, L - i,
    16), one multiplet each, ``MPS.random`` with ``seed``."""
    from tenet import network
    from tenet.structure import GradedSpace
    from tenet.symmetry import SU2

    phys = GradedSpace.new(SU2, {SU2.sector(1): 1})
    bonds = [GradedSpace.new(SU2, {SU2.sector(j): 1
                                   for j in range(i % 2, min(i, L - i, max_2j) + 1, 2)})
             for i in range(L + 1)]
    return network.MPS.random(phys, bonds, seed=seed)


def derive_bond(args) -> None:
    """Grow the L = 64 chain to a cap of ``--derive-chi`` multiplets per bond (cutoff 1e-14,
    so the cap binds; ncv = 20) and print the converged mid-chain bond's multiplets per
    spin and the run's per-sweep energies and times: the bond histogram of the large-bond
    matvec workload."""
    import torch

    from tenet import network

    L = 64
    psi = chain64_start(L)
    t0 = time.perf_counter()
    rec = []
    out = network.dmrg_(psi, network.heisenberg_mpo_su2(L), chi=args.derive_chi,
                        cutoff=1e-14, ncv=20, max_sweeps=args.derive_sweeps, budget="reduced",
                        callback=lambda o: rec.append((o.energy, time.perf_counter() - t0)))
    torch.cuda.synchronize()
    bonds = {n: {int(a.two_j): m for a, m in psi[n].legs[0].space.sectors}
             for n in (L // 2 - 1, L // 2, L // 2 + 1)}
    print(json.dumps({"derive_bond": {"L": L, "chi_multiplets": args.derive_chi,
                                      "sweeps": out.sweeps, "energy": out.energy,
                                      "per_sweep": rec, "bonds": bonds}}))


def max_over_ranks(ms: float, device) -> float:
    """The slowest rank's time: every rank of an initialised process group calls this at
    the same point (one all-reduce); a single process gets its own time back."""
    import torch
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return ms
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_value(flops: int, steps: int, world: int, ms: float) -> float:
    """Whole-job TFLOP/s: every rank's ``steps`` matvecs of ``flops`` each over the slowest
    rank's time ``ms``."""
    return flops * steps * world / (ms * 1e-3) / 1e12


def run_reference(args) -> None:
    """The reference's algorithm for the path on the host cores: the oracle's NumPy
    restatement of ``Env.heff2`` (the reference is Python and cannot travel to the GPU
    host; the oracle is pinned to its outputs), all BLAS threads, on the same workload.
    Only the oracle is imported, never the tenet package.  Rank 0 alone runs it."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import oracle.tenet_oracle as O

    ot = oracle_workload()
    O.FLOPS[0] = 0
    O.heff2(*ot)
    flops = O.FLOPS[0]
    for _ in range(max(0, args.warmup - 1)):
        O.heff2(*ot)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        O.heff2(*ot)
        times.append(time.perf_counter() - t0)
    total = sum(times)
    value = flops * len(times) / total / 1e12
    print(json.dumps({
        "metric": METRIC, "value": value, "unit": "TFLOP/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total / len(times) * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "impl": "reference", "config": bench_config(args.gpus),
        "flops_per_matvec": flops,
        "cpu_baseline": {"value": value, "unit": "TFLOP/s", "cores": host_cores(),
                         "kind": "port",
                         "sample": f"{len(times)} oracle heff2 matvecs, one per step, after "
                                   f"{max(1, args.warmup)} warm-up calls"},
        "e2e": {"value": value, "unit": "TFLOP/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }))


def dmrg_solve(args) -> dict:
    """Config-2 solves end to end on the GPU: the L = 64 SU(2) Heisenberg chain from the
    seeded start, chi = 256 (dense), cutoff 1e-10, ncv = 20, the reference's convergence
    tolerances, at most 10 sweeps -- first from empty plan caches (planning included),
    then again with the caches warm, and in the 3xBF16 precision form; energies against
    the reference's own run.  Beside it, the oracle's DMRG (the reference's algorithm in
    NumPy) on the host cores for its first sweep, a bounded sample of the same solve."""
    import torch

    from tenet import network

    L = 64
    out = {"workload": "L=64 SU(2) Heisenberg, chi=256 dense, cutoff 1e-10, ncv=20, max 10 "
                       "sweeps, seeded start 2j<=16", "reference_energy": REF_DMRG["energy"],
           "reference_sweeps": REF_DMRG["sweeps"]}
    for name, kw in (("f64_cold", {}), ("f64_warm", {}), ("3xbf16", {"precision": "3xbf16"})):
        psi = chain64_start(L)
        stamps = []
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        o = network.dmrg_(psi, network.heisenberg_mpo_su2(L), chi=256, cutoff=1e-10, ncv=20,
                          max_sweeps=10, callback=lambda r: stamps.append(time.perf_counter()),
                          **kw)
        torch.cuda.synchronize()
        sec = time.perf_counter() - t0
        out[name] = {"seconds": sec, "solves_per_s": 1.0 / sec, "sweeps": o.sweeps,
                     "energy": o.energy,
                     "abs_dE_per_site_vs_reference": abs(o.energy - REF_DMRG["energy"]) / L,
                     "first_sweep_s": stamps[0] - t0 if stamps else None}
    if not args.no_cpu:
        import oracle.tenet_oracle as O

        phys = tuple(PHYS.items())
        bonds = [tuple((j, 1) for j in range(i % 2, min(i, L - i, 16) + 1, 2))
                 for i in range(L + 1)]
        psi = [O.random(O.Structure(O.SU2, (O.Leg(bonds[i], O.OUT), O.Leg(phys, O.OUT),
                                            O.Leg(bonds[i + 1], O.IN))), i) for i in range(L)]
        t0 = time.perf_counter()
        stamps = []
        O.dmrg(psi, O.heisenberg_mpo_su2(L), chi=256, cutoff=1e-10, ncv=20, max_sweeps=1,
               on_sweep=lambda k, p, e: stamps.append((time.perf_counter() - t0, e)))
        out["cpu_baseline"] = {
            "kind": "port", "cores": host_cores(),
            "sample": "the oracle's DMRG, first sweep of the same solve (canonisation and "
                      "environment set-up included)",
            "first_sweep_s": stamps[0][0], "first_sweep_energy": stamps[0][1],
            "gpu_first_sweep_speedup": stamps[0][0] / out["f64_cold"]["first_sweep_s"]}
    return out


def run_tenet(args) -> None:
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120))

    from tenet import _exec, _lib, network
    from tenet.program import GraphMatvec, heff2_folded_program, heff2_program

    tensors = build_workload(seed=rank)
    fl, w1, w2, fr, aa = tensors
    # the metric's work: the reference's four-contraction lowering (sum of 2 M K N)
    flops = heff2_flops()
    launches_eager = launches_per_matvec(tensors)
    # the timed form: the environments' default, the MPO-folded two-contraction chain
    lf, rf = network.fold_left(fl, w1), network.fold_right(w2, fr)
    prog = heff2_folded_program(lf, rf, aa.structure)
    site = heff2_program(fl, w1, w2, fr, aa.structure)
    assert site.flops == flops
    gm = GraphMatvec(prog)
    gm.x.copy_(aa.arena)
    flush = torch.empty(256 * 1024 * 1024 // 8, dtype=torch.float64, device="cuda")

    def timed(fn, steps):
        """Device time of ``steps`` calls, L2 flushed (untimed) between them."""
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(steps)]
        torch.cuda.synchronize()
        for k in range(steps):
            flush.fill_(float(k))
            ev[k][0].record()
            fn()
            ev[k][1].record()
        torch.cuda.synchronize()
        return sum(a.elapsed_time(b) for a, b in ev)

    # other forms, for comparison: the plain FP64 form (eager, op by op), the reference's
    # four-contraction order as a graph, the folded chain without a graph, without
    # programmatic dependent launch, and as one persistent launch
    gm_site = GraphMatvec(site)
    gm_site.x.copy_(aa.arena)
    forms_ms = {}
    for name, fn in (("eager_ops", lambda: network.heff2(fl, w1, w2, fr, aa)),
                     ("eager_chain", lambda: prog.run(gm.x, gm.y)),
                     ("graph_site_order", gm_site.replay)):
        for _ in range(args.warmup):
            fn()
        forms_ms[name] = timed(fn, args.steps) / args.steps
    from tenet import program as _program

    lib = _lib.load()
    lib.tnb_set_pdl(0)
    gm_plain = GraphMatvec(prog)
    lib.tnb_set_pdl(1)
    _exec.FUSE = True
    gm_fused = GraphMatvec(prog)
    _exec.FUSE = False
    # the same chain planned for one launch on one thread-block cluster (off by default)
    _exec.CLUSTER = True
    _program._HEFF_TABLES.clear()
    prog_cl = heff2_folded_program(lf, rf, aa.structure)
    gm_cluster = GraphMatvec(prog_cl) if prog_cl.cluster is not None else None
    _exec.CLUSTER = False
    _program._HEFF_TABLES.clear()
    for name, g in (("graph_without_pdl", gm_plain), ("graph_grid_fused_one_launch", gm_fused),
                    ("graph_cluster_one_launch", gm_cluster)):
        if g is None:
            continue
        for _ in range(args.warmup):
            g.replay()
        forms_ms[name] = timed(g.replay, args.steps) / args.steps

    # the precision form: the sector products big enough to be dense contractions on the
    # tcgen05 tensor cores (and, for comparison, every non-skinny product there)
    mixed = {}
    ref_out = site(aa).numpy_arena()
    for precision, tc_min in (("3xbf16", None), ("tf32", None), ("3xbf16", 0), ("tf32", 0)):
        mprog = heff2_folded_program(lf, rf, aa.structure, precision=precision,
                                     tc_min_flops=tc_min)
        mg = GraphMatvec(mprog)
        mg.x.copy_(aa.arena)
        for _ in range(args.warmup):
            mg.replay()
        mms = timed(mg.replay, args.steps) / args.steps
        got = mg(aa).numpy_arena()
        mixed[precision + ("_all_products" if tc_min == 0 else "")] = {
            "ms_per_matvec": mms, "tflops": flops / (mms * 1e-3) / 1e12,
            "tensor_core_products": sum(len(p.table) for lk in mprog.links
                                        for p in lk.gemm.parts if p.kind in (3, 4)),
            "rel_error_vs_f64": float(np.linalg.norm(got - ref_out) / np.linalg.norm(ref_out))}

    # the other bond histograms: graph matvec, folded and in the reference's order
    others = {}
    for wname, bond in WORKLOADS.items():
        t5 = build_workload(seed=rank, bond=bond)
        wf = heff2_flops(bond)
        pf = heff2_folded_program(network.fold_left(t5[0], t5[1]),
                                  network.fold_right(t5[2], t5[3]), t5[4].structure)
        ps = heff2_program(*t5[:4], t5[4].structure)
        row = {"bond_multiplets": {str(k): v for k, v in bond.items()}, "flops_per_matvec": wf}
        for tag, pp in (("folded", pf), ("site_order", ps)):
            g = GraphMatvec(pp)
            g.x.copy_(t5[4].arena)
            for _ in range(args.warmup):
                g.replay()
            wms = timed(g.replay, args.steps) / args.steps
            row[tag] = {"ms_per_matvec": wms, "tflops": wf / (wms * 1e-3) / 1e12,
                        "launches": pp.launches}
        others[wname] = row

    for _ in range(args.warmup):
        gm.replay()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    with Clocks(local) as clk:
        ms = timed(gm.replay, args.steps)
        # the timed steps take well under the 200 ms sampling period: keep the same replay
        # loop running for a second so the sampler sees it under load
        t_end = time.perf_counter() + 1.0
        while time.perf_counter() < t_end:
            for _ in range(50):
                gm.replay()
            torch.cuda.synchronize()
    ms = max_over_ranks(ms, "cuda")
    if world > 1:
        dist.barrier()
    value = job_value(flops, args.steps, world, ms)
    launches_per_step = prog.launches

    # kernel timing pass: the same steps, each enqueued behind a GPU-side head start so
    # the per-launch events bracket device execution only (no host gaps)
    log = _exec.LaunchLog(timed=True)
    for k in range(args.steps):
        flush.fill_(float(k))
        torch.cuda._sleep(2_000_000)
        with log:
            prog.run(gm.x, gm.y)
    kernels = log.summary()
    # the one-cluster launch alone, timed the same way (head start, events on the stream)
    cluster_ms = None
    if prog.cluster is not None:
        evs = []
        for k in range(args.steps):
            flush.fill_(float(k))
            torch.cuda._sleep(2_000_000)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            prog.run(gm.x, gm.y)
            b.record()
            evs.append((a, b))
        torch.cuda.synchronize()
        cluster_ms = sum(a.elapsed_time(b) for a, b in evs) / args.steps
    # algorithmic bytes of one matvec: every gather's source terms and destination, every
    # product's A, B and C (FP64)
    gemm_bytes = 8 * sum(int(M) * int(K) + int(K) * int(N) + int(M) * int(N)
                         for lk in prog.links for part in lk.gemm.parts
                         for M, N, K in (r[:3] for r in part.table))
    gather_bytes = kernels.get("block_gather", {"work": 0})["work"] / args.steps
    matvec_bytes = gemm_bytes + gather_bytes

    # end to end through the public API with host buffers: every step copies the input
    # from pinned host memory, runs the chain and copies the result back, all three in
    # one graph launch (GraphMatvec with host_io)
    gm_host = GraphMatvec(prog, host_io=True)
    gm_host.host_x.copy_(aa.arena.detach().cpu())
    out_size = aa.arena.numel()

    def e2e_step():
        gm_host.replay_host()

    for _ in range(max(1, args.warmup)):
        e2e_step()
    e_ms = max_over_ranks(timed(e2e_step, args.steps), "cuda")
    e2e_value = job_value(flops, args.steps, world, e_ms)
    torch.cuda.synchronize()
    gm.replay()
    torch.cuda.synchronize()
    assert torch.equal(gm_host.host_y, gm.y.cpu()), "the host-buffer matvec differs"
    assert _lib.device_error(0) == 0, "a kernel raised the device error word during the bench"

    if rank == 0:
        pk = peaks()
        dgemm = measure_dgemm_peak(torch)
        # per kernel class: its share of the kernel time and its achieved rate (GEMMs in
        # executed TFLOP/s against cuBLAS DGEMM; gathers and gather-fused GEMMs in GB/s of
        # algorithmic bytes against HBM)
        classes = {k: v for k, v in kernels.items() if v["ms"] > 0}
        total_kernel_ms = sum(v["ms"] for v in classes.values())
        table = {}
        for k, v in classes.items():
            is_flops = k == "grouped_gemm_f64"
            rate = v["work"] / (v["ms"] * 1e-3) / (1e12 if is_flops else 1e9)
            table[k] = {"launches": v["launches"], "ms": v["ms"],
                        "share": v["ms"] / total_kernel_ms if total_kernel_ms else 0,
                        ("tflops_executed" if is_flops else "gbs"): rate,
                        ("dgemm_peak_tflops" if is_flops else "hbm_peak_gbs"):
                            dgemm if is_flops else pk["hbm_gbs"]}
        key = max(classes, key=lambda k: classes[k]["ms"]) if classes else "block_gather"
        dom = table.get(key, {})
        is_flops = key == "grouped_gemm_f64"
        roofline = {
            "bound": "tensor" if is_flops else "hbm",
            "kernel": key,
            "achieved": dom.get("tflops_executed" if is_flops else "gbs", 0.0),
            "peak": dgemm if is_flops else pk["hbm_gbs"],
            "unit": "TFLOP/s" if is_flops else "GB/s",
            "peak_source": ("cuBLAS DGEMM 8192^3 measured in this run (FP64 has no entry in "
                            "MEASURED_PEAKS.json)") if is_flops
            else f"MEASURED_PEAKS.json hbm_gbs ({pk['src']})",
            # DRAM bytes per launch (read + write) of the same kernel on this workload, from
            # one ncu capture of this build (cold cache; in the graph replay the operands
            # sit in L2), in bytes, mean over the captured launches
            "traffic": NCU_TRAFFIC.get(key),
            "kernels": table,
            "kernel_ms_per_step": total_kernel_ms / args.steps,
            "graph_ms_per_step": ms / args.steps,
        }
        if cluster_ms is not None:
            # the whole matvec is one kernel: its algorithmic bytes over its duration
            roofline.update({
                "bound": "hbm", "kernel": "chain_cluster_kernel",
                "achieved": matvec_bytes / (cluster_ms * 1e-3) / 1e9, "peak": pk["hbm_gbs"],
                "unit": "GB/s", "peak_source": f"MEASURED_PEAKS.json hbm_gbs ({pk['src']})",
                "traffic": NCU_TRAFFIC.get("chain_cluster_kernel"),
                "algorithmic_bytes_per_launch": matvec_bytes,
                "kernel_ms_per_launch": cluster_ms,
                "cluster_ctas": prog.cluster_ctas,
                "note": "the kernels entry times the same stages launched one by one"})
        roofline["frac"] = roofline["achieved"] / roofline["peak"] if roofline["peak"] else None
        base = cpu_baseline(flops, budget_s=args.cpu_budget) if not args.no_cpu else None
        solve = dmrg_solve(args) if args.dmrg else None
        solves = serving(args) if args.serve_requests > 0 else None
        env3 = batched_env_updates(args) if args.config3_n > 0 else None
        bmv = (batched_matvecs(args, forms_ms["eager_ops"], ms / args.steps)
               if args.batch_n > 0 else None)
        gprobe = gemm_probe(args.gemm_n, dgemm) if args.gemm_n > 0 else None
        print(json.dumps({
            "metric": METRIC, "value": value, "unit": "TFLOP/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": bench_config(world),
            "flops_per_matvec": flops, "gemm_flops_executed_per_matvec": prog.flops,
            "elements_aa": int(aa.arena.numel()),
            "e2e": {"value": e2e_value, "unit": "TFLOP/s",
                    "h2d_bytes_per_step": int(aa.arena.numel() * 8),
                    "d2h_bytes_per_step": int(out_size * 8)},
            "gpu_launches": int(args.steps * launches_per_step),
            "launches_per_step": launches_per_step,
            "forms_ms_per_matvec": {"graph_folded": ms / args.steps, **forms_ms},
            "forms_tflops": {"graph_folded": flops / (ms / args.steps * 1e-3) / 1e12,
                             **{k: flops / (v * 1e-3) / 1e12 for k, v in forms_ms.items()}},
            "launches_per_matvec_eager_ops": launches_eager,
            "launches_per_matvec_site_order": site.launches,
            "other_workloads": others,
            "mixed_precision_forms": mixed,
            "dmrg_solve": solve,
            "serving": solves,
            "batched_env_updates": env3,
            "batched_matvecs": bmv,
            "gemm_probe": gprobe,
            "roofline": roofline,
            "cpu_baseline": base,
            "clocks": clk.summary(),
        }))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="tenet", choices=["tenet", "reference"])
    ap.add_argument("--cpu-budget", type=float, default=20.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--serve-requests", type=int, default=6,
                    help="served DMRG requests in the solves/s comparison (0: skip)")
    ap.add_argument("--serve-slots", type=int, default=8)
    ap.add_argument("--serve-workers", type=int, default=4,
                    help="worker processes of the host-parallel serving arms")
    ap.add_argument("--batch-n", type=int, default=32,
                    help="members of the batched heff2 matvec (0: skip)")
    ap.add_argument("--config3-n", type=int, default=64,
                    help="members of the batched U1xU1xfZ2 environment update (0: skip)")
    ap.add_argument("--serve-full", action="store_true",
                    help="draw the requests from the full L / chi distribution")
    ap.add_argument("--gemm-n", type=int, default=4096,
                    help="size of the square product of the GEMM tile-kind probe (0: skip)")
    ap.add_argument("--profile-gemm", type=int, default=0,
                    help="only run each GEMM tile kind once on this square size (for "
                         "profiling the tensor-core kernels) and exit")
    ap.add_argument("--profile-heff2", type=int, default=0,
                    help="only run the headline matvec's stage launches this many times (a "
                         "small, fixed launch sequence for profiling its kernels) and exit")
    ap.add_argument("--profile-config3", action="store_true",
                    help="only run the batched environment update a few times (a small, "
                         "fixed launch sequence for profiling its kernels) and exit")
    ap.add_argument("--serve-stream", action="store_true",
                    help="only serve the full config-5 stream (--serve-requests requests, "
                         "--serve-workers workers) at three arrival rates, print and exit")
    ap.add_argument("--serve-rate-requests", type=int, default=0,
                    help="requests of each Poisson arm of --serve-stream (0: all)")
    ap.add_argument("--serve-plain-sample", type=int, default=12,
                    help="requests of the stream the plain FP64 form solves for the baseline")
    ap.add_argument("--no-dmrg", dest="dmrg", action="store_false",
                    help="skip the config-2 DMRG time-to-solution leg")
    ap.add_argument("--derive-bond", action="store_true",
                    help="grow the L = 64 chain to --derive-chi multiplets and print its "
                         "mid-chain bond histogram, then exit")
    ap.add_argument("--derive-chi", type=int, default=256)
    ap.add_argument("--derive-sweeps", type=int, default=6)
    args = ap.parse_args()
    if args.derive_bond:
        derive_bond(args)
        return
    if args.serve_stream:
        serve_stream(args)
        return
    if args.warmup < 3:
        args.warmup = 3
    if args.profile_gemm > 0:
        gemm_probe(args.profile_gemm, None, reps=1)
        return
    if args.profile_heff2:
        import torch

        from tenet import network
        from tenet.program import heff2_folded_program

        fl, w1, w2, fr, aa = build_workload()
        prog = heff2_folded_program(network.fold_left(fl, w1), network.fold_right(w2, fr),
                                    aa.structure)
        y = torch.empty_like(aa.arena)
        for _ in range(args.profile_heff2):
            prog.run(aa.arena, y)
        torch.cuda.synchronize()
        return
    if args.profile_config3:
        import torch

        from tenet import batch

        F, A, W = config3_batch(args.config3_n)
        for _ in range(3):
            batch.env_update_last(F, A, W)
        torch.cuda.synchronize()
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_tenet(args)


if __name__ == "__main__":
    main()
