"""Generate the golden vectors in ``tests/golden/`` by running the reference itself.

Run in a container that has the reference source (it is imported, never copied)::

    python tests/golden/make_golden.py /path/to/TeNeT-py

The reference's missing third-party dependencies are replaced by the test-only shims in
``tests/golden/_refshim`` (a NumPy ``autoray`` subset, an ``opt_einsum`` stub that refuses,
and an SU(2) ``racah`` stand-in computed by ``oracle/racah_su2.py``).  Everything written
here is the reference's own output on seeded inputs:

* ``cases.npz`` + ``cases.json``: operand and result tensors of transpose / repartition /
  tensordot / einsum / inner / norm / svd_truncated over U(1), Z2, fZ2 and SU(2), with the
  exact block keys of every structure;
* ``config1.json``: the U(1) ``einsum("abcd,cdef->abef")`` at full size (operands are
  regenerated from their seeds by the test), recorded as per-block checksums;
* ``heff.npz`` + ``heff.json``: one SU(2) Heisenberg two-site ``Env.heff2`` application on a
  mid-chain bond (site-tensor path), its Lanczos ground energy at ``ncv=20``, and the
  truncated SVD of the result;
* ``dmrg.json``: reference DMRG energies and per-bond kept sectors, and the spread of the
  reference's own first-sweep energy when its canonised start is perturbed at the
  rounding level (the ``spread`` part);
* ``dmrg64.json``: the L = 64, chi = 256 SU(2) Heisenberg DMRG (site-tensor and prepared
  paths) with its per-sweep history and final bond spaces;
* ``ctmrg.json``: Z2 Ising CTMRG (beta = 0.44 at chi = 16 and 128 for a fixed number of
  moves; beta = 0.40, chi = 16 to convergence): per-sweep corner-spectrum changes, final
  corner spectrum and bond sectors, the reference's beta f estimate and Onsager's;
* ``su2_tables.npz``: the reference's full SU(2) F and R fixture tables;
* ``su2_f_sample.txt``: every 37th row of the reference's F-symbol fixture with the
  value the reference's F-symbol route returns.

No test reads the reference at run time; only these files are committed.
"""

from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]


def _setup(ref: Path) -> None:
    sys.path[:0] = [str(HERE / "_refshim"), str(REPO), str(ref / "src")]


# ---------------------------------------------------------------------------------------
# serialisation: legs as JSON, blocks concatenated in block_order (C order each)


def _sector_int(s) -> int:
    for name in ("charge", "parity", "two_j"):
        if hasattr(s, name):
            return int(getattr(s, name))
    raise TypeError(s)


def _legs(t) -> list:
    return [
        {
            "provider": leg.provider.name,
            "sectors": [[_sector_int(a), m] for a, m in leg.space.sectors],
            "side": leg.side.value,
            "dual": bool(leg.dual),
        }
        for leg in t.legs
    ]


def _tree(tr) -> list:
    return [[_sector_int(u) for u in tr.uncoupled], [_sector_int(u) for u in tr.inner],
            _sector_int(tr.coupled)]


def _keys(t) -> list:
    return [[_tree(k.output_tree), _tree(k.input_tree)] for k in t.structure.block_order]


def _arena(t) -> np.ndarray:
    if not t.blocks:
        return np.zeros(0)
    return np.concatenate([np.asarray(b, dtype=np.float64).ravel() for b in t.blocks])


class Store:
    def __init__(self) -> None:
        self.meta: dict = {}
        self.arrays: dict = {}

    def tensor(self, name: str, t) -> dict:
        self.arrays[name] = _arena(t)
        return {"legs": _legs(t), "keys": _keys(t), "arena": name}

    def dump(self, stem: str) -> None:
        (HERE / f"{stem}.json").write_text(json.dumps(self.meta, indent=1))
        np.savez_compressed(HERE / f"{stem}.npz", **self.arrays)


# ---------------------------------------------------------------------------------------


def make_cases(store: Store) -> None:
    import tenet
    from tenet import IN, OUT, GradedSpace, Leg, SymmetricTensor
    from tenet.symmetry import SU2, U1, Z2, SU2Sector, U1Sector, Z2Sector, fZ2, FZ2Sector

    def rnd(legs, seed):
        return SymmetricTensor.random(tuple(legs), seed=seed)

    cases = []

    def record(name, op, operands, output, **args):
        entry = {"name": name, "op": op, "args": args}
        entry["operands"] = [store.tensor(f"{name}/in{i}", t) for i, t in enumerate(operands)]
        if output is not None:
            entry["output"] = store.tensor(f"{name}/out", output)
        cases.append(entry)

    # --- U(1): config-1 shape class at reduced degeneracy -----------------------------
    V = GradedSpace.new(U1, {U1Sector(q): max(1, round(4 * np.exp(-q * q / 4))) for q in range(-3, 4)})
    A = rnd([Leg(V, OUT)] * 4, 0)
    B = rnd([Leg(V, IN), Leg(V, IN), Leg(V, OUT), Leg(V, OUT)], 1)
    record("u1_einsum_abcd_cdef", "einsum", [A, B], tenet.einsum("abcd,cdef->abef", A, B),
           equation="abcd,cdef->abef")
    W = GradedSpace.new(U1, {U1Sector(-2): 1, U1Sector(0): 2, U1Sector(1): 3, U1Sector(3): 1})
    T = rnd([Leg(W, OUT), Leg(V, IN), Leg(W, OUT, True), Leg(V, IN, True)], 2)
    record("u1_transpose", "transpose", [T], tenet.transpose(T, (2, 3, 0, 1)), axes=[2, 3, 0, 1])
    record("u1_repartition", "repartition", [T], tenet.repartition(T, (1, 3), (0, 2)),
           outputs=[1, 3], inputs=[0, 2])
    X = rnd([Leg(W, OUT), Leg(V, OUT), Leg(W, IN)], 3)
    Y = rnd([Leg(W, OUT), Leg(V, IN), Leg(W, OUT, True)], 4)
    record("u1_tensordot_bend", "tensordot", [X, Y], tenet.tensordot(X, Y, ((0, 2), (2, 0))),
           axes=[[0, 2], [2, 0]])
    record("u1_inner", "inner", [T, rnd(T.legs, 5)], None, value=float(tenet.inner(T, rnd(T.legs, 5))))

    # --- Z2 and fZ2 ---------------------------------------------------------------------
    for prov, S, tag in ((Z2, Z2Sector, "z2"), (fZ2, FZ2Sector, "fz2")):
        P = GradedSpace.new(prov, {S(0): 3, S(1): 2})
        Q = GradedSpace.new(prov, {S(0): 2, S(1): 4})
        a = rnd([Leg(P, OUT), Leg(Q, OUT), Leg(P, IN), Leg(Q, IN)], 10)
        b = rnd([Leg(Q, OUT), Leg(P, OUT), Leg(Q, IN)], 11)
        record(f"{tag}_transpose", "transpose", [a], tenet.transpose(a, (1, 0, 3, 2)),
               axes=[1, 0, 3, 2])
        record(f"{tag}_repartition", "repartition", [a], tenet.repartition(a, (0, 3, 1), (2,)),
               outputs=[0, 3, 1], inputs=[2])
        record(f"{tag}_einsum", "einsum", [a, b], tenet.einsum("abcd,dce->abe", a, b),
               equation="abcd,dce->abe")
        b2 = rnd([Leg(Q, IN), Leg(P, OUT), Leg(Q, IN)], 12)
        record(f"{tag}_einsum_perm", "einsum", [a, b2], tenet.einsum("abcd,bef->acdef", a, b2),
               equation="abcd,bef->acdef")

    # --- SU(2) ----------------------------------------------------------------------------
    H = GradedSpace.new(SU2, {SU2Sector(1): 1})
    Bd = GradedSpace.new(SU2, {SU2Sector(0): 2, SU2Sector(2): 3, SU2Sector(4): 1})
    Bo = GradedSpace.new(SU2, {SU2Sector(1): 2, SU2Sector(3): 2, SU2Sector(5): 1})
    aa = rnd([Leg(Bd, OUT), Leg(H, OUT), Leg(H, OUT), Leg(Bd, IN)], 20)
    record("su2_transpose_braid", "transpose", [aa], tenet.transpose(aa, (0, 2, 1, 3)),
           axes=[0, 2, 1, 3])
    record("su2_transpose_cycle", "transpose", [aa], tenet.transpose(aa, (2, 0, 1, 3)),
           axes=[2, 0, 1, 3])
    record("su2_repartition", "repartition", [aa], tenet.repartition(aa, (0, 1), (2, 3)),
           outputs=[0, 1], inputs=[2, 3])
    record("su2_repartition_back", "repartition", [aa], tenet.repartition(aa, (3, 1), (2, 0)),
           outputs=[3, 1], inputs=[2, 0])
    Mw = GradedSpace.new(SU2, {SU2Sector(0): 2, SU2Sector(2): 1})
    f = rnd([Leg(Bd, OUT), Leg(Mw, IN, True), Leg(Bd, IN)], 21)
    record("su2_einsum_apqr_rys", "einsum", [aa, f], tenet.einsum("apqr,rys->apqys", aa, f),
           equation="apqr,rys->apqys")
    g = rnd([Leg(Bd, IN), Leg(H, IN), Leg(Bo, OUT)], 22)
    record("su2_einsum_bend", "einsum", [aa, g], tenet.einsum("apqr,aps->qrs", aa, g),
           equation="apqr,aps->qrs")
    record("su2_inner", "inner", [aa, rnd(aa.legs, 23)], None,
           value=float(tenet.inner(aa, rnd(aa.legs, 23))))
    record("su2_norm", "norm", [aa], None, value=float(tenet.norm(aa)))
    u, s, vh = tenet.linalg.svd_truncated(aa, ((0, 1), (2, 3)), max_bond=12, cutoff=1e-10)
    record("su2_svd_truncated", "svd_truncated", [aa], s, axes=[[0, 1], [2, 3]], max_bond=12,
           cutoff=1e-10, bond=[[_sector_int(c), m] for c, m in s.legs[0].space.sectors])
    record("su2_svd_truncated_u", "svd_truncated_u", [aa], u)
    record("su2_svd_truncated_vh", "svd_truncated_vh", [aa], vh)
    store.meta["cases"] = cases


def make_config1() -> dict:
    import tenet
    from tenet import IN, OUT, GradedSpace, Leg, SymmetricTensor
    from tenet.symmetry import U1, U1Sector

    V = GradedSpace.new(U1, {U1Sector(q): round(12 * np.exp(-q * q / 4)) for q in range(-3, 4)})
    A = SymmetricTensor.random((Leg(V, OUT),) * 4, seed=0)
    B = SymmetricTensor.random((Leg(V, IN), Leg(V, IN), Leg(V, OUT), Leg(V, OUT)), seed=1)
    C = tenet.einsum("abcd,cdef->abef", A, B)
    probe = np.random.default_rng(12345)
    blocks = []
    for blk in C.blocks:
        x = np.asarray(blk).ravel()
        w = probe.standard_normal(x.size)
        blocks.append([float(x.sum()), float((x * x).sum()), float(w @ x)])
    return {
        "degeneracies": [[q, round(12 * np.exp(-q * q / 4))] for q in range(-3, 4)],
        "equation": "abcd,cdef->abef",
        "out_legs": _legs(C),
        "keys": _keys(C),
        "checksum_seed": 12345,
        "blocks_sum_sumsq_probe": blocks,
        "first_block": np.asarray(C.blocks[0]).ravel().tolist(),
    }


def make_heff(store: Store) -> dict:
    """SU(2) Heisenberg L=12: a converged chi=32 state, its mid-chain matvec and Lanczos."""
    import tenet
    from tenet import GradedSpace
    from tenet.models import spin_half
    from tenet.network import MPO, MPS, Env, dmrg_, lanczos
    from tenet.network.dmrg import _pair
    from tenet.symmetry import SU2, SU2Sector

    site = spin_half(SU2)
    L = 12
    h = MPO.from_terms(L, [(1.0, [(site.ops["S.S"], (i, i + 1))]) for i in range(L - 1)])
    hm = h.materialize()
    bonds = [GradedSpace.new(SU2, {SU2Sector(j): 1 for j in range(i % 2, min(i, L - i) + 1, 2)})
             for i in range(L + 1)]
    out = dmrg_(MPS.random(site.phys, bonds, seed=0), hm, chi=32, max_sweeps=2)
    psi = out.psi
    psi.canonize_(0)
    env = Env(psi, hm).setup_(0)
    n_mid = L // 2 - 1
    for n in range(n_mid):  # sweep the centre to the bond (n_mid, n_mid + 1)
        aa = _pair(psi[n], psi[n + 1])
        u, s, vh = tenet.linalg.svd_truncated(aa, ((0, 1), (2, 3)), max_bond=10**6, cutoff=1e-14)
        psi[n] = u
        psi[n + 1] = tenet.einsum("xy,yqr->xqr", s, vh)
        env.clear_(n, n + 1)
        env.update_(n, to="last")
    aa = _pair(psi[n_mid], psi[n_mid + 1])
    hv = env.heff2(n_mid, aa)
    meta = {
        "L": L, "n": n_mid,
        "aa": store.tensor("aa", aa),
        "fl": store.tensor("fl", env.F[n_mid - 1, n_mid]),
        "fr": store.tensor("fr", env.F[n_mid + 2, n_mid + 1]),
        "w1": store.tensor("w1", hm[n_mid]),
        "w2": store.tensor("w2", hm[n_mid + 1]),
        "heff_aa": store.tensor("heff_aa", hv),
    }
    e, v = lanczos(lambda x: env.heff2(n_mid, x), aa, ncv=20)
    meta["lanczos_ncv20_energy"] = e
    meta["lanczos_vec"] = store.tensor("lanczos_vec", v)
    u, s, vh = tenet.linalg.svd_truncated(v, ((0, 1), (2, 3)), max_bond=16, cutoff=1e-10)
    meta["svd_bond"] = [[_sector_int(c), m] for c, m in s.legs[0].space.sectors]
    meta["svd_s"] = store.tensor("svd_s", s)
    # the first and last sites of the materialised MPO, for boundary handling
    meta["w_first"] = store.tensor("w_first", hm[0])
    meta["w_last"] = store.tensor("w_last", hm[L - 1])
    return meta


def make_dmrg() -> dict:
    from tenet import GradedSpace
    from tenet.models import spin_half
    from tenet.network import MPO, MPS, dmrg_
    from tenet.symmetry import SU2, SU2Sector

    site = spin_half(SU2)
    runs = {}
    for L, chi, sweeps in ((12, 32, 4), (16, 24, 3)):
        h = MPO.from_terms(L, [(1.0, [(site.ops["S.S"], (i, i + 1))]) for i in range(L - 1)])
        bonds = [GradedSpace.new(SU2, {SU2Sector(j): 1 for j in range(i % 2, min(i, L - i) + 1, 2)})
                 for i in range(L + 1)]
        out = dmrg_(MPS.random(site.phys, bonds, seed=0), h.materialize(), chi=chi,
                    max_sweeps=sweeps, ncv=20, cutoff=1e-10)
        runs[f"L{L}_chi{chi}"] = {
            "L": L, "chi": chi, "sweeps": out.sweeps, "energy": out.energy,
            "history": [float(r[0]) for r in out.history],
            "bonds": [[[_sector_int(a), m] for a, m in out.psi[i].legs[0].space.sectors]
                      for i in range(L)],
        }
    return runs


def make_first_sweep_spread(runs: dict, samples: int = 60) -> None:
    """The reference's own sensitivity of a growth sweep to rounding: its first-sweep
    energy when every element of the canonised start (``MPS.canonize_``) is multiplied by
    ``1 + r eps`` with r ~ N(0, 1) and eps alternating 1e-14 and 1e-13 (the size of a
    different summation order), over ``samples`` seeds.  The sweeps that still grow the
    bonds solve spaces smaller than ncv = 20 with an unreorthogonalised Lanczos, whose Ritz
    vector then carries amplified rounding, and a truncation decision near the cutoff can
    follow it.  Stores ``first_sweep_spread`` (the largest |dE|/L seen) in each run."""
    import numpy as np

    from tenet import GradedSpace
    from tenet.models import spin_half
    from tenet.network import MPO, MPS, dmrg_
    from tenet.symmetry import SU2, SU2Sector

    site = spin_half(SU2)
    canonize = MPS.canonize_
    for rec in runs.values():
        L, chi = rec["L"], rec["chi"]
        h = MPO.from_terms(L, [(1.0, [(site.ops["S.S"], (i, i + 1))]) for i in range(L - 1)])
        h = h.materialize()
        bonds = [GradedSpace.new(SU2, {SU2Sector(j): 1 for j in range(i % 2, min(i, L - i) + 1, 2)})
                 for i in range(L + 1)]

        def first(seed, eps, L=L, chi=chi, h=h, bonds=bonds):
            def noisy(self, *a, **k):
                out = canonize(self, *a, **k)
                rng = np.random.default_rng(seed)
                for n in range(L):
                    for b in self[n].blocks:
                        flat = np.asarray(b).reshape(-1)
                        flat *= 1.0 + eps * rng.standard_normal(flat.size)
                return out

            MPS.canonize_ = noisy
            try:
                out = dmrg_(MPS.random(site.phys, bonds, seed=0), h, chi=chi, max_sweeps=1,
                            ncv=20, cutoff=1e-10)
            finally:
                MPS.canonize_ = canonize
            return float(out.history[0][0])

        e0 = rec["history"][0]
        spread = max(abs(first(100 + s, 1e-14 if s % 2 else 1e-13) - e0) / L
                     for s in range(samples))
        rec["first_sweep_spread"] = spread
        rec["first_sweep_spread_samples"] = samples


def make_dmrg64(ref: Path) -> dict:
    """The SU(2) Heisenberg chain at L = 64 through the reference's own ``dmrg_``
    (``network/dmrg.py:620-843``): ``chi = 256`` in the reference's dense sense, cutoff
    1e-10, ncv = 20, at most 10 sweeps with its default convergence tolerances, from the
    seeded random start whose bond spins are 2j <= min(i, L - i, 16).  Recorded for the
    site-tensor path (the MPO materialised: the matvec this build runs) with per-sweep
    history and every final bond space, and for the prepared path (``MPO.from_terms`` as
    given) as per-sweep energies; plus the MPSKit N = 64, chi = 256 energy of the
    reference's fixture ``tests/fixtures/mpskit_heisenberg.json``."""
    import time

    from tenet import GradedSpace
    from tenet.models import spin_half
    from tenet.network import MPO, MPS, dmrg_
    from tenet.symmetry import SU2, SU2Sector

    site = spin_half(SU2)
    L, chi = 64, 256
    h = MPO.from_terms(L, [(1.0, [(site.ops["S.S"], (i, i + 1))]) for i in range(L - 1)])
    bonds = [GradedSpace.new(SU2, {SU2Sector(j): 1
                                   for j in range(i % 2, min(i, L - i, 16) + 1, 2)})
             for i in range(L + 1)]
    rec = {"L": L, "chi": chi, "ncv": 20, "cutoff": 1e-10, "max_sweeps": 10, "max_2j": 16}
    for name, op in (("site", h.materialize()), ("prepared", h)):
        t0 = time.perf_counter()
        per_sweep = []

        def record(o, per_sweep=per_sweep):
            per_sweep.append([[[_sector_int(a), m] for a, m in o.psi[i].legs[0].space.sectors]
                              for i in range(L)])

        out = dmrg_(MPS.random(site.phys, bonds, seed=0), op, chi=chi, cutoff=1e-10, ncv=20,
                    max_sweeps=10, callback=record)
        run = {"sweeps": out.sweeps, "energy": out.energy,
               "history": [[float(x) for x in r] for r in out.history],
               "seconds": time.perf_counter() - t0}
        if name == "site":
            run["bonds"] = per_sweep[-1]
            run["bonds_per_sweep"] = per_sweep
        rec[name] = run
    fix = json.loads((ref / "tests/fixtures/mpskit_heisenberg.json").read_text())
    rec["mpskit_N64_chi256"] = fix["N64"]["chi256"]["energy"]
    return rec


def make_ctmrg(ref: Path) -> dict:
    """Z2 CTMRG of the 2D Ising model (``network/ctmrg.py:451-660``): beta = 0.44 near the
    critical point (a fixed number of moves, chi = 16 and 128) and beta = 0.40 run to its
    1e-10 tolerance with the reference's free-energy estimator on the result."""
    sys.path.insert(0, str(ref / "examples" / "toy_codes"))
    import ctmrg as toy  # examples/toy_codes/ctmrg.py: ising_bulk, beta_free_energy, onsager

    from tenet.network import ctmrg, single_layer_ctm
    from tenet.network.common import spectrum

    out = {}
    for name, beta, chi, tol, sweeps in (("b044_chi16", 0.44, 16, 0.0, 60),
                                         ("b044_chi128", 0.44, 128, 0.0, 20),
                                         ("b040_chi16", 0.40, 16, 1e-10, 200)):
        bulk = toy.ising_bulk(beta)
        res = ctmrg(*single_layer_ctm(bulk), chi=chi, tol=tol, max_sweeps=sweeps)
        c, e, bond = res.env
        out[name] = {
            "beta": beta, "chi": chi, "tol": tol, "max_sweeps": sweeps, "sweeps": res.sweeps,
            "converged": bool(res.converged), "history": [float(x) for x in res.history],
            "spectrum": spectrum(c), "bond": [[_sector_int(a), m] for a, m in bond.sectors],
            "bulk": {"legs": _legs(bulk), "keys": _keys(bulk), "arena": _arena(bulk).tolist()},
        }
        if res.converged:
            out[name]["beta_f"] = float(toy.beta_free_energy(beta, res.env, k=0))
            out[name]["onsager_beta_f"] = float(toy.onsager(beta))
    return out


def make_su2_tables(ref: Path) -> None:
    """The reference's full SU(2) coefficient fixtures as a compact archive: every row of
    ``tests/fixtures/su2_f.txt`` (109,900 F-symbols, 2j <= 12) and ``su2_r.txt`` (616
    R-symbol signs), the tables its ``tests/symmetry/test_su2_recoupling.py`` checks."""
    f = np.loadtxt(ref / "tests/fixtures/su2_f.txt")
    r = np.loadtxt(ref / "tests/fixtures/su2_r.txt", dtype=np.int64)
    np.savez_compressed(HERE / "su2_tables.npz", f_dj=f[:, :6].astype(np.int8),
                        f_value=f[:, 6], r_dj=r[:, :3].astype(np.int8),
                        r_value=r[:, 3].astype(np.int8))


def make_f_sample(ref: Path) -> None:
    from tenet.symmetry import SU2, SU2Sector

    rows = [r for r in (ref / "tests/fixtures/su2_f.txt").read_text().splitlines()
            if not r.startswith("#")]
    lines = ["# every 37th row of the reference fixture tests/fixtures/su2_f.txt",
             "# columns: dj1 dj2 dj3 dj4 dj5 dj6 fixture_value reference_f_symbol"]
    for r in rows[::37]:
        parts = r.split()
        dj = tuple(int(x) for x in parts[:6])
        val = SU2.f_symbol(*(SU2Sector(x) for x in dj))
        lines.append(" ".join(parts[:7]) + f" {val!r}")
    (HERE / "su2_f_sample.txt").write_text("\n".join(lines) + "\n")


def main() -> None:
    if len(sys.argv) not in (2, 3):
        raise SystemExit("usage: python tests/golden/make_golden.py <path to the TeNeT-py tree>"
                         " [dmrg64 | su2tables | spread]")
    ref = Path(sys.argv[1])
    _setup(ref)
    if len(sys.argv) == 3:  # one part alone
        if sys.argv[2] == "dmrg64":
            (HERE / "dmrg64.json").write_text(json.dumps(make_dmrg64(ref)))
        elif sys.argv[2] == "su2tables":
            make_su2_tables(ref)
        elif sys.argv[2] == "spread":
            runs = json.loads((HERE / "dmrg.json").read_text())
            make_first_sweep_spread(runs)
            (HERE / "dmrg.json").write_text(json.dumps(runs, indent=1))
        else:
            raise SystemExit(f"unknown part {sys.argv[2]!r}")
        return
    store = Store()
    make_cases(store)
    store.dump("cases")
    (HERE / "config1.json").write_text(json.dumps(make_config1()))
    hs = Store()
    hs.meta = make_heff(hs)
    hs.dump("heff")
    runs = make_dmrg()
    make_first_sweep_spread(runs)
    (HERE / "dmrg.json").write_text(json.dumps(runs, indent=1))
    (HERE / "ctmrg.json").write_text(json.dumps(make_ctmrg(ref)))
    (HERE / "dmrg64.json").write_text(json.dumps(make_dmrg64(ref)))
    make_f_sample(ref)
    make_su2_tables(ref)


if __name__ == "__main__":
    main()
