"""Parity of the CUDA path with the reference's golden vectors and with the oracle.

Every test calls the library through the package's public API (which drives the C ABI)
and compares against (a) outputs of the reference itself (``tests/golden``), at 1e-12
relative per block -- the tolerance stated for the FP64 plain form -- and
(b) the oracle on seeded random inputs at sizes the oracle finishes in seconds.  Block
keys must be identical.  After each test the sticky device error word must be clear.
"""

import json
from pathlib import Path

import numpy as np
import pytest
import torch

import oracle.tenet_oracle as O
import tenet
from tenet import _lib, linalg, network
from tenet.structure import IN, OUT, GradedSpace, Leg, TensorStructure, layout
from tenet.symmetry import SU2, U1, Z2, fZ2

pytestmark = pytest.mark.gpu
PROV = {"U1": U1, "Z2": Z2, "fZ2": fZ2, "SU2": SU2}
RTOL = 1e-12


def struct(legs_json):
    p = PROV[legs_json[0]["provider"]]
    return TensorStructure(tuple(
        Leg(GradedSpace.new(p, {p.sector(a): m for a, m in leg["sectors"]}),
            OUT if leg["side"] == "out" else IN, bool(leg["dual"])) for leg in legs_json))


def keys(d):
    t = lambda x: (tuple(x[0]), tuple(x[1]), x[2])  # noqa: E731
    return tuple((t(o), t(i)) for o, i in d["keys"])


def load(arrays, d):
    s = struct(d["legs"])
    assert s.keys == keys(d)
    return tenet.SymmetricTensor.from_numpy_arena(s, arrays[d["arena"]])


def close(got, want, rtol=RTOL):
    """``got`` within ``rtol`` of ``want``.  For a tensor the bound holds per block,
    relative to that block's own largest entry (an all-zero block is measured against the
    whole tensor's largest entry); for a plain array, relative to its largest entry."""
    blocks = None
    if isinstance(got, tenet.SymmetricTensor):
        lay = layout(got.structure)
        blocks = [(int(o), int(n)) for o, n in zip(lay.offsets, lay.sizes)]
        got = got.numpy_arena()
    got, want = np.asarray(got), np.asarray(want)
    assert got.shape == want.shape
    if not want.size:
        return
    whole = max(np.abs(want).max(), 1e-300)
    if blocks is None:
        err = np.abs(got - want).max() / whole
        assert err <= rtol, f"relative error {err:.3e} > {rtol:.1e}"
        return
    worst, at = 0.0, -1
    for b, (o, n) in enumerate(blocks):
        if n == 0:
            continue
        w = want[o:o + n]
        err = np.abs(got[o:o + n] - w).max() / (np.abs(w).max() or whole)
        if err > worst:
            worst, at = err, b
    assert worst <= rtol, f"block {at}: relative error {worst:.3e} > {rtol:.1e}"


@pytest.fixture(autouse=True)
def _device_error_clear():
    yield
    torch.cuda.synchronize()
    assert _lib.device_error(0) == 0, "a kernel raised the device error word"


@pytest.fixture(scope="module")
def cases(golden_dir):
    return json.loads((golden_dir / "cases.json").read_text()), np.load(golden_dir / "cases.npz")


def test_golden_cases(cases):
    meta, arrays = cases
    done = 0
    for c in meta["cases"]:
        op, a = c["op"], c["args"]
        ins = [load(arrays, d) for d in c["operands"]]
        if op == "einsum":
            out = tenet.einsum(a["equation"], *ins)
        elif op == "transpose":
            out = tenet.transpose(ins[0], a["axes"])
        elif op == "repartition":
            out = tenet.repartition(ins[0], a["outputs"], a["inputs"])
        elif op == "tensordot":
            out = tenet.tensordot(ins[0], ins[1], a["axes"])
        elif op == "inner":
            assert tenet.inner(*ins) == pytest.approx(a["value"], rel=RTOL)
            continue
        elif op == "norm":
            assert tenet.norm(*ins) == pytest.approx(a["value"], rel=RTOL)
            continue
        elif op == "svd_truncated":
            u, s, vh = linalg.svd_truncated(ins[0], a["axes"], max_bond=a["max_bond"],
                                            cutoff=a["cutoff"])
            want = struct(c["output"]["legs"])
            assert s.structure == want, "kept bond sectors differ from the reference"
            close(s, arrays[c["output"]["arena"]])
            # U S Vh reconstructs the truncated tensor (vectors carry a sign gauge)
            rec = tenet.einsum("abx,xy->aby", u, s)
            rec = tenet.compose(tenet.repartition(rec, (0, 1), (2,)), vh)
            ref = O.svd_truncated(O.from_arena(O.structure_from_json(c["operands"][0]["legs"]),
                                               arrays[c["operands"][0]["arena"]]),
                                  a["axes"], max_bond=a["max_bond"], cutoff=a["cutoff"])
            want_rec = O.compose(O.repartition(O.einsum("abx,xy->aby", ref[0], ref[1]), (0, 1),
                                               (2,)), ref[2]).arena()
            close(rec, want_rec, 1e-11)
            continue
        else:
            continue
        assert out.structure == struct(c["output"]["legs"]), c["name"]
        close(out, arrays[c["output"]["arena"]])
        done += 1
    assert done >= 15


def test_heff2_lanczos_svd_golden(golden_dir):
    m = json.loads((golden_dir / "heff.json").read_text())
    h = np.load(golden_dir / "heff.npz")
    T = {k: load(h, m[k]) for k in ("aa", "fl", "fr", "w1", "w2")}
    out = network.heff2(T["fl"], T["w1"], T["w2"], T["fr"], T["aa"])
    assert out.structure == struct(m["heff_aa"]["legs"])
    close(out, h[m["heff_aa"]["arena"]])
    e, v = network.lanczos(lambda x: network.heff2(T["fl"], T["w1"], T["w2"], T["fr"], x),
                           T["aa"], ncv=20)
    assert e == pytest.approx(m["lanczos_ncv20_energy"], rel=1e-12)
    _, s, _ = linalg.svd_truncated(v, ((0, 1), (2, 3)), max_bond=16, cutoff=1e-10)
    assert [[SU2.label(a), k] for a, k in s.legs[0].space.sectors] == m["svd_bond"]
    close(s, h[m["svd_s"]["arena"]], 1e-9)


def test_env_folds_match_oracle(golden_dir):
    """Both environment folds on a seeded site tensor (``network/env.py:620-629``)."""
    m = json.loads((golden_dir / "heff.json").read_text())
    h = np.load(golden_dir / "heff.npz")
    fl, fr, w1 = (load(h, m[k]) for k in ("fl", "fr", "w1"))
    ofl, ofr, ow1 = (O.from_arena(O.structure_from_json(m[k]["legs"]), h[m[k]["arena"]])
                     for k in ("fl", "fr", "w1"))
    bond, phys = m["aa"]["legs"][0], m["aa"]["legs"][1]
    site = [dict(bond, side="out"), dict(phys, side="out"), dict(bond, side="in")]
    a = tenet.SymmetricTensor.random(struct(site).legs, seed=5)
    oa = O.random(O.structure_from_json(site), 5)
    got, want = network.env_update_last(fl, a, w1), O.env_update_last(ofl, oa, ow1)
    assert got.structure.keys == O.block_order(want.structure)
    close(got, want.arena())
    got, want = network.env_update_first(fr, a, w1), O.env_update_first(ofr, oa, ow1)
    assert got.structure.keys == O.block_order(want.structure)
    close(got, want.arena())


def test_folded_env_updates_match_the_three_contraction_ones(golden_dir):
    """Growing an environment through the folded one (``F . W`` kept from the bond's
    matvec) gives the same environment as the reference's three contractions."""
    m = json.loads((golden_dir / "heff.json").read_text())
    h = np.load(golden_dir / "heff.npz")
    fl, fr, w1, w2 = (load(h, m[k]) for k in ("fl", "fr", "w1", "w2"))
    bond, phys = m["aa"]["legs"][0], m["aa"]["legs"][1]
    site = [dict(bond, side="out"), dict(phys, side="out"), dict(bond, side="in")]
    a = tenet.SymmetricTensor.random(struct(site).legs, seed=7)
    want = network.env_update_last(fl, a, w1)
    got = network.env_update_last_folded(network.fold_left(fl, w1), a)
    assert got.structure == want.structure
    close(got, want.numpy_arena(), 1e-13)
    want = network.env_update_first(fr, a, w2)
    got = network.env_update_first_folded(network.fold_right(w2, fr), a)
    assert got.structure == want.structure
    close(got, want.numpy_arena(), 1e-13)


def test_config1_full_size_against_reference_checksums(golden_dir):
    g = json.loads((golden_dir / "config1.json").read_text())
    V = GradedSpace.new(U1, {U1.sector(q): d for q, d in g["degeneracies"]})
    A = tenet.SymmetricTensor.random((Leg(V, OUT),) * 4, seed=0)
    B = tenet.SymmetricTensor.random((Leg(V, IN), Leg(V, IN), Leg(V, OUT), Leg(V, OUT)), seed=1)
    C = tenet.einsum(g["equation"], A, B)
    assert C.structure.keys == keys(g)
    probe = np.random.default_rng(g["checksum_seed"])
    for blk, (s, ss, pr) in zip(C.blocks, g["blocks_sum_sumsq_probe"]):
        x = blk.cpu().numpy().ravel()
        w = probe.standard_normal(x.size)
        assert float((x * x).sum()) == pytest.approx(ss, rel=1e-12)
        assert float(w @ x) == pytest.approx(pr, rel=1e-10, abs=1e-9)
    close(C.blocks[0].cpu().numpy().ravel(), np.array(g["first_block"]))
    # element by element at full size against the oracle (pinned to the same checksums
    # by the CPU suite), 1e-12 relative per block
    sec = tuple((q, d) for q, d in g["degeneracies"])
    oA = O.random(O.Structure(O.U1, (O.Leg(sec, O.OUT),) * 4), 0)
    oB = O.random(O.Structure(O.U1, (O.Leg(sec, O.IN), O.Leg(sec, O.IN), O.Leg(sec, O.OUT),
                                     O.Leg(sec, O.OUT))), 1)
    close(C, O.einsum(g["equation"], oA, oB).arena())


SU2_SPACES = [
    {0: 2, 2: 3, 4: 1},
    {1: 2, 3: 1},
    {0: 1, 2: 2, 4: 2, 6: 1},
]


def _o_leg(p, sec, side, dual=False):
    return O.Leg(tuple(sorted(sec.items())), side, dual)


def _leg(p, sec, side, dual=False):
    return Leg(GradedSpace.new(p, {p.sector(a): m for a, m in sec.items()}), side, dual)


@pytest.mark.parametrize("seed", range(6))
def test_random_su2_contractions_against_oracle(seed):
    rng = np.random.default_rng(100 + seed)
    bond = SU2_SPACES[seed % 3]
    half = {1: 1}
    sides = [OUT if x else IN for x in rng.integers(0, 2, 4)]
    duals = [bool(x) for x in rng.integers(0, 2, 4)]
    spaces = [bond, half, half, bond]
    legs = [_leg(SU2, sp, sd, du) for sp, sd, du in zip(spaces, sides, duals)]
    olegs = [_o_leg(SU2, sp, O.OUT if sd is OUT else O.IN, du)
             for sp, sd, du in zip(spaces, sides, duals)]
    a = tenet.SymmetricTensor.random(legs, seed=seed)
    oa = O.random(O.Structure(O.SU2, tuple(olegs)), seed)
    if oa.arena().size == 0:
        pytest.skip("no allowed block for this random leg pattern")
    perm = tuple(int(x) for x in rng.permutation(4))
    close(tenet.transpose(a, perm), O.transpose(oa, perm).arena())
    outs = tuple(int(x) for x in rng.permutation(4)[:2])
    ins = tuple(i for i in range(4) if i not in outs)
    close(tenet.repartition(a, outs, ins), O.repartition(oa, outs, ins).arena())
    # contract legs 2,3 against a partner built to be contractible
    plegs = [Leg(legs[2].space, legs[2].side, not legs[2].dual),
             Leg(legs[3].space, legs[3].side, not legs[3].dual), _leg(SU2, bond, OUT)]
    oplegs = [O.Leg(olegs[2].sectors, olegs[2].side, not olegs[2].dual),
              O.Leg(olegs[3].sectors, olegs[3].side, not olegs[3].dual),
              _o_leg(SU2, bond, O.OUT)]
    b = tenet.SymmetricTensor.random(plegs, seed=seed + 50)
    ob = O.random(O.Structure(O.SU2, tuple(oplegs)), seed + 50)
    got = tenet.einsum("abcd,cde->eab", a, b)
    want = O.einsum("abcd,cde->eab", oa, ob)
    assert got.structure.keys == O.block_order(want.structure)
    close(got, want.arena())


@pytest.mark.parametrize("prov", ["U1", "fZ2", "Z2"])
def test_random_abelian_contractions_against_oracle(prov):
    p, op = PROV[prov], {"U1": O.U1, "fZ2": O.FZ2, "Z2": O.Z2}[prov]
    sec = {-1: 2, 0: 3, 1: 2} if prov == "U1" else {0: 3, 1: 2}
    A = [(sec, OUT, False), (sec, IN, False), (sec, OUT, True), (sec, IN, False)]
    a = tenet.SymmetricTensor.random([_leg(p, *x) for x in A], seed=7)
    oa = O.random(O.Structure(op, tuple(_o_leg(op, s, O.OUT if sd is OUT else O.IN, d)
                                        for s, sd, d in A)), 7)
    B = [(sec, OUT, False), (sec, OUT, False), (sec, IN, False)]
    b = tenet.SymmetricTensor.random([_leg(p, *x) for x in B], seed=8)
    ob = O.random(O.Structure(op, tuple(_o_leg(op, s, O.OUT if sd is OUT else O.IN, d)
                                        for s, sd, d in B)), 8)
    for eq in ("abcd,dbe->ace", "abcd,bef->acdfe"):
        got = tenet.einsum(eq, a, b)
        want = O.einsum(eq, oa, ob)
        assert got.structure.keys == O.block_order(want.structure)
        close(got, want.arena())
    close(tenet.transpose(a, (3, 1, 0, 2)), O.transpose(oa, (3, 1, 0, 2)).arena())


def test_vector_ops_and_cabi_direct():
    """The C ABI called with raw device pointers: axpby and the weighted dot."""
    import ctypes

    n = 100_003
    x = torch.randn(n, dtype=torch.float64, device="cuda")
    y = torch.randn(n, dtype=torch.float64, device="cuda")
    out = torch.empty_like(x)
    lib = _lib.load()
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert lib.tnb_axpby(n, 2.0, x.data_ptr(), -0.5, y.data_ptr(), out.data_ptr(), s) == 0
    close(out.cpu().numpy(), 2.0 * x.cpu().numpy() - 0.5 * y.cpu().numpy(), 1e-15)
    starts = torch.tensor([0, 10, 50_000, n], dtype=torch.int64, device="cuda")
    w = torch.tensor([1.0, 3.0, 2.0], dtype=torch.float64, device="cuda")
    work = torch.zeros(lib.tnb_dot_work_bytes(n), dtype=torch.uint8, device="cuda")
    res = torch.empty(1, dtype=torch.float64, device="cuda")
    for _ in range(2):  # the workspace is reusable
        assert lib.tnb_weighted_dot(x.data_ptr(), y.data_ptr(), n, starts.data_ptr(),
                                    w.data_ptr(), 3, work.data_ptr(), res.data_ptr(), s) == 0
        xh, yh = x.cpu().numpy(), y.cpu().numpy()
        want = (xh[:10] @ yh[:10]) + 3 * (xh[10:50000] @ yh[10:50000]) + 2 * (xh[50000:] @ yh[50000:])
        assert res.item() == pytest.approx(want, rel=1e-12)


def test_empty_and_degenerate_inputs():
    # a U(1) leg pattern with no charge-conserving block: empty arena end to end
    V = GradedSpace.new(U1, {U1.sector(1): 2})
    t = tenet.SymmetricTensor.random((Leg(V, OUT), Leg(V, OUT)), seed=0)
    assert t.arena.numel() == 0
    assert tenet.transpose(t, (1, 0)).arena.numel() == 0
    assert tenet.norm(t) == 0.0
    # outer product: no contracted axis
    W = GradedSpace.new(U1, {U1.sector(0): 2, U1.sector(1): 1})
    a = tenet.SymmetricTensor.random((Leg(W, OUT), Leg(W, IN)), seed=1)
    b = tenet.SymmetricTensor.random((Leg(W, OUT), Leg(W, IN)), seed=2)
    oa = O.random(O.Structure(O.U1, (O.Leg(((0, 2), (1, 1)), O.OUT), O.Leg(((0, 2), (1, 1)), O.IN))), 1)
    ob = O.random(O.Structure(O.U1, (O.Leg(((0, 2), (1, 1)), O.OUT), O.Leg(((0, 2), (1, 1)), O.IN))), 2)
    close(tenet.tensordot(a, b, ((), ())), O.tensordot(oa, ob, ((), ())).arena())


def test_compiled_chain_and_graph_match_golden(golden_dir):
    """The compiled heff2 program (eager and CUDA-graph replay) against the reference."""
    from tenet.program import GraphMatvec, heff2_program

    m = json.loads((golden_dir / "heff.json").read_text())
    h = np.load(golden_dir / "heff.npz")
    T = {k: load(h, m[k]) for k in ("aa", "fl", "fr", "w1", "w2")}
    prog = heff2_program(T["fl"], T["w1"], T["w2"], T["fr"], T["aa"].structure)
    want = h[m["heff_aa"]["arena"]]
    close(prog(T["aa"]), want)
    gm = GraphMatvec(prog)
    for _ in range(3):  # replays are repeatable
        close(gm(T["aa"]), want)
    e, _ = network.lanczos(gm, T["aa"], ncv=20)
    assert e == pytest.approx(m["lanczos_ncv20_energy"], rel=1e-12)


def test_folded_heff2_matches_golden_and_site_order(golden_dir):
    """The folded two-contraction matvec (MPO sites folded into the environments) against
    the reference's heff2 output, per block at 1e-12, eagerly and as a compiled graph;
    and against the four-contraction program on the bench workload."""
    import bench
    from tenet.program import GraphMatvec, heff2_folded_program, heff2_program

    m = json.loads((golden_dir / "heff.json").read_text())
    h = np.load(golden_dir / "heff.npz")
    T = {k: load(h, m[k]) for k in ("aa", "fl", "fr", "w1", "w2")}
    lf, rf = network.fold_left(T["fl"], T["w1"]), network.fold_right(T["w2"], T["fr"])
    want = h[m["heff_aa"]["arena"]]
    close(network.heff2_folded(lf, rf, T["aa"]), want)
    prog = heff2_folded_program(lf, rf, T["aa"].structure)
    assert prog.launches <= 5
    close(prog(T["aa"]), want)
    close(GraphMatvec(prog)(T["aa"]), want)
    fl, w1, w2, fr, aa = bench.build_workload()
    site = heff2_program(fl, w1, w2, fr, aa.structure)(aa).numpy_arena()
    folded = heff2_folded_program(network.fold_left(fl, w1), network.fold_right(w2, fr),
                                  aa.structure)
    close(GraphMatvec(folded)(aa), site)


def test_cluster_chain_is_bit_identical_to_stage_by_stage(golden_dir):
    """A compact chain (every stage a few dozen items) runs as one launch on one
    thread-block cluster: the same tables and arithmetic as the stage-by-stage replay,
    identical bits, repeatedly, through a captured graph and in a device Lanczos solve."""
    import bench
    from tenet import _exec
    from tenet.program import GraphMatvec, heff2_folded_program, heff2_program

    from tenet import program

    m = json.loads((golden_dir / "heff.json").read_text())
    h = np.load(golden_dir / "heff.npz")
    T = {k: load(h, m[k]) for k in ("aa", "fl", "fr", "w1", "w2")}
    fl, w1, w2, fr, aa = bench.build_workload()
    _exec.CLUSTER = True  # planned for the cluster launch (off by default)
    program._HEFF_TABLES.clear()
    try:
        cases = [(heff2_folded_program(network.fold_left(fl, w1), network.fold_right(w2, fr),
                                       aa.structure), aa),
                 (heff2_program(fl, w1, w2, fr, aa.structure), aa),
                 (heff2_folded_program(network.fold_left(T["fl"], T["w1"]),
                                       network.fold_right(T["w2"], T["fr"]),
                                       T["aa"].structure), T["aa"])]
        _check_cluster_cases(cases)
    finally:
        _exec.CLUSTER = False
        program._HEFF_TABLES.clear()
    close(GraphMatvec(cases[2][0])(T["aa"]), h[m["heff_aa"]["arena"]])


def _check_cluster_cases(cases):
    from tenet import _exec
    from tenet.program import GraphMatvec

    for prog, x in cases:
        assert prog.compact and prog.cluster is not None and prog.launches == 1
        try:
            _exec.CLUSTER = False
            want = GraphMatvec(prog)(x).numpy_arena()
        finally:
            _exec.CLUSTER = True
        g = GraphMatvec(prog)
        for _ in range(3):
            assert np.array_equal(g(x).numpy_arena(), want)
        assert np.array_equal(prog(x).numpy_arena(), want)
        lz = network.DeviceLanczos(prog, 12)
        e1, v1 = lz.solve(x)
        try:
            _exec.CLUSTER = False
            e0, v0 = network.DeviceLanczos(prog, 12).solve(x)
        finally:
            _exec.CLUSTER = True
        assert e1 == e0 and np.array_equal(v1.numpy_arena(), v0.numpy_arena())


def test_gather_fused_gemm_matches_the_two_launch_link(golden_dir):
    """A link whose A gather runs inside its GEMM (``tnb_grouped_gemm_gather_a``) gives
    the products of the gather-then-GEMM pair (within 1e-13 per block: the pair splits
    long K, the fused tile does not) and the reference's heff2 (1e-12 per block); the
    headline matvec becomes 3 launches, replayed from a graph and in a device Lanczos
    solve."""
    import bench
    from tenet import _exec, program
    from tenet.program import GraphMatvec, heff2_folded_program

    m = json.loads((golden_dir / "heff.json").read_text())
    h = np.load(golden_dir / "heff.npz")
    T = {k: load(h, m[k]) for k in ("aa", "fl", "fr", "w1", "w2")}
    fl, w1, w2, fr, aa = bench.build_workload()
    cases = [(network.fold_left(fl, w1), network.fold_right(w2, fr), aa),
             (network.fold_left(T["fl"], T["w1"]), network.fold_right(T["w2"], T["fr"]),
              T["aa"])]
    outs = {}
    for fuse in (True, False):
        _exec.FUSE_A = fuse
        program._HEFF_TABLES.clear()
        try:
            for k, (lf, rf, x) in enumerate(cases):
                prog = heff2_folded_program(lf, rf, x.structure)
                if fuse:
                    assert any(lk.ga is not None for lk in prog.links)
                    if k == 0:
                        assert prog.launches == 3
                    e, _ = network.DeviceLanczos(prog, 12).solve(x)
                    outs[("lanczos", k)] = e
                outs[(fuse, k)] = GraphMatvec(prog)(x)
        finally:
            _exec.FUSE_A = False
            program._HEFF_TABLES.clear()
    for k in range(len(cases)):
        close(outs[(True, k)], outs[(False, k)].numpy_arena(), 1e-13)
    close(outs[(True, 1)], h[m["heff_aa"]["arena"]])


def test_bench_workload_program_matches_oracle():
    """The bench's 256-multiplet workload: compiled chain against the oracle, per block."""
    import bench

    tensors = bench.build_workload()
    from tenet.program import heff2_program

    prog = heff2_program(*tensors[:4], tensors[4].structure)
    assert prog.flops == bench.heff2_flops()
    got = prog(tensors[4]).numpy_arena()
    want = O.heff2(*bench.oracle_workload()).arena()
    close(got, want)


@pytest.mark.parametrize("kind", [0, 1, 2, 5])
def test_grouped_gemm_kinds_against_numpy(kind):
    """Every tile kind on uneven products, K = 0 included, through the C ABI."""
    from tenet import _exec

    rng = np.random.default_rng(kind)
    if kind == 2:
        shapes = [(1000, 3, 3), (777, 1, 1), (5, 16, 16), (300, 2, 0)]
    elif kind == 5:
        shapes = [(3, 1000, 3), (1, 777, 1), (16, 5, 16), (2, 300, 0), (4, 25790, 4)]
    else:
        shapes = [(176, 236, 60), (9, 11, 2), (64, 64, 64), (65, 33, 17), (40, 7, 0), (1, 1, 1),
                  (176, 60, 236), (41, 10, 511), (3, 2, 1000)]
    a_off = b_off = c_off = 0
    prods, mats = [], []
    for M, N, K in shapes:
        prods.append((M, N, K, a_off, K, b_off, N, c_off, N))
        mats.append((a_off, b_off, c_off))
        a_off += M * K
        b_off += K * N
        c_off += M * N
    A = rng.standard_normal(a_off)
    B = rng.standard_normal(b_off)
    table = _exec.make_gemm(prods, kind)
    if kind in (0, 1):
        assert table.n_counters > 0, "the long-K products must take the split-K path"
    ta, tb = torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda()
    for _ in range(2):  # the split-K counters must be left zero for the next run
        tc = torch.full((c_off,), float("nan"), dtype=torch.float64, device="cuda")
        table.run(ta, tb, tc)
        C = tc.cpu().numpy()
        for (M, N, K), (ao, bo, co) in zip(shapes, mats):
            want = A[ao:ao + M * K].reshape(M, K) @ B[bo:bo + K * N].reshape(K, N)
            close(C[co:co + M * N].reshape(M, N), want, 1e-13)


def test_heisenberg_mpo_matches_reference_site_tensors(golden_dir):
    """The SU(2) Heisenberg MPO builder against the reference's materialised W (L = 12)."""
    m = json.loads((golden_dir / "heff.json").read_text())
    h = np.load(golden_dir / "heff.npz")
    mpo = network.heisenberg_mpo_su2(12)
    for site, key in ((5, "w1"), (6, "w2")):
        assert mpo[site].structure == struct(m[key]["legs"])
        close(mpo[site], h[m[key]["arena"]], 1e-14)  # the reference splits S.S by an SVD
    # boundary sites: same spaces as the reference's, up to the dual flag of a spin-0 leg
    for site, key in ((0, "w_first"), (11, "w_last")):
        got = [leg.space for leg in mpo[site].legs]
        want = [leg.space for leg in struct(m[key]["legs"]).legs]
        assert got == want


@pytest.mark.parametrize("fold", [True, False])
@pytest.mark.parametrize("run", ["L12_chi32", "L16_chi24"])
def test_dmrg_su2_matches_reference(golden_dir, run, fold):
    """Full two-site DMRG on the GPU against the reference's own run (``dmrg_`` at
    ncv = 20, cutoff 1e-10, same seeded start): the same number of sweeps, every kept
    bond space identical, every sweep after the first within 1e-8 per site and the last
    one within 1e-10 relative.  The first sweep grows the bonds from one multiplet per
    spin: it solves spaces smaller than ncv = 20 with an unreorthogonalised Lanczos, whose
    Ritz vector then carries amplified rounding, and a truncation near the cutoff can
    follow it.  The reference itself moves that sweep's energy by up to
    ``first_sweep_spread`` per site (2.1e-7 at L = 12) when its canonised start changes at
    the rounding level (``make_golden.py ... spread``, 60 seeds); the first sweep is held
    to five times that.  Both matvec forms: the folded two-contraction one (default) and
    the reference's four-contraction order."""
    g = json.loads((golden_dir / "dmrg.json").read_text())[run]
    L, chi = g["L"], g["chi"]
    phys = GradedSpace.new(SU2, {SU2.sector(1): 1})
    bonds = [GradedSpace.new(SU2, {SU2.sector(j): 1 for j in range(i % 2, min(i, L - i) + 1, 2)})
             for i in range(L + 1)]
    psi = network.MPS.random(phys, bonds, seed=0)
    out = network.dmrg_(psi, network.heisenberg_mpo_su2(L), chi=chi, cutoff=1e-10,
                        ncv=20, max_sweeps=g["sweeps"], fold=fold)
    assert out.sweeps == g["sweeps"] and out.psi is psi
    first_tol = max(1e-8, 5.0 * g["first_sweep_spread"])
    for k, (got, want) in enumerate(zip(out.history, g["history"])):
        assert abs(got[0] - want) / L <= (first_tol if k == 0 else 1e-8), k
    assert out.energy == pytest.approx(g["history"][-1], rel=1e-10)
    kept = [[[SU2.label(a), k] for a, k in psi[i].legs[0].space.sectors] for i in range(L)]
    assert kept == g["bonds"], "kept bond sectors differ from the reference's"


def test_programmatic_dependent_launch_changes_nothing(golden_dir):
    """The chain with and without programmatic dependent launch: bit-identical results."""
    from tenet.program import GraphMatvec, heff2_program

    m = json.loads((golden_dir / "heff.json").read_text())
    h = np.load(golden_dir / "heff.npz")
    T = {k: load(h, m[k]) for k in ("aa", "fl", "fr", "w1", "w2")}
    lib = _lib.load()
    outs = []
    try:
        for flag in (0, 1):
            lib.tnb_set_pdl(flag)
            prog = heff2_program(T["fl"], T["w1"], T["w2"], T["fr"], T["aa"].structure)
            gm = GraphMatvec(prog)
            outs.append([gm(T["aa"]).numpy_arena() for _ in range(3)])
    finally:
        lib.tnb_set_pdl(1)
    for a, b in zip(outs[0], outs[1]):
        assert np.array_equal(a, b)
    close(tenet.SymmetricTensor.from_numpy_arena(T["aa"].structure, outs[1][0]),
          h[m["heff_aa"]["arena"]])


@pytest.mark.parametrize("name", ["b044_chi16", "b040_chi16", "b044_chi128"])
def test_ctmrg_z2_ising_matches_reference(golden_dir, name):
    """Z2 Ising CTMRG on the GPU against the reference's runs: the bulk tensor, the sweep
    count, every per-sweep corner-spectrum change, the final spectrum, the even/odd bond
    split, and (converged run) the free energy vs the reference and Onsager."""
    r = json.loads((golden_dir / "ctmrg.json").read_text())[name]
    bulk = network.ising_bulk(r["beta"])
    assert bulk.structure == struct(r["bulk"]["legs"])
    close(bulk, np.array(r["bulk"]["arena"]), 1e-14)
    c, e, bond, hist = network.ctmrg(*network.single_layer_ctm(bulk), chi=r["chi"], tol=r["tol"],
                                     max_sweeps=r["max_sweeps"])
    assert len(hist) == r["sweeps"]
    np.testing.assert_allclose(hist, r["history"], rtol=1e-5, atol=1e-10)
    np.testing.assert_allclose(network.spectrum(c), r["spectrum"], rtol=1e-8, atol=1e-12)
    assert [[Z2.label(a), m] for a, m in bond.sectors] == r["bond"]
    if "beta_f" in r:
        bf = network.beta_free_energy(c, e, bulk)
        assert bf == pytest.approx(r["beta_f"], rel=1e-10)
        assert bf == pytest.approx(r["onsager_beta_f"], rel=1e-6)


def test_device_lanczos_matches_reference(golden_dir):
    """The whole recurrence from one library call: the reference's ncv=20 energy and the
    same Ritz vector (up to sign) as the host-driven Lanczos; repeated solves agree."""
    from tenet.program import heff2_program

    m = json.loads((golden_dir / "heff.json").read_text())
    h = np.load(golden_dir / "heff.npz")
    T = {k: load(h, m[k]) for k in ("aa", "fl", "fr", "w1", "w2")}
    prog = heff2_program(T["fl"], T["w1"], T["w2"], T["fr"], T["aa"].structure)
    lg = network.DeviceLanczos(prog, 20)
    e_host, v_host = network.lanczos(prog, T["aa"], ncv=20)
    for _ in range(2):
        e, v = lg.solve(T["aa"])
        assert e == pytest.approx(m["lanczos_ncv20_energy"], rel=1e-12)
        assert e == pytest.approx(e_host, rel=1e-13)
        a, b = v.numpy_arena(), v_host.numpy_arena()
        sign = np.sign(a @ b)
        close(sign * a, b, 1e-10)
    # a Krylov space that breaks down early (ncv larger than the space allows)
    small = network.DeviceLanczos(prog, 60)
    e60, _ = small.solve(T["aa"])
    assert e60 == pytest.approx(network.lanczos(prog, T["aa"], ncv=60)[0], rel=1e-10)


def test_device_lanczos_graph_replay_is_bit_identical(golden_dir):
    """With ``GRAPH`` on, from its second solve on a solver replays the whole recurrence
    from a CUDA graph: the same energy and Ritz vector bits as its first (eager) solve,
    from another start vector too, and as a solver that never captures.  The step kernel that carries the
    recurrence for small vectors (``tnb_lanczos_step``) runs in both."""
    from tenet.program import heff2_program

    m = json.loads((golden_dir / "heff.json").read_text())
    h = np.load(golden_dir / "heff.npz")
    T = {k: load(h, m[k]) for k in ("aa", "fl", "fr", "w1", "w2")}
    prog = heff2_program(T["fl"], T["w1"], T["w2"], T["fr"], T["aa"].structure)
    from tenet import ops

    other = ops.add(T["aa"] * 0.5, tenet.SymmetricTensor.random(T["aa"].legs, seed=11) * 0.1)
    lg = network.DeviceLanczos(prog, 20)
    lg.GRAPH = True
    runs = [lg.solve(v) for v in (T["aa"], T["aa"], other, T["aa"])]
    assert lg._graph not in (None, False)
    eager = network.DeviceLanczos(prog, 20)
    eager.GRAPH = False
    want = {0: eager.solve(T["aa"]), 2: eager.solve(other)}
    for k, (e, v) in enumerate(runs):
        we, wv = want[2 if k == 2 else 0]
        assert e == we
        assert np.array_equal(v.numpy_arena(), wv.numpy_arena())


@pytest.mark.parametrize("n", [1500, 6000])
def test_lanczos_step_kernel_against_the_five_launches(n):
    """``tnb_lanczos_step`` (one CTA) against tnb_weighted_dot + tnb_lanczos_update +
    tnb_weighted_dot + tnb_lanczos_next on the same state: bit-identical while the dots
    are one chunk (n <= 2048), within rounding beyond; also the stop at j + 1 == ncv and
    the zero vector once stopped."""
    lib = _lib.load()
    P = lambda t: t.data_ptr()  # noqa: E731
    g = torch.Generator(device="cuda").manual_seed(5)
    v, vp, w0 = (torch.randn(n, dtype=torch.float64, device="cuda", generator=g)
                 for _ in range(3))
    starts = torch.tensor([0, n // 3, n // 2, n], dtype=torch.int64, device="cuda")
    weights = torch.tensor([1.0, 3.0, 2.0], dtype=torch.float64, device="cuda")
    ncv, j = 8, 3
    st0 = torch.zeros(3 * ncv + 2, dtype=torch.float64, device="cuda")
    st0[ncv + j - 1] = 0.7
    work = torch.zeros(int(lib.tnb_dot_work_bytes(n)), dtype=torch.uint8, device="cuda")
    outs = []
    for fused in (False, True):
        st, w = st0.clone(), w0.clone()
        nxt = torch.full((n,), np.nan, dtype=torch.float64, device="cuda")
        if fused:
            _lib.call("tnb_lanczos_step", n, P(w), P(v), P(vp), P(nxt), P(st), j, ncv, 1e-13,
                      P(starts), P(weights), 3, None)
        else:
            _lib.call("tnb_weighted_dot", P(v), P(w), n, P(starts), P(weights), 3, P(work),
                      P(st) + 8 * j, None)
            _lib.call("tnb_lanczos_update", n, P(w), P(v), P(vp), P(st), j, ncv, None)
            _lib.call("tnb_weighted_dot", P(w), P(w), n, P(starts), P(weights), 3, P(work),
                      P(st) + 8 * (2 * ncv + j), None)
            _lib.call("tnb_lanczos_next", n, P(w), P(nxt), P(st), j, ncv, 1e-13, None)
        torch.cuda.synchronize()
        outs.append((st.cpu().numpy(), w.cpu().numpy(), nxt.cpu().numpy()))
    (s1, w1, x1), (s2, w2, x2) = outs
    if n <= 2048:
        assert np.array_equal(s1, s2) and np.array_equal(w1, w2) and np.array_equal(x1, x2)
    else:
        assert np.allclose(s1, s2, rtol=1e-13, atol=0) and np.abs(x1 - x2).max() < 1e-13
    assert s2[3 * ncv] == j + 2 and s2[3 * ncv + 1] == 0.0
    # the last step stops; a stopped recurrence only zeroes the next vector
    st, w = st0.clone(), w0.clone()
    nxt = torch.ones(n, dtype=torch.float64, device="cuda")
    _lib.call("tnb_lanczos_step", n, P(w), P(v), P(vp), P(nxt), P(st), ncv - 1, ncv, 1e-13,
              P(starts), P(weights), 3, None)
    _lib.call("tnb_lanczos_step", n, P(w), P(v), P(vp), P(nxt), P(st), ncv - 1, ncv, 1e-13,
              P(starts), P(weights), 3, None)
    torch.cuda.synchronize()
    assert st[3 * ncv].item() == ncv and st[3 * ncv + 1].item() == 1.0
    assert (nxt == 0).all()
    assert lib.tnb_lanczos_step_max_n() >= 6000


def test_multi_dot_and_reorth_kernels():
    """The reorthogonalisation primitives through the C ABI against NumPy."""
    import ctypes

    lib = _lib.load()
    n, k = 70_001, 7
    g = torch.Generator(device="cuda").manual_seed(3)
    V = torch.randn((k, n), dtype=torch.float64, device="cuda", generator=g)
    x = torch.randn(n, dtype=torch.float64, device="cuda", generator=g)
    ptrs = torch.tensor([V[i].data_ptr() for i in range(k)], dtype=torch.int64, device="cuda")
    starts = torch.tensor([0, 100, n], dtype=torch.int64, device="cuda")
    w = torch.tensor([2.0, 1.0], dtype=torch.float64, device="cuda")
    work = torch.zeros(lib.tnb_multi_dot_work_bytes(n, k), dtype=torch.uint8, device="cuda")
    out = torch.empty(k, dtype=torch.float64, device="cuda")
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for _ in range(2):
        assert lib.tnb_multi_dot(n, k, ptrs.data_ptr(), x.data_ptr(), starts.data_ptr(),
                                 w.data_ptr(), 2, work.data_ptr(), out.data_ptr(), s) == 0
        Vh, xh = V.cpu().numpy(), x.cpu().numpy()
        want = 2.0 * Vh[:, :100] @ xh[:100] + Vh[:, 100:] @ xh[100:]
        close(out.cpu().numpy(), want, 1e-12)
    y = x.clone()
    assert lib.tnb_lanczos_reorth(n, k, out.data_ptr(), ptrs.data_ptr(), y.data_ptr(), None, 1,
                                  s) == 0
    close(y.cpu().numpy(), xh - out.cpu().numpy() @ Vh, 1e-12)


def test_recorded_sequence_replays_the_chain_bit_identically(golden_dir):
    """A chain program's recorded launch sequence, replayed with its placeholder buffers
    patched to other vectors, gives bit-identical results to launching the same tables
    one by one from the host, and can be captured in a CUDA graph."""
    from tenet import _exec
    from tenet.program import heff2_program

    m = json.loads((golden_dir / "heff.json").read_text())
    h = np.load(golden_dir / "heff.npz")
    T = {k: load(h, m[k]) for k in ("aa", "fl", "fr", "w1", "w2")}
    prog = heff2_program(T["fl"], T["w1"], T["w2"], T["fr"], T["aa"].structure, defer=True)
    assert len(prog.seq) == prog.launches == 6
    assert [lk.deferred for lk in prog.links] == [False, True, True, False]
    x = T["aa"].arena
    y_seq = torch.full_like(prog.y_slot, float("nan"))
    y_py = torch.full_like(prog.y_slot, float("nan"))
    prog.run(x, y_seq)
    prog._run_tables(x, y_py)
    assert torch.equal(y_seq, y_py)
    close(tenet.SymmetricTensor.from_numpy_arena(T["aa"].structure, y_seq.cpu().numpy()),
          load(h, m["heff_aa"]).numpy_arena(), 1e-12)
    # the product-source gathers give the bits of the GEMM-then-gather chain they replace
    plain = heff2_program(T["fl"], T["w1"], T["w2"], T["fr"], T["aa"].structure, defer=False)
    assert plain.launches == 8 and not any(lk.deferred for lk in plain.links)
    y_plain = torch.full_like(prog.y_slot, float("nan"))
    plain.run(x, y_plain)
    assert torch.equal(y_plain, y_seq)
    # a sequence appended to itself twice replays both copies
    s2 = _exec.Seq()
    _lib.call("tnb_seq_append", s2.handle, prog.seq.handle)
    _lib.call("tnb_seq_append", s2.handle, prog.seq.handle)
    assert len(s2) == 2 * len(prog.seq)
    # graph capture of a replay
    g = torch.cuda.CUDAGraph()
    y_g = torch.zeros_like(y_py)
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        prog.run(x, y_g)
    torch.cuda.current_stream().wait_stream(side)
    y_g.zero_()
    with torch.cuda.graph(g):
        prog.run(x, y_g)
    g.replay()
    torch.cuda.synchronize()
    assert torch.equal(y_g, y_py)
    # the host-buffer graph: pinned input in, the chain, pinned output back, one launch
    from tenet.program import GraphMatvec

    gh = GraphMatvec(prog, host_io=True)
    gh.host_x.copy_(x.cpu())
    gh.replay_host()
    torch.cuda.synchronize()
    assert torch.equal(gh.host_y, y_py.cpu())


def _ed_j1j2(L: int, j1: float, j2: float) -> float:
    """Ground energy of the dense spin-1/2 J1-J2 chain (open ends) by exact diagonalisation."""
    sx = np.array([[0, 0.5], [0.5, 0]])
    sy = np.array([[0, -0.5j], [0.5j, 0]])
    sz = np.array([[0.5, 0], [0, -0.5]])

    def site_op(op, i):
        out = np.eye(1)
        for k in range(L):
            out = np.kron(out, op if k == i else np.eye(2))
        return out

    ops_ = [[site_op(o, i) for o in (sx, sy, sz)] for i in range(L)]
    H = np.zeros((2 ** L, 2 ** L), dtype=complex)
    for i in range(L):
        for d, jj in ((1, j1), (2, j2)):
            if jj and i + d < L:
                H += jj * sum(a @ b for a, b in zip(ops_[i], ops_[i + d]))
    return float(np.linalg.eigvalsh(H)[0])


@pytest.mark.parametrize("j2", [0.0, 0.25, 0.4])
def test_j1j2_dmrg_matches_exact_diagonalisation(j2):
    """The SU(2) J1-J2 MPO (spectator channel for the next-nearest S.S) through two-site
    DMRG on the device gives the exact ground energy of the dense chain."""
    from tenet.structure import GradedSpace
    from tenet.symmetry import SU2

    L = 8
    phys = GradedSpace.new(SU2, {SU2.sector(1): 1})
    bonds = [GradedSpace.new(SU2, {SU2.sector(j): 1 for j in range(i % 2, min(i, L - i) + 1, 2)})
             for i in range(L + 1)]
    h = network.heisenberg_mpo_su2(L, 1.0, j2)
    out = network.dmrg_(network.MPS.random(phys, bonds, seed=0), h, chi=64,
                        cutoff=1e-14, ncv=20, max_sweeps=12)
    assert out.energy == pytest.approx(_ed_j1j2(L, 1.0, j2), abs=1e-9)


def test_fused_chain_is_bit_identical_to_stage_by_stage(golden_dir):
    """The persistent one-launch chain runs the same tables and arithmetic as the
    stage-by-stage replay: identical bits on the golden heff2 and on the bench workload,
    repeatedly (its grid barrier and split-K counters return to zero).  It runs gathers
    and GEMMs only, so its programs are planned without product-source gathers; the
    six-launch chain with them gives the same bits."""
    import bench
    from tenet import _exec, program
    from tenet.program import heff2_program

    m = json.loads((golden_dir / "heff.json").read_text())
    h = np.load(golden_dir / "heff.npz")
    T = {k: load(h, m[k]) for k in ("aa", "fl", "fr", "w1", "w2")}
    w = bench.build_workload()
    # the persistent chain runs gathers and plain GEMMs: plan without gather-fused links
    assert not _exec.FUSE_A
    _fused_chain_cases(T, w)


def _fused_chain_cases(T, w):
    from tenet import _exec
    from tenet.program import heff2_program

    for ops4, aa in (((T["fl"], T["w1"], T["w2"], T["fr"]), T["aa"]), (w[:4], w[4])):
        prog = heff2_program(*ops4, aa.structure, defer=False)
        assert prog.fused is not None and len(prog.fused) == 1
        default_prog = heff2_program(*ops4, aa.structure, defer=True)
        assert default_prog.fused is None
        y_default = torch.full_like(prog.y_slot, float("nan"))
        default_prog.run(aa.arena, y_default)
        outs = [y_default]
        default = _exec.FUSE
        for fuse in (True, False, True, True):
            _exec.FUSE = fuse
            try:
                y = torch.full_like(prog.y_slot, float("nan"))
                prog.run(aa.arena, y)
                torch.cuda.synchronize()
                outs.append(y)
            finally:
                _exec.FUSE = default
        for y in outs[1:]:
            assert torch.equal(y, outs[0])
        assert int(prog.barrier[0].item()) == 0


def test_save_load_round_trip_on_the_device(tmp_path):
    """``tenet.save`` / ``tenet.load`` and ``MPS.save`` / ``MPS.load`` through the device."""
    import tenet
    from tenet.structure import GradedSpace
    from tenet.symmetry import SU2

    m = json.loads((Path(__file__).resolve().parent / "golden" / "heff.json").read_text())
    h = np.load(Path(__file__).resolve().parent / "golden" / "heff.npz")
    t = load(h, m["aa"])
    tenet.save(t, tmp_path / "aa.npz")
    back = tenet.load(tmp_path / "aa.npz")
    assert back.structure == t.structure
    assert torch.equal(back.arena, t.arena)
    L = 6
    phys = GradedSpace.new(SU2, {SU2.sector(1): 1})
    bonds = [GradedSpace.new(SU2, {SU2.sector(j): 1 for j in range(i % 2, min(i, L - i) + 1, 2)})
             for i in range(L + 1)]
    psi = network.MPS.random(phys, bonds, seed=2).canonize_(0)
    psi.save(tmp_path / "psi")
    psi2 = network.MPS.load(tmp_path / "psi")
    assert psi2.center == psi.center == 0
    for n in range(L):
        assert torch.equal(psi2[n].arena, psi[n].arena)


def test_host_copies_refuse_pageable_memory():
    """``tnb_copy_f64`` and ``tnb_mapped_address`` reach host memory only through pinned
    buffers' mapped addresses: a pageable buffer is refused on the host, before any
    launch, with the library's error status; pinned and device buffers work."""
    import ctypes

    lib = _lib.load()
    n = 1000
    pageable = np.arange(n, dtype=np.float64)
    dev = torch.zeros(n, dtype=torch.float64, device="cuda")
    pinned = torch.arange(n, dtype=torch.float64).pin_memory()
    s = torch.cuda.current_stream().cuda_stream
    assert lib.tnb_copy_f64(n, pageable.ctypes.data, dev.data_ptr(), s) != 0
    assert b"pinned" in lib.tnb_last_error()
    out = ctypes.c_void_p()
    assert lib.tnb_mapped_address(pageable.ctypes.data, ctypes.byref(out)) != 0
    assert lib.tnb_copy_f64(n, pinned.data_ptr(), dev.data_ptr(), s) == 0
    back = torch.zeros(n, dtype=torch.float64).pin_memory()
    assert lib.tnb_copy_f64(n - 1, dev.data_ptr() + 8, back.data_ptr(), s) == 0  # unaligned
    torch.cuda.synchronize()
    assert torch.equal(dev.cpu(), pinned)
    assert torch.equal(back[:n - 1], pinned[1:])
    assert lib.tnb_mapped_address(dev.data_ptr(), ctypes.byref(out)) == 0
    assert out.value == dev.data_ptr()


def test_chain_direct_gathers_are_bit_identical():
    """With ``CHAIN_DIRECT_GATHER`` on, a compiled matvec records its gathers in the
    per-chunk-row form (``tnb_seq_add_gather_direct``) when every segment has rank <= 4:
    the same bits as the
    chunk-map recording, through the graph and the device Lanczos, on the bench's three
    bonds; the one-launch chain still builds from a chunk-map recording."""
    import bench
    from tenet import _exec
    from tenet import program as _program
    from tenet.program import GraphMatvec, heff2_folded_program

    for bond in (bench.BOND, *bench.WORKLOADS.values()):
        fl, w1, w2, fr, aa = bench.build_workload(seed=5, bond=bond)
        lf, rf = network.fold_left(fl, w1), network.fold_right(w2, fr)
        outs = []
        for direct in (False, True):
            _exec.CHAIN_DIRECT_GATHER = direct
            _program._HEFF_TABLES.clear()
            try:
                prog = heff2_folded_program(lf, rf, aa.structure)
                y = GraphMatvec(prog)(aa).numpy_arena()
                e, v = network.DeviceLanczos(prog, 12).solve(aa)
                outs.append((y, e, v.numpy_arena(), prog.fused is not None))
            finally:
                _exec.CHAIN_DIRECT_GATHER = False
                _program._HEFF_TABLES.clear()
        (y0, e0, v0, f0), (y1, e1, v1, f1) = outs
        assert np.array_equal(y0, y1) and e0 == e1 and np.array_equal(v0, v1)
        assert f0 == f1
    torch.cuda.synchronize()
    assert _lib.device_error(0) == 0
