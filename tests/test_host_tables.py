"""Host planner and descriptor tables against the reference's golden vectors, on CPU.

The planner must reproduce the reference's block keys exactly; its gather and grouped-
GEMM tables, executed by a NumPy emulation of the kernels' documented semantics
(``tests/_emulate.py``), must reproduce the reference's results.  No GPU is needed.
"""

import json

import numpy as np
import pytest

import _emulate
from tenet import _exec, ops
from tenet.plan import repartition_plan, transpose_plan
from tenet.structure import IN, OUT, GradedSpace, Leg, TensorStructure, layout
from tenet._exec import gather_rows, make_gather
from tenet.symmetry import SU2, U1, Z2, fZ2

PROV = {"U1": U1, "Z2": Z2, "fZ2": fZ2, "SU2": SU2}


def structure_from_json(legs):
    p = PROV[legs[0]["provider"]]
    return TensorStructure(tuple(
        Leg(GradedSpace.new(p, {p.sector(a): m for a, m in leg["sectors"]}),
            OUT if leg["side"] == "out" else IN, bool(leg["dual"])) for leg in legs))


def keys_from_json(keys):
    t = lambda x: (tuple(x[0]), tuple(x[1]), x[2])  # noqa: E731
    return tuple((t(o), t(i)) for o, i in keys)


def _load(arrays, d):
    s = structure_from_json(d["legs"])
    assert s.keys == keys_from_json(d["keys"]), "block keys differ from the reference"
    return s, np.array(arrays[d["arena"]], dtype=np.float64)


def run_map(src_s, arena, plan):
    dst, perm, terms = plan
    table = make_gather(gather_rows(src_s, "arena", dst, "arena", perm, terms))
    out = np.full(layout(dst).size, np.nan)
    _emulate.gather(table, arena, out)
    return dst, out


def run_tensordot(sa, a, sb, b, axes, out_axes=None):
    ex = ops.contraction_exec(sa, sb, ops._validated_axes(sa, sb, axes), "f64", None, out_axes)
    ap, bp, cp = np.full(ex.a_mat, np.nan), np.full(ex.b_mat, np.nan), np.full(ex.c_mat, np.nan)
    _emulate.gather(ex.pack, a, ap, b, bp)
    _emulate.gemm(ex.gemm, ap, bp, cp)
    out = np.full(layout(ex.out).size, np.nan)
    _emulate.gather(ex.unpack, cp, out)
    return ex.out, out


def run_einsum(eq, ops_):
    lhs, outl = eq.split("->")
    ta, tb = lhs.split(",")
    (sa, a), (sb, b) = ops_
    shared = [x for x in ta if x in tb]
    axes = (tuple(ta.index(x) for x in shared), tuple(tb.index(x) for x in shared))
    free = [x for x in ta if x not in shared] + [x for x in tb if x not in shared]
    # the product path folds the output transpose into the unpack; the two-step form
    # (unpack, then a transpose) must give the same numbers
    folded = run_tensordot(sa, a, sb, b, axes, tuple(free.index(x) for x in outl))
    s, c = run_tensordot(sa, a, sb, b, axes)
    two_step = run_map(s, c, transpose_plan(s, tuple(free.index(x) for x in outl)))
    assert folded[0] == two_step[0]
    np.testing.assert_allclose(folded[1], two_step[1], rtol=1e-13, atol=1e-14)
    return folded


@pytest.fixture(scope="module")
def cases(golden_dir):
    return json.loads((golden_dir / "cases.json").read_text()), np.load(golden_dir / "cases.npz")


def test_block_keys_match_reference(cases):
    meta, arrays = cases
    n = 0
    for c in meta["cases"]:
        for d in c["operands"] + ([c["output"]] if "output" in c else []):
            _load(arrays, d)
            n += 1
    assert n > 40


def test_tables_reproduce_reference(cases):
    meta, arrays = cases
    done = 0
    for c in meta["cases"]:
        op, a = c["op"], c["args"]
        if op not in ("einsum", "transpose", "repartition", "tensordot"):
            continue
        ins = [_load(arrays, d) for d in c["operands"]]
        es, ex = _load(arrays, c["output"])
        if op == "einsum":
            s, out = run_einsum(a["equation"], ins)
        elif op == "transpose":
            s, out = run_map(ins[0][0], ins[0][1], transpose_plan(ins[0][0], tuple(a["axes"])))
        elif op == "repartition":
            s, out = run_map(ins[0][0], ins[0][1],
                             repartition_plan(ins[0][0], tuple(a["outputs"]), tuple(a["inputs"])))
        else:
            s, out = run_tensordot(ins[0][0], ins[0][1], ins[1][0], ins[1][1], a["axes"])
        assert s == es, c["name"]
        assert not np.isnan(out).any(), c["name"]
        np.testing.assert_allclose(out, ex, rtol=1e-12, atol=1e-12 * np.abs(ex).max(),
                                   err_msg=c["name"])
        done += 1
    assert done >= 15


def test_heff2_tables_reproduce_reference(golden_dir):
    m = json.loads((golden_dir / "heff.json").read_text())
    h = np.load(golden_dir / "heff.npz")
    T = {k: _load(h, m[k]) for k in ("aa", "fl", "fr", "w1", "w2", "heff_aa")}

    def composed(eq, A, B, bend):
        lhs, out = eq.split("->")
        ta, tb = lhs.split(",")

        def bent(t, term):
            s, arr = t
            flip = set(bend)
            outs = tuple(i for i, ch in enumerate(term) if (s.legs[i].side is OUT) != (ch in flip))
            ins = tuple(i for i in range(len(term)) if i not in outs)
            return run_map(s, arr, repartition_plan(s, outs, ins)), "".join(term[i] for i in (*outs, *ins))

        A, ta = bent(A, ta)
        B, tb = bent(B, tb)
        return run_einsum(f"{ta},{tb}->{out}", [A, B])

    t = run_einsum("apqr,rys->apqys", [T["aa"], T["fr"]])
    t = composed("apqys,mQqy->apQms", t, T["w2"], "q")
    t = composed("apQms,xPpm->aPQxs", t, T["w1"], "p")
    s, out = composed("aPQxs,axB->BPQs", t, T["fl"], "a")
    es, ex = T["heff_aa"]
    assert s == es
    np.testing.assert_allclose(out, ex, rtol=1e-12, atol=1e-12 * np.abs(ex).max())


def test_config1_plan_sizes(golden_dir):
    g = json.loads((golden_dir / "config1.json").read_text())
    V = GradedSpace.new(U1, {U1.sector(q): d for q, d in g["degeneracies"]})
    sa = TensorStructure((Leg(V, OUT),) * 4)
    sb = TensorStructure((Leg(V, IN), Leg(V, IN), Leg(V, OUT), Leg(V, OUT)))
    ex = ops.contraction_exec(sa, sb, ((2, 3), (0, 1)))
    assert ex.out.keys == keys_from_json(g["keys"])
    assert layout(sa).size == 387756 and ex.gemm.n_gemm == 13
    assert ex.flops == 215_736_784 or abs(ex.flops - 2.157e8) / 2.157e8 < 1e-3


@pytest.mark.parametrize("defer", [False, True])
def test_heff2_chain_program_reproduces_reference(golden_dir, defer):
    """The compiled chain (5 gathers + 4 GEMMs, fixed operands pre-packed) on CPU, with
    and without the MPO links' products computed by the gathers that read them."""
    from types import SimpleNamespace

    from tenet.program import heff2_program

    m = json.loads((golden_dir / "heff.json").read_text())
    h = np.load(golden_dir / "heff.npz")
    T = {k: _load(h, m[k]) for k in ("aa", "fl", "fr", "w1", "w2", "heff_aa")}
    ops_ = {k: SimpleNamespace(structure=T[k][0]) for k in ("fl", "w1", "w2", "fr")}
    prog = heff2_program(ops_["fl"], ops_["w1"], ops_["w2"], ops_["fr"], T["aa"][0],
                         allocate=False, defer=defer)
    # the first link's A gather permutes whole rows only: its products read the input;
    # the two MPO links' skinny products are computed by the gathers that read them
    assert [lk.a_direct for lk in prog.links] == [True, False, False, False]
    assert [lk.deferred for lk in prog.links] == [False, defer, defer, False]
    assert not any(lk.ga is not None for lk in prog.links)  # gather fusion is off by default
    assert prog.launches == (6 if defer else 8)
    src, pending = T["aa"][1], None
    for lk in prog.links:
        name = next(k for k in ("fl", "w1", "w2", "fr") if ops_[k] is lk.b_tensor)
        bbuf = np.full(lk.b_size, np.nan)
        _emulate.gather(lk.b_gather, T[name][1], bbuf)
        cbuf = np.full(lk.c_size, np.nan)
        if lk.a_direct:
            abuf = src
        else:
            abuf = np.full(lk.a_size, np.nan)
            if isinstance(lk.a_gather, _exec.ProductGather):
                _emulate.gather_product(lk.a_gather, *pending, abuf)
            else:
                _emulate.gather(lk.a_gather, src, abuf)
        if lk.deferred:
            pending = (abuf, bbuf)
        else:
            _emulate.gemm(lk.gemm, abuf, bbuf, cbuf)
        src = cbuf
    out = np.full(layout(prog.out_struct).size, np.nan)
    if isinstance(prog.out_gather, _exec.ProductGather):
        _emulate.gather_product(prog.out_gather, *pending, out)
    else:
        _emulate.gather(prog.out_gather, src, out)
    es, ex = T["heff_aa"]
    assert prog.out_struct == es
    np.testing.assert_allclose(out, ex, rtol=1e-12, atol=1e-12 * np.abs(ex).max())


def _compose_spec(terms, following):
    by_src: dict = {}
    for s, d, c in following:
        by_src.setdefault(s, []).append((d, c))
    merged: dict = {}
    for s, m, c in terms:
        for d, o in by_src.get(m, ()):
            merged[(s, d)] = merged.get((s, d), 0.0) + c * o
    return [(s, d, c) for (s, d), c in merged.items()]


def _normalise_spec(dims, dstr, rstr, cstr):
    order = sorted(range(len(dims)), key=lambda k: (-dstr[k], -cstr[k], -rstr[k]))
    out = []
    for k in order:
        if dims[k] == 1:
            continue
        d, a, b, c = dims[k], dstr[k], rstr[k], cstr[k]
        if out and out[-1][1] == a * d and out[-1][2] == b * d and out[-1][3] == c * d:
            out[-1] = (out[-1][0] * d, a, b, c)
            continue
        out.append((d, a, b, c))
    return out or [(1, 1, 0, 0)]


def test_native_compose_matches_the_sparse_product_rule():
    from tenet.plan import compose_terms

    rng = np.random.default_rng(7)
    for trial in range(40):
        na, nb, nm = rng.integers(0, 60), rng.integers(0, 60), rng.integers(1, 12)
        a = [(int(rng.integers(0, 20)), int(rng.integers(0, nm)), float(rng.standard_normal()))
             for _ in range(na)]
        b = [(int(rng.integers(0, nm)), int(rng.integers(0, 20)), float(rng.choice([1.0, -1.0, 0.5])))
             for _ in range(nb)]
        got = compose_terms(a, b)
        want = np.array(_compose_spec(a, b), dtype=np.float64).reshape(-1, 3)
        assert got.shape == want.shape and np.array_equal(got, want)


def _plan_rows(D, DS, RS, CS, d_off, sizes, tb, te, buf):
    """``tnb_plan_gather_rows`` on host arrays (raises ValueError on a refused row)."""
    from tenet import _lib

    D = np.asarray(D)
    R, nd = D.shape
    rows = np.zeros((R, _exec.SEG_W), np.int64)
    arrs = [np.ascontiguousarray(x, dtype=np.int64) for x in (D, DS, RS, CS, d_off, sizes, tb, te)]
    if _lib.load().tnb_plan_gather_rows(R, nd, *(x.ctypes.data for x in arrs), buf,
                                        rows.ctypes.data) != 0:
        raise ValueError("refused")
    return rows


def test_native_gather_rows_match_the_normalisation_rule():
    rng = np.random.default_rng(3)
    R, nd = 200, 5
    D = rng.integers(1, 4, size=(R, nd))
    DS, RS, CS = (rng.integers(0, 6, size=(R, nd)) for _ in range(3))
    # contiguous runs so that merges happen
    DS[:, -1], DS[:, -2] = 1, D[:, -1]
    CS[:, -1], CS[:, -2] = 1, D[:, -1]
    off, size = rng.integers(0, 1000, R), D.prod(axis=1)
    tb = np.arange(R)
    rows = _plan_rows(D, DS, RS, CS, off, size, tb, tb + 1, 1)
    for r in range(R):
        segs = _normalise_spec(list(D[r]), list(DS[r]), list(RS[r]), list(CS[r]))
        row = rows[r]
        assert tuple(row[:6]) == (off[r], size[r], len(segs), r, r + 1, 1)
        for k, (d, a, b, c) in enumerate(segs):
            assert (row[8 + k], row[16 + k], row[24 + k], row[32 + k]) == (d, a, b, c)
    with pytest.raises(ValueError):
        big = np.full((1, 9), 2)
        primes = np.array([[29, 23, 19, 17, 13, 11, 7, 5, 3]])  # no two dims merge
        _plan_rows(big, primes, big * 0, big * 0, [0], [512], [0], [0], 0)


def test_native_gather_table_matches_the_grouping_rule():
    """``tnb_plan_gather_table``: kept destination blocks' terms grouped by block in block
    order (given order inside a group), one row each with the first term's source strides
    permuted, then a zero-writing row per kept block without terms; term outputs in the
    grouped order."""
    import ctypes

    from tenet import _lib

    rng = np.random.default_rng(11)
    for trial in range(30):
        nd = int(rng.integers(1, 5))
        n_src, n_dst, nt = int(rng.integers(1, 9)), int(rng.integers(1, 9)), int(rng.integers(0, 25))
        s_off, s_ld = rng.integers(0, 500, n_src), rng.integers(0, 9, n_src)
        s_rs, s_cs = rng.integers(0, 5, (n_src, nd)), rng.integers(0, 5, (n_src, nd))
        d_off, d_str = rng.integers(0, 500, n_dst), rng.integers(0, 7, (n_dst, nd))
        d_shape = rng.integers(1, 4, (n_dst, nd))
        d_size = d_shape.prod(axis=1)
        keep = (rng.random(n_dst) < 0.8).astype(np.uint8)
        perm = rng.permutation(nd)
        ts, td = rng.integers(0, n_src, nt), rng.integers(0, n_dst, nt)
        tc = rng.standard_normal(nt)
        rows = np.zeros((n_dst, _exec.SEG_W), np.int64)
        o_src, o_ld, o_cf, counts = (np.zeros(nt, np.int64), np.zeros(nt, np.int64),
                                     np.zeros(nt), np.zeros(2, np.int64))
        arrs = [np.ascontiguousarray(x, dtype=np.int64)
                for x in (ts, td, s_off, s_ld, s_rs, s_cs, d_off, d_str, d_shape, d_size, perm)]
        st = _lib.load().tnb_plan_gather_table(
            nt, arrs[0].ctypes.data, arrs[1].ctypes.data, tc.ctypes.data, n_src,
            *(a.ctypes.data for a in arrs[2:6]), n_dst, *(a.ctypes.data for a in arrs[6:10]),
            keep.ctypes.data, nd, arrs[10].ctypes.data, 0, rows.ctypes.data, o_src.ctypes.data,
            o_cf.ctypes.data, o_ld.ctypes.data, counts.ctypes.data)
        assert st == 0
        sel = sorted((t for t in range(nt) if keep[td[t]]), key=lambda t: td[t])
        assert counts[1] == len(sel)
        assert np.array_equal(o_src[:len(sel)], s_off[ts[sel]])
        assert np.array_equal(o_ld[:len(sel)], s_ld[ts[sel]])
        assert np.array_equal(o_cf[:len(sel)], tc[sel])
        want, q = [], 0
        while q < len(sel):
            j, e = td[sel[q]], q
            while e < len(sel) and td[sel[e]] == j:
                e += 1
            i0 = ts[sel[q]]
            want.append((j, s_rs[i0][perm], s_cs[i0][perm], q, e))
            q = e
        covered = set(td.tolist())
        want += [(j, np.zeros(nd, int), np.zeros(nd, int), len(sel), len(sel))
                 for j in range(n_dst) if keep[j] and j not in covered]
        assert counts[0] == len(want)
        for row, (j, rs, cs, tb, te) in zip(rows, want):
            segs = _normalise_spec(list(d_shape[j]), list(d_str[j]), list(rs), list(cs))
            assert tuple(row[:5]) == (d_off[j], d_size[j], len(segs), tb, te)
            for k, (d, a, b, c) in enumerate(segs):
                assert (row[8 + k], row[16 + k], row[24 + k], row[32 + k]) == (d, a, b, c)
        # an out-of-range block index is refused
        bad = arrs[1].copy()
        if nt:
            bad[0] = n_dst
            assert _lib.load().tnb_plan_gather_table(
                nt, arrs[0].ctypes.data, bad.ctypes.data, tc.ctypes.data, n_src,
                *(a.ctypes.data for a in arrs[2:6]), n_dst, *(a.ctypes.data for a in arrs[6:10]),
                keep.ctypes.data, nd, arrs[10].ctypes.data, 0, rows.ctypes.data,
                o_src.ctypes.data, o_cf.ctypes.data, o_ld.ctypes.data, counts.ctypes.data) != 0


def _seg(dst_off, dims, dstr, rstr, cstr, t0, t1):
    row = np.zeros(_exec.SEG_W, np.int64)
    rank = len(dims)
    row[0], row[1], row[2], row[3], row[4] = dst_off, int(np.prod(dims)), rank, t0, t1
    row[8:8 + rank], row[16:16 + rank] = dims, dstr
    row[24:24 + rank], row[32:32 + rank] = rstr, cstr
    return row


def test_product_gather_plans_windows_and_refuses_the_rest():
    """``product_gather`` maps each term of a gather over a product's C arena to its
    product row and first (row, column); computing the elements from A and B (the
    kernel's semantics, emulated) gives what the gather gives over the materialised C.
    It refuses long K, split-K and tensor-core tables, and windows that leave a block."""
    prods = [(5, 3, 2, 0, 2, 0, 3, 0, 3), (4, 2, 3, 10, 3, 6, 2, 15, 2)]
    table = _exec.make_gemm(prods, _exec.TILE_SKINNY)
    rng = np.random.default_rng(3)
    a, b = rng.standard_normal(22), rng.standard_normal(12)
    # one destination block, the sum of a 3 x 2 window of product 0 (rows 1-3, columns
    # 1-2) and a 3 x 2 window of product 1 (rows 0-2), transposed into the destination
    rows = np.array([_seg(0, (3, 2), (1, 3), (1, 0), (0, 1), 0, 2)])
    g = make_gather((rows, np.array([4, 15]), np.array([0.5, -2.0]), np.array([3, 2])))
    pg = _exec.product_gather(g, table)
    assert pg is not None
    assert pg.tprod.tolist() == [0, 1] and pg.tsrc.tolist() == [1, 0] and pg.tld.tolist() == [1, 0]
    c = np.full(23, np.nan)
    _emulate.gemm(table, a, b, c)
    want, got = np.full(6, np.nan), np.full(6, np.nan)
    _emulate.gather(g, c, want)
    _emulate.gather_product(pg, a, b, got)
    np.testing.assert_allclose(got, want, rtol=1e-14, atol=1e-14)
    # a contiguous run across rows of product 1 is not a (row, column) window
    run = make_gather((np.array([_seg(0, (4,), (1,), (0,), (1,), 0, 1)]), np.array([17]),
                       np.array([1.0]), np.array([0])))
    assert _exec.product_gather(run, table) is None
    # a window reaching past its block's last row
    tall = make_gather((np.array([_seg(0, (3, 2), (1, 3), (1, 0), (0, 1), 0, 1)]),
                        np.array([15 + 2 * 2]), np.array([1.0]), np.array([2])))
    assert _exec.product_gather(tall, table) is None
    # long K, tensor-core and split-K tables
    assert _exec.product_gather(g, _exec.make_gemm(
        [(5, 3, 5, 0, 5, 0, 3, 0, 3), (4, 2, 3, 25, 3, 15, 2, 15, 2)], _exec.TILE_SKINNY)) is None
    assert _exec.product_gather(g, _exec.make_gemm(prods, _exec.TILE_TC_3XBF16)) is None
    split = _exec.make_gemm(prods, _exec.TILE_SKINNY)
    split.table = split.table.copy()
    split.table[0, 12] = 2
    assert _exec.product_gather(g, split) is None


def test_graph_matvec_refuses_an_unknown_host_copy_mode():
    """``GraphMatvec(host_copy=...)`` is checked before anything touches the device."""
    from tenet.program import GraphMatvec

    with pytest.raises(ValueError, match="host_copy"):
        GraphMatvec(None, host_io=True, host_copy="zero-copy")


def test_su2_invariant_two_site_operator_coefficients():
    """``T = a S.S + b 1`` read off the two reduced values of an invariant two-site operator
    (what ``MPO.from_terms`` splits); other leg shapes are refused."""
    from tenet.network import su2_invariant_coefficients
    from tenet.structure import IN, OUT, GradedSpace, Leg, TensorStructure
    from tenet.symmetry import SU2

    phys = GradedSpace.new(SU2, {SU2.sector(1): 1})
    s = TensorStructure((Leg(phys, OUT), Leg(phys, OUT), Leg(phys, IN), Leg(phys, IN)))
    ss = np.array([-0.75 if key[0][2] == 0 else 0.25 for key in s.keys])
    assert su2_invariant_coefficients(s, ss) == (1.0, 0.0)
    assert su2_invariant_coefficients(s, 2.0 * ss + 1.0) == (2.0, 1.0)
    bad = TensorStructure((Leg(phys, OUT), Leg(phys, IN), Leg(phys, OUT), Leg(phys, IN)))
    with pytest.raises(ValueError, match="invariant"):
        su2_invariant_coefficients(bad, np.zeros(2))


def test_dmrg_record_and_schmidt_change_follow_the_reference():
    """``DMRG_out`` and ``Sweep`` carry the reference's fields and defaults; the Schmidt
    change is the zero-padded worst-bond distance (``network/dmrg.py:545-561``)."""
    from tenet import network

    assert network.DMRG_out._fields == ("sweeps", "energy", "denergy", "max_dSchmidt",
                                        "max_discarded_weight", "history", "schedule", "psi")
    assert network.Sweep() == (64, 1e-14, 0.0, "wavefunction")
    assert network._schmidt_change({}, {0: [1.0]}) == float("inf")
    got = network._schmidt_change({0: [0.8, 0.6], 1: [1.0]}, {0: [0.8], 1: [1.0], 2: [1.0]})
    assert got == pytest.approx(1.0)


def test_gather_csr_reproduces_the_gather_element_by_element():
    """The element-level view of a gather (what the gather-fused GEMM reads its A
    through) gives every destination element the same terms in the same order: summed
    from zero in that order it equals the table's emulation, on every A gather of the
    folded heff2 chain of the bench's bonds."""
    import bench
    from tenet import network  # noqa: F401  (the folded structures come from its einsums)
    from tenet.plan import transpose_plan
    from tenet.program import ChainProgram

    def einsum_s(eq, sa, sb):
        lhs, out = eq.split("->")
        ta, tb = lhs.split(",")
        shared = [x for x in ta if x in tb]
        axes = (tuple(ta.index(x) for x in shared), tuple(tb.index(x) for x in shared))
        ex = ops.contraction_exec(sa, sb, axes)
        free = [x for x in ta if x not in shared] + [x for x in tb if x not in shared]
        return transpose_plan(ex.out, tuple(free.index(x) for x in out))[0]

    class S:
        def __init__(self, st):
            self.structure = st

    for bond in (bench.BOND, bench.WORKLOADS["L64_cutoff1e-14_mid_bond"]):
        fl, w1, w2, fr, aa = bench.workload_structures(bond)
        lf, rf = einsum_s("axB,xPpm->aBPpm", fl, w1), einsum_s("mQqy,rys->mQqrs", w2, fr)
        p = ChainProgram(aa)
        p.einsum("apqr,mQqrs->apmQs", S(rf))
        p.einsum("apmQs,aBPpm->BPQs", S(lf))
        _exec.FUSE_A = True
        try:
            p.finish(False)
        finally:
            _exec.FUSE_A = False
        rng = np.random.default_rng(0)
        srcs = [rng.standard_normal(layout(aa).size), None]
        assert p.links[0].ga is not None
        for lk in p.links:
            assert (lk.ga is not None) == (max(q[2] for q in lk.gemm.products) <= _exec.GA_MAX_K)
            src = srcs[0] if srcs[1] is None else srcs[1]
            want = np.zeros(lk.a_size)
            _emulate.gather(lk.a_gather, src, want)
            ptr, s_idx, cf = _exec.gather_csr(lk.a_gather, lk.a_size)
            got = np.array([sum(cf[t] * src[s_idx[t]] for t in range(ptr[e], ptr[e + 1]))
                            for e in range(lk.a_size)])
            assert np.allclose(got, want, rtol=1e-15, atol=1e-15)
            srcs[1] = rng.standard_normal(lk.c_size)
        if bond == bench.BOND:
            assert p.launches == 3


def test_two_operand_einsum_plan_and_its_refusals():
    """The cached two-operand plan: shared labels contracted in the first operand's order,
    the output order of the free labels; every malformed equation still refused, and
    refused again on a repeat (a refusal is never cached)."""
    from tenet import ops

    axes, perm = ops._pair_plan("apx,xy->apy", 3, 2)
    assert axes == ((2,), (0,)) and perm == (0, 1, 2)
    axes, perm = ops._pair_plan("apmQs,aBPpm->BPQs", 5, 5)
    assert axes == ((0, 1, 2), (0, 3, 4)) and perm == (2, 3, 0, 1)
    for eq, na, nb in (("ab,bc->ac", 3, 2), ("a.b,bc->ac", 2, 2), ("ab,bb->a", 2, 2),
                       ("ab,bc->a", 2, 2), ("ab,bc,cd->ad", 2, 2)):
        for _ in range(2):
            with pytest.raises(ValueError):
                ops._pair_plan(eq, na, nb)


def test_per_chunk_gather_rows_reproduce_the_gather():
    """``GatherTable.chunk_rows`` (the table of ``tnb_block_gather_direct``): executed chunk
    by chunk from those rows alone -- inline first terms for one-term segments -- the pack
    and unpack tables of a U(1) x U(1) x fZ2 environment-update contraction and of an SU(2)
    two-site contraction give the standard gather's result bit for bit, and every chunk
    row carries its segment's words."""
    import bench
    from tenet.structure import IN, OUT, Leg, TensorStructure, layout

    V, M, Pp = bench.config3_spaces(1000, 24.0, 256)
    sf = TensorStructure((Leg(V, IN), Leg(M, OUT, True), Leg(V, OUT)))
    sa = TensorStructure((Leg(V, OUT), Leg(Pp, OUT), Leg(V, IN)))
    fl, w1, w2, fr, aa = bench.workload_structures(bench.WORKLOADS["L64_cutoff1e-14_mid_bond"])
    rng = np.random.default_rng(9)
    cases = []
    for x, y, axes in ((sf, sa, ((0,), (0,))), (aa, fr, ((3,), (0,)))):
        ex = ops.contraction_exec(x, y, axes)
        cases.append((ex.pack, (layout(x).size, layout(y).size), (ex.a_mat, ex.b_mat)))
        cases.append((ex.unpack, (ex.c_mat, 0), (layout(ex.out).size, 0)))
    for t, (n0, n1), (d0, d1) in cases:
        rows = t.chunk_rows()
        assert rows.shape == (t.chunks, _exec.CHUNK_ROW_W)
        assert np.array_equal(rows[:, :_exec.SEG_W], t.seg[t.chunk_map])
        srcs = [rng.standard_normal(max(n0, 1)), rng.standard_normal(max(n1, 1))]
        want = [np.full(max(d0, 1), np.nan), np.full(max(d1, 1), np.nan)]
        got = [np.full(max(d0, 1), np.nan), np.full(max(d1, 1), np.nan)]
        two = n1 > 0
        _emulate.gather(t, srcs[0], want[0], srcs[1] if two else None, want[1] if two else None)
        _emulate.gather_direct(rows, t.tsrc, t.tcf, t.tld, srcs[0], got[0],
                               srcs[1] if two else None, got[1] if two else None)
        for w, g in zip(want, got):
            assert np.array_equal(w, g, equal_nan=True)
        # the division constants: floor(n / d) by multiply and shift for every n < 2^31
        mags = rows[:, _exec.CHUNK_ROW_MAGIC:_exec.CHUNK_ROW_MAGIC + 8]
        for d, mag in zip(rows[:, 8:16].reshape(-1).tolist(), mags.reshape(-1).tolist()):
            if d <= 1:
                assert mag == 0
                continue
            mul, shr = mag & 0xFFFFFFFF, mag >> 32
            for n in (0, 1, d - 1, d, 2 ** 31 - 1, *rng.integers(0, 2 ** 31, 8).tolist()):
                assert ((n * mul) >> 32) >> shr == n // d


def test_division_constants_at_the_extremes():
    """``_exec.division_constants`` (the per-chunk rows' multiply-shift constants): for
    extents 2 .. 2^31 - 1, powers of two and their neighbours, floor(n / d) = (n mul) >>
    (32 + shift) for n from 0 to 2^31 - 1, and 0 for extents of 0 or 1."""
    rng = np.random.default_rng(12)
    ds = [2, 3, 5, 7, 25, 1000, 2 ** 31 - 1]
    ds += [2 ** k + o for k in range(2, 31) for o in (-1, 0, 1)]
    mags = _exec.division_constants(np.array([0, 1, *ds], dtype=np.int64))
    assert mags[0] == 0 and mags[1] == 0
    for d, mag in zip(ds, mags[2:].tolist()):
        mul, shr = mag & 0xFFFFFFFF, mag >> 32
        assert 0 < mul < 2 ** 32 and shr == (d - 1).bit_length() - 1
        ns = [0, 1, d - 1, d, d + 1, 2 ** 31 - 1, (2 ** 31 - 1) // d * d - 1,
              *rng.integers(0, 2 ** 31, 16).tolist()]
        for n in ns:
            if 0 <= n < 2 ** 31:
                assert ((n * mul) >> 32) >> shr == n // d, (d, n)
