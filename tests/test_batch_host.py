"""The U(1) x U(1) x fZ2 provider and batched execution, on the CPU: the planner's tables
for single and batched environment updates, executed by the NumPy emulation of the
kernels, against the oracle's fZ2 update on coarsened tensors (``tests/_coarsen.py``)."""

import numpy as np
import pytest

import _emulate
import oracle.tenet_oracle as O
from _coarsen import coarsen, rel
from tenet import batch, ops
from tenet.structure import IN, OUT, Leg, TensorStructure, layout
from tenet.symmetry import ProductSector as PS
from tenet.symmetry import U1xU1xfZ2 as P


def spaces():
    import bench

    return bench.config3_spaces(7, 2.5, 4)


def structures():
    V, M, Pp = spaces()
    return (TensorStructure((Leg(V, IN), Leg(M, OUT, True), Leg(V, OUT))),
            TensorStructure((Leg(V, OUT), Leg(Pp, OUT), Leg(V, IN))),
            TensorStructure((Leg(M, IN, True), Leg(Pp, OUT), Leg(Pp, IN), Leg(M, OUT, True))))


def test_product_provider_labels_fusion_and_braiding():
    a, b = PS(1, 1, 1), PS(-1, 1, 1)
    assert P.fusion(a, b) == (PS(0, 2, 0),)
    assert P.dual(a) == PS(-1, -1, 1) and P.unit == PS(0, 0, 0)
    assert P.r_symbol(a, b, PS(0, 2, 0)) == -1 and P.r_symbol(a, PS(0, 0, 0), a) == 1
    labs = [P.label(x) for x in sorted([PS(1, -5, 0), PS(0, 0, 1), PS(0, 1, 0), PS(-2, 3, 1)])]
    assert labs == sorted(labs)  # labels order like sectors
    assert all(P.sector(P.label(x)) == x for x in (a, b, PS(-4, 4, 0)))
    with pytest.raises(ValueError):
        PS(0, 0, 2)


def _map(s, kind, x, host, n):
    dst, table = batch._unary(s, kind, x, None, n)
    if table is None:
        return dst, host
    out = np.full(n * layout(dst).size, np.nan)
    _emulate.gather(table, host.reshape(-1), out)
    return dst, out.reshape(n, -1)


def _einsum(eq, sa, a, a_shared, sb, b, b_shared, n):
    (ta, tb), o = ops._parse(eq, 2)
    sh = [x for x in ta if x in tb]
    axes = (tuple(ta.index(x) for x in sh), tuple(tb.index(x) for x in sh))
    free = [x for x in ta if x not in sh] + [x for x in tb if x not in sh]
    bc = batch._contraction(sa, sb, axes, n, a_shared, b_shared, "f64", None,
                            tuple(free.index(x) for x in o))
    ap = np.full(max(1, (1 if bc.a_shared else n) * bc.a_mat), np.nan)
    bp = np.full(max(1, (1 if bc.b_shared else n) * bc.b_mat), np.nan)
    cp = np.full(n * bc.c_mat, np.nan)
    _emulate.gather(bc.pack, a.reshape(-1), ap, b.reshape(-1), bp)
    _emulate.gemm(bc.gemm, ap, bp, cp)
    out = np.full(n * bc.out_size, np.nan)
    _emulate.gather(bc.unpack, cp, out)
    return bc.out, out.reshape(n, -1)


def test_batched_env_update_tables_match_the_oracle_per_member():
    sf, sa, sw = structures()
    n = 3
    rng = np.random.default_rng(0)
    f = np.stack([rng.standard_normal(layout(sf).size) for _ in range(n)])
    a = np.stack([rng.standard_normal(layout(sa).size) for _ in range(n)])
    w = rng.standard_normal(layout(sw).size)
    sbra, bra = _map(sa, "a", None, a, n)
    s1, t1 = _einsum("axB,apr->xBpr", sf, f, False, sa, a, False, n)
    s2, t2 = _einsum("xPpm,xBpr->BrPm", sw, w, True, s1, t1, False, n)  # W shared, on the left
    s3, t3 = _einsum("BPs,BrPm->rms", sbra, bra, False, s2, t2, False, n)
    for k in range(n):
        want = O.env_update_last(coarsen(sf, f[k]), coarsen(sa, a[k]), coarsen(sw, w))
        got = coarsen(s3, t3[k])
        assert got.structure == want.structure
        assert rel(got.arena(), want.arena()) <= 1e-13
