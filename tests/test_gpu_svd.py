"""The blockwise SVD and the device truncation decision (K4), through the C ABI.

Singular values against NumPy's LAPACK SVD (relative to each sector's largest, 1e-13),
both factors isometric and the product reconstructing the matrix to 1e-13; exactly
rank-deficient sectors (zero rows, zero columns, rank one) still give orthonormal
factors; sectors too large for shared memory take the global work path.  The decision
kernel is compared with the host restatement of the reference's keep rule (``decide``)
on seeded spectra with ties across sectors, in every cutoff mode and both budgets.  The
blockwise LQ is compared element by element with NumPy's LAPACK QR of each transpose (the
reference's gauge), through both work paths, and bit for bit on the one-row sectors of a
multiplicity-one start state."""

import numpy as np
import pytest
import torch

from tenet import _exec, _lib, linalg
from tenet.symmetry import SU2

pytestmark = pytest.mark.gpu
P = _exec.ptr


def _svd_batch(mats, force_global=False):
    lib = _lib.load()
    smax = int(lib.tnb_block_svd_smem_doubles())
    rows, a_parts, uo, so, vo, wo, smem, a_off = [], [], 0, 0, 0, 0, 0, 0
    for a in mats:
        m, n = a.shape
        k = min(m, n)
        need = max(m, n) * k + k * k + 2 * k
        if need <= smax and not force_global:
            w, smem = -1, max(smem, need)
        else:
            w, wo = wo, wo + need
        rows.append((m, n, a_off, uo, so, vo, w, 0))
        a_parts.append(a.ravel())
        a_off += a.size
        uo, so, vo = uo + m * k, so + k, vo + k * n
    dev = "cuda"
    A = torch.tensor(np.concatenate(a_parts) if a_parts else np.zeros(1), device=dev)
    U, S, V = (torch.full((max(1, x),), np.nan, dtype=torch.float64, device=dev)
               for x in (uo, so, vo))
    W = torch.zeros(max(1, wo), dtype=torch.float64, device=dev)
    R = torch.tensor(rows, dtype=torch.int64, device=dev)
    info = torch.full((len(rows),), 7, dtype=torch.int32, device=dev)
    _lib.call("tnb_block_svd", P(R), len(rows), P(A), A.numel(), P(U), U.numel(), P(S),
              S.numel(), P(V), V.numel(), P(W), wo, P(info), smem, _exec.stream_ptr())
    torch.cuda.synchronize()
    assert _lib.device_error(0) == 0
    assert (info == 0).all(), info
    U, S, V = U.cpu().numpy(), S.cpu().numpy(), V.cpu().numpy()
    out = []
    for (m, n, _, uo, so, vo, _, _) in rows:
        k = min(m, n)
        out.append((U[uo:uo + m * k].reshape(m, k), S[so:so + k], V[vo:vo + k * n].reshape(k, n)))
    return out


def _check(a, u, s, vh):
    m, n = a.shape
    k = min(m, n)
    want = np.linalg.svd(a, compute_uv=False)
    top = max(want.max() if want.size else 0.0, 1e-300)
    assert np.all(np.diff(s) <= 0)
    assert np.abs(s - want).max() <= 1e-13 * top
    assert np.abs(u.T @ u - np.eye(k)).max() <= 1e-13
    assert np.abs(vh @ vh.T - np.eye(k)).max() <= 1e-13
    assert np.abs(u @ np.diag(s) @ vh - a).max() <= 1e-13 * max(np.abs(a).max(), 1e-300)


def test_block_svd_shapes_and_paths():
    rng = np.random.default_rng(3)
    shapes = [(1, 1), (1, 5), (5, 1), (7, 3), (3, 7), (22, 22), (30, 50), (64, 64), (100, 40),
              (270, 120)]
    mats = [rng.standard_normal(sh) for sh in shapes]
    for a, (u, s, vh) in zip(mats, _svd_batch(mats)):
        _check(a, u, s, vh)
    # the same sectors through the global work path
    for a, (u, s, vh) in zip(mats[:6], _svd_batch(mats[:6], force_global=True)):
        _check(a, u, s, vh)


def test_block_svd_rank_deficient_and_graded_spectra():
    rng = np.random.default_rng(4)
    zero_cols = rng.standard_normal((12, 8))
    zero_cols[:, [1, 5]] = 0.0
    zero_rows = rng.standard_normal((6, 9))
    zero_rows[[0, 3], :] = 0.0
    rank_one = np.outer(rng.standard_normal(10), rng.standard_normal(7))
    # singular values spread over 14 decades (a converged DMRG bond's spectrum)
    q1, _ = np.linalg.qr(rng.standard_normal((40, 40)))
    q2, _ = np.linalg.qr(rng.standard_normal((40, 40)))
    graded = q1 @ np.diag(10.0 ** -np.linspace(0, 14, 40)) @ q2.T
    mats = [zero_cols, zero_rows, rank_one, np.zeros((4, 3)), graded]
    out = _svd_batch(mats)
    for a, (u, s, vh) in zip(mats[:4], out[:4]):
        _check(a, u, s, vh)
    u, s, vh = out[4]
    want = 10.0 ** -np.linspace(0, 14, 40)
    # high relative accuracy down the spectrum, as far as the input's own rounding allows
    assert np.abs(s - want).max() <= 1e-13
    assert np.all(np.abs(s[:25] - want[:25]) <= 1e-9 * want[:25])


def _lq_batch(mats, force_global=False):
    smax = int(_lib.load().tnb_block_svd_smem_doubles())
    rows, parts, b_off, lo, qo, wo, smem = [], [], 0, 0, 0, 0, 0
    for b in mats:
        mb, nb = b.shape
        k = min(mb, nb)
        need = nb * mb + nb * k + 2 * k
        if need <= smax and not force_global:
            w, smem = -1, max(smem, need)
        else:
            w, wo = wo, wo + need
        rows.append((mb, nb, b_off, lo, qo, w, 0, 0))
        parts.append(b.ravel())
        b_off, lo, qo = b_off + b.size, lo + mb * k, qo + k * nb
    dev = "cuda"
    B = torch.tensor(np.concatenate(parts), device=dev)
    L, Q = (torch.full((max(1, x),), np.nan, dtype=torch.float64, device=dev) for x in (lo, qo))
    W = torch.zeros(max(1, wo), dtype=torch.float64, device=dev)
    R = torch.tensor(rows, dtype=torch.int64, device=dev)
    _lib.call("tnb_block_lq", P(R), len(rows), P(B), B.numel(), P(L), L.numel(), P(Q),
              Q.numel(), P(W), wo, smem, _exec.stream_ptr())
    torch.cuda.synchronize()
    assert _lib.device_error(0) == 0
    L, Q = L.cpu().numpy(), Q.cpu().numpy()
    out = []
    for (mb, nb, _, lo, qo, _, _, _) in rows:
        k = min(mb, nb)
        out.append((L[lo:lo + mb * k].reshape(mb, k), Q[qo:qo + k * nb].reshape(k, nb)))
    return out


def test_block_lq_matches_lapack_gauge():
    rng = np.random.default_rng(5)
    shapes = [(1, 1), (1, 6), (6, 1), (7, 3), (3, 7), (22, 22), (30, 50), (64, 64), (100, 40),
              (40, 100), (200, 180)]
    mats = [rng.standard_normal(sh) for sh in shapes]
    for force in (False, True):
        for b, (lf, qf) in zip(mats, _lq_batch(mats, force_global=force)):
            q, r = np.linalg.qr(b.T)  # LAPACK dgeqrf + dorgqr
            scale = max(np.abs(b).max(), 1e-300)
            assert np.abs(lf - r.T).max() <= 1e-12 * scale, b.shape
            assert np.abs(qf - q.T).max() <= 1e-12, b.shape
            assert np.abs(lf @ qf - b).max() <= 1e-13 * scale


def test_block_lq_one_row_sectors_bit_exact():
    """A 1 x 2 sector (every sector of a start state with one multiplet per bond spin):
    one reflection whose norm is formed as LAPACK's dlapy2 forms it, so L and Q equal
    NumPy's QR of the transpose bit for bit."""
    rng = np.random.default_rng(7)
    mats = [rng.standard_normal((1, 2)) * 10.0 ** rng.uniform(-3, 6) for _ in range(400)]
    for b, (lf, qf) in zip(mats, _lq_batch(mats)):
        q, r = np.linalg.qr(b.T)
        assert np.array_equal(lf, r.T) and np.array_equal(qf, q.T), b


def test_block_lq_rank_deficient():
    """Zero rows or columns and rank one: the factors still reconstruct the block and Q
    stays a right isometry."""
    rng = np.random.default_rng(6)
    zero_rows = rng.standard_normal((9, 12))
    zero_rows[[2, 7], :] = 0.0
    zero_cols = rng.standard_normal((8, 5))
    zero_cols[:, [0, 3]] = 0.0
    rank_one = np.outer(rng.standard_normal(10), rng.standard_normal(7))
    mats = [zero_rows, zero_cols, rank_one, np.zeros((4, 3))]
    for b, (lf, qf) in zip(mats, _lq_batch(mats)):
        k = min(b.shape)
        assert np.abs(qf @ qf.T - np.eye(k)).max() <= 1e-13
        assert np.abs(lf @ qf - b).max() <= 1e-13 * max(np.abs(b).max(), 1.0)
        assert np.all(np.triu(lf, 1) == 0.0)


@pytest.mark.parametrize("mode", ["abs", "rel", "sum2", "rsum2", "sum1", "rsum1"])
@pytest.mark.parametrize("budget", ["dense", "reduced"])
def test_device_decision_matches_the_keep_rule(mode, budget):
    rng = np.random.default_rng(sum(map(ord, mode + budget)))
    labels = [0, 2, 4, 6]
    spectra = {}
    for c in labels:
        x = np.sort(rng.choice(np.array([1.0, 0.5, 0.25, 0.125, 1e-3, 1e-6, 1e-9]),
                               size=rng.integers(1, 12)))[::-1]
        spectra[c] = x * rng.choice([1.0, 1.0, 0.7])  # equal values across sectors: ties
    cut = {"abs": 1e-4, "rel": 1e-4, "sum2": 1e-7, "rsum2": 1e-7, "sum1": 1e-4,
           "rsum1": 1e-4}[mode]
    for max_bond in (None, 9, 25):
        for cutoff in (cut, None):
            if max_bond is None and cutoff is None:
                continue
            spectrum = sorted(((float(x), c, i) for c in labels
                               for i, x in enumerate(spectra[c])),
                              key=lambda e: (-e[0], e[1], e[2]))
            want = linalg.decide(spectrum, SU2, max_bond, cutoff, mode, budget=budget)
            dev = "cuda"
            s = torch.tensor(np.concatenate([spectra[c] for c in labels]), device=dev)
            offs = np.cumsum([0] + [len(spectra[c]) for c in labels])
            sec = torch.tensor([(len(spectra[c]), offs[k], c, 0) for k, c in enumerate(labels)],
                               dtype=torch.int64, device=dev)
            qd = torch.tensor([float(c + 1) for c in labels], dtype=torch.float64, device=dev)
            T = s.numel()
            keep = torch.zeros(len(labels), dtype=torch.int64, device=dev)
            ss = torch.zeros(T, dtype=torch.float64, device=dev)
            sc = torch.zeros(T, dtype=torch.int32, device=dev)
            st = torch.zeros(8, dtype=torch.float64, device=dev)
            _lib.call("tnb_truncate_decide", P(sec), P(qd), len(labels), P(s), T,
                      -1.0 if cutoff is None else cutoff, linalg._MODES[mode],
                      -1.0 if max_bond is None else float(max_bond),
                      0 if budget == "dense" else 1, P(keep), P(ss), P(sc), P(st),
                      _exec.stream_ptr())
            torch.cuda.synchronize()
            got = {c: int(k) for c, k in zip(labels, keep.cpu().numpy()) if k}
            assert got == want.keep, (max_bond, cutoff)
            stats = st.cpu().numpy()
            assert int(stats[0]) == want.reduced_dim
            assert stats[1] == want.dense_dim
            assert stats[2] == pytest.approx(want.discarded_weight, rel=1e-15, abs=1e-300)
            order = [(float(x), labels[k]) for x, k in zip(ss.cpu().numpy(), sc.cpu().numpy())]
            assert order == [(x, c) for x, c, _ in spectrum]


def test_truncations_in_flight_on_two_streams():
    """Two truncations of the same structure launched on two streams before either reads
    its decision back (what the serving loop does across requests): each gets its own
    result, equal to the same truncation run alone."""
    import tenet
    from tenet.structure import IN, OUT, GradedSpace, Leg

    V = GradedSpace.new(SU2, {SU2.sector(0): 6, SU2.sector(2): 5, SU2.sector(4): 3})
    P = GradedSpace.new(SU2, {SU2.sector(1): 1})
    legs = (Leg(V, OUT), Leg(P, OUT), Leg(P, OUT), Leg(V, IN))
    a, b = (tenet.SymmetricTensor.random(legs, seed=s) for s in (21, 22))
    kw = dict(max_bond=20, cutoff=1e-12)
    alone = [linalg.svd_truncated_selected(t, ((0, 1), (2, 3)), **kw) for t in (a, b)]
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    torch.cuda.synchronize()
    with torch.cuda.stream(s1):
        pa = linalg.svd_truncated_launch(a, ((0, 1), (2, 3)), **kw)
    with torch.cuda.stream(s2):
        pb = linalg.svd_truncated_launch(b, ((0, 1), (2, 3)), **kw)
    with torch.cuda.stream(s1):
        ra = linalg.svd_truncated_finish(pa)
    with torch.cuda.stream(s2):
        rb = linalg.svd_truncated_finish(pb)
    torch.cuda.synchronize()
    for got, want in zip((ra, rb), alone):
        assert got[3].keep == want[3].keep and got[4] == want[4]
        for x, y in zip(got[:3], want[:3]):
            assert np.array_equal(x.numpy_arena(), y.numpy_arena())
