"""Batched U(1) x U(1) x fZ2 environment updates on the device, against the oracle's fZ2
update on coarsened tensors (``tests/_coarsen.py``), the unbatched device path, and, in
reduced precision, the FP64 batch."""

import numpy as np
import pytest
import torch

import oracle.tenet_oracle as O
from _coarsen import coarsen as _coarsen
from _coarsen import rel
from tenet import _lib, batch, network, ops

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _device_error_clear():
    yield
    torch.cuda.synchronize()
    assert _lib.device_error(0) == 0, "a kernel raised the device error word"


def coarsen(t):
    return _coarsen(t.structure, t.numpy_arena())


def test_batched_product_env_update_matches_oracle_and_unbatched():
    import bench

    n = 3
    F, A, W = bench.config3_batch(n, seed=7, lam=2.5, max_deg=4)
    out = batch.env_update_last(F, A, W)
    assert out.arena.shape[0] == n
    for k in range(n):
        got = out[k]
        want = O.env_update_last(coarsen(F[k]), coarsen(A[k]), coarsen(W[k]))
        c = coarsen(got)
        assert c.structure == want.structure
        assert rel(c.arena(), want.arena()) <= 1e-12
        # the unbatched device path on the same member
        one = network.env_update_last(F[k], A[k], W[k])
        assert one.structure == got.structure
        assert rel(got.numpy_arena(), one.numpy_arena()) <= 1e-13


@pytest.mark.parametrize("precision,tol", [("3xbf16", 1e-4), ("tf32", 1e-2)])
def test_batched_product_env_update_in_reduced_precision(precision, tol):
    import bench

    F, A, W = bench.config3_batch(4, seed=3, lam=6.0, max_deg=16)
    exact = batch.env_update_last(F, A, W).arena.cpu().numpy()
    with ops.precision(precision, 0):
        got = batch.env_update_last(F, A, W).arena.cpu().numpy()
    for k in range(4):
        assert rel(got[k], exact[k]) <= tol


def test_autotuned_tiles_compute_the_same_products():
    """The autotuner only chooses among tile kinds that compute the same products: the
    tuned batch agrees with the heuristic one to rounding."""
    import bench

    F, A, W = bench.config3_batch(4, seed=5, lam=6.0, max_deg=16)
    batch.AUTOTUNE = False
    try:
        ref = batch.env_update_last(F, A, W).arena.cpu().numpy()
    finally:
        batch.AUTOTUNE = True
    got = batch.env_update_last(F, A, W).arena.cpu().numpy()
    assert rel(got, ref) <= 1e-13


def test_batched_heff2_matches_each_member():
    """n two-site matvecs of the bench workload's structures (own environments and
    vectors, shared MPO) in one batch: each member equals ``network.heff2`` on it."""
    import bench

    n = 3
    members = [bench.build_workload(seed=10 * k) for k in range(n)]
    fl, w1, w2, fr, aa = (batch.TensorBatch.stack([m[i] for m in members]) for i in range(5))
    w1 = batch.TensorBatch.broadcast(members[0][1], n)
    w2 = batch.TensorBatch.broadcast(members[0][2], n)
    out = batch.heff2(fl, w1, w2, fr, aa)
    compiled = batch.BatchedHeff2(fl, w1, w2, fr, aa.structure)(aa)
    # the MPO links' products computed by the gathers that read them: the same bits
    deferred = batch.BatchedHeff2(fl, w1, w2, fr, aa.structure, defer=True)
    assert sum(bl.deferred for bl in deferred.links) == 2
    assert torch.equal(deferred(aa).arena, compiled.arena)
    for k, (f, _, _, r, a) in enumerate(members):
        want = network.heff2(f, members[0][1], members[0][2], r, a)
        assert out.structure == want.structure == compiled.structure
        assert rel(out[k].numpy_arena(), want.numpy_arena()) <= 1e-13
        assert rel(compiled[k].numpy_arena(), want.numpy_arena()) <= 1e-13


def test_per_chunk_row_gathers_are_bit_identical():
    """``tnb_block_gather_direct`` (a row per chunk, one-term segments' terms inline) and
    ``tnb_grouped_gemm_f64_rows`` (a row per tile) against ``tnb_block_gather`` and
    ``tnb_grouped_gemm_f64`` on the same tables: a U(1) x U(1) x fZ2 environment-update
    batch with every table forced onto the row forms (size-rule and autotuned tile kinds,
    split-K included) and an SU(2) braid's multi-term table -- the same bits, and no bounds
    error."""
    import bench
    from tenet import _exec
    from tenet.structure import layout

    F, A, W = bench.config3_batch(8)
    outs = []
    # never, then every gather from its chunk rows and every FP64 GEMM from its tile rows
    for least in (10 ** 9, 0):
        old = (_exec.DIRECT_MIN_CHUNKS, _exec.DIRECT_MIN_TILES)
        _exec.DIRECT_MIN_CHUNKS = _exec.DIRECT_MIN_TILES = least
        try:
            for autotune in (False, True):  # the size rule's kinds, then the tuned ones
                batch.AUTOTUNE = autotune
                outs.append(batch.env_update_last(F, A, W).arena.cpu().numpy())
        finally:
            _exec.DIRECT_MIN_CHUNKS, _exec.DIRECT_MIN_TILES = old
            batch.AUTOTUNE = True
    assert np.array_equal(outs[0], outs[2]) and np.array_equal(outs[1], outs[3])

    fl, w1, w2, fr, aa = bench.build_workload(seed=3, bond=bench.WORKLOADS["L64_cutoff1e-14_mid_bond"])
    # swapping the two physical legs is an F R F move: segments of several terms
    dst, table = ops._map_exec(aa.structure, "t", (0, 2, 1, 3), None)
    assert np.any(table.seg[:, 4] - table.seg[:, 3] > 1)
    res = []
    for min_chunks in (10 ** 9, 0):
        _exec.DIRECT_MIN_CHUNKS, old = min_chunks, _exec.DIRECT_MIN_CHUNKS
        try:
            out = torch.full((layout(dst).size,), np.nan, dtype=torch.float64, device="cuda")
            table.run(aa.arena, out)
            res.append([out.cpu().numpy()])
        finally:
            _exec.DIRECT_MIN_CHUNKS = old
    torch.cuda.synchronize()
    assert _lib.device_error(0) == 0
    for a, b in zip(*res):
        assert np.array_equal(a, b, equal_nan=True)
