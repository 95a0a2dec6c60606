"""NumPy emulation of the CUDA library's table-driven kernels, for CPU-only tests.

Each function executes a descriptor table exactly as ``include/tenet_b200.h`` documents
the kernel semantics, so the host planner's tables can be verified on a machine without
a GPU.  This is test infrastructure; the shipped package never runs it.
"""

import numpy as np


def gather(table, src0, dst0, src1=None, dst1=None):
    srcs, dsts = (src0, src1), (dst0, dst1)
    for row in table.seg:
        dst_off, size, rank, t0, t1, buf = (int(x) for x in row[:6])
        dims = [int(x) for x in row[8:8 + rank]]
        dstr, rstr, cstr = (np.array(row[o:o + rank], dtype=np.int64) for o in (16, 24, 32))
        J = np.indices(dims).reshape(rank, -1)
        doff = dst_off + (J * dstr[:, None]).sum(0)
        R = (J * rstr[:, None]).sum(0)
        C = (J * cstr[:, None]).sum(0)
        acc = np.zeros(J.shape[1])
        for t in range(t0, t1):
            o = table.tsrc[t] + table.tld[t] * R + C
            assert o.min() >= 0 and o.max() < srcs[buf].size, "source out of bounds"
            acc = acc + table.tcf[t] * srcs[buf][o]
        assert doff.min() >= 0 and doff.max() < dsts[buf].size, "destination out of bounds"
        dsts[buf][doff] = acc


def gather_product(table, a, b, dst):
    """``tnb_block_gather_product``: the gather of C = A x B over ``table.gemm``; term t
    reads C[tsrc[t] + R, tld[t] + C] of product row ``table.tprod[t]``."""
    rows = table.gemm.table
    for row in table.seg:
        dst_off, size, rank, t0, t1, buf = (int(x) for x in row[:6])
        assert buf == 0, "a product-source gather has one buffer pair"
        dims = [int(x) for x in row[8:8 + rank]]
        dstr, rstr, cstr = (np.array(row[o:o + rank], dtype=np.int64) for o in (16, 24, 32))
        J = np.indices(dims).reshape(rank, -1)
        doff = dst_off + (J * dstr[:, None]).sum(0)
        R = (J * rstr[:, None]).sum(0)
        C = (J * cstr[:, None]).sum(0)
        acc = np.zeros(J.shape[1])
        for t in range(t0, t1):
            M, N, K, ao, lda, bo, ldb = (int(x) for x in rows[table.tprod[t], :7])
            m, n = table.tsrc[t] + R, table.tld[t] + C
            assert m.min() >= 0 and m.max() < M and n.min() >= 0 and n.max() < N, \
                "term reads outside its product"
            v = np.zeros(len(m))
            for k in range(K):
                v = v + a[ao + m * lda + k] * b[bo + k * ldb + n]
            acc = acc + table.tcf[t] * v
        assert doff.min() >= 0 and doff.max() < dst.size, "destination out of bounds"
        dst[doff] = acc


def gemm(table, a, b, c):
    parts = getattr(table, "parts", None)
    if parts is not None:
        for p in parts:
            gemm(p, a, b, c)
        return
    for row in table.table:
        M, N, K, ao, lda, bo, ldb, co, ldc = (int(x) for x in row[:9])
        if K == 0:
            for m in range(M):
                c[co + m * ldc: co + m * ldc + N] = 0.0
            continue
        A = np.lib.stride_tricks.as_strided(a[ao:], (M, K), (lda * 8, 8))
        B = np.lib.stride_tricks.as_strided(b[bo:], (K, N), (ldb * 8, 8))
        out = A @ B
        for m in range(M):
            c[co + m * ldc: co + m * ldc + N] = out[m]


def gather_direct(rows, tsrc, tcf, tld, src0, dst0, src1=None, dst1=None, chunk=1024):
    """``tnb_block_gather_direct`` from its per-chunk rows: each chunk its own slice of its
    segment, a one-term segment's term taken from the row's inline words."""
    srcs, dsts = (src0, src1), (dst0, dst1)
    for k, row in enumerate(rows):
        dst_off, size, rank, t0, t1, buf, first, ce = (int(x) for x in row[:8])
        ce = ce or chunk
        lo, hi = (k - first) * ce, min(size, (k - first + 1) * ce)
        dims = [int(x) for x in row[8:8 + rank]]
        dstr, rstr, cstr = (np.array(row[o:o + rank], dtype=np.int64) for o in (16, 24, 32))
        J = np.indices(dims).reshape(rank, -1)[:, lo:hi]
        doff = dst_off + (J * dstr[:, None]).sum(0)
        R = (J * rstr[:, None]).sum(0)
        C = (J * cstr[:, None]).sum(0)
        if t1 - t0 == 1:
            terms = [(int(row[40]), float(np.int64(row[41]).view(np.float64)), int(row[42]))]
        else:
            terms = [(int(tsrc[t]), float(tcf[t]), int(tld[t])) for t in range(t0, t1)]
        acc = np.zeros(J.shape[1])
        for s, cf, ld in terms:
            o = s + ld * R + C
            acc = acc + cf * srcs[buf][o]
        dsts[buf][doff] = acc
