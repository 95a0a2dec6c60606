"""Device execution: plans become descriptor tables, tables drive the CUDA library.

A gather table is one row per destination block (the layout of a row is documented in
``include/tenet_b200.h``).  Source and destination may each be a tensor *arena* (blocks
concatenated in block order, C-contiguous in public axis order) or a packed
*coupled-sector matrix* buffer (map-view lowering, rows = OUT trees, cols = IN trees).
Before a row is emitted its dims are reordered so the innermost dim has the smallest
destination stride (coalesced stores), extent-1 dims are dropped and dims that are
contiguous in both source and destination are merged, so a pure reshape becomes a
rank-1 copy.

Tables are built once per (structure, plan) and cached as device tensors; a call then
costs one ctypes launch per kernel.
"""

from __future__ import annotations

import ctypes
import threading
from dataclasses import dataclass

from contextlib import contextmanager

import numpy as np
import torch

from tenet import _lib
from tenet.structure import TensorStructure, layout, matrix_layout

SEG_W = 40
GEMM_W = 16
#: words of a per-chunk gather row (``tnb_block_gather_direct``): the segment row, its
#: first term inline, a pad word, then its extents' division constants
CHUNK_ROW_W = 56
CHUNK_ROW_MAGIC = 48


def division_constants(dims: np.ndarray) -> np.ndarray:
    """Per extent d >= 2: mul = ceil(2^(31 + l) / d), l = ceil(log2 d), packed as mul | (l
    - 1) << 32 (0 for d <= 1), so that floor(n / d) = (n mul) >> (31 + l) for n < 2^31
    (Granlund and Montgomery, 1994)."""
    out = np.zeros(dims.shape, dtype=np.int64)
    flat, res = dims.reshape(-1), out.reshape(-1)
    for i, d in enumerate(flat.tolist()):
        if d >= 2:
            l = (d - 1).bit_length()
            res[i] = ((1 << (31 + l)) + d - 1) // d | (l - 1) << 32
    return out
CHUNK = 1024
MAX_RANK = 8
TILE_64, TILE_32, TILE_SKINNY, TILE_TC_TF32, TILE_TC_3XBF16, TILE_WIDE = 0, 1, 2, 3, 4, 5
TC_KINDS = {"tf32": TILE_TC_TF32, "3xbf16": TILE_TC_3XBF16}
SKINNY_ROWS, SKINNY_MAX = 256, 16
# tensor-core tiles: 128 x 128 outputs, K slabs of 32; each packed operand slab (one
# 128-row x 32 chunk, every part: BF16 hi + lo, or one TF32) is 16 KB
TC_TILE, TC_BK, TC_SLAB_BYTES = 128, 32, 16384
N_SM = 148


def device() -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("tenet_b200 needs a CUDA device: there is no CPU execution path")
    return torch.device("cuda", torch.cuda.current_device())


def stream_ptr() -> int:
    """The raw ``cudaStream_t`` of the current device's current stream."""
    return torch._C._cuda_getCurrentRawStream(torch._C._cuda_getDevice())


def ptr(t: torch.Tensor | None) -> int:
    return 0 if t is None or t.numel() == 0 else t.data_ptr()


class Seq:
    """A recorded launch sequence (``tnb_seq`` in ``include/tenet_b200.h``): gathers and
    grouped GEMMs recorded once and replayed by one library call, optionally with buffer
    pointers substituted.  The owner keeps every recorded table and buffer alive."""

    def __init__(self) -> None:
        lib = _lib.load()
        h = ctypes.c_void_p()
        _lib.call("tnb_seq_create", ctypes.byref(h))
        self.handle = h.value
        self._destroy = lib.tnb_seq_destroy

    def __del__(self):
        if getattr(self, "handle", None):
            self._destroy(self.handle)
            self.handle = None

    def __len__(self) -> int:
        return int(_lib.load().tnb_seq_length(self.handle))

    def __enter__(self):
        self._prev = recording()
        _TLS.rec = self
        return self

    def __exit__(self, *exc):
        _TLS.rec = self._prev

    def run(self, patch: dict | None = None) -> None:
        """Replay on the current stream; ``patch`` maps recorded buffer addresses to the
        addresses to use instead."""
        if patch:
            n = len(patch)
            src = (ctypes.c_void_p * n)(*patch.keys())
            dst = (ctypes.c_void_p * n)(*patch.values())
            _lib.call("tnb_seq_run", self.handle, n, src, dst, stream_ptr())
        else:
            _lib.call("tnb_seq_run", self.handle, 0, None, None, stream_ptr())


# per host thread: the sequence being recorded, if any (threads of the serving loop record
# their own programs concurrently)
_TLS = threading.local()


def recording() -> Seq | None:
    """The sequence launches are being recorded into on this thread (None: launch)."""
    return getattr(_TLS, "rec", None)

#: Run compiled chains as one persistent launch when every stage fuses.  Off by default:
#: on B200 the stage-by-stage replay (a CUDA graph, programmatic dependent launch) is
#: faster at the sizes measured, because the FP64 tile holds the persistent kernel to one
#: CTA per SM, which starves its latency-bound gather stages.  The fused launch gives
#: bit-identical results and stays available for comparison.
FUSE = False
#: plan a small chain (every stage at most ``CLUSTER_MAX_ITEMS`` work items) to run as one
#: launch on a single thread-block cluster (``tnb_seq_fuse_cluster``).  Off by default:
#: bit-identical, but measured slower than the graph of stage launches on B200 (43 against
#: 22.5 us for the L = 64 mid-bond matvec: each stage's table loads sit on its critical
#: path after every barrier, where the stage launches overlap them with the previous
#: kernel through programmatic dependent launch)
CLUSTER = False
CLUSTER_MAX_ITEMS = 48
CLUSTER_CTAS = 16



class _Staging:
    """A pinned host ring through which plan tables reach the device: a table is packed
    into the next free bytes of the ring and copied asynchronously, so an upload costs a
    host memcpy and one queued copy.  Before the ring wraps, every copy still reading it
    is waited for."""

    def __init__(self, nbytes: int = 64 << 20) -> None:
        self.nbytes = nbytes
        self.buf = None
        self.pos = 0
        self.pending: list = []
        self.lock = threading.Lock()

    def stage(self, packed: np.ndarray):
        with self.lock:
            return self._stage(packed)

    def _stage(self, packed: np.ndarray):
        n = packed.nbytes
        if n > self.nbytes // 4:
            return None
        if self.buf is None:
            self.buf = torch.empty(self.nbytes, dtype=torch.uint8).pin_memory()
            self.host = self.buf.numpy()
        if self.pos + n > self.nbytes:
            for ev in self.pending:
                ev.synchronize()
            self.pending.clear()
            self.pos = 0
        view = self.buf[self.pos:self.pos + n]
        self.host[self.pos:self.pos + n] = packed
        self.pos = -(-(self.pos + n) // 256) * 256
        return view


_STAGING = _Staging()


class _DevArray:
    """One array of an upload as the library's calls take it: a device address and an
    element count (``ptr`` reads both).  The upload's buffer keeps the memory alive."""

    __slots__ = ("_ptr", "_n")

    def __init__(self, address: int, n: int) -> None:
        self._ptr, self._n = address, n

    def data_ptr(self) -> int:
        return self._ptr

    def numel(self) -> int:
        return self._n


class _UploadSlice:
    """A table's share of an upload made for several tables at once."""

    __slots__ = ("up", "lo", "hi")

    def __init__(self, up, lo: int, hi: int) -> None:
        self.up, self.lo, self.hi = up, lo, hi

    def ready(self) -> tuple:
        return self.up.ready()[self.lo:self.hi]


def upload_together(tables) -> None:
    """One upload (one staging copy, one device buffer, one event) for the arrays of every
    table in ``tables`` not yet on the device, instead of one each at its first run."""
    todo, arrays, spans = [], [], []
    for t in tables:
        if t is None or getattr(t, "_dev", 1) is not None:
            continue
        arrs = t.host_arrays()
        todo.append(t)
        spans.append((len(arrays), len(arrays) + len(arrs)))
        arrays.extend(arrs)
    if not todo:
        return
    up = Uploaded(arrays)
    for t, (lo, hi) in zip(todo, spans):
        t._dev = _UploadSlice(up, lo, hi)


class Uploaded:
    """Device copies of host arrays, made on the current stream.  A copy from pageable
    host memory may still be in flight when the call returns, so a kernel on another
    stream waits for the upload's event before first reading them (the serving loop runs
    requests that share plan tables on different streams).  The arrays come back as
    address-and-count holders over one device buffer (tables are only ever handed to
    the library), which spares a torch view per array on every upload."""

    __slots__ = ("arrays", "stream", "event", "buf")

    def __init__(self, host_arrays) -> None:
        # one host->device copy: the arrays packed at 16-byte aligned offsets of one
        # buffer, then typed views into its device copy
        host_arrays = [np.ascontiguousarray(x) for x in host_arrays]
        offs, total = [], 0
        for x in host_arrays:
            offs.append(total)
            total += -(-x.nbytes // 16) * 16
        packed = np.zeros(max(total, 16), dtype=np.uint8)
        for x, o in zip(host_arrays, offs):
            packed[o:o + x.nbytes] = x.reshape(-1).view(np.uint8)
        staged = None if torch.cuda.is_current_stream_capturing() else _STAGING.stage(packed)
        if staged is not None:
            dev_buf = torch.empty(packed.nbytes, dtype=torch.uint8, device=device())
            dev_buf.copy_(staged, non_blocking=True)
        else:
            dev_buf = torch.from_numpy(packed).to(device())
        base = dev_buf.data_ptr()
        self.buf = dev_buf
        self.arrays = tuple(_DevArray(base + o, x.size) for x, o in zip(host_arrays, offs))
        self.stream = stream_ptr()
        self.event = torch.cuda.Event()
        self.event.record()
        if staged is not None:
            _STAGING.pending.append(self.event)

    def ready(self) -> tuple:
        if self.event is not None and stream_ptr() != self.stream \
                and not torch.cuda.is_current_stream_capturing():
            if self.event.query():
                self.event = None
            else:
                torch.cuda.current_stream().wait_event(self.event)
        return self.arrays


class LaunchLog:
    """Optional per-launch record: ``(kind, start event, end event, work)`` for every
    library kernel launched while installed, events on the launching stream.  ``work``
    is algorithmic bytes for gathers and flops for GEMMs."""

    def __init__(self, timed: bool = True) -> None:
        self.timed = timed
        self.records: list = []
        self.count = 0

    def __enter__(self):
        global _LOG
        self._prev, _LOG = _LOG, self
        return self

    def __exit__(self, *exc):
        global _LOG
        _LOG = self._prev

    def begin(self):
        self.count += 1
        if not self.timed:
            return None
        ev = torch.cuda.Event(enable_timing=True)
        ev.record()
        return ev

    def end(self, kind: str, start, work: int) -> None:
        if start is None:
            return
        ev = torch.cuda.Event(enable_timing=True)
        ev.record()
        self.records.append((kind, start, ev, work))

    def summary(self) -> dict:
        torch.cuda.synchronize()
        out: dict = {}
        for kind, a, b, work in self.records:
            d = out.setdefault(kind, {"launches": 0, "ms": 0.0, "work": 0})
            d["launches"] += 1
            d["ms"] += a.elapsed_time(b)
            d["work"] += work
        return out


_LOG: LaunchLog | None = None


# ---------------------------------------------------------------------------------------
# gather tables


def gather_rows(src_s: TensorStructure, src_kind: str, dst_s: TensorStructure, dst_kind: str,
                perm, terms, buf: int = 0, dst_keep=None):
    """Rows + term arrays executing ``dst[j] = sum c * transpose(src[i], perm)``: one row
    per destination block that has terms (in block order, its terms in the order given),
    then one zero-writing row per destination block without any.  ``dst_keep``
    optionally restricts the emitted destination blocks (a boolean mask).  Returns
    ``(rows (R, SEG_W), term sources, term coefficients, term leading dimensions)`` as
    arrays, term ranges relative to this part.  The grouping and the rows are built by
    the library's host planner (``tnb_plan_gather_table``)."""
    sl, dl = layout(src_s), layout(dst_s)
    if src_kind == "matrix":
        sm = matrix_layout(src_s)
        s_off, s_ld, s_rs, s_cs = sm.block_off, sm.block_ld, sm.rstride, sm.cstride
    else:
        s_off, s_ld = sl.offsets, _zeros_like_cached(sl.offsets)
        s_rs, s_cs = _zeros_like_cached(sl.strides), sl.strides
    if dst_kind == "matrix":
        dm = matrix_layout(dst_s)
        d_off = dm.block_off
        d_str = dm.rstride * dm.block_ld[:, None] + dm.cstride
    else:
        d_off, d_str = dl.offsets, dl.strides
    n_dst, nd = dl.shapes.shape
    keep = np.ones(n_dst, np.uint8) if dst_keep is None else np.asarray(dst_keep, np.uint8)
    if len(terms):
        tarr = np.asarray(terms, dtype=np.float64).reshape(-1, 3)
        ts, td, tc = tarr[:, 0].astype(np.int64), tarr[:, 1].astype(np.int64), tarr[:, 2].copy()
    else:
        ts = td = np.zeros(0, np.int64)
        tc = np.zeros(0)
    nt = len(ts)
    c = lambda x, t=np.int64: np.ascontiguousarray(x, dtype=t)  # noqa: E731
    args = [c(s_off), c(s_ld), c(s_rs), c(s_cs), c(d_off), c(d_str), c(dl.shapes), c(dl.sizes)]
    perm = c(perm)
    rows = np.zeros((n_dst, SEG_W), np.int64)
    out_src, out_ld, out_coef = np.zeros(nt, np.int64), np.zeros(nt, np.int64), np.zeros(nt)
    counts = np.zeros(2, np.int64)
    status = _lib.load().tnb_plan_gather_table(
        nt, ts.ctypes.data, td.ctypes.data, tc.ctypes.data, len(s_off), args[0].ctypes.data,
        args[1].ctypes.data, args[2].ctypes.data, args[3].ctypes.data, n_dst,
        args[4].ctypes.data, args[5].ctypes.data, args[6].ctypes.data, args[7].ctypes.data,
        keep.ctypes.data, nd, perm.ctypes.data, buf, rows.ctypes.data, out_src.ctypes.data,
        out_coef.ctypes.data, out_ld.ctypes.data, counts.ctypes.data)
    if status != 0:
        raise ValueError(f"a gather plan with a block of rank above the kernel's {MAX_RANK}, "
                         "or an out-of-range block index")
    R, T = int(counts[0]), int(counts[1])
    return rows[:R], out_src[:T], out_coef[:T], out_ld[:T]


_ZEROS: dict = {}


def _zeros_like_cached(a: np.ndarray) -> np.ndarray:
    """A read-only zero array of ``a``'s shape, shared per shape."""
    z = _ZEROS.get(a.shape)
    if z is None:
        z = np.zeros(a.shape, np.int64)
        z.flags.writeable = False
        _ZEROS[a.shape] = z
    return z


class GatherTable:
    """A gather program: host arrays (inspectable on a CPU-only machine) uploaded to the
    current device on first use."""

    def __init__(self, seg: np.ndarray, tsrc, tcf, tld) -> None:
        self.seg = seg
        self.tsrc = np.asarray(tsrc, dtype=np.int64)
        self.tcf = np.asarray(tcf, dtype=np.float64)
        self.tld = np.asarray(tld, dtype=np.int64)
        self.n_seg = len(seg)
        self.n_term = len(self.tsrc)
        ce = np.where(seg[:, 7] > 0, seg[:, 7], CHUNK) if len(seg) else np.zeros(0, np.int64)
        per = (seg[:, 1] + ce - 1) // ce if len(seg) else np.zeros(0, np.int64)
        self.chunks = int(per.sum()) if len(seg) else 0
        self.elems = int(seg[:, 1].sum()) if len(seg) else 0
        self.term_elems = int((seg[:, 1] * (seg[:, 4] - seg[:, 3])).sum()) if len(seg) else 0
        self.chunk_map = np.repeat(np.arange(len(seg), dtype=np.int32), per)
        self._dev = None
        self._ddev = None

    @property
    def bytes_moved(self) -> int:
        """Algorithmic HBM bytes of one run: every term's source read once, every
        destination element written once."""
        return 8 * (self.elems + self.term_elems)

    def host_arrays(self) -> tuple:
        return (self.seg, self.tsrc, self.tcf, self.tld, self.chunk_map)

    def device_arrays(self):
        if self._dev is None:
            self._dev = Uploaded(self.host_arrays())
        return self._dev.ready()

    @property
    def direct_ok(self) -> bool:
        """Whether ``tnb_block_gather_direct`` takes this table (every segment of rank <=
        4)."""
        return bool(self.n_seg) and int(self.seg[:, 2].max()) <= DIRECT_MAX_RANK

    def chunk_rows(self) -> np.ndarray:
        """The table as one ``CHUNK_ROW_W`` row per chunk: the chunk's segment row, the
        segment's first term (source, coefficient bits, leading dimension) inline, and the
        division constants of its extents."""
        rows = np.zeros((self.chunks, CHUNK_ROW_W), dtype=np.int64)
        if self.chunks:
            own = self.seg[self.chunk_map]
            rows[:, :SEG_W] = own
            has = own[:, 4] > own[:, 3]
            t0 = own[has, 3]
            rows[has, SEG_W] = self.tsrc[t0]
            rows[has, SEG_W + 1] = self.tcf[t0].view(np.int64)
            rows[has, SEG_W + 2] = self.tld[t0]
            mags = division_constants(self.seg[:, 8:8 + 8])
            rows[:, CHUNK_ROW_MAGIC:CHUNK_ROW_MAGIC + 8] = mags[self.chunk_map]
        return rows

    def direct_arrays(self):
        if self._ddev is None:
            self._ddev = Uploaded((self.chunk_rows(), self.tsrc, self.tcf, self.tld))
        return self._ddev.ready()

    def run(self, src0, dst0, src1=None, dst1=None) -> None:
        if self.n_seg == 0:
            return
        rec = recording()
        if rec is not None and CHAIN_DIRECT_GATHER and not _STANDARD[0] and self.direct_ok:
            crows, tsrc, tcf, tld = self.direct_arrays()
            _lib.call("tnb_seq_add_gather_direct", rec.handle, ptr(crows), self.chunks,
                      ptr(tsrc), ptr(tcf), ptr(tld), self.n_term, ptr(src0), src0.numel(),
                      ptr(dst0), dst0.numel(), ptr(src1), 0 if src1 is None else src1.numel(),
                      ptr(dst1), 0 if dst1 is None else dst1.numel())
            return
        if rec is None and DIRECT_GATHER and self.chunks >= DIRECT_MIN_CHUNKS and self.direct_ok:
            crows, tsrc, tcf, tld = self.direct_arrays()
            mark = _LOG.begin() if _LOG is not None else None
            _lib.call("tnb_block_gather_direct", ptr(crows), self.chunks, ptr(tsrc), ptr(tcf),
                      ptr(tld), self.n_term, ptr(src0), src0.numel(), ptr(dst0), dst0.numel(),
                      ptr(src1), 0 if src1 is None else src1.numel(),
                      ptr(dst1), 0 if dst1 is None else dst1.numel(), stream_ptr())
            if _LOG is not None:
                _LOG.end("block_gather", mark, self.bytes_moved)
            return
        seg, tsrc, tcf, tld, cmap = self.device_arrays()
        if rec is not None:
            _lib.call("tnb_seq_add_gather", rec.handle, ptr(seg), self.n_seg, ptr(cmap),
                      self.chunks, ptr(tsrc), ptr(tcf), ptr(tld), self.n_term,
                      ptr(src0), src0.numel(), ptr(dst0), dst0.numel(),
                      ptr(src1), 0 if src1 is None else src1.numel(),
                      ptr(dst1), 0 if dst1 is None else dst1.numel())
            return
        mark = _LOG.begin() if _LOG is not None else None
        _lib.call("tnb_block_gather", ptr(seg), self.n_seg, ptr(cmap), self.chunks, ptr(tsrc),
                  ptr(tcf), ptr(tld), self.n_term,
                  ptr(src0), src0.numel(), ptr(dst0), dst0.numel(),
                  ptr(src1), 0 if src1 is None else src1.numel(),
                  ptr(dst1), 0 if dst1 is None else dst1.numel(), stream_ptr())
        if _LOG is not None:
            _LOG.end("block_gather", mark, self.bytes_moved)


#: run gathers of at least DIRECT_MIN_CHUNKS chunks (more than two waves of resident
#: CTAs, where each CTA's table loads are not hidden behind another kernel) from their
#: per-chunk rows (``tnb_block_gather_direct``): one round of table loads per CTA
DIRECT_GATHER = True
DIRECT_MIN_CHUNKS = 2 * 3 * N_SM + 1
DIRECT_MAX_RANK = 4
#: record the gathers of compiled chains (a matvec's recorded sequence) in the per-chunk-row
#: form whatever their size.  Off by default: the same bits, but a one-wave gather's table
#: wait already overlaps the previous launch (programmatic dependent launch), and with a
#: cold L2 the larger rows cost more than the saved round trips (headline matvec 22.6-25.4
#: against 21.7-22.6 us, L2 flushed; equal with a warm L2)
CHAIN_DIRECT_GATHER = False
_STANDARD = [0]  # > 0 inside standard_gathers()


@contextmanager
def standard_gathers():
    """Record chunk-map gathers only (the one-launch chain kernels take no other form)."""
    _STANDARD[0] += 1
    try:
        yield
    finally:
        _STANDARD[0] -= 1
#: likewise FP64 grouped GEMMs of at least DIRECT_MIN_TILES tiles from one row per tile
#: (``tnb_grouped_gemm_f64_rows``): one table load per tile instead of two dependent ones
DIRECT_GEMM = True
DIRECT_MIN_TILES = 4 * N_SM

#: resident gather CTAs per SM (the kernels' launch bounds): plain, product-source
GATHER_CTAS_PER_SM = 3
PRODUCT_GATHER_CTAS_PER_SM = 2


def chunk_size(sizes, ctas_per_sm: int = GATHER_CTAS_PER_SM) -> int:
    """Elements per gather chunk for a table whose segments hold ``sizes`` elements: the
    largest of 1024, 512, 256 whose chunks still fill one wave of resident CTAs.  Every
    CTA pays a chain of dependent loads (chunk map, row, terms) before its data loads, so
    a small, latency-bound table wants one wave of CTAs with two or four elements per
    thread rather than two waves of one; a big table keeps four elements per thread."""
    sizes = np.asarray(sizes, dtype=np.int64)
    wave = ctas_per_sm * N_SM
    for ce in (CHUNK, CHUNK // 2):
        if int(((sizes + ce - 1) // ce).sum()) >= wave:
            return ce
    return CHUNK // 4


def _chunked(seg: np.ndarray, ctas_per_sm: int = GATHER_CTAS_PER_SM) -> np.ndarray:
    """``seg`` with the chunk size (column 7) and chunk prefix sums (column 6) set."""
    seg = seg.copy()
    if len(seg):
        seg[:, 7] = chunk_size(seg[:, 1], ctas_per_sm)
        per = (seg[:, 1] + seg[:, 7] - 1) // seg[:, 7]
        seg[:, 6] = np.cumsum(per) - per
    return seg


class ProductGather(GatherTable):
    """A gather whose source is the product C = A x B of an FP64 GEMM table with K <= 4
    (an MPO link's products), never materialised: each source element is computed where
    it is read (``tnb_block_gather_product``), so the GEMM launch and the round trip of C
    through memory disappear.  ``base`` is the plain gather over a materialised C; term
    ``t`` reads C[m0[t] + R, n0[t] + C] of product row ``tprod[t]`` (its ``tsrc`` and
    ``tld`` hold m0 and n0).  Built by ``product_gather``."""

    def __init__(self, base: GatherTable, gemm: "GemmTable", tprod, m0, n0) -> None:
        super().__init__(_chunked(base.seg, PRODUCT_GATHER_CTAS_PER_SM), m0, base.tcf, n0)
        self.base, self.gemm = base, gemm
        self.tprod = np.asarray(tprod, dtype=np.int64)

    @property
    def bytes_moved(self) -> int:
        """Algorithmic bytes: every destination element written once and the product's
        operands read once (A is M x K, B is K x N per product row); the re-reads of an A
        row for the N columns and the terms that share it hit in cache."""
        r = self.gemm.table
        return 8 * (self.elems + int((r[:, 0] * r[:, 2] + r[:, 2] * r[:, 1]).sum()))

    def host_arrays(self) -> tuple:
        return (self.seg, self.tsrc, self.tcf, self.tld, self.chunk_map, self.tprod)

    def device_arrays(self):
        if self._dev is None:
            self._dev = Uploaded(self.host_arrays())
        return self._dev.ready()

    def run(self, a, b, dst) -> None:
        """``dst`` = the gather of C = A x B (``a``, ``b``: the product's operand buffers)
        on the current stream."""
        if self.n_seg == 0:
            return
        seg, tsrc, tcf, tld, cmap, tprod = self.device_arrays()
        table, _ = self.gemm.device_tables()
        args = (ptr(seg), self.n_seg, ptr(cmap), self.chunks, ptr(tsrc), ptr(tcf), ptr(tld),
                ptr(tprod), self.n_term, ptr(table), self.gemm.n_gemm, ptr(a), a.numel(),
                ptr(b), b.numel(), ptr(dst), dst.numel())
        rec = recording()
        if rec is not None:
            _lib.call("tnb_seq_add_gather_product", rec.handle, *args)
            return
        mark = _LOG.begin() if _LOG is not None else None
        _lib.call("tnb_block_gather_product", *args, stream_ptr())
        if _LOG is not None:
            _LOG.end("block_gather", mark, self.bytes_moved)


#: longest K of a skinny product that a gather computes where it reads it
PRODUCT_MAX_K = 4


def product_gather(g: GatherTable, part):
    """``g`` (a gather over the C arena of the FP64 GEMM table ``part``) as a
    ``ProductGather``, or None when it cannot be one: ``part`` is a tensor-core or split-K
    table or has a product with K > ``PRODUCT_MAX_K``, a row uses the second buffer pair,
    or a term's window is not a window of one product's M x N block.  Every FP64 kind
    without split-K sums k ascending from zero in one FMA chain, as the product-source
    gather does, so the values are bit-identical.

    Term t reads offsets tsrc + tld R + C with R = sum_d j_d rstride_d and C = sum_d j_d
    cstride_d over the box 0 <= j_d < dims_d.  When tld is the block's ldc and, with
    tsrc - c_off = m0 ldc + n0, every C stays in [-n0, N - n0) and every R in [-m0, M - m0),
    the element is exactly C[m0 + R, n0 + C] of that product; R and C are linear over the
    box, so their extremes follow from the strides' signs."""
    if (g is None or g.n_seg == 0 or part.n_gemm == 0
            or part.kind not in (TILE_64, TILE_32, TILE_SKINNY, TILE_WIDE)):
        return None
    rows, seg = part.table, g.seg
    if np.any(rows[:, 2] > PRODUCT_MAX_K) or np.any(rows[:, 12] > 1) or np.any(seg[:, 5] != 0):
        return None
    if seg[0, 3] != 0 or seg[-1, 4] != g.n_term or np.any(seg[1:, 3] != seg[:-1, 4]):
        return None  # terms are not stored row by row
    owner = np.repeat(np.arange(g.n_seg), seg[:, 4] - seg[:, 3])  # term -> its row
    rk = seg[owner, 2][:, None]
    span = np.where(np.arange(8)[None, :] < rk, np.maximum(seg[owner, 8:16] - 1, 0), 0)
    rs, cs = span * seg[owner, 24:32], span * seg[owner, 32:40]
    r_lo, r_hi = np.minimum(rs, 0).sum(1), np.maximum(rs, 0).sum(1)
    c_lo, c_hi = np.minimum(cs, 0).sum(1), np.maximum(cs, 0).sum(1)
    coff = rows[:, 7]
    order = np.argsort(coff, kind="stable")
    pos = np.searchsorted(coff[order], g.tsrc, side="right") - 1
    if np.any(pos < 0):
        return None
    tprod = order[pos]
    M, N, ldc = rows[tprod, 0], rows[tprod, 1], rows[tprod, 8]
    if np.any(g.tld != ldc) or np.any(ldc <= 0):
        return None
    m0, n0 = np.divmod(g.tsrc - coff[tprod], ldc)
    if (np.any(m0 + r_lo < 0) or np.any(m0 + r_hi >= M)
            or np.any(n0 + c_lo < 0) or np.any(n0 + c_hi >= N)):
        return None
    return ProductGather(g, part, tprod, m0, n0)


def make_gather(*parts) -> GatherTable:
    """Concatenate one or more ``gather_rows`` results into a single table."""
    rows, tsrc, tcf, tld = [], [], [], []
    base = 0
    for r, ts, tc, tl in parts:
        r = np.array(r, dtype=np.int64).reshape(-1, SEG_W)
        r[:, 3:5] += base
        rows.append(r)
        tsrc.append(np.asarray(ts, np.int64))
        tcf.append(np.asarray(tc, np.float64))
        tld.append(np.asarray(tl, np.int64))
        base += len(ts)
    seg = _chunked(np.concatenate(rows) if rows else np.zeros((0, SEG_W), np.int64))
    return GatherTable(seg, np.concatenate(tsrc) if tsrc else np.zeros(0, np.int64),
                       np.concatenate(tcf) if tcf else np.zeros(0),
                       np.concatenate(tld) if tld else np.zeros(0, np.int64))


# ---------------------------------------------------------------------------------------
# grouped GEMM tables


class GemmTable:
    """A grouped-GEMM program (one tile kind); host table uploaded on first use."""

    def __init__(self, table: np.ndarray, tiles: int, flops: int, kind: int,
                 n_counters: int = 0, n_parts: int = 0) -> None:
        self.table = table
        self.n_gemm = len(table)
        self.tiles = tiles
        self.flops = flops
        self.kind = kind
        self.n_counters = n_counters
        self.work_bytes = (((4 * n_counters + 255) // 256) * 256 + 8 * n_parts) if n_counters else 0
        per = table[:, 11] if len(table) else np.zeros(0, np.int64)
        self.tile_map = np.repeat(np.arange(len(table), dtype=np.int32), per)
        self._dev = None
        self._rows_dev = None
        self._work: dict = {}
        self._private = False

    @property
    def launches(self) -> int:
        """Kernels one ``run`` launches: tensor-core tables pack A and B first."""
        if self.n_gemm == 0:
            return 0
        if self.kind in (TILE_TC_TF32, TILE_TC_3XBF16):
            return 1 + int(self.n_counters > 0)
        return 1

    def private(self) -> GemmTable:
        """The same table with a split-K work buffer of its own (a compiled program's
        copy, so that programs sharing a cached table can run on different streams)."""
        import copy

        q = copy.copy(self)
        q._work = {}
        q._private = True
        return q

    def work(self):
        """The split-K scratch: the table's own when private, else one per stream."""
        if not self.work_bytes:
            return None
        key = 0 if self._private else stream_ptr()
        buf = self._work.get(key)
        if buf is None:
            buf = torch.zeros(self.work_bytes, dtype=torch.uint8, device=device())
            self._work[key] = buf
        return buf

    def host_arrays(self) -> tuple:
        return (self.table, self.tile_map)

    def device_tables(self):
        """(table, tile_map) on the current device, uploaded on first use."""
        if self._dev is None:
            self._dev = Uploaded(self.host_arrays())
        return self._dev.ready()

    def tile_rows(self) -> np.ndarray:
        """The table as one row per tile (``tnb_grouped_gemm_f64_rows``)."""
        return np.ascontiguousarray(self.table[self.tile_map])

    def run(self, a, b, c) -> None:
        """Launch on the current stream.  The split-K counters of a private table belong
        to it, so one private table must not run on two streams at once."""
        if self.n_gemm == 0:
            return
        work = self.work()
        rec = recording()
        if (rec is None and DIRECT_GEMM and self.tiles >= DIRECT_MIN_TILES
                and self.kind in (TILE_64, TILE_32, TILE_SKINNY, TILE_WIDE)):
            if self._rows_dev is None:
                self._rows_dev = Uploaded((self.tile_rows(),))
            (rows,) = self._rows_dev.ready()
            mark = _LOG.begin() if _LOG is not None else None
            _lib.call("tnb_grouped_gemm_f64_rows", ptr(rows), self.tiles, self.kind, ptr(a),
                      a.numel(), ptr(b), b.numel(), ptr(c), c.numel(), ptr(work),
                      self.work_bytes, self.n_counters, stream_ptr())
            if _LOG is not None:
                _LOG.end("grouped_gemm_f64", mark, self.flops)
            return
        table, tile_map = self.device_tables()
        if rec is not None:
            _lib.call("tnb_seq_add_gemm", rec.handle, ptr(table), self.n_gemm, ptr(tile_map),
                      self.tiles, self.kind, ptr(a), a.numel(), ptr(b), b.numel(), ptr(c),
                      c.numel(), ptr(work), self.work_bytes, self.n_counters)
            return
        mark = _LOG.begin() if _LOG is not None else None
        _lib.call("tnb_grouped_gemm_f64", ptr(table), self.n_gemm, ptr(tile_map),
                  self.tiles, self.kind, ptr(a), a.numel(), ptr(b), b.numel(), ptr(c),
                  c.numel(), ptr(work), self.work_bytes, self.n_counters, stream_ptr())
        if _LOG is not None:
            _LOG.end("grouped_gemm_tc" if self.kind in (TILE_TC_TF32, TILE_TC_3XBF16)
                     else "grouped_gemm_f64", mark, self.flops)


#: longest contracted dimension of a product whose A gather runs inside its GEMM
#: (``GatherAGemm``, ``tnb_grouped_gemm_gather_a``), and the most gather terms one of its
#: 32-row tiles may read (they are staged in shared memory)
GA_MAX_K = 128
GA_MAX_TERMS = 5120
#: fold an eligible link's A gather into its GEMM launch (``ChainProgram``).  Off by
#: default: the same results, measured slower on B200 (folded heff2 at the L = 64 mid bond
#: 20.5 against 16.4 us in 3 against 5 launches; 43.5 against 39.0 us at 256 multiplets):
#: a tile's A elements, their terms and its K reduction land on the few CTAs of the
#: product's output tiles, where the separate gather spreads them over 9-32 CTAs and
#: overlaps its table loads with the previous kernel
FUSE_A = False


def gather_csr(g: GatherTable, n_dst: int):
    """The element-level view of a gather into a buffer of ``n_dst`` elements: for every
    destination element, its terms ``(source offset, coefficient)`` in the gather's own
    order (``ptr`` of ``n_dst + 1`` entries, int32 ``src``, float64 ``cf``).  Elements no
    segment covers get no terms (they read as zero).  None when the gather uses its
    second buffer pair or the sizes exceed int32."""
    seg = g.seg
    if g.n_seg and np.any(seg[:, 5] != 0):
        return None
    dsts, srcs, cfs = [], [], []
    for row in seg:
        size, rank, t0, t1 = int(row[1]), int(row[2]), int(row[3]), int(row[4])
        if size == 0:
            continue
        dims = [int(x) for x in row[8:8 + rank]]
        idx = np.indices(dims).reshape(rank, -1)  # outermost first, C order = element order
        dst = int(row[0]) + (row[16:16 + rank, None] * idx).sum(axis=0)
        R = (row[24:24 + rank, None] * idx).sum(axis=0)
        C = (row[32:32 + rank, None] * idx).sum(axis=0)
        if t1 == t0:
            continue
        for t in range(t0, t1):
            dsts.append(dst)
            srcs.append(int(g.tsrc[t]) + int(g.tld[t]) * R + C)
            cfs.append(np.full(dst.size, float(g.tcf[t])))
    if dsts:
        d = np.concatenate(dsts)
        sv = np.concatenate(srcs)
        cv = np.concatenate(cfs)
        order = np.argsort(d, kind="stable")  # per element, terms stay in table order
        d, sv, cv = d[order], sv[order], cv[order]
    else:
        d = sv = np.zeros(0, np.int64)
        cv = np.zeros(0)
    if d.size and (d.min() < 0 or d.max() >= n_dst):
        raise ValueError("gather_csr: a destination lies outside the buffer")
    if sv.size and (sv.min() < 0 or sv.max() >= 2 ** 31 - 1) or d.size >= 2 ** 31 - 1:
        return None
    ptr = np.zeros(n_dst + 1, np.int64)
    np.add.at(ptr, d + 1, 1)
    ptr = np.cumsum(ptr)
    return ptr.astype(np.int32), sv.astype(np.int32), cv.astype(np.float64)


class GatherAGemm:
    """A link's A gather and grouped FP64 GEMM as one launch (``tnb_grouped_gemm_gather_a``):
    32 x 32 output tiles without split-K over products with K <= ``GA_MAX_K``, each CTA
    evaluating its A tile from the gather's element-level terms."""

    def __init__(self, csr, products, n_a: int) -> None:
        rows, tile, flops = [], 0, 0
        for M, N, K, ao, lda, bo, ldb, co, ldc in products:
            if not (M and N):
                continue
            out_tiles, tn = _tiles(M, N, TILE_32)
            rows.append([M, N, K, ao, lda, bo, ldb, co, ldc, tile, tn, out_tiles, 0, 0, 0, 0])
            tile += out_tiles
            flops += 2 * M * N * K
        self.table = np.array(rows, dtype=np.int64).reshape(-1, GEMM_W)
        self.n_gemm = len(rows)
        self.tiles = tile
        self.flops = flops
        per = self.table[:, 11] if len(rows) else np.zeros(0, np.int64)
        self.tile_map = np.repeat(np.arange(len(rows), dtype=np.int32), per)
        self.a_ptr, self.a_src, self.a_cf = csr
        self.n_a = n_a
        # algorithmic bytes of one launch: every A term's source element, B and C once
        self.bytes = 8 * len(self.a_cf) + sum(8 * (K * N + M * N) for M, N, K, *_ in rows)
        self._dev = None

    launches = 1

    @staticmethod
    def eligible(products) -> bool:
        return all(p[2] <= GA_MAX_K and (p[2] == 0 or p[4] == p[2]) for p in products)

    @staticmethod
    def fits(csr, products) -> bool:
        """Whether every 32-row tile's A elements have at most ``GA_MAX_TERMS`` terms."""
        a_ptr = csr[0]
        for M, N, K, ao, *_ in products:
            if not (M and N and K):
                continue
            for m0 in range(0, M, 32):
                rows = min(32, M - m0)
                lo, hi = ao + m0 * K, ao + (m0 + rows) * K
                if hi >= len(a_ptr) or a_ptr[hi] - a_ptr[lo] > GA_MAX_TERMS:
                    return False
        return True

    def host_arrays(self) -> tuple:
        return (self.table, self.tile_map, self.a_ptr, self.a_src, self.a_cf)

    def device_tables(self):
        if self._dev is None:
            self._dev = Uploaded(self.host_arrays())
        return self._dev.ready()

    def private(self):
        return self

    def run(self, src, b, c) -> None:
        if self.n_gemm == 0:
            return
        table, tile_map, a_ptr, a_src, a_cf = self.device_tables()
        args = (ptr(table), self.n_gemm, ptr(tile_map), self.tiles, ptr(a_ptr),
                a_ptr.numel(), ptr(a_src), ptr(a_cf), a_cf.numel(), ptr(src), src.numel(),
                ptr(b), b.numel(), ptr(c), c.numel())
        rec = recording()
        if rec is not None:
            _lib.call("tnb_seq_add_gemm_gather_a", rec.handle, *args)
            return
        mark = _LOG.begin() if _LOG is not None else None
        _lib.call("tnb_grouped_gemm_gather_a", *args, stream_ptr())
        if _LOG is not None:
            _LOG.end("grouped_gemm_gather_a", mark, self.bytes)


def _tiles(M, N, kind):
    if kind == TILE_SKINNY:
        return (M + SKINNY_ROWS - 1) // SKINNY_ROWS, 1
    if kind == TILE_WIDE:
        return (N + SKINNY_ROWS - 1) // SKINNY_ROWS, 1
    if kind in (TILE_TC_TF32, TILE_TC_3XBF16):
        tn = (N + TC_TILE - 1) // TC_TILE
        return ((M + TC_TILE - 1) // TC_TILE) * tn, tn
    t = 64 if kind == TILE_64 else 32
    tn = (N + t - 1) // t
    return ((M + t - 1) // t) * tn, tn


def choose_kind(products) -> int:
    """Skinny when every product is tall and thin; else 64x64 tiles unless they would
    not fill two waves of the GPU, then 32x32."""
    live = [p for p in products if p[0] and p[1]]
    if live and all(_is_skinny(p, thin_rows(live)) for p in live):
        return TILE_SKINNY
    big = sum(_tiles(p[0], p[1], TILE_64)[0] for p in live)
    return TILE_64 if big >= 2 * N_SM else TILE_32


def _is_skinny(p, thin_rows: int = 0) -> bool:
    """A tall product (at most 16 columns and 16 contracted) goes to the one-thread-per-row
    kernel when it has many rows, or whenever its composition's thin products hold
    ``SKINNY_BULK`` rows or more in all (``thin_rows``): then a 64- or 32-wide tile would
    leave most of its columns idle on a lot of work.  A few small thin products stay in
    the tiled launch (no second launch for little work)."""
    thin = p[1] <= SKINNY_MAX and p[2] <= SKINNY_MAX
    return thin and (p[0] >= SKINNY_ROWS or thin_rows >= SKINNY_BULK)


#: total rows of thin products above which every thin product of a composition runs on
#: the one-thread-per-row kernel
SKINNY_BULK = 1 << 16


def thin_rows(products) -> int:
    return sum(p[0] for p in products if p[1] and p[1] <= SKINNY_MAX and p[2] <= SKINNY_MAX)


def wide_cols(products) -> int:
    return sum(p[1] for p in products if p[0] and p[0] <= SKINNY_MAX and p[2] <= SKINNY_MAX)


def _is_wide(p, cols: int = 0) -> bool:
    """The transpose of ``_is_skinny``: at most 16 rows and 16 contracted, a long N (or
    many such columns in the composition) -- one thread per output column."""
    flat = p[0] <= SKINNY_MAX and p[2] <= SKINNY_MAX
    return flat and (p[1] >= SKINNY_ROWS or cols >= SKINNY_BULK)


#: A coupled-sector product goes to the tensor cores in the precision form only when it
#: is at least 2 x 128 x 64 x 64 flops (half a 128 x 128 x 64 tile's work); smaller ones
#: stay on the FP64 path.
TC_MIN_FLOPS = 2 * 128 * 64 * 64


def tc_worthy(p, min_flops: int | None = None) -> bool:
    M, N, K = p[0], p[1], p[2]
    return K >= 16 and 2 * M * N * K >= (TC_MIN_FLOPS if min_flops is None else min_flops)


# ---------------------------------------------------------------------------------------
# autotuning of the FP64 tile kind


AUTOTUNE_CACHE: dict = {}


def histogram_key(products) -> tuple:
    """The block-size histogram of a composition: product counts per (log2 M, log2 N,
    log2 K) bin.  Compositions with the same histogram share a tuning decision."""
    from collections import Counter

    c = Counter((int(p[0]).bit_length(), int(p[1]).bit_length(), int(p[2]).bit_length())
                for p in products if p[0] and p[1])
    return tuple(sorted(c.items()))


def autotune(products) -> tuple[int, bool]:
    """``(tile kind, split-K)`` for the FP64 products of a composition, measured: each
    candidate -- 64 x 64 or 32 x 32 tiles, with or without split-K -- runs three times
    on scratch operands of the composition's extents (CUDA events on the current
    stream, after one untimed run), and the fastest is cached under the block-size
    histogram.  Every candidate computes the same products; split-K changes the order
    in which a long K is summed, so results are reproducible for a fixed decision."""
    key = histogram_key(products)
    hit = AUTOTUNE_CACHE.get(key)
    if hit is not None:
        return hit
    live = [p for p in products if p[0] and p[1]]
    dev = device()
    f64 = dict(dtype=torch.float64, device=dev)
    na = max([p[3] + (p[0] - 1) * p[4] + p[2] for p in live if p[2]] + [1])
    nb = max([p[5] + (p[2] - 1) * p[6] + p[1] for p in live if p[2]] + [1])
    nc = max([p[7] + (p[0] - 1) * p[8] + p[1] for p in live] + [1])
    a, b, c = torch.zeros(na, **f64), torch.zeros(nb, **f64), torch.empty(nc, **f64)
    best, best_ms = (choose_kind(live), True), float("inf")
    for kind in (TILE_64, TILE_32):
        for split in (True, False):
            t = make_gemm(live, kind, split_k=split)
            t.run(a, b, c)
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
            ev[0].record()
            for _ in range(3):
                t.run(a, b, c)
            ev[1].record()
            ev[1].synchronize()
            ms = ev[0].elapsed_time(ev[1])
            if ms < best_ms:
                best, best_ms = (kind, split), ms
    AUTOTUNE_CACHE[key] = best
    return best


class GemmGroup:
    """One composition's products in at most four launches: the tall skinny ones, the wide
    flat ones, the rest in FP64 tiles, and -- in the precision form -- the products big
    enough to be dense contractions on the tcgen05 tensor cores (``tc_min_flops``
    overrides the size rule).  ``tuned`` picks the FP64 tile kind by ``autotune``
    instead of the size heuristic."""

    def __init__(self, products, precision: str = "f64", tc_min_flops: int | None = None,
                 tuned: bool = False, split_k: bool = True):
        bulk, cols = thin_rows(products), wide_cols(products)
        skinny = [p for p in products if _is_skinny(p, bulk)]
        wide = [p for p in products if not _is_skinny(p, bulk) and _is_wide(p, cols)]
        rest = [p for p in products if not _is_skinny(p, bulk) and not _is_wide(p, cols)]
        tc = []
        if precision in TC_KINDS:
            tc = [p for p in rest if tc_worthy(p, tc_min_flops)]
            rest = [p for p in rest if not tc_worthy(p, tc_min_flops)]
        self.parts = []
        if tc:
            self.parts.append(make_gemm(tc, TC_KINDS[precision]))
        if rest:
            if tuned:  # the measured tile kind for this block-size histogram
                kind, split = autotune(rest)
                self.parts.append(make_gemm(rest, kind, split_k=split))
            else:
                self.parts.append(make_gemm(rest, choose_kind(rest), split_k=split_k))
        if skinny:
            self.parts.append(make_gemm(skinny, TILE_SKINNY))
        if wide:
            self.parts.append(make_gemm(wide, TILE_WIDE))
        self.tensor_core = bool(tc)
        self.products = list(products)
        self.flops = sum(p.flops for p in self.parts)
        self.tiles = sum(p.tiles for p in self.parts)
        self.n_gemm = sum(p.n_gemm for p in self.parts)
        self.launches = sum(p.launches for p in self.parts)

    @property
    def table(self):
        return np.concatenate([p.table for p in self.parts]) if self.parts else \
            np.zeros((0, GEMM_W), np.int64)

    def run(self, a, b, c) -> None:
        for p in self.parts:
            p.run(a, b, c)

    def private(self) -> GemmGroup:
        import copy

        q = copy.copy(self)
        q.parts = [p.private() for p in self.parts]
        return q


#: CTAs a composition's split-K tiles aim for (two per SM)
SPLITK_TARGET_CTAS = 2 * N_SM


def _splits(K: int, out_tiles_total: int) -> tuple[int, int]:
    """K splits for a long-K product when the composition's output tiles cannot fill two
    waves: (splits, ksplit) with ksplit a multiple of 16 and at least 32."""
    if K <= 64 or out_tiles_total >= SPLITK_TARGET_CTAS:
        return 1, 0
    want = max(1, -(-SPLITK_TARGET_CTAS // max(out_tiles_total, 1)))
    ks = max(32, -(-K // want))
    ks = -(-ks // 16) * 16
    return -(-K // ks), ks


def make_gemm(products, kind: int | None = None, split_k: bool = True) -> GemmTable:
    """``products``: iterable of (M, N, K, a_off, lda, b_off, ldb, c_off, ldc)."""
    products = [p for p in products if p[0] and p[1]]
    if kind is None:
        kind = choose_kind(products)
    tw = 64 if kind == TILE_64 else 32  # split-K partial tile width (tiled FP64 kinds only)
    out_total = sum(_tiles(p[0], p[1], kind)[0] for p in products)
    rows = []
    tile = flops = n_cnt = n_parts = 0
    for M, N, K, ao, lda, bo, ldb, co, ldc in products:
        out_tiles, tn = _tiles(M, N, kind)
        S, ks = (1, 0)
        if split_k and kind in (TILE_64, TILE_32):
            S, ks = _splits(K, out_total)
        row = [M, N, K, ao, lda, bo, ldb, co, ldc, tile, tn, out_tiles * S, 0, 0, 0, 0]
        if S > 1:
            row[12:16] = [S, ks, n_parts, n_cnt]
            n_parts += out_tiles * S * tw * tw
            n_cnt += out_tiles
        rows.append(row)
        tile += out_tiles * S
        flops += 2 * M * N * K
    arr = np.array(rows, dtype=np.int64).reshape(-1, GEMM_W)
    if kind in (TILE_TC_TF32, TILE_TC_3XBF16):
        # operand packing: per row the first A slab (M tiles x K slabs) and B slab (N tiles
        # x K slabs) in the packed work buffer; the counts travel in n_counters
        a_tot = b_tot = 0
        for row in arr:
            M, N, K = int(row[0]), int(row[1]), int(row[2])
            ks = (K + TC_BK - 1) // TC_BK
            row[12], row[13] = a_tot, b_tot
            a_tot += ((M + TC_TILE - 1) // TC_TILE) * ks
            b_tot += ((N + TC_TILE - 1) // TC_TILE) * ks
        t = GemmTable(arr, tile, flops, kind)
        t.n_counters = a_tot | (b_tot << 32)
        t.work_bytes = (a_tot + b_tot) * TC_SLAB_BYTES
        return t
    return GemmTable(arr, tile, flops, kind, n_cnt, n_parts)


# ---------------------------------------------------------------------------------------
# weighted runs for inner / norm


class DotRuns:
    """Equal-weight element runs of a structure (device arrays, see ``Uploaded``)."""

    def __init__(self, starts, weights) -> None:
        self._up = Uploaded((np.asarray(starts, dtype=np.int64),
                             np.asarray(weights, dtype=np.float64)))
        self.n_runs = len(weights)

    @property
    def start(self) -> _DevArray:
        return self._up.ready()[0]

    @property
    def weight(self) -> _DevArray:
        return self._up.ready()[1]


def make_runs(s: TensorStructure) -> DotRuns:
    lay = layout(s)
    p = s.provider
    starts, weights = [], []
    for b in range(len(lay.sizes)):
        w = p._qdim(int(lay.coupled[b]))
        if weights and weights[-1] == w:
            continue
        starts.append(int(lay.offsets[b]))
        weights.append(w)
    starts.append(lay.size)
    return DotRuns(starts, weights)


_WORK: dict = {}


def dot_workspace(n: int) -> torch.Tensor:
    """A zero-initialised scratch buffer per (device, stream), grown on demand."""
    need = int(_lib.load().tnb_dot_work_bytes(n))
    key = (torch.cuda.current_device(), torch.cuda.current_stream().cuda_stream)
    buf = _WORK.get(key)
    if buf is None or buf.numel() < need:
        buf = torch.zeros(max(need, 4096), dtype=torch.uint8, device=device())
        _WORK[key] = buf
    return buf
