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
from dataclasses import dataclass

import numpy as np
import torch

from tenet import _lib
from tenet.structure import TensorStructure, layout, matrix_layout

SEG_W = 40
GEMM_W = 16
CHUNK = 1024
MAX_RANK = 8
TILE_64, TILE_32, TILE_SKINNY, TILE_TC_TF32, TILE_TC_3XBF16 = 0, 1, 2, 3, 4
TC_KINDS = {"tf32": TILE_TC_TF32, "3xbf16": TILE_TC_3XBF16}
SKINNY_ROWS, SKINNY_MAX = 256, 16
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
        global _REC
        self._prev, _REC = _REC, self
        return self

    def __exit__(self, *exc):
        global _REC
        _REC = self._prev

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


_REC: Seq | None = None


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


def _group(terms):
    by_dst: dict = {}
    for s, d, c in terms:
        by_dst.setdefault(d, []).append((s, c))
    return by_dst


def _normalise(dims, dstr, rstr, cstr):
    """Order dims by destination stride (descending), drop extent-1 dims, merge dims that
    are contiguous in destination and source alike."""
    order = sorted(range(len(dims)), key=lambda k: (-dstr[k], -cstr[k], -rstr[k]))
    out = []
    for k in order:
        if dims[k] == 1:
            continue
        d, a, b, c = dims[k], dstr[k], rstr[k], cstr[k]
        if out:
            pd, pa, pb, pc = out[-1]
            if pa == a * d and pb == b * d and pc == c * d:
                out[-1] = (pd * d, a, b, c)
                continue
        out.append((d, a, b, c))
    if not out:
        out = [(1, 1, 0, 0)]
    if len(out) > MAX_RANK:
        raise ValueError(f"a block of rank {len(out)} exceeds the kernel's {MAX_RANK}")
    return out


def gather_rows(src_s: TensorStructure, src_kind: str, dst_s: TensorStructure, dst_kind: str,
                perm, terms, buf: int = 0, dst_keep=None):
    """Rows + term arrays executing ``dst[j] = sum c * transpose(src[i], perm)``.

    ``dst_keep`` optionally restricts the emitted destination blocks (a boolean mask).
    """
    sl, dl = layout(src_s), layout(dst_s)
    if src_kind == "matrix":
        sm = matrix_layout(src_s)
        s_off, s_ld, s_rs, s_cs = sm.block_off, sm.block_ld, sm.rstride, sm.cstride
    else:
        s_off, s_ld = sl.offsets, np.zeros_like(sl.offsets)
        s_rs, s_cs = np.zeros_like(sl.strides), sl.strides
    if dst_kind == "matrix":
        dm = matrix_layout(dst_s)
        d_off = dm.block_off
        d_str = dm.rstride * dm.block_ld[:, None] + dm.cstride
    else:
        d_off, d_str = dl.offsets, dl.strides
    perm = list(perm)
    rows, tsrc, tcf, tld = [], [], [], []
    for j, lst in sorted(_group(terms).items()):
        if dst_keep is not None and not dst_keep[j]:
            continue
        i0 = lst[0][0]
        dims = [int(x) for x in dl.shapes[j]]
        segs = _normalise(dims, [int(x) for x in d_str[j]], [int(s_rs[i0][p]) for p in perm],
                          [int(s_cs[i0][p]) for p in perm])
        row = np.zeros(SEG_W, dtype=np.int64)
        row[0] = d_off[j]
        row[1] = dl.sizes[j]
        row[2] = len(segs)
        row[3] = len(tsrc)
        row[4] = len(tsrc) + len(lst)
        row[5] = buf
        for k, (d, a, b, c) in enumerate(segs):
            row[8 + k], row[16 + k], row[24 + k], row[32 + k] = d, a, b, c
        rows.append(row)
        for i, c in lst:
            tsrc.append(int(s_off[i]))
            tcf.append(float(c))
            tld.append(int(s_ld[i]))
    # destination blocks with no term at all are written as zeros
    covered = set(_group(terms))
    for j in range(len(dl.sizes)):
        if j in covered or (dst_keep is not None and not dst_keep[j]):
            continue
        dims = [int(x) for x in dl.shapes[j]]
        segs = _normalise(dims, [int(x) for x in d_str[j]], [0] * len(dims), [0] * len(dims))
        row = np.zeros(SEG_W, dtype=np.int64)
        row[0], row[1], row[2] = d_off[j], dl.sizes[j], len(segs)
        row[3] = row[4] = len(tsrc)
        row[5] = buf
        for k, (d, a, b, c) in enumerate(segs):
            row[8 + k], row[16 + k], row[24 + k], row[32 + k] = d, a, b, c
        rows.append(row)
    return rows, tsrc, tcf, tld


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
        self.chunks = int(((seg[:, 1] + CHUNK - 1) // CHUNK).sum()) if len(seg) else 0
        self.elems = int(seg[:, 1].sum()) if len(seg) else 0
        self.term_elems = int((seg[:, 1] * (seg[:, 4] - seg[:, 3])).sum()) if len(seg) else 0
        per = (seg[:, 1] + CHUNK - 1) // CHUNK if len(seg) else np.zeros(0, np.int64)
        self.chunk_map = np.repeat(np.arange(len(seg), dtype=np.int32), per)
        self._dev = None

    @property
    def bytes_moved(self) -> int:
        """Algorithmic HBM bytes of one run: every term's source read once, every
        destination element written once."""
        return 8 * (self.elems + self.term_elems)

    def device_arrays(self):
        if self._dev is None:
            dev = device()
            self._dev = tuple(torch.from_numpy(x).to(dev) for x in
                              (self.seg, self.tsrc, self.tcf, self.tld, self.chunk_map))
        return self._dev

    def run(self, src0, dst0, src1=None, dst1=None) -> None:
        if self.n_seg == 0:
            return
        seg, tsrc, tcf, tld, cmap = self.device_arrays()
        if _REC is not None:
            _lib.call("tnb_seq_add_gather", _REC.handle, ptr(seg), self.n_seg, ptr(cmap),
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


def make_gather(*parts) -> GatherTable:
    """Concatenate one or more ``gather_rows`` results into a single table."""
    rows, tsrc, tcf, tld = [], [], [], []
    for r, s, c, ld in parts:
        base = len(tsrc)
        for row in r:
            row = row.copy()
            row[3] += base
            row[4] += base
            rows.append(row)
        tsrc += s
        tcf += c
        tld += ld
    chunk = 0
    for row in rows:
        row[6] = chunk
        chunk += (int(row[1]) + CHUNK - 1) // CHUNK
    seg = np.stack(rows) if rows else np.zeros((0, SEG_W), np.int64)
    return GatherTable(seg, tsrc, tcf, tld)


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

    def run(self, a, b, c) -> None:
        """Launch on the current stream.  The split-K work buffer belongs to this table, so
        one table must not run on two streams at once."""
        if self.n_gemm == 0:
            return
        if self._dev is None:
            dev = device()
            work = torch.zeros(max(self.work_bytes, 1), dtype=torch.uint8, device=dev)
            self._dev = (torch.from_numpy(self.table).to(dev),
                         torch.from_numpy(self.tile_map).to(dev), work)
        if _REC is not None:
            _lib.call("tnb_seq_add_gemm", _REC.handle, ptr(self._dev[0]), self.n_gemm,
                      ptr(self._dev[1]), self.tiles, self.kind, ptr(a), a.numel(), ptr(b),
                      b.numel(), ptr(c), c.numel(),
                      ptr(self._dev[2]) if self.work_bytes else None, self.work_bytes,
                      self.n_counters)
            return
        mark = _LOG.begin() if _LOG is not None else None
        _lib.call("tnb_grouped_gemm_f64", ptr(self._dev[0]), self.n_gemm, ptr(self._dev[1]),
                  self.tiles, self.kind, ptr(a), a.numel(), ptr(b), b.numel(), ptr(c),
                  c.numel(), ptr(self._dev[2]) if self.work_bytes else None, self.work_bytes,
                  self.n_counters, stream_ptr())
        if _LOG is not None:
            _LOG.end("grouped_gemm_tc" if self.kind in (TILE_TC_TF32, TILE_TC_3XBF16)
                     else "grouped_gemm_f64", mark, self.flops)


def _tiles(M, N, kind):
    if kind == TILE_SKINNY:
        return (M + SKINNY_ROWS - 1) // SKINNY_ROWS, 1
    if kind in (TILE_TC_TF32, TILE_TC_3XBF16):
        tn = (N + 63) // 64
        return ((M + 127) // 128) * tn, tn
    t = 64 if kind == TILE_64 else 32
    tn = (N + t - 1) // t
    return ((M + t - 1) // t) * tn, tn


def choose_kind(products) -> int:
    """Skinny when every product is tall and thin; else 64x64 tiles unless they would
    not fill two waves of the GPU, then 32x32."""
    live = [p for p in products if p[0] and p[1]]
    if live and all(_is_skinny(p) for p in live):
        return TILE_SKINNY
    big = sum(_tiles(p[0], p[1], TILE_64)[0] for p in live)
    return TILE_64 if big >= 2 * N_SM else TILE_32


def _is_skinny(p) -> bool:
    """A tall product (many rows, at most 16 columns and 16 contracted) goes to the
    one-thread-per-row kernel; a small one stays in the tiled launch."""
    return p[0] >= SKINNY_ROWS and p[1] <= SKINNY_MAX and p[2] <= SKINNY_MAX


class GemmGroup:
    """One composition's products, split into at most two launches: the tall skinny ones
    and the rest (so an MPO-like product never occupies a 64-wide tile)."""

    def __init__(self, products, precision: str = "f64") -> None:
        skinny = [p for p in products if _is_skinny(p)]
        rest = [p for p in products if not _is_skinny(p)]
        self.parts = []
        if rest:
            kind = TC_KINDS[precision] if precision in TC_KINDS else choose_kind(rest)
            self.parts.append(make_gemm(rest, kind))
        if skinny:
            self.parts.append(make_gemm(skinny, TILE_SKINNY))
        self.flops = sum(p.flops for p in self.parts)
        self.tiles = sum(p.tiles for p in self.parts)
        self.n_gemm = sum(p.n_gemm for p in self.parts)
        self.launches = len(self.parts)

    @property
    def table(self):
        return np.concatenate([p.table for p in self.parts]) if self.parts else \
            np.zeros((0, GEMM_W), np.int64)

    def run(self, a, b, c) -> None:
        for p in self.parts:
            p.run(a, b, c)


def _splits(K: int, out_tiles_total: int) -> tuple[int, int]:
    """K splits for a long-K product when the composition's output tiles cannot fill two
    waves: (splits, ksplit) with ksplit a multiple of 16 and at least 32."""
    if K <= 64 or out_tiles_total >= 2 * N_SM:
        return 1, 0
    want = max(1, -(-2 * N_SM // max(out_tiles_total, 1)))
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
    return GemmTable(arr, tile, flops, kind, n_cnt, n_parts)


# ---------------------------------------------------------------------------------------
# weighted runs for inner / norm


@dataclass
class DotRuns:
    start: torch.Tensor
    weight: torch.Tensor
    n_runs: int


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
    dev = device()
    return DotRuns(torch.tensor(starts, dtype=torch.int64, device=dev),
                   torch.tensor(weights, dtype=torch.float64, device=dev), len(weights))


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
