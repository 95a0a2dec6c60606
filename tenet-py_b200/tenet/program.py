"""Compiled contraction chains: a matvec as a fixed sequence of kernel launches.

The two-site matvec (``network/env.py:416-432``) is a chain: each pairwise contraction's
left operand is the previous result, its right operand a tensor that does not change
during a Lanczos solve (an environment or an MPO site).  In the reference every link is
``repartition -> to_matrices -> matmul -> from_matrices -> repartition -> transpose``
(``ops/contraction.py:368-376``), plus the explicit bends of ``_composed``
(``network/env.py:60-90``).  Here the chain is planned once:

* each fixed operand is packed into its coupled-sector matrices once per program;
* everything between two GEMMs -- the previous product's ``from_matrices``, its
  restoring repartition, the einsum's final transpose, the next bend and the next
  operand's repartition and ``to_matrices`` -- composes into one block map, executed by
  one gather straight from the previous product's packed matrices into the next
  operand's packed matrices;
* every buffer is allocated once, so ``run`` is a fixed launch sequence that a CUDA
  graph captures and replays.

For ``heff2`` that is 5 gathers and 4 grouped GEMMs per matvec, 8 launches in the FP64
form: the first link's A gather only permutes whole rows of the input's blocks, so its
products read the input in place (``_direct_products``).  Optionally (``defer``) the two
MPO links' products (K <= 4) are computed by the gathers that read them
(``_defer_skinny``): 6 launches, the same bits.
"""

from __future__ import annotations

import numpy as np
import torch

from tenet import _exec, _lib
from tenet.plan import chain, repartition_plan, transpose_plan
from tenet.structure import IN, OUT, TensorStructure, layout, matrix_layout
from tenet.tensor import SymmetricTensor

__all__ = ["ChainProgram", "heff2_folded_program", "heff2_program"]

#: stage capacity of one fused launch (``tnb_seq_fuse``)
FUSED_MAX_STAGES = 24


class _StructureOnly:
    """Stand-in for a fixed operand in a shared program template: its structure only."""

    __slots__ = ("structure",)

    def __init__(self, structure) -> None:
        self.structure = structure


def _identity_plan(s: TensorStructure):
    return s, tuple(range(s.ndim)), tuple((i, i, 1.0) for i in range(s.num_blocks))


def _direct_products(g, products):
    """The link's products reading its source in place, or None.

    When the A gather only moves whole rows of the coupled-sector matrices -- every
    segment a contiguous run (rank 1, unit strides) copied with one term of coefficient 1,
    covering complete rows of one product's A -- the gather is a row permutation, and a
    product whose A rows come from several runs is the same product split by rows: one
    product per run (runs contiguous in the source merged), A read from the source where
    the run lies, C rows where they were.  Every C element keeps its FMA chain over K."""
    if g is None or g.n_seg == 0:
        return None
    seg = g.seg
    t0 = seg[:, 3]
    single = seg[:, 1] == 1  # a one-element run has no stride
    if (np.any(seg[:, 2] != 1) or np.any(seg[:, 4] - t0 != 1) or np.any(seg[:, 5] != 0)
            or np.any((seg[:, 16] != 1) & ~single) or np.any((seg[:, 32] != 1) & ~single)):
        return None
    if np.any(g.tcf[t0] != 1.0) or np.any((g.tld[t0] * seg[:, 24] != 0) & ~single):
        return None
    runs = sorted(zip(seg[:, 0].tolist(), seg[:, 1].tolist(), g.tsrc[t0].tolist()))
    out, r = [], 0
    for M, N, K, ao, lda, bo, ldb, co, ldc in sorted(products, key=lambda p: (p[2] == 0, p[3])):
        if K == 0:
            out.append((M, N, K, ao, lda, bo, ldb, co, ldc))
            continue
        if lda != K:
            return None
        end, pos, mine = ao + M * K, ao, []
        while r < len(runs) and runs[r][0] < end:
            d, size, src = runs[r]
            if d != pos or size % K or d + size > end:
                return None
            if mine and mine[-1][2] + mine[-1][1] == src:  # contiguous in the source too
                mine[-1] = (mine[-1][0], mine[-1][1] + size, mine[-1][2])
            else:
                mine.append((d, size, src))
            pos, r = d + size, r + 1
        if pos != end:
            return None
        for d, size, src in mine:
            out.append((size // K, N, K, src, K, bo, ldb, co + ((d - ao) // K) * ldc, ldc))
    return out if r == len(runs) else None


class _Link:
    """One contraction of the chain, with its gathers and GEMM table."""

    def __init__(self, src_struct, src_kind, a_plan, b_tensor, b_plan, axes, precision="f64",
                 tc_min_flops=None):
        ca, cb = axes
        sa_logical = a_plan[0]
        sb_logical = b_plan[0]
        fa = tuple(i for i in range(sa_logical.ndim) if i not in ca)
        fb = tuple(j for j in range(sb_logical.ndim) if j not in cb)
        for i, j in zip(ca, cb):
            x, y = sa_logical.legs[i], sb_logical.legs[j]
            if x.space != y.space or (x.dual != (x.side is IN)) == (y.dual != (y.side is IN)):
                raise ValueError(f"chain: axis {i} and axis {j} do not contract")
        sa2, pa, ta = chain(a_plan, repartition_plan(sa_logical, fa, ca))
        sb2, pb, tb = chain(b_plan, repartition_plan(sb_logical, cb, fb))
        sc = TensorStructure((*sa2.codomain, *sb2.domain))
        free = (*(sa_logical.legs[i] for i in fa), *(sb_logical.legs[j] for j in fb))
        ro = tuple(k for k, leg in enumerate(free) if leg.side is OUT)
        ri = tuple(k for k, leg in enumerate(free) if leg.side is IN)
        pos = {k: q for q, k in enumerate((*ro, *ri))}
        ft = tuple(pos[k] for k in range(len(free)))
        rp = repartition_plan(sc, ro, ri)
        self.after = chain(rp, transpose_plan(rp[0], ft))  # C' -> tensordot output
        assert self.after[0].legs == free
        ma, mb, mc = matrix_layout(sa2), matrix_layout(sb2), matrix_layout(sc)
        products, used = [], set()
        for c in mc.sectors:
            M, N = mc.shape[c]
            if c in ma.shape and c in mb.shape:
                K = ma.shape[c][1]
                products.append((M, N, K, ma.base[c], K, mb.base[c], N, mc.base[c], N))
                used.add(c)
            else:
                products.append((M, N, 0, 0, 0, 0, N, mc.base[c], N))
        keep_a = [int(x) in used for x in ma.block_sector]
        keep_b = [int(x) in used for x in mb.block_sector]
        self.a_gather = _exec.make_gather(
            _exec.gather_rows(src_struct, src_kind, sa2, "matrix", pa, ta, 0, keep_a))
        self.b_gather = _exec.make_gather(
            _exec.gather_rows(b_tensor.structure, "arena", sb2, "matrix", pb, tb, 0, keep_b))
        self.a_size = ma.size
        # the FP64 form reads a row-permuting A gather's source in place (the tensor-core
        # form keeps the packed A: its 128-row tiles would run half empty on split rows)
        direct = _direct_products(self.a_gather, products) if precision == "f64" else None
        self.a_direct = direct is not None
        self.deferred = False  # the consumer gather computes this link's skinny product
        if self.a_direct:
            products, self.a_gather, self.a_size = direct, None, 0
        self.gemm = _exec.GemmGroup(products, precision, tc_min_flops)
        self.ga = None  # the A gather and the GEMM as one launch (ChainProgram._fuse_gathers)
        self.c_struct = sc
        self.b_size, self.c_size = mb.size, mc.size
        self.b_tensor = b_tensor


class ChainProgram:
    """``y = chain(x)`` for a fixed input structure; see the module docstring."""

    def __init__(self, in_struct: TensorStructure, precision: str = "f64",
                 tc_min_flops: int | None = None, defer: bool = False) -> None:
        """``precision``: "f64" (the plain FP64 form), or "tf32" / "3xbf16" to run the
        coupled-sector products big enough to be dense contractions (at least
        ``tc_min_flops``, default ``_exec.TC_MIN_FLOPS``) on the tcgen05 tensor cores.
        ``defer``: let the gather that consumes a short-K link's product compute it where
        it reads it (``_exec.ProductGather``) instead of launching the GEMM.  Off by
        default: bit-identical and two launches fewer on heff2, but slower there (65.5
        against 57.4 us per SU(2) matvec on B200), because each product element is read
        by 2.4 gather terms on average and is recomputed for each."""
        self.precision = precision
        self.defer = defer
        self.tc_min_flops = tc_min_flops
        self.in_struct = in_struct
        self.src = (in_struct, "arena")
        self.pending = _identity_plan(in_struct)
        self.links: list[_Link] = []
        self._built = False

    # --- building -----------------------------------------------------------------------
    @property
    def structure(self) -> TensorStructure:
        return self.pending[0]

    def transpose(self, axes) -> ChainProgram:
        self.pending = chain(self.pending, transpose_plan(self.structure, tuple(axes)))
        return self

    def repartition(self, outputs, inputs) -> ChainProgram:
        self.pending = chain(self.pending, repartition_plan(self.structure, tuple(outputs),
                                                           tuple(inputs)))
        return self

    def contract(self, b: SymmetricTensor, axes, b_plan=None) -> ChainProgram:
        b_plan = b_plan or _identity_plan(b.structure)
        link = _Link(self.src[0], self.src[1], self.pending, b, b_plan, axes, self.precision,
                     self.tc_min_flops)
        self.links.append(link)
        self.src = (link.c_struct, "matrix")
        self.pending = link.after
        return self

    def einsum(self, equation: str, b: SymmetricTensor, bend: str = "") -> ChainProgram:
        """``einsum(equation, <chain>, b)`` with the wires in ``bend`` bent first on both
        operands (the reference's ``_composed``)."""
        lhs, out = equation.split("->")
        ta, tb = lhs.split(",")
        b_plan = _identity_plan(b.structure)
        if bend:
            flip = set(bend)
            s = self.structure
            outs = tuple(i for i, ch in enumerate(ta) if (s.legs[i].side is OUT) != (ch in flip))
            ins = tuple(i for i in range(len(ta)) if i not in outs)
            self.repartition(outs, ins)
            ta = "".join(ta[i] for i in (*outs, *ins))
            sb = b.structure
            bo = tuple(i for i, ch in enumerate(tb) if (sb.legs[i].side is OUT) != (ch in flip))
            bi = tuple(i for i in range(len(tb)) if i not in bo)
            b_plan = repartition_plan(sb, bo, bi)
            tb = "".join(tb[i] for i in (*bo, *bi))
        shared = [x for x in ta if x in tb]
        axes = (tuple(ta.index(x) for x in shared), tuple(tb.index(x) for x in shared))
        self.contract(b, axes, b_plan)
        free = [x for x in ta if x not in shared] + [x for x in tb if x not in shared]
        return self.transpose(tuple(free.index(x) for x in out))

    def finish(self, allocate: bool = True) -> ChainProgram:
        dst, perm, terms = self.pending
        self.out_struct = dst
        self.out_gather = _exec.make_gather(
            _exec.gather_rows(self.src[0], self.src[1], dst, "arena", perm, terms))
        if self.defer:
            self._defer_skinny()
        self.compact = self._compact()
        if not self.compact:
            self._fuse_gathers()
        if allocate:
            self.allocate()
        return self

    def _fuse_gathers(self) -> None:
        """Fold each link's A gather into its GEMM launch (``_exec.GatherAGemm``) when the
        link's products are FP64 with K <= ``_exec.GA_MAX_K``: the link becomes one launch
        and its packed A is never written."""
        if not _exec.FUSE_A or self.precision != "f64":
            return
        for lk in self.links:
            if lk.a_gather is None or lk.a_direct or lk.deferred or lk.gemm.tensor_core:
                continue
            if type(lk.a_gather) is not _exec.GatherTable or \
                    not _exec.GatherAGemm.eligible(lk.gemm.products):
                continue
            csr = _exec.gather_csr(lk.a_gather, lk.a_size)
            if csr is not None and _exec.GatherAGemm.fits(csr, lk.gemm.products):
                lk.ga = _exec.GatherAGemm(csr, lk.gemm.products, lk.a_size)

    def _compact(self) -> bool:
        """Whether every stage has at most ``_exec.CLUSTER_MAX_ITEMS`` work items (gather
        chunks, GEMM tiles per CTA-sized item) once split-K is off: such a chain runs as one
        launch on one thread-block cluster.  Its GEMM tables are then rebuilt without
        split-K, which only pays across many SMs."""
        if not _exec.CLUSTER or self.uses_tensor_cores or any(lk.deferred for lk in self.links):
            return False
        groups = [_exec.GemmGroup(lk.gemm.products, self.precision, self.tc_min_flops,
                                  split_k=False) for lk in self.links]
        items = [self.out_gather.chunks]
        for lk, gg in zip(self.links, groups):
            if lk.a_gather is not None:
                items.append(lk.a_gather.chunks)
            for part in gg.parts:
                if part.kind not in (_exec.TILE_64, _exec.TILE_32, _exec.TILE_SKINNY):
                    return False
                items.append(-(-part.tiles // 4) if part.kind == _exec.TILE_32 else part.tiles)
        if max(items) > _exec.CLUSTER_MAX_ITEMS:
            return False
        for lk, gg in zip(self.links, groups):
            lk.gemm = gg
        return True

    def _consumer(self, i: int):
        """The gather that reads link ``i``'s product, or None (a GEMM reads it)."""
        if i + 1 < len(self.links):
            nxt = self.links[i + 1]
            return None if nxt.a_direct else nxt.a_gather
        return self.out_gather

    def _set_consumer(self, i: int, g) -> None:
        if i + 1 < len(self.links):
            self.links[i + 1].a_gather = g
        else:
            self.out_gather = g

    def _defer_skinny(self) -> None:
        """Fold every link whose products all have K <= 4 (the MPO links) into the gather
        that consumes its product, when that gather's terms each read inside one product
        block (``_exec.product_gather``): one launch and one round trip of the product
        fewer per such link, bit-identical results."""
        for i, lk in enumerate(self.links):
            parts = lk.gemm.parts
            consumer = self._consumer(i)
            if len(parts) != 1 or consumer is None:
                continue
            pg = _exec.product_gather(consumer, parts[0])
            if pg is not None:
                lk.deferred = True
                self._set_consumer(i, pg)

    def rebind(self, operands: dict) -> ChainProgram:
        """A new program sharing this one's tables, with the fixed operands replaced by
        tensors of the same structures (``operands`` maps the names given at planning)."""
        import copy

        q = copy.copy(self)
        q.links = []
        for lk, name in zip(self.links, self.operand_names):
            t = operands[name]
            if t.structure != lk.b_tensor.structure:
                raise ValueError("ChainProgram.rebind: operand structure differs")
            nl = copy.copy(lk)
            nl.b_tensor = t
            q.links.append(nl)
        q._built = False
        return q

    def finish_alloc(self, allocate: bool) -> ChainProgram:
        if allocate:
            self.allocate()
        return self

    def allocate(self) -> None:
        """Allocate every buffer once and pack the fixed operands (needs the device)."""
        dev = _exec.device()
        f64 = dict(dtype=torch.float64, device=dev)
        # every table of the chain in one upload, made on the shared template's tables
        # (programs rebound from one template upload once; private copies share it)
        _exec.upload_together([t for lk in self.links
                               for t in ((lk.ga, lk.b_gather) if lk.ga is not None else
                                         (lk.a_gather, lk.b_gather, *lk.gemm.parts))]
                              + [self.out_gather])
        for lk in self.links:  # split-K scratch of this program's own
            lk.gemm = lk.gemm.private()
        self.a_bufs = [torch.empty(max(1, 0 if lk.ga is not None else lk.a_size), **f64)
                       for lk in self.links]
        self.c_bufs = [torch.empty(max(1, lk.c_size), **f64) for lk in self.links]
        self.b_bufs = [torch.empty(max(1, lk.b_size), **f64) for lk in self.links]
        # placeholder input/output: the recorded sequence reads and writes these, and a
        # replay substitutes the caller's vectors for them
        self.x_slot = torch.zeros(max(1, layout(self.in_struct).size), **f64)
        self.y_slot = torch.zeros(max(1, layout(self.out_struct).size), **f64)
        self.refresh()
        self.seq = _exec.Seq()
        with self.seq:
            self._run_tables(self.x_slot, self.y_slot)
        # the one-launch forms fuse a chunk-map recording of the same stages
        std = self.seq
        if _exec.CHAIN_DIRECT_GATHER:
            std = _exec.Seq()
            with _exec.standard_gathers(), std:
                self._run_tables(self.x_slot, self.y_slot)
        self._std_seq = std
        # the same stages as one persistent launch, when they all fuse (no tensor-core
        # stage, no product-source gather, at most the kernel's stage count)
        self.cluster = None
        if getattr(self, "compact", False) and _exec.CLUSTER and \
                0 < len(std) <= FUSED_MAX_STAGES:
            import ctypes

            from tenet import _lib

            cl, ctas = _exec.Seq(), ctypes.c_int32(0)
            _lib.call("tnb_seq_fuse_cluster", std.handle, self.x_slot.data_ptr(),
                      self.y_slot.data_ptr(), _exec.CLUSTER_CTAS, ctypes.byref(ctas),
                      cl.handle)
            self.cluster, self.cluster_ctas = cl, ctas.value
        self.fused = None
        if (not self.uses_tensor_cores and not any(lk.deferred for lk in self.links)
                and not any(lk.ga is not None for lk in self.links)
                and 0 < len(std) <= FUSED_MAX_STAGES):
            from tenet import _lib

            self.barrier = torch.zeros(2, dtype=torch.int32, device=dev)
            fused = _exec.Seq()
            _lib.call("tnb_seq_fuse", std.handle, self.x_slot.data_ptr(),
                      self.y_slot.data_ptr(), self.barrier.data_ptr(), fused.handle)
            self.fused = fused
        self._built = True

    @property
    def exec_seq(self) -> _exec.Seq:
        """The sequence a replay runs: the one-cluster launch of a compact chain (when
        ``_exec.CLUSTER``), the grid-wide fused launch (when ``_exec.FUSE``), else the
        stage-by-stage sequence."""
        if self.cluster is not None and _exec.CLUSTER:
            return self.cluster
        return self.fused if (self.fused is not None and _exec.FUSE) else self.seq

    def refresh(self) -> None:
        """Re-pack the fixed operands (after their values changed, same structures)."""
        for lk, buf in zip(self.links, self.b_bufs):
            lk.b_gather.run(lk.b_tensor.arena, buf)

    # --- running ------------------------------------------------------------------------
    @property
    def flops(self) -> int:
        return sum(lk.gemm.flops for lk in self.links)

    @property
    def launches(self) -> int:
        if getattr(self, "cluster", None) is not None and _exec.CLUSTER:
            return 1
        return sum(1 if lk.ga is not None else
                   (0 if lk.deferred else lk.gemm.launches) + (not lk.a_direct)
                   for lk in self.links) + 1

    @property
    def uses_tensor_cores(self) -> bool:
        return any(lk.gemm.tensor_core for lk in self.links)

    def tensor_core_candidates(self, min_flops: int | None = None) -> bool:
        """Whether the precision form of this chain would put any product on the tensor
        cores (``_exec.tc_worthy``)."""
        return any(_exec.tc_worthy(p, min_flops)
                   and not _exec._is_skinny(p, _exec.thin_rows(lk.gemm.products))
                   and not _exec._is_wide(p, _exec.wide_cols(lk.gemm.products))
                   for lk in self.links for p in lk.gemm.products)

    def run(self, x: torch.Tensor, out: torch.Tensor) -> torch.Tensor:
        """``out = chain(x)`` on the current stream: one replay of the recorded stages (or
        of the fused one-launch chain when ``_exec.FUSE`` is on; launch by launch while a
        ``LaunchLog`` times each kernel).  One program must not run on two streams at
        once."""
        if _exec._LOG is None and _exec.recording() is None:
            self.exec_seq.run({self.x_slot.data_ptr(): x.data_ptr(),
                               self.y_slot.data_ptr(): out.data_ptr()})
            return out
        return self._run_tables(x, out)

    def _run_tables(self, x: torch.Tensor, out: torch.Tensor) -> torch.Tensor:
        src, pending = x, None  # pending: the operands of a deferred link's product
        for lk, ab, bb, cb in zip(self.links, self.a_bufs, self.b_bufs, self.c_bufs):
            if lk.ga is not None:
                lk.ga.run(src, bb, cb)
                src = cb
                continue
            a = src if lk.a_direct else ab
            if isinstance(lk.a_gather, _exec.ProductGather):
                lk.a_gather.run(*pending, ab)
            elif not lk.a_direct:
                lk.a_gather.run(src, ab)
            if lk.deferred:
                pending = (a, bb)
            else:
                lk.gemm.run(a, bb, cb)
            src = cb
        if isinstance(self.out_gather, _exec.ProductGather):
            self.out_gather.run(*pending, out)
        else:
            self.out_gather.run(src, out)
        return out

    def __call__(self, x: SymmetricTensor) -> SymmetricTensor:
        if x.structure != self.in_struct:
            raise ValueError("ChainProgram: input structure differs from the compiled one")
        out = SymmetricTensor.empty(self.out_struct)
        self.run(x.arena, out.arena)
        return out


class _Mapped:
    """A pinned host tensor seen through its kernel address (``_lib.mapped_address``):
    the two methods a chain program's ``run`` reads of its output."""

    __slots__ = ("_ptr", "_n")

    def __init__(self, host: torch.Tensor) -> None:
        self._ptr, self._n = _lib.mapped_address(host.data_ptr()), host.numel()

    def data_ptr(self) -> int:
        return self._ptr

    def numel(self) -> int:
        return self._n


class GraphMatvec:
    """A ``ChainProgram`` captured in a CUDA graph: copy in, replay, copy out.

    With ``host_io`` the graph also moves the data between pinned host buffers and the
    device: ``host_x`` -> device, the chain, the result -> ``host_y``, so a host caller
    pays one graph launch per matvec (``replay_host``).  ``host_copy`` "kernel" reads
    ``host_x`` with a copy kernel (``tnb_copy_f64``) and lets the chain's last gather
    write its result straight into ``host_y`` through the buffer's mapped address
    (every output element is written once); "dma" uses the copy engines
    (``cudaMemcpyAsync``) both ways."""

    def __init__(self, program: ChainProgram, warmup: int = 2, host_io: bool = False,
                 host_copy: str = "kernel") -> None:
        if host_copy not in ("kernel", "dma"):
            raise ValueError(f"GraphMatvec: host_copy {host_copy!r} is not 'kernel' or 'dma'")
        self.program = program
        dev = _exec.device()
        self.x = torch.zeros(layout(program.in_struct).size, dtype=torch.float64, device=dev)
        self.y = torch.empty(layout(program.out_struct).size, dtype=torch.float64, device=dev)
        self.host_x = self.host_y = None
        if host_io:
            self.host_x = torch.zeros(self.x.numel(), dtype=torch.float64).pin_memory()
            self.host_y = torch.zeros(self.y.numel(), dtype=torch.float64).pin_memory()

        def move(src, dst):
            if host_copy == "kernel":
                _lib.call("tnb_copy_f64", src.numel(), src.data_ptr(), dst.data_ptr(),
                          _exec.stream_ptr())
            else:
                dst.copy_(src, non_blocking=True)

        direct_out = host_io and host_copy == "kernel"
        out = _Mapped(self.host_y) if direct_out else self.y

        def body():
            if host_io:
                move(self.host_x, self.x)
            program.run(self.x, out)
            if host_io and not direct_out:
                move(self.y, self.host_y)

        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            for _ in range(warmup):
                body()
        torch.cuda.current_stream().wait_stream(side)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            body()

    def __call__(self, x: SymmetricTensor) -> SymmetricTensor:
        self.x.copy_(x.arena)
        self.graph.replay()
        return SymmetricTensor(self.program.out_struct, arena=self.y.clone())

    def replay(self) -> None:
        self.graph.replay()

    def replay_host(self) -> torch.Tensor:
        """``host_y`` = H ``host_x`` (host_io graphs): enqueue on the current stream; the
        result is in ``host_y`` once the stream reaches this point."""
        if self.host_x is None:
            raise ValueError("GraphMatvec.replay_host: built without host_io")
        self.graph.replay()
        return self.host_y


_HEFF_TABLES: dict = {}
_HEFF_TABLES_MAX = 512


def heff2_program(fl, w1, w2, fr, in_struct: TensorStructure, allocate: bool = True,
                  precision: str = "f64", tc_min_flops: int | None = None,
                  defer: bool = False) -> ChainProgram:
    """The site-tensor two-site matvec (``network/env.py:416-432``) as a chain program.
    ``fl``, ``w1``, ``w2``, ``fr`` need only ``.structure`` when ``allocate`` is False.

    The program's tables depend on the five structures and the precision only, so they
    are planned once per such key and shared: a later call with the same structures
    builds a fresh program (own buffers, bound to the given tensors) around them."""
    key = (fl.structure, w1.structure, w2.structure, fr.structure, in_struct, precision,
           tc_min_flops, defer)
    cached = _HEFF_TABLES.get(key)
    if cached is not None:
        return cached.rebind(dict(zip(cached.operand_names, (fr, w2, w1, fl)))) \
            .finish_alloc(allocate)
    p = ChainProgram(in_struct, precision, tc_min_flops, defer)
    p.einsum("apqr,rys->apqys", fr)
    p.einsum("apqys,mQqy->apQms", w2, bend="q")
    p.einsum("apQms,xPpm->aPQxs", w1, bend="p")
    p.einsum("aPQxs,axB->BPQs", fl, bend="a")
    p.operand_names = ("fr", "w2", "w1", "fl")
    p.finish(False)
    bound = dict(zip(p.operand_names, (fr, w2, w1, fl)))
    for lk in p.links:  # the shared template keeps structures, never device tensors
        lk.b_tensor = _StructureOnly(lk.b_tensor.structure)
    if len(_HEFF_TABLES) >= _HEFF_TABLES_MAX:
        _HEFF_TABLES.pop(next(iter(_HEFF_TABLES)))
    _HEFF_TABLES[key] = p
    return p.rebind(bound).finish_alloc(allocate)


def heff2_folded_program(lf, rf, in_struct: TensorStructure, allocate: bool = True,
                         precision: str = "f64", tc_min_flops: int | None = None) -> ChainProgram:
    """The two-site matvec with each MPO site folded into its environment: ``rf =
    W[n+1] . F[(n+2, n+1)]`` on ``(m, Q, q, r, s)`` and ``lf = F[(n-1, n)] . W[n]`` on
    ``(a, B, P, p, m)`` (``network.fold_right`` / ``fold_left``, formed once per
    environment), then ``H aa = (aa . rf) . lf``: two contractions instead of four.

    The same operator as ``heff2_program`` (the reference's four-contraction order,
    ``network/env.py:416-432``), with the sums associated differently -- the reference's
    prepared path (``env.py:158-325``) also folds the environments before applying the
    operator.  It trades about 1.8x the GEMM flops for half the launches: the two MPO
    links (K <= 3, bandwidth-bound) and their gathers disappear, and the two remaining
    products have K of a whole bond times a physical leg.  Tables are shared per
    structure key as in ``heff2_program``."""
    key = ("folded", lf.structure, rf.structure, in_struct, precision, tc_min_flops)
    cached = _HEFF_TABLES.get(key)
    if cached is not None:
        return cached.rebind(dict(zip(cached.operand_names, (rf, lf)))).finish_alloc(allocate)
    p = ChainProgram(in_struct, precision, tc_min_flops)
    p.einsum("apqr,mQqrs->apmQs", rf)
    p.einsum("apmQs,aBPpm->BPQs", lf)
    p.operand_names = ("rf", "lf")
    p.finish(False)
    if p.out_struct != in_struct:
        raise ValueError("heff2_folded_program: the folded operands do not map the two-site "
                         "space to itself")
    bound = dict(zip(p.operand_names, (rf, lf)))
    for lk in p.links:
        lk.b_tensor = _StructureOnly(lk.b_tensor.structure)
    if len(_HEFF_TABLES) >= _HEFF_TABLES_MAX:
        _HEFF_TABLES.pop(next(iter(_HEFF_TABLES)))
    _HEFF_TABLES[key] = p
    return p.rebind(bound).finish_alloc(allocate)
