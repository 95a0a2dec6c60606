"""``SymmetricTensor``: a structure plus one HBM arena holding every block.

The reference stores ``blocks`` as a tuple of independent backend arrays
(``tensor.py:60-112``).  Here all blocks of a tensor live in one contiguous FP64 CUDA
buffer (the *arena*), in ``structure.block_order``, each block C-contiguous in public
axis order; ``blocks`` hands out torch views into it, so code written against the
reference's block tuple keeps working while every kernel sees one pointer plus the
structure's offset table.
"""

from __future__ import annotations

from typing import Any

import numpy as np
import torch

from tenet import _exec
from tenet.structure import TensorStructure, layout

__all__ = ["SymmetricTensor"]


class SymmetricTensor:
    __slots__ = ("structure", "arena")

    def __init__(self, structure: TensorStructure, blocks: Any = None, *, arena=None) -> None:
        if not isinstance(structure, TensorStructure):
            structure = TensorStructure(tuple(structure))
        lay = layout(structure)
        if arena is None:
            blocks = tuple(blocks) if blocks is not None else ()
            if len(blocks) != len(lay.sizes):
                raise ValueError(f"expected {len(lay.sizes)} blocks, got {len(blocks)}")
            for i, b in enumerate(blocks):
                if tuple(b.shape) != tuple(int(x) for x in lay.shapes[i]):
                    raise ValueError(f"block {i} has shape {tuple(b.shape)}, expected "
                                     f"{tuple(int(x) for x in lay.shapes[i])}")
            dev = _exec.device()
            if blocks:
                flat = [torch.as_tensor(b).reshape(-1) for b in blocks]
                arena = torch.cat([f.to(device=dev, dtype=torch.float64) for f in flat])
            else:
                arena = torch.zeros(0, dtype=torch.float64, device=dev)
        else:
            if arena.dim() != 1 or arena.numel() != lay.size:
                raise ValueError(f"arena has {arena.numel()} elements, structure needs {lay.size}")
            if arena.dtype != torch.float64 or not arena.is_cuda:
                raise ValueError("the arena must be a CUDA float64 tensor")
        self.structure = structure
        self.arena = arena

    # --- constructors -----------------------------------------------------------------
    @classmethod
    def from_arena(cls, structure: TensorStructure, arena: torch.Tensor) -> SymmetricTensor:
        return cls(structure, arena=arena)

    @classmethod
    def empty(cls, structure: TensorStructure) -> SymmetricTensor:
        return cls(structure, arena=torch.empty(layout(structure).size, dtype=torch.float64,
                                                device=_exec.device()))

    @classmethod
    def zeros(cls, legs, dtype=None) -> SymmetricTensor:
        s = legs if isinstance(legs, TensorStructure) else TensorStructure(tuple(legs))
        return cls(s, arena=torch.zeros(layout(s).size, dtype=torch.float64,
                                        device=_exec.device()))

    @classmethod
    def random(cls, legs, *, seed: int | None = None, dtype=None) -> SymmetricTensor:
        """Standard-normal blocks from ``np.random.default_rng(seed)``, one draw per block
        in block order -- the reference's stream exactly (``tensor.py:232-262``), so a
        seeded tensor here holds the same numbers as the reference's."""
        s = legs if isinstance(legs, TensorStructure) else TensorStructure(tuple(legs))
        lay = layout(s)
        rng = np.random.default_rng(seed)
        host = np.empty(lay.size, dtype=np.float64)
        for b in range(len(lay.sizes)):
            o, n = int(lay.offsets[b]), int(lay.sizes[b])
            host[o:o + n] = rng.standard_normal(tuple(int(x) for x in lay.shapes[b])).ravel()
        return cls(s, arena=torch.from_numpy(host).to(_exec.device()))

    @classmethod
    def from_numpy_arena(cls, structure: TensorStructure, host: np.ndarray) -> SymmetricTensor:
        return cls(structure, arena=torch.from_numpy(np.ascontiguousarray(host, np.float64))
                   .to(_exec.device()))

    # --- views ------------------------------------------------------------------------
    @property
    def blocks(self) -> tuple:
        lay = layout(self.structure)
        return tuple(self.arena[int(o):int(o) + int(n)].view(*(int(x) for x in sh))
                     for o, n, sh in zip(lay.offsets, lay.sizes, lay.shapes))

    def items(self):
        return zip(self.structure.block_order, self.blocks)

    def block(self, key):
        return self.blocks[self.structure.index_of(key)]

    @property
    def legs(self) -> tuple:
        return self.structure.legs

    @property
    def ndim(self) -> int:
        return self.structure.ndim

    @property
    def provider(self):
        return self.structure.provider

    @property
    def codomain(self) -> tuple:
        return self.structure.codomain

    @property
    def domain(self) -> tuple:
        return self.structure.domain

    @property
    def dtype(self):
        return self.arena.dtype

    @property
    def device(self):
        return self.arena.device

    @property
    def backend(self) -> str:
        return "torch"

    @property
    def shape(self) -> tuple[int, ...]:
        return tuple(leg.space.dim for leg in self.legs)

    @property
    def reduced_shape(self) -> tuple[int, ...]:
        return tuple(leg.space.reduced_dim for leg in self.legs)

    def numpy_arena(self) -> np.ndarray:
        return self.arena.detach().cpu().numpy()

    def copy(self) -> SymmetricTensor:
        return SymmetricTensor(self.structure, arena=self.arena.clone())

    # --- operator sugar ---------------------------------------------------------------
    def transpose(self, *axes):
        from tenet import ops

        if len(axes) == 1 and not isinstance(axes[0], int):
            axes = tuple(axes[0])
        return ops.transpose(self, axes or None)

    def repartition(self, outputs, inputs):
        from tenet import ops

        return ops.repartition(self, outputs, inputs)

    def adjoint(self):
        from tenet import ops

        return ops.adjoint(self)

    def conj(self):
        return self  # real FP64 blocks

    def norm(self):
        from tenet import ops

        return ops.norm(self)

    def __add__(self, other):
        from tenet import ops

        return ops.add(self, other)

    def __sub__(self, other):
        from tenet import ops

        return ops.subtract(self, other)

    def __neg__(self):
        from tenet import ops

        return ops.multiply(self, -1.0)

    def __mul__(self, s):
        from tenet import ops

        return ops.multiply(self, s)

    __rmul__ = __mul__

    def __truediv__(self, s):
        from tenet import ops

        return ops.divide(self, s)

    def __matmul__(self, other):
        from tenet import ops

        return ops.compose(self, other)

    def __repr__(self) -> str:
        return f"SymmetricTensor(ndim={self.ndim}, blocks={self.structure.num_blocks}, " \
               f"elements={self.arena.numel()})"
