"""tenet (B200 build): block-sparse symmetric tensors with every block op on sm_100a.

A drop-in for the hot path of TeNeT-py's ``tenet`` package: the same ``SymmetricTensor``
/ ``einsum`` / ``tensordot`` / ``linalg.svd_truncated`` API, blocks held in one CUDA
arena per tensor, and the per-block execution loops replaced by the kernels of
``libtenet_b200.so`` (declared in ``include/tenet_b200.h``).  There is no CPU execution
path; the host only plans.
"""

from tenet import linalg, network, symmetry
from tenet.serialize import load, save
from tenet.ops import add, adjoint, block_sqrt, compose, contractible, divide, einsum, inner, multiply, \
    norm, outward_dual, repartition, subtract, tensordot, transpose
from tenet.structure import IN, OUT, FusionBlockKey, FusionTree, GradedSpace, Leg, Side, \
    TensorStructure
from tenet.tensor import SymmetricTensor

__all__ = [
    "IN", "OUT", "FusionBlockKey", "FusionTree", "GradedSpace", "Leg", "Side",
    "SymmetricTensor", "TensorStructure", "add", "adjoint", "block_sqrt", "compose", "contractible",
    "divide", "einsum", "inner", "linalg", "load", "multiply", "network", "norm",
    "outward_dual", "repartition", "save", "subtract", "symmetry", "tensordot", "transpose",
]
