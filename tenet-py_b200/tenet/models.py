"""Site definitions (``models/sites.py``): the spin-1/2 site graded by SU(2).

``spin_half(SU2)`` returns the reference's ``Site``: the physical space (one ``j = 1/2``
multiplet), its operator set -- under SU(2) the invariant two-site ``S.S`` alone, as a
rank-4 tensor (``models/sites.py:121-195``) -- and the dense matrices.  The U(1) grading
of the reference (rank-3 charge-leg ``Sz``, ``S+``, ``S-``) is not part of this build.
"""

from __future__ import annotations

from typing import NamedTuple

import numpy as np

__all__ = ["Site", "spin_half"]

_SZ = np.diag([0.5, -0.5])
_SP = np.array([[0.0, 1.0], [0.0, 0.0]])
_SS = (np.kron(_SZ, _SZ) + 0.5 * (np.kron(_SP, _SP.T) + np.kron(_SP.T, _SP)))


class Site(NamedTuple):
    """A physical site: its graded space, operators as tensors, and dense matrices."""

    phys: object
    ops: dict
    matrices: dict


def spin_half(symmetry=None) -> Site:
    """The spin-1/2 site graded by ``SU2`` (one ``j = 1/2`` multiplet): ``ops["S.S"]`` is
    the invariant two-site Heisenberg term that ``MPO.from_terms`` splits."""
    from tenet.network import local_op
    from tenet.structure import GradedSpace
    from tenet.symmetry import SU2

    if symmetry is not SU2:
        raise ValueError("spin_half: this build ships the SU2 grading; pass tenet.symmetry.SU2")
    phys = GradedSpace.new(SU2, {SU2.sector(1): 1})
    return Site(phys, {"S.S": local_op(_SS, phys=phys)}, {"S.S": _SS.copy()})
