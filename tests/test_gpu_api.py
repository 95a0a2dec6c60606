"""The drop-in API around the sweep: ``spin_half(SU2)``, ``MPO.from_terms``,
``dmrg_``'s reference arguments and record, the two-state environment."""

import json

import numpy as np
import pytest

import tenet
from tenet import models, network
from tenet.structure import GradedSpace
from tenet.symmetry import SU2

pytestmark = pytest.mark.gpu


class _Site:
    """``spin_half(SU2)``, built on first use (its operator lives on the device)."""

    def __getattr__(self, name):
        site = models.spin_half(SU2)
        self.phys, self.ops, self.matrices = site
        return getattr(site, name)


SITE = _Site()


def _equal_mpo(a, b):
    assert len(a) == len(b)
    for x, y in zip(a.sites, b.sites):
        assert x.structure == y.structure
        np.testing.assert_allclose(x.numpy_arena(), y.numpy_arena(), rtol=0, atol=1e-15)


def test_from_terms_builds_the_chain_mpo():
    op = SITE.ops["S.S"]
    L = 10
    h = network.MPO.from_terms(L, [(1.0, [(op, (i, i + 1))]) for i in range(L - 1)])
    _equal_mpo(h, network.heisenberg_mpo_su2(L))
    terms = [(1.0, [(op, (i, i + 1))]) for i in range(L - 1)]
    terms += [(0.3, [(op, (i, i + 2))]) for i in range(L - 2)]
    _equal_mpo(network.MPO.from_terms(L, terms), network.heisenberg_mpo_su2(L, 1.0, 0.3))
    with pytest.raises(ValueError, match="neighbours"):
        network.MPO.from_terms(L, [(1.0, [(op, (0, 3))])])


def test_su2_example_script_runs_unchanged_in_its_su2_half(golden_dir):
    """``examples/su2_heisenberg.py``'s SU(2) run, spelled as it spells it (its U(1) half
    is out of this build), against the MPSKit N = 20 SU(2) energy the reference's own
    fixture validates."""
    from tenet.network import MPO, MPS, dmrg_
    from tenet.symmetry import SU2Sector

    def su2_mpo(n_sites):
        op = SITE.ops["S.S"]
        return MPO.from_terms(n_sites, [(1.0, [(op, (i, i + 1))]) for i in range(n_sites - 1)])

    def bond_spaces(n_sites):
        tri = GradedSpace.new(SU2, {SU2Sector(0): 1})
        mid = GradedSpace.new(SU2, {SU2Sector(0): 2, SU2Sector(1): 2, SU2Sector(2): 1})
        return [tri] + [mid] * (n_sites - 1) + [tri]

    n_sites, chi = 20, 64
    psi = MPS.random(SITE.phys, bond_spaces(n_sites), seed=0)
    su2 = dmrg_(psi, su2_mpo(n_sites), chi=chi)
    assert isinstance(su2, network.DMRG_out) and su2.psi is psi
    assert su2.energy == pytest.approx(-8.682473334399202, abs=1e-9)
    assert len(su2.history) == su2.sweeps == len(su2.schedule)
    mid = su2.psi[n_sites // 2].legs[0].space
    assert sum((a.two_j + 1) * m for a, m in mid.sectors) <= chi


def test_dmrg_schedule_callback_and_refusals():
    L = 8
    h = network.heisenberg_mpo_su2(L)
    phys = SITE.phys
    bonds = [GradedSpace.new(SU2, {SU2.sector(j): 1 for j in range(i % 2, min(i, L - i) + 1, 2)})
             for i in range(L + 1)]
    seen = []
    sched = [network.Sweep(8, 1e-10, noise=1e-4), network.Sweep(16, 1e-12)]
    out = network.dmrg_(network.MPS.random(phys, bonds, seed=0), h, schedule=sched, ncv=8,
                        max_sweeps=6, callback=lambda o: seen.append(o.sweeps))
    assert seen == list(range(1, out.sweeps + 1))
    assert out.schedule[0] == sched[0] and all(s == sched[1] for s in out.schedule[1:])
    with pytest.raises(ValueError, match="not both"):
        network.dmrg_(network.MPS.random(phys, bonds, seed=0), h, schedule=sched, chi=8)
    with pytest.raises(ValueError, match="empty"):
        network.dmrg_(network.MPS.random(phys, bonds, seed=0), h, schedule=[])
    with pytest.raises(ValueError, match="noise_type"):
        network.dmrg_(network.MPS.random(phys, bonds, seed=0), h,
                      schedule=[network.Sweep(8, noise=1e-4, noise_type="other")])


def test_excited_state_is_orthogonal_to_the_ground_state():
    L = 8
    h = network.heisenberg_mpo_su2(L)
    bonds = [GradedSpace.new(SU2, {SU2.sector(j): 1 for j in range(i % 2, min(i, L - i) + 1, 2)})
             for i in range(L + 1)]
    g = network.dmrg_(network.MPS.random(SITE.phys, bonds, seed=0), h, chi=64, ncv=12)
    e = network.dmrg_(network.MPS.random(SITE.phys, bonds, seed=1), h, chi=64, ncv=12,
                      orthogonal_to=[g.psi], max_sweeps=20)
    assert e.energy > g.energy + 1e-3
    # the overlap through a two-state environment over the identity MPO
    env = network.Env(g.psi, network.MPO.identity(L, SITE.phys), bra=e.psi).setup_(0)
    pair = tenet.einsum("apx,xqr->apqr", g.psi[0], g.psi[1])
    bb = tenet.einsum("apx,xqr->apqr", e.psi[0], e.psi[1])
    assert abs(float(tenet.inner(env.project2(0, pair), bb))) < 1e-8


def test_canonize_leaves_right_orthonormal_sites():
    """``canonize_``: each site n >= 1 is a right isometry on the bond of min(rows, cols)
    per sector, and the state is normalised on site 0."""
    from tenet import ops

    L = 10
    bonds = [GradedSpace.new(SU2, {SU2.sector(j): 1 + (j % 3)
                                   for j in range(i % 2, min(i, L - i) + 1, 2)})
             for i in range(L + 1)]
    psi = network.MPS.random(SITE.phys, bonds, seed=3)
    psi.canonize_(0)
    for n in range(1, L):
        q = ops.repartition(psi[n], (0,), (1, 2))
        eye = ops.identity((q.legs[0],))
        got = ops.compose(q, ops.adjoint(q))
        assert got.structure == eye.structure
        np.testing.assert_allclose(got.numpy_arena(), eye.numpy_arena(), atol=1e-13)
    assert abs(ops.norm(psi[0]) - 1.0) < 1e-12
