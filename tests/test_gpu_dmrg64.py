"""SU(2) Heisenberg DMRG at L = 64, chi = 256 on the GPU against the reference's own run.

The reference's ``dmrg_`` (``network/dmrg.py:620-843``) was run on the same seeded start
(bond spins 2j <= min(i, L - i, 16), ``MPS.random`` seed 0), ``chi = 256`` in its dense
sense, cutoff 1e-10, ncv = 20, at most 10 sweeps with its default convergence tolerances,
and recorded in ``tests/golden/dmrg64.json`` (``make_golden.py ... dmrg64``).  Here the
whole solve runs on the device -- graph-captured matvecs, device-resident Lanczos, the
GPU SVD -- and must stop at the same sweep with the same per-sweep energies, the same
kept bond space at every bond, and an energy per site within 1e-8 of the MPSKit value the
reference's own integration test reads (``tests/integration/test_dmrg.py:88``).
"""

import json

import pytest

from tenet import network
from tenet.structure import GradedSpace
from tenet.symmetry import SU2

pytestmark = pytest.mark.gpu


def _start(g):
    L = g["L"]
    phys = GradedSpace.new(SU2, {SU2.sector(1): 1})
    bonds = [GradedSpace.new(SU2, {SU2.sector(j): 1
                                   for j in range(i % 2, min(i, L - i, g["max_2j"]) + 1, 2)})
             for i in range(L + 1)]
    return network.MPS.random(phys, bonds, seed=0)


@pytest.fixture(scope="module")
def golden(golden_dir):
    return json.loads((golden_dir / "dmrg64.json").read_text())


@pytest.mark.parametrize("fold", [True, False])
def test_dmrg_su2_L64_chi256_matches_reference(golden, fold):
    """Same number of sweeps, every bond's kept space identical after every sweep, each
    sweep's energy within 1e-8 per site (the first sweeps grow the bonds with Lanczos at
    ncv = 20 without reorthogonalisation, whose Ritz values move at the 1e-7 relative
    level with the matvec's summation order -- measured alike for a host-driven
    recurrence with the reference's own operation order), the converged energy within
    1e-10 relative."""
    g, site = golden, golden["site"]
    L = g["L"]
    psi = _start(g)
    seen = []
    out = network.dmrg_(psi, network.heisenberg_mpo_su2(L), chi=g["chi"], cutoff=g["cutoff"],
                        ncv=g["ncv"], max_sweeps=g["max_sweeps"], fold=fold,
                        callback=lambda o: seen.append(
                            [[[SU2.label(a), k] for a, k in o.psi[i].legs[0].space.sectors]
                             for i in range(L)]))
    assert out.sweeps == site["sweeps"]
    for got, want in zip(out.history, site["history"]):
        assert abs(got[0] - want[0]) / L <= 1e-8
    assert out.energy == pytest.approx(site["energy"], rel=1e-10)
    for k, (got, want) in enumerate(zip(seen, site["bonds_per_sweep"])):
        assert got == want, f"kept bond sectors differ from the reference's after sweep {k + 1}"
    assert abs(out.energy - g["prepared"]["energy"]) / L <= 1e-10
    assert abs(out.energy - g["mpskit_N64_chi256"]) / L <= 1e-8


@pytest.mark.parametrize("precision", ["3xbf16", "tf32"])
def test_dmrg_su2_L64_precision_form_within_1e8_per_site(golden, precision):
    """The precision form through the same solve: tensor-core matvec products, FP64
    Lanczos orthogonalisation, correction, SVD and truncation."""
    g = golden
    L = g["L"]
    out = network.dmrg_(_start(g), network.heisenberg_mpo_su2(L), chi=g["chi"],
                        cutoff=g["cutoff"], ncv=g["ncv"], max_sweeps=g["max_sweeps"],
                        precision=precision)
    assert abs(out.energy - g["site"]["energy"]) / L <= 1e-8
