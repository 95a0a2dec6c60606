"""The oracle against the reference's own outputs (golden vectors) and F/R fixtures.

These pins are what make the oracle trustworthy as the checker of the CUDA path: every
case in ``tests/golden`` was produced by running the reference itself
(``tests/golden/make_golden.py``), and the oracle must reproduce its block keys exactly and
its values to 1e-12 relative (in practice it is bit-identical on every transpose, bend and
contraction case).
"""

import json

import numpy as np
import pytest

import oracle.tenet_oracle as O
from oracle import racah_su2


def _load(meta, arrays, d):
    s = O.structure_from_json(d["legs"])
    assert O.block_order(s) == O.keys_from_json(d["keys"]), "block keys differ from the reference"
    return O.from_arena(s, arrays[d["arena"]])


@pytest.fixture(scope="module")
def cases(golden_dir):
    return json.loads((golden_dir / "cases.json").read_text()), np.load(golden_dir / "cases.npz")


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)) if b.size else 0.0


def test_every_case_matches_reference(cases):
    meta, arrays = cases
    seen = 0
    for c in meta["cases"]:
        ops = [_load(meta, arrays, d) for d in c["operands"]]
        a, op = c["args"], c["op"]
        if op == "einsum":
            out = O.einsum(a["equation"], *ops)
        elif op == "transpose":
            out = O.transpose(ops[0], a["axes"])
        elif op == "repartition":
            out = O.repartition(ops[0], a["outputs"], a["inputs"])
        elif op == "tensordot":
            out = O.tensordot(ops[0], ops[1], a["axes"])
        elif op == "inner":
            assert O.inner(*ops) == pytest.approx(a["value"], rel=1e-12)
            continue
        elif op == "norm":
            assert O.norm(*ops) == pytest.approx(a["value"], rel=1e-12)
            continue
        elif op == "svd_truncated":
            _, s, _ = O.svd_truncated(ops[0], a["axes"], max_bond=a["max_bond"], cutoff=a["cutoff"])
            exp = _load(meta, arrays, c["output"])
            assert s.structure == exp.structure
            assert _rel(s.arena(), exp.arena()) < 1e-12
            assert [list(x) for x in s.structure.legs[0].sectors] == a["bond"]
            continue
        else:
            continue
        exp = _load(meta, arrays, c["output"])
        assert out.structure == exp.structure, c["name"]
        assert exp.arena().size > 0
        assert _rel(out.arena(), exp.arena()) < 1e-12, c["name"]
        seen += 1
    assert seen >= 15


def test_heff2_lanczos_svd_match_reference(golden_dir):
    m = json.loads((golden_dir / "heff.json").read_text())
    h = np.load(golden_dir / "heff.npz")
    aa, fl, fr, w1, w2, ex = (_load(m, h, m[k]) for k in ("aa", "fl", "fr", "w1", "w2", "heff_aa"))
    out = O.heff2(fl, w1, w2, fr, aa)
    assert out.structure == ex.structure
    assert _rel(out.arena(), ex.arena()) < 1e-12
    e, v = O.lanczos(lambda x: O.heff2(fl, w1, w2, fr, x), aa, ncv=20)
    assert e == pytest.approx(m["lanczos_ncv20_energy"], rel=1e-12)
    _, s, _ = O.svd_truncated(v, ((0, 1), (2, 3)), max_bond=16, cutoff=1e-10)
    assert [list(x) for x in s.structure.legs[0].sectors] == m["svd_bond"]


def test_config1_keys_and_checksums(golden_dir):
    """Full-size U(1) config: operands regenerated from their seeds, result checksummed."""
    g = json.loads((golden_dir / "config1.json").read_text())
    sec = tuple((q, d) for q, d in g["degeneracies"])
    V = lambda side: O.Leg(sec, side)  # noqa: E731
    A = O.random(O.Structure(O.U1, (V(O.OUT),) * 4), 0)
    B = O.random(O.Structure(O.U1, (V(O.IN), V(O.IN), V(O.OUT), V(O.OUT))), 1)
    C = O.einsum(g["equation"], A, B)
    assert O.block_order(C.structure) == O.keys_from_json(g["keys"])
    probe = np.random.default_rng(g["checksum_seed"])
    for blk, (s, ss, pr) in zip(C.blocks, g["blocks_sum_sumsq_probe"]):
        x = blk.ravel()
        w = probe.standard_normal(x.size)
        assert float(x.sum()) == pytest.approx(s, rel=1e-10, abs=1e-9)
        assert float((x * x).sum()) == pytest.approx(ss, rel=1e-12)
        assert float(w @ x) == pytest.approx(pr, rel=1e-10, abs=1e-9)


def test_su2_f_symbols_match_fixture_sample(golden_dir):
    """F-symbols against the reference's TensorKitSectors fixture (every 37th row)."""
    rows = [r.split() for r in (golden_dir / "su2_f_sample.txt").read_text().splitlines()
            if not r.startswith("#")]
    assert len(rows) > 2900
    worst = 0.0
    for r in rows:
        dj = tuple(int(x) for x in r[:6])
        got = racah_su2.f_symbol(*dj)
        worst = max(worst, abs(got - float(r[6])), abs(got - float(r[7])))
    assert worst <= 1e-13


def test_su2_r_and_frobenius_schur():
    assert racah_su2.r_symbol(1, 1, 0) == -1 and racah_su2.r_symbol(1, 1, 2) == 1
    assert [racah_su2.frobenius_schur(j) for j in range(5)] == [1, -1, 1, -1, 1]
    # CG orthonormality, j <= 3
    for a in range(0, 5):
        for b in range(0, 5):
            rows = [racah_su2.cg_tensor(a, b, c)[..., 0].reshape(-1, c + 1)
                    for c in range(abs(a - b), a + b + 1, 2)]
            m = np.concatenate(rows, axis=1)
            assert np.allclose(m.T @ m, np.eye(m.shape[1]), atol=1e-14)


def test_ctmrg_matches_reference(golden_dir):
    """Z2 Ising CTMRG: sweeps, per-sweep spectrum change, corner spectrum, bond split and
    the free-energy estimate against the reference's own runs."""
    g = json.loads((golden_dir / "ctmrg.json").read_text())
    for name in ("b044_chi16", "b040_chi16"):
        r = g[name]
        bs = O.structure_from_json(r["bulk"]["legs"])
        bulk = O.from_arena(bs, np.array(r["bulk"]["arena"]))
        c, e, bond, hist = O.ctmrg(bulk, chi=r["chi"], tol=r["tol"], max_sweeps=r["max_sweeps"])
        assert len(hist) == r["sweeps"]
        np.testing.assert_allclose(hist, r["history"], rtol=1e-6, atol=1e-11)
        np.testing.assert_allclose(O.corner_spectrum(c), r["spectrum"], rtol=1e-9, atol=1e-12)
        assert [list(x) for x in bond] == r["bond"]
        if "beta_f" in r:
            assert O.beta_free_energy(c, e, bulk) == pytest.approx(r["beta_f"], rel=1e-10)
            assert O.beta_free_energy(c, e, bulk) == pytest.approx(r["onsager_beta_f"], rel=1e-6)


def test_onsager_restatement_matches_the_reference_value(golden_dir):
    import json

    r = json.loads((golden_dir / "ctmrg.json").read_text())["b040_chi16"]
    assert O.onsager_beta_f(r["beta"]) == pytest.approx(r["onsager_beta_f"], rel=1e-12)


def test_oracle_dmrg_matches_reference_run(golden_dir):
    """The oracle's two-site DMRG driver and MPO against the reference's own L = 12 run:
    per-sweep energies, every kept bond space, and the bulk MPO site tensors."""
    g = json.loads((golden_dir / "dmrg.json").read_text())["L12_chi32"]
    m = json.loads((golden_dir / "heff.json").read_text())
    h = np.load(golden_dir / "heff.npz")
    L = g["L"]
    W = O.heisenberg_mpo_su2(L)
    for key, n in (("w1", 5), ("w2", 6)):
        want = O.from_arena(O.structure_from_json(m[key]["legs"]), h[m[key]["arena"]])
        assert W[n].structure == want.structure
        assert np.abs(W[n].arena() - want.arena()).max() <= 1e-14
    phys = ((1, 1),)
    bonds = [tuple((j, 1) for j in range(i % 2, min(i, L - i) + 1, 2)) for i in range(L + 1)]
    psi = [O.random(O.Structure(O.SU2, (O.Leg(bonds[i], O.OUT), O.Leg(phys, O.OUT),
                                        O.Leg(bonds[i + 1], O.IN))), i) for i in range(L)]
    energies, psi = O.dmrg(psi, W, chi=g["chi"], cutoff=1e-10, ncv=20, max_sweeps=g["sweeps"])
    assert len(energies) == g["sweeps"]
    np.testing.assert_allclose(energies, g["history"], rtol=1e-12)
    assert [[list(x) for x in psi[i].structure.legs[0].sectors] for i in range(L)] == g["bonds"]
