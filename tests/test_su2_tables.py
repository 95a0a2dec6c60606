"""SU(2) coefficients against the reference's full fixture tables and the coherence laws.

``su2_tables.npz`` holds every row of the reference's ``tests/fixtures/su2_f.txt`` (F, 2j
<= 12) and ``su2_r.txt`` (R signs), the tables its ``tests/symmetry/test_su2_recoupling.py``
checks at 1e-13.  Both the planner's coefficients (``tenet._su2``) and the oracle's
(``oracle/racah_su2.py``) must reproduce them.  Beyond 2j = 12 no fixture exists, so the
planner's symbols are held to the laws that fix a unitary braided gauge up to the values
already pinned: pentagon, hexagon, unitarity of every F-matrix and the snake relation of
the bend coefficient (the reference's ``symmetry/coherence.py:77-360``), over label sets
that reach 2j = 17 -- the largest bond spin of the benchmarked matvec -- with inner lines
as large as fusion makes them.
"""

import itertools

import numpy as np
import pytest

from oracle import racah_su2
from tenet import _su2


@pytest.fixture(scope="module")
def tables(golden_dir):
    with np.load(golden_dir / "su2_tables.npz") as z:
        return {k: z[k] for k in z.files}


def test_full_f_table_matches_fixture(tables):
    dj, want = tables["f_dj"].astype(int), tables["f_value"]
    assert dj.shape == (109_900, 6)
    for impl in (_su2.f_symbol, racah_su2.f_symbol):
        got = np.fromiter((impl(*row) for row in map(tuple, dj.tolist())), float, len(dj))
        dev = np.abs(got - want)
        worst = int(dev.argmax())
        assert dev[worst] <= 1e-13, f"{impl.__module__}: {dev[worst]:.2e} at {tuple(dj[worst])}"


def test_full_r_table_matches_fixture(tables):
    dj, want = tables["r_dj"].astype(int), tables["r_value"].astype(int)
    assert dj.shape == (616, 3)
    for impl in (_su2.r_symbol, racah_su2.r_symbol):
        got = [impl(*row) for row in map(tuple, dj.tolist())]
        assert all(abs(g) == 1 for g in got)
        assert [g > 0 for g in got] == [w > 0 for w in want]


def _channels(a, b):
    return range(abs(a - b), a + b + 1, 2)


F, R, B = _su2.f_symbol, _su2.r_symbol, _su2.b_symbol
# outer labels: the small spins of the MPO and physical legs, and the large bond spins
# beyond the fixture
BUDGET = (0, 1, 2, 13, 14, 15, 16, 17)


def test_pentagon_up_to_2j_17():
    rng = np.random.default_rng(0)
    checked = 0
    quads = [q for q in itertools.product(BUDGET, repeat=4) if max(q) >= 13]
    for i in rng.choice(len(quads), size=40, replace=False):
        a, b, c, d = quads[i]
        for f in _channels(a, b):
            for g in _channels(f, c):
                for ell in _channels(c, d):
                    for e in _channels(g, d):
                        if not _su2.triangle(f, ell, e):
                            continue
                        for k in _channels(b, ell):
                            if not _su2.triangle(a, k, e):
                                continue
                            lhs = F(f, c, d, e, g, ell) * F(a, b, ell, e, f, k)
                            rhs = sum(F(a, b, c, g, f, h) * F(a, h, d, e, g, k)
                                      * F(b, c, d, k, h, ell) for h in _channels(b, c))
                            assert abs(lhs - rhs) <= 1e-12, (a, b, c, d, e, f, g, k, ell)
                            checked += 1
    assert checked > 2_000


def test_hexagon_up_to_2j_17():
    checked = 0
    for a, b, c, d in itertools.product(BUDGET, repeat=4):
        if max(a, b, c, d) < 13:
            continue
        for e in _channels(c, a):
            if not _su2.triangle(e, b, d):
                continue
            for g in _channels(c, b):
                if not _su2.triangle(a, g, d):
                    continue
                lhs = R(c, a, e) * F(a, c, b, d, e, g) * R(c, b, g)
                rhs = sum(F(c, a, b, d, e, f) * R(c, f, d) * F(a, b, c, d, f, g)
                          for f in _channels(a, b))
                assert abs(lhs - rhs) <= 1e-12, (a, b, c, d, e, g)
                checked += 1
    assert checked > 1_000


def test_f_matrices_unitary_and_snake_up_to_2j_17():
    labels = range(0, 18)
    checked = 0
    for a, b, c in itertools.product(labels, repeat=3):
        for d in range(0, a + b + c + 1):
            es = [e for e in _channels(a, b) if _su2.triangle(e, c, d)]
            fs = [f for f in _channels(b, c) if _su2.triangle(a, f, d)]
            if not es:
                continue
            assert len(es) == len(fs)
            m = np.array([[F(a, b, c, d, e, f) for f in fs] for e in es])
            assert np.abs(m @ m.T - np.eye(len(es))).max() <= 1e-12, (a, b, c, d)
            checked += 1
    assert checked > 10_000
    for a, b in itertools.product(labels, repeat=2):
        for c in _channels(a, b):  # SU(2) irreps are self-dual
            want = ((a + 1) * (b + 1) / (c + 1)) ** 0.5 * F(a, b, b, a, c, 0)
            assert abs(B(a, b, c) - want) <= 1e-12
