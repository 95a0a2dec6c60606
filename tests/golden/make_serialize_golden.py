"""Golden files of the reference's on-disk format (``serialize.py``, ``network/mps.py``).

Run in a container that has the reference source (it is imported, never copied)::

    python tests/golden/make_serialize_golden.py /path/to/TeNeT-py

with the test-only shims of ``tests/golden/_refshim`` (see ``make_golden.py``).  Writes
``tests/golden/serialize/``:

* ``ref_<case>.npz`` -- tensors written by the reference's ``tenet.save`` (U(1), Z2, fZ2,
  SU(2)), and ``ref_mps/`` -- an SU(2) MPS directory written by ``MPS.save``;
* ``serialize.json`` -- per case the reference's block keys (sector labels) and arena,
  and whether the reference's ``tenet.load`` read back, bit for bit, the file this
  library's ``serialize.save_arena`` wrote for the same tensor.
"""

from __future__ import annotations

import json
import shutil
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
OUT = HERE / "serialize"


def main(ref: Path) -> None:
    sys.path[:0] = [str(HERE / "_refshim"), str(REPO), str(ref / "src"),
                    str(REPO / "tenet-py_b200")]
    import tenet as R  # the reference package (first on the path)
    from tenet import IN, OUT as ROUT, GradedSpace, Leg, SymmetricTensor
    from tenet.network import MPS
    from tenet.symmetry import SU2, U1, Z2, FZ2Sector, SU2Sector, U1Sector, Z2Sector, fZ2

    if OUT.exists():
        shutil.rmtree(OUT)
    OUT.mkdir(parents=True)
    cases = {
        "u1": (U1, U1Sector, {-1: 2, 0: 3, 1: 1}),
        "z2": (Z2, Z2Sector, {0: 2, 1: 3}),
        "fz2": (fZ2, FZ2Sector, {0: 2, 1: 2}),
        "su2": (SU2, SU2Sector, {0: 1, 1: 2, 2: 1}),
    }
    meta: dict = {}
    for name, (p, S, sec) in cases.items():
        V = GradedSpace.new(p, {S(a): m for a, m in sec.items()})
        legs = (Leg(V, ROUT), Leg(V, ROUT, dual=True), Leg(V, IN))
        t = SymmetricTensor.random(legs, seed=7)
        path = OUT / f"ref_{name}.npz"
        R.save(t, path)
        keys = []
        for k in t.structure.block_order:
            def tree(tr):
                lab = lambda s: int(next(getattr(s, f) for f in ("charge", "parity", "two_j")  # noqa: E731
                                         if hasattr(s, f)))
                return [[lab(s) for s in tr.uncoupled], [lab(s) for s in tr.inner], lab(tr.coupled)]
            keys.append([tree(k.output_tree), tree(k.input_tree)])
        arena = np.concatenate([np.asarray(b).ravel() for b in t.blocks])
        meta[name] = {"file": path.name, "keys": keys, "arena": arena.tolist()}

    # this library's writer, read by the reference's loader
    sys.path.insert(0, str(REPO / "tenet-py_b200"))
    import importlib

    for mod in [m for m in sys.modules if m == "tenet" or m.startswith("tenet.")]:
        del sys.modules[mod]
    sys.path.remove(str(ref / "src"))
    ours = importlib.import_module("tenet.serialize")
    ostruct = importlib.import_module("tenet.structure")
    osym = importlib.import_module("tenet.symmetry")
    for name, (_, _, sec) in cases.items():
        P = {"u1": osym.U1, "z2": osym.Z2, "fz2": osym.fZ2, "su2": osym.SU2}[name]
        V = ostruct.GradedSpace.new(P, {P.sector(a): m for a, m in sec.items()})
        s = ostruct.TensorStructure((ostruct.Leg(V, ostruct.OUT), ostruct.Leg(V, ostruct.OUT, True),
                                     ostruct.Leg(V, ostruct.IN)))
        ours.save_arena(s, np.array(meta[name]["arena"]), OUT / f"ours_{name}.npz")
    for mod in [m for m in sys.modules if m == "tenet" or m.startswith("tenet.")]:
        del sys.modules[mod]
    sys.path.remove(str(REPO / "tenet-py_b200"))
    sys.path.insert(0, str(ref / "src"))
    R = importlib.import_module("tenet")
    for name in cases:
        back = R.load(OUT / f"ours_{name}.npz")
        arena = np.concatenate([np.asarray(b).ravel() for b in back.blocks])
        meta[name]["reference_loads_ours_bit_exact"] = bool(
            np.array_equal(arena, np.array(meta[name]["arena"])))
        (OUT / f"ours_{name}.npz").unlink()

    # an SU(2) MPS directory
    from tenet.network import MPS as RMPS
    from tenet.symmetry import SU2 as RSU2, SU2Sector as RS

    phys = R.GradedSpace.new(RSU2, {RS(1): 1})
    bonds = [R.GradedSpace.new(RSU2, {RS(j): 1 for j in range(i % 2, min(i, 4 - i) + 1, 2)})
             for i in range(5)]
    psi = RMPS.random(phys, bonds, seed=3)
    psi.save(OUT / "ref_mps")
    meta["mps"] = {"dir": "ref_mps", "n_sites": len(psi), "center": psi.center,
                   "arenas": [np.concatenate([np.asarray(b).ravel() for b in psi[n].blocks]).tolist()
                              for n in range(len(psi))]}
    (OUT / "serialize.json").write_text(json.dumps(meta))
    print("wrote", OUT)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: python tests/golden/make_serialize_golden.py "
                         "<path to the TeNeT-py tree>")
    main(Path(sys.argv[1]))
