"""The on-disk format (``serialize.py``, ``network/mps.py:567-676``) on the CPU: files written
by the reference itself (``tests/golden/serialize``, made by ``make_serialize_golden.py``)
load here with the reference's block keys and values; files written here load in the
reference (recorded when the fixtures were made); round trips for every provider; the
loader's refusals; MPS directories."""

import json
import shutil
from pathlib import Path

import numpy as np
import pytest

from tenet import serialize
from tenet.structure import IN, OUT, GradedSpace, Leg, TensorStructure, layout
from tenet.symmetry import SU2, U1, Z2, ProductSector, U1xU1xfZ2, fZ2

G = Path(__file__).resolve().parent / "golden" / "serialize"
META = json.loads((G / "serialize.json").read_text())


@pytest.mark.parametrize("case", ["u1", "z2", "fz2", "su2"])
def test_reference_files_load_with_the_reference_keys_and_values(case):
    m = META[case]
    s, host = serialize.load_arena(G / m["file"])
    keys = [[[tuple(o[0]), tuple(o[1]), o[2]], [tuple(i[0]), tuple(i[1]), i[2]]]
            for o, i in m["keys"]]
    ours = [[list(o), list(i)] for o, i in s.keys]
    assert ours == keys
    assert np.array_equal(host, np.array(m["arena"]))
    assert m["reference_loads_ours_bit_exact"]


def _structures():
    out = []
    for p, labs in ((U1, (-1, 0, 2)), (Z2, (0, 1)), (fZ2, (0, 1)), (SU2, (0, 1, 2, 3))):
        V = GradedSpace.new(p, {p.sector(a): k + 1 for k, a in enumerate(labs)})
        out.append(TensorStructure((Leg(V, OUT), Leg(V, OUT, True, "mid"), Leg(V, IN))))
    V = GradedSpace.new(U1xU1xfZ2, {ProductSector(0, 0, 0): 2, ProductSector(1, 1, 1): 1,
                                    ProductSector(1, -1, 1): 2, ProductSector(2, 0, 0): 1})
    out.append(TensorStructure((Leg(V, OUT), Leg(V, OUT), Leg(V, IN, True))))
    return out


@pytest.mark.parametrize("k", range(5))
def test_round_trip_keeps_structure_and_values(tmp_path, k):
    s = _structures()[k]
    host = np.random.default_rng(k).standard_normal(layout(s).size)
    serialize.save_arena(s, host, tmp_path / "t.npz")
    s2, h2 = serialize.load_arena(tmp_path / "t.npz")
    assert s2 == s and np.array_equal(h2, host)
    serialize.save_arena(s, host, tmp_path / "c.npz", compress=True)
    assert np.array_equal(serialize.load_arena(tmp_path / "c.npz")[1], host)


def test_loader_refusals(tmp_path):
    s = _structures()[3]  # SU(2)
    host = np.zeros(layout(s).size)
    serialize.save_arena(s, host, tmp_path / "t.npz")
    with np.load(tmp_path / "t.npz") as z:
        header = json.loads(str(z["header"].item()))
        blocks = {f: z[f] for f in z.files if f != "header"}

    def write(name, hdr, bl):
        np.savez(tmp_path / name, header=np.array(json.dumps(hdr)), **bl)
        return tmp_path / name

    with pytest.raises(ValueError, match="newer"):
        serialize.load_arena(write("f.npz", {**header, "format": 2}, blocks))
    with pytest.raises(ValueError, match="gauge"):
        serialize.load_arena(write("g.npz", {**header, "gauges": {"SU2": "other"}}, blocks))
    # a racah build of unknown coefficients is refused, a known or accepted one loads
    unknown = write("u.npz", {**header, "gauges": {"SU2": "su2=racah;unknown-build"}}, blocks)
    with pytest.raises(ValueError, match="gauge"):
        serialize.load_arena(unknown)
    serialize.load_arena(write("k.npz", {**header, "gauges": {
        "SU2": "su2=racah;racah-shim-su2-exact-racah-formula"}}, blocks))
    serialize.accept_su2_gauge("su2=racah;unknown-build")
    try:
        serialize.load_arena(unknown)
    finally:
        serialize._SU2_KNOWN.discard("su2=racah;unknown-build")
    with pytest.raises(ValueError, match="blocks"):
        serialize.load_arena(write("n.npz", {**header, "num_blocks": 1}, blocks))
    with pytest.raises(ValueError, match="unexpected"):
        serialize.load_arena(write("x.npz", header, {**blocks, "extra": np.zeros(1)}))
    with pytest.raises(ValueError, match="missing"):
        serialize.load_arena(write("m.npz", header, {k: v for k, v in blocks.items()
                                                    if k != "b0"}))
    with pytest.raises(ValueError, match="shape"):
        serialize.load_arena(write("s.npz", header, {**blocks, "b0": np.zeros((9, 9, 9))}))
    with pytest.raises(KeyError):
        bad = json.loads(json.dumps(header))
        bad["legs"][0]["space"]["provider"]["kind"] = "SU3"
        serialize.load_arena(write("k.npz", bad, blocks))
    with pytest.raises(TypeError, match="leg name"):
        V = GradedSpace.new(U1, {U1.sector(0): 1})
        serialize.save_arena(TensorStructure((Leg(V, OUT, False, 1.5), Leg(V, IN))),
                             np.zeros(1), tmp_path / "y.npz")


def test_reference_mps_directory_loads_and_is_checked(tmp_path):
    m = META["mps"]
    sites, center = serialize.load_mps_arenas(G / m["dir"])
    assert len(sites) == m["n_sites"] and center == m["center"]
    for (s, h), want in zip(sites, m["arenas"]):
        assert np.array_equal(h, np.array(want))
    d = tmp_path / "mps"
    shutil.copytree(G / m["dir"], d)
    (d / "003.npz").unlink()
    with pytest.raises(ValueError, match="do not match"):
        serialize.load_mps_arenas(d)
    shutil.copy(G / m["dir"] / "003.npz", d / "003.npz")
    (d / "mps.json").write_text(json.dumps({"format": 1, "n_sites": 4, "center": 7}))
    with pytest.raises(ValueError, match="out of range"):
        serialize.load_mps_arenas(d)
    (d / "mps.json").write_text(json.dumps({"format": 1, "n_sites": 4, "center": None}))
    shutil.copy(G / m["dir"] / "000.npz", d / "002.npz")  # a site whose bonds do not fit
    with pytest.raises(ValueError, match="disagrees"):
        serialize.load_mps_arenas(d)
