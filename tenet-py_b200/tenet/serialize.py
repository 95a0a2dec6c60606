"""``save`` / ``load`` of tensors and MPS in the reference's on-disk format.

A tensor is one ``.npz``: a JSON ``header`` member (format version, the legs with their
spaces, the coefficient-gauge fingerprints of the providers present, the block count)
and one member ``b{i}`` per block in block order (``serialize.py:209-346``).  Nothing
derived is written -- block order, shapes and fusion trees are functions of the legs --
and on load the block count, member set, block shapes and gauges are checked before any
block moves.  An MPS is a directory: one ``NNN.npz`` per site plus ``mps.json`` with the
format, the site count and the canonical center (``network/mps.py:567-676``).

The arithmetic lives on the host (``save_arena`` / ``load_arena`` take and return a
structure and a NumPy arena); ``save`` / ``load`` move the arena to and from the device.
A loaded tensor lives on the current CUDA device (the reference loads NumPy blocks and
places them with ``to_backend``).

Gauges.  fZ2 blocks follow the reference's fZ2 conventions (its fingerprint is written
and required).  This build's SU(2) coefficients are the TensorKit ``SU2Irrep`` gauge the
reference accepts on load as its legacy SU(2) fingerprint, which is what is written;
files the reference writes carry ``su2=racah;<fingerprint>``, and the reference measured
that gauge to agree with the legacy one to 4.95e-14, so both are accepted here.
"""

from __future__ import annotations

import json
import pathlib

import numpy as np

from tenet.structure import IN, OUT, GradedSpace, Leg, TensorStructure, layout
from tenet.symmetry import SU2, U1, Z2, ProductSector, Provider, U1xU1xfZ2, fZ2

__all__ = ["FORMAT_VERSION", "MPS_FORMAT_VERSION", "accept_su2_gauge", "load", "load_arena",
           "load_mps", "save", "save_arena", "save_mps"]

FORMAT_VERSION = 1
MPS_FORMAT_VERSION = 1
VERSION = "tenet_b200 0.1"

_FZ2_GAUGE = "f=1;r=fermionic;fs=+1;twist=(-1)^p;perm=koszul"
_SU2_GAUGE = "3j=condon-shortley;cg=condon-shortley;f=tks-su2irrep;r=tks-su2irrep;fs=tks-su2irrep"
# SU(2) gauges a file may carry besides the one written here, each naming a coefficient
# source whose F / R / B values are known to equal this build's (to 4.4e-16 on every row
# of the reference's F fixture): the racah build the reference's on-disk fixtures were
# written under.  Any other ``su2=racah;<fingerprint>`` is refused, as the reference
# refuses a racah release that moves coefficient values (``serialize.py:99-103``).
# ``accept_su2_gauge`` adds one for a racah build a caller has checked against the table.
_SU2_KNOWN = {"su2=racah;racah-shim-su2-exact-racah-formula"}
_SIMPLE = {"U1": U1, "Z2": Z2, "fZ2": fZ2, "SU2": SU2}


def _encode_provider(p: Provider) -> dict:
    if p is U1xU1xfZ2:
        return {"kind": "Product", "factors": [{"kind": "U1", "name": "U1"},
                                               {"kind": "U1", "name": "U1"},
                                               {"kind": "fZ2", "name": "fZ2"}]}
    return {"kind": p.name, "name": p.name}


def _decode_provider(d) -> Provider:
    kind = d["kind"]
    if kind == "Product":
        kinds = [f["kind"] for f in d["factors"]]
        names = [f.get("name", f["kind"]) for f in d["factors"]]
        if kinds == ["U1", "U1", "fZ2"] and names == kinds:
            return U1xU1xfZ2
        raise ValueError(f"unsupported product provider {kinds}")
    if kind not in _SIMPLE:
        raise KeyError(f"unknown provider kind {kind!r}; known kinds are {sorted(_SIMPLE)}")
    if d.get("name", kind) != kind:
        raise ValueError(f"provider {kind} named {d['name']!r} is a different symmetry")
    return _SIMPLE[kind]


def _encode_sector(p: Provider, a) -> list:
    if p is U1xU1xfZ2:
        return [[a.n], [a.two_sz], [a.parity]]
    return [p.label(a)]


def _decode_sector(p: Provider, args):
    if p is U1xU1xfZ2:
        (n,), (sz,), (par,) = args
        return ProductSector(int(n), int(sz), int(par))
    (x,) = args
    return p.sector(int(x))


def _encode_leg(leg: Leg, axis: int) -> dict:
    if not (leg.name is None or isinstance(leg.name, (str, int))):
        raise TypeError(f"public axis {axis}: leg name {leg.name!r} cannot be written to JSON; "
                        "only None, str and int names are supported")
    p = leg.space.provider
    return {"side": "out" if leg.side is OUT else "in", "dual": bool(leg.dual), "name": leg.name,
            "space": {"provider": _encode_provider(p),
                      "sectors": [[_encode_sector(p, a), int(m)] for a, m in leg.space.sectors]}}


def _decode_leg(d) -> Leg:
    p = _decode_provider(d["space"]["provider"])
    space = GradedSpace.new(p, [(_decode_sector(p, a), int(m)) for a, m in d["space"]["sectors"]])
    side = {"out": OUT, "in": IN}[d["side"]]
    return Leg(space, side, bool(d["dual"]), d.get("name"))


def _gauges(s: TensorStructure) -> dict:
    p = s.provider
    out = {}
    if p is SU2:
        out["SU2"] = _SU2_GAUGE
    if p is fZ2 or p is U1xU1xfZ2:
        out["fZ2"] = _FZ2_GAUGE
    return out


def _check_gauges(path, gauges: dict) -> None:
    for kind, gauge in gauges.items():
        ok = {"SU2": gauge == _SU2_GAUGE or gauge in _SU2_KNOWN,
              "fZ2": gauge == _FZ2_GAUGE}.get(kind, True)
        if not ok:
            raise ValueError(f"{path}: {kind} coefficient gauge on disk is {gauge!r}; this build "
                             "runs a different convention and the blocks are not comparable")


def accept_su2_gauge(gauge: str) -> None:
    """Accept files whose SU(2) gauge string is ``gauge`` (e.g. ``"su2=racah;<fingerprint>"``
    of a racah build whose coefficients the caller has checked equal this build's)."""
    if not isinstance(gauge, str) or not gauge:
        raise TypeError("gauge must be a non-empty string")
    _SU2_KNOWN.add(gauge)


def save_arena(s: TensorStructure, host: np.ndarray, path, *, compress: bool = False) -> None:
    """Write structure ``s`` with the block arena ``host`` to ``path``."""
    lay = layout(s)
    host = np.asarray(host, dtype=np.float64)
    if host.shape != (lay.size,):
        raise ValueError(f"save: arena of {host.shape}, expected ({lay.size},)")
    header = {"format": FORMAT_VERSION, "tenet": VERSION,
              "legs": [_encode_leg(leg, i) for i, leg in enumerate(s.legs)],
              "gauges": _gauges(s), "num_blocks": s.num_blocks}
    blocks = {f"b{b}": host[int(lay.offsets[b]):int(lay.offsets[b]) + int(lay.sizes[b])]
              .reshape(tuple(int(x) for x in lay.shapes[b])) for b in range(s.num_blocks)}
    (np.savez_compressed if compress else np.savez)(
        path, header=np.array(json.dumps(header)), **blocks)


def load_arena(path) -> tuple[TensorStructure, np.ndarray]:
    """``(structure, arena)`` of a file written by ``save`` (here or by the reference)."""
    with np.load(path, allow_pickle=False) as z:
        header = json.loads(str(z["header"].item()))
        if header["format"] > FORMAT_VERSION:
            raise ValueError(f"{path}: file format {header['format']} is newer than this "
                             f"library's format {FORMAT_VERSION}")
        _check_gauges(path, header.get("gauges", {}))
        s = TensorStructure(tuple(_decode_leg(d) for d in header["legs"]))
        n = header["num_blocks"]
        if n != s.num_blocks:
            raise ValueError(f"{path}: header says {n} blocks but the structure it describes "
                             f"has {s.num_blocks}")
        expected = {"header", *(f"b{i}" for i in range(n))}
        extra = sorted(set(z.files) - expected)
        if extra:
            raise ValueError(f"{path}: unexpected members {extra} in the archive")
        lay = layout(s)
        host = np.empty(lay.size)
        for b in range(n):
            try:
                blk = z[f"b{b}"]
            except KeyError:
                raise ValueError(f"{path}: missing block member 'b{b}'") from None
            shape = tuple(int(x) for x in lay.shapes[b])
            if blk.shape != shape:
                raise ValueError(f"{path}: block {b} has shape {blk.shape}, expected {shape}")
            o = int(lay.offsets[b])
            host[o:o + blk.size] = np.asarray(blk, dtype=np.float64).ravel()
    return s, host


def save(t, path, *, compress: bool = False) -> None:
    """``tenet.save``: write a ``SymmetricTensor`` (copied to the host) to ``path``."""
    save_arena(t.structure, t.numpy_arena(), path, compress=compress)


def load(path):
    """``tenet.load``: the saved tensor, its arena on the current CUDA device."""
    from tenet.tensor import SymmetricTensor

    s, host = load_arena(path)
    return SymmetricTensor.from_numpy_arena(s, host)


def save_mps(psi, path) -> None:
    """``MPS.save``: a directory of ``NNN.npz`` site files plus ``mps.json``."""
    path = pathlib.Path(path)
    path.mkdir(parents=True, exist_ok=True)
    for n in range(len(psi)):
        save(psi[n], path / f"{n:03d}.npz")
    meta = {"format": MPS_FORMAT_VERSION, "n_sites": len(psi), "center": psi.center}
    (path / "mps.json").write_text(json.dumps(meta))


def load_mps_arenas(path) -> tuple[list, object]:
    """Host side of ``load_mps``: ``([(structure, arena), ...], center)`` after the
    directory checks (``network/mps.py:609-676``)."""
    path = pathlib.Path(path)
    meta_path = path / "mps.json"
    if not meta_path.is_file():
        raise ValueError(f"{meta_path}: not found; an MPS directory must contain mps.json")
    meta = json.loads(meta_path.read_text())
    if meta["format"] > MPS_FORMAT_VERSION:
        raise ValueError(f"{meta_path}: MPS directory format {meta['format']} is newer than "
                         f"this library's format {MPS_FORMAT_VERSION}")
    n_sites, center = meta["n_sites"], meta["center"]
    expected = {f"{n:03d}.npz" for n in range(n_sites)}
    found = {p.name for p in path.iterdir()} - {"mps.json"}
    if found != expected:
        raise ValueError(f"{path}: site files {sorted(found)} do not match n_sites={n_sites}")
    if center is not None and not 0 <= center < n_sites:
        raise ValueError(f"{path}: center {center} out of range for {n_sites} sites")
    sites = [load_arena(path / f"{n:03d}.npz") for n in range(n_sites)]
    for n in range(n_sites - 1):
        r, l = sites[n][0].legs[-1], sites[n + 1][0].legs[0]
        if r.space != l.space:
            raise ValueError(f"{path}: the bond between sites {n} and {n + 1} disagrees")
    return sites, center


def load_mps(path):
    """``MPS.load``: the saved state on the current CUDA device, ``center`` included."""
    from tenet.network import MPS
    from tenet.tensor import SymmetricTensor

    sites, center = load_mps_arenas(path)
    return MPS([SymmetricTensor.from_numpy_arena(s, h) for s, h in sites], center)
