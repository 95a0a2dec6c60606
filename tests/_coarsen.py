"""U(1) x U(1) x fZ2 tensors as the oracle's fZ2 tensors (test infrastructure).

The reference's product provider cannot bend, so U(1) x U(1) x fZ2 environment updates
have no reference run.  The check is the oracle's fZ2 update (pinned to the reference's
fZ2 golden vectors) on the same tensors coarsened to fZ2: every (N, 2Sz) sector of a leg
merged into the parity sector it belongs to, in sector order.  A U(1) x U(1) x fZ2 tensor
is an fZ2 tensor whose blocks vanish away from charge-conserving positions, and every
fusion and braiding coefficient on this path depends on the parities alone, so
coarsening commutes with the update exactly.
"""

import numpy as np

import oracle.tenet_oracle as O
from tenet.structure import OUT, layout


def coarsen(s, host):
    """The fZ2 oracle tensor of structure ``s`` with arena ``host`` (a NumPy array)."""
    p = s.provider
    legs, offs = [], []
    for leg in s.legs:
        cnt, off = [0, 0], {}
        for a, m in leg.space.sectors:
            lab = p.label(a)
            off[lab] = (lab & 1, cnt[lab & 1])
            cnt[lab & 1] += m
        legs.append(O.Leg(tuple((q, cnt[q]) for q in (0, 1) if cnt[q]),
                          O.OUT if leg.side is OUT else O.IN, bool(leg.dual)))
        offs.append(off)
    sf = O.Structure(O.FZ2, tuple(legs))
    blocks = {k: np.zeros(O.block_shape(sf, k)) for k in O.block_order(sf)}
    lay = layout(s)
    oa, ia = s.out_axes, s.in_axes
    for b, (ot, it) in enumerate(s.keys):
        labs = dict(zip(oa, ot[0])) | dict(zip(ia, it[0]))
        out_u = tuple(labs[ax] & 1 for ax in oa)
        in_u = tuple(labs[ax] & 1 for ax in ia)
        c = int(np.bitwise_xor.reduce(out_u)) if out_u else 0
        key = (O.fusion_trees(O.FZ2, out_u, c)[0], O.fusion_trees(O.FZ2, in_u, c)[0])
        sl = []
        for ax, leg in enumerate(s.legs):
            space_label = p._dual(labs[ax]) if leg.dual else labs[ax]
            sl.append(slice(offs[ax][space_label][1],
                            offs[ax][space_label][1] + int(lay.shapes[b, ax])))
        o0 = int(lay.offsets[b])
        blocks[key][tuple(sl)] = host[o0:o0 + int(lay.sizes[b])].reshape(tuple(lay.shapes[b]))
    return O.Tensor(sf, [blocks[k] for k in O.block_order(sf)])


def rel(a, b) -> float:
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
