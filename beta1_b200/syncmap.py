"""Compiled boundary synchronisations (the composed gather tables given to
mhd_set_sync_map).

A LunarBoundary::Sync(group) (Z4_Lunar/src/boundary/Boundary_Sync_.cpp:4-65)
is an ordered sequence of copies: physical handlers, corner defaults
(src/6_boundary/Boundary.cpp:178-270) and the face, edge and vertex halo
gathers (src/4_halo/1_MPCNS_Halo_Inner.cpp:3-217).  Composing the sequence
gives, for every point it touches, the one point whose pre-sync value it ends
up holding; that composition is what the device applies in one gather.

This module builds the composition for topologies it knows:

* ``periodic``: one block connected to itself on all six faces.  Every ghost
  point of every field takes the value of the point with the same component
  whose index, along each direction where the ghost lies outside the inner
  range, is wrapped modulo the cell count n of that direction; directions in
  which the point is inside the inner range keep their index (inner ranges
  are [0, n) for cell-like and [0, n] for nodal directions).  This is what the
  reference's inner face/edge/vertex patches of a self-periodic block produce
  (checked point by point against the reference's own Sync in the tests).
"""
from __future__ import annotations

from typing import Dict, List, Tuple

import numpy as np

GROUPS: Dict[str, List[str]] = {
    "Ucell": ["U_H"],
    "Bface": ["B_xi", "B_eta", "B_zeta"],
    "Eface": ["Eface_xi", "Eface_eta", "Eface_zeta"],
    "Eedge": ["E_xi", "E_eta", "E_zeta"],
    "B_cell": ["B_cell", "Bind_cell"],
    "Jedge": ["J_xi", "J_eta", "J_zeta"],
    "J_cell": ["J_cell"],
    "Uplus": ["U_plus"],
    "Eres": ["Eres_xi", "Eres_eta", "Eres_zeta"],
    "Eres1form": ["Eres_xi", "Eres_eta", "Eres_zeta"],
    "dB": ["dB_xi", "dB_eta", "dB_zeta"],
}

# +1 planes per axis of each location code (restart numbering)
PLUS = {0: (0, 0, 0), 1: (1, 0, 0), 2: (0, 1, 0), 3: (0, 0, 1), 4: (0, 1, 1), 5: (1, 0, 1), 6: (1, 1, 0)}


def aos_index(lo, hi, ncomp, i, j, k, m):
    n1 = hi[1] - lo[1]
    n2 = hi[2] - lo[2]
    return (((i - lo[0]) * n1 + (j - lo[1])) * n2 + (k - lo[2])) * ncomp + m


def periodic_field_map(info: dict, ncell: Tuple[int, int, int]):
    """(dst, src) AoS indices of the periodic ghost fill of one field."""
    lo, hi, nc, loc = info["lo"], info["hi"], info["ncomp"], info["loc"]
    pl = PLUS[loc]
    I, J, K = np.meshgrid(np.arange(lo[0], hi[0]), np.arange(lo[1], hi[1]), np.arange(lo[2], hi[2]), indexing="ij")
    ghost = ((I < 0) | (J < 0) | (K < 0) | (I >= ncell[0] + pl[0]) | (J >= ncell[1] + pl[1])
             | (K >= ncell[2] + pl[2]))
    I, J, K = I[ghost], J[ghost], K[ghost]
    def wrap(x, n, p):
        return np.where((x < 0) | (x >= n + p), np.mod(x, n), x)

    Is, Js, Ks = wrap(I, ncell[0], pl[0]), wrap(J, ncell[1], pl[1]), wrap(K, ncell[2], pl[2])
    dst, src = [], []
    for m in range(nc):
        dst.append(aos_index(lo, hi, nc, I, J, K, m))
        src.append(aos_index(lo, hi, nc, Is, Js, Ks, m))
    return np.concatenate(dst).astype(np.int64), np.concatenate(src).astype(np.int64)


def install_periodic(ctx, ncell) -> Dict[str, int]:
    """Sets the periodic gather table of every group on a one-block context."""
    sizes = {}
    for group, fields in GROUPS.items():
        dsts, srcs = [], []
        for f in fields:
            info = ctx.field_info(f, 0)
            base = ctx.point_base(f, 0)
            d, s = periodic_field_map(info, ncell)
            dsts.append(d + base)
            srcs.append(s + base)
        dst = np.concatenate(dsts)
        src = np.concatenate(srcs)
        ctx.set_sync_map(group, dst, src)
        sizes[group] = int(dst.size)
    return sizes
