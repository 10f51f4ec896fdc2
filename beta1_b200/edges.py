"""Edge ownership and the implicit resistive unknowns.

An edge shared by several blocks (block interfaces, periodic wraps) is one
physical unknown.  The reference identifies edges through node equivalence
classes and makes the smallest (rank, block, i, j, k, dir) copy the owner
(src/2_topology/2_MPCNS_Topology_Equiv.cpp:378-531); the other copies are
aliases that receive the owner's value times the orientation sign
(HALO_OWNER::sync_edge_1form, src/4_halo/9_MPCNS_Halo_EdgeOwner_sync.cpp:52-68,
274-285).  The implicit resistive unknowns are the owner edges whose
resistivity is positive, in owner order
(LunarSolver::BuildImplicitResistiveEdgeDofMap_,
Z4_Lunar/src/implicit/Lunar_ImplicitResistive.cpp:147-164).
"""
from __future__ import annotations

import math

import numpy as np

# edge direction 1/2/3 = xi/eta/zeta; +1 cells along its own axis, nodes across
_EXT = {1: (0, 1, 1), 2: (1, 0, 1), 3: (1, 1, 0)}


def local_edges(ncell):
    """All edges of a block's inner range: arrays (dir, i, j, k)."""
    out = []
    for d in (1, 2, 3):
        p = _EXT[d]
        I, J, K = np.meshgrid(np.arange(ncell[0] + p[0]), np.arange(ncell[1] + p[1]), np.arange(ncell[2] + p[2]),
                              indexing="ij")
        out.append(np.stack([np.full(I.size, d), I.ravel(), J.ravel(), K.ravel()], axis=1))
    return np.concatenate(out)


def tiled_owners(ncell, tiles, periodic_i=False):
    """(alias, owner) pairs of a tiled layout with identity orientation, as
    arrays of (block, dir, i, j, k); all signs are +1.  periodic_i also
    identifies the node planes i = 0 and i = n_i (a self-periodic block)."""
    TJ, TK = tiles
    nb = TJ * TK
    NJ, NK = ncell[1] * TJ, ncell[2] * TK
    rows = []
    for b in range(nb):
        tj, tk = b // TK, b % TK
        e = local_edges(ncell)
        gi = np.mod(e[:, 1], ncell[0]) if periodic_i else e[:, 1]
        gj = np.mod(tj * ncell[1] + e[:, 2], NJ)
        gk = np.mod(tk * ncell[2] + e[:, 3], NK)
        rows.append(np.stack([np.full(len(e), b), e[:, 0], e[:, 1], e[:, 2], e[:, 3], gi, gj, gk], axis=1))
    R = np.concatenate(rows)  # block, dir, i, j, k, key_i, key_j, key_k
    # owner = min (block, i, j, k, dir) within each key (dir, gi, gj, gk)
    order = np.lexsort((R[:, 1], R[:, 4], R[:, 3], R[:, 2], R[:, 0], R[:, 7], R[:, 6], R[:, 5], R[:, 1]))
    R = R[order]
    key = R[:, [1, 5, 6, 7]]
    newgrp = np.ones(len(R), dtype=bool)
    newgrp[1:] = np.any(key[1:] != key[:-1], axis=1)
    gid = np.cumsum(newgrp) - 1
    first = np.nonzero(newgrp)[0]
    owner = R[first][gid]
    alias = ~newgrp
    return R[alias][:, :5], owner[alias][:, :5], R[newgrp][:, :5]


def eta_at_edges(edges, nodes, inver_Rem):
    """Resistivity of edges (block, dir, i, j, k): inver_Rem times the tanh
    shell profile of the edge-midpoint radius, zero outside 0.84 < r < 1.04
    and on collapsed edges (LunarSolver::ImplicitResistiveEtaAtEdge_,
    Z4_Lunar/src/implicit/Lunar_ImplicitResistive.cpp:166-199).  The radius
    and length follow the reference's operation order; the profile uses the
    C library's tanh, as the reference does."""
    edges = np.asarray(edges)
    eta = np.zeros(len(edges))
    for b in np.unique(edges[:, 0]) if len(edges) else []:
        X = nodes[int(b)]
        o = X.off
        sel = np.nonzero(edges[:, 0] == b)[0]
        d, i, j, k = (edges[sel, c] for c in range(1, 5))
        p0 = X.a[i + o, j + o, k + o]
        p1 = X.a[i + (d == 1) + o, j + (d == 2) + o, k + (d == 3) + o]
        dx, dy, dz = (p1[:, c] - p0[:, c] for c in range(3))
        dl = np.sqrt(dx * dx + dy * dy + dz * dz)
        xm, ym, zm = (0.5 * (p0[:, c] + p1[:, c]) for c in range(3))
        r = np.sqrt(xm * xm + ym * ym + zm * zm)
        live = ~(np.abs(dl) <= 1.0e-12) & ~(r <= 0.84) & ~(r >= 1.04)
        for q in np.nonzero(live)[0]:
            rq = float(r[q])
            eta[sel[q]] = inver_Rem * (0.5 * (math.tanh((rq - 0.84) / 0.02) - math.tanh((rq - 1.04) / 0.02)))
    return eta


def resistive_dofs(owners, nodes, inver_Rem):
    """Owner edges with eta > 0 in owner order (block, i, j, k, dir), and eta."""
    o = owners[np.lexsort((owners[:, 1], owners[:, 4], owners[:, 3], owners[:, 2], owners[:, 0]))]
    eta = eta_at_edges(o, nodes, inver_Rem)
    keep = eta > 0.0
    return o[keep], eta[keep]


def shell_profile(nodes, ncell):
    """yita0(r) of every inner edge of a block (per axis an array over the
    edge's inner box): 0.5 [tanh((r - 0.84)/0.02) - tanh((r - 1.04)/0.02)] of
    the edge-midpoint radius, zero outside 0.84 < r < 1.04
    (LunarSolver::AddResistiveEdgeEMF_To_,
    Z4_Lunar/src/physics/LunarSolver_MagExplicit_Resis.cpp:72-88, 160-167).
    `nodes` is the block's node array with its ghost layers (geometry.Padded)."""
    o = nodes.off
    out = []
    for d in (1, 2, 3):
        p = _EXT[d]
        n = (ncell[0] + p[0], ncell[1] + p[1], ncell[2] + p[2])
        di, dj, dk = (d == 1), (d == 2), (d == 3)
        p0 = nodes.a[o:o + n[0], o:o + n[1], o:o + n[2]]
        p1 = nodes.a[o + di:o + di + n[0], o + dj:o + dj + n[1], o + dk:o + dk + n[2]]
        xm, ym, zm = (0.5 * (p0[..., c] + p1[..., c]) for c in range(3))
        r = np.sqrt(xm * xm + ym * ym + zm * zm)
        y = np.zeros(r.shape)
        for idx in zip(*np.nonzero(~(r <= 0.84) & ~(r >= 1.04))):
            rr = float(r[idx])
            y[idx] = 0.5 * (math.tanh((rr - 0.84) / 0.02) - math.tanh((rr - 1.04) / 0.02))
        out.append(y)
    return out
