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
    "Badd": ["Badd_xi", "Badd_eta", "Badd_zeta"],
    "Ehall": ["Ehall_xi", "Ehall_eta", "Ehall_zeta"],
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


def periodic_maps(ctx, ncell) -> Dict[str, dict]:
    """group -> gather table (dst, src point ids; no constants or walls) of
    the periodic one-block layout; ctx: a context or a HostLayout."""
    out = {}
    for group, fields in GROUPS.items():
        dsts, srcs = [], []
        for f in fields:
            info = ctx.field_info(f, 0)
            base = ctx.point_base(f, 0)
            d, s = periodic_field_map(info, ncell)
            dsts.append(d + base)
            srcs.append(s + base)
        out[group] = dict(dst=np.concatenate(dsts), src=np.concatenate(srcs), cdst=np.zeros(0, dtype=np.int64),
                          cval=np.zeros(0), walls=[])
    return out


def install_periodic(ctx, ncell) -> Dict[str, int]:
    """Sets the periodic gather table of every group on a one-block context."""
    sizes = {}
    for group, m in periodic_maps(ctx, ncell).items():
        ctx.set_sync_map(group, m["dst"], m["src"])
        sizes[group] = int(m["dst"].size)
    return sizes


def merge_runs(per_run) -> Dict[str, dict]:
    """One table per group for a batch of runs: per_run holds (tables of a
    run compiled on its own blocks 0, 1, ..., first block of the run in the
    batch); the runs' tables are shifted to their blocks and concatenated
    (runs share no halo)."""
    out: Dict[str, dict] = {}
    for maps, off in per_run:
        for group, m in shift_blocks(maps, off).items():
            o = out.setdefault(group, dict(dst=[], src=[], dst2=[], src2=[], cdst=[], cval=[], walls=[]))
            for k in ("dst", "src", "dst2", "src2", "cdst", "cval"):
                o[k].append(m[k])
            o["walls"] += m["walls"]
    for o in out.values():
        for k in ("dst", "src", "dst2", "src2", "cdst"):
            o[k] = np.concatenate(o[k]).astype(np.int64)
        o["cval"] = np.concatenate(o["cval"]).astype(np.float64)
    return out


def shift_blocks(maps: Dict[str, dict], off: int) -> Dict[str, dict]:
    """The tables of a layout whose blocks become blocks off, off + 1, ... of
    a larger context (point ids carry the block in bits 40-55)."""
    sh = np.int64(off) << np.int64(40)
    none = np.zeros(0, dtype=np.int64)
    return {g: dict(dst=m["dst"] + sh, src=m["src"] + sh, dst2=m.get("dst2", none) + sh,
                    src2=m.get("src2", none) + sh, cdst=m["cdst"] + sh, cval=m["cval"],
                    walls=[(b + off, d) for (b, d) in m["walls"]]) for g, m in maps.items()}


# ---------------------------------------------------------------------------
# Tiled layouts with physical walls
# ---------------------------------------------------------------------------
#
# Blocks of one orientation tile the transverse (j, k) directions
# periodically; the radial direction i ends in a Solid_Surface (i = 0) and a
# Farfield (i = n_i).  A Sync(group) then is
#   phase A: the physical handlers that compute or set values
#            (Z4_Lunar/src/boundary/Boundary_Condition_Fluid.cpp,
#             Boundary_Condition.cpp, Boundary_Condition_EM.cpp),
#   phase B: every copy -- default physical copies of the ghost slab from the
#            first inner layer (src/6_boundary/Boundary.cpp:303-331) and the
#            face/edge/vertex halos -- composed into one gather.
# The composition is obtained by replaying the copies on an index map.

# what each handler of the shipped Lunar set-up does to a field on the
# Solid_Surface / Farfield faces (Z4_Lunar/src/boundary/Boundary_Build.cpp:5-271):
#   copy        ghost slab <- first inner layer
#   nop         nothing
#   wall_u      Solid_Surface fluid handler (phase A kernel)
#   ghost_const ghost slab <- constant (phase A)
#   slab_zero_copy   inner slab (and, for J_cell, the next layer) <- 0, then copy
#   slab_const_copy  inner slab <- E_inf . dr (zero-curl far field), then copy
#   eface_ghost_zero normal component field: inner slab <- 0; ghost slab <- 0


def wall_rules(field: str, resistive: bool):
    """(Solid_Surface rule, Farfield rule) of a field."""
    if field == "U_H":
        return "wall_u", "ghost_const"
    if field == "U_plus":
        return "nop", "nop"
    if field in ("B_xi", "B_eta", "B_zeta"):
        return "copy", "nop"
    if field == "B_cell":
        return "copy", "ghost_const"
    if field == "Bind_cell":
        return "copy", "ghost_const"
    if field == "J_cell":
        return ("copy" if resistive else "slab_zero2_copy"), "copy"
    if field.startswith("Eface_"):
        return ("eface_ghost_zero" if resistive else "slab_zero_copy"), "nop"
    if field in ("E_xi", "E_eta", "E_zeta"):
        return ("copy" if resistive else "nop"), "slab_const_copy"
    if field in ("Eres_xi", "Eres_eta", "Eres_zeta"):
        # the zero-curl handler recognises only E_xi/E_eta/E_zeta and falls
        # back to the default copy for any other field (Boundary_Condition.cpp:573-597)
        return "copy", "copy"
    return "copy", "copy"


class TiledLayout:
    """Block b sits at tile (b // TK, b % TK); all blocks have the same cells."""

    def __init__(self, ncell, tiles):
        self.n = tuple(ncell)
        self.TJ, self.TK = tiles

    def tile(self, b):
        return b // self.TK, b % self.TK

    def block(self, tj, tk):
        return (tj % self.TJ) * self.TK + (tk % self.TK)


def _field_points(info):
    lo, hi = info["lo"], info["hi"]
    I, J, K = np.meshgrid(np.arange(lo[0], hi[0]), np.arange(lo[1], hi[1]), np.arange(lo[2], hi[2]), indexing="ij")
    return I.ravel(), J.ravel(), K.ravel()


def compile_tiled(ctx, layout: TiledLayout, resistive: bool, farfield_consts, node_coords):
    """Builds phase A tables and the composed gather of every group.
    farfield_consts: dict with 'qinf' (5), 'B_imf' (3), 'E_inf' (3).
    node_coords: per block, Padded node array (ghost nodes included).
    Returns {group: dict(dst, src, cdst, cval, walls)}."""
    n = layout.n
    nb = layout.TJ * layout.TK
    out = {}
    for group, fields in GROUPS.items():
        dsts, srcs, cd, cv, walls = [], [], [], [], []
        for f in fields:
            info0 = ctx.field_info(f, 0)
            loc, nc = info0["loc"], info0["ncomp"]
            lo, hi = info0["lo"], info0["hi"]
            pl = PLUS[loc]
            inner_hi = (n[0] + pl[0], n[1] + pl[1], n[2] + pl[2])
            shape = (hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2])
            npt = shape[0] * shape[1] * shape[2]
            I, J, K = _field_points(info0)
            # src_of as (block, point-offset) pairs over all blocks of this field
            sb = np.repeat(np.arange(nb), npt)
            sp = np.tile(np.arange(npt), nb)
            phaseA = np.zeros(nb * npt, dtype=bool)

            def off(i, j, k):
                return ((i - lo[0]) * shape[1] + (j - lo[1])) * shape[2] + (k - lo[2])

            solid, far = wall_rules(f, resistive)
            tin = (J >= 0) & (J < inner_hi[1]) & (K >= 0) & (K < inner_hi[2])
            g_lo = tin & (I < 0)
            g_hi = tin & (I >= inner_hi[0])
            slab_lo = tin & (I == 0)
            slab_hi = tin & (I == inner_hi[0] - 1)
            for b in range(nb):
                base = b * npt
                # Solid_Surface (i = 0)
                if solid == "copy":
                    idx = np.nonzero(g_lo)[0]
                    sp[base + idx] = off(np.zeros_like(I[idx]), J[idx], K[idx])
                elif solid == "wall_u":
                    sel = g_lo | slab_lo
                    phaseA[base + np.nonzero(sel)[0]] = True
                    walls.append((b, -1))
                elif solid in ("slab_zero_copy", "slab_zero2_copy"):
                    zsel = slab_lo | (tin & (I == 1)) if solid == "slab_zero2_copy" else slab_lo
                    for m in range(nc):
                        for q in np.nonzero(zsel)[0]:
                            pass
                    zidx = np.nonzero(zsel)[0]
                    phaseA[base + zidx] = True
                    for m in range(nc):
                        cd.append((f, b, I[zidx], J[zidx], K[zidx], m))
                        cv.append(np.zeros(zidx.size))
                    idx = np.nonzero(g_lo)[0]
                    sp[base + idx] = off(np.zeros_like(I[idx]), J[idx], K[idx])
                elif solid == "eface_ghost_zero":
                    normal = f == "Eface_xi"
                    zsel = g_lo | (slab_lo if normal else np.zeros_like(g_lo))
                    zidx = np.nonzero(zsel)[0]
                    phaseA[base + zidx] = True
                    for m in range(nc):
                        cd.append((f, b, I[zidx], J[zidx], K[zidx], m))
                        cv.append(np.zeros(zidx.size))
                # Farfield (i = n_i)
                if far == "copy":
                    idx = np.nonzero(g_hi)[0]
                    sp[base + idx] = off(np.full_like(I[idx], inner_hi[0] - 1), J[idx], K[idx])
                elif far == "ghost_const":
                    idx = np.nonzero(g_hi)[0]
                    phaseA[base + idx] = True
                    vals = {"U_H": farfield_consts["qinf"], "B_cell": farfield_consts["B_imf"],
                            "Bind_cell": [0.0, 0.0, 0.0]}[f]
                    for m in range(nc):
                        cd.append((f, b, I[idx], J[idx], K[idx], m))
                        cv.append(np.full(idx.size, float(vals[m])))
                elif far == "slab_const_copy":
                    sidx = np.nonzero(slab_hi)[0]
                    phaseA[base + sidx] = True
                    X = node_coords[b]
                    d = {"E_xi": (1, 0, 0), "Eres_xi": (1, 0, 0), "E_eta": (0, 1, 0), "Eres_eta": (0, 1, 0),
                         "E_zeta": (0, 0, 1), "Eres_zeta": (0, 0, 1)}[f]
                    Ei, Ej, Ek = I[sidx], J[sidx], K[sidx]
                    o = X.off
                    p0 = X.a[Ei + o, Ej + o, Ek + o]
                    p1 = X.a[Ei + d[0] + o, Ej + d[1] + o, Ek + d[2] + o]
                    E = farfield_consts["E_inf"]
                    val = (E[0] * (p1[:, 0] - p0[:, 0]) + E[1] * (p1[:, 1] - p0[:, 1])) + E[2] * (p1[:, 2] - p0[:, 2])
                    cd.append((f, b, Ei, Ej, Ek, 0))
                    cv.append(val)
                    idx = np.nonzero(g_hi)[0]
                    sp[base + idx] = off(np.full_like(I[idx], inner_hi[0] - 1), J[idx], K[idx])
            # transverse halos: tangential ghost -> owner tile's point (i unchanged)
            tg = ~tin
            for b in range(nb):
                tj, tk = layout.tile(b)
                idx = np.nonzero(tg)[0]
                Jg, Kg = J[idx], K[idx]
                wj = (Jg < 0) | (Jg >= inner_hi[1])
                wk = (Kg < 0) | (Kg >= inner_hi[2])
                gj = tj * n[1] + Jg
                gk = tk * n[2] + Kg
                otj = np.where(wj, np.floor_divide(gj, n[1]), tj)
                otk = np.where(wk, np.floor_divide(gk, n[2]), tk)
                jj = np.where(wj, gj - otj * n[1], Jg)
                kk = np.where(wk, gk - otk * n[2], Kg)
                ob = (np.mod(otj, layout.TJ) * layout.TK + np.mod(otk, layout.TK))
                opt = off(I[idx], jj, kk)
                srcflat = ob * npt + opt
                sb[b * npt + idx] = sb[srcflat]
                sp[b * npt + idx] = sp[srcflat]
                phaseA[b * npt + idx] = False
            allp = np.arange(nb * npt)
            own_b = allp // npt
            own_p = allp % npt
            moved = ~phaseA & ~((sb == own_b) & (sp == own_p))
            mi = np.nonzero(moved)[0]
            bases = np.array([ctx.point_base(f, b) for b in range(nb)], dtype=np.int64)
            for m in range(nc):
                dsts.append(bases[own_b[mi]] + own_p[mi] * nc + m)
                srcs.append(bases[sb[mi]] + sp[mi] * nc + m)
        cdst = []
        cval = []
        for (f, b, Ii, Jj, Kk, m), v in zip(cd, cv):
            info = ctx.field_info(f, b)
            base = ctx.point_base(f, b)
            cdst.append(base + aos_index(info["lo"], info["hi"], info["ncomp"], Ii, Jj, Kk, m))
            cval.append(v)
        out[group] = dict(dst=np.concatenate(dsts) if dsts else np.zeros(0, np.int64),
                          src=np.concatenate(srcs) if srcs else np.zeros(0, np.int64),
                          cdst=np.concatenate(cdst).astype(np.int64) if cdst else np.zeros(0, np.int64),
                          cval=np.concatenate(cval) if cval else np.zeros(0),
                          walls=sorted(set(walls)))
    return out


# ---------------------------------------------------------------------------
# The single-block spherical shell: Solid_Surface / Farfield in i, Pole at
# both ends of j, k periodic onto itself
# ---------------------------------------------------------------------------
#
# A Sync(group) there is (Z4_Lunar/src/boundary/Boundary_Sync_.cpp:4-65), per
# field, the physical handlers in the topology's patch order -- Pole j min,
# Pole j max, Farfield (i max), Solid_Surface (i min) -- then the corner
# default where a wall meets a Pole (every ghost point of the corner takes the
# value of the nearest inner point, BoundaryCore::ApplyPhysicalCornerDefault,
# src/6_boundary/Boundary.cpp:178-260), then the periodic halo in k.
#
# What the Pole handler of the shipped set-up does to a field
# (Z4_Lunar/src/boundary/Boundary_Build.cpp:27-269, eta Poles):
#   copy   the ghost slab <- the first inner layer (DefaultPhysicalCopy)
#   nop    nothing
#   ring   the device computes the first inner layer (the pole ring): U_H's
#          k average (BC_Pole_Cell_), the B_cell / Bind_cell collapse, B_xi's
#          k average (BC_Pole_Bface_Collapse_), E_xi from -u x B
#          (BC_Pole_Eedge_Axis), E_eta's and Eres_eta's regulation
#          (BC_Pole_Eedge_RegulateK_Norm); then the ghost copy
#   zero   the first inner layer <- 0, then the ghost copy (B_eta's norm face,
#          BC_Pole_Eedge_Zero_Rotate of E_zeta, J_xi, J_zeta, Eres_xi, Eres_zeta)
#   ring_ghost_zero  the device computes the first inner layer (J_eta,
#          BC_Pole_Jedge_RegulateK_Norm); the ghost slab <- 0
SHELL_POLE_RULES = {"U_plus": "nop", "U_H": "ring", "B_cell": "ring", "Bind_cell": "ring", "B_xi": "ring",
                    "E_xi": "ring", "E_eta": "ring", "B_eta": "zero", "E_zeta": "zero", "J_xi": "zero",
                    "J_zeta": "zero", "J_eta": "ring_ghost_zero", "Eres_xi": "zero", "Eres_eta": "ring",
                    "Eres_zeta": "zero"}

# groups with a computing Pole handler (the device runs their ring kernels
# before the group's tables)
SHELL_POLE_HANDLED = ("Ucell", "Bface", "Eedge", "B_cell", "Jedge", "Eres", "Eres1form")

# groups whose Sync runs the halo exchange only (no physical handlers, no
# corner default): Sync("Uplus") after calc_Uplus
SHELL_HALO_ONLY = ("Uplus",)

# resistive groups: compiled only for a resistive set-up
SHELL_SKIPPED = ("Eres", "Eres1form")


def shell_pole_rule(field: str) -> str:
    """What the Pole handler of the shipped Lunar set-up does to a field
    (eta Poles: Eres_xi and Eres_zeta Zero_Rotate, Eres_eta regulated,
    Z4_Lunar/src/boundary/Boundary_Build.cpp:208-239)."""
    return SHELL_POLE_RULES.get(field, "copy")


def compile_shell(ctx, ncell, resistive: bool, farfield_consts=None, nodes=None):
    """Tables of every Sync group of the shell; the resistive groups and
    handlers with `resistive` (is_Lunar_resistance: the Solid_Surface
    handlers of J_cell, Eface and the edge EMF of Boundary_Build.cpp:93-163).
    ctx: a context or HostLayout of the one block; farfield_consts: dict with
    'qinf' (5), 'B_imf' (3), 'E_inf' (3); nodes: the block's Padded ghost node
    mesh (both needed by the groups with Farfield values).

    The Sync is replayed in the reference's order on a map that holds, per
    point, the point whose value it takes and when that value is read, or a
    constant.  The device runs a shell Sync as
      1. the Pole ring kernels (in place, on the first inner layer),
      2. the gather `dst/src`: sources read after the rings, before the walls,
      3. the Solid_Surface fluid handler (`walls`; in place, wall layer and ghosts),
      4. the gather `dst2/src2`: sources the wall handler wrote,
      5. the fixed values `cdst/cval`.
    A copy here can read a point before a later handler overwrites it (the
    Pole ghost copy at i = 0 reads the wall layer before the wall handler
    zeroes or rewrites it), hence the copies before the fixed values, and the
    two gathers around the wall.
    Returns {group: dict(dst, src, dst2, src2, cdst, cval, walls)}."""
    n = tuple(ncell)
    out = {}
    for group, fields in GROUPS.items():
        if group in SHELL_SKIPPED and not resistive:
            continue
        physical = group not in SHELL_HALO_ONLY
        dsts, srcs, dsts2, srcs2, cdst, cval, walls = [], [], [], [], [], [], []
        for f in fields:
            info = ctx.field_info(f, 0)
            loc, nc, ng = info["loc"], info["ncomp"], info["nghost"]
            lo, hi = info["lo"], info["hi"]
            pl = PLUS[loc]
            ih = (n[0] + pl[0], n[1] + pl[1], n[2] + pl[2])
            shape = (hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2])
            npt = shape[0] * shape[1] * shape[2]
            I, J, K = _field_points(info)

            def off(i, j, k):
                return ((i - lo[0]) * shape[1] + (j - lo[1])) * shape[2] + (k - lo[2])

            src = np.arange(npt)               # point whose value a point ends up holding
            ver = np.zeros(npt, dtype=np.int8)  # ... read before (0) or after (1) the wall handler
            isc = np.zeros(npt, dtype=bool)     # ... or a constant
            cv = np.zeros((npt, nc))

            def copy(sel, i, j, k):
                idx = np.nonzero(sel)[0]
                o = off(i(idx), j(idx), k(idx))
                src[idx] = src[o]
                ver[idx] = ver[o]
                isc[idx] = isc[o]
                cv[idx] = cv[o]

            def const(sel, vals):
                idx = np.nonzero(sel)[0]
                isc[idx] = True
                cv[idx] = np.asarray(vals, dtype=np.float64).reshape(-1, nc) if np.ndim(vals) == 2 else vals

            if physical:
                pin = (I >= 0) & (I < ih[0]) & (K >= 0) & (K < ih[2])
                tin = (J >= 0) & (J < ih[1]) & (K >= 0) & (K < ih[2])
                rule = shell_pole_rule(f)
                for side in (-1, +1):
                    jr = 0 if side < 0 else ih[1] - 1
                    ghost = pin & ((J < 0) if side < 0 else (J >= ih[1]))
                    if rule == "nop":
                        continue
                    if rule == "zero":
                        const(pin & (J == jr), 0.0)
                    if rule == "ring_ghost_zero":
                        const(ghost, 0.0)
                        continue
                    copy(ghost, lambda x: I[x], lambda x, jr=jr: np.full_like(J[x], jr), lambda x: K[x])
                solid, far = wall_rules(f, resistive)
                # Farfield (i max)
                g_hi = tin & (I >= ih[0])
                if far == "copy":
                    copy(g_hi, lambda x: np.full_like(I[x], ih[0] - 1), lambda x: J[x], lambda x: K[x])
                elif far == "ghost_const":
                    vals = {"U_H": farfield_consts["qinf"], "B_cell": farfield_consts["B_imf"],
                            "Bind_cell": [0.0, 0.0, 0.0]}[f]
                    const(g_hi, [float(v) for v in vals])
                elif far == "slab_const_copy":
                    sl = tin & (I == ih[0] - 1)
                    idx = np.nonzero(sl)[0]
                    d = {"E_xi": (1, 0, 0), "E_eta": (0, 1, 0), "E_zeta": (0, 0, 1)}[f]
                    o = nodes.off
                    p0 = nodes.a[I[idx] + o, J[idx] + o, K[idx] + o]
                    p1 = nodes.a[I[idx] + d[0] + o, J[idx] + d[1] + o, K[idx] + d[2] + o]
                    E = farfield_consts["E_inf"]
                    val = (E[0] * (p1[:, 0] - p0[:, 0]) + E[1] * (p1[:, 1] - p0[:, 1])) + E[2] * (p1[:, 2] - p0[:, 2])
                    const(sl, val[:, None])
                    copy(g_hi, lambda x: np.full_like(I[x], ih[0] - 1), lambda x: J[x], lambda x: K[x])
                elif far != "nop":
                    raise ValueError(f"Farfield rule {far} of {f} is not compiled for the shell")
                # Solid_Surface (i min)
                g_lo = tin & (I < 0)
                if solid == "copy":
                    copy(g_lo, lambda x: np.zeros_like(I[x]), lambda x: J[x], lambda x: K[x])
                elif solid in ("slab_zero_copy", "slab_zero2_copy"):
                    const(tin & ((I == 0) | ((I == 1) & (solid == "slab_zero2_copy"))), 0.0)
                    copy(g_lo, lambda x: np.zeros_like(I[x]), lambda x: J[x], lambda x: K[x])
                elif solid == "eface_ghost_zero":
                    # BC_Solid_Surface_Eface_ghots_zero: the normal field's wall
                    # layer and every field's ghost slab <- 0
                    const(g_lo | (tin & (I == 0) & (f == "Eface_xi")), 0.0)
                elif solid == "wall_u":
                    # the wall handler rewrites the wall layer and its ghosts in place
                    w = np.nonzero(tin & (I <= 0))[0]
                    src[w] = w
                    ver[w] = 1
                    isc[w] = False
                    walls = [(0, -1)]
                elif solid != "nop":
                    raise ValueError(f"Solid_Surface rule {solid} of {f} is not compiled for the shell")
                # corner default where a wall meets a Pole (along k)
                cor = (K >= 0) & (K < ih[2]) & ((I < 0) | (I >= ih[0])) & ((J < 0) | (J >= ih[1]))
                copy(cor, lambda x: np.clip(I[x], 0, ih[0] - 1), lambda x: np.clip(J[x], 0, ih[1] - 1), lambda x: K[x])
            # the periodic halo in k (the plane k = n_k of k-staggered fields is inner)
            copy((K < 0) | (K >= ih[2]), lambda x: I[x], lambda x: J[x], lambda x: np.mod(K[x], n[2]))
            base = ctx.point_base(f, 0)
            moved = ~isc & (src != np.arange(npt))
            g1 = np.nonzero(moved & (ver == 0))[0]
            g2 = np.nonzero(moved & (ver == 1))[0]
            c = np.nonzero(isc)[0]
            for m in range(nc):
                dsts.append(base + g1 * nc + m)
                srcs.append(base + src[g1] * nc + m)
                dsts2.append(base + g2 * nc + m)
                srcs2.append(base + src[g2] * nc + m)
                cdst.append(base + c * nc + m)
                cval.append(cv[c, m])
        out[group] = dict(dst=np.concatenate(dsts).astype(np.int64), src=np.concatenate(srcs).astype(np.int64),
                          dst2=np.concatenate(dsts2).astype(np.int64), src2=np.concatenate(srcs2).astype(np.int64),
                          cdst=np.concatenate(cdst).astype(np.int64), cval=np.concatenate(cval), walls=walls)
    return out
