"""The numpy restatement of the Hall edge EMF (oracle/mhd_oracle.py) against
the reference's own BuildHallFaceEMF_Rusanov_diff_ (fixtures written by the
reference solver, tests/golden/make_golden.py hall()): a periodic box and a
4-block slab whose Solid_Surface zeroing reaches 20 node layers inwards."""
import os
import sys

import numpy as np
import pytest

from conftest import ROOT, load_golden, rel_l2

sys.path.insert(0, os.path.join(ROOT, "oracle"))
import mhd_oracle  # noqa: E402

from beta1_b200 import case, geometry, physics  # noqa: E402

TOL = 1e-12
GEO = ["dr_xi", "dr_eta", "dr_zeta", "Area_xi", "Area_eta", "Area_zeta", "dl_xi", "dl_eta", "dl_zeta"]


def hall_case(kind):
    if kind == "periodic":
        return case.periodic_box_case((8, 6, 5)), load_golden("hall_periodic_8x6x5.npz"), []
    spec = case.slab_case(24, (5, 6), (2, 2))
    n = spec.blocks[0].ncell
    # the slab's inner wall: a Solid_Surface patch on the i-minimum face of every block
    patches = [("Solid_Surface", -1, (0, 0, 0), (1, n[1] + 1, n[2] + 1))]
    return spec, load_golden("hall_slab_24x5x6_t2x2.npz"), patches


@pytest.mark.parametrize("kind", ["periodic", "slab"])
def test_oracle_hall_emf_matches_reference(kind):
    spec, g, patches = hall_case(kind)
    c = physics.constants(spec.params)
    consts = dict(M_H=c["M_H"], M_ref=c["M_ref"], ne_hall_floor=c["ne_hall_floor"])
    o = mhd_oracle.Oracle([b.ncell for b in spec.blocks], consts)
    for ib, b in enumerate(spec.blocks):
        blk = o.blocks[ib]
        geo = geometry.build(geometry.ghost_mesh(b.x, b.y, b.z, 4), b.ncell, 4)
        for name in GEO:
            lo, hi, a = geo[name]
            blk.set_ref(name, lo, a)
        for name in ("B_cell", "J_cell", "U_H", "B_xi", "B_eta", "B_zeta"):
            blk.set_ref(name, tuple(g["b%d/%s__lo" % (ib, name)]), g["b%d/%s" % (ib, name)])
        o.hall_emf(blk, c["hall_coef"], o.hall_zero_boxes(b.ncell, patches))
        for name in ("Ehall_xi", "Ehall_eta", "Ehall_zeta"):
            got = blk.get_ref(name)
            ref = g["b%d/%s" % (ib, name)]
            assert got.shape == ref.shape, name
            assert rel_l2(got, ref) <= TOL, (kind, ib, name, rel_l2(got, ref))
