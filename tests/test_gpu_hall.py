"""GPU Hall edge EMF (MHD_STAGE_HALL_EMF) against the reference's own
BuildHallFaceEMF_Rusanov_diff_ on a periodic box and on a 4-block slab whose
Solid_Surface zeroing reaches 20 node layers inwards (fixtures written by the
reference solver, tests/golden/make_golden.py hall()).  FP64 in the
reference's operation order: the bound is the 1e-12 relative L2 of the FP64
parity tests."""
import numpy as np
import pytest

from conftest import load_golden, rel_l2

from beta1_b200 import case, mhd, rst, solver

pytestmark = pytest.mark.gpu

TOL = 1e-12
LOCS = {"U_H": rst.CELL, "B_xi": rst.FACE_XI, "B_eta": rst.FACE_ET, "B_zeta": rst.FACE_ZE}


def state_of(g, spec):
    st = rst.RestartFile(0, 0.0, len(spec.blocks), {})
    for name, loc in LOCS.items():
        rec = rst.FieldRecord(name, loc, 5 if name == "U_H" else 1, 4)
        for b in range(len(spec.blocks)):
            a = g["init/b%d/%s" % (b, name)]
            lo = tuple(int(v) for v in g["init/b%d/%s__lo" % (b, name)])
            rec.blocks.append(rst.FieldArray(lo, tuple(l + s for l, s in zip(lo, a.shape[:3])), a))
        st.fields[name] = rec
    return st


@pytest.mark.parametrize("kind", ["periodic", "slab"])
def test_hall_emf_matches_reference(kind):
    if kind == "periodic":
        spec, g, topo = case.periodic_box_case((8, 6, 5)), load_golden("hall_periodic_8x6x5.npz"), "periodic"
    else:
        spec, g, topo = case.slab_case(24, (5, 6), (2, 2)), load_golden("hall_slab_24x5x6_t2x2.npz"), "tiled"
    s = solver.Solver(spec, topology=topo)
    try:
        s.load_state(state_of(g, spec))
        s.ctx.stage(mhd.STAGE_HALL_EMF)
        worst = 0.0
        for b in range(len(spec.blocks)):
            for name in ("Ehall_xi", "Ehall_eta", "Ehall_zeta"):
                got, ref = s.field(name, b), g["b%d/%s" % (b, name)]
                assert got.shape == ref.shape
                e = rel_l2(got, ref)
                worst = max(worst, e)
                assert e <= TOL, (kind, b, name, e)
        print("Hall EMF %s: max rel L2 %.3e" % (kind, worst))
    finally:
        s.ctx.close()
