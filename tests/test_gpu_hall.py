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


# k_hall_edge variants: 0 reads each edge's four cells, 2 the seven cells of
# a staggered point once; both give the reference's bits
@pytest.mark.parametrize("variant", [0, 2])
@pytest.mark.parametrize("kind", ["periodic", "slab"])
def test_hall_emf_matches_reference(kind, variant):
    if kind == "periodic":
        spec, g, topo = case.periodic_box_case((8, 6, 5)), load_golden("hall_periodic_8x6x5.npz"), "periodic"
    else:
        spec, g, topo = case.slab_case(24, (5, 6), (2, 2)), load_golden("hall_slab_24x5x6_t2x2.npz"), "tiled"
    s = solver.Solver(spec, topology=topo)
    try:
        s.ctx.set_tune({"k_hall_edge": variant})
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


# the reference's Newton stops at ||F|| <= 1e-12 ||F0|| with an approximate
# Jacobian, the device at 1e-12 with finite-difference products: both are
# that close to the same root, so the Hall EMF agrees to about 1e-12
# relative and the updated B (dt times its curl) closer still
HALL_TOL = {"Ehall": 1e-10, "B": 1e-12}


def test_step_with_implicit_hall_runs():
    """A whole StepOnce with the implicit Hall solve after the explicit part
    (the split-graph path): finite fields, a converged solve."""
    spec, g = case.slab_case(24, (5, 6), (2, 2)), load_golden("hallstep_slab_24x5x6_t2x2.npz")
    s = solver.Solver(spec, topology="tiled")
    try:
        s.load_state(state_of(g, spec))
        s.install_hall_implicit("tiled", rtol=1e-10)
        s.step(2)
        st = s.ctx.hall_stats()
        assert st["reason"] in (2, 3), st
        for name in ("U_H", "B_xi", "Ehall_xi"):
            assert np.all(np.isfinite(s.field(name, 1)))
    finally:
        s.ctx.close()


@pytest.mark.parametrize("kind", ["periodic", "slab"])
def test_implicit_hall_solve_matches_reference(kind):
    if kind == "periodic":
        spec, g, topo = case.periodic_box_case((8, 6, 5)), load_golden("hallstep_periodic_8x6x5.npz"), "periodic"
    else:
        spec, g, topo = case.slab_case(24, (5, 6), (2, 2)), load_golden("hallstep_slab_24x5x6_t2x2.npz"), "tiled"
    s = solver.Solver(spec, topology=topo)
    try:
        s.load_state(state_of(g, spec))
        s.ctx.stage(mhd.STAGE_TIMESTEP)
        assert s.ctx.get_time()[0] == float(g["dt"])
        s.install_hall_implicit(topo, rtol=1e-12, atol=1e-30, maxit=200, ksp_rtol=1e-10, ksp_maxit=2000)
        s.ctx.stage(mhd.STAGE_HALL_SOLVE)
        st = s.ctx.hall_stats()
        assert st["reason"] in (2, 3), st
        worst = {}
        for b in range(len(spec.blocks)):
            for name in ("Ehall_xi", "Ehall_eta", "Ehall_zeta", "B_xi", "B_eta", "B_zeta", "B_cell"):
                got, ref = s.field(name, b), g["b%d/%s" % (b, name)]
                e = rel_l2(got, ref)
                key = "Ehall" if name.startswith("Ehall") else "B"
                worst[key] = max(worst.get(key, 0.0), e)
                assert e <= HALL_TOL[key], (kind, b, name, e, st)
        print("implicit Hall %s: %s, solver %s" % (kind, worst, st))
    finally:
        s.ctx.close()
