"""Whole steps with the implicit Hall solve against the reference.

The device's step with the implicit Hall solve is one CUDA graph: the
Newton steps, the GMRES cycles, the Arnoldi steps, the restart product and
the line-search trials are conditional nodes whose conditions the device
sets, so no residual is read back by the host.  The reference runs its
StepOnce as compiled with HALL_IMPLICIT == 1 (oracle/_ref/ref_lunar
hallrun: the Euler stage, SolveOneStep at the step's dt with the nonlinear
solve tightened to ||F|| <= 1e-12 ||F0||, calc_Bcell, the closing syncs and
derived fields) on the same restart file.

Every state, derived and intermediate field, the converged Hall EMF and dt
are compared after each step, except the face EMF Eface_*: the reference's
Jacobian (its linearised whistler operator, BuildLinearHallFaceEMF_,
Z4_Lunar/src/implicit/Hall_Implicit_Solver.cpp:964-1080) uses those fields
as scratch, so after its solve they hold the last linearised Hall face EMF,
not the step's ideal face EMF; the device, whose products are differences
of the residual, leaves them as the explicit part wrote them.  Bound: 1e-10 relative L2 per field (the two
Newton iterations stop at 1e-12 of ||F0|| with different Jacobians, so they
agree on the root to about that; the rest of the step is the FP64 path of
the parity tests).  The first step's dt, computed before any solve, is
compared bit for bit."""
import numpy as np
import pytest

from conftest import reference_run, rel_l2

from beta1_b200 import case, mhd, solver

pytestmark = pytest.mark.gpu

TOL = 1e-10
FIELDS = ["U_H", "B_xi", "B_eta", "B_zeta", "PV_H", "U_plus", "B_cell", "Bind_cell", "J_xi", "J_eta", "J_zeta",
          "J_cell", "E_xi", "E_eta", "E_zeta", "RHS_H", "RHS_B_xi",
          "RHS_B_eta", "RHS_B_zeta", "Ehall_xi", "Ehall_eta", "Ehall_zeta", "divB"]


def cases():
    return {
        "periodic": (case.periodic_box_case((8, 6, 5)), "periodic", "initial"),
        "slab": (case.slab_case(24, (5, 6), (2, 2)), "tiled", "inflow"),
    }


@pytest.mark.parametrize("kind", ["periodic", "slab"])
def test_steps_with_implicit_hall_match_reference(kind, tmp_path):
    spec, topo, init = cases()[kind]
    st = case.initial_state(spec, seed=20261205) if init == "initial" else case.inflow_state(spec, seed=20261205)
    steps = 2
    ref = reference_run(spec, st, steps, str(tmp_path), command="hallrun")
    s = solver.Solver(spec, topology=topo)
    try:
        s.load_state(st)
        s.install_hall_implicit(topo, rtol=1e-12, atol=1e-30, maxit=200, ksp_rtol=1e-10, ksp_maxit=2000)
        worst = 0.0
        for n in range(1, steps + 1):
            l0 = s.ctx.launches()
            dt, _ = s.step(1)
            stats = s.ctx.hall_stats()
            assert stats["reason"] in (2, 3), (kind, n, stats)
            # the solve's loops ran on the device: at least one Newton step of
            # at least one Arnoldi step, counted from the device's pass counters
            assert stats["its"] >= 1 and stats["linear_its"] >= 1, stats
            assert s.ctx.launches() - l0 > 30, (kind, n)
            rdt = float(ref[n].fields["dt"].blocks[0].data.reshape(()))
            if n == 1:
                assert dt == rdt, (kind, dt, rdt)
            else:
                assert abs(dt - rdt) <= TOL * abs(rdt), (kind, n, dt, rdt)
            s.ctx.stage(mhd.STAGE_DIVB)
            for b in range(len(spec.blocks)):
                for f in FIELDS:
                    want = ref[n].fields[f].blocks[b].data
                    got = s.field(f, b)
                    assert got.shape == want.shape, (kind, n, b, f)
                    if f == "divB":
                        assert np.abs(got - want).max() <= 1e-10, (kind, n, b, f)
                        continue
                    e = rel_l2(got, want)
                    worst = max(worst, e)
                    assert e <= TOL, f"{kind} step {n} block {b} field {f}: rel L2 {e:.3e} ({stats})"
        print("Hall steps %s: max rel L2 %.3e, solver %s" % (kind, worst, stats))
    finally:
        s.ctx.close()


def test_newton_step_limit_ends_the_solve_on_the_device():
    """A Newton step limit of one with an unreachable tolerance: the
    device-steered loop stops after one step with the iteration-limit reason
    (-5, as SNES_DIVERGED_MAX_IT), and the step completes with finite fields;
    the GMRES iteration limit bounds each linear solve the same way."""
    spec = case.slab_case(24, (5, 6), (2, 2))
    st = case.inflow_state(spec, seed=20261205)
    s = solver.Solver(spec, topology="tiled")
    try:
        s.load_state(st)
        s.install_hall_implicit("tiled", rtol=1e-300, atol=1e-300, maxit=1, ksp_rtol=1e-300, ksp_maxit=3)
        s.step(2)
        stats = s.ctx.hall_stats()
        assert stats["reason"] == -5 and stats["its"] == 1, stats
        assert 1 <= stats["linear_its"] <= 3, stats
        assert stats["fnorm"] < stats["fnorm0"], stats
        for name in ("U_H", "B_xi", "Ehall_xi"):
            assert np.all(np.isfinite(s.field(name, 1))), name
    finally:
        s.ctx.close()
