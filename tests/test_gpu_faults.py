"""Failure detection on the device, in forms that fault, trap or hang nothing.

* dt guard: the reference aborts a run whose CFL time step falls below
  1e-7 or is NaN (Z4_Lunar/src/physics/LunarSolver_Timestep.cpp:128-139).
  Here a state injected on the host (one cell moving at 1e9) makes the step
  return MHD_EDT; the context then steps again, and matches the reference,
  once a good state is loaded.
* Krylov limit: a resistive solve capped at one iteration reports the
  reason KSP_DIVERGED_ITS (-3) and the step goes on, as the reference's
  KSPSolve does (Z4_Lunar/src/implicit/Lunar_ImplicitResistive.cpp:457-491
  prints the reason and continues).
* Grid barrier: every wait of the persistent Krylov kernel polls a bounded
  number of times.  A test hook makes one barrier wait for an arrival that
  never comes, with a short polling limit; the step returns MHD_EKRYLOV, and
  the next step from a good state matches the reference.
"""
import time

import numpy as np
import pytest

from conftest import load_golden, periodic_setup, rel_l2, slab_setup

from beta1_b200 import mhd, solver

pytestmark = pytest.mark.gpu

STATE = ["U_H", "B_xi", "B_eta", "B_zeta"]


def _fast_cell_state(st):
    """the restart state with one cell's x momentum set to 1e9 rho"""
    bad = st.__class__(st.step, st.time, st.nblock, {})
    for name, rec in st.fields.items():
        r = rec.__class__(rec.name, rec.loc, rec.ncomp, rec.nghost, [])
        for fa in rec.blocks:
            r.blocks.append(fa.__class__(fa.lo, fa.hi, fa.data.copy()))
        bad.fields[name] = r
    fa = bad.fields["U_H"].blocks[0]
    i, j, k = (2 - fa.lo[0], 3 - fa.lo[1], 1 - fa.lo[2])
    fa.data[i, j, k, 1] = 1e9 * fa.data[i, j, k, 0]
    return bad


def test_dt_guard_returns_edt_then_recovers(golden_periodic):
    g = golden_periodic["steps"]
    spec, st = periodic_setup(g)
    s = solver.Solver(spec)
    try:
        s.load_state(_fast_cell_state(st))
        with pytest.raises(mhd.MHDError, match="EDT"):
            s.step(1)
        s.ctx.set_time(0.0, 0.0, 0)
        s.load_state(st)
        dt, _ = s.step(1)
        assert dt == float(g["s1/dt"])
        for f in STATE:
            assert np.array_equal(s.field(f), g["s1/" + f]), f
    finally:
        s.ctx.close()


def _resistive_slab(maxit=None):
    g = load_golden("slab_6x5x6_t2x2_r11_steps.npz")
    spec, st = slab_setup(g)
    if maxit is not None:
        spec.params["implicit_resistive_ksp_max_it"] = maxit
    s = solver.Solver(spec, topology="tiled")
    s.load_state(st)
    return g, spec, st, s


def test_krylov_iteration_limit_reports_reason_and_continues():
    g, spec, st, s = _resistive_slab(maxit=1)
    try:
        s.step(1)
        stats = s.ctx.resistive_stats()
        assert stats["reason"] == -3, stats
        assert stats["its"] == 1, stats
        assert stats["rnorm"] > 0.0 and np.isfinite(stats["rnorm"])
        # the unconverged solve still updates B
        assert np.all(np.isfinite(s.field("B_xi", 0)))
    finally:
        s.ctx.close()


def test_stalled_grid_barrier_returns_ekrylov_then_recovers():
    g, spec, st, s = _resistive_slab()
    try:
        s.ctx.test_stall_barrier(4096)
        t0 = time.perf_counter()
        with pytest.raises(mhd.MHDError, match="EKRYLOV"):
            s.step(1)
        assert time.perf_counter() - t0 < 30.0
        s.ctx.set_time(0.0, 0.0, 0)
        s.load_state(st)
        dt, _ = s.step(1)
        assert abs(dt - float(g["s1/dt"])) <= 1e-10 * float(g["s1/dt"])
        for b in range(len(spec.blocks)):
            for f in STATE:
                assert rel_l2(s.field(f, b), g["s1/b%d/%s" % (b, f)]) <= 1e-10, (b, f)
        stats = s.ctx.resistive_stats()
        assert stats["reason"] in (2, 3), stats
    finally:
        s.ctx.close()


def test_stall_hook_needs_a_persistent_solve(golden_periodic):
    spec, st = periodic_setup(golden_periodic["steps"])
    s = solver.Solver(spec)
    try:
        with pytest.raises(mhd.MHDError, match="ESTATE"):
            s.ctx.test_stall_barrier(100)
    finally:
        s.ctx.close()
