"""GPU parity on the spherical shell with Pole patches against the reference.

The shell is one block: Solid_Surface at r = 1 and Farfield at r = 8 in i,
a Pole patch at both ends of theta (j = 0 and j = n_j), and phi (k) periodic
onto itself -- the grid the reference's shipped boundary table describes
(Z4_Lunar/9999setup/2_Boundary_Condition.txt:1-7).  Its Syncs run the Pole
handlers of Z4_Lunar/src/boundary/Boundary_Condition_Fluid.cpp:186-219 and
Boundary_Condition_EM.cpp:3-380, and its derived-field pass the Pole repairs
of Z4_Lunar/src/physics/LunarSolver_Tools.cpp (the B_zeta rewrite :242-307,
the J_cell ring least squares :894-1296, the divB zeroing :729-772).

The fixture tests/golden/shell_8x6x8_steps.npz holds the reference's own
fields after its load and after each of two StepOnce.  The FP64 kernels follow
the reference's operation order, so every field is compared bit for bit (the
1e-12 relative L2 bound of the FP64 path is asserted as well), dt included.
"""
import os
import sys

import numpy as np
import pytest

from conftest import ROOT, load_golden, rel_l2, shell_setup

from beta1_b200 import case, mhd, solver

pytestmark = pytest.mark.gpu

TOL = 1e-12
FIELDS = ["U_H", "B_xi", "B_eta", "B_zeta", "PV_H", "U_plus", "B_cell", "Bind_cell", "J_xi", "J_eta", "J_zeta",
          "J_cell", "E_xi", "E_eta", "E_zeta", "Eface_xi", "Eface_eta", "Eface_zeta", "RHS_H", "RHS_B_xi",
          "RHS_B_eta", "RHS_B_zeta", "divB"]
STATE = ["U_H", "B_xi", "B_eta", "B_zeta"]


@pytest.fixture(scope="module")
def shell_run():
    g = load_golden("shell_8x6x8_steps.npz")
    spec, st = shell_setup(g)
    s = solver.Solver(spec, topology="shell")
    s.load_state(st)
    s.ctx.stage(mhd.STAGE_DIVB)
    out = {0: {f: s.field(f) for f in FIELDS}}
    dts = {}
    for n in (1, 2):
        dts[n], _ = s.step(1)
        s.ctx.stage(mhd.STAGE_DIVB)
        out[n] = {f: s.field(f) for f in FIELDS}
    diag = s.ctx.diagnostics()
    s.ctx.close()
    return g, out, dts, diag


@pytest.mark.parametrize("step", [0, 1, 2])
def test_shell_fields_bitwise(shell_run, step):
    g, out, dts, _ = shell_run
    checked = 0
    for f in FIELDS:
        if step == 0 and f.startswith(("E", "RHS")):
            continue  # not computed before the first step
        ref = g["s%d/b0/%s" % (step, f)]
        got = out[step][f]
        assert got.shape == ref.shape, (step, f, got.shape, ref.shape)
        assert rel_l2(got, ref) <= TOL, (step, f, rel_l2(got, ref))
        bad = np.argwhere(got != ref)
        assert bad.size == 0, f"step {step} field {f}: {len(bad)} points differ, first {bad[:3].tolist()}"
        checked += 1
    assert checked == (13 if step == 0 else len(FIELDS))


def test_shell_dt_bitwise(shell_run):
    g, out, dts, _ = shell_run
    for n in (1, 2):
        assert dts[n] == float(g["s%d/dt" % n]), (n, dts[n], float(g["s%d/dt" % n]))


def test_shell_diagnostics_print_equals_reference(shell_run):
    """mhd_diagnostics after the two steps, printed as the reference's
    PrintMinMaxDiagnostics_ prints them (Z4_Lunar/src/tools/LunarSolver_PrintDiag.cpp:7-85),
    equals the reference's own lines."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import mhd_oracle
    _, _, _, (mins, maxs) = shell_run
    with open(os.path.join(ROOT, "tests", "golden", "shell_8x6x8_diag.txt")) as fh:
        ref = [ln.rstrip() for ln in fh if ln.strip()]
    assert mhd_oracle.Oracle.format_diagnostics(mins, maxs) == ref


def test_batch_of_shells_equals_runs_alone():
    """Shells of different sizes and inflows in one batch context: each run
    equals the same run advanced alone, bit for bit, dt included."""
    g = load_golden("shell_8x6x8_steps.npz")
    spec0, st0 = shell_setup(g)
    spec1 = case.shell_case(10, 8, 12, mach_u=6.0)
    st1 = case.inflow_state(spec1, seed=77)
    runs = [(spec0, st0), (spec1, st1)]
    for prec in (mhd.PREC_FP64, mhd.PREC_MIXED):
        bt = solver.Batch([(sp, "shell") for sp, _ in runs], precision=prec)
        bt.load_states([st for _, st in runs])
        bt.step(3)
        for r, (sp, st) in enumerate(runs):
            s = solver.Solver(sp, topology="shell", precision=prec)
            s.load_state(st)
            s.step(3)
            for f in STATE + ["B_cell", "J_cell", "PV_H"]:
                a, b = bt.field(r, f), s.field(f)
                assert np.array_equal(a, b), (prec, r, f, rel_l2(a, b))
            assert bt.ctx.run_time(r) == s.ctx.run_time(0), (prec, r)
            s.ctx.close()
        bt.ctx.close()


def test_shell_first_step_matches_reference_in_batch():
    """The fixture's shell inside a batch with a second shell still equals
    the reference's own first step bitwise."""
    g = load_golden("shell_8x6x8_steps.npz")
    spec0, st0 = shell_setup(g)
    spec1 = case.shell_case(6, 4, 8)
    st1 = case.inflow_state(spec1, seed=78)
    bt = solver.Batch([(spec0, "shell"), (spec1, "shell")])
    bt.load_states([st0, st1])
    bt.step(1)
    bt.ctx.stage(mhd.STAGE_DIVB)
    for f in FIELDS:
        assert np.array_equal(bt.field(0, f), g["s1/b0/" + f]), f
    assert bt.ctx.run_time(0)[0] == float(g["s1/dt"])
    bt.ctx.close()


def test_resistive_shell_steps_match_reference():
    """Two StepOnce with the explicit resistive sub-cycles (two per step, peak
    resistivity 1) on the Pole shell: each sub-cycle's B_cell / J pass with
    the B_zeta rewrite and the pole-shell J_cell, Sync("Eres") with the
    Eres_eta regulation on the pole rings (Z4_Lunar/src/boundary/Boundary_Build.cpp:208-239)
    and the resistive Solid_Surface handlers, against the reference's own
    fields (tests/golden/shell_8x6x8_r10_steps.npz): every field, Eres
    included, bit for bit, dt included (the 1e-12 relative L2 bound of the
    FP64 path is asserted first, so that a failure reports its size)."""
    g = load_golden("shell_8x6x8_r10_steps.npz")
    spec, st = shell_setup(g)
    assert spec.params["is_Lunar_resistance"] and int(spec.params["n_resistive_subcycles"]) == 2
    s = solver.Solver(spec, topology="shell")
    names = FIELDS + ["Eres_xi", "Eres_eta", "Eres_zeta"]
    try:
        s.load_state(st)
        exact = total = 0
        worst = 0.0
        for n in (1, 2):
            dt, _ = s.step(1)
            ref_dt = float(g["s%d/dt" % n])
            assert abs(dt - ref_dt) <= TOL * abs(ref_dt), (n, dt, ref_dt)
            assert dt == ref_dt, (n, dt, ref_dt)
            s.ctx.stage(mhd.STAGE_DIVB)
            for f in names:
                ref = g["s%d/b0/%s" % (n, f)]
                got = s.field(f)
                assert got.shape == ref.shape, (n, f)
                if f == "divB":
                    assert np.abs(got - ref).max() <= TOL, (n, f)
                else:
                    e = rel_l2(got, ref)
                    worst = max(worst, e)
                    assert e <= TOL, (n, f, e)
                exact += int(np.array_equal(got, ref))
                total += 1
        # the resistive EMF reaches the pole rings: the regulated Eres_eta is not zero there
        assert np.abs(g["s2/b0/Eres_eta"]).max() > 0.0
        print("resistive shell: %d of %d fields bitwise, max rel L2 %.3e" % (exact, total, worst))
        assert exact == total
    finally:
        s.ctx.close()
