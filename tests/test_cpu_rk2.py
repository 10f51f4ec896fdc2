"""SSP-RK2 in the oracle against the reference's own stages.

The reference integrates with one forward-Euler stage per StepOnce.  The
SSP-RK2 form composes two of its Euler stages at the dt of the step's start
and their convex average (Shu and Osher, 1988).  The fixture
tests/golden/periodic_8x6x5_rk2.npz holds the reference harness's rk2
command (the reference's own ZeroRHS_, Scheme_U_, AddSourceToRHS_Fluid,
AssembleRHS_Induction_CT_, ApplyUpdate_Euler_, Syncs and
UpdateDerivedFields_); the oracle's rk2_step must equal it bit for bit."""
import numpy as np
import pytest

from conftest import load_golden
from test_cpu_oracle import COMPARE, build_periodic_oracle

import mhd_oracle  # noqa: F401  (on the path via test_cpu_oracle)


@pytest.fixture(scope="module")
def rk2_run(golden_periodic):
    g = load_golden("periodic_8x6x5_rk2.npz")
    o = build_periodic_oracle(golden_periodic)
    o.sync("Ucell")
    o.sync("Bface")
    o.update_derived()
    out, dts = {}, {}
    for s in (1, 2):
        dts[s] = o.rk2_step()
        o.calc_divb()
        out[s] = {f: o.blocks[0].get_ref(f) for f in COMPARE}
    return g, out, dts


@pytest.mark.parametrize("step", [1, 2])
def test_oracle_rk2_equals_reference_stages(rk2_run, step):
    g, out, dts = rk2_run
    assert dts[step] == float(g["s%d/dt" % step])
    for f in ("U_H", "B_xi", "B_eta", "B_zeta", "PV_H", "B_cell", "J_cell", "divB"):
        assert np.array_equal(out[step][f], g["s%d/%s" % (step, f)]), (step, f)


def test_rk2_differs_from_euler_and_keeps_time(rk2_run, golden_periodic):
    g, out, dts = rk2_run
    e = golden_periodic["steps"]
    assert float(g["s1/dt"]) == float(e["s1/dt"])  # same state, same CFL step
    assert not np.array_equal(g["s1/U_H"], e["s1/U_H"])
    assert float(g["s2/time"]) == float(g["s1/dt"]) + float(g["s2/dt"])
