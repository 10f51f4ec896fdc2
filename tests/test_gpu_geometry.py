"""The device geometry builder (mhd_build_geometry) against the host geometry.

From a block's ghost node mesh the device computes every geometry field the
reference builds at set-up (src/3_field/4_MPCNS_Geometry.cpp:4-640: JD, Jac,
face areas, beta, dl, Astar, alpha, dr; the least-squares weights of
Z4_Lunar/src/LunarSolver.cpp:243-915; the uniform-field Badd).  The host
geometry (beta1_b200.geometry) equals the reference's own dump bitwise
(tests/test_cpu_geometry.py), and the device builder follows the same
operation order, so the two must agree bit for bit on every field, and a step
from either set-up must give the same state.  Cases: the periodic box, the
4-block slab and the Pole shell."""
import numpy as np
import pytest

from conftest import load_golden, periodic_setup, shell_setup, slab_setup

from beta1_b200 import solver

pytestmark = pytest.mark.gpu

FIELDS = solver.GEOM_FIELDS + ["Badd_xi", "Badd_eta", "Badd_zeta"]
STATE = ["U_H", "B_xi", "B_eta", "B_zeta", "B_cell", "J_cell"]


def _case(name):
    if name == "periodic":
        spec, st = periodic_setup(load_golden("periodic_8x6x5_steps.npz"))
        return spec, st, "periodic"
    if name == "slab":
        spec, st = slab_setup(load_golden("slab_6x5x6_t2x2_r00_steps.npz"))
        return spec, st, "tiled"
    spec, st = shell_setup(load_golden("shell_8x6x8_steps.npz"))
    return spec, st, "shell"


@pytest.mark.parametrize("name", ["periodic", "slab", "shell"])
def test_device_geometry_equals_host_geometry(name):
    spec, st, topo = _case(name)
    host = solver.Solver(spec, topology=topo, geometry_on="host")
    dev = solver.Solver(spec, topology=topo, geometry_on="device")
    try:
        for b in range(len(spec.blocks)):
            for f in FIELDS:
                a, d = host.field(f, b), dev.field(f, b)
                assert a.shape == d.shape, (f, b)
                bad = np.argwhere(a != d)
                assert bad.size == 0, f"{name} block {b} field {f}: {len(bad)} points differ, first {bad[:3].tolist()}"
        host.load_state(st)
        dev.load_state(st)
        ha, da = host.step(2), dev.step(2)
        assert ha == da
        for b in range(len(spec.blocks)):
            for f in STATE:
                assert np.array_equal(host.field(f, b), dev.field(f, b)), (name, b, f)
    finally:
        host.ctx.close()
        dev.ctx.close()
