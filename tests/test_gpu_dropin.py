"""The reference's own driver with the B200 drop-in of LunarSolver's driver.

oracle/_ref/ref_lunar_b200_stock is the reference's Z4_Lunar/main.cpp and
every reference source unchanged, except that
beta1_b200/dropin/LunarSolver_Driver_B200.cpp links in place of
Z4_Lunar/src/LunarSolver_Driver.cpp: Advance / StepOnce /
UpdateControlAndOutput run every step on the device through the C ABI and
read the fields back for the reference's own writers.  Both it and the stock
build (oracle/_ref/ref_lunar_stock) run the same CASE directory from the
reference's own initial condition for a few steps and write the reference's
restart file at the last step; the two files must agree on every field (bit
for bit for ideal MHD and the resistive shell, to 1e-12 with the explicit
resistive sub-cycles on the slab, to 1e-10 with the implicit resistive
solve), and where bit for bit the output-step diagnostics both print must be
the same lines.  With the explicit sub-cycles the driver forms the edge
resistivity profile from the reference's own node coordinates."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, load_golden, rel_l2, shell_setup, slab_setup

from beta1_b200 import case, rst, tables

pytestmark = pytest.mark.gpu

STOCK = os.path.join(ROOT, "oracle", "_ref", "ref_lunar_stock")
DROPIN = os.path.join(ROOT, "oracle", "_ref", "ref_lunar_b200_stock")
STEPS = 3


def _case(name):
    """(case, topology, relative L2 bound, bit for bit)"""
    if name == "slab_ideal":
        spec, _ = slab_setup(load_golden("slab_6x5x6_t2x2_r00_steps.npz"))
        return spec, "tiled", 1e-12, True
    if name == "slab_implicit_resistive":
        spec, _ = slab_setup(load_golden("slab_6x5x6_t2x2_r11_steps.npz"))
        return spec, "tiled", 1e-10, False
    if name == "slab_explicit_resistive":
        spec, _ = slab_setup(load_golden("slab_6x5x6_t2x2_r10_steps.npz"))
        return spec, "tiled", 1e-12, False
    if name == "shell_explicit_resistive":
        spec, _ = shell_setup(load_golden("shell_8x6x8_r10_steps.npz"))
        return spec, "shell", 1e-12, True
    spec, _ = shell_setup(load_golden("shell_8x6x8_steps.npz"))
    return spec, "shell", 1e-12, True


def _run(binary, d, spec, topo):
    spec.params.update(max_Nstep=STEPS, output_step=STEPS, output_residual=STEPS, continue_calc=0)
    case.write_case(d, spec)
    if binary == DROPIN:
        tables.write(os.path.join(d, "CASE", "b200_tables.bin"), tables.compile_case(spec, topo))
    r = subprocess.run([binary], cwd=d, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True, timeout=600)
    assert r.returncode == 0, (binary, r.stderr[-2000:])
    diag = [ln.rstrip() for ln in r.stdout.splitlines() if ln.strip().startswith(("rho=", "Bx =", "Pmag="))]
    return rst.read(os.path.join(d, "DATA", "flow_field0000.bin")), diag


@pytest.mark.parametrize("name", ["slab_ideal", "slab_implicit_resistive", "slab_explicit_resistive", "shell",
                                  "shell_explicit_resistive"])
def test_dropin_driver_equals_stock_driver(name, tmp_path):
    if not (os.path.exists(STOCK) and os.path.exists(DROPIN)):
        pytest.skip("oracle/_ref/ref_lunar_stock or ref_lunar_b200_stock is not built (make -C oracle)")
    spec, topo, tol, bitwise = _case(name)
    a, b = tmp_path / "stock", tmp_path / "b200"
    a.mkdir()
    b.mkdir()
    ref, dref = _run(STOCK, str(a), spec, topo)
    got, dgot = _run(DROPIN, str(b), spec, topo)
    assert got.step == ref.step == STEPS
    assert abs(got.time - ref.time) <= tol * ref.time
    assert set(got.fields) == set(ref.fields)
    for f, rec in ref.fields.items():
        for bi, fa in enumerate(rec.blocks):
            g = got.fields[f].blocks[bi].data
            if fa.data is None:
                continue
            assert g.shape == fa.data.shape, (f, bi)
            assert rel_l2(g, fa.data) <= tol, (name, f, bi, rel_l2(g, fa.data))
            if bitwise:
                assert np.array_equal(g, fa.data), (name, f, bi)
    assert dref and len(dgot) == len(dref)
    if bitwise:
        assert dgot == dref
