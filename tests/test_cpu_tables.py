"""The set-up file the C++ drop-in driver reads (beta1_b200.tables): written
and read back, every table survives bit for bit, and its sync tables are the
ones the Python solver installs (beta1_b200.syncmap on the same case)."""
import numpy as np
import pytest

from conftest import load_golden, shell_setup, slab_setup

from beta1_b200 import geometry, mhd, solver, tables


@pytest.mark.parametrize("fixture,topo", [("slab_6x5x6_t2x2_r11_steps.npz", "tiled"),
                                          ("slab_6x5x6_t2x2_r10_steps.npz", "tiled"),
                                          ("shell_8x6x8_steps.npz", "shell"),
                                          ("shell_8x6x8_r10_steps.npz", "shell")])
def test_tables_round_trip(fixture, topo, tmp_path):
    setup = slab_setup if topo == "tiled" else shell_setup
    spec, _ = setup(load_golden(fixture))
    c = tables.compile_case(spec, topo)
    p = str(tmp_path / "t.bin")
    tables.write(p, c)
    r = tables.read(p)
    assert set(r["groups"]) == set(c["groups"])
    for g, m in c["groups"].items():
        for k in ("dst", "src", "cdst"):
            assert np.array_equal(np.asarray(m[k], dtype=np.int64).ravel(), r["groups"][g][k]), (g, k)
        assert np.array_equal(np.asarray(m["cval"], dtype=np.float64).ravel(), r["groups"][g]["cval"]), g
        if m.get("dst2") is not None:
            assert np.array_equal(np.asarray(m["dst2"], dtype=np.int64).ravel(), r["groups"][g]["dst2"]), g
        assert [tuple(w) for w in m["walls"]] == [tuple(w) for w in r["groups"][g]["walls"]], g
    assert [tuple(p) for p in c["poles"]] == [tuple(p) for p in r["poles"]]
    resistive = bool(spec.params.get("is_Lunar_resistance", 0))
    implicit = resistive and bool(spec.params.get("use_implicit_lunar_resistance", 0))
    # the resistive sync groups are exported with the resistive handlers
    assert ("Eres" in r["groups"]) == resistive
    if topo == "shell":
        assert sorted(tuple(p) for p in r["poles"]) == [(0, -2), (0, 2)]
    if not implicit:
        # no implicit system; the explicit sub-cycles' profile is formed by the driver
        assert r["resistive"] is None
    else:
        res = r["resistive"]
        assert res is not None and res["unknowns"].size > 0
        assert np.array_equal(res["unknowns"], c["resistive"]["unknowns"])
        assert res["rtol"] == float(spec.params["implicit_resistive_ksp_rtol"])


@pytest.mark.parametrize("fixture", ["shell_8x6x8_steps.npz", "shell_8x6x8_r10_steps.npz"])
def test_shell_tables_equal_solver_tables(fixture):
    spec, _ = shell_setup(load_golden(fixture))
    c = tables.compile_case(spec, "shell")
    nodes = [geometry.block_ghost_mesh(b, int(spec.params["ngg"])) for b in spec.blocks]
    ref = solver.shell_tables(spec, nodes[0], mhd.HostLayout([b.ncell for b in spec.blocks]))
    for g, m in ref.items():
        assert np.array_equal(np.asarray(m["dst"]), np.asarray(c["groups"][g]["dst"])), g
        assert np.array_equal(np.asarray(m["src"]), np.asarray(c["groups"][g]["src"])), g
