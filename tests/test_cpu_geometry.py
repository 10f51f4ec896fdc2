"""Geometry set-up (beta1_b200.geometry) against the reference's own geometry
fields (Jacobian, face-area vectors, Hodge scales, B/J reconstruction
weights and ghost node coordinates of a periodic box, dumped by the
reference solver).  The restatement follows the reference's operation
order, so every field must agree bit for bit."""
import numpy as np

from beta1_b200 import case, geometry

FIELDS = ["Jac", "JDxi", "JDet", "JDze", "beta_xi", "beta_eta", "beta_zeta", "alpha_xi", "alpha_eta",
          "alpha_zeta", "dr_xi", "dr_eta", "dr_zeta", "Bcell_from_Bface_w", "Jcell_from_Jedge_w", "Area_xi", "Area_eta",
          "Area_zeta", "dl_xi", "dl_eta", "dl_zeta"]


def test_ghost_nodes_bitwise(golden_periodic):
    geom = golden_periodic["geom"]
    n = tuple(int(v) for v in golden_periodic["steps"]["n"])
    b = case.periodic_box_case(n).blocks[0]
    X = geometry.ghost_mesh(b.x, b.y, b.z, 4)
    assert X.a.shape == geom["X_node"].shape
    assert np.array_equal(X.a, geom["X_node"])


def test_geometry_fields_bitwise(golden_periodic):
    geom = golden_periodic["geom"]
    n = tuple(int(v) for v in golden_periodic["steps"]["n"])
    b = case.periodic_box_case(n).blocks[0]
    g = geometry.build(geometry.ghost_mesh(b.x, b.y, b.z, 4), b.ncell, 4)
    for name in FIELDS:
        lo, hi, a = g[name]
        assert tuple(lo) == tuple(int(v) for v in geom[name + "__lo"]), name
        assert a.shape == geom[name].shape, name
        assert np.array_equal(a, geom[name]), (name, np.abs(a - geom[name]).max())


def test_pole_shell_geometry_bitwise():
    """A single-block spherical shell with Pole patches at both ends of the
    polar index: the ghost node rows past each pole collapse onto the pole
    row (Grid::MeshTrans_Inner_Pole), and every geometry field, degenerate
    cells included, equals the reference's."""
    from conftest import load_golden
    geom = load_golden("shell_8x6x8_geom.npz")
    b = case.shell_case(8, 6, 8).blocks[0]
    X = geometry.block_ghost_mesh(b, 4)
    assert np.array_equal(X.a, geom["X_node"])
    with np.errstate(all="ignore"):
        g = geometry.build(X, b.ncell, 4)
    for name in FIELDS:
        lo, hi, a = g[name]
        assert tuple(lo) == tuple(int(v) for v in geom[name + "__lo"]), name
        assert np.array_equal(a, geom[name]), (name, np.abs(a - geom[name]).max())


def test_pole_shell_fixture_starts_from_the_seeded_state():
    """The Pole shell's step fixture (the reference's StepOnce on Pole
    patches) starts from the state regenerated from (case, seed)."""
    from conftest import load_golden
    g = load_golden("shell_8x6x8_steps.npz")
    n = tuple(int(v) for v in g["n"])
    spec = case.shell_case(*n)
    st = case.inflow_state(spec, seed=int(g["seed"]))
    for name in ("U_H", "B_xi", "B_eta", "B_zeta"):
        assert np.array_equal(st.fields[name].blocks[0].data, g["init/b0/" + name]), name
    assert float(g["s1/dt"]) > 0.0 and np.isfinite(g["s2/b0/U_H"]).all()


def test_block_ghost_mesh_without_poles_is_the_reflected_mesh():
    b = case.slab_case(6, (5, 6), (2, 2)).blocks[0]
    assert np.array_equal(geometry.block_ghost_mesh(b, 4).a, geometry.ghost_mesh(b.x, b.y, b.z, 4).a)


def test_pole_patch_rules():
    import pytest
    # the reference requires zeta as the rotation direction and an even,
    # unsplit azimuthal cell count (Grid::MeshTrans_Inner_Pole)
    with pytest.raises(ValueError):
        case.shell_case(4, 4, 5)
    b = case.shell_case(4, 4, 6).blocks[0]
    X = geometry.ghost_mesh(b.x, b.y, b.z, 4)
    with pytest.raises(ValueError):
        geometry.pole_ghosts(X, b.ncell, [((0, 4, 0, 4, 0, 0), "Pole")])
    Y = geometry.block_ghost_mesh(b, 4)
    o = Y.off
    # every ghost row past the low pole repeats the pole row over the inner i, k range
    for g in range(1, o + 1):
        assert np.array_equal(Y.a[o:o + 5, o - g, o:o + 7], Y.a[o:o + 5, o, o:o + 7])
        assert np.array_equal(Y.a[o:o + 5, o + 4 + g, o:o + 7], Y.a[o:o + 5, o + 4, o:o + 7])


def test_mercury_setup_has_every_key_the_solver_reads(tmp_path):
    """The setup files of a Mercury case (case.mercury_params) hold every key
    MercurySolver and the shared core read (Param::GetDou / GetInt / GetBoo
    keys of Z5_Mercury and src/), and a dipole list in the reference's LIST
    syntax."""
    from beta1_b200 import case
    keys = ["Archive_Output_Time", "CFL", "J_range_on", "J_range_start", "arti_eta_max", "continue_calc", "dimension",
            "eta_max_mercury", "implicit_resistive_ksp_atol", "implicit_resistive_ksp_max_it",
            "implicit_resistive_ksp_rtol", "is_Ambipolar_Efield", "is_Mercury_resistance",
            "is_local_artificial_resistivity", "local_arti_eta_max", "local_arti_r_cutoff", "local_arti_r_decay",
            "local_arti_x0", "local_arti_y0", "local_arti_z0", "max_Nstep", "max_Time", "mole_mass1", "mole_mass2",
            "n_resistive_subcycles", "ngg", "num_of_dipole", "output_residual", "output_step", "r_max", "r_min",
            "use_implicit_mercury_resistance"]
    dip = dict(x0=0.0, y0=0.0, z0=4.88e5, mx=0.0, my=0.0, mz=-2.83e19, a=5.0e2)
    p = case.mercury_params(num_of_dipole=1, dipoles=[dip])
    spec = case.CaseSpec(case.slab_blocks(6, (4, 4), (1, 1)), case.slab_interfaces(6, (4, 4), (1, 1)), p)
    case.write_case(str(tmp_path), spec)
    d = tmp_path / "CASE" / "setup"
    text = "".join((d / f).read_text() for f in ("0_General_Setting.txt", "1_Initial_condition.txt",
                                                 "2_Boundary_Condition.txt", "3_MHD_Control.txt"))
    words = set(text.split())
    assert [k for k in keys if k not in words] == []
    assert "eta_max_lunar" not in words and "is_Lunar_resistance" not in words
    ctl = (d / "3_MHD_Control.txt").read_text().splitlines()
    i = ctl.index("Dipole1         7")
    assert ctl[i + 2].split() == ["x0", "y0", "z0", "mx", "my", "mz", "a"]
    assert float(ctl[i + 3].split()[5]) == -2.83e19
