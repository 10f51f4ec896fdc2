"""Host logic of parameter sweeps: the sweep's random draws and the merged
sync tables of a batch of runs (no GPU)."""
import numpy as np

from beta1_b200 import case, mhd, physics, syncmap


def test_mt19937_64_known_answer():
    # the C++ standard's check value of std::mt19937_64 ([rand.predef]):
    # the 10000th output of a default-constructed engine (seed 5489)
    g = case.MT19937_64(5489)
    for _ in range(9999):
        g.next()
    assert g.next() == 9981545732273789042


def test_sweep_draws_in_range_and_reproducible():
    a = case.sweep_cases(nruns=48)
    b = case.sweep_cases(nruns=48)
    assert [d for _, d in a] == [d for _, d in b]
    for spec, d in a:
        assert 32 <= d["nr"] <= 128 and 24 <= d["nt"] <= 96
        assert 4.0 <= d["mach"] < 12.0 and 0.0 <= d["angle"] < 180.0
        assert spec.blocks[0].ncell == (d["nr"], d["nt"], d["nt"])
        q, B = physics.farfield_state(spec.params)
        assert abs(q[1] / q[0] + d["mach"]) < 1e-12
    # uneven sizes
    assert len({d["nr"] * d["nt"] ** 2 for _, d in a}) > 40


def _tiled_maps(spec):
    from beta1_b200 import geometry
    b = spec.blocks[0]
    X = [geometry.ghost_mesh(bb.x, bb.y, bb.z, 4) for bb in spec.blocks]
    lay = mhd.HostLayout([bb.ncell for bb in spec.blocks])
    q, B = physics.farfield_state(spec.params)
    u = [q[1] / q[0], q[2] / q[0], q[3] / q[0]]
    E = [B[1] * u[2] - B[2] * u[1], B[2] * u[0] - B[0] * u[2], B[0] * u[1] - B[1] * u[0]]
    return syncmap.compile_tiled(lay, syncmap.TiledLayout(b.ncell, spec.tiles), False, dict(qinf=q, B_imf=B, E_inf=E),
                                 X)


def test_merged_tables_address_each_runs_own_blocks():
    runs = [case.slab_case(6, (5, 6), (2, 2)), case.slab_case(7, (4, 4), (1, 1), mach_u=5.0),
            case.periodic_box_case((5, 4, 3))]
    per_run, off = [], 0
    for spec in runs:
        if len(spec.blocks) == 1 and not hasattr(spec, "tiles"):
            maps = syncmap.periodic_maps(mhd.HostLayout([spec.blocks[0].ncell]), spec.blocks[0].ncell)
        else:
            maps = _tiled_maps(spec)
        per_run.append((maps, off))
        off += len(spec.blocks)
    merged = syncmap.merge_runs(per_run)
    all_cells = [b.ncell for spec in runs for b in spec.blocks]
    lay = mhd.HostLayout(all_cells)
    for group, m in merged.items():
        n = 0
        for (maps, o), spec in zip(per_run, runs):
            mm = maps[group]
            k = mm["dst"].size
            blk_d = (m["dst"][n:n + k] >> 40) & 0xFFFF
            blk_s = (m["src"][n:n + k] >> 40) & 0xFFFF
            # a run's copies stay inside its own blocks
            assert ((blk_d >= o) & (blk_d < o + len(spec.blocks))).all()
            assert ((blk_s >= o) & (blk_s < o + len(spec.blocks))).all()
            # and are the run's own table with the block field moved
            assert np.array_equal(m["dst"][n:n + k] - (np.int64(o) << 40), mm["dst"])
            n += k
        assert n == m["dst"].size
        assert all(0 <= b < len(all_cells) for b, _ in m["walls"])
    # the batch layout's point ids are those of the shifted tables
    assert lay.point_base("U_H", 4) == syncmap.shift_blocks({"g": dict(
        dst=np.array([mhd.HostLayout([(1, 1, 1)]).point_base("U_H", 0)]), src=np.zeros(1, np.int64),
        cdst=np.zeros(0, np.int64), cval=np.zeros(0), walls=[])}, 4)["g"]["dst"][0]


def test_shell_sweep_same_draws():
    """grid="shell": the same draws, each run a spherical shell with Poles and
    an even azimuthal cell count (Nt rounded up)."""
    from beta1_b200 import case, solver
    slab = case.sweep_cases(6)
    shell = case.sweep_cases(6, grid="shell")
    for (sp_a, va), (sp_b, vb) in zip(slab, shell):
        assert va == vb
        n = sp_b.blocks[0].ncell
        assert n == (va["nr"], va["nt"], va["nt"] + (va["nt"] & 1))
        assert solver.pole_directions(sp_b.blocks[0]) == [-2, 2]
        assert sp_b.params["INITIAL"] == sp_a.params["INITIAL"]
