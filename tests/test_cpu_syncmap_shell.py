"""Compiled synchronisation of the single-block spherical shell (Solid_Surface
and Farfield in r, Pole patches at both ends of theta, phi periodic onto
itself), in the order the device runs it: the Pole ring kernels, the gather
of values read before the wall handler, the wall handler, the gather of
values it wrote, then the fixed values (syncmap.compile_shell).

That order is emulated here on the oracle's arrays (the ring kernels are the
oracle's restatement of the reference's Pole handlers) and compared, bitwise
and for every Sync group,
* with the reference's own Sync: the probe fixture (tests/golden/make_golden.py,
  shell_probe) holds what it leaves in every point after the group's fields
  were filled with their own point indices;
* with the oracle's Sync in the reference's order on a state in mid-run."""
import copy

import numpy as np
import pytest

from conftest import load_golden
from test_cpu_oracle_shell import build_shell_oracle, mhd_oracle, resistive_shell_params

from beta1_b200 import case, mhd, physics, syncmap

MASK = (1 << 40) - 1


def shell_tables(n=(8, 6, 8), resistive=False):
    spec = case.shell_case(*n)
    b = spec.blocks[0]
    q, B = physics.farfield_state(spec.params)
    u = [q[1] / q[0], q[2] / q[0], q[3] / q[0]]
    E_inf = [B[1] * u[2] - B[2] * u[1], B[2] * u[0] - B[0] * u[2], B[0] * u[1] - B[1] * u[0]]
    from beta1_b200 import geometry
    lay = mhd.HostLayout([b.ncell])
    maps = syncmap.compile_shell(lay, b.ncell, resistive, dict(qinf=q, B_imf=B, E_inf=E_inf),
                                 geometry.block_ghost_mesh(b, 4))
    return lay, maps


@pytest.fixture(scope="module")
def tables():
    return shell_tables()


def _points(o, names, ids):
    ids = np.asarray(ids, dtype=np.int64)
    fi = ids >> 56
    for f in np.unique(fi):
        sel = np.nonzero(fi == f)[0]
        assert np.all(((ids[sel] >> 40) & 0xFFFF) == 0)
        m, I, J, K = o.aos_points(names[f], 0, ids[sel] & MASK)
        G = o.blocks[0].G
        yield sel, o.blocks[0].f[names[f]], (m, I + G, J + G, K + G)


def _read(o, names, ids):
    v = np.empty(len(ids))
    for sel, arr, idx in _points(o, names, ids):
        v[sel] = arr[idx]
    return v


def _write(o, names, ids, v):
    for sel, arr, idx in _points(o, names, ids):
        arr[idx] = v[sel]


def device_order_sync(o, names, group, t):
    o.pole_rings(group)
    _write(o, names, t["dst"], _read(o, names, t["src"]))
    for (b, d) in t["walls"]:
        o.wall_u(b, d)
    _write(o, names, t["dst2"], _read(o, names, t["src2"]))
    _write(o, names, t["cdst"], t["cval"])


def test_table_structure(tables):
    lay, maps = tables
    assert set(maps) == set(syncmap.GROUPS) - set(syncmap.SHELL_SKIPPED)
    for group, t in maps.items():
        d1, s1, d2, s2 = t["dst"], t["src"], t["dst2"], t["src2"]
        # every point is written once, and no source is written by a gather
        allw = np.concatenate([d1, d2, t["cdst"]])
        assert np.unique(allw).size == allw.size, group
        assert np.intersect1d(np.concatenate([d1, d2]), np.concatenate([s1, s2])).size == 0, group
        # only the wall handler's group has copies after it
        assert (d2.size > 0) == bool(t["walls"]), group
    assert maps["Ucell"]["walls"] == [(0, -1)]


@pytest.fixture(scope="module")
def shell_oracle_mid():
    o = build_shell_oracle()
    o.step()
    return o


@pytest.mark.parametrize("group", [g for g in syncmap.GROUPS if g not in syncmap.SHELL_SKIPPED])
def test_device_order_equals_reference_sync(tables, shell_oracle_mid, group):
    lay, maps = tables
    names = [t[0] for t in lay.table]
    probe = load_golden("shell_8x6x8_probe.npz")
    o = copy.deepcopy(build_shell_oracle())
    blk = o.blocks[0]
    for f in syncmap.GROUPS[group]:
        loc, nc, ng = mhd_oracle.FIELDS[f]
        p = mhd_oracle.PLUS[loc]
        shape = tuple(blk.n[a] + p[a] + 2 * ng for a in range(3)) + (nc,)
        blk.set_ref(f, (-ng, -ng, -ng), (np.arange(np.prod(shape), dtype=np.float64) + 1.0).reshape(shape))
    device_order_sync(o, names, group, maps[group])
    for f in syncmap.GROUPS[group]:
        got = blk.get_ref(f).reshape(-1)
        ref = np.arange(got.size, dtype=np.float64) + 1.0
        ref[probe["%s/%s/0/dst" % (group, f)]] = probe["%s/%s/0/val" % (group, f)]
        bad = np.nonzero(got != ref)[0]
        assert bad.size == 0, (group, f, bad.size)
    # in mid-run: the device order against the reference's order
    a = copy.deepcopy(shell_oracle_mid)
    b = copy.deepcopy(shell_oracle_mid)
    a.sync(group)
    device_order_sync(b, names, group, maps[group])
    for f in syncmap.GROUPS[group]:
        assert np.array_equal(a.blocks[0].get_ref(f), b.blocks[0].get_ref(f)), (group, f)


def test_pole_directions_and_patches():
    from beta1_b200 import solver
    spec = case.shell_case(8, 6, 8)
    b = spec.blocks[0]
    assert solver.pole_directions(b) == [-2, 2]
    pats = solver.topology_patches("shell", b.ncell, b)
    assert [(p[0], p[1]) for p in pats] == [("Solid_Surface", -1), ("Pole", -2), ("Pole", 2)]
    assert pats[2][2] == (0, 6, 0) and pats[2][3] == (9, 7, 9)
    rows = solver.hall_zero_boxes(b.ncell, pats)
    # the eta Poles zero the xi and zeta edges of their node planes
    assert [0, 0, 0, 0, 8, 1, 9] in rows and [2, 0, 6, 0, 9, 7, 8] in rows
    assert solver.topology_patches("periodic", b.ncell, b) == []


def test_batch_of_shells_merges_every_list():
    from beta1_b200 import geometry, solver
    specs = [case.shell_case(6, 4, 6), case.shell_case(8, 6, 8)]
    lays = [mhd.HostLayout([s.blocks[0].ncell]) for s in specs]
    per_run = [(solver.shell_tables(s, geometry.block_ghost_mesh(s.blocks[0], 4), lay), r)
               for r, (s, lay) in enumerate(zip(specs, lays))]
    merged = syncmap.merge_runs(per_run)
    for group in merged:
        for key in ("dst", "src", "dst2", "src2", "cdst"):
            assert merged[group][key].size == sum(m[group][key].size for m, _ in per_run), (group, key)
        blocks = (merged[group]["dst2"] >> 40) & 0xFFFF
        assert set(blocks.tolist()) <= {0, 1}
    assert merged["Ucell"]["walls"] == [(0, -1), (1, -1)]
    assert set(((merged["Ucell"]["dst2"] >> 40) & 0xFFFF).tolist()) == {0, 1}


def test_device_order_steps_equal_reference(tables):
    """Two StepOnce with every Sync in the device order (compiled tables) and
    the device's derived-field order: the reference's fields bitwise."""
    lay, maps = tables
    names = [t[0] for t in lay.table]

    class DeviceOrder(mhd_oracle.ShellOracle):
        def sync(self, group):
            device_order_sync(self, names, group, maps[group])

        def update_magnetic_derived(self):
            # k_bcell, Sync, B_zeta rewrite, k_jedge, Sync, J_cell, its ring, Sync
            blk = self.blocks[0]
            self.calc_bcell(blk)
            self.sync("B_cell")
            self.bzeta_pole_rewrite()
            self.curl_adj(blk, ("B_xi", "B_eta", "B_zeta"), ("J_xi", "J_eta", "J_zeta"))
            self.sync("Jedge")
            self.calc_jcell(blk)
            self.jcell_pole_repair()
            self.sync("J_cell")

    ref = build_shell_oracle()
    o = DeviceOrder.__new__(DeviceOrder)
    o.__dict__.update(copy.deepcopy(ref.__dict__))
    # restart load through the device order
    g = load_golden("shell_8x6x8_steps.npz")
    from conftest import shell_setup
    spec, st = shell_setup(g)
    for name in ("U_H", "B_xi", "B_eta", "B_zeta"):
        fa = st.fields[name].blocks[0]
        o.blocks[0].set_ref(name, fa.lo, fa.data)
    o.sync("Ucell")
    o.sync("Bface")
    o.update_derived()
    for s in (0, 1, 2):
        if s:
            assert o.step() == float(g["s%d/dt" % s])
        o.calc_divb()
        for key in g.files:
            if not key.startswith("s%d/b0/" % s) or key.endswith("__lo"):
                continue
            f = key.split("/")[-1]
            if s == 0 and f.startswith(("E", "RHS")):
                continue
            assert np.array_equal(o.blocks[0].get_ref(f), g[key]), (s, f)


@pytest.mark.parametrize("n", [(10, 5, 12), (6, 2, 4)])
def test_device_order_on_other_shells(n):
    """Other shell sizes (an odd polar count; two polar cells, where the two
    pole rings are neighbours): every group in the device order equals the
    oracle's Sync in the reference's order, in mid-run."""
    lay, maps = shell_tables(n)
    names = [t[0] for t in lay.table]
    spec = case.shell_case(*n)
    mid = build_shell_oracle(n, seed=31)
    mid.step()
    for group in maps:
        a = copy.deepcopy(mid)
        b = copy.deepcopy(mid)
        a.sync(group)
        device_order_sync(b, names, group, maps[group])
        for f in syncmap.GROUPS[group]:
            assert np.array_equal(a.blocks[0].get_ref(f), b.blocks[0].get_ref(f)), (n, group, f)
    assert spec.blocks[0].ncell == n


@pytest.fixture(scope="module")
def resistive_tables():
    return shell_tables(resistive=True)


def test_resistive_tables_hold_every_group(resistive_tables):
    lay, maps = resistive_tables
    assert set(maps) == set(syncmap.GROUPS)
    for group, t in maps.items():
        allw = np.concatenate([t["dst"], t["dst2"], t["cdst"]])
        assert np.unique(allw).size == allw.size, group


@pytest.mark.parametrize("group", ["Eres", "Eres1form", "J_cell", "Eface", "Eedge", "Jedge", "B_cell", "Ucell"])
def test_resistive_device_order_equals_reference_sync(resistive_tables, group):
    """With is_Lunar_resistance: the compiled tables (after the Eres_eta
    regulation on the pole rings) equal the reference's Sync on the probe
    fixture, and the oracle's Sync in the reference's order in mid-run."""
    lay, maps = resistive_tables
    names = [t[0] for t in lay.table]
    probe = load_golden("shell_8x6x8_r10_probe.npz")
    over = resistive_shell_params()
    o = build_shell_oracle(**over)
    blk = o.blocks[0]
    for f in syncmap.GROUPS[group]:
        loc, nc, ng = mhd_oracle.FIELDS[f]
        p = mhd_oracle.PLUS[loc]
        shape = tuple(blk.n[a] + p[a] + 2 * ng for a in range(3)) + (nc,)
        blk.set_ref(f, (-ng, -ng, -ng), (np.arange(np.prod(shape), dtype=np.float64) + 1.0).reshape(shape))
    device_order_sync(o, names, group, maps[group])
    for f in syncmap.GROUPS[group]:
        got = blk.get_ref(f).reshape(-1)
        ref = np.arange(got.size, dtype=np.float64) + 1.0
        ref[probe["%s/%s/0/dst" % (group, f)]] = probe["%s/%s/0/val" % (group, f)]
        assert np.count_nonzero(got != ref) == 0, (group, f)
    mid = build_shell_oracle(**over)
    mid.step()
    a = copy.deepcopy(mid)
    b = copy.deepcopy(mid)
    a.sync(group)
    device_order_sync(b, names, group, maps[group])
    for f in syncmap.GROUPS[group]:
        assert np.array_equal(a.blocks[0].get_ref(f), b.blocks[0].get_ref(f)), (group, f)


def test_resistive_device_order_steps_equal_reference(resistive_tables):
    """Two StepOnce with the explicit resistive sub-cycles, every Sync in the
    device order (compiled resistive tables) and the device's derived-field
    order in each sub-cycle: the reference's fields bitwise, Eres included."""
    lay, maps = resistive_tables
    names = [t[0] for t in lay.table]

    class DeviceOrder(mhd_oracle.ShellOracle):
        def sync(self, group):
            device_order_sync(self, names, group, maps[group])

    ref = build_shell_oracle(**resistive_shell_params())
    o = DeviceOrder.__new__(DeviceOrder)
    o.__dict__.update(copy.deepcopy(ref.__dict__))
    g = load_golden("shell_8x6x8_r10_steps.npz")
    for s in (1, 2):
        assert o.step() == float(g["s%d/dt" % s])
        o.calc_divb()
        for key in g.files:
            if not key.startswith("s%d/b0/" % s) or key.endswith("__lo"):
                continue
            f = key.split("/")[-1]
            assert np.array_equal(o.blocks[0].get_ref(f), g[key]), (s, f)


@pytest.mark.parametrize("n", [(10, 5, 12), (6, 2, 4)])
def test_resistive_device_order_on_other_shells(n):
    """The resistive tables on other shell sizes (an odd polar count; two
    polar cells): every group, the Eres groups included, in the device order
    equals the oracle's Sync in the reference's order after a step with the
    explicit resistive sub-cycles."""
    lay, maps = shell_tables(n, resistive=True)
    names = [t[0] for t in lay.table]
    mid = build_shell_oracle(n, seed=33, **resistive_shell_params())
    mid.step()
    assert np.abs(mid.blocks[0].get_ref("Eres_eta")).max() > 0.0
    for group in maps:
        a = copy.deepcopy(mid)
        b = copy.deepcopy(mid)
        a.sync(group)
        device_order_sync(b, names, group, maps[group])
        for f in syncmap.GROUPS[group]:
            assert np.array_equal(a.blocks[0].get_ref(f), b.blocks[0].get_ref(f)), (n, group, f)
