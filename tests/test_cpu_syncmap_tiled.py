"""Compiled boundary/halo synchronisation of a tiled slab (4 blocks, periodic
transverse wraps, Solid_Surface inner wall, Farfield outer boundary) against
the reference's own Sync, group by group.

The probe fixtures record what the reference's LunarBoundary::Sync leaves
in every point of every field of a group after each point was pre-filled
with its own index (tests/golden/make_golden.py).  From the compiled tables
(composed copies + fixed values) the same end state is predicted and must
match exactly; the Solid_Surface fluid handler computes values from the
index-filled state, so its cells are excluded here (it is checked by the
step parity tests).
"""
import numpy as np
import pytest

from conftest import load_golden

from beta1_b200 import case, geometry, mhd, physics, syncmap

NR, NT, TILES = 6, (5, 6), (2, 2)


def compile_maps(resistive):
    spec = case.slab_case(NR, NT, TILES, is_Lunar_resistance=resistive, use_implicit_lunar_resistance=resistive)
    lay = mhd.HostLayout([b.ncell for b in spec.blocks])
    q, B = physics.farfield_state(spec.params)
    u = [q[1] / q[0], q[2] / q[0], q[3] / q[0]]
    E_inf = [B[1] * u[2] - B[2] * u[1], B[2] * u[0] - B[0] * u[2], B[0] * u[1] - B[1] * u[0]]
    X = [geometry.ghost_mesh(b.x, b.y, b.z, 4) for b in spec.blocks]
    maps = syncmap.compile_tiled(lay, syncmap.TiledLayout(spec.blocks[0].ncell, TILES), bool(resistive),
                                 dict(qinf=q, B_imf=B, E_inf=E_inf), X)
    return lay, maps


def final_arrays(probe, group, field, lay):
    out = []
    for b in range(TILES[0] * TILES[1]):
        info = lay.field_info(field, b)
        size = int(np.prod([h - l for l, h in zip(info["lo"], info["hi"])])) * info["ncomp"]
        v = np.arange(size, dtype=np.float64) + b * 2.0 ** 32 + 1.0
        v[probe["%s/%s/%d/dst" % (group, field, b)]] = probe["%s/%s/%d/val" % (group, field, b)]
        out.append(v)
    return out


def wall_mask(lay, b, field, maps_group):
    info = lay.field_info(field, b)
    size = int(np.prod([h - l for l, h in zip(info["lo"], info["hi"])])) * info["ncomp"]
    if field != "U_H" or (b, -1) not in maps_group["walls"]:
        return np.zeros(size, dtype=bool)
    I, J, K = np.meshgrid(*[np.arange(l, h) for l, h in zip(info["lo"], info["hi"])], indexing="ij")
    w = ((I <= 0) & (J >= 0) & (J < NT[0]) & (K >= 0) & (K < NT[1])).ravel()
    return np.repeat(w, info["ncomp"])


@pytest.mark.parametrize("resistive", [0, 1])
def test_tiled_maps_equal_reference_sync(resistive):
    probe = load_golden("slab_%dx%dx%d_t%dx%d_r%d%d_probe.npz" % ((NR,) + NT + TILES + (resistive, resistive)))
    lay, maps = compile_maps(resistive)
    checked = 0
    for group, fields in syncmap.GROUPS.items():
        m = maps[group]
        for field in fields:
            fi = lay.index[field]
            ref = final_arrays(probe, group, field, lay)
            for b in range(len(ref)):
                pred = np.arange(ref[b].size, dtype=np.float64) + b * 2.0 ** 32 + 1.0
                sel = ((m["dst"] >> 56) == fi) & (((m["dst"] >> 40) & 0xFFFF) == b)
                dd = m["dst"][sel] & ((1 << 40) - 1)
                ss = m["src"][sel]
                assert np.all((ss >> 56) == fi), (group, field)
                # a composed copy delivers the value its source holds once the group's fixed
                # values and handlers ran; sources are never copy destinations themselves
                sb = (ss >> 40) & 0xFFFF
                so = ss & ((1 << 40) - 1)
                pred[dd] = np.array([ref[int(x)][int(y)] for x, y in zip(sb, so)]) if ss.size else pred[dd]
                cs = ((m["cdst"] >> 56) == fi) & (((m["cdst"] >> 40) & 0xFFFF) == b)
                pred[m["cdst"][cs] & ((1 << 40) - 1)] = m["cval"][cs]
                bad = (pred != ref[b]) & ~wall_mask(lay, b, field, m)
                assert not bad.any(), (group, field, b, int(bad.sum()))
                checked += 1
    assert checked == sum(len(f) for f in syncmap.GROUPS.values()) * TILES[0] * TILES[1]


def test_composed_sources_are_not_destinations():
    lay, maps = compile_maps(1)
    for group, m in maps.items():
        assert not np.isin(m["src"], m["dst"]).any(), group
