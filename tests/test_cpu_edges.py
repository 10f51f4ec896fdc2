"""Edge ownership (alias -> owner table) and the implicit resistive unknowns
of a tiled slab against the reference's own tables (HALO_OWNER local
aliases and LunarSolver::implicit_resistive_dofs_, dumped by the reference
solver, tests/golden/make_golden.py)."""
import numpy as np

from conftest import load_golden

from beta1_b200 import case, edges, geometry, physics

NR, NT, TILES = 6, (5, 6), (2, 2)


def test_alias_owner_table_matches_reference():
    g = load_golden("slab_%dx%dx%d_t%dx%d_r11_owners.npz" % ((NR,) + NT + TILES))
    alias, owner, owners = edges.tiled_owners((NR,) + NT, TILES)
    ref = g["alias"]
    mine = np.concatenate([alias, owner, np.ones((len(alias), 1), dtype=alias.dtype)], axis=1)
    key = lambda a: a[np.lexsort(a[:, :5].T[::-1])]
    assert mine.shape == ref.shape
    assert np.array_equal(key(mine), key(ref.astype(mine.dtype)))
    assert len(owners) == int(g["n_owner"])


def test_resistive_unknowns_and_eta_match_reference():
    g = load_golden("slab_%dx%dx%d_t%dx%d_r11_owners.npz" % ((NR,) + NT + TILES))
    over = {k.split("/", 1)[1]: g[k].item() for k in g.files if k.startswith("param/")}
    spec = case.slab_case(NR, NT, TILES, is_Lunar_resistance=1, use_implicit_lunar_resistance=1, **over)
    X = [geometry.ghost_mesh(b.x, b.y, b.z, 4) for b in spec.blocks]
    _, _, owners = edges.tiled_owners((NR,) + NT, TILES)
    dofs, eta = edges.resistive_dofs(owners, X, physics.constants(spec.params)["inver_Rem"])
    assert len(dofs) > 0
    assert np.array_equal(dofs, g["dof"].astype(dofs.dtype))  # same unknowns, same solve order
    assert np.array_equal(eta, g["eta"])
