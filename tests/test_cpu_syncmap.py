"""The compiled periodic Sync tables equal, point by point, what the
reference's own LunarBoundary::Sync does on a self-periodic block (probe
fixtures: every point pre-filled with its own index, then the reference Sync
ran, tests/golden/make_golden.py)."""
import numpy as np

from beta1_b200 import rst, syncmap

LOCS = {"U_H": 0, "B_xi": 1, "B_eta": 2, "B_zeta": 3, "Eface_xi": 1, "Eface_eta": 2, "Eface_zeta": 3,
        "E_xi": 4, "E_eta": 5, "E_zeta": 6, "J_xi": 4, "J_eta": 5, "J_zeta": 6, "B_cell": 0, "Bind_cell": 0,
        "J_cell": 0, "U_plus": 0}
NCOMP = {"U_H": 5, "Eface_xi": 3, "Eface_eta": 3, "Eface_zeta": 3, "B_cell": 3, "Bind_cell": 3, "J_cell": 3,
         "U_plus": 3}


def test_periodic_maps_equal_reference_probe(golden_periodic):
    probe = golden_periodic["probe"]
    n = tuple(int(v) for v in golden_periodic["steps"]["n"])
    checked = 0
    for key in probe.files:
        if not key.endswith("/dst"):
            continue
        group, field, _ = key.split("/")
        assert field in syncmap.GROUPS[group]
        loc = LOCS[field]
        lo, hi = rst.extent(loc, n, 4)
        info = dict(lo=lo, hi=hi, ncomp=NCOMP.get(field, 1), loc=loc)
        d, s = syncmap.periodic_field_map(info, n)
        order = np.argsort(d)
        ref_d = probe[key]
        ref_s = probe[key[:-3] + "src"]
        ro = np.argsort(ref_d)
        assert np.array_equal(d[order], ref_d[ro]), (group, field)
        assert np.array_equal(s[order], ref_s[ro]), (group, field)
        checked += 1
    assert checked == 17
