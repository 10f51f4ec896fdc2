"""Compiled synchronisation of the single-block spherical shell (Solid_Surface
and Farfield in r, Pole patches at both ends of theta, phi periodic onto
itself) against the reference's own Sync, for every group whose Pole
handling is a copy: U_plus, the face EMF, J_cell, dB, Badd and the Hall edge
EMF.  The probe fixture (tests/golden/make_golden.py, shell_probe) holds what
the reference's Sync leaves in every point after each point was pre-filled
with its own index.  The shell's gather entries deliver pre-sync values (a
Pole ghost copy reads the wall slab before the wall handler zeroes it), so a
copied point must hold its source's index, a fixed point its constant, and
every other point its own index."""
import numpy as np

from conftest import load_golden

from beta1_b200 import case, mhd, syncmap


def test_shell_tables_equal_reference_sync():
    probe = load_golden("shell_8x6x8_probe.npz")
    spec = case.shell_case(8, 6, 8)
    lay = mhd.HostLayout([spec.blocks[0].ncell])
    maps = syncmap.compile_shell(lay, spec.blocks[0].ncell, False)
    assert set(maps) == set(syncmap.GROUPS) - set(syncmap.SHELL_POLE_HANDLED)
    mask = (1 << 40) - 1
    checked = 0
    for group, m in maps.items():
        for field in syncmap.GROUPS[group]:
            fi = lay.index[field]
            info = lay.field_info(field, 0)
            size = int(np.prod([h - l for l, h in zip(info["lo"], info["hi"])])) * info["ncomp"]
            ref = np.arange(size, dtype=np.float64) + 1.0
            ref[probe["%s/%s/0/dst" % (group, field)]] = probe["%s/%s/0/val" % (group, field)]
            pred = np.arange(size, dtype=np.float64) + 1.0
            sel = (m["dst"] >> 56) == fi
            dd, ss = m["dst"][sel] & mask, m["src"][sel] & mask
            assert np.all((m["src"][sel] >> 56) == fi)
            # sources are never destinations: one gather of pre-sync values
            assert np.intersect1d(dd, ss).size == 0, (group, field)
            pred[dd] = ss + 1.0
            cs = (m["cdst"] >> 56) == fi
            pred[m["cdst"][cs] & mask] = m["cval"][cs]
            bad = np.nonzero(pred != ref)[0]
            assert bad.size == 0, (group, field, bad.size)
            checked += dd.size
    assert checked > 10000

