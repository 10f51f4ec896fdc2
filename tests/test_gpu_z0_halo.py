"""Z0-style halo smoke driver (oracle/_ref/z0_halo_b200, source
beta1_b200/dropin/z0_halo_b200.cpp): the reference's kept grid / topology /
field / halo API sets the case up, the device gather of U_H and the face B
fields is derived from the reference's own face, edge and vertex exchanges,
and on seeded random fields the device's gather must equal the reference's
host exchange at every point, bit for bit.  Layouts: the periodic box (a
block periodic onto itself), the 4-block tiled slab (face, edge and vertex
halos across blocks) and the Pole shell."""
import os
import subprocess

import pytest

from conftest import ROOT, load_golden, periodic_setup, shell_setup, slab_setup

from beta1_b200 import case

pytestmark = pytest.mark.gpu

BIN = os.path.join(ROOT, "oracle", "_ref", "z0_halo_b200")
CASES = {"periodic": (periodic_setup, "periodic_8x6x5_steps.npz"),
         "slab": (slab_setup, "slab_6x5x6_t2x2_r00_steps.npz"),
         "shell": (shell_setup, "shell_8x6x8_steps.npz")}


@pytest.mark.parametrize("name", list(CASES))
def test_device_halo_gather_equals_reference_exchange(name, tmp_path):
    if not os.path.exists(BIN):
        pytest.skip("oracle/_ref/z0_halo_b200 is not built (make -C oracle dropin)")
    setup, fixture = CASES[name]
    spec, _ = setup(load_golden(fixture))
    case.write_case(str(tmp_path), spec)
    r = subprocess.run([BIN], cwd=str(tmp_path), stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True,
                       timeout=300)
    assert r.returncode == 0, (r.stdout[-1500:], r.stderr[-1500:])
    lines = [ln for ln in r.stdout.splitlines() if "gather entries" in ln]
    assert len(lines) == 4, r.stdout[-1500:]
    for ln in lines:
        assert ln.endswith(" 0 differ"), ln
        assert int(ln.split(":")[1].split()[0]) > 0, ln  # every field has ghost copies
