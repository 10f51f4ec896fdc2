"""Discrete identities of the path (known answers with no fixture): the face
area vectors of every cell close (the geometric conservation law), the
curl of any edge field has no cell divergence, and a uniform state stays
uniform through a StepOnce.  Checked on the oracle and the host geometry,
which the reference and the device match bit for bit (the parity tests), so
the identities hold there to the same round-off."""
import os
import sys

import numpy as np
import pytest

from conftest import ROOT

from beta1_b200 import case, geometry

sys.path.insert(0, os.path.join(ROOT, "oracle"))
import mhd_oracle  # noqa: E402

GRIDS = {"periodic": lambda: case.periodic_box_case((8, 6, 5)),
         "slab": lambda: case.slab_case(6, (5, 6), (1, 1)),
         "shell": lambda: case.shell_case(8, 6, 8)}


@pytest.mark.parametrize("name", list(GRIDS))
def test_face_vectors_of_every_cell_close(name):
    spec = GRIDS[name]()
    b = spec.blocks[0]
    n = b.ncell
    g = geometry.build(geometry.block_ghost_mesh(b, 4), n, 4)

    def face(nm, di, dj, dk):
        lo, hi, a = g[nm]
        return a[di - lo[0]:di - lo[0] + n[0], dj - lo[1]:dj - lo[1] + n[1], dk - lo[2]:dk - lo[2] + n[2]]

    s = (face("JDxi", 1, 0, 0) - face("JDxi", 0, 0, 0) + face("JDet", 0, 1, 0) - face("JDet", 0, 0, 0)
         + face("JDze", 0, 0, 1) - face("JDze", 0, 0, 0))
    scale = max(np.abs(g[k][2]).max() for k in ("JDxi", "JDet", "JDze"))
    assert np.abs(s).max() <= 1e-13 * scale, (name, np.abs(s).max() / scale)


def test_curl_of_edge_field_has_no_divergence():
    n = (8, 6, 8)
    o = mhd_oracle.Oracle([n], {})
    blk = o.blocks[0]
    rng = np.random.default_rng(11)
    for nm in ("E_xi", "E_eta", "E_zeta"):
        blk.f[nm][...] = rng.standard_normal(blk.f[nm].shape)
    o.curl_e2f(blk, ("E_xi", "E_eta", "E_zeta"), ("RHS_B_xi", "RHS_B_eta", "RHS_B_zeta"), -1.0)
    lo, hi = blk.inner(0)
    bx = lambda d: blk.box("RHS_B_xi", 0, lo, hi, d)
    be = lambda d: blk.box("RHS_B_eta", 0, lo, hi, d)
    bz = lambda d: blk.box("RHS_B_zeta", 0, lo, hi, d)
    z = (0, 0, 0)
    div = bx((1, 0, 0)) - bx(z) + be((0, 1, 0)) - be(z) + bz((0, 0, 1)) - bz(z)
    assert np.abs(div).max() <= 1e-14 * np.abs(bx(z)).max() * 10


def test_uniform_state_stays_uniform(golden_periodic):
    """Uniform rho, v and p with a uniform applied field (Badd = B0 . JD, no
    induced field): after a StepOnce the state is unchanged and the induced
    field still zero, to round-off, on the periodic curvilinear box."""
    from test_cpu_oracle import build_periodic_oracle
    from beta1_b200 import solver
    o = build_periodic_oracle(golden_periodic)
    blk = o.blocks[0]
    n = blk.n
    st = case.initial_state(case.periodic_box_case(n), B0=None, sigma=0.0)
    for name in ("U_H", "B_xi", "B_eta", "B_zeta"):
        fa = st.fields[name].blocks[0]
        blk.set_ref(name, fa.lo, fa.data)
    B0 = (0.3, -0.2, 0.5)
    for fname, jd in (("Badd_xi", "JDxi"), ("Badd_eta", "JDet"), ("Badd_zeta", "JDze")):
        JD = blk.get_ref(jd)
        loc, nc, ng = mhd_oracle.FIELDS[jd]
        blk.set_ref(fname, (-ng, -ng, -ng), solver.badd_faces(JD, B0))
    o.sync("Ucell")
    o.sync("Bface")
    o.update_derived()
    lo, hi = blk.inner(0)
    U0 = [blk.box("U_H", m, lo, hi).copy() for m in range(5)]
    for m in range(5):
        assert np.ptp(U0[m]) == 0.0
    o.step()
    for m in range(5):
        U1 = blk.box("U_H", m, lo, hi)
        assert np.abs(U1 - U0[m]).max() <= 1e-13 * max(1.0, np.abs(U0[m]).max()), m
    scale = np.abs(blk.f["Badd_xi"]).max()
    for nm in ("B_xi", "B_eta", "B_zeta"):
        assert np.abs(blk.f[nm]).max() <= 1e-13 * scale, nm


def test_fast_cell_drives_dt_below_the_abort_threshold(golden_periodic):
    """The premise of the device's dt-guard test: one cell moving at 1e9 (a
    state injected on the host) bounds the CFL time step below dt_abort = 1e-7
    (LunarSolver_Timestep.cpp:128-139), where StepOnce aborts and the device
    step returns MHD_EDT instead."""
    from test_cpu_oracle import build_periodic_oracle
    o = build_periodic_oracle(golden_periodic)
    blk = o.blocks[0]
    G = blk.G
    rho = blk.f["U_H"][0][G + 2, G + 3, G + 1]
    blk.f["U_H"][1][G + 2, G + 3, G + 1] = 1e9 * rho
    o.sync("Ucell")
    o.sync("Bface")
    o.update_derived()
    assert o.compute_timestep() < 1e-7
