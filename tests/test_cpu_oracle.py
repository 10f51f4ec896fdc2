"""Pins the numpy restatement in oracle/mhd_oracle.py against the reference.

The oracle is given exactly what the reference used (geometry fields, the
initial state, and the reference's own Sync tables read off its probe
fixture) and must reproduce the reference's fields after every StepOnce of
the committed golden run.  It follows the reference's floating-point
operation order, so the expected agreement is bitwise; the bound is the
FP64 tolerance of 1e-12 relative L2 per field per step.
"""
import os
import sys

import numpy as np
import pytest

from conftest import ROOT, rel_l2

sys.path.insert(0, os.path.join(ROOT, "oracle"))
import mhd_oracle  # noqa: E402

TOL = 1e-12
GEOM = ["Jac", "JDxi", "JDet", "JDze", "beta_xi", "beta_eta", "beta_zeta", "alpha_xi", "alpha_eta", "alpha_zeta",
        "Bcell_from_Bface_w", "Jcell_from_Jedge_w", "Badd_xi", "Badd_eta", "Badd_zeta"]
COMPARE = ["U_H", "B_xi", "B_eta", "B_zeta", "PV_H", "U_plus", "B_cell", "Bind_cell", "J_xi", "J_eta", "J_zeta",
           "J_cell", "E_xi", "E_eta", "E_zeta", "Eface_xi", "Eface_eta", "Eface_zeta", "RHS_H", "RHS_B_xi",
           "RHS_B_eta", "RHS_B_zeta", "divB"]


def oracle_consts(params):
    from beta1_b200 import physics
    c = physics.constants(params)
    return dict(gamma=c["gamma"], cfl=c["cfl"], inver_MA2=c["inver_MA2"], momentum_hall_coeff=c["momentum_hall_coeff"],
                state_coeff=c["state_coeff"], M_H=c["M_H"], M_ref=c["M_ref"], ne_hall_floor=c["ne_hall_floor"])


def build_periodic_oracle(gp):
    g, geom, probe = gp["steps"], gp["geom"], gp["probe"]
    from beta1_b200 import case
    n = tuple(int(v) for v in g["n"])
    o = mhd_oracle.Oracle([n], oracle_consts(case.periodic_box_case(n).params))
    blk = o.blocks[0]
    for name in GEOM:
        blk.set_ref(name, tuple(geom[name + "__lo"]), geom[name])
    for name in ("U_H", "B_xi", "B_eta", "B_zeta"):
        blk.set_ref(name, tuple(g["init/" + name + "__lo"]), g["init/" + name])
    for key in probe.files:
        if key.endswith("/dst"):
            group, field, _ = key.split("/")
            o.add_copies(group, field, 0, probe[key], field, 0, probe[key[:-3] + "src"])
    return o


@pytest.fixture(scope="module")
def oracle_run(golden_periodic):
    g = golden_periodic["steps"]
    o = build_periodic_oracle(golden_periodic)
    o.sync("Ucell")
    o.sync("Bface")
    o.update_derived()
    o.calc_divb()
    out = {0: {f: o.blocks[0].get_ref(f) for f in COMPARE}}
    dts = {}
    nsteps = max(int(k.split("/")[0][1:]) for k in g.files if k[0] == "s" and k[1].isdigit())
    for s in range(1, nsteps + 1):
        dts[s] = o.step()
        o.calc_divb()
        out[s] = {f: o.blocks[0].get_ref(f) for f in COMPARE}
    return g, out, dts, nsteps


def test_oracle_matches_reference_steps(oracle_run):
    g, out, dts, nsteps = oracle_run
    worst = 0.0
    for s in range(nsteps + 1):
        for f in COMPARE:
            if s == 0 and f.startswith(("E", "RHS")):
                continue
            ref = g["s%d/%s" % (s, f)]
            got = out[s][f]
            assert got.shape == ref.shape, (s, f, got.shape, ref.shape)
            e = rel_l2(got, ref)
            worst = max(worst, e)
            assert e <= TOL, f"step {s} field {f}: rel L2 {e:.3e}"
    print("oracle vs reference: max rel L2 %.3e" % worst)


def test_oracle_state_bitwise(oracle_run):
    g, out, dts, nsteps = oracle_run
    for s in range(1, nsteps + 1):
        for f in ("U_H", "B_xi", "B_eta", "B_zeta"):
            assert np.array_equal(out[s][f], g["s%d/%s" % (s, f)]), (s, f)


def test_oracle_dt_exact(oracle_run):
    g, out, dts, nsteps = oracle_run
    for s in range(1, nsteps + 1):
        assert dts[s] == float(g["s%d/dt" % s])


# --------------------------------------------------------------------------
# tiled slab: 4 blocks, Solid_Surface wall, Farfield, with and without the
# implicit resistive solve
# --------------------------------------------------------------------------
SLAB_FIELDS = COMPARE + ["Eres_xi", "Eres_eta", "Eres_zeta"]
SLAB_CASES = {"ideal": ("slab_6x5x6_t2x2_r00_steps.npz", 1e-12),
              "implicit_resistive": ("slab_6x5x6_t2x2_r11_steps.npz", 1e-10),
              "explicit_resistive": ("slab_6x5x6_t2x2_r10_steps.npz", 1e-12),
              "single_tile": ("slab_6x5x6_t1x1_r00_steps.npz", 1e-12)}


def build_slab_oracle(g):
    from beta1_b200 import edges, geometry, mhd, physics, solver, syncmap
    from conftest import slab_setup
    spec, st = slab_setup(g)
    blocks = [b.ncell for b in spec.blocks]
    o = mhd_oracle.Oracle(blocks, oracle_consts(spec.params))
    q, B = physics.farfield_state(spec.params)
    X = []
    for ib, b in enumerate(spec.blocks):
        Xb = geometry.ghost_mesh(b.x, b.y, b.z, 4)
        X.append(Xb)
        geo = geometry.build(Xb, b.ncell, 4)
        for name in GEOM[:12] + ["dr_xi", "dr_eta", "dr_zeta"]:
            lo, hi, a = geo[name]
            o.blocks[ib].set_ref(name, lo, a)
        for fname, jd in (("Badd_xi", "JDxi"), ("Badd_eta", "JDet"), ("Badd_zeta", "JDze")):
            lo, hi, a = geo[jd]
            o.blocks[ib].set_ref(fname, lo, solver.badd_faces(a, B))
        for name in ("U_H", "B_xi", "B_eta", "B_zeta"):
            fa = st.fields[name].blocks[ib]
            o.blocks[ib].set_ref(name, fa.lo, fa.data)
    lay = mhd.HostLayout(blocks)
    names = [t[0] for t in lay.table]
    u = [q[1] / q[0], q[2] / q[0], q[3] / q[0]]
    E_inf = [B[1] * u[2] - B[2] * u[1], B[2] * u[0] - B[0] * u[2], B[0] * u[1] - B[1] * u[0]]
    resistive = bool(spec.params.get("is_Lunar_resistance", 0))
    maps = syncmap.compile_tiled(lay, syncmap.TiledLayout(blocks[0], spec.tiles), resistive,
                                 dict(qinf=q, B_imf=B, E_inf=E_inf), X)
    for group, m in maps.items():
        o.add_point_tables(group, names, m["dst"], m["src"], m["cdst"], m["cval"], m["walls"])
    o.sync("Badd")
    if resistive and spec.params.get("use_implicit_lunar_resistance", 0):
        alias, owner, owners = edges.tiled_owners(blocks[0], spec.tiles)
        dofs, eta = edges.resistive_dofs(owners, X, physics.constants(spec.params)["inver_Rem"])
        o.set_resistive(dofs, eta, alias, owner, np.ones(len(alias)))
    elif resistive:
        nodes = [Xb.a[Xb.off:Xb.off + b.ncell[0] + 1, Xb.off:Xb.off + b.ncell[1] + 1, Xb.off:Xb.off + b.ncell[2] + 1]
                 for Xb, b in zip(X, spec.blocks)]
        o.set_explicit_resistive(nodes, physics.constants(spec.params)["inver_Rem"],
                                 spec.params["n_resistive_subcycles"])
    return o


@pytest.fixture(scope="module", params=list(SLAB_CASES))
def oracle_slab(request):
    from conftest import load_golden
    fname, tol = SLAB_CASES[request.param]
    g = load_golden(fname)
    o = build_slab_oracle(g)
    o.sync("Ucell")
    o.sync("Bface")
    o.update_derived()
    o.calc_divb()
    nb = len(o.blocks)
    out = {0: {(f, b): o.blocks[b].get_ref(f) for f in SLAB_FIELDS for b in range(nb)}}
    dts = {}
    nsteps = max(int(k.split("/")[0][1:]) for k in g.files if k[0] == "s" and k[1].isdigit())
    for s in range(1, nsteps + 1):
        dts[s] = o.step()
        o.calc_divb()
        out[s] = {(f, b): o.blocks[b].get_ref(f) for f in SLAB_FIELDS for b in range(nb)}
    return g, out, dts, nsteps, nb, tol, o


def test_oracle_slab_matches_reference(oracle_slab):
    g, out, dts, nsteps, nb, tol, o = oracle_slab
    worst = 0.0
    for s in range(nsteps + 1):
        for f in SLAB_FIELDS:
            if s == 0 and f.startswith(("E", "RHS")):
                continue
            if f.startswith("Eres") and not int(g["resistive"][0]):
                continue
            for b in range(nb):
                ref = g["s%d/b%d/%s" % (s, b, f)]
                got = out[s][(f, b)]
                assert got.shape == ref.shape, (s, b, f)
                if f == "divB":
                    # round-off quantity (~1e-16): compared absolutely
                    assert np.abs(got - ref).max() <= tol, (s, b, f)
                    continue
                e = rel_l2(got, ref)
                worst = max(worst, e)
                assert e <= tol, f"step {s} block {b} field {f}: rel L2 {e:.3e}"
    for s in range(1, nsteps + 1):
        assert abs(dts[s] - float(g["s%d/dt" % s])) <= tol * abs(float(g["s%d/dt" % s]))
    print("oracle slab: max rel L2 %.3e" % worst)
