"""The oracle on the Pole shell (one block: Solid_Surface and Farfield in r,
Pole patches at both ends of theta, phi periodic onto itself) against the
reference itself:

* every Sync group, Pole handlers included (the U_H ring average, the B_cell
  and face-B collapses, the axis and regulated edge EMF, the J edge
  regulation), at every point of the index-filled field of the probe fixture;
* the derived fields after the reference's load (with the B_zeta rewrite, the
  J_cell ring repair and the divB zeroing of the Pole layers) and two StepOnce,
  every field bitwise.

This oracle is the checker of the device Pole path."""
import copy
import os
import sys

import numpy as np
import pytest

from conftest import ROOT, load_golden

sys.path.insert(0, os.path.join(ROOT, "oracle"))
import mhd_oracle  # noqa: E402
from test_cpu_oracle import GEOM, oracle_consts  # noqa: E402

SEED = 20261207
SHELL_GEOM = GEOM[:12] + ["dr_xi", "dr_eta", "dr_zeta", "dl_xi", "dl_eta", "dl_zeta", "Astar_xi", "Astar_eta",
                          "Astar_zeta"]


def resistive_shell_params():
    """case parameters of the resistive shell fixture (explicit sub-cycles)"""
    g = load_golden("shell_8x6x8_r10_steps.npz")
    over = {k[len("param/"):]: g[k].item() for k in g.files if k.startswith("param/")}
    return dict(is_Lunar_resistance=1, use_implicit_lunar_resistance=0, **over)


def build_shell_oracle(n=(8, 6, 8), seed=SEED, **over):
    """The oracle after the reference's load_state + UpdateDerivedFields_ on the
    seeded inflow state of the shell (what every fixture of the shell starts
    from); `over`: case parameters (the explicit resistive sub-cycles with
    is_Lunar_resistance)."""
    from beta1_b200 import case, geometry, physics, solver
    spec = case.shell_case(*n, **over)
    b = spec.blocks[0]
    q, B = physics.farfield_state(spec.params)
    Xb = geometry.block_ghost_mesh(b, 4)
    resistive = bool(spec.params.get("is_Lunar_resistance", 0))
    o = mhd_oracle.ShellOracle(b.ncell, oracle_consts(spec.params), Xb, q, B, resistive=resistive)
    if resistive:
        o.set_explicit_resistive([Xb.a[Xb.off:Xb.off + b.ncell[0] + 1, Xb.off:Xb.off + b.ncell[1] + 1,
                                       Xb.off:Xb.off + b.ncell[2] + 1]],
                                 physics.constants(spec.params)["inver_Rem"], spec.params["n_resistive_subcycles"])
    geo = geometry.build(Xb, b.ncell, 4)
    blk = o.blocks[0]
    for name in SHELL_GEOM:
        lo, hi, a = geo[name]
        blk.set_ref(name, lo, a)
    for fname, jd in (("Badd_xi", "JDxi"), ("Badd_eta", "JDet"), ("Badd_zeta", "JDze")):
        lo, hi, a = geo[jd]
        blk.set_ref(fname, lo, solver.badd_faces(a, B))
    st = case.inflow_state(spec, seed=seed)
    for name in ("U_H", "B_xi", "B_eta", "B_zeta"):
        fa = st.fields[name].blocks[0]
        blk.set_ref(name, fa.lo, fa.data)
    o.sync("Badd")
    o.sync("Ucell")
    o.sync("Bface")
    o.update_derived()
    return o


@pytest.fixture(scope="module")
def shell_oracle():
    return build_shell_oracle()


def test_every_shell_sync_equals_reference_probe(shell_oracle):
    from beta1_b200 import syncmap
    probe = load_golden("shell_8x6x8_probe.npz")
    o = shell_oracle
    blk = o.blocks[0]
    saved = copy.deepcopy(blk.f)
    checked = 0
    try:
        for grp, fields in syncmap.GROUPS.items():
            if grp in ("Eres", "Eres1form"):
                continue  # resistive groups: the shell fixtures are ideal
            blk.f = copy.deepcopy(saved)
            for f in fields:
                loc, nc, ng = mhd_oracle.FIELDS[f]
                p = mhd_oracle.PLUS[loc]
                shape = tuple(blk.n[a] + p[a] + 2 * ng for a in range(3)) + (nc,)
                blk.set_ref(f, (-ng, -ng, -ng), (np.arange(np.prod(shape), dtype=np.float64) + 1.0).reshape(shape))
            o.sync(grp)
            for f in fields:
                got = blk.get_ref(f).reshape(-1)
                ref = np.arange(got.size, dtype=np.float64) + 1.0
                dst = probe["%s/%s/0/dst" % (grp, f)]
                ref[dst] = probe["%s/%s/0/val" % (grp, f)]
                bad = np.nonzero(got != ref)[0]
                assert bad.size == 0, (grp, f, bad.size)
                checked += dst.size
    finally:
        blk.f = saved
    assert checked > 100000


@pytest.fixture(scope="module")
def shell_run(shell_oracle):
    o = build_shell_oracle()
    o.calc_divb()
    out = {0: {f: o.blocks[0].get_ref(f) for f in mhd_oracle.FIELDS}}
    dts = {}
    for s in (1, 2):
        dts[s] = o.step()
        o.calc_divb()
        out[s] = {f: o.blocks[0].get_ref(f) for f in mhd_oracle.FIELDS}
    return out, dts


@pytest.mark.parametrize("step", [0, 1, 2])
def test_shell_oracle_steps_bitwise(shell_run, step):
    g = load_golden("shell_8x6x8_steps.npz")
    out, dts = shell_run
    checked = 0
    for key in g.files:
        if not key.startswith("s%d/b0/" % step) or key.endswith("__lo"):
            continue
        f = key.split("/")[-1]
        if step == 0 and f.startswith(("E", "RHS")):
            continue  # not yet computed at load
        assert np.array_equal(out[step][f], g[key]), (step, f)
        checked += 1
    assert checked >= 13
    if step:
        assert dts[step] == float(g["s%d/dt" % step])


def test_shell_oracle_diagnostics_equal_reference_print(shell_run):
    """PrintMinMaxDiagnostics_ after two steps: the oracle's minima / maxima,
    printed as the reference prints them, equal the reference's lines
    (tests/golden/shell_8x6x8_diag.txt)."""
    o = build_shell_oracle()
    for _ in range(2):
        o.step()
    o.calc_divb()
    mins, maxs = o.minmax_diagnostics()
    with open(os.path.join(ROOT, "tests", "golden", "shell_8x6x8_diag.txt")) as f:
        ref = [ln.rstrip() for ln in f if ln.strip()]
    assert o.format_diagnostics(mins, maxs) == ref


def test_resistive_shell_syncs_equal_reference_probe():
    """The Sync groups of the resistive set-up (the Eres groups with their
    Pole handlers: Zero_Rotate of Eres_xi / Eres_zeta, the regulation of
    Eres_eta; the Solid_Surface copies of J_cell and the edge EMF, the Eface
    ghost zeroing) against the reference's probe with is_Lunar_resistance."""
    from beta1_b200 import syncmap
    probe = load_golden("shell_8x6x8_r10_probe.npz")
    o = build_shell_oracle(**resistive_shell_params())
    blk = o.blocks[0]
    saved = copy.deepcopy(blk.f)
    checked = 0
    for grp in ("Eres", "Eres1form", "J_cell", "Eface", "Eedge", "Ucell", "Bface", "Jedge", "B_cell"):
        blk.f = copy.deepcopy(saved)
        fields = syncmap.GROUPS[grp]
        for f in fields:
            loc, nc, ng = mhd_oracle.FIELDS[f]
            p = mhd_oracle.PLUS[loc]
            shape = tuple(blk.n[a] + p[a] + 2 * ng for a in range(3)) + (nc,)
            blk.set_ref(f, (-ng, -ng, -ng), (np.arange(np.prod(shape), dtype=np.float64) + 1.0).reshape(shape))
        o.sync(grp)
        for f in fields:
            got = blk.get_ref(f).reshape(-1)
            ref = np.arange(got.size, dtype=np.float64) + 1.0
            dst = probe["%s/%s/0/dst" % (grp, f)]
            ref[dst] = probe["%s/%s/0/val" % (grp, f)]
            bad = np.nonzero(got != ref)[0]
            assert bad.size == 0, (grp, f, bad.size)
            checked += dst.size
    assert checked > 50000


@pytest.fixture(scope="module")
def resistive_shell_run():
    o = build_shell_oracle(**resistive_shell_params())
    o.calc_divb()
    out = {0: {f: o.blocks[0].get_ref(f) for f in mhd_oracle.FIELDS}}
    dts = {}
    for s in (1, 2):
        dts[s] = o.step()
        o.calc_divb()
        out[s] = {f: o.blocks[0].get_ref(f) for f in mhd_oracle.FIELDS}
    return out, dts


@pytest.mark.parametrize("step", [0, 1, 2])
def test_resistive_shell_oracle_steps_bitwise(resistive_shell_run, step):
    """Two StepOnce with the explicit resistive sub-cycles (two per step) on
    the Pole shell: every field, Eres included, equals the reference's."""
    g = load_golden("shell_8x6x8_r10_steps.npz")
    out, dts = resistive_shell_run
    checked = 0
    for key in g.files:
        if not key.startswith("s%d/b0/" % step) or key.endswith("__lo"):
            continue
        f = key.split("/")[-1]
        if step == 0 and f.startswith(("E", "RHS")):
            continue  # not yet computed at load
        assert np.array_equal(out[step][f], g[key]), (step, f, np.abs(out[step][f] - g[key]).max())
        checked += 1
    assert checked >= 13 if step == 0 else checked >= 26
    if step:
        assert dts[step] == float(g["s%d/dt" % step])
