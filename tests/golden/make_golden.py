"""Generates the committed golden fixtures from the reference itself.

Runs the reference Lunar solver, compiled from its own sources against the
single-rank MPI / PETSc-subset shims (oracle/Makefile -> oracle/_ref/ref_lunar),
on small seeded cases written in the reference's own input formats, and
stores its outputs as compressed numpy archives:

* periodic_<n>_geom.npz    every geometry field and the ghost node coordinates
* periodic_<n>_probe.npz   for each Sync group, the point each ghost is copied from
* periodic_<n>_steps.npz   state + derived + intermediate fields after 0..S StepOnce

Needs the reference tree (default /root/reference) and a built oracle; run
    make -C oracle -j8 && python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from beta1_b200 import case, rst  # noqa: E402

REF_BIN = os.path.join(ROOT, "oracle", "_ref", "ref_lunar")
OUT = os.path.dirname(os.path.abspath(__file__))

STEP_FIELDS = ["U_H", "B_xi", "B_eta", "B_zeta", "PV_H", "U_plus", "B_cell", "Bind_cell", "J_xi", "J_eta", "J_zeta",
               "J_cell", "E_xi", "E_eta", "E_zeta", "Eface_xi", "Eface_eta", "Eface_zeta", "RHS_H", "RHS_B_xi",
               "RHS_B_eta", "RHS_B_zeta", "divB"]
GROUPS = ["Ucell", "Bface", "Eface", "Eedge", "B_cell", "Jedge", "J_cell", "Uplus"]


def run(args, cwd):
    subprocess.run([REF_BIN] + args, cwd=cwd, check=True, stdout=subprocess.PIPE)


def flatten(rf: rst.RestartFile, names, block=0):
    out = {}
    for n in names:
        fa = rf.fields[n].blocks[block]
        out[n] = fa.data
        out[n + "__lo"] = np.array(fa.lo, dtype=np.int32)
    return out


def periodic(n=(8, 6, 5), steps=2, seed=20261203):
    tag = "periodic_%dx%dx%d" % n
    with tempfile.TemporaryDirectory() as d:
        spec = case.periodic_box_case(n)
        case.write_case(d, spec)
        st = case.initial_state(spec, seed=seed)
        rst.write(os.path.join(d, "init.rst"), st)
        run(["geom", "geom.bin"], d)
        g = rst.read(os.path.join(d, "geom.bin"))
        np.savez_compressed(os.path.join(OUT, tag + "_geom.npz"), **flatten(g, list(g.fields)))
        probes = {}
        for grp in GROUPS:
            run(["probe", "init.rst", grp, "p.bin"], d)
            p = rst.read(os.path.join(d, "p.bin"))
            for fname, rec in p.fields.items():
                v = rec.blocks[0].data.reshape(-1)
                own = np.arange(v.size, dtype=np.float64) + 1.0
                changed = np.nonzero(v != own)[0]
                probes[grp + "/" + fname + "/dst"] = changed.astype(np.int64)
                probes[grp + "/" + fname + "/src"] = (v[changed] - 1.0).astype(np.int64)
        np.savez_compressed(os.path.join(OUT, tag + "_probe.npz"), **probes)
        run(["run", "init.rst", str(steps), "step"], d)
        arr = {}
        init = flatten(st, ["U_H", "B_xi", "B_eta", "B_zeta"])
        for k, v in init.items():
            arr["init/" + k] = v
        for s in range(steps + 1):
            r = rst.read(os.path.join(d, "step_%04d.bin" % s))
            for k, v in flatten(r, STEP_FIELDS).items():
                arr["s%d/%s" % (s, k)] = v
            arr["s%d/dt" % s] = r.fields["dt"].blocks[0].data.reshape(())
            arr["s%d/time" % s] = np.array(r.time)
        arr["n"] = np.array(n)
        arr["seed"] = np.array(seed)
        np.savez_compressed(os.path.join(OUT, tag + "_steps.npz"), **arr)
    print("wrote", tag)


def periodic_rk2(n=(8, 6, 5), steps=2, seed=20261203):
    """SSP-RK2 steps of the periodic box, each two of the reference's Euler
    stages at one dt and their convex average (harness command rk2)."""
    tag = "periodic_%dx%dx%d_rk2" % n
    with tempfile.TemporaryDirectory() as d:
        spec = case.periodic_box_case(n)
        case.write_case(d, spec)
        st = case.initial_state(spec, seed=seed)
        rst.write(os.path.join(d, "init.rst"), st)
        run(["rk2", "init.rst", str(steps), "step"], d)
        arr = {}
        for k, v in flatten(st, ["U_H", "B_xi", "B_eta", "B_zeta"]).items():
            arr["init/" + k] = v
        for s_ in range(steps + 1):
            r = rst.read(os.path.join(d, "step_%04d.bin" % s_))
            for k, v in flatten(r, STEP_FIELDS).items():
                arr["s%d/%s" % (s_, k)] = v
            arr["s%d/dt" % s_] = r.fields["dt"].blocks[0].data.reshape(())
            arr["s%d/time" % s_] = np.array(r.time)
        arr["n"] = np.array(n)
        arr["seed"] = np.array(seed)
        np.savez_compressed(os.path.join(OUT, tag + ".npz"), **arr)
    print("wrote", tag)


def slab(nr=6, nt=(5, 6), tiles=(2, 2), steps=2, resistive=0, implicit=0, seed=20261204, **over):
    tag = "slab_%dx%dx%d_t%dx%d_r%d%d" % ((nr,) + tuple(nt) + tuple(tiles) + (resistive, implicit))
    with tempfile.TemporaryDirectory() as d:
        spec = case.slab_case(nr, nt, tiles, is_Lunar_resistance=resistive, use_implicit_lunar_resistance=implicit,
                              **over)
        case.write_case(d, spec)
        st = case.inflow_state(spec, seed=seed)
        rst.write(os.path.join(d, "init.rst"), st)
        run(["run", "init.rst", str(steps), "step"], d)
        arr = {}
        for b in range(len(spec.blocks)):
            for k, v in flatten(st, ["U_H", "B_xi", "B_eta", "B_zeta"], b).items():
                arr["init/b%d/%s" % (b, k)] = v
        for s_ in range(steps + 1):
            r = rst.read(os.path.join(d, "step_%04d.bin" % s_))
            for b in range(len(spec.blocks)):
                for k, v in flatten(r, STEP_FIELDS + ["Eres_xi", "Eres_eta", "Eres_zeta"], b).items():
                    arr["s%d/b%d/%s" % (s_, b, k)] = v
            arr["s%d/dt" % s_] = r.fields["dt"].blocks[0].data.reshape(())
        arr["nr"] = np.array(nr)
        arr["nt"] = np.array(nt)
        arr["tiles"] = np.array(tiles)
        arr["resistive"] = np.array([resistive, implicit])
        for k, v in over.items():
            arr["param/" + k] = np.array(v)
        arr["seed"] = np.array(seed)
        np.savez_compressed(os.path.join(OUT, tag + "_steps.npz"), **arr)
    print("wrote", tag)


LONG_FIELDS = ["U_H", "B_xi", "B_eta", "B_zeta", "PV_H", "B_cell", "J_cell", "divB"]


def slab_long(nr=16, nt=(8, 8), tiles=(2, 2), steps=100, resistive=0, implicit=0, seed=20261206, **over):
    """The reference's state after `steps` StepOnce of a slab (only the
    initial and the final state are kept): the FP64 target of the
    long-horizon parity and of the mixed-precision error report."""
    tag = "slab_%dx%dx%d_t%dx%d_r%d%d_long%d" % ((nr,) + tuple(nt) + tuple(tiles) + (resistive, implicit, steps))
    with tempfile.TemporaryDirectory() as d:
        spec = case.slab_case(nr, nt, tiles, is_Lunar_resistance=resistive, use_implicit_lunar_resistance=implicit,
                              **over)
        case.write_case(d, spec)
        st = case.inflow_state(spec, seed=seed)
        rst.write(os.path.join(d, "init.rst"), st)
        run(["run", "init.rst", str(steps), "step"], d)
        # the initial state is regenerated from (case, seed) by the reader;
        # the final fields are kept on the inner points only
        arr = {}
        r = rst.read(os.path.join(d, "step_%04d.bin" % steps))
        for b, blk in enumerate(spec.blocks):
            for name in LONG_FIELDS:
                fa = r.fields[name].blocks[b]
                hi = [n + (1 if name == "B_" + ax else 0) for n, ax in zip(blk.ncell, ("xi", "eta", "zeta"))]
                sl = tuple(slice(-lo, -lo + h) for lo, h in zip(fa.lo, hi))
                arr["final/b%d/%s" % (b, name)] = np.ascontiguousarray(fa.data[sl])
        t = 0.0
        for s_ in range(1, steps + 1):
            t += float(rst.read(os.path.join(d, "step_%04d.bin" % s_)).fields["dt"].blocks[0].data.reshape(()))
        arr["time"] = np.array(t)
        arr["steps"] = np.array(steps)
        arr["nr"] = np.array(nr)
        arr["nt"] = np.array(nt)
        arr["tiles"] = np.array(tiles)
        arr["resistive"] = np.array([resistive, implicit])
        for k, v in over.items():
            arr["param/" + k] = np.array(v)
        arr["seed"] = np.array(seed)
        np.savez_compressed(os.path.join(OUT, tag + ".npz"), **arr)
    print("wrote", tag)


def shell_geom(nr=8, nth=6, nph=8):
    """The reference's geometry of a single-block spherical shell with Pole
    patches at both ends of the polar index (and its ghost node mesh)."""
    tag = "shell_%dx%dx%d" % (nr, nth, nph)
    with tempfile.TemporaryDirectory() as d:
        spec = case.shell_case(nr, nth, nph)
        case.write_case(d, spec)
        run(["geom", "geom.bin"], d)
        g = rst.read(os.path.join(d, "geom.bin"))
        np.savez_compressed(os.path.join(OUT, tag + "_geom.npz"), **flatten(g, list(g.fields)))
    print("wrote", tag)


def shell_tag(nr, nth, nph, resistive):
    """fixture name of a shell; resistive shells (explicit sub-cycles) add _r10"""
    return "shell_%dx%dx%d" % (nr, nth, nph) + ("_r10" if resistive else "")


def shell_steps(nr=8, nth=6, nph=8, steps=2, seed=20261207, resistive=0, **over):
    """The reference's fields after 0..steps StepOnce on the Pole shell (the
    target of a device Pole path; the initial state is regenerated from
    (case, seed) and kept here too).  resistive: the explicit resistive
    sub-cycles (is_Lunar_resistance with use_implicit_lunar_resistance 0)."""
    tag = shell_tag(nr, nth, nph, resistive)
    with tempfile.TemporaryDirectory() as d:
        spec = case.shell_case(nr, nth, nph, is_Lunar_resistance=resistive, use_implicit_lunar_resistance=0, **over)
        case.write_case(d, spec)
        st = case.inflow_state(spec, seed=seed)
        rst.write(os.path.join(d, "init.rst"), st)
        run(["run", "init.rst", str(steps), "step"], d)
        arr = {}
        for k, v in flatten(st, ["U_H", "B_xi", "B_eta", "B_zeta"], 0).items():
            arr["init/b0/%s" % k] = v
        names = STEP_FIELDS + (["Eres_xi", "Eres_eta", "Eres_zeta"] if resistive else [])
        for s_ in range(steps + 1):
            r = rst.read(os.path.join(d, "step_%04d.bin" % s_))
            for k, v in flatten(r, names, 0).items():
                arr["s%d/b0/%s" % (s_, k)] = v
            arr["s%d/dt" % s_] = r.fields["dt"].blocks[0].data.reshape(())
        arr["n"] = np.array([nr, nth, nph])
        arr["seed"] = np.array(seed)
        arr["resistive"] = np.array([resistive, 0])
        for k, v in over.items():
            arr["param/" + k] = np.array(v)
        np.savez_compressed(os.path.join(OUT, tag + "_steps.npz"), **arr)
    print("wrote", tag, "steps")


def shell_diag(nr=8, nth=6, nph=8, seed=20261207, steps=2):
    """The reference's output-step diagnostics (calc_divB, then
    PrintMinMaxDiagnostics_) after `steps` StepOnce on the Pole shell: the
    lines it prints."""
    tag = "shell_%dx%dx%d" % (nr, nth, nph)
    with tempfile.TemporaryDirectory() as d:
        spec = case.shell_case(nr, nth, nph)
        case.write_case(d, spec)
        rst.write(os.path.join(d, "init.rst"), case.inflow_state(spec, seed=seed))
        out = subprocess.run([REF_BIN, "diag", "init.rst", str(steps)], cwd=d, capture_output=True, text=True,
                             check=True).stdout
    lines = [ln.rstrip() for ln in out.splitlines() if ln.strip().startswith(("rho=", "Bx", "Pmag"))]
    with open(os.path.join(OUT, tag + "_diag.txt"), "w") as f:
        f.write("\n".join(lines) + "\n")
    print("wrote", tag + "_diag")


def shell_probe(nr=8, nth=6, nph=8, seed=20261207, resistive=0):
    """Every Sync group of the Pole shell probed on the reference (as
    slab_probe); resistive: the handlers of a resistive set-up."""
    from beta1_b200 import syncmap
    tag = shell_tag(nr, nth, nph, resistive)
    with tempfile.TemporaryDirectory() as d:
        spec = case.shell_case(nr, nth, nph, is_Lunar_resistance=resistive, use_implicit_lunar_resistance=0)
        case.write_case(d, spec)
        rst.write(os.path.join(d, "init.rst"), case.inflow_state(spec, seed=seed))
        arr = {}
        for grp in syncmap.GROUPS:
            run(["probe", "init.rst", grp, "p.bin"], d)
            p = rst.read(os.path.join(d, "p.bin"))
            for fname, rec in p.fields.items():
                v = rec.blocks[0].data.reshape(-1)
                own = np.arange(v.size, dtype=np.float64) + 1.0
                changed = np.nonzero(v != own)[0]
                arr["%s/%s/0/dst" % (grp, fname)] = changed.astype(np.int32)
                arr["%s/%s/0/val" % (grp, fname)] = v[changed]
        np.savez_compressed(os.path.join(OUT, tag + "_probe.npz"), **arr)
    print("wrote", tag + "_probe")


def shell_resistive():
    """The explicit resistive sub-cycles on the Pole shell: the reference's
    steps and Sync probe with the resistive handlers (peak resistivity 1,
    two sub-cycles per step)."""
    eta = 1.0 * case.MU0 * case.ref_scales()["U"] * case.ref_scales()["L_ref"]
    shell_steps(resistive=1, eta_max_lunar=eta, n_resistive_subcycles=2)
    shell_probe(resistive=1)


def hall(spec_kind, seed=20261205):
    """The reference's Hall edge EMF (BuildHallFaceEMF_Rusanov_diff_) of a
    seeded state: a periodic box (no walls) and a slab whose Solid_Surface
    zeroing reaches 20 node layers into the block."""
    if spec_kind == "periodic":
        spec = case.periodic_box_case((8, 6, 5))
        st = case.initial_state(spec, seed=seed)
        tag = "hall_periodic_8x6x5"
    else:
        spec = case.slab_case(24, (5, 6), (2, 2))
        st = case.inflow_state(spec, seed=seed)
        tag = "hall_slab_24x5x6_t2x2"
    with tempfile.TemporaryDirectory() as d:
        case.write_case(d, spec)
        rst.write(os.path.join(d, "init.rst"), st)
        run(["hall", "init.rst", "hall.bin"], d)
        r = rst.read(os.path.join(d, "hall.bin"))
        arr = {}
        for b in range(len(spec.blocks)):
            for name in ("U_H", "B_xi", "B_eta", "B_zeta"):
                fa = st.fields[name].blocks[b]
                arr["init/b%d/%s" % (b, name)] = fa.data
                arr["init/b%d/%s__lo" % (b, name)] = np.array(fa.lo, dtype=np.int32)
            for name in ("Ehall_xi", "Ehall_eta", "Ehall_zeta", "B_cell", "J_cell", "U_H", "B_xi", "B_eta", "B_zeta"):
                fa = r.fields[name].blocks[b]
                arr["b%d/%s" % (b, name)] = fa.data
                arr["b%d/%s__lo" % (b, name)] = np.array(fa.lo, dtype=np.int32)
        arr["kind"] = np.array(spec_kind)
        np.savez_compressed(os.path.join(OUT, tag + ".npz"), **arr)
    print("wrote", tag)


def hallstep(spec_kind, seed=20261205):
    """One implicit Hall solve of the reference (ImplicitHallSolver::SolveOneStep
    at the state's CFL dt, nonlinear tolerance 1e-12) from a seeded state:
    the face B after the solve, the converged Hall EMF and B_cell."""
    if spec_kind == "periodic":
        spec = case.periodic_box_case((8, 6, 5))
        st = case.initial_state(spec, seed=seed)
        tag = "hallstep_periodic_8x6x5"
    else:
        spec = case.slab_case(24, (5, 6), (2, 2))
        st = case.inflow_state(spec, seed=seed)
        tag = "hallstep_slab_24x5x6_t2x2"
    with tempfile.TemporaryDirectory() as d:
        case.write_case(d, spec)
        rst.write(os.path.join(d, "init.rst"), st)
        run(["hallstep", "init.rst", "out.bin"], d)
        r = rst.read(os.path.join(d, "out.bin"))
        arr = {}
        for b in range(len(spec.blocks)):
            for name in ("U_H", "B_xi", "B_eta", "B_zeta"):
                fa = st.fields[name].blocks[b]
                arr["init/b%d/%s" % (b, name)] = fa.data
                arr["init/b%d/%s__lo" % (b, name)] = np.array(fa.lo, dtype=np.int32)
            for name in ("B_xi", "B_eta", "B_zeta", "Ehall_xi", "Ehall_eta", "Ehall_zeta", "B_cell", "RHS_B_xi",
                         "RHS_B_eta", "RHS_B_zeta"):
                fa = r.fields[name].blocks[b]
                arr["b%d/%s" % (b, name)] = fa.data
                arr["b%d/%s__lo" % (b, name)] = np.array(fa.lo, dtype=np.int32)
        arr["dt"] = r.fields["dt"].blocks[0].data.reshape(())
        np.savez_compressed(os.path.join(OUT, tag + ".npz"), **arr)
    print("wrote", tag)


def slab_probe(nr=6, nt=(5, 6), tiles=(2, 2), resistive=0, seed=20261204):
    """Every Sync group of a tiled slab probed on the reference: for each
    (group, field, block) the offsets whose value the Sync changed and the
    value it left there (an encoded source point, a boundary constant, or a
    wall-handler value)."""
    from beta1_b200 import syncmap
    tag = "slab_%dx%dx%d_t%dx%d_r%d%d" % ((nr,) + tuple(nt) + tuple(tiles) + (resistive, resistive))
    with tempfile.TemporaryDirectory() as d:
        spec = case.slab_case(nr, nt, tiles, is_Lunar_resistance=resistive, use_implicit_lunar_resistance=resistive)
        case.write_case(d, spec)
        rst.write(os.path.join(d, "init.rst"), case.inflow_state(spec, seed=seed))
        arr = {}
        for grp in syncmap.GROUPS:
            run(["probe", "init.rst", grp, "p.bin"], d)
            p = rst.read(os.path.join(d, "p.bin"))
            for fname, rec in p.fields.items():
                for b, fa in enumerate(rec.blocks):
                    v = fa.data.reshape(-1)
                    own = np.arange(v.size, dtype=np.float64) + b * 2.0 ** 32 + 1.0
                    changed = np.nonzero(v != own)[0]
                    arr["%s/%s/%d/dst" % (grp, fname, b)] = changed.astype(np.int32)
                    arr["%s/%s/%d/val" % (grp, fname, b)] = v[changed]
        np.savez_compressed(os.path.join(OUT, tag + "_probe.npz"), **arr)
    print("wrote", tag + "_probe")


def slab_owners(nr=6, nt=(5, 6), tiles=(2, 2), seed=20261204, **over):
    """Edge alias/owner table and the implicit resistive unknowns (with eta)
    of a tiled slab, as the reference builds them."""
    tag = "slab_%dx%dx%d_t%dx%d_r11" % ((nr,) + tuple(nt) + tuple(tiles))
    with tempfile.TemporaryDirectory() as d:
        spec = case.slab_case(nr, nt, tiles, is_Lunar_resistance=1, use_implicit_lunar_resistance=1, **over)
        case.write_case(d, spec)
        rst.write(os.path.join(d, "init.rst"), case.inflow_state(spec, seed=seed))
        run(["owners", "owners.txt"], d)
        alias, dof, eta, n_owner = [], [], [], None
        for line in open(os.path.join(d, "owners.txt")):
            t = line.split()
            if t[0] == "alias":
                alias.append([int(x) for x in t[1:6]] + [int(x) for x in t[7:12]] + [int(t[13])])
            elif t[0] == "dof":
                dof.append([int(x) for x in t[1:6]])
                eta.append(float(t[7]))
            elif t[0] == "n_owner":
                n_owner = int(t[1])
        arr = dict(alias=np.array(alias, dtype=np.int32), dof=np.array(dof, dtype=np.int32),
                   eta=np.array(eta), n_owner=np.array(n_owner))
        for k, v in over.items():
            arr["param/" + k] = np.array(v)
        np.savez_compressed(os.path.join(OUT, tag + "_owners.npz"), **arr)
    print("wrote", tag + "_owners")


if __name__ == "__main__":
    if not os.path.exists(REF_BIN):
        sys.exit("build the oracle first: make -C oracle -j8")
    if len(sys.argv) > 1:
        # named generators only, with their default arguments
        for name in sys.argv[1:]:
            globals()[name]()
        sys.exit(0)
    periodic_rk2()
    periodic((8, 6, 5), steps=2)
    slab(steps=2)
    # implicit resistive shell with peak resistivity 1 (inver_Rem = 1), solved to rtol 1e-13
    slab(steps=2, resistive=1, implicit=1, eta_max_lunar=1.0 * case.MU0 * case.ref_scales()["U"]
         * case.ref_scales()["L_ref"], implicit_resistive_ksp_rtol=1e-13, implicit_resistive_ksp_atol=1e-30,
         implicit_resistive_ksp_max_it=300)
    # explicit resistive sub-cycles (two per step) with the same resistivity
    slab(steps=2, resistive=1, implicit=0, eta_max_lunar=1.0 * case.MU0 * case.ref_scales()["U"]
         * case.ref_scales()["L_ref"], n_resistive_subcycles=2)
    # one block periodic onto itself across the transverse directions
    slab(steps=2, tiles=(1, 1))
    shell_geom()
    shell_steps()
    shell_probe()
    shell_diag()
    # the shell with the explicit resistive sub-cycles (two per step) at peak resistivity 1
    shell_resistive()
    slab_probe(resistive=0)
    slab_probe(resistive=1)
    hall("periodic")
    hall("slab")
    hallstep("periodic")
    hallstep("slab")
    slab_long()
    slab_long(resistive=1, implicit=1, eta_max_lunar=0.1 * case.MU0 * case.ref_scales()["U"]
              * case.ref_scales()["L_ref"], implicit_resistive_ksp_rtol=1e-12, implicit_resistive_ksp_atol=1e-30,
              implicit_resistive_ksp_max_it=300)
    slab_owners(eta_max_lunar=1.0 * case.MU0 * case.ref_scales()["U"] * case.ref_scales()["L_ref"])
