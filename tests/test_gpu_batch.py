"""Batches of independent runs (mhd_batch_create) against the reference.

Three runs of different sizes and layouts advance in one context: the
periodic 8 x 6 x 5 box, the 4-block slab (Solid_Surface and Farfield walls,
2 x 2 transverse tiles) and the single-block slab periodic onto itself.  The
blocks are uneven, so every hot-path stage runs as one flattened launch
holding exactly the CTAs of every block, and each run keeps its own time
step.  Every run must reproduce its own reference outputs (the fixtures of
the single-run parity tests) to the FP64 bound of 1e-12 relative L2 per
field per step, with its conserved state and dt bit for bit; the
mixed-precision batch must equal the mixed-precision runs advanced alone.
"""
import numpy as np
import pytest

from conftest import load_golden, periodic_setup, rel_l2, slab_setup

from beta1_b200 import mhd, solver

pytestmark = pytest.mark.gpu

TOL = 1e-12
FIELDS = ["U_H", "B_xi", "B_eta", "B_zeta", "PV_H", "U_plus", "B_cell", "Bind_cell", "J_xi", "J_eta", "J_zeta",
          "J_cell", "E_xi", "E_eta", "E_zeta", "Eface_xi", "Eface_eta", "Eface_zeta", "RHS_H", "RHS_B_xi",
          "RHS_B_eta", "RHS_B_zeta", "divB"]
STATE = ["U_H", "B_xi", "B_eta", "B_zeta"]


def ref_key(kind, s, b, f):
    return "s%d/%s" % (s, f) if kind == "periodic" else "s%d/b%d/%s" % (s, b, f)


@pytest.fixture(scope="module")
def cases():
    out = []
    g = load_golden("periodic_8x6x5_steps.npz")
    spec, st = periodic_setup(g)
    out.append(("periodic", g, spec, "periodic", st))
    for name in ("slab_6x5x6_t2x2_r00_steps.npz", "slab_6x5x6_t1x1_r00_steps.npz"):
        g = load_golden(name)
        spec, st = slab_setup(g)
        out.append(("slab", g, spec, "tiled", st))
    return out


def snapshot(bt, r, nb):
    return {(f, b): bt.field(r, f, b) for f in FIELDS for b in range(nb)}


@pytest.fixture(scope="module")
def batch_run(cases):
    bt = solver.Batch([(c[2], c[3]) for c in cases])
    bt.load_states([c[4] for c in cases])
    bt.ctx.stage(mhd.STAGE_DIVB)
    nbs = [len(c[2].blocks) for c in cases]
    out = {0: [snapshot(bt, r, nb) for r, nb in enumerate(nbs)]}
    dts = {}
    nsteps = 2
    for n in range(1, nsteps + 1):
        bt.step(1)
        bt.ctx.stage(mhd.STAGE_DIVB)
        out[n] = [snapshot(bt, r, nb) for r, nb in enumerate(nbs)]
        dts[n] = [bt.ctx.run_time(r) for r in range(len(cases))]
    flat = bt.ctx.nruns
    bt.ctx.close()
    return out, dts, nsteps, nbs, flat


def test_batch_runs_match_reference(cases, batch_run):
    out, dts, nsteps, nbs, nruns = batch_run
    assert nruns == 3
    worst = 0.0
    for r, (kind, g, spec, topo, st) in enumerate(cases):
        for n in range(nsteps + 1):
            for f in FIELDS:
                if n == 0 and f.startswith(("E", "RHS")):
                    continue
                for b in range(nbs[r]):
                    ref = g[ref_key(kind, n, b, f)]
                    got = out[n][r][(f, b)]
                    assert got.shape == ref.shape, (r, n, b, f)
                    if f == "divB":
                        assert np.abs(got - ref).max() <= TOL, (r, n, b, f)
                        continue
                    if f in STATE and n > 0:
                        assert np.array_equal(got, ref), (r, n, b, f)
                    e = rel_l2(got, ref)
                    worst = max(worst, e)
                    assert e <= TOL, f"run {r} step {n} block {b} field {f}: rel L2 {e:.3e}"
    print("batch of %d runs: max rel L2 %.3e" % (len(cases), worst))


def test_batch_dt_per_run(cases, batch_run):
    out, dts, nsteps, nbs, _ = batch_run
    t = [0.0] * len(cases)
    for n in range(1, nsteps + 1):
        for r, (kind, g, spec, topo, st) in enumerate(cases):
            dt, time, steps = dts[n][r]
            assert dt == float(g["s%d/dt" % n]), (r, n, dt)
            t[r] += dt
            assert steps == n and time == t[r]
    # the runs do have different time steps
    assert len({dts[1][r][0] for r in range(len(cases))}) > 1


def test_batch_step_reports_every_run(cases):
    bt = solver.Batch([(c[2], c[3]) for c in cases])
    bt.load_states([c[4] for c in cases])
    dts, times = bt.ctx.batch_step(2)
    for r, (kind, g, spec, topo, st) in enumerate(cases):
        assert dts[r] == float(g["s2/dt"]), (r, dts[r])
        assert times[r] == float(g["s1/dt"]) + float(g["s2/dt"]), (r, times[r])
        assert bt.ctx.run_time(r)[:2] == (dts[r], times[r])
    bt.ctx.close()


def test_mixed_batch_equals_runs_alone(cases):
    bt = solver.Batch([(c[2], c[3]) for c in cases], precision=mhd.PREC_MIXED)
    bt.load_states([c[4] for c in cases])
    bt.step(3)
    for r, (kind, g, spec, topo, st) in enumerate(cases):
        s = solver.Solver(spec, topology=topo, precision=mhd.PREC_MIXED)
        s.load_state(st)
        s.step(3)
        for b in range(len(spec.blocks)):
            for f in STATE + ["B_cell", "J_cell"]:
                assert np.array_equal(bt.field(r, f, b), s.field(f, b)), (r, b, f)
        assert bt.ctx.run_time(r) == s.ctx.run_time(0)
        s.ctx.close()
    bt.ctx.close()
