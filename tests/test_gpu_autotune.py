"""The autotuner (mhd_autotune): it picks one register / occupancy variant
per hot kernel by timing them on the context's own state.  The variants are
the same code under different launch bounds, so a tuned context must still
reproduce the reference bit for bit: the 4-block slab (ideal MHD) and the
implicit resistive slab against their reference fixtures after tuning."""
import numpy as np
import pytest

from conftest import load_golden, rel_l2, slab_setup

from beta1_b200 import mhd, solver

pytestmark = pytest.mark.gpu

STATE = ["U_H", "B_xi", "B_eta", "B_zeta"]
DERIVED = ["PV_H", "U_plus", "B_cell", "J_cell", "E_xi", "E_eta", "E_zeta", "RHS_H"]


@pytest.mark.parametrize("fname,tol", [("slab_6x5x6_t2x2_r00_steps.npz", 0.0), ("slab_6x5x6_t2x2_r11_steps.npz", 1e-10)])
def test_tuned_context_matches_reference(fname, tol):
    g = load_golden(fname)
    spec, st = slab_setup(g)
    s = solver.Solver(spec, topology="tiled")
    s.load_state(st)
    chosen = s.ctx.autotune(reps=3)
    assert set(chosen) == {"k_pv_uplus_dt", "k_fluid_ucontra", "k_bcell_jedge", "k_eface", "k_curl_e2f", "k_eedge",
                           "k_fluid_mixed", "k_gmres_resist", "k_hall_edge"}
    # minimum CTAs per SM of the chosen variant (0: no launch bounds)
    assert all(v >= 0 for v in chosen.values())
    nb = len(spec.blocks)
    for n in (1, 2):
        s.step(1)
        for b in range(nb):
            for f in STATE + DERIVED:
                ref = g["s%d/b%d/%s" % (n, b, f)]
                got = s.field(f, b)
                if tol == 0.0:
                    assert np.array_equal(got, ref), (n, b, f)
                else:
                    assert rel_l2(got, ref) <= tol, (n, b, f)
    s.ctx.close()


def test_tuned_mixed_equals_default_mixed():
    g = load_golden("slab_6x5x6_t2x2_r00_steps.npz")
    spec, st = slab_setup(g)
    a = solver.Solver(spec, topology="tiled", precision=mhd.PREC_MIXED)
    a.load_state(st)
    a.ctx.autotune(reps=3)
    a.step(3)
    b = solver.Solver(spec, topology="tiled", precision=mhd.PREC_MIXED)
    b.load_state(st)
    b.step(3)
    for blk in range(len(spec.blocks)):
        for f in STATE:
            assert np.array_equal(a.field(f, blk), b.field(f, blk)), (blk, f)
    a.ctx.close()
    b.ctx.close()


def test_tuning_leaves_the_implicit_hall_start_untouched():
    # the implicit Hall solve starts Newton from the edge EMF of the last
    # step; tuning must restore it, so a tuned and an untuned context take
    # bit-identical steps
    g = load_golden("slab_6x5x6_t2x2_r00_steps.npz")
    spec, st = slab_setup(g)
    out = []
    for tune in (True, False):
        s = solver.Solver(spec, topology="tiled")
        s.install_hall_implicit("tiled", rtol=1e-10)
        s.load_state(st)
        s.step(1)
        if tune:
            s.ctx.autotune(reps=2)
        s.step(1)
        out.append({(f, b): s.field(f, b) for f in ("B_xi", "B_eta", "B_zeta", "Ehall_xi") for b in range(4)})
        s.ctx.close()
    for key in out[0]:
        assert np.array_equal(out[0][key], out[1][key]), key


@pytest.mark.parametrize("variant", [12, 16, 0, 2])
def test_flux_variants_give_the_same_bits(variant):
    """The mixed flux pass in each of its variants -- the face-tiled kernel
    (12: every face flux evaluated once per tile, shared through shared
    memory; 16: the same with the tile's face states staged in shared memory
    by asynchronous copies) and the per-cell kernel under other launch
    bounds -- against the
    default per-cell variant, bit for bit, on a batch of uneven shells and a
    slab (tiles cut the blocks at every alignment)."""
    from beta1_b200 import case
    from conftest import shell_setup
    g = load_golden("shell_8x6x8_steps.npz")
    spec0, st0 = shell_setup(g)
    spec1 = case.shell_case(10, 8, 12, mach_u=6.0)
    st1 = case.inflow_state(spec1, seed=77)
    runs = [(spec0, "shell", st0), (spec1, "shell", st1)]
    out = []
    for v in (3, variant):
        bt = solver.Batch([(sp, topo) for sp, topo, _ in runs], precision=mhd.PREC_MIXED)
        bt.ctx.set_tune({"k_fluid_mixed": v})
        bt.load_states([st for _, _, st in runs])
        bt.step(3)
        out.append({(r, f): bt.field(r, f) for r in range(2) for f in STATE + ["RHS_H", "B_cell", "J_cell"]})
        bt.ctx.close()
    for key in out[0]:
        assert np.array_equal(out[0][key], out[1][key]), (variant, key)
    gs = load_golden("slab_6x5x6_t2x2_r00_steps.npz")
    spec, st = slab_setup(gs)
    res = []
    for v in (3, variant):
        s = solver.Solver(spec, topology="tiled", precision=mhd.PREC_MIXED)
        s.ctx.set_tune({"k_fluid_mixed": v})
        s.load_state(st)
        s.step(2)
        res.append({(f, b): s.field(f, b) for f in STATE + ["RHS_H"] for b in range(len(spec.blocks))})
        s.ctx.close()
    for key in res[0]:
        assert np.array_equal(res[0][key], res[1][key]), (variant, key)


@pytest.mark.parametrize("precision", [mhd.PREC_FP64, mhd.PREC_MIXED])
def test_split_derived_pass_gives_the_same_bits(precision):
    """k_pv_uplus_dt variant 14 -- J_cell in a pass of its own before the PV /
    U_plus / CFL pass -- against the fused default (4), bit for bit, on a
    batch of uneven shells (the Pole path, whose J_cell ring repair follows
    the pass) and the tiled slab, in both precisions."""
    from beta1_b200 import case
    from conftest import shell_setup
    g = load_golden("shell_8x6x8_steps.npz")
    spec0, st0 = shell_setup(g)
    spec1 = case.shell_case(10, 8, 12, mach_u=6.0)
    st1 = case.inflow_state(spec1, seed=77)
    runs = [(spec0, "shell", st0), (spec1, "shell", st1)]
    out = []
    for v in (4, 14):
        bt = solver.Batch([(sp, topo) for sp, topo, _ in runs], precision=precision)
        bt.ctx.set_tune({"k_pv_uplus_dt": v})
        bt.load_states([st for _, _, st in runs])
        bt.step(3)
        out.append({(r, f): bt.field(r, f) for r in range(2) for f in STATE + ["U_plus", "B_cell", "J_cell"]})
        out[-1]["dt"] = bt.ctx.get_time()
        bt.ctx.close()
    for key in out[0]:
        assert np.array_equal(np.asarray(out[0][key]), np.asarray(out[1][key])), (precision, key)
    gs = load_golden("slab_6x5x6_t2x2_r00_steps.npz")
    spec, st = slab_setup(gs)
    res = []
    for v in (4, 14):
        s = solver.Solver(spec, topology="tiled", precision=precision)
        s.ctx.set_tune({"k_pv_uplus_dt": v})
        s.load_state(st)
        s.step(2)
        res.append({(f, b): s.field(f, b) for f in STATE + ["J_cell", "PV_H"] for b in range(len(spec.blocks))})
        s.ctx.close()
    for key in res[0]:
        assert np.array_equal(res[0][key], res[1][key]), (precision, key)


def test_set_tune_rejects_unknown_variants(golden_periodic):
    from conftest import periodic_setup
    spec, st = periodic_setup(golden_periodic["steps"])
    s = solver.Solver(spec)
    try:
        with pytest.raises(mhd.MHDError, match="EINVAL"):
            s.ctx.set_tune({"k_fluid_mixed": 7})
    finally:
        s.ctx.close()
