"""Long-horizon parity and the mixed-precision error report.

A 4-block slab (16 x 8 x 8 cells per block, Solid_Surface and Farfield
walls) is advanced 100 steps by the reference (tests/golden/make_golden.py,
slab_long()) and here, from the same seeded initial state regenerated from
(case, seed).  The fixtures hold the reference's final fields on the inner
points.

* FP64 form: every field within 1e-12 relative L2 of the reference after
  100 steps (1e-9 with the implicit resistive solve, where GMRES stops at
  the solver tolerance, 1e-12 of ||b||, on both sides and the difference in
  orthogonalisation order is carried over 100 steps).
* Mixed form (FP32 face fluxes and contravariant velocities, FP64 CT, curl,
  state update, residuals): every field within 1e-5 relative L2 of the
  reference after 100 steps, and max |div B| * dx / |B| <= 1e-12 with dx the
  cube root of the cell volume, i.e. div B stays at FP64 round-off.
"""
import numpy as np
import pytest

from conftest import load_golden, rel_l2

from beta1_b200 import case, mhd, solver

pytestmark = pytest.mark.gpu

FIELDS = ["U_H", "B_xi", "B_eta", "B_zeta", "PV_H", "B_cell", "J_cell"]
CASES = {"ideal": ("slab_16x8x8_t2x2_r00_long100.npz", 1e-12),
         "implicit_resistive": ("slab_16x8x8_t2x2_r11_long100.npz", 1e-9)}
MIXED_TOL = 1e-5
DIVB_TOL = 1e-12


def long_setup(g):
    over = {k.split("/", 1)[1]: g[k].item() for k in g.files if k.startswith("param/")}
    res = [int(v) for v in g["resistive"]]
    spec = case.slab_case(int(g["nr"]), tuple(int(v) for v in g["nt"]), tuple(int(v) for v in g["tiles"]),
                          is_Lunar_resistance=res[0], use_implicit_lunar_resistance=res[1], **over)
    return spec, case.inflow_state(spec, seed=int(g["seed"]))


def inner(ctx, name, b, a):
    """the inner points of a downloaded field (cells [0, n), faces [0, n])"""
    inf = ctx.field_info(name, b)
    blk = ctx.ncells[b]
    hi = [n + (1 if name == "B_" + ax else 0) for n, ax in zip(blk, ("xi", "eta", "zeta"))]
    return a[tuple(slice(-lo, -lo + h) for lo, h in zip(inf["lo"], hi))]


def run_long(spec, st, precision, steps):
    s = solver.Solver(spec, topology="tiled", precision=precision)
    s.load_state(st)
    t = 0.0
    for _ in range(steps):
        dt, _ = s.step(1)
        t += dt
    s.ctx.stage(mhd.STAGE_DIVB)
    nb = len(spec.blocks)
    out = {(f, b): inner(s.ctx, f, b, s.field(f, b)) for f in FIELDS + ["divB", "Jac"] for b in range(nb)}
    s.ctx.close()
    return out, t


def field_errors(g, out, nb):
    err = {}
    for f in FIELDS:
        got = np.concatenate([out[(f, b)].ravel() for b in range(nb)])
        ref = np.concatenate([g["final/b%d/%s" % (b, f)].ravel() for b in range(nb)])
        err[f] = rel_l2(got, ref)
    return err


def divb_ratio(out, nb):
    worst = 0.0
    for b in range(nb):
        dx = np.cbrt(np.abs(out[("Jac", b)][..., 0]))
        bmag = np.linalg.norm(out[("B_cell", b)], axis=-1)
        worst = max(worst, float(np.max(np.abs(out[("divB", b)][..., 0]) * dx / bmag)))
    return worst


@pytest.fixture(scope="module", params=list(CASES))
def long_runs(request):
    fname, tol = CASES[request.param]
    g = load_golden(fname)
    spec, st = long_setup(g)
    steps = int(g["steps"])
    fp64 = run_long(spec, st, mhd.PREC_FP64, steps)
    mixed = run_long(spec, st, mhd.PREC_MIXED, steps)
    return g, len(spec.blocks), tol, fp64, mixed


def test_fp64_matches_reference_after_100_steps(long_runs):
    g, nb, tol, (out, t), _ = long_runs
    err = field_errors(g, out, nb)
    print("fp64 after %d steps: %s" % (int(g["steps"]), {k: "%.2e" % v for k, v in err.items()}))
    for f, e in err.items():
        assert e <= tol, (f, e)
    assert abs(t - float(g["time"])) <= tol * float(g["time"])


def test_mixed_error_report(long_runs):
    g, nb, tol, _, (out, t) = long_runs
    err = field_errors(g, out, nb)
    r = divb_ratio(out, nb)
    print("mixed after %d steps: %s, max |divB| dx/|B| %.2e" % (int(g["steps"]), {k: "%.2e" % v for k, v in err.items()},
                                                                r))
    for f, e in err.items():
        assert e <= MIXED_TOL, (f, e)
    assert r <= DIVB_TOL
    assert abs(t - float(g["time"])) <= MIXED_TOL * float(g["time"])
