"""The allocation-free read-out (mhd_download_field_noalloc).

Some callers of this library cannot allocate device memory when they read
fields out: a driver writing an emergency restart dump after an allocation
has failed, or one that gave all of the GPU's memory to its own pool.  For
them the library has one read-out that stages through a fixed array compiled
into it instead of a buffer allocated on first use.  These tests check,
through the C ABI, that it returns the same values as mhd_download_field on
consecutive calls (the shared array keeps the previous call's contents), and
that it refuses a field larger than the array.

Kept in a file of its own that pytest collects last."""
import ctypes as C

import numpy as np
import pytest

from conftest import periodic_setup, rel_l2

from beta1_b200 import case, mhd, solver

pytestmark = pytest.mark.gpu

TOL = 1e-12  # the FP64 tolerance of the parity tests; the values here are copies, so they match exactly
FIELDS = ["U_H", "B_xi", "PV_H", "U_plus", "Eface_eta", "E_zeta", "J_cell", "RHS_H"]


@pytest.fixture(scope="module")
def stepped(golden_periodic):
    spec, st = periodic_setup(golden_periodic["steps"])
    s = solver.Solver(spec)
    s.load_state(st)
    s.step(2)
    yield s
    s.ctx.close()


def test_noalloc_readout_matches_download_on_consecutive_calls(stepped):
    ctx = stepped.ctx
    for name in FIELDS:
        want = ctx.download(name)
        first = ctx.download_noalloc(name)
        second = ctx.download_noalloc(name)
        assert first.shape == want.shape
        assert rel_l2(first, want) <= TOL, name
        assert rel_l2(second, want) <= TOL, name
        assert np.array_equal(first, want) and np.array_equal(second, want), name


def test_noalloc_readout_after_further_steps(stepped):
    ctx = stepped.ctx
    stepped.step(1)
    a = ctx.download_noalloc("U_H")
    b = ctx.download_noalloc("B_eta")
    assert rel_l2(a, ctx.download("U_H")) <= TOL
    assert rel_l2(b, ctx.download("B_eta")) <= TOL


def test_noalloc_readout_rejects_fields_beyond_its_array():
    # a 64^3 block: its 36-component J-cell weights exceed the staging array
    ctx = mhd.Context([(64, 64, 64)], solver.make_params(case.periodic_box_case((8, 8, 8)).params))
    try:
        inf = ctx.field_info("Jcell_from_Jedge_w", 0)
        n = int(np.prod([h - l for l, h in zip(inf["lo"], inf["hi"])])) * inf["ncomp"]
        assert n > mhd.NOALLOC_MAX_DOUBLES
        out = np.empty(n)
        rc = ctx.lib.mhd_download_field_noalloc(ctx.h, b"Jcell_from_Jedge_w", 0, out.ctypes.data, n)
        assert mhd.ERRORS.get(rc) == "EINVAL"
        buf = C.create_string_buffer(512)
        ctx.lib.mhd_last_error(ctx.h, buf, 512)
        assert b"at most" in buf.value
    finally:
        ctx.close()
