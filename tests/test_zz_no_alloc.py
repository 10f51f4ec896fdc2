"""The allocation-free read-out (mhd_download_field_noalloc).

Some callers of this library cannot allocate device memory when they read
fields out: a driver writing an emergency restart dump after an allocation
has failed, or one that gave all of the GPU's memory to its own pool.  For
them the library has one read-out that stages through a fixed array compiled
into it instead of a buffer allocated on first use.  These tests check,
through the C ABI, that:

* on a fresh context it allocates nothing: read before any other read-out,
  the device's free memory does not change, and the values equal the
  reference's own (the golden fixture);
* it returns the same values as mhd_download_field on consecutive calls
  (the shared array keeps the previous call's contents);
* it refuses a field larger than the array (MHD_EINVAL) and a context whose
  sync tables are not on the device yet (MHD_ESTATE).

Kept in a file of its own that pytest collects last."""
import ctypes as C

import numpy as np
import pytest

from conftest import periodic_setup, rel_l2

from beta1_b200 import case, mhd, solver

pytestmark = pytest.mark.gpu

TOL = 1e-12  # the FP64 tolerance of the parity tests; the values here are copies, so they match exactly
FIELDS = ["U_H", "B_xi", "PV_H", "U_plus", "Eface_eta", "E_zeta", "J_cell", "RHS_H"]


def _raw_noalloc(ctx, name, block=0):
    """the entry point called through the C ABI; returns (status, array)"""
    inf = ctx.field_info(name, block)
    shape = tuple(h - l for l, h in zip(inf["lo"], inf["hi"])) + (inf["ncomp"],)
    out = np.empty(shape, dtype=np.float64)
    rc = ctx.lib.mhd_download_field_noalloc(ctx.h, name.encode(), block, out.ctypes.data, out.size)
    return rc, out


def _free_bytes():
    import torch
    torch.cuda.synchronize()
    return torch.cuda.mem_get_info()[0]


def test_fresh_context_reads_out_without_allocating(golden_periodic):
    """The first read-outs of a fresh context, before any mhd_download_field:
    the device's free memory is unchanged, and the values equal the
    reference's after two steps.  The 20^3 block's geometry is built on the
    device, so the context's own staging buffer (set up by uploads) holds at
    most the 5-component state; the 36-component J_cell weights (7 MB) read
    out here would need a larger one, well above the 2 MiB granularity of
    device allocations, so a fall-back to it would show in the free memory."""
    big = solver.Solver(case.periodic_box_case((20, 20, 20)), geometry_on="device")
    big.load_state(case.initial_state(big.spec, seed=5))
    big.step(1)
    free0 = _free_bytes()
    rc, w = _raw_noalloc(big.ctx, "Jcell_from_Jedge_w")
    assert rc == mhd.MHD_OK
    rc2, u = _raw_noalloc(big.ctx, "U_H")
    assert rc2 == mhd.MHD_OK
    assert _free_bytes() == free0
    assert w.nbytes > 3 * 1024 * 1024
    assert np.array_equal(w, big.field("Jcell_from_Jedge_w")) and np.array_equal(u, big.field("U_H"))
    big.ctx.close()

    g = golden_periodic["steps"]
    spec, st = periodic_setup(g)
    s = solver.Solver(spec)
    s.load_state(st)
    s.step(2)
    for name in ("U_H", "B_xi", "B_eta", "B_zeta", "J_cell"):
        rc, got = _raw_noalloc(s.ctx, name)
        assert rc == mhd.MHD_OK
        assert np.array_equal(got, g["s2/" + name]), name
    s.ctx.close()


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


def test_noalloc_readout_refuses_before_the_sync_tables_are_built(golden_periodic):
    """Before the first step some of the context's sync tables are not on
    the device; building them would allocate, so the read-out refuses with
    MHD_ESTATE, and works after the first step."""
    spec, st = periodic_setup(golden_periodic["steps"])
    s = solver.Solver(spec)
    try:
        rc, _ = _raw_noalloc(s.ctx, "U_H")
        assert mhd.ERRORS.get(rc) == "ESTATE"
        s.load_state(st)
        s.step(1)
        rc, u = _raw_noalloc(s.ctx, "U_H")
        assert rc == mhd.MHD_OK
        assert np.array_equal(u, s.field("U_H"))
    finally:
        s.ctx.close()
