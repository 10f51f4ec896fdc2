"""End-to-end steps through host buffers (mhd_step_host, mhd_step_host_inner).

The state goes up from host AoS arrays (U_H, then B_xi / B_eta / B_zeta of
every block), the device runs the Syncs, the derived fields and the steps,
and the state comes back.  mhd_step_host moves the whole arrays, ghost
layers included; mhd_step_host_inner only the inner points (cells [0, n),
faces [0, n] along their own axis), the ghost points the step reads being
formed on the device by the Syncs.  Both must give the reference's own
steps bit for bit: the periodic box after two steps and the Pole shell
after one (fixtures written by the reference solver).  The host input is the
restart state as the reference loads it, before UpdateDerivedFields_: the
call runs the derived pass first, and on a Pole grid that pass rewrites the
first cell layer's B_zeta, so a state read back after one derived pass is
not the same input.  The inner form is checked from a device whose ghost
layers hold another state, so that a step reading a stale ghost point would
show."""
import numpy as np
import pytest

from conftest import load_golden, periodic_setup, shell_setup

from beta1_b200 import case, solver

pytestmark = pytest.mark.gpu

STATE = ("U_H", "B_xi", "B_eta", "B_zeta")


def inner_of(ctx, name, b, a):
    """the inner points of a field array of block b (cells [0, n), faces [0, n])"""
    inf = ctx.field_info(name, b)
    # the array spans points [lo, hi) with lo = -ghosts and hi = n + ghosts
    # (n + 1 + ghosts along a face's own axis): array index = point - lo, so
    # the inner points [0, hi + lo) sit at indices [-lo, hi)
    lo, hi = inf["lo"], inf["hi"]
    return a[tuple(slice(-l, h) for l, h in zip(lo, hi))]


def host_state(ctx, arrays, inner):
    """the concatenated host state of one block from its restart arrays
    (whole field boxes, ghost layers included)"""
    parts = []
    for name in STATE:
        a = arrays[name]
        assert a.shape == ctx.download(name, 0).shape, name
        if inner:
            a = inner_of(ctx, name, 0, a)
        parts.append(np.ascontiguousarray(a).ravel())
    return np.concatenate(parts)


def split_state(ctx, nblocks, flat, inner):
    """the host state back into per-(block, field) arrays"""
    out, off = {}, 0
    for b in range(nblocks):
        for name in STATE:
            shape = ctx.download(name, b).shape
            if inner:
                shape = inner_of(ctx, name, b, np.empty(shape)).shape
            n = int(np.prod(shape))
            out[(b, name)] = flat[off:off + n].reshape(shape)
            off += n
    assert off == flat.size
    return out


@pytest.mark.parametrize("kind", ["periodic", "shell"])
def test_host_buffer_steps_match_reference(kind):
    if kind == "periodic":
        g = load_golden("periodic_8x6x5_steps.npz")
        spec, st = periodic_setup(g)
        topo, steps, key = "periodic", 2, "%s"
    else:
        g = load_golden("shell_8x6x8_steps.npz")
        spec, st = shell_setup(g)
        topo, steps, key = "shell", 1, "b0/%s"

    def want(name):
        return g[("s%d/" % steps) + key % name]

    init = {name: g["init/" + key % name] for name in STATE}
    nb = len(spec.blocks)
    # whole arrays
    s = solver.Solver(spec, topology=topo)
    try:
        s.load_state(st)
        full_in = host_state(s.ctx, init, inner=False)
        inner_in = host_state(s.ctx, init, inner=True)
        assert full_in.size == s.ctx.state_count() and inner_in.size == s.ctx.state_count_inner()
        out = np.empty_like(full_in)
        s.ctx.step_host(steps, full_in, out)
        got = split_state(s.ctx, nb, out, inner=False)
        for name in STATE:
            assert np.array_equal(got[(0, name)], want(name)), (kind, "full", name)
    finally:
        s.ctx.close()
    # inner points only, on a device that holds another state
    other = case.inflow_state(spec, seed=4242) if kind == "shell" else case.initial_state(spec, seed=4242)
    s = solver.Solver(spec, topology=topo)
    try:
        s.load_state(other)
        out = np.empty_like(inner_in)
        s.ctx.step_host_inner(steps, inner_in, out)
        got = split_state(s.ctx, nb, out, inner=True)
        for name in STATE:
            ref = inner_of(s.ctx, name, 0, want(name))
            assert np.array_equal(got[(0, name)], ref), (kind, "inner", name)
    finally:
        s.ctx.close()
