"""The device's Pole work items (beta1_b200/csrc/mhd_pole.cuh, run by the
kernel k_pole), compiled for the host (tests/pole_host.cpp) and run on the
oracle's arrays -- which have the device's padded structure-of-arrays layout
-- against the oracle's restatement of each Pole handler and repair, bitwise,
on a shell in mid-run."""
import copy
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ROOT
from test_cpu_oracle_shell import build_shell_oracle, mhd_oracle

from beta1_b200 import mhd

OPS = ["POLE_RING_U", "POLE_RING_BXI", "POLE_BCELL", "POLE_EXI_AXIS", "POLE_EETA_REG", "POLE_JETA", "POLE_BZETA",
       "POLE_JCELL", "POLE_DIVB", "POLE_ERES_REG"]
OP = {name: i for i, name in enumerate(OPS)}
# fields each operation writes: overwritten with noise first, so that the
# operation has to produce them (the mid-run state already holds its results)
OUTPUTS = {"POLE_RING_U": ["U_H"], "POLE_RING_BXI": ["B_xi"], "POLE_BCELL": ["B_cell", "Bind_cell"],
           "POLE_EXI_AXIS": ["E_xi"], "POLE_EETA_REG": ["E_eta"], "POLE_JETA": ["J_eta"], "POLE_BZETA": ["B_zeta"],
           "POLE_JCELL": ["J_cell"], "POLE_DIVB": ["divB"], "POLE_ERES_REG": ["Eres_eta"]}


@pytest.fixture(scope="module")
def host_lib(tmp_path_factory):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no host C++ compiler")
    out = str(tmp_path_factory.mktemp("pole") / "libpole_host.so")
    subprocess.run([cxx, "-std=c++17", "-O2", "-ffp-contract=off", "-shared", "-fPIC",
                    os.path.join(ROOT, "tests", "pole_host.cpp"), "-o", out], check=True)
    lib = C.CDLL(out)
    lib.pole_host.argtypes = [C.c_int] * 6 + [C.POINTER(C.c_void_p), C.c_int]
    return lib


@pytest.fixture(scope="module", params=[(8, 6, 8), (6, 2, 4)], ids=["8x6x8", "6x2x4"])
def mid_run(request):
    o = build_shell_oracle(request.param, seed=31)
    o.step()
    return o


def run_host(lib, o, op, sides=(-1, 1)):
    """op on the oracle's own arrays (fields the oracle does not keep get zero planes)"""
    names = [t[0] for t in mhd.field_table()]
    assert lib.pole_nfields() == len(names)
    blk = o.blocks[0]
    spare = []
    ptrs = (C.c_void_p * len(names))()
    for f, name in enumerate(names):
        a = blk.f.get(name)
        if a is None:
            a = np.zeros((mhd_oracle_ncomp(name),) + blk.f["U_H"].shape[1:])
            spare.append(a)
        assert a.flags.c_contiguous and a.dtype == np.float64
        ptrs[f] = a.ctypes.data
    for side in sides:
        assert lib.pole_host(OP[op], side, blk.n[0], blk.n[1], blk.n[2], blk.G, ptrs, len(names)) == 0


def mhd_oracle_ncomp(name):
    return {t[0]: t[2] for t in mhd.field_table()}[name]


def oracle_op(o, op):
    S = o.POLES
    if op == "POLE_RING_U":
        for s in S:
            o._pole_cell(s)
    elif op == "POLE_RING_BXI":
        for s in S:
            o._pole_ring_average("B_xi", s)
    elif op == "POLE_BCELL":
        for s in S:
            o._pole_bcell("B_cell", s)
            o._pole_bcell("Bind_cell", s)
    elif op == "POLE_EXI_AXIS":
        for s in S:
            o._pole_eedge_axis(s)
    elif op == "POLE_EETA_REG":
        for s in S:
            o._pole_eedge_regulate(s, ghosts=False)
    elif op == "POLE_ERES_REG":
        for s in S:
            o._pole_eedge_regulate(s, ghosts=False, name="Eres_eta")
    elif op == "POLE_JETA":
        for s in S:
            o._pole_jedge_regulate(s, ghosts=False)
    elif op == "POLE_BZETA":
        o.bzeta_pole_rewrite()
    elif op == "POLE_JCELL":
        o.jcell_pole_repair()
    elif op == "POLE_DIVB":
        o.calc_divb()


@pytest.mark.parametrize("op", OPS)
def test_pole_work_items_equal_oracle(host_lib, mid_run, op):
    start = copy.deepcopy(mid_run)
    rng = np.random.default_rng(OP[op])
    for name in OUTPUTS[op]:
        arr = start.blocks[0].f[name]
        arr += 0.25 * (np.abs(arr).max() + 1.0) * rng.standard_normal(arr.shape)
    a = copy.deepcopy(start)
    b = copy.deepcopy(start)
    oracle_op(a, op)
    if op == "POLE_DIVB":
        mhd_oracle.Oracle.calc_divb(b)  # divB without the Pole zeroing, then the work items
    run_host(host_lib, b, op)
    changed = 0
    for name, arr in a.blocks[0].f.items():
        other = b.blocks[0].f[name]
        assert np.array_equal(arr, other), (op, name, int(np.count_nonzero(arr != other)))
        changed += int(np.count_nonzero(arr != start.blocks[0].f[name]))
    assert changed > 0, op


def test_diag_keys_order_and_round_trip(host_lib):
    """diag_key orders doubles as their values (-0 just below +0) and
    diag_unkey inverts it bit for bit."""
    rng = np.random.default_rng(5)
    x = np.concatenate([rng.standard_normal(2000) * 10.0 ** rng.integers(-300, 300, 2000),
                        [0.0, -0.0, np.inf, -np.inf, 5e-324, -5e-324, 1.7976931348623157e308]])
    k = np.zeros(x.size, dtype=np.uint64)
    back = np.zeros(x.size)
    host_lib.diag_keys.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
    host_lib.diag_keys(x.ctypes.data, k.ctypes.data, back.ctypes.data, x.size)
    assert np.array_equal(back.view(np.uint64), x.view(np.uint64))
    order = np.argsort(k, kind="stable")
    xs = x[order]
    assert np.all(xs[:-1] <= xs[1:])


def test_diag_reduction_equals_oracle(host_lib, mid_run):
    """k_diag's per-cell values and key reduction (host build) against the
    oracle's PrintMinMaxDiagnostics_ restatement, on the shell in mid-run."""
    o = copy.deepcopy(mid_run)
    o.calc_divb()
    names = [t[0] for t in mhd.field_table()]
    blk = o.blocks[0]
    spare = []
    ptrs = (C.c_void_p * len(names))()
    for f, name in enumerate(names):
        a = blk.f.get(name)
        if a is None:
            a = np.zeros((mhd_oracle_ncomp(name),) + blk.f["U_H"].shape[1:])
            spare.append(a)
        ptrs[f] = a.ctypes.data
    mins = (C.c_double * 6)()
    maxs = (C.c_double * 7)()
    host_lib.diag_host.argtypes = [C.c_int] * 4 + [C.POINTER(C.c_void_p), C.c_int, C.c_void_p, C.c_void_p]
    assert host_lib.diag_host(blk.n[0], blk.n[1], blk.n[2], blk.G, ptrs, len(names), mins, maxs) == 0
    rmins, rmaxs = o.minmax_diagnostics()
    assert list(mins) == rmins and list(maxs) == rmaxs
