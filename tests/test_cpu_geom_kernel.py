"""The device geometry builder (beta1_b200/csrc/mhd_geom.cuh, run by the
kernel k_geometry behind mhd_build_geometry), compiled for the host
(tests/geom_host.cpp) and run on the device's padded layout, against the host
geometry (beta1_b200/geometry.py, itself bitwise against the reference's own
geometry): every field bitwise, on a periodic box, a slab block and the Pole
shell with its collapsed cells."""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ROOT

from beta1_b200 import case, geometry, mhd, solver

GROUPS = 6  # GEOM_FACE_VEC .. GEOM_WJ; GEOM_BADD = 6
G = 4


@pytest.fixture(scope="module")
def host_lib(tmp_path_factory):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no host C++ compiler")
    out = str(tmp_path_factory.mktemp("geom") / "libgeom_host.so")
    subprocess.run([cxx, "-std=c++17", "-O2", "-ffp-contract=off", "-shared", "-fPIC",
                    os.path.join(ROOT, "tests", "geom_host.cpp"), "-o", out], check=True)
    lib = C.CDLL(out)
    lib.geom_host.argtypes = [C.c_int] * 4 + [C.c_void_p, C.POINTER(C.c_void_p), C.c_int, C.c_int, C.c_void_p]
    return lib


CASES = {"periodic": lambda: case.periodic_box_case((8, 6, 5)),
         "slab": lambda: case.slab_case(6, (5, 6), (1, 1)),
         "shell": lambda: case.shell_case(8, 6, 8),
         "shell_two_polar_cells": lambda: case.shell_case(6, 2, 4)}


@pytest.mark.parametrize("name", list(CASES))
def test_device_geometry_equals_host_geometry(host_lib, name):
    spec = CASES[name]()
    b = spec.blocks[0]
    n = b.ncell
    X = geometry.block_ghost_mesh(b, G)
    assert X.off == G + 1
    nodes = np.ascontiguousarray(X.a, dtype=np.float64)
    ref = geometry.build(X, n, G)
    table = mhd.field_table()
    vol_shape = (n[0] + 1 + 2 * G, n[1] + 1 + 2 * G, n[2] + 1 + 2 * G)
    fields = [np.zeros((nc,) + vol_shape) for _, _, nc, _ in table]
    ptrs = (C.c_void_p * len(fields))(*[a.ctypes.data for a in fields])
    Bimf = np.array([0.0, 0.3, -0.2])
    for g in range(GROUPS + 1):
        assert host_lib.geom_host(n[0], n[1], n[2], G, nodes.ctypes.data, ptrs, len(fields), g,
                                  Bimf.ctypes.data) == 0
    lay = mhd.HostLayout([n])
    index = {t[0]: i for i, t in enumerate(table)}
    expect = {nm: ref[nm] for nm in solver.GEOM_FIELDS}
    for fname, jd in (("Badd_xi", "JDxi"), ("Badd_eta", "JDet"), ("Badd_zeta", "JDze")):
        lo, hi, a = ref[jd]
        expect[fname] = (lo, hi, solver.badd_faces(a, Bimf))
    for nm, (lo, hi, a) in expect.items():
        info = lay.field_info(nm, 0)
        assert tuple(lo) == tuple(info["lo"]) and tuple(hi) == tuple(info["hi"]), nm
        arr = fields[index[nm]]
        box = arr[:, lo[0] + G:hi[0] + G, lo[1] + G:hi[1] + G, lo[2] + G:hi[2] + G]
        got = np.moveaxis(box, 0, -1)
        same = (got == a) | (np.isnan(got) & np.isnan(a))
        assert same.all(), (name, nm, int((~same).sum()))
