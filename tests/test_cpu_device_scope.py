"""Device binding of the C ABI's entry points, checked on the host.

A context lives on the device that was current at its creation; every entry
point makes that device current for the call and restores the caller's
device afterwards (beta1_b200/csrc/mhd_device_scope.h).  The same header is
compiled here against a fake device API (tests/device_scope_host.cpp) and
each scenario's sequence of device calls is checked."""
import ctypes as C
import os
import shutil
import subprocess

import pytest

from conftest import ROOT

GET = 1000


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no host C++ compiler")
    out = str(tmp_path_factory.mktemp("scope") / "libscope.so")
    subprocess.run([cxx, "-std=c++17", "-O2", "-shared", "-fPIC", os.path.join(ROOT, "tests", "device_scope_host.cpp"),
                    "-o", out], check=True)
    lib = C.CDLL(out)
    lib.scope_trace.argtypes = [C.c_int] * 5 + [C.POINTER(C.c_int)] * 3
    return lib


def trace(lib, current, want, nested=0, fail_set=-1, fail_get=0):
    log = (C.c_int * 16)()
    n = C.c_int()
    during = C.c_int()
    r = lib.scope_trace(current, want, nested, fail_set, fail_get, log, C.byref(n), C.byref(during))
    return r // 10, r % 10, list(log[:n.value]), during.value


def test_other_device_is_bound_and_restored(lib):
    ok, after, log, during = trace(lib, current=0, want=3)
    assert ok and during == 3 and after == 0
    assert log == [GET, 3, 0]


def test_same_device_makes_no_set_call(lib):
    ok, after, log, during = trace(lib, current=2, want=2)
    assert ok and during == 2 and after == 2 and log == [GET]


def test_nested_entry_points_restore_once(lib):
    ok, after, log, during = trace(lib, current=1, want=4, nested=1)
    assert ok and during == 4 and after == 1
    assert log == [GET, 4, GET, 1]


def test_null_context_touches_nothing(lib):
    ok, after, log, during = trace(lib, current=5, want=-1)
    assert ok and after == 5 and log == []


def test_failed_bind_reports_and_changes_nothing(lib):
    ok, after, log, during = trace(lib, current=0, want=6, fail_set=6)
    assert not ok and after == 0 and during == 0 and log == [GET, 6]
    ok, after, log, during = trace(lib, current=0, want=6, fail_get=1)
    assert not ok and after == 0 and log == [GET]
