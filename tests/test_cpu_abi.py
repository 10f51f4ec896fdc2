"""The C-ABI library loads without a GPU and exports every entry point that
include/beta1_mhd.h declares; its field table and point-id layout agree with
the reference's field registrations."""
import ctypes
import os
import re

import pytest

from conftest import ROOT

from beta1_b200 import mhd

HEADER = os.path.join(ROOT, "include", "beta1_mhd.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(mhd_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(mhd.LIB_PATH):
        pytest.fail("libbeta1_mhd.so is not built (python -c 'import __graft_entry__ as g; g.build()')")
    return mhd.load()


def test_header_declares_the_bound_symbols():
    assert declared_functions() == sorted(mhd.exported_symbols())


def test_library_exports_every_declared_symbol(lib):
    raw = ctypes.CDLL(mhd.LIB_PATH)
    for name in declared_functions():
        assert hasattr(raw, name), name


def test_field_table_matches_registrations(lib):
    table = {t[0]: t[1:] for t in mhd.field_table()}
    # (location, components, ghost layers) of the reference's registrations
    expect = {"U_H": (0, 5, 4), "B_xi": (1, 1, 4), "B_eta": (2, 1, 4), "B_zeta": (3, 1, 4), "PV_H": (0, 5, 4),
              "J_xi": (4, 1, 4), "E_zeta": (6, 1, 4), "Eface_eta": (2, 3, 4), "RHS_H": (0, 5, 0),
              "Jac": (0, 1, 3), "JDxi": (1, 3, 4), "beta_zeta": (3, 1, 3), "alpha_xi": (4, 1, 3),
              "Bcell_from_Bface_w": (0, 18, 3), "Jcell_from_Jedge_w": (0, 36, 3), "Eres_xi": (4, 1, 4)}
    for name, v in expect.items():
        assert table[name] == v, (name, table[name], v)


def test_kernel_names_and_errors_without_gpu(lib):
    assert lib.mhd_kernel_name(0) is not None
    # a null context is rejected, not dereferenced
    assert lib.mhd_sync(None, b"Ucell") == 1
    assert lib.mhd_update_derived(None) == 1


def test_tunable_kernels_match_the_python_defaults(lib):
    # every tunable kernel of the library has a default variant on the Python
    # side, in the library's order, and no more
    names = [lib.mhd_tune_name(i) for i in range(len(mhd.DEFAULT_TUNE) + 1)]
    assert [n.decode() for n in names[:-1]] == list(mhd.DEFAULT_TUNE)
    assert names[-1] is None


def test_host_layout_point_ids(lib):
    lay = mhd.HostLayout([(8, 6, 5), (4, 4, 4)])
    info = lay.field_info("B_eta", 1)
    assert info["lo"] == (-4, -4, -4) and info["hi"] == (8, 9, 8)
    pid = lay.point_base("B_eta", 1)
    assert pid >> 56 == lay.index["B_eta"] and (pid >> 40) & 0xFFFF == 1


def test_host_state_buffers_are_checked_before_the_call():
    """The host-buffer step's wrapper refuses buffers the library would read
    or write past: wrong size, dtype or layout, or a read-only output."""
    import numpy as np
    n = 12
    good = np.zeros(n)
    mhd.check_state_buffers(good, np.zeros(n), n)
    mhd.check_state_buffers(good, good, n)  # in place
    with pytest.raises(ValueError):
        mhd.check_state_buffers(good, np.zeros(n - 1), n)
    with pytest.raises(ValueError):
        mhd.check_state_buffers(np.zeros(n + 1), np.zeros(n + 1), n)
    with pytest.raises(TypeError):
        mhd.check_state_buffers(np.zeros(n, dtype=np.float32), good, n)
    with pytest.raises(TypeError):
        mhd.check_state_buffers(good, np.zeros(2 * n)[::2], n)
    ro = np.zeros(n)
    ro.flags.writeable = False
    with pytest.raises(ValueError):
        mhd.check_state_buffers(good, ro, n)
