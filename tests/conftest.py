import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def load_golden(name):
    return np.load(os.path.join(GOLDEN, name), allow_pickle=False)


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.linalg.norm(b.ravel())
    num = np.linalg.norm((a - b).ravel())
    return num / den if den > 0 else num


@pytest.fixture(scope="session")
def golden_periodic():
    return {
        "steps": load_golden("periodic_8x6x5_steps.npz"),
        "geom": load_golden("periodic_8x6x5_geom.npz"),
        "probe": load_golden("periodic_8x6x5_probe.npz"),
    }


def slab_setup(g):
    """(case spec, restart state) of a committed slab fixture."""
    from beta1_b200 import case, rst
    LOCS = {"U_H": rst.CELL, "B_xi": rst.FACE_XI, "B_eta": rst.FACE_ET, "B_zeta": rst.FACE_ZE}
    nr = int(g["nr"])
    nt = tuple(int(v) for v in g["nt"])
    tiles = tuple(int(v) for v in g["tiles"])
    res = [int(v) for v in g["resistive"]]
    over = {k.split("/", 1)[1]: g[k].item() for k in g.files if k.startswith("param/")}
    spec = case.slab_case(nr, nt, tiles, is_Lunar_resistance=res[0], use_implicit_lunar_resistance=res[1], **over)
    st = rst.RestartFile(0, 0.0, len(spec.blocks), {})
    for name, loc in LOCS.items():
        rec = rst.FieldRecord(name, loc, 5 if name == "U_H" else 1, 4)
        for b in range(len(spec.blocks)):
            a = g["init/b%d/%s" % (b, name)]
            lo = tuple(int(v) for v in g["init/b%d/%s__lo" % (b, name)])
            rec.blocks.append(rst.FieldArray(lo, tuple(l + s for l, s in zip(lo, a.shape[:3])), a))
        st.fields[name] = rec
    return spec, st


def shell_setup(g):
    """(case spec, restart state) of a committed Pole-shell fixture (with the
    explicit resistive sub-cycles when the fixture's flag says so)."""
    from beta1_b200 import case, rst
    LOCS = {"U_H": rst.CELL, "B_xi": rst.FACE_XI, "B_eta": rst.FACE_ET, "B_zeta": rst.FACE_ZE}
    over = {}
    if "resistive" in g.files and int(g["resistive"][0]):
        over = {k[len("param/"):]: g[k].item() for k in g.files if k.startswith("param/")}
        over.update(is_Lunar_resistance=1, use_implicit_lunar_resistance=0)
    spec = case.shell_case(*(int(v) for v in g["n"]), **over)
    st = rst.RestartFile(0, 0.0, 1, {})
    for name, loc in LOCS.items():
        rec = rst.FieldRecord(name, loc, 5 if name == "U_H" else 1, 4)
        a = g["init/b0/%s" % name]
        lo = tuple(int(v) for v in g["init/b0/%s__lo" % name])
        rec.blocks.append(rst.FieldArray(lo, tuple(l + s for l, s in zip(lo, a.shape[:3])), a))
        st.fields[name] = rec
    return spec, st


def periodic_setup(g):
    """(case spec, restart state) of the committed periodic fixture."""
    from beta1_b200 import case, rst
    n = tuple(int(v) for v in g["n"])
    spec = case.periodic_box_case(n)
    st = rst.RestartFile(0, 0.0, 1, {})
    for name, loc in (("U_H", rst.CELL), ("B_xi", rst.FACE_XI), ("B_eta", rst.FACE_ET), ("B_zeta", rst.FACE_ZE)):
        a = g["init/" + name]
        lo = tuple(int(v) for v in g["init/" + name + "__lo"])
        hi = tuple(l + s for l, s in zip(lo, a.shape[:3]))
        st.fields[name] = rst.FieldRecord(name, loc, a.shape[3], 4, [rst.FieldArray(lo, hi, a)])
    return spec, st



REF_BIN = os.path.join(ROOT, "oracle", "_ref", "ref_lunar")


def reference_run(spec, st, steps, workdir, command="run"):
    """The reference's own StepOnce (oracle/_ref/ref_lunar, built from the
    reference's sources by __graft_entry__.build) on a case written in its
    input formats: returns [RestartFile after the load, after step 1, ...]
    with every state, derived and intermediate field and dt.  command "rk2":
    SSP-RK2 steps of two of the reference's Euler stages each.  Skips the
    calling test when the reference binary is not built."""
    import subprocess

    from beta1_b200 import case, rst
    if not os.path.exists(REF_BIN):
        pytest.skip("oracle/_ref/ref_lunar is not built (make -C oracle)")
    case.write_case(workdir, spec)
    rst.write(os.path.join(workdir, "init.rst"), st)
    subprocess.run([REF_BIN, command, "init.rst", str(steps), "step"], cwd=workdir, check=True,
                   stdout=subprocess.DEVNULL)
    return [rst.read(os.path.join(workdir, "step_%04d.bin" % s)) for s in range(steps + 1)]
