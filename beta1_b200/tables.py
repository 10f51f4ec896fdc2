"""The device set-up a C++ driver cannot derive from the reference alone, in
one binary file: the compiled Sync tables of every group (beta1_b200.syncmap),
the Pole patches, and the implicit resistive system (unknowns, resistivity,
edge aliases).  The C++ drop-in of LunarSolver's driver
(beta1_b200/dropin/LunarSolver_Driver_B200.cpp) reads it at its first
StepOnce; geometry and state it takes from the reference's own FieldBlocks.

Point ids are the library's (field index << 56 | block << 40 | AoS offset),
so the file fits a context with the same blocks.  compile_case() takes the
CaseSpec (beta1_b200.case) the CASE directory was written from.

Layout (little-endian): b"B1TB", int32 version 1, int32 ngroups, then per
group: int32 name length, name, and five arrays (int64 count, then values):
dst, src (int64), dst2, src2 (int64, copies after the wall handlers),
cdst (int64) and cval (float64) as one count, then int32 nwalls and
(int32 block, int32 direction) pairs; int32 npoles and (block, direction)
pairs; int32 has_resistive, and if 1: int64 n, unknowns int64[n], eta
f64[n], int64 na, alias int64[na], owner int64[na], sign f64[na], f64 rtol,
f64 atol, int32 maxit, int32 restart.
"""
from __future__ import annotations

import struct

import numpy as np

from . import edges, mhd, physics, solver, syncmap


def compile_case(spec, topology: str) -> dict:
    """Sync tables, Poles and resistive system of a case, compiled on the
    host (no GPU)."""
    from . import geometry
    ngg = int(spec.params["ngg"])
    nodes = [geometry.block_ghost_mesh(b, ngg) for b in spec.blocks]
    lay = mhd.HostLayout([b.ncell for b in spec.blocks])
    resistive = bool(spec.params.get("is_Lunar_resistance", 0))
    implicit = resistive and bool(spec.params.get("use_implicit_lunar_resistance", 0))
    # the explicit resistive sub-cycles need only the resistive sync groups:
    # the driver forms their edge profile from its own node coordinates
    if topology == "tiled":
        consts = solver.farfield_consts(spec.params)
        groups = syncmap.compile_tiled(lay, syncmap.TiledLayout(spec.blocks[0].ncell, spec.tiles), resistive, consts,
                                       nodes)
    elif implicit:
        raise NotImplementedError("the implicit resistive solve is exported for the tiled layout only")
    elif resistive and topology != "shell":
        raise NotImplementedError("the resistive handlers are compiled for the tiled layout and the shell")
    else:
        groups = solver.run_tables(spec, topology, nodes)
    poles = []
    if topology == "shell":
        poles = [(0, d) for d in solver.pole_directions(spec.blocks[0])]
    res = None
    if implicit:
        n = spec.blocks[0].ncell
        tiles = spec.tiles
        alias, owner, owners = edges.tiled_owners(n, tiles)
        c = physics.constants(spec.params)
        dofs, eta = edges.resistive_dofs(owners, nodes, c["inver_Rem"])
        names = {1: "Eres_xi", 2: "Eres_eta", 3: "Eres_zeta"}

        def ids(rows):
            rows = np.asarray(rows, dtype=np.int64).reshape(-1, 5)
            out = np.empty(len(rows), dtype=np.int64)
            for r, (b, d, i, j, k) in enumerate(rows.tolist()):
                inf = lay.field_info(names[d], b)
                out[r] = lay.point_base(names[d], b) + syncmap.aos_index(inf["lo"], inf["hi"], 1, i, j, k, 0)
            return out

        p = spec.params
        res = dict(unknowns=ids(dofs), eta=np.asarray(eta, dtype=np.float64), alias=ids(alias), owner=ids(owner),
                   sign=np.ones(len(alias)), rtol=float(p["implicit_resistive_ksp_rtol"]),
                   atol=float(p["implicit_resistive_ksp_atol"]), maxit=int(p["implicit_resistive_ksp_max_it"]),
                   restart=30)
    return dict(groups=groups, poles=poles, resistive=res)


def _arr(f, a, dtype):
    a = np.ascontiguousarray(np.asarray(a, dtype=dtype).ravel())
    f.write(struct.pack("<q", a.size))
    f.write(a.astype("<" + np.dtype(dtype).str[1:]).tobytes())


def write(path: str, compiled: dict) -> None:
    with open(path, "wb") as f:
        f.write(b"B1TB")
        f.write(struct.pack("<ii", 1, len(compiled["groups"])))
        for name, m in compiled["groups"].items():
            nb = name.encode()
            f.write(struct.pack("<i", len(nb)))
            f.write(nb)
            _arr(f, m["dst"], np.int64)
            _arr(f, m["src"], np.int64)
            d2 = m.get("dst2")
            _arr(f, d2 if d2 is not None else [], np.int64)
            _arr(f, m.get("src2") if d2 is not None else [], np.int64)
            _arr(f, m["cdst"], np.int64)
            cv = np.ascontiguousarray(np.asarray(m["cval"], dtype=np.float64).ravel())
            f.write(cv.tobytes())
            f.write(struct.pack("<i", len(m["walls"])))
            for b, d in m["walls"]:
                f.write(struct.pack("<ii", int(b), int(d)))
        f.write(struct.pack("<i", len(compiled["poles"])))
        for b, d in compiled["poles"]:
            f.write(struct.pack("<ii", int(b), int(d)))
        r = compiled["resistive"]
        f.write(struct.pack("<i", 1 if r else 0))
        if r:
            _arr(f, r["unknowns"], np.int64)
            f.write(np.ascontiguousarray(r["eta"], dtype=np.float64).tobytes())
            _arr(f, r["alias"], np.int64)
            f.write(np.ascontiguousarray(r["owner"], dtype=np.int64).tobytes())
            f.write(np.ascontiguousarray(r["sign"], dtype=np.float64).tobytes())
            f.write(struct.pack("<ddii", r["rtol"], r["atol"], r["maxit"], r["restart"]))


def read(path: str) -> dict:
    """The inverse of write() (the C++ reader's twin, for tests)."""
    with open(path, "rb") as f:
        buf = f.read()
    pos = [0]

    def take(fmt):
        v = struct.unpack_from(fmt, buf, pos[0])
        pos[0] += struct.calcsize(fmt)
        return v

    def arr(dtype, n=None):
        if n is None:
            n = take("<q")[0]
        a = np.frombuffer(buf, dtype=dtype, count=n, offset=pos[0]).copy()
        pos[0] += n * np.dtype(dtype).itemsize
        return a

    if buf[:4] != b"B1TB":
        raise ValueError("not a set-up file (no B1TB tag)")
    pos[0] = 4
    ver, ng = take("<ii")
    if ver != 1:
        raise ValueError(f"set-up file version {ver}, expected 1")
    groups = {}
    for _ in range(ng):
        (ln,) = take("<i")
        name = buf[pos[0]:pos[0] + ln].decode()
        pos[0] += ln
        m = dict(dst=arr("<i8"), src=arr("<i8"), dst2=arr("<i8"), src2=arr("<i8"))
        m["cdst"] = arr("<i8")
        m["cval"] = arr("<f8", m["cdst"].size)
        (nw,) = take("<i")
        m["walls"] = [take("<ii") for _ in range(nw)]
        groups[name] = m
    (npol,) = take("<i")
    poles = [take("<ii") for _ in range(npol)]
    (hr,) = take("<i")
    res = None
    if hr:
        u = arr("<i8")
        eta = arr("<f8", u.size)
        al = arr("<i8")
        ow = arr("<i8", al.size)
        sg = arr("<f8", al.size)
        rtol, atol, maxit, restart = take("<ddii")
        res = dict(unknowns=u, eta=eta, alias=al, owner=ow, sign=sg, rtol=rtol, atol=atol, maxit=maxit,
                   restart=restart)
    return dict(groups=groups, poles=poles, resistive=res)
