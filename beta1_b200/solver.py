"""Solver facade: sets a case up on the device the way the reference's
LunarSolver constructor prepares its fields (Z4_Lunar/src/LunarSolver.cpp:12-235),
then steps it with the CUDA library."""
from __future__ import annotations

from typing import Optional

import numpy as np

from . import case as case_mod
from . import edges, geometry, mhd, physics, rst, syncmap

GEOM_FIELDS = ["Jac", "JDxi", "JDet", "JDze", "beta_xi", "beta_eta", "beta_zeta", "alpha_xi", "alpha_eta",
               "alpha_zeta", "dr_xi", "dr_eta", "dr_zeta", "Bcell_from_Bface_w", "Jcell_from_Jedge_w", "Area_xi",
               "Area_eta", "Area_zeta", "dl_xi", "dl_eta", "dl_zeta", "Astar_xi", "Astar_eta", "Astar_zeta"]

_EDGE_PLUS = {0: (0, 1, 1), 1: (1, 0, 1), 2: (1, 1, 0)}


def hall_zero_boxes(ncell, patches):
    """Edge boxes the Hall EMF zeroes (LunarSolver::BuildHallFaceEMF_Rusanov_diff_,
    Z4_Lunar/src/physics/LunarSolver_MagExplicit_Hall.cpp:300-450): the node box
    of every Solid_Surface patch widened 20 node layers inwards, and every Pole
    patch's node box (eta edges for a xi-normal pole, xi edges for an
    eta-normal pole, zeta edges always), as half-open edge boxes clipped to
    the inner edges.  patches: (bc name, direction, node lo, node hi).
    Returns rows (edge axis, lo[3], hi[3])."""
    out = []
    for name, direction, nlo, nhi in patches:
        ax = abs(direction) - 1
        for ea in range(3):
            if name == "Pole":
                if not ((abs(direction) == 1 and ea == 1) or (abs(direction) == 2 and ea == 0) or ea == 2):
                    continue
            elif name != "Solid_Surface":
                continue
            lo, hi = list(nlo), list(nhi)
            if name == "Solid_Surface":
                if direction < 0:
                    hi[ax] += 20
                else:
                    lo[ax] -= 20
            hi[ea] -= 1
            plus = _EDGE_PLUS[ea]
            lo = [max(lo[a], 0) for a in range(3)]
            hi = [min(hi[a], ncell[a] + plus[a]) for a in range(3)]
            if all(lo[a] < hi[a] for a in range(3)):
                out.append([ea] + lo + hi)
    return out
STATE_FIELDS = ["U_H", "B_xi", "B_eta", "B_zeta"]


def pole_directions(block) -> list:
    """Directions of a block's eta Pole patches: -2 for the node plane j = 0,
    +2 for j = n_j (the patch's node range is one plane in j)."""
    out = []
    for (ist, ied, jst, jed, kst, ked), name in block.physical:
        if name != "Pole":
            continue
        if jst != jed or jst not in (0, block.ncell[1]):
            raise ValueError("only Pole patches on a j face (eta Poles) are supported")
        out.append(-2 if jst == 0 else 2)
    return out


def topology_patches(topology, ncell, block=None):
    """(bc name, direction, node lo, node hi) of the physical patches the Hall
    EMF zeroes next to: the Solid_Surface face i = 0 of the tiled slab and the
    shell, and the shell's Poles."""
    n = ncell
    if topology not in ("tiled", "shell"):
        return []
    out = [("Solid_Surface", -1, (0, 0, 0), (1, n[1] + 1, n[2] + 1))]
    if topology == "shell":
        for d in pole_directions(block):
            j = 0 if d < 0 else n[1]
            out.append(("Pole", d, (0, j, 0), (n[0] + 1, j + 1, n[2] + 1)))
    return out


def make_params(p, precision=mhd.PREC_FP64) -> mhd.Params:
    c = physics.constants(p)
    return mhd.Params(gamma=c["gamma"], cfl=c["cfl"], inver_MA2=c["inver_MA2"],
                      momentum_hall_coeff=c["momentum_hall_coeff"], state_coeff=c["state_coeff"], M_H=c["M_H"],
                      M_ref=c["M_ref"], ne_hall_floor=c["ne_hall_floor"], dt_abort=1e-7, ngg=int(p["ngg"]),
                      precision=int(precision))


def badd_faces(JD: np.ndarray, B0) -> np.ndarray:
    """Applied field flux of the IMF on every face (DipoleField::Build_Badd_FaceFlux
    without dipoles, Z4_Lunar/include/operators/Dipole.h:89-375): B0 . JD."""
    return ((B0[0] * JD[..., 0] + B0[1] * JD[..., 1]) + B0[2] * JD[..., 2])[..., None]


# host-side set-up of a case (geometry, node arrays, compiled sync tables),
# kept for solvers of the same case (e.g. the FP64 and the mixed-precision
# form side by side)
_HOST_CACHE: dict = {}


class Solver:
    def __init__(self, spec: case_mod.CaseSpec, topology: str = "periodic", precision=mhd.PREC_FP64,
                 geometry_on: str = "host"):
        """geometry_on: "host" builds the geometry fields with beta1_b200.geometry
        and uploads them; "device" sends only the ghost node meshes and builds
        them with mhd_build_geometry (the same values)."""
        if geometry_on not in ("host", "device"):
            raise ValueError(f"unknown geometry builder {geometry_on}")
        self.spec = spec
        ngg = int(spec.params["ngg"])
        self.ctx = mhd.Context([b.ncell for b in spec.blocks], make_params(spec.params, precision))
        cache = _HOST_CACHE.get(id(spec))
        if cache is None or cache["spec"] is not spec:
            cache = {"spec": spec, "geom": [None] * len(spec.blocks), "nodes": []}
            for b in spec.blocks:
                cache["nodes"].append(geometry.block_ghost_mesh(b, ngg))
            _HOST_CACHE.clear()
            _HOST_CACHE[id(spec)] = cache
        if geometry_on == "host":
            for ib, b in enumerate(spec.blocks):
                if cache["geom"][ib] is None:
                    cache["geom"][ib] = geometry.build(cache["nodes"][ib], b.ncell, ngg)
        self._cache = cache
        if precision == mhd.PREC_MIXED:
            q0, _ = physics.farfield_state(spec.params)
            u0 = [q0[1] / q0[0], q0[2] / q0[0], q0[3] / q0[0]]
            p0 = (physics.constants(spec.params)["gamma"] - 1.0) * (
                q0[4] - 0.5 * q0[0] * (u0[0] ** 2 + u0[1] ** 2 + u0[2] ** 2))
            self.ctx.set_flux_reference([q0[0]] + u0 + [p0])
        self.geom = []
        self.nodes = []
        _, B_imf = physics.farfield_state(spec.params)
        for ib, b in enumerate(spec.blocks):
            X = cache["nodes"][ib]
            g = cache["geom"][ib] if geometry_on == "host" else None
            if g is None:
                self.ctx.build_geometry(ib, X.a, B_imf)
            else:
                for name in GEOM_FIELDS:
                    lo, hi, a = g[name]
                    self.ctx.upload(name, ib, a)
                if any(v != 0.0 for v in B_imf):
                    for fname, jd in (("Badd_xi", "JDxi"), ("Badd_eta", "JDet"), ("Badd_zeta", "JDze")):
                        self.ctx.upload(fname, ib, badd_faces(g[jd][2], B_imf))
            self.geom.append(g)
            self.nodes.append(X)
        if topology == "periodic":
            if len(spec.blocks) != 1:
                raise ValueError("a periodic box has one block")
            self.sync_sizes = syncmap.install_periodic(self.ctx, spec.blocks[0].ncell)
        elif topology == "tiled":
            self.install_tiled()
        elif topology == "shell":
            self.install_shell()
        else:
            raise ValueError(f"unknown topology {topology}")
        self.ctx.sync("Badd")
        self.install_hall(topology)
        p = spec.params
        if float(p.get("arti_eta_max", 0.0)) > 0.0:
            raise NotImplementedError("the artificial-resistivity edge EMF is not supported by this build")
        if p.get("is_Lunar_resistance", 0):
            if p.get("use_implicit_lunar_resistance", 0):
                self.install_resistive(topology)
            else:
                self.install_explicit_resistive()

    def _edge_ids(self, rows, names):
        """point ids of edge rows (block, axis 1..3, i, j, k) in the fields
        names[axis]; one field lookup per (field, block), vectorised over rows"""
        rows = np.asarray(rows, dtype=np.int64).reshape(-1, 5)
        out = np.empty(len(rows), dtype=np.int64)
        for d in np.unique(rows[:, 1]).tolist():
            for b in np.unique(rows[rows[:, 1] == d, 0]).tolist():
                sel = (rows[:, 1] == d) & (rows[:, 0] == b)
                info = self.ctx.field_info(names[d], b)
                r = rows[sel]
                out[sel] = self.ctx.point_base(names[d], b) + syncmap.aos_index(info["lo"], info["hi"], 1, r[:, 2],
                                                                                  r[:, 3], r[:, 4], 0)
        return out

    def install_resistive(self, topology):
        """Unknowns, resistivity and edge aliases of the implicit resistive
        solve (LunarSolver::SetupImplicitResistiveDiffusion_)."""
        spec = self.spec
        n = spec.blocks[0].ncell
        tiles = spec.tiles if topology == "tiled" else (1, 1)
        alias, owner, owners = edges.tiled_owners(n, tiles)
        c = physics.constants(spec.params)
        dofs, eta = edges.resistive_dofs(owners, self.nodes, c["inver_Rem"])
        names = {1: "Eres_xi", 2: "Eres_eta", 3: "Eres_zeta"}

        def ids(rows):
            return self._edge_ids(rows, names)

        p = spec.params
        self.ctx.set_resistive(ids(dofs), eta, ids(alias), ids(owner), np.ones(len(alias)),
                               float(p["implicit_resistive_ksp_rtol"]), float(p["implicit_resistive_ksp_atol"]),
                               int(p["implicit_resistive_ksp_max_it"]), 30)
        self.resistive_dofs = (dofs, eta)

    def install_hall(self, topology):
        """Hall coefficient and the Hall EMF's zeroed edge boxes: the tiled
        slab has a Solid_Surface patch on the i-minimum face of every block,
        the periodic box has no physical patch."""
        rows = []
        for ib, b in enumerate(self.spec.blocks):
            rows += [[ib] + r for r in hall_zero_boxes(b.ncell, topology_patches(topology, b.ncell, b))]
        self.ctx.set_hall(physics.constants(self.spec.params)["hall_coef"], rows)

    def install_hall_implicit(self, topology, rtol=1e-8, atol=1e-50, maxit=50, ksp_rtol=1e-5, ksp_maxit=10000):
        """Owner edges and aliases of the implicit Hall unknowns
        (ImplicitHallSolver: owner_edges_sorted_ and the edge 1-form table)."""
        n = self.spec.blocks[0].ncell
        tiles = self.spec.tiles if topology == "tiled" else (1, 1)
        alias, owner, owners = edges.tiled_owners(n, tiles, periodic_i=(topology == "periodic"))
        names = {1: "Ehall_xi", 2: "Ehall_eta", 3: "Ehall_zeta"}

        def ids(rows):
            return self._edge_ids(rows, names)

        self.ctx.set_hall_implicit(ids(owners), ids(alias), ids(owner), np.ones(len(alias)), rtol, atol, maxit,
                                   ksp_rtol, ksp_maxit)

    def install_explicit_resistive(self):
        """Shell profile of every inner edge and the sub-cycle count of
        LunarSolver::ResistiveDiffusionSubcycles_."""
        spec = self.spec
        for ib, b in enumerate(spec.blocks):
            for name, y in zip(("eta_edge_xi", "eta_edge_eta", "eta_edge_zeta"),
                               edges.shell_profile(self.nodes[ib], b.ncell)):
                self.ctx.upload(name, ib, y[..., None])
        c = physics.constants(spec.params)
        self.ctx.set_resistive_explicit(c["inver_Rem"], max(1, int(spec.params["n_resistive_subcycles"])))

    def install_tiled(self):
        spec = self.spec
        q, B = physics.farfield_state(spec.params)
        u = [q[1] / q[0], q[2] / q[0], q[3] / q[0]]
        E_inf = [B[1] * u[2] - B[2] * u[1], B[2] * u[0] - B[0] * u[2], B[0] * u[1] - B[1] * u[0]]
        resistive = bool(spec.params.get("is_Lunar_resistance", 0))
        key = ("maps", resistive)
        if key not in self._cache:
            self._cache[key] = syncmap.compile_tiled(self.ctx, syncmap.TiledLayout(spec.blocks[0].ncell, spec.tiles),
                                                     resistive, dict(qinf=q, B_imf=B, E_inf=E_inf), self.nodes)
        maps = self._cache[key]
        self.sync_sizes = {}
        for group, m in maps.items():
            self.ctx.set_sync_map(group, m["dst"], m["src"])
            self.ctx.set_sync_consts(group, m["cdst"], m["cval"])
            for (b, d) in m["walls"]:
                self.ctx.set_sync_wall(group, b, d)
            self.sync_sizes[group] = (int(m["dst"].size), int(m["cdst"].size), len(m["walls"]))

    def install_shell(self):
        """The single-block spherical shell: Solid_Surface and Farfield in i,
        eta Poles at both ends of j, k periodic onto itself (ideal MHD, or
        the explicit resistive sub-cycles)."""
        spec = self.spec
        if len(spec.blocks) != 1:
            raise ValueError("a shell has one block")
        p = spec.params
        if p.get("is_Lunar_resistance", 0) and p.get("use_implicit_lunar_resistance", 0):
            raise NotImplementedError("the implicit resistive solve is not built for a shell")
        key = ("shell_maps", bool(p.get("is_Lunar_resistance", 0)))
        if key not in self._cache:
            self._cache[key] = shell_tables(spec, self.nodes[0], self.ctx)
        self.sync_sizes = install_maps(self.ctx, self._cache[key])
        for d in pole_directions(spec.blocks[0]):
            self.ctx.set_pole(0, d)

    def load_state(self, state: rst.RestartFile):
        """Restart load + the syncs that make ghosts consistent, then
        UpdateDerivedFields_ (the state the first StepOnce starts from)."""
        for name in STATE_FIELDS:
            rec = state.fields[name]
            for ib, fa in enumerate(rec.blocks):
                self.ctx.upload(name, ib, fa.data)
        self.ctx.sync("Ucell")
        self.ctx.sync("Bface")
        self.ctx.update_derived()

    def step(self, n=1):
        return self.ctx.step(n)

    def field(self, name, block=0) -> np.ndarray:
        return self.ctx.download(name, block)


def farfield_consts(params):
    """q_inf, B_imf and the zero-curl far-field EMF E_inf = -u_inf x B_imf"""
    q, B = physics.farfield_state(params)
    u = [q[1] / q[0], q[2] / q[0], q[3] / q[0]]
    E_inf = [B[1] * u[2] - B[2] * u[1], B[2] * u[0] - B[0] * u[2], B[0] * u[1] - B[1] * u[0]]
    return dict(qinf=q, B_imf=B, E_inf=E_inf)


def shell_tables(spec: case_mod.CaseSpec, nodes, layout=None):
    """Sync tables of a single-block shell (syncmap.compile_shell), with the
    resistive handlers when the case sets is_Lunar_resistance."""
    b = spec.blocks[0]
    lay = layout if layout is not None else mhd.HostLayout([b.ncell])
    return syncmap.compile_shell(lay, b.ncell, bool(spec.params.get("is_Lunar_resistance", 0)),
                                 farfield_consts(spec.params), nodes)


def install_maps(ctx, maps):
    """Gives a context its compiled sync tables; returns the sizes per group."""
    sizes = {}
    for group, m in maps.items():
        ctx.set_sync_map(group, m["dst"], m["src"])
        if m.get("dst2") is not None and m["dst2"].size:
            ctx.set_sync_map_post(group, m["dst2"], m["src2"])
        if m["cdst"].size:
            ctx.set_sync_consts(group, m["cdst"], m["cval"])
        for (b, d) in m["walls"]:
            ctx.set_sync_wall(group, b, d)
        sizes[group] = (int(m["dst"].size), int(m["cdst"].size), len(m["walls"]))
    return sizes


def host_setup(spec: case_mod.CaseSpec, topology: Optional[str] = None, geometry_on: str = "host"):
    """Host-side set-up of a case: per block the ghost node mesh and (unless
    the device builds it) the geometry fields, and (given the topology) the
    run's sync tables compiled on its own blocks 0, 1, ...  A pure function
    of the case, safe to run in worker processes.  Returns (nodes, geom, tables
    or None); geom holds None per block when geometry_on is "device"."""
    ngg = int(spec.params["ngg"])
    nodes, geom = [], []
    for b in spec.blocks:
        X = geometry.block_ghost_mesh(b, ngg)
        nodes.append(X)
        geom.append(geometry.build(X, b.ncell, ngg) if geometry_on == "host" else None)
    return nodes, geom, (run_tables(spec, topology, nodes) if topology else None)


def host_setup_run(run):
    """host_setup of a (spec, topology[, geometry_on]) tuple (process-pool entry)"""
    return host_setup(*run)


def run_tables(spec: case_mod.CaseSpec, topology: str, nodes):
    """Sync tables of one non-resistive run on its own blocks 0, 1, ..."""
    lay = mhd.HostLayout([b.ncell for b in spec.blocks])
    if topology == "periodic":
        return syncmap.periodic_maps(lay, spec.blocks[0].ncell)
    if topology == "shell":
        return shell_tables(spec, nodes[0], lay)
    if topology != "tiled":
        raise ValueError(f"unknown topology {topology}")
    q, B = physics.farfield_state(spec.params)
    u = [q[1] / q[0], q[2] / q[0], q[3] / q[0]]
    E_inf = [B[1] * u[2] - B[2] * u[1], B[2] * u[0] - B[0] * u[2], B[0] * u[1] - B[1] * u[0]]
    return syncmap.compile_tiled(lay, syncmap.TiledLayout(spec.blocks[0].ncell, spec.tiles), False,
                                 dict(qinf=q, B_imf=B, E_inf=E_inf), nodes)


def _farfield_prim(params):
    q0, _ = physics.farfield_state(params)
    u0 = [q0[1] / q0[0], q0[2] / q0[0], q0[3] / q0[0]]
    p0 = (physics.constants(params)["gamma"] - 1.0) * (q0[4] - 0.5 * q0[0] * (u0[0] ** 2 + u0[1] ** 2 + u0[2] ** 2))
    return [q0[0]] + u0 + [p0]


class Batch:
    """Independent runs in one context (mhd_batch_create): a parameter sweep
    whose runs differ in grid size, inflow and IMF, each with its own time
    step, all advanced by one step graph.  runs: (case spec, topology) per
    run, topology "periodic" (one block), "tiled" or "shell" (one block with
    Poles; a batch with shells holds shells only); the runs must agree on
    the constants of the step (gamma, CFL, the J x B and state scales) and
    may not use the resistive or Hall solves.  host: optional iterable of
    the host_setup(spec, topology) results of the runs in order (e.g. from a
    process pool); each is uploaded and released as it arrives.  A run whose
    host set-up holds no geometry (host_setup(..., geometry_on="device")) has
    it built on the device from its node mesh."""

    CONSTS = ("gamma", "cfl", "inver_MA2", "momentum_hall_coeff", "state_coeff", "M_H", "M_ref", "ne_hall_floor")

    def __init__(self, runs, precision=mhd.PREC_FP64, host=None, geometry_on: str = "host"):
        self.runs = [(spec, topo) for spec, topo in runs]
        c0 = physics.constants(self.runs[0][0].params)
        for spec, topo in self.runs:
            c = physics.constants(spec.params)
            bad = [k for k in self.CONSTS if c[k] != c0[k]]
            if bad:
                raise ValueError(f"runs of a batch must share the step constants; differing: {bad}")
            if spec.params.get("is_Lunar_resistance", 0):
                raise ValueError("resistive runs cannot be batched")
            if topo in ("periodic", "shell") and len(spec.blocks) != 1:
                raise ValueError(f"a {topo} run has one block")
        shells = [topo == "shell" for _, topo in self.runs]
        if any(shells) and not all(shells):
            # a context with Poles runs every sync in the shell's order
            raise ValueError("a batch with shells holds shells only")
        ncells, run_of, self.offset = [], [], []
        for r, (spec, _) in enumerate(self.runs):
            self.offset.append(len(ncells))
            ncells += [b.ncell for b in spec.blocks]
            run_of += [r] * len(spec.blocks)
        self.ctx = mhd.Context(ncells, make_params(self.runs[0][0].params, precision), runs=run_of)
        if host is None:
            host = (host_setup(spec, topo, geometry_on) for spec, topo in self.runs)
        per_run = []
        zero_rows = []
        poles = []
        for r, ((spec, topo), (nodes, geom, maps)) in enumerate(zip(self.runs, host)):
            off = self.offset[r]
            q, B = physics.farfield_state(spec.params)
            for ib, g in enumerate(geom):
                if g is None:
                    self.ctx.build_geometry(off + ib, nodes[ib].a, B)
                    continue
                for name in GEOM_FIELDS:
                    self.ctx.upload(name, off + ib, g[name][2])
                if any(v != 0.0 for v in B):
                    for fname, jd in (("Badd_xi", "JDxi"), ("Badd_eta", "JDet"), ("Badd_zeta", "JDze")):
                        self.ctx.upload(fname, off + ib, badd_faces(g[jd][2], B))
            if maps is None:
                maps = run_tables(spec, topo, nodes)
            per_run.append((maps, off))
            del nodes, geom
            for ib, b in enumerate(spec.blocks):
                zero_rows += [[off + ib] + row for row in hall_zero_boxes(b.ncell, topology_patches(topo, b.ncell, b))]
                if topo == "shell":
                    for d in pole_directions(b):
                        poles.append((off + ib, d))
            if precision == mhd.PREC_MIXED:
                self.ctx.set_flux_reference(_farfield_prim(spec.params), run=r)
        self.sync_sizes = install_maps(self.ctx, syncmap.merge_runs(per_run))
        for b, d in poles:
            self.ctx.set_pole(b, d)
        self.ctx.sync("Badd")
        self.ctx.set_hall(c0["hall_coef"], zero_rows)

    @property
    def cells(self):
        return [sum(b.ncell[0] * b.ncell[1] * b.ncell[2] for b in spec.blocks) for spec, _ in self.runs]

    def load_states(self, states):
        """Restart state of every run, then the syncs and UpdateDerivedFields_."""
        for r, st in enumerate(states):
            for name in STATE_FIELDS:
                for ib, fa in enumerate(st.fields[name].blocks):
                    self.ctx.upload(name, self.offset[r] + ib, fa.data)
        self.ctx.sync("Ucell")
        self.ctx.sync("Bface")
        self.ctx.update_derived()

    def step(self, n=1):
        return self.ctx.step(n)

    def field(self, run, name, block=0) -> np.ndarray:
        return self.ctx.download(name, self.offset[run] + block)

