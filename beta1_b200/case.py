"""Case writer: grids, boundary files, parameter files and initial states in
the reference's on-disk formats, so that the reference driver and this
library read identical inputs.

Formats written (all under ``<dir>/CASE``):

* ``setup/filenames`` and the four parameter files, in the key/value + LIST
  syntax parsed by src/0_basic/1_MPCNS_Parameter.cpp:4-66 (the shipped
  Z4_Lunar/9999setup/* files are the template).
* ``geometry/grid   0.grd``: binary grid, Read_Method 2
  (src/1_grid/1_MPCNS_Grid.cpp:125-230): int32 nblock, per block an int32
  byte count plus NUL-terminated name, per block int32 imax/jmax/kmax (node
  counts), then per block x, y, z as float64 with i fastest.
* ``geometry/boundary_condition/boundary   0.txt``: per block the number of
  physical faces, then "ist ied jst jed kst ked bctype" with 0-based node
  indices (src/1_grid/1_MPCNS_Grid.cpp:232-296).
* ``geometry/boundary_condition/boundary_name.fvbnd``: header line, name of
  type 0, further names from type 2 on, terminated by BOUNDARIES
  (src/1_grid/1_MPCNS_Grid.cpp:298-334).
* ``geometry/boundary_condition/inner   0.txt``: total count, per-block
  counts, a comment line, then one line per interface with 1-based node
  ranges whose signs encode the in-plane axis pairing, the signed 1-based
  block number (negative = periodic) and block name for both sides
  (src/1_grid/1_MPCNS_Grid.cpp:413-520, include/1_grid/Grid_Boundary.h:236-330).
* ``geometry/boundary_condition/parallel   0.txt``: no inter-rank faces.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple

import numpy as np

from . import rst

# Physical constants of the shipped Lunar setup (Z4_Lunar/9999setup/0_General_Setting.txt:23-28)
GAMMA = 1.6667
NA = 6.02e23
R_UNI = 8.314
MU0 = 1.256637061e-6
Q_E = 1.602e-19

BC_NAMES = ["Solid_Surface", "Farfield", "Pole", "Outflow"]  # types 2, 3, 4, 5


@dataclass
class BlockGrid:
    name: str
    x: np.ndarray  # (imax, jmax, kmax) node coordinates
    y: np.ndarray
    z: np.ndarray
    physical: List[Tuple[Tuple[int, int, int, int, int, int], str]] = field(default_factory=list)

    @property
    def ncell(self):
        return tuple(s - 1 for s in self.x.shape)


@dataclass
class InnerFace:
    """One side of a block interface in the inner-file convention: 1-based
    node ranges (ist, ied, jst, jed, kst, ked) whose signs/order encode the
    axis pairing, plus the 1-based block number (negative for periodic)."""
    this_range: Tuple[int, int, int, int, int, int]
    this_block: int
    tar_range: Tuple[int, int, int, int, int, int]
    tar_block: int


@dataclass
class CaseSpec:
    blocks: List[BlockGrid]
    inner: List[List[InnerFace]]  # per block
    params: Dict[str, object]


def ref_scales(U=4.61e5, n=7.0e6, M=0.001, T=1.2e5, L=1.7374e6):
    """Reference scales chosen so that inver_MA2 = momentum_hall_coeff = 1
    (Z4_Lunar/src/physics/LunarSolver_Tools.cpp:37-39): B_ref = U*sqrt(mu0*rho_ref)."""
    rho_ref = M * n / NA
    B = U * math.sqrt(MU0 * rho_ref)
    return dict(U=U, T=T, n=n, Molecular_mass=M, B_ref=B, L_ref=L)


def default_params(**over):
    p = dict(
        CFL=0.4, max_Time=0.0, max_Nstep=100000000, output_step=0, output_residual=0,
        Archive_Output_Time=0.0, continue_calc=0, dimension=3, ngg=4, Read_Method=2,
        corner_treat=2, scale=1.0, mole_mass1=0.001, eta_max_lunar=1.25e7,
        REF=ref_scales(),
        INITIAL=None,  # dict(U, T, n, Molecular_mass, c_y, c_z, Bx, By, Bz)
        num_of_dipole=0, is_Lunar_resistance=0, use_implicit_lunar_resistance=0,
        n_resistive_subcycles=1, implicit_resistive_ksp_rtol=1e-10,
        implicit_resistive_ksp_atol=1e-30, implicit_resistive_ksp_max_it=200,
        arti_eta_max=0.0, J_range_start=800.0, J_range_on=3000.0,
    )
    p.update(over)
    if p["INITIAL"] is None:
        r = p["REF"]
        p["INITIAL"] = dict(U=r["U"], T=r["T"], n=r["n"], Molecular_mass=r["Molecular_mass"],
                            c_y=0.0, c_z=0.0, Bx=0.0, By=0.0, Bz=0.0)
    return p


def _num(v) -> str:
    if isinstance(v, bool):
        return "1" if v else "0"
    if isinstance(v, int):
        return str(v)
    return repr(float(v))


def write_setup(case_dir: str, p: Dict[str, object]) -> None:
    d = os.path.join(case_dir, "CASE", "setup")
    os.makedirs(d, exist_ok=True)
    with open(os.path.join(d, "filenames"), "w") as f:
        f.write("0_General_Setting.txt\n1_Initial_condition.txt\n2_Boundary_Condition.txt\n3_MHD_Control.txt\n###END###\n")
    g = []
    g.append(f"double  CFL                     {_num(p['CFL'])}")
    g.append(f"double  max_Time                {_num(p['max_Time'])}")
    g.append(f"int     max_Nstep               {_num(p['max_Nstep'])}")
    g.append(f"int     output_step             {_num(p['output_step'])}")
    g.append(f"int     output_residual         {_num(p['output_residual'])}")
    g.append(f"double  Archive_Output_Time     {_num(p['Archive_Output_Time'])}")
    g.append(f"bool    continue_calc           {_num(p['continue_calc'])}")
    g.append(f"int     dimension               {_num(p['dimension'])}")
    g.append(f"int     ngg                     {_num(p['ngg'])}")
    g.append(f"int     Read_Method             {_num(p['Read_Method'])}")
    g.append(f"int     corner_treat            {_num(p['corner_treat'])}")
    g.append(f"double  scale                   {_num(p['scale'])}")
    g.append(f"double  mole_mass1              {_num(p['mole_mass1'])}")
    if p.get("solver") == "mercury":
        g.append(f"double  mole_mass2              {_num(p['mole_mass2'])}")
        g.append(f"double  eta_max_mercury         {_num(p['eta_max_mercury'])}")
    else:
        g.append(f"double  eta_max_lunar           {_num(p['eta_max_lunar'])}")
    g.append("")
    g.append("LIST==================================================================")
    g.append("constant        5")
    g.append("(double)")
    g.append("gamma           NA              R_uni       mu_mag             q_e")
    g.append(f"{_num(GAMMA)} {_num(NA)} {_num(R_UNI)} {_num(MU0)} {_num(Q_E)}")
    g.append("LIST==================================================================")
    g.append("")
    g.append("END_OF_FILE")
    with open(os.path.join(d, "0_General_Setting.txt"), "w") as f:
        f.write("\n".join(g) + "\n")
    r = p["REF"]
    ini = p["INITIAL"]
    s = []
    s.append("LIST==================================================================")
    s.append("REF             6")
    s.append("(double)")
    s.append("U               T               n           Molecular_mass  B_ref   L_ref")
    s.append(" ".join(_num(r[k]) for k in ["U", "T", "n", "Molecular_mass", "B_ref", "L_ref"]))
    s.append("LIST==================================================================")
    s.append("")
    s.append("LIST==================================================================")
    s.append("INITIAL         9")
    s.append("(double)")
    s.append("U               T               n           Molecular_mass  c_y     c_z     Bx      By      Bz")
    s.append(" ".join(_num(ini[k]) for k in ["U", "T", "n", "Molecular_mass", "c_y", "c_z", "Bx", "By", "Bz"]))
    s.append("LIST==================================================================")
    s.append("")
    s.append("END_OF_FILE")
    with open(os.path.join(d, "1_Initial_condition.txt"), "w") as f:
        f.write("\n".join(s) + "\n")
    with open(os.path.join(d, "2_Boundary_Condition.txt"), "w") as f:
        f.write("LIST==================================================================\n"
                "Boundary_Priority      5\n(int)\n"
                "Pole                   Outflow     Absorbing   Solid_Surface   Farfield\n"
                "0                      4           2           3               1\n"
                "LIST==================================================================\n\nEND_OF_FILE\n")
    m = []
    m.append(f"int     num_of_dipole                   {_num(p['num_of_dipole'])}")
    mercury = p.get("solver") == "mercury"
    if mercury:
        # DipoleField::load_from_param (Z5_Mercury/include/operators/Dipole.h:44-88)
        for i, dp in enumerate(p.get("dipoles", [])[:int(p["num_of_dipole"])], start=1):
            m.append("LIST==================================================================")
            m.append(f"Dipole{i}         7")
            m.append("(double)")
            m.append("x0              y0              z0          mx          my          mz          a")
            m.append(" ".join(_num(dp[k]) for k in ["x0", "y0", "z0", "mx", "my", "mz", "a"]))
            m.append("LIST==================================================================")
        m.append(f"bool    is_Mercury_resistance           {_num(p['is_Mercury_resistance'])}")
        m.append(f"bool    use_implicit_mercury_resistance {_num(p['use_implicit_mercury_resistance'])}")
        m.append(f"bool    is_Ambipolar_Efield             {_num(p['is_Ambipolar_Efield'])}")
        m.append(f"double  r_min                           {_num(p['r_min'])}")
        m.append(f"double  r_max                           {_num(p['r_max'])}")
        m.append(f"bool    is_local_artificial_resistivity {_num(p['is_local_artificial_resistivity'])}")
        for k in ("local_arti_eta_max", "local_arti_x0", "local_arti_y0", "local_arti_z0", "local_arti_r_decay",
                  "local_arti_r_cutoff"):
            m.append(f"double  {k:<31} {_num(p[k])}")
    else:
        m.append(f"bool    is_Lunar_resistance           {_num(p['is_Lunar_resistance'])}")
        m.append(f"bool    use_implicit_lunar_resistance {_num(p['use_implicit_lunar_resistance'])}")
    m.append(f"int     n_resistive_subcycles           {_num(p['n_resistive_subcycles'])}")
    m.append(f"double  implicit_resistive_ksp_rtol     {_num(p['implicit_resistive_ksp_rtol'])}")
    m.append(f"double  implicit_resistive_ksp_atol     {_num(p['implicit_resistive_ksp_atol'])}")
    m.append(f"int     implicit_resistive_ksp_max_it   {_num(p['implicit_resistive_ksp_max_it'])}")
    m.append(f"double  arti_eta_max                    {_num(p['arti_eta_max'])}")
    m.append(f"double  J_range_start                   {_num(p['J_range_start'])}")
    m.append(f"double  J_range_on                      {_num(p['J_range_on'])}")
    m.append("")
    m.append("END_OF_FILE")
    with open(os.path.join(d, "3_MHD_Control.txt"), "w") as f:
        f.write("\n".join(m) + "\n")


def write_geometry(case_dir: str, spec: CaseSpec) -> None:
    gdir = os.path.join(case_dir, "CASE", "geometry")
    bdir = os.path.join(gdir, "boundary_condition")
    os.makedirs(bdir, exist_ok=True)
    rank = "   0"
    with open(os.path.join(gdir, f"grid{rank}.grd"), "wb") as f:
        f.write(np.int32(len(spec.blocks)).tobytes())
        for b in spec.blocks:
            nm = b.name.encode() + b"\0"
            f.write(np.int32(len(nm)).tobytes())
            f.write(nm)
        for b in spec.blocks:
            f.write(np.array(b.x.shape, dtype="<i4").tobytes())
        for b in spec.blocks:
            for c in (b.x, b.y, b.z):
                # stored with i fastest, then j, then k
                f.write(np.ascontiguousarray(np.transpose(c, (2, 1, 0)), dtype="<f8").tobytes())
    with open(os.path.join(bdir, f"boundary{rank}.txt"), "w") as f:
        for b in spec.blocks:
            f.write(f"{len(b.physical)}\n")
            for rng, name in b.physical:
                f.write(" ".join(str(v) for v in rng) + f" {2 + BC_NAMES.index(name)}\n")
    with open(os.path.join(bdir, "boundary_name.fvbnd"), "w") as f:
        f.write("FVBND 1 4\nUnspecified\n")
        for n in BC_NAMES:
            f.write(n + "\n")
        f.write("BOUNDARIES\n")
    total = sum(len(x) for x in spec.inner)
    with open(os.path.join(bdir, f"inner{rank}.txt"), "w") as f:
        f.write(f"{total}\n")
        f.write(" ".join(str(len(x)) for x in spec.inner) + "\n")
        f.write("imin imax jmin jmax kmin kmax block name | target imin imax jmin jmax kmin kmax block name\n")
        for ib, faces in enumerate(spec.inner):
            for fc in faces:
                f.write(" ".join(str(v) for v in fc.this_range) + f" {fc.this_block} {spec.blocks[ib].name} "
                        + " ".join(str(v) for v in fc.tar_range)
                        + f" {fc.tar_block} {spec.blocks[abs(fc.tar_block) - 1].name}\n")
    with open(os.path.join(bdir, f"parallel{rank}.txt"), "w") as f:
        f.write(f"{len(spec.blocks)}\n0\n" + " ".join("0" for _ in spec.blocks) + "\nno inter-rank faces\n")


def write_case(case_dir: str, spec: CaseSpec) -> None:
    write_setup(case_dir, spec.params)
    write_geometry(case_dir, spec)


# --------------------------------------------------------------------------
# Grids
# --------------------------------------------------------------------------

def periodic_box(n: Tuple[int, int, int], amp: float = 0.05) -> BlockGrid:
    """Unit cube with the sinusoidal map x = xi + a sin(2 pi eta),
    y = eta + a sin(2 pi zeta), z = zeta + a sin(2 pi xi), nodes at xi = i/n."""
    ni, nj, nk = n
    xi = np.arange(ni + 1) / ni
    et = np.arange(nj + 1) / nj
    ze = np.arange(nk + 1) / nk
    XI, ET, ZE = np.meshgrid(xi, et, ze, indexing="ij")
    x = XI + amp * np.sin(2.0 * np.pi * ET)
    y = ET + amp * np.sin(2.0 * np.pi * ZE)
    z = ZE + amp * np.sin(2.0 * np.pi * XI)
    return BlockGrid("Fluid", x, y, z)


def periodic_inner(n: Tuple[int, int, int]) -> List[InnerFace]:
    """Self-periodic interfaces of one block (block number -1 = periodic).
    In-plane pairing convention: the second tangential axis carries negative
    indices on both sides, so the transform is the identity up to the normal
    offset (include/1_grid/Grid_Boundary.h:274-299)."""
    I, J, K = n[0] + 1, n[1] + 1, n[2] + 1
    faces = []
    # i faces: tangential j (primary), k (secondary, negative)
    lo_i = (1, 1, 1, J, -1, -K)
    hi_i = (I, I, 1, J, -1, -K)
    lo_j = (1, I, 1, 1, -1, -K)
    hi_j = (1, I, J, J, -1, -K)
    lo_k = (1, I, -1, -J, 1, 1)
    hi_k = (1, I, -1, -J, K, K)
    for a, b in ((lo_i, hi_i), (lo_j, hi_j), (lo_k, hi_k)):
        faces.append(InnerFace(a, -1, b, -1))
        faces.append(InnerFace(b, -1, a, -1))
    return faces


def periodic_box_case(n=(64, 64, 64), **param_over) -> CaseSpec:
    blk = periodic_box(n)
    return CaseSpec([blk], [periodic_inner(n)], default_params(**param_over))


# --------------------------------------------------------------------------
# Initial states
# --------------------------------------------------------------------------

def _face_area_vectors(x, y, z):
    """Face area vectors S = 0.5 * (d1 x d2) of the bilinear faces spanned by
    node arrays (same construction as the reference's JDxi/JDet/JDze,
    src/3_field/4_MPCNS_Geometry.cpp:98-197).  Returns three arrays of shape
    (ni+1, nj, nk, 3), (ni, nj+1, nk, 3), (ni, nj, nk+1, 3) over interior faces."""
    P = np.stack([x, y, z], axis=-1)

    def quad(p0, pa, pb, pab):
        rx = pa - p0
        ry = pb - p0
        rx_ = pb - pab
        ry_ = pa - pab
        return 0.5 * (np.cross(rx, ry) + np.cross(rx_, ry_))

    Sxi = quad(P[:, :-1, :-1], P[:, 1:, :-1], P[:, :-1, 1:], P[:, 1:, 1:])
    Set = quad(P[:-1, :, :-1], P[:-1, :, 1:], P[1:, :, :-1], P[1:, :, 1:])
    Sze = quad(P[:-1, :-1, :], P[1:, :-1, :], P[:-1, 1:, :], P[1:, 1:, :])
    return Sxi, Set, Sze


def _curl_edge_to_face(axi, aet, aze):
    """Face circulation of edge 1-forms with the reference's orientation
    (Z4_Lunar/src/operators/CTOperators.cpp:6-56, multiplier +1).  Edge arrays
    cover interior edges: axi (ni, nj+1, nk+1), aet (ni+1, nj, nk+1),
    aze (ni+1, nj+1, nk)."""
    bxi = (aet[:, :, :-1] - aet[:, :, 1:]) + (aze[:, 1:, :] - aze[:, :-1, :])
    bet = (axi[:, :, 1:] - axi[:, :, :-1]) + (aze[:-1, :, :] - aze[1:, :, :])
    bze = (axi[:, :-1, :] - axi[:, 1:, :]) + (aet[1:, :, :] - aet[:-1, :, :])
    return bxi, bet, bze


def _embed(interior: np.ndarray, loc: int, ncell, nghost: int, ncomp: int) -> rst.FieldArray:
    lo, hi = rst.extent(loc, ncell, nghost)
    shape = (hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2], ncomp)
    a = np.zeros(shape)
    g = nghost
    s = interior.shape
    a[g:g + s[0], g:g + s[1], g:g + s[2], :] = interior.reshape(s[0], s[1], s[2], ncomp)
    return rst.FieldArray(lo, hi, a)


def initial_state(spec: CaseSpec, rho0=1.0, p0=0.1, v0=(0.1, 0.0, 0.0), B0=(1.0, 0.0, 0.0),
                  sigma=1e-3, seed=20261203, periodic=True, gamma=GAMMA) -> rst.RestartFile:
    """See _initial_state; B0 = None leaves the induced field to the noise
    alone (the applied field then lives in Badd)."""
    return _initial_state(spec, rho0, p0, v0, B0, sigma, seed, periodic, gamma)


def inflow_state(spec: CaseSpec, sigma=1e-3, seed=20261203) -> rst.RestartFile:
    """Farfield state everywhere plus seeded noise; the induced B is the curl
    of a random edge potential only (the IMF enters through Badd)."""
    from . import physics
    q, _ = physics.farfield_state(spec.params)
    p0 = (GAMMA - 1.0) * (q[4] - 0.5 * (q[1] ** 2 + q[2] ** 2 + q[3] ** 2) / q[0])
    return _initial_state(spec, q[0], p0, (q[1] / q[0], q[2] / q[0], q[3] / q[0]), None, sigma, seed, False, GAMMA)


def _initial_state(spec, rho0, p0, v0, B0, sigma, seed, periodic, gamma) -> rst.RestartFile:
    """Uniform state plus seeded Gaussian noise (numpy PCG64): rho and the
    three velocity components per cell, then a random edge potential whose
    face circulation is added to B, so div B stays at round-off.  U_H holds
    (rho, rho u, rho v, rho w, E) with E = p/(gamma-1) + rho|u|^2/2 (the fluid
    energy excludes the magnetic energy, Z4_Lunar/src/boundary/Boundary_Condition_Fluid.cpp:179).
    Ghost layers are left at zero; the reader fills them by a Sync."""
    rng = np.random.Generator(np.random.PCG64(seed))
    ng = spec.params["ngg"]
    fields = {nm: rst.FieldRecord(nm, loc, nc, ng) for nm, loc, nc in
              (("U_H", rst.CELL, 5), ("B_xi", rst.FACE_XI, 1), ("B_eta", rst.FACE_ET, 1), ("B_zeta", rst.FACE_ZE, 1))}
    for blk in spec.blocks:
        ni, nj, nk = blk.ncell
        rho = rho0 + sigma * rng.standard_normal((ni, nj, nk))
        vel = [v0[c] + sigma * rng.standard_normal((ni, nj, nk)) for c in range(3)]
        E = p0 / (gamma - 1.0) + 0.5 * rho * (vel[0] ** 2 + vel[1] ** 2 + vel[2] ** 2)
        U = np.stack([rho, rho * vel[0], rho * vel[1], rho * vel[2], E], axis=-1)
        fields["U_H"].blocks.append(_embed(U, rst.CELL, (ni, nj, nk), ng, 5))
        Sxi, Set, Sze = _face_area_vectors(blk.x, blk.y, blk.z)
        b = np.asarray(B0 if B0 is not None else (0.0, 0.0, 0.0), dtype=float)
        bxi, bet, bze = Sxi @ b, Set @ b, Sze @ b
        h2 = float(np.mean(np.linalg.norm(Sxi, axis=-1)))
        if periodic:
            a_u = [sigma * h2 * rng.standard_normal((ni, nj, nk)) for _ in range(3)]
            axi = np.pad(a_u[0], ((0, 0), (0, 1), (0, 1)), mode="wrap")
            aet = np.pad(a_u[1], ((0, 1), (0, 0), (0, 1)), mode="wrap")
            aze = np.pad(a_u[2], ((0, 1), (0, 1), (0, 0)), mode="wrap")
        else:
            axi = sigma * h2 * rng.standard_normal((ni, nj + 1, nk + 1))
            aet = sigma * h2 * rng.standard_normal((ni + 1, nj, nk + 1))
            aze = sigma * h2 * rng.standard_normal((ni + 1, nj + 1, nk))
        dxi, det, dze = _curl_edge_to_face(axi, aet, aze)
        fields["B_xi"].blocks.append(_embed(bxi + dxi, rst.FACE_XI, (ni, nj, nk), ng, 1))
        fields["B_eta"].blocks.append(_embed(bet + det, rst.FACE_ET, (ni, nj, nk), ng, 1))
        fields["B_zeta"].blocks.append(_embed(bze + dze, rst.FACE_ZE, (ni, nj, nk), ng, 1))
    return rst.RestartFile(0, 0.0, len(spec.blocks), fields)


# --------------------------------------------------------------------------
# Six-block cubed-sphere shell
# --------------------------------------------------------------------------

# cube faces: centre direction, first and second tangential axes; (r, e1, e2)
# is right-handed for every face
_CUBE_FACES = [
    ((1, 0, 0), (0, 1, 0), (0, 0, 1)),
    ((-1, 0, 0), (0, -1, 0), (0, 0, 1)),
    ((0, 1, 0), (-1, 0, 0), (0, 0, 1)),
    ((0, -1, 0), (1, 0, 0), (0, 0, 1)),
    ((0, 0, 1), (0, 1, 0), (-1, 0, 0)),
    ((0, 0, -1), (0, 1, 0), (1, 0, 0)),
]


def cubed_sphere_blocks(nr: int, na: int, r0: float = 1.0, r1: float = 8.0) -> List[BlockGrid]:
    """Six blocks of nr log-spaced radial cells over [r0, r1] (index i, outward)
    times na x na equiangular gnomonic cells (indices j, k).  Inner radius is a
    Solid_Surface, outer radius a Farfield."""
    r = r0 * (r1 / r0) ** (np.arange(nr + 1) / nr)
    a = -np.pi / 4 + (np.pi / 2) * np.arange(na + 1) / na
    TA, TB = np.meshgrid(np.tan(a), np.tan(a), indexing="ij")
    blocks = []
    for c, e1, e2 in _CUBE_FACES:
        c, e1, e2 = (np.asarray(v, dtype=float) for v in (c, e1, e2))
        d = c[None, None, :] + TA[..., None] * e1[None, None, :] + TB[..., None] * e2[None, None, :]
        d = d / np.linalg.norm(d, axis=-1, keepdims=True)
        P = r[:, None, None, None] * d[None, :, :, :]
        blk = BlockGrid("Fluid", P[..., 0].copy(), P[..., 1].copy(), P[..., 2].copy())
        blk.physical = [((0, 0, 0, na, 0, na), "Solid_Surface"), ((nr, nr, 0, na, 0, na), "Farfield")]
        blocks.append(blk)
    return blocks


def _face_nodes(b: BlockGrid, axis: int, side: int) -> np.ndarray:
    P = np.stack([b.x, b.y, b.z], axis=-1)
    idx = [slice(None)] * 3
    idx[axis] = 0 if side == 0 else P.shape[axis] - 1
    return P[tuple(idx)]


def match_interfaces(blocks: List[BlockGrid], tol: float = 1e-9) -> List[List[InnerFace]]:
    """Finds conforming block faces by node coordinates and writes each pair in
    the inner-file convention: on the first side the first tangential axis
    runs 1..N (positive), the second -1..-N (negative); on the target side the
    axis matching the first carries positive, the one matching the second
    negative indices, each descending where the target runs the opposite way
    (pairing rules of include/1_grid/Grid_Boundary.h:236-330 and
    src/2_topology/2_MPCNS_Topology.cpp:76-160).  The neighbour's entry is
    the exact mirror (its range = our target range and vice versa), which is
    how the reader pairs the two sides (src/1_grid/1_MPCNS_Grid.cpp:468-520)."""
    inner: List[List[InnerFace]] = [[] for _ in blocks]
    done = {}
    faces = [(ia, ax, sd) for ia in range(len(blocks)) for ax in range(3) for sd in (0, 1)]
    for (ia, axA, sA) in faces:
        A = blocks[ia]
        if (ia, axA, sA) in done:
            continue
        FA = _face_nodes(A, axA, sA)
        found = None
        for (ib, axB, sB) in faces:
            if (ib, axB, sB) == (ia, axA, sA):
                continue
            m = _match(FA, _face_nodes(blocks[ib], axB, sB), tol)
            if m is not None:
                found = (ib, axB, sB, m)
                break
        if not found:
            continue
        ib, axB, sB, (t1B, rev1, t2B, rev2) = found
        B = blocks[ib]
        nA = [s_ - 1 for s_ in A.x.shape]
        nB = [s_ - 1 for s_ in B.x.shape]
        tA = [d for d in range(3) if d != axA]
        tBax = [d for d in range(3) if d != axB]
        rngA = [0] * 6
        rngB = [0] * 6
        for d in range(3):
            if d == axA:
                v = 1 if sA == 0 else nA[d] + 1
                rngA[2 * d], rngA[2 * d + 1] = v, v
            elif d == tA[0]:
                rngA[2 * d], rngA[2 * d + 1] = 1, nA[d] + 1
            else:
                rngA[2 * d], rngA[2 * d + 1] = -1, -(nA[d] + 1)
        for d in range(3):
            if d == axB:
                v = 1 if sB == 0 else nB[d] + 1
                rngB[2 * d], rngB[2 * d + 1] = v, v
            elif d == tBax[t1B]:
                lo_, hi_ = 1, nB[d] + 1
                rngB[2 * d], rngB[2 * d + 1] = (hi_, lo_) if rev1 else (lo_, hi_)
            else:
                lo_, hi_ = -1, -(nB[d] + 1)
                rngB[2 * d], rngB[2 * d + 1] = (hi_, lo_) if rev2 else (lo_, hi_)
        inner[ia].append(InnerFace(tuple(rngA), ia + 1, tuple(rngB), ib + 1))
        inner[ib].append(InnerFace(tuple(rngB), ib + 1, tuple(rngA), ia + 1))
        done[(ia, axA, sA)] = True
        done[(ib, axB, sB)] = True
    return inner


def _match(FA: np.ndarray, FB: np.ndarray, tol: float):
    """If face node arrays coincide up to an axis swap/reversal, returns
    (which B tangential axis matches A's first, reversed?, the one matching
    A's second, reversed?)."""
    for swap in (False, True):
        G = np.transpose(FB, (1, 0, 2)) if swap else FB
        if G.shape[:2] != FA.shape[:2]:
            continue
        for r1 in (False, True):
            for r2 in (False, True):
                H = G[::-1] if r1 else G
                H = H[:, ::-1] if r2 else H
                if np.max(np.abs(H - FA)) < tol:
                    # A axis 0 <-> B axis (1 if swap else 0)
                    t1B = 1 if swap else 0
                    t2B = 0 if swap else 1
                    rev1 = r1
                    rev2 = r2
                    return t1B, rev1, t2B, rev2
    return None


def cubed_sphere_case(nr=96, na=48, **param_over) -> CaseSpec:
    blocks = cubed_sphere_blocks(nr, na)
    return CaseSpec(blocks, match_interfaces(blocks), default_params(**param_over))


def inflow_params(mach_u=8.0, B=(0.0, 0.5 / math.sqrt(2.0), 0.5 / math.sqrt(2.0)), p0=0.05, **over):
    """Parameters whose Farfield/initial state (BuildLunarBackgroundState,
    Z4_Lunar/include/0_BackgroundState.h:20-66) is rho = 1, v = (-mach_u, 0, 0),
    p = p0 and B = `B` in nondimensional units."""
    p = default_params(**over)
    r = p["REF"]
    k_B = R_UNI / NA
    rho_ref = r["Molecular_mass"] / NA * r["n"]
    T = p0 * rho_ref * r["U"] * r["U"] / (r["n"] * k_B)
    p["INITIAL"] = dict(U=mach_u * r["U"], T=T, n=r["n"], Molecular_mass=r["Molecular_mass"], c_y=0.0, c_z=0.0,
                        Bx=B[0] * r["B_ref"], By=B[1] * r["B_ref"], Bz=B[2] * r["B_ref"])
    return p


def mercury_params(**over):
    """Parameters of the reference's Mercury (two-fluid) solver: the inflow
    parameters plus the keys MercurySolver reads (Z5_Mercury/9999setup/*,
    MercurySolver.cpp, MercurySolver_Tools.cpp); every optional term off
    unless set.  dipoles: [dict(x0, y0, z0, mx, my, mz, a)] in SI units."""
    base = dict(solver="mercury", mole_mass2=0.023, eta_max_mercury=0.0, is_Mercury_resistance=0,
                use_implicit_mercury_resistance=0, is_Ambipolar_Efield=0, r_min=1.1, r_max=1.2,
                is_local_artificial_resistivity=0, local_arti_eta_max=0.0, local_arti_x0=0.0, local_arti_y0=0.0,
                local_arti_z0=0.0, local_arti_r_decay=0.05, local_arti_r_cutoff=0.05, dipoles=[])
    base.update(over)
    return inflow_params(**base)


def cubed_sphere_inflow_case(nr=96, na=48, **over) -> CaseSpec:
    blocks = cubed_sphere_blocks(nr, na)
    return CaseSpec(blocks, match_interfaces(blocks), inflow_params(**over))


# --------------------------------------------------------------------------
# Tiled slab: radial direction bounded by a Solid_Surface (x = r0) and a
# Farfield (x = r1), transverse directions periodic and split into tiles
# --------------------------------------------------------------------------

def slab_blocks(nr: int, nt: Tuple[int, int], tiles: Tuple[int, int], r0: float = 1.0, r1: float = 8.0,
                amp: float = 0.03) -> List[BlockGrid]:
    """Blocks of nr log-spaced cells over x in [r0, r1] (index i) times
    nt[0] x nt[1] cells (indices j, k) each, tiles[0] x tiles[1] tiles over
    the square [-1/2, 1/2)^2 in (Y, Z) with the map y = Y + amp sin(2 pi Z),
    z = Z + amp sin(2 pi Y), periodic with period 1 in Y and Z.  All blocks
    share one orientation (interfaces map indices by translation).  The
    reference's resistive shell 0.84 < |x| < 1.04 then covers the patch of
    the wall around y = z = 0."""
    TJ, TK = tiles
    NJ, NK = nt[0] * TJ, nt[1] * TK
    X = r0 * (r1 / r0) ** (np.arange(nr + 1) / nr)
    blocks = []
    for tj in range(TJ):
        for tk in range(TK):
            Y = (tj * nt[0] + np.arange(nt[0] + 1)) / NJ - 0.5
            Z = (tk * nt[1] + np.arange(nt[1] + 1)) / NK - 0.5
            XX, YY, ZZ = np.meshgrid(X, Y, Z, indexing="ij")
            x = XX.copy()
            y = YY + amp * np.sin(2.0 * np.pi * ZZ)
            z = ZZ + amp * np.sin(2.0 * np.pi * YY)
            blk = BlockGrid("Fluid", x, y, z)
            blk.physical = [((0, 0, 0, nt[0], 0, nt[1]), "Solid_Surface"),
                            ((nr, nr, 0, nt[0], 0, nt[1]), "Farfield")]
            blocks.append(blk)
    return blocks


def slab_interfaces(nr: int, nt: Tuple[int, int], tiles: Tuple[int, int]) -> List[List[InnerFace]]:
    """Transverse interfaces of the tile array (with wrap-around).  Every
    interface is flagged periodic (negative block numbers), so that ghost
    nodes are built by reflection (the reference skips the node copy for
    periodic interfaces, src/1_grid/1_MPCNS_Grid.cpp:1262-1281)."""
    TJ, TK = tiles
    I, J, K = nr + 1, nt[0] + 1, nt[1] + 1

    def bid(tj, tk):
        return (tj % TJ) * TK + (tk % TK)

    inner = [[] for _ in range(TJ * TK)]
    jmin = (1, I, 1, 1, -1, -K)
    jmax = (1, I, J, J, -1, -K)
    kmin = (1, I, -1, -J, 1, 1)
    kmax = (1, I, -1, -J, K, K)
    for tj in range(TJ):
        for tk in range(TK):
            b = bid(tj, tk)
            inner[b].append(InnerFace(jmin, -(b + 1), jmax, -(bid(tj - 1, tk) + 1)))
            inner[b].append(InnerFace(jmax, -(b + 1), jmin, -(bid(tj + 1, tk) + 1)))
            inner[b].append(InnerFace(kmin, -(b + 1), kmax, -(bid(tj, tk - 1) + 1)))
            inner[b].append(InnerFace(kmax, -(b + 1), kmin, -(bid(tj, tk + 1) + 1)))
    return inner


def shell_blocks(nr: int, nth: int, nph: int, r0: float = 1.0, r1: float = 8.0) -> List[BlockGrid]:
    """One spherical-shell block: nr log-spaced radial cells over [r0, r1]
    (index i), nth polar cells over theta in [0, pi] (index j) and nph
    azimuthal cells over phi in [0, 2 pi) (index k, nph even), with
    x = r sin(theta) cos(phi), y = r sin(theta) sin(phi), z = r cos(theta).
    Physical patches: Solid_Surface at i = 0, Farfield at i = nr, Pole at
    j = 0 and j = nth (the node rows on the z axis)."""
    if nph % 2:
        raise ValueError("a Pole patch needs an even number of azimuthal cells")
    r = r0 * (r1 / r0) ** (np.arange(nr + 1) / nr)
    th = np.pi * np.arange(nth + 1) / nth
    ph = 2.0 * np.pi * np.arange(nph + 1) / nph
    R, T, P = np.meshgrid(r, th, ph, indexing="ij")
    x = R * np.sin(T) * np.cos(P)
    y = R * np.sin(T) * np.sin(P)
    z = R * np.cos(T)
    # the pole rows lie exactly on the axis
    x[:, 0, :] = 0.0
    y[:, 0, :] = 0.0
    x[:, nth, :] = 0.0
    y[:, nth, :] = 0.0
    blk = BlockGrid("Fluid", x, y, z)
    blk.physical = [((0, 0, 0, nth, 0, nph), "Solid_Surface"), ((nr, nr, 0, nth, 0, nph), "Farfield"),
                    ((0, nr, 0, 0, 0, nph), "Pole"), ((0, nr, nth, nth, 0, nph), "Pole")]
    return [blk]


def shell_case(nr=16, nth=8, nph=12, **over) -> CaseSpec:
    """The single-block spherical shell with Pole patches and its azimuthal
    direction periodic onto itself (inflow parameters as the slab's)."""
    I, J, K = nr + 1, nth + 1, nph + 1
    kmin = (1, I, -1, -J, 1, 1)
    kmax = (1, I, -1, -J, K, K)
    inner = [[InnerFace(kmin, -1, kmax, -1), InnerFace(kmax, -1, kmin, -1)]]
    return CaseSpec(shell_blocks(nr, nth, nph), inner, inflow_params(**over))


def slab_case(nr=96, nt=(48, 48), tiles=(3, 2), **over) -> CaseSpec:
    blocks = slab_blocks(nr, nt, tiles)
    spec = CaseSpec(blocks, slab_interfaces(nr, nt, tiles), inflow_params(**over))
    spec.tiles = tiles
    return spec


# --------------------------------------------------------------------------
# Parameter sweep: independent single-block runs of uneven sizes
# --------------------------------------------------------------------------

class MT19937_64:
    """The 64-bit Mersenne Twister (Matsumoto and Nishimura, 2000) with the
    parameters of std::mt19937_64, for the sweep's draws."""

    N, M = 312, 156
    UPPER, LOWER = 0xFFFFFFFF80000000, 0x7FFFFFFF
    MASK = (1 << 64) - 1

    def __init__(self, seed: int):
        self.mt = [0] * self.N
        self.mt[0] = seed & self.MASK
        for i in range(1, self.N):
            self.mt[i] = (6364136223846793005 * (self.mt[i - 1] ^ (self.mt[i - 1] >> 62)) + i) & self.MASK
        self.i = self.N

    def _twist(self):
        mt = self.mt
        for i in range(self.N):
            x = (mt[i] & self.UPPER) | (mt[(i + 1) % self.N] & self.LOWER)
            xa = x >> 1
            if x & 1:
                xa ^= 0xB5026F5AA96619E9
            mt[i] = mt[(i + self.M) % self.N] ^ xa
        self.i = 0

    def next(self) -> int:
        if self.i >= self.N:
            self._twist()
        y = self.mt[self.i]
        self.i += 1
        y ^= (y >> 29) & 0x5555555555555555
        y ^= (y << 17) & 0x71D67FFFEDA60000
        y ^= (y << 37) & 0xFFF7EEE000000000
        y ^= y >> 43
        return y & self.MASK

    def integer(self, lo: int, hi: int) -> int:
        """lo + x mod (hi - lo + 1): uniform on {lo..hi} up to a bias below 1e-16"""
        return lo + self.next() % (hi - lo + 1)

    def real(self, lo: float, hi: float) -> float:
        """lo + (hi - lo) u with u the top 53 bits of a draw over 2^53"""
        return lo + (hi - lo) * ((self.next() >> 11) * 2.0 ** -53)


def sweep_cases(nruns: int = 48, seed: int = 5, nr=(32, 128), nt=(24, 96), mach=(4.0, 12.0), angle=(0.0, 180.0),
                grid: str = "slab"):
    """Runs of a parameter sweep: per run (drawn in this order from
    MT19937_64(seed)) radial cells Nr, transverse cells Nt, inflow speed
    `mach` (v = (-mach, 0, 0) in units of the reference speed) and IMF clock
    angle theta in degrees, B = 0.5 (0, cos theta, sin theta).  grid "slab":
    each run is one Nr x Nt x Nt slab block between a Solid_Surface and a
    Farfield, periodic onto itself transversally; grid "shell": one
    spherical shell of Nr x Nt x Nph cells with Pole patches (shell_case),
    Nph = Nt rounded up to even (the Pole's ghost rows pair phi with
    phi + pi).  Returns [(spec, dict of the drawn values)]."""
    if grid not in ("slab", "shell"):
        raise ValueError(f"unknown sweep grid {grid}")
    g = MT19937_64(seed)
    out = []
    for _ in range(nruns):
        n_r = g.integer(*nr)
        n_t = g.integer(*nt)
        m = g.real(*mach)
        th = g.real(*angle)
        B = (0.0, 0.5 * math.cos(math.radians(th)), 0.5 * math.sin(math.radians(th)))
        if grid == "shell":
            spec = shell_case(n_r, n_t, n_t + (n_t & 1), mach_u=m, B=B)
        else:
            spec = slab_case(n_r, (n_t, n_t), (1, 1), mach_u=m, B=B)
        out.append((spec, dict(nr=n_r, nt=n_t, mach=m, angle=th)))
    return out
