"""CPU restatement of the reference's per-step MHD algorithm (numpy).

TEST INFRASTRUCTURE ONLY: this module is the checker the GPU path is
compared against in tests/, __graft_entry__.smoke() and bench.py's CPU
baseline; nothing in beta1_b200/ imports it.

It restates LunarSolver::StepOnce (Z4_Lunar/src/LunarSolver_Driver.cpp:21-92)
stage by stage with whole-array numpy operations in the reference's floating
point operation order, so on the reference's own inputs it reproduces the
reference's outputs (pinned against the fixtures in tests/golden, which the
reference solver itself produced).  Boundary synchronisations of the
periodic box and the tiled slab apply the same composed tables the device
receives (their own equality with the reference's Sync is pinned separately
against the reference's probe fixtures); on the Pole shell (ShellOracle) the
Sync runs the reference's handlers themselves, in the reference's order.

Data layout: per block, a field is a float64 array (ncomp, NI, NJ, NK) over
the padded logical box [-G, n + 1 + G) in each direction.
"""
from __future__ import annotations

import numpy as np

# name: (location code of the restart file, components, ghost layers), as the
# reference registers them (Z4_Lunar/main.cpp:61-123, src/3_field/4_MPCNS_Geometry.cpp:4-69)
FIELDS = {
    "U_H": (0, 5, 4), "B_xi": (1, 1, 4), "B_eta": (2, 1, 4), "B_zeta": (3, 1, 4), "PV_H": (0, 5, 4),
    "U_plus": (0, 3, 4), "B_cell": (0, 3, 4), "Bind_cell": (0, 3, 4), "J_xi": (4, 1, 4), "J_eta": (5, 1, 4),
    "J_zeta": (6, 1, 4), "J_cell": (0, 3, 4), "Eface_xi": (1, 3, 4), "Eface_eta": (2, 3, 4),
    "Eface_zeta": (3, 3, 4), "E_xi": (4, 1, 4), "E_eta": (5, 1, 4), "E_zeta": (6, 1, 4), "RHS_H": (0, 5, 0),
    "RHS_B_xi": (1, 1, 0), "RHS_B_eta": (2, 1, 0), "RHS_B_zeta": (3, 1, 0), "Badd_xi": (1, 1, 4),
    "Badd_eta": (2, 1, 4), "Badd_zeta": (3, 1, 4), "Jac": (0, 1, 3), "JDxi": (1, 3, 4), "JDet": (2, 3, 4),
    "JDze": (3, 3, 4), "beta_xi": (1, 1, 3), "beta_eta": (2, 1, 3), "beta_zeta": (3, 1, 3), "alpha_xi": (4, 1, 3),
    "alpha_eta": (5, 1, 3), "alpha_zeta": (6, 1, 3), "Bcell_from_Bface_w": (0, 18, 3),
    "Jcell_from_Jedge_w": (0, 36, 3), "Eres_xi": (4, 1, 4), "Eres_eta": (5, 1, 4), "Eres_zeta": (6, 1, 4),
    "dB_xi": (1, 1, 4), "dB_eta": (2, 1, 4), "dB_zeta": (3, 1, 4), "dJ_xi": (4, 1, 4), "dJ_eta": (5, 1, 4),
    "dJ_zeta": (6, 1, 4), "RHS_Bres_xi": (1, 1, 0), "RHS_Bres_eta": (2, 1, 0), "RHS_Bres_zeta": (3, 1, 0),
    "divB": (0, 1, 1), "dr_xi": (4, 3, 3), "dr_eta": (5, 3, 3), "dr_zeta": (6, 3, 3),
    "Area_xi": (1, 1, 3), "Area_eta": (2, 1, 3), "Area_zeta": (3, 1, 3), "dl_xi": (4, 1, 3), "dl_eta": (5, 1, 3),
    "dl_zeta": (6, 1, 3), "Ehall_xi": (4, 1, 4), "Ehall_eta": (5, 1, 4), "Ehall_zeta": (6, 1, 4),
    "Astar_xi": (4, 1, 3), "Astar_eta": (5, 1, 3), "Astar_zeta": (6, 1, 3),
}
PLUS = {0: (0, 0, 0), 1: (1, 0, 0), 2: (0, 1, 0), 3: (0, 0, 1), 4: (0, 1, 1), 5: (1, 0, 1), 6: (1, 1, 0)}


class Block:
    def __init__(self, n, G=4):
        self.n = tuple(n)
        self.G = G
        self.f = {}
        for name, (loc, nc, _) in FIELDS.items():
            self.f[name] = np.zeros((nc, n[0] + 1 + 2 * G, n[1] + 1 + 2 * G, n[2] + 1 + 2 * G))

    def s(self, lo, hi):
        """slices of the logical box [lo, hi)"""
        G = self.G
        return tuple(slice(l + G, h + G) for l, h in zip(lo, hi))

    def sh(self, lo, hi, d):
        """box shifted by d"""
        return self.s(tuple(l + x for l, x in zip(lo, d)), tuple(h + x for h, x in zip(hi, d)))

    def box(self, name, m, lo, hi, d=(0, 0, 0)):
        return self.f[name][m][self.sh(lo, hi, d)]

    def inner(self, loc):
        p = PLUS[loc]
        return (0, 0, 0), (self.n[0] + p[0], self.n[1] + p[1], self.n[2] + p[2])

    def set_ref(self, name, lo, data):
        """store a reference-layout array (ni, nj, nk, ncomp) whose logical origin is lo"""
        sl = tuple(slice(l + self.G, l + self.G + s) for l, s in zip(lo, data.shape[:3]))
        for m in range(data.shape[3]):
            self.f[name][m][sl] = data[..., m]

    def get_ref(self, name):
        """the field's logical box [lo, hi) in reference layout (ni, nj, nk, ncomp)"""
        loc, nc, ng = FIELDS[name]
        p = PLUS[loc]
        lo = (-ng, -ng, -ng)
        hi = (self.n[0] + p[0] + ng, self.n[1] + p[1] + ng, self.n[2] + p[2] + ng)
        return np.stack([self.box(name, m, lo, hi) for m in range(nc)], axis=-1)


def smax(a, b):
    """std::max(a, b) elementwise (first argument unless the second is larger)."""
    return np.where(a < b, b, a)


class Oracle:
    def __init__(self, ncells, consts, G=4):
        self.blocks = [Block(n, G) for n in ncells]
        self.c = consts
        self.dt = 0.0
        self.time = 0.0
        self.syncs = {}  # group -> dict(gather=(dst, src) as (field, block, m, i, j, k) arrays, consts, walls)

    # ------------------------------------------------------------------ syncs
    def aos_points(self, name, b, offsets):
        """(m, I, J, K) of AoS offsets within field `name`'s logical box on block b
        (FieldBlock storage order, include/3_field/Field_Array.h:177)."""
        blk = self.blocks[b]
        loc, nc, ng = FIELDS[name]
        p = PLUS[loc]
        ext = [blk.n[a] + p[a] + 2 * ng for a in range(3)]
        o = np.asarray(offsets, dtype=np.int64)
        m = o % nc
        t = o // nc
        K = t % ext[2] - ng
        t = t // ext[2]
        J = t % ext[1] - ng
        I = t // ext[1] - ng
        return m, I, J, K

    def add_copies(self, group, dst_name, dst_block, dst_off, src_name, src_block, src_off):
        """Composed copies of a Sync group: point dst[n] takes the value src[n] had before the sync."""
        g = self.syncs.setdefault(group, dict(copies=[], consts=[], walls=[]))
        g["copies"].append(((dst_name, dst_block) + self.aos_points(dst_name, dst_block, dst_off),
                            (src_name, src_block) + self.aos_points(src_name, src_block, src_off)))

    def add_consts(self, group, name, block, off, val):
        g = self.syncs.setdefault(group, dict(copies=[], consts=[], walls=[]))
        g["consts"].append(((name, block) + self.aos_points(name, block, off), np.asarray(val, dtype=np.float64)))

    def add_wall(self, group, block, direction):
        g = self.syncs.setdefault(group, dict(copies=[], consts=[], walls=[]))
        g["walls"].append((block, direction))

    def add_point_tables(self, group, names, dst, src, cdst=(), cval=(), walls=()):
        """A group's tables in point-id form ((field index << 56) | (block << 40) | AoS offset,
        `names` maps field indices to names)."""
        dst, src = np.asarray(dst, dtype=np.int64), np.asarray(src, dtype=np.int64)
        mask = (1 << 40) - 1
        key = np.stack([dst >> 56, (dst >> 40) & 0xFFFF, src >> 56, (src >> 40) & 0xFFFF], axis=1)
        if len(key):
            uk, inv = np.unique(key, axis=0, return_inverse=True)
            for q, (fd, bd, fs, bs) in enumerate(uk.tolist()):
                sel = inv.ravel() == q
                self.add_copies(group, names[fd], bd, dst[sel] & mask, names[fs], bs, src[sel] & mask)
        cdst = np.asarray(cdst, dtype=np.int64)
        cval = np.asarray(cval, dtype=np.float64)
        if len(cdst):
            ck = np.stack([cdst >> 56, (cdst >> 40) & 0xFFFF], axis=1)
            uk, inv = np.unique(ck, axis=0, return_inverse=True)
            for q, (f, b) in enumerate(uk.tolist()):
                sel = inv.ravel() == q
                self.add_consts(group, names[f], b, cdst[sel] & mask, cval[sel])
        for (b, d) in walls:
            self.add_wall(group, b, d)
        self.syncs.setdefault(group, dict(copies=[], consts=[], walls=[]))

    def _view(self, pt):
        name, b, m, I, J, K = pt
        blk = self.blocks[b]
        return blk.f[name], (m, I + blk.G, J + blk.G, K + blk.G)

    def sync(self, group):
        """LunarBoundary::Sync(group) (Z4_Lunar/src/boundary/Boundary.cpp:30-40): fixed values and wall
        handlers first, then every copy reads the values from before the sync."""
        s = self.syncs.get(group)
        if s is None:
            return
        for pt, val in s["consts"]:
            arr, idx = self._view(pt)
            arr[idx] = val
        for (b, d) in s["walls"]:
            self.wall_u(b, d)
        vals = []
        for _, src in s["copies"]:
            arr, idx = self._view(src)
            vals.append(arr[idx].copy())
        for (dst, _), v in zip(s["copies"], vals):
            arr, idx = self._view(dst)
            arr[idx] = v

    def wall_u(self, b, d):
        """LunarBoundary::BC_Solid_Surface_ on the i-minimum face
        (Z4_Lunar/src/boundary/Boundary_Condition_Fluid.cpp:19-185)."""
        assert d == -1
        blk = self.blocks[b]
        g = self.c["gamma"]
        U = blk.f["U_H"]
        G = blk.G
        n = blk.n
        J, K = slice(G, G + n[1]), slice(G, G + n[2])

        def pressure(rho, mx, my, mz, E):
            rho = smax(rho, 2.5e-3)
            ke = 0.5 * (mx * mx + my * my + mz * mz) / rho
            eint = E - ke
            eint = np.where(eint < 0.0, 0.0, eint)
            return smax((g - 1.0) * eint, 1e-12)

        r = [U[m][G + 1, J, K] for m in range(5)]
        rho_r = smax(r[0], 2.5e-3)
        p_r = pressure(rho_r, r[1], r[2], r[3], r[4])
        zero = 0.0
        ke_g = 0.5 * rho_r * (zero * zero + zero * zero + zero * zero)
        U[0][G, J, K] = rho_r
        U[1][G, J, K] = rho_r * zero
        U[2][G, J, K] = rho_r * zero
        U[3][G, J, K] = rho_r * zero
        U[4][G, J, K] = p_r / (g - 1.0) + ke_g
        rho_r = smax(U[0][G, J, K], 2.5e-3)
        p_r = pressure(rho_r, U[1][G, J, K], U[2][G, J, K], U[3][G, J, K], U[4][G, J, K])
        ke_g = 0.5 * rho_r * (zero * zero + zero * zero + zero * zero)
        for ng in range(1, G + 1):
            U[0][G - ng, J, K] = rho_r
            U[1][G - ng, J, K] = rho_r * zero
            U[2][G - ng, J, K] = rho_r * zero
            U[3][G - ng, J, K] = rho_r * zero
            U[4][G - ng, J, K] = p_r / (g - 1.0) + ke_g

    # ------------------------------------------------------- derived fields
    def calc_bcell(self, blk):
        """calc_Bcell (Z4_Lunar/src/physics/LunarSolver_Tools.cpp:163-240)"""
        lo, hi = blk.inner(0)
        bx = lambda d=(0, 0, 0): blk.box("B_xi", 0, lo, hi, d)
        be = lambda d=(0, 0, 0): blk.box("B_eta", 0, lo, hi, d)
        bz = lambda d=(0, 0, 0): blk.box("B_zeta", 0, lo, hi, d)
        ax = lambda d=(0, 0, 0): blk.box("Badd_xi", 0, lo, hi, d)
        ae = lambda d=(0, 0, 0): blk.box("Badd_eta", 0, lo, hi, d)
        az = lambda d=(0, 0, 0): blk.box("Badd_zeta", 0, lo, hi, d)
        tot = [-bx() - ax(), bx((1, 0, 0)) + ax((1, 0, 0)), -be() - ae(), be((0, 1, 0)) + ae((0, 1, 0)),
               -bz() - az(), bz((0, 0, 1)) + az((0, 0, 1))]
        ind = [-bx(), bx((1, 0, 0)), -be(), be((0, 1, 0)), -bz(), bz((0, 0, 1))]
        W = lambda q: blk.box("Bcell_from_Bface_w", q, lo, hi)
        acc_t = [0.0, 0.0, 0.0]
        acc_i = [0.0, 0.0, 0.0]
        for q in range(6):
            for c in range(3):
                w = W(6 * c + q)
                acc_t[c] = acc_t[c] + w * tot[q]
                acc_i[c] = acc_i[c] + w * ind[q]
        for c in range(3):
            blk.f["B_cell"][c][blk.s(lo, hi)] = acc_t[c]
            blk.f["Bind_cell"][c][blk.s(lo, hi)] = acc_i[c]

    def curl_adj(self, blk, fB, fJ, mult=1.0):
        """CTOperators::CurlAdjFaceToEdge times alpha
        (Z4_Lunar/src/operators/CTOperators.cpp:58-110, LunarSolver_Tools.cpp:777-835)"""
        Fx, Fe, Fz = fB
        for ea, nm in enumerate(fJ):
            lo, hi = blk.inner(4 + ea)
            bx = lambda d: blk.box("beta_xi", 0, lo, hi, d) * blk.box(Fx, 0, lo, hi, d)
            be = lambda d: blk.box("beta_eta", 0, lo, hi, d) * blk.box(Fe, 0, lo, hi, d)
            bz = lambda d: blk.box("beta_zeta", 0, lo, hi, d) * blk.box(Fz, 0, lo, hi, d)
            z = (0, 0, 0)
            if ea == 0:
                val = (be((0, 0, -1)) - be(z)) + (bz(z) - bz((0, -1, 0)))
            elif ea == 1:
                val = (bx(z) - bx((0, 0, -1))) + (bz((-1, 0, 0)) - bz(z))
            else:
                val = (bx((0, -1, 0)) - bx(z)) + (be(z) - be((-1, 0, 0)))
            alpha = blk.box(("alpha_xi", "alpha_eta", "alpha_zeta")[ea], 0, lo, hi)
            blk.f[nm][0][blk.s(lo, hi)] = (mult * val) * alpha

    def calc_jcell(self, blk):
        """calc_Jcell (LunarSolver_Tools.cpp:837-892)"""
        lo, hi = blk.inner(0)
        jx = lambda d: blk.box("J_xi", 0, lo, hi, d)
        je = lambda d: blk.box("J_eta", 0, lo, hi, d)
        jz = lambda d: blk.box("J_zeta", 0, lo, hi, d)
        s = [jx((0, 0, 0)), jx((0, 1, 0)), jx((0, 0, 1)), jx((0, 1, 1)), je((0, 0, 0)), je((1, 0, 0)),
             je((0, 0, 1)), je((1, 0, 1)), jz((0, 0, 0)), jz((1, 0, 0)), jz((0, 1, 0)), jz((1, 1, 0))]
        acc = [0.0, 0.0, 0.0]
        for q in range(12):
            for c in range(3):
                acc[c] = acc[c] + blk.box("Jcell_from_Jedge_w", 12 * c + q, lo, hi) * s[q]
        for c in range(3):
            blk.f["J_cell"][c][blk.s(lo, hi)] = acc[c]

    def calc_pv_uplus(self, blk):
        """calc_PV + calc_Uplus over the whole array (LunarSolver_Tools.cpp:58-141)"""
        g = self.c["gamma"]
        U = blk.f["U_H"]
        rho = smax(U[0], 1e-12)
        u = U[1] / rho
        v = U[2] / rho
        w = U[3] / rho
        ke = 0.5 * rho * (u * u + v * v + w * w)
        eint = U[4] - ke
        eint = np.where(eint < 0.0, 0.0, eint)
        p = smax((g - 1.0) * eint, 1e-12)
        T = p / (rho * self.c["state_coeff"])
        PV = blk.f["PV_H"]
        PV[0], PV[1], PV[2], PV[3], PV[4] = u, v, w, p, T
        has = U[0] > 1e-20
        Up = blk.f["U_plus"]
        Up[0] = np.where(has, u, 0.0)
        Up[1] = np.where(has, v, 0.0)
        Up[2] = np.where(has, w, 0.0)

    def update_magnetic_derived(self):
        """UpdateMagneticDerivedFields_ (LunarSolver_Tools.cpp:149-155)"""
        for blk in self.blocks:
            self.calc_bcell(blk)
        self.sync("B_cell")
        for blk in self.blocks:
            self.curl_adj(blk, ("B_xi", "B_eta", "B_zeta"), ("J_xi", "J_eta", "J_zeta"))
        self.sync("Jedge")
        for blk in self.blocks:
            self.calc_jcell(blk)
        self.sync("J_cell")

    def update_derived(self):
        """UpdateDerivedFields_ (LunarSolver_Tools.cpp:157-161)"""
        self.update_magnetic_derived()
        for blk in self.blocks:
            self.calc_pv_uplus(blk)
        self.sync("Uplus")

    # ---------------------------------------------------------------- time step
    def compute_timestep(self):
        """Compute_Timestep (Z4_Lunar/src/physics/LunarSolver_Timestep.cpp:8-140)"""
        g = self.c["gamma"]
        best = 1e100
        for blk in self.blocks:
            lo, hi = blk.inner(0)
            V = np.abs(blk.box("Jac", 0, lo, hi))
            U = [blk.box("U_H", m, lo, hi) for m in range(5)]
            rho = smax(U[0], 1e-2)
            ux, uy, uz = U[1] / rho, U[2] / rho, U[3] / rho
            ke = 0.5 * rho * (ux * ux + uy * uy + uz * uz)
            p = (g - 1.0) * (U[4] - ke)
            cs2 = g * p / rho
            Bx, By, Bz = (blk.box("B_cell", c, lo, hi) for c in range(3))
            B2 = Bx * Bx + By * By + Bz * Bz
            denom = np.zeros(V.shape)
            for nm, d in (("JDxi", (1, 0, 0)), ("JDet", (0, 1, 0)), ("JDze", (0, 0, 1))):
                for shift, outward in (((0, 0, 0), False), (d, True)):
                    ax, ay, az = (blk.box(nm, c, lo, hi, shift) for c in range(3))
                    A = np.sqrt(ax * ax + ay * ay + az * az)
                    with np.errstate(invalid="ignore", divide="ignore"):
                        nx, ny, nz = ax / A, ay / A, az / A
                    if not outward:
                        nx, ny, nz = -nx, -ny, -nz
                    un = ux * nx + uy * ny + uz * nz
                    Bn = Bx * nx + By * ny + Bz * nz
                    vA2 = self.c["inver_MA2"] * B2 / rho
                    vAn2 = self.c["inver_MA2"] * (Bn * Bn) / rho
                    term = cs2 + vA2
                    disc = term * term - 4.0 * cs2 * vAn2
                    disc = np.where(disc < 0.0, 0.0, disc)
                    cf = np.sqrt(0.5 * (term + np.sqrt(disc)))
                    denom = denom + np.where(A <= 0.0, 0.0, (np.abs(un) + cf) * A)
            ok = (V > 0.0) & (denom > 0.0)
            with np.errstate(invalid="ignore", divide="ignore"):
                dtc = np.where(ok, self.c["cfl"] * V / denom, 1e100)
            best = min(best, float(np.min(dtc)))
        self.dt = best
        return best

    # --------------------------------------------------------------- fluid RHS
    def _face_flux(self, blk, d, lo, hi, shift):
        """Reconstruction_Rusanov on the faces [lo, hi) + shift of direction d
        (Z4_Lunar/src/physics/LunarSolver_FluidRHS.cpp:34-111)"""
        g = self.c["gamma"]
        nm = ("JDxi", "JDet", "JDze")[d]
        e = tuple(-1 if q == d else 0 for q in range(3))
        sL = tuple(a + b for a, b in zip(shift, e))
        k1, k2, k3 = (blk.box(nm, c, lo, hi, shift) for c in range(3))
        rhoL = blk.box("U_H", 0, lo, hi, sL)
        rhoR = blk.box("U_H", 0, lo, hi, shift)
        uL, vL, wL, pL = (blk.box("PV_H", c, lo, hi, sL) for c in range(4))
        uR, vR, wR, pR = (blk.box("PV_H", c, lo, hi, shift) for c in range(4))
        UL = [rhoL, rhoL * uL, rhoL * vL, rhoL * wL, pL / (g - 1.0) + 0.5 * rhoL * (uL * uL + vL * vL + wL * wL)]
        UR = [rhoR, rhoR * uR, rhoR * vR, rhoR * wR, pR / (g - 1.0) + 0.5 * rhoR * (uR * uR + vR * vR + wR * wR)]
        kk = (k1 * k1 + k2 * k2 + k3 * k3)

        def rad(rho, u, v, w, p):
            uvw = k1 * u + k2 * v + k3 * w
            c = np.sqrt(smax(0.0, g * p / smax(rho, 1e-30)))
            return np.abs(uvw) + c * np.sqrt(kk)

        def flux(rho, u, v, w, p):
            uvw = k1 * u + k2 * v + k3 * w
            rhoe = p / (g - 1.0) + 0.5 * rho * (u * u + v * v + w * w)
            return [rho * uvw, rho * uvw * u + k1 * p, rho * uvw * v + k2 * p, rho * uvw * w + k3 * p,
                    uvw * (rhoe + p)]

        r = smax(rad(rhoL, uL, vL, wL, pL), rad(rhoR, uR, vR, wR, pR))
        FL = flux(rhoL, uL, vL, wL, pL)
        FR = flux(rhoR, uR, vR, wR, pR)
        return [0.5 * (FL[m] + FR[m]) - 0.5 * r * (UR[m] - UL[m]) for m in range(5)]

    def fluid_rhs(self):
        """ZeroRHS_ + Scheme_U_ + AddSourceToRHS_Fluid
        (LunarSolver_Advance.cpp:4-59, LunarSolver_FluidRHS.cpp:3-201, :528-568)"""
        c = self.c
        for blk in self.blocks:
            lo, hi = blk.inner(0)
            invJ = 1.0 / blk.box("Jac", 0, lo, hi)
            dF = []
            for d in range(3):
                e = tuple(1 if q == d else 0 for q in range(3))
                Fm = self._face_flux(blk, d, lo, hi, (0, 0, 0))
                Fp = self._face_flux(blk, d, lo, hi, e)
                dF.append([Fp[m] - Fm[m] for m in range(5)])
            R = []
            for m in range(5):
                r = 0.0 - dF[0][m] * invJ
                r = r - dF[1][m] * invJ
                r = r - dF[2][m] * invJ
                R.append(r)
            rho = blk.box("U_H", 0, lo, hi)
            n_true = smax(rho, 0.0) / c["M_H"] * c["M_ref"]
            ne = np.sqrt(n_true * n_true + c["ne_hall_floor"] * c["ne_hall_floor"])
            fc = c["momentum_hall_coeff"] * (n_true / ne)
            Jx, Jy, Jz = (blk.box("J_cell", q, lo, hi) for q in range(3))
            Bx, By, Bz = (blk.box("B_cell", q, lo, hi) for q in range(3))
            jxb = [Jy * Bz - Jz * By, Jz * Bx - Jx * Bz, Jx * By - Jy * Bx]
            PV = [blk.box("PV_H", q, lo, hi) for q in range(3)]
            R[1] = R[1] + fc * jxb[0]
            R[2] = R[2] + fc * jxb[1]
            R[3] = R[3] + fc * jxb[2]
            R[4] = R[4] + fc * (jxb[0] * PV[0] + jxb[1] * PV[1] + jxb[2] * PV[2])
            for m in range(5):
                blk.f["RHS_H"][m][blk.s(lo, hi)] = R[m]

    # ------------------------------------------------------------- induction
    def _ucon(self, blk, axis, lo, hi, d):
        """cell_u_contra (LunarSolver_MagExplicit_Ideal.cpp:95-115) on cells [lo,hi)+d"""
        nm = ("JDxi", "JDet", "JDze")[axis]
        e = tuple(x + (1 if q == axis else 0) for q, x in enumerate(d))
        kx = 0.5 * (blk.box(nm, 0, lo, hi, d) + blk.box(nm, 0, lo, hi, e))
        ky = 0.5 * (blk.box(nm, 1, lo, hi, d) + blk.box(nm, 1, lo, hi, e))
        kz = 0.5 * (blk.box(nm, 2, lo, hi, d) + blk.box(nm, 2, lo, hi, e))
        inv = 1.0 / (np.abs(blk.box("Jac", 0, lo, hi, d)) + 1.0e-30)
        return (kx * blk.box("U_plus", 0, lo, hi, d) + ky * blk.box("U_plus", 1, lo, hi, d)
                + kz * blk.box("U_plus", 2, lo, hi, d)) * inv

    def eface(self, blk):
        """AssembleOneDirectionEMF_ for the three directions (LunarSolver_MagExplicit_Ideal.cpp:348-496)"""
        Bn = ("B_xi", "B_eta", "B_zeta")
        An = ("Badd_xi", "Badd_eta", "Badd_zeta")
        for fa in range(3):
            lo, hi = blk.inner(1 + fa)
            L = tuple(-1 if q == fa else 0 for q in range(3))
            z = (0, 0, 0)
            tot = lambda ax, d: blk.box(Bn[ax], 0, lo, hi, d) + blk.box(An[ax], 0, lo, hi, d)
            ind = lambda ax, d: blk.box(Bn[ax], 0, lo, hi, d)
            bff = tot(fa, z)

            def G(ba):
                e = tuple(1 if q == ba else 0 for q in range(3))
                Le = tuple(a + b for a, b in zip(L, e))
                btL = 0.5 * (tot(ba, L) + tot(ba, Le))
                btR = 0.5 * (tot(ba, z) + tot(ba, e))
                biL = 0.5 * (ind(ba, L) + ind(ba, Le))
                biR = 0.5 * (ind(ba, z) + ind(ba, e))
                ufL = self._ucon(blk, fa, lo, hi, L)
                ufR = self._ucon(blk, fa, lo, hi, z)
                ubL = self._ucon(blk, ba, lo, hi, L)
                ubR = self._ucon(blk, ba, lo, hi, z)
                GL = ufL * btL - ubL * bff
                GR = ufR * btR - ubR * bff
                radius = smax(np.abs(ufL), np.abs(ufR))
                return 0.5 * (GL + GR) - 0.5 * radius * (biR - biL)

            zero = np.zeros(bff.shape)
            if fa == 0:
                e = [zero, G(2), -G(1)]
            elif fa == 1:
                e = [-G(2), zero, G(0)]
            else:
                e = [G(1), -G(0), zero]
            nm = ("Eface_xi", "Eface_eta", "Eface_zeta")[fa]
            for c in range(3):
                blk.f[nm][c][blk.s(lo, hi)] = e[c]

    def eedge(self, blk):
        """AssembleEdgeEMF_FromFaceE_Ideal_ after zeroing E_edge
        (LunarSolver_MagExplicit_Ideal.cpp:53-287, LunarSolver_MagneticRHS.cpp:9-28)"""
        for nm in ("E_xi", "E_eta", "E_zeta"):
            blk.f[nm][:] = 0.0
        C = 0.5
        z = (0, 0, 0)

        def a4(axis, lo, hi, cells):
            a = 0.0
            for d in cells:
                a = smax(a, np.abs(self._ucon(blk, axis, lo, hi, d)))
            return a

        B = lambda nm, lo, hi, d: blk.box(nm, 0, lo, hi, d)
        lo, hi = blk.inner(4)
        Ec = 0.25 * (blk.box("Eface_eta", 0, lo, hi, z) + blk.box("Eface_eta", 0, lo, hi, (0, 0, -1))
                     + blk.box("Eface_zeta", 0, lo, hi, z) + blk.box("Eface_zeta", 0, lo, hi, (0, -1, 0)))
        cells = [z, (0, -1, 0), (0, 0, -1), (0, -1, -1)]
        ae, az = a4(1, lo, hi, cells), a4(2, lo, hi, cells)
        dz = B("B_zeta", lo, hi, z) - B("B_zeta", lo, hi, (0, -1, 0))
        de = B("B_eta", lo, hi, z) - B("B_eta", lo, hi, (0, 0, -1))
        blk.f["E_xi"][0][blk.s(lo, hi)] = Ec + C * (0.5 * ae * dz - 0.5 * az * de)
        lo, hi = blk.inner(5)
        Ec = 0.25 * (blk.box("Eface_xi", 1, lo, hi, z) + blk.box("Eface_xi", 1, lo, hi, (0, 0, -1))
                     + blk.box("Eface_zeta", 1, lo, hi, z) + blk.box("Eface_zeta", 1, lo, hi, (-1, 0, 0)))
        cells = [z, (-1, 0, 0), (0, 0, -1), (-1, 0, -1)]
        az, ax = a4(2, lo, hi, cells), a4(0, lo, hi, cells)
        dx = B("B_xi", lo, hi, z) - B("B_xi", lo, hi, (0, 0, -1))
        dz = B("B_zeta", lo, hi, z) - B("B_zeta", lo, hi, (-1, 0, 0))
        blk.f["E_eta"][0][blk.s(lo, hi)] = Ec + C * (0.5 * az * dx - 0.5 * ax * dz)
        lo, hi = blk.inner(6)
        Ec = 0.25 * (blk.box("Eface_xi", 2, lo, hi, z) + blk.box("Eface_xi", 2, lo, hi, (0, -1, 0))
                     + blk.box("Eface_eta", 2, lo, hi, z) + blk.box("Eface_eta", 2, lo, hi, (-1, 0, 0)))
        cells = [z, (-1, 0, 0), (0, -1, 0), (-1, -1, 0)]
        ax, ae = a4(0, lo, hi, cells), a4(1, lo, hi, cells)
        de = B("B_eta", lo, hi, z) - B("B_eta", lo, hi, (-1, 0, 0))
        dx = B("B_xi", lo, hi, z) - B("B_xi", lo, hi, (0, -1, 0))
        blk.f["E_zeta"][0][blk.s(lo, hi)] = Ec + C * (0.5 * ax * de - 0.5 * ae * dx)

    def curl_e2f(self, blk, fE, fF, mult):
        """CTOperators::CurlEdgeToFace (Z4_Lunar/src/operators/CTOperators.cpp:6-56)"""
        Ex, Ee, Ez = fE
        z = (0, 0, 0)
        for fa, nm in enumerate(fF):
            lo, hi = blk.inner(1 + fa)
            e = lambda f_, d: blk.box(f_, 0, lo, hi, d)
            if fa == 0:
                c = (e(Ee, z) - e(Ee, (0, 0, 1))) + (e(Ez, (0, 1, 0)) - e(Ez, z))
            elif fa == 1:
                c = (e(Ex, (0, 0, 1)) - e(Ex, z)) + (e(Ez, z) - e(Ez, (1, 0, 0)))
            else:
                c = (e(Ex, z) - e(Ex, (0, 1, 0))) + (e(Ee, (1, 0, 0)) - e(Ee, z))
            blk.f[nm][0][blk.s(lo, hi)] = mult * c

    def step(self):
        """One LunarSolver::StepOnce (Z4_Lunar/src/LunarSolver_Driver.cpp:21-92): CFL time step,
        fluid RHS, CT induction, forward-Euler update, the implicit resistive
        solve when it is set up, then the closing syncs and derived fields."""
        self.compute_timestep()
        dt = self.dt
        self.euler_stage(dt)
        self.time += dt
        self.sync("Ucell")
        self.sync("Bface")
        self.update_derived()
        return dt

    STATE = (("U_H", 0, 5), ("B_xi", 1, 1), ("B_eta", 2, 1), ("B_zeta", 3, 1))

    def rk2_step(self):
        """SSP-RK2 (Shu and Osher, 1988) from two StepOnce Euler stages at the
        dt of the step's start (the composition the reference harness's rk2
        command runs with the reference's own stage functions): U1 = U^n +
        dt L(U^n) with the closing syncs and derived fields, U2 = U1 + dt L(U1),
        U^{n+1} = 0.5 (U^n + U2) on the inner cells and faces, then the closing
        syncs and derived fields."""
        self.compute_timestep()
        dt = self.dt
        saved = []
        for blk in self.blocks:
            keep = {}
            for name, loc, nc in self.STATE:
                lo, hi = blk.inner(loc)
                keep[name] = [blk.box(name, m, lo, hi).copy() for m in range(nc)]
            saved.append(keep)
        self.euler_stage(dt)
        self.sync("Ucell")
        self.sync("Bface")
        self.update_derived()
        self.euler_stage(dt)
        for blk, keep in zip(self.blocks, saved):
            for name, loc, nc in self.STATE:
                lo, hi = blk.inner(loc)
                for m in range(nc):
                    blk.f[name][m][blk.s(lo, hi)] = 0.5 * (keep[name][m] + blk.box(name, m, lo, hi))
        self.time += dt
        self.sync("Ucell")
        self.sync("Bface")
        self.update_derived()
        return dt

    def euler_stage(self, dt):
        """The forward-Euler stage of StepOnce at a given dt (fluid RHS, CT
        induction, update, resistive part), without the closing syncs."""
        self.fluid_rhs()
        for blk in self.blocks:
            self.eface(blk)
        self.sync("Eface")
        for blk in self.blocks:
            self.eedge(blk)
        self.sync("Eedge")
        for blk in self.blocks:
            self.curl_e2f(blk, ("E_xi", "E_eta", "E_zeta"), ("RHS_B_xi", "RHS_B_eta", "RHS_B_zeta"), -1.0)
        for blk in self.blocks:
            lo, hi = blk.inner(0)
            for m in range(5):
                blk.f["U_H"][m][blk.s(lo, hi)] += dt * blk.box("RHS_H", m, lo, hi)
            for fa, (bn, rn) in enumerate((("B_xi", "RHS_B_xi"), ("B_eta", "RHS_B_eta"), ("B_zeta", "RHS_B_zeta"))):
                lo, hi = blk.inner(1 + fa)
                blk.f[bn][0][blk.s(lo, hi)] += dt * blk.box(rn, 0, lo, hi)
        if self.resist is not None:
            self.resistive_step()
        elif self.explicit is not None:
            self.resistive_subcycles()

    # ------------------------------------------------------ implicit resistivity
    def set_resistive(self, unknowns, eta, alias, owner, sign):
        """Unknown edges (block, dir, i, j, k) with dir 1/2/3 = xi/eta/zeta in solve order and their
        resistivity (BuildImplicitResistiveEdgeDofMap_, Z4_Lunar/src/implicit/Lunar_ImplicitResistive.cpp:147-164),
        and the edge alias -> owner table with orientation signs (HALO_OWNER::sync_edge_1form)."""
        self.resist = dict(u=np.asarray(unknowns), eta=np.asarray(eta, dtype=np.float64), alias=np.asarray(alias),
                           owner=np.asarray(owner), sign=np.asarray(sign, dtype=np.float64))

    resist = None
    EDGE3 = {1: "_xi", 2: "_eta", 3: "_zeta"}

    def _edge_get(self, prefix, rows):
        out = np.empty(len(rows))
        for d in (1, 2, 3):
            sel = rows[:, 1] == d
            for b in np.unique(rows[sel, 0]):
                s2 = sel & (rows[:, 0] == b)
                blk = self.blocks[int(b)]
                G = blk.G
                out[s2] = blk.f[prefix + self.EDGE3[d]][0][rows[s2, 2] + G, rows[s2, 3] + G, rows[s2, 4] + G]
        return out

    def _edge_set(self, prefix, rows, vals):
        for d in (1, 2, 3):
            sel = rows[:, 1] == d
            for b in np.unique(rows[sel, 0]):
                s2 = sel & (rows[:, 0] == b)
                blk = self.blocks[int(b)]
                G = blk.G
                blk.f[prefix + self.EDGE3[d]][0][rows[s2, 2] + G, rows[s2, 3] + G, rows[s2, 4] + G] = vals[s2]

    def _alias(self, prefix):
        R = self.resist
        if len(R["alias"]):
            self._edge_set(prefix, R["alias"], R["sign"] * self._edge_get(prefix, R["owner"]))

    def _clear(self, prefix):
        for blk in self.blocks:
            for sfx in ("_xi", "_eta", "_zeta"):
                blk.f[prefix + sfx][:] = 0.0

    def _unpack(self, x):
        """UnpackVecToImplicitEres_ (Lunar_ImplicitResistive.cpp:332-360)"""
        self._clear("Eres")
        self._edge_set("Eres", self.resist["u"], x)
        self._alias("Eres")
        self.sync("Eres1form")

    def resistive_matvec(self, x):
        """MatMultImplicitResistive_ (Lunar_ImplicitResistive.cpp:380-427):
        y = x - eta * alpha curlAdj(beta (-dt) curl(x))."""
        self._unpack(x)
        self._clear("dB")
        for blk in self.blocks:
            self.curl_e2f(blk, ("Eres_xi", "Eres_eta", "Eres_zeta"), ("dB_xi", "dB_eta", "dB_zeta"), -self.dt)
        self.sync("dB")
        self._clear("dJ")
        for blk in self.blocks:
            self.curl_adj(blk, ("dB_xi", "dB_eta", "dB_zeta"), ("dJ_xi", "dJ_eta", "dJ_zeta"))
        self._alias("dJ")
        R = self.resist
        return self._edge_get("Eres", R["u"]) - R["eta"] * self._edge_get("dJ", R["u"])

    def resistive_step(self):
        """SolveImplicitResistiveDiffusion_ + ApplyImplicitResistiveUpdate_
        (Lunar_ImplicitResistive.cpp:430-518).  The linear system is solved
        directly (dense LU over the operator's columns) instead of by GMRES:
        the result is the exact solution the Krylov solve approaches to its
        tolerance, so it checks a GMRES solution to that tolerance."""
        R = self.resist
        self.sync("Bface")
        self.sync("Bface")
        for blk in self.blocks:
            self.curl_adj(blk, ("B_xi", "B_eta", "B_zeta"), ("J_xi", "J_eta", "J_zeta"))
        self.sync("Jedge")
        n = len(R["u"])
        if n:
            b = 0.0 + R["eta"] * self._edge_get("J", R["u"])
            A = np.empty((n, n))
            e = np.zeros(n)
            for q in range(n):
                e[q] = 1.0
                A[:, q] = self.resistive_matvec(e)
                e[q] = 0.0
            x = np.linalg.solve(A, b)
            self.resist_last = dict(b=b, x=x, A=A)
        else:
            x = np.zeros(0)
        self._unpack(x)
        self.sync("Eres1form")
        self._clear("RHS_Bres")
        for blk in self.blocks:
            self.curl_e2f(blk, ("Eres_xi", "Eres_eta", "Eres_zeta"), ("RHS_Bres_xi", "RHS_Bres_eta", "RHS_Bres_zeta"),
                          -1.0)
            for fa, (bn, rn) in enumerate((("B_xi", "RHS_Bres_xi"), ("B_eta", "RHS_Bres_eta"),
                                           ("B_zeta", "RHS_Bres_zeta"))):
                lo, hi = blk.inner(1 + fa)
                blk.f[bn][0][blk.s(lo, hi)] += self.dt * blk.box(rn, 0, lo, hi)
        self.sync("Bface")

    # ------------------------------------------------------- divB diagnostic
    def calc_divb(self):
        """calc_divB without Pole patches (Z4_Lunar/src/physics/LunarSolver_Tools.cpp:685-775)"""
        for blk in self.blocks:
            lo, hi = blk.inner(0)
            z = (0, 0, 0)
            bx = lambda d: blk.box("B_xi", 0, lo, hi, d)
            be = lambda d: blk.box("B_eta", 0, lo, hi, d)
            bz = lambda d: blk.box("B_zeta", 0, lo, hi, d)
            num = bx((1, 0, 0)) - bx(z) + be((0, 1, 0)) - be(z) + bz((0, 0, 1)) - bz(z)
            blk.f["divB"][0][blk.s(lo, hi)] = num / blk.box("Jac", 0, lo, hi)

    # ------------------------------------------------------- diagnostics
    def minmax_diagnostics(self):
        """PrintMinMaxDiagnostics_ (Z4_Lunar/src/tools/LunarSolver_PrintDiag.cpp:7-85):
        over the inner cells of every block the minima of rho, p, Bx, By, Bz,
        |B|^2 / 2 and their maxima plus max |divB| (std::min / std::max skip
        NaN).  Returns (mins[6], maxs[7])."""
        mins = [np.inf] * 6
        maxs = [-np.inf] * 6 + [0.0]
        for blk in self.blocks:
            lo, hi = blk.inner(0)
            bx, by, bz = (blk.box("B_cell", c, lo, hi) for c in range(3))
            vals = [blk.box("U_H", 0, lo, hi), blk.box("PV_H", 3, lo, hi), bx, by, bz,
                    0.5 * (bx * bx + by * by + bz * bz)]
            for q, v in enumerate(vals):
                v = v[~np.isnan(v)]
                if v.size:
                    mins[q] = min(mins[q], float(v.min()))
                    maxs[q] = max(maxs[q], float(v.max()))
            d = np.abs(blk.box("divB", 0, lo, hi))
            d = d[~np.isnan(d)]
            if d.size:
                maxs[6] = max(maxs[6], float(d.max()))
        return mins, maxs

    @staticmethod
    def format_diagnostics(mins, maxs):
        """the three lines PrintMinMaxDiagnostics_ prints"""
        b_abs_max = np.sqrt(max(0.0, 2.0 * maxs[5]))
        return ["           rho=[%.3e, %.3e]  p=[%.3e, %.3e]" % (mins[0], maxs[0], mins[1], maxs[1]),
                "           Bx =[%.3e, %.3e]  By=[%.3e, %.3e]  Bz=[%.3e, %.3e]" % (mins[2], maxs[2], mins[3],
                                                                                  maxs[3], mins[4], maxs[4]),
                "           Pmag=[%.3e, %.3e]  |B|max=%.3e  divB_max=%.3e" % (mins[5], maxs[5], b_abs_max, maxs[6])]

    # ------------------------------------------------ explicit resistivity
    explicit = None

    def set_explicit_resistive(self, nodes, inver_Rem, nsub):
        """ResistiveDiffusionSubcycles_ set-up: edge-midpoint radii of the inner
        edges from the node coordinates (per block a (ni+1, nj+1, nk+1, 3)
        array of the inner nodes) and the tanh shell profile yita0
        (Z4_Lunar/src/physics/LunarSolver_MagExplicit_Resis.cpp:72-88, 160-167)."""
        import math
        prof = []
        for blk, X in zip(self.blocks, nodes):
            per = []
            for ea, (di, dj, dk) in enumerate(((1, 0, 0), (0, 1, 0), (0, 0, 1))):
                lo, hi = blk.inner(4 + ea)
                p0 = X[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]]
                p1 = X[lo[0] + di:hi[0] + di, lo[1] + dj:hi[1] + dj, lo[2] + dk:hi[2] + dk]
                xm, ym, zm = (0.5 * (p0[..., c] + p1[..., c]) for c in range(3))
                r = np.sqrt(xm * xm + ym * ym + zm * zm)
                y = np.zeros(r.shape)
                for idx in zip(*np.nonzero((r > 0.84) & (r < 1.04))):
                    rr = float(r[idx])
                    y[idx] = 0.5 * (math.tanh((rr - 0.84) / 0.02) - math.tanh((rr - 1.04) / 0.02))
                per.append(y)
            prof.append(per)
        self.explicit = dict(yita0=prof, inver_Rem=float(inver_Rem), nsub=max(1, int(nsub)))

    def eres_explicit(self, blk, yita0):
        """AddResistiveEdgeEMF_To_ on zeroed Eres (LunarSolver_MagExplicit_Resis.cpp:67-209)"""
        cells = {0: [(0, 0, 0), (0, -1, 0), (0, 0, -1), (0, -1, -1)],
                 1: [(0, 0, 0), (-1, 0, 0), (0, 0, -1), (-1, 0, -1)],
                 2: [(0, 0, 0), (-1, 0, 0), (0, -1, 0), (-1, -1, 0)]}
        for ea, (en, dn) in enumerate((("Eres_xi", "dr_xi"), ("Eres_eta", "dr_eta"), ("Eres_zeta", "dr_zeta"))):
            lo, hi = blk.inner(4 + ea)
            J = [0.0, 0.0, 0.0]
            for d in cells[ea]:
                for c in range(3):
                    J[c] = J[c] + blk.box("J_cell", c, lo, hi, d)
            J = [x * 0.25 for x in J]
            Jedge = J[0] * blk.box(dn, 0, lo, hi) + J[1] * blk.box(dn, 1, lo, hi) + J[2] * blk.box(dn, 2, lo, hi)
            y = yita0[ea]
            with np.errstate(invalid="ignore"):
                val = 0.0 + (self.explicit["inver_Rem"] * y) * Jedge
            blk.f[en][0][blk.s(lo, hi)] = np.where(y == 0.0, 0.0, val)

    def resistive_subcycles(self):
        """ResistiveDiffusionSubcycles_ (Z4_Lunar/src/physics/LunarSolver_MagneticRHS.cpp:53-115)"""
        nsub = self.explicit["nsub"]
        dt_res = self.dt / float(nsub)
        for _ in range(nsub):
            self.sync("Bface")
            self.update_magnetic_derived()
            self._clear("Eres")
            self._clear("RHS_Bres")
            for blk, y in zip(self.blocks, self.explicit["yita0"]):
                self.eres_explicit(blk, y)
            self.sync("Eres")
            for blk in self.blocks:
                self.curl_e2f(blk, ("Eres_xi", "Eres_eta", "Eres_zeta"),
                              ("RHS_Bres_xi", "RHS_Bres_eta", "RHS_Bres_zeta"), -1.0)
                for fa, (bn, rn) in enumerate((("B_xi", "RHS_Bres_xi"), ("B_eta", "RHS_Bres_eta"),
                                               ("B_zeta", "RHS_Bres_zeta"))):
                    lo, hi = blk.inner(1 + fa)
                    blk.f[bn][0][blk.s(lo, hi)] += dt_res * blk.box(rn, 0, lo, hi)
            self.sync("Bface")

    # ------------------------------------------------------------ Hall EMF
    @staticmethod
    def hall_zero_boxes(n, patches):
        """Edge boxes (axis, lo, hi) that BuildHallFaceEMF_Rusanov_diff_ zeroes
        (Z4_Lunar/src/physics/LunarSolver_MagExplicit_Hall.cpp:300-450): the
        node box of every Solid_Surface patch widened 20 layers inwards, and
        of every Pole patch, turned into edge boxes and clipped to the inner
        edges.  patches: (bc name, direction, node lo, node hi)."""
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
                plus = PLUS[4 + ea]
                lo = [max(lo[a], 0) for a in range(3)]
                hi = [min(hi[a], n[a] + plus[a]) for a in range(3)]
                if all(lo[a] < hi[a] for a in range(3)):
                    out.append((ea, tuple(lo), tuple(hi)))
        return out

    def hall_emf(self, blk, hall_coef, zero_boxes=()):
        """BuildHallFaceEMF_Rusanov_diff_ (Z4_Lunar/src/physics/LunarSolver_MagExplicit_Hall.cpp:8-457):
        Ehc = alpha (J x B) and beta = |alpha| |B| on every cell of the array
        (alpha = hall_coef / ne_eff of Hall_Num_Limiter), then per inner edge the
        4-cell mean of Ehc along dr minus the whistler diffusion of the face-B
        jumps, zeroed in zero_boxes."""
        c = self.c
        G = blk.G
        ng = FIELDS["B_cell"][2]
        n = blk.n
        lo, hi = (-ng, -ng, -ng), (n[0] + ng, n[1] + ng, n[2] + ng)
        rho = blk.box("U_H", 0, lo, hi)
        n_true = smax(rho, 0.0) / c["M_H"] * c["M_ref"]
        ne = np.sqrt(n_true * n_true + c["ne_hall_floor"] * c["ne_hall_floor"])
        alpha = hall_coef / ne
        Jx, Jy, Jz = (blk.box("J_cell", q, lo, hi) for q in range(3))
        Bx, By, Bz = (blk.box("B_cell", q, lo, hi) for q in range(3))
        shape = blk.f["B_cell"][0].shape
        Ehc = np.zeros((3,) + shape)
        beta = np.zeros(shape)
        sl = blk.s(lo, hi)
        Ehc[0][sl] = alpha * (Jy * Bz - Jz * By)
        Ehc[1][sl] = alpha * (Jz * Bx - Jx * Bz)
        Ehc[2][sl] = alpha * (Jx * By - Jy * Bx)
        beta[sl] = np.abs(alpha) * np.sqrt(Bx * Bx + By * By + Bz * Bz)
        eps, Cwh = 1e-14, 0.1
        # per edge axis: the 4 cells, the two transverse axes (t1, t2) and
        # the face areas that give h_t1 and h_t2
        spec = {0: ([(0, -1, -1), (0, -1, 0), (0, 0, -1), (0, 0, 0)], "B_zeta", (0, -1, 0), "B_eta", (0, 0, -1),
                    "Area_zeta", (0, -1, 0), "Area_eta", (0, 0, -1), "dl_xi", "dr_xi"),
                1: ([(-1, 0, -1), (-1, 0, 0), (0, 0, -1), (0, 0, 0)], "B_xi", (0, 0, -1), "B_zeta", (-1, 0, 0),
                    "Area_xi", (0, 0, -1), "Area_zeta", (-1, 0, 0), "dl_eta", "dr_eta"),
                2: ([(-1, -1, 0), (-1, 0, 0), (0, -1, 0), (0, 0, 0)], "B_eta", (-1, 0, 0), "B_xi", (0, -1, 0),
                    "Area_eta", (-1, 0, 0), "Area_xi", (0, -1, 0), "dl_zeta", "dr_zeta")}
        for ea in range(3):
            cells, Bm, dm, Bp, dp, Am, dAm, Ap, dAp, dln, drn = spec[ea]
            elo, ehi = blk.inner(4 + ea)
            cbox = lambda arr, d: arr[blk.sh(elo, ehi, d)]
            Ec = []
            for q in range(3):
                a, b_, c2, d2 = (cbox(Ehc[q], d) for d in cells)
                Ec.append(0.25 * (a + b_ + c2 + d2))
            Ecen = Ec[0] * blk.box(drn, 0, elo, ehi) + Ec[1] * blk.box(drn, 1, elo, ehi) + Ec[2] * blk.box(drn, 2, elo, ehi)
            b0, b1, b2, b3 = (cbox(beta, d) for d in cells)
            beta_e = smax(smax(b0, b1), smax(b2, b3))
            L = smax(blk.box(dln, 0, elo, ehi), eps)
            z = (0, 0, 0)
            Abar_m = 0.5 * (blk.box(Am, 0, elo, ehi) + blk.box(Am, 0, elo, ehi, dAm))
            inv_m = L / smax(Abar_m, eps)
            mu_m = Cwh * beta_e * inv_m * inv_m
            Abar_p = 0.5 * (blk.box(Ap, 0, elo, ehi) + blk.box(Ap, 0, elo, ehi, dAp))
            inv_p = L / smax(Abar_p, eps)
            mu_p = Cwh * beta_e * inv_p * inv_p
            dB_m = blk.box(Bm, 0, elo, ehi) - blk.box(Bm, 0, elo, ehi, dm)
            dB_p = blk.box(Bp, 0, elo, ehi) - blk.box(Bp, 0, elo, ehi, dp)
            E = Ecen - 0.5 * mu_m * dB_m + 0.5 * mu_p * dB_p
            name = ("Ehall_xi", "Ehall_eta", "Ehall_zeta")[ea]
            blk.f[name][0][blk.s(elo, ehi)] = E
            for (za, zlo, zhi) in zero_boxes:
                if za == ea:
                    blk.f[name][0][blk.s(zlo, zhi)] = 0.0


# ---------------------------------------------------------------------------
# The single-block spherical shell: Solid_Surface (i min) and Farfield (i max)
# in r, Pole patches at both ends of theta (j), phi (k) periodic onto itself
# ---------------------------------------------------------------------------

def _solve3_gj(A, b):
    """Gauss-Jordan elimination with partial pivoting on [A | b], the 3x3 solve
    of the reference's Pole handlers and repairs (Z4_Lunar/src/boundary/
    Boundary_Condition.cpp:244-292, Boundary_Condition_EM.cpp:107-165,
    Z4_Lunar/src/physics/LunarSolver_Tools.cpp:894-944); None when a pivot
    falls below 1e-300."""
    M = [[A[r][0], A[r][1], A[r][2], b[r]] for r in range(3)]
    for c in range(3):
        piv = c
        amax = abs(M[c][c])
        for r0 in range(c + 1, 3):
            av = abs(M[r0][c])
            if av > amax:
                amax = av
                piv = r0
        if amax < 1.0e-300:
            return None
        if piv != c:
            for q in range(c, 4):
                M[c][q], M[piv][q] = M[piv][q], M[c][q]
        inv = 1.0 / M[c][c]
        for q in range(c, 4):
            M[c][q] *= inv
        for r0 in range(3):
            if r0 == c:
                continue
            fac = M[r0][c]
            for q in range(c, 4):
                M[r0][q] -= fac * M[c][q]
    return [M[0][3], M[1][3], M[2][3]]


def _cmax(a, b):
    """std::max(a, b) on scalars"""
    return b if a < b else a


class ShellOracle(Oracle):
    """The oracle on one spherical-shell block.  Sync(group) runs the
    reference's handlers in place, in the reference's order
    (Z4_Lunar/src/boundary/Boundary_Sync_.cpp:4-65): per field the physical
    handlers of the topology's patches (Pole j min, Pole j max, Farfield,
    Solid_Surface; Z4_Lunar/src/boundary/Boundary_Build.cpp:5-271 names the
    handler of every field and patch), the corner default where a wall meets
    a Pole (src/6_boundary/Boundary.cpp:178-260), then the periodic halo in k.
    The derived-field pass adds the reference's Pole repairs: the B_zeta flux
    rewrite after Sync("B_cell"), the least-squares J_cell of the pole shell
    and the divB zeroing next to the Poles.  resistive: the handlers the
    reference registers when is_Lunar_resistance is set (the Solid_Surface
    handlers of J_cell, Eface and the edge EMF, Boundary_Build.cpp:93-163)
    and the Eres groups with their Pole handlers (Boundary_Build.cpp:208-239)."""

    POLES = (-1, +1)  # j min (direction -2), j max (direction +2)

    def __init__(self, ncell, consts, nodes, qinf, B_imf, resistive=False, G=4):
        super().__init__([ncell], consts, G)
        self.resistive = bool(resistive)
        self.nodes = nodes      # Padded ghost node mesh (..., 3) of the block
        self.qinf = np.asarray(qinf, dtype=np.float64)
        self.B_imf = np.asarray(B_imf, dtype=np.float64)
        u = [qinf[1] / qinf[0], qinf[2] / qinf[0], qinf[3] / qinf[0]]
        # BC_Farfield_Eedge_set_zerocurl (Boundary_Condition.cpp:559-600): E_inf = -u_inf x B_imf
        self.E_inf = [B_imf[1] * u[2] - B_imf[2] * u[1], B_imf[2] * u[0] - B_imf[0] * u[2],
                      B_imf[0] * u[1] - B_imf[1] * u[0]]

    # ------------------------------------------------------------ helpers
    def _ih(self, name):
        p = PLUS[FIELDS[name][0]]
        n = self.blocks[0].n
        return (n[0] + p[0], n[1] + p[1], n[2] + p[2])

    def _at(self, name, i, j, k, m=0):
        blk = self.blocks[0]
        G = blk.G
        return float(blk.f[name][m][i + G, j + G, k + G])

    def _put(self, name, i, j, k, m, v):
        blk = self.blocks[0]
        G = blk.G
        blk.f[name][m][i + G, j + G, k + G] = v

    def _slab(self, name, axis, side):
        """(index of the inner slab along axis, slices of the tangential inner range)"""
        ih = self._ih(name)
        G = self.blocks[0].G
        ref = 0 if side < 0 else ih[axis] - 1
        tang = [slice(G, G + ih[a]) for a in range(3)]
        return ref, tang

    def _copy_ghosts(self, name, axis, side):
        """DefaultPhysicalCopy (src/6_boundary/Boundary.cpp:303-332): every ghost
        layer of the slab takes the first inner layer."""
        blk = self.blocks[0]
        G = blk.G
        ng = FIELDS[name][2]
        ref, t = self._slab(name, axis, side)
        src = list(t)
        src[axis] = ref + G
        for g in range(1, ng + 1):
            dst = list(t)
            dst[axis] = ref + side * g + G
            blk.f[name][(slice(None),) + tuple(dst)] = blk.f[name][(slice(None),) + tuple(src)]

    def _set_ghosts(self, name, axis, side, vals):
        blk = self.blocks[0]
        G = blk.G
        ng = FIELDS[name][2]
        ref, t = self._slab(name, axis, side)
        for g in range(1, ng + 1):
            dst = list(t)
            dst[axis] = ref + side * g + G
            for m, v in enumerate(vals):
                blk.f[name][(m,) + tuple(dst)] = v

    def _zero_slab(self, name, axis, side, layers=1):
        blk = self.blocks[0]
        G = blk.G
        ref, t = self._slab(name, axis, side)
        for q in range(layers):
            dst = list(t)
            dst[axis] = ref - side * q + G
            blk.f[name][(slice(None),) + tuple(dst)] = 0.0

    # ------------------------------------------------------- Pole handlers
    def _pole(self, name, side):
        """The Pole handler of a field (Boundary_Build.cpp:27-269)."""
        if name == "U_plus":
            return
        if name == "U_H":
            self._pole_cell(side)
        elif name in ("B_cell", "Bind_cell"):
            self._pole_bcell(name, side)
        elif name == "B_xi":
            self._pole_ring_average("B_xi", side)
        elif name == "B_eta":
            self._zero_slab("B_eta", 1, side)
        elif name == "E_xi":
            self._pole_eedge_axis(side)
        elif name in ("E_eta", "Eres_eta"):
            self._pole_eedge_regulate(side, name=name)
            return
        elif name in ("E_zeta", "J_xi", "J_zeta", "Eres_xi", "Eres_zeta"):
            # BC_Pole_Eedge_Zero_Rotate (Boundary_Condition.cpp:165-177); on an
            # eta Pole Eres_xi takes it too (Boundary_Build.cpp:208-216)
            self._zero_slab(name, 1, side)
        elif name == "J_eta":
            self._pole_jedge_regulate(side)
            return
        self._copy_ghosts(name, 1, side)

    def _pole_cell(self, side):
        """BC_Pole_Cell_ (Z4_Lunar/src/boundary/Boundary_Condition_Fluid.cpp:186-219):
        the first cell layer at the pole becomes its average over k (summed in
        k order, divided by the count)."""
        self._pole_ring_average("U_H", side)

    def _pole_ring_average(self, name, side):
        """k-ring average of the inner slab (BC_Pole_Cell_ and the axis-face
        branch of BC_Pole_Bface_Collapse_, Boundary_Condition_EM.cpp:620-670)"""
        blk = self.blocks[0]
        G = blk.G
        ih = self._ih(name)
        j = (0 if side < 0 else ih[1] - 1) + G
        I = slice(G, G + ih[0])
        for m in range(FIELDS[name][1]):
            acc = np.zeros(ih[0])
            for k in range(ih[2]):
                acc = acc + blk.f[name][m][I, j, G + k]
            avg = acc / float(ih[2])
            blk.f[name][m][I, j, G:G + ih[2]] = avg[:, None]

    def _pole_bcell(self, name, side):
        """BC_Pole_Bcell_Collapse_ for an eta Pole (Boundary_Condition_EM.cpp:3-380):
        per ring the cell vector that best reproduces, in least squares, the
        fluxes of the outer eta face and the two xi faces of every cell of the
        ring (the total fields add Badd), written to the whole ring."""
        total = name == "B_cell"
        n = self.blocks[0].n
        j0 = 0 if side < 0 else n[1] - 1
        jn = j0 + 1 if side < 0 else j0
        sn = 1.0 if side < 0 else -1.0

        def face(F, Fa, i, j, k):
            v = self._at(F, i, j, k)
            if total:
                v += self._at(Fa, i, j, k)
            return v

        for i in range(n[0]):
            M = [[0.0] * 3 for _ in range(3)]
            b = [0.0, 0.0, 0.0]

            def push(S, phi):
                sn2 = S[0] * S[0] + S[1] * S[1] + S[2] * S[2]
                if sn2 <= 1.0e-300:
                    return
                for a in range(3):
                    b[a] += phi * S[a]
                    for c in range(3):
                        M[a][c] += S[a] * S[c]

            for k in range(n[2]):
                push([sn * self._at("JDet", i, jn, k, m) for m in range(3)], sn * face("B_eta", "Badd_eta", i, jn, k))
                push([-self._at("JDxi", i, j0, k, m) for m in range(3)], -face("B_xi", "Badd_xi", i, j0, k))
                push([self._at("JDxi", i + 1, j0, k, m) for m in range(3)], face("B_xi", "Badd_xi", i + 1, j0, k))
            tr = abs(M[0][0]) + abs(M[1][1]) + abs(M[2][2])
            reg = 1.0e-12 * _cmax(1.0, tr)
            for a in range(3):
                M[a][a] += reg
            Bp = _solve3_gj(M, b)
            if Bp is None:
                continue
            for k in range(n[2]):
                for m in range(3):
                    self._put(name, i, j0, k, m, Bp[m])

    def _pole_eedge_axis(self, side):
        """BC_Pole_Eedge_Axis for E_xi on an eta Pole (Boundary_Condition.cpp:27-164):
        E = -u_plus x B_cell of the first cell layer, projected on dr_xi."""
        ih = self._ih("E_xi")
        j = 0 if side < 0 else ih[1] - 1
        jc = j if side < 0 else j - 1
        for i in range(ih[0]):
            for k in range(ih[2]):
                ux, uy, uz = (self._at("U_plus", i, jc, k, m) for m in range(3))
                Bx, By, Bz = (self._at("B_cell", i, jc, k, m) for m in range(3))
                E = [-(uy * Bz - uz * By), -(uz * Bx - ux * Bz), -(ux * By - uy * Bx)]
                dl = [self._at("dr_xi", i, j, k, m) for m in range(3)]
                self._put("E_xi", i, j, k, 0, E[0] * dl[0] + E[1] * dl[1] + E[2] * dl[2])

    def _pole_eedge_regulate(self, side, ghosts=True, name="E_eta"):
        """BC_Pole_Eedge_RegulateK_Norm for E_eta (or Eres_eta) on an eta Pole
        (Boundary_Condition.cpp:179-477): per ring the Cartesian vector whose
        projections best reproduce the edge values (k = n_k excluded: it is
        k = 0), projected back onto every edge; then the ghost copy."""
        ih = self._ih(name)
        j = 0 if side < 0 else ih[1] - 1
        for i in range(ih[0]):
            A = [[0.0] * 3 for _ in range(3)]
            b = [0.0, 0.0, 0.0]
            cnt = 0
            for k in range(ih[2] - 1):
                dl = [self._at("dr_eta", i, j, k, m) for m in range(3)]
                L = np.sqrt(dl[0] * dl[0] + dl[1] * dl[1] + dl[2] * dl[2])
                if L < 1.0e-14:
                    continue
                invL = 1.0 / L
                tau = [dl[0] * invL, dl[1] * invL, dl[2] * invL]
                y = self._at(name, i, j, k) * invL
                for a in range(3):
                    b[a] += y * tau[a]
                    for c in range(3):
                        A[a][c] += tau[a] * tau[c]
                cnt += 1
            if cnt <= 0:
                for k in range(ih[2]):
                    self._put(name, i, j, k, 0, 0.0)
                continue
            trA = A[0][0] + A[1][1] + A[2][2]
            reg = 1.0e-12 * _cmax(1.0, trA)
            for a in range(3):
                A[a][a] += reg
            Ev = _solve3_gj(A, b)
            if Ev is None:
                avg = 0.0
                for k in range(ih[2]):
                    avg += self._at(name, i, j, k)
                avg /= float(ih[2])
                for k in range(ih[2]):
                    self._put(name, i, j, k, 0, avg)
                continue
            for k in range(ih[2]):
                dl = [self._at("dr_eta", i, j, k, m) for m in range(3)]
                L = np.sqrt(dl[0] * dl[0] + dl[1] * dl[1] + dl[2] * dl[2])
                v = 0.0 if L < 1.0e-14 else Ev[0] * dl[0] + Ev[1] * dl[1] + Ev[2] * dl[2]
                self._put(name, i, j, k, 0, v)
        if ghosts:
            self._copy_ghosts(name, 1, side)

    def _pole_jedge_regulate(self, side, ghosts=True):
        """BC_Pole_Jedge_RegulateK_Norm for J_eta on an eta Pole
        (Boundary_Condition.cpp:478-548): the circulation of beta_zeta B_zeta
        around the dual edge times dl_eta / Astar_eta; the ghost slab is zeroed."""
        blk = self.blocks[0]
        G = blk.G
        ih = self._ih("J_eta")
        j = 0 if side < 0 else ih[1] - 1
        lo, hi = (0, j, 0), (ih[0], j + 1, ih[2])
        bz = lambda d: blk.box("beta_zeta", 0, lo, hi, d) * blk.box("B_zeta", 0, lo, hi, d)
        circ = bz((-1, 0, 0)) - bz((0, 0, 0))
        Ast = blk.box("Astar_eta", 0, lo, hi)
        dl = blk.box("dl_eta", 0, lo, hi)
        with np.errstate(divide="ignore", invalid="ignore"):
            v = np.where(np.abs(Ast) <= 1.0e-300, 0.0, (dl / Ast) * circ)
        blk.f["J_eta"][0][blk.s(lo, hi)] = v
        if ghosts:
            self._set_ghosts("J_eta", 1, side, [0.0])

    def pole_rings(self, group):
        """Only the values the Pole handlers of a group compute on the first
        inner layer (both Poles), none of their copies or zeros."""
        for side in self.POLES:
            if group == "Ucell":
                self._pole_cell(side)
            elif group == "Bface":
                self._pole_ring_average("B_xi", side)
            elif group == "B_cell":
                self._pole_bcell("B_cell", side)
                self._pole_bcell("Bind_cell", side)
            elif group == "Eedge":
                self._pole_eedge_axis(side)
                self._pole_eedge_regulate(side, ghosts=False)
            elif group == "Jedge":
                self._pole_jedge_regulate(side, ghosts=False)
            elif group in ("Eres", "Eres1form"):
                self._pole_eedge_regulate(side, ghosts=False, name="Eres_eta")

    # -------------------------------------------- Farfield / Solid_Surface
    def _farfield(self, name):
        """Farfield handler (i max) of the non-resistive set-up (Boundary_Build.cpp:5-271)."""
        if name in ("U_plus", "B_xi", "B_eta", "B_zeta", "Eface_xi", "Eface_eta", "Eface_zeta"):
            return
        if name == "U_H":
            self._set_ghosts("U_H", 0, +1, self.qinf)       # BC_UH_Farfield_H_
        elif name == "B_cell":
            self._set_ghosts("B_cell", 0, +1, self.B_imf)   # BC_Farfield_Bface
        elif name == "Bind_cell":
            self._set_ghosts("Bind_cell", 0, +1, [0.0, 0.0, 0.0])
        elif name in ("E_xi", "E_eta", "E_zeta"):
            # BC_Farfield_Eedge_set_zerocurl: slab <- E_inf . (x(edge end) - x(edge start)), then copy
            blk = self.blocks[0]
            G = blk.G
            ih = self._ih(name)
            d = {"E_xi": (1, 0, 0), "E_eta": (0, 1, 0), "E_zeta": (0, 0, 1)}[name]
            i = ih[0] - 1
            X, o = self.nodes.a, self.nodes.off
            p0 = X[i + o, o:o + ih[1], o:o + ih[2]]
            p1 = X[i + d[0] + o, o + d[1]:o + d[1] + ih[1], o + d[2]:o + d[2] + ih[2]]
            E = self.E_inf
            blk.f[name][0][i + G, G:G + ih[1], G:G + ih[2]] = (E[0] * (p1[..., 0] - p0[..., 0])
                                                               + E[1] * (p1[..., 1] - p0[..., 1])
                                                               + E[2] * (p1[..., 2] - p0[..., 2]))
            self._copy_ghosts(name, 0, +1)
        else:
            self._copy_ghosts(name, 0, +1)

    def _solid(self, name):
        """Solid_Surface handler (i min).  With resistivity the reference
        registers no J_cell or edge-EMF handler there (the default copy runs)
        and zeroes only the Eface ghosts (with the normal field's wall layer)."""
        if name == "U_plus" or (name in ("E_xi", "E_eta", "E_zeta") and not self.resistive):
            return
        if name == "U_H":
            self.wall_u(0, -1)                  # BC_Solid_Surface_
            return
        if name.startswith("Eface_") and self.resistive:
            # BC_Solid_Surface_Eface_ghots_zero (Boundary_Condition_EM.cpp)
            if name == "Eface_xi":
                self._zero_slab(name, 0, -1)
            self._set_ghosts(name, 0, -1, [0.0, 0.0, 0.0])
            return
        if name == "J_cell" and not self.resistive:
            self._zero_slab("J_cell", 0, -1, layers=2)   # BC_Solid_Surface_Jcell (EM.cpp:382-427)
        elif name.startswith("Eface_"):
            self._zero_slab(name, 0, -1)        # BC_Solid_Surface_Eface_ (EM.cpp:787-803)
        self._copy_ghosts(name, 0, -1)

    def _corner_default(self, name):
        """ApplyPhysicalCornerDefault on the four wall/Pole edges along k."""
        blk = self.blocks[0]
        G = blk.G
        ng = FIELDS[name][2]
        ih = self._ih(name)
        K = slice(G, G + ih[2])
        for ig in list(range(-ng, 0)) + list(range(ih[0], ih[0] + ng)):
            for jg in list(range(-ng, 0)) + list(range(ih[1], ih[1] + ng)):
                ic = min(max(ig, 0), ih[0] - 1)
                jc = min(max(jg, 0), ih[1] - 1)
                blk.f[name][:, ig + G, jg + G, K] = blk.f[name][:, ic + G, jc + G, K]

    def _halo_k(self, name):
        """The block's periodic halo in k: a ghost plane takes plane k mod n_k."""
        blk = self.blocks[0]
        G = blk.G
        ng = FIELDS[name][2]
        ih = self._ih(name)
        nk = blk.n[2]
        for kg in list(range(-ng, 0)) + list(range(ih[2], ih[2] + ng)):
            blk.f[name][:, :, :, kg + G] = blk.f[name][:, :, :, (kg % nk) + G]

    HALO_ONLY = ("Uplus",)

    def sync(self, group):
        from_groups = {
            "Ucell": ["U_H"], "Bface": ["B_xi", "B_eta", "B_zeta"], "Eface": ["Eface_xi", "Eface_eta", "Eface_zeta"],
            "Eedge": ["E_xi", "E_eta", "E_zeta"], "B_cell": ["B_cell", "Bind_cell"], "Jedge": ["J_xi", "J_eta", "J_zeta"],
            "J_cell": ["J_cell"], "Uplus": ["U_plus"], "dB": ["dB_xi", "dB_eta", "dB_zeta"],
            "Badd": ["Badd_xi", "Badd_eta", "Badd_zeta"], "Ehall": ["Ehall_xi", "Ehall_eta", "Ehall_zeta"],
            "Eres": ["Eres_xi", "Eres_eta", "Eres_zeta"], "Eres1form": ["Eres_xi", "Eres_eta", "Eres_zeta"]}
        fields = from_groups[group]
        if group not in self.HALO_ONLY:
            for f in fields:
                for side in self.POLES:
                    self._pole(f, side)
                self._farfield(f)
                self._solid(f)
            for f in fields:
                self._corner_default(f)
        for f in fields:
            self._halo_k(f)

    # ------------------------------------------------ Pole repairs
    def bzeta_pole_rewrite(self):
        """calc_Bcell after Sync("B_cell") (Z4_Lunar/src/physics/LunarSolver_Tools.cpp:242-307):
        on the first cell layer at each eta Pole, B_zeta becomes the flux of
        Bind_cell through the zeta face, k = 0 .. n_k."""
        blk = self.blocks[0]
        n = blk.n
        for side in self.POLES:
            jc = 0 if side < 0 else n[1] - 1
            lo, hi = (0, jc, 0), (n[0], jc + 1, n[2] + 1)
            bi = [blk.box("Bind_cell", m, lo, hi) for m in range(3)]
            A = [blk.box("JDze", m, lo, hi) for m in range(3)]
            blk.f["B_zeta"][0][blk.s(lo, hi)] = bi[0] * A[0] + bi[1] * A[1] + bi[2] * A[2]

    def jcell_pole_repair(self):
        """The least-squares J_cell of the first cell layer at each eta Pole
        (calc_Jcell, LunarSolver_Tools.cpp:945-1090): per ring the Cartesian
        vector that best reproduces the J edge 1-forms of the ring's norm
        edges on the Pole layer and its axis / rotate edges one node layer away."""
        n = self.blocks[0].n
        for side in self.POLES:
            jc = 0 if side < 0 else n[1] - 1
            jt = jc + 1 if side < 0 else jc
            for i in range(n[0]):
                A = [[0.0] * 3 for _ in range(3)]
                b = [0.0, 0.0, 0.0]
                cnt = 0

                def push(Je, dr, ii, jj, kk):
                    nonlocal cnt
                    d = [self._at(dr, ii, jj, kk, m) for m in range(3)]
                    L = np.sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2])
                    if L < 1.0e-14:
                        return
                    tau = [d[0] / L, d[1] / L, d[2] / L]
                    y = self._at(Je, ii, jj, kk) / L
                    for a in range(3):
                        b[a] += y * tau[a]
                        for c in range(3):
                            A[a][c] += tau[a] * tau[c]
                    cnt += 1

                for k in range(n[2]):
                    push("J_eta", "dr_eta", i, jc, k)
                    push("J_eta", "dr_eta", i + 1, jc, k)
                    push("J_eta", "dr_eta", i, jc, k + 1)
                    push("J_eta", "dr_eta", i + 1, jc, k + 1)
                    push("J_xi", "dr_xi", i, jt, k)
                    push("J_xi", "dr_xi", i, jt, k + 1)
                    push("J_zeta", "dr_zeta", i, jt, k)
                    push("J_zeta", "dr_zeta", i + 1, jt, k)
                if cnt <= 0:
                    continue
                trA = A[0][0] + A[1][1] + A[2][2]
                reg = 1.0e-12 * _cmax(1.0, trA)
                for a in range(3):
                    A[a][a] += reg
                Jp = _solve3_gj(A, b)
                if Jp is None:
                    continue
                for k in range(n[2]):
                    for m in range(3):
                        self._put("J_cell", i, jc, k, m, Jp[m])

    def update_magnetic_derived(self):
        blk = self.blocks[0]
        self.calc_bcell(blk)
        self.sync("B_cell")
        self.bzeta_pole_rewrite()
        self.curl_adj(blk, ("B_xi", "B_eta", "B_zeta"), ("J_xi", "J_eta", "J_zeta"))
        self.sync("Jedge")
        self.calc_jcell(blk)
        self.jcell_pole_repair()
        self.sync("J_cell")

    def calc_divb(self):
        """calc_divB with the Pole zeroing of the first cell layer at each
        Pole (LunarSolver_Tools.cpp:685-775)."""
        super().calc_divb()
        blk = self.blocks[0]
        n = blk.n
        for side in self.POLES:
            jc = 0 if side < 0 else n[1] - 1
            blk.f["divB"][0][blk.s((0, jc, 0), (n[0], jc + 1, n[2]))] = 0.0
