"""Host-side geometry builder: the metric and Hodge-star arrays the hot path
reads, computed from block node coordinates with the same formulas and the
same floating-point operation order as the reference set-up, so the arrays
agree bit for bit.

Followed reference code:
* ghost nodes by reflection: src/1_grid/1_MPCNS_Grid.cpp:591-820 (Block::Add_ghostmesh)
* cell centres (dual grid): src/1_grid/1_MPCNS_Grid_GCL.cpp:6-24
* face area vectors JDxi/JDet/JDze: src/3_field/4_MPCNS_Geometry.cpp:98-197
* cell volume Jac: src/3_field/4_MPCNS_Geometry.cpp:199-318
* Area, dlstar, beta, dl, Sstar, Astar, alpha: src/3_field/4_MPCNS_Geometry.cpp:320-640
* dr edge vectors: src/3_field/4_MPCNS_Geometry.cpp:1249-1318
* B and J reconstruction weights: Z4_Lunar/src/LunarSolver.cpp:284-915

Arrays are "padded" numpy views: ``Padded(a, off)`` stores logical index i at
a[i + off].  All builders return dicts of Padded arrays on the reference's
logical index ranges (include/3_field/1_Field_Block.h, Field_Block.cpp:51-131).
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Dict, Tuple

import numpy as np


@dataclass
class Padded:
    """Array with a logical origin: logical (i, j, k) is a[i+o, j+o, k+o]."""
    a: np.ndarray
    off: int

    def sl(self, lo, hi):
        """Slices for the logical half-open box [lo, hi)."""
        o = self.off
        return tuple(slice(l + o, h + o) for l, h in zip(lo, hi))

    def box(self, lo, hi):
        return self.a[self.sl(lo, hi)]


# ----------------------------------------------------------------------------
# ghost nodes
# ----------------------------------------------------------------------------

def ghost_mesh(x: np.ndarray, y: np.ndarray, z: np.ndarray, ngg: int) -> Padded:
    """Node coordinates extended by ngg+1 ghost layers by point reflection
    through the boundary node, layer by layer, then the 12 edge strips and 8
    corners by parallelogram completion (Block::Add_ghostmesh, 3-D branch).
    Returns Padded array (..., 3) with logical node range [-(ngg+1), m+ngg+2)."""
    mx, my, mz = (s - 1 for s in x.shape)
    G = ngg + 1
    P = np.zeros((mx + 1 + 2 * G, my + 1 + 2 * G, mz + 1 + 2 * G, 3))
    o = G
    P[o:o + mx + 1, o:o + my + 1, o:o + mz + 1, 0] = x
    P[o:o + mx + 1, o:o + my + 1, o:o + mz + 1, 1] = y
    P[o:o + mx + 1, o:o + my + 1, o:o + mz + 1, 2] = z

    def r(lo, hi):
        return slice(lo + o, hi + o)

    for gh in range(1, G + 1):
        gimin, gimax = -gh, mx + gh
        gjmin, gjmax = -gh, my + gh
        gkmin, gkmax = -gh, mz + gh
        J = r(gjmin + 1, gjmax)
        K = r(gkmin + 1, gkmax)
        I = r(gimin + 1, gimax)
        # i faces
        P[gimin + o, J, K] = 2 * P[0 + o, J, K] - P[-gimin + o, J, K]
        P[gimax + o, J, K] = 2 * P[mx + o, J, K] - P[2 * mx - gimax + o, J, K]
        # j faces
        P[I, gjmin + o, K] = 2 * P[I, 0 + o, K] - P[I, -gjmin + o, K]
        P[I, gjmax + o, K] = 2 * P[I, my + o, K] - P[I, 2 * my - gjmax + o, K]
        # k faces
        P[I, J, gkmin + o] = 2 * P[I, J, 0 + o] - P[I, J, -gkmin + o]
        P[I, J, gkmax + o] = 2 * P[I, J, mz + o] - P[I, J, 2 * mz - gkmax + o]
        # edges along k
        for (ic, isn), (jc, jsn) in (((gimin, 1), (gjmin, 1)), ((gimax, -1), (gjmin, 1)),
                                     ((gimin, 1), (gjmax, -1)), ((gimax, -1), (gjmax, -1))):
            P[ic + o, jc + o, K] = (P[ic + isn + o, jc + o, K] + P[ic + o, jc + jsn + o, K]) - P[ic + isn + o, jc + jsn + o, K]
        # edges along j
        for (ic, isn), (kc, ksn) in (((gimin, 1), (gkmin, 1)), ((gimax, -1), (gkmin, 1)),
                                     ((gimin, 1), (gkmax, -1)), ((gimax, -1), (gkmax, -1))):
            P[ic + o, J, kc + o] = (P[ic + isn + o, J, kc + o] + P[ic + o, J, kc + ksn + o]) - P[ic + isn + o, J, kc + ksn + o]
        # edges along i, including the 8 corners
        Ifull = r(gimin, gimax + 1)
        for (jc, jsn), (kc, ksn) in (((gjmin, 1), (gkmin, 1)), ((gjmax, -1), (gkmin, 1)),
                                     ((gjmin, 1), (gkmax, -1)), ((gjmax, -1), (gkmax, -1))):
            P[Ifull, jc + o, kc + o] = (P[Ifull, jc + jsn + o, kc + o] + P[Ifull, jc + o, kc + ksn + o]) - P[Ifull, jc + jsn + o, kc + ksn + o]
    return Padded(P, o)


def pole_ghosts(X: Padded, ncell: Tuple[int, int, int], patches) -> Padded:
    """Grid::MeshTrans_Inner_Pole (src/1_grid/1_MPCNS_Grid_GCL.cpp:564-616):
    beyond a Pole patch (normal xi or eta, rotation direction zeta), the
    ngg+1 ghost node layers over the patch's own tangential range repeat the
    patch's node row, so the ghost cells past the axis collapse.  patches:
    ((imin, imax, jmin, jmax, kmin, kmax), name) node ranges (0-based) of the
    block's physical patches; only "Pole" ones are applied, after the
    reflected ghost mesh and the interface copies."""
    P = X.a
    o = X.off
    G = o
    for rng, name in patches:
        if name != "Pole":
            continue
        sub = [min(abs(rng[2 * a]), abs(rng[2 * a + 1])) for a in range(3)]
        sup = [max(abs(rng[2 * a]), abs(rng[2 * a + 1])) for a in range(3)]
        cyc = [0, 0, 0]
        for a in range(3):
            if sub[a] == sup[a]:
                cyc[a] = -1 if sub[a] == 0 else 1
        if cyc[2] != 0 or sub[2] != 0 or sup[2] != ncell[2] or ncell[2] % 2:
            raise ValueError("a Pole patch needs zeta as its rotation direction, unsplit, with an even cell count")
        for index in range(1, G + 1):
            dst = tuple(slice(sub[a] + index * cyc[a] + o, sup[a] + index * cyc[a] + o + 1) for a in range(3))
            src = tuple(slice(sub[a] + o, sup[a] + o + 1) for a in range(3))
            P[dst] = P[src]
    return X


def block_ghost_mesh(b, ngg: int) -> Padded:
    """Ghost node mesh of a case block (BlockGrid): reflection, then the Pole
    collapse of its Pole patches."""
    return pole_ghosts(ghost_mesh(b.x, b.y, b.z, ngg), b.ncell, b.physical)


# ----------------------------------------------------------------------------
# helpers with the reference's operation order
# ----------------------------------------------------------------------------

def _cross(a, b):
    return np.stack([a[..., 1] * b[..., 2] - a[..., 2] * b[..., 1],
                     a[..., 2] * b[..., 0] - a[..., 0] * b[..., 2],
                     a[..., 0] * b[..., 1] - a[..., 1] * b[..., 0]], axis=-1)


def _norm3(a):
    return np.sqrt(a[..., 0] * a[..., 0] + a[..., 1] * a[..., 1] + a[..., 2] * a[..., 2])


def _avg4(a, b, c, d):
    return 0.25 * (((a + b) + c) + d)


def _avg8(a0, a1, a2, a3, a4, a5, a6, a7):
    return 0.125 * (((((((a0 + a1) + a2) + a3) + a4) + a5) + a6) + a7)


def _extent(loc: str, n, g):
    ni, nj, nk = n
    plus = dict(cell=(0, 0, 0), fxi=(1, 0, 0), fet=(0, 1, 0), fze=(0, 0, 1),
                exi=(0, 1, 1), eet=(1, 0, 1), eze=(1, 1, 0), node=(1, 1, 1))[loc]
    return (-g, -g, -g), (ni + plus[0] + g, nj + plus[1] + g, nk + plus[2] + g)


def _idx(lo, hi):
    """Open-mesh logical index grids for the box [lo, hi)."""
    return np.meshgrid(np.arange(lo[0], hi[0]), np.arange(lo[1], hi[1]), np.arange(lo[2], hi[2]), indexing="ij")


def _take(P: Padded, I, J, K):
    """P at the logical points (I, J, K).  The callers pass index grids of a
    box (from _idx) shifted by constants, which become a strided slice; any
    other index arrays take the general gather."""
    o = P.off
    n = I.shape
    if len(n) == 3 and J.shape == n and K.shape == n and min(n) > 0:
        i0, j0, k0 = int(I[0, 0, 0]), int(J[0, 0, 0]), int(K[0, 0, 0])
        if (I[-1, 0, 0] - i0 == n[0] - 1 and J[0, -1, 0] - j0 == n[1] - 1 and K[0, 0, -1] - k0 == n[2] - 1
                and I[0, -1, -1] == i0 and J[-1, 0, -1] == j0 and K[-1, -1, 0] == k0
                and np.array_equal(I[:, 0, 0], np.arange(i0, i0 + n[0]))
                and np.array_equal(J[0, :, 0], np.arange(j0, j0 + n[1]))
                and np.array_equal(K[0, 0, :], np.arange(k0, k0 + n[2]))
                and i0 + o >= 0 and j0 + o >= 0 and k0 + o >= 0):
            # a grid iff each index varies along its own axis only
            if ((I == I[:, :1, :1]).all() and (J == J[:1, :, :1]).all() and (K == K[:1, :1, :]).all()):
                return P.a[i0 + o:i0 + o + n[0], j0 + o:j0 + o + n[1], k0 + o:k0 + o + n[2]]
    return P.a[I + o, J + o, K + o]


# ----------------------------------------------------------------------------
# geometry fields
# ----------------------------------------------------------------------------

def build(X: Padded, ncell: Tuple[int, int, int], ngg: int) -> Dict[str, Tuple[tuple, tuple, np.ndarray]]:
    """All geometry fields on their reference extents.  Returns name ->
    (lo, hi, data) with data shaped (ni, nj, nk, ncomp)."""
    n = ncell
    out: Dict[str, Tuple[tuple, tuple, np.ndarray]] = {}

    def face_area(loc, da, db):
        lo, hi = _extent(loc, n, ngg)
        I, J, K = _idx(lo, hi)
        ori = _take(X, I, J, K)
        xp = _take(X, I + da[0], J + da[1], K + da[2])
        yp = _take(X, I + db[0], J + db[1], K + db[2])
        xyp = _take(X, I + da[0] + db[0], J + da[1] + db[1], K + da[2] + db[2])
        rx = xp - ori
        ry = yp - ori
        rx_ = yp - xyp
        ry_ = xp - xyp
        A = _cross(rx, ry) + _cross(rx_, ry_)
        return lo, hi, 0.5 * A

    out["JDxi"] = face_area("fxi", (0, 1, 0), (0, 0, 1))
    out["JDet"] = face_area("fet", (0, 0, 1), (1, 0, 0))
    out["JDze"] = face_area("fze", (1, 0, 0), (0, 1, 0))

    # cell centres: dual(i,j,k) = mean of the 8 nodes around (i-1..i, j-1..j, k-1..k)
    gd = ngg
    dlo = (-gd, -gd, -gd)
    dhi = (n[0] + gd + 1, n[1] + gd + 1, n[2] + gd + 1)
    I, J, K = _idx(dlo, dhi)
    Dc = _avg8(_take(X, I, J, K), _take(X, I - 1, J, K), _take(X, I, J - 1, K), _take(X, I - 1, J - 1, K),
               _take(X, I, J, K - 1), _take(X, I - 1, J, K - 1), _take(X, I, J - 1, K - 1),
               _take(X, I - 1, J - 1, K - 1))
    D = Padded(Dc, gd)

    def jd(name):
        lo, hi, a = out[name]
        return Padded(a, -lo[0])

    JDxi, JDet, JDze = jd("JDxi"), jd("JDet"), jd("JDze")

    # Jac = (1/3) sum over the 6 faces of S_out . (x_face - x_c)
    lo, hi = _extent("cell", n, ngg - 1)
    I, J, K = _idx(lo, hi)
    xc = _take(D, I + 1, J + 1, K + 1)

    def dot(a, b):
        return (a[..., 0] * b[..., 0] + a[..., 1] * b[..., 1]) + a[..., 2] * b[..., 2]

    def fc(a, b, c, d):
        return _avg4(_take(X, *a), _take(X, *b), _take(X, *c), _take(X, *d))

    V = np.zeros(I.shape)
    V = V + dot(-_take(JDxi, I, J, K), fc((I, J, K), (I, J + 1, K), (I, J, K + 1), (I, J + 1, K + 1)) - xc)
    V = V + dot(_take(JDxi, I + 1, J, K), fc((I + 1, J, K), (I + 1, J + 1, K), (I + 1, J, K + 1), (I + 1, J + 1, K + 1)) - xc)
    V = V + dot(-_take(JDet, I, J, K), fc((I, J, K), (I + 1, J, K), (I, J, K + 1), (I + 1, J, K + 1)) - xc)
    V = V + dot(_take(JDet, I, J + 1, K), fc((I, J + 1, K), (I + 1, J + 1, K), (I, J + 1, K + 1), (I + 1, J + 1, K + 1)) - xc)
    V = V + dot(-_take(JDze, I, J, K), fc((I, J, K), (I + 1, J, K), (I, J + 1, K), (I + 1, J + 1, K)) - xc)
    V = V + dot(_take(JDze, I, J, K + 1), fc((I, J, K + 1), (I + 1, J, K + 1), (I, J + 1, K + 1), (I + 1, J + 1, K + 1)) - xc)
    out["Jac"] = (lo, hi, (V / 3.0)[..., None])

    # face Area, dlstar, beta
    eps = 1e-25
    for loc, nm, jdp, sh in (("fxi", "xi", JDxi, (0, 1, 1)), ("fet", "eta", JDet, (1, 0, 1)), ("fze", "zeta", JDze, (1, 1, 0))):
        lo, hi = _extent(loc, n, ngg - 1)
        I, J, K = _idx(lo, hi)
        S = _take(jdp, I, J, K)
        Smag = _norm3(S)
        cL = _take(D, I + sh[0], J + sh[1], K + sh[2])
        cR = _take(D, I + 1, J + 1, K + 1)
        Lstar = _norm3(cR - cL)
        with np.errstate(divide="ignore", invalid="ignore"):
            beta = np.where(Smag < eps, 0.0, Lstar / Smag)
        out["Area_" + nm] = (lo, hi, Smag[..., None])
        out["dlstar_" + nm] = (lo, hi, Lstar[..., None])
        out["beta_" + nm] = (lo, hi, beta[..., None])

    # edge dl, Sstar, Astar, alpha (with the dual-face collapse cap)
    ratio = 1e-3
    tol = 1e-12

    def quad(p00, p10, p01, p11):
        a0 = _cross(p10 - p00, p01 - p00)
        a1 = _cross(p01 - p11, p10 - p11)
        return 0.5 * (a0 + a1)

    edge_defs = (
        ("exi", "xi", (1, 0, 0), [(1, 0, 0), (1, 1, 0), (1, 0, 1), (1, 1, 1)]),
        ("eet", "eta", (0, 1, 0), [(0, 1, 0), (1, 1, 0), (0, 1, 1), (1, 1, 1)]),
        ("eze", "zeta", (0, 0, 1), [(0, 0, 1), (1, 0, 1), (0, 1, 1), (1, 1, 1)]),
    )
    for loc, nm, d, cells in edge_defs:
        lo, hi = _extent(loc, n, ngg - 1)
        I, J, K = _idx(lo, hi)
        r0 = _take(X, I, J, K)
        r1 = _take(X, I + d[0], J + d[1], K + d[2])
        L = _norm3(r1 - r0)
        p00, p10, p01, p11 = (_take(D, I + c[0], J + c[1], K + c[2]) for c in cells)
        Avec = quad(p00, p10, p01, p11)
        Amag = _norm3(Avec)
        with np.errstate(divide="ignore", invalid="ignore"):
            alpha_raw = np.where(Amag < eps, 0.0, L / Amag)
        d00_10 = _norm3(p10 - p00)
        d00_01 = _norm3(p01 - p00)
        d10_11 = _norm3(p11 - p10)
        d01_11 = _norm3(p11 - p01)
        d00_11 = _norm3(p11 - p00)
        d10_01 = _norm3(p01 - p10)
        href = np.maximum(np.maximum(np.maximum(d00_10, d00_01), np.maximum(d10_11, d01_11)),
                          np.maximum(np.maximum(d00_11, d10_01), np.maximum(L, eps)))
        side_min = np.minimum(np.minimum(d00_10, d00_01), np.minimum(d10_11, d01_11))
        diag_min = np.minimum(d00_11, d10_01)
        touch = (L < tol) | (side_min < ratio * href) | (diag_min < ratio * href) | (Amag < ratio * href * href)
        alpha = np.where(touch, 0.0, alpha_raw)
        out["dl_" + nm] = (lo, hi, L[..., None])
        out["Sstar_" + nm] = (lo, hi, Avec)
        out["Astar_" + nm] = (lo, hi, Amag[..., None])
        out["alpha_" + nm] = (lo, hi, alpha[..., None])
        out["dr_" + nm] = (lo, hi, r1 - r0)

    out["Bcell_from_Bface_w"] = _bcell_weights(X, JDxi, JDet, JDze, n, ngg - 1)
    out["Jcell_from_Jedge_w"] = _jcell_weights(X, n, ngg - 1)
    return out


# ----------------------------------------------------------------------------
# reconstruction weights (pseudo-inverse least squares)
# ----------------------------------------------------------------------------

def _sym_eig_3x3(A):
    """Cyclic Jacobi eigen-solver for a batch of symmetric 3x3 matrices, 12
    sweeps over (0,1), (0,2), (1,2), then eigenvalues sorted descending with
    the eigenvector columns permuted alongside
    (Z4_Lunar/src/LunarSolver.cpp:306-380).  A: (..., 3, 3), modified."""
    shp = A.shape[:-2]
    V = np.zeros(shp + (3, 3))
    V[..., 0, 0] = V[..., 1, 1] = V[..., 2, 2] = 1.0
    for _ in range(12):
        for p, q in ((0, 1), (0, 2), (1, 2)):
            apq = A[..., p, q].copy()
            act = ~(np.abs(apq) < 1e-300)
            if not act.any():
                continue
            app = A[..., p, p].copy()
            aqq = A[..., q, q].copy()
            safe = np.where(act, apq, 1.0)
            tau = (aqq - app) / (2.0 * safe)
            with np.errstate(over="ignore", divide="ignore", invalid="ignore"):
                sq = np.sqrt(1.0 + tau * tau)
                t = np.where(tau >= 0.0, 1.0 / (tau + sq), -1.0 / (-tau + sq))
            c = 1.0 / np.sqrt(1.0 + t * t)
            s = t * c
            k = 3 - p - q
            Akp = A[..., k, p].copy()
            Akq = A[..., k, q].copy()
            nkp = c * Akp - s * Akq
            nkq = s * Akp + c * Akq
            app_new = ((c * c) * app - ((2.0 * s) * c) * apq) + (s * s) * aqq
            aqq_new = ((s * s) * app + ((2.0 * s) * c) * apq) + (c * c) * aqq
            for (a, b, v) in ((k, p, nkp), (p, k, nkp), (k, q, nkq), (q, k, nkq),
                              (p, p, app_new), (q, q, aqq_new)):
                A[..., a, b] = np.where(act, v, A[..., a, b])
            A[..., p, q] = np.where(act, 0.0, A[..., p, q])
            A[..., q, p] = np.where(act, 0.0, A[..., q, p])
            for kk in range(3):
                Vkp = V[..., kk, p].copy()
                Vkq = V[..., kk, q].copy()
                V[..., kk, p] = np.where(act, c * Vkp - s * Vkq, Vkp)
                V[..., kk, q] = np.where(act, s * Vkp + c * Vkq, Vkq)
    d = np.stack([A[..., 0, 0], A[..., 1, 1], A[..., 2, 2]], axis=-1)
    for a in range(2):
        for b in range(a + 1, 3):
            sw = d[..., b] > d[..., a]
            da, db = d[..., a].copy(), d[..., b].copy()
            d[..., a] = np.where(sw, db, da)
            d[..., b] = np.where(sw, da, db)
            for kk in range(3):
                va, vb = V[..., kk, a].copy(), V[..., kk, b].copy()
                V[..., kk, a] = np.where(sw, vb, va)
                V[..., kk, b] = np.where(sw, va, vb)
    return V, d


def _pinv_weights(Sx, Sy, Sz, mu, active, valid, tau_eig=1e-10, eps_abs=1e-300):
    """W[q*nf + f] = (M^+ mu_f S_f)_q with M = sum_f mu_f S_f S_f^T and the
    pseudo-inverse from the eigen-decomposition with relative truncation."""
    nf = Sx.shape[-1]
    M = np.zeros(Sx.shape[:-1] + (3, 3))
    m00 = np.zeros(Sx.shape[:-1]); m01 = m00.copy(); m02 = m00.copy()
    m11 = m00.copy(); m12 = m00.copy(); m22 = m00.copy()
    for f in range(nf):
        a = active[..., f]
        u = mu[..., f]
        x, y, z = Sx[..., f], Sy[..., f], Sz[..., f]
        m00 = np.where(a, m00 + (u * x) * x, m00)
        m01 = np.where(a, m01 + (u * x) * y, m01)
        m02 = np.where(a, m02 + (u * x) * z, m02)
        m11 = np.where(a, m11 + (u * y) * y, m11)
        m12 = np.where(a, m12 + (u * y) * z, m12)
        m22 = np.where(a, m22 + (u * z) * z, m22)
    M[..., 0, 0], M[..., 0, 1], M[..., 0, 2] = m00, m01, m02
    M[..., 1, 0], M[..., 1, 1], M[..., 1, 2] = m01, m11, m12
    M[..., 2, 0], M[..., 2, 1], M[..., 2, 2] = m02, m12, m22
    V, lam = _sym_eig_3x3(M.copy())
    lam_max = np.maximum(lam[..., 0], np.maximum(lam[..., 1], lam[..., 2]))
    ok = valid & ~(lam_max <= eps_abs)
    inv = np.zeros_like(lam)
    for q in range(3):
        with np.errstate(divide="ignore", invalid="ignore"):
            inv[..., q] = np.where(lam[..., q] > tau_eig * lam_max, 1.0 / lam[..., q], 0.0)
    Minv = np.zeros(M.shape)
    for a in range(3):
        for b in range(3):
            acc = np.zeros(lam.shape[:-1])
            for q in range(3):
                acc = acc + (V[..., a, q] * inv[..., q]) * V[..., b, q]
            Minv[..., a, b] = acc
    W = np.zeros(Sx.shape[:-1] + (3 * nf,))
    for f in range(nf):
        a = active[..., f] & ok
        rx = mu[..., f] * Sx[..., f]
        ry = mu[..., f] * Sy[..., f]
        rz = mu[..., f] * Sz[..., f]
        for q in range(3):
            w = (Minv[..., q, 0] * rx + Minv[..., q, 1] * ry) + Minv[..., q, 2] * rz
            W[..., q * nf + f] = np.where(a, w, 0.0)
    return W


def _bcell_weights(X, JDxi, JDet, JDze, n, g):
    """Weights of the 6 signed face fluxes for the cell-centred B
    (Z4_Lunar/src/LunarSolver.cpp:386-625); nonzero on inner cells only."""
    lo, hi = _extent("cell", n, g)
    W = np.zeros((hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2], 18))
    I, J, K = _idx((0, 0, 0), n)

    def nd(di, dj, dk):
        return _take(X, I + di, J + dj, K + dk)

    c = _avg8(nd(0, 0, 0), nd(1, 0, 0), nd(0, 1, 0), nd(1, 1, 0), nd(0, 0, 1), nd(1, 0, 1), nd(0, 1, 1), nd(1, 1, 1))
    fcs = [
        _avg4(nd(0, 0, 0), nd(0, 1, 0), nd(0, 0, 1), nd(0, 1, 1)),
        _avg4(nd(1, 0, 0), nd(1, 1, 0), nd(1, 0, 1), nd(1, 1, 1)),
        _avg4(nd(0, 0, 0), nd(1, 0, 0), nd(0, 0, 1), nd(1, 0, 1)),
        _avg4(nd(0, 1, 0), nd(1, 1, 0), nd(0, 1, 1), nd(1, 1, 1)),
        _avg4(nd(0, 0, 0), nd(1, 0, 0), nd(0, 1, 0), nd(1, 1, 0)),
        _avg4(nd(0, 0, 1), nd(1, 0, 1), nd(0, 1, 1), nd(1, 1, 1)),
    ]
    S = [-_take(JDxi, I, J, K), _take(JDxi, I + 1, J, K), -_take(JDet, I, J, K), _take(JDet, I, J + 1, K),
         -_take(JDze, I, J, K), _take(JDze, I, J, K + 1)]
    Sx = np.stack([s[..., 0] for s in S], axis=-1)
    Sy = np.stack([s[..., 1] for s in S], axis=-1)
    Sz = np.stack([s[..., 2] for s in S], axis=-1)
    Smag = np.sqrt(Sx * Sx + Sy * Sy + Sz * Sz)
    Sref = np.zeros(I.shape)
    for f in range(6):
        Sref = np.maximum(Sref, Smag[..., f])
    dist = np.stack([_norm3(fcs[f] - c) for f in range(6)], axis=-1)
    valid = ~(Sref <= 1e-300)
    active = Smag > 1e-10 * Sref[..., None]
    mu = np.where(active, 1.0 / np.maximum(dist, 1e-14), 0.0)
    Win = _pinv_weights(Sx, Sy, Sz, mu, active, valid)
    W[-lo[0]:-lo[0] + n[0], -lo[1]:-lo[1] + n[1], -lo[2]:-lo[2] + n[2]] = Win
    return lo, hi, W


def _jcell_weights(X, n, g):
    """Weights of the 12 edge currents for the cell-centred J
    (Z4_Lunar/src/LunarSolver.cpp:627-915); nonzero on inner cells only."""
    lo, hi = _extent("cell", n, g)
    W = np.zeros((hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2], 36))
    I, J, K = _idx((0, 0, 0), n)

    def nd(di, dj, dk):
        return _take(X, I + di, J + dj, K + dk)

    pairs = [((0, 0, 0), (1, 0, 0)), ((0, 1, 0), (1, 1, 0)), ((0, 0, 1), (1, 0, 1)), ((0, 1, 1), (1, 1, 1)),
             ((0, 0, 0), (0, 1, 0)), ((1, 0, 0), (1, 1, 0)), ((0, 0, 1), (0, 1, 1)), ((1, 0, 1), (1, 1, 1)),
             ((0, 0, 0), (0, 0, 1)), ((1, 0, 0), (1, 0, 1)), ((0, 1, 0), (0, 1, 1)), ((1, 1, 0), (1, 1, 1))]
    ls = [nd(*b) - nd(*a) for a, b in pairs]
    Lx = np.stack([l[..., 0] for l in ls], axis=-1)
    Ly = np.stack([l[..., 1] for l in ls], axis=-1)
    Lz = np.stack([l[..., 2] for l in ls], axis=-1)
    L = np.sqrt(Lx * Lx + Ly * Ly + Lz * Lz)
    Lref = np.zeros(I.shape)
    for e in range(12):
        Lref = np.maximum(Lref, L[..., e])
    valid = ~(Lref <= 1e-300)
    active = L > 1e-10 * Lref[..., None]
    mu = np.where(active, 1.0, 0.0)
    Win = _pinv_weights(Lx, Ly, Lz, mu, active, valid)
    W[-lo[0]:-lo[0] + n[0], -lo[1]:-lo[1] + n[1], -lo[2]:-lo[2] + n[2]] = Win
    return lo, hi, W
