// Geometry of a block from its ghost node mesh, point by point: face area
// vectors, cell volumes, the face and edge Hodge ratios, edge vectors and
// lengths, and the least-squares weights of the cell-centred B and J
// (src/3_field/4_MPCNS_Geometry.cpp:4-640, Z4_Lunar/src/LunarSolver.cpp:243-915).
// Every point is computed from the nodes alone, in the reference's operation
// order (face vectors and cell centres are recomputed where a later quantity
// needs them), so the device kernel k_geometry and host builds of this code
// produce the same values as the reference.
#pragma once

#include <cmath>
#include <cstdint>

#include "mhd_layout.cuh"

namespace mhd
{

// The ghost node mesh: logical node (i, j, k), i in [-off, n_i + 1 + off),
// at a[((i + off) * NJ + (j + off)) * NK + (k + off)] * 3 + c
struct NodeMesh
{
    const double *a;
    int off;
    int NJ, NK;
};

// point groups of the builder (one launch row each)
enum GeomGroup : int
{
    GEOM_FACE_VEC = 0, // JDxi, JDet, JDze (face area vectors)
    GEOM_JAC,          // Jac (cell volume)
    GEOM_FACE_HODGE,   // Area_*, beta_*
    GEOM_EDGE,         // dl_*, Astar_*, alpha_*, dr_*
    GEOM_WB,           // Bcell_from_Bface_w
    GEOM_WJ,           // Jcell_from_Jedge_w
    GEOM_BADD,         // Badd_*: the uniform field's face fluxes
    NGEOM_GROUP
};

struct V3
{
    double x, y, z;
};

__host__ __device__ inline V3 gnode(const NodeMesh &m, int i, int j, int k)
{
    const int64_t p = ((int64_t(i + m.off) * m.NJ + (j + m.off)) * m.NK + (k + m.off)) * 3;
    return V3{m.a[p], m.a[p + 1], m.a[p + 2]};
}
__host__ __device__ inline V3 gsub(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__host__ __device__ inline V3 gadd(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__host__ __device__ inline V3 gneg(V3 a) { return V3{-a.x, -a.y, -a.z}; }
__host__ __device__ inline V3 gscale(double s, V3 a) { return V3{s * a.x, s * a.y, s * a.z}; }
__host__ __device__ inline V3 gcross(V3 a, V3 b)
{
    return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__host__ __device__ inline double gnorm(V3 a) { return sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
__host__ __device__ inline double gdot(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
__host__ __device__ inline V3 gavg4(V3 a, V3 b, V3 c, V3 d)
{
    return gscale(0.25, gadd(gadd(gadd(a, b), c), d));
}
__host__ __device__ inline V3 gavg8(V3 a0, V3 a1, V3 a2, V3 a3, V3 a4, V3 a5, V3 a6, V3 a7)
{
    return gscale(0.125, gadd(gadd(gadd(gadd(gadd(gadd(gadd(a0, a1), a2), a3), a4), a5), a6), a7));
}
__host__ __device__ inline double gmax(double a, double b) { return (a < b) ? b : a; } // np.maximum on numbers
__host__ __device__ inline double gmin(double a, double b) { return (b < a) ? b : a; } // np.minimum on numbers

// face area vector of face family fa (0 xi, 1 eta, 2 zeta) at (i, j, k):
// half the sum of the two triangle cross products of the face's quad
__host__ __device__ inline V3 geom_face(const NodeMesh &m, int fa, int i, int j, int k)
{
    const int da[3][3] = {{0, 1, 0}, {0, 0, 1}, {1, 0, 0}};
    const int db[3][3] = {{0, 0, 1}, {1, 0, 0}, {0, 1, 0}};
    const V3 ori = gnode(m, i, j, k);
    const V3 xp = gnode(m, i + da[fa][0], j + da[fa][1], k + da[fa][2]);
    const V3 yp = gnode(m, i + db[fa][0], j + db[fa][1], k + db[fa][2]);
    const V3 xyp = gnode(m, i + da[fa][0] + db[fa][0], j + da[fa][1] + db[fa][1], k + da[fa][2] + db[fa][2]);
    const V3 A = gadd(gcross(gsub(xp, ori), gsub(yp, ori)), gcross(gsub(yp, xyp), gsub(xp, xyp)));
    return gscale(0.5, A);
}

// cell centre of the dual index (i, j, k): mean of the nodes (i-1..i, j-1..j, k-1..k)
__host__ __device__ inline V3 geom_dual(const NodeMesh &m, int i, int j, int k)
{
    return gavg8(gnode(m, i, j, k), gnode(m, i - 1, j, k), gnode(m, i, j - 1, k), gnode(m, i - 1, j - 1, k),
                 gnode(m, i, j, k - 1), gnode(m, i - 1, j, k - 1), gnode(m, i, j - 1, k - 1),
                 gnode(m, i - 1, j - 1, k - 1));
}

// Cyclic Jacobi eigen-solver of a symmetric 3x3 matrix, 12 sweeps over
// (0,1), (0,2), (1,2), eigenvalues sorted descending with the eigenvector
// columns alongside (Z4_Lunar/src/LunarSolver.cpp:306-380)
__host__ __device__ inline void geom_eig3(double A[3][3], double V[3][3], double d[3])
{
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b)
            V[a][b] = (a == b) ? 1.0 : 0.0;
    const int P[3] = {0, 0, 1}, Q[3] = {1, 2, 2};
    for (int sweep = 0; sweep < 12; ++sweep)
        for (int r = 0; r < 3; ++r)
        {
            const int p = P[r], q = Q[r];
            const double apq = A[p][q];
            if (fabs(apq) < 1e-300)
                continue;
            const double app = A[p][p], aqq = A[q][q];
            const double tau = (aqq - app) / (2.0 * apq);
            const double sq = sqrt(1.0 + tau * tau);
            const double t = (tau >= 0.0) ? 1.0 / (tau + sq) : -1.0 / (-tau + sq);
            const double c = 1.0 / sqrt(1.0 + t * t);
            const double s = t * c;
            const int k = 3 - p - q;
            const double Akp = A[k][p], Akq = A[k][q];
            const double nkp = c * Akp - s * Akq;
            const double nkq = s * Akp + c * Akq;
            const double app_new = ((c * c) * app - ((2.0 * s) * c) * apq) + (s * s) * aqq;
            const double aqq_new = ((s * s) * app + ((2.0 * s) * c) * apq) + (c * c) * aqq;
            A[k][p] = nkp;
            A[p][k] = nkp;
            A[k][q] = nkq;
            A[q][k] = nkq;
            A[p][p] = app_new;
            A[q][q] = aqq_new;
            A[p][q] = 0.0;
            A[q][p] = 0.0;
            for (int kk = 0; kk < 3; ++kk)
            {
                const double Vkp = V[kk][p], Vkq = V[kk][q];
                V[kk][p] = c * Vkp - s * Vkq;
                V[kk][q] = s * Vkp + c * Vkq;
            }
        }
    d[0] = A[0][0];
    d[1] = A[1][1];
    d[2] = A[2][2];
    for (int a = 0; a < 2; ++a)
        for (int b = a + 1; b < 3; ++b)
            if (d[b] > d[a])
            {
                const double t = d[a];
                d[a] = d[b];
                d[b] = t;
                for (int kk = 0; kk < 3; ++kk)
                {
                    const double u = V[kk][a];
                    V[kk][a] = V[kk][b];
                    V[kk][b] = u;
                }
            }
}

// W[q * nf + f] = (M^+ mu_f S_f)_q with M = sum_f mu_f S_f S_f^T and the
// pseudo-inverse from the eigen-decomposition with relative truncation 1e-10
template <int NF>
__host__ __device__ inline void geom_pinv_weights(const V3 S[NF], const double mu[NF], const bool active[NF],
                                                  bool valid, double *W, int64_t wstride)
{
    double m00 = 0.0, m01 = 0.0, m02 = 0.0, m11 = 0.0, m12 = 0.0, m22 = 0.0;
    for (int f = 0; f < NF; ++f)
    {
        if (!active[f])
            continue;
        const double u = mu[f], x = S[f].x, y = S[f].y, z = S[f].z;
        m00 = m00 + (u * x) * x;
        m01 = m01 + (u * x) * y;
        m02 = m02 + (u * x) * z;
        m11 = m11 + (u * y) * y;
        m12 = m12 + (u * y) * z;
        m22 = m22 + (u * z) * z;
    }
    double A[3][3] = {{m00, m01, m02}, {m01, m11, m12}, {m02, m12, m22}};
    double V[3][3], lam[3];
    geom_eig3(A, V, lam);
    const double lam_max = gmax(lam[0], gmax(lam[1], lam[2]));
    const bool ok = valid && !(lam_max <= 1e-300);
    double inv[3];
    for (int q = 0; q < 3; ++q)
        inv[q] = (lam[q] > 1e-10 * lam_max) ? 1.0 / lam[q] : 0.0;
    double Minv[3][3];
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b)
        {
            double acc = 0.0;
            for (int q = 0; q < 3; ++q)
                acc = acc + (V[a][q] * inv[q]) * V[b][q];
            Minv[a][b] = acc;
        }
    for (int f = 0; f < NF; ++f)
    {
        const bool a = active[f] && ok;
        const double rx = mu[f] * S[f].x, ry = mu[f] * S[f].y, rz = mu[f] * S[f].z;
        for (int q = 0; q < 3; ++q)
        {
            const double w = (Minv[q][0] * rx + Minv[q][1] * ry) + Minv[q][2] * rz;
            W[int64_t(q * NF + f) * wstride] = a ? w : 0.0;
        }
    }
}

// does (i, j, k) lie in the box of location loc widened by g ghost layers
__host__ __device__ inline bool geom_in(const BlockView &b, int loc, int g, int i, int j, int k)
{
    int pi, pj, pk;
    loc_plus(loc, pi, pj, pk);
    return i >= -g && j >= -g && k >= -g && i < b.ni + pi + g && j < b.nj + pj + g && k < b.nk + pk + g;
}

// the fields of one group at one point (i, j, k) of the padded box; points
// outside a field's extent are left alone.  G: the ghost layers of the
// geometry (ngg), gb: the uniform applied field of GEOM_BADD
__host__ __device__ inline void geom_point(const NodeMesh &m, const BlockView &b, int group, int i, int j, int k,
                                           int G, const double *gb)
{
    const int64_t v = b.vol;
    const int64_t p = pidx(b, i, j, k);
    switch (group)
    {
    case GEOM_FACE_VEC:
        for (int fa = 0; fa < 3; ++fa)
            if (geom_in(b, LOC_FXI + fa, G, i, j, k))
            {
                const V3 A = geom_face(m, fa, i, j, k);
                double *F = b.f[F_JDxi + fa];
                F[p] = A.x;
                F[v + p] = A.y;
                F[2 * v + p] = A.z;
            }
        break;
    case GEOM_JAC:
        if (geom_in(b, LOC_CELL, G - 1, i, j, k))
        {
            const V3 xc = geom_dual(m, i + 1, j + 1, k + 1);
            auto fc = [&](int a0, int a1, int a2, int b0, int b1, int b2, int c0, int c1, int c2, int d0, int d1,
                          int d2) {
                return gavg4(gnode(m, a0, a1, a2), gnode(m, b0, b1, b2), gnode(m, c0, c1, c2), gnode(m, d0, d1, d2));
            };
            double V = 0.0;
            V = V + gdot(gneg(geom_face(m, 0, i, j, k)), gsub(fc(i, j, k, i, j + 1, k, i, j, k + 1, i, j + 1, k + 1), xc));
            V = V + gdot(geom_face(m, 0, i + 1, j, k),
                         gsub(fc(i + 1, j, k, i + 1, j + 1, k, i + 1, j, k + 1, i + 1, j + 1, k + 1), xc));
            V = V + gdot(gneg(geom_face(m, 1, i, j, k)), gsub(fc(i, j, k, i + 1, j, k, i, j, k + 1, i + 1, j, k + 1), xc));
            V = V + gdot(geom_face(m, 1, i, j + 1, k),
                         gsub(fc(i, j + 1, k, i + 1, j + 1, k, i, j + 1, k + 1, i + 1, j + 1, k + 1), xc));
            V = V + gdot(gneg(geom_face(m, 2, i, j, k)), gsub(fc(i, j, k, i + 1, j, k, i, j + 1, k, i + 1, j + 1, k), xc));
            V = V + gdot(geom_face(m, 2, i, j, k + 1),
                         gsub(fc(i, j, k + 1, i + 1, j, k + 1, i, j + 1, k + 1, i + 1, j + 1, k + 1), xc));
            b.f[F_Jac][p] = V / 3.0;
        }
        break;
    case GEOM_FACE_HODGE:
    {
        const int sh[3][3] = {{0, 1, 1}, {1, 0, 1}, {1, 1, 0}};
        for (int fa = 0; fa < 3; ++fa)
            if (geom_in(b, LOC_FXI + fa, G - 1, i, j, k))
            {
                const double Smag = gnorm(geom_face(m, fa, i, j, k));
                const V3 cL = geom_dual(m, i + sh[fa][0], j + sh[fa][1], k + sh[fa][2]);
                const V3 cR = geom_dual(m, i + 1, j + 1, k + 1);
                const double Lstar = gnorm(gsub(cR, cL));
                b.f[F_Areaxi + fa][p] = Smag;
                b.f[F_betaxi + fa][p] = (Smag < 1e-25) ? 0.0 : Lstar / Smag;
            }
        break;
    }
    case GEOM_EDGE:
    {
        // edge direction and the four cells around the edge (dual indices)
        const int d[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
        const int cells[3][4][3] = {{{1, 0, 0}, {1, 1, 0}, {1, 0, 1}, {1, 1, 1}},
                                    {{0, 1, 0}, {1, 1, 0}, {0, 1, 1}, {1, 1, 1}},
                                    {{0, 0, 1}, {1, 0, 1}, {0, 1, 1}, {1, 1, 1}}};
        const double eps = 1e-25, ratio = 1e-3, tol = 1e-12;
        for (int ea = 0; ea < 3; ++ea)
            if (geom_in(b, LOC_EXI + ea, G - 1, i, j, k))
            {
                const V3 r0 = gnode(m, i, j, k);
                const V3 r1 = gnode(m, i + d[ea][0], j + d[ea][1], k + d[ea][2]);
                const V3 dr = gsub(r1, r0);
                const double L = gnorm(dr);
                const V3 p00 = geom_dual(m, i + cells[ea][0][0], j + cells[ea][0][1], k + cells[ea][0][2]);
                const V3 p10 = geom_dual(m, i + cells[ea][1][0], j + cells[ea][1][1], k + cells[ea][1][2]);
                const V3 p01 = geom_dual(m, i + cells[ea][2][0], j + cells[ea][2][1], k + cells[ea][2][2]);
                const V3 p11 = geom_dual(m, i + cells[ea][3][0], j + cells[ea][3][1], k + cells[ea][3][2]);
                const V3 Avec = gscale(0.5, gadd(gcross(gsub(p10, p00), gsub(p01, p00)), gcross(gsub(p01, p11), gsub(p10, p11))));
                const double Amag = gnorm(Avec);
                const double alpha_raw = (Amag < eps) ? 0.0 : L / Amag;
                const double d00_10 = gnorm(gsub(p10, p00)), d00_01 = gnorm(gsub(p01, p00));
                const double d10_11 = gnorm(gsub(p11, p10)), d01_11 = gnorm(gsub(p11, p01));
                const double d00_11 = gnorm(gsub(p11, p00)), d10_01 = gnorm(gsub(p01, p10));
                const double href = gmax(gmax(gmax(d00_10, d00_01), gmax(d10_11, d01_11)),
                                         gmax(gmax(d00_11, d10_01), gmax(L, eps)));
                const double side_min = gmin(gmin(d00_10, d00_01), gmin(d10_11, d01_11));
                const double diag_min = gmin(d00_11, d10_01);
                const bool touch = (L < tol) || (side_min < ratio * href) || (diag_min < ratio * href) ||
                                   (Amag < ratio * href * href);
                b.f[F_dlxi + ea][p] = L;
                b.f[F_Astarxi + ea][p] = Amag;
                b.f[F_alphaxi + ea][p] = touch ? 0.0 : alpha_raw;
                double *D = b.f[F_drxi + ea];
                D[p] = dr.x;
                D[v + p] = dr.y;
                D[2 * v + p] = dr.z;
            }
        break;
    }
    case GEOM_WB:
        if (geom_in(b, LOC_CELL, G - 1, i, j, k))
        {
            double *W = b.f[F_WB] + p;
            if (i < 0 || j < 0 || k < 0 || i >= b.ni || j >= b.nj || k >= b.nk)
            {
                for (int q = 0; q < 18; ++q)
                    W[int64_t(q) * v] = 0.0;
                break;
            }
            auto nd = [&](int di, int dj, int dk) { return gnode(m, i + di, j + dj, k + dk); };
            const V3 c = gavg8(nd(0, 0, 0), nd(1, 0, 0), nd(0, 1, 0), nd(1, 1, 0), nd(0, 0, 1), nd(1, 0, 1), nd(0, 1, 1),
                               nd(1, 1, 1));
            const V3 fcs[6] = {gavg4(nd(0, 0, 0), nd(0, 1, 0), nd(0, 0, 1), nd(0, 1, 1)),
                               gavg4(nd(1, 0, 0), nd(1, 1, 0), nd(1, 0, 1), nd(1, 1, 1)),
                               gavg4(nd(0, 0, 0), nd(1, 0, 0), nd(0, 0, 1), nd(1, 0, 1)),
                               gavg4(nd(0, 1, 0), nd(1, 1, 0), nd(0, 1, 1), nd(1, 1, 1)),
                               gavg4(nd(0, 0, 0), nd(1, 0, 0), nd(0, 1, 0), nd(1, 1, 0)),
                               gavg4(nd(0, 0, 1), nd(1, 0, 1), nd(0, 1, 1), nd(1, 1, 1))};
            const V3 S[6] = {gneg(geom_face(m, 0, i, j, k)), geom_face(m, 0, i + 1, j, k),
                             gneg(geom_face(m, 1, i, j, k)), geom_face(m, 1, i, j + 1, k),
                             gneg(geom_face(m, 2, i, j, k)), geom_face(m, 2, i, j, k + 1)};
            double Smag[6], Sref = 0.0;
            for (int f = 0; f < 6; ++f)
            {
                Smag[f] = sqrt(S[f].x * S[f].x + S[f].y * S[f].y + S[f].z * S[f].z);
                Sref = gmax(Sref, Smag[f]);
            }
            const bool valid = !(Sref <= 1e-300);
            double mu[6];
            bool active[6];
            for (int f = 0; f < 6; ++f)
            {
                active[f] = Smag[f] > 1e-10 * Sref;
                mu[f] = active[f] ? 1.0 / gmax(gnorm(gsub(fcs[f], c)), 1e-14) : 0.0;
            }
            geom_pinv_weights<6>(S, mu, active, valid, W, v);
        }
        break;
    case GEOM_WJ:
        if (geom_in(b, LOC_CELL, G - 1, i, j, k))
        {
            double *W = b.f[F_WJ] + p;
            if (i < 0 || j < 0 || k < 0 || i >= b.ni || j >= b.nj || k >= b.nk)
            {
                for (int q = 0; q < 36; ++q)
                    W[int64_t(q) * v] = 0.0;
                break;
            }
            // the 12 cell edges: xi edges, then eta, then zeta (start and end node offsets)
            const int E[12][6] = {{0, 0, 0, 1, 0, 0}, {0, 1, 0, 1, 1, 0}, {0, 0, 1, 1, 0, 1}, {0, 1, 1, 1, 1, 1},
                                  {0, 0, 0, 0, 1, 0}, {1, 0, 0, 1, 1, 0}, {0, 0, 1, 0, 1, 1}, {1, 0, 1, 1, 1, 1},
                                  {0, 0, 0, 0, 0, 1}, {1, 0, 0, 1, 0, 1}, {0, 1, 0, 0, 1, 1}, {1, 1, 0, 1, 1, 1}};
            V3 Lv[12];
            double L[12], Lref = 0.0;
            for (int e = 0; e < 12; ++e)
            {
                Lv[e] = gsub(gnode(m, i + E[e][3], j + E[e][4], k + E[e][5]), gnode(m, i + E[e][0], j + E[e][1], k + E[e][2]));
                L[e] = sqrt(Lv[e].x * Lv[e].x + Lv[e].y * Lv[e].y + Lv[e].z * Lv[e].z);
                Lref = gmax(Lref, L[e]);
            }
            const bool valid = !(Lref <= 1e-300);
            double mu[12];
            bool active[12];
            for (int e = 0; e < 12; ++e)
            {
                active[e] = L[e] > 1e-10 * Lref;
                mu[e] = active[e] ? 1.0 : 0.0;
            }
            geom_pinv_weights<12>(Lv, mu, active, valid, W, v);
        }
        break;
    case GEOM_BADD:
        for (int fa = 0; fa < 3; ++fa)
            if (geom_in(b, LOC_FXI + fa, G, i, j, k))
            {
                const double *F = b.f[F_JDxi + fa];
                b.f[F_Baddxi + fa][p] = (gb[0] * F[p] + gb[1] * F[v + p]) + gb[2] * F[2 * v + p];
            }
        break;
    default:
        break;
    }
}

} // namespace mhd
