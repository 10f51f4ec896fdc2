// Pole handlers and repairs of eta Poles (a block face j = 0, direction -2,
// or j = n_j, direction +2, whose ring runs around the k direction), as
// per-thread work shared by the device kernel k_pole and host builds of the
// same code: each operation works on the pole ring of the first inner layer,
// and sums over a ring run in k order in one work item, as in the reference.
#pragma once

#include <cmath>
#include <cstdint>

#include "mhd_layout.cuh"

namespace mhd
{

enum PoleOp : int
{
    POLE_RING_U = 0, // U_H: k average of the first cell layer
    POLE_RING_BXI,   // B_xi: k average of the first layer
    POLE_BCELL,      // B_cell and Bind_cell: least-squares collapse of the ring
    POLE_EXI_AXIS,   // E_xi on the pole line: -u_plus x B_cell . dr_xi
    POLE_EETA_REG,   // E_eta: regulation of the ring by one Cartesian vector
    POLE_JETA,       // J_eta: (dl / A*) times the circulation of beta_zeta B_zeta
    POLE_BZETA,      // B_zeta of the first cell layer: flux of Bind_cell
    POLE_JCELL,      // J_cell of the first cell layer: least-squares ring vector
    POLE_DIVB,       // divB of the first cell layer: 0
    POLE_ERES_REG,   // Eres_eta: the regulation of POLE_EETA_REG on the resistive edge EMF
    NPOLE_OP
};

// work items one Pole of a block with (ni, nj, nk) cells needs for an operation
__host__ __device__ inline int64_t pole_work(int op, int ni, int nk)
{
    switch (op)
    {
    case POLE_RING_U:
        return int64_t(ni) * 5;
    case POLE_RING_BXI:
    case POLE_EETA_REG:
    case POLE_ERES_REG:
        return ni + 1;
    case POLE_BCELL:
        return int64_t(ni) * 2;
    case POLE_EXI_AXIS:
    case POLE_BZETA:
        return int64_t(ni) * (nk + 1);
    case POLE_JETA:
        return int64_t(ni + 1) * (nk + 1);
    case POLE_JCELL:
        return ni;
    case POLE_DIVB:
        return int64_t(ni) * nk;
    default:
        return 0;
    }
}

// Gauss-Jordan elimination with partial pivoting on [A | b] (the 3x3 solve of
// Z4_Lunar/src/boundary/Boundary_Condition.cpp:244-292,
// Boundary_Condition_EM.cpp:107-165, Z4_Lunar/src/physics/LunarSolver_Tools.cpp:894-944);
// false when a pivot falls below 1e-300
__host__ __device__ inline bool pole_solve3(const double A[3][3], const double b[3], double x[3])
{
    double M[3][4];
#pragma unroll
    for (int r = 0; r < 3; ++r)
    {
        M[r][0] = A[r][0];
        M[r][1] = A[r][1];
        M[r][2] = A[r][2];
        M[r][3] = b[r];
    }
    for (int c = 0; c < 3; ++c)
    {
        int piv = c;
        double amax = fabs(M[c][c]);
        for (int r0 = c + 1; r0 < 3; ++r0)
        {
            const double av = fabs(M[r0][c]);
            if (av > amax)
            {
                amax = av;
                piv = r0;
            }
        }
        if (amax < 1.0e-300)
            return false;
        if (piv != c)
            for (int q = c; q < 4; ++q)
            {
                const double t = M[c][q];
                M[c][q] = M[piv][q];
                M[piv][q] = t;
            }
        const double inv = 1.0 / M[c][c];
        for (int q = c; q < 4; ++q)
            M[c][q] *= inv;
        for (int r0 = 0; r0 < 3; ++r0)
        {
            if (r0 == c)
                continue;
            const double fac = M[r0][c];
            for (int q = c; q < 4; ++q)
                M[r0][q] -= fac * M[c][q];
        }
    }
    x[0] = M[0][3];
    x[1] = M[1][3];
    x[2] = M[2][3];
    return true;
}

// A += s s^T, b += phi s
__host__ __device__ inline void pole_push(double A[3][3], double b[3], const double s[3], double phi)
{
#pragma unroll
    for (int a = 0; a < 3; ++a)
    {
        b[a] += phi * s[a];
#pragma unroll
        for (int c = 0; c < 3; ++c)
            A[a][c] += s[a] * s[c];
    }
}

__host__ __device__ inline double pole_max1(double t)
{
    return (1.0 < t) ? t : 1.0; // std::max(1.0, t)
}

// work item t of operation op on the Pole of block b on side -1 (j = 0) or
// +1 (j = n_j); items past pole_work do nothing
__host__ __device__ inline void pole_one(const BlockView &b, int side, int op, int64_t t)
{
    const int ni = b.ni, nj = b.nj, nk = b.nk;
    if (t < 0 || t >= pole_work(op, ni, nk))
        return;
    const int64_t v = b.vol;
    const int jc = side < 0 ? 0 : nj - 1; // first cell layer (and j-cell-centred fields)
    switch (op)
    {
    case POLE_RING_U: // BC_Pole_Cell_ (Z4_Lunar/src/boundary/Boundary_Condition_Fluid.cpp:186-219)
    case POLE_RING_BXI: // axis faces of BC_Pole_Bface_Collapse_ (Boundary_Condition_EM.cpp:620-670)
    {
        const bool u = op == POLE_RING_U;
        const int i = u ? int(t / 5) : int(t);
        const int m = u ? int(t % 5) : 0;
        double *F = b.f[u ? F_U : F_Bxi] + int64_t(m) * v;
        double acc = 0.0;
        for (int k = 0; k < nk; ++k)
            acc = acc + F[pidx(b, i, jc, k)];
        const double avg = acc / double(nk);
        for (int k = 0; k < nk; ++k)
            F[pidx(b, i, jc, k)] = avg;
        break;
    }
    case POLE_BCELL: // BC_Pole_Bcell_Collapse_, eta Pole (Boundary_Condition_EM.cpp:3-380)
    {
        const int i = int(t >> 1);
        const bool total = (t & 1) == 0;
        const int jn = side < 0 ? jc + 1 : jc; // outer eta face of the ring
        const double sn = side < 0 ? 1.0 : -1.0;
        const double *Aet = b.f[F_JDeta], *Axi = b.f[F_JDxi];
        const double *Bet = b.f[F_Beta], *Bxi = b.f[F_Bxi], *Aadd = b.f[F_Baddeta], *Xadd = b.f[F_Baddxi];
        double A[3][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
        double rhs[3] = {0.0, 0.0, 0.0};
        auto push = [&](const double S[3], double phi) {
            const double sn2 = S[0] * S[0] + S[1] * S[1] + S[2] * S[2];
            if (sn2 <= 1.0e-300)
                return;
            pole_push(A, rhs, S, phi);
        };
        for (int k = 0; k < nk; ++k)
        {
            const int64_t pn = pidx(b, i, jn, k), p0 = pidx(b, i, jc, k), p1 = pidx(b, i + 1, jc, k);
            {
                const double S[3] = {sn * Aet[pn], sn * Aet[v + pn], sn * Aet[2 * v + pn]};
                double f = Bet[pn];
                if (total)
                    f += Aadd[pn];
                push(S, sn * f);
            }
            {
                const double S[3] = {-Axi[p0], -Axi[v + p0], -Axi[2 * v + p0]};
                double f = Bxi[p0];
                if (total)
                    f += Xadd[p0];
                push(S, -f);
            }
            {
                const double S[3] = {Axi[p1], Axi[v + p1], Axi[2 * v + p1]};
                double f = Bxi[p1];
                if (total)
                    f += Xadd[p1];
                push(S, f);
            }
        }
        const double tr = fabs(A[0][0]) + fabs(A[1][1]) + fabs(A[2][2]);
        const double reg = 1.0e-12 * pole_max1(tr);
        A[0][0] += reg;
        A[1][1] += reg;
        A[2][2] += reg;
        double Bp[3];
        if (!pole_solve3(A, rhs, Bp))
            break;
        double *Out = b.f[total ? F_Bcell : F_Bind];
        for (int k = 0; k < nk; ++k)
        {
            const int64_t p = pidx(b, i, jc, k);
            Out[p] = Bp[0];
            Out[v + p] = Bp[1];
            Out[2 * v + p] = Bp[2];
        }
        break;
    }
    case POLE_EXI_AXIS: // BC_Pole_Eedge_Axis, E_xi on an eta Pole (Boundary_Condition.cpp:27-164)
    {
        const int i = int(t / (nk + 1)), k = int(t % (nk + 1));
        const int jn = side < 0 ? 0 : nj; // the pole line (node plane)
        const int64_t pc = pidx(b, i, jc, k), pe = pidx(b, i, jn, k);
        const double *Up = b.f[F_Uplus], *Bc = b.f[F_Bcell], *dr = b.f[F_drxi];
        const double ux = Up[pc], uy = Up[v + pc], uz = Up[2 * v + pc];
        const double Bx = Bc[pc], By = Bc[v + pc], Bz = Bc[2 * v + pc];
        const double E0 = -(uy * Bz - uz * By), E1 = -(uz * Bx - ux * Bz), E2 = -(ux * By - uy * Bx);
        b.f[F_Exi][pe] = E0 * dr[pe] + E1 * dr[v + pe] + E2 * dr[2 * v + pe];
        break;
    }
    case POLE_EETA_REG: // BC_Pole_Eedge_RegulateK_Norm, E_eta on an eta Pole (Boundary_Condition.cpp:179-477)
    case POLE_ERES_REG: // ... and Eres_eta (Boundary_Build.cpp:218-226)
    {
        const int i = int(t);
        double *E = b.f[op == POLE_ERES_REG ? F_Ereseta : F_Eeta];
        const double *dr = b.f[F_dreta];
        double A[3][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
        double rhs[3] = {0.0, 0.0, 0.0};
        int cnt = 0;
        for (int k = 0; k < nk; ++k) // k = n_k is the same edge as k = 0
        {
            const int64_t p = pidx(b, i, jc, k);
            const double d0 = dr[p], d1 = dr[v + p], d2 = dr[2 * v + p];
            const double L = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
            if (L < 1.0e-14)
                continue;
            const double invL = 1.0 / L;
            const double tau[3] = {d0 * invL, d1 * invL, d2 * invL};
            pole_push(A, rhs, tau, E[p] * invL);
            ++cnt;
        }
        if (cnt <= 0)
        {
            for (int k = 0; k <= nk; ++k)
                E[pidx(b, i, jc, k)] = 0.0;
            break;
        }
        const double trA = A[0][0] + A[1][1] + A[2][2];
        const double reg = 1.0e-12 * pole_max1(trA);
        A[0][0] += reg;
        A[1][1] += reg;
        A[2][2] += reg;
        double Ev[3];
        if (!pole_solve3(A, rhs, Ev))
        {
            double avg = 0.0;
            for (int k = 0; k <= nk; ++k)
                avg += E[pidx(b, i, jc, k)];
            avg /= double(nk + 1);
            for (int k = 0; k <= nk; ++k)
                E[pidx(b, i, jc, k)] = avg;
            break;
        }
        for (int k = 0; k <= nk; ++k)
        {
            const int64_t p = pidx(b, i, jc, k);
            const double d0 = dr[p], d1 = dr[v + p], d2 = dr[2 * v + p];
            const double L = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
            E[p] = (L < 1.0e-14) ? 0.0 : Ev[0] * d0 + Ev[1] * d1 + Ev[2] * d2;
        }
        break;
    }
    case POLE_JETA: // BC_Pole_Jedge_RegulateK_Norm, J_eta on an eta Pole (Boundary_Condition.cpp:478-548)
    {
        const int i = int(t / (nk + 1)), k = int(t % (nk + 1));
        const int64_t p = pidx(b, i, jc, k), pm = pidx(b, i - 1, jc, k);
        const double *bz = b.f[F_betazeta], *Bz = b.f[F_Bzeta];
        const double circ = bz[pm] * Bz[pm] - bz[p] * Bz[p];
        const double Ast = b.f[F_Astareta][p];
        const double dl = b.f[F_dleta][p];
        b.f[F_Jeta][p] = (fabs(Ast) <= 1.0e-300) ? 0.0 : (dl / Ast) * circ;
        break;
    }
    case POLE_BZETA: // calc_Bcell after Sync("B_cell") (LunarSolver_Tools.cpp:242-307)
    {
        const int i = int(t / (nk + 1)), k = int(t % (nk + 1));
        const int64_t p = pidx(b, i, jc, k);
        const double *Bi = b.f[F_Bind], *Az = b.f[F_JDzeta];
        b.f[F_Bzeta][p] = Bi[p] * Az[p] + Bi[v + p] * Az[v + p] + Bi[2 * v + p] * Az[2 * v + p];
        break;
    }
    case POLE_JCELL: // the pole-shell least squares of calc_Jcell (LunarSolver_Tools.cpp:945-1090)
    {
        const int i = int(t);
        const int jt = side < 0 ? jc + 1 : jc; // node plane one layer away from the Pole
        double A[3][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
        double rhs[3] = {0.0, 0.0, 0.0};
        int cnt = 0;
        auto push = [&](int fJ, int fdr, int ii, int jj, int kk) {
            const int64_t p = pidx(b, ii, jj, kk);
            const double *dr = b.f[fdr];
            const double dx = dr[p], dy = dr[v + p], dz = dr[2 * v + p];
            const double L = sqrt(dx * dx + dy * dy + dz * dz);
            if (L < 1.0e-14)
                return;
            const double tau[3] = {dx / L, dy / L, dz / L};
            pole_push(A, rhs, tau, b.f[fJ][p] / L);
            ++cnt;
        };
        for (int k = 0; k < nk; ++k)
        {
            push(F_Jeta, F_dreta, i, jc, k);
            push(F_Jeta, F_dreta, i + 1, jc, k);
            push(F_Jeta, F_dreta, i, jc, k + 1);
            push(F_Jeta, F_dreta, i + 1, jc, k + 1);
            push(F_Jxi, F_drxi, i, jt, k);
            push(F_Jxi, F_drxi, i, jt, k + 1);
            push(F_Jzeta, F_drzeta, i, jt, k);
            push(F_Jzeta, F_drzeta, i + 1, jt, k);
        }
        if (cnt <= 0)
            break;
        const double trA = A[0][0] + A[1][1] + A[2][2];
        const double reg = 1.0e-12 * pole_max1(trA);
        A[0][0] += reg;
        A[1][1] += reg;
        A[2][2] += reg;
        double Jp[3];
        if (!pole_solve3(A, rhs, Jp))
            break;
        double *Jc = b.f[F_Jcell];
        for (int k = 0; k < nk; ++k)
        {
            const int64_t p = pidx(b, i, jc, k);
            Jc[p] = Jp[0];
            Jc[v + p] = Jp[1];
            Jc[2 * v + p] = Jp[2];
        }
        break;
    }
    case POLE_DIVB: // calc_divB's zeroing next to a Pole (LunarSolver_Tools.cpp:729-772)
    {
        const int i = int(t / nk), k = int(t % nk);
        b.f[F_divB][pidx(b, i, jc, k)] = 0.0;
        break;
    }
    default:
        break;
    }
}

} // namespace mhd
