// FP64 hot-path kernels for sm_100a.
//
// Each kernel evaluates one stage of LunarSolver::StepOnce with the same
// floating-point operation order as the reference's loops; this translation
// unit is compiled with -fmad=false so that no multiply-add is contracted,
// and the results agree with the reference bit for bit.  The stencils are
// HBM-bound (about 1-3 flop per byte), so they run on the CUDA cores with
// coalesced k-fastest accesses; no tensor cores are involved.
#include "mhd_kernels.cuh"

#include <cfloat>
#include <cmath>

namespace mhd
{

// std::max / std::min semantics (return the first argument unless the
// second compares greater / smaller), which differ from fmax on NaN.
__device__ __forceinline__ double smax(double a, double b) { return (a < b) ? b : a; }
__device__ __forceinline__ double smin(double a, double b) { return (b < a) ? b : a; }

__device__ __forceinline__ double at(const BlockView &b, int f, int m, int i, int j, int k)
{
    return b.f[f][m * b.vol + pidx(b, i, j, k)];
}

// Thread -> (block, i, j, k) over a box [lo, lo + n) with k fastest.
__device__ __forceinline__ bool box_point(const int lo[3], const int n[3], int64_t t, int &i, int &j, int &k)
{
    const int64_t tot = int64_t(n[0]) * n[1] * n[2];
    if (t >= tot)
        return false;
    k = lo[2] + int(t % n[2]);
    t /= n[2];
    j = lo[1] + int(t % n[1]);
    i = lo[0] + int(t / n[1]);
    return true;
}

// Box of a location on block b: inner range [0, n + plus) widened by g.
__device__ __forceinline__ void loc_box(const BlockView &b, int loc, int g, int lo[3], int n[3])
{
    int pi, pj, pk;
    loc_plus(loc, pi, pj, pk);
    lo[0] = lo[1] = lo[2] = -g;
    n[0] = b.ni + pi + 2 * g;
    n[1] = b.nj + pj + 2 * g;
    n[2] = b.nk + pk + 2 * g;
}

// ---------------------------------------------------------------------------
// Scheme_U_ + AddSourceToRHS_Fluid
// (Z4_Lunar/src/physics/LunarSolver_FluidRHS.cpp:3-201, :528-568)
// ---------------------------------------------------------------------------

// One Rusanov face flux (Reconstruction_Rusanov, piecewise-constant states).
// The sound speed sqrt(max(0, gamma p / max(rho, 1e-30))) and the total
// energy p / (gamma - 1) + rho |u|^2 / 2 of each cell, and the face area
// |k|, are the reference's expressions evaluated once (k_pv_uplus_dt,
// k_face_normals) instead of once per face side; the values are identical.
__device__ __forceinline__ void rusanov_face(const BlockView &b, const Consts &c, int dir, int i, int j, int k,
                                             double out[5])
{
    const int JD = (dir == 0) ? F_JDxi : (dir == 1) ? F_JDeta : F_JDzeta;
    const int64_t p = pidx(b, i, j, k);
    const double k1 = b.f[JD][p];
    const double k2 = b.f[JD][b.vol + p];
    const double k3 = b.f[JD][2 * b.vol + p];
    const double area = b.f[F_NAxi + dir][p];
    const int iL = i - (dir == 0), jL = j - (dir == 1), kL = k - (dir == 2);
    const int64_t pL = pidx(b, iL, jL, kL);
    const double *U = b.f[F_U];
    const double *PV = b.f[F_PV];
    const int64_t v = b.vol;

    const double rhoL = U[pL], uL = PV[pL], vL = PV[v + pL], wL = PV[2 * v + pL], pLp = PV[3 * v + pL];
    const double rhoR = U[p], uR = PV[p], vR = PV[v + p], wR = PV[2 * v + p], pR = PV[3 * v + p];
    const double rhoeL = b.f[F_RhoE][pL], rhoeR = b.f[F_RhoE][p];
    const double cL = b.f[F_Cs][pL], cR = b.f[F_Cs][p];

    double UL[5], UR[5];
    UL[0] = rhoL;
    UL[1] = rhoL * uL;
    UL[2] = rhoL * vL;
    UL[3] = rhoL * wL;
    UL[4] = rhoeL;
    UR[0] = rhoR;
    UR[1] = rhoR * uR;
    UR[2] = rhoR * vR;
    UR[3] = rhoR * wR;
    UR[4] = rhoeR;

    const double uvwL = k1 * uL + k2 * vL + k3 * wL;
    const double uvwR = k1 * uR + k2 * vR + k3 * wR;
    const double radL = fabs(uvwL) + cL * area;
    const double radR = fabs(uvwR) + cR * area;
    const double rad = smax(radL, radR);

    double FL[5], FR[5];
    FL[0] = rhoL * uvwL;
    FL[1] = rhoL * uvwL * uL + k1 * pLp;
    FL[2] = rhoL * uvwL * vL + k2 * pLp;
    FL[3] = rhoL * uvwL * wL + k3 * pLp;
    FL[4] = uvwL * (rhoeL + pLp);
    FR[0] = rhoR * uvwR;
    FR[1] = rhoR * uvwR * uR + k1 * pR;
    FR[2] = rhoR * uvwR * vR + k2 * pR;
    FR[3] = rhoR * uvwR * wR + k3 * pR;
    FR[4] = uvwR * (rhoeR + pR);
#pragma unroll
    for (int m = 0; m < 5; ++m)
        out[m] = 0.5 * (FL[m] + FR[m]) - 0.5 * rad * (UR[m] - UL[m]);
}

// |JD| and JD / |JD| of every face (geometry; once per set-up)
__global__ void k_face_normals(const BlockView *__restrict__ bvs)
{
    const BlockView &b = bvs[blockIdx.y];
    const int fa = blockIdx.z;
    int lo[3], n[3];
    loc_box(b, LOC_FXI + fa, b.G, lo, n);
    int i, j, k;
    if (!box_point(lo, n, int64_t(blockIdx.x) * blockDim.x + threadIdx.x, i, j, k))
        return;
    const int64_t p = pidx(b, i, j, k);
    const int64_t v = b.vol;
    const double *M = b.f[F_JDxi + fa];
    const double ax = M[p], ay = M[v + p], az = M[2 * v + p];
    const double A = sqrt(ax * ax + ay * ay + az * az);
    double *N = b.f[F_NAxi + fa];
    N[p] = A;
    N[v + p] = ax / A;
    N[2 * v + p] = ay / A;
    N[3 * v + p] = az / A;
}

__device__ __forceinline__ void fluid_one(const BlockView &b, const Consts &c, int i, int j, int k)
{
    const int64_t p = pidx(b, i, j, k);
    const int64_t v = b.vol;
    double Fm[5], Fp[5];
    double r[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    const double invJ = 1.0 / b.f[F_Jac][p];

    // each component takes its three flux differences in the reference's
    // order, r -= dx / J, r -= dy / J, r -= dz / J; they are applied as each
    // direction completes (the same operations per component), so no
    // direction's differences stay live
    rusanov_face(b, c, 0, i, j, k, Fm);
    rusanov_face(b, c, 0, i + 1, j, k, Fp);
#pragma unroll
    for (int m = 0; m < 5; ++m)
        r[m] -= (Fp[m] - Fm[m]) * invJ;
    rusanov_face(b, c, 1, i, j, k, Fm);
    rusanov_face(b, c, 1, i, j + 1, k, Fp);
#pragma unroll
    for (int m = 0; m < 5; ++m)
        r[m] -= (Fp[m] - Fm[m]) * invJ;
    rusanov_face(b, c, 2, i, j, k, Fm);
    rusanov_face(b, c, 2, i, j, k + 1, Fp);
#pragma unroll
    for (int m = 0; m < 5; ++m)
        r[m] -= (Fp[m] - Fm[m]) * invJ;

    // J x B force with the Hall_Num_Limiter weight (LunarSolver_Tools.cpp:47-56)
    const double rho = b.f[F_U][p];
    const double n_true = smax(rho, 0.0) / c.M_H * c.M_ref;
    const double ne_eff = sqrt(n_true * n_true + c.ne_floor * c.ne_floor);
    const double w = n_true / ne_eff;
    const double fc = c.mom_hall * w;
    const double *J = b.f[F_Jcell];
    const double *B = b.f[F_Bcell];
    const double jx = J[p], jy = J[v + p], jz = J[2 * v + p];
    const double bx = B[p], by = B[v + p], bz = B[2 * v + p];
    const double jxb_x = jy * bz - jz * by;
    const double jxb_y = jz * bx - jx * bz;
    const double jxb_z = jx * by - jy * bx;
    const double *PV = b.f[F_PV];
    r[1] += fc * jxb_x;
    r[2] += fc * jxb_y;
    r[3] += fc * jxb_z;
    r[4] += fc * (jxb_x * PV[p] + jxb_y * PV[v + p] + jxb_z * PV[2 * v + p]);

    double *R = b.f[F_RHS];
#pragma unroll
    for (int m = 0; m < 5; ++m)
        R[m * v + p] = r[m];
}

__global__ void k_fluid_rhs(const BlockView *__restrict__ bvs, Consts c, int64_t /*maxpts*/)
{
    const BlockView &b = bvs[blockIdx.y];
    int lo[3], n[3];
    loc_box(b, LOC_CELL, 0, lo, n);
    int i, j, k;
    if (!box_point(lo, n, int64_t(blockIdx.x) * blockDim.x + threadIdx.x, i, j, k))
        return;
    fluid_one(b, c, i, j, k);
}

// ---------------------------------------------------------------------------
// AssembleOneDirectionEMF_ (Z4_Lunar/src/physics/LunarSolver_MagExplicit_Ideal.cpp:348-496)
// ---------------------------------------------------------------------------

__device__ __forceinline__ double face_ind(const BlockView &b, int axis, int i, int j, int k)
{
    const int F = (axis == 0) ? F_Bxi : (axis == 1) ? F_Beta : F_Bzeta;
    return b.f[F][pidx(b, i, j, k)];
}
__device__ __forceinline__ double face_tot(const BlockView &b, int axis, int i, int j, int k)
{
    const int F = (axis == 0) ? F_Bxi : (axis == 1) ? F_Beta : F_Bzeta;
    const int A = (axis == 0) ? F_Baddxi : (axis == 1) ? F_Baddeta : F_Baddzeta;
    const int64_t p = pidx(b, i, j, k);
    return b.f[F][p] + b.f[A][p];
}
// contravariant velocity of a cell along `axis` (cell_u_contra,
// LunarSolver_MagExplicit_Ideal.cpp:95-115)
__device__ __forceinline__ double u_contra(const BlockView &b, int axis, int i, int j, int k)
{
    const int JD = (axis == 0) ? F_JDxi : (axis == 1) ? F_JDeta : F_JDzeta;
    const int64_t p = pidx(b, i, j, k);
    const int64_t q = pidx(b, i + (axis == 0), j + (axis == 1), k + (axis == 2));
    const int64_t v = b.vol;
    const double *M = b.f[JD];
    const double kx = 0.5 * (M[p] + M[q]);
    const double ky = 0.5 * (M[v + p] + M[v + q]);
    const double kz = 0.5 * (M[2 * v + p] + M[2 * v + q]);
    const double inv_jac = 1.0 / (fabs(b.f[F_Jac][p]) + 1.0e-30);
    const double *Up = b.f[F_Uplus];
    return (kx * Up[p] + ky * Up[v + p] + kz * Up[2 * v + p]) * inv_jac;
}

// the three contravariant velocities of every cell within one layer of the
// inner range, stored once per step instead of being recomputed by every
// face and edge stencil that needs them (up to eight times per point)
__global__ void k_ucontra(const BlockView *__restrict__ bvs)
{
    const BlockView &b = bvs[blockIdx.y];
    int lo[3], n[3];
    loc_box(b, LOC_CELL, 1, lo, n);
    int i, j, k;
    if (!box_point(lo, n, int64_t(blockIdx.x) * blockDim.x + threadIdx.x, i, j, k))
        return;
    const int64_t p = pidx(b, i, j, k);
    double *UC = b.f[F_UC];
    UC[p] = u_contra(b, 0, i, j, k);
    UC[b.vol + p] = u_contra(b, 1, i, j, k);
    UC[2 * b.vol + p] = u_contra(b, 2, i, j, k);
}

// the fluid RHS of the inner cells and the contravariant velocities of the
// cells within one ghost layer in one pass (both read JD and Jac around the
// same cells; U_contra is read only by the EMF kernels that follow)
__device__ __forceinline__ void k_fluid_ucontra_body(const BlockView *__restrict__ bvs, Consts c)
{
    int64_t t;
    const BlockView &b = bvs[cta_block(bvs, KIND_CELL1, t)];
    int lo[3], n[3];
    loc_box(b, LOC_CELL, 1, lo, n);
    int i, j, k;
    if (!box_point(lo, n, t, i, j, k))
        return;
    if (i >= 0 && j >= 0 && k >= 0 && i < b.ni && j < b.nj && k < b.nk)
        fluid_one(b, c, i, j, k);
    const int64_t p = pidx(b, i, j, k);
    double *UC = b.f[F_UC];
    UC[p] = u_contra(b, 0, i, j, k);
    UC[b.vol + p] = u_contra(b, 1, i, j, k);
    UC[2 * b.vol + p] = u_contra(b, 2, i, j, k);
}

template <int MINB> __global__ void __launch_bounds__(256, MINB) k_fluid_ucontra_t(const BlockView *__restrict__ bvs, Consts c)
{
    k_fluid_ucontra_body(bvs, c);
}
// the compiler's own register allocation (no launch bounds)
__global__ void k_fluid_ucontra_free(const BlockView *__restrict__ bvs, Consts c)
{
    k_fluid_ucontra_body(bvs, c);
}


// contravariant velocity of a cell, as stored by the fluid pass
__device__ __forceinline__ double uc(const BlockView &b, int axis, int i, int j, int k)
{
    return b.f[F_UC][axis * b.vol + pidx(b, i, j, k)];
}

__device__ __forceinline__ double emf_flux(const BlockView &b, int ba, int fa, int iL, int jL, int kL, int iR, int jR,
                                           int kR, double bff)
{
    const int sa = (ba == 0), sb = (ba == 1), sc = (ba == 2);
    const double btL = 0.5 * (face_tot(b, ba, iL, jL, kL) + face_tot(b, ba, iL + sa, jL + sb, kL + sc));
    const double btR = 0.5 * (face_tot(b, ba, iR, jR, kR) + face_tot(b, ba, iR + sa, jR + sb, kR + sc));
    const double biL = 0.5 * (face_ind(b, ba, iL, jL, kL) + face_ind(b, ba, iL + sa, jL + sb, kL + sc));
    const double biR = 0.5 * (face_ind(b, ba, iR, jR, kR) + face_ind(b, ba, iR + sa, jR + sb, kR + sc));
    const double ufL = uc(b, fa, iL, jL, kL);
    const double ufR = uc(b, fa, iR, jR, kR);
    const double ubL = uc(b, ba, iL, jL, kL);
    const double ubR = uc(b, ba, iR, jR, kR);
    const double GL = ufL * btL - ubL * bff;
    const double GR = ufR * btR - ubR * bff;
    const double radius = smax(fabs(ufL), fabs(ufR));
    return 0.5 * (GL + GR) - 0.5 * radius * (biR - biL);
}

// the two non-zero Eface components of face (i, j, k) of axis fa
__device__ __forceinline__ void eface_one(const BlockView &b, int fa, int i, int j, int k)
{
    const int iL = i - (fa == 0), jL = j - (fa == 1), kL = k - (fa == 2);
    const double bff = face_tot(b, fa, i, j, k);
    double e0 = 0.0, e1 = 0.0, e2 = 0.0;
    if (fa == 0)
    {
        const double G_eta_xi = emf_flux(b, 1, 0, iL, jL, kL, i, j, k, bff);
        const double G_zeta_xi = emf_flux(b, 2, 0, iL, jL, kL, i, j, k, bff);
        e1 = G_zeta_xi;
        e2 = -G_eta_xi;
    }
    else if (fa == 1)
    {
        const double G_xi_eta = emf_flux(b, 0, 1, iL, jL, kL, i, j, k, bff);
        const double G_zeta_eta = emf_flux(b, 2, 1, iL, jL, kL, i, j, k, bff);
        e0 = -G_zeta_eta;
        e2 = G_xi_eta;
    }
    else
    {
        const double G_xi_zeta = emf_flux(b, 0, 2, iL, jL, kL, i, j, k, bff);
        const double G_eta_zeta = emf_flux(b, 1, 2, iL, jL, kL, i, j, k, bff);
        e0 = G_eta_zeta;
        e1 = -G_xi_zeta;
    }
    const int F = F_Efxi + fa;
    const int64_t p = pidx(b, i, j, k);
    b.f[F][p] = e0;
    b.f[F][b.vol + p] = e1;
    b.f[F][2 * b.vol + p] = e2;
}

// Staggered points (i, j, k) of a block in [0, n + 1) per axis, one thread
// each, or in the box rng[6 * block] (lo[3], hi[3], within [0, n + 1)^3)
// when a region table is given; the kernels below handle all three face or
// edge axes of a point in one thread so that the fields they share are read
// once.
__device__ __forceinline__ bool stagger_point(const BlockView &b, const int *rng, int blk, int64_t t, int &i, int &j,
                                              int &k)
{
    int lo[3] = {0, 0, 0};
    int n[3] = {b.ni + 1, b.nj + 1, b.nk + 1};
    if (rng)
    {
        const int *r = rng + 6 * blk;
        for (int a = 0; a < 3; ++a)
        {
            lo[a] = r[a];
            n[a] = r[3 + a] - r[a];
        }
    }
    return box_point(lo, n, t, i, j, k);
}

// is (i, j, k) an inner point of the face (kind 0) or edge (kind 1) axis a
__device__ __forceinline__ bool inner_of(const BlockView &b, int kind, int a, int i, int j, int k)
{
    int pl[3];
    loc_plus((kind == 0 ? LOC_FXI : LOC_EXI) + a, pl[0], pl[1], pl[2]);
    return i < b.ni + pl[0] && j < b.nj + pl[1] && k < b.nk + pl[2];
}

__device__ __forceinline__ void k_eface_body(const BlockView *__restrict__ bvs)
{
    int64_t t;
    const BlockView &b = bvs[cta_block(bvs, KIND_STAG, t)];
    int i, j, k;
    if (!stagger_point(b, nullptr, 0, t, i, j, k))
        return;
#pragma unroll
    for (int fa = 0; fa < 3; ++fa)
        if (inner_of(b, 0, fa, i, j, k))
            eface_one(b, fa, i, j, k);
}

template <int MINB> __global__ void __launch_bounds__(256, MINB) k_eface_t(const BlockView *__restrict__ bvs)
{
    k_eface_body(bvs);
}
// the compiler's own register allocation (no launch bounds)
__global__ void k_eface_free(const BlockView *__restrict__ bvs)
{
    k_eface_body(bvs);
}


// ---------------------------------------------------------------------------
// AssembleEdgeEMF_FromFaceE_Ideal_ (LunarSolver_MagExplicit_Ideal.cpp:53-287)
// with the zeroing of E_edge over the whole array (LunarSolver_MagneticRHS.cpp:9-28)
// ---------------------------------------------------------------------------

__device__ __forceinline__ double max_abs_u4(const BlockView &b, int axis, int i0, int j0, int k0, int i1, int j1,
                                             int k1, int i2, int j2, int k2, int i3, int j3, int k3)
{
    double a = 0.0;
    a = smax(a, fabs(uc(b, axis, i0, j0, k0)));
    a = smax(a, fabs(uc(b, axis, i1, j1, k1)));
    a = smax(a, fabs(uc(b, axis, i2, j2, k2)));
    a = smax(a, fabs(uc(b, axis, i3, j3, k3)));
    return a;
}

// edge EMF of edge (i, j, k) of axis ea (inner edges)
__device__ __forceinline__ double eedge_one(const BlockView &b, int ea, int i, int j, int k)
{
    const double Cuct = 0.5;
    double E = 0.0;
    if (ea == 0)
    {
        const double *Fe = b.f[F_Efeta];
        const double *Fz = b.f[F_Efzeta];
        const double Ec = 0.25 * (Fe[pidx(b, i, j, k)] + Fe[pidx(b, i, j, k - 1)] + Fz[pidx(b, i, j, k)] +
                                  Fz[pidx(b, i, j - 1, k)]);
        const double a_eta = max_abs_u4(b, 1, i, j, k, i, j - 1, k, i, j, k - 1, i, j - 1, k - 1);
        const double a_zeta = max_abs_u4(b, 2, i, j, k, i, j - 1, k, i, j, k - 1, i, j - 1, k - 1);
        const double dBzeta_eta = face_ind(b, 2, i, j, k) - face_ind(b, 2, i, j - 1, k);
        const double dBeta_zeta = face_ind(b, 1, i, j, k) - face_ind(b, 1, i, j, k - 1);
        E = Ec + Cuct * (0.5 * a_eta * dBzeta_eta - 0.5 * a_zeta * dBeta_zeta);
    }
    else if (ea == 1)
    {
        const double *Fx = b.f[F_Efxi];
        const double *Fz = b.f[F_Efzeta];
        const int64_t v = b.vol;
        const double Ec = 0.25 * (Fx[v + pidx(b, i, j, k)] + Fx[v + pidx(b, i, j, k - 1)] +
                                  Fz[v + pidx(b, i, j, k)] + Fz[v + pidx(b, i - 1, j, k)]);
        const double a_zeta = max_abs_u4(b, 2, i, j, k, i - 1, j, k, i, j, k - 1, i - 1, j, k - 1);
        const double a_xi = max_abs_u4(b, 0, i, j, k, i - 1, j, k, i, j, k - 1, i - 1, j, k - 1);
        const double dBxi_zeta = face_ind(b, 0, i, j, k) - face_ind(b, 0, i, j, k - 1);
        const double dBzeta_xi = face_ind(b, 2, i, j, k) - face_ind(b, 2, i - 1, j, k);
        E = Ec + Cuct * (0.5 * a_zeta * dBxi_zeta - 0.5 * a_xi * dBzeta_xi);
    }
    else
    {
        const double *Fx = b.f[F_Efxi];
        const double *Fe = b.f[F_Efeta];
        const int64_t v2 = 2 * b.vol;
        const double Ec = 0.25 * (Fx[v2 + pidx(b, i, j, k)] + Fx[v2 + pidx(b, i, j - 1, k)] +
                                  Fe[v2 + pidx(b, i, j, k)] + Fe[v2 + pidx(b, i - 1, j, k)]);
        const double a_xi = max_abs_u4(b, 0, i, j, k, i - 1, j, k, i, j - 1, k, i - 1, j - 1, k);
        const double a_eta = max_abs_u4(b, 1, i, j, k, i - 1, j, k, i, j - 1, k, i - 1, j - 1, k);
        const double dBeta_xi = face_ind(b, 1, i, j, k) - face_ind(b, 1, i - 1, j, k);
        const double dBxi_eta = face_ind(b, 0, i, j, k) - face_ind(b, 0, i, j - 1, k);
        E = Ec + Cuct * (0.5 * a_xi * dBeta_xi - 0.5 * a_eta * dBxi_eta);
    }
    return E;
}

// inner edges of all three axes; ghost edges keep the zero of
// AssembleRHS_Induction_CT_ except where the Eedge sync writes them
__device__ __forceinline__ void k_eedge_body(const BlockView *__restrict__ bvs)
{
    int64_t t;
    const BlockView &b = bvs[cta_block(bvs, KIND_STAG, t)];
    int i, j, k;
    if (!stagger_point(b, nullptr, 0, t, i, j, k))
        return;
#pragma unroll
    for (int ea = 0; ea < 3; ++ea)
        if (inner_of(b, 1, ea, i, j, k))
            b.f[F_Exi + ea][pidx(b, i, j, k)] = eedge_one(b, ea, i, j, k);
}

template <int MINB> __global__ void __launch_bounds__(256, MINB) k_eedge_t(const BlockView *__restrict__ bvs)
{
    k_eedge_body(bvs);
}
// the compiler's own register allocation (no launch bounds)
__global__ void k_eedge_free(const BlockView *__restrict__ bvs)
{
    k_eedge_body(bvs);
}


// ---------------------------------------------------------------------------
// CTOperators::CurlEdgeToFace (Z4_Lunar/src/operators/CTOperators.cpp:6-56)
// with multiplier `mult`, written to RHS_B, optionally followed by the face
// part of ApplyUpdate_Euler_ (LunarSolver_Advance.cpp:95-121): B += dt*RHS_B.
// ---------------------------------------------------------------------------
// the three inner faces at staggered point (i, j, k): RHS = mult * curl E,
// optionally B += dtB * RHS
__device__ __forceinline__ void curl_point(const BlockView &b, int fE0, int fR0, int fB0, double mult, double dtB,
                                           int i, int j, int k)
{
    const double *Ex = b.f[fE0], *Ee = b.f[fE0 + 1], *Ez = b.f[fE0 + 2];
    const int64_t p = pidx(b, i, j, k);
#pragma unroll
    for (int fa = 0; fa < 3; ++fa)
    {
        if (!inner_of(b, 0, fa, i, j, k))
            continue;
        double curl;
        if (fa == 0)
            curl = (Ee[p] - Ee[pidx(b, i, j, k + 1)]) + (Ez[pidx(b, i, j + 1, k)] - Ez[p]);
        else if (fa == 1)
            curl = (Ex[pidx(b, i, j, k + 1)] - Ex[p]) + (Ez[p] - Ez[pidx(b, i + 1, j, k)]);
        else
            curl = (Ex[p] - Ex[pidx(b, i, j + 1, k)]) + (Ee[pidx(b, i + 1, j, k)] - Ee[p]);
        const double rhs = mult * curl;
        if (fR0 >= 0)
            b.f[fR0 + fa][p] = rhs;
        if (fB0 >= 0)
            b.f[fB0 + fa][p] += dtB * rhs;
    }
}

// The implicit Hall trial's face update from the snapshot B*: on the inner
// faces RHS = mult curl E and B = B* + dt RHS, B* read from its snapshot (bs:
// per block the B*_xi, B*_eta, B*_zeta arrays, in the pool's point layout).
// The same operands and operations as restoring B = B* and then B += dt RHS,
// so the same bits, without the copy.
__global__ void k_curl_from_snapshot(const BlockView *__restrict__ bvs, int fE0, int fR0, int fB0, double mult,
                                     const double *__restrict__ dtp, const double *const *__restrict__ bs)
{
    int64_t t;
    const int bi = cta_block(bvs, KIND_STAG, t);
    const BlockView &b = bvs[bi];
    int i, j, k;
    if (!stagger_point(b, nullptr, 0, t, i, j, k))
        return;
    const double dtB = dtp[b.run] / 1.0;
    const double *Ex = b.f[fE0], *Ee = b.f[fE0 + 1], *Ez = b.f[fE0 + 2];
    const int64_t p = pidx(b, i, j, k);
#pragma unroll
    for (int fa = 0; fa < 3; ++fa)
    {
        if (!inner_of(b, 0, fa, i, j, k))
            continue;
        double curl;
        if (fa == 0)
            curl = (Ee[p] - Ee[pidx(b, i, j, k + 1)]) + (Ez[pidx(b, i, j + 1, k)] - Ez[p]);
        else if (fa == 1)
            curl = (Ex[pidx(b, i, j, k + 1)] - Ex[p]) + (Ez[p] - Ez[pidx(b, i + 1, j, k)]);
        else
            curl = (Ex[p] - Ex[pidx(b, i, j + 1, k)]) + (Ee[pidx(b, i + 1, j, k)] - Ee[p]);
        const double rhs = mult * curl;
        b.f[fR0 + fa][p] = rhs;
        b.f[fB0 + fa][p] = bs[3 * bi + fa][p] + dtB * rhs;
    }
}

// the discrete curl curl_point forms on face axis fa at (i, j, k)
__device__ __forceinline__ double face_curl(const BlockView &b, int fE0, int fa, int i, int j, int k)
{
    const double *Ex = b.f[fE0], *Ee = b.f[fE0 + 1], *Ez = b.f[fE0 + 2];
    const int64_t p = pidx(b, i, j, k);
    if (fa == 0)
        return (Ee[p] - Ee[pidx(b, i, j, k + 1)]) + (Ez[pidx(b, i, j + 1, k)] - Ez[p]);
    if (fa == 1)
        return (Ex[pidx(b, i, j, k + 1)] - Ex[p]) + (Ez[p] - Ez[pidx(b, i + 1, j, k)]);
    return (Ex[p] - Ex[pidx(b, i, j + 1, k)]) + (Ee[pidx(b, i + 1, j, k)] - Ee[p]);
}

__device__ __forceinline__ void k_curl_e2f_body(const BlockView *__restrict__ bvs, int fE0, int fR0, int fB0, double mult,
                           const double *__restrict__ dtp, double dtdiv, int mult_is_neg_dt, const int *__restrict__ rng)
{
    int64_t t;
    const int bi = cta_block(bvs, KIND_STAG, t);
    const BlockView &b = bvs[bi];
    if (mult_is_neg_dt)
        mult = -dtp[b.run];
    int i, j, k;
    if (!stagger_point(b, rng, bi, t, i, j, k))
        return;
    curl_point(b, fE0, fR0, fB0, mult, fB0 >= 0 ? dtp[b.run] / dtdiv : 0.0, i, j, k);
}

template <int MINB> __global__ void __launch_bounds__(256, MINB) k_curl_e2f_t(const BlockView *__restrict__ bvs, int fE0, int fR0, int fB0, double mult,
                           const double *__restrict__ dtp, double dtdiv, int mult_is_neg_dt, const int *__restrict__ rng)
{
    k_curl_e2f_body(bvs, fE0, fR0, fB0, mult, dtp, dtdiv, mult_is_neg_dt, rng);
}
// the compiler's own register allocation (no launch bounds)
__global__ void k_curl_e2f_free(const BlockView *__restrict__ bvs, int fE0, int fR0, int fB0, double mult,
                           const double *__restrict__ dtp, double dtdiv, int mult_is_neg_dt, const int *__restrict__ rng)
{
    k_curl_e2f_body(bvs, fE0, fR0, fB0, mult, dtp, dtdiv, mult_is_neg_dt, rng);
}


// calc_divB on inner cells (Z4_Lunar/src/physics/LunarSolver_Tools.cpp:685-775;
// layouts with Pole patches, whose first shell the reference zeroes, are not
// handled here)
__global__ void k_divb(const BlockView *__restrict__ bvs)
{
    const BlockView &b = bvs[blockIdx.y];
    int lo[3], n[3];
    loc_box(b, LOC_CELL, 0, lo, n);
    int i, j, k;
    if (!box_point(lo, n, int64_t(blockIdx.x) * blockDim.x + threadIdx.x, i, j, k))
        return;
    const int64_t p = pidx(b, i, j, k);
    const double *Bx = b.f[F_Bxi], *Be = b.f[F_Beta], *Bz = b.f[F_Bzeta];
    const double num = Bx[pidx(b, i + 1, j, k)] - Bx[p] + Be[pidx(b, i, j + 1, k)] - Be[p] + Bz[pidx(b, i, j, k + 1)] -
                       Bz[p];
    b.f[F_divB][p] = num / b.f[F_Jac][p];
}

// Explicit resistive edge EMF, AddResistiveEdgeEMF_To_ on a zeroed Eres
// (Z4_Lunar/src/physics/LunarSolver_MagExplicit_Resis.cpp:67-209): on inner
// edges with a non-zero shell profile yita0 (eta_edge_*, from the edge
// midpoint radius), Eres = (inver_Rem yita0) (J_avg . dr) with J_avg the mean
// cell current of the four cells around the edge; zero elsewhere.
__global__ void k_eres_explicit(const BlockView *__restrict__ bvs, double inver_Rem)
{
    int64_t t;
    const BlockView &b = bvs[cta_block(bvs, KIND_STAG, t)];
    int i, j, k;
    if (!stagger_point(b, nullptr, 0, t, i, j, k))
        return;
    const double *Jc = b.f[F_Jcell];
    const int64_t v = b.vol;
    const int64_t p = pidx(b, i, j, k);
#pragma unroll
    for (int ea = 0; ea < 3; ++ea)
    {
        if (!inner_of(b, 1, ea, i, j, k))
            continue;
        const double yita0 = b.f[F_etaxi + ea][p];
        double E = 0.0;
        if (yita0 != 0.0)
        {
            int64_t c[4];
            if (ea == 0)
            {
                c[0] = p;
                c[1] = pidx(b, i, j - 1, k);
                c[2] = pidx(b, i, j, k - 1);
                c[3] = pidx(b, i, j - 1, k - 1);
            }
            else if (ea == 1)
            {
                c[0] = p;
                c[1] = pidx(b, i - 1, j, k);
                c[2] = pidx(b, i, j, k - 1);
                c[3] = pidx(b, i - 1, j, k - 1);
            }
            else
            {
                c[0] = p;
                c[1] = pidx(b, i - 1, j, k);
                c[2] = pidx(b, i, j - 1, k);
                c[3] = pidx(b, i - 1, j - 1, k);
            }
            double Jx = 0.0, Jy = 0.0, Jz = 0.0;
#pragma unroll
            for (int q = 0; q < 4; ++q)
            {
                Jx += Jc[c[q]];
                Jy += Jc[v + c[q]];
                Jz += Jc[2 * v + c[q]];
            }
            Jx *= 0.25;
            Jy *= 0.25;
            Jz *= 0.25;
            const double *dr = b.f[F_drxi + ea];
            const double Jedge = Jx * dr[p] + Jy * dr[v + p] + Jz * dr[2 * v + p];
            E = 0.0 + (inver_Rem * yita0) * Jedge;
        }
        b.f[F_Eresxi + ea][p] = E;
    }
}

// ---------------------------------------------------------------------------
// Hall edge EMF, BuildHallFaceEMF_Rusanov_diff_
// (Z4_Lunar/src/physics/LunarSolver_MagExplicit_Hall.cpp:8-457)
// ---------------------------------------------------------------------------

// Ehc = alpha (J x B) and beta = |alpha| |B| on every cell of the array, with
// alpha = hall_coef / ne_eff (Hall_Num_Limiter)
__global__ void k_hall_cell(const BlockView *__restrict__ bvs, Consts c, double hall_coef)
{
    const BlockView &b = bvs[blockIdx.y];
    int lo[3], n[3];
    loc_box(b, LOC_CELL, b.G, lo, n);
    int i, j, k;
    if (!box_point(lo, n, int64_t(blockIdx.x) * blockDim.x + threadIdx.x, i, j, k))
        return;
    const int64_t p = pidx(b, i, j, k);
    const int64_t v = b.vol;
    const double n_true = smax(b.f[F_U][p], 0.0) / c.M_H * c.M_ref;
    const double ne = sqrt(n_true * n_true + c.ne_floor * c.ne_floor);
    const double alpha = hall_coef / ne;
    const double *J = b.f[F_Jcell], *B = b.f[F_Bcell];
    const double Jx = J[p], Jy = J[v + p], Jz = J[2 * v + p];
    const double Bx = B[p], By = B[v + p], Bz = B[2 * v + p];
    double *E = b.f[F_Ehc];
    E[p] = alpha * (Jy * Bz - Jz * By);
    E[v + p] = alpha * (Jz * Bx - Jx * Bz);
    E[2 * v + p] = alpha * (Jx * By - Jy * Bx);
    b.f[F_HallBeta][p] = fabs(alpha) * sqrt(Bx * Bx + By * By + Bz * Bz);
}

// one inner edge of axis ea: 4-cell mean of Ehc along dr, minus the
// whistler diffusion of the two face-B jumps across the edge.  E[q][c] and
// be[q] are the Ehc components and beta of the edge's four cells, in the
// order the reference sums them.
__device__ __forceinline__ double hall_edge_one(const BlockView &b, int ea, int i, int j, int k, const double (&E)[4][3],
                                                const double (&be)[4])
{
    const double eps = 1e-14, Cwh = 0.1;
    const int64_t v = b.vol;
    const int64_t p = pidx(b, i, j, k);
    int Fm, Fp, Am, Ap;
    int64_t qm, qp, am, ap;
    if (ea == 0)
    {
        Fm = F_Bzeta, qm = pidx(b, i, j - 1, k), Fp = F_Beta, qp = pidx(b, i, j, k - 1);
        Am = F_Areazeta, am = pidx(b, i, j - 1, k), Ap = F_Areaeta, ap = pidx(b, i, j, k - 1);
    }
    else if (ea == 1)
    {
        Fm = F_Bxi, qm = pidx(b, i, j, k - 1), Fp = F_Bzeta, qp = pidx(b, i - 1, j, k);
        Am = F_Areaxi, am = pidx(b, i, j, k - 1), Ap = F_Areazeta, ap = pidx(b, i - 1, j, k);
    }
    else
    {
        Fm = F_Beta, qm = pidx(b, i - 1, j, k), Fp = F_Bxi, qp = pidx(b, i, j - 1, k);
        Am = F_Areaeta, am = pidx(b, i - 1, j, k), Ap = F_Areaxi, ap = pidx(b, i, j - 1, k);
    }
    const double Ecx = 0.25 * (E[0][0] + E[1][0] + E[2][0] + E[3][0]);
    const double Ecy = 0.25 * (E[0][1] + E[1][1] + E[2][1] + E[3][1]);
    const double Ecz = 0.25 * (E[0][2] + E[1][2] + E[2][2] + E[3][2]);
    const double *dr = b.f[F_drxi + ea];
    const double Ecen = Ecx * dr[p] + Ecy * dr[v + p] + Ecz * dr[2 * v + p];
    const double beta_e = smax(smax(be[0], be[1]), smax(be[2], be[3]));
    const double L = smax(b.f[F_dlxi + ea][p], eps);
    const double Abar_m = 0.5 * (b.f[Am][p] + b.f[Am][am]);
    const double inv_m = L / smax(Abar_m, eps);
    const double mu_m = Cwh * beta_e * inv_m * inv_m;
    const double Abar_p = 0.5 * (b.f[Ap][p] + b.f[Ap][ap]);
    const double inv_p = L / smax(Abar_p, eps);
    const double mu_p = Cwh * beta_e * inv_p * inv_p;
    const double dB_m = b.f[Fm][p] - b.f[Fm][qm];
    const double dB_p = b.f[Fp][p] - b.f[Fp][qp];
    return Ecen - 0.5 * mu_m * dB_m + 0.5 * mu_p * dB_p;
}

// zero box test of the Hall edge EMF (Solid_Surface layers and Pole edges)
__device__ __forceinline__ bool hall_zeroed(const int *__restrict__ zb, int nzb, int bi, int ea, int i, int j, int k)
{
    bool zero = false;
    for (int q = 0; q < nzb && !zero; ++q)
    {
        const int *z = zb + 8 * q;
        zero = (z[0] == bi && z[1] == ea && i >= z[2] && j >= z[3] && k >= z[4] && i < z[5] && j < z[6] && k < z[7]);
    }
    return zero;
}

// the four cells of each edge axis, in the reference's order, as offsets
// into the seven cells around a staggered point: 0 (0,0,0), 1 (0,-1,0),
// 2 (0,0,-1), 3 (0,-1,-1), 4 (-1,0,0), 5 (-1,0,-1), 6 (-1,-1,0) (a
// compile-time table: every use sits in a fully unrolled loop)
__device__ __forceinline__ constexpr int hall_cells(int ea, int q)
{
    return ea == 0 ? (q == 0 ? 3 : q == 1 ? 1 : q == 2 ? 2 : 0)
                   : ea == 1 ? (q == 0 ? 5 : q == 1 ? 4 : q == 2 ? 2 : 0) : (q == 0 ? 6 : q == 1 ? 4 : q == 2 ? 1 : 0);
}

__device__ __forceinline__ int64_t hall_cell_of(const BlockView &b, int q, int i, int j, int k)
{
    const int di = (q >= 4) ? -1 : 0;
    const int dj = (q == 1 || q == 3 || q == 6) ? -1 : 0;
    const int dk = (q == 2 || q == 3 || q == 5) ? -1 : 0;
    return pidx(b, i + di, j + dj, k + dk);
}

// one inner edge of axis ea, its cells read here: 4-cell mean of Ehc along
// dr, minus the whistler diffusion of the two face-B jumps across the edge
__device__ __forceinline__ double hall_edge_direct(const BlockView &b, int ea, int i, int j, int k)
{
    const double eps = 1e-14, Cwh = 0.1;
    const int64_t v = b.vol;
    const int64_t p = pidx(b, i, j, k);
    int64_t c[4];
    int Fm, Fp, Am, Ap;
    int64_t qm, qp, am, ap;
    if (ea == 0)
    {
        c[0] = pidx(b, i, j - 1, k - 1);
        c[1] = pidx(b, i, j - 1, k);
        c[2] = pidx(b, i, j, k - 1);
        c[3] = p;
        Fm = F_Bzeta, qm = pidx(b, i, j - 1, k), Fp = F_Beta, qp = pidx(b, i, j, k - 1);
        Am = F_Areazeta, am = pidx(b, i, j - 1, k), Ap = F_Areaeta, ap = pidx(b, i, j, k - 1);
    }
    else if (ea == 1)
    {
        c[0] = pidx(b, i - 1, j, k - 1);
        c[1] = pidx(b, i - 1, j, k);
        c[2] = pidx(b, i, j, k - 1);
        c[3] = p;
        Fm = F_Bxi, qm = pidx(b, i, j, k - 1), Fp = F_Bzeta, qp = pidx(b, i - 1, j, k);
        Am = F_Areaxi, am = pidx(b, i, j, k - 1), Ap = F_Areazeta, ap = pidx(b, i - 1, j, k);
    }
    else
    {
        c[0] = pidx(b, i - 1, j - 1, k);
        c[1] = pidx(b, i - 1, j, k);
        c[2] = pidx(b, i, j - 1, k);
        c[3] = p;
        Fm = F_Beta, qm = pidx(b, i - 1, j, k), Fp = F_Bxi, qp = pidx(b, i, j - 1, k);
        Am = F_Areaeta, am = pidx(b, i - 1, j, k), Ap = F_Areaxi, ap = pidx(b, i, j - 1, k);
    }
    const double *E = b.f[F_Ehc], *be = b.f[F_HallBeta];
    const double Ecx = 0.25 * (E[c[0]] + E[c[1]] + E[c[2]] + E[c[3]]);
    const double Ecy = 0.25 * (E[v + c[0]] + E[v + c[1]] + E[v + c[2]] + E[v + c[3]]);
    const double Ecz = 0.25 * (E[2 * v + c[0]] + E[2 * v + c[1]] + E[2 * v + c[2]] + E[2 * v + c[3]]);
    const double *dr = b.f[F_drxi + ea];
    const double Ecen = Ecx * dr[p] + Ecy * dr[v + p] + Ecz * dr[2 * v + p];
    const double beta_e = smax(smax(be[c[0]], be[c[1]]), smax(be[c[2]], be[c[3]]));
    const double L = smax(b.f[F_dlxi + ea][p], eps);
    const double Abar_m = 0.5 * (b.f[Am][p] + b.f[Am][am]);
    const double inv_m = L / smax(Abar_m, eps);
    const double mu_m = Cwh * beta_e * inv_m * inv_m;
    const double Abar_p = 0.5 * (b.f[Ap][p] + b.f[Ap][ap]);
    const double inv_p = L / smax(Abar_p, eps);
    const double mu_p = Cwh * beta_e * inv_p * inv_p;
    const double dB_m = b.f[Fm][p] - b.f[Fm][qm];
    const double dB_p = b.f[Fp][p] - b.f[Fp][qp];
    return Ecen - 0.5 * mu_m * dB_m + 0.5 * mu_p * dB_p;
}

// inner Hall edge EMF of all three axes; zero inside the boxes zb[8 q ..]:
// block, edge axis, lo[3], hi[3] (Solid_Surface layers and Pole edges).
// Per-edge form: each edge reads its four cells (the compiler's own
// register allocation).
__global__ void k_hall_edge_percell(const BlockView *__restrict__ bvs, const int *__restrict__ zb, int nzb)
{
    int64_t t;
    const int bi = cta_block(bvs, KIND_STAG, t);
    const BlockView &b = bvs[bi];
    int i, j, k;
    if (!stagger_point(b, nullptr, 0, t, i, j, k))
        return;
    const int64_t p = pidx(b, i, j, k);
#pragma unroll
    for (int ea = 0; ea < 3; ++ea)
    {
        if (!inner_of(b, 1, ea, i, j, k))
            continue;
        bool zero = false;
        for (int q = 0; q < nzb && !zero; ++q)
        {
            const int *z = zb + 8 * q;
            zero = (z[0] == bi && z[1] == ea && i >= z[2] && j >= z[3] && k >= z[4] && i < z[5] &&
                    j < z[6] && k < z[7]);
        }
        b.f[F_Ehxi + ea][p] = zero ? 0.0 : hall_edge_direct(b, ea, i, j, k);
    }
}

// Shared-cell form: the seven cells the three edges of a staggered point
// share are read once, and every edge is formed before any is stored (at
// least 2 CTAs per SM).
__global__ void __launch_bounds__(256, 2) k_hall_edge_shared(const BlockView *__restrict__ bvs,
                                                             const int *__restrict__ zb, int nzb)
{
    int64_t t;
    const int bi = cta_block(bvs, KIND_STAG, t);
    const BlockView &b = bvs[bi];
    int i, j, k;
    if (!stagger_point(b, nullptr, 0, t, i, j, k))
        return;
    const int64_t v = b.vol;
    const double *Ec = b.f[F_Ehc], *bec = b.f[F_HallBeta];
    double E7[7][3], be7[7];
#pragma unroll
    for (int q = 0; q < 7; ++q)
    {
        const int64_t c = hall_cell_of(b, q, i, j, k);
        E7[q][0] = Ec[c];
        E7[q][1] = Ec[v + c];
        E7[q][2] = Ec[2 * v + c];
        be7[q] = bec[c];
    }
    double out[3] = {0.0, 0.0, 0.0};
    bool inner[3];
#pragma unroll
    for (int ea = 0; ea < 3; ++ea)
    {
        inner[ea] = inner_of(b, 1, ea, i, j, k);
        if (!inner[ea] || hall_zeroed(zb, nzb, bi, ea, i, j, k))
            continue;
        double E[4][3], be[4];
#pragma unroll
        for (int q = 0; q < 4; ++q)
        {
            E[q][0] = E7[hall_cells(ea, q)][0];
            E[q][1] = E7[hall_cells(ea, q)][1];
            E[q][2] = E7[hall_cells(ea, q)][2];
            be[q] = be7[hall_cells(ea, q)];
        }
        out[ea] = hall_edge_one(b, ea, i, j, k, E, be);
    }
    const int64_t p = pidx(b, i, j, k);
#pragma unroll
    for (int ea = 0; ea < 3; ++ea)
        if (inner[ea])
            b.f[F_Ehxi + ea][p] = out[ea];
}

int launch_k_hall_edge(int variant, dim3 grid, cudaStream_t st, const BlockView *bvs, const int *zb, int nzb)
{
    switch (variant)
    {
    case 0:
        k_hall_edge_percell<<<grid, 256, 0, st>>>(bvs, zb, nzb);
        break;
    case 1:
        k_hall_edge_shared<<<grid, 256, 0, st>>>(bvs, zb, nzb);
        break;
    default:
        return -1;
    }
    return 0;
}

// cell part of ApplyUpdate_Euler_ (LunarSolver_Advance.cpp:82-93): U += dt*RHS_H
__global__ void k_update_u(const BlockView *__restrict__ bvs, const double *__restrict__ dtp)
{
    int64_t t;
    const BlockView &b = bvs[cta_block(bvs, KIND_CELL0, t)];
    int lo[3], n[3];
    loc_box(b, LOC_CELL, 0, lo, n);
    int i, j, k;
    if (!box_point(lo, n, t, i, j, k))
        return;
    const double dt = dtp[b.run];
    const int64_t p = pidx(b, i, j, k);
#pragma unroll
    for (int m = 0; m < 5; ++m)
        b.f[F_U][m * b.vol + p] += dt * b.f[F_RHS][m * b.vol + p];
}

// SSP-RK2 (Shu and Osher, 1988) from two Euler stages at one dt: the state
// of the step's start on the points the Euler update writes (inner cells,
// inner faces), then U^{n+1} = 0.5 (U^n + U2) there.  save = 1 stores,
// save = 0 averages.
__global__ void k_rk2(const BlockView *__restrict__ bvs, int save)
{
    int64_t t;
    const BlockView &b = bvs[cta_block(bvs, KIND_STAG, t)];
    int i, j, k;
    if (!stagger_point(b, nullptr, 0, t, i, j, k))
        return;
    const int64_t p = pidx(b, i, j, k);
    const int64_t v = b.vol;
    double *r = b.rk;
    if (i < b.ni && j < b.nj && k < b.nk)
    {
        double *U = b.f[F_U];
#pragma unroll
        for (int m = 0; m < 5; ++m)
        {
            if (save)
                r[m * v + p] = U[m * v + p];
            else
                U[m * v + p] = 0.5 * (r[m * v + p] + U[m * v + p]);
        }
    }
#pragma unroll
    for (int fa = 0; fa < 3; ++fa)
        if (inner_of(b, 0, fa, i, j, k))
        {
            double *B = b.f[F_Bxi + fa];
            double *R = r + (5 + fa) * v;
            if (save)
                R[p] = B[p];
            else
                B[p] = 0.5 * (R[p] + B[p]);
        }
}

// least-squares weight planes of a block: the FP64 field, or its FP32 copy
template <typename WT> __device__ __forceinline__ const WT *weights(const BlockView &b, int f, int plane32);
template <> __device__ __forceinline__ const double *weights<double>(const BlockView &b, int f, int)
{
    return b.f[f];
}
template <> __device__ __forceinline__ const float *weights<float>(const BlockView &b, int, int plane32)
{
    return b.w32 + int64_t(plane32) * b.vol;
}

// plane q of axis a's face data: q = 0 the area, 1..3 the unit normal (the
// FP64 field Anorm_*, or its FP32 copies)
template <typename WT> __device__ __forceinline__ const WT *face_planes(const BlockView &b, int a, int q);
template <> __device__ __forceinline__ const double *face_planes<double>(const BlockView &b, int a, int q)
{
    return b.f[F_NAxi + a] + int64_t(q) * b.vol;
}
template <> __device__ __forceinline__ const float *face_planes<float>(const BlockView &b, int a, int q)
{
    return b.g32 + int64_t(q == 0 ? G32_AREA + a : G32_NRM + 3 * a + q - 1) * b.vol;
}

// ---------------------------------------------------------------------------
// calc_Bcell (Z4_Lunar/src/physics/LunarSolver_Tools.cpp:163-241)
// ---------------------------------------------------------------------------
// WT: double (the reference's weights, FP64 form) or float (their FP32
// copies, mixed form: the products and sums stay FP64)
template <typename WT>
__device__ __forceinline__ void bcell_one(const BlockView &b, int i, int j, int k)
{
    const double *Bx = b.f[F_Bxi], *Be = b.f[F_Beta], *Bz = b.f[F_Bzeta];
    const double *Ax = b.f[F_Baddxi], *Ae = b.f[F_Baddeta], *Az = b.f[F_Baddzeta];
    const int64_t p = pidx(b, i, j, k);
    const int64_t pi1 = pidx(b, i + 1, j, k), pj1 = pidx(b, i, j + 1, k), pk1 = pidx(b, i, j, k + 1);
    const double phi_tot[6] = {-Bx[p] - Ax[p], Bx[pi1] + Ax[pi1], -Be[p] - Ae[p],
                               Be[pj1] + Ae[pj1], -Bz[p] - Az[p], Bz[pk1] + Az[pk1]};
    const double phi_ind[6] = {-Bx[p], Bx[pi1], -Be[p], Be[pj1], -Bz[p], Bz[pk1]};
    const int64_t v = b.vol;
    const WT *W = weights<WT>(b, F_WB, W32_B);
    double bxt = 0.0, byt = 0.0, bzt = 0.0, bxi = 0.0, byi = 0.0, bzi = 0.0;
#pragma unroll
    for (int q = 0; q < 6; ++q)
    {
        const double wx = double(W[q * v + p]);
        const double wy = double(W[(6 + q) * v + p]);
        const double wz = double(W[(12 + q) * v + p]);
        bxt += wx * phi_tot[q];
        byt += wy * phi_tot[q];
        bzt += wz * phi_tot[q];
        bxi += wx * phi_ind[q];
        byi += wy * phi_ind[q];
        bzi += wz * phi_ind[q];
    }
    double *Bc = b.f[F_Bcell], *Bi = b.f[F_Bind];
    Bc[p] = bxt;
    Bc[v + p] = byt;
    Bc[2 * v + p] = bzt;
    Bi[p] = bxi;
    Bi[v + p] = byi;
    Bi[2 * v + p] = bzi;
}

template <typename WT> __global__ void k_bcell_w(const BlockView *__restrict__ bvs)
{
    const BlockView &b = bvs[blockIdx.y];
    int lo[3], n[3];
    loc_box(b, LOC_CELL, 0, lo, n);
    int i, j, k;
    if (!box_point(lo, n, int64_t(blockIdx.x) * blockDim.x + threadIdx.x, i, j, k))
        return;
    bcell_one<WT>(b, i, j, k);
}

void launch_k_bcell(bool w32, dim3 grid, cudaStream_t st, const BlockView *bvs)
{
    if (w32)
        k_bcell_w<float><<<grid, 256, 0, st>>>(bvs);
    else
        k_bcell_w<double><<<grid, 256, 0, st>>>(bvs);
}

// ---------------------------------------------------------------------------
// Calc_J_Edge: CTOperators::CurlAdjFaceToEdge (CTOperators.cpp:58-110) with
// the face Hodge scale beta, times the edge scale alpha
// (LunarSolver_Tools.cpp:777-835).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void jedge_one(const BlockView &b, int ea, int i, int j, int k, int fB0, int fJ0,
                                          double mult)
{
    const double *Fx = b.f[fB0], *Fe = b.f[fB0 + 1], *Fz = b.f[fB0 + 2];
    const double *bx = b.f[F_betaxi], *be = b.f[F_betaeta], *bz = b.f[F_betazeta];
    const int64_t c0 = pidx(b, i, j, k);
    double val;
    if (ea == 0)
    {
        const int64_t a = pidx(b, i, j, k - 1), d = pidx(b, i, j - 1, k);
        val = (be[a] * Fe[a] - be[c0] * Fe[c0]) + (bz[c0] * Fz[c0] - bz[d] * Fz[d]);
    }
    else if (ea == 1)
    {
        const int64_t a = pidx(b, i, j, k - 1), d = pidx(b, i - 1, j, k);
        val = (bx[c0] * Fx[c0] - bx[a] * Fx[a]) + (bz[d] * Fz[d] - bz[c0] * Fz[c0]);
    }
    else
    {
        const int64_t a = pidx(b, i, j - 1, k), d = pidx(b, i - 1, j, k);
        val = (bx[a] * Fx[a] - bx[c0] * Fx[c0]) + (be[c0] * Fe[c0] - be[d] * Fe[d]);
    }
    const double J = mult * val;
    b.f[fJ0 + ea][c0] = J * b.f[F_alphaxi + ea][c0];
}

__global__ void k_jedge(const BlockView *__restrict__ bvs, int fB0, int fJ0, double mult, const int *__restrict__ rng)
{
    int64_t t;
    const int bi = cta_block(bvs, KIND_STAG, t);
    const BlockView &b = bvs[bi];
    int i, j, k;
    if (!stagger_point(b, rng, bi, t, i, j, k))
        return;
#pragma unroll
    for (int ea = 0; ea < 3; ++ea)
        if (inner_of(b, 1, ea, i, j, k))
            jedge_one(b, ea, i, j, k, fB0, fJ0, mult);
}

// calc_Bcell and Calc_J_Edge in one pass over the staggered points: both
// read the face B around the same points (the B_cell sync between them in
// the reference touches neither input)
template <typename WT> __device__ __forceinline__ void k_bcell_jedge_body(const BlockView *__restrict__ bvs)
{
    int64_t t;
    const BlockView &b = bvs[cta_block(bvs, KIND_STAG, t)];
    int i, j, k;
    if (!stagger_point(b, nullptr, 0, t, i, j, k))
        return;
    if (i < b.ni && j < b.nj && k < b.nk)
        bcell_one<WT>(b, i, j, k);
#pragma unroll
    for (int ea = 0; ea < 3; ++ea)
        if (inner_of(b, 1, ea, i, j, k))
            jedge_one(b, ea, i, j, k, F_Bxi, F_Jxi, 1.0);
}

template <typename WT, int MINB>
__global__ void __launch_bounds__(256, MINB) k_bcell_jedge_t(const BlockView *__restrict__ bvs)
{
    k_bcell_jedge_body<WT>(bvs);
}
// the compiler's own register allocation (no launch bounds)
template <typename WT> __global__ void k_bcell_jedge_free(const BlockView *__restrict__ bvs)
{
    k_bcell_jedge_body<WT>(bvs);
}


// ---------------------------------------------------------------------------
// calc_Jcell (LunarSolver_Tools.cpp:837-892)
// ---------------------------------------------------------------------------
template <typename WT> __device__ __forceinline__ void jcell_one(const BlockView &b, int i, int j, int k)
{
    const double *Jx = b.f[F_Jxi], *Je = b.f[F_Jeta], *Jz = b.f[F_Jzeta];
    const double s[12] = {Jx[pidx(b, i, j, k)],         Jx[pidx(b, i, j + 1, k)],     Jx[pidx(b, i, j, k + 1)],
                          Jx[pidx(b, i, j + 1, k + 1)], Je[pidx(b, i, j, k)],         Je[pidx(b, i + 1, j, k)],
                          Je[pidx(b, i, j, k + 1)],     Je[pidx(b, i + 1, j, k + 1)], Jz[pidx(b, i, j, k)],
                          Jz[pidx(b, i + 1, j, k)],     Jz[pidx(b, i, j + 1, k)],     Jz[pidx(b, i + 1, j + 1, k)]};
    const WT *W = weights<WT>(b, F_WJ, W32_J);
    const int64_t p = pidx(b, i, j, k);
    const int64_t v = b.vol;
    double jx = 0.0, jy = 0.0, jz = 0.0;
#pragma unroll
    for (int q = 0; q < 12; ++q)
    {
        jx += double(W[q * v + p]) * s[q];
        jy += double(W[(12 + q) * v + p]) * s[q];
        jz += double(W[(24 + q) * v + p]) * s[q];
    }
    double *Jc = b.f[F_Jcell];
    Jc[p] = jx;
    Jc[v + p] = jy;
    Jc[2 * v + p] = jz;
}

__global__ void k_jcell(const BlockView *__restrict__ bvs)
{
    const BlockView &b = bvs[blockIdx.y];
    int lo[3], n[3];
    loc_box(b, LOC_CELL, 0, lo, n);
    int i, j, k;
    if (!box_point(lo, n, int64_t(blockIdx.x) * blockDim.x + threadIdx.x, i, j, k))
        return;
    jcell_one<double>(b, i, j, k);
}

// J_cell in a pass of its own over the flattened inner-cell grid (the split
// variant of the derived-field pass: the weight stream with the compiler's
// own register budget, the PV / CFL pass without it)
template <typename WT> __global__ void k_jcell_w(const BlockView *__restrict__ bvs)
{
    int64_t t;
    const BlockView &b = bvs[cta_block(bvs, KIND_CELL0, t)];
    int lo[3], n[3];
    loc_box(b, LOC_CELL, 0, lo, n);
    int i, j, k;
    if (!box_point(lo, n, t, i, j, k))
        return;
    jcell_one<WT>(b, i, j, k);
}

void launch_k_jcell(bool w32, dim3 grid, cudaStream_t st, const BlockView *bvs)
{
    if (w32)
        k_jcell_w<float><<<grid, 256, 0, st>>>(bvs);
    else
        k_jcell_w<double><<<grid, 256, 0, st>>>(bvs);
}

// ---------------------------------------------------------------------------
// calc_PV + calc_Uplus (LunarSolver_Tools.cpp:58-141) on the inner cells
// and `depth` ghost layers (the reference covers the whole array) and, on
// inner cells, the CFL time-step bound of the next Compute_Timestep
// (LunarSolver_Timestep.cpp:8-140) reduced with warp shuffles and one
// atomicMin per thread block.
// ---------------------------------------------------------------------------

// one face of the CFL bound: (|u . n| + c_f) A with n the outward unit
// normal (A and JD / A precomputed per face, k_face_normals), in the
// arithmetic of the face planes: FP64 with the FP64 planes (the reference's
// values and operations), FP32 with their FP32 copies (the mixed form: the
// speeds in FP32, summed over the faces in FP64)
template <typename T>
__device__ __forceinline__ T cfl_face_term(const T *Ap, const T *N0, const T *N1, const T *N2, int64_t p,
                                           bool outward_plus, T ux, T uy, T uz, T Bx, T By, T Bz, T B2, T rho, T cs2,
                                           T inver_MA2)
{
    const T A = Ap[p];
    if (A <= T(0))
        return T(0);
    T nx = N0[p], ny = N1[p], nz = N2[p];
    if (!outward_plus)
    {
        nx = -nx;
        ny = -ny;
        nz = -nz;
    }
    const T un = ux * nx + uy * ny + uz * nz;
    const T Bn = Bx * nx + By * ny + Bz * nz;
    const T vA2 = inver_MA2 * B2 / rho;
    const T vAn2 = inver_MA2 * (Bn * Bn) / rho;
    const T term = cs2 + vA2;
    T disc = term * term - T(4) * cs2 * vAn2;
    if (disc < T(0))
        disc = T(0);
    const T cf = sqrt(T(0.5) * (term + sqrt(disc)));
    return (fabs(un) + cf) * A;
}

__device__ __forceinline__ unsigned long long dbl_key(double x)
{
    // order-preserving key for non-negative doubles (NaN maps above +inf)
    return (unsigned long long)__double_as_longlong(x);
}

// variants: at least 4 CTAs per SM (64 registers; the default: the extra
// warps hide more of the weight-stream latency, 0.216 -> 0.205 ms on the C2
// step against the uncapped 80 registers), uncapped, at least 5
template <typename WT>
__device__ __forceinline__ void k_pv_uplus_dt_body(const BlockView *__restrict__ bvs, Consts c, unsigned long long *dt_key, int depth,
                              int with_jcell)
{
    int64_t t;
    const BlockView &b = bvs[cta_block(bvs, KIND_CELL1, t)];
    int lo[3], n[3];
    loc_box(b, LOC_CELL, depth, lo, n);
    int i, j, k;
    double dtc = 1e100;
    if (box_point(lo, n, t, i, j, k))
    {
        // calc_Jcell on inner cells in the same pass: its weight stream
        // overlaps this kernel's FP64 work (J_cell is not read here)
        if (with_jcell && i >= 0 && j >= 0 && k >= 0 && i < b.ni && j < b.nj && k < b.nk)
            jcell_one<WT>(b, i, j, k);
        const int64_t p = pidx(b, i, j, k);
        const int64_t v = b.vol;
        const double *U = b.f[F_U];
        const double U0 = U[p], U1 = U[v + p], U2 = U[2 * v + p], U3 = U[3 * v + p], U4 = U[4 * v + p];
        const double rho_pv = smax(U0, 1e-12);
        const double u = U1 / rho_pv, vv = U2 / rho_pv, w = U3 / rho_pv;
        {
            const double rho = rho_pv;
            const double ke = 0.5 * rho * (u * u + vv * vv + w * w);
            double eint = U4 - ke;
            if (eint < 0.0)
                eint = 0.0;
            double pr = (c.gamma - 1.0) * eint;
            pr = smax(pr, 1e-12);
            if (sizeof(WT) == sizeof(double))
            {
                // PV_H (the mixed form's pass leaves it to read-out: its flux
                // reads the FP32 face states, its J x B source the velocities
                // from U)
                const double T = pr / (rho * c.state_coeff);
                double *PV = b.f[F_PV];
                PV[p] = u;
                PV[v + p] = vv;
                PV[2 * v + p] = w;
                PV[3 * v + p] = pr;
                PV[4 * v + p] = T;
            }
            const bool has_plasma = U0 > 1e-20;
            double *Up = b.f[F_Uplus];
            Up[p] = has_plasma ? u : 0.0;
            Up[v + p] = has_plasma ? vv : 0.0;
            Up[2 * v + p] = has_plasma ? w : 0.0;
            // sound speed and total energy of the Rusanov face states
            // (Reconstruction_Rusanov, LunarSolver_FluidRHS.cpp:34-111)
            const double cs = sqrt(smax(0.0, c.gamma * pr / smax(U0, 1e-30)));
            const double rhoe = pr / (c.gamma - 1.0) + 0.5 * U0 * (u * u + vv * vv + w * w);
            if (sizeof(WT) == sizeof(double))
            {
                // FP64 face states of the FP64 flux (the mixed form's flux
                // reads the FP32 copies below instead)
                b.f[F_Cs][p] = cs;
                b.f[F_RhoE][p] = rhoe;
            }
            if (b.q32)
            {
                // FP32 face states of the mixed-precision flux: deviations
                // from the reference state (formed in FP64), sound speed
                float *q = b.q32;
                const double *q0 = b.qref;
                q[Q32_RHO * v + p] = float(U0 - q0[0]);
                q[(Q32_U + 0) * v + p] = float(u - q0[1]);
                q[(Q32_U + 1) * v + p] = float(vv - q0[2]);
                q[(Q32_U + 2) * v + p] = float(w - q0[3]);
                q[Q32_P * v + p] = float(pr - q0[4]);
                q[Q32_RHOE * v + p] = float(rhoe - q0[5]);
                q[Q32_C * v + p] = float(cs);
            }
        }
        const bool inner = (i >= 0 && j >= 0 && k >= 0 && i < b.ni && j < b.nj && k < b.nk);
        if (inner && dt_key)
        {
            const double V = fabs(b.f[F_Jac][p]);
            if (V > 0.0)
            {
                const double rho = smax(U0, 1e-2);
                // same quotients as the primitive velocities when both floors leave rho alone
                const bool same = (rho == rho_pv);
                const double ux = same ? u : U1 / rho, uy = same ? vv : U2 / rho, uz = same ? w : U3 / rho;
                const double ke = 0.5 * rho * (ux * ux + uy * uy + uz * uz);
                const double eint = U4 - ke;
                const double pr = (c.gamma - 1.0) * eint;
                const double cs2 = c.gamma * pr / rho;
                const double *Bc = b.f[F_Bcell];
                const double Bx = Bc[p], By = Bc[v + p], Bz = Bc[2 * v + p];
                const double B2 = Bx * Bx + By * By + Bz * Bz;
                // the mixed form reads the FP32 copies of the face areas and normals
                const WT *P[3][4];
#pragma unroll
                for (int a = 0; a < 3; ++a)
#pragma unroll
                    for (int q = 0; q < 4; ++q)
                        P[a][q] = face_planes<WT>(b, a, q);
                const int64_t pa1[3] = {pidx(b, i + 1, j, k), pidx(b, i, j + 1, k), pidx(b, i, j, k + 1)};
                // the face speeds in the planes' arithmetic (identity casts in FP64)
                const WT uxw = WT(ux), uyw = WT(uy), uzw = WT(uz), Bxw = WT(Bx), Byw = WT(By), Bzw = WT(Bz);
                const WT B2w = WT(B2), rhow = WT(rho), cs2w = WT(cs2), iMA2 = WT(c.inver_MA2);
                double denom = 0.0;
#pragma unroll
                for (int a = 0; a < 3; ++a)
                {
                    denom += double(cfl_face_term<WT>(P[a][0], P[a][1], P[a][2], P[a][3], p, false, uxw, uyw, uzw, Bxw,
                                                      Byw, Bzw, B2w, rhow, cs2w, iMA2));
                    denom += double(cfl_face_term<WT>(P[a][0], P[a][1], P[a][2], P[a][3], pa1[a], true, uxw, uyw, uzw,
                                                      Bxw, Byw, Bzw, B2w, rhow, cs2w, iMA2));
                }
                // cells with denom <= 0 (or NaN) do not bound dt, as in the reference
                if (denom > 0.0)
                    dtc = c.cfl * V / denom;
            }
        }
    }
    if (!dt_key)
        return;
    // block-wide minimum of the order-preserving keys
    unsigned long long key = dbl_key(dtc);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
    {
        const unsigned long long o = __shfl_xor_sync(0xffffffffu, key, off);
        key = (o < key) ? o : key;
    }
    __shared__ unsigned long long wmin[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0)
        wmin[warp] = key;
    __syncthreads();
    if (warp == 0)
    {
        const int nw = (blockDim.x + 31) >> 5;
        key = (lane < nw) ? wmin[lane] : ~0ull;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1)
        {
            const unsigned long long o = __shfl_xor_sync(0xffffffffu, key, off);
            key = (o < key) ? o : key;
        }
        if (lane == 0)
            atomicMin(dt_key + b.run, key);
    }
}

template <typename WT, int MINB>
__global__ void __launch_bounds__(256, MINB) k_pv_uplus_dt_t(const BlockView *__restrict__ bvs, Consts c, unsigned long long *dt_key, int depth,
                              int with_jcell)
{
    k_pv_uplus_dt_body<WT>(bvs, c, dt_key, depth, with_jcell);
}
// the compiler's own register allocation (no launch bounds)
template <typename WT>
__global__ void k_pv_uplus_dt_free(const BlockView *__restrict__ bvs, Consts c, unsigned long long *dt_key, int depth,
                              int with_jcell)
{
    k_pv_uplus_dt_body<WT>(bvs, c, dt_key, depth, with_jcell);
}


// Start of StepOnce: dt = global minimum of the CFL bounds, abort check
// (dt < dt_abort or NaN sets the error word, LunarSolver_Timestep.cpp:128-139).
__global__ void k_begin_step(const unsigned long long *dt_key, double *dt, int *err, double dt_abort, int nruns)
{
    for (int r = threadIdx.x; r < nruns; r += blockDim.x)
    {
        const double d = __longlong_as_double((long long)dt_key[r]);
        dt[r] = d;
        if (!isfinite(d) || d < dt_abort)
            err[0] = MHD_EDT;
    }
}

// Arms the dt reductions with the reference's initial bound (dt_local = 1e100).
__global__ void k_arm_dt(unsigned long long *dt_key, int nruns)
{
    for (int r = threadIdx.x; r < nruns; r += blockDim.x)
        dt_key[r] = dbl_key(1e100);
}

// End of StepOnce: run-data counters (Z4_Lunar/src/LunarSolver_Driver.cpp:75-79)
__global__ void k_end_step(const double *dt, double *time, long long *step, int nruns)
{
    for (int r = threadIdx.x; r < nruns; r += blockDim.x)
    {
        time[r] += dt[r];
        step[r] += 1;
    }
}

// ---------------------------------------------------------------------------
// compiled Sync: dst <- src over the field pool
// ---------------------------------------------------------------------------
__global__ void k_gather(double *__restrict__ pool, const uint64_t *__restrict__ dst, const uint64_t *__restrict__ src,
                         int64_t n)
{
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t < n)
        pool[dst[t]] = pool[src[t]];
}

__global__ void k_gather32(double *__restrict__ pool, const uint32_t *__restrict__ dst,
                           const uint32_t *__restrict__ src, int64_t n)
{
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t < n)
        pool[dst[t]] = pool[src[t]];
}

// phase A of a Sync: points set to fixed values by physical handlers
// (Farfield states, zero-curl edge EMF, zeroed wall layers)
__global__ void k_set_consts(double *__restrict__ pool, const uint64_t *__restrict__ dst,
                             const double *__restrict__ val, int64_t n)
{
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t < n)
        pool[dst[t]] = val[t];
}

// phase A of Sync("Ucell") on a Solid_Surface face: LunarBoundary::BC_Solid_Surface_
// (Z4_Lunar/src/boundary/Boundary_Condition_Fluid.cpp:19-185).  The first inner
// cell layer takes the density of the next cell inwards (floored at 2.5e-3),
// zero velocity and its pressure; every ghost layer then repeats that
// layer's state.  One thread per boundary cell column; dir = +-1, +-2, +-3.
__device__ __forceinline__ void wall_u_one(const BlockView &b, int dir, double gamma, int64_t t);

__global__ void k_wall_u(const BlockView *__restrict__ bvs, int blk, int dir, double gamma)
{
    wall_u_one(bvs[blk], dir, gamma, int64_t(blockIdx.x) * blockDim.x + threadIdx.x);
}

// all Solid_Surface handlers of a sync in one launch: walls[2 q] = block,
// walls[2 q + 1] = direction of handler q = blockIdx.y
__global__ void k_wall_u_all(const BlockView *__restrict__ bvs, const int *__restrict__ walls, double gamma)
{
    const int q = blockIdx.y;
    wall_u_one(bvs[walls[2 * q]], walls[2 * q + 1], gamma, int64_t(blockIdx.x) * blockDim.x + threadIdx.x);
}

__device__ __forceinline__ void wall_u_one(const BlockView &b, int dir, double gamma, int64_t t)
{
    const int ax = (dir < 0 ? -dir : dir) - 1;
    const int sgn = dir > 0 ? 1 : -1;
    const int n[3] = {b.ni, b.nj, b.nk};
    const int t1 = (ax == 0) ? 1 : 0;
    const int t2 = (ax == 2) ? 1 : 2;
    if (t >= int64_t(n[t1]) * n[t2])
        return;
    int c[3];
    c[t1] = int(t / n[t2]);
    c[t2] = int(t % n[t2]);
    c[ax] = (sgn < 0) ? 0 : n[ax] - 1;
    const double rho_floor = 2.5e-3, p_floor = 1e-12;
    double *U = b.f[F_U];
    const int64_t v = b.vol;
    auto pressure = [&](double rho, double mx, double my, double mz, double E) {
        rho = smax(rho, rho_floor);
        const double ke = 0.5 * (mx * mx + my * my + mz * mz) / rho;
        double eint = E - ke;
        if (eint < 0.0)
            eint = 0.0;
        double p = (gamma - 1.0) * eint;
        return smax(p, p_floor);
    };
    // first layer from the cell one further inside
    int r[3] = {c[0], c[1], c[2]};
    r[ax] -= sgn;
    const int64_t pr = pidx(b, r[0], r[1], r[2]);
    const int64_t p0 = pidx(b, c[0], c[1], c[2]);
    {
        const double rho_r = smax(U[pr], rho_floor);
        const double p_r = pressure(rho_r, U[v + pr], U[2 * v + pr], U[3 * v + pr], U[4 * v + pr]);
        const double vz = 0.0;
        const double ke_g = 0.5 * rho_r * (vz * vz + vz * vz + vz * vz);
        U[p0] = rho_r;
        U[v + p0] = rho_r * vz;
        U[2 * v + p0] = rho_r * vz;
        U[3 * v + p0] = rho_r * vz;
        U[4 * v + p0] = p_r / (gamma - 1.0) + ke_g;
    }
    // ghost layers repeat the (updated) first layer
    const double rho_r = smax(U[p0], rho_floor);
    const double p_r = pressure(rho_r, U[v + p0], U[2 * v + p0], U[3 * v + p0], U[4 * v + p0]);
    const double vz = 0.0;
    const double ke_g = 0.5 * rho_r * (vz * vz + vz * vz + vz * vz);
    for (int ng = 1; ng <= b.G; ++ng)
    {
        int gidx[3] = {c[0], c[1], c[2]};
        gidx[ax] += ng * sgn;
        const int64_t pg = pidx(b, gidx[0], gidx[1], gidx[2]);
        U[pg] = rho_r;
        U[v + pg] = rho_r * vz;
        U[2 * v + pg] = rho_r * vz;
        U[3 * v + pg] = rho_r * vz;
        U[4 * v + pg] = p_r / (gamma - 1.0) + ke_g;
    }
}

// two-phase variant when a source is also a destination
__global__ void k_gather_stage(double *__restrict__ tmp, const double *__restrict__ pool,
                               const uint64_t *__restrict__ src, int64_t n)
{
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t < n)
        tmp[t] = pool[src[t]];
}
__global__ void k_scatter_stage(double *__restrict__ pool, const double *__restrict__ tmp,
                                const uint64_t *__restrict__ dst, int64_t n)
{
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t < n)
        pool[dst[t]] = tmp[t];
}

// ---------------------------------------------------------------------------
// AoS (reference host layout) <-> padded SoA, on the device
// ---------------------------------------------------------------------------
__global__ void k_aos_to_soa(const BlockView *__restrict__ bvs, int blk, int fid, int ncomp, int lo0, int lo1,
                             int lo2, int n0, int n1, int n2, const double *__restrict__ aos)
{
    const BlockView &b = bvs[blk];
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const int64_t tot = int64_t(n0) * n1 * n2 * ncomp;
    if (t >= tot)
        return;
    int64_t r = t;
    const int m = int(r % ncomp);
    r /= ncomp;
    const int k = lo2 + int(r % n2);
    r /= n2;
    const int j = lo1 + int(r % n1);
    const int i = lo0 + int(r / n1);
    b.f[fid][m * b.vol + pidx(b, i, j, k)] = aos[t];
}

__global__ void k_soa_to_aos(const BlockView *__restrict__ bvs, int blk, int fid, int ncomp, int lo0, int lo1,
                             int lo2, int n0, int n1, int n2, double *__restrict__ aos)
{
    const BlockView &b = bvs[blk];
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const int64_t tot = int64_t(n0) * n1 * n2 * ncomp;
    if (t >= tot)
        return;
    int64_t r = t;
    const int m = int(r % ncomp);
    r /= ncomp;
    const int k = lo2 + int(r % n2);
    r /= n2;
    const int j = lo1 + int(r % n1);
    const int i = lo0 + int(r / n1);
    aos[t] = b.f[fid][m * b.vol + pidx(b, i, j, k)];
}

// ---------------------------------------------------------------------------
// The implicit resistive solve in one persistent kernel
// (SolveImplicitResistiveDiffusion_, Z4_Lunar/src/implicit/Lunar_ImplicitResistive.cpp:430-491,
// with the operator MatMultImplicitResistive_, :369-427)
//
// Launched cooperatively (every CTA resident), so CTAs can wait for one
// another at grid barriers.  Every barrier wait is bounded: a CTA that gives
// up sets the error word and leaves, and the others give up at their next
// barrier.  Dot products: each CTA writes its partial sums, and after the
// barrier every CTA adds all partials in the same fixed order, so all CTAs
// hold bit-identical results and take the same control decisions without a
// second barrier.  The GMRES scalars (Hessenberg matrix, rotations, counters)
// live in each CTA's shared memory; CTA 0 writes them back at the end.
// ---------------------------------------------------------------------------

constexpr long long kBarrierSpins = 1ll << 22; // about a second of polling

// bar[0]: arrival count, bar[1]: generation, bar[2]: polling limit of every
// wait (0: kBarrierSpins; a smaller limit is set only by the failure-
// detection hook mhd_test_stall_barrier, and the host clears it after use)
__device__ __forceinline__ bool grid_barrier(unsigned *bar, int *err)
{
    __shared__ int ok; // one decision for the whole CTA
    __syncthreads();
    if (threadIdx.x == 0)
    {
        volatile unsigned *gen = bar + 1;
        const unsigned g = *gen;
        const unsigned lim = *(volatile unsigned *)(bar + 2);
        const long long limit = lim ? (long long)lim : kBarrierSpins;
        __threadfence();
        if (atomicAdd(bar, 1u) + 1u == gridDim.x)
        {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        }
        else
        {
            long long spins = 0;
            while (*gen == g)
            {
                if (++spins > limit)
                {
                    atomicExch(err, MHD_EKRYLOV);
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        ok = *(volatile int *)err != MHD_EKRYLOV;
    }
    __syncthreads();
    return ok != 0;
}

struct GmresScalars
{
    double H[31 * 31], cs[31], sn[31], g[32], hcol[32], y[31], d[32];
    double beta, resid, bnorm, ttol;
    int j, its, reason, breakdown, inner, outer, cycles;
};

// out[c] = V_c . w for c < nv, or out[0] = w . w (V null); with_self also
// out[nv] = w . w in the same reduction; every CTA ends with the same values
// in out (shared memory)
__device__ bool grid_dots(const ResistSolve &a, const double *V, int nv, const double *w, double *out, int &pbuf,
                          bool with_self = false)
{
    __shared__ double wred[8][8];
    const int G = gridDim.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    double *part = a.partial + int64_t(pbuf) * 32 * G;
    pbuf ^= 1;
    const int nd = nv + (with_self ? 1 : 0);
    for (int c0 = 0; c0 < nd; c0 += 8)
    {
        double acc[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        for (int64_t t = int64_t(blockIdx.x) * blockDim.x + tid; t < a.n; t += int64_t(G) * blockDim.x)
        {
            const double wt = w[t];
#pragma unroll
            for (int q = 0; q < 8; ++q)
                if (c0 + q < nd)
                    acc[q] += ((V && c0 + q < nv) ? V[int64_t(c0 + q) * a.n + t] : wt) * wt;
        }
#pragma unroll
        for (int q = 0; q < 8; ++q)
            for (int off = 16; off > 0; off >>= 1)
                acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], off);
        if (lane == 0)
            for (int q = 0; q < 8; ++q)
                wred[warp][q] = acc[q];
        __syncthreads();
        if (tid < 8 && c0 + tid < nd)
        {
            double sum = 0.0;
            for (int wp = 0; wp < int(blockDim.x >> 5); ++wp)
                sum += wred[wp][tid];
            part[int64_t(c0 + tid) * G + blockIdx.x] = sum;
        }
        __syncthreads();
    }
    if (!grid_barrier(a.bar, a.err))
        return false;
    for (int c = warp; c < nd; c += int(blockDim.x >> 5))
    {
        double sum = 0.0;
        for (int g = lane; g < G; g += 32)
            sum += __ldcg(&part[int64_t(c) * G + g]);
        for (int off = 16; off > 0; off >>= 1)
            sum += __shfl_xor_sync(0xffffffffu, sum, off);
        if (lane == 0)
            out[c] = sum;
    }
    __syncthreads();
    return true;
}

// fixed values (unless already written) then copies of a point list
__device__ bool grid_apply(const ResistSolve &a, const DevCopy &l, bool consts_done)
{
    const int64_t t0 = int64_t(blockIdx.x) * blockDim.x + threadIdx.x, ts = int64_t(gridDim.x) * blockDim.x;
    if (l.nconst > 0 && !consts_done)
    {
        for (int64_t t = t0; t < l.nconst; t += ts)
            a.pool[l.cdst[t]] = l.cval[t];
        if (!grid_barrier(a.bar, a.err))
            return false;
    }
    if (l.n == 0)
        return true;
    if (l.tmp)
    {
        for (int64_t t = t0; t < l.n; t += ts)
            l.tmp[t] = a.pool[l.src[t]];
        if (!grid_barrier(a.bar, a.err))
            return false;
        for (int64_t t = t0; t < l.n; t += ts)
            a.pool[l.dst[t]] = __ldcg(&l.tmp[t]);
    }
    else
        for (int64_t t = t0; t < l.n; t += ts)
            a.pool[l.dst[t]] = a.pool[l.src[t]];
    return grid_barrier(a.bar, a.err);
}

// y = A (src / div) (MatMultImplicitResistive_): Eres at the unknowns and
// their aliases, Sync("Eres1form"), dB = -dt curl Eres on the region,
// Sync("dB"), then per unknown dJ = alpha curlAdj(beta dB) at its edge and
// y = Eres - eta dJ.  src must be complete at entry unless first_barrier:
// the aliases read other threads' elements.  src / div is the stored basis
// vector bit for bit (the same division), so the basis vector itself need
// not be complete.
__device__ bool grid_matvec(const ResistSolve &a, const double *src, double div, bool first_barrier, double *y)
{
    const int64_t t0 = int64_t(blockIdx.x) * blockDim.x + threadIdx.x, ts = int64_t(gridDim.x) * blockDim.x;
    if (first_barrier && !grid_barrier(a.bar, a.err))
        return false;
    const double mdt = -a.dtp[0];
    if (a.fa.n >= 0)
    {
        // one phase: every Eres point the unknowns, aliases and Sync("Eres1form") set
        for (int64_t q = t0; q < a.fa.n; q += ts)
        {
            const int kd = a.fa.kind[q];
            const int64_t ix = a.fa.idx[q];
            double v;
            if (kd == FUSE_UNKNOWN)
                v = src[ix] / div;
            else if (kd == FUSE_ALIAS)
                v = a.fa.val[q] * (src[ix] / div);
            else if (kd == FUSE_CONST)
                v = a.fa.val[q];
            else
                v = a.pool[ix];
            a.pool[a.fa.dst[q]] = v;
        }
        if (!grid_barrier(a.bar, a.err))
            return false;
    }
    else
    {
        for (int64_t t = t0; t < a.n; t += ts)
            a.pool[a.e[t]] = src[t] / div;
        for (int64_t q = t0; q < a.nalias; q += ts)
            a.pool[a.alias[q]] = a.sign[q] * (src[a.alias_of[q]] / div);
        if (a.merge1)
            for (int64_t t = t0; t < a.eres1form.nconst; t += ts)
                a.pool[a.eres1form.cdst[t]] = a.eres1form.cval[t];
        if (!grid_barrier(a.bar, a.err))
            return false;
        if (!grid_apply(a, a.eres1form, a.merge1 != 0))
            return false;
    }
    const int64_t np = int64_t(a.nblocks) * a.nreg;
    for (int64_t q = t0; q < np; q += ts)
    {
        const int blk = int(q / a.nreg);
        const BlockView &b = a.bvs[blk];
        int i, j, k;
        if (stagger_point(b, a.rng, blk, q % a.nreg, i, j, k))
            curl_point(b, F_Eresxi, F_dBxi, -1, mdt, 0.0, i, j, k);
    }
    if (a.merge2)
        for (int64_t t = t0; t < a.db.nconst; t += ts)
            a.pool[a.db.cdst[t]] = a.db.cval[t];
    if (a.fb.n >= 0)
    {
        // the Sync("dB") copies in the same phase: each destination takes
        // the curl at its source directly (fixed values were written above)
        for (int64_t q = t0; q < a.fb.n; q += ts)
        {
            const int kd = a.fb.kind[q];
            const int64_t ix = a.fb.idx[q];
            double v;
            if (kd == FUSE_CURL)
            {
                const int k = int(ix % 4096) - 64, j = int((ix / 4096) % 4096) - 64;
                const int i = int((ix / (int64_t(4096) * 4096)) % 4096) - 64, fa = int(ix / (int64_t(4096) * 4096 * 4096));
                v = mdt * face_curl(a.bvs[a.fb.blk[q]], F_Eresxi, fa, i, j, k);
            }
            else if (kd == FUSE_CONST)
                v = a.fb.val[q];
            else
                v = a.pool[ix];
            a.pool[a.fb.dst[q]] = v;
        }
        if (!grid_barrier(a.bar, a.err))
            return false;
    }
    else
    {
        if (!grid_barrier(a.bar, a.err))
            return false;
        if (!grid_apply(a, a.db, a.merge2 != 0))
            return false;
    }
    for (int64_t t = t0; t < a.n; t += ts)
    {
        const int *u = a.uloc + 5 * t;
        jedge_one(a.bvs[u[0]], u[1], u[2], u[3], u[4], F_dBxi, F_dJxi, 1.0);
        y[t] = a.pool[a.e[t]] - a.eta[t] * a.pool[a.dj[t]];
    }
    return true;
}

__global__ void __launch_bounds__(256) k_gmres_resist(ResistSolve a)
{
    __shared__ GmresScalars S;
    __shared__ double dv[32];
    const int tid = threadIdx.x;
    const int64_t t0 = int64_t(blockIdx.x) * blockDim.x + tid, ts = int64_t(gridDim.x) * blockDim.x;
    const int64_t n = a.n;
    int pbuf = 0;
    // right-hand side b = eta J at the unknowns (PackImplicitJedgeToVec_), x = 0
    for (int64_t t = t0; t < n; t += ts)
    {
        a.b[t] = 0.0 + a.eta[t] * a.pool[a.j[t]];
        a.x[t] = 0.0;
    }
    if (!grid_dots(a, nullptr, 1, a.b, dv, pbuf))
        return;
    if (tid == 0)
    {
        S.bnorm = sqrt(dv[0]);
        S.ttol = fmax(a.rtol * S.bnorm, a.atol);
        S.its = 0;
        S.reason = 0;
        S.cycles = 0;
        S.resid = S.bnorm;
    }
    __syncthreads();
    for (;;)
    {
        // cycle start: r = b - A x, beta = ||r||
        if (!grid_matvec(a, a.x, 1.0, true, a.w))
            return;
        for (int64_t t = t0; t < n; t += ts)
            a.r[t] = a.b[t] - a.w[t];
        if (!grid_dots(a, nullptr, 1, a.r, dv, pbuf))
            return;
        if (tid == 0)
        {
            S.beta = sqrt(dv[0]);
            for (int q = 0; q < 32; ++q)
                S.g[q] = 0.0;
            S.g[0] = S.beta;
            S.resid = S.beta;
            S.breakdown = 0;
            S.j = 0;
            S.inner = 1;
            if (S.beta <= S.ttol)
            {
                S.reason = (S.beta <= a.atol) ? 3 : 2;
                S.inner = 0;
            }
            else if (S.its >= a.maxit)
            {
                S.reason = -3;
                S.inner = 0;
            }
        }
        __syncthreads();
        if (S.inner)
            for (int64_t t = t0; t < n; t += ts)
                a.V[t] = a.r[t] / S.beta;
        while (S.inner)
        {
            const int j = S.j;
            // V_j = r / beta (j = 0) or the previous step's w / ||w||, both
            // complete at the last reduction's barrier
            if (!grid_matvec(a, j == 0 ? a.r : a.w, j == 0 ? S.beta : S.hcol[j], false, a.w))
                return;
            // classical Gram-Schmidt, twice
            if (!grid_dots(a, a.V, j + 1, a.w, S.hcol, pbuf))
                return;
            for (int64_t t = t0; t < n; t += ts)
            {
                double s = a.w[t];
                for (int c = 0; c <= j; ++c)
                    s -= S.hcol[c] * a.V[int64_t(c) * n + t];
                a.w[t] = s;
            }
            // second pass, its dots and ||w'||^2 in one reduction: with V
            // orthonormal, ||w' - V d||^2 = ||w'||^2 - ||d||^2
            if (!grid_dots(a, a.V, j + 1, a.w, S.d, pbuf, true))
                return;
            for (int64_t t = t0; t < n; t += ts)
            {
                double s = a.w[t];
                for (int c = 0; c <= j; ++c)
                    s -= S.d[c] * a.V[int64_t(c) * n + t];
                a.w[t] = s;
            }
            if (tid <= j)
                S.hcol[tid] += S.d[tid];
            __syncthreads();
            if (tid == 0)
            {
                // new column: rotations, residual estimate
                double dd = 0.0;
                for (int c = 0; c <= j; ++c)
                    dd += S.d[c] * S.d[c];
                const double nw2 = S.d[j + 1] - dd;
                S.hcol[j + 1] = sqrt(nw2 > 0.0 ? nw2 : 0.0);
                for (int i = 0; i <= j + 1; ++i)
                    S.H[i * 31 + j] = S.hcol[i];
                for (int i = 0; i < j; ++i)
                {
                    const double x0 = S.H[i * 31 + j], x1 = S.H[(i + 1) * 31 + j];
                    S.H[i * 31 + j] = S.cs[i] * x0 + S.sn[i] * x1;
                    S.H[(i + 1) * 31 + j] = -S.sn[i] * x0 + S.cs[i] * x1;
                }
                const double x0 = S.H[j * 31 + j], x1 = S.H[(j + 1) * 31 + j];
                const double den = sqrt(x0 * x0 + x1 * x1);
                S.cs[j] = den > 0.0 ? x0 / den : 1.0;
                S.sn[j] = den > 0.0 ? x1 / den : 0.0;
                S.H[j * 31 + j] = den;
                S.H[(j + 1) * 31 + j] = 0.0;
                S.g[j + 1] = -S.sn[j] * S.g[j];
                S.g[j] = S.cs[j] * S.g[j];
                S.resid = fabs(S.g[j + 1]);
                S.breakdown = (S.hcol[j + 1] == 0.0) ? 1 : 0;
            }
            __syncthreads();
            if (!S.breakdown)
                for (int64_t t = t0; t < n; t += ts)
                    a.V[int64_t(j + 1) * n + t] = a.w[t] / S.hcol[j + 1];
            __syncthreads();
            if (tid == 0)
            {
                S.its += 1;
                S.j += 1;
                S.inner = !(S.resid <= S.ttol || S.breakdown || S.j >= a.m || S.its >= a.maxit);
            }
            __syncthreads();
        }
        // cycle end: H y = g, x += V y
        if (tid == 0)
        {
            const int m = S.j;
            for (int i = m - 1; i >= 0; --i)
            {
                double s = S.g[i];
                for (int q = i + 1; q < m; ++q)
                    s -= S.H[i * 31 + q] * S.y[q];
                S.y[i] = s / S.H[i * 31 + i];
            }
            S.cycles += 1;
        }
        __syncthreads();
        for (int64_t t = t0; t < n; t += ts)
        {
            double s = a.x[t];
            for (int c = 0; c < S.j; ++c)
                s += S.y[c] * a.V[int64_t(c) * n + t];
            a.x[t] = s;
        }
        if (tid == 0)
        {
            S.outer = 0;
            if (S.reason != 0)
                S.outer = 0;
            else if (S.resid <= S.ttol || S.breakdown)
                S.reason = (S.resid <= a.atol) ? 3 : 2;
            else if (S.its >= a.maxit)
                S.reason = -3;
            else
                S.outer = 1;
        }
        __syncthreads();
        if (!S.outer)
            break;
    }
    if (blockIdx.x == 0 && tid == 0)
    {
        GmresState *st = a.st;
        st->its = S.its;
        st->resid = S.resid;
        st->bnorm = S.bnorm;
        st->ttol = S.ttol;
        st->reason = S.reason;
        st->j = S.j;
        st->total_its += S.its;
        st->total_cycles += S.cycles;
    }
}

// launchers of the register / occupancy variants (tuned by mhd_autotune)
template <typename WT>
int launch_pv_variant(int variant, dim3 grid, cudaStream_t st, const BlockView *bvs, Consts c, unsigned long long *dt_key,
                      int depth, int with_jcell)
{
    switch (variant)
    {
    case 0:
        k_pv_uplus_dt_t<WT, 4><<<grid, 256, 0, st>>>(bvs, c, dt_key, depth, with_jcell);
        break;
    case 1:
        k_pv_uplus_dt_free<WT><<<grid, 256, 0, st>>>(bvs, c, dt_key, depth, with_jcell);
        break;
    case 2:
        k_pv_uplus_dt_t<WT, 5><<<grid, 256, 0, st>>>(bvs, c, dt_key, depth, with_jcell);
        break;
    case 3:
        // split: J_cell runs in its own pass (launch_k_jcell) before this one
        k_pv_uplus_dt_t<WT, 4><<<grid, 256, 0, st>>>(bvs, c, dt_key, depth, 0);
        break;
    default:
        return -1;
    }
    return 0;
}

// w32: the mixed form's FP32 weight copies (a separate instantiation, so the
// FP64 form's kernel is unchanged)
int launch_k_pv_uplus_dt(int variant, bool w32, dim3 grid, cudaStream_t st, const BlockView *bvs, Consts c,
                         unsigned long long *dt_key, int depth, int with_jcell)
{
    return w32 ? launch_pv_variant<float>(variant, grid, st, bvs, c, dt_key, depth, with_jcell)
               : launch_pv_variant<double>(variant, grid, st, bvs, c, dt_key, depth, with_jcell);
}

int launch_k_fluid_ucontra(int variant, dim3 grid, cudaStream_t st, const BlockView *bvs, Consts c)
{
    switch (variant)
    {
    case 0:
        k_fluid_ucontra_free<<<grid, 256, 0, st>>>(bvs, c);
        break;
    case 1:
        k_fluid_ucontra_t<3><<<grid, 256, 0, st>>>(bvs, c);
        break;
    default:
        return -1;
    }
    return 0;
}

template <typename WT> int launch_bcell_jedge_variant(int variant, dim3 grid, cudaStream_t st, const BlockView *bvs)
{
    switch (variant)
    {
    case 0:
        k_bcell_jedge_free<WT><<<grid, 256, 0, st>>>(bvs);
        break;
    case 1:
        k_bcell_jedge_t<WT, 6><<<grid, 256, 0, st>>>(bvs);
        break;
    default:
        return -1;
    }
    return 0;
}

int launch_k_bcell_jedge(int variant, bool w32, dim3 grid, cudaStream_t st, const BlockView *bvs)
{
    return w32 ? launch_bcell_jedge_variant<float>(variant, grid, st, bvs)
               : launch_bcell_jedge_variant<double>(variant, grid, st, bvs);
}

int launch_k_eface(int variant, dim3 grid, cudaStream_t st, const BlockView *bvs)
{
    switch (variant)
    {
    case 0:
        k_eface_free<<<grid, 256, 0, st>>>(bvs);
        break;
    case 1:
        k_eface_t<6><<<grid, 256, 0, st>>>(bvs);
        break;
    default:
        return -1;
    }
    return 0;
}

int launch_k_curl_e2f(int variant, dim3 grid, cudaStream_t st, const BlockView *bvs, int fE0, int fR0, int fB0, double mult,
                           const double *dtp, double dtdiv, int mult_is_neg_dt, const int *rng)
{
    switch (variant)
    {
    case 0:
        k_curl_e2f_free<<<grid, 256, 0, st>>>(bvs, fE0, fR0, fB0, mult, dtp, dtdiv, mult_is_neg_dt, rng);
        break;
    case 1:
        k_curl_e2f_t<6><<<grid, 256, 0, st>>>(bvs, fE0, fR0, fB0, mult, dtp, dtdiv, mult_is_neg_dt, rng);
        break;
    default:
        return -1;
    }
    return 0;
}

int launch_k_eedge(int variant, dim3 grid, cudaStream_t st, const BlockView *bvs)
{
    switch (variant)
    {
    case 0:
        k_eedge_free<<<grid, 256, 0, st>>>(bvs);
        break;
    case 1:
        k_eedge_t<8><<<grid, 256, 0, st>>>(bvs);
        break;
    default:
        return -1;
    }
    return 0;
}

// Geometry of one block from its ghost node mesh (mhd_geom.cuh): one thread
// per point of the padded box, one grid row per group (group0, group0 + 1, ...)
__global__ void k_geometry(const BlockView *__restrict__ bvs, int blk, NodeMesh m, int G, int group0, double b0,
                           double b1, double b2)
{
    const BlockView &b = bvs[blk];
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= b.vol)
        return;
    const int k = int(t % b.NK) - b.G;
    const int j = int((t / b.NK) % b.NJ) - b.G;
    const int i = int(t / (int64_t(b.NK) * b.NJ)) - b.G;
    const double gb[3] = {b0, b1, b2};
    geom_point(m, b, group0 + int(blockIdx.y), i, j, k, G, gb);
}

// output-step diagnostics: minima start at +inf, maxima at -inf, max |divB| at 0
__global__ void k_diag_init(unsigned long long *keys)
{
    const int t = threadIdx.x;
    if (t < DIAG_NMIN)
        keys[t] = diag_key(INFINITY);
    else if (t < DIAG_NMIN + DIAG_NQ - 1)
        keys[t] = diag_key(-INFINITY);
    else if (t == DIAG_NMIN + DIAG_NQ - 1)
        keys[t] = diag_key(0.0);
}

// one inner cell per thread, one grid row per block; NaN values are skipped
// (std::min / std::max keep the running value against a NaN)
__global__ void k_diag(const BlockView *__restrict__ bvs, int run, unsigned long long *keys)
{
    const BlockView &b = bvs[blockIdx.y];
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    unsigned long long kmin[DIAG_NMIN], kmax[DIAG_NQ];
#pragma unroll
    for (int q = 0; q < DIAG_NQ; ++q)
    {
        if (q < DIAG_NMIN)
            kmin[q] = ~0ull;
        kmax[q] = 0ull;
    }
    if ((run < 0 || b.run == run) && t < int64_t(b.ni) * b.nj * b.nk)
    {
        const int k = int(t % b.nk), j = int((t / b.nk) % b.nj), i = int(t / (int64_t(b.nk) * b.nj));
        double v[DIAG_NQ];
        diag_cell(b, i, j, k, v);
#pragma unroll
        for (int q = 0; q < DIAG_NQ; ++q)
            if (v[q] == v[q])
            {
                const unsigned long long key = diag_key(v[q]);
                if (q < DIAG_NMIN)
                    kmin[q] = key;
                kmax[q] = key;
            }
    }
#pragma unroll
    for (int q = 0; q < DIAG_NQ; ++q)
    {
        unsigned long long lo = (q < DIAG_NMIN) ? kmin[q] : ~0ull, hi = kmax[q];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1)
        {
            const unsigned long long olo = __shfl_xor_sync(0xffffffffu, lo, off);
            const unsigned long long ohi = __shfl_xor_sync(0xffffffffu, hi, off);
            lo = (olo < lo) ? olo : lo;
            hi = (ohi > hi) ? ohi : hi;
        }
        if ((threadIdx.x & 31) == 0)
        {
            if (q < DIAG_NMIN && lo != ~0ull)
                atomicMin(&keys[q], lo);
            if (hi != 0ull)
                atomicMax(&keys[DIAG_NMIN + q], hi);
        }
    }
}

// Pole handlers and repairs: one thread per pole_one work item (mhd_pole.cuh)
__global__ void k_pole(const BlockView *__restrict__ bvs, const int *__restrict__ poles, int op)
{
    const BlockView &b = bvs[poles[2 * blockIdx.y]];
    const int side = poles[2 * blockIdx.y + 1] > 0 ? 1 : -1;
    pole_one(b, side, op, int64_t(blockIdx.x) * blockDim.x + threadIdx.x);
}

// The J edges that read a B_zeta face the Pole rewrite changed (POLE_BZETA
// writes the first cell layer jc at each Pole: J_xi at j = jc, jc + 1 and
// J_eta at j = jc read it): Calc_J_Edge again on the staggered points
// j = jc, jc + 1 of each Pole, after the rewrite.  Every other J edge was
// formed before the rewrite, in the fused B_cell / J-edge pass, from the
// same faces, so the J edges are those of the reference's order (calc_Bcell
// with the rewrite, then Calc_J_Edge) bit for bit.  Work items per Pole:
// (ni + 1) x 2 x (nk + 1).
__global__ void k_pole_jedge(const BlockView *__restrict__ bvs, const int *__restrict__ poles)
{
    const BlockView &b = bvs[poles[2 * blockIdx.y]];
    const int side = poles[2 * blockIdx.y + 1] > 0 ? 1 : -1;
    const int jc = side < 0 ? 0 : b.nj - 1;
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= int64_t(b.ni + 1) * 2 * (b.nk + 1))
        return;
    const int k = int(t % (b.nk + 1)), j = jc + int((t / (b.nk + 1)) % 2), i = int(t / (2 * int64_t(b.nk + 1)));
#pragma unroll
    for (int ea = 0; ea < 2; ++ea)
        if (inner_of(b, 1, ea, i, j, k))
            jedge_one(b, ea, i, j, k, F_Bxi, F_Jxi, 1.0);
}

// ---------------------------------------------------------------------------
// The ring least squares of POLE_BCELL, POLE_EETA_REG and POLE_JCELL with one
// warp per ring.  The lanes form the pushed vectors and values of 32 k at a
// time (square roots and divisions in parallel, the same operations as
// pole_one).  Each sum then runs in one lane over the pushes in the
// reference's order (k, then the handler's order within k), so it equals the
// one-thread ring sum bit for bit: the normal matrix A and the count depend
// on the geometry only and are summed once per geometry (build), nine lanes
// one entry each; every application sums the right-hand side, three lanes
// one component each, and lane 0 regularises, solves and broadcasts.
// ---------------------------------------------------------------------------
constexpr int kPoleWarps = 4; // warps (rings) per CTA
constexpr int kPoleTerms = 8; // at most 8 pushes per k (J_cell)

struct PoleTerm
{
    double s[3], phi;
    int ok;
};

// one chunk of pushes: build: lane q < 9 sums s[q / 3] s[q % 3] (A), lane 9
// counts; apply: lane a < 3 sums phi s[a]
__device__ __forceinline__ void pole_accumulate(const PoleTerm *sh, int nterm, bool build, double &acc, int &cnt)
{
    const int lane = threadIdx.x & 31;
    if (build)
    {
        if (lane < 9)
        {
            const int a = lane / 3, c = lane % 3;
            for (int q = 0; q < nterm; ++q)
                if (sh[q].ok)
                    acc += sh[q].s[a] * sh[q].s[c];
        }
        else if (lane == 9)
            for (int q = 0; q < nterm; ++q)
                cnt += sh[q].ok ? 1 : 0;
    }
    else if (lane < 3)
        for (int q = 0; q < nterm; ++q)
            if (sh[q].ok)
                acc += sh[q].phi * sh[q].s[lane];
}

// build: store the ring's A and count (cache[0..8], cache[9]); apply: lane 0
// loads them, regularises (trace of |A_aa| or of A_aa), solves and
// broadcasts x.  status: 0 solved, 1 no usable push (count_guard), 2 singular
__device__ bool pole_finish(double acc, int cnt, bool build, double *cache, bool trace_abs, bool count_guard,
                            double x[3], int &status)
{
    const int lane = threadIdx.x & 31;
    if (build)
    {
        if (lane < 9)
            cache[lane] = acc;
        else if (lane == 9)
            cache[9] = double(cnt);
        status = 3;
        return false;
    }
    const double r0 = __shfl_sync(0xffffffffu, acc, 0), r1 = __shfl_sync(0xffffffffu, acc, 1),
                 r2 = __shfl_sync(0xffffffffu, acc, 2);
    int st = 0;
    double xs[3] = {0.0, 0.0, 0.0};
    if (lane == 0)
    {
        if (count_guard && int(cache[9]) <= 0)
            st = 1;
        else
        {
            double A[3][3] = {{cache[0], cache[1], cache[2]}, {cache[3], cache[4], cache[5]}, {cache[6], cache[7], cache[8]}};
            const double rhs[3] = {r0, r1, r2};
            const double tr = trace_abs ? fabs(A[0][0]) + fabs(A[1][1]) + fabs(A[2][2]) : A[0][0] + A[1][1] + A[2][2];
            const double reg = 1.0e-12 * pole_max1(tr);
            A[0][0] += reg;
            A[1][1] += reg;
            A[2][2] += reg;
            st = pole_solve3(A, rhs, xs) ? 0 : 2;
        }
    }
    status = __shfl_sync(0xffffffffu, st, 0);
#pragma unroll
    for (int c = 0; c < 3; ++c)
        x[c] = __shfl_sync(0xffffffffu, xs[c], 0);
    return status == 0;
}

__device__ void pole_bcell_warp(const BlockView &b, int side, int64_t t, PoleTerm *sh, double *cache, bool build)
{
    const int lane = threadIdx.x & 31;
    const int nj = b.nj, nk = b.nk;
    const int64_t v = b.vol;
    const int i = int(t >> 1);
    const bool total = (t & 1) == 0;
    if (build && !total)
        return; // one A per ring, shared by the total and the induced field
    const int jc = side < 0 ? 0 : nj - 1;
    const int jn = side < 0 ? jc + 1 : jc;
    const double sn = side < 0 ? 1.0 : -1.0;
    const double *Aet = b.f[F_JDeta], *Axi = b.f[F_JDxi];
    const double *Bet = b.f[F_Beta], *Bxi = b.f[F_Bxi], *Aadd = b.f[F_Baddeta], *Xadd = b.f[F_Baddxi];
    double acc = 0.0;
    int cnt = 0;
    for (int k0 = 0; k0 < nk; k0 += 32)
    {
        const int k = k0 + lane;
        if (k < nk)
        {
            const int64_t pn = pidx(b, i, jn, k), p0 = pidx(b, i, jc, k), p1 = pidx(b, i + 1, jc, k);
            PoleTerm *o = sh + 3 * lane;
            double f = Bet[pn];
            if (total)
                f += Aadd[pn];
            o[0] = PoleTerm{{sn * Aet[pn], sn * Aet[v + pn], sn * Aet[2 * v + pn]}, sn * f, 0};
            f = Bxi[p0];
            if (total)
                f += Xadd[p0];
            o[1] = PoleTerm{{-Axi[p0], -Axi[v + p0], -Axi[2 * v + p0]}, -f, 0};
            f = Bxi[p1];
            if (total)
                f += Xadd[p1];
            o[2] = PoleTerm{{Axi[p1], Axi[v + p1], Axi[2 * v + p1]}, f, 0};
            for (int q = 0; q < 3; ++q)
            {
                const double *S = o[q].s;
                o[q].ok = !((S[0] * S[0] + S[1] * S[1] + S[2] * S[2]) <= 1.0e-300);
            }
        }
        __syncwarp();
        pole_accumulate(sh, 3 * min(32, nk - k0), build, acc, cnt);
        __syncwarp();
    }
    // BC_Pole_Bcell_Collapse_ solves whenever the regularised system is regular
    double Bp[3];
    int st;
    if (!pole_finish(acc, cnt, build, cache, true, false, Bp, st))
        return;
    double *Out = b.f[total ? F_Bcell : F_Bind];
    for (int k = lane; k < nk; k += 32)
    {
        const int64_t p = pidx(b, i, jc, k);
        Out[p] = Bp[0];
        Out[v + p] = Bp[1];
        Out[2 * v + p] = Bp[2];
    }
}

// the regulation of E_eta (field F_Eeta) or Eres_eta (F_Ereseta): both are
// eta edges of the same ring, so their normal matrices (from dr_eta) are one
__device__ void pole_eeta_warp(const BlockView &b, int side, int64_t t, PoleTerm *sh, double *cache, bool build,
                               int field)
{
    const int lane = threadIdx.x & 31;
    const int nj = b.nj, nk = b.nk;
    const int64_t v = b.vol;
    const int i = int(t);
    const int jc = side < 0 ? 0 : nj - 1;
    double *E = b.f[field];
    const double *dr = b.f[F_dreta];
    double acc = 0.0;
    int cnt = 0;
    for (int k0 = 0; k0 < nk; k0 += 32) // k = n_k is the same edge as k = 0
    {
        const int k = k0 + lane;
        if (k < nk)
        {
            const int64_t p = pidx(b, i, jc, k);
            const double d0 = dr[p], d1 = dr[v + p], d2 = dr[2 * v + p];
            const double L = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
            PoleTerm &o = sh[lane];
            o.ok = !(L < 1.0e-14);
            if (o.ok)
            {
                const double invL = 1.0 / L;
                o.s[0] = d0 * invL;
                o.s[1] = d1 * invL;
                o.s[2] = d2 * invL;
                o.phi = build ? 0.0 : E[p] * invL;
            }
        }
        __syncwarp();
        pole_accumulate(sh, min(32, nk - k0), build, acc, cnt);
        __syncwarp();
    }
    double Ev[3];
    int st;
    if (pole_finish(acc, cnt, build, cache, false, true, Ev, st))
    {
        for (int k = lane; k <= nk; k += 32)
        {
            const int64_t p = pidx(b, i, jc, k);
            const double d0 = dr[p], d1 = dr[v + p], d2 = dr[2 * v + p];
            const double L = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
            E[p] = (L < 1.0e-14) ? 0.0 : Ev[0] * d0 + Ev[1] * d1 + Ev[2] * d2;
        }
        return;
    }
    if (st == 1) // no usable edge
    {
        for (int k = lane; k <= nk; k += 32)
            E[pidx(b, i, jc, k)] = 0.0;
        return;
    }
    if (st != 2)
        return; // build
    // singular system: the ring average, summed in k order by lane 0
    double avg = 0.0;
    if (lane == 0)
    {
        for (int k = 0; k <= nk; ++k)
            avg += E[pidx(b, i, jc, k)];
        avg /= double(nk + 1);
    }
    avg = __shfl_sync(0xffffffffu, avg, 0);
    for (int k = lane; k <= nk; k += 32)
        E[pidx(b, i, jc, k)] = avg;
}

__device__ void pole_jcell_warp(const BlockView &b, int side, int64_t t, PoleTerm *sh, double *cache, bool build)
{
    const int lane = threadIdx.x & 31;
    const int nj = b.nj, nk = b.nk;
    const int64_t v = b.vol;
    const int i = int(t);
    const int jc = side < 0 ? 0 : nj - 1;
    const int jt = side < 0 ? jc + 1 : jc; // node plane one layer away from the Pole
    // the 8 pushes of each k, in the order of the reference's loop
    const int di[8] = {0, 1, 0, 1, 0, 0, 0, 1};
    const int dk[8] = {0, 0, 1, 1, 0, 1, 0, 0};
    const int fj[8] = {F_Jeta, F_Jeta, F_Jeta, F_Jeta, F_Jxi, F_Jxi, F_Jzeta, F_Jzeta};
    const int fd[8] = {F_dreta, F_dreta, F_dreta, F_dreta, F_drxi, F_drxi, F_drzeta, F_drzeta};
    double acc = 0.0;
    int cnt = 0;
    for (int k0 = 0; k0 < nk; k0 += 32)
    {
        const int k = k0 + lane;
        if (k < nk)
        {
#pragma unroll
            for (int q = 0; q < 8; ++q)
            {
                const int64_t p = pidx(b, i + di[q], q < 4 ? jc : jt, k + dk[q]);
                const double *dr = b.f[fd[q]];
                const double dx = dr[p], dy = dr[v + p], dz = dr[2 * v + p];
                const double L = sqrt(dx * dx + dy * dy + dz * dz);
                PoleTerm &o = sh[8 * lane + q];
                o.ok = !(L < 1.0e-14);
                if (o.ok)
                {
                    o.s[0] = dx / L;
                    o.s[1] = dy / L;
                    o.s[2] = dz / L;
                    o.phi = build ? 0.0 : b.f[fj[q]][p] / L;
                }
            }
        }
        __syncwarp();
        pole_accumulate(sh, 8 * min(32, nk - k0), build, acc, cnt);
        __syncwarp();
    }
    double Jp[3];
    int st;
    if (!pole_finish(acc, cnt, build, cache, false, true, Jp, st))
        return;
    double *Jc = b.f[F_Jcell];
    for (int k = lane; k < nk; k += 32)
    {
        const int64_t p = pidx(b, i, jc, k);
        Jc[p] = Jp[0];
        Jc[v + p] = Jp[1];
        Jc[2 * v + p] = Jp[2];
    }
}

// which of the three least-squares operations (cache slot), -1 otherwise
__host__ __device__ inline int pole_lsq_slot(int op)
{
    return op == POLE_BCELL ? 0 : (op == POLE_EETA_REG || op == POLE_ERES_REG) ? 1 : op == POLE_JCELL ? 2 : -1;
}

// cache: per Pole, per least-squares operation, per ring i (stride rings):
// A (9 values) and the push count
__global__ void __launch_bounds__(32 * kPoleWarps) k_pole_warp(const BlockView *__restrict__ bvs,
                                                               const int *__restrict__ poles, int op,
                                                               double *__restrict__ cache, int stride, int build)
{
    __shared__ PoleTerm sh[kPoleWarps][32 * kPoleTerms];
    const BlockView &b = bvs[poles[2 * blockIdx.y]];
    const int side = poles[2 * blockIdx.y + 1] > 0 ? 1 : -1;
    const int warp = threadIdx.x >> 5;
    const int64_t t = int64_t(blockIdx.x) * kPoleWarps + warp;
    if (t >= pole_work(op, b.ni, b.nk))
        return; // the whole warp leaves together
    const int ring = (op == POLE_BCELL) ? int(t >> 1) : int(t);
    double *c = cache + ((int64_t(blockIdx.y) * 3 + pole_lsq_slot(op)) * stride + ring) * 10;
    if (op == POLE_BCELL)
        pole_bcell_warp(b, side, t, sh[warp], c, build != 0);
    else if (op == POLE_EETA_REG || op == POLE_ERES_REG)
        pole_eeta_warp(b, side, t, sh[warp], c, build != 0, op == POLE_ERES_REG ? F_Ereseta : F_Eeta);
    else
        pole_jcell_warp(b, side, t, sh[warp], c, build != 0);
}

void launch_pole_op(int op, int64_t work, int npoles, cudaStream_t st, const BlockView *bvs, const int *poles,
                    double *cache, int stride, int build)
{
    if (pole_lsq_slot(op) >= 0)
        k_pole_warp<<<dim3(unsigned((work + kPoleWarps - 1) / kPoleWarps), unsigned(npoles)), 32 * kPoleWarps, 0,
                      st>>>(bvs, poles, op, cache, stride, build);
    else if (!build)
        k_pole<<<dim3(unsigned((work + 255) / 256), unsigned(npoles)), 256, 0, st>>>(bvs, poles, op);
}

} // namespace mhd
