// Mixed-precision kernels (MHD_PREC_MIXED).  The Rusanov face fluxes of the
// fluid right-hand side are evaluated in FP32 and accumulated in FP32, in
// deviation form: the face states are stored as FP32 deviations from a
// constant reference state q0 (the far-field inflow), and each face computes
//     dF = Rusanov(qL, qR; k) - Phi0(k),   Phi0(k) = F_phys(q0) . k
// from the deviations with the algebra rearranged so that no large term is
// formed and then cancelled (rho U - rho0 U0 = drho U + rho0 dU, etc.).  The
// part Phi0 is linear in the face vector k, so its divergence is
// Phi0(sum of the cell's signed face vectors), evaluated in FP64 from the
// FP64 metric.  FP32 rounding therefore scales with the departure from q0,
// not with the flux itself.  The J x B source, the stored RHS_H, the
// conserved update, the contravariant velocities of the CT EMF, the EMF
// itself, its curl and the face-B update stay FP64 (the contravariant
// velocities here, the rest in other translation units), so div B stays at
// FP64 round-off.  Compiled without contracted multiply-adds, so that the
// per-cell and the face-tiled flux kernels give the same bits.
#include "mhd_kernels.cuh"

namespace mhd
{

__device__ __forceinline__ float fmaxs(float a, float b) { return (a < b) ? b : a; }

// FP32 copies of the face areas |JD|, the unit face normals and the
// B_cell / J_cell least-squares weights on every point of the padded box
__global__ void k_geom32(const BlockView *__restrict__ bvs)
{
    const BlockView &b = bvs[blockIdx.y];
    const int64_t v = b.vol;
    const int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= v)
        return;
#pragma unroll
    for (int a = 0; a < 3; ++a)
    {
        b.g32[(G32_AREA + a) * v + p] = float(b.f[F_NAxi + a][p]);
#pragma unroll
        for (int c = 0; c < 3; ++c)
            b.g32[(G32_NRM + 3 * a + c) * v + p] = float(b.f[F_NAxi + a][(1 + c) * v + p]);
    }
    for (int q = 0; q < 18; ++q)
        b.w32[(W32_B + q) * v + p] = float(b.f[F_WB][q * v + p]);
    for (int q = 0; q < 36; ++q)
        b.w32[(W32_J + q) * v + p] = float(b.f[F_WJ][q * v + p]);
}

// reference-state constants of the deviation flux, FP32
struct Ref32
{
    float rho, u[3], H; // rho0, u0, E0 + p0
};

// one Rusanov face flux minus the reference-state flux Phi0(k), in FP32:
// face vector (k1, k2, k3), face area, left cell pL, right cell p.  Per side,
// with U = k . u = U0 + dU:
//   mass    rho U - rho0 U0               = drho U + rho0 dU          (= dm)
//   mom x   rho U u + k1 p - (same at q0) = dm u + rho0 U0 du + k1 dp
//   energy  U (E + p) - U0 (E0 + p0)      = dU (E + p) + U0 (dE + dp)
// and the dissipation uses conserved differences of the deviations
// (rho u - rho0 u0 = drho u + rho0 du).
// the FP32 face states of a cell: its planes in the pool (index: the cell's
// pool offset) or in a tile staged in shared memory (index: its place there)
struct QPool
{
    const float *q;
    int64_t v;
    __device__ __forceinline__ float operator()(int plane, int64_t c) const { return q[plane * v + c]; }
};
constexpr int QS_I = TILE_I + 2, QS_J = TILE_J + 2, QS_K = TILE_K + 2; // a tile and one halo cell each side
constexpr int QS_N = QS_I * QS_J * QS_K;
struct QTile
{
    const float *q;
    __device__ __forceinline__ float operator()(int plane, int64_t c) const { return q[plane * QS_N + c]; }
};

template <class Q>
__device__ __forceinline__ void rusanov_dev32q(const Q &q, const Ref32 &r0, float k1, float k2, float k3, float area,
                                               int64_t p, int64_t pL, float out[5])
{
    const float U0 = k1 * r0.u[0] + k2 * r0.u[1] + k3 * r0.u[2];
    float dF[2][5], dC[2][5], rad = 0.0f;
#pragma unroll
    for (int s = 0; s < 2; ++s)
    {
        const int64_t c = s ? p : pL;
        const float dr = q(Q32_RHO, c);
        const float du = q(Q32_U, c), dv = q(Q32_U + 1, c), dw = q(Q32_U + 2, c);
        const float dp = q(Q32_P, c), dE = q(Q32_RHOE, c), cs = q(Q32_C, c);
        const float u = r0.u[0] + du, vv = r0.u[1] + dv, w = r0.u[2] + dw;
        const float dU = k1 * du + k2 * dv + k3 * dw;
        const float U = U0 + dU;
        const float dm = dr * U + r0.rho * dU;
        const float mU0 = r0.rho * U0;
        dF[s][0] = dm;
        dF[s][1] = dm * u + mU0 * du + k1 * dp;
        dF[s][2] = dm * vv + mU0 * dv + k2 * dp;
        dF[s][3] = dm * w + mU0 * dw + k3 * dp;
        dF[s][4] = dU * (r0.H + dE + dp) + U0 * (dE + dp);
        dC[s][0] = dr;
        dC[s][1] = dr * u + r0.rho * du;
        dC[s][2] = dr * vv + r0.rho * dv;
        dC[s][3] = dr * w + r0.rho * dw;
        dC[s][4] = dE;
        rad = fmaxs(rad, fabsf(U) + cs * area);
    }
#pragma unroll
    for (int m = 0; m < 5; ++m)
        out[m] = 0.5f * (dF[0][m] + dF[1][m]) - 0.5f * rad * (dC[1][m] - dC[0][m]);
}

__device__ __forceinline__ void rusanov_dev32(const BlockView &b, const Ref32 &r0, float k1, float k2, float k3,
                                              float area, int64_t p, int64_t pL, float out[5])
{
    rusanov_dev32q(QPool{b.q32, b.vol}, r0, k1, k2, k3, area, p, pL, out);
}

// RHS_H of one inner cell from its FP32 flux-deviation sum r: the FP64
// divergence of the reference-state flux Phi0(S) (S the sum of the cell's
// signed face vectors), the FP64 J x B force with the Hall_Num_Limiter weight
// and its work, over the FP64 cell volume
__device__ __forceinline__ void mixed_rhs(const BlockView &b, const Consts &c, int64_t p, double jac,
                                          const double S[3], const float r[5])
{
    const int64_t v = b.vol;
    const double *q0 = b.qref;
    const double US = S[0] * q0[1] + S[1] * q0[2] + S[2] * q0[3];
    const double mS = q0[0] * US;
    const double phi[5] = {mS, mS * q0[1] + S[0] * q0[4], mS * q0[2] + S[1] * q0[4], mS * q0[3] + S[2] * q0[4],
                           US * (q0[5] + q0[4])};
    const double rho = b.f[F_U][p];
    const double n_true = ((rho < 0.0) ? 0.0 : rho) / c.M_H * c.M_ref;
    const double fc = c.mom_hall * (n_true / sqrt(n_true * n_true + c.ne_floor * c.ne_floor));
    const double *J = b.f[F_Jcell], *B = b.f[F_Bcell], *U = b.f[F_U];
    const double jx = J[p], jy = J[v + p], jz = J[2 * v + p];
    const double bx = B[p], by = B[v + p], bz = B[2 * v + p];
    const double fx = jy * bz - jz * by, fy = jz * bx - jx * bz, fz = jx * by - jy * bx;
    const double invJ = 1.0 / jac;
    // the work uses calc_PV's velocities U_m / max(rho, 1e-12) (the mixed
    // form's derived pass leaves PV_H to read-out), as one quotient
    const double rho_pv = (rho < 1e-12) ? 1e-12 : rho;
    const double fU = fx * U[v + p] + fy * U[2 * v + p] + fz * U[3 * v + p];
    double *R = b.f[F_RHS];
    R[p] = -(double(r[0]) + phi[0]) * invJ;
    R[v + p] = -(double(r[1]) + phi[1]) * invJ + fc * fx;
    R[2 * v + p] = -(double(r[2]) + phi[2]) * invJ + fc * fy;
    R[3 * v + p] = -(double(r[3]) + phi[3]) * invJ + fc * fz;
    R[4 * v + p] = -(double(r[4]) + phi[4]) * invJ + fc * (fU / rho_pv);
}

// Fluid RHS of the inner cells (FP32 flux divergence, FP64 J x B source) and
// the FP64 contravariant velocities of the cells within one ghost layer; the
// FP64 face metric read for the velocities is the one the fluxes round.
// variants: at least 3 CTAs per SM (80 registers; the default: 1.73 -> 1.52 ms
// per step on the shell sweep against 2 CTAs per SM), uncapped (96
// registers), at least 2
__device__ __forceinline__ void k_fluid_mixed_body(const BlockView *__restrict__ bvs, Consts c)
{
    int64_t t;
    const BlockView &b = bvs[cta_block(bvs, KIND_CELL1, t)];
    const int lo = -1;
    const int n0 = b.ni + 2, n1 = b.nj + 2, n2 = b.nk + 2;
    if (t >= int64_t(n0) * n1 * n2)
        return;
    const int k = lo + int(t % n2);
    t /= n2;
    const int j = lo + int(t % n1);
    const int i = lo + int(t / n1);
    const int64_t v = b.vol;
    const int64_t p = pidx(b, i, j, k);
    const double jac = b.f[F_Jac][p];
    const bool inner = i >= 0 && j >= 0 && k >= 0 && i < b.ni && j < b.nj && k < b.nk;
    // contravariant velocities (cell_u_contra): (k-bar . U_plus) / (|Jac| + 1e-30)
    const double *Up = b.f[F_Uplus];
    const double ux = Up[p], uy = Up[v + p], uz = Up[2 * v + p];
    const double inv_jac = 1.0 / (fabs(jac) + 1.0e-30);
    double *UC = b.f[F_UC];
    const float *g = b.g32;
    const double *q0 = b.qref;
    const Ref32 r0 = {float(q0[0]), {float(q0[1]), float(q0[2]), float(q0[3])}, float(q0[5] + q0[4])};
    // one axis at a time: its face metric at the low (p) and high (pp) face,
    // the cell's velocity along it, its share of the FP64 sum of signed face
    // vectors, and (inner cells) its two FP32 face fluxes -- the same
    // operations in the same order as forming all three axes first, with a
    // third of the metric live at once
    double S[3] = {0.0, 0.0, 0.0};
    float r[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int a = 0; a < 3; ++a)
    {
        const int64_t pp = a == 0 ? pidx(b, i + 1, j, k) : a == 1 ? pidx(b, i, j + 1, k) : pidx(b, i, j, k + 1);
        const double *M = b.f[F_JDxi + a];
        double m_[3], p_[3];
        float km[3], kp[3];
#pragma unroll
        for (int d = 0; d < 3; ++d)
        {
            m_[d] = M[d * v + p];
            p_[d] = M[d * v + pp];
            km[d] = float(m_[d]);
            kp[d] = float(p_[d]);
            S[d] += p_[d] - m_[d];
        }
        const double kx = 0.5 * (m_[0] + p_[0]);
        const double ky = 0.5 * (m_[1] + p_[1]);
        const double kz = 0.5 * (m_[2] + p_[2]);
        UC[a * v + p] = (kx * ux + ky * uy + kz * uz) * inv_jac;
        if (inner)
        {
            const int64_t pm = a == 0 ? pidx(b, i - 1, j, k) : a == 1 ? pidx(b, i, j - 1, k) : pidx(b, i, j, k - 1);
            float Fm[5], Fp[5];
            rusanov_dev32(b, r0, km[0], km[1], km[2], g[(G32_AREA + a) * v + p], p, pm, Fm);
            rusanov_dev32(b, r0, kp[0], kp[1], kp[2], g[(G32_AREA + a) * v + pp], pp, p, Fp);
#pragma unroll
            for (int m = 0; m < 5; ++m)
                r[m] += Fp[m] - Fm[m];
        }
    }
    if (inner)
        mixed_rhs(b, c, p, jac, S, r);
}

template <int MINB>
__global__ void __launch_bounds__(256, MINB) k_fluid_mixed_t(const BlockView *__restrict__ bvs, Consts c)
{
    k_fluid_mixed_body(bvs, c);
}
// the compiler's own register allocation (no launch bounds)
__global__ void k_fluid_mixed_free(const BlockView *__restrict__ bvs, Consts c)
{
    k_fluid_mixed_body(bvs, c);
}


// ---------------------------------------------------------------------------
// Face-tiled variants: a CTA covers TILE_I x TILE_J x TILE_K cells of the
// depth-1 box (k fastest, one warp per (i, j) row of 32 k).  Every thread
// forms its cell's contravariant velocities as above; then each face flux
// needed by an inner cell is evaluated once -- a cell's three low faces by its
// own thread, the high faces of the tile's last layer in each direction by the
// threads of that layer -- into shared memory, and after one barrier each
// inner cell sums its six faces.  The two cells of a face call the same flux
// with the same arguments (face metric and area of the face, the two cells'
// states), so the fluxes and the RHS are bit for bit those of the per-cell
// variant (the file is compiled without contracted multiply-adds).
//
// STAGED: the FP32 face states of the tile and a one-cell halo are copied
// into shared memory with asynchronous copies issued first thing, which run
// while the threads form the FP64 contravariant velocities; the fluxes then
// read them there.  The loads are in flight without holding registers.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void cp_async4(float *dst, const float *src)
{
    const unsigned d = unsigned(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all()
{
    asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;\n" ::: "memory");
}

template <bool STAGED> __device__ __forceinline__ void k_fluid_mixed_tile_body(const BlockView *__restrict__ bvs, Consts c)
{
    __shared__ float Fx[TILE_I + 1][TILE_J][TILE_K][5];
    __shared__ float Fy[TILE_I][TILE_J + 1][TILE_K][5];
    __shared__ float Fz[TILE_I][TILE_J][TILE_K + 1][5];
    __shared__ float qs[STAGED ? 7 * QS_N : 1];
    int64_t t;
    const BlockView &b = bvs[cta_block(bvs, KIND_TILE1, t)];
    const int ntj = (b.nj + 2 + TILE_J - 1) / TILE_J, ntk = (b.nk + 2 + TILE_K - 1) / TILE_K;
    const int64_t tile = t / 256;
    if (tile >= int64_t((b.ni + 2 + TILE_I - 1) / TILE_I) * ntj * ntk)
        return; // the whole CTA
    const int i0 = -1 + int(tile / (int64_t(ntj) * ntk)) * TILE_I;
    const int j0 = -1 + int((tile / ntk) % ntj) * TILE_J;
    const int k0 = -1 + int(tile % ntk) * TILE_K;
    const int64_t v = b.vol;
    if (STAGED)
    {
        // the tile's cells and one halo cell each side, where the padded
        // array has them (the halo beyond the box's last cell is never read)
        const int G = b.G;
        for (int e = threadIdx.x; e < QS_N; e += blockDim.x)
        {
            const int gk = k0 - 1 + e % QS_K, gj = j0 - 1 + (e / QS_K) % QS_J, gi = i0 - 1 + e / (QS_K * QS_J);
            if (gi < -G || gj < -G || gk < -G || gi > b.ni + G || gj > b.nj + G || gk > b.nk + G)
                continue;
            const int64_t gp = pidx(b, gi, gj, gk);
#pragma unroll
            for (int m = 0; m < 7; ++m)
                cp_async4(&qs[m * QS_N + e], &b.q32[m * v + gp]);
        }
    }
    const int tk = threadIdx.x & 31, tj = (threadIdx.x >> 5) % TILE_J, ti = (threadIdx.x >> 5) / TILE_J;
    const int i = i0 + ti, j = j0 + tj, k = k0 + tk;
    const bool valid = i <= b.ni && j <= b.nj && k <= b.nk;
    const bool inner = i >= 0 && j >= 0 && k >= 0 && i < b.ni && j < b.nj && k < b.nk;
    const int64_t p = pidx(b, i, j, k);
    const int64_t pp[3] = {pidx(b, i + 1, j, k), pidx(b, i, j + 1, k), pidx(b, i, j, k + 1)};
    const int64_t pm[3] = {pidx(b, i - 1, j, k), pidx(b, i, j - 1, k), pidx(b, i, j, k - 1)};
    // the same cells in the staged tile
    const int64_t sp = (int64_t(ti + 1) * QS_J + (tj + 1)) * QS_K + (tk + 1);
    const int64_t sd[3] = {int64_t(QS_J) * QS_K, QS_K, 1};
    float km[3][3], kp[3][3];
    double S[3] = {0.0, 0.0, 0.0};
    double jac = 0.0;
    if (valid)
    {
        jac = b.f[F_Jac][p];
        const double *Up = b.f[F_Uplus];
        const double ux = Up[p], uy = Up[v + p], uz = Up[2 * v + p];
        const double inv_jac = 1.0 / (fabs(jac) + 1.0e-30);
        double *UC = b.f[F_UC];
#pragma unroll
        for (int a = 0; a < 3; ++a)
        {
            const double *M = b.f[F_JDxi + a];
            double m_[3], p_[3];
#pragma unroll
            for (int d = 0; d < 3; ++d)
            {
                m_[d] = M[d * v + p];
                p_[d] = M[d * v + pp[a]];
                km[a][d] = float(m_[d]);
                kp[a][d] = float(p_[d]);
                S[d] += p_[d] - m_[d];
            }
            const double kx = 0.5 * (m_[0] + p_[0]);
            const double ky = 0.5 * (m_[1] + p_[1]);
            const double kz = 0.5 * (m_[2] + p_[2]);
            UC[a * v + p] = (kx * ux + ky * uy + kz * uz) * inv_jac;
        }
    }
    if (STAGED)
    {
        cp_async_wait_all();
        __syncthreads();
    }
    const double *q0 = b.qref;
    const Ref32 r0 = {float(q0[0]), {float(q0[1]), float(q0[2]), float(q0[3])}, float(q0[5] + q0[4])};
    const float *g = b.g32;
    // the low face of axis a of this cell joins cells -1 and 0 along a: needed
    // by an inner cell when the cell's own index along a is in [0, n_a] and
    // the other two are inner
    const int idx[3] = {i, j, k}, n[3] = {b.ni, b.nj, b.nk};
    const int last[3] = {ti == TILE_I - 1, tj == TILE_J - 1, tk == TILE_K - 1};
    if (valid)
    {
#pragma unroll
        for (int a = 0; a < 3; ++a)
        {
            bool others = true;
#pragma unroll
            for (int d = 0; d < 3; ++d)
                if (d != a && (idx[d] < 0 || idx[d] >= n[d]))
                    others = false;
            if (!others)
                continue;
            float F[5];
            if (idx[a] >= 0 && idx[a] <= n[a])
            {
                if (STAGED)
                    rusanov_dev32q(QTile{qs}, r0, km[a][0], km[a][1], km[a][2], g[(G32_AREA + a) * v + p], sp,
                                   sp - sd[a], F);
                else
                    rusanov_dev32(b, r0, km[a][0], km[a][1], km[a][2], g[(G32_AREA + a) * v + p], p, pm[a], F);
                float *dst = a == 0 ? Fx[ti][tj][tk] : a == 1 ? Fy[ti][tj][tk] : Fz[ti][tj][tk];
#pragma unroll
                for (int m = 0; m < 5; ++m)
                    dst[m] = F[m];
            }
            // the high face of the tile's last layer (the next tile's low face)
            if (last[a] && idx[a] + 1 >= 0 && idx[a] + 1 <= n[a])
            {
                if (STAGED)
                    rusanov_dev32q(QTile{qs}, r0, kp[a][0], kp[a][1], kp[a][2], g[(G32_AREA + a) * v + pp[a]],
                                   sp + sd[a], sp, F);
                else
                    rusanov_dev32(b, r0, kp[a][0], kp[a][1], kp[a][2], g[(G32_AREA + a) * v + pp[a]], pp[a], p, F);
                float *dst = a == 0 ? Fx[TILE_I][tj][tk] : a == 1 ? Fy[ti][TILE_J][tk] : Fz[ti][tj][TILE_K];
#pragma unroll
                for (int m = 0; m < 5; ++m)
                    dst[m] = F[m];
            }
        }
    }
    __syncthreads();
    if (!inner)
        return;
    float r[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
    {
        const float *Fm = Fx[ti][tj][tk], *Fp = Fx[ti + 1][tj][tk];
#pragma unroll
        for (int m = 0; m < 5; ++m)
            r[m] += Fp[m] - Fm[m];
    }
    {
        const float *Fm = Fy[ti][tj][tk], *Fp = Fy[ti][tj + 1][tk];
#pragma unroll
        for (int m = 0; m < 5; ++m)
            r[m] += Fp[m] - Fm[m];
    }
    {
        const float *Fm = Fz[ti][tj][tk], *Fp = Fz[ti][tj][tk + 1];
#pragma unroll
        for (int m = 0; m < 5; ++m)
            r[m] += Fp[m] - Fm[m];
    }
    mixed_rhs(b, c, p, jac, S, r);
}

__global__ void __launch_bounds__(256, 2) k_fluid_mixed_tile(const BlockView *__restrict__ bvs, Consts c)
{
    k_fluid_mixed_tile_body<false>(bvs, c);
}

__global__ void __launch_bounds__(256, 2) k_fluid_mixed_staged(const BlockView *__restrict__ bvs, Consts c)
{
    k_fluid_mixed_tile_body<true>(bvs, c);
}

// launchers of the register / occupancy variants (tuned by mhd_autotune);
// variant 3 is the face-tiled kernel, 4 the same with the staged face states
// (both on the KIND_TILE1 grid)
int launch_k_fluid_mixed(int variant, dim3 grid, cudaStream_t st, const BlockView *bvs, Consts c)
{
    switch (variant)
    {
    case 3:
        k_fluid_mixed_tile<<<grid, 256, 0, st>>>(bvs, c);
        break;
    case 4:
        k_fluid_mixed_staged<<<grid, 256, 0, st>>>(bvs, c);
        break;
    case 0:
        k_fluid_mixed_t<3><<<grid, 256, 0, st>>>(bvs, c);
        break;
    case 1:
        k_fluid_mixed_free<<<grid, 256, 0, st>>>(bvs, c);
        break;
    case 2:
        k_fluid_mixed_t<2><<<grid, 256, 0, st>>>(bvs, c);
        break;
    default:
        return -1;
    }
    return 0;
}

} // namespace mhd
