// Output-step diagnostics on the device (LunarSolver::PrintMinMaxDiagnostics_,
// Z4_Lunar/src/tools/LunarSolver_PrintDiag.cpp:7-85): per inner cell the
// values whose minima and maxima the reference prints, and an
// order-preserving integer key of a double for atomic min / max.  Shared by
// the kernel k_diag and host builds of the same code.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>

#include "mhd_layout.cuh"

namespace mhd
{

// quantities: rho, p, Bx, By, Bz, |B|^2 / 2 (minimum and maximum), |divB| (maximum)
constexpr int DIAG_NQ = 7;
constexpr int DIAG_NMIN = 6;

__host__ __device__ inline void diag_cell(const BlockView &b, int i, int j, int k, double v[DIAG_NQ])
{
    const int64_t vol = b.vol;
    const int64_t p = pidx(b, i, j, k);
    const double bx = b.f[F_Bcell][p], by = b.f[F_Bcell][vol + p], bz = b.f[F_Bcell][2 * vol + p];
    v[0] = b.f[F_U][p];
    v[1] = b.f[F_PV][3 * vol + p];
    v[2] = bx;
    v[3] = by;
    v[4] = bz;
    v[5] = 0.5 * (bx * bx + by * by + bz * bz);
    v[6] = fabs(b.f[F_divB][p]);
}

// unsigned key with key(a) < key(b) iff a < b for ordered doubles (-0 below +0)
__host__ __device__ inline unsigned long long diag_key(double x)
{
    unsigned long long u;
    memcpy(&u, &x, sizeof u);
    return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}

__host__ __device__ inline double diag_unkey(unsigned long long k)
{
    const unsigned long long u = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
    double x;
    memcpy(&x, &u, sizeof x);
    return x;
}

} // namespace mhd
