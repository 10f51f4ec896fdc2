// Host build of the device geometry builder's points (beta1_b200/csrc/mhd_geom.cuh)
// for the CPU tests: the same source the kernel k_geometry runs, compiled for
// the host without contracted multiply-adds.  Test infrastructure.
#define __host__
#define __device__
#define __forceinline__ inline
#include "../beta1_b200/csrc/mhd_geom.cuh"

// one group of a block's geometry on every point of its padded box; fields
// as in the library (component planes of vol doubles, library field order)
extern "C" int geom_host(int ni, int nj, int nk, int G, const double *nodes, double **fields, int nfields, int group,
                         const double *gb)
{
    if (nfields != mhd::NFIELD || group < 0 || group >= mhd::NGEOM_GROUP)
        return 1;
    mhd::BlockView b{};
    for (int f = 0; f < mhd::NFIELD; ++f)
        b.f[f] = fields[f];
    b.ni = ni;
    b.nj = nj;
    b.nk = nk;
    b.G = G;
    b.NJ = nj + 1 + 2 * G;
    b.NK = nk + 1 + 2 * G;
    b.vol = int64_t(ni + 1 + 2 * G) * b.NJ * b.NK;
    const int off = G + 1;
    const mhd::NodeMesh m{nodes, off, nj + 1 + 2 * off, nk + 1 + 2 * off};
    for (int64_t t = 0; t < b.vol; ++t)
    {
        const int k = int(t % b.NK) - G;
        const int j = int((t / b.NK) % b.NJ) - G;
        const int i = int(t / (int64_t(b.NK) * b.NJ)) - G;
        mhd::geom_point(m, b, group, i, j, k, G, gb);
    }
    return 0;
}
