// Host build of the Pole work items of beta1_b200/csrc/mhd_pole.cuh for the
// CPU tests: the same source the device kernel k_pole runs, compiled for the
// host without contracted multiply-adds (IEEE +, -, *, / and sqrt round as
// on the device).  Test infrastructure.
#define __host__
#define __device__
#define __forceinline__ inline
#include "../beta1_b200/csrc/mhd_pole.cuh"

// runs every work item of one operation on one Pole of a block whose fields
// are host arrays on the padded box (fields[f]: component planes of vol
// doubles, in the library's field order)
extern "C" int pole_host(int op, int side, int ni, int nj, int nk, int G, double **fields, int nfields)
{
    if (nfields != mhd::NFIELD || op < 0 || op >= mhd::NPOLE_OP || (side != -1 && side != 1))
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
    const int64_t w = mhd::pole_work(op, ni, nk);
    for (int64_t t = 0; t < w; ++t)
        mhd::pole_one(b, side, op, t);
    return 0;
}

extern "C" int pole_nfields() { return mhd::NFIELD; }
