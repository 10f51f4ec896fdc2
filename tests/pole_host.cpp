// Host build of the Pole work items of beta1_b200/csrc/mhd_pole.cuh and of
// the output diagnostics of mhd_output.cuh for the CPU tests: the same source
// the device kernels k_pole and k_diag run, compiled for the host without
// contracted multiply-adds (IEEE +, -, *, / and sqrt round as on the
// device).  Test infrastructure.
#define __host__
#define __device__
#define __forceinline__ inline
#include "../beta1_b200/csrc/mhd_pole.cuh"
#include "../beta1_b200/csrc/mhd_output.cuh"

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

static mhd::BlockView host_view(int ni, int nj, int nk, int G, double **fields)
{
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
    return b;
}

// k_diag's reduction over one block, sequentially: mins[6], maxs[7]
extern "C" int diag_host(int ni, int nj, int nk, int G, double **fields, int nfields, double *mins, double *maxs)
{
    if (nfields != mhd::NFIELD)
        return 1;
    const mhd::BlockView b = host_view(ni, nj, nk, G, fields);
    unsigned long long kmin[mhd::DIAG_NMIN], kmax[mhd::DIAG_NQ];
    for (int q = 0; q < mhd::DIAG_NQ; ++q)
    {
        if (q < mhd::DIAG_NMIN)
            kmin[q] = mhd::diag_key(INFINITY);
        kmax[q] = mhd::diag_key(q < mhd::DIAG_NMIN ? -INFINITY : 0.0);
    }
    for (int i = 0; i < ni; ++i)
        for (int j = 0; j < nj; ++j)
            for (int k = 0; k < nk; ++k)
            {
                double v[mhd::DIAG_NQ];
                mhd::diag_cell(b, i, j, k, v);
                for (int q = 0; q < mhd::DIAG_NQ; ++q)
                    if (v[q] == v[q])
                    {
                        const unsigned long long key = mhd::diag_key(v[q]);
                        if (q < mhd::DIAG_NMIN && key < kmin[q])
                            kmin[q] = key;
                        if (key > kmax[q])
                            kmax[q] = key;
                    }
            }
    for (int q = 0; q < mhd::DIAG_NQ; ++q)
    {
        if (q < mhd::DIAG_NMIN)
            mins[q] = mhd::diag_unkey(kmin[q]);
        maxs[q] = mhd::diag_unkey(kmax[q]);
    }
    return 0;
}

// the order-preserving keys of n doubles
extern "C" void diag_keys(const double *x, unsigned long long *k, double *back, int n)
{
    for (int t = 0; t < n; ++t)
    {
        k[t] = mhd::diag_key(x[t]);
        back[t] = mhd::diag_unkey(k[t]);
    }
}
