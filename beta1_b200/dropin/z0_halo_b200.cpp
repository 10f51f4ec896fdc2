// Z0-style halo smoke driver on the B200 (the reference's Z0_NULL/main.cpp
// exercises the inter-block ghost fill; it no longer compiles against the
// reference's current API, so this driver does the same job against the kept
// API: Param, Grid_Preprocess, build_topology, Field, Halo).
//
// Run inside a case directory holding ./CASE.  For the cell field U_H (5
// components) and the face fields B_xi / B_eta / B_zeta:
//
// 1. The device gather table is derived from the reference's own halo
//    exchange: every point is filled with block * 2^32 + AoS offset + 1
//    (exact in a double), the reference's face, edge and vertex exchanges run
//    (Halo::data_trans_1DCorner / 2DCorner / 3DCorner,
//    include/4_halo/1_MPCNS_Halo.h:24-42), and every point that now holds
//    another point's code is a copy from that point.  The composition of the
//    three exchanges is one gather: point dst[n] takes the value src[n] had
//    before the exchange.
// 2. The fields are filled with seeded random values; the reference exchanges
//    them on the host while the device runs the gather (mhd_sync); the two
//    must agree at every point, bit for bit.
//
// Prints one line per field and exits 0 when every field agrees, 1 otherwise.
#include "0_basic/MPI_WRAPPER.h"
#include "1_grid/1_MPCNS_Grid.h"
#include "2_topology/2_MPCNS_Topology.h"
#include "3_field/2_MPCNS_Field.h"
#include "4_halo/1_MPCNS_Halo.h"

#include "beta1_mhd.h"

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <string>
#include <vector>

namespace
{

void check(mhd_ctx *ctx, int rc, const char *what)
{
    if (rc == MHD_OK)
        return;
    char msg[512] = "";
    if (ctx)
        mhd_last_error(ctx, msg, int32_t(sizeof msg));
    std::fprintf(stderr, "[z0_halo_b200] %s failed (status %d): %s\n", what, rc, msg);
    std::abort();
}

std::vector<double> &storage(Field *fld, const std::string &name, int ib)
{
    return fld->field(name, ib).raw_data().GetV3();
}

// the reference's halo exchange of one field: faces, edges, vertices
void exchange(Halo *hal, std::string name)
{
    hal->data_trans_1DCorner(name);
    hal->data_trans_2DCorner(name);
    hal->data_trans_3DCorner(name);
}

} // namespace

int main(int argc, char **argv)
{
    int myid = 0;
    PARALLEL::mpi_initial(argc, argv);
    PARALLEL::mpi_rank(&myid);
    Param *par = new Param;
    par->ReadParam(myid);
    Grid *grd = new Grid;
    grd->Grid_Preprocess(par);
    TOPO::Topology topology = TOPO::build_topology(*grd, myid, par->GetInt("dimension"));
    const int ngg = par->GetInt("ngg");
    Field *fld = new Field(grd, par, ngg);
    fld->register_field({"U_H", StaggerLocation::Cell, 5, ngg});
    fld->register_field({"B_xi", StaggerLocation::FaceXi, 1, ngg});
    fld->register_field({"B_eta", StaggerLocation::FaceEt, 1, ngg});
    fld->register_field({"B_zeta", StaggerLocation::FaceZe, 1, ngg});
    Halo *hal = new Halo(fld, &topology);
    const char *names[4] = {"U_H", "B_xi", "B_eta", "B_zeta"};
    const char *groups[4] = {"Ucell", "Bface", "Bface", "Bface"};
    for (const char *n : names)
        hal->register_halo_field(n);
    hal->build_registered_patterns();

    const int nb = fld->num_blocks();
    std::vector<mhd_block_desc> blocks;
    for (int ib = 0; ib < nb; ++ib)
    {
        FieldBlock &U = fld->field(std::string("U_H"), ib);
        const Int3 lo = U.inner_lo(), hi = U.inner_hi();
        blocks.push_back({hi.i - lo.i, hi.j - lo.j, hi.k - lo.k});
    }
    // 1. gather tables from the reference's exchange of index codes
    std::vector<int64_t> dst[2], src[2];
    int32_t fidx[4];
    for (int f = 0; f < 4; ++f)
    {
        // the library's field index of the name (point ids carry it)
        fidx[f] = -1;
        for (int32_t q = 0;; ++q)
        {
            const char *nm = nullptr;
            int32_t loc, nc, ng;
            if (mhd_field_spec(q, &nm, &loc, &nc, &ng) != MHD_OK)
                break;
            if (std::string(nm) == names[f])
                fidx[f] = q;
        }
        if (fidx[f] < 0)
        {
            std::fprintf(stderr, "[z0_halo_b200] the library has no field %s\n", names[f]);
            return 2;
        }
        for (int ib = 0; ib < nb; ++ib)
        {
            std::vector<double> &v = storage(fld, names[f], ib);
            for (size_t q = 0; q < v.size(); ++q)
                v[q] = double(int64_t(ib) << 32) + double(q) + 1.0;
        }
        exchange(hal, names[f]);
        const int g = (f == 0) ? 0 : 1;
        for (int ib = 0; ib < nb; ++ib)
        {
            const std::vector<double> &v = storage(fld, names[f], ib);
            for (size_t q = 0; q < v.size(); ++q)
            {
                const double own = double(int64_t(ib) << 32) + double(q) + 1.0;
                if (v[q] == own)
                    continue;
                const int64_t code = int64_t(v[q]) - 1;
                if (double(code + 1) != v[q] || code < 0)
                {
                    std::fprintf(stderr, "[z0_halo_b200] %s block %d offset %zu: not a copy\n", names[f], ib, q);
                    return 2;
                }
                const int64_t sb = code >> 32, so = code & 0xffffffffll;
                dst[g].push_back((int64_t(fidx[f]) << 56) | (int64_t(ib) << 40) | int64_t(q));
                src[g].push_back((int64_t(fidx[f]) << 56) | (sb << 40) | so);
            }
        }
    }
    mhd_params p{};
    p.gamma = 5.0 / 3.0;
    p.cfl = 0.4;
    p.inver_MA2 = p.momentum_hall_coeff = p.state_coeff = p.M_H = p.M_ref = 1.0;
    p.dt_abort = 1e-7;
    p.ngg = ngg;
    p.precision = MHD_PREC_FP64;
    mhd_ctx *ctx = nullptr;
    check(nullptr, mhd_ctx_create(blocks.data(), nb, &p, &ctx), "mhd_ctx_create");

    for (int g = 0; g < 2; ++g)
        check(ctx, mhd_set_sync_map(ctx, g == 0 ? "Ucell" : "Bface", dst[g].data(), src[g].data(),
                                    int64_t(dst[g].size())),
              "mhd_set_sync_map");

    // 2. random fields: the reference's host exchange against the device gather
    std::mt19937_64 rng(20261203);
    std::normal_distribution<double> nd(0.0, 1.0);
    int bad_fields = 0;
    for (int f = 0; f < 4; ++f)
    {
        for (int ib = 0; ib < nb; ++ib)
        {
            std::vector<double> &v = storage(fld, names[f], ib);
            for (double &x : v)
                x = nd(rng);
            check(ctx, mhd_upload_field(ctx, names[f], ib, v.data(), int64_t(v.size())), "mhd_upload_field");
        }
    }
    check(ctx, mhd_sync(ctx, "Ucell"), "mhd_sync");
    check(ctx, mhd_sync(ctx, "Bface"), "mhd_sync");
    for (int f = 0; f < 4; ++f)
    {
        exchange(hal, names[f]);
        int64_t diff = 0, points = 0;
        for (int ib = 0; ib < nb; ++ib)
        {
            const std::vector<double> &want = storage(fld, names[f], ib);
            std::vector<double> got(want.size());
            check(ctx, mhd_download_field(ctx, names[f], ib, got.data(), int64_t(got.size())), "mhd_download_field");
            for (size_t q = 0; q < got.size(); ++q)
                diff += (std::memcmp(&got[q], &want[q], sizeof(double)) != 0);
            points += int64_t(got.size());
        }
        std::printf("%s (%s): %lld gather entries, %lld points, %lld differ\n", names[f], groups[f],
                    (long long)(f == 0 ? dst[0].size() : dst[1].size()), (long long)points, (long long)diff);
        bad_fields += diff != 0;
    }
    mhd_ctx_destroy(ctx);
    PARALLEL::mpi_finalize();
    delete hal;
    delete fld;
    delete par;
    delete grd;
    return bad_fields ? 1 : 0;
}
