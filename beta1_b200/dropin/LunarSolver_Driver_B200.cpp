// Drop-in replacement of the reference's Z4_Lunar/src/LunarSolver_Driver.cpp
// that runs every StepOnce on the B200 through the C ABI (include/beta1_mhd.h).
//
// The reference's driver (Z4_Lunar/main.cpp) and every other reference
// source stay unchanged: a build links this file in place of
// LunarSolver_Driver.cpp, plus libbeta1_mhd.so.  It defines the same three
// members of LunarSolver (Z4_Lunar/include/LunarSolver.h:62-64, 225-226):
//
// * Advance(): the reference's loop -- derived fields, output switches and
//   the step-0 output on the host, then StepOnce() until the stop switch.
// * StepOnce(): the first call sets the device up from the solver's own
//   FieldBlocks (geometry, applied field, state) and the compiled set-up file
//   (Sync tables, Pole patches, implicit resistive system; written by
//   beta1_b200.tables from the CaseSpec of the CASE directory, path in
//   BETA1_TABLES, default ./CASE/b200_tables.bin); every call is one device
//   step (mhd_step: CFL dt, fluid RHS, CT induction, Euler update, implicit
//   resistive solve, closing syncs and derived fields), then the run data
//   and switches as the reference records them.
// * UpdateControlAndOutput(): at output steps the state and derived fields
//   are first read back into the FieldBlocks, then the reference's own
//   diagnostics and writers run on them (the same calls, in the same order,
//   as Z4_Lunar/src/LunarSolver_Driver.cpp:94-128).
//
// Errors follow the reference's convention: a message on stderr, then abort.
// The implicit Hall solve (HALL_IMPLICIT 1) is not routed through the device
// by this driver.  The explicit resistive sub-cycles are: their edge profile
// is formed here from the solver's own node coordinates.
#include "LunarSolver.h"

#include "beta1_mhd.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <string>
#include <vector>

namespace
{

void die(mhd_ctx *ctx, int rc, const char *what)
{
    char msg[512] = "";
    if (ctx)
        mhd_last_error(ctx, msg, int32_t(sizeof msg));
    std::fprintf(stderr, "[beta1_mhd] %s failed (status %d): %s\n", what, rc, msg);
    std::abort();
}

void check(mhd_ctx *ctx, int rc, const char *what)
{
    if (rc != MHD_OK)
        die(ctx, rc, what);
}

// ---- the compiled set-up file (format: beta1_b200/tables.py) ----
struct Group
{
    std::string name;
    std::vector<int64_t> dst, src, dst2, src2, cdst;
    std::vector<double> cval;
    std::vector<int32_t> walls; // block, direction pairs
};

struct Resistive
{
    std::vector<int64_t> unknowns, alias, owner;
    std::vector<double> eta, sign;
    double rtol = 0.0, atol = 0.0;
    int32_t maxit = 0, restart = 30;
};

struct Tables
{
    std::vector<Group> groups;
    std::vector<int32_t> poles; // block, direction pairs
    bool has_res = false;
    Resistive res;
};

class Reader
{
  public:
    explicit Reader(const std::string &path) : in_(path, std::ios::binary)
    {
        if (!in_)
        {
            std::fprintf(stderr, "[beta1_mhd] cannot open the set-up file %s\n", path.c_str());
            std::abort();
        }
    }
    template <class T> T get()
    {
        T v{};
        in_.read(reinterpret_cast<char *>(&v), sizeof v);
        if (!in_)
            bad();
        return v;
    }
    template <class T> std::vector<T> values(int64_t n)
    {
        if (n < 0)
            bad();
        std::vector<T> v(static_cast<size_t>(n));
        if (n > 0)
            in_.read(reinterpret_cast<char *>(v.data()), std::streamsize(n * int64_t(sizeof(T))));
        if (!in_)
            bad();
        return v;
    }
    template <class T> std::vector<T> counted() { return values<T>(get<int64_t>()); }
    std::string text(int32_t n)
    {
        std::string s(static_cast<size_t>(n), 0);
        in_.read(&s[0], n);
        if (!in_)
            bad();
        return s;
    }

  private:
    [[noreturn]] void bad()
    {
        std::fprintf(stderr, "[beta1_mhd] the set-up file is truncated or malformed\n");
        std::abort();
    }
    std::ifstream in_;
};

Tables read_tables(const std::string &path)
{
    Reader r(path);
    Tables t;
    if (r.text(4) != "B1TB" || r.get<int32_t>() != 1)
    {
        std::fprintf(stderr, "[beta1_mhd] %s is not a version-1 set-up file\n", path.c_str());
        std::abort();
    }
    const int32_t ng = r.get<int32_t>();
    for (int32_t g = 0; g < ng; ++g)
    {
        Group grp;
        grp.name = r.text(r.get<int32_t>());
        grp.dst = r.counted<int64_t>();
        grp.src = r.counted<int64_t>();
        grp.dst2 = r.counted<int64_t>();
        grp.src2 = r.counted<int64_t>();
        grp.cdst = r.counted<int64_t>();
        grp.cval = r.values<double>(int64_t(grp.cdst.size()));
        const int32_t nw = r.get<int32_t>();
        grp.walls = r.values<int32_t>(2 * int64_t(nw));
        t.groups.push_back(std::move(grp));
    }
    t.poles = r.values<int32_t>(2 * int64_t(r.get<int32_t>()));
    t.has_res = r.get<int32_t>() != 0;
    if (t.has_res)
    {
        t.res.unknowns = r.counted<int64_t>();
        t.res.eta = r.values<double>(int64_t(t.res.unknowns.size()));
        t.res.alias = r.counted<int64_t>();
        t.res.owner = r.values<int64_t>(int64_t(t.res.alias.size()));
        t.res.sign = r.values<double>(int64_t(t.res.alias.size()));
        t.res.rtol = r.get<double>();
        t.res.atol = r.get<double>();
        t.res.maxit = r.get<int32_t>();
        t.res.restart = r.get<int32_t>();
    }
    return t;
}

// ---- one device context per solver ----
struct Device
{
    mhd_ctx *ctx = nullptr;
};

std::map<const LunarSolver *, Device> &devices()
{
    // left to process teardown: the CUDA runtime may be gone by the time
    // static objects are destroyed
    static auto *m = new std::map<const LunarSolver *, Device>;
    return *m;
}

Device *device_of(const LunarSolver *s)
{
    auto it = devices().find(s);
    return (it != devices().end() && it->second.ctx) ? &it->second : nullptr;
}

// FieldBlock storage is the ABI's host layout: the field's logical box in
// (i, j, k, m) order, component fastest
void upload(mhd_ctx *ctx, FieldBlock &fb, const char *name, int ib)
{
    std::vector<double> &v = fb.raw_data().GetV3();
    check(ctx, mhd_upload_field(ctx, name, ib, v.data(), int64_t(v.size())), name);
}

void download(mhd_ctx *ctx, FieldBlock &fb, const char *name, int ib)
{
    std::vector<double> &v = fb.raw_data().GetV3();
    check(ctx, mhd_download_field(ctx, name, ib, v.data(), int64_t(v.size())), name);
}

// geometry and applied-field arrays the device reads, as the reference built them
const char *const kGeometry[] = {"Jac",      "JDxi",     "JDet",      "JDze",      "beta_xi",   "beta_eta",
                                 "beta_zeta", "alpha_xi", "alpha_eta", "alpha_zeta", "dr_xi",     "dr_eta",
                                 "dr_zeta",  "Area_xi",  "Area_eta",  "Area_zeta", "dl_xi",     "dl_eta",
                                 "dl_zeta",  "Astar_xi", "Astar_eta", "Astar_zeta", "Bcell_from_Bface_w",
                                 "Jcell_from_Jedge_w", "Badd_xi", "Badd_eta", "Badd_zeta"};
const char *const kState[] = {"U_H", "B_xi", "B_eta", "B_zeta"};

// The resistivity profile of LunarSolver::AddResistiveEdgeEMF_To_
// (Z4_Lunar/src/physics/LunarSolver_MagExplicit_Resis.cpp:72-88, 160-167) at
// every inner edge of a block: yita0 of the radius of the edge's midpoint,
// as the eta_edge_xi / eta_edge_eta / eta_edge_zeta fields the device's
// resistive edge EMF reads (no ghost layers; edge box n + 1 across the edge).
void upload_resistive_profile(mhd_ctx *ctx, Block &blk, int ib, int ni, int nj, int nk)
{
    const char *const names[3] = {"eta_edge_xi", "eta_edge_eta", "eta_edge_zeta"};
    for (int ea = 0; ea < 3; ++ea)
    {
        const int di = ea == 0, dj = ea == 1, dk = ea == 2;
        const int n0 = ni + (ea != 0), n1 = nj + (ea != 1), n2 = nk + (ea != 2);
        std::vector<double> y(size_t(n0) * size_t(n1) * size_t(n2), 0.0);
        for (int i = 0; i < n0; ++i)
            for (int j = 0; j < n1; ++j)
                for (int k = 0; k < n2; ++k)
                {
                    const double xm = 0.5 * (blk.x(i, j, k) + blk.x(i + di, j + dj, k + dk));
                    const double ym = 0.5 * (blk.y(i, j, k) + blk.y(i + di, j + dj, k + dk));
                    const double zm = 0.5 * (blk.z(i, j, k) + blk.z(i + di, j + dj, k + dk));
                    const double r = std::sqrt(xm * xm + ym * ym + zm * zm);
                    double v = 0.0;
                    if (!(r <= 0.84 || r >= 1.04))
                        v = 0.5 * (std::tanh((r - 0.84) / 0.02) - std::tanh((r - 1.04) / 0.02));
                    y[(size_t(i) * size_t(n1) + size_t(j)) * size_t(n2) + size_t(k)] = v;
                }
        check(ctx, mhd_upload_field(ctx, names[ea], ib, y.data(), int64_t(y.size())), names[ea]);
    }
}
// what the reference's diagnostics and writers read at output steps
const char *const kOutput[] = {"U_H",   "B_xi",   "B_eta",  "B_zeta",    "PV_H",    "U_plus",
                               "B_cell", "Bind_cell", "J_xi", "J_eta",   "J_zeta",  "J_cell",
                               "E_xi",  "E_eta",  "E_zeta", "Eres_xi", "Eres_eta", "Eres_zeta"};

} // namespace

void LunarSolver::Advance()
{
    // the reference's own loop (Z4_Lunar/src/LunarSolver_Driver.cpp:6-19)
    UpdateDerivedFields_();
    control_.UpdateSwitches(*run_data_);
    UpdateControlAndOutput();
    while (!control_.if_stop)
        StepOnce();
}

bool LunarSolver::StepOnce()
{
    Device &d = devices()[this];
    if (!d.ctx)
    {
        const int nb = fld_->num_blocks();
        std::vector<mhd_block_desc> blocks;
        for (int ib = 0; ib < nb; ++ib)
        {
            const FieldBlock &U = fld_->field(fid_.fid_U_H, ib);
            const Int3 lo = U.inner_lo(), hi = U.inner_hi();
            blocks.push_back({hi.i - lo.i, hi.j - lo.j, hi.k - lo.k});
        }
        mhd_params p{};
        p.gamma = gamma_;
        p.cfl = CFL;
        p.inver_MA2 = inver_MA2;
        p.momentum_hall_coeff = momentum_hall_coeff;
        p.state_coeff = state_coeff_H;
        p.M_H = M_H;
        p.M_ref = M_ref;
        p.ne_hall_floor = ne_hall_floor;
        p.dt_abort = 1e-7; // the abort threshold of Compute_Timestep
        p.ngg = par_->GetInt("ngg");
        p.precision = MHD_PREC_FP64;
        check(nullptr, mhd_ctx_create(blocks.data(), nb, &p, &d.ctx), "mhd_ctx_create");
        for (int ib = 0; ib < nb; ++ib)
        {
            for (const char *name : kGeometry)
                if (fld_->has_field(name))
                    upload(d.ctx, fld_->field(std::string(name), ib), name, ib);
            for (const char *name : kState)
                upload(d.ctx, fld_->field(std::string(name), ib), name, ib);
        }
        const char *env = std::getenv("BETA1_TABLES");
        const Tables t = read_tables(env ? env : "./CASE/b200_tables.bin");
        for (const Group &g : t.groups)
        {
            check(d.ctx, mhd_set_sync_map(d.ctx, g.name.c_str(), g.dst.data(), g.src.data(), int64_t(g.dst.size())),
                  "mhd_set_sync_map");
            if (!g.dst2.empty())
                check(d.ctx, mhd_set_sync_map_post(d.ctx, g.name.c_str(), g.dst2.data(), g.src2.data(),
                                                   int64_t(g.dst2.size())),
                      "mhd_set_sync_map_post");
            if (!g.cdst.empty())
                check(d.ctx, mhd_set_sync_consts(d.ctx, g.name.c_str(), g.cdst.data(), g.cval.data(),
                                                 int64_t(g.cdst.size())),
                      "mhd_set_sync_consts");
            for (size_t w = 0; w + 1 < g.walls.size(); w += 2)
                check(d.ctx, mhd_set_sync_wall(d.ctx, g.name.c_str(), g.walls[w], g.walls[w + 1]),
                      "mhd_set_sync_wall");
        }
        for (size_t q = 0; q + 1 < t.poles.size(); q += 2)
            check(d.ctx, mhd_set_pole(d.ctx, t.poles[q], t.poles[q + 1]), "mhd_set_pole");
        if (resist_control.is_Lunar_resistance && resist_control.use_implicit_lunar_resistance)
        {
            if (!t.has_res)
            {
                std::fprintf(stderr, "[beta1_mhd] the set-up file holds no implicit resistive system\n");
                std::abort();
            }
            const Resistive &r = t.res;
            check(d.ctx, mhd_set_resistive(d.ctx, int64_t(r.unknowns.size()), r.unknowns.data(), r.eta.data(),
                                           int64_t(r.alias.size()), r.alias.data(), r.owner.data(), r.sign.data(),
                                           r.rtol, r.atol, r.maxit, r.restart),
                  "mhd_set_resistive");
        }
        else if (resist_control.is_Lunar_resistance)
        {
            // ResistiveDiffusionSubcycles_ (Z4_Lunar/src/physics/LunarSolver_MagneticRHS.cpp:53-115)
            for (int ib = 0; ib < nb; ++ib)
                upload_resistive_profile(d.ctx, fld_->grd->grids(ib), ib, blocks[size_t(ib)].ni,
                                         blocks[size_t(ib)].nj, blocks[size_t(ib)].nk);
            check(d.ctx, mhd_set_resistive_explicit(d.ctx, inver_Rem, std::max(1, resist_control.n_subcycles)),
                  "mhd_set_resistive_explicit");
        }
        check(d.ctx, mhd_set_time(d.ctx, run_data_->dt, run_data_->time, run_data_->step), "mhd_set_time");
        // the host state's derived fields were computed by Advance(); the
        // device computes its own from the same state
        check(d.ctx, mhd_update_derived(d.ctx), "mhd_update_derived");
    }
    double t = 0.0;
    check(d.ctx, mhd_step(d.ctx, 1, &dt, &t), "mhd_step");
    // Record and update the run data, as StepOnce does
    run_data_->dt = dt;
    run_data_->time += dt;
    run_data_->step += 1;
    control_.UpdateSwitches(*run_data_);
    return UpdateControlAndOutput();
}

bool LunarSolver::UpdateControlAndOutput()
{
    RunData &run = io_.Run();
    if (Device *d = device_of(this))
        if (control_.if_outres || control_.if_outfile)
            for (int ib = 0; ib < fld_->num_blocks(); ++ib)
                for (const char *name : kOutput)
                    if (fld_->has_field(name))
                        download(d->ctx, fld_->field(std::string(name), ib), name, ib);

    // the reference's diagnostics and writers, in its order
    if (control_.if_outres)
    {
        calc_divB();
        runtime_data_->UpdateOnOutres(run);
        runtime_data_->PrintLineMinimal(run);
        PrintMinMaxDiagnostics_();
    }
    if (control_.if_outfile)
    {
        io_.BackupDataDirectory("./DATA_backup");
        io_.WriteTecplotBinFile(run.step, run.time);
        io_.WriteRestartBinFile(run.step, run.time);
        io_.WriteRunDataFile();
        io_.MaybeArchiveDataDirectory(run.step, run.time);
    }
    return control_.if_stop;
}
