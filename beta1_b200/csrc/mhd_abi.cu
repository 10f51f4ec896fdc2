// C-ABI of the B200 MHD hot path (see include/beta1_mhd.h): context and
// field pool management, host<->device transfers, compiled boundary syncs,
// and the per-step launch sequence replayed as a CUDA graph.
#include "mhd_device_scope.h"
#include "mhd_kernels.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <unordered_set>
#include <vector>

using namespace mhd;

// Staging array of the allocation-free read-out (mhd_download_field_noalloc):
// every device that loads the library holds it until the process exits.  Its
// name is a host-side stand-in in host code; the device address is looked up
// with cudaGetSymbolAddress when a context is created on that device.
static __device__ __align__(256) double g_noalloc_staging[MHD_NOALLOC_MAX_DOUBLES];

namespace
{

struct CudaDeviceApi
{
    static int get(int *d) { return cudaGetDevice(d) == cudaSuccess ? 0 : 1; }
    static int set(int d) { return cudaSetDevice(d) == cudaSuccess ? 0 : 1; }
};

// makes the context's device current for the rest of the entry point and
// restores the caller's device on return
#define BIND_DEVICE(ctx)                                                                        \
    DeviceScope<CudaDeviceApi> dev_scope_((ctx) ? (ctx)->device : -1);                          \
    if (!dev_scope_.ok())                                                                       \
        return MHD_ECUDA

struct FieldSpec
{
    const char *name;
    int loc;
    int ncomp;
    int nghost;
};

const FieldSpec kFields[NFIELD] = {
#define MHD_SPEC(id, name, loc, nc, ng) {name, loc, nc, ng},
    MHD_FIELD_LIST(MHD_SPEC)
#undef MHD_SPEC
};

int field_by_name(const char *name)
{
    if (!name)
        return -1;
    for (int f = 0; f < NFIELD; ++f)
        if (std::strcmp(kFields[f].name, name) == 0)
            return f;
    return -1;
}

// Device lists of one sync: fixed values (phase A) and composed copies (phase B).
struct CopyList
{
    uint64_t *cdst = nullptr;
    double *cval = nullptr;
    int64_t nconst = 0;
    uint64_t *dst = nullptr;
    uint64_t *src = nullptr;
    double *tmp = nullptr; // non-null when a source is also a destination
    int64_t n = 0;
    // the same copies with 32-bit offsets, when the pool has fewer than 2^32
    // points and no copy is staged (a quarter less traffic per copy)
    uint32_t *dst32 = nullptr, *src32 = nullptr;
};

// One sync group.  The full tables are what the reference's Sync writes.
// The hot lists keep only the points a later kernel of the step reads (the
// ghost layers within each field's stencil depth, and inner points); the
// rest is written by the full lists when a field is read out (materialised),
// which gives the same values because a composed copy's source does not
// change between the sync and the read-out.
struct SyncMap
{
    std::vector<uint64_t> hd, hs, hcd; // full tables (pool offsets) on the host
    std::vector<double> hcv;
    std::vector<std::pair<int, int>> walls; // (block, direction) of Solid_Surface fluid handlers
    // Pole contexts: composed copies whose sources the wall handlers write
    // (run after them)
    std::vector<uint64_t> hd2, hs2;
    bool staged = false;
    bool built = false; // device lists match the host tables
    CopyList full, hot, post;
    // Pole contexts: the copies and fixed values a step leaves for read-out
    // (cold), written then without the rings, walls and post-wall copies
    CopyList cold;
    int *dwalls = nullptr;  // walls on the device (block, direction pairs)
    int64_t wall_cols = 0;  // boundary cell columns of the largest wall
};

constexpr int kThreads = 256;

const char *const kKernelNames[] = {
    "k_fluid_rhs",    "k_eface",       "k_eedge",        "k_curl_e2f",     "k_update_u",      "k_bcell",
    "k_jedge",        "k_jcell",       "k_pv_uplus_dt",  "k_begin_step",   "k_arm_dt",        "k_end_step",
    "k_gather",       "k_gather_stage", "k_scatter_stage", "k_aos_to_soa", "k_soa_to_aos",    "k_set_consts",
    "k_wall_u",       "k_alias_copy",  "k_scatter_vec",  "k_resist_out",   "k_resist_rhs",    "k_dots",
    "k_sub_proj",    "k_add_small",    "k_div_guard",    "k_div_next",      "k_gmres_init",
    "k_cycle_start",  "k_gmres_column", "k_inner_check", "k_gmres_solve_y", "k_add_basis",    "k_outer_check",
    "k_zero",         "k_residual",    "k_ucontra",      "k_face_normals", "k_divb",          "k_eres_explicit",
    "k_bcell_jedge",  "k_fluid_ucontra", "k_wall_u_all",   "k_hall_cell",    "k_hall_edge",
    "k_pack_vec",     "k_geom32",       "k_fluid_mixed",  "k_gmres_resist", "k_pole",
    "k_geometry",     "k_diag_init",   "k_diag",        "k_rk2",          "k_hall_begin",    "k_hall_step_begin",
    "k_hall_gmres_init", "k_hall_cycle_prep", "k_hall_ls_begin", "k_hall_ls_check", "k_hall_accept", "k_hall_column",
    "k_hall_trial",   "k_hall_jv_dots", "k_hall_proj_dots", "k_hall_next",  "k_hall_res_dots", "k_hall_restart_r",
    "k_hall_gmres_prologue", "k_norm2", "k_hall_take",    "k_copy_segments"};
constexpr int kNumKernelNames = int(sizeof(kKernelNames) / sizeof(kKernelNames[0]));

} // namespace

// kernels compiled in register / occupancy variants (mhd_kernels.cuh)
enum TuneId
{
    TUNE_k_pv_uplus_dt,
    TUNE_k_fluid_ucontra,
    TUNE_k_bcell_jedge,
    TUNE_k_eface,
    TUNE_k_curl_e2f,
    TUNE_k_eedge,
    TUNE_k_fluid_mixed,
    TUNE_k_gmres_resist,
    TUNE_k_hall_edge,
    NTUNE
};
const char *const kTuneNames[NTUNE] = {"k_pv_uplus_dt", "k_fluid_ucontra", "k_bcell_jedge",  "k_eface",
                                       "k_curl_e2f",    "k_eedge",         "k_fluid_mixed",  "k_gmres_resist",
                                       "k_hall_edge"};
// minimum CTAs per SM of each variant (variant 0 first; 0: the compiler's
// own allocation, no launch bounds) and the number of variants
// per variant the reported value: the minimum CTAs per SM of its launch
// bounds (0: none); 12 for the face-tiled k_fluid_mixed (2 CTAs per SM), 16
// for the same with its face states staged in shared memory, 14
// for k_pv_uplus_dt with J_cell in a pass of its own (the PV pass at 4); for
// the persistent k_gmres_resist the CTAs of its grid (0: two per SM); for
// k_hall_edge 2 selects the form that reads the seven cells of a staggered
// point once
const int kTuneMinCtas[NTUNE][5] = {{4, 0, 5, 14, 0}, {0, 3, 0, 0, 0},        {0, 6, 0, 0, 0},
                                    {0, 6, 0, 0, 0},  {0, 6, 0, 0, 0},        {0, 8, 0, 0, 0},
                                    {3, 0, 2, 12, 16}, {0, 148, 64, 32, 0},   {0, 2, 0, 0, 0}};
const int kTuneCount[NTUNE] = {4, 2, 2, 2, 2, 2, 5, 4, 2};
constexpr int kPvSplit = 3; // variant index of k_pv_uplus_dt's split form

// loop bodies of the device-steered implicit Hall solve
enum
{
    HALL_KB_NEWTON,
    HALL_KB_CYCLE,
    HALL_KB_INNER,
    HALL_KB_RESTART,
    HALL_KB_LS,
    HALL_KB_N
};

struct mhd_ctx
{
    int device = -1;               // CUDA device the context lives on
    double *noalloc = nullptr;     // device address of g_noalloc_staging on it
    int nblocks = 0;
    mhd_params prm{};
    Consts c{};
    int G = 4;
    std::vector<BlockView> hbv;
    BlockView *dbv = nullptr;
    double *pool = nullptr;
    size_t pool_n = 0;
    float *pool32 = nullptr; // FP32 planes of the mixed-precision form
    std::vector<std::vector<size_t>> base; // [field][block] offset in pool
    cudaStream_t stream = nullptr;
    cudaGraph_t graph = nullptr, graph_a = nullptr, graph_c = nullptr;
    cudaGraphExec_t gexec = nullptr, gexec_a = nullptr, gexec_c = nullptr;
    int64_t graph_kernels = 0, graph_kernels_a = 0, graph_kernels_c = 0;
    // independent runs (a batch): per run its dt reduction key, dt, time and
    // step count, and the reference state of the mixed-precision flux
    int nruns = 1;
    unsigned long long *dt_key = nullptr;
    double *dt = nullptr;
    double *time = nullptr;
    long long *step = nullptr;
    int *err = nullptr;
    double *qref = nullptr; // [nruns][6]
    // flattened launches (batches): block of every CTA per launch kind
    bool flat = false;
    int *cta_tab = nullptr;
    int64_t cta_total[NKIND] = {};
    std::map<std::string, SyncMap> syncs;
    // eta Poles: (block, direction) pairs; a context with Poles runs every
    // sync in the topology order of the Pole shell
    std::vector<int> poles;
    int *dpoles = nullptr;
    double *pole_cache = nullptr; // normal matrices of the Pole rings' least squares
    int pole_stride = 0;          // rings per Pole and operation in pole_cache
    unsigned long long *diag_keys = nullptr; // output-step minima / maxima (mhd_diagnostics)
    // materialisation state: groups whose last sync ran its hot list only,
    // and PV / U_plus computed on the first ghost layer only
    std::map<std::string, bool> dirty;
    bool pv_dirty = false;
    bool geom_dirty = true; // face areas / normals to recompute from JD
    std::vector<std::string> field_group = std::vector<std::string>(NFIELD); // group that syncs a field
    double *staging = nullptr;
    size_t staging_n = 0;
    int64_t launches = 0;
    int64_t max_cells = 0;
    bool capturing = false;
    std::string msg;
    // implicit resistive solve (LunarSolver::SolveImplicitResistiveDiffusion_)
    struct Resistive
    {
        bool on = false;
        int64_t n = 0;                 // unknowns (owner edges with eta > 0)
        uint64_t *e = nullptr;         // pool offsets of the unknowns in Eres_*
        uint64_t *dj = nullptr;        // ... in dJ_*
        uint64_t *j = nullptr;         // ... in J_*
        double *eta = nullptr;
        int64_t nalias = 0;            // aliases of unknown owners (sync_edge_1form)
        uint64_t *alias_e = nullptr, *owner_e = nullptr;
        double *sign = nullptr;
        // the operator's active region: copies with a destination inside it,
        // and per (block, axis) sub-ranges of the inner faces / edges
        CopyList eres1form, db;
        int *rng = nullptr;      // per block: region box lo[3], hi[3] within [0, n + 1)^3
        int64_t nreg_max = 0;    // points of the largest region box
        double rtol = 1e-8, atol = 1e-12;
        int maxit = 200, restart = 30;
        // workspace
        double *V = nullptr, *w = nullptr, *x = nullptr, *b = nullptr, *r = nullptr;
        double *partial = nullptr, *dots = nullptr;
        GmresState *st = nullptr;
        int ngroups = 1;
        // launch accounting of the graph-resident loops
        int64_t k_cycle = 0, k_inner = 0;        // kernels per restart cycle / per Arnoldi step
        long long its_eager = 0, cycles_eager = 0;
        bool graph_loops = true;                 // conditional graph nodes usable
        std::vector<uint64_t> seed;              // unknown and alias offsets (Eres), for the region
        // the persistent solve (one cooperative kernel per solve)
        int64_t *alias_of = nullptr;             // unknown index of each alias's owner
        int *uloc = nullptr;                     // per unknown: block, edge axis, i, j, k
        int merge1 = 0, merge2 = 0;              // fixed values written in the phase before
        double *ppartial = nullptr;              // per-CTA partial dot products, double-buffered
        unsigned *bar = nullptr;                 // grid barrier: arrival count, generation
        int pgrid = 0;                           // CTAs of the persistent kernel (0: unavailable)
        // fused operator phases of the persistent solve (n < 0: the copy-list phases)
        struct Fused
        {
            uint64_t *dst = nullptr;
            int *kind = nullptr;
            int64_t *idx = nullptr;
            double *val = nullptr;
            int *blk = nullptr;
            int64_t n = -1;
        } fa, fb;
    } res;
    // implicit Hall solve (ImplicitHallSolver::SolveOneStep): Newton on
    // F(X) = X - Ehall(B* - theta dt curl X) over the inner Hall edges of
    // every block, GMRES on finite-difference Jacobian-vector products
    struct HallImplicit
    {
        bool on = false;
        int64_t n = 0;
        uint64_t *e = nullptr;                     // pool offsets of the unknowns (owner Hall edges)
        int64_t nalias = 0;                        // alias <- sign * owner (edge 1-form sync)
        uint64_t *alias = nullptr, *owner = nullptr;
        double *sign = nullptr;
        double rtol = 1e-8, atol = 1e-50;          // Newton stopping test (PETSc SNES defaults)
        int maxit = 50;
        double ksp_rtol = 1e-5;                    // linear solves (PETSc KSP default)
        int ksp_maxit = 10000, restart = 30;
        double *bstar = nullptr;                   // snapshot of the face B arrays (one range per block)
        int64_t *seg_snap = nullptr, *seg_restore = nullptr; // per block: dst offset, src offset, length
        int copy_ctas = 1;
        const double **bs = nullptr;               // per block: the snapshot's B_xi, B_eta, B_zeta
        // trials read B* from the snapshot instead of restoring it: exact when
        // Sync("Bface") writes every destination from points no trial writes
        // (no staged copies, no wall handler), so the points neither the curl
        // nor the sync writes keep B*
        bool from_snapshot = false;
        double *X = nullptr, *F = nullptr, *Xt = nullptr, *Ft = nullptr, *dx = nullptr, *b = nullptr, *r = nullptr;
        double *V = nullptr, *w = nullptr, *partial = nullptr, *dots = nullptr;
        unsigned *done = nullptr;                  // CTAs finished in a reduction pass
        GmresState *st = nullptr;
        HallCtl *ctl = nullptr;                    // Newton / line-search control and statistics
        int ngroups = 1;
        // launch accounting: kernels per pass of each loop body (captured),
        // passes run eagerly
        int64_t kb[HALL_KB_N] = {0, 0, 0, 0, 0};
        int64_t kb_nested = 0;                     // kernels of one captured Newton pass, nested bodies included
        long long eager[HALL_KB_N] = {0, 0, 0, 0, 0};
    } hall;
    // Hall edge EMF: coefficient and zero boxes (block, axis, lo[3], hi[3])
    double hall_coef = 0.0;
    int *hall_zb = nullptr;
    int hall_nzb = 0;
    // time integrator (MHD_INTEGRATOR_*) and the SSP-RK2 start-of-step state
    int integrator = MHD_INTEGRATOR_EULER;
    double *rk = nullptr;
    // explicit resistive sub-cycles (ResistiveDiffusionSubcycles_): 0 = off
    int res_nsub = 0;
    double res_inver_Rem = 0.0;
    cudaStream_t spare[4] = {nullptr, nullptr, nullptr, nullptr}; // capture streams of conditional bodies
    int spare_depth = 0;

    // register / occupancy variant of each tunable kernel (mhd_autotune)
    int tune[NTUNE] = {0, 0, 0, 0, 0, 0, 0, 0, 0};

    // eager profiling: one event pair per launch
    bool profiling = false;
    std::vector<const char *> prof_names;
    std::vector<cudaEvent_t> prof_ev;
};

static void free_resistive(mhd_ctx *ctx);
static int resistive_region(mhd_ctx *ctx, const std::vector<uint64_t> &seed);
static void free_list(CopyList &m);
static int build_all_syncs(mhd_ctx *ctx);
static int materialise_field(mhd_ctx *ctx, int f);
static int materialise_group(mhd_ctx *ctx, const std::string &group);
static int materialise_all(mhd_ctx *ctx);
static void mark_dirty(mhd_ctx *ctx);
int build_sync(mhd_ctx *ctx, const std::string &group, SyncMap &m);

namespace
{

int fail(mhd_ctx *ctx, int code, const char *fmt, ...)
{
    if (ctx)
    {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        std::vsnprintf(buf, sizeof(buf), fmt, ap);
        va_end(ap);
        ctx->msg = buf;
    }
    return code;
}

#define CK(ctx, call)                                                                           \
    do                                                                                          \
    {                                                                                           \
        cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess)                                                                  \
            return fail(ctx, MHD_ECUDA, "%s failed: %s", #call, cudaGetErrorString(e_));        \
    } while (0)

void field_box(const mhd_ctx *ctx, int f, int b, int lo[3], int hi[3])
{
    const BlockView &v = ctx->hbv[b];
    int pi, pj, pk;
    loc_plus(kFields[f].loc, pi, pj, pk);
    const int g = kFields[f].nghost;
    lo[0] = lo[1] = lo[2] = -g;
    hi[0] = v.ni + pi + g;
    hi[1] = v.nj + pj + g;
    hi[2] = v.nk + pk + g;
}

int64_t field_count(const mhd_ctx *ctx, int f, int b)
{
    int lo[3], hi[3];
    field_box(ctx, f, b, lo, hi);
    return int64_t(hi[0] - lo[0]) * (hi[1] - lo[1]) * (hi[2] - lo[2]) * kFields[f].ncomp;
}

unsigned grid_for(int64_t n) { return unsigned((n + kThreads - 1) / kThreads); }

// number of points of a location box (max over blocks), g = widening
int64_t max_box(const mhd_ctx *ctx, int loc, int g)
{
    int64_t m = 0;
    for (const auto &v : ctx->hbv)
    {
        int pi, pj, pk;
        loc_plus(loc, pi, pj, pk);
        const int64_t n = int64_t(v.ni + pi + 2 * g) * (v.nj + pj + 2 * g) * (v.nk + pk + 2 * g);
        m = n > m ? n : m;
    }
    return m;
}

// staggered points [0, n + 1)^3 of the largest block
int64_t max_stagger(const mhd_ctx *ctx)
{
    int64_t m = 0;
    for (const auto &v : ctx->hbv)
        m = std::max(m, int64_t(v.ni + 1) * (v.nj + 1) * (v.nk + 1));
    return m;
}

// points of a block in a launch kind's box
int64_t kind_points(const BlockView &v, int kind)
{
    if (kind == KIND_CELL0)
        return int64_t(v.ni) * v.nj * v.nk;
    if (kind == KIND_CELL1)
        return int64_t(v.ni + 2) * (v.nj + 2) * (v.nk + 2);
    if (kind == KIND_TILE1) // one CTA of kThreads per tile
        return int64_t((v.ni + 2 + TILE_I - 1) / TILE_I) * ((v.nj + 2 + TILE_J - 1) / TILE_J) *
               ((v.nk + 2 + TILE_K - 1) / TILE_K) * kThreads;
    return int64_t(v.ni + 1) * (v.nj + 1) * (v.nk + 1);
}

// grid of a hot-path launch: one row of exactly the CTAs every block needs
// (batches of uneven blocks), else one row per block sized for the largest
dim3 grid_kind(const mhd_ctx *ctx, int kind)
{
    if (ctx->flat)
        return dim3(unsigned(ctx->cta_total[kind]), 1);
    int64_t m = 0;
    for (const auto &v : ctx->hbv)
        m = std::max(m, kind_points(v, kind));
    return dim3(unsigned(grid_for(m)), unsigned(ctx->nblocks));
}

int ensure_staging(mhd_ctx *ctx, size_t n)
{
    if (ctx->staging_n >= n)
        return MHD_OK;
    if (ctx->staging)
        cudaFree(ctx->staging);
    ctx->staging = nullptr;
    ctx->staging_n = 0;
    CK(ctx, cudaMalloc(&ctx->staging, n * sizeof(double)));
    ctx->staging_n = n;
    return MHD_OK;
}

#define RUN(x)                 \
    do                         \
    {                          \
        int rc_ = (x);         \
        if (rc_ != MHD_OK)     \
            return rc_;        \
    } while (0)

// ---- launch helpers (all on ctx->stream) ----
// Eager profiling: prof_begin() records an event before a launch, launched()
// one after it, so each kernel's duration is measured on the launching stream.
void prof_begin(mhd_ctx *ctx, const char *name)
{
    if (!ctx->profiling)
        return;
    cudaEvent_t e;
    cudaEventCreate(&e);
    cudaEventRecord(e, ctx->stream);
    ctx->prof_ev.push_back(e);
    ctx->prof_names.push_back(name);
}

int launched(mhd_ctx *ctx, int nk = 1)
{
    if (ctx->profiling)
    {
        cudaEvent_t e;
        cudaEventCreate(&e);
        cudaEventRecord(e, ctx->stream);
        ctx->prof_ev.push_back(e);
    }
    ctx->launches += nk;
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return fail(ctx, MHD_ECUDA, "kernel launch failed: %s", cudaGetErrorString(e));
    return MHD_OK;
}

// phase B of a sync: the composed copies
int gather_map(mhd_ctx *ctx, const CopyList &s)
{
    if (s.n == 0)
        return MHD_OK;
    if (s.tmp)
    {
        prof_begin(ctx, "k_gather_stage");
        k_gather_stage<<<grid_for(s.n), kThreads, 0, ctx->stream>>>(s.tmp, ctx->pool, s.src, s.n);
        RUN(launched(ctx));
        prof_begin(ctx, "k_scatter_stage");
        k_scatter_stage<<<grid_for(s.n), kThreads, 0, ctx->stream>>>(ctx->pool, s.tmp, s.dst, s.n);
        return launched(ctx);
    }
    prof_begin(ctx, "k_gather");
    if (s.dst32)
        k_gather32<<<grid_for(s.n), kThreads, 0, ctx->stream>>>(ctx->pool, s.dst32, s.src32, s.n);
    else
        k_gather<<<grid_for(s.n), kThreads, 0, ctx->stream>>>(ctx->pool, s.dst, s.src, s.n);
    return launched(ctx);
}

// fixed values then copies of a list (no wall handlers)
int apply_list(mhd_ctx *ctx, const CopyList &l)
{
    if (l.nconst > 0)
    {
        prof_begin(ctx, "k_set_consts");
        k_set_consts<<<grid_for(l.nconst), kThreads, 0, ctx->stream>>>(ctx->pool, l.cdst, l.cval, l.nconst);
        RUN(launched(ctx));
    }
    return gather_map(ctx, l);
}

// one Pole operation on every Pole of the context
int launch_pole(mhd_ctx *ctx, int op)
{
    const int np = int(ctx->poles.size() / 2);
    if (np == 0)
        return MHD_OK;
    int64_t w = 0;
    for (int q = 0; q < np; ++q)
    {
        const BlockView &v = ctx->hbv[size_t(ctx->poles[size_t(2 * q)])];
        w = std::max(w, pole_work(op, v.ni, v.nk));
    }
    prof_begin(ctx, "k_pole");
    launch_pole_op(op, w, np, ctx->stream, ctx->dbv, ctx->dpoles, ctx->pole_cache, ctx->pole_stride, 0);
    return launched(ctx);
}

// the values the Pole handlers of a group compute on the pole rings
// (Z4_Lunar/src/boundary/Boundary_Build.cpp:61-269)
int pole_rings(mhd_ctx *ctx, const std::string &group)
{
    if (group == "Ucell")
        return launch_pole(ctx, POLE_RING_U);
    if (group == "Bface")
        return launch_pole(ctx, POLE_RING_BXI);
    if (group == "B_cell")
        return launch_pole(ctx, POLE_BCELL);
    if (group == "Eedge")
    {
        RUN(launch_pole(ctx, POLE_EXI_AXIS));
        return launch_pole(ctx, POLE_EETA_REG);
    }
    if (group == "Jedge")
        return launch_pole(ctx, POLE_JETA);
    if (group == "Eres" || group == "Eres1form")
        return launch_pole(ctx, POLE_ERES_REG);
    return MHD_OK;
}

// LunarBoundary::Sync(group): phase A (fixed values, wall handlers), then
// the composed copies; the hot lists unless `full`.  In a context with
// Poles: the topology order of the Pole shell -- the Pole rings, the copies
// read before the wall handlers, the wall handlers, the copies of what they
// wrote, then the fixed values -- always with the full lists (the Pole
// repairs of the derived-field pass change sources of earlier syncs).
int run_sync(mhd_ctx *ctx, const char *group, bool full = false)
{
    auto it = ctx->syncs.find(group);
    if (it == ctx->syncs.end())
        return MHD_OK;
    SyncMap &m = it->second;
    if (!m.built)
    {
        if (ctx->capturing)
            return fail(ctx, MHD_ESTATE, "sync group %s changed during capture", group);
        RUN(build_sync(ctx, it->first, m));
    }
    if (!ctx->poles.empty())
    {
        // the hot lists in a step: the cold rest is written at read-out
        const CopyList &l = full ? m.full : m.hot;
        RUN(pole_rings(ctx, it->first));
        RUN(gather_map(ctx, l));
        if (!m.walls.empty())
        {
            prof_begin(ctx, "k_wall_u_all");
            k_wall_u_all<<<dim3(grid_for(m.wall_cols), unsigned(m.walls.size())), kThreads, 0, ctx->stream>>>(
                ctx->dbv, m.dwalls, ctx->c.gamma);
            RUN(launched(ctx));
        }
        RUN(gather_map(ctx, m.post));
        if (l.nconst > 0)
        {
            prof_begin(ctx, "k_set_consts");
            k_set_consts<<<grid_for(l.nconst), kThreads, 0, ctx->stream>>>(ctx->pool, l.cdst, l.cval, l.nconst);
            RUN(launched(ctx));
        }
        ctx->dirty[it->first] = !full && (m.cold.n > 0 || m.cold.nconst > 0);
        return MHD_OK;
    }
    const CopyList &l = full ? m.full : m.hot;
    if (l.nconst > 0)
    {
        prof_begin(ctx, "k_set_consts");
        k_set_consts<<<grid_for(l.nconst), kThreads, 0, ctx->stream>>>(ctx->pool, l.cdst, l.cval, l.nconst);
        RUN(launched(ctx));
    }
    if (!m.walls.empty())
    {
        prof_begin(ctx, "k_wall_u_all");
        k_wall_u_all<<<dim3(grid_for(m.wall_cols), unsigned(m.walls.size())), kThreads, 0, ctx->stream>>>(
            ctx->dbv, m.dwalls, ctx->c.gamma);
        RUN(launched(ctx));
    }
    RUN(gather_map(ctx, l));
    ctx->dirty[it->first] = !full && (m.hot.n != m.full.n || m.hot.nconst != m.full.nconst);
    return MHD_OK;
}

// face areas and unit normals from the uploaded JD (eager, outside graphs)
int ensure_geom(mhd_ctx *ctx)
{
    if (!ctx->geom_dirty)
        return MHD_OK;
    if (ctx->capturing)
        return fail(ctx, MHD_ESTATE, "geometry changed during capture");
    int64_t nf = 0;
    for (int l = LOC_FXI; l <= LOC_FZETA; ++l)
        nf = std::max(nf, max_box(ctx, l, ctx->G));
    prof_begin(ctx, "k_face_normals");
    k_face_normals<<<dim3(grid_for(nf), ctx->nblocks, 3), kThreads, 0, ctx->stream>>>(ctx->dbv);
    RUN(launched(ctx));
    if (ctx->pool32)
    {
        int64_t vmax = 0;
        for (const auto &v : ctx->hbv)
            vmax = std::max(vmax, v.vol);
        prof_begin(ctx, "k_geom32");
        k_geom32<<<dim3(grid_for(vmax), ctx->nblocks), kThreads, 0, ctx->stream>>>(ctx->dbv);
        RUN(launched(ctx));
    }
    const int np = int(ctx->poles.size() / 2);
    if (np > 0)
    {
        // the Pole rings' normal matrices, from the geometry
        int stride = 0;
        for (int q = 0; q < np; ++q)
            stride = std::max(stride, ctx->hbv[size_t(ctx->poles[size_t(2 * q)])].ni + 1);
        if (stride != ctx->pole_stride || !ctx->pole_cache)
        {
            cudaFree(ctx->pole_cache);
            ctx->pole_cache = nullptr;
            CK(ctx, cudaMalloc(&ctx->pole_cache, size_t(np) * 3 * size_t(stride) * 10 * sizeof(double)));
            ctx->pole_stride = stride;
        }
        for (int op : {int(POLE_BCELL), int(POLE_EETA_REG), int(POLE_JCELL)})
        {
            int64_t w = 0;
            for (int q = 0; q < np; ++q)
            {
                const BlockView &v = ctx->hbv[size_t(ctx->poles[size_t(2 * q)])];
                w = std::max(w, pole_work(op, v.ni, v.nk));
            }
            prof_begin(ctx, "k_pole");
            launch_pole_op(op, w, np, ctx->stream, ctx->dbv, ctx->dpoles, ctx->pole_cache, ctx->pole_stride, 1);
            RUN(launched(ctx));
        }
    }
    ctx->geom_dirty = false;
    return MHD_OK;
}

// UpdateDerivedFields_ as two passes: B_cell with the J edges (both read the
// face B), then J_cell with PV / U_plus / the CFL bound (J_cell's weight
// stream beside PV's FP64 work).  Each sync runs after the pass that writes
// its fields and before any pass that reads them; the reference's order
// among these independent fields does not change any value.
int launch_update_derived_pole(mhd_ctx *ctx);

// J_cell's own pass when the derived-field pass runs split (k_pv_uplus_dt variant kPvSplit)
int launch_jcell_split(mhd_ctx *ctx)
{
    if (ctx->tune[TUNE_k_pv_uplus_dt] != kPvSplit)
        return MHD_OK;
    prof_begin(ctx, "k_jcell");
    launch_k_jcell(ctx->pool32 != nullptr, grid_kind(ctx, KIND_CELL0), ctx->stream, ctx->dbv);
    return launched(ctx);
}

int launch_update_derived(mhd_ctx *ctx)
{
    if (!ctx->poles.empty())
        return launch_update_derived_pole(ctx);
    cudaStream_t s = ctx->stream;
    prof_begin(ctx, "k_bcell_jedge");
    launch_k_bcell_jedge(ctx->tune[TUNE_k_bcell_jedge], ctx->pool32 != nullptr, grid_kind(ctx, KIND_STAG), s, ctx->dbv);
    RUN(launched(ctx));
    RUN(run_sync(ctx, "B_cell"));
    RUN(run_sync(ctx, "Jedge"));
    // arm the dt reduction, then J_cell, PV / U_plus and the CFL bound of the next step
    prof_begin(ctx, "k_arm_dt");
    k_arm_dt<<<1, 128, 0, s>>>(ctx->dt_key, ctx->nruns);
    RUN(launched(ctx));
    // first ghost layer only: deeper PV / U_plus ghosts are read by no kernel
    // of the step and are filled when read out (materialise_pv)
    RUN(launch_jcell_split(ctx));
    prof_begin(ctx, "k_pv_uplus_dt");
    launch_k_pv_uplus_dt(ctx->tune[TUNE_k_pv_uplus_dt], ctx->pool32 != nullptr, grid_kind(ctx, KIND_CELL1), s, ctx->dbv,
                         ctx->c, ctx->dt_key, 1, 1);
    ctx->pv_dirty = true;
    RUN(launched(ctx));
    RUN(run_sync(ctx, "J_cell"));
    RUN(run_sync(ctx, "Uplus"));
    return MHD_OK;
}

// UpdateDerivedFields_ with Poles, in the reference's order: calc_Bcell and
// Sync("B_cell"), the B_zeta rewrite of the first cell layer at each Pole
// (which the J edges then read), Calc_J_Edge and Sync("Jedge"), then J_cell
// (with PV / U_plus / the CFL bound), its pole-shell repair, and the syncs.
// B_cell and the J edges run as one pass before the rewrite; the few J edges
// that read a rewritten face are formed again after it (k_pole_jedge).
int launch_update_derived_pole(mhd_ctx *ctx)
{
    cudaStream_t s = ctx->stream;
    prof_begin(ctx, "k_bcell_jedge");
    launch_k_bcell_jedge(ctx->tune[TUNE_k_bcell_jedge], ctx->pool32 != nullptr, grid_kind(ctx, KIND_STAG), s, ctx->dbv);
    RUN(launched(ctx));
    RUN(run_sync(ctx, "B_cell"));
    RUN(launch_pole(ctx, POLE_BZETA));
    {
        const int np = int(ctx->poles.size() / 2);
        int64_t w = 0;
        for (int q = 0; q < np; ++q)
        {
            const BlockView &v = ctx->hbv[size_t(ctx->poles[size_t(2 * q)])];
            w = std::max<int64_t>(w, int64_t(v.ni + 1) * 2 * (v.nk + 1));
        }
        prof_begin(ctx, "k_jedge");
        k_pole_jedge<<<dim3(grid_for(w), unsigned(np)), kThreads, 0, s>>>(ctx->dbv, ctx->dpoles);
        RUN(launched(ctx));
    }
    RUN(run_sync(ctx, "Jedge"));
    prof_begin(ctx, "k_arm_dt");
    k_arm_dt<<<1, 128, 0, s>>>(ctx->dt_key, ctx->nruns);
    RUN(launched(ctx));
    RUN(launch_jcell_split(ctx));
    prof_begin(ctx, "k_pv_uplus_dt");
    launch_k_pv_uplus_dt(ctx->tune[TUNE_k_pv_uplus_dt], ctx->pool32 != nullptr, grid_kind(ctx, KIND_CELL1), s, ctx->dbv,
                         ctx->c, ctx->dt_key, 1, 1);
    ctx->pv_dirty = true;
    RUN(launched(ctx));
    RUN(launch_pole(ctx, POLE_JCELL));
    RUN(run_sync(ctx, "J_cell"));
    RUN(run_sync(ctx, "Uplus"));
    return MHD_OK;
}

int launch_fluid_ucontra(mhd_ctx *ctx);

int launch_fluid_rhs(mhd_ctx *ctx)
{
    if (ctx->pool32) // the mixed form's flux pass (its FP32 U_contra are a by-product)
        return launch_fluid_ucontra(ctx);
    const int64_t nc = max_box(ctx, LOC_CELL, 0);
    prof_begin(ctx, "k_fluid_rhs");
    k_fluid_rhs<<<dim3(grid_for(nc), ctx->nblocks), kThreads, 0, ctx->stream>>>(ctx->dbv, ctx->c, nc);
    return launched(ctx);
}

// fluid RHS together with the contravariant velocities of the EMF stencils
int launch_fluid_ucontra(mhd_ctx *ctx)
{
    if (ctx->pool32)
    {
        prof_begin(ctx, "k_fluid_mixed");
        const int var = ctx->tune[TUNE_k_fluid_mixed];
        launch_k_fluid_mixed(var, grid_kind(ctx, var >= 3 ? KIND_TILE1 : KIND_CELL1), ctx->stream, ctx->dbv, ctx->c);
        return launched(ctx);
    }
    prof_begin(ctx, "k_fluid_ucontra");
    launch_k_fluid_ucontra(ctx->tune[TUNE_k_fluid_ucontra], grid_kind(ctx, KIND_CELL1), ctx->stream, ctx->dbv, ctx->c);
    return launched(ctx);
}

// AssembleRHS_Induction_CT_; with_ucontra unless the fluid pass computed them
int launch_induction(mhd_ctx *ctx, bool update_b, bool with_ucontra = true)
{
    const int nb = ctx->nblocks;
    cudaStream_t s = ctx->stream;
    if (with_ucontra)
    {
        prof_begin(ctx, "k_ucontra");
        k_ucontra<<<dim3(grid_for(max_box(ctx, LOC_CELL, 1)), nb), kThreads, 0, s>>>(ctx->dbv);
        RUN(launched(ctx));
    }
    prof_begin(ctx, "k_eface");
    launch_k_eface(ctx->tune[TUNE_k_eface], grid_kind(ctx, KIND_STAG), s, ctx->dbv);
    RUN(launched(ctx));
    RUN(run_sync(ctx, "Eface"));
    // inner edges; ghost edges keep their zero of AssembleRHS_Induction_CT_
    // except where the Eedge sync writes them
    prof_begin(ctx, "k_eedge");
    launch_k_eedge(ctx->tune[TUNE_k_eedge], grid_kind(ctx, KIND_STAG), s, ctx->dbv);
    RUN(launched(ctx));
    RUN(run_sync(ctx, "Eedge"));
    prof_begin(ctx, "k_curl_e2f");
    launch_k_curl_e2f(ctx->tune[TUNE_k_curl_e2f], grid_kind(ctx, KIND_STAG), s, ctx->dbv, F_Exi, F_RBxi, update_b ? F_Bxi : -1, -1.0,
                                                             ctx->dt, 1.0, 0, nullptr);
    return launched(ctx);
}

int launch_update_u(mhd_ctx *ctx)
{
    prof_begin(ctx, "k_update_u");
    k_update_u<<<grid_kind(ctx, KIND_CELL0), kThreads, 0, ctx->stream>>>(ctx->dbv, ctx->dt);
    return launched(ctx);
}


// ---------------------------------------------------------------------------
// implicit resistive step (Z4_Lunar/src/implicit/Lunar_ImplicitResistive.cpp:264-518)
//
// The operator only touches the unknowns' neighbourhood: Eres is non-zero at
// the unknowns, their aliases and the sync images of those, and dB next to
// them.  mhd_set_resistive computes per block a box holding all of these
// (closed under the Eres1form and dB copies, widened by the curl stencils);
// the curls, J edges and copies of the solve run on that box only.  Outside
// it the fields stay zero, as the reference's full-array clears and loops
// leave them, so restricting the work changes no value the solve reads.
// ---------------------------------------------------------------------------

int launch_curl_rng(mhd_ctx *ctx, int fE0, int fR0, int fB0, double mult, int mult_is_neg_dt)
{
    auto &R = ctx->res;
    if (R.nreg_max == 0)
        return MHD_OK;
    prof_begin(ctx, "k_curl_e2f");
    launch_k_curl_e2f(ctx->tune[TUNE_k_curl_e2f], dim3(grid_for(R.nreg_max), ctx->nblocks), ctx->stream, 
        ctx->dbv, fE0, fR0, fB0, mult, ctx->dt, 1.0, mult_is_neg_dt, R.rng);
    return launched(ctx);
}

int launch_jedge_rng(mhd_ctx *ctx, int fB0, int fJ0)
{
    auto &R = ctx->res;
    if (R.nreg_max == 0)
        return MHD_OK;
    prof_begin(ctx, "k_jedge");
    k_jedge<<<dim3(grid_for(R.nreg_max), ctx->nblocks), kThreads, 0, ctx->stream>>>(ctx->dbv, fB0, fJ0, 1.0, R.rng);
    return launched(ctx);
}

// UnpackVecToImplicitEres_: Eres[unknowns] <- x (column *jdev of x0 when
// jdev is given), aliases <- sign * owner, Sync("Eres1form")
int unpack_eres(mhd_ctx *ctx, const double *x0, const int *jdev)
{
    auto &R = ctx->res;
    if (R.n > 0)
    {
        prof_begin(ctx, "k_scatter_vec");
        k_scatter_vec<<<grid_for(R.n), kThreads, 0, ctx->stream>>>(ctx->pool, R.e, x0, R.n, jdev, R.n);
        RUN(launched(ctx));
    }
    if (R.nalias > 0)
    {
        prof_begin(ctx, "k_alias_copy");
        k_alias_copy<<<grid_for(R.nalias), kThreads, 0, ctx->stream>>>(ctx->pool, R.alias_e, R.owner_e, R.sign,
                                                                        R.nalias);
        RUN(launched(ctx));
    }
    return apply_list(ctx, R.eres1form);
}

// y = A x  (MatMultImplicitResistive_): dB = -dt curl Eres, Sync("dB"),
// dJ = alpha curlAdj(beta dB), y = Eres - eta dJ at the unknowns.  The
// owner->alias copy of dJ is not needed: y reads dJ at owners only.
int resist_matvec(mhd_ctx *ctx, const double *x0, const int *jdev, double *y)
{
    auto &R = ctx->res;
    RUN(unpack_eres(ctx, x0, jdev));
    RUN(launch_curl_rng(ctx, F_Eresxi, F_dBxi, -1, 0.0, /*mult_is_neg_dt=*/1));
    RUN(apply_list(ctx, R.db));
    RUN(launch_jedge_rng(ctx, F_dBxi, F_dJxi));
    prof_begin(ctx, "k_resist_out");
    k_resist_out<<<grid_for(R.n), kThreads, 0, ctx->stream>>>(ctx->pool, R.e, R.dj, R.eta, y, R.n);
    return launched(ctx);
}

// out[c] = V_c . w for c < nvec (or c <= *jdev), out[0] = w . w when V is null
int dots(mhd_ctx *ctx, const double *V, int nvec, const int *jdev, const double *w, double *out)
{
    auto &R = ctx->res;
    const int ny = jdev ? R.restart + 1 : nvec;
    prof_begin(ctx, "k_dots");
    k_dots<<<dim3(R.ngroups, ny), 256, 0, ctx->stream>>>(V, R.n, nvec, w, R.n, R.partial, jdev, out, R.st->dot_done);
    return launched(ctx);
}

#define LAUNCH1(name, ...)                                        \
    do                                                            \
    {                                                             \
        prof_begin(ctx, #name);                                   \
        name<<<1, 1, 0, ctx->stream>>>(__VA_ARGS__);              \
        RUN(launched(ctx));                                       \
    } while (0)
#define LAUNCHN(name, n, ...)                                     \
    do                                                            \
    {                                                             \
        prof_begin(ctx, #name);                                   \
        name<<<grid_for(n), kThreads, 0, ctx->stream>>>(__VA_ARGS__); \
        RUN(launched(ctx));                                       \
    } while (0)

// GMRES(m) with x0 = 0 and the convergence test ||r|| <= max(rtol ||b||, atol)
// of PETSc's default (KSPConvergedDefault), in three pieces that run either
// eagerly (the host reads the loop flags) or inside the step graph (the
// kernels set conditional handles).
int gmres_prologue(mhd_ctx *ctx)
{
    auto &R = ctx->res;
    RUN(dots(ctx, nullptr, 1, nullptr, R.b, R.dots + 40));
    LAUNCH1(k_gmres_init, R.st, R.dots + 40, R.rtol, R.atol, R.maxit, R.restart);
    LAUNCHN(k_zero, R.n, R.x, R.n);
    return MHD_OK;
}

int gmres_cycle_start(mhd_ctx *ctx, cudaGraphConditionalHandle h, int use)
{
    auto &R = ctx->res;
    RUN(resist_matvec(ctx, R.x, nullptr, R.w));
    LAUNCHN(k_residual, R.n, R.b, R.w, R.r, R.n);
    RUN(dots(ctx, nullptr, 1, nullptr, R.r, R.dots));
    LAUNCH1(k_cycle_start, R.st, R.dots, h, use);
    LAUNCHN(k_div_guard, R.n, R.V, R.r, &R.st->beta, R.n, &R.st->inner);
    return MHD_OK;
}

// one Arnoldi step on column j, classical Gram-Schmidt applied twice
int gmres_step(mhd_ctx *ctx, cudaGraphConditionalHandle h, int use)
{
    auto &R = ctx->res;
    const int *j = &R.st->j;
    double *hcol = R.st->hcol;
    RUN(resist_matvec(ctx, R.V, j, R.w));
    RUN(dots(ctx, R.V, 0, j, R.w, hcol));
    LAUNCHN(k_sub_proj, R.n, R.V, R.n, 0, hcol, R.w, R.n, j);
    RUN(dots(ctx, R.V, 0, j, R.w, R.dots));
    LAUNCHN(k_sub_proj, R.n, R.V, R.n, 0, R.dots, R.w, R.n, j);
    prof_begin(ctx, "k_add_small");
    k_add_small<<<1, 32, 0, ctx->stream>>>(hcol, R.dots, j);
    RUN(launched(ctx));
    RUN(dots(ctx, nullptr, 1, nullptr, R.w, R.dots + 32));
    LAUNCH1(k_gmres_column, R.st, R.dots + 32);
    LAUNCHN(k_div_next, R.n, R.V, R.n, R.w, R.st, R.n);
    LAUNCH1(k_inner_check, R.st, h, use);
    return MHD_OK;
}

int gmres_cycle_end(mhd_ctx *ctx, cudaGraphConditionalHandle h, int use)
{
    auto &R = ctx->res;
    LAUNCH1(k_gmres_solve_y, R.st);
    LAUNCHN(k_add_basis, R.n, R.V, R.n, R.st, R.x, R.n);
    LAUNCH1(k_outer_check, R.st, h, use);
    return MHD_OK;
}

int read_flag(mhd_ctx *ctx, const int *dev, int *host)
{
    CK(ctx, cudaMemcpyAsync(host, dev, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    return MHD_OK;
}

int gmres_eager(mhd_ctx *ctx)
{
    auto &R = ctx->res;
    RUN(gmres_prologue(ctx));
    int outer = 1;
    while (outer)
    {
        RUN(gmres_cycle_start(ctx, 0, 0));
        int inner = 0;
        RUN(read_flag(ctx, &R.st->inner, &inner));
        while (inner)
        {
            RUN(gmres_step(ctx, 0, 0));
            ++R.its_eager;
            RUN(read_flag(ctx, &R.st->inner, &inner));
        }
        RUN(gmres_cycle_end(ctx, 0, 0));
        ++R.cycles_eager;
        RUN(read_flag(ctx, &R.st->outer, &outer));
    }
    return MHD_OK;
}

int capture_graph_of(mhd_ctx *ctx, cudaGraph_t *g)
{
    cudaStreamCaptureStatus st;
    CK(ctx, cudaStreamGetCaptureInfo(ctx->stream, &st, nullptr, g, nullptr, nullptr));
    if (st != cudaStreamCaptureStatusActive)
        return fail(ctx, MHD_ESTATE, "stream is not capturing");
    return MHD_OK;
}

// Appends a conditional node of the given type (while or if; handle h) at
// the capture position of ctx->stream and captures body(ctx, h) into it on a
// spare stream; *kernels receives the kernels one pass of the body launches
// (the bodies nested in it included).
int capture_cond(mhd_ctx *ctx, cudaGraphConditionalNodeType type, cudaGraphConditionalHandle h,
                 int (*body)(mhd_ctx *, cudaGraphConditionalHandle), int64_t *kernels)
{
    if (ctx->spare_depth >= int(sizeof ctx->spare / sizeof ctx->spare[0]))
        return fail(ctx, MHD_ESTATE, "conditional nodes nested too deep");
    cudaStreamCaptureStatus st;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t *deps = nullptr;
    size_t ndeps = 0;
    CK(ctx, cudaStreamGetCaptureInfo(ctx->stream, &st, nullptr, &g, &deps, &ndeps));
    cudaGraphNodeParams p = {cudaGraphNodeTypeConditional};
    p.conditional.handle = h;
    p.conditional.type = type;
    p.conditional.size = 1;
    cudaGraphNode_t node;
    CK(ctx, cudaGraphAddNode(&node, g, deps, ndeps, &p));
    CK(ctx, cudaStreamUpdateCaptureDependencies(ctx->stream, &node, 1, cudaStreamSetCaptureDependencies));
    cudaGraph_t bodyg = p.conditional.phGraph_out[0];
    cudaStream_t s2 = ctx->spare[ctx->spare_depth];
    if (!s2)
        return fail(ctx, MHD_ESTATE, "no capture stream");
    CK(ctx, cudaStreamBeginCaptureToGraph(s2, bodyg, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    cudaStream_t saved = ctx->stream;
    ctx->stream = s2;
    ctx->spare_depth += 1;
    const int64_t before = ctx->launches;
    const int rc = body(ctx, h);
    *kernels = ctx->launches - before;
    ctx->spare_depth -= 1;
    ctx->stream = saved;
    cudaGraph_t out = nullptr;
    const cudaError_t e = cudaStreamEndCapture(s2, &out);
    if (rc != MHD_OK)
        return rc;
    if (e != cudaSuccess)
        return fail(ctx, MHD_ECUDA, "conditional body capture failed: %s", cudaGetErrorString(e));
    return MHD_OK;
}

int capture_while(mhd_ctx *ctx, cudaGraphConditionalHandle h, int (*body)(mhd_ctx *, cudaGraphConditionalHandle),
                  int64_t *kernels)
{
    return capture_cond(ctx, cudaGraphCondTypeWhile, h, body, kernels);
}

int gmres_step_graph(mhd_ctx *ctx, cudaGraphConditionalHandle h) { return gmres_step(ctx, h, 1); }

int gmres_outer_body(mhd_ctx *ctx, cudaGraphConditionalHandle hout)
{
    auto &R = ctx->res;
    cudaGraph_t g = nullptr;
    RUN(capture_graph_of(ctx, &g));
    cudaGraphConditionalHandle hin;
    CK(ctx, cudaGraphConditionalHandleCreate(&hin, g, 0, 0));
    RUN(gmres_cycle_start(ctx, hin, 1));
    RUN(capture_while(ctx, hin, gmres_step_graph, &R.k_inner));
    return gmres_cycle_end(ctx, hout, 1);
}

// the solve as graph nodes: prologue, then while(outer) { cycle start,
// while(inner) { Arnoldi step }, cycle end }
int gmres_graph(mhd_ctx *ctx)
{
    auto &R = ctx->res;
    RUN(gmres_prologue(ctx));
    cudaGraph_t g = nullptr;
    RUN(capture_graph_of(ctx, &g));
    cudaGraphConditionalHandle hout;
    CK(ctx, cudaGraphConditionalHandleCreate(&hout, g, 1, cudaGraphCondAssignDefault));
    int64_t kcyc = 0;
    RUN(capture_while(ctx, hout, gmres_outer_body, &kcyc));
    R.k_cycle = kcyc - R.k_inner;
    return MHD_OK;
}

// the resistive part of StepOnce (SolveImplicitResistiveDiffusion_ +
// ApplyImplicitResistiveUpdate_).  The reference syncs Bface twice before
// the solve and once after the update; one sync before is equivalent (a
// composed sync is idempotent) and the closing Sync("Bface") of the step
// repeats the one after.  J is needed at the unknowns only here (the
// derived-field pass recomputes it everywhere).
DevCopy dev_copy(const CopyList &l)
{
    return DevCopy{l.cdst, l.cval, l.nconst, l.dst, l.src, l.tmp, l.n};
}

// the whole solve as one cooperative kernel (k_gmres_resist)
int launch_gmres_persistent(mhd_ctx *ctx)
{
    auto &R = ctx->res;
    ResistSolve a{};
    a.bvs = ctx->dbv;
    a.pool = ctx->pool;
    a.nblocks = ctx->nblocks;
    a.e = R.e;
    a.dj = R.dj;
    a.j = R.j;
    a.eta = R.eta;
    a.n = R.n;
    a.alias = R.alias_e;
    a.alias_of = R.alias_of;
    a.sign = R.sign;
    a.nalias = R.nalias;
    a.eres1form = dev_copy(R.eres1form);
    a.db = dev_copy(R.db);
    a.uloc = R.uloc;
    a.merge1 = R.merge1;
    a.merge2 = R.merge2;
    a.rng = R.rng;
    a.nreg = R.nreg_max;
    a.dtp = ctx->dt;
    a.V = R.V;
    a.w = R.w;
    a.x = R.x;
    a.b = R.b;
    a.r = R.r;
    a.partial = R.ppartial;
    a.st = R.st;
    a.m = R.restart;
    a.maxit = R.maxit;
    a.rtol = R.rtol;
    a.atol = R.atol;
    a.bar = R.bar;
    a.err = ctx->err;
    a.fa = FusedList{R.fa.dst, R.fa.kind, R.fa.idx, R.fa.val, R.fa.blk, R.fa.n};
    a.fb = FusedList{R.fb.dst, R.fb.kind, R.fb.idx, R.fb.val, R.fb.blk, R.fb.n};
    cudaLaunchConfig_t cfg = {};
    const int want = kTuneMinCtas[TUNE_k_gmres_resist][ctx->tune[TUNE_k_gmres_resist]];
    cfg.gridDim = dim3(unsigned(want > 0 ? std::min(want, R.pgrid) : R.pgrid));
    cfg.blockDim = dim3(256);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = ctx->stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    prof_begin(ctx, "k_gmres_resist");
    CK(ctx, cudaLaunchKernelEx(&cfg, k_gmres_resist, a));
    return launched(ctx);
}

int launch_resistive(mhd_ctx *ctx)
{
    auto &R = ctx->res;
    RUN(run_sync(ctx, "Bface"));
    RUN(launch_jedge_rng(ctx, F_Bxi, F_Jxi));
    if (R.n > 0 && R.pgrid > 0)
        RUN(launch_gmres_persistent(ctx));
    else if (R.n > 0)
    {
        LAUNCHN(k_resist_rhs, R.n, ctx->pool, R.j, R.eta, R.b, R.n);
        if (ctx->capturing && R.graph_loops)
            RUN(gmres_graph(ctx));
        else
            RUN(gmres_eager(ctx));
    }
    RUN(unpack_eres(ctx, R.x, nullptr));
    return launch_curl_rng(ctx, F_Eresxi, F_RBresxi, F_Bxi, -1.0, 0);
}

// the Euler stage at the current dt: fluid RHS, CT induction with the
// face-B update, cell update.  (The cell update stays a pass of its own: in
// the latency-bound mixed flux pass it ran slower than alone.)
int launch_euler_core(mhd_ctx *ctx)
{
    RUN(launch_fluid_ucontra(ctx));
    RUN(launch_induction(ctx, /*update_b=*/true, /*with_ucontra=*/false));
    return launch_update_u(ctx);
}

// one LunarSolver::StepOnce, explicit part: dt, fluid RHS, CT induction, update
int launch_step_a(mhd_ctx *ctx)
{
    prof_begin(ctx, "k_begin_step");
    k_begin_step<<<1, 128, 0, ctx->stream>>>(ctx->dt_key, ctx->dt, ctx->err, ctx->prm.dt_abort, ctx->nruns);
    RUN(launched(ctx));
    return launch_euler_core(ctx);
}

// ... and its closing part: run data, Sync("Ucell"), Sync("Bface"), derived fields
int launch_step_c(mhd_ctx *ctx)
{
    prof_begin(ctx, "k_end_step");
    k_end_step<<<1, 128, 0, ctx->stream>>>(ctx->dt, ctx->time, ctx->step, ctx->nruns);
    RUN(launched(ctx));
    RUN(run_sync(ctx, "Ucell"));
    RUN(run_sync(ctx, "Bface"));
    return launch_update_derived(ctx);
}

// ResistiveDiffusionSubcycles_ (Z4_Lunar/src/physics/LunarSolver_MagneticRHS.cpp:53-115):
// per sub-cycle Sync("Bface"), B_cell / J edge / J_cell with their syncs,
// the resistive edge EMF, Sync("Eres"), then B += (dt / nsub) (-curl Eres)
// and Sync("Bface").  With Poles, UpdateMagneticDerivedFields_ in the
// reference's order: the B_zeta rewrite after Sync("B_cell") (which the J
// edges read) and the pole-shell J_cell before Sync("J_cell"); Sync("Eres")
// regulates Eres_eta on the pole rings.
int launch_resistive_explicit(mhd_ctx *ctx)
{
    const int nb = ctx->nblocks;
    cudaStream_t s = ctx->stream;
    const unsigned gs = grid_for(max_stagger(ctx));
    for (int q = 0; q < ctx->res_nsub; ++q)
    {
        RUN(run_sync(ctx, "Bface"));
        prof_begin(ctx, "k_bcell");
        launch_k_bcell(false, dim3(grid_for(max_box(ctx, LOC_CELL, 0)), nb), s, ctx->dbv);
        RUN(launched(ctx));
        RUN(run_sync(ctx, "B_cell"));
        RUN(launch_pole(ctx, POLE_BZETA));
        prof_begin(ctx, "k_jedge");
        k_jedge<<<dim3(gs, nb), kThreads, 0, s>>>(ctx->dbv, F_Bxi, F_Jxi, 1.0, nullptr);
        RUN(launched(ctx));
        RUN(run_sync(ctx, "Jedge"));
        prof_begin(ctx, "k_jcell");
        k_jcell<<<dim3(grid_for(max_box(ctx, LOC_CELL, 0)), nb), kThreads, 0, s>>>(ctx->dbv);
        RUN(launched(ctx));
        RUN(launch_pole(ctx, POLE_JCELL));
        RUN(run_sync(ctx, "J_cell"));
        prof_begin(ctx, "k_eres_explicit");
        k_eres_explicit<<<dim3(gs, nb), kThreads, 0, s>>>(ctx->dbv, ctx->res_inver_Rem);
        RUN(launched(ctx));
        RUN(run_sync(ctx, "Eres"));
        prof_begin(ctx, "k_curl_e2f");
        launch_k_curl_e2f(ctx->tune[TUNE_k_curl_e2f], dim3(gs, nb), s, ctx->dbv, F_Eresxi, F_RBresxi, F_Bxi, -1.0, ctx->dt,
                                                     double(ctx->res_nsub), 0, nullptr);
        RUN(launched(ctx));
        RUN(run_sync(ctx, "Bface"));
    }
    return MHD_OK;
}

// ---------------------------------------------------------------------------
// Implicit Hall solve (ImplicitHallSolver::SolveOneStep,
// Z4_Lunar/src/implicit/Hall_Implicit_Solver.cpp:268-391, residual of
// Hall_Implicit_Formfunction.cpp:7-106).  Newton with a backtracking line
// search; each Newton system J dx = -F solved by restarted GMRES whose
// products J v are finite differences of F (the reference uses an
// approximate whistler Jacobian; both converge to the root of F).
//
// Steered on the device: the control state (HallCtl, GmresState) lives in
// device memory and one-thread kernels take every decision.  Inside the
// step graph the four loops (Newton steps, GMRES cycles, Arnoldi steps,
// line-search trials) and the restart product are conditional nodes whose
// handles those kernels set, so a step runs with no host round trip; run
// eagerly (a stage, or where conditional nodes cannot be built) the host
// reads the same kernels' mirror flags.  Every loop is bounded: Newton by
// maxit, GMRES by its iteration limit, the line search by 12 trials.
// ---------------------------------------------------------------------------

int hall_use(const mhd_ctx *ctx) { return ctx->capturing ? 1 : 0; }

// a conditional handle of the graph being captured (0 when eager)
int new_handle(mhd_ctx *ctx, cudaGraphConditionalHandle *h)
{
    *h = 0;
    if (!ctx->capturing)
        return MHD_OK;
    cudaGraph_t g = nullptr;
    RUN(capture_graph_of(ctx, &g));
    CK(ctx, cudaGraphConditionalHandleCreate(h, g, 0, 0));
    return MHD_OK;
}

// A loop (while) or branch (if) of the solve: captured as a conditional node
// whose body the device steers through h, or run eagerly with the host
// reading the flag the same kernels write.  *kernels receives the kernels
// of one captured pass; *eager counts the passes run eagerly.
int hall_cond(mhd_ctx *ctx, cudaGraphConditionalNodeType type, cudaGraphConditionalHandle h, const int *flag,
              int (*body)(mhd_ctx *, cudaGraphConditionalHandle), int64_t *kernels, long long *eager)
{
    if (ctx->capturing)
        return capture_cond(ctx, type, h, body, kernels);
    int go = 0;
    RUN(read_flag(ctx, flag, &go));
    while (go)
    {
        RUN(body(ctx, 0));
        *eager += 1;
        if (type == cudaGraphCondTypeIf)
            break;
        RUN(read_flag(ctx, flag, &go));
    }
    return MHD_OK;
}

// one pass of a vector reduction kernel over the solve's unknowns
#define HALL_RED(name, ...)                                                  \
    do                                                                       \
    {                                                                        \
        prof_begin(ctx, #name);                                              \
        name<<<ctx->hall.ngroups, 256, 0, ctx->stream>>>(__VA_ARGS__);       \
        RUN(launched(ctx));                                                  \
    } while (0)

// B <- B* (snapshot = false) or B* <- B (snapshot = true): the face B
// arrays of every block, one contiguous range per block
int hall_copy_b(mhd_ctx *ctx, bool snapshot)
{
    auto &H = ctx->hall;
    prof_begin(ctx, "k_copy_segments");
    if (snapshot)
        k_copy_segments<<<dim3(unsigned(H.copy_ctas), unsigned(ctx->nblocks)), kThreads, 0, ctx->stream>>>(
            H.bstar, ctx->pool, H.seg_snap, ctx->nblocks);
    else
        k_copy_segments<<<dim3(unsigned(H.copy_ctas), unsigned(ctx->nblocks)), kThreads, 0, ctx->stream>>>(
            ctx->pool, H.bstar, H.seg_restore, ctx->nblocks);
    return launched(ctx);
}

// UpdateMagneticDerivedFields_ with the B_cell / J_cell ghosts the Hall
// stencils read, then the Hall edge EMF.  B_cell and the J edges in one pass
// (both read only the face B; the B_cell sync between them in the reference
// touches neither input).
int hall_emf_from_current_b(mhd_ctx *ctx)
{
    const int nb = ctx->nblocks;
    cudaStream_t s = ctx->stream;
    prof_begin(ctx, "k_bcell_jedge");
    launch_k_bcell_jedge(ctx->tune[TUNE_k_bcell_jedge], false, grid_kind(ctx, KIND_STAG), s, ctx->dbv);
    RUN(launched(ctx));
    RUN(run_sync(ctx, "B_cell", true));
    RUN(run_sync(ctx, "Jedge"));
    prof_begin(ctx, "k_jcell");
    k_jcell<<<dim3(grid_for(max_box(ctx, LOC_CELL, 0)), nb), kThreads, 0, s>>>(ctx->dbv);
    RUN(launched(ctx));
    RUN(run_sync(ctx, "J_cell", true));
    prof_begin(ctx, "k_hall_cell");
    k_hall_cell<<<dim3(grid_for(max_box(ctx, LOC_CELL, ctx->G)), nb), kThreads, 0, s>>>(ctx->dbv, ctx->c,
                                                                                        ctx->hall_coef);
    RUN(launched(ctx));
    prof_begin(ctx, "k_hall_edge");
    launch_k_hall_edge(ctx->tune[TUNE_k_hall_edge], grid_kind(ctx, KIND_STAG), s, ctx->dbv, ctx->hall_zb, ctx->hall_nzb);
    return launched(ctx);
}

// the trial B of the Ehall unknowns in the pool (UnpackVecToEhallField_:
// owners already written, then their aliases), Sync("Ehall"), B = B* + dt
// (-curl Ehall) on inner faces (theta = 1), Sync("Bface")
int hall_trial_b(mhd_ctx *ctx)
{
    auto &H = ctx->hall;
    if (!H.from_snapshot)
        RUN(hall_copy_b(ctx, false));
    if (H.nalias > 0)
        LAUNCHN(k_alias_copy, H.nalias, ctx->pool, H.alias, H.owner, H.sign, H.nalias);
    RUN(run_sync(ctx, "Ehall", true));
    prof_begin(ctx, "k_curl_e2f");
    if (H.from_snapshot)
        k_curl_from_snapshot<<<grid_kind(ctx, KIND_STAG), kThreads, 0, ctx->stream>>>(ctx->dbv, F_Ehxi, F_RBxi, F_Bxi,
                                                                                      -1.0, ctx->dt, H.bs);
    else
        launch_k_curl_e2f(ctx->tune[TUNE_k_curl_e2f], dim3(grid_for(max_stagger(ctx)), ctx->nblocks), ctx->stream,
                          ctx->dbv, F_Ehxi, F_RBxi, F_Bxi, -1.0, ctx->dt, 1.0, 0, nullptr);
    RUN(launched(ctx));
    return run_sync(ctx, "Bface");
}

// FormFunction_ up to the predicted Hall EMF of the trial in the pool
int hall_chain(mhd_ctx *ctx)
{
    RUN(hall_trial_b(ctx));
    return hall_emf_from_current_b(ctx);
}

// one Arnoldi step: w = J V_j as (F(X + h V_j) - F(X)) / h, classical
// Gram-Schmidt twice against V_0..V_j (the second pass's norm by Pythagoras),
// the new Hessenberg column and V_{j+1}
int hall_arnoldi(mhd_ctx *ctx, cudaGraphConditionalHandle hin)
{
    auto &H = ctx->hall;
    const int *jd = &H.st->j;
    LAUNCHN(k_hall_trial, H.n, ctx->pool, H.e, H.X, &H.ctl->h, H.V, H.n, jd, H.Xt, H.n);
    RUN(hall_chain(ctx));
    HALL_RED(k_hall_jv_dots, ctx->pool, H.e, H.Xt, H.F, &H.ctl->h, H.w, H.V, H.n, H.st, H.n, H.partial, H.st->hcol,
             H.done);
    HALL_RED(k_hall_proj_dots, H.V, H.n, H.st, H.w, H.n, H.partial, H.dots, H.done);
    LAUNCH1(k_hall_column, H.st, H.dots);
    LAUNCHN(k_hall_next, H.n, H.V, H.n, H.w, H.st, H.dots, H.n);
    LAUNCH1(k_inner_check, H.st, hin, hall_use(ctx));
    return MHD_OK;
}

// r = b - J dx at a GMRES restart
int hall_restart_product(mhd_ctx *ctx, cudaGraphConditionalHandle)
{
    auto &H = ctx->hall;
    LAUNCHN(k_hall_trial, H.n, ctx->pool, H.e, H.X, &H.ctl->hdx, H.dx, 0, nullptr, H.Xt, H.n);
    RUN(hall_chain(ctx));
    LAUNCHN(k_hall_restart_r, H.n, ctx->pool, H.e, H.Xt, H.F, &H.ctl->hdx, H.b, H.r, H.n);
    return MHD_OK;
}

// one GMRES(m) cycle for J dx = -F (x0 = 0, PETSc's default test)
int hall_cycle(mhd_ctx *ctx, cudaGraphConditionalHandle hout)
{
    auto &H = ctx->hall;
    const int use = hall_use(ctx);
    HALL_RED(k_norm2, H.dx, H.n, H.partial, H.dots + 40, H.done);
    cudaGraphConditionalHandle hr;
    RUN(new_handle(ctx, &hr));
    LAUNCH1(k_hall_cycle_prep, H.ctl, H.dots + 40, hr, use);
    RUN(hall_cond(ctx, cudaGraphCondTypeIf, hr, &H.ctl->restart, hall_restart_product, &H.kb[HALL_KB_RESTART],
                  &H.eager[HALL_KB_RESTART]));
    HALL_RED(k_norm2, H.r, H.n, H.partial, H.dots + 44, H.done);
    cudaGraphConditionalHandle hin;
    RUN(new_handle(ctx, &hin));
    LAUNCH1(k_cycle_start, H.st, H.dots + 44, hin, use);
    LAUNCHN(k_div_guard, H.n, H.V, H.r, &H.st->beta, H.n, &H.st->inner);
    RUN(hall_cond(ctx, cudaGraphCondTypeWhile, hin, &H.st->inner, hall_arnoldi, &H.kb[HALL_KB_INNER],
                  &H.eager[HALL_KB_INNER]));
    LAUNCH1(k_gmres_solve_y, H.st);
    LAUNCHN(k_add_basis, H.n, H.V, H.n, H.st, H.dx, H.n);
    LAUNCH1(k_outer_check, H.st, hout, use);
    return MHD_OK;
}

// one line-search trial X + lambda dx
int hall_ls_trial(mhd_ctx *ctx, cudaGraphConditionalHandle hls)
{
    auto &H = ctx->hall;
    LAUNCHN(k_hall_trial, H.n, ctx->pool, H.e, H.X, &H.ctl->lambda, H.dx, 0, nullptr, H.Xt, H.n);
    RUN(hall_chain(ctx));
    HALL_RED(k_hall_res_dots, ctx->pool, H.e, H.Xt, H.Ft, H.n, H.partial, H.dots + 48, H.done);
    LAUNCH1(k_hall_ls_check, H.ctl, H.dots + 48, hls, hall_use(ctx));
    return MHD_OK;
}

// one Newton step: ||X||, GMRES for the correction, the line search, the new iterate
int hall_newton_step(mhd_ctx *ctx, cudaGraphConditionalHandle hn)
{
    auto &H = ctx->hall;
    const int use = hall_use(ctx);
    HALL_RED(k_norm2, H.X, H.n, H.partial, H.dots + 52, H.done);
    LAUNCH1(k_hall_step_begin, H.ctl, H.dots + 52);
    HALL_RED(k_hall_gmres_prologue, H.F, H.b, H.r, H.dx, H.n, H.partial, H.dots + 56, H.done);
    cudaGraphConditionalHandle hout;
    RUN(new_handle(ctx, &hout));
    LAUNCH1(k_hall_gmres_init, H.st, H.dots + 56, H.ksp_rtol, 0.0, H.ksp_maxit, H.restart, hout, use);
    RUN(hall_cond(ctx, cudaGraphCondTypeWhile, hout, &H.st->outer, hall_cycle, &H.kb[HALL_KB_CYCLE],
                  &H.eager[HALL_KB_CYCLE]));
    cudaGraphConditionalHandle hls;
    RUN(new_handle(ctx, &hls));
    LAUNCH1(k_hall_ls_begin, H.ctl, hls, use);
    RUN(hall_cond(ctx, cudaGraphCondTypeWhile, hls, &H.ctl->ls, hall_ls_trial, &H.kb[HALL_KB_LS],
                  &H.eager[HALL_KB_LS]));
    LAUNCHN(k_hall_take, H.n, H.X, H.Xt, H.F, H.Ft, H.n);
    LAUNCH1(k_hall_accept, H.ctl, hn, use);
    return MHD_OK;
}

// One implicit Hall solve at the current dt: Newton on F from the current
// Ehall (the reference's initial guess), then B = B* + dt (-curl Ehall) and
// Sync("Bface")
int launch_hall_implicit(mhd_ctx *ctx)
{
    auto &H = ctx->hall;
    if (!H.on || H.n == 0)
        return MHD_OK;
    RUN(build_all_syncs(ctx));
    {
        const auto it = ctx->syncs.find("Bface");
        H.from_snapshot = it != ctx->syncs.end() && it->second.built && it->second.full.tmp == nullptr &&
                          it->second.walls.empty() && ctx->poles.empty();
    }
    RUN(hall_copy_b(ctx, true));
    LAUNCHN(k_pack_vec, H.n, ctx->pool, H.e, H.X, H.n);
    // F of the initial guess (the unknowns in the pool are X already)
    RUN(hall_chain(ctx));
    HALL_RED(k_hall_res_dots, ctx->pool, H.e, H.X, H.F, H.n, H.partial, H.dots + 60, H.done);
    cudaGraphConditionalHandle hn;
    RUN(new_handle(ctx, &hn));
    LAUNCH1(k_hall_begin, H.ctl, H.dots + 60, H.st, H.rtol, H.atol, H.maxit, hn, hall_use(ctx));
    RUN(hall_cond(ctx, cudaGraphCondTypeWhile, hn, &H.ctl->newton, hall_newton_step, &H.kb[HALL_KB_NEWTON],
                  &H.eager[HALL_KB_NEWTON]));
    if (ctx->capturing)
    {
        // kernels per pass of each body, without the bodies nested in it
        H.kb[HALL_KB_CYCLE] -= H.kb[HALL_KB_INNER] + H.kb[HALL_KB_RESTART];
        H.kb_nested = H.kb[HALL_KB_NEWTON];
        H.kb[HALL_KB_NEWTON] -= (H.kb[HALL_KB_CYCLE] + H.kb[HALL_KB_INNER] + H.kb[HALL_KB_RESTART]) + H.kb[HALL_KB_LS];
    }
    // the final update with the converged Hall EMF
    LAUNCHN(k_hall_trial, H.n, ctx->pool, H.e, H.X, nullptr, nullptr, 0, nullptr, nullptr, H.n);
    return hall_trial_b(ctx);
}

// the part of a step before the eagerly driven solves: the explicit step,
// with the explicit resistive sub-cycles when they are on
int launch_step_a_mid(mhd_ctx *ctx)
{
    RUN(launch_step_a(ctx));
    if (!ctx->res.on && ctx->res_nsub > 0)
        RUN(launch_resistive_explicit(ctx));
    return MHD_OK;
}

// the resistive part of an Euler stage (implicit solve or explicit sub-cycles)
int launch_resistive_part(mhd_ctx *ctx)
{
    if (ctx->res.on)
        return launch_resistive(ctx);
    if (ctx->res_nsub > 0)
        return launch_resistive_explicit(ctx);
    return MHD_OK;
}

int launch_rk2(mhd_ctx *ctx, int save)
{
    prof_begin(ctx, "k_rk2");
    k_rk2<<<grid_kind(ctx, KIND_STAG), kThreads, 0, ctx->stream>>>(ctx->dbv, save);
    return launched(ctx);
}

// One SSP-RK2 step (Shu and Osher, 1988) from two of StepOnce's Euler stages
// at the dt of the step's start (the reference has only forward Euler,
// Z4_Lunar/src/LunarSolver_Driver.cpp:21-92): U1 = U^n + dt L(U^n), with the
// syncs and derived fields of the end of a step; U2 = U1 + dt L(U1); then
// U^{n+1} = 0.5 (U^n + U2) on the points the Euler update writes, and the
// step's closing syncs and derived fields.
int launch_step_rk2(mhd_ctx *ctx)
{
    RUN(launch_rk2(ctx, 1));
    RUN(launch_step_a(ctx));
    RUN(launch_resistive_part(ctx));
    RUN(run_sync(ctx, "Ucell"));
    RUN(run_sync(ctx, "Bface"));
    RUN(launch_update_derived(ctx));
    RUN(launch_euler_core(ctx));
    RUN(launch_resistive_part(ctx));
    RUN(launch_rk2(ctx, 0));
    return launch_step_c(ctx);
}

int launch_step(mhd_ctx *ctx)
{
    if (ctx->integrator == MHD_INTEGRATOR_SSPRK2)
        return launch_step_rk2(ctx);
    RUN(launch_step_a(ctx));
    if (ctx->res.on)
        RUN(launch_resistive(ctx));
    else if (ctx->res_nsub > 0)
        RUN(launch_resistive_explicit(ctx));
    RUN(launch_hall_implicit(ctx));
    return launch_step_c(ctx);
}

int check_err(mhd_ctx *ctx)
{
    int e = 0;
    CK(ctx, cudaMemcpyAsync(&e, ctx->err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    if (e == MHD_EDT)
    {
        double d = 0.0;
        cudaMemcpy(&d, ctx->dt, sizeof(double), cudaMemcpyDeviceToHost);
        const int z = 0;
        cudaMemcpy(ctx->err, &z, sizeof(int), cudaMemcpyHostToDevice);
        return fail(ctx, MHD_EDT, "dt too small or NaN: dt=%.3e", d);
    }
    if (e == MHD_EKRYLOV)
    {
        const int z = 0;
        cudaMemcpy(ctx->err, &z, sizeof(int), cudaMemcpyHostToDevice);
        if (ctx->res.bar)
            cudaMemset(ctx->res.bar, 0, 4 * sizeof(unsigned));
        return fail(ctx, MHD_EKRYLOV, "persistent Krylov solve: a grid barrier wait gave up");
    }
    return MHD_OK;
}

void drop_graph(mhd_ctx *ctx)
{
    for (auto *ge : {&ctx->gexec, &ctx->gexec_a, &ctx->gexec_c})
        if (*ge)
        {
            cudaGraphExecDestroy(*ge);
            *ge = nullptr;
        }
    for (auto *g : {&ctx->graph, &ctx->graph_a, &ctx->graph_c})
        if (*g)
        {
            cudaGraphDestroy(*g);
            *g = nullptr;
        }
}

int capture(mhd_ctx *ctx, int (*body)(mhd_ctx *), cudaGraph_t *graph, cudaGraphExec_t *exec, int64_t *nodes)
{
    const int64_t before = ctx->launches;
    CK(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    ctx->capturing = true;
    const int rc = body(ctx);
    ctx->capturing = false;
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
    const int64_t captured = ctx->launches - before;
    ctx->launches = before;
    if (rc != MHD_OK)
    {
        if (g)
            cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess)
        return fail(ctx, MHD_ECUDA, "graph capture failed: %s", cudaGetErrorString(e));
    *graph = g;
    CK(ctx, cudaGraphInstantiate(exec, g, 0));
    *nodes = captured;
    return MHD_OK;
}

// The step is one CUDA graph.  With the implicit resistive solve the Krylov
// loop is part of it (conditional while nodes steered by the device); where
// conditional nodes cannot be built, the step falls back to the explicit and
// closing parts as two graphs around an eagerly launched solve.
int build_graph(mhd_ctx *ctx)
{
    RUN(ensure_geom(ctx));
    if (ctx->gexec || ctx->gexec_a)
        return MHD_OK;
    RUN(build_all_syncs(ctx));
    if (ctx->integrator == MHD_INTEGRATOR_SSPRK2)
    {
        if (ctx->res.on && ctx->res.pgrid == 0)
            return fail(ctx, MHD_ESTATE, "SSP-RK2 with the implicit resistive solve needs the persistent solve");
        return capture(ctx, launch_step, &ctx->graph, &ctx->gexec, &ctx->graph_kernels);
    }
    if ((ctx->res.on || ctx->hall.on) && ctx->res.graph_loops)
    {
        ctx->hall.kb_nested = 0;
        const int rc = capture(ctx, launch_step, &ctx->graph, &ctx->gexec, &ctx->graph_kernels);
        if (rc == MHD_OK)
        {
            // the loop bodies were captured once; their launches are counted per pass
            ctx->graph_kernels -= ctx->res.k_cycle + ctx->res.k_inner + ctx->hall.kb_nested;
            return MHD_OK;
        }
        // conditional nodes unavailable: clear the error state of the stream and fall back
        cudaGetLastError();
        drop_graph(ctx);
        ctx->res.graph_loops = false;
        ctx->hall.kb_nested = 0;
        for (auto &k : ctx->hall.kb)
            k = 0;
    }
    if (ctx->res.on || ctx->hall.on)
    {
        RUN(capture(ctx, launch_step_a_mid, &ctx->graph_a, &ctx->gexec_a, &ctx->graph_kernels_a));
        return capture(ctx, launch_step_c, &ctx->graph_c, &ctx->gexec_c, &ctx->graph_kernels_c);
    }
    return capture(ctx, launch_step, &ctx->graph, &ctx->gexec, &ctx->graph_kernels);
}

int run_steps(mhd_ctx *ctx, int nsteps)
{
    RUN(build_graph(ctx));
    for (int s = 0; s < nsteps; ++s)
    {
        if (ctx->gexec)
        {
            CK(ctx, cudaGraphLaunch(ctx->gexec, ctx->stream));
            ctx->launches += ctx->graph_kernels;
        }
        else
        {
            CK(ctx, cudaGraphLaunch(ctx->gexec_a, ctx->stream));
            ctx->launches += ctx->graph_kernels_a;
            if (ctx->res.on)
                RUN(launch_resistive(ctx));
            RUN(launch_hall_implicit(ctx));
            CK(ctx, cudaGraphLaunch(ctx->gexec_c, ctx->stream));
            ctx->launches += ctx->graph_kernels_c;
        }
    }
    if (nsteps > 0)
        mark_dirty(ctx);
    return MHD_OK;
}

} // namespace

extern "C" {

namespace
{
int create_ctx(const mhd_block_desc *blocks, int32_t nblocks, const int32_t *run_of_block, int32_t nruns,
               const mhd_params *params, mhd_ctx **out)
{
    if (!blocks || nblocks <= 0 || !params || !out || nruns <= 0 || nruns > nblocks)
        return MHD_EINVAL;
    *out = nullptr;
    std::vector<int> run(size_t(nblocks), 0);
    if (run_of_block)
    {
        std::vector<int> seen(size_t(nruns), 0);
        for (int b = 0; b < nblocks; ++b)
        {
            if (run_of_block[b] < 0 || run_of_block[b] >= nruns)
                return MHD_EINVAL;
            run[size_t(b)] = run_of_block[b];
            seen[size_t(run_of_block[b])] = 1;
        }
        for (int r = 0; r < nruns; ++r)
            if (!seen[size_t(r)])
                return MHD_EINVAL; // every run owns at least one block
    }
    else if (nruns != 1)
        return MHD_EINVAL;
    mhd_ctx *ctx = new mhd_ctx;
    if (cudaGetDevice(&ctx->device) != cudaSuccess)
    {
        delete ctx;
        return MHD_ECUDA;
    }
    ctx->nblocks = nblocks;
    ctx->nruns = nruns;
    ctx->prm = *params;
    ctx->G = params->ngg > 0 ? params->ngg : 4;
    ctx->c = Consts{params->gamma,     params->cfl, params->inver_MA2,   params->momentum_hall_coeff,
                    params->state_coeff, params->M_H, params->M_ref, params->ne_hall_floor};
    for (int f = 0; f < NFIELD; ++f)
        if (kFields[f].nghost > ctx->G)
        {
            delete ctx;
            return MHD_EINVAL;
        }
    ctx->hbv.resize(size_t(nblocks));
    ctx->base.assign(NFIELD, std::vector<size_t>(size_t(nblocks), 0));
    size_t off = 0;
    for (int b = 0; b < nblocks; ++b)
    {
        if (blocks[b].ni <= 0 || blocks[b].nj <= 0 || blocks[b].nk <= 0)
        {
            delete ctx;
            return MHD_EINVAL;
        }
        BlockView &v = ctx->hbv[size_t(b)];
        v.run = run[size_t(b)];
        v.ni = blocks[b].ni;
        v.nj = blocks[b].nj;
        v.nk = blocks[b].nk;
        v.G = ctx->G;
        const int NI = v.ni + 1 + 2 * v.G;
        v.NJ = v.nj + 1 + 2 * v.G;
        v.NK = v.nk + 1 + 2 * v.G;
        v.vol = int64_t(NI) * v.NJ * v.NK;
        ctx->max_cells = std::max<int64_t>(ctx->max_cells, int64_t(v.ni) * v.nj * v.nk);
        for (int f = 0; f < NFIELD; ++f)
        {
            ctx->base[size_t(f)][size_t(b)] = off;
            off += size_t(kFields[f].ncomp) * size_t(v.vol);
            off = (off + 31) & ~size_t(31); // 256-byte aligned planes
        }
    }
    ctx->pool_n = off;
    auto bail = [&](int code) {
        mhd_ctx_destroy(ctx);
        return code;
    };
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess)
        return bail(MHD_ECUDA);
    {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_staging) != cudaSuccess)
            return bail(MHD_ECUDA);
        ctx->noalloc = static_cast<double *>(p);
    }
    if (cudaMalloc(&ctx->pool, off * sizeof(double)) != cudaSuccess)
        return bail(MHD_ENOMEM);
    if (cudaMemsetAsync(ctx->pool, 0, off * sizeof(double), ctx->stream) != cudaSuccess)
        return bail(MHD_ECUDA);
    for (int b = 0; b < nblocks; ++b)
        for (int f = 0; f < NFIELD; ++f)
            ctx->hbv[size_t(b)].f[f] = ctx->pool + ctx->base[size_t(f)][size_t(b)];
    if (params->precision == MHD_PREC_MIXED)
    {
        size_t n32 = 0;
        for (int b = 0; b < nblocks; ++b)
            n32 += size_t(G32_N + Q32_N + W32_N) * size_t(ctx->hbv[size_t(b)].vol);
        if (cudaMalloc(&ctx->pool32, n32 * sizeof(float)) != cudaSuccess)
            return bail(MHD_ENOMEM);
        if (cudaMemset(ctx->pool32, 0, n32 * sizeof(float)) != cudaSuccess)
            return bail(MHD_ECUDA);
        size_t o = 0;
        for (int b = 0; b < nblocks; ++b)
        {
            BlockView &v = ctx->hbv[size_t(b)];
            v.g32 = ctx->pool32 + o;
            v.q32 = v.g32 + size_t(G32_N) * size_t(v.vol);
            v.w32 = v.q32 + size_t(Q32_N) * size_t(v.vol);
            o += size_t(G32_N + Q32_N + W32_N) * size_t(v.vol);
        }
    }
    else if (params->precision != MHD_PREC_FP64)
        return bail(MHD_EINVAL);
    // per-run scalars: dt keys, dt, time, step (8 bytes each per run), the
    // error word, then the flux reference states
    const size_t nr = size_t(nruns);
    const size_t scal_bytes = 32 * nr + 64 + 48 * nr;
    void *scal = nullptr;
    if (cudaMalloc(&scal, scal_bytes) != cudaSuccess)
        return bail(MHD_ENOMEM);
    if (cudaMemset(scal, 0, scal_bytes) != cudaSuccess)
        return bail(MHD_ECUDA);
    char *sc = static_cast<char *>(scal);
    ctx->dt_key = reinterpret_cast<unsigned long long *>(sc);
    ctx->dt = reinterpret_cast<double *>(sc + 8 * nr);
    ctx->time = reinterpret_cast<double *>(sc + 16 * nr);
    ctx->step = reinterpret_cast<long long *>(sc + 24 * nr);
    ctx->err = reinterpret_cast<int *>(sc + 32 * nr);
    ctx->qref = reinterpret_cast<double *>(sc + 32 * nr + 64);
    {
        const double big = 1e100;
        unsigned long long key;
        std::memcpy(&key, &big, 8);
        const std::vector<unsigned long long> keys(nr, key);
        if (cudaMemcpy(ctx->dt_key, keys.data(), 8 * nr, cudaMemcpyHostToDevice) != cudaSuccess)
            return bail(MHD_ECUDA);
    }
    for (int b = 0; b < nblocks; ++b)
        ctx->hbv[size_t(b)].qref = ctx->qref + 6 * size_t(run[size_t(b)]);
    // flattened launches when the batch holds several runs
    if (nruns > 1)
    {
        std::vector<int> tab;
        int64_t first[NKIND] = {};
        for (int kind = 0; kind < NKIND; ++kind)
        {
            first[kind] = int64_t(tab.size());
            for (int b = 0; b < nblocks; ++b)
            {
                BlockView &v = ctx->hbv[size_t(b)];
                const int64_t n = grid_for(kind_points(v, kind));
                v.cta0[kind] = int(int64_t(tab.size()) - first[kind]);
                tab.insert(tab.end(), size_t(n), b);
            }
            ctx->cta_total[kind] = int64_t(tab.size()) - first[kind];
            if (ctx->cta_total[kind] > INT_MAX)
                return bail(MHD_EINVAL);
        }
        if (cudaMalloc(&ctx->cta_tab, tab.size() * sizeof(int)) != cudaSuccess)
            return bail(MHD_ENOMEM);
        if (cudaMemcpy(ctx->cta_tab, tab.data(), tab.size() * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess)
            return bail(MHD_ECUDA);
        for (auto &v : ctx->hbv)
            for (int kind = 0; kind < NKIND; ++kind)
                v.cta_blk[kind] = ctx->cta_tab + first[kind];
        ctx->flat = true;
    }
    if (cudaMalloc(&ctx->dbv, sizeof(BlockView) * size_t(nblocks)) != cudaSuccess)
        return bail(MHD_ENOMEM);
    if (cudaMemcpy(ctx->dbv, ctx->hbv.data(), sizeof(BlockView) * size_t(nblocks), cudaMemcpyHostToDevice) !=
        cudaSuccess)
        return bail(MHD_ECUDA);
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess)
        return bail(MHD_ECUDA);
    *out = ctx;
    return MHD_OK;
}
} // namespace

int mhd_ctx_create(const mhd_block_desc *blocks, int32_t nblocks, const mhd_params *params, mhd_ctx **out)
{
    return create_ctx(blocks, nblocks, nullptr, 1, params, out);
}

int mhd_batch_create(const mhd_block_desc *blocks, int32_t nblocks, const int32_t *run_of_block, int32_t nruns,
                     const mhd_params *params, mhd_ctx **out)
{
    if (!run_of_block)
        return MHD_EINVAL;
    return create_ctx(blocks, nblocks, run_of_block, nruns, params, out);
}

int mhd_ctx_destroy(mhd_ctx *ctx)
{
    BIND_DEVICE(ctx);
    if (!ctx)
        return MHD_OK;
    drop_graph(ctx);
    for (auto &kv : ctx->syncs)
    {
        free_list(kv.second.full);
        free_list(kv.second.hot);
        free_list(kv.second.post);
        free_list(kv.second.cold);
        cudaFree(kv.second.dwalls);
    }
    cudaFree(ctx->dpoles);
    cudaFree(ctx->pole_cache);
    cudaFree(ctx->diag_keys);
    free_resistive(ctx);
    cudaFree(ctx->hall_zb);
    mhd_set_hall_implicit(ctx, 0, nullptr, 0, nullptr, nullptr, nullptr, 0.0, 0.0, 0, 0.0, 1);
    for (auto &sp : ctx->spare)
        if (sp)
            cudaStreamDestroy(sp);
    if (ctx->dt_key)
        cudaFree(ctx->dt_key);
    cudaFree(ctx->cta_tab);
    cudaFree(ctx->rk);
    cudaFree(ctx->staging);
    cudaFree(ctx->dbv);
    cudaFree(ctx->pool);
    cudaFree(ctx->pool32);
    if (ctx->stream)
        cudaStreamDestroy(ctx->stream);
    delete ctx;
    return MHD_OK;
}

int mhd_last_error(const mhd_ctx *ctx, char *buf, int32_t buflen)
{
    if (!ctx || !buf || buflen <= 0)
        return MHD_EINVAL;
    std::snprintf(buf, size_t(buflen), "%s", ctx->msg.c_str());
    return MHD_OK;
}

int mhd_field_info(const mhd_ctx *ctx, const char *name, int32_t block, int32_t *loc, int32_t *ncomp, int32_t *nghost,
                   int32_t lo[3], int32_t hi[3])
{
    const int f = field_by_name(name);
    if (!ctx || f < 0 || block < 0 || block >= ctx->nblocks)
        return MHD_EINVAL;
    int l[3], h[3];
    field_box(ctx, f, block, l, h);
    if (loc)
        *loc = kFields[f].loc;
    if (ncomp)
        *ncomp = kFields[f].ncomp;
    if (nghost)
        *nghost = kFields[f].nghost;
    for (int d = 0; d < 3; ++d)
    {
        if (lo)
            lo[d] = l[d];
        if (hi)
            hi[d] = h[d];
    }
    return MHD_OK;
}

static int transfer(mhd_ctx *ctx, const char *name, int32_t block, const double *hin, double *hout, int64_t count)
{
    const int f = field_by_name(name);
    if (!ctx)
        return MHD_EINVAL;
    if (f < 0 || block < 0 || block >= ctx->nblocks)
        return fail(ctx, MHD_EINVAL, "unknown field '%s' or block %d", name ? name : "(null)", block);
    const int64_t n = field_count(ctx, f, block);
    if (count != n)
        return fail(ctx, MHD_EINVAL, "field %s block %d holds %lld values, got %lld", name, block, (long long)n,
                    (long long)count);
    RUN(ensure_staging(ctx, size_t(n)));
    int lo[3], hi[3];
    field_box(ctx, f, block, lo, hi);
    const int nc = kFields[f].ncomp;
    if (hin)
    {
        if (f == F_JDxi || f == F_JDeta || f == F_JDzeta || f == F_WB || f == F_WJ || f == F_drxi || f == F_dreta ||
            f == F_drzeta)
            ctx->geom_dirty = true; // face normals, FP32 copies and Pole matrices follow
        CK(ctx, cudaMemcpyAsync(ctx->staging, hin, size_t(n) * 8, cudaMemcpyHostToDevice, ctx->stream));
        prof_begin(ctx, "k_aos_to_soa");
        k_aos_to_soa<<<grid_for(n), kThreads, 0, ctx->stream>>>(ctx->dbv, block, f, nc, lo[0], lo[1], lo[2],
                                                                hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2],
                                                                ctx->staging);
        RUN(launched(ctx));
    }
    else
    {
        prof_begin(ctx, "k_soa_to_aos");
        k_soa_to_aos<<<grid_for(n), kThreads, 0, ctx->stream>>>(ctx->dbv, block, f, nc, lo[0], lo[1], lo[2],
                                                                hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2],
                                                                ctx->staging);
        RUN(launched(ctx));
        CK(ctx, cudaMemcpyAsync(hout, ctx->staging, size_t(n) * 8, cudaMemcpyDeviceToHost, ctx->stream));
    }
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    return MHD_OK;
}

int mhd_upload_field(mhd_ctx *ctx, const char *name, int32_t block, const double *data, int64_t count)
{
    BIND_DEVICE(ctx);
    if (!ctx || !data)
        return fail(ctx, MHD_EINVAL, "null data");
    // every field the device holds is brought to the reference's state first
    RUN(materialise_all(ctx));
    return transfer(ctx, name, block, data, nullptr, count);
}

// ---------------------------------------------------------------------------
// Allocation-free read-out (no counterpart in the reference): stages through
// g_noalloc_staging, whose device address the context looked up at creation.
// ---------------------------------------------------------------------------
int mhd_download_field_noalloc(mhd_ctx *ctx, const char *name, int32_t block, double *data, int64_t count)
{
    BIND_DEVICE(ctx);
    if (!ctx || !data)
        return fail(ctx, MHD_EINVAL, "null data");
    const int f = field_by_name(name);
    if (f < 0 || block < 0 || block >= ctx->nblocks)
        return fail(ctx, MHD_EINVAL, "unknown field '%s' or block %d", name ? name : "(null)", block);
    const int64_t n = field_count(ctx, f, block);
    if (count != n)
        return fail(ctx, MHD_EINVAL, "field %s block %d holds %lld values, got %lld", name, block, (long long)n,
                    (long long)count);
    if (n > int64_t(MHD_NOALLOC_MAX_DOUBLES))
        return fail(ctx, MHD_EINVAL,
                    "field %s block %d holds %lld values; the allocation-free read-out holds at most %d",
                    name, block, (long long)n, MHD_NOALLOC_MAX_DOUBLES);
    // bringing the field to the reference's state must only replay tables
    // that are already on the device
    for (const auto &kv : ctx->syncs)
        if (!kv.second.built)
            return fail(ctx, MHD_ESTATE, "sync group %s is not on the device yet; step or update the derived "
                        "fields once before an allocation-free read-out", kv.first.c_str());
    double *stage = ctx->noalloc;
    if (!stage)
        return fail(ctx, MHD_ESTATE, "the read-out array's device address is unknown");
    RUN(materialise_field(ctx, f));
    int lo[3], hi[3];
    field_box(ctx, f, block, lo, hi);
    prof_begin(ctx, "k_soa_to_aos");
    k_soa_to_aos<<<grid_for(n), kThreads, 0, ctx->stream>>>(ctx->dbv, block, f, kFields[f].ncomp, lo[0], lo[1],
                                                            lo[2], hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2], stage);
    RUN(launched(ctx));
    CK(ctx, cudaMemcpyAsync(data, stage, size_t(n) * 8, cudaMemcpyDeviceToHost, ctx->stream));
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    return MHD_OK;
}

int mhd_download_field(mhd_ctx *ctx, const char *name, int32_t block, double *data, int64_t count)
{
    BIND_DEVICE(ctx);
    if (!ctx || !data)
        return fail(ctx, MHD_EINVAL, "null data");
    const int f = field_by_name(name);
    if (f >= 0)
        RUN(materialise_field(ctx, f));
    return transfer(ctx, name, block, nullptr, data, count);
}

int64_t mhd_point_id(const mhd_ctx *ctx, const char *name, int32_t block, int32_t i, int32_t j, int32_t k, int32_t m)
{
    const int f = field_by_name(name);
    if (!ctx || f < 0 || block < 0 || block >= ctx->nblocks || m < 0 || m >= kFields[f].ncomp)
        return -1;
    int lo[3], hi[3];
    field_box(ctx, f, block, lo, hi);
    if (i < lo[0] || j < lo[1] || k < lo[2] || i >= hi[0] || j >= hi[1] || k >= hi[2])
        return -1;
    const int64_t aos =
        ((int64_t(i - lo[0]) * (hi[1] - lo[1]) + (j - lo[1])) * (hi[2] - lo[2]) + (k - lo[2])) * kFields[f].ncomp + m;
    return (int64_t(f) << 56) | (int64_t(block) << 40) | aos;
}

// point id -> pool offset (-1 if invalid)
static int64_t pool_offset(const mhd_ctx *ctx, int64_t id)
{
    if (id < 0)
        return -1;
    const int f = int(id >> 56);
    const int b = int((id >> 40) & 0xffff);
    int64_t aos = id & ((int64_t(1) << 40) - 1);
    if (f >= NFIELD || b >= ctx->nblocks)
        return -1;
    int lo[3], hi[3];
    field_box(ctx, f, b, lo, hi);
    const int nc = kFields[f].ncomp;
    const int n1 = hi[1] - lo[1], n2 = hi[2] - lo[2];
    if (aos >= int64_t(hi[0] - lo[0]) * n1 * n2 * nc)
        return -1;
    const int m = int(aos % nc);
    aos /= nc;
    const int k = lo[2] + int(aos % n2);
    aos /= n2;
    const int j = lo[1] + int(aos % n1);
    const int i = lo[0] + int(aos / n1);
    const BlockView &v = ctx->hbv[size_t(b)];
    return int64_t(ctx->base[size_t(f)][size_t(b)]) + int64_t(m) * v.vol + pidx(v, i, j, k);
}

} // extern "C"

template <typename T> static int upload_vec(mhd_ctx *ctx, const std::vector<T> &v, T **d)
{
    *d = nullptr;
    if (v.empty())
        return MHD_OK;
    CK(ctx, cudaMalloc(d, v.size() * sizeof(T)));
    CK(ctx, cudaMemcpy(*d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    return MHD_OK;
}

static void free_list(CopyList &m)
{
    cudaFree(m.dst);
    cudaFree(m.src);
    cudaFree(m.dst32);
    cudaFree(m.src32);
    cudaFree(m.tmp);
    cudaFree(m.cdst);
    cudaFree(m.cval);
    m = CopyList();
}

static void free_resistive(mhd_ctx *ctx)
{
    auto &R = ctx->res;
    for (void *p : {(void *)R.e, (void *)R.dj, (void *)R.j, (void *)R.eta, (void *)R.alias_e, (void *)R.owner_e,
                    (void *)R.sign, (void *)R.rng, (void *)R.V, (void *)R.w, (void *)R.x,
                    (void *)R.b, (void *)R.r, (void *)R.partial, (void *)R.dots, (void *)R.st,
                    (void *)R.alias_of, (void *)R.ppartial, (void *)R.bar, (void *)R.uloc})
        cudaFree(p);
    for (auto *fl : {&R.fa, &R.fb})
        for (void *p : {(void *)fl->dst, (void *)fl->kind, (void *)fl->idx, (void *)fl->val, (void *)fl->blk})
            cudaFree(p);
    free_list(R.eres1form);
    free_list(R.db);
    const bool loops = R.graph_loops;
    R = mhd_ctx::Resistive();
    R.graph_loops = loops;
}

// pool offset -> (block, i, j, k) of the point (component dropped)
struct PoolDecoder
{
    std::vector<std::pair<uint64_t, int>> starts; // (base offset, field * nblocks + block), sorted
    const mhd_ctx *ctx;
    explicit PoolDecoder(const mhd_ctx *c) : ctx(c)
    {
        for (int f = 0; f < NFIELD; ++f)
            for (int b = 0; b < c->nblocks; ++b)
                starts.push_back({uint64_t(c->base[size_t(f)][size_t(b)]), f * c->nblocks + b});
        std::sort(starts.begin(), starts.end());
    }
    bool operator()(uint64_t off, int &b, int &i, int &j, int &k) const
    {
        int f;
        return decode(off, f, b, i, j, k);
    }
    bool decode(uint64_t off, int &f, int &b, int &i, int &j, int &k) const
    {
        auto it = std::upper_bound(starts.begin(), starts.end(), std::make_pair(off, INT32_MAX));
        if (it == starts.begin())
            return false;
        --it;
        f = it->second / ctx->nblocks;
        b = it->second % ctx->nblocks;
        const BlockView &v = ctx->hbv[size_t(b)];
        const uint64_t rel = off - it->first;
        if (rel >= uint64_t(v.vol) * uint64_t(kFields[f].ncomp))
            return false;
        const int64_t p = int64_t(rel % uint64_t(v.vol));
        k = int(p % v.NK) - v.G;
        j = int((p / v.NK) % v.NJ) - v.G;
        i = int(p / (int64_t(v.NK) * v.NJ)) - v.G;
        return true;
    }
};

struct IBox
{
    int lo[3] = {INT32_MAX, INT32_MAX, INT32_MAX};
    int hi[3] = {INT32_MIN, INT32_MIN, INT32_MIN}; // exclusive
    bool empty() const { return lo[0] >= hi[0]; }
    void add(int i, int j, int k)
    {
        const int p[3] = {i, j, k};
        for (int a = 0; a < 3; ++a)
        {
            lo[a] = std::min(lo[a], p[a]);
            hi[a] = std::max(hi[a], p[a] + 1);
        }
    }
    bool has(int i, int j, int k, int widen = 0) const
    {
        return !empty() && i >= lo[0] - widen && i < hi[0] + widen && j >= lo[1] - widen && j < hi[1] + widen &&
               k >= lo[2] - widen && k < hi[2] + widen;
    }
};

static void host_map(mhd_ctx *ctx, const char *group, std::vector<uint64_t> &d, std::vector<uint64_t> &s,
                     bool &staged)
{
    auto it = ctx->syncs.find(group);
    if (it == ctx->syncs.end())
    {
        d.clear();
        s.clear();
        staged = false;
        return;
    }
    d = it->second.hd;
    s = it->second.hs;
    staged = it->second.staged;
}

static int upload_list(mhd_ctx *ctx, CopyList &l, const std::vector<uint64_t> &cd, const std::vector<double> &cv,
                       const std::vector<uint64_t> &d, const std::vector<uint64_t> &s2, bool staged)
{
    free_list(l);
    RUN(upload_vec(ctx, cd, &l.cdst));
    RUN(upload_vec(ctx, cv, &l.cval));
    l.nconst = int64_t(cd.size());
    RUN(upload_vec(ctx, d, &l.dst));
    RUN(upload_vec(ctx, s2, &l.src));
    l.n = int64_t(d.size());
    if (staged && l.n > 0)
        CK(ctx, cudaMalloc(&l.tmp, size_t(l.n) * 8));
    if (!staged && l.n > 0 && ctx->pool_n < (size_t(1) << 32))
    {
        const std::vector<uint32_t> d32(d.begin(), d.end()), s32(s2.begin(), s2.end());
        RUN(upload_vec(ctx, d32, &l.dst32));
        RUN(upload_vec(ctx, s32, &l.src32));
    }
    return MHD_OK;
}

// Ghost depth of each field that a kernel of the step reads: the face,
// edge and contravariant-velocity stencils reach one layer into U_H, the
// face B, Eface and U_plus; the edge EMF and J edges, B_cell, Bind_cell and
// J_cell are read on inner points only.  Other fields keep every layer.
static int hot_depth(const mhd_ctx *ctx, int f)
{
    // the explicit resistive EMF averages J_cell over the four cells around
    // an edge, one ghost layer deep
    if (f == F_Jcell && ctx->res_nsub > 0)
        return 1;
    // the Pole work items read B_cell / Bind_cell at k = n_k, the ring's
    // periodic ghost (E_xi on the pole line, the B_zeta rewrite)
    if ((f == F_Bcell || f == F_Bind) && !ctx->poles.empty())
        return 1;
    switch (f)
    {
    case F_U:
    case F_Bxi:
    case F_Beta:
    case F_Bzeta:
    case F_Efxi:
    case F_Efeta:
    case F_Efzeta:
    case F_Uplus:
        return 1;
    case F_Exi:
    case F_Eeta:
    case F_Ezeta:
    case F_Bcell:
    case F_Bind:
    case F_Jxi:
    case F_Jeta:
    case F_Jzeta:
    case F_Jcell:
    case F_Eresxi:
    case F_Ereseta:
    case F_Ereszeta:
        return 0;
    default:
        return 1 << 20;
    }
}

static bool hot_point(const mhd_ctx *ctx, const PoolDecoder &dec, uint64_t off)
{
    int f, b, i, j, k;
    if (!dec.decode(off, f, b, i, j, k))
        return true;
    const int d = hot_depth(ctx, f);
    const BlockView &v = ctx->hbv[size_t(b)];
    int pl[3];
    loc_plus(kFields[f].loc, pl[0], pl[1], pl[2]);
    return i >= -d && j >= -d && k >= -d && i < v.ni + pl[0] + d && j < v.nj + pl[1] + d && k < v.nk + pl[2] + d;
}

// Hot and cold lists of a Pole context's group.  Its Sync runs the rings,
// the copies, the wall handlers, the post-wall copies, then the fixed values;
// a step runs the hot part and read-out the cold part (copies, then fixed
// values).  A copy may wait for read-out only when its destination is read
// by no kernel of the step (not a hot point) and its source holds at read-out
// what it held when the copies ran: not a point the wall handlers, the
// post-wall copies or the fixed values of the same Sync write, and not in a
// group whose sources a later Pole repair rewrites (Bface: the B_zeta rewrite
// of the derived-field pass); nor may the wall handlers or the post-wall
// copies overwrite its destination.  A fixed value is hot at a hot point or at the
// destination of a hot copy (it overwrites the copy), cold otherwise.
static int build_sync_pole(mhd_ctx *ctx, const std::string &group, SyncMap &m, const PoolDecoder &dec)
{
    std::vector<uint64_t> d, s2, cd, dc, sc, cdc;
    std::vector<double> cv, cvc;
    const bool all_hot = (group == "Bface");
    std::unordered_set<uint64_t> later(m.hcd.begin(), m.hcd.end());
    later.insert(m.hd2.begin(), m.hd2.end());
    // points the wall handlers write: the boundary cell layer and the ghost
    // layers beyond it on the wall's face
    auto wall_point = [&](uint64_t off) {
        int f, b, i, j, k;
        if (m.walls.empty() || !dec.decode(off, f, b, i, j, k))
            return false;
        for (const auto &w : m.walls)
        {
            if (w.first != b)
                continue;
            const BlockView &v = ctx->hbv[size_t(b)];
            const int ax = std::abs(w.second) - 1;
            const int p[3] = {i, j, k}, n[3] = {v.ni, v.nj, v.nk};
            if ((w.second < 0 && p[ax] <= 0) || (w.second > 0 && p[ax] >= n[ax] - 1))
                return true;
        }
        return false;
    };
    std::unordered_set<uint64_t> hot_dst, post_dst(m.hd2.begin(), m.hd2.end());
    for (size_t t = 0; t < m.hd.size(); ++t)
    {
        // a copy the wall handlers or the post-wall copies overwrite in the
        // same Sync must run before them, in the step
        const bool hot = all_hot || hot_point(ctx, dec, m.hd[t]) || later.count(m.hs[t]) || wall_point(m.hs[t]) ||
                         wall_point(m.hd[t]) || post_dst.count(m.hd[t]);
        (hot ? d : dc).push_back(m.hd[t]);
        (hot ? s2 : sc).push_back(m.hs[t]);
        if (hot)
            hot_dst.insert(m.hd[t]);
    }
    for (size_t t = 0; t < m.hcd.size(); ++t)
    {
        const bool hot = all_hot || hot_point(ctx, dec, m.hcd[t]) || hot_dst.count(m.hcd[t]);
        (hot ? cd : cdc).push_back(m.hcd[t]);
        (hot ? cv : cvc).push_back(m.hcv[t]);
    }
    RUN(upload_list(ctx, m.hot, cd, cv, d, s2, m.staged));
    RUN(upload_list(ctx, m.cold, cdc, cvc, dc, sc, m.staged));
    int f, b, i, j, k;
    for (const auto *tab : {&m.hd, &m.hcd})
        for (uint64_t off : *tab)
            if (dec.decode(off, f, b, i, j, k))
                ctx->field_group[size_t(f)] = group;
    m.built = true;
    return MHD_OK;
}

// device lists of a group from its host tables: the full lists, and the hot
// ones (copies to hot points; fixed values at hot points or at sources of
// hot copies)
int build_sync(mhd_ctx *ctx, const std::string &group, SyncMap &m)
{
    RUN(upload_list(ctx, m.full, m.hcd, m.hcv, m.hd, m.hs, m.staged));
    RUN(upload_list(ctx, m.post, {}, {}, m.hd2, m.hs2, false));
    cudaFree(m.dwalls);
    m.dwalls = nullptr;
    m.wall_cols = 0;
    std::vector<int> wv;
    for (const auto &w : m.walls)
    {
        const BlockView &v = ctx->hbv[size_t(w.first)];
        const int ax = std::abs(w.second) - 1;
        const int64_t ncol = (ax == 0) ? int64_t(v.nj) * v.nk : (ax == 1) ? int64_t(v.ni) * v.nk : int64_t(v.ni) * v.nj;
        m.wall_cols = std::max(m.wall_cols, ncol);
        wv.push_back(w.first);
        wv.push_back(w.second);
    }
    RUN(upload_vec(ctx, wv, &m.dwalls));
    const PoolDecoder dec(ctx);
    std::vector<uint64_t> d, s2, cd;
    std::vector<double> cv;
    if (!ctx->poles.empty())
        return build_sync_pole(ctx, group, m, dec);
    for (size_t t = 0; t < m.hd.size(); ++t)
        if (hot_point(ctx, dec, m.hd[t]))
        {
            d.push_back(m.hd[t]);
            s2.push_back(m.hs[t]);
        }
    std::unordered_set<uint64_t> srcs(s2.begin(), s2.end());
    for (size_t t = 0; t < m.hcd.size(); ++t)
        if (hot_point(ctx, dec, m.hcd[t]) || srcs.count(m.hcd[t]))
        {
            cd.push_back(m.hcd[t]);
            cv.push_back(m.hcv[t]);
        }
    RUN(upload_list(ctx, m.hot, cd, cv, d, s2, m.staged));
    int f, b, i, j, k;
    for (const auto *tab : {&m.hd, &m.hcd})
        for (uint64_t off : *tab)
            if (dec.decode(off, f, b, i, j, k))
                ctx->field_group[size_t(f)] = group;
    m.built = true;
    return MHD_OK;
}

static int build_all_syncs(mhd_ctx *ctx)
{
    for (auto &kv : ctx->syncs)
        if (!kv.second.built)
            RUN(build_sync(ctx, kv.first, kv.second));
    return MHD_OK;
}

// read-out of fields whose last sync ran its hot list only
// cold copies then cold fixed values of a Pole context's group (the order
// of the full Sync: its fixed values come last)
static int run_cold(mhd_ctx *ctx, const std::string &group)
{
    auto it = ctx->syncs.find(group);
    if (it == ctx->syncs.end())
        return MHD_OK;
    const CopyList &c = it->second.cold;
    RUN(gather_map(ctx, c));
    if (c.nconst > 0)
    {
        prof_begin(ctx, "k_set_consts");
        k_set_consts<<<grid_for(c.nconst), kThreads, 0, ctx->stream>>>(ctx->pool, c.cdst, c.cval, c.nconst);
        RUN(launched(ctx));
    }
    ctx->dirty[group] = false;
    return MHD_OK;
}

static int materialise_group(mhd_ctx *ctx, const std::string &group)
{
    auto it = ctx->dirty.find(group);
    if (it == ctx->dirty.end() || !it->second)
        return MHD_OK;
    if (!ctx->poles.empty())
        return run_cold(ctx, group);
    return run_sync(ctx, group.c_str(), true);
}

static int materialise_pv(mhd_ctx *ctx)
{
    const bool up = ctx->dirty.count("Uplus") && ctx->dirty["Uplus"];
    if (!ctx->pv_dirty && !up)
        return MHD_OK;
    RUN(materialise_group(ctx, "Ucell"));
    RUN(ensure_geom(ctx));
    prof_begin(ctx, "k_pv_uplus_dt");
    launch_k_pv_uplus_dt(ctx->tune[TUNE_k_pv_uplus_dt], false, dim3(grid_for(max_box(ctx, LOC_CELL, ctx->G)), ctx->nblocks),
                         ctx->stream, ctx->dbv, ctx->c, nullptr, ctx->G, 0);
    RUN(launched(ctx));
    RUN(run_sync(ctx, "Uplus", true));
    ctx->pv_dirty = false;
    return MHD_OK;
}

static int materialise_field(mhd_ctx *ctx, int f)
{
    if (f == F_PV || f == F_Uplus)
        return materialise_pv(ctx);
    if (!ctx->field_group[size_t(f)].empty())
        return materialise_group(ctx, ctx->field_group[size_t(f)]);
    return MHD_OK;
}

static int materialise_all(mhd_ctx *ctx)
{
    RUN(materialise_pv(ctx));
    std::vector<std::string> dirty;
    for (auto &kv : ctx->dirty)
        if (kv.second)
            dirty.push_back(kv.first);
    for (const auto &g : dirty)
        RUN(materialise_group(ctx, g));
    return MHD_OK;
}

// after graph replays: every group ran its hot list
static void mark_dirty(mhd_ctx *ctx)
{
    // a context with Poles leaves its cold lists (copies whose sources the
    // step no longer changes) for read-out; the whole Sync is not run again
    // there (it is not idempotent: the ring averages need not reproduce a
    // ring, and the Pole repairs change sources after their syncs)
    for (auto &kv : ctx->syncs)
        if (kv.second.built)
            ctx->dirty[kv.first] = ctx->poles.empty() ? (kv.second.hot.n != kv.second.full.n ||
                                                         kv.second.hot.nconst != kv.second.full.nconst)
                                                      : (kv.second.cold.n > 0 || kv.second.cold.nconst > 0);
    ctx->pv_dirty = true;
}

// The region of the resistive operator.  Eres can be non-zero only at the
// unknown and alias edges and at their images under the Eres1form copies
// (closed point by point).  dB can be non-zero only on faces next to those
// edges (their bounding box widened by one point) and at the images of those
// faces under the dB copies.  The region of block b is the bounding box of
// all these points widened by one more point for the curl-adjoint stencil.
// Builds the per (block, axis) face and edge sub-ranges and the copy lists
// restricted to destinations inside the region.
static int resistive_region(mhd_ctx *ctx, const std::vector<uint64_t> &seed)
{
    auto &R = ctx->res;
    const int nb = ctx->nblocks;
    const PoolDecoder dec(ctx);
    std::vector<uint64_t> md[2], ms[2];
    bool staged[2];
    host_map(ctx, "Eres1form", md[0], ms[0], staged[0]);
    host_map(ctx, "dB", md[1], ms[1], staged[1]);
    int b, i, j, k;
    // Eres: exact closure of the seed under the Eres1form copies
    std::unordered_set<uint64_t> enz(seed.begin(), seed.end());
    for (int iter = 0; iter < 64; ++iter)
    {
        bool changed = false;
        for (size_t t = 0; t < md[0].size(); ++t)
            if (enz.count(ms[0][t]) && enz.insert(md[0][t]).second)
                changed = true;
        if (!changed)
            break;
    }
    std::vector<IBox> ebox(static_cast<size_t>(nb)), box(static_cast<size_t>(nb));
    for (uint64_t off : enz)
    {
        if (!dec(off, b, i, j, k))
            return fail(ctx, MHD_EINVAL, "resistive point outside the pool");
        ebox[size_t(b)].add(i, j, k);
        box[size_t(b)].add(i, j, k);
    }
    // dB: faces within one point of the Eres box, closed under the dB copies
    std::unordered_set<uint64_t> fnz;
    for (int iter = 0; iter < 64; ++iter)
    {
        bool changed = false;
        for (size_t t = 0; t < md[1].size(); ++t)
        {
            const uint64_t src = ms[1][t];
            const bool live = fnz.count(src) || (dec(src, b, i, j, k) && ebox[size_t(b)].has(i, j, k, 1));
            if (live && fnz.insert(md[1][t]).second)
                changed = true;
        }
        if (!changed)
            break;
    }
    for (uint64_t off : fnz)
        if (dec(off, b, i, j, k))
            box[size_t(b)].add(i, j, k);
    for (int q = 0; q < nb; ++q)
    {
        IBox &x = box[size_t(q)];
        if (x.empty())
            continue;
        const BlockView &v = ctx->hbv[size_t(q)];
        const int n[3] = {v.ni, v.nj, v.nk};
        for (int a = 0; a < 3; ++a)
        {
            x.lo[a] = std::max(x.lo[a] - 2, -v.G);
            x.hi[a] = std::min(x.hi[a] + 2, n[a] + 1 + v.G);
        }
    }
    // per block: the region box within the staggered points [0, n + 1)^3
    std::vector<int> rg(size_t(nb) * 6, 0);
    R.nreg_max = 0;
    for (int q = 0; q < nb; ++q)
    {
        const BlockView &v = ctx->hbv[size_t(q)];
        const int n[3] = {v.ni, v.nj, v.nk};
        int64_t cnt = 1;
        for (int d = 0; d < 3; ++d)
        {
            const int lo = box[size_t(q)].empty() ? 0 : std::max(0, box[size_t(q)].lo[d]);
            const int hi = box[size_t(q)].empty() ? 0 : std::min(n[d] + 1, box[size_t(q)].hi[d]);
            rg[size_t(q) * 6 + d] = lo;
            rg[size_t(q) * 6 + 3 + d] = std::max(lo, hi);
            cnt *= std::max(0, hi - lo);
        }
        R.nreg_max = std::max(R.nreg_max, cnt);
    }
    RUN(upload_vec(ctx, rg, &R.rng));
    // copies with a destination inside the region
    CopyList *out[2] = {&R.eres1form, &R.db};
    const char *names[2] = {"Eres1form", "dB"};
    for (int q = 0; q < 2; ++q)
    {
        std::vector<uint64_t> d, s2, cd;
        std::vector<double> cv;
        for (size_t t = 0; t < md[q].size(); ++t)
            if (dec(md[q][t], b, i, j, k) && box[size_t(b)].has(i, j, k))
            {
                d.push_back(md[q][t]);
                s2.push_back(ms[q][t]);
            }
        auto it = ctx->syncs.find(names[q]);
        if (it != ctx->syncs.end())
            for (size_t t = 0; t < it->second.hcd.size(); ++t)
                if (dec(it->second.hcd[t], b, i, j, k) && box[size_t(b)].has(i, j, k))
                {
                    cd.push_back(it->second.hcd[t]);
                    cv.push_back(it->second.hcv[t]);
                }
        RUN(upload_list(ctx, *out[q], cd, cv, d, s2, staged[q]));
    }
    return MHD_OK;
}

// The persistent solve's operator in fewer grid-wide phases.  Phase A: the
// unknowns, their aliases, Sync("Eres1form")'s fixed values and copies,
// written in that order by the reference, become one list with a single
// writer per point, each copy taking the expression of the value its source
// holds after the writes before it.  Phase B: Sync("dB")'s copies are
// written with the curl, each destination computing the curl at its source,
// when no copy lands on a point the curl or a fixed value writes.  Neither
// fusion applies when a copy's source is another copy's destination (the
// chained case keeps the staged copy lists).  The values are the same bits
// as the phase-by-phase operator's.
static int build_fused_operator(mhd_ctx *ctx, const std::vector<uint64_t> &he, const std::vector<uint64_t> &ae,
                                const std::vector<int64_t> &aidx, const std::vector<double> &asign)
{
    auto &R = ctx->res;
    R.fa.n = R.fb.n = -1;
    struct E
    {
        int kind;
        int64_t idx;
        double val;
        int blk;
    };
    auto fetch = [&](const CopyList &l, std::vector<uint64_t> &d, std::vector<uint64_t> &sr, std::vector<uint64_t> &cd,
                     std::vector<double> &cv) -> int {
        d.resize(size_t(l.n));
        sr.resize(size_t(l.n));
        cd.resize(size_t(l.nconst));
        cv.resize(size_t(l.nconst));
        if (l.n > 0)
        {
            CK(ctx, cudaMemcpy(d.data(), l.dst, size_t(l.n) * 8, cudaMemcpyDeviceToHost));
            CK(ctx, cudaMemcpy(sr.data(), l.src, size_t(l.n) * 8, cudaMemcpyDeviceToHost));
        }
        if (l.nconst > 0)
        {
            CK(ctx, cudaMemcpy(cd.data(), l.cdst, size_t(l.nconst) * 8, cudaMemcpyDeviceToHost));
            CK(ctx, cudaMemcpy(cv.data(), l.cval, size_t(l.nconst) * 8, cudaMemcpyDeviceToHost));
        }
        return MHD_OK;
    };
    auto chained = [](const std::vector<uint64_t> &d, const std::vector<uint64_t> &sr) {
        std::unordered_set<uint64_t> ds(d.begin(), d.end());
        for (uint64_t x : sr)
            if (ds.count(x))
                return true;
        return false;
    };
    auto upload = [&](mhd_ctx::Resistive::Fused &out, const std::vector<uint64_t> &order,
                      const std::map<uint64_t, E> &m) -> int {
        std::vector<uint64_t> d;
        std::vector<int> kd, bl;
        std::vector<int64_t> ix;
        std::vector<double> vl;
        for (uint64_t o : order)
        {
            const E &e = m.at(o);
            d.push_back(o);
            kd.push_back(e.kind);
            ix.push_back(e.idx);
            vl.push_back(e.val);
            bl.push_back(e.blk);
        }
        RUN(upload_vec(ctx, d, &out.dst));
        RUN(upload_vec(ctx, kd, &out.kind));
        RUN(upload_vec(ctx, ix, &out.idx));
        RUN(upload_vec(ctx, vl, &out.val));
        RUN(upload_vec(ctx, bl, &out.blk));
        out.n = int64_t(order.size());
        return MHD_OK;
    };
    std::vector<uint64_t> d1, s1, cd1, d2, s2, cd2;
    std::vector<double> cv1, cv2;
    RUN(fetch(R.eres1form, d1, s1, cd1, cv1));
    RUN(fetch(R.db, d2, s2, cd2, cv2));
    // phase A
    if (!chained(d1, s1))
    {
        std::map<uint64_t, E> m;
        std::vector<uint64_t> order;
        auto put = [&](uint64_t dst, const E &e) {
            auto it = m.find(dst);
            if (it == m.end())
            {
                m.emplace(dst, e);
                order.push_back(dst);
            }
            else
                it->second = e;
        };
        for (size_t t = 0; t < he.size(); ++t)
            put(he[t], E{FUSE_UNKNOWN, int64_t(t), 0.0, 0});
        for (size_t q = 0; q < ae.size(); ++q)
            put(ae[q], E{FUSE_ALIAS, aidx[q], asign[q], 0});
        for (size_t c = 0; c < cd1.size(); ++c)
            put(cd1[c], E{FUSE_CONST, 0, cv1[c], 0});
        std::vector<std::pair<uint64_t, E>> cps;
        for (size_t c = 0; c < d1.size(); ++c)
        {
            auto it = m.find(s1[c]);
            cps.push_back({d1[c], it != m.end() ? it->second : E{FUSE_POOL, int64_t(s1[c]), 0.0, 0}});
        }
        for (const auto &pr : cps)
            put(pr.first, pr.second);
        RUN(upload(R.fa, order, m));
    }
    // phase B
    if (R.merge2 && !chained(d2, s2))
    {
        std::vector<int> rg(size_t(ctx->nblocks) * 6);
        CK(ctx, cudaMemcpy(rg.data(), R.rng, rg.size() * sizeof(int), cudaMemcpyDeviceToHost));
        const PoolDecoder dec(ctx);
        // is the dB point `off` a face the curl writes (inner face in the region)?
        auto curl_face = [&](uint64_t off, int &b, int &fa, int &i, int &j, int &k) {
            int f;
            if (!dec.decode(off, f, b, i, j, k) || f < F_dBxi || f > F_dBxi + 2)
                return false;
            fa = f - F_dBxi;
            const BlockView &v = ctx->hbv[size_t(b)];
            const int *r = rg.data() + 6 * b;
            const int p[3] = {i, j, k};
            for (int a = 0; a < 3; ++a)
                if (p[a] < r[a] || p[a] >= r[3 + a])
                    return false;
            return i >= 0 && j >= 0 && k >= 0 && i < v.ni + (fa == 0) && j < v.nj + (fa == 1) && k < v.nk + (fa == 2);
        };
        std::unordered_set<uint64_t> consts(cd2.begin(), cd2.end());
        std::map<uint64_t, E> m;
        std::vector<uint64_t> order;
        bool ok = true;
        int b, fa, i, j, k;
        for (size_t c = 0; c < d2.size() && ok; ++c)
        {
            if (consts.count(d2[c]) || curl_face(d2[c], b, fa, i, j, k) || m.count(d2[c]))
            {
                ok = false; // a copy onto a written point: keep the phase-by-phase operator
                break;
            }
            E e{FUSE_POOL, int64_t(s2[c]), 0.0, 0};
            if (consts.count(s2[c]))
            {
                for (size_t q = 0; q < cd2.size(); ++q)
                    if (cd2[q] == s2[c])
                        e = E{FUSE_CONST, 0, cv2[q], 0};
            }
            else if (curl_face(s2[c], b, fa, i, j, k))
                e = E{FUSE_CURL, fuse_pack(fa, i, j, k), 0.0, b};
            m.emplace(d2[c], e);
            order.push_back(d2[c]);
        }
        if (ok)
            RUN(upload(R.fb, order, m));
    }
    return MHD_OK;
}

extern "C" {

int mhd_set_sync_map(mhd_ctx *ctx, const char *group, const int64_t *dst, const int64_t *src, int64_t n)
{
    BIND_DEVICE(ctx);
    if (!ctx || !group || n < 0 || (n > 0 && (!dst || !src)))
        return fail(ctx, MHD_EINVAL, "bad sync map arguments");
    std::vector<uint64_t> d(static_cast<size_t>(n)), s(static_cast<size_t>(n));
    for (int64_t t = 0; t < n; ++t)
    {
        const int64_t od = pool_offset(ctx, dst[t]);
        const int64_t os = pool_offset(ctx, src[t]);
        if (od < 0 || os < 0)
            return fail(ctx, MHD_EINVAL, "sync map entry %lld has an invalid point id", (long long)t);
        d[size_t(t)] = uint64_t(od);
        s[size_t(t)] = uint64_t(os);
    }
    // staged (gather, then scatter) when a source is also a destination
    std::vector<uint64_t> sorted_d(d);
    std::sort(sorted_d.begin(), sorted_d.end());
    bool staged = false;
    for (int64_t t = 0; t < n && !staged; ++t)
        staged = std::binary_search(sorted_d.begin(), sorted_d.end(), s[size_t(t)]);
    SyncMap &m = ctx->syncs[group];
    m.hd.swap(d);
    m.hs.swap(s);
    m.staged = staged;
    m.built = false;
    drop_graph(ctx);
    // the resistive operator's region depends on these two groups
    if (ctx->res.on && (std::strcmp(group, "Eres1form") == 0 || std::strcmp(group, "dB") == 0))
    {
        cudaFree(ctx->res.rng);
        ctx->res.rng = nullptr;
        RUN(resistive_region(ctx, ctx->res.seed));
    }
    return MHD_OK;
}

int mhd_set_sync_consts(mhd_ctx *ctx, const char *group, const int64_t *dst, const double *val, int64_t n)
{
    BIND_DEVICE(ctx);
    if (!ctx || !group || n < 0 || (n > 0 && (!dst || !val)))
        return fail(ctx, MHD_EINVAL, "bad sync constant arguments");
    std::vector<uint64_t> d(static_cast<size_t>(n));
    for (int64_t t = 0; t < n; ++t)
    {
        const int64_t od = pool_offset(ctx, dst[t]);
        if (od < 0)
            return fail(ctx, MHD_EINVAL, "sync constant %lld has an invalid point id", (long long)t);
        d[size_t(t)] = uint64_t(od);
    }
    SyncMap &m = ctx->syncs[group];
    m.hcd.swap(d);
    m.hcv.assign(val, val + n);
    m.built = false;
    drop_graph(ctx);
    if (ctx->res.on && (std::strcmp(group, "Eres1form") == 0 || std::strcmp(group, "dB") == 0))
    {
        cudaFree(ctx->res.rng);
        ctx->res.rng = nullptr;
        RUN(resistive_region(ctx, ctx->res.seed));
    }
    return MHD_OK;
}

int mhd_set_sync_map_post(mhd_ctx *ctx, const char *group, const int64_t *dst, const int64_t *src, int64_t n)
{
    BIND_DEVICE(ctx);
    if (!ctx || !group || n < 0 || (n > 0 && (!dst || !src)))
        return fail(ctx, MHD_EINVAL, "bad sync map arguments");
    std::vector<uint64_t> d(static_cast<size_t>(n)), s(static_cast<size_t>(n));
    for (int64_t t = 0; t < n; ++t)
    {
        const int64_t od = pool_offset(ctx, dst[t]);
        const int64_t os = pool_offset(ctx, src[t]);
        if (od < 0 || os < 0)
            return fail(ctx, MHD_EINVAL, "sync map entry %lld has an invalid point id", (long long)t);
        d[size_t(t)] = uint64_t(od);
        s[size_t(t)] = uint64_t(os);
    }
    // one gather: no source may be a destination
    std::vector<uint64_t> sorted_d(d);
    std::sort(sorted_d.begin(), sorted_d.end());
    for (int64_t t = 0; t < n; ++t)
        if (std::binary_search(sorted_d.begin(), sorted_d.end(), s[size_t(t)]))
            return fail(ctx, MHD_EINVAL, "post-wall copy %lld reads a point the same list writes", (long long)t);
    SyncMap &m = ctx->syncs[group];
    m.hd2.swap(d);
    m.hs2.swap(s);
    m.built = false;
    drop_graph(ctx);
    return MHD_OK;
}

int mhd_build_geometry(mhd_ctx *ctx, int32_t block, const double *nodes, int64_t count, const double *B_imf)
{
    BIND_DEVICE(ctx);
    if (!ctx || block < 0 || block >= ctx->nblocks || !nodes)
        return fail(ctx, MHD_EINVAL, "bad geometry arguments");
    if (ctx->capturing)
        return fail(ctx, MHD_ESTATE, "geometry changed during capture");
    const BlockView &v = ctx->hbv[size_t(block)];
    const int off = ctx->G + 1;
    NodeMesh m{nullptr, off, v.nj + 1 + 2 * off, v.nk + 1 + 2 * off};
    const int64_t want = int64_t(v.ni + 1 + 2 * off) * m.NJ * m.NK * 3;
    if (count != want)
        return fail(ctx, MHD_EINVAL, "node mesh of block %d: %lld values, expected %lld", block, (long long)count,
                    (long long)want);
    RUN(ensure_staging(ctx, size_t(count)));
    CK(ctx, cudaMemcpyAsync(ctx->staging, nodes, size_t(count) * 8, cudaMemcpyHostToDevice, ctx->stream));
    m.a = ctx->staging;
    prof_begin(ctx, "k_geometry");
    k_geometry<<<dim3(grid_for(v.vol), GEOM_BADD), kThreads, 0, ctx->stream>>>(ctx->dbv, block, m, ctx->G, 0, 0.0,
                                                                                  0.0, 0.0);
    RUN(launched(ctx));
    if (B_imf && (B_imf[0] != 0.0 || B_imf[1] != 0.0 || B_imf[2] != 0.0))
    {
        prof_begin(ctx, "k_geometry");
        k_geometry<<<dim3(grid_for(v.vol), 1), kThreads, 0, ctx->stream>>>(ctx->dbv, block, m, ctx->G, GEOM_BADD,
                                                                             B_imf[0], B_imf[1], B_imf[2]);
        RUN(launched(ctx));
    }
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    ctx->geom_dirty = true;
    drop_graph(ctx);
    return MHD_OK;
}

int mhd_diagnostics(mhd_ctx *ctx, int32_t run, double *mins, double *maxs)
{
    BIND_DEVICE(ctx);
    if (!ctx || !mins || !maxs || run >= ctx->nruns)
        return fail(ctx, MHD_EINVAL, "bad diagnostics arguments");
    if (ctx->capturing)
        return fail(ctx, MHD_ESTATE, "diagnostics during capture");
    if (!ctx->diag_keys)
        CK(ctx, cudaMalloc(&ctx->diag_keys, (DIAG_NMIN + DIAG_NQ) * sizeof(unsigned long long)));
    RUN(materialise_field(ctx, F_PV)); // the pressure of PV_H
    prof_begin(ctx, "k_diag_init");
    k_diag_init<<<1, 32, 0, ctx->stream>>>(ctx->diag_keys);
    RUN(launched(ctx));
    prof_begin(ctx, "k_diag");
    k_diag<<<dim3(grid_for(ctx->max_cells), unsigned(ctx->nblocks)), kThreads, 0, ctx->stream>>>(ctx->dbv, run,
                                                                                                 ctx->diag_keys);
    RUN(launched(ctx));
    unsigned long long keys[DIAG_NMIN + DIAG_NQ];
    CK(ctx, cudaMemcpyAsync(keys, ctx->diag_keys, sizeof keys, cudaMemcpyDeviceToHost, ctx->stream));
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    for (int q = 0; q < DIAG_NMIN; ++q)
        mins[q] = diag_unkey(keys[q]);
    for (int q = 0; q < DIAG_NQ; ++q)
        maxs[q] = diag_unkey(keys[DIAG_NMIN + q]);
    return MHD_OK;
}

int mhd_set_pole(mhd_ctx *ctx, int32_t block, int32_t direction)
{
    BIND_DEVICE(ctx);
    if (!ctx || block < 0 || block >= ctx->nblocks || (direction != -2 && direction != 2))
        return fail(ctx, MHD_EINVAL, "bad Pole arguments (eta Poles: direction -2 or +2)");
    const BlockView &v = ctx->hbv[size_t(block)];
    if (v.nj < 2)
        return fail(ctx, MHD_EINVAL, "a block with Poles needs at least two cells in j");
    if (ctx->res.on || ctx->hall.n > 0)
        return fail(ctx, MHD_ESTATE, "Poles are not available with the implicit resistive or Hall solves");
    for (size_t q = 0; q < ctx->poles.size(); q += 2)
        if (ctx->poles[q] == block && ctx->poles[q + 1] == direction)
            return MHD_OK;
    ctx->poles.push_back(block);
    ctx->poles.push_back(direction);
    cudaFree(ctx->dpoles);
    ctx->dpoles = nullptr;
    RUN(upload_vec(ctx, ctx->poles, &ctx->dpoles));
    for (auto &kv : ctx->syncs)
        kv.second.built = false;
    ctx->geom_dirty = true; // the rings' normal matrices
    drop_graph(ctx);
    return MHD_OK;
}

int mhd_set_sync_wall(mhd_ctx *ctx, const char *group, int32_t block, int32_t direction)
{
    BIND_DEVICE(ctx);
    if (!ctx || !group || block < 0 || block >= ctx->nblocks || direction == 0 || direction < -3 || direction > 3)
        return fail(ctx, MHD_EINVAL, "bad wall handler arguments");
    ctx->syncs[group].walls.emplace_back(block, direction);
    drop_graph(ctx);
    return MHD_OK;
}

int mhd_set_resistive(mhd_ctx *ctx, int64_t n, const int64_t *unknowns, const double *eta, int64_t nalias,
                      const int64_t *alias, const int64_t *owner, const double *sign, double rtol, double atol,
                      int32_t maxit, int32_t restart)
{
    BIND_DEVICE(ctx);
    if (!ctx || n < 0 || nalias < 0 || (n > 0 && (!unknowns || !eta)) || (nalias > 0 && (!alias || !owner || !sign)))
        return fail(ctx, MHD_EINVAL, "bad resistive arguments");
    if (ctx->nruns > 1 && n > 0)
        return fail(ctx, MHD_ESTATE, "the implicit resistive solve is not available in a batch of runs (one shared dt per solve)");
    if (!ctx->poles.empty() && n > 0)
        return fail(ctx, MHD_ESTATE, "the implicit resistive solve is not available with Poles");
    if (restart <= 0 || restart > kMaxRestart)
        return fail(ctx, MHD_EINVAL, "GMRES restart must be in [1, %d]", kMaxRestart);
    if (maxit < 0)
        return fail(ctx, MHD_EINVAL, "negative iteration limit");
    auto &R = ctx->res;
    free_resistive(ctx);
    drop_graph(ctx);
    // Eres point ids -> pool offsets in Eres, dJ and J (same locations, same boxes)
    auto remap = [&](const int64_t *ids, int64_t cnt, int to0, std::vector<uint64_t> &out) -> int {
        out.resize(size_t(cnt));
        for (int64_t t = 0; t < cnt; ++t)
        {
            const int f = int(ids[t] >> 56);
            if (f < F_Eresxi || f > F_Eresxi + 2)
                return fail(ctx, MHD_EINVAL, "resistive point %lld is not an Eres point", (long long)t);
            const int64_t id = (int64_t(to0 + (f - F_Eresxi)) << 56) | (ids[t] & ((int64_t(1) << 56) - 1));
            const int64_t o = pool_offset(ctx, id);
            if (o < 0)
                return fail(ctx, MHD_EINVAL, "resistive point %lld is outside its field", (long long)t);
            out[size_t(t)] = uint64_t(o);
        }
        return MHD_OK;
    };
    std::vector<uint64_t> he, hdj, hj, ae, oe;
    RUN(remap(unknowns, n, F_Eresxi, he));
    RUN(remap(unknowns, n, F_dJxi, hdj));
    RUN(remap(unknowns, n, F_Jxi, hj));
    RUN(remap(alias, nalias, F_Eresxi, ae));
    RUN(remap(owner, nalias, F_Eresxi, oe));
    // only aliases of unknown owners can be non-zero
    std::vector<uint64_t> sorted_e(he);
    std::sort(sorted_e.begin(), sorted_e.end());
    std::vector<uint64_t> fa, fo;
    std::vector<double> fs;
    std::vector<int64_t> fidx; // unknown index of the owner
    std::map<uint64_t, int64_t> index_of;
    for (int64_t t = 0; t < n; ++t)
        index_of[he[size_t(t)]] = t;
    for (int64_t t = 0; t < nalias; ++t)
        if (std::binary_search(sorted_e.begin(), sorted_e.end(), oe[size_t(t)]))
        {
            fa.push_back(ae[size_t(t)]);
            fo.push_back(oe[size_t(t)]);
            fs.push_back(sign[t]);
            fidx.push_back(index_of[oe[size_t(t)]]);
        }
    RUN(upload_vec(ctx, he, &R.e));
    RUN(upload_vec(ctx, hdj, &R.dj));
    RUN(upload_vec(ctx, hj, &R.j));
    RUN(upload_vec(ctx, fa, &R.alias_e));
    RUN(upload_vec(ctx, fo, &R.owner_e));
    RUN(upload_vec(ctx, fs, &R.sign));
    RUN(upload_vec(ctx, fidx, &R.alias_of));
    std::vector<double> heta(eta, eta + n);
    RUN(upload_vec(ctx, heta, &R.eta));
    R.n = n;
    R.nalias = int64_t(fa.size());
    // the operator's active region
    R.seed = he;
    R.seed.insert(R.seed.end(), fa.begin(), fa.end());
    RUN(resistive_region(ctx, R.seed));
    // the persistent solve's phase merges and unknown locations
    {
        PoolDecoder dec(ctx);
        std::vector<int> uloc(size_t(5 * n));
        for (int64_t t = 0; t < n; ++t)
        {
            int f, b, i, j, k;
            if (!dec.decode(he[size_t(t)], f, b, i, j, k))
                return fail(ctx, MHD_EINVAL, "resistive unknown %lld does not decode", (long long)t);
            const int loc[5] = {b, f - F_Eresxi, i, j, k};
            std::copy(loc, loc + 5, uloc.begin() + 5 * t);
        }
        RUN(upload_vec(ctx, uloc, &R.uloc));
        auto fetch = [&](const CopyList &l, std::vector<uint64_t> &h) -> int {
            h.resize(size_t(l.nconst));
            if (l.nconst > 0)
                CK(ctx, cudaMemcpy(h.data(), l.cdst, size_t(l.nconst) * 8, cudaMemcpyDeviceToHost));
            return MHD_OK;
        };
        // Sync("Eres1form")'s fixed values may be written with the unknowns
        // and aliases when they touch none of them
        std::vector<uint64_t> c1, c2;
        RUN(fetch(R.eres1form, c1));
        RUN(fetch(R.db, c2));
        std::vector<uint64_t> written(he);
        written.insert(written.end(), fa.begin(), fa.end());
        std::sort(written.begin(), written.end());
        R.merge1 = 1;
        for (uint64_t o : c1)
            if (std::binary_search(written.begin(), written.end(), o))
                R.merge1 = 0;
        // Sync("dB")'s fixed values may be written with the curl, which
        // writes inner faces only, when none of them is an inner face
        R.merge2 = 1;
        for (uint64_t o : c2)
        {
            int f, b, i, j, k;
            if (!dec.decode(o, f, b, i, j, k))
            {
                R.merge2 = 0;
                continue;
            }
            const BlockView &v = ctx->hbv[size_t(b)];
            const int a = f - F_dBxi;
            if (i >= 0 && j >= 0 && k >= 0 && i < v.ni + (a == 0) && j < v.nj + (a == 1) && k < v.nk + (a == 2))
                R.merge2 = 0;
        }
        RUN(build_fused_operator(ctx, he, fa, fidx, fs));
    }
    // every point of the solve's fields starts at zero
    for (int f0 : {int(F_Eresxi), int(F_dBxi), int(F_dJxi), int(F_RBresxi)})
        for (int f = f0; f < f0 + 3; ++f)
            for (int b = 0; b < ctx->nblocks; ++b)
                CK(ctx, cudaMemset(ctx->pool + ctx->base[size_t(f)][size_t(b)], 0,
                                   size_t(ctx->hbv[size_t(b)].vol) * 8 * size_t(kFields[f].ncomp)));
    R.restart = restart;
    R.rtol = rtol;
    R.atol = atol;
    R.maxit = maxit;
    R.ngroups = int(std::min<int64_t>(std::max<int64_t>((n + 255) / 256, 1), 592));
    const size_t nn = size_t(n > 0 ? n : 1);
    CK(ctx, cudaMalloc(&R.V, nn * size_t(restart + 1) * 8));
    CK(ctx, cudaMalloc(&R.w, nn * 8));
    CK(ctx, cudaMalloc(&R.x, nn * 8));
    CK(ctx, cudaMalloc(&R.b, nn * 8));
    CK(ctx, cudaMalloc(&R.r, nn * 8));
    CK(ctx, cudaMalloc(&R.partial, size_t(R.ngroups) * size_t(restart + 2) * 8));
    CK(ctx, cudaMalloc(&R.dots, 64 * 8));
    CK(ctx, cudaMalloc(&R.st, sizeof(GmresState)));
    CK(ctx, cudaMemset(R.x, 0, nn * 8));
    CK(ctx, cudaMemset(R.st, 0, sizeof(GmresState)));
    // the persistent solve: as many CTAs as the work needs, at most two per
    // SM (more gave no further gain) and no more than can be resident
    // together (cooperative launch)
    {
        int dev = 0, sms = 0, per_sm = 0, coop = 0;
        CK(ctx, cudaGetDevice(&dev));
        CK(ctx, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        CK(ctx, cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
        CK(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_gmres_resist, 256, 0));
        const int64_t work = std::max<int64_t>(n, int64_t(ctx->nblocks) * R.nreg_max);
        const int64_t want = std::max<int64_t>(1, (work + 255) / 256);
        R.pgrid = (coop && per_sm > 0) ? int(std::min<int64_t>(want, int64_t(sms) * std::min(per_sm, 2))) : 0;
        if (R.pgrid > 0)
        {
            CK(ctx, cudaMalloc(&R.ppartial, size_t(2 * 32) * size_t(R.pgrid) * 8));
            CK(ctx, cudaMalloc(&R.bar, 4 * sizeof(unsigned)));
            CK(ctx, cudaMemset(R.bar, 0, 4 * sizeof(unsigned)));
        }
    }
    R.its_eager = R.cycles_eager = 0;
    R.k_cycle = R.k_inner = 0;
    for (auto &sp : ctx->spare)
        if (!sp)
            CK(ctx, cudaStreamCreateWithFlags(&sp, cudaStreamNonBlocking));
    R.on = true;
    return MHD_OK;
}

int mhd_set_hall(mhd_ctx *ctx, double hall_coef, const int32_t *zero_boxes, int32_t nbox)
{
    BIND_DEVICE(ctx);
    if (!ctx || nbox < 0 || (nbox > 0 && !zero_boxes))
        return fail(ctx, MHD_EINVAL, "bad Hall arguments");
    for (int q = 0; q < nbox; ++q)
    {
        const int32_t *z = zero_boxes + 8 * q;
        if (z[0] < 0 || z[0] >= ctx->nblocks || z[1] < 0 || z[1] > 2)
            return fail(ctx, MHD_EINVAL, "Hall zero box %d: bad block or axis", q);
    }
    cudaFree(ctx->hall_zb);
    ctx->hall_zb = nullptr;
    ctx->hall_nzb = 0;
    if (nbox > 0)
    {
        CK(ctx, cudaMalloc(&ctx->hall_zb, size_t(nbox) * 8 * sizeof(int)));
        CK(ctx, cudaMemcpy(ctx->hall_zb, zero_boxes, size_t(nbox) * 8 * sizeof(int), cudaMemcpyHostToDevice));
    }
    ctx->hall_nzb = nbox;
    ctx->hall_coef = hall_coef;
    return MHD_OK;
}

int mhd_set_hall_implicit(mhd_ctx *ctx, int64_t n, const int64_t *unknowns, int64_t nalias, const int64_t *alias,
                          const int64_t *owner, const double *sign, double rtol, double atol, int32_t maxit,
                          double ksp_rtol, int32_t ksp_maxit)
{
    BIND_DEVICE(ctx);
    if (!ctx || n < 0 || nalias < 0 || maxit < 0 || ksp_maxit < 1 || (n > 0 && !unknowns) ||
        (nalias > 0 && (!alias || !owner || !sign)))
        return fail(ctx, MHD_EINVAL, "bad implicit Hall arguments");
    if (n > 0 && ctx->integrator != MHD_INTEGRATOR_EULER)
        return fail(ctx, MHD_ESTATE, "the implicit Hall solve runs with the Euler integrator only");
    if (ctx->nruns > 1 && n > 0)
        return fail(ctx, MHD_ESTATE, "the implicit Hall solve is not available in a batch of runs (one shared dt per solve)");
    if (!ctx->poles.empty() && n > 0)
        return fail(ctx, MHD_ESTATE, "the implicit Hall solve is not available with Poles");
    auto &H = ctx->hall;
    for (void *p : {(void *)H.e, (void *)H.alias, (void *)H.owner, (void *)H.sign, (void *)H.bstar, (void *)H.X,
                    (void *)H.F, (void *)H.Xt, (void *)H.Ft, (void *)H.dx, (void *)H.b, (void *)H.r, (void *)H.V,
                    (void *)H.w, (void *)H.partial, (void *)H.dots, (void *)H.st, (void *)H.ctl, (void *)H.done,
                    (void *)H.seg_snap, (void *)H.seg_restore, (void *)H.bs})
        cudaFree(p);
    H = mhd_ctx::HallImplicit();
    drop_graph(ctx);
    if (n == 0)
        return MHD_OK;
    auto remap = [&](const int64_t *ids, int64_t cnt, std::vector<uint64_t> &out) -> int {
        out.resize(size_t(cnt));
        for (int64_t t = 0; t < cnt; ++t)
        {
            const int f = int(ids[t] >> 56);
            const int64_t o = pool_offset(ctx, ids[t]);
            if (f < F_Ehxi || f > F_Ehxi + 2 || o < 0)
                return fail(ctx, MHD_EINVAL, "implicit Hall point %lld is not an Ehall point", (long long)t);
            out[size_t(t)] = uint64_t(o);
        }
        return MHD_OK;
    };
    std::vector<uint64_t> he, ha, ho;
    RUN(remap(unknowns, n, he));
    RUN(remap(alias, nalias, ha));
    RUN(remap(owner, nalias, ho));
    RUN(upload_vec(ctx, he, &H.e));
    RUN(upload_vec(ctx, ha, &H.alias));
    RUN(upload_vec(ctx, ho, &H.owner));
    std::vector<double> hs(sign, sign + nalias);
    RUN(upload_vec(ctx, hs, &H.sign));
    H.n = n;
    H.nalias = nalias;
    H.rtol = rtol;
    H.atol = atol;
    H.maxit = maxit;
    H.ksp_rtol = ksp_rtol;
    H.ksp_maxit = ksp_maxit;
    H.ngroups = int(std::min<int64_t>(std::max<int64_t>((H.n + 255) / 256, 1), 592));
    // the face B arrays of a block are one range of the pool (B_xi, B_eta,
    // B_zeta consecutive, with the alignment gaps between them)
    std::vector<int64_t> snap, restore;
    size_t nbs = 0;
    int64_t seg_max = 0;
    for (int b = 0; b < ctx->nblocks; ++b)
    {
        const int64_t lo = int64_t(ctx->base[F_Bxi][size_t(b)]);
        const int64_t len = int64_t(ctx->base[F_Bzeta][size_t(b)]) + ctx->hbv[size_t(b)].vol - lo;
        snap.insert(snap.end(), {int64_t(nbs), lo, len});
        restore.insert(restore.end(), {lo, int64_t(nbs), len});
        nbs += size_t(len);
        seg_max = std::max(seg_max, len);
    }
    H.copy_ctas = int(std::min<int64_t>(std::max<int64_t>((seg_max + kThreads - 1) / kThreads, 1), 1184));
    RUN(upload_vec(ctx, snap, &H.seg_snap));
    RUN(upload_vec(ctx, restore, &H.seg_restore));
    CK(ctx, cudaMalloc(&H.bstar, nbs * 8));
    {
        std::vector<const double *> bsp;
        for (int b = 0; b < ctx->nblocks; ++b)
            for (int f = F_Bxi; f <= F_Bzeta; ++f)
                bsp.push_back(H.bstar + snap[size_t(3 * b)] +
                              (int64_t(ctx->base[size_t(f)][size_t(b)]) - int64_t(ctx->base[F_Bxi][size_t(b)])));
        CK(ctx, cudaMalloc(&H.bs, bsp.size() * sizeof(double *)));
        CK(ctx, cudaMemcpy(H.bs, bsp.data(), bsp.size() * sizeof(double *), cudaMemcpyHostToDevice));
    }
    const size_t nn = size_t(H.n);
    for (double **p : {&H.X, &H.F, &H.Xt, &H.Ft, &H.dx, &H.b, &H.r, &H.w})
        CK(ctx, cudaMalloc(p, nn * 8));
    CK(ctx, cudaMalloc(&H.V, nn * size_t(H.restart + 1) * 8));
    CK(ctx, cudaMalloc(&H.partial, size_t(H.ngroups) * size_t(kMdMax) * 8));
    CK(ctx, cudaMalloc(&H.dots, 64 * 8));
    CK(ctx, cudaMalloc(&H.st, sizeof(GmresState)));
    CK(ctx, cudaMemset(H.st, 0, sizeof(GmresState)));
    CK(ctx, cudaMalloc(&H.ctl, sizeof(HallCtl)));
    CK(ctx, cudaMemset(H.ctl, 0, sizeof(HallCtl)));
    CK(ctx, cudaMalloc(&H.done, sizeof(unsigned)));
    CK(ctx, cudaMemset(H.done, 0, sizeof(unsigned)));
    for (auto &sp : ctx->spare)
        if (!sp)
            CK(ctx, cudaStreamCreateWithFlags(&sp, cudaStreamNonBlocking));
    H.on = true;
    return MHD_OK;
}

int mhd_hall_stats(const mhd_ctx *ctx, int32_t *newton_its, int32_t *linear_its, double *fnorm, double *fnorm0,
                   int32_t *reason)
{
    BIND_DEVICE(ctx);
    if (!ctx)
        return MHD_EINVAL;
    const auto &H = ctx->hall;
    HallCtl c{};
    GmresState g{};
    if (H.ctl)
    {
        // the statistics live in the solve's device state
        if (cudaMemcpyAsync(&c, H.ctl, sizeof c, cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess ||
            cudaMemcpyAsync(&g, H.st, sizeof g, cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess ||
            cudaStreamSynchronize(ctx->stream) != cudaSuccess)
            return MHD_ECUDA;
    }
    if (newton_its)
        *newton_its = c.it;
    if (linear_its)
        *linear_its = int32_t(g.total_its - c.lin0);
    if (fnorm)
        *fnorm = c.f;
    if (fnorm0)
        *fnorm0 = c.f0;
    if (reason)
        *reason = c.reason;
    return MHD_OK;
}

int mhd_set_resistive_explicit(mhd_ctx *ctx, double inver_Rem, int32_t nsub)
{
    BIND_DEVICE(ctx);
    if (!ctx || nsub < 0)
        return fail(ctx, MHD_EINVAL, "bad explicit resistive arguments");
    if (ctx->nruns > 1 && nsub > 0)
        return fail(ctx, MHD_ESTATE, "the explicit resistive sub-cycling is not available in a batch of runs (one shared dt per solve)");
    if (nsub > 0 && ctx->res.on)
        return fail(ctx, MHD_ESTATE, "the implicit resistive solve is set up; the two are exclusive");
    ctx->res_nsub = nsub;
    ctx->res_inver_Rem = inver_Rem;
    // the hot sync lists depend on it (J_cell ghost depth)
    for (auto &kv : ctx->syncs)
        kv.second.built = false;
    drop_graph(ctx);
    return MHD_OK;
}

int mhd_set_flux_reference_run(mhd_ctx *ctx, int32_t run, const double prim[5])
{
    BIND_DEVICE(ctx);
    if (!ctx || !prim)
        return fail(ctx, MHD_EINVAL, "null flux reference");
    if (run < -1 || run >= ctx->nruns)
        return fail(ctx, MHD_EINVAL, "run %d out of range", run);
    for (int m = 0; m < 5; ++m)
        if (!std::isfinite(prim[m]))
            return fail(ctx, MHD_EINVAL, "non-finite flux reference");
    const double rho = prim[0], u = prim[1], v = prim[2], w = prim[3], p = prim[4];
    const double q[6] = {rho, u, v, w, p, p / (ctx->c.gamma - 1.0) + 0.5 * rho * (u * u + v * v + w * w)};
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    for (int r = (run < 0 ? 0 : run); r < (run < 0 ? ctx->nruns : run + 1); ++r)
        CK(ctx, cudaMemcpy(ctx->qref + 6 * size_t(r), q, sizeof(q), cudaMemcpyHostToDevice));
    return MHD_OK;
}

int mhd_set_flux_reference(mhd_ctx *ctx, const double prim[5])
{
    return mhd_set_flux_reference_run(ctx, -1, prim);
}

int mhd_autotune(mhd_ctx *ctx, int32_t reps, int32_t *min_ctas, int32_t n)
{
    BIND_DEVICE(ctx);
    if (!ctx || reps < 1 || n < 0 || (n > 0 && !min_ctas))
        return fail(ctx, MHD_EINVAL, "bad autotune arguments");
    if (ctx->capturing)
        return fail(ctx, MHD_ESTATE, "autotune during capture");
    RUN(ensure_geom(ctx));
    cudaStream_t s = ctx->stream;
    // snapshot of the state (U_H and the face B of every block; with the
    // implicit Hall solve also its edge EMF, which starts the next Newton
    // solve) and of the run clocks (dt keys, dt, time, step: one contiguous
    // allocation)
    std::vector<int> sf = {F_U, F_Bxi, F_Beta, F_Bzeta};
    if (ctx->hall.on)
        for (int a = 0; a < 3; ++a)
            sf.push_back(F_Ehxi + a);
    size_t tot = 0;
    for (int f : sf)
        for (int b = 0; b < ctx->nblocks; ++b)
            tot += size_t(kFields[f].ncomp) * size_t(ctx->hbv[size_t(b)].vol);
    const size_t clock_bytes = 32 * size_t(ctx->nruns);
    double *snap = nullptr;
    CK(ctx, cudaMalloc(&snap, tot * 8 + clock_bytes));
    auto copy_state = [&](bool save) -> int {
        size_t o = 0;
        for (int f : sf)
            for (int b = 0; b < ctx->nblocks; ++b)
            {
                const size_t cnt = size_t(kFields[f].ncomp) * size_t(ctx->hbv[size_t(b)].vol);
                double *field = ctx->pool + ctx->base[size_t(f)][size_t(b)];
                CK(ctx, cudaMemcpyAsync(save ? snap + o : field, save ? field : snap + o, cnt * 8,
                                        cudaMemcpyDeviceToDevice, s));
                o += cnt;
            }
        char *clk = reinterpret_cast<char *>(snap + tot);
        CK(ctx, cudaMemcpyAsync(save ? static_cast<void *>(clk) : static_cast<void *>(ctx->dt_key),
                                save ? static_cast<const void *>(ctx->dt_key) : static_cast<const void *>(clk),
                                clock_bytes, cudaMemcpyDeviceToDevice, s));
        if (!save)
            RUN(launch_update_derived(ctx)); // derived fields of the restored state
        return MHD_OK;
    };
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    CK(ctx, cudaEventCreate(&e0));
    CK(ctx, cudaEventCreate(&e1));
    // `reps` whole steps (the step graph) from the saved state, after one
    // step that builds the graph
    auto time_steps = [&](float &ms) -> int {
        RUN(copy_state(false));
        RUN(run_steps(ctx, 1));
        RUN(copy_state(false));
        CK(ctx, cudaEventRecord(e0, s));
        RUN(run_steps(ctx, reps));
        CK(ctx, cudaEventRecord(e1, s));
        CK(ctx, cudaEventSynchronize(e1));
        CK(ctx, cudaEventElapsedTime(&ms, e0, e1));
        return check_err(ctx);
    };
    // the faster of two timings of kernel t in variant v (clock and cache noise)
    auto trial = [&](int t, int v, float &ms) -> int {
        ctx->tune[t] = v;
        drop_graph(ctx);
        float a = 0.0f, b = 0.0f;
        RUN(time_steps(a));
        RUN(time_steps(b));
        ms = std::min(a, b);
        return MHD_OK;
    };
    int rc = copy_state(true);
    // bring the clocks up before anything is compared
    for (int w = 0; w < 3 && rc == MHD_OK; ++w)
    {
        float ms = 0.0f;
        rc = time_steps(ms);
    }
    for (int t = 0; t < NTUNE && rc == MHD_OK; ++t)
    {
        // the flux kernel of the precision in use only
        if ((t == TUNE_k_fluid_mixed && !ctx->pool32) || (t == TUNE_k_fluid_ucontra && ctx->pool32))
            continue;
        // the persistent resistive solve's grid, where it runs
        if (t == TUNE_k_gmres_resist && !(ctx->res.on && ctx->res.pgrid > 0))
            continue;
        // the Hall edge EMF, where the implicit Hall solve runs it
        if (t == TUNE_k_hall_edge && !ctx->hall.on)
            continue;
        int keep = ctx->tune[t];
        for (int v = 0; v < kTuneCount[t] && rc == MHD_OK; ++v)
        {
            if (v == keep)
                continue;
            // the candidate and the kept variant timed back to back; the
            // candidate replaces it only when the step is clearly faster
            float ms_v = 0.0f, ms_k = 0.0f;
            rc = trial(t, v, ms_v);
            if (rc == MHD_OK)
                rc = trial(t, keep, ms_k);
            if (rc == MHD_OK && ms_v < 0.97f * ms_k)
                keep = v;
        }
        ctx->tune[t] = keep;
        drop_graph(ctx);
    }
    if (rc == MHD_OK)
        rc = copy_state(false);
    cudaStreamSynchronize(s);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(snap);
    drop_graph(ctx);
    RUN(rc);
    for (int i = 0; i < n && i < NTUNE; ++i)
        min_ctas[i] = kTuneMinCtas[i][ctx->tune[i]];
    return MHD_OK;
}

const char *mhd_tune_name(int32_t i) { return (i >= 0 && i < NTUNE) ? kTuneNames[i] : nullptr; }

int mhd_set_tune(mhd_ctx *ctx, const int32_t *min_ctas, int32_t n)
{
    BIND_DEVICE(ctx);
    if (!ctx || n < 0 || n > NTUNE || (n > 0 && !min_ctas))
        return fail(ctx, MHD_EINVAL, "bad variant list");
    if (ctx->capturing)
        return fail(ctx, MHD_ESTATE, "variants changed during capture");
    int chosen[NTUNE];
    for (int t = 0; t < NTUNE; ++t)
    {
        chosen[t] = ctx->tune[t];
        if (t >= n)
            continue;
        chosen[t] = -1;
        for (int v = 0; v < kTuneCount[t]; ++v)
            if (kTuneMinCtas[t][v] == min_ctas[t])
                chosen[t] = v;
        if (chosen[t] < 0)
            return fail(ctx, MHD_EINVAL, "kernel %s has no variant %d", kTuneNames[t], min_ctas[t]);
    }
    for (int t = 0; t < NTUNE; ++t)
        ctx->tune[t] = chosen[t];
    drop_graph(ctx);
    return MHD_OK;
}

int mhd_resistive_stats(const mhd_ctx *ctx, int32_t *its, double *rnorm, double *bnorm, int32_t *reason)
{
    BIND_DEVICE(ctx);
    if (!ctx)
        return MHD_EINVAL;
    GmresState h;
    std::memset(&h, 0, sizeof(h));
    if (ctx->res.st)
    {
        if (cudaMemcpyAsync(&h, ctx->res.st, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess ||
            cudaStreamSynchronize(ctx->stream) != cudaSuccess)
            return MHD_ECUDA;
    }
    if (its)
        *its = h.its;
    if (rnorm)
        *rnorm = h.resid;
    if (bnorm)
        *bnorm = h.bnorm;
    if (reason)
        *reason = h.reason;
    return MHD_OK;
}

int mhd_set_integrator(mhd_ctx *ctx, int32_t integrator)
{
    BIND_DEVICE(ctx);
    if (!ctx)
        return MHD_EINVAL;
    if (integrator != MHD_INTEGRATOR_EULER && integrator != MHD_INTEGRATOR_SSPRK2)
        return fail(ctx, MHD_EINVAL, "unknown integrator %d", integrator);
    if (ctx->capturing)
        return fail(ctx, MHD_ESTATE, "integrator changed during capture");
    if (integrator == MHD_INTEGRATOR_SSPRK2)
    {
        if (ctx->hall.on)
            return fail(ctx, MHD_ESTATE, "SSP-RK2 is not available with the implicit Hall solve");
        if (!ctx->rk)
        {
            size_t n = 0;
            for (const auto &v : ctx->hbv)
                n += 8 * size_t(v.vol);
            CK(ctx, cudaMalloc(&ctx->rk, n * sizeof(double)));
            CK(ctx, cudaMemsetAsync(ctx->rk, 0, n * sizeof(double), ctx->stream));
            size_t o = 0;
            for (auto &v : ctx->hbv)
            {
                v.rk = ctx->rk + o;
                o += 8 * size_t(v.vol);
            }
            CK(ctx, cudaMemcpyAsync(ctx->dbv, ctx->hbv.data(), sizeof(BlockView) * ctx->hbv.size(),
                                    cudaMemcpyHostToDevice, ctx->stream));
            CK(ctx, cudaStreamSynchronize(ctx->stream));
        }
    }
    if (integrator != ctx->integrator)
    {
        ctx->integrator = integrator;
        drop_graph(ctx);
    }
    return MHD_OK;
}

int mhd_test_stall_barrier(mhd_ctx *ctx, uint32_t spin_limit)
{
    BIND_DEVICE(ctx);
    if (!ctx || spin_limit == 0)
        return MHD_EINVAL;
    auto &R = ctx->res;
    if (!R.on || !R.bar)
        return fail(ctx, MHD_ESTATE, "test_stall_barrier: no persistent implicit resistive solve is set up");
    // arrival count one short of the grid for good (no CTA completes the
    // barrier), and a short polling limit for every wait
    const unsigned w[4] = {0xFFFFFFFFu, 0u, spin_limit, 0u};
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    CK(ctx, cudaMemcpy(R.bar, w, sizeof(w), cudaMemcpyHostToDevice));
    return MHD_OK;
}

int mhd_sync(mhd_ctx *ctx, const char *group)
{
    BIND_DEVICE(ctx);
    if (!ctx || !group)
        return MHD_EINVAL;
    RUN(ensure_geom(ctx));
    RUN(run_sync(ctx, group, true));
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    return MHD_OK;
}

int mhd_update_derived(mhd_ctx *ctx)
{
    BIND_DEVICE(ctx);
    if (!ctx)
        return MHD_EINVAL;
    RUN(ensure_geom(ctx));
    RUN(launch_update_derived(ctx));
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    return MHD_OK;
}

int mhd_step(mhd_ctx *ctx, int32_t nsteps, double *dt_out, double *time_out)
{
    BIND_DEVICE(ctx);
    if (!ctx || nsteps < 0)
        return MHD_EINVAL;
    RUN(run_steps(ctx, nsteps));
    RUN(check_err(ctx));
    if (dt_out)
        CK(ctx, cudaMemcpy(dt_out, ctx->dt, 8, cudaMemcpyDeviceToHost));
    if (time_out)
        CK(ctx, cudaMemcpy(time_out, ctx->time, 8, cudaMemcpyDeviceToHost));
    return MHD_OK;
}

int mhd_batch_step(mhd_ctx *ctx, int32_t nsteps, double *dt_out, double *time_out, int32_t nruns)
{
    BIND_DEVICE(ctx);
    if (!ctx || nsteps < 0 || (nruns > 0 && (!dt_out && !time_out)))
        return fail(ctx, MHD_EINVAL, "bad batch step arguments");
    if (nruns != 0 && nruns != ctx->nruns)
        return fail(ctx, MHD_EINVAL, "the context holds %d runs, not %d", ctx->nruns, nruns);
    RUN(run_steps(ctx, nsteps));
    RUN(check_err(ctx));
    const size_t nr = size_t(nruns);
    if (dt_out && nr)
        CK(ctx, cudaMemcpy(dt_out, ctx->dt, 8 * nr, cudaMemcpyDeviceToHost));
    if (time_out && nr)
        CK(ctx, cudaMemcpy(time_out, ctx->time, 8 * nr, cudaMemcpyDeviceToHost));
    return MHD_OK;
}

namespace
{
// the host state's box of field f in block b: the whole array (ghosts
// included) or its inner points only (cells [0, n), faces [0, n] along
// their own axis)
void state_box(const mhd_ctx *ctx, int f, int b, bool inner, int lo[3], int hi[3])
{
    field_box(ctx, f, b, lo, hi);
    if (!inner)
        return;
    const int g = kFields[f].nghost;
    for (int a = 0; a < 3; ++a)
    {
        lo[a] = 0;
        hi[a] -= g;
    }
}

int64_t state_count(const mhd_ctx *ctx, bool inner)
{
    int64_t n = 0;
    for (int b = 0; b < ctx->nblocks; ++b)
        for (int f : {int(F_U), int(F_Bxi), int(F_Beta), int(F_Bzeta)})
        {
            int lo[3], hi[3];
            state_box(ctx, f, b, inner, lo, hi);
            n += int64_t(hi[0] - lo[0]) * (hi[1] - lo[1]) * (hi[2] - lo[2]) * kFields[f].ncomp;
        }
    return n;
}

// upload, syncs, derived fields, steps, download of the state's boxes
int step_host(mhd_ctx *ctx, int32_t nsteps, const double *state_in, double *state_out, int64_t count, double *dt_out,
              bool inner)
{
    if (!state_in || !state_out || nsteps < 0)
        return MHD_EINVAL;
    if (count != state_count(ctx, inner))
        return fail(ctx, MHD_EINVAL, "state holds %lld values, expected %lld", (long long)count,
                    (long long)state_count(ctx, inner));
    RUN(ensure_staging(ctx, size_t(count)));
    CK(ctx, cudaMemcpyAsync(ctx->staging, state_in, size_t(count) * 8, cudaMemcpyHostToDevice, ctx->stream));
    int64_t off = 0;
    for (int b = 0; b < ctx->nblocks; ++b)
        for (int f : {int(F_U), int(F_Bxi), int(F_Beta), int(F_Bzeta)})
        {
            int lo[3], hi[3];
            state_box(ctx, f, b, inner, lo, hi);
            const int64_t n = int64_t(hi[0] - lo[0]) * (hi[1] - lo[1]) * (hi[2] - lo[2]) * kFields[f].ncomp;
            prof_begin(ctx, "k_aos_to_soa");
            k_aos_to_soa<<<grid_for(n), kThreads, 0, ctx->stream>>>(ctx->dbv, b, f, kFields[f].ncomp, lo[0], lo[1],
                                                                    lo[2], hi[0] - lo[0], hi[1] - lo[1],
                                                                    hi[2] - lo[2], ctx->staging + off);
            RUN(launched(ctx));
            off += n;
        }
    RUN(ensure_geom(ctx));
    RUN(run_sync(ctx, "Ucell"));
    RUN(run_sync(ctx, "Bface"));
    RUN(launch_update_derived(ctx));
    RUN(run_steps(ctx, nsteps));
    for (int f : {int(F_U), int(F_Bxi)})
        RUN(materialise_field(ctx, f));
    off = 0;
    for (int b = 0; b < ctx->nblocks; ++b)
        for (int f : {int(F_U), int(F_Bxi), int(F_Beta), int(F_Bzeta)})
        {
            int lo[3], hi[3];
            state_box(ctx, f, b, inner, lo, hi);
            const int64_t n = int64_t(hi[0] - lo[0]) * (hi[1] - lo[1]) * (hi[2] - lo[2]) * kFields[f].ncomp;
            prof_begin(ctx, "k_soa_to_aos");
            k_soa_to_aos<<<grid_for(n), kThreads, 0, ctx->stream>>>(ctx->dbv, b, f, kFields[f].ncomp, lo[0], lo[1],
                                                                    lo[2], hi[0] - lo[0], hi[1] - lo[1],
                                                                    hi[2] - lo[2], ctx->staging + off);
            RUN(launched(ctx));
            off += n;
        }
    CK(ctx, cudaMemcpyAsync(state_out, ctx->staging, size_t(count) * 8, cudaMemcpyDeviceToHost, ctx->stream));
    RUN(check_err(ctx));
    if (dt_out)
        CK(ctx, cudaMemcpy(dt_out, ctx->dt, 8, cudaMemcpyDeviceToHost));
    return MHD_OK;
}
} // namespace

int64_t mhd_state_count(const mhd_ctx *ctx)
{
    return ctx ? state_count(ctx, false) : -1;
}

int64_t mhd_state_count_inner(const mhd_ctx *ctx)
{
    return ctx ? state_count(ctx, true) : -1;
}

int mhd_step_host(mhd_ctx *ctx, int32_t nsteps, const double *state_in, double *state_out, int64_t count,
                  double *dt_out)
{
    BIND_DEVICE(ctx);
    if (!ctx)
        return MHD_EINVAL;
    return step_host(ctx, nsteps, state_in, state_out, count, dt_out, false);
}

int mhd_step_host_inner(mhd_ctx *ctx, int32_t nsteps, const double *state_in, double *state_out, int64_t count,
                        double *dt_out)
{
    BIND_DEVICE(ctx);
    if (!ctx)
        return MHD_EINVAL;
    return step_host(ctx, nsteps, state_in, state_out, count, dt_out, true);
}

int mhd_host_alloc(int64_t bytes, void **ptr)
{
    if (!ptr || bytes <= 0)
        return MHD_EINVAL;
    return cudaHostAlloc(ptr, size_t(bytes), cudaHostAllocDefault) == cudaSuccess ? MHD_OK : MHD_ENOMEM;
}

int mhd_host_free(void *ptr)
{
    return cudaFreeHost(ptr) == cudaSuccess ? MHD_OK : MHD_ECUDA;
}

int mhd_stage(mhd_ctx *ctx, int32_t stage_id)
{
    BIND_DEVICE(ctx);
    if (!ctx)
        return MHD_EINVAL;
    RUN(ensure_geom(ctx));
    switch (stage_id)
    {
    case MHD_STAGE_TIMESTEP:
        prof_begin(ctx, "k_begin_step");
        k_begin_step<<<1, 128, 0, ctx->stream>>>(ctx->dt_key, ctx->dt, ctx->err, ctx->prm.dt_abort, ctx->nruns);
        RUN(launched(ctx));
        break;
    case MHD_STAGE_FLUID_RHS:
        RUN(launch_fluid_rhs(ctx));
        break;
    case MHD_STAGE_INDUCTION:
        RUN(launch_induction(ctx, false));
        break;
    case MHD_STAGE_UPDATE:
        RUN(launch_update_u(ctx));
        {
            prof_begin(ctx, "k_curl_e2f");
            launch_k_curl_e2f(ctx->tune[TUNE_k_curl_e2f], grid_kind(ctx, KIND_STAG), ctx->stream, ctx->dbv, F_Exi, -1, F_Bxi, -1.0,
                                                                                ctx->dt, 1.0, 0, nullptr);
            RUN(launched(ctx));
        }
        break;
    case MHD_STAGE_HALL_EMF:
        // the edge stencils read B_cell / J_cell one ghost layer deep
        RUN(materialise_group(ctx, "B_cell"));
        RUN(materialise_group(ctx, "J_cell"));
        prof_begin(ctx, "k_hall_cell");
        k_hall_cell<<<dim3(grid_for(max_box(ctx, LOC_CELL, ctx->G)), ctx->nblocks), kThreads, 0, ctx->stream>>>(
            ctx->dbv, ctx->c, ctx->hall_coef);
        RUN(launched(ctx));
        prof_begin(ctx, "k_hall_edge");
        launch_k_hall_edge(ctx->tune[TUNE_k_hall_edge], grid_kind(ctx, KIND_STAG), ctx->stream, ctx->dbv,
                           ctx->hall_zb, ctx->hall_nzb);
        RUN(launched(ctx));
        break;
    case MHD_STAGE_HALL_SOLVE:
        // one implicit Hall solve at the current dt, then calc_Bcell (as StepOnce)
        if (!ctx->hall.on)
            return fail(ctx, MHD_ESTATE, "the implicit Hall solve is not set up");
        RUN(launch_hall_implicit(ctx));
        prof_begin(ctx, "k_bcell");
        launch_k_bcell(false, dim3(grid_for(max_box(ctx, LOC_CELL, 0)), ctx->nblocks), ctx->stream, ctx->dbv);
        RUN(launched(ctx));
        RUN(run_sync(ctx, "B_cell"));
        break;
    case MHD_STAGE_DIVB:
        prof_begin(ctx, "k_divb");
        k_divb<<<dim3(grid_for(max_box(ctx, LOC_CELL, 0)), ctx->nblocks), kThreads, 0, ctx->stream>>>(ctx->dbv);
        RUN(launched(ctx));
        RUN(launch_pole(ctx, POLE_DIVB)); // the first cell layer next to a Pole: 0
        break;
    default:
        return fail(ctx, MHD_EINVAL, "unknown stage %d", stage_id);
    }
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    return check_err(ctx);
}

int mhd_run_time(mhd_ctx *ctx, int32_t run, double *dt, double *time, int64_t *step)
{
    BIND_DEVICE(ctx);
    if (!ctx || run < 0 || run >= ctx->nruns)
        return MHD_EINVAL;
    double d = 0.0, t = 0.0;
    long long s = 0;
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    CK(ctx, cudaMemcpy(&d, ctx->dt + run, 8, cudaMemcpyDeviceToHost));
    CK(ctx, cudaMemcpy(&t, ctx->time + run, 8, cudaMemcpyDeviceToHost));
    CK(ctx, cudaMemcpy(&s, ctx->step + run, 8, cudaMemcpyDeviceToHost));
    if (dt)
        *dt = d;
    if (time)
        *time = t;
    if (step)
        *step = s;
    return MHD_OK;
}

int mhd_get_time(mhd_ctx *ctx, double *dt, double *time, int64_t *step)
{
    BIND_DEVICE(ctx);
    return mhd_run_time(ctx, 0, dt, time, step);
}

int mhd_set_time(mhd_ctx *ctx, double dt, double time, int64_t step)
{
    BIND_DEVICE(ctx);
    if (!ctx)
        return MHD_EINVAL;
    const size_t nr = size_t(ctx->nruns);
    const std::vector<double> d(nr, dt), t(nr, time);
    const std::vector<long long> s(nr, step);
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    CK(ctx, cudaMemcpy(ctx->dt, d.data(), 8 * nr, cudaMemcpyHostToDevice));
    CK(ctx, cudaMemcpy(ctx->time, t.data(), 8 * nr, cudaMemcpyHostToDevice));
    CK(ctx, cudaMemcpy(ctx->step, s.data(), 8 * nr, cudaMemcpyHostToDevice));
    return MHD_OK;
}

int64_t mhd_kernel_launches(const mhd_ctx *ctx)
{
    if (!ctx)
        return -1;
    int64_t n = ctx->launches;
    const auto &R = ctx->res;
    if (R.st && (R.k_cycle > 0 || R.k_inner > 0))
    {
        // passes of the graph-resident Krylov loops, counted on the device
        GmresState h;
        if (cudaMemcpyAsync(&h, R.st, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream) == cudaSuccess &&
            cudaStreamSynchronize(ctx->stream) == cudaSuccess)
            n += R.k_cycle * (h.total_cycles - R.cycles_eager) + R.k_inner * (h.total_its - R.its_eager);
    }
    const auto &H = ctx->hall;
    if (H.ctl && H.kb_nested > 0)
    {
        // passes of the graph-resident Hall loops, counted on the device
        HallCtl c;
        GmresState g;
        if (cudaMemcpyAsync(&c, H.ctl, sizeof c, cudaMemcpyDeviceToHost, ctx->stream) == cudaSuccess &&
            cudaMemcpyAsync(&g, H.st, sizeof g, cudaMemcpyDeviceToHost, ctx->stream) == cudaSuccess &&
            cudaStreamSynchronize(ctx->stream) == cudaSuccess)
        {
            const long long pass[HALL_KB_N] = {c.pass[0], g.total_cycles, g.total_its, c.pass[1], c.pass[2]};
            for (int q = 0; q < HALL_KB_N; ++q)
                n += H.kb[q] * (pass[q] - H.eager[q]);
        }
    }
    return n;
}

int mhd_field_spec(int32_t index, const char **name, int32_t *loc, int32_t *ncomp, int32_t *nghost)
{
    if (index < 0 || index >= NFIELD)
        return MHD_EINVAL;
    if (name)
        *name = kFields[index].name;
    if (loc)
        *loc = kFields[index].loc;
    if (ncomp)
        *ncomp = kFields[index].ncomp;
    if (nghost)
        *nghost = kFields[index].nghost;
    return MHD_OK;
}

int mhd_profile_step(mhd_ctx *ctx, int32_t cap, int32_t *kernel_ids, float *ms, int32_t *count)
{
    BIND_DEVICE(ctx);
    if (!ctx || !count || cap < 0)
        return MHD_EINVAL;
    RUN(ensure_geom(ctx));
    RUN(build_all_syncs(ctx));
    ctx->profiling = true;
    ctx->prof_ev.clear();
    ctx->prof_names.clear();
    const int rc = launch_step(ctx);
    ctx->profiling = false;
    if (rc != MHD_OK)
        return rc;
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    const int n = int(ctx->prof_names.size());
    *count = n;
    for (int q = 0; q < n && q < cap; ++q)
    {
        float t = 0.0f;
        cudaEventElapsedTime(&t, ctx->prof_ev[size_t(2 * q)], ctx->prof_ev[size_t(2 * q + 1)]);
        if (ms)
            ms[q] = t;
        if (kernel_ids)
        {
            int id = 0;
            for (; id < kNumKernelNames; ++id)
                if (std::strcmp(kKernelNames[id], ctx->prof_names[size_t(q)]) == 0)
                    break;
            kernel_ids[q] = id;
        }
    }
    for (auto e : ctx->prof_ev)
        cudaEventDestroy(e);
    ctx->prof_ev.clear();
    ctx->prof_names.clear();
    return check_err(ctx);
}

const char *mhd_kernel_name(int32_t id) { return (id >= 0 && id < kNumKernelNames) ? kKernelNames[id] : ""; }

void *mhd_stream(const mhd_ctx *ctx) { return ctx ? static_cast<void *>(ctx->stream) : nullptr; }

} // extern "C"
