// C-ABI of the B200 MHD hot path (see include/beta1_mhd.h): context and
// field pool management, host<->device transfers, compiled boundary syncs,
// and the per-step launch sequence replayed as a CUDA graph.
#include "mhd_kernels.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

using namespace mhd;

namespace
{

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

struct SyncMap
{
    // phase A: constants and wall handlers
    uint64_t *cdst = nullptr;
    double *cval = nullptr;
    int64_t nconst = 0;
    std::vector<std::pair<int, int>> walls; // (block, direction) of Solid_Surface fluid handlers
    // phase B: composed copies
    uint64_t *dst = nullptr;
    uint64_t *src = nullptr;
    double *tmp = nullptr; // non-null when a source is also a destination
    int64_t n = 0;
};

constexpr int kThreads = 256;

const char *const kKernelNames[] = {"k_fluid_rhs",   "k_eface",        "k_eedge",         "k_curl_e2f",
                                    "k_update_u",    "k_bcell",        "k_jedge",         "k_jcell",
                                    "k_pv_uplus_dt", "k_begin_step",   "k_arm_dt",        "k_end_step",
                                    "k_gather",      "k_gather_stage", "k_scatter_stage", "k_aos_to_soa",
                                    "k_soa_to_aos",  "k_set_consts",   "k_wall_u"};
constexpr int kNumKernelNames = int(sizeof(kKernelNames) / sizeof(kKernelNames[0]));

} // namespace

struct mhd_ctx
{
    int nblocks = 0;
    mhd_params prm{};
    Consts c{};
    int G = 4;
    std::vector<BlockView> hbv;
    BlockView *dbv = nullptr;
    double *pool = nullptr;
    size_t pool_n = 0;
    std::vector<std::vector<size_t>> base; // [field][block] offset in pool
    cudaStream_t stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    int64_t graph_kernels = 0;
    // device scalars
    unsigned long long *dt_key = nullptr;
    double *dt = nullptr;
    double *time = nullptr;
    long long *step = nullptr;
    int *err = nullptr;
    std::map<std::string, SyncMap> syncs;
    double *staging = nullptr;
    size_t staging_n = 0;
    int64_t launches = 0;
    int64_t max_cells = 0;
    bool capturing = false;
    std::string msg;
    // eager profiling: one event pair per launch
    bool profiling = false;
    std::vector<const char *> prof_names;
    std::vector<cudaEvent_t> prof_ev;
};

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

int run_sync(mhd_ctx *ctx, const char *group)
{
    auto it = ctx->syncs.find(group);
    if (it == ctx->syncs.end())
        return MHD_OK;
    SyncMap &s = it->second;
    if (s.nconst > 0)
    {
        prof_begin(ctx, "k_set_consts");
        k_set_consts<<<grid_for(s.nconst), kThreads, 0, ctx->stream>>>(ctx->pool, s.cdst, s.cval, s.nconst);
        RUN(launched(ctx));
    }
    for (const auto &w : s.walls)
    {
        const BlockView &v = ctx->hbv[size_t(w.first)];
        const int ax = std::abs(w.second) - 1;
        const int64_t ncol = (ax == 0) ? int64_t(v.nj) * v.nk : (ax == 1) ? int64_t(v.ni) * v.nk : int64_t(v.ni) * v.nj;
        prof_begin(ctx, "k_wall_u");
        k_wall_u<<<grid_for(ncol), kThreads, 0, ctx->stream>>>(ctx->dbv, w.first, w.second, ctx->c.gamma);
        RUN(launched(ctx));
    }
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
    k_gather<<<grid_for(s.n), kThreads, 0, ctx->stream>>>(ctx->pool, s.dst, s.src, s.n);
    return launched(ctx);
}

int launch_update_derived(mhd_ctx *ctx)
{
    const int nb = ctx->nblocks;
    cudaStream_t s = ctx->stream;
    const int64_t nc = max_box(ctx, LOC_CELL, 0);
    prof_begin(ctx, "k_bcell");
    k_bcell<<<dim3(grid_for(nc), nb), kThreads, 0, s>>>(ctx->dbv);
    RUN(launched(ctx));
    RUN(run_sync(ctx, "B_cell"));
    const int64_t ne = max_box(ctx, LOC_EZETA, 0) > max_box(ctx, LOC_EXI, 0) ? max_box(ctx, LOC_EZETA, 0)
                                                                              : max_box(ctx, LOC_EXI, 0);
    const int64_t ne2 = max_box(ctx, LOC_EETA, 0) > ne ? max_box(ctx, LOC_EETA, 0) : ne;
    prof_begin(ctx, "k_jedge");
    k_jedge<<<dim3(grid_for(ne2), nb, 3), kThreads, 0, s>>>(ctx->dbv, F_Bxi, F_Jxi, 1.0);
    RUN(launched(ctx));
    RUN(run_sync(ctx, "Jedge"));
    prof_begin(ctx, "k_jcell");
    k_jcell<<<dim3(grid_for(nc), nb), kThreads, 0, s>>>(ctx->dbv);
    RUN(launched(ctx));
    RUN(run_sync(ctx, "J_cell"));
    // arm the dt reduction, then PV / U_plus / CFL bound of the next step
    prof_begin(ctx, "k_arm_dt");
    k_arm_dt<<<1, 1, 0, s>>>(ctx->dt_key);
    RUN(launched(ctx));
    const int64_t ng = max_box(ctx, LOC_CELL, ctx->G);
    prof_begin(ctx, "k_pv_uplus_dt");
    k_pv_uplus_dt<<<dim3(grid_for(ng), nb), kThreads, 0, s>>>(ctx->dbv, ctx->c, ctx->dt_key);
    RUN(launched(ctx));
    RUN(run_sync(ctx, "Uplus"));
    return MHD_OK;
}

int launch_fluid_rhs(mhd_ctx *ctx)
{
    const int64_t nc = max_box(ctx, LOC_CELL, 0);
    prof_begin(ctx, "k_fluid_rhs");
    k_fluid_rhs<<<dim3(grid_for(nc), ctx->nblocks), kThreads, 0, ctx->stream>>>(ctx->dbv, ctx->c, nc);
    return launched(ctx);
}

int launch_induction(mhd_ctx *ctx, bool update_b)
{
    const int nb = ctx->nblocks;
    cudaStream_t s = ctx->stream;
    int64_t nf = 0;
    for (int l = LOC_FXI; l <= LOC_FZETA; ++l)
        nf = max_box(ctx, l, 0) > nf ? max_box(ctx, l, 0) : nf;
    prof_begin(ctx, "k_eface");
    k_eface<<<dim3(grid_for(nf), nb, 3), kThreads, 0, s>>>(ctx->dbv);
    RUN(launched(ctx));
    RUN(run_sync(ctx, "Eface"));
    int64_t ne = 0;
    for (int l = LOC_EXI; l <= LOC_EZETA; ++l)
        ne = max_box(ctx, l, ctx->G) > ne ? max_box(ctx, l, ctx->G) : ne;
    prof_begin(ctx, "k_eedge");
    k_eedge<<<dim3(grid_for(ne), nb, 3), kThreads, 0, s>>>(ctx->dbv, ctx->G);
    RUN(launched(ctx));
    RUN(run_sync(ctx, "Eedge"));
    prof_begin(ctx, "k_curl_e2f");
    k_curl_e2f<<<dim3(grid_for(nf), nb, 3), kThreads, 0, s>>>(ctx->dbv, F_Exi, F_RBxi, update_b ? F_Bxi : -1,
                                                               -1.0, ctx->dt, 1.0);
    return launched(ctx);
}

int launch_update_u(mhd_ctx *ctx)
{
    const int64_t nc = max_box(ctx, LOC_CELL, 0);
    prof_begin(ctx, "k_update_u");
    k_update_u<<<dim3(grid_for(nc), ctx->nblocks), kThreads, 0, ctx->stream>>>(ctx->dbv, ctx->dt);
    return launched(ctx);
}

// one LunarSolver::StepOnce
int launch_step(mhd_ctx *ctx)
{
    cudaStream_t s = ctx->stream;
    prof_begin(ctx, "k_begin_step");
    k_begin_step<<<1, 1, 0, s>>>(ctx->dt_key, ctx->dt, ctx->err, ctx->prm.dt_abort);
    RUN(launched(ctx));
    RUN(launch_fluid_rhs(ctx));
    RUN(launch_induction(ctx, /*update_b=*/true));
    RUN(launch_update_u(ctx));
    prof_begin(ctx, "k_end_step");
    k_end_step<<<1, 1, 0, s>>>(ctx->dt, ctx->time, ctx->step);
    RUN(launched(ctx));
    RUN(run_sync(ctx, "Ucell"));
    RUN(run_sync(ctx, "Bface"));
    RUN(launch_update_derived(ctx));
    return MHD_OK;
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
    return MHD_OK;
}

void drop_graph(mhd_ctx *ctx)
{
    if (ctx->gexec)
        cudaGraphExecDestroy(ctx->gexec);
    if (ctx->graph)
        cudaGraphDestroy(ctx->graph);
    ctx->gexec = nullptr;
    ctx->graph = nullptr;
}

int build_graph(mhd_ctx *ctx)
{
    if (ctx->gexec)
        return MHD_OK;
    const int64_t before = ctx->launches;
    CK(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    const int rc = launch_step(ctx);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
    ctx->launches = before;
    if (rc != MHD_OK)
    {
        if (g)
            cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess)
        return fail(ctx, MHD_ECUDA, "graph capture failed: %s", cudaGetErrorString(e));
    ctx->graph = g;
    CK(ctx, cudaGraphInstantiate(&ctx->gexec, g, 0));
    size_t nn = 0;
    CK(ctx, cudaGraphGetNodes(g, nullptr, &nn));
    ctx->graph_kernels = int64_t(nn);
    return MHD_OK;
}

} // namespace

extern "C" {

int mhd_ctx_create(const mhd_block_desc *blocks, int32_t nblocks, const mhd_params *params, mhd_ctx **out)
{
    if (!blocks || nblocks <= 0 || !params || !out)
        return MHD_EINVAL;
    *out = nullptr;
    mhd_ctx *ctx = new mhd_ctx;
    ctx->nblocks = nblocks;
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
    int rc = MHD_OK;
    auto bail = [&](int code) {
        mhd_ctx_destroy(ctx);
        return code;
    };
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess)
        return bail(MHD_ECUDA);
    if (cudaMalloc(&ctx->pool, off * sizeof(double)) != cudaSuccess)
        return bail(MHD_ENOMEM);
    if (cudaMemsetAsync(ctx->pool, 0, off * sizeof(double), ctx->stream) != cudaSuccess)
        return bail(MHD_ECUDA);
    for (int b = 0; b < nblocks; ++b)
        for (int f = 0; f < NFIELD; ++f)
            ctx->hbv[size_t(b)].f[f] = ctx->pool + ctx->base[size_t(f)][size_t(b)];
    if (cudaMalloc(&ctx->dbv, sizeof(BlockView) * size_t(nblocks)) != cudaSuccess)
        return bail(MHD_ENOMEM);
    if (cudaMemcpy(ctx->dbv, ctx->hbv.data(), sizeof(BlockView) * size_t(nblocks), cudaMemcpyHostToDevice) !=
        cudaSuccess)
        return bail(MHD_ECUDA);
    void *scal = nullptr;
    if (cudaMalloc(&scal, 256) != cudaSuccess)
        return bail(MHD_ENOMEM);
    cudaMemset(scal, 0, 256);
    char *sc = static_cast<char *>(scal);
    ctx->dt_key = reinterpret_cast<unsigned long long *>(sc);
    ctx->dt = reinterpret_cast<double *>(sc + 8);
    ctx->time = reinterpret_cast<double *>(sc + 16);
    ctx->step = reinterpret_cast<long long *>(sc + 24);
    ctx->err = reinterpret_cast<int *>(sc + 32);
    const double big = 1e100;
    unsigned long long key;
    std::memcpy(&key, &big, 8);
    if (cudaMemcpy(ctx->dt_key, &key, 8, cudaMemcpyHostToDevice) != cudaSuccess)
        return bail(MHD_ECUDA);
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess)
        return bail(MHD_ECUDA);
    (void)rc;
    *out = ctx;
    return MHD_OK;
}

int mhd_ctx_destroy(mhd_ctx *ctx)
{
    if (!ctx)
        return MHD_OK;
    drop_graph(ctx);
    for (auto &kv : ctx->syncs)
    {
        cudaFree(kv.second.dst);
        cudaFree(kv.second.src);
        cudaFree(kv.second.tmp);
        cudaFree(kv.second.cdst);
        cudaFree(kv.second.cval);
    }
    if (ctx->dt_key)
        cudaFree(ctx->dt_key);
    cudaFree(ctx->staging);
    cudaFree(ctx->dbv);
    cudaFree(ctx->pool);
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
    if (!data)
        return fail(ctx, MHD_EINVAL, "null data");
    return transfer(ctx, name, block, data, nullptr, count);
}

int mhd_download_field(mhd_ctx *ctx, const char *name, int32_t block, double *data, int64_t count)
{
    if (!data)
        return fail(ctx, MHD_EINVAL, "null data");
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

int mhd_set_sync_map(mhd_ctx *ctx, const char *group, const int64_t *dst, const int64_t *src, int64_t n)
{
    if (!ctx || !group || n < 0 || (n > 0 && (!dst || !src)))
        return fail(ctx, MHD_EINVAL, "bad sync map arguments");
    std::vector<uint64_t> d(static_cast<size_t>(n)), s(static_cast<size_t>(n));
    std::vector<char> is_dst(ctx->pool_n, 0);
    for (int64_t t = 0; t < n; ++t)
    {
        const int64_t od = pool_offset(ctx, dst[t]);
        const int64_t os = pool_offset(ctx, src[t]);
        if (od < 0 || os < 0)
            return fail(ctx, MHD_EINVAL, "sync map entry %lld has an invalid point id", (long long)t);
        d[size_t(t)] = uint64_t(od);
        s[size_t(t)] = uint64_t(os);
        is_dst[size_t(od)] = 1;
    }
    bool staged = false;
    for (int64_t t = 0; t < n && !staged; ++t)
        staged = is_dst[size_t(s[size_t(t)])] != 0;
    SyncMap &m = ctx->syncs[group];
    cudaFree(m.dst);
    cudaFree(m.src);
    cudaFree(m.tmp);
    m.dst = m.src = nullptr;
    m.tmp = nullptr;
    m.n = 0;
    drop_graph(ctx);
    if (n == 0)
        return MHD_OK;
    CK(ctx, cudaMalloc(&m.dst, size_t(n) * 8));
    CK(ctx, cudaMalloc(&m.src, size_t(n) * 8));
    CK(ctx, cudaMemcpy(m.dst, d.data(), size_t(n) * 8, cudaMemcpyHostToDevice));
    CK(ctx, cudaMemcpy(m.src, s.data(), size_t(n) * 8, cudaMemcpyHostToDevice));
    if (staged)
        CK(ctx, cudaMalloc(&m.tmp, size_t(n) * 8));
    m.n = n;
    return MHD_OK;
}

int mhd_set_sync_consts(mhd_ctx *ctx, const char *group, const int64_t *dst, const double *val, int64_t n)
{
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
    cudaFree(m.cdst);
    cudaFree(m.cval);
    m.cdst = nullptr;
    m.cval = nullptr;
    m.nconst = 0;
    drop_graph(ctx);
    if (n == 0)
        return MHD_OK;
    CK(ctx, cudaMalloc(&m.cdst, size_t(n) * 8));
    CK(ctx, cudaMalloc(&m.cval, size_t(n) * 8));
    CK(ctx, cudaMemcpy(m.cdst, d.data(), size_t(n) * 8, cudaMemcpyHostToDevice));
    CK(ctx, cudaMemcpy(m.cval, val, size_t(n) * 8, cudaMemcpyHostToDevice));
    m.nconst = n;
    return MHD_OK;
}

int mhd_set_sync_wall(mhd_ctx *ctx, const char *group, int32_t block, int32_t direction)
{
    if (!ctx || !group || block < 0 || block >= ctx->nblocks || direction == 0 || direction < -3 || direction > 3)
        return fail(ctx, MHD_EINVAL, "bad wall handler arguments");
    ctx->syncs[group].walls.emplace_back(block, direction);
    drop_graph(ctx);
    return MHD_OK;
}

int mhd_sync(mhd_ctx *ctx, const char *group)
{
    if (!ctx || !group)
        return MHD_EINVAL;
    RUN(run_sync(ctx, group));
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    return MHD_OK;
}

int mhd_update_derived(mhd_ctx *ctx)
{
    if (!ctx)
        return MHD_EINVAL;
    RUN(launch_update_derived(ctx));
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    return MHD_OK;
}

int mhd_step(mhd_ctx *ctx, int32_t nsteps, double *dt_out, double *time_out)
{
    if (!ctx || nsteps < 0)
        return MHD_EINVAL;
    RUN(build_graph(ctx));
    for (int s = 0; s < nsteps; ++s)
    {
        CK(ctx, cudaGraphLaunch(ctx->gexec, ctx->stream));
        ctx->launches += ctx->graph_kernels;
    }
    RUN(check_err(ctx));
    if (dt_out)
        CK(ctx, cudaMemcpy(dt_out, ctx->dt, 8, cudaMemcpyDeviceToHost));
    if (time_out)
        CK(ctx, cudaMemcpy(time_out, ctx->time, 8, cudaMemcpyDeviceToHost));
    return MHD_OK;
}

int64_t mhd_state_count(const mhd_ctx *ctx)
{
    if (!ctx)
        return -1;
    int64_t n = 0;
    for (int b = 0; b < ctx->nblocks; ++b)
        for (int f : {int(F_U), int(F_Bxi), int(F_Beta), int(F_Bzeta)})
            n += field_count(ctx, f, b);
    return n;
}

int mhd_step_host(mhd_ctx *ctx, int32_t nsteps, const double *state_in, double *state_out, int64_t count,
                  double *dt_out)
{
    if (!ctx || !state_in || !state_out || nsteps < 0)
        return MHD_EINVAL;
    if (count != mhd_state_count(ctx))
        return fail(ctx, MHD_EINVAL, "state holds %lld values, expected %lld", (long long)count,
                    (long long)mhd_state_count(ctx));
    RUN(ensure_staging(ctx, size_t(count)));
    CK(ctx, cudaMemcpyAsync(ctx->staging, state_in, size_t(count) * 8, cudaMemcpyHostToDevice, ctx->stream));
    int64_t off = 0;
    for (int b = 0; b < ctx->nblocks; ++b)
        for (int f : {int(F_U), int(F_Bxi), int(F_Beta), int(F_Bzeta)})
        {
            int lo[3], hi[3];
            field_box(ctx, f, b, lo, hi);
            const int64_t n = field_count(ctx, f, b);
            prof_begin(ctx, "k_aos_to_soa");
            k_aos_to_soa<<<grid_for(n), kThreads, 0, ctx->stream>>>(ctx->dbv, b, f, kFields[f].ncomp, lo[0], lo[1],
                                                                    lo[2], hi[0] - lo[0], hi[1] - lo[1],
                                                                    hi[2] - lo[2], ctx->staging + off);
            RUN(launched(ctx));
            off += n;
        }
    RUN(run_sync(ctx, "Ucell"));
    RUN(run_sync(ctx, "Bface"));
    RUN(launch_update_derived(ctx));
    RUN(build_graph(ctx));
    for (int s = 0; s < nsteps; ++s)
    {
        CK(ctx, cudaGraphLaunch(ctx->gexec, ctx->stream));
        ctx->launches += ctx->graph_kernels;
    }
    off = 0;
    for (int b = 0; b < ctx->nblocks; ++b)
        for (int f : {int(F_U), int(F_Bxi), int(F_Beta), int(F_Bzeta)})
        {
            int lo[3], hi[3];
            field_box(ctx, f, b, lo, hi);
            const int64_t n = field_count(ctx, f, b);
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
    if (!ctx)
        return MHD_EINVAL;
    switch (stage_id)
    {
    case MHD_STAGE_TIMESTEP:
        prof_begin(ctx, "k_begin_step");
        k_begin_step<<<1, 1, 0, ctx->stream>>>(ctx->dt_key, ctx->dt, ctx->err, ctx->prm.dt_abort);
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
            int64_t nf = 0;
            for (int l = LOC_FXI; l <= LOC_FZETA; ++l)
                nf = max_box(ctx, l, 0) > nf ? max_box(ctx, l, 0) : nf;
            prof_begin(ctx, "k_curl_e2f");
            k_curl_e2f<<<dim3(grid_for(nf), ctx->nblocks, 3), kThreads, 0, ctx->stream>>>(ctx->dbv, F_Exi, -1, F_Bxi,
                                                                                         -1.0, ctx->dt, 1.0);
            RUN(launched(ctx));
        }
        break;
    default:
        return fail(ctx, MHD_EINVAL, "unknown stage %d", stage_id);
    }
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    return check_err(ctx);
}

int mhd_get_time(mhd_ctx *ctx, double *dt, double *time, int64_t *step)
{
    if (!ctx)
        return MHD_EINVAL;
    double d[2];
    long long s = 0;
    CK(ctx, cudaMemcpy(d, ctx->dt, 16, cudaMemcpyDeviceToHost));
    CK(ctx, cudaMemcpy(&s, ctx->step, 8, cudaMemcpyDeviceToHost));
    if (dt)
        *dt = d[0];
    if (time)
        *time = d[1];
    if (step)
        *step = s;
    return MHD_OK;
}

int mhd_set_time(mhd_ctx *ctx, double dt, double time, int64_t step)
{
    if (!ctx)
        return MHD_EINVAL;
    const double d[2] = {dt, time};
    const long long s = step;
    CK(ctx, cudaMemcpy(ctx->dt, d, 16, cudaMemcpyHostToDevice));
    CK(ctx, cudaMemcpy(ctx->step, &s, 8, cudaMemcpyHostToDevice));
    return MHD_OK;
}

int64_t mhd_kernel_launches(const mhd_ctx *ctx) { return ctx ? ctx->launches : -1; }

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
    if (!ctx || !count || cap < 0)
        return MHD_EINVAL;
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
