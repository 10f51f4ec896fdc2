// Matrix-free restarted GMRES on the device, replacing the PETSc KSPSolve of
// the implicit resistive step (Z4_Lunar/src/implicit/Lunar_ImplicitResistive.cpp:430-491).
//
// Vectors are dense over the solve's unknowns (owner edges with eta > 0).
// Orthogonalisation is classical Gram-Schmidt applied twice (CGS2): every
// pass needs only one batched dot-product kernel, instead of one reduction
// per basis vector with modified Gram-Schmidt.  All reductions are
// two-stage (per-CTA partial sums, then a fixed-order final sum), so a solve
// is bit-reproducible from run to run.
//
// The whole control state lives in device memory (GmresState): the
// Hessenberg matrix, the Givens rotations, the residual estimate, the column
// and iteration counters and the two loop conditions.  One-thread kernels
// update it and, when the solve runs inside a CUDA graph, set the graph's
// conditional handles (an inner while loop over Arnoldi steps, an outer one
// over restart cycles), so a solve needs no host round trip.  Run eagerly,
// the host reads the two loop flags instead.  Kernels that work on "column
// j" read j from the state.
#include "mhd_kernels.cuh"

namespace mhd
{

constexpr int kRedThreads = 256;

__global__ void k_dots(const double *__restrict__ V, int64_t ldv, int nvec, const double *__restrict__ w, int64_t n,
                       double *__restrict__ partial, const int *__restrict__ jdev, double *__restrict__ out,
                       unsigned int *__restrict__ done)
{
    const int c = blockIdx.y;
    const int nv = jdev ? jdev[0] + 1 : nvec;
    if (c >= nv)
        return;
    const double *v = V ? V + int64_t(c) * ldv : w;
    double s = 0.0;
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < n; t += int64_t(gridDim.x) * blockDim.x)
        s += v[t] * w[t];
    __shared__ double red[kRedThreads];
    __shared__ bool last;
    red[threadIdx.x] = s;
    __syncthreads();
    for (int off = blockDim.x / 2; off > 0; off >>= 1)
    {
        if (threadIdx.x < off)
            red[threadIdx.x] += red[threadIdx.x + off];
        __syncthreads();
    }
    if (threadIdx.x == 0)
    {
        partial[int64_t(c) * gridDim.x + blockIdx.x] = red[0];
        __threadfence();
        last = (atomicAdd(&done[c], 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (!last)
        return;
    // the last CTA: partials of product c in a fixed order
    double q = 0.0;
    for (int b = threadIdx.x; b < int(gridDim.x); b += blockDim.x)
        q += __ldcg(&partial[int64_t(c) * gridDim.x + b]);
    red[threadIdx.x] = q;
    __syncthreads();
    for (int off = blockDim.x / 2; off > 0; off >>= 1)
    {
        if (threadIdx.x < off)
            red[threadIdx.x] += red[threadIdx.x + off];
        __syncthreads();
    }
    if (threadIdx.x == 0)
    {
        out[c] = red[0];
        done[c] = 0u;
    }
}

// w -= sum_c h[c] V_c
__global__ void k_sub_proj(const double *__restrict__ V, int64_t ldv, int nvec, const double *__restrict__ h,
                           double *__restrict__ w, int64_t n, const int *__restrict__ jdev)
{
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= n)
        return;
    const int nv = jdev ? jdev[0] + 1 : nvec;
    double s = w[t];
    for (int c = 0; c < nv; ++c)
        s -= h[c] * V[int64_t(c) * ldv + t];
    w[t] = s;
}

// a[c] += b[c] for c <= j
__global__ void k_add_small(double *__restrict__ a, const double *__restrict__ b, const int *__restrict__ jdev)
{
    const int c = threadIdx.x;
    if (c <= jdev[0])
        a[c] += b[c];
}

// y = x / a[0] unless guard[0] == 0
__global__ void k_div_guard(double *__restrict__ y, const double *__restrict__ x, const double *__restrict__ a,
                            int64_t n, const int *__restrict__ guard)
{
    if (guard && guard[0] == 0)
        return;
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t < n)
        y[t] = x[t] / a[0];
}

// V_{j+1} = w / ||w|| (skipped on breakdown)
__global__ void k_div_next(double *__restrict__ V, int64_t ldv, const double *__restrict__ w,
                           const GmresState *__restrict__ st, int64_t n)
{
    if (st->breakdown)
        return;
    const int j = st->j;
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t < n)
        V[int64_t(j + 1) * ldv + t] = w[t] / st->hcol[j + 1];
}

// start of a solve: ||b||, the stopping threshold, counters
__device__ __forceinline__ void gmres_init_state(GmresState *st, const double *__restrict__ b2, double rtol,
                                                 double atol, int maxit, int m)
{
    const double bnorm = sqrt(b2[0]);
    st->bnorm = bnorm;
    st->ttol = fmax(rtol * bnorm, atol);
    st->atol = atol;
    st->maxit = maxit;
    st->m = m;
    st->its = 0;
    st->reason = 0;
    st->j = 0;
    st->inner = 0;
    st->outer = 1;
}

__global__ void k_gmres_init(GmresState *st, const double *__restrict__ b2, double rtol, double atol, int maxit, int m)
{
    gmres_init_state(st, b2, rtol, atol, maxit, m);
}

// start of a cycle: beta = ||r||, g = beta e1; decides whether the cycle runs
__global__ void k_cycle_start(GmresState *st, const double *__restrict__ beta2, cudaGraphConditionalHandle h,
                              int use_handle)
{
    const double beta = sqrt(beta2[0]);
    st->beta = beta;
    for (int i = 0; i < 32; ++i)
        st->g[i] = 0.0;
    st->g[0] = beta;
    st->resid = beta;
    st->breakdown = 0;
    st->j = 0;
    int go = 1;
    if (beta <= st->ttol)
    {
        st->reason = (beta <= st->atol) ? 3 : 2;
        go = 0;
    }
    else if (st->its >= st->maxit)
    {
        st->reason = -3;
        go = 0;
    }
    st->inner = go;
    if (use_handle)
        cudaGraphSetConditional(h, unsigned(go));
}

// new column j: hcol[j + 1] = ||w||, H[0..j+1, j] = hcol; apply the
// previous rotations, form a new one, update g and the residual estimate
__device__ __forceinline__ void gmres_rotate_column(GmresState *st)
{
    const int j = st->j;
    double *H = st->H;
    for (int i = 0; i <= j + 1; ++i)
        H[i * 31 + j] = st->hcol[i];
    for (int i = 0; i < j; ++i)
    {
        const double a = H[i * 31 + j], b = H[(i + 1) * 31 + j];
        H[i * 31 + j] = st->cs[i] * a + st->sn[i] * b;
        H[(i + 1) * 31 + j] = -st->sn[i] * a + st->cs[i] * b;
    }
    const double a = H[j * 31 + j], b = H[(j + 1) * 31 + j];
    const double den = sqrt(a * a + b * b);
    st->cs[j] = den > 0.0 ? a / den : 1.0;
    st->sn[j] = den > 0.0 ? b / den : 0.0;
    H[j * 31 + j] = den;
    H[(j + 1) * 31 + j] = 0.0;
    st->g[j + 1] = -st->sn[j] * st->g[j];
    st->g[j] = st->cs[j] * st->g[j];
    st->resid = fabs(st->g[j + 1]);
    st->breakdown = (st->hcol[j + 1] == 0.0) ? 1 : 0;
}

__global__ void k_gmres_column(GmresState *st, const double *__restrict__ wnorm2)
{
    st->hcol[st->j + 1] = sqrt(wnorm2[0]);
    gmres_rotate_column(st);
}

// end of an Arnoldi step: counters and the inner loop condition
__global__ void k_inner_check(GmresState *st, cudaGraphConditionalHandle h, int use_handle)
{
    st->its += 1;
    st->total_its += 1;
    st->j += 1;
    const int go = !(st->resid <= st->ttol || st->breakdown || st->j >= st->m || st->its >= st->maxit);
    st->inner = go;
    if (use_handle)
        cudaGraphSetConditional(h, unsigned(go));
}

// back substitution H y = g over the cycle's j columns
__global__ void k_gmres_solve_y(GmresState *st)
{
    const int m = st->j;
    for (int i = m - 1; i >= 0; --i)
    {
        double s = st->g[i];
        for (int q = i + 1; q < m; ++q)
            s -= st->H[i * 31 + q] * st->y[q];
        st->y[i] = s / st->H[i * 31 + i];
    }
}

// x += V y over the cycle's j columns
__global__ void k_add_basis(const double *__restrict__ V, int64_t ldv, const GmresState *__restrict__ st,
                            double *__restrict__ x, int64_t n)
{
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= n)
        return;
    const int m = st->j;
    double s = x[t];
    for (int c = 0; c < m; ++c)
        s += st->y[c] * V[int64_t(c) * ldv + t];
    x[t] = s;
}

// end of a cycle: converged (PETSc's default test), out of iterations, or restart
__global__ void k_outer_check(GmresState *st, cudaGraphConditionalHandle h, int use_handle)
{
    st->total_cycles += 1;
    int go = 0;
    if (st->reason != 0)
        go = 0;
    else if (st->resid <= st->ttol || st->breakdown)
        st->reason = (st->resid <= st->atol) ? 3 : 2;
    else if (st->its >= st->maxit)
        st->reason = -3;
    else
        go = 1;
    st->outer = go;
    if (use_handle)
        cudaGraphSetConditional(h, unsigned(go));
}

__global__ void k_zero(double *__restrict__ x, int64_t n)
{
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t < n)
        x[t] = 0.0;
}

// r = b - y
__global__ void k_residual(const double *__restrict__ b, const double *__restrict__ y, double *__restrict__ r,
                           int64_t n)
{
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t < n)
        r[t] = b[t] - y[t];
}

// ---------------------------------------------------------------------------
// Resistive operator pieces (LunarSolver::MatMultImplicitResistive_ and its
// helpers, Z4_Lunar/src/implicit/Lunar_ImplicitResistive.cpp:264-427)
// ---------------------------------------------------------------------------

// pool[dst[t]] = x[t]   (UnpackVecToImplicitEres_)
__global__ void k_scatter_vec(double *__restrict__ pool, const uint64_t *__restrict__ dst,
                              const double *__restrict__ x0, int64_t ldx, const int *__restrict__ jdev, int64_t n)
{
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= n)
        return;
    const double *x = jdev ? x0 + int64_t(jdev[0]) * ldx : x0;
    pool[dst[t]] = x[t];
}

// y[t] = pool[e[t]] - eta[t] * pool[dj[t]]   (end of MatMultImplicitResistive_)
__global__ void k_resist_out(const double *__restrict__ pool, const uint64_t *__restrict__ e,
                             const uint64_t *__restrict__ dj, const double *__restrict__ eta, double *__restrict__ y,
                             int64_t n)
{
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t < n)
        y[t] = pool[e[t]] - eta[t] * pool[dj[t]];
}

// b[t] = 0.0 + eta[t] * pool[j[t]]   (PackImplicitJedgeToVec_ with multiply_eta)
__global__ void k_resist_rhs(const double *__restrict__ pool, const uint64_t *__restrict__ j,
                             const double *__restrict__ eta, double *__restrict__ b, int64_t n)
{
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t < n)
        b[t] = 0.0 + eta[t] * pool[j[t]];
}

// alias <- sign * owner (HALO_OWNER::sync_edge_1form)
__global__ void k_alias_copy(double *__restrict__ pool, const uint64_t *__restrict__ alias,
                             const uint64_t *__restrict__ owner, const double *__restrict__ sign, int64_t n)
{
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t < n)
        pool[alias[t]] = sign[t] * pool[owner[t]];
}

// ---------------------------------------------------------------------------
// Vector pieces of the implicit Hall Newton-Krylov solve
// (ImplicitHallSolver::SolveOneStep / FormFunction_,
// Z4_Lunar/src/implicit/Hall_Implicit_Solver.cpp:268-391, Hall_Implicit_Formfunction.cpp:7-106)
// ---------------------------------------------------------------------------

// x[t] = pool[src[t]]   (pack an edge field into a vector)
__global__ void k_pack_vec(const double *__restrict__ pool, const uint64_t *__restrict__ src, double *__restrict__ x,
                           int64_t n)
{
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t < n)
        x[t] = pool[src[t]];
}


// ---------------------------------------------------------------------------
// The implicit Hall solve steered on the device (ImplicitHallSolver::
// SolveOneStep, Z4_Lunar/src/implicit/Hall_Implicit_Solver.cpp:268-391):
// one-thread control kernels over HallCtl, and vector passes that fuse the
// finite-difference product, the Gram-Schmidt projections and the dot
// products a GMRES step needs (three passes over the basis per step).
// ---------------------------------------------------------------------------

namespace
{
__device__ __forceinline__ void set_cond(cudaGraphConditionalHandle h, int use, int v)
{
    if (use)
        cudaGraphSetConditional(h, unsigned(v));
}

// sqrt of the FP64 unit roundoff: the relative difference step
__device__ __forceinline__ double fd_scale() { return sqrt(2.220446049250313e-16); }

// the Newton loop test of SNESSolve's default convergence test
__device__ void hall_newton_test(HallCtl *c, cudaGraphConditionalHandle h, int use)
{
    int go = 0;
    if (c->f <= c->atol)
        c->reason = 2;
    else if (c->f <= c->rtol * c->f0)
        c->reason = 3;
    else if (c->it >= c->maxit)
        c->reason = -5;
    else
        go = 1;
    c->newton = go;
    set_cond(h, use, go);
}

// Grid reductions in a fixed order, so every pass is reproducible: each CTA
// adds its threads' sums (warp shuffles, then the warps in order) into one
// partial per product; the last CTA to finish adds the partials in CTA
// order.  Products are taken in chunks of at most kChunk per pass over the
// vectors (registers per thread stay bounded whatever the basis size).
constexpr int kChunk = 8;

// the CTA's partial sums of products c0 + q (q < N, c0 + q < nd)
template <int N>
__device__ __forceinline__ void block_partials(const double (&acc)[N], int c0, int nd, double *__restrict__ partial)
{
    constexpr int kWarps = kRedThreads / 32;
    __shared__ double red[N][kWarps];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < N; ++q)
        if (c0 + q < nd)
        {
            double v = acc[q];
            for (int o = 16; o > 0; o >>= 1)
                v += __shfl_down_sync(0xffffffffu, v, o);
            if (lane == 0)
                red[q][wid] = v;
        }
    __syncthreads();
    if (int(threadIdx.x) < N && c0 + int(threadIdx.x) < nd)
    {
        double s = 0.0;
        for (int w = 0; w < kWarps; ++w)
            s += red[threadIdx.x][w];
        partial[int64_t(c0 + int(threadIdx.x)) * gridDim.x + blockIdx.x] = s;
    }
    __syncthreads();
}

// out[c] for c < nd from the CTAs' partials, by the last CTA to arrive
__device__ void grid_finish(int nd, const double *__restrict__ partial, double *__restrict__ out,
                            unsigned *__restrict__ done)
{
    constexpr int kWarps = kRedThreads / 32;
    __shared__ bool last;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0)
        last = (atomicAdd(done, 1u) == gridDim.x - 1);
    __syncthreads();
    if (!last)
        return;
    __threadfence();
    for (int c = wid; c < nd; c += kWarps)
    {
        double s = 0.0;
        for (int b = lane; b < int(gridDim.x); b += 32)
            s += __ldcg(&partial[int64_t(c) * gridDim.x + b]);
        for (int o = 16; o > 0; o >>= 1)
            s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0)
            out[c] = s;
    }
    if (threadIdx.x == 0)
        *done = 0u;
}
} // namespace

__global__ void k_hall_begin(HallCtl *c, const double *__restrict__ f2, const GmresState *__restrict__ st, double rtol,
                             double atol, int maxit, cudaGraphConditionalHandle h, int use)
{
    c->f = sqrt(f2[0]);
    c->f0 = c->f;
    c->rtol = rtol;
    c->atol = atol;
    c->maxit = maxit;
    c->it = 0;
    c->reason = -5;
    c->lin0 = st->total_its;
    hall_newton_test(c, h, use);
}

// start of a Newton step: ||X|| and the difference step of unit vectors
__global__ void k_hall_step_begin(HallCtl *c, const double *__restrict__ x2)
{
    c->xnorm = sqrt(x2[0]);
    c->h = fd_scale() * (1.0 + c->xnorm) / 1.0;
    c->first = 1;
}

__global__ void k_hall_gmres_init(GmresState *st, const double *__restrict__ b2, double rtol, double atol, int maxit,
                                  int m, cudaGraphConditionalHandle hout, int use)
{
    gmres_init_state(st, b2, rtol, atol, maxit, m);
    set_cond(hout, use, 1);
}

// top of a GMRES cycle: a restart needs r = b - J dx, one product with dx
// (none on the first cycle, where r = b, nor when dx = 0)
__global__ void k_hall_cycle_prep(HallCtl *c, const double *__restrict__ dx2, cudaGraphConditionalHandle h, int use)
{
    const double dn = sqrt(dx2[0]);
    const int go = !c->first && dn > 0.0;
    if (go)
    {
        c->hdx = fd_scale() * (1.0 + c->xnorm) / dn;
        c->pass[1] += 1;
    }
    c->first = 0;
    c->restart = go;
    set_cond(h, use, go);
}

__global__ void k_hall_ls_begin(HallCtl *c, cudaGraphConditionalHandle h, int use)
{
    c->lambda = 1.0;
    c->cut = 0;
    c->ls = 1;
    set_cond(h, use, 1);
}

// backtracking: accept when ||F(X + lambda dx)|| <= (1 - 1e-4 lambda) ||F(X)||,
// else halve lambda, at most 12 trials (the last one is taken regardless)
__global__ void k_hall_ls_check(HallCtl *c, const double *__restrict__ ft2, cudaGraphConditionalHandle h, int use)
{
    const double ft = sqrt(ft2[0]);
    c->ft = ft;
    c->pass[2] += 1;
    int go = 0;
    if (!(ft <= (1.0 - 1e-4 * c->lambda) * c->f) && c->cut < 11)
    {
        c->lambda *= 0.5;
        c->cut += 1;
        go = 1;
    }
    c->ls = go;
    set_cond(h, use, go);
}

__global__ void k_hall_accept(HallCtl *c, cudaGraphConditionalHandle h, int use)
{
    c->f = c->ft;
    c->it += 1;
    c->pass[0] += 1;
    hall_newton_test(c, h, use);
}

// the column of a CGS2 step whose second pass gave d: h += d, and
// ||w''||^2 = ||w'||^2 - ||d||^2 (w'' = w' - V d with V orthonormal)
__global__ void k_hall_column(GmresState *st, const double *__restrict__ d)
{
    const int j = st->j;
    double s2 = d[j + 1];
    for (int c = 0; c <= j; ++c)
    {
        st->hcol[c] += d[c];
        s2 -= d[c] * d[c];
    }
    st->hcol[j + 1] = sqrt(fmax(s2, 0.0));
    gmres_rotate_column(st);
}

__global__ void k_hall_trial(double *__restrict__ pool, const uint64_t *__restrict__ e, const double *__restrict__ X,
                             const double *__restrict__ a, const double *__restrict__ v0, int64_t ldv,
                             const int *__restrict__ jdev, double *__restrict__ Xt, int64_t n)
{
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= n)
        return;
    double x = X[t];
    if (a)
    {
        const double *v = jdev ? v0 + int64_t(jdev[0]) * ldv : v0;
        x = x + a[0] * v[t];
    }
    if (Xt)
        Xt[t] = x;
    pool[e[t]] = x;
}

__global__ void __launch_bounds__(kRedThreads) k_hall_jv_dots(const double *__restrict__ pool,
                                                              const uint64_t *__restrict__ e,
                                                              const double *__restrict__ Xt,
                                                              const double *__restrict__ F,
                                                              const double *__restrict__ h, double *__restrict__ w,
                                                              const double *__restrict__ V, int64_t ldv,
                                                              const GmresState *__restrict__ st, int64_t n,
                                                              double *__restrict__ partial, double *__restrict__ out,
                                                              unsigned *__restrict__ done)
{
    const int nv = st->j + 1;
    const double hh = h[0];
    const int64_t t0 = int64_t(blockIdx.x) * blockDim.x + threadIdx.x, ts = int64_t(gridDim.x) * blockDim.x;
    for (int c0 = 0; c0 < nv; c0 += kChunk)
    {
        double acc[kChunk];
#pragma unroll
        for (int q = 0; q < kChunk; ++q)
            acc[q] = 0.0;
        for (int64_t t = t0; t < n; t += ts)
        {
            double wt;
            if (c0 == 0)
            {
                wt = ((Xt[t] - pool[e[t]]) - F[t]) / hh;
                w[t] = wt;
            }
            else
                wt = w[t];
#pragma unroll
            for (int q = 0; q < kChunk; ++q)
                if (c0 + q < nv)
                    acc[q] += V[int64_t(c0 + q) * ldv + t] * wt;
        }
        block_partials(acc, c0, nv, partial);
    }
    grid_finish(nv, partial, out, done);
}

__global__ void __launch_bounds__(kRedThreads) k_hall_proj_dots(const double *__restrict__ V, int64_t ldv,
                                                                const GmresState *__restrict__ st,
                                                                double *__restrict__ w, int64_t n,
                                                                double *__restrict__ partial,
                                                                double *__restrict__ out, unsigned *__restrict__ done)
{
    __shared__ double hs[kMdMax];
    const int nv = st->j + 1;
    if (int(threadIdx.x) < nv)
        hs[threadIdx.x] = st->hcol[threadIdx.x];
    __syncthreads();
    const int64_t t0 = int64_t(blockIdx.x) * blockDim.x + threadIdx.x, ts = int64_t(gridDim.x) * blockDim.x;
    // the subtraction, the first chunk of products and w . w in one pass
    {
        double acc[kChunk], self[1] = {0.0};
#pragma unroll
        for (int q = 0; q < kChunk; ++q)
            acc[q] = 0.0;
        for (int64_t t = t0; t < n; t += ts)
        {
            double wt = w[t];
#pragma unroll 4
            for (int c = 0; c < nv; ++c)
                wt -= hs[c] * V[int64_t(c) * ldv + t];
            w[t] = wt;
            self[0] += wt * wt;
#pragma unroll
            for (int q = 0; q < kChunk; ++q)
                if (q < nv)
                    acc[q] += V[int64_t(q) * ldv + t] * wt;
        }
        block_partials(acc, 0, nv, partial);
        block_partials(self, nv, nv + 1, partial);
    }
    for (int c0 = kChunk; c0 < nv; c0 += kChunk)
    {
        double acc[kChunk];
#pragma unroll
        for (int q = 0; q < kChunk; ++q)
            acc[q] = 0.0;
        for (int64_t t = t0; t < n; t += ts)
        {
            const double wt = w[t];
#pragma unroll
            for (int q = 0; q < kChunk; ++q)
                if (c0 + q < nv)
                    acc[q] += V[int64_t(c0 + q) * ldv + t] * wt;
        }
        block_partials(acc, c0, nv, partial);
    }
    grid_finish(nv + 1, partial, out, done);
}

__global__ void k_hall_next(double *__restrict__ V, int64_t ldv, const double *__restrict__ w,
                            const GmresState *__restrict__ st, const double *__restrict__ d, int64_t n)
{
    if (st->breakdown)
        return;
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= n)
        return;
    const int j = st->j;
    double s = w[t];
    for (int c = 0; c <= j; ++c)
        s -= d[c] * V[int64_t(c) * ldv + t];
    V[int64_t(j + 1) * ldv + t] = s / st->hcol[j + 1];
}

__global__ void __launch_bounds__(kRedThreads) k_hall_res_dots(const double *__restrict__ pool,
                                                               const uint64_t *__restrict__ e,
                                                               const double *__restrict__ Xt, double *__restrict__ Ft,
                                                               int64_t n, double *__restrict__ partial,
                                                               double *__restrict__ out, unsigned *__restrict__ done)
{
    double acc[1] = {0.0};
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < n; t += int64_t(gridDim.x) * blockDim.x)
    {
        const double f = Xt[t] - pool[e[t]];
        Ft[t] = f;
        acc[0] += f * f;
    }
    block_partials(acc, 0, 1, partial);
    grid_finish(1, partial, out, done);
}

__global__ void k_hall_restart_r(const double *__restrict__ pool, const uint64_t *__restrict__ e,
                                 const double *__restrict__ Xt, const double *__restrict__ F,
                                 const double *__restrict__ h, const double *__restrict__ b, double *__restrict__ r,
                                 int64_t n)
{
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t < n)
        r[t] = b[t] - ((Xt[t] - pool[e[t]]) - F[t]) / h[0];
}

__global__ void __launch_bounds__(kRedThreads) k_hall_gmres_prologue(const double *__restrict__ F,
                                                                     double *__restrict__ b, double *__restrict__ r,
                                                                     double *__restrict__ dx, int64_t n,
                                                                     double *__restrict__ partial,
                                                                     double *__restrict__ out,
                                                                     unsigned *__restrict__ done)
{
    double acc[1] = {0.0};
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < n; t += int64_t(gridDim.x) * blockDim.x)
    {
        const double v = -F[t];
        b[t] = v;
        r[t] = v;
        dx[t] = 0.0;
        acc[0] += v * v;
    }
    block_partials(acc, 0, 1, partial);
    grid_finish(1, partial, out, done);
}

__global__ void __launch_bounds__(kRedThreads) k_norm2(const double *__restrict__ x, int64_t n,
                                                       double *__restrict__ partial, double *__restrict__ out,
                                                       unsigned *__restrict__ done)
{
    double acc[1] = {0.0};
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < n; t += int64_t(gridDim.x) * blockDim.x)
        acc[0] += x[t] * x[t];
    block_partials(acc, 0, 1, partial);
    grid_finish(1, partial, out, done);
}

__global__ void k_hall_take(double *__restrict__ X, const double *__restrict__ Xt, double *__restrict__ F,
                            const double *__restrict__ Ft, int64_t n)
{
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t < n)
    {
        X[t] = Xt[t];
        F[t] = Ft[t];
    }
}

__global__ void k_copy_segments(double *__restrict__ dst, const double *__restrict__ src,
                                const int64_t *__restrict__ seg, int nseg)
{
    const int s = blockIdx.y;
    if (s >= nseg)
        return;
    const int64_t d0 = seg[3 * s], s0 = seg[3 * s + 1], len = seg[3 * s + 2];
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < len; t += int64_t(gridDim.x) * blockDim.x)
        dst[d0 + t] = src[s0 + t];
}
} // namespace mhd
