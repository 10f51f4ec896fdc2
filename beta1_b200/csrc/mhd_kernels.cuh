// Kernel declarations shared by the C-ABI implementation.
#pragma once

#include "mhd_layout.cuh"
#include "mhd_pole.cuh"
#include "mhd_geom.cuh"
#include "mhd_output.cuh"
#include "../../include/beta1_mhd.h"

namespace mhd
{

// Nondimensional constants passed by value to the kernels.
struct Consts
{
    double gamma;
    double cfl;
    double inver_MA2;
    double mom_hall;
    double state_coeff;
    double M_H, M_ref;
    double ne_floor;
};

__global__ void k_fluid_rhs(const BlockView *bvs, Consts c, int64_t maxpts);
__global__ void k_ucontra(const BlockView *bvs);
__global__ void k_face_normals(const BlockView *bvs);
// Face / edge kernels run one thread per staggered point (i, j, k) in
// [0, n + 1)^3 and handle all three axes there.  rng (may be null): per
// block a region box lo[3], hi[3]; only points inside it are processed.
__global__ void k_update_u(const BlockView *bvs, const double *dtp);
__global__ void k_divb(const BlockView *bvs);
// mixed precision (mhd_kernels_mixed.cu)
__global__ void k_geom32(const BlockView *bvs);
__global__ void k_rk2(const BlockView *bvs, int save);
__global__ void k_hall_cell(const BlockView *bvs, Consts c, double hall_coef);
// the Hall edge EMF, variant 0: per-edge cell reads (no launch bounds), 1: the
// seven cells of a staggered point read once (at least 2 CTAs per SM); the
// same bits
int launch_k_hall_edge(int variant, dim3 grid, cudaStream_t st, const BlockView *bvs, const int *zb, int nzb);
__global__ void k_eres_explicit(const BlockView *bvs, double inver_Rem);
// calc_Bcell on the inner cells (2-D launch, one grid row per block); w32:
// from the FP32 weight copies (mixed form)
void launch_k_bcell(bool w32, dim3 grid, cudaStream_t st, const BlockView *bvs);
__global__ void k_jedge(const BlockView *bvs, int fB0, int fJ0, double mult, const int *rng);
__global__ void k_jcell(const BlockView *bvs);
// RHS = mult curl E and B = B* + dt RHS on the inner faces, B* from a snapshot
// (bs[3 * block + axis]: the snapshot's B arrays of each block, pool layout)
__global__ void k_curl_from_snapshot(const BlockView *bvs, int fE0, int fR0, int fB0, double mult, const double *dtp,
                                     const double *const *bs);
// J_cell on the inner cells over the flattened KIND_CELL0 grid (w32: FP32 weights)
void launch_k_jcell(bool w32, dim3 grid, cudaStream_t st, const BlockView *bvs);

// Pole handlers and repairs on eta Poles (mhd_pole.cuh): per Pole a
// (block, direction) pair in `poles`, one grid row per Pole
__global__ void k_pole(const BlockView *bvs, const int *poles, int op);
// Calc_J_Edge again on the J_xi / J_eta edges that read the B_zeta faces
// POLE_BZETA rewrote (staggered layers jc, jc + 1 of each Pole; grid.y: Poles)
__global__ void k_pole_jedge(const BlockView *bvs, const int *poles);
// one Pole operation over every Pole (work items per Pole: pole_work); the
// ring least squares run one warp per ring, with their geometry-only normal
// matrices in `cache` (per Pole, per least-squares operation, `stride`
// rings, 10 values each), which build = 1 fills (after every geometry change)
void launch_pole_op(int op, int64_t work, int npoles, cudaStream_t st, const BlockView *bvs, const int *poles,
                    double *cache, int stride, int build);
__global__ void k_geometry(const BlockView *bvs, int blk, NodeMesh m, int G, int group0, double b0, double b1,
                           double b2);
// output-step minima / maxima over the inner cells of a run's blocks (run < 0:
// every block); keys[0..DIAG_NMIN) minima, keys[DIAG_NMIN..DIAG_NMIN + DIAG_NQ) maxima
__global__ void k_diag_init(unsigned long long *keys);
__global__ void k_diag(const BlockView *bvs, int run, unsigned long long *keys);
__global__ void k_begin_step(const unsigned long long *dt_key, double *dt, int *err, double dt_abort, int nruns);
__global__ void k_arm_dt(unsigned long long *dt_key, int nruns);
__global__ void k_end_step(const double *dt, double *time, long long *step, int nruns);
__global__ void k_gather(double *pool, const uint64_t *dst, const uint64_t *src, int64_t n);
// the same with 32-bit pool offsets (pools of fewer than 2^32 points)
__global__ void k_gather32(double *pool, const uint32_t *dst, const uint32_t *src, int64_t n);
__global__ void k_set_consts(double *pool, const uint64_t *dst, const double *val, int64_t n);
__global__ void k_wall_u(const BlockView *bvs, int blk, int dir, double gamma);
__global__ void k_wall_u_all(const BlockView *bvs, const int *walls, double gamma);
__global__ void k_gather_stage(double *tmp, const double *pool, const uint64_t *src, int64_t n);
__global__ void k_scatter_stage(double *pool, const double *tmp, const uint64_t *dst, int64_t n);
__global__ void k_aos_to_soa(const BlockView *bvs, int blk, int fid, int ncomp, int lo0, int lo1, int lo2, int n0,
                             int n1, int n2, const double *aos);
__global__ void k_soa_to_aos(const BlockView *bvs, int blk, int fid, int ncomp, int lo0, int lo1, int lo2, int n0,
                             int n1, int n2, double *aos);

// Krylov (mhd_krylov.cu).  GMRES state kept on the device, including the
// loop control, so that a whole solve runs inside one CUDA graph (conditional
// while nodes) or, eagerly, with the host reading the two loop flags.
// Restart length at most kMaxRestart.
constexpr int kMaxRestart = 30;
struct GmresState
{
    double H[31 * 31]; // H[i * 31 + j]: row i, column j (upper Hessenberg, rotated in place)
    double cs[31], sn[31], g[32];
    double hcol[32]; // h of the current column, then ||w|| at hcol[j + 1]
    double resid;    // |g[j + 1]|
    double beta;     // initial residual norm of the cycle
    double y[31];
    int breakdown;
    // control
    int j;                  // columns built in the current cycle
    int its;                // iterations of the current solve
    int m, maxit;           // restart length, iteration limit
    double ttol, atol;      // max(rtol ||b||, atol), atol
    double bnorm;
    int reason;             // 0 running, 2 rtol, 3 atol, -3 iteration limit
    int inner, outer;       // loop conditions (mirrors of the graph conditionals)
    long long total_its;    // cumulative over all solves
    long long total_cycles; // cumulative over all solves
    unsigned int dot_done[32]; // CTAs finished per dot product (the last one sums the partials)
};
// The implicit resistive solve as one persistent (cooperative) kernel:
// GMRES(m) with the operator, the orthogonalisation and the control flow
// all on the device, CTAs meeting at grid barriers between phases.
struct DevCopy // fixed values then copies of a point list (apply_list)
{
    const uint64_t *cdst;
    const double *cval;
    int64_t nconst;
    const uint64_t *dst, *src;
    double *tmp; // staging when a source is also a destination
    int64_t n;
};
// One point-wise write list of the fused resistive operator: pool[dst[q]] =
// kind 0: x[idx] / div (an unknown), 1: val * (x[idx] / div) (an alias),
// 2: val (a fixed value), 3: pool[idx] (a point no phase writes),
// 4: -dt * (discrete curl of Eres at the face packed in idx, block blk)
struct FusedList
{
    const uint64_t *dst;
    const int *kind;
    const int64_t *idx;
    const double *val;
    const int *blk;
    int64_t n;
};
enum : int
{
    FUSE_UNKNOWN = 0,
    FUSE_ALIAS = 1,
    FUSE_CONST = 2,
    FUSE_POOL = 3,
    FUSE_CURL = 4
};
// face packed as ((fa * 4096 + i + 64) * 4096 + j + 64) * 4096 + k + 64
__host__ __device__ inline int64_t fuse_pack(int fa, int i, int j, int k)
{
    return ((int64_t(fa) * 4096 + (i + 64)) * 4096 + (j + 64)) * 4096 + (k + 64);
}

struct ResistSolve
{
    const BlockView *bvs;
    double *pool;
    int nblocks;
    const uint64_t *e, *dj, *j; // unknowns' offsets in Eres, dJ and J
    const double *eta;
    int64_t n;
    const uint64_t *alias; // aliases of unknown owners ...
    const int64_t *alias_of; // ... and the owner's unknown index
    const double *sign;
    int64_t nalias;
    DevCopy eres1form, db;
    const int *uloc; // per unknown: block, edge axis, i, j, k
    int merge1;      // Sync("Eres1form")'s fixed values may go with the unknowns' writes
    int merge2;      // Sync("dB")'s fixed values may go with the curl
    const int *rng; // per block region box
    int64_t nreg;   // points of the largest region box
    const double *dtp;
    double *V, *w, *x, *b, *r;
    double *partial; // 2 x 32 x gridDim.x
    GmresState *st;
    int m, maxit;
    double rtol, atol;
    unsigned *bar; // arrival count, generation
    int *err;      // set to MHD_EKRYLOV when a barrier wait gives up
    // fused operator phases (n < 0: not fused, the copy-list phases run):
    // A: every Eres point the unknowns' writes and Sync("Eres1form") set,
    // each as one expression of the basis vector; B: the Sync("dB") copies,
    // each as the curl at its source (or a fixed or unchanged value)
    FusedList fa, fb;
};
__global__ void k_gmres_resist(ResistSolve a);

// dot products out[c] = V_c . w for c < nvec (nvec = *jdev + 1 when jdev is
// given); V == nullptr computes w . w.  Each CTA stores its partial sum; the
// last CTA of each product adds the partials in a fixed order.
__global__ void k_dots(const double *V, int64_t ldv, int nvec, const double *w, int64_t n, double *partial,
                       const int *jdev, double *out, unsigned int *done);
__global__ void k_sub_proj(const double *V, int64_t ldv, int nvec, const double *h, double *w, int64_t n,
                           const int *jdev);
__global__ void k_add_small(double *a, const double *b, const int *jdev);
__global__ void k_div_guard(double *y, const double *x, const double *a, int64_t n, const int *guard);
__global__ void k_div_next(double *V, int64_t ldv, const double *w, const GmresState *st, int64_t n);
__global__ void k_gmres_init(GmresState *st, const double *b2, double rtol, double atol, int maxit, int m);
__global__ void k_cycle_start(GmresState *st, const double *beta2, cudaGraphConditionalHandle h, int use_handle);
__global__ void k_gmres_column(GmresState *st, const double *wnorm2);
__global__ void k_inner_check(GmresState *st, cudaGraphConditionalHandle h, int use_handle);
__global__ void k_gmres_solve_y(GmresState *st);
__global__ void k_add_basis(const double *V, int64_t ldv, const GmresState *st, double *x, int64_t n);
__global__ void k_outer_check(GmresState *st, cudaGraphConditionalHandle h, int use_handle);
__global__ void k_zero(double *x, int64_t n);
__global__ void k_residual(const double *b, const double *y, double *r, int64_t n);
// pool[dst[t]] = x[t] with x = x0 + (*jdev) * ldx when jdev is given
__global__ void k_scatter_vec(double *pool, const uint64_t *dst, const double *x0, int64_t ldx, const int *jdev,
                              int64_t n);
__global__ void k_resist_out(const double *pool, const uint64_t *e, const uint64_t *dj, const double *eta, double *y,
                             int64_t n);
__global__ void k_resist_rhs(const double *pool, const uint64_t *j, const double *eta, double *b, int64_t n);
__global__ void k_alias_copy(double *pool, const uint64_t *alias, const uint64_t *owner, const double *sign,
                             int64_t n);
__global__ void k_pack_vec(const double *pool, const uint64_t *src, double *x, int64_t n);

// Control state of the implicit Hall solve on the device: Newton with a
// backtracking line search around GMRES on finite-difference products.
// One-thread kernels update it and set the loop conditions (the graph's
// conditional handles inside a graph; the mirror flags, read by the host,
// when run eagerly).
struct HallCtl
{
    double f, f0, ft; // ||F|| of the iterate, of the initial guess, of the line-search trial
    double xnorm;     // ||X|| at the start of the Newton step
    double h;         // difference step of a product with a unit basis vector
    double hdx;       // ... with the correction dx (restart residual)
    double lambda;    // line-search step
    double rtol, atol;
    int it, maxit;    // Newton steps taken / allowed
    int cut;          // line-search halvings in this step
    int reason;       // 2 ||F|| <= atol, 3 ||F|| <= rtol ||F0||, -5 step limit
    int first;        // the first GMRES cycle of the Newton step (r = b, no product)
    int newton, ls, restart; // loop conditions
    long long lin0;          // cumulative GMRES iterations before this solve
    long long pass[3];       // cumulative: Newton steps, restart products, line-search trials
};
// products per multi-dot pass: up to kMaxRestart + 1 basis vectors and one norm
constexpr int kMdMax = 32;
__global__ void k_hall_begin(HallCtl *c, const double *f2, const GmresState *st, double rtol, double atol, int maxit,
                             cudaGraphConditionalHandle h, int use);
__global__ void k_hall_step_begin(HallCtl *c, const double *x2);
__global__ void k_hall_gmres_init(GmresState *st, const double *b2, double rtol, double atol, int maxit, int m,
                                  cudaGraphConditionalHandle hout, int use);
__global__ void k_hall_cycle_prep(HallCtl *c, const double *dx2, cudaGraphConditionalHandle h, int use);
__global__ void k_hall_ls_begin(HallCtl *c, cudaGraphConditionalHandle h, int use);
__global__ void k_hall_ls_check(HallCtl *c, const double *ft2, cudaGraphConditionalHandle h, int use);
__global__ void k_hall_accept(HallCtl *c, cudaGraphConditionalHandle h, int use);
__global__ void k_hall_column(GmresState *st, const double *d);
// Xt = X + (*a) v (v = v0 + (*jdev) ldv; Xt = X when a is null), written into the pool's unknowns
__global__ void k_hall_trial(double *pool, const uint64_t *e, const double *X, const double *a, const double *v0,
                             int64_t ldv, const int *jdev, double *Xt, int64_t n);
// w = ((Xt - pool[e]) - F) / *h and out[c] = V_c . w for c <= j
__global__ void k_hall_jv_dots(const double *pool, const uint64_t *e, const double *Xt, const double *F,
                               const double *h, double *w, const double *V, int64_t ldv, const GmresState *st,
                               int64_t n, double *partial, double *out, unsigned *done);
// w -= sum_c hcol[c] V_c; out[c] = V_c . w (c <= j), out[j + 1] = w . w
__global__ void k_hall_proj_dots(const double *V, int64_t ldv, const GmresState *st, double *w, int64_t n,
                                 double *partial, double *out, unsigned *done);
// V_{j+1} = (w - sum_c d[c] V_c) / hcol[j + 1]
__global__ void k_hall_next(double *V, int64_t ldv, const double *w, const GmresState *st, const double *d,
                            int64_t n);
// Ft = Xt - pool[e]; out[0] = Ft . Ft
__global__ void k_hall_res_dots(const double *pool, const uint64_t *e, const double *Xt, double *Ft, int64_t n,
                                double *partial, double *out, unsigned *done);
// r = b - ((Xt - pool[e]) - F) / *h
__global__ void k_hall_restart_r(const double *pool, const uint64_t *e, const double *Xt, const double *F,
                                 const double *h, const double *b, double *r, int64_t n);
// b = -F, r = b, dx = 0; out[0] = b . b
__global__ void k_hall_gmres_prologue(const double *F, double *b, double *r, double *dx, int64_t n, double *partial,
                                      double *out, unsigned *done);
// out[0] = x . x
__global__ void k_norm2(const double *x, int64_t n, double *partial, double *out, unsigned *done);
// X = Xt, F = Ft
__global__ void k_hall_take(double *X, const double *Xt, double *F, const double *Ft, int64_t n);
// dst = src over nseg segments (seg: dst offset, src offset, length)
__global__ void k_copy_segments(double *dst, const double *src, const int64_t *seg, int nseg);


// Hot stencil kernels in register / occupancy variants (the same code under
// different __launch_bounds__ minimum CTAs per SM; 0 = no launch bounds, the
// compiler's own allocation); variant 0 is the default.  Returns -1 for an
// unknown variant.
// k_pv_uplus_dt: minimum CTAs per SM 4, 0, 5, and variant 3: at 4 without
// J_cell, which launch_k_jcell computes in a pass of its own before it; w32:
// J_cell from the FP32 weight copies (mixed form)
int launch_k_pv_uplus_dt(int variant, bool w32, dim3 grid, cudaStream_t st, const BlockView *bvs, Consts c,
                         unsigned long long *dt_key, int depth, int with_jcell);
// k_fluid_ucontra: minimum CTAs per SM 0, 3
int launch_k_fluid_ucontra(int variant, dim3 grid, cudaStream_t st, const BlockView *bvs, Consts c);
// k_bcell_jedge: minimum CTAs per SM 0, 6; w32 as above
int launch_k_bcell_jedge(int variant, bool w32, dim3 grid, cudaStream_t st, const BlockView *bvs);
// k_eface: minimum CTAs per SM 0, 6
int launch_k_eface(int variant, dim3 grid, cudaStream_t st, const BlockView *bvs);
// k_curl_e2f: minimum CTAs per SM 0, 6
int launch_k_curl_e2f(int variant, dim3 grid, cudaStream_t st, const BlockView *bvs, int fE0, int fR0, int fB0,
                      double mult, const double *dtp, double dtdiv, int mult_is_neg_dt, const int *rng);
// k_eedge: minimum CTAs per SM 0, 8
int launch_k_eedge(int variant, dim3 grid, cudaStream_t st, const BlockView *bvs);
// k_fluid_mixed: minimum CTAs per SM 3, 0, 2
int launch_k_fluid_mixed(int variant, dim3 grid, cudaStream_t st, const BlockView *bvs, Consts c);

} // namespace mhd
