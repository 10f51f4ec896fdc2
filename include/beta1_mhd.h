/*
 * beta1_mhd.h -- C ABI of the B200 (sm_100a) per-timestep MHD hot path.
 *
 * One context holds every block of a multi-block structured grid on one GPU,
 * one CUDA stream, the device copies of the solver's fields and the gather
 * tables of its boundary/halo synchronisations.  All entry points return 0 on
 * success and a positive MHD_E* code otherwise; nothing here exits or throws.
 * A context is not thread-safe; different contexts are independent.  A
 * context lives on the CUDA device that was current when it was created;
 * every entry point makes that device current for the duration of the call
 * and restores the caller's current device before it returns.
 *
 * Field data cross this boundary in the reference's own host layout: a field
 * on block b is the half-open logical box [lo, hi) of its stagger location
 * (include/3_field/1_Field_Block.h:29-35, src/3_field/1_Field_Block.cpp:51-131),
 * stored as float64 in (i, j, k, m) order with the component m fastest
 * (include/3_field/Field_Array.h:177).  Field names are the reference's
 * (Z4_Lunar/main.cpp:61-123, src/3_field/4_MPCNS_Geometry.cpp:4-69).
 *
 * Each entry point below names the reference interface it replaces.
 */
#ifndef BETA1_MHD_H
#define BETA1_MHD_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define MHD_OK 0
#define MHD_EINVAL 1      /* bad argument (unknown name, size mismatch, null) */
#define MHD_ECUDA 2       /* a CUDA runtime call failed */
#define MHD_ENOMEM 3      /* device or host allocation failed */
#define MHD_EDT 4         /* time step underflow or NaN (dt < dt_abort) */
#define MHD_ESTATE 5      /* call out of order (e.g. step before set-up) */
#define MHD_EKRYLOV 6     /* a persistent Krylov solve gave up waiting at a grid barrier (a solve that
                             does not converge is no error: it continues, as the reference does,
                             with the reason in mhd_resistive_stats) */

/* stagger locations, numbered as the reference's restart writer does
   (src/5_io/IOModule_Bin.cpp:62-85) */
#define MHD_LOC_CELL 0
#define MHD_LOC_FACE_XI 1
#define MHD_LOC_FACE_ETA 2
#define MHD_LOC_FACE_ZETA 3
#define MHD_LOC_EDGE_XI 4
#define MHD_LOC_EDGE_ETA 5
#define MHD_LOC_EDGE_ZETA 6

/* precision of the flux / EMF / Krylov-operator arithmetic */
#define MHD_PREC_FP64 0   /* FP64 throughout, operation order of the reference */
#define MHD_PREC_MIXED 1  /* FP32 face fluxes, FP64 CT, state and residuals */

typedef struct mhd_ctx mhd_ctx;

/* Cell counts of one block (Block::mx/my/mz, include/1_grid/1_MPCNS_Grid.h:34-44). */
typedef struct
{
    int32_t ni, nj, nk;
} mhd_block_desc;

/* Nondimensional constants of the solver, as LunarSolver::calc_physical_constant
   computes them (Z4_Lunar/src/physics/LunarSolver_Tools.cpp:3-45). */
typedef struct
{
    double gamma;               /* ratio of specific heats */
    double cfl;                 /* CFL number of Compute_Timestep */
    double inver_MA2;           /* 1 / Alfven Mach^2 scale of v_A^2 */
    double momentum_hall_coeff; /* J x B force coefficient */
    double state_coeff;         /* p = rho T state_coeff */
    double M_H, M_ref;          /* molar masses in Hall_Num_Limiter */
    double ne_hall_floor;       /* electron-density floor of Hall_Num_Limiter */
    double dt_abort;            /* abort threshold of Compute_Timestep (1e-7) */
    int32_t ngg;                /* ghost layers of the state fields (4) */
    int32_t precision;          /* MHD_PREC_* */
} mhd_params;

/* LunarSolver ctor + Field registration (Z4_Lunar/src/LunarSolver.cpp:12-235,
   Z4_Lunar/main.cpp:57-123): allocates every hot-path field of every block
   on the current CUDA device, zero-filled. */
int mhd_ctx_create(const mhd_block_desc *blocks, int32_t nblocks, const mhd_params *params, mhd_ctx **out);

/* A batch of independent runs in one context (no counterpart in the
   reference, which advances one grid per process): run_of_block[b] in
   [0, nruns) names the run of block b, every run owns at least one block.
   Each run has its own time step (the CFL minimum over its own blocks), time
   and step count; the blocks of all runs advance together, every hot-path
   stage as one launch whose grid holds exactly the CTAs of every block
   (blocks of uneven sizes waste no CTAs), and the whole step is one CUDA
   graph.  Blocks of different runs share no halo: the sync tables the caller
   installs connect blocks of the same run only.  Every other entry point
   works on a batch, with block indices over all runs; mhd_step and
   mhd_get_time report run 0, mhd_run_time any run.  The implicit resistive
   and Hall solves and the explicit resistive sub-cycles are rejected on a
   batch (MHD_ESTATE). */
int mhd_batch_create(const mhd_block_desc *blocks, int32_t nblocks, const int32_t *run_of_block, int32_t nruns,
                     const mhd_params *params, mhd_ctx **out);

/* dt of the last step, simulated time and step count of one run. */
int mhd_run_time(mhd_ctx *ctx, int32_t run, double *dt, double *time, int64_t *step);

/* nsteps steps of every run of a batch (each run its own dt), then every
   run's last dt and time into dt_out[nruns] and time_out[nruns] (either may
   be null; nruns must be the batch's run count, or 0 for no read-back). */
int mhd_batch_step(mhd_ctx *ctx, int32_t nsteps, double *dt_out, double *time_out, int32_t nruns);

/* ~LunarSolver / delete fld (Z4_Lunar/main.cpp:216-222). */
int mhd_ctx_destroy(mhd_ctx *ctx);

/* Message of the last failing call on this context (NUL-terminated). */
int mhd_last_error(const mhd_ctx *ctx, char *buf, int32_t buflen);

/* Descriptor of a named field: location, components, ghost layers and the
   logical box [lo, hi) on block `block` (FieldBlock::get_lo/get_hi,
   include/3_field/1_Field_Block.h:29-35). */
int mhd_field_info(const mhd_ctx *ctx, const char *name, int32_t block, int32_t *loc, int32_t *ncomp,
                   int32_t *nghost, int32_t lo[3], int32_t hi[3]);

/* FieldBlock host storage <-> device (the reference reads/writes FieldBlock
   storage directly, src/3_field/1_Field_Block.cpp:3-25).  `data` holds the
   field's full logical box in AoS order; `count` must equal its size. */
int mhd_upload_field(mhd_ctx *ctx, const char *name, int32_t block, const double *data, int64_t count);
int mhd_download_field(mhd_ctx *ctx, const char *name, int32_t block, double *data, int64_t count);

/* Allocation-free read-out.  No counterpart in the reference: its drivers
   read FieldBlock storage directly.  Same result as mhd_download_field, but
   the device-side AoS staging goes through a fixed array of
   MHD_NOALLOC_MAX_DOUBLES doubles (16 MiB) compiled into the library, instead
   of a staging buffer the context allocates on first use.  Every GPU that
   loads the library holds that array until the process exits.

   Callers that cannot allocate:
   - a driver that writes an emergency restart dump after a device allocation
     has failed, where a further cudaMalloc would fail too;
   - a driver that hands the GPU's memory to its own pool up front, sizing the
     solver's blocks to fill it, so that no memory is left at output steps.

   Limits and rules:
   - A field of one block larger than MHD_NOALLOC_MAX_DOUBLES values is
     rejected with MHD_EINVAL.
   - The context must have taken at least one step (mhd_step or
     mhd_batch_step) before the call, so that every sync table the read-out
     may replay is already on the device.  Otherwise the call returns
     MHD_ESTATE.
   - The array's device address on the context's GPU is looked up when the
     context is created (mhd_ctx_create / mhd_batch_create), so the read-out
     itself does no set-up.
   - All calls share the one array, whichever context makes them.  Each call
     overwrites the part it uses and waits for its copy to finish before it
     returns; the array keeps the last call's values.  Calls that overlap on
     the same GPU (other host threads, other contexts) race. */
#define MHD_NOALLOC_MAX_DOUBLES (1 << 21)
int mhd_download_field_noalloc(mhd_ctx *ctx, const char *name, int32_t block, double *data, int64_t count);

/* Field table of the library (no context, no GPU needed): name, location,
   components and ghost layers of field `index`; MHD_EINVAL past the end.
   A point id (below) is (index << 56) | (block << 40) | AoS offset of the
   point within the field's logical box on that block. */
int mhd_field_spec(int32_t index, const char **name, int32_t *loc, int32_t *ncomp, int32_t *nghost);

/* Point id of (field, block, i, j, k, m) for the gather tables below. */
int64_t mhd_point_id(const mhd_ctx *ctx, const char *name, int32_t block, int32_t i, int32_t j, int32_t k,
                     int32_t m);

/* Compiled boundary synchronisation of one group (LunarBoundary::Sync,
   Z4_Lunar/src/boundary/Boundary.cpp:30-40 and Boundary_Sync_.cpp:4-65:
   physical handlers, corner defaults, face/edge/vertex halos of
   src/4_halo/1_MPCNS_Halo_Inner.cpp:3-217).  The group's whole ordered
   sequence of copies is given as its composition: after the sync, point
   dst[n] holds the value point src[n] had before it.  Groups: "Ucell",
   "Bface", "Eface", "Eedge", "B_cell", "Jedge", "J_cell", "Uplus",
   "Eres", "Eres1form", "dB", "Badd". */
int mhd_set_sync_map(mhd_ctx *ctx, const char *group, const int64_t *dst, const int64_t *src, int64_t n);

/* Phase A of a group's sync, run before its composed copies: points that
   the physical handlers set to fixed values (the Farfield state of
   BC_UH_Farfield_H_ and BC_Farfield_Bface, the zero-curl edge EMF of
   BC_Farfield_Eedge_set_zerocurl, the zeroed wall layers of
   BC_Solid_Surface_Jcell / BC_Solid_Surface_Eface_*, Z4_Lunar/src/boundary/
   Boundary_Condition*.cpp), and the Solid_Surface fluid handler
   BC_Solid_Surface_ (Boundary_Condition_Fluid.cpp:19-185) on a block face
   (direction +-1, +-2, +-3 as in PhysicalPatch::direction). */
int mhd_set_sync_consts(mhd_ctx *ctx, const char *group, const int64_t *dst, const double *val, int64_t n);
int mhd_set_sync_wall(mhd_ctx *ctx, const char *group, int32_t block, int32_t direction);

/* Pole patches (the "Pole" boundary of Z4_Lunar/src/boundary/Boundary_Build.cpp:27-269)
   on a block face j = 0 (direction -2) or j = n_j (direction +2) whose
   ring runs around the k direction (k periodic onto itself).  From then on
   every Sync of the context runs in the topology order of the Pole shell
   (Pole, Pole, Farfield, Solid_Surface, Boundary_Sync_.cpp:4-65): the Pole
   rings the handlers compute (BC_Pole_Cell_, BC_Pole_Bcell_Collapse_,
   BC_Pole_Bface_Collapse_, BC_Pole_Eedge_Axis, BC_Pole_Eedge_RegulateK_Norm,
   BC_Pole_Jedge_RegulateK_Norm, and in the resistive groups Eres / Eres1form
   the regulation of Eres_eta), the composed copies of mhd_set_sync_map
   (sources read after the rings, before the wall handlers), the wall
   handlers, the copies of mhd_set_sync_map_post (sources the wall handlers
   wrote), then the fixed values of mhd_set_sync_consts.  The derived-field
   pass adds the Pole repairs of Z4_Lunar/src/physics/LunarSolver_Tools.cpp
   (B_zeta of the first cell layer after Sync("B_cell"), :242-307; the
   least-squares J_cell of the pole shell, :945-1090) and MHD_STAGE_DIVB
   zeroes divB there (:729-772); the explicit resistive sub-cycles
   (mhd_set_resistive_explicit) run the same repairs in each sub-cycle's
   UpdateMagneticDerivedFields_.  Needs the geometry field Astar_eta.  Not
   available with the implicit resistive or implicit Hall solves (MHD_ESTATE). */
int mhd_set_pole(mhd_ctx *ctx, int32_t block, int32_t direction);

/* Geometry of a block built on the device from its ghost node mesh
   (Block::Add_ghostmesh and, with Poles, Grid::MeshTrans_Inner_Pole done by
   the caller): JDxi/JDet/JDze, Jac, Area_*, beta_*, dl_*, Astar_*, alpha_*,
   dr_*, Bcell_from_Bface_w and Jcell_from_Jedge_w on their reference extents
   (src/3_field/4_MPCNS_Geometry.cpp:4-640, Z4_Lunar/src/LunarSolver.cpp:243-915),
   in place of uploading each with mhd_upload_field; with B_imf (3 values, or
   null) not zero also Badd_* = B_imf . JD.  nodes: (n_i + 1 + 2 (G + 1)) x
   (n_j + ...) x (n_k + ...) x 3 doubles, G = mhd_params.ngg, logical node
   (i, j, k) at ((i + G + 1) * NJ + j + G + 1) * NK + k + G + 1, x y z last. */
int mhd_build_geometry(mhd_ctx *ctx, int32_t block, const double *nodes, int64_t count, const double *B_imf);

/* Output-step diagnostics of LunarSolver::PrintMinMaxDiagnostics_
   (Z4_Lunar/src/tools/LunarSolver_PrintDiag.cpp:7-85) over the inner cells of
   a run's blocks (run -1: every block): mins[6] = the minima of rho, p, Bx,
   By, Bz, |B|^2 / 2, maxs[7] = their maxima and max |divB| (NaN values are
   skipped).  Reads U_H, PV_H, B_cell and divB: call MHD_STAGE_DIVB first, as
   the reference calls calc_divB first. */
int mhd_diagnostics(mhd_ctx *ctx, int32_t run, double *mins, double *maxs);
int mhd_set_sync_map_post(mhd_ctx *ctx, const char *group, const int64_t *dst, const int64_t *src, int64_t n);

/* Implicit resistive step (LunarSolver::SolveImplicitResistiveDiffusion_,
   Z4_Lunar/src/implicit/Lunar_ImplicitResistive.cpp:430-518, with the
   PETSc KSPSolve/MatShell of :95-124 replaced by a device GMRES): unknowns
   are Eres_xi/Eres_eta/Eres_zeta point ids of the owner edges with eta > 0
   in solve order (BuildImplicitResistiveEdgeDofMap_, :147-164), `eta` their
   resistivity; alias/owner/sign is the edge 1-form sync table
   (HALO_OWNER::sync_edge_1form).  Convergence: ||r|| <= max(rtol ||b||, atol)
   from x = 0, at most maxit iterations, restart <= 30.  Enables the solve in
   every following StepOnce. */
int mhd_set_resistive(mhd_ctx *ctx, int64_t n, const int64_t *unknowns, const double *eta, int64_t nalias,
                      const int64_t *alias, const int64_t *owner, const double *sign, double rtol, double atol,
                      int32_t maxit, int32_t restart);

/* Hall edge EMF set-up (LunarSolver::BuildHallFaceEMF_Rusanov_diff_,
   Z4_Lunar/src/physics/LunarSolver_MagExplicit_Hall.cpp:8-457): the Hall
   coefficient (hall_coef of calc_physical_constant) and the edge boxes the
   reference zeroes, 8 int32 each: block, edge axis (0/1/2 = xi/eta/zeta),
   lo[3], hi[3] (half-open, inner edge indices) -- the Solid_Surface node box
   widened 20 layers inwards and the Pole node boxes, turned into edge boxes.
   The geometry fields Area_* and dl_* must be uploaded.  MHD_STAGE_HALL_EMF
   then computes Ehall_xi / Ehall_eta / Ehall_zeta of the current state. */
int mhd_set_hall(mhd_ctx *ctx, double hall_coef, const int32_t *zero_boxes, int32_t nbox);

/* Implicit Hall solve in every following StepOnce, after the resistive
   part (ImplicitHallSolver::SolveOneStep with theta = 1,
   Z4_Lunar/src/implicit/Hall_Implicit_Solver.cpp:268-391, the step the
   reference runs when HALL_IMPLICIT is 1).  The unknowns are the owner edges
   of Ehall (`unknowns`: Ehall_xi / Ehall_eta / Ehall_zeta point ids, the
   reference's owner_edges_sorted_), alias/owner/sign the edge 1-form table of
   HALO_OWNER (unpack_owner_edge_1form_local).  Newton on
   F(E) = E - E_hall(B* - dt curl E) from the current Ehall, with a
   backtracking line search; each Newton system is solved by restarted
   GMRES(30) with finite-difference Jacobian-vector products.  Stops at
   ||F|| <= max(rtol ||F0||, atol) or after maxit Newton steps (PETSc SNES
   defaults: 1e-8, 1e-50, 50); ksp_rtol / ksp_maxit bound the linear
   solves.  The solve is steered on the device: in mhd_step its loops are
   conditional nodes of the step's CUDA graph, with no host round trip.
   Needs mhd_set_hall and the "Ehall" sync group.  n = 0 switches it off. */
int mhd_set_hall_implicit(mhd_ctx *ctx, int64_t n, const int64_t *unknowns, int64_t nalias, const int64_t *alias,
                          const int64_t *owner, const double *sign, double rtol, double atol, int32_t maxit,
                          double ksp_rtol, int32_t ksp_maxit);

/* Newton steps, GMRES iterations, final and initial ||F|| and reason
   (2 atol, 3 rtol, -5 Newton iteration limit) of the last implicit Hall solve
   (read from the device; waits for the context's stream). */
int mhd_hall_stats(const mhd_ctx *ctx, int32_t *newton_its, int32_t *linear_its, double *fnorm, double *fnorm0,
                   int32_t *reason);

/* Explicit resistive sub-cycles (LunarSolver::ResistiveDiffusionSubcycles_,
   Z4_Lunar/src/physics/LunarSolver_MagneticRHS.cpp:53-115, with the edge EMF of
   AddResistiveEdgeEMF_To_, Z4_Lunar/src/physics/LunarSolver_MagExplicit_Resis.cpp:67-209):
   `nsub` sub-cycles of dt / nsub in every following StepOnce (0 switches them
   off).  The shell profile yita0(r) of every inner edge is read from the
   fields eta_edge_xi / eta_edge_eta / eta_edge_zeta, which the caller
   uploads; the EMF is (inver_Rem yita0) (J . dr).  Exclusive with
   mhd_set_resistive. */
int mhd_set_resistive_explicit(mhd_ctx *ctx, double inver_Rem, int32_t nsub);

/* Reference state of the mixed-precision flux (no counterpart in the
   reference, which has no mixed-precision form): primitive rho, u, v, w, p
   of a constant state, normally the far-field inflow.  The FP32 face states
   are stored as deviations from it and the Rusanov flux is evaluated in FP32
   in deviation form, with the reference-state part added in FP64, so the
   FP32 rounding scales with the departure from this state.  Any state gives
   the same result up to that rounding (zero, the default, is the plain FP32
   flux).  Sets every run of a batch.  Takes effect at the next
   UpdateDerivedFields_ (mhd_update_derived, or the end of a step); has no
   effect in MHD_PREC_FP64. */
int mhd_set_flux_reference(mhd_ctx *ctx, const double prim[5]);
/* The same for one run of a batch (run -1: every run). */
int mhd_set_flux_reference_run(mhd_ctx *ctx, int32_t run, const double prim[5]);

/* Autotuner (no counterpart in the reference): the hot stencil kernels are
   compiled in register / occupancy variants (the same code under different
   minimum-CTAs-per-SM launch bounds, so every variant gives bit-identical
   results).  mhd_autotune times whole steps (`reps` graph launches, after a
   warm-up) with one kernel's variant changed at a time, the candidate and
   the kept variant back to back and each the faster of two timings, and
   keeps a candidate when the step gets at least 3 % faster; every trial
   starts from a snapshot of the state taken
   at entry, and the state and run clocks are restored at the end, so the
   call does not advance the simulation.  Call it after the state is loaded.
   min_ctas[i] (i < n, at most MHD_NTUNE) receives the chosen minimum CTAs
   per SM of kernel mhd_tune_name(i) (0: no launch bounds, the compiler's own
   register allocation; 12: the face-tiled k_fluid_mixed, 16: the same with
   its FP32 face states staged in shared memory; 14: k_pv_uplus_dt
   with J_cell in a pass of its own).  For the persistent k_gmres_resist the
   value is the CTAs of its grid (0: two per SM); its partial sums group
   differently per grid, so its results agree to round-off, not bitwise.
   k_hall_edge 2: the seven cells of a staggered point read once. */
#define MHD_NTUNE 9
int mhd_autotune(mhd_ctx *ctx, int32_t reps, int32_t *min_ctas, int32_t n);
const char *mhd_tune_name(int32_t i);

/* Applies a variant choice (no counterpart in the reference): min_ctas[i]
   (i < n) in the values mhd_autotune reports, e.g. one it returned in an
   earlier run.  For k_fluid_mixed the value 12 selects the face-tiled kernel
   (each face flux evaluated once per 2 x 4 x 32-cell tile and shared
   through shared memory; the same bits as the per-cell variants), 16 the
   same with the tile's FP32 face states copied into shared memory by
   asynchronous copies first.
   MHD_EINVAL for a value that names no variant. */
int mhd_set_tune(mhd_ctx *ctx, const int32_t *min_ctas, int32_t n);

/* Iterations, final residual norm, ||b|| and convergence reason (2 rtol,
   3 atol, -3 iteration limit, as KSPConvergedReason) of the last solve. */
int mhd_resistive_stats(const mhd_ctx *ctx, int32_t *its, double *rnorm, double *bnorm, int32_t *reason);

/* Time integrator of every following step.  The reference has one: a single
   forward-Euler stage per StepOnce (Z4_Lunar/src/LunarSolver_Driver.cpp:21-92,
   Z4_Lunar/src/physics/LunarSolver_Advance.cpp:61-122), MHD_INTEGRATOR_EULER,
   the default.  MHD_INTEGRATOR_SSPRK2 composes two of those Euler stages at
   the dt of the step's start (Shu-Osher SSP-RK2): U1 = U^n + dt L(U^n), with
   Sync("Ucell"), Sync("Bface") and UpdateDerivedFields_ after it, then
   U^{n+1} = 0.5 (U^n + (U1 + dt L(U1))) on the inner cells and faces, then
   the step's closing syncs and derived fields.  Each stage includes the
   resistive part.  Not available with the implicit Hall solve (MHD_ESTATE).
   Allocates the start-of-step copy of U_H and face B on first use. */
#define MHD_INTEGRATOR_EULER 0
#define MHD_INTEGRATOR_SSPRK2 1
int mhd_set_integrator(mhd_ctx *ctx, int32_t integrator);

/* Failure-detection hook (no counterpart in the reference, whose solves
   cannot stall): makes the grid barrier of the next persistent implicit
   resistive solve wait for an arrival that never comes, and bounds every
   wait of that solve at spin_limit polls (about 0.1 us each).  The solve
   gives up, the step returns MHD_EKRYLOV, the barrier is reset, and the
   context steps again once a good state is loaded.  Nothing faults or hangs:
   every wait is bounded.  MHD_ESTATE without a persistent solve. */
int mhd_test_stall_barrier(mhd_ctx *ctx, uint32_t spin_limit);

/* LunarBoundary::Sync(group) on the device. */
int mhd_sync(mhd_ctx *ctx, const char *group);

/* LunarSolver::UpdateDerivedFields_ (Z4_Lunar/src/physics/LunarSolver_Tools.cpp:157-161):
   B_cell, J_edge, J_cell, PV, U_plus with their syncs; also the CFL time step
   of the next StepOnce (LunarSolver::Compute_Timestep,
   Z4_Lunar/src/physics/LunarSolver_Timestep.cpp:8-140). */
int mhd_update_derived(mhd_ctx *ctx);

/* `nsteps` x LunarSolver::StepOnce (Z4_Lunar/src/LunarSolver_Driver.cpp:21-92),
   replayed as one CUDA graph per step.  dt_out / time_out (may be NULL)
   receive the last step's dt and the accumulated time. */
int mhd_step(mhd_ctx *ctx, int32_t nsteps, double *dt_out, double *time_out);

/* End-to-end step through host buffers: uploads U_H and B_xi/B_eta/B_zeta of
   every block from host AoS arrays (concatenated block after block), runs
   Sync("Ucell"), Sync("Bface"), UpdateDerivedFields_ and `nsteps` StepOnce,
   downloads the same fields back.  state_in and state_out each hold `count`
   values (mhd_state_count); the input is read in full before the output is
   written, so they may be the same array.  The host arrays may be pinned (see
   mhd_host_alloc) for full copy bandwidth.  Each call starts as a restart
   does: the state is taken as read from a restart file, before
   UpdateDerivedFields_ (on a grid with Poles that pass rewrites B_zeta on the
   first cell layer, so feeding a call's output back in applies it twice). */
int mhd_step_host(mhd_ctx *ctx, int32_t nsteps, const double *state_in, double *state_out, int64_t count,
                  double *dt_out);

/* Size in doubles of the concatenated host state used by mhd_step_host. */
int64_t mhd_state_count(const mhd_ctx *ctx);

/* The same end-to-end step with the state's inner points only (no
   counterpart in the reference, whose arrays carry their ghost layers):
   cells [0, n) and faces [0, n] along their own axis, AoS, block after
   block, U_H then B_xi / B_eta / B_zeta.  The ghost points the step reads
   are formed on the device by the Syncs, as in mhd_step_host; ghost points
   no Sync writes keep their device values and are not read by the step.
   mhd_state_count_inner gives the size in doubles. */
int mhd_step_host_inner(mhd_ctx *ctx, int32_t nsteps, const double *state_in, double *state_out, int64_t count,
                        double *dt_out);
int64_t mhd_state_count_inner(const mhd_ctx *ctx);

/* Page-locked host memory for the state buffers (cudaHostAlloc). */
int mhd_host_alloc(int64_t bytes, void **ptr);
int mhd_host_free(void *ptr);

/* Individual stages, for stage-level parity checks and for drivers that keep
   their own step loop.  Stage ids: */
#define MHD_STAGE_TIMESTEP 1   /* Compute_Timestep (dt of the current state) */
#define MHD_STAGE_FLUID_RHS 2  /* ZeroRHS_ + Scheme_U_ + AddSourceToRHS_Fluid -> RHS_H */
#define MHD_STAGE_INDUCTION 3  /* AssembleRHS_Induction_CT_ -> Eface, E, RHS_B */
#define MHD_STAGE_UPDATE 4     /* ApplyUpdate_Euler_ with the current dt */
#define MHD_STAGE_DIVB 5       /* calc_divB -> divB (inner cells; 0 next to a Pole) */
#define MHD_STAGE_HALL_EMF 6   /* BuildHallFaceEMF_Rusanov_diff_ -> Ehall_xi/eta/zeta (see mhd_set_hall) */
#define MHD_STAGE_HALL_SOLVE 7 /* ImplicitHallSolver::SolveOneStep at the current dt, then calc_Bcell */
int mhd_stage(mhd_ctx *ctx, int32_t stage_id);

/* Current dt / time / step counters (device -> host; run 0 of a batch).
   mhd_set_time sets every run. */
int mhd_get_time(mhd_ctx *ctx, double *dt, double *time, int64_t *step);
int mhd_set_time(mhd_ctx *ctx, double dt, double time, int64_t step);

/* Launch statistics: number of kernels this library launched since creation. */
int64_t mhd_kernel_launches(const mhd_ctx *ctx);

/* One StepOnce launched kernel by kernel (no graph) with a CUDA event pair
   around every launch: fills kernel_ids[q] / ms[q] for the first `cap`
   launches and *count with the number of launches. */
int mhd_profile_step(mhd_ctx *ctx, int32_t cap, int32_t *kernel_ids, float *ms, int32_t *count);

/* Name of a kernel id reported by mhd_profile_step. */
const char *mhd_kernel_name(int32_t id);

/* CUDA stream of the context (cudaStream_t), for callers that time with events. */
void *mhd_stream(const mhd_ctx *ctx);

#ifdef __cplusplus
}
#endif

#endif /* BETA1_MHD_H */
