// Device data layout of the MHD hot path.
//
// Every field of a block lives on one common padded box so that a single
// (i, j, k) -> offset map serves all stagger locations: logical indices run
// over [-G, n + 1 + G) in each direction (G = ghost layers of the state
// fields, the "+1" covers the extra face/edge/node plane), k fastest, and
// each component is a separate plane of `vol` doubles (structure of arrays).
// A field's own reference extent is a sub-box of this padded box.
#pragma once

#include <cstdint>

namespace mhd
{

// Field table: reference name, stagger location (restart-file numbering),
// components and ghost layers of the reference registration
// (Z4_Lunar/main.cpp:61-123, src/3_field/4_MPCNS_Geometry.cpp:4-69).
#define MHD_FIELD_LIST(X)                                  \
    X(U, "U_H", 0, 5, 4)                                   \
    X(Bxi, "B_xi", 1, 1, 4)                                \
    X(Beta, "B_eta", 2, 1, 4)                              \
    X(Bzeta, "B_zeta", 3, 1, 4)                            \
    X(PV, "PV_H", 0, 5, 4)                                 \
    X(Uplus, "U_plus", 0, 3, 4)                            \
    X(Bcell, "B_cell", 0, 3, 4)                            \
    X(Bind, "Bind_cell", 0, 3, 4)                          \
    X(Jxi, "J_xi", 4, 1, 4)                                \
    X(Jeta, "J_eta", 5, 1, 4)                              \
    X(Jzeta, "J_zeta", 6, 1, 4)                            \
    X(Jcell, "J_cell", 0, 3, 4)                            \
    X(Efxi, "Eface_xi", 1, 3, 4)                           \
    X(Efeta, "Eface_eta", 2, 3, 4)                         \
    X(Efzeta, "Eface_zeta", 3, 3, 4)                       \
    X(Exi, "E_xi", 4, 1, 4)                                \
    X(Eeta, "E_eta", 5, 1, 4)                              \
    X(Ezeta, "E_zeta", 6, 1, 4)                            \
    X(RHS, "RHS_H", 0, 5, 0)                               \
    X(RBxi, "RHS_B_xi", 1, 1, 0)                           \
    X(RBeta, "RHS_B_eta", 2, 1, 0)                         \
    X(RBzeta, "RHS_B_zeta", 3, 1, 0)                       \
    X(divB, "divB", 0, 1, 1)                               \
    X(Baddxi, "Badd_xi", 1, 1, 4)                          \
    X(Baddeta, "Badd_eta", 2, 1, 4)                        \
    X(Baddzeta, "Badd_zeta", 3, 1, 4)                      \
    X(Jac, "Jac", 0, 1, 3)                                 \
    X(JDxi, "JDxi", 1, 3, 4)                               \
    X(JDeta, "JDet", 2, 3, 4)                              \
    X(JDzeta, "JDze", 3, 3, 4)                             \
    X(betaxi, "beta_xi", 1, 1, 3)                          \
    X(betaeta, "beta_eta", 2, 1, 3)                        \
    X(betazeta, "beta_zeta", 3, 1, 3)                      \
    X(alphaxi, "alpha_xi", 4, 1, 3)                        \
    X(alphaeta, "alpha_eta", 5, 1, 3)                      \
    X(alphazeta, "alpha_zeta", 6, 1, 3)                    \
    X(drxi, "dr_xi", 4, 3, 3)                              \
    X(dreta, "dr_eta", 5, 3, 3)                            \
    X(drzeta, "dr_zeta", 6, 3, 3)                          \
    X(WB, "Bcell_from_Bface_w", 0, 18, 3)                  \
    X(WJ, "Jcell_from_Jedge_w", 0, 36, 3)                  \
    X(Eresxi, "Eres_xi", 4, 1, 4)                          \
    X(Ereseta, "Eres_eta", 5, 1, 4)                        \
    X(Ereszeta, "Eres_zeta", 6, 1, 4)                      \
    X(RBresxi, "RHS_Bres_xi", 1, 1, 0)                     \
    X(RBreseta, "RHS_Bres_eta", 2, 1, 0)                   \
    X(RBreszeta, "RHS_Bres_zeta", 3, 1, 0)                 \
    X(dBxi, "dB_xi", 1, 1, 4)                              \
    X(dBeta, "dB_eta", 2, 1, 4)                            \
    X(dBzeta, "dB_zeta", 3, 1, 4)                          \
    X(dJxi, "dJ_xi", 4, 1, 4)                              \
    X(dJeta, "dJ_eta", 5, 1, 4)                            \
    X(dJzeta, "dJ_zeta", 6, 1, 4)                          \
    X(etaxi, "eta_edge_xi", 4, 1, 0)                         \
    X(etaeta, "eta_edge_eta", 5, 1, 0)                     \
    X(etazeta, "eta_edge_zeta", 6, 1, 0)                   \
    X(UC, "U_contra_cell", 0, 3, 1)                        \
    X(NAxi, "Anorm_xi", 1, 4, 4)                           \
    X(NAeta, "Anorm_eta", 2, 4, 4)                         \
    X(NAzeta, "Anorm_zeta", 3, 4, 4)                       \
    X(Cs, "Csound_cell", 0, 1, 1)                          \
    X(RhoE, "RhoE_cell", 0, 1, 1)                          \
    X(Areaxi, "Area_xi", 1, 1, 3)                          \
    X(Areaeta, "Area_eta", 2, 1, 3)                        \
    X(Areazeta, "Area_zeta", 3, 1, 3)                      \
    X(dlxi, "dl_xi", 4, 1, 3)                              \
    X(dleta, "dl_eta", 5, 1, 3)                            \
    X(dlzeta, "dl_zeta", 6, 1, 3)                          \
    X(Ehxi, "Ehall_xi", 4, 1, 4)                           \
    X(Eheta, "Ehall_eta", 5, 1, 4)                         \
    X(Ehzeta, "Ehall_zeta", 6, 1, 4)                       \
    X(Ehc, "Ehall_cell", 0, 3, 4)                          \
    X(HallBeta, "hall_beta_cell", 0, 1, 4)                 \
    X(Astarxi, "Astar_xi", 4, 1, 3)                        \
    X(Astareta, "Astar_eta", 5, 1, 3)                      \
    X(Astarzeta, "Astar_zeta", 6, 1, 3)

enum FieldId : int
{
#define MHD_ENUM(id, name, loc, nc, ng) F_##id,
    MHD_FIELD_LIST(MHD_ENUM)
#undef MHD_ENUM
        NFIELD
};

enum Loc : int
{
    LOC_CELL = 0,
    LOC_FXI = 1,
    LOC_FETA = 2,
    LOC_FZETA = 3,
    LOC_EXI = 4,
    LOC_EETA = 5,
    LOC_EZETA = 6
};

// +1 planes of a stagger location per axis
__host__ __device__ inline void loc_plus(int loc, int &pi, int &pj, int &pk)
{
    pi = (loc == LOC_FXI || loc == LOC_EETA || loc == LOC_EZETA) ? 1 : 0;
    pj = (loc == LOC_FETA || loc == LOC_EXI || loc == LOC_EZETA) ? 1 : 0;
    pk = (loc == LOC_FZETA || loc == LOC_EXI || loc == LOC_EETA) ? 1 : 0;
}

struct BlockView
{
    double *f[NFIELD];
    int ni, nj, nk;   // cells
    int G;            // padding ghost layers
    int NJ, NK;       // padded extents (j, k)
    int64_t vol;      // doubles per component plane
    // mixed precision only (null otherwise): FP32 planes on the same padded box
    float *g32;       // face area xi, eta, zeta, then their unit normals
    float *q32;       // face-state quantities rho, u, v, w, p, rhoE, c
    float *w32;       // least-squares weights: Bcell_from_Bface_w (18 planes), Jcell_from_Jedge_w (36)
    // SSP-RK2 only (null otherwise): the state at the step's start, U_H 5
    // planes then B_xi, B_eta, B_zeta, on the same padded box
    double *rk;
    // run (independent time line) the block belongs to, and that run's
    // reference state of the mixed-precision flux (rho, u, v, w, p, E)
    int run;
    const double *qref;
    // flattened launches over blocks of uneven sizes: per launch kind the
    // block of every CTA (same table in every view; null = 2-D launches with
    // one grid row per block) and this block's first CTA
    const int *cta_blk[4];
    int cta0[4];
};

// launch kinds of the flattened grids: cells with depth 0, cells with depth
// 1, the staggered box [0, n + 1)^3 of the face / edge kernels, and tiles of
// TILE_I x TILE_J x TILE_K cells over the depth-1 box (one CTA each)
enum : int
{
    KIND_CELL0 = 0,
    KIND_CELL1 = 1,
    KIND_STAG = 2,
    KIND_TILE1 = 3,
    NKIND = 4
};
constexpr int TILE_I = 2, TILE_J = 4, TILE_K = 32; // TILE_I * TILE_J * TILE_K = 256 threads

#ifdef __CUDACC__
// Block and thread-in-block of the calling thread: flattened launches (one
// grid row) look the block up per CTA, 2-D launches take blockIdx.y.
__device__ __forceinline__ int cta_block(const BlockView *bvs, int kind, int64_t &t)
{
    const int *tab = bvs[0].cta_blk[kind];
    if (tab && gridDim.y == 1)
    {
        const int bi = tab[blockIdx.x];
        t = int64_t(blockIdx.x - bvs[bi].cta0[kind]) * blockDim.x + threadIdx.x;
        return bi;
    }
    t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    return int(blockIdx.y);
}
#endif

// plane indices of BlockView::g32 / q32
enum : int
{
    G32_AREA = 0, // face area of axis a: plane a
    G32_NRM = 3,  // unit normal of axis a, component c: plane 3 + 3 a + c
    G32_N = 12,
    Q32_RHO = 0,
    Q32_U = 1,
    Q32_P = 4,
    Q32_RHOE = 5,
    Q32_C = 6,
    Q32_N = 7,
    W32_B = 0,
    W32_J = 18,
    W32_N = 54
};

__host__ __device__ inline int64_t pidx(const BlockView &b, int i, int j, int k)
{
    return (int64_t(i + b.G) * b.NJ + (j + b.G)) * b.NK + (k + b.G);
}

} // namespace mhd
