/* Minimal stand-in for the PETSc API subset the reference calls.
 *
 * Test infrastructure only (CPU oracle).  Vectors are plain host arrays on one
 * rank, matrices are shells with a user MatMult, KSP is restarted GMRES(30)
 * with modified Gram-Schmidt (Saad & Schultz 1986) and the convergence test
 * ||r_k|| < max(rtol*||b||, atol); SNES is Newton with a backtracking line
 * search (Dennis & Schnabel 1983, alg. A6.3.1).  Call sites in the reference:
 * Z4_Lunar/src/implicit/Lunar_ImplicitResistive.cpp:95-124,457-491 and
 * Z4_Lunar/src/implicit/Hall_Implicit_Solver.cpp:147-220,268-300.
 */
#ifndef ORACLE_SHIM_PETSCSYS_H
#define ORACLE_SHIM_PETSCSYS_H

#include "mpi.h"
#include <cstdio>
#include <cstdlib>

typedef int PetscErrorCode;
typedef int PetscInt;
typedef double PetscScalar;
typedef double PetscReal;
typedef enum { PETSC_FALSE = 0, PETSC_TRUE = 1 } PetscBool;

#define PETSC_COMM_WORLD MPI_COMM_WORLD
#define MPIU_INT MPI_INT
#define MPIU_REAL MPI_DOUBLE
#define MPIU_SCALAR MPI_DOUBLE
#define PETSC_DEFAULT (-2)
#define PETSC_DECIDE (-1)
#define PETSC_DETERMINE (-1)
#define PETSC_ERR_ARG_NULL 85
#define PETSC_ERR_LIB 76
#define PETSC_ERR_PLIB 77
#define PETSC_ERR_ARG_WRONG 62
#define PETSC_ERR_ARG_OUTOFRANGE 63
#define PETSC_ERR_NOT_CONVERGED 91
#define PETSC_SUCCESS 0

typedef enum { NORM_1 = 0, NORM_2 = 1, NORM_FROBENIUS = 2, NORM_INFINITY = 3 } NormType;
typedef enum { MATOP_MULT = 3 } MatOperation;

typedef struct ShimVec_ *Vec;
typedef struct ShimMat_ *Mat;
typedef struct ShimKSP_ *KSP;
typedef struct ShimPC_ *PC;
typedef struct ShimSNES_ *SNES;

typedef const char *KSPType;
typedef const char *PCType;
typedef const char *SNESType;
#define KSPGMRES "gmres"
#define PCNONE "none"
#define PCSHELL "shell"
#define PCJACOBI "jacobi"
#define SNESNEWTONLS "newtonls"

typedef enum
{
    KSP_CONVERGED_ITERATING = 0,
    KSP_CONVERGED_RTOL = 2,
    KSP_CONVERGED_ATOL = 3,
    KSP_DIVERGED_ITS = -3,
    KSP_DIVERGED_BREAKDOWN = -5
} KSPConvergedReason;

typedef enum
{
    SNES_CONVERGED_ITERATING = 0,
    SNES_CONVERGED_FNORM_ABS = 2,
    SNES_CONVERGED_FNORM_RELATIVE = 3,
    SNES_CONVERGED_SNORM_RELATIVE = 4,
    SNES_DIVERGED_MAX_IT = -5,
    SNES_DIVERGED_LINE_SEARCH = -6
} SNESConvergedReason;

#define PetscCall(expr)                       \
    do                                        \
    {                                         \
        PetscErrorCode shim_ierr_ = (expr);   \
        if (shim_ierr_)                       \
            return shim_ierr_;                \
    } while (0)

#define PetscCallAbort(comm, expr)                                                  \
    do                                                                              \
    {                                                                               \
        PetscErrorCode shim_ierr_ = (expr);                                         \
        if (shim_ierr_)                                                             \
        {                                                                           \
            std::fprintf(stderr, "[petsc shim] error %d at %s:%d\n", shim_ierr_,    \
                         __FILE__, __LINE__);                                       \
            std::abort();                                                           \
        }                                                                           \
    } while (0)

#define SETERRQ(comm, code, ...)                                   \
    do                                                             \
    {                                                              \
        std::fprintf(stderr, "[petsc shim] ");                     \
        std::fprintf(stderr, __VA_ARGS__);                         \
        std::fprintf(stderr, "\n");                                \
        return (code);                                             \
    } while (0)

#define PetscCheck(cond, comm, code, ...) \
    do                                    \
    {                                     \
        if (!(cond))                      \
            SETERRQ(comm, code, __VA_ARGS__); \
    } while (0)

#define PetscFunctionBeginUser
#define PetscFunctionBegin
#define PetscFunctionReturn(x) return (x)

PetscErrorCode PetscInitialize(int *argc, char ***argv, const char *file, const char *help);
PetscErrorCode PetscFinalize(void);
PetscErrorCode PetscInitialized(PetscBool *flag);

/* Vec */
PetscErrorCode VecCreateMPI(MPI_Comm comm, PetscInt n, PetscInt N, Vec *v);
PetscErrorCode VecCreateSeq(MPI_Comm comm, PetscInt n, Vec *v);
PetscErrorCode VecDuplicate(Vec x, Vec *y);
PetscErrorCode VecDestroy(Vec *v);
PetscErrorCode VecSet(Vec x, PetscScalar a);
PetscErrorCode VecCopy(Vec x, Vec y);
PetscErrorCode VecAXPY(Vec y, PetscScalar a, Vec x);
PetscErrorCode VecAYPX(Vec y, PetscScalar b, Vec x);
PetscErrorCode VecWAXPY(Vec w, PetscScalar a, Vec x, Vec y);
PetscErrorCode VecScale(Vec x, PetscScalar a);
PetscErrorCode VecNorm(Vec x, NormType t, PetscReal *val);
PetscErrorCode VecDot(Vec x, Vec y, PetscScalar *val);
PetscErrorCode VecGetArray(Vec x, PetscScalar **a);
PetscErrorCode VecRestoreArray(Vec x, PetscScalar **a);
PetscErrorCode VecGetArrayRead(Vec x, const PetscScalar **a);
PetscErrorCode VecRestoreArrayRead(Vec x, const PetscScalar **a);
PetscErrorCode VecGetLocalSize(Vec x, PetscInt *n);
PetscErrorCode VecGetSize(Vec x, PetscInt *n);

/* Mat */
PetscErrorCode MatCreateShell(MPI_Comm comm, PetscInt m, PetscInt n, PetscInt M, PetscInt N, void *ctx, Mat *A);
PetscErrorCode MatShellSetOperation(Mat A, MatOperation op, void (*f)(void));
PetscErrorCode MatShellGetContext(Mat A, void *ctx);
PetscErrorCode MatMult(Mat A, Vec x, Vec y);
PetscErrorCode MatDestroy(Mat *A);
PetscErrorCode MatCreateSNESMF(SNES snes, Mat *J);
PetscErrorCode MatMFFDComputeJacobian(SNES snes, Vec x, Mat J, Mat P, void *ctx);

/* PC */
PetscErrorCode PCSetType(PC pc, PCType t);
PetscErrorCode PCShellSetContext(PC pc, void *ctx);
PetscErrorCode PCShellGetContext(PC pc, void *ctx);
PetscErrorCode PCShellSetApply(PC pc, PetscErrorCode (*apply)(PC, Vec, Vec));
PetscErrorCode PCShellSetName(PC pc, const char *name);
PetscErrorCode PCApply(PC pc, Vec x, Vec y);

/* KSP */
PetscErrorCode KSPCreate(MPI_Comm comm, KSP *ksp);
PetscErrorCode KSPSetOperators(KSP ksp, Mat A, Mat P);
PetscErrorCode KSPSetType(KSP ksp, KSPType t);
PetscErrorCode KSPGetPC(KSP ksp, PC *pc);
PetscErrorCode KSPSetTolerances(KSP ksp, PetscReal rtol, PetscReal atol, PetscReal dtol, PetscInt maxits);
PetscErrorCode KSPSetFromOptions(KSP ksp);
PetscErrorCode KSPSetInitialGuessNonzero(KSP ksp, PetscBool flg);
PetscErrorCode KSPSolve(KSP ksp, Vec b, Vec x);
PetscErrorCode KSPGetConvergedReason(KSP ksp, KSPConvergedReason *r);
PetscErrorCode KSPGetIterationNumber(KSP ksp, PetscInt *its);
PetscErrorCode KSPGetResidualNorm(KSP ksp, PetscReal *rnorm);
PetscErrorCode KSPDestroy(KSP *ksp);

/* SNES */
typedef PetscErrorCode (*SNESFunctionFn)(SNES, Vec, Vec, void *);
typedef PetscErrorCode (*SNESJacobianFn)(SNES, Vec, Mat, Mat, void *);
PetscErrorCode SNESCreate(MPI_Comm comm, SNES *snes);
PetscErrorCode SNESSetFunction(SNES snes, Vec r, SNESFunctionFn f, void *ctx);
PetscErrorCode SNESSetJacobian(SNES snes, Mat A, Mat P, SNESJacobianFn f, void *ctx);
PetscErrorCode SNESSetType(SNES snes, SNESType t);
PetscErrorCode SNESGetKSP(SNES snes, KSP *ksp);
PetscErrorCode SNESSetFromOptions(SNES snes);
PetscErrorCode SNESSetTolerances(SNES snes, PetscReal abstol, PetscReal rtol, PetscReal stol, PetscInt maxit,
                                 PetscInt maxf);
PetscErrorCode SNESSolve(SNES snes, Vec b, Vec x);
PetscErrorCode SNESGetConvergedReason(SNES snes, SNESConvergedReason *r);
PetscErrorCode SNESGetIterationNumber(SNES snes, PetscInt *its);
PetscErrorCode SNESGetFunctionNorm(SNES snes, PetscReal *fnorm);
PetscErrorCode SNESDestroy(SNES *snes);

#endif
