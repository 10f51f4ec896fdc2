// PETSc-subset stand-in: single-rank host vectors, shell matrices,
// restarted GMRES(30) and a Newton line-search nonlinear solver.
// Test infrastructure for the CPU oracle only.
#include "petscsys_shim.h"

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

struct ShimVec_
{
    std::vector<double> a;
};

struct ShimMat_
{
    void *ctx = nullptr;
    PetscErrorCode (*mult)(Mat, Vec, Vec) = nullptr;
    bool mffd = false;
    SNES snes = nullptr;
};

struct ShimPC_
{
    std::string type = PCNONE;
    void *ctx = nullptr;
    PetscErrorCode (*apply)(PC, Vec, Vec) = nullptr;
};

struct ShimKSP_
{
    Mat A = nullptr;
    ShimPC_ pc;
    double rtol = 1e-5, atol = 1e-50, dtol = 1e5;
    int maxits = 10000;
    int restart = 30;
    bool guess_nonzero = false;
    KSPConvergedReason reason = KSP_CONVERGED_ITERATING;
    int its = 0;
    double rnorm = 0.0;
};

struct ShimSNES_
{
    Vec r = nullptr;
    SNESFunctionFn f = nullptr;
    void *fctx = nullptr;
    Mat J = nullptr;
    SNESJacobianFn jac = nullptr;
    void *jctx = nullptr;
    ShimKSP_ ksp;
    double abstol = 1e-50, rtol = 1e-8, stol = 1e-8;
    int maxit = 50;
    SNESConvergedReason reason = SNES_CONVERGED_ITERATING;
    int its = 0;
    double fnorm = 0.0;
};

static bool g_petsc_init = false;

PetscErrorCode PetscInitialize(int *, char ***, const char *, const char *)
{
    g_petsc_init = true;
    return 0;
}
PetscErrorCode PetscFinalize(void)
{
    g_petsc_init = false;
    return 0;
}
PetscErrorCode PetscInitialized(PetscBool *flag)
{
    *flag = g_petsc_init ? PETSC_TRUE : PETSC_FALSE;
    return 0;
}

// ---------------------------------------------------------------- Vec
PetscErrorCode VecCreateMPI(MPI_Comm, PetscInt n, PetscInt, Vec *v)
{
    *v = new ShimVec_;
    (*v)->a.assign(size_t(n > 0 ? n : 0), 0.0);
    return 0;
}
PetscErrorCode VecCreateSeq(MPI_Comm c, PetscInt n, Vec *v) { return VecCreateMPI(c, n, n, v); }
PetscErrorCode VecDuplicate(Vec x, Vec *y)
{
    *y = new ShimVec_;
    (*y)->a.assign(x->a.size(), 0.0);
    return 0;
}
PetscErrorCode VecDestroy(Vec *v)
{
    delete *v;
    *v = nullptr;
    return 0;
}
PetscErrorCode VecSet(Vec x, PetscScalar a)
{
    for (auto &e : x->a)
        e = a;
    return 0;
}
PetscErrorCode VecCopy(Vec x, Vec y)
{
    y->a = x->a;
    return 0;
}
PetscErrorCode VecAXPY(Vec y, PetscScalar a, Vec x)
{
    for (size_t i = 0; i < y->a.size(); ++i)
        y->a[i] += a * x->a[i];
    return 0;
}
PetscErrorCode VecAYPX(Vec y, PetscScalar b, Vec x)
{
    for (size_t i = 0; i < y->a.size(); ++i)
        y->a[i] = x->a[i] + b * y->a[i];
    return 0;
}
PetscErrorCode VecWAXPY(Vec w, PetscScalar a, Vec x, Vec y)
{
    for (size_t i = 0; i < w->a.size(); ++i)
        w->a[i] = a * x->a[i] + y->a[i];
    return 0;
}
PetscErrorCode VecScale(Vec x, PetscScalar a)
{
    for (auto &e : x->a)
        e *= a;
    return 0;
}
static double dot_(const std::vector<double> &x, const std::vector<double> &y)
{
    double s = 0.0;
    for (size_t i = 0; i < x.size(); ++i)
        s += x[i] * y[i];
    return s;
}
PetscErrorCode VecNorm(Vec x, NormType t, PetscReal *val)
{
    if (t == NORM_INFINITY)
    {
        double m = 0.0;
        for (double e : x->a)
            m = std::max(m, std::abs(e));
        *val = m;
    }
    else if (t == NORM_1)
    {
        double s = 0.0;
        for (double e : x->a)
            s += std::abs(e);
        *val = s;
    }
    else
        *val = std::sqrt(dot_(x->a, x->a));
    return 0;
}
PetscErrorCode VecDot(Vec x, Vec y, PetscScalar *val)
{
    *val = dot_(x->a, y->a);
    return 0;
}
PetscErrorCode VecGetArray(Vec x, PetscScalar **a)
{
    *a = x->a.data();
    return 0;
}
PetscErrorCode VecRestoreArray(Vec, PetscScalar **a)
{
    *a = nullptr;
    return 0;
}
PetscErrorCode VecGetArrayRead(Vec x, const PetscScalar **a)
{
    *a = x->a.data();
    return 0;
}
PetscErrorCode VecRestoreArrayRead(Vec, const PetscScalar **a)
{
    *a = nullptr;
    return 0;
}
PetscErrorCode VecGetLocalSize(Vec x, PetscInt *n)
{
    *n = PetscInt(x->a.size());
    return 0;
}
PetscErrorCode VecGetSize(Vec x, PetscInt *n) { return VecGetLocalSize(x, n); }

// ---------------------------------------------------------------- Mat
PetscErrorCode MatCreateShell(MPI_Comm, PetscInt, PetscInt, PetscInt, PetscInt, void *ctx, Mat *A)
{
    *A = new ShimMat_;
    (*A)->ctx = ctx;
    return 0;
}
PetscErrorCode MatShellSetOperation(Mat A, MatOperation op, void (*f)(void))
{
    if (op == MATOP_MULT)
        A->mult = reinterpret_cast<PetscErrorCode (*)(Mat, Vec, Vec)>(f);
    return 0;
}
PetscErrorCode MatShellGetContext(Mat A, void *ctx)
{
    *static_cast<void **>(ctx) = A->ctx;
    return 0;
}
PetscErrorCode MatMult(Mat A, Vec x, Vec y)
{
    if (!A->mult)
        SETERRQ(0, PETSC_ERR_ARG_NULL, "MatMult on a shell without MATOP_MULT");
    return A->mult(A, x, y);
}
PetscErrorCode MatDestroy(Mat *A)
{
    delete *A;
    *A = nullptr;
    return 0;
}
PetscErrorCode MatCreateSNESMF(SNES snes, Mat *J)
{
    *J = new ShimMat_;
    (*J)->mffd = true;
    (*J)->snes = snes;
    return 0;
}
PetscErrorCode MatMFFDComputeJacobian(SNES, Vec, Mat, Mat, void *) { return 0; }

// ---------------------------------------------------------------- PC
PetscErrorCode PCSetType(PC pc, PCType t)
{
    pc->type = t;
    return 0;
}
PetscErrorCode PCShellSetContext(PC pc, void *ctx)
{
    pc->ctx = ctx;
    return 0;
}
PetscErrorCode PCShellGetContext(PC pc, void *ctx)
{
    *static_cast<void **>(ctx) = pc->ctx;
    return 0;
}
PetscErrorCode PCShellSetApply(PC pc, PetscErrorCode (*apply)(PC, Vec, Vec))
{
    pc->apply = apply;
    return 0;
}
PetscErrorCode PCShellSetName(PC, const char *) { return 0; }
PetscErrorCode PCApply(PC pc, Vec x, Vec y)
{
    if (pc->type == PCSHELL && pc->apply)
        return pc->apply(pc, x, y);
    return VecCopy(x, y);
}

// ---------------------------------------------------------------- KSP
PetscErrorCode KSPCreate(MPI_Comm, KSP *ksp)
{
    *ksp = new ShimKSP_;
    return 0;
}
PetscErrorCode KSPSetOperators(KSP ksp, Mat A, Mat)
{
    ksp->A = A;
    return 0;
}
PetscErrorCode KSPSetType(KSP, KSPType) { return 0; }
PetscErrorCode KSPGetPC(KSP ksp, PC *pc)
{
    *pc = &ksp->pc;
    return 0;
}
PetscErrorCode KSPSetTolerances(KSP ksp, PetscReal rtol, PetscReal atol, PetscReal dtol, PetscInt maxits)
{
    if (rtol != PETSC_DEFAULT)
        ksp->rtol = rtol;
    if (atol != PETSC_DEFAULT)
        ksp->atol = atol;
    if (dtol != PETSC_DEFAULT)
        ksp->dtol = dtol;
    if (maxits != PETSC_DEFAULT)
        ksp->maxits = maxits;
    return 0;
}
PetscErrorCode KSPSetFromOptions(KSP) { return 0; }
PetscErrorCode KSPSetInitialGuessNonzero(KSP ksp, PetscBool flg)
{
    ksp->guess_nonzero = (flg == PETSC_TRUE);
    return 0;
}

// Right-preconditioned restarted GMRES with modified Gram-Schmidt and Givens
// rotations.  Without a preconditioner this is plain GMRES(m).  Convergence:
// the Hessenberg residual estimate drops below max(rtol*||b||, atol).
static PetscErrorCode gmres_solve(ShimKSP_ &k, Vec b, Vec x)
{
    const size_t n = b->a.size();
    const int m = k.restart;
    k.its = 0;
    k.reason = KSP_CONVERGED_ITERATING;
    if (!k.guess_nonzero)
        std::fill(x->a.begin(), x->a.end(), 0.0);

    ShimVec_ r, w, z;
    r.a.assign(n, 0.0);
    w.a.assign(n, 0.0);
    z.a.assign(n, 0.0);
    const double bnorm = std::sqrt(dot_(b->a, b->a));
    const double ttol = std::max(k.rtol * bnorm, k.atol);

    std::vector<std::vector<double>> V(size_t(m + 1), std::vector<double>(n, 0.0));
    std::vector<std::vector<double>> H(size_t(m + 1), std::vector<double>(size_t(m), 0.0));
    std::vector<double> cs(size_t(m), 0.0), sn(size_t(m), 0.0), g(size_t(m + 1), 0.0);

    while (true)
    {
        // r = b - A x
        PetscCall(MatMult(k.A, x, &r));
        for (size_t i = 0; i < n; ++i)
            r.a[i] = b->a[i] - r.a[i];
        double beta = std::sqrt(dot_(r.a, r.a));
        k.rnorm = beta;
        if (beta <= ttol)
        {
            k.reason = (beta <= k.atol) ? KSP_CONVERGED_ATOL : KSP_CONVERGED_RTOL;
            return 0;
        }
        if (k.its >= k.maxits)
        {
            k.reason = KSP_DIVERGED_ITS;
            return 0;
        }
        for (size_t i = 0; i < n; ++i)
            V[0][i] = r.a[i] / beta;
        std::fill(g.begin(), g.end(), 0.0);
        g[0] = beta;
        int j = 0;
        bool done = false;
        for (; j < m && k.its < k.maxits; ++j)
        {
            // w = A M^{-1} v_j
            ShimVec_ vj;
            vj.a = V[size_t(j)];
            PetscCall(PCApply(&k.pc, &vj, &z));
            PetscCall(MatMult(k.A, &z, &w));
            for (int i = 0; i <= j; ++i)
            {
                const double h = dot_(w.a, V[size_t(i)]);
                H[size_t(i)][size_t(j)] = h;
                for (size_t q = 0; q < n; ++q)
                    w.a[q] -= h * V[size_t(i)][q];
            }
            const double hn = std::sqrt(dot_(w.a, w.a));
            H[size_t(j + 1)][size_t(j)] = hn;
            if (hn > 0.0)
                for (size_t q = 0; q < n; ++q)
                    V[size_t(j + 1)][q] = w.a[q] / hn;
            for (int i = 0; i < j; ++i)
            {
                const double t = cs[size_t(i)] * H[size_t(i)][size_t(j)] + sn[size_t(i)] * H[size_t(i + 1)][size_t(j)];
                H[size_t(i + 1)][size_t(j)] =
                    -sn[size_t(i)] * H[size_t(i)][size_t(j)] + cs[size_t(i)] * H[size_t(i + 1)][size_t(j)];
                H[size_t(i)][size_t(j)] = t;
            }
            const double a = H[size_t(j)][size_t(j)], bb = H[size_t(j + 1)][size_t(j)];
            const double den = std::sqrt(a * a + bb * bb);
            cs[size_t(j)] = den > 0.0 ? a / den : 1.0;
            sn[size_t(j)] = den > 0.0 ? bb / den : 0.0;
            H[size_t(j)][size_t(j)] = den;
            H[size_t(j + 1)][size_t(j)] = 0.0;
            g[size_t(j + 1)] = -sn[size_t(j)] * g[size_t(j)];
            g[size_t(j)] = cs[size_t(j)] * g[size_t(j)];
            ++k.its;
            k.rnorm = std::abs(g[size_t(j + 1)]);
            if (k.rnorm <= ttol || hn == 0.0)
            {
                done = true;
                ++j;
                break;
            }
        }
        // solve H y = g (upper triangular j x j), x += M^{-1} V y
        std::vector<double> y(size_t(j), 0.0);
        for (int i = j - 1; i >= 0; --i)
        {
            double s = g[size_t(i)];
            for (int q = i + 1; q < j; ++q)
                s -= H[size_t(i)][size_t(q)] * y[size_t(q)];
            y[size_t(i)] = s / H[size_t(i)][size_t(i)];
        }
        std::fill(w.a.begin(), w.a.end(), 0.0);
        for (int i = 0; i < j; ++i)
            for (size_t q = 0; q < n; ++q)
                w.a[q] += y[size_t(i)] * V[size_t(i)][q];
        PetscCall(PCApply(&k.pc, &w, &z));
        for (size_t q = 0; q < n; ++q)
            x->a[q] += z.a[q];
        if (done)
        {
            k.reason = (k.rnorm <= k.atol) ? KSP_CONVERGED_ATOL : KSP_CONVERGED_RTOL;
            return 0;
        }
        if (k.its >= k.maxits)
        {
            k.reason = KSP_DIVERGED_ITS;
            return 0;
        }
    }
}

PetscErrorCode KSPSolve(KSP ksp, Vec b, Vec x) { return gmres_solve(*ksp, b, x); }
PetscErrorCode KSPGetConvergedReason(KSP ksp, KSPConvergedReason *r)
{
    *r = ksp->reason;
    return 0;
}
PetscErrorCode KSPGetIterationNumber(KSP ksp, PetscInt *its)
{
    *its = ksp->its;
    return 0;
}
PetscErrorCode KSPGetResidualNorm(KSP ksp, PetscReal *rnorm)
{
    *rnorm = ksp->rnorm;
    return 0;
}
PetscErrorCode KSPDestroy(KSP *ksp)
{
    delete *ksp;
    *ksp = nullptr;
    return 0;
}

// ---------------------------------------------------------------- SNES
PetscErrorCode SNESCreate(MPI_Comm, SNES *snes)
{
    *snes = new ShimSNES_;
    (*snes)->ksp.rtol = 1e-5;
    return 0;
}
PetscErrorCode SNESSetFunction(SNES snes, Vec r, SNESFunctionFn f, void *ctx)
{
    snes->r = r;
    snes->f = f;
    snes->fctx = ctx;
    return 0;
}
PetscErrorCode SNESSetJacobian(SNES snes, Mat A, Mat, SNESJacobianFn f, void *ctx)
{
    snes->J = A;
    snes->jac = f;
    snes->jctx = ctx;
    return 0;
}
PetscErrorCode SNESSetType(SNES, SNESType) { return 0; }
PetscErrorCode SNESGetKSP(SNES snes, KSP *ksp)
{
    *ksp = &snes->ksp;
    return 0;
}
PetscErrorCode SNESSetFromOptions(SNES) { return 0; }
PetscErrorCode SNESSetTolerances(SNES snes, PetscReal abstol, PetscReal rtol, PetscReal stol, PetscInt maxit,
                                 PetscInt)
{
    if (abstol != PETSC_DEFAULT)
        snes->abstol = abstol;
    if (rtol != PETSC_DEFAULT)
        snes->rtol = rtol;
    if (stol != PETSC_DEFAULT)
        snes->stol = stol;
    if (maxit != PETSC_DEFAULT)
        snes->maxit = maxit;
    return 0;
}

// Newton iteration x <- x - lambda J^{-1} F(x) with a backtracking line
// search on ||F||^2 (Armijo constant 1e-4, halving, at most 10 cuts).
PetscErrorCode SNESSolve(SNES snes, Vec, Vec x)
{
    const size_t n = x->a.size();
    ShimVec_ F, dx, xt, Ft;
    F.a.assign(n, 0.0);
    dx.a.assign(n, 0.0);
    xt.a.assign(n, 0.0);
    Ft.a.assign(n, 0.0);
    snes->its = 0;
    snes->reason = SNES_CONVERGED_ITERATING;
    PetscCall(snes->f(snes, x, &F, snes->fctx));
    double fn = std::sqrt(dot_(F.a, F.a));
    const double fn0 = fn;
    snes->fnorm = fn;
    if (fn <= snes->abstol)
    {
        snes->reason = SNES_CONVERGED_FNORM_ABS;
        return 0;
    }
    snes->ksp.A = snes->J;
    while (snes->its < snes->maxit)
    {
        if (snes->jac)
            PetscCall(snes->jac(snes, x, snes->J, snes->J, snes->jctx));
        snes->ksp.guess_nonzero = false;
        PetscCall(gmres_solve(snes->ksp, &F, &dx));
        double lambda = 1.0;
        double ftn = 0.0;
        bool accepted = false;
        for (int cut = 0; cut < 10; ++cut)
        {
            for (size_t q = 0; q < n; ++q)
                xt.a[q] = x->a[q] - lambda * dx.a[q];
            PetscCall(snes->f(snes, &xt, &Ft, snes->fctx));
            ftn = std::sqrt(dot_(Ft.a, Ft.a));
            if (ftn * ftn <= (1.0 - 2.0e-4 * lambda) * fn * fn)
            {
                accepted = true;
                break;
            }
            lambda *= 0.5;
        }
        ++snes->its;
        if (!accepted)
        {
            snes->reason = SNES_DIVERGED_LINE_SEARCH;
            return 0;
        }
        const double dxn = lambda * std::sqrt(dot_(dx.a, dx.a));
        const double xn = std::sqrt(dot_(xt.a, xt.a));
        x->a = xt.a;
        F.a = Ft.a;
        fn = ftn;
        snes->fnorm = fn;
        if (fn <= snes->abstol)
        {
            snes->reason = SNES_CONVERGED_FNORM_ABS;
            return 0;
        }
        if (fn <= snes->rtol * fn0)
        {
            snes->reason = SNES_CONVERGED_FNORM_RELATIVE;
            return 0;
        }
        if (dxn <= snes->stol * xn)
        {
            snes->reason = SNES_CONVERGED_SNORM_RELATIVE;
            return 0;
        }
    }
    snes->reason = SNES_DIVERGED_MAX_IT;
    return 0;
}
PetscErrorCode SNESGetConvergedReason(SNES snes, SNESConvergedReason *r)
{
    *r = snes->reason;
    return 0;
}
PetscErrorCode SNESGetIterationNumber(SNES snes, PetscInt *its)
{
    *its = snes->its;
    return 0;
}
PetscErrorCode SNESGetFunctionNorm(SNES snes, PetscReal *fnorm)
{
    *fnorm = snes->fnorm;
    return 0;
}
PetscErrorCode SNESDestroy(SNES *snes)
{
    delete *snes;
    *snes = nullptr;
    return 0;
}
