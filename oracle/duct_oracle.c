/*
 * duct_oracle.c -- CPU FP64 restatement of the duct reference hot path.
 *
 * TEST INFRASTRUCTURE ONLY (checker and CPU baseline; see duct_oracle.h for
 * the parity-pin statement).  Each function cites the reference routine it
 * restates.  LAPACK/BLAS come from the OpenBLAS build bundled with SciPy
 * (symbols scipy_dgeev_, scipy_dgetrf_, scipy_dgetri_, scipy_dgemm_), i.e.
 * the same routines the reference calls (src/pseudomat.f90:110,131,141-142,
 * 244,254-255; src/solvediag.f90:51-80,140-219).
 */
#include "duct_oracle.h"
#include "orc_fft.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ---- LAPACK / BLAS (gfortran ABI: trailing hidden string lengths) ------- */
extern void scipy_dgeev_(const char *jobvl, const char *jobvr, const int *n,
                         double *a, const int *lda, double *wr, double *wi,
                         double *vl, const int *ldvl, double *vr,
                         const int *ldvr, double *work, const int *lwork,
                         int *info, size_t, size_t);
extern void scipy_dgetrf_(const int *m, const int *n, double *a,
                          const int *lda, int *ipiv, int *info);
extern void scipy_dgetri_(const int *n, double *a, const int *lda,
                          const int *ipiv, double *work, const int *lwork,
                          int *info);
extern void scipy_dgemm_(const char *ta, const char *tb, const int *m,
                         const int *n, const int *k, const double *alpha,
                         const double *a, const int *lda, const double *b,
                         const int *ldb, const double *beta, double *c,
                         const int *ldc, size_t, size_t);
extern void scipy_dsygv_(const int *itype, const char *jobz, const char *uplo,
                         const int *n, double *a, const int *lda, double *b,
                         const int *ldb, double *w, double *work,
                         const int *lwork, int *info, size_t, size_t);
extern void scipy_dptsv_(const int *n, const int *nrhs, double *d, double *e,
                         double *b, const int *ldb, int *info);
extern void scipy_openblas_set_num_threads(int);

void orc_set_blas_threads(int n) { scipy_openblas_set_num_threads(n); }

#define IX(i, j, ld) ((size_t)(i) + (size_t)(j) * (size_t)(ld))

static void dgemm_tn(int n, const double *A, const double *B, double *C)
{
    /* C = A^T * B, all n x n with leading dimension n (the reference's
     * dgemm('t','n',mm2+1,...) calls).                                      */
    const double one = 1.0, zero = 0.0;
    scipy_dgemm_("t", "n", &n, &n, &n, &one, A, &n, B, &n, &zero, C, &n, 1, 1);
}

static int invert(int n, double *A)
{
    /* dgetrf + dgetri, as src/pseudomat.f90:141-142, 254-255, 177-178.      */
    int info = 0, lwk = 64 * (n > 4 ? n : 4);
    int *ipiv = (int *)malloc(sizeof(int) * (size_t)n);
    double *wk = (double *)malloc(sizeof(double) * (size_t)lwk);
    scipy_dgetrf_(&n, &n, A, &n, ipiv, &info);
    if (info == 0) scipy_dgetri_(&n, A, &n, ipiv, wk, &lwk, &info);
    free(ipiv);
    free(wk);
    return info;
}

static int eigen(int n, double *A, double *wr, double *wi, double *vr)
{
    /* dgeev('n','v',...) as src/pseudomat.f90:131-132, 244-245.              */
    int info = 0, lwk = 64 * n, one = 1;
    double dummy = 0.0;
    double *wk = (double *)calloc((size_t)lwk, sizeof(double));
    scipy_dgeev_("n", "v", &n, A, &n, wr, wi, &dummy, &one, vr, &n, wk, &lwk,
                 &info, 1, 1);
    free(wk);
    return info;
}

/* pseudomat, src/pseudomat.f90:2-312 (both the 'd' and the 'n' branch).   */
int orc_pseudomat(int m, orc_ops *o)
{
    if (m < 4) return -1;
    memset(o, 0, sizeof(*o));
    const int n = m - 1, mm2 = m - 2;
    const double pi = 4.0 * atan(1.0);
    o->m = m;
    o->xcol = (double *)calloc((size_t)m, sizeof(double));
    o->DC = (double *)calloc((size_t)m * m, sizeof(double));
    o->D2 = (double *)calloc((size_t)m * m, sizeof(double));
    o->ED = (double *)calloc((size_t)mm2, sizeof(double));
    o->EDim = (double *)calloc((size_t)mm2, sizeof(double));
    o->EN = (double *)calloc((size_t)mm2, sizeof(double));
    o->ENim = (double *)calloc((size_t)mm2, sizeof(double));
    o->PD = (double *)calloc((size_t)mm2 * mm2, sizeof(double));
    o->PDM1 = (double *)calloc((size_t)mm2 * mm2, sizeof(double));
    o->PN = (double *)calloc((size_t)mm2 * mm2, sizeof(double));
    o->PNM1 = (double *)calloc((size_t)mm2 * mm2, sizeof(double));
    o->D2Bd = (double *)calloc((size_t)mm2 * mm2, sizeof(double));
    o->D2Bn = (double *)calloc((size_t)mm2 * mm2, sizeof(double));
    double *dd = (double *)calloc((size_t)m, sizeof(double));
    double *D2B = (double *)calloc((size_t)mm2 * mm2, sizeof(double));
    double *x = o->xcol, *DC = o->DC, *D2 = o->D2;

    /* dd and nodes: :72-85 */
    dd[0] = 2.0;
    for (int i = 1; i < m - 1; ++i) dd[i] = 1.0;
    dd[m - 1] = 2.0;
    for (int j = 0; j < m; ++j) x[j] = -cos(pi * (double)j / (double)n);

    /* derivative matrix, CHQZ p.69: :90-107 (1-based l,j -> 0-based) */
    DC[IX(0, 0, m)] = -(2.0 * (double)n * (double)n + 1.0) / 6.0;
    DC[IX(m - 1, m - 1, m)] = -DC[IX(0, 0, m)];
    for (int i = 1; i < n; ++i)
        DC[IX(i, i, m)] = -0.5 * x[i] / (1.0 - x[i] * x[i]);
    for (int l = 0; l < m; ++l) {
        for (int j = 0; j < l; ++j) {
            double coef = dd[l] / dd[j];
            double sgn = ((l + j) % 2 == 0) ? 1.0 : -1.0;
            DC[IX(l, j, m)] = coef * sgn / (x[l] - x[j]);
        }
        for (int j = l + 1; j < m; ++j) {
            double coef = dd[l] / dd[j];
            double sgn = ((l + j) % 2 == 0) ? 1.0 : -1.0;
            DC[IX(l, j, m)] = coef * sgn / (x[l] - x[j]);
        }
    }
    /* D2 = DC*DC: :110 */
    {
        const double one = 1.0, zero = 0.0;
        scipy_dgemm_("n", "n", &m, &m, &m, &one, DC, &m, DC, &m, &zero, D2, &m,
                     1, 1);
    }

    int info = 0;
    /* ---- Dirichlet: :223-263 ---- */
    for (int j = 0; j < mm2; ++j)
        for (int i = 0; i < mm2; ++i)
            D2B[IX(i, j, mm2)] = D2[IX(i + 1, j + 1, m)];
    memcpy(o->D2Bd, D2B, sizeof(double) * (size_t)mm2 * mm2);
    info = eigen(mm2, D2B, o->ED, o->EDim, o->PD);
    if (info) goto done;
    memcpy(o->PDM1, o->PD, sizeof(double) * (size_t)mm2 * mm2);
    info = invert(mm2, o->PDM1);
    if (info) goto done;

    /* ---- Neumann: :114-186 ---- */
    {
        const double Det = DC[IX(0, 0, m)] * DC[IX(m - 1, m - 1, m)] -
                           DC[IX(0, m - 1, m)] * DC[IX(m - 1, 0, m)];
        for (int i = 1; i < n; ++i)
            for (int j = 1; j < n; ++j) {
                double ter1 = D2[IX(i, 0, m)] *
                              (DC[IX(0, m - 1, m)] * DC[IX(m - 1, j, m)] -
                               DC[IX(m - 1, m - 1, m)] * DC[IX(0, j, m)]) /
                              Det;
                double ter3 = D2[IX(i, m - 1, m)] *
                              (DC[IX(m - 1, 0, m)] * DC[IX(0, j, m)] -
                               DC[IX(0, 0, m)] * DC[IX(m - 1, j, m)]) /
                              Det;
                D2B[IX(i - 1, j - 1, mm2)] = ter1 + D2[IX(i, j, m)] + ter3;
            }
        memcpy(o->D2Bn, D2B, sizeof(double) * (size_t)mm2 * mm2);
        info = eigen(mm2, D2B, o->EN, o->ENim, o->PN);
        if (info) goto done;
        memcpy(o->PNM1, o->PN, sizeof(double) * (size_t)mm2 * mm2);
        info = invert(mm2, o->PNM1);
        if (info) goto done;
        /* location of the zero eigenvalue: :146-152 (strict "ne" update) */
        double eigmin = 1.0e6;
        o->iofzero = 0;
        for (int i = 0; i < mm2; ++i) {
            double eig = fmin(eigmin, fabs(o->EN[i]));
            if (eig != eigmin) {
                o->iofzero = i + 1;
                eigmin = eig;
            }
        }
        o->wanted = 0.0;
        /* AM1: :158-178, Fortran AM1(r,c) -> AM1[(r-1)+(c-1)*4] */
        double *A = o->AM1;
        const double d11 = DC[IX(0, 0, m)], d1m = DC[IX(0, m - 1, m)];
        const double dm1 = DC[IX(m - 1, 0, m)], dmm = DC[IX(m - 1, m - 1, m)];
        A[0 + 0 * 4] = 2.0 * d11; A[0 + 1 * 4] = d1m;
        A[0 + 2 * 4] = 0.0;       A[0 + 3 * 4] = d1m;
        A[1 + 0 * 4] = -dm1;      A[1 + 1 * 4] = d11 - dmm;
        A[1 + 2 * 4] = d1m;       A[1 + 3 * 4] = 0.0;
        A[2 + 0 * 4] = 0.0;       A[2 + 1 * 4] = dm1;
        A[2 + 2 * 4] = 2.0 * dmm; A[2 + 3 * 4] = dm1;
        A[3 + 0 * 4] = -dm1;      A[3 + 1 * 4] = 0.0;
        A[3 + 2 * 4] = d1m;       A[3 + 3 * 4] = d11 - dmm;
        info = invert(4, A);
    }
done:
    free(dd);
    free(D2B);
    return info;
}

void orc_ops_free(orc_ops *o)
{
    free(o->xcol); free(o->DC); free(o->D2);
    free(o->ED); free(o->EDim); free(o->PD); free(o->PDM1);
    free(o->EN); free(o->ENim); free(o->PN); free(o->PNM1);
    free(o->D2Bd); free(o->D2Bn);
    memset(o, 0, sizeof(*o));
}

/* Padded (m-1)^2 transposed operators exactly as the reference stores them
 * (PDT, PDM1T, PNT, PNM1T of src/pseudomat.f90:181-186, 258-263).          */
static void padded_transpose(int mm2, const double *P, double *PT)
{
    const int np1 = mm2 + 1;
    memset(PT, 0, sizeof(double) * (size_t)np1 * np1);
    for (int i = 0; i < mm2; ++i)
        for (int j = 0; j < mm2; ++j) PT[IX(i, j, np1)] = P[IX(j, i, mm2)];
}

typedef struct {
    double *F, *FT, *tmprt, *PT, *PM1T;
} orc_work;

static void work_alloc(orc_work *w, int m)
{
    const size_t np1 = (size_t)(m - 1);
    w->F = (double *)calloc(np1 * np1, sizeof(double));
    w->FT = (double *)calloc(np1 * np1, sizeof(double));
    w->tmprt = (double *)calloc(np1 * np1, sizeof(double));
    w->PT = (double *)calloc(np1 * np1, sizeof(double));
    w->PM1T = (double *)calloc(np1 * np1, sizeof(double));
}
static void work_free(orc_work *w)
{
    free(w->F); free(w->FT); free(w->tmprt); free(w->PT); free(w->PM1T);
}

/* solvediag, src/solvediag.f90:2-330 (the ngpu=0 branch).                   */
static int solvediag_w(double *U, const orc_ops *o, char bound, double xlambda,
                       orc_work *w)
{
    const int m = o->m, mm2 = m - 2, np1 = m - 1;
    const size_t nn = (size_t)np1 * np1;
    double *F = w->F, *FT = w->FT, *tmprt = w->tmprt;
    memset(F, 0, nn * sizeof(double));
    memset(FT, 0, nn * sizeof(double));
    memset(tmprt, 0, nn * sizeof(double));
    /* interior copy: :30-34 */
    for (int j = 1; j < m - 1; ++j)
        for (int i = 1; i < m - 1; ++i) F[IX(i - 1, j - 1, np1)] = U[IX(i, j, m)];

    if (bound == 'd') {
        const double *D2 = o->D2;
        /* boundary-value correction: :39-45 (D2bx = D2by = D2(:,{1,m})) */
        for (int j = 0; j < mm2; ++j)
            for (int i = 0; i < mm2; ++i) {
                double bcontv = D2[IX(i + 1, 0, m)] * U[IX(0, j + 1, m)] +
                                D2[IX(i + 1, m - 1, m)] * U[IX(m - 1, j + 1, m)];
                double bconth = D2[IX(j + 1, 0, m)] * U[IX(i + 1, 0, m)] +
                                D2[IX(j + 1, m - 1, m)] * U[IX(i + 1, m - 1, m)];
                F[IX(i, j, np1)] -= bcontv + bconth;
            }
        padded_transpose(mm2, o->PD, w->PT);
        padded_transpose(mm2, o->PDM1, w->PM1T);
        /* hot loop: :51-80 */
        dgemm_tn(np1, w->PM1T, F, FT);
        for (int i = 0; i < np1; ++i)
            for (int j = 0; j < np1; ++j) tmprt[IX(i, j, np1)] = FT[IX(j, i, np1)];
        dgemm_tn(np1, tmprt, w->PM1T, F);
        for (int j = 0; j < mm2; ++j)
            for (int i = 0; i < mm2; ++i)
                FT[IX(i, j, np1)] =
                    F[IX(i, j, np1)] / ((o->ED[i] + o->ED[j]) - xlambda);
        dgemm_tn(np1, w->PT, FT, F);
        for (int i = 0; i < np1; ++i)
            for (int j = 0; j < np1; ++j) tmprt[IX(i, j, np1)] = F[IX(j, i, np1)];
        dgemm_tn(np1, tmprt, w->PT, FT);
        /* write-back: :131-135 */
        for (int j = 0; j < mm2; ++j)
            for (int i = 0; i < mm2; ++i) U[IX(i + 1, j + 1, m)] = FT[IX(i, j, np1)];
        return 0;
    }
    if (bound != 'n') return -1;

    /* ---- Neumann: :137-322 ---- */
    const double *EN = o->EN, *PN = o->PN, *DC = o->DC;
    padded_transpose(mm2, o->PN, w->PT);
    padded_transpose(mm2, o->PNM1, w->PM1T);
    dgemm_tn(np1, w->PM1T, F, FT);
    for (int i = 0; i < mm2; ++i)
        for (int j = 0; j < mm2; ++j) tmprt[IX(i, j, np1)] = FT[IX(j, i, np1)];
    dgemm_tn(np1, tmprt, w->PM1T, F);
    if (fabs(xlambda) > 1.0e-10) {
        for (int j = 0; j < mm2; ++j)
            for (int i = 0; i < mm2; ++i)
                FT[IX(i, j, np1)] = F[IX(i, j, np1)] / (EN[i] + EN[j] - xlambda);
    } else {
        /* singular mode: :163-206 */
        const int io = o->iofzero - 1;
        for (int j = 0; j < mm2; ++j)
            for (int i = 0; i < mm2; ++i) {
                if (i == io && j == io) continue;
                FT[IX(i, j, np1)] = F[IX(i, j, np1)] / (EN[i] + EN[j] - xlambda);
            }
        FT[IX(io, io, np1)] = 0.0;
        double valore = 0.0;
        for (int l = 0; l < mm2; ++l) {
            double val = 0.0;
            for (int k = 0; k < mm2; ++k) val += PN[IX(io, k, mm2)] * FT[IX(l, k, np1)];
            valore += PN[IX(io, l, mm2)] * val;
        }
        FT[IX(io, io, np1)] =
            (o->wanted - valore) / (PN[IX(io, io, mm2)] * PN[IX(io, io, mm2)]);
    }
    dgemm_tn(np1, w->PT, FT, F);
    for (int i = 0; i < mm2; ++i)
        for (int j = 0; j < mm2; ++j) tmprt[IX(i, j, np1)] = F[IX(j, i, np1)];
    dgemm_tn(np1, tmprt, w->PT, FT);
    for (int j = 0; j < mm2; ++j)
        for (int i = 0; i < mm2; ++i) U[IX(i + 1, j + 1, m)] = FT[IX(i, j, np1)];

    /* Neumann wall lines: :253-276 */
    const double d11 = DC[IX(0, 0, m)], d1m = DC[IX(0, m - 1, m)];
    const double dm1 = DC[IX(m - 1, 0, m)], dmm = DC[IX(m - 1, m - 1, m)];
    const double det = d11 * dmm - d1m * dm1;
    for (int i = 1; i < m - 1; ++i) {
        double sumb = 0.0, sumt = 0.0;
        for (int j = 0; j < mm2; ++j) {
            sumb += DC[IX(0, j + 1, m)] * FT[IX(i - 1, j, np1)];
            sumt += DC[IX(m - 1, j + 1, m)] * FT[IX(i - 1, j, np1)];
        }
        U[IX(i, 0, m)] = (-dmm * sumb + d1m * sumt) / det;
        U[IX(i, m - 1, m)] = (dm1 * sumb - d11 * sumt) / det;
    }
    for (int j = 1; j < m - 1; ++j) {
        double suml = 0.0, sumr = 0.0;
        for (int i = 0; i < mm2; ++i) {
            suml += DC[IX(0, i + 1, m)] * FT[IX(i, j - 1, np1)];
            sumr += DC[IX(m - 1, i + 1, m)] * FT[IX(i, j - 1, np1)];
        }
        U[IX(0, j, m)] = (-dmm * suml + d1m * sumr) / det;
        U[IX(m - 1, j, m)] = (dm1 * suml - d11 * sumr) / det;
    }
    /* corners: :280-322 */
    double ff[4] = {0, 0, 0, 0};
    for (int i = 1; i < m - 1; ++i)
        ff[0] = ff[0] - DC[IX(0, i, m)] * (U[IX(i, 0, m)] + U[IX(0, i, m)]);
    for (int i = 1; i < m - 1; ++i)
        ff[1] = ff[1] - DC[IX(0, i, m)] * U[IX(m - 1, i, m)] +
                DC[IX(m - 1, i, m)] * U[IX(i, 0, m)];
    for (int i = 1; i < m - 1; ++i)
        ff[2] = ff[2] - DC[IX(m - 1, i, m)] * (U[IX(i, m - 1, m)] + U[IX(m - 1, i, m)]);
    for (int i = 1; i < m - 1; ++i)
        ff[3] = ff[3] - DC[IX(0, i, m)] * U[IX(i, m - 1, m)] +
                DC[IX(m - 1, i, m)] * U[IX(0, i, m)];
    const double *A = o->AM1;
    double c[4];
    for (int r = 0; r < 4; ++r) {
        c[r] = 0.0;
        for (int i = 0; i < 4; ++i) c[r] += A[r + 4 * i] * ff[i];
    }
    U[IX(0, 0, m)] = c[0];
    U[IX(m - 1, 0, m)] = c[1];
    U[IX(m - 1, m - 1, m)] = c[2];
    U[IX(0, m - 1, m)] = c[3];
    return 0;
}

int orc_solvediag(double *U, const orc_ops *o, char bound, double xlambda)
{
    orc_work w;
    work_alloc(&w, o->m);
    int r = solvediag_w(U, o, bound, xlambda, &w);
    work_free(&w);
    return r;
}

/* helm3d + int2d3d + com2re/re2com: src/helm3d.f90:36-72,
 * src/int2d3d.f90:2-53, 55-109.                                            */
int orc_helm3d(double *rhs, double *sol, int my, int mz, int ib, int ie,
               const double *xalp, char bound, double alambda,
               const orc_ops *o, int nthreads)
{
    if (my != mz || my != o->m) return -2;
    if (bound != 'd' && bound != 'n') return -1;
    const int nmodes = ie - ib + 1;
    const size_t plane = (size_t)my * mz;
    if (bound == 'd') {
        for (int i = 0; i < nmodes; ++i) {
            double *r = rhs + 2 * plane * (size_t)i;
            for (int j = 0; j < my; ++j) {
                r[2 * IX(j, 0, my)] = r[2 * IX(j, 0, my) + 1] = 0.0;
                r[2 * IX(j, mz - 1, my)] = r[2 * IX(j, mz - 1, my) + 1] = 0.0;
            }
            for (int k = 0; k < mz; ++k) {
                r[2 * IX(0, k, my)] = r[2 * IX(0, k, my) + 1] = 0.0;
                r[2 * IX(my - 1, k, my)] = r[2 * IX(my - 1, k, my) + 1] = 0.0;
            }
        }
    }
    if (nthreads < 1) nthreads = 1;
    int err = 0;
#pragma omp parallel num_threads(nthreads) reduction(| : err)
    {
        orc_work w;
        work_alloc(&w, my);
        double *U = (double *)malloc(sizeof(double) * plane);
#pragma omp for schedule(dynamic, 1)
        for (int i = 0; i < nmodes; ++i) {
            const int imode = ib + i;
            const double xlambda = alambda + xalp[i] * xalp[i];
            const double *r = rhs + 2 * plane * (size_t)i;
            double *s = sol + 2 * plane * (size_t)i;
            for (size_t p = 0; p < plane; ++p) U[p] = r[2 * p];
            err |= solvediag_w(U, o, bound, xlambda, &w);
            for (size_t p = 0; p < plane; ++p) {
                s[2 * p] = U[p];
                s[2 * p + 1] = 0.0;
            }
            if (imode == 0) continue;
            for (size_t p = 0; p < plane; ++p) U[p] = r[2 * p + 1];
            err |= solvediag_w(U, o, bound, xlambda, &w);
            for (size_t p = 0; p < plane; ++p) s[2 * p + 1] += U[p];
        }
        free(U);
        work_free(&w);
    }
    return err ? -1 : 0;
}

/* ---- Chebyshev transforms ------------------------------------------------ */

/* FFTW REDFT00 of length nn: X_k = x_0 + (-1)^k x_{N} + 2 sum x_j cos(pi jk/N)
 * with N = nn-1, evaluated directly with an exact-angle cosine table.      */
static void redft00(const double *x, double *X, int nn, const double *ctab)
{
    const int N = nn - 1;
    for (int k = 0; k < nn; ++k) {
        double s = x[0] + ((k & 1) ? -x[N] : x[N]);
        double acc = 0.0;
        for (int j = 1; j < N; ++j) acc += x[j] * ctab[(size_t)((long)j * k % (2 * N))];
        X[k] = s + 2.0 * acc;
    }
}

static double *cos_table(int nn)
{
    const int N = nn - 1;
    const double pi = 4.0 * atan(1.0);
    double *t = (double *)malloc(sizeof(double) * (size_t)(2 * N));
    for (int q = 0; q < 2 * N; ++q) t[q] = cos(pi * (double)q / (double)N);
    return t;
}

/* REDFT00 through the complex FFT of the even extension (length 2N):
 * X_k = Re FFT(x_0, x_1, .., x_N, x_{N-1}, .., x_1)_k -- the O(N log N) route
 * FFTW takes; used for the longer lines (nn >= 64), where the direct sum
 * would dominate the oracle's time.                                         */
static void redft00_fft(const double *x, double *X, int nn, const orc_fft_plan *p, double *wa, double *wb)
{
    const int N = nn - 1;
    for (int j = 0; j <= N; ++j) { wa[2 * j] = x[j]; wa[2 * j + 1] = 0.0; }
    for (int j = 1; j < N; ++j) { wa[2 * (2 * N - j)] = x[j]; wa[2 * (2 * N - j) + 1] = 0.0; }
    orc_fft(p, wa, wb, 0);
    for (int k = 0; k < nn; ++k) X[k] = wb[2 * k];
}

/* tcheb_fftw, src/tchebw.f:62-192 (one direction; identical for y and z). */
void orc_tcheb(double *cr, long ise, long isa, long nlines, int nn, int iopt)
{
    double *ctab = cos_table(nn);
    const double dn1 = 1.0 / (double)(nn - 1), dn2 = 0.5 * dn1;
    const int use_fft = nn >= 64;
    orc_fft_plan plan;
    orc_fft_plan_init(&plan, use_fft ? 2 * (nn - 1) : 1);
#pragma omp parallel
    {
        double *buf = (double *)malloc(sizeof(double) * (size_t)nn);
        double *out = (double *)malloc(sizeof(double) * (size_t)nn);
        double *wa = (double *)malloc(sizeof(double) * 4 * (size_t)nn);
        double *wb = (double *)malloc(sizeof(double) * 4 * (size_t)nn);
#define REDFT00(x, X) (use_fft ? redft00_fft(x, X, nn, &plan, wa, wb) : redft00(x, X, nn, ctab))
#pragma omp for
        for (long k = 0; k < nlines; ++k) {
            double *c = cr + k * isa;
            for (int j = 0; j < nn; ++j) buf[j] = c[j * ise];
            if (iopt < 0) {
                REDFT00(buf, out);
                for (int j = 1; j < nn - 1; ++j) c[j * ise] = dn1 * out[j];
                c[0] = dn2 * out[0];
                c[(long)(nn - 1) * ise] = dn2 * out[nn - 1];
            } else {
                buf[0] *= 2.0;
                buf[nn - 1] *= 2.0;
                REDFT00(buf, out);
                for (int j = 0; j < nn; ++j) c[j * ise] = 0.5 * out[j];
            }
        }
#undef REDFT00
        free(buf);
        free(out);
        free(wa);
        free(wb);
    }
    orc_fft_plan_free(&plan);
    free(ctab);
}

/* transyz, src/chebyshev.f90:458-540.                                       */
void orc_transyz(double *cheb, int my, int mz, int nmodes, char cdir, int iopt)
{
    if (cdir == 'y') {
        const long nn = (long)mz * nmodes;
        orc_tcheb(cheb, 2, 2L * my, nn, my, iopt);
        orc_tcheb(cheb + 1, 2, 2L * my, nn, my, iopt);
    } else {
        for (int i = 0; i < nmodes; ++i) {
            double *c = cheb + (size_t)i * my * mz * 2;
            orc_tcheb(c, 2L * my, 2, my, mz, iopt);
            orc_tcheb(c + 1, 2L * my, 2, my, mz, iopt);
        }
    }
}

/* transyz_plane, src/chebyshev.f90:542-595.                                 */
void orc_transyz_plane(double *cheb, int my, int mz, int iopt)
{
    orc_tcheb(cheb, 1, my, mz, my, iopt);
    orc_tcheb(cheb, my, 1, my, mz, iopt);
}

/* One backward recurrence line (src/chebyshev.f90:44-58 pattern):
 * out_k = -d_k for k>=1, out_0 = -d_0/2 with d_{k-1} = d_{k+1} + 2k c_k.    */
static void deriv_line(const double *c, long st, double *out, long so, int n,
                       double fac, int accumulate)
{
    double aari = 0.0, bri = 0.0, tri = 0.0, cri;
    int ia = n;
    for (int ii = 1; ii <= n - 1; ++ii) {
        const int kk = n - ii;
        cri = bri + 2.0 * (double)kk * c[(long)(ia - 1) * st];
        if (accumulate) out[(long)(ia - 1) * so] += -tri * fac;
        else out[(long)(ia - 1) * so] = -tri * fac;
        bri = aari;
        tri = cri;
        aari = cri;
        ia -= 1;
    }
    if (accumulate) out[(long)(ia - 1) * so] += -0.5 * tri * fac;
    else out[(long)(ia - 1) * so] = -0.5 * tri * fac;
}

/* derivyz, src/chebyshev.f90:1-295.  Complex lines: real and imaginary parts
 * follow the same real recurrence (scal is real).                           */
void orc_derivyz(const double *u, double *du, int my, int mz, int nmodes,
                 char cdir, int ider, double scal, char what, double aspect)
{
    const int acc = (what != 'n');
    const int n = (cdir == 'y') ? my : mz;
    const double fz = (cdir == 'y') ? 1.0 : (ider == 1 ? 1.0 / aspect : 1.0 / (aspect * aspect));
    double *aux = (double *)malloc(sizeof(double) * (size_t)n);
    for (int i = 0; i < nmodes; ++i) {
        const size_t base = (size_t)i * my * mz * 2;
        const long nlines = (cdir == 'y') ? mz : my;
        for (long l = 0; l < nlines; ++l) {
            for (int part = 0; part < 2; ++part) {
                size_t off;
                long st;
                if (cdir == 'y') { off = base + 2 * (size_t)l * my + part; st = 2; }
                else { off = base + 2 * (size_t)l + part; st = 2L * my; }
                if (ider == 1) {
                    deriv_line(u + off, st, du + off, st, n, scal * fz, acc);
                } else {
                    deriv_line(u + off, st, aux, 1, n, 1.0, 0);
                    deriv_line(aux, 1, du + off, st, n, scal * fz, acc);
                }
            }
        }
    }
    free(aux);
}

/* cheb2_integral, src/chebyshev.f90:692-723.                                */
double orc_cheb2_integral(const double *u, int ny, int nz, double aspect)
{
    double sum = 0.0;
    for (int j = 0; j < nz; j += 2)
        for (int i = 0; i < ny; i += 2)
            sum += u[IX(i, j, ny)] * 4.0 * aspect /
                   ((double)(j * j - 1) * (double)(i * i - 1));
    return sum;
}

/* cxyz2yzx / cyzx2xyz, src/parallel.F:476-529 (complex*16 elements).       */
void orc_cxyz2yzx(const double *phys, double *phys2, int nmodes, int my, int nz)
{
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < my; ++j)
            for (int i = 0; i < nmodes; ++i) {
                size_t s = (size_t)i + (size_t)nmodes * (j + (size_t)my * k);
                size_t d = (size_t)j + (size_t)my * (k + (size_t)nz * i);
                phys2[2 * d] = phys[2 * s];
                phys2[2 * d + 1] = phys[2 * s + 1];
            }
}

void orc_cyzx2xyz(double *phys, const double *phys2, int nmodes, int my, int nz)
{
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < my; ++j)
            for (int i = 0; i < nmodes; ++i) {
                size_t s = (size_t)j + (size_t)my * (k + (size_t)nz * i);
                size_t d = (size_t)i + (size_t)nmodes * (j + (size_t)my * k);
                phys[2 * d] = phys2[2 * s];
                phys[2 * d + 1] = phys2[2 * s + 1];
            }
}


/* ---- rectangular / general-BC solver --------------------------------- */

/* pseudomaty_temp / pseudomatz_temp, src/pseudomat_temp.f90:2-320.        */
int orc_pseudomat_temp(int m, double sc, char b1, char b2, orc_dir *d)
{
    if (m < 4) return -1;
    memset(d, 0, sizeof(*d));
    const int n = m - 1, mm2 = m - 2;
    const double pi = 4.0 * atan(1.0);
    d->m = m; d->s = sc; d->b1 = b1; d->b2 = b2;
    d->D = (double *)calloc((size_t)m * m, sizeof(double));
    d->D2 = (double *)calloc((size_t)m * m, sizeof(double));
    d->E = (double *)calloc((size_t)mm2, sizeof(double));
    d->P = (double *)calloc((size_t)mm2 * mm2, sizeof(double));
    d->PM1 = (double *)calloc((size_t)mm2 * mm2, sizeof(double));
    d->B = (double *)calloc((size_t)mm2 * mm2, sizeof(double));
    double *y = (double *)calloc((size_t)m, sizeof(double));
    double *dd = (double *)calloc((size_t)m, sizeof(double));
    double *eii = (double *)calloc((size_t)mm2, sizeof(double));
    double *Bt = (double *)calloc((size_t)mm2 * mm2, sizeof(double));
    double *D = d->D, *D2 = d->D2;
    dd[0] = 2.0;
    for (int i = 1; i < m - 1; ++i) dd[i] = 1.0;
    dd[m - 1] = 2.0;
    for (int j = 0; j < m; ++j) y[j] = -cos(pi * (double)j / (double)n);
    D[IX(0, 0, m)] = -(2.0 * (double)n * (double)n + 1.0) / 6.0;
    D[IX(m - 1, m - 1, m)] = -D[IX(0, 0, m)];
    for (int i = 1; i < n; ++i) D[IX(i, i, m)] = -0.5 * y[i] / (1.0 - y[i] * y[i]);
    for (int l = 0; l < m; ++l)
        for (int j = 0; j < m; ++j) {
            if (j == l) continue;
            const double sgn = ((l + j) % 2 == 0) ? 1.0 : -1.0;
            D[IX(l, j, m)] = dd[l] / dd[j] * sgn / (y[l] - y[j]);
        }
    for (size_t i = 0; i < (size_t)m * m; ++i) D[i] *= 1.0 / sc;   /* dscal(1/s) :77 */
    {
        const double one = 1.0, zero = 0.0;
        scipy_dgemm_("n", "n", &m, &m, &m, &one, D, &m, D, &m, &zero, D2, &m, 1, 1);
    }
    const double d11 = D[IX(0, 0, m)], d1m = D[IX(0, m - 1, m)];
    const double dm1 = D[IX(m - 1, 0, m)], dmm = D[IX(m - 1, m - 1, m)];
    for (int i = 1; i < n; ++i)
        for (int j = 1; j < n; ++j) {
            double v;
            if (b1 == 'n' && b2 == 'n') {
                const double Det = d11 * dmm - d1m * dm1;
                const double ter1 = D2[IX(i, 0, m)] * (d1m * D[IX(m - 1, j, m)] - dmm * D[IX(0, j, m)]) / Det;
                const double ter3 = D2[IX(i, m - 1, m)] * (dm1 * D[IX(0, j, m)] - d11 * D[IX(m - 1, j, m)]) / Det;
                v = ter1 + D2[IX(i, j, m)] + ter3;
            } else if (b1 == 'd' && b2 == 'n') {
                v = D2[IX(i, j, m)] - D2[IX(i, m - 1, m)] * D[IX(m - 1, j, m)] / dmm;
            } else if (b1 == 'n' && b2 == 'd') {
                v = D2[IX(i, j, m)] - D2[IX(i, 0, m)] * D[IX(0, j, m)] / d11;
            } else {
                v = D2[IX(i, j, m)];
            }
            d->B[IX(i - 1, j - 1, mm2)] = v;
        }
    memcpy(Bt, d->B, sizeof(double) * (size_t)mm2 * mm2);
    int info = eigen(mm2, Bt, d->E, eii, d->P);
    if (!info) {
        memcpy(d->PM1, d->P, sizeof(double) * (size_t)mm2 * mm2);
        info = invert(mm2, d->PM1);
    }
    free(y); free(dd); free(eii); free(Bt);
    return info;
}

void orc_dir_free(orc_dir *d)
{
    free(d->D); free(d->D2); free(d->E); free(d->P); free(d->PM1); free(d->B);
    memset(d, 0, sizeof(*d));
}

static int argmin_abs(const double *E, int n)
{
    int k = 0;
    for (int i = 1; i < n; ++i)
        if (fabs(E[i]) < fabs(E[k])) k = i;
    return k;
}

/* solvediag_temp + mod_term_FTy/z + edge_value_y/z.                        */
int orc_solvediag_temp(double *U, const orc_dir *yd, const orc_dir *zd, double xlambda,
                       const double *bcy, const double *bcz, int sing)
{
    const int my = yd->m, mz = zd->m, ny = my - 2, nz = mz - 2;
    double *F = (double *)calloc((size_t)ny * nz, sizeof(double));
    double *FT = (double *)calloc((size_t)ny * nz, sizeof(double));
    const double *DY = yd->D, *DZ = zd->D, *D2Y = yd->D2, *D2Z = zd->D2;
    for (int j = 1; j < mz - 1; ++j)
        for (int i = 1; i < my - 1; ++i) F[IX(i - 1, j - 1, ny)] = U[IX(i, j, my)];
    /* mod_term_FTy / mod_term_FTz (src/solvediag_temp.f90:86-239) */
    for (int j = 1; j < mz - 1; ++j)
        for (int i = 1; i < my - 1; ++i) {
            double v = 0.0, h = 0.0;
            if (bcy) {
                const double c1 = bcy[j], c2 = bcy[j + mz];
                const double a1 = D2Y[IX(i, 0, my)], a2 = D2Y[IX(i, my - 1, my)];
                if (yd->b1 == 'd' && yd->b2 == 'd') v = -a1 * c1 - a2 * c2;
                else if (yd->b1 == 'd' && yd->b2 == 'n')
                    v = -a1 * c1 - a2 * (c2 - DY[IX(my - 1, 0, my)] * c1) / DY[IX(my - 1, my - 1, my)];
                else if (yd->b1 == 'n' && yd->b2 == 'd')
                    v = -a1 * (c1 - DY[IX(0, my - 1, my)] * c2) / DY[IX(0, 0, my)] - a2 * c2;
                else {
                    const double Det = DY[IX(0, 0, my)] * DY[IX(my - 1, my - 1, my)] - DY[IX(0, my - 1, my)] * DY[IX(my - 1, 0, my)];
                    v = a1 * (DY[IX(0, my - 1, my)] * c2 - DY[IX(my - 1, my - 1, my)] * c1) / Det +
                        a2 * (DY[IX(my - 1, 0, my)] * c1 - DY[IX(0, 0, my)] * c2) / Det;
                }
            }
            if (bcz) {
                const double c1 = bcz[i], c2 = bcz[i + my];
                const double a1 = D2Z[IX(j, 0, mz)], a2 = D2Z[IX(j, mz - 1, mz)];
                if (zd->b1 == 'd' && zd->b2 == 'd') h = -a1 * c1 - a2 * c2;
                else if (zd->b1 == 'd' && zd->b2 == 'n')
                    h = -a1 * c1 - a2 * (c2 - DZ[IX(mz - 1, 0, mz)] * c1) / DZ[IX(mz - 1, mz - 1, mz)];
                else if (zd->b1 == 'n' && zd->b2 == 'd')
                    h = -a1 * (c1 - DZ[IX(0, mz - 1, mz)] * c2) / DZ[IX(0, 0, mz)] - a2 * c2;
                else {
                    const double Det = DZ[IX(0, 0, mz)] * DZ[IX(mz - 1, mz - 1, mz)] - DZ[IX(0, mz - 1, mz)] * DZ[IX(mz - 1, 0, mz)];
                    h = a1 * (DZ[IX(0, mz - 1, mz)] * c2 - DZ[IX(mz - 1, mz - 1, mz)] * c1) / Det +
                        a2 * (DZ[IX(mz - 1, 0, mz)] * c1 - DZ[IX(0, 0, mz)] * c2) / Det;
                }
            }
            F[IX(i - 1, j - 1, ny)] += v + h;
        }
    /* F = PTYM1 F PTZM1^T ; divide ; FT = PTY F PTZ^T  (:47-64) */
    {
        const double one = 1.0, zero = 0.0;
        scipy_dgemm_("n", "n", &ny, &nz, &ny, &one, yd->PM1, &ny, F, &ny, &zero, FT, &ny, 1, 1);
        scipy_dgemm_("n", "t", &ny, &nz, &nz, &one, FT, &ny, zd->PM1, &nz, &zero, F, &ny, 1, 1);
        const int iy0 = argmin_abs(yd->E, ny), iz0 = argmin_abs(zd->E, nz);
        for (int j = 0; j < nz; ++j)
            for (int i = 0; i < ny; ++i) {
                if (sing && i == iy0 && j == iz0) { FT[IX(i, j, ny)] = 0.0; continue; }
                FT[IX(i, j, ny)] = F[IX(i, j, ny)] / (yd->E[i] + zd->E[j] - xlambda);
            }
        scipy_dgemm_("n", "n", &ny, &nz, &ny, &one, yd->P, &ny, FT, &ny, &zero, F, &ny, 1, 1);
        scipy_dgemm_("n", "t", &ny, &nz, &nz, &one, F, &ny, zd->P, &nz, &zero, FT, &ny, 1, 1);
    }
    for (int j = 0; j < nz; ++j)
        for (int i = 0; i < ny; ++i) U[IX(i + 1, j + 1, my)] = FT[IX(i, j, ny)];
    /* edge_value_y (:241-300): walls y = -1, +1 for interior columns j */
    for (int j = 1; j < mz - 1; ++j) {
        const double c1 = bcy ? bcy[j] : 0.0, c2 = bcy ? bcy[j + mz] : 0.0;
        double a = 0.0, b = 0.0;
        for (int i = 1; i < my - 1; ++i) {
            a += DY[IX(0, i, my)] * U[IX(i, j, my)];
            b += DY[IX(my - 1, i, my)] * U[IX(i, j, my)];
        }
        if (yd->b1 == 'd' && yd->b2 == 'd') { U[IX(0, j, my)] = c1; U[IX(my - 1, j, my)] = c2; }
        else if (yd->b1 == 'd' && yd->b2 == 'n') {
            U[IX(0, j, my)] = c1;
            U[IX(my - 1, j, my)] = (c2 - DY[IX(my - 1, 0, my)] * U[IX(0, j, my)] - b) / DY[IX(my - 1, my - 1, my)];
        } else if (yd->b1 == 'n' && yd->b2 == 'd') {
            U[IX(my - 1, j, my)] = c2;
            U[IX(0, j, my)] = (c1 - DY[IX(0, my - 1, my)] * U[IX(my - 1, j, my)] - a) / DY[IX(0, 0, my)];
        } else {
            const double Det = DY[IX(0, 0, my)] * DY[IX(my - 1, my - 1, my)] - DY[IX(0, my - 1, my)] * DY[IX(my - 1, 0, my)];
            U[IX(0, j, my)] = (DY[IX(my - 1, my - 1, my)] * (c1 - a) - DY[IX(0, my - 1, my)] * (c2 - b)) / Det;
            U[IX(my - 1, j, my)] = (-DY[IX(my - 1, 0, my)] * (c1 - a) + DY[IX(0, 0, my)] * (c2 - b)) / Det;
        }
    }
    /* edge_value_z (:302-351) */
    for (int i = 1; i < my - 1; ++i) {
        const double c1 = bcz ? bcz[i] : 0.0, c2 = bcz ? bcz[i + my] : 0.0;
        double a = 0.0, b = 0.0;
        for (int j = 1; j < mz - 1; ++j) {
            a += DZ[IX(0, j, mz)] * U[IX(i, j, my)];
            b += DZ[IX(mz - 1, j, mz)] * U[IX(i, j, my)];
        }
        if (zd->b1 == 'd' && zd->b2 == 'd') { U[IX(i, 0, my)] = c1; U[IX(i, mz - 1, my)] = c2; }
        else if (zd->b1 == 'd' && zd->b2 == 'n') {
            U[IX(i, 0, my)] = c1;
            U[IX(i, mz - 1, my)] = (c2 - DZ[IX(mz - 1, 0, mz)] * U[IX(i, 0, my)] - b) / DZ[IX(mz - 1, mz - 1, mz)];
        } else if (zd->b1 == 'n' && zd->b2 == 'd') {
            U[IX(i, mz - 1, my)] = c2;
            U[IX(i, 0, my)] = (c1 - DZ[IX(0, mz - 1, mz)] * U[IX(i, mz - 1, my)] - a) / DZ[IX(0, 0, mz)];
        } else {
            const double Det = DZ[IX(0, 0, mz)] * DZ[IX(mz - 1, mz - 1, mz)] - DZ[IX(0, mz - 1, mz)] * DZ[IX(mz - 1, 0, mz)];
            U[IX(i, 0, my)] = (DZ[IX(mz - 1, mz - 1, mz)] * (c1 - a) - DZ[IX(0, mz - 1, mz)] * (c2 - b)) / Det;
            U[IX(i, mz - 1, my)] = (-DZ[IX(mz - 1, 0, mz)] * (c1 - a) + DZ[IX(0, 0, mz)] * (c2 - b)) / Det;
        }
    }
    free(F);
    free(FT);
    return 0;
}

int orc_helm3d_temp(const double *rhs, double *sol, int my, int mz, int ib, int ie,
                    const double *xalp, double alambda, const orc_dir *yd, const orc_dir *zd,
                    const double *bcy, const double *bcz, int nthreads)
{
    const int nmodes = ie - ib + 1;
    const size_t plane = (size_t)my * mz;
    if (nthreads < 1) nthreads = 1;
#pragma omp parallel num_threads(nthreads)
    {
        double *U = (double *)malloc(sizeof(double) * plane);
#pragma omp for schedule(dynamic, 1)
        for (int i = 0; i < nmodes; ++i) {
            const int imode = ib + i;
            const double xl = alambda + xalp[i] * xalp[i];
            const int sing = (yd->b1 == 'n' && yd->b2 == 'n' && zd->b1 == 'n' && zd->b2 == 'n' && fabs(xl) <= 1.0e-10);
            const double *r = rhs + 2 * plane * (size_t)i;
            double *s = sol + 2 * plane * (size_t)i;
            const double *by = bcy ? bcy + (size_t)2 * mz * i : NULL;
            const double *bz = bcz ? bcz + (size_t)2 * my * i : NULL;
            for (size_t p = 0; p < plane; ++p) U[p] = r[2 * p];
            orc_solvediag_temp(U, yd, zd, xl, by, bz, sing);
            for (size_t p = 0; p < plane; ++p) { s[2 * p] = U[p]; s[2 * p + 1] = 0.0; }
            if (imode == 0) continue;
            for (size_t p = 0; p < plane; ++p) U[p] = r[2 * p + 1];
            orc_solvediag_temp(U, yd, zd, xl, by, bz, sing);
            for (size_t p = 0; p < plane; ++p) s[2 * p + 1] += U[p];
        }
        free(U);
    }
    return 0;
}

/* ---- Shen-Legendre Galerkin solver ------------------------------------- */
/* generalized symmetric eigenproblem A x = w B x (itype 1), as the
 * reference's dsygv call (src/preshen.f90:463-496).                        */
static int sygv(int n, double *A, double *B, double *w)
{
    int itype = 1, info = 0, lwk = -1;
    double q = 0.0;
    scipy_dsygv_(&itype, "V", "U", &n, A, &n, B, &n, w, &q, &lwk, &info, 1, 1);
    lwk = (int)q + 16;
    double *wk = (double *)malloc(sizeof(double) * (size_t)lwk);
    scipy_dsygv_(&itype, "V", "U", &n, A, &n, B, &n, w, wk, &lwk, &info, 1, 1);
    free(wk);
    return info;
}

/* preshen + makeMS + precomeigen (src/preshen.f90:2-535) and leg_cheb_mat
 * (src/legendre.f90:3-110).                                               */
int orc_shen_setup(int m, char bound, orc_shen *s)
{
    if (m < 5 || (m % 2) == 0) return -1;
    memset(s, 0, sizeof(*s));
    const int n = m - 2, nm1 = m - 1;
    s->m = m;
    s->bound = bound;
    s->b = (double *)calloc((size_t)m, sizeof(double));
    s->M = (double *)calloc((size_t)n * n, sizeof(double));
    s->S = (double *)calloc((size_t)n * n, sizeof(double));
    s->E = (double *)calloc((size_t)n, sizeof(double));
    s->P = (double *)calloc((size_t)n * n, sizeof(double));
    s->PSM1 = (double *)calloc((size_t)n * n, sizeof(double));
    s->A = (double *)calloc((size_t)m * m, sizeof(double));
    s->B = (double *)calloc((size_t)m * m, sizeof(double));
    for (int kk = 0; kk < m; ++kk)                      /* makeMS :359-371 */
        s->b[kk] = (bound == 'd') ? -1.0 : -(double)(kk * (kk + 1)) / (double)((kk + 2) * (kk + 3));
    for (int k = 0; k < n; ++k) {                       /* precomeigen :450-460 */
        s->S[IX(k, k, n)] = -s->b[k] * (double)(4 * k + 6);
        s->M[IX(k, k, n)] = 2.0 / (double)(2 * k + 1) + 2.0 * s->b[k] * s->b[k] / (double)(2 * k + 5);
    }
    if (bound == 'n') s->S[0] = 2.0;
    for (int k = 0; k < n - 2; ++k) {
        const double v = s->b[k] * 2.0 / (double)(2 * k + 5);
        s->M[IX(k, k + 2, n)] = v;
        s->M[IX(k + 2, k, n)] = v;
    }
    int info = 0;
    if (bound == 'd') {
        double *Pv = (double *)malloc(sizeof(double) * (size_t)n * n);
        double *St = (double *)malloc(sizeof(double) * (size_t)n * n);
        memcpy(Pv, s->M, sizeof(double) * (size_t)n * n);
        memcpy(St, s->S, sizeof(double) * (size_t)n * n);
        info = sygv(n, Pv, St, s->E);
        memcpy(s->P, Pv, sizeof(double) * (size_t)n * n);
        free(Pv); free(St);
    } else {
        const int n1 = n - 1;                            /* :479-496 */
        double *M1 = (double *)calloc((size_t)n1 * n1, sizeof(double));
        double *S1 = (double *)calloc((size_t)n1 * n1, sizeof(double));
        double *E1 = (double *)calloc((size_t)n1, sizeof(double));
        for (int j = 0; j < n1; ++j)
            for (int i = 0; i < n1; ++i) {
                M1[IX(i, j, n1)] = s->M[IX(i + 1, j + 1, n)];
                S1[IX(i, j, n1)] = s->S[IX(i + 1, j + 1, n)];
            }
        info = sygv(n1, M1, S1, E1);
        s->P[0] = 1.0;
        s->E[0] = 1.0;
        for (int i = 0; i < n1; ++i) {
            s->E[i + 1] = E1[i];
            for (int j = 0; j < n1; ++j) s->P[IX(i + 1, j + 1, n)] = M1[IX(i, j, n1)];
        }
        free(M1); free(S1); free(E1);
    }
    if (info) return info;
    memcpy(s->PSM1, s->P, sizeof(double) * (size_t)n * n);   /* :516-530 */
    if ((info = invert(n, s->PSM1))) return info;
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) s->PSM1[IX(i, j, n)] /= s->S[IX(j, j, n)];
    /* leg_cheb_mat: A upper triangular by the recurrence :56-82 */
    double *A = s->A;
    A[IX(0, 0, m)] = 1.0;
    A[IX(1, 1, m)] = 1.0;
    for (int k = 2; k <= nm1; ++k) A[IX(k, k, m)] = 2.0 * (double)k / (double)(2 * k - 1) * A[IX(k - 1, k - 1, m)];
    for (int k = 2; k <= nm1; k += 2) A[IX(0, k, m)] = -1.0 / (double)(k * k - 1);
    for (int j = 2; j <= nm1 - 1; ++j) {                 /* Fortran j=2..n-1, jj=j+1 */
        const int jj = j + 1;
        for (int i = 1; i <= j; ++i) {
            const int ii = i + 1;
            const double c1 = (double)(2 * i + 2) / (double)(2 * i + 3);
            const double c2 = (double)(2 * i) / (double)(2 * i - 1);
            /* A(ii,jj+1)=c1*A(ii+1,jj)+c2*A(ii-1,jj)-A(ii,jj-1), 1-based */
            A[IX(ii - 1, jj, m)] = c1 * A[IX(ii, jj - 1, m)] + c2 * A[IX(ii - 2, jj - 1, m)] - A[IX(ii - 1, jj - 2, m)];
        }
    }
    memcpy(s->B, A, sizeof(double) * (size_t)m * m);
    return invert(m, s->B);
}

void orc_shen_free(orc_shen *s)
{
    free(s->b); free(s->M); free(s->S); free(s->E); free(s->P); free(s->PSM1); free(s->A); free(s->B);
    memset(s, 0, sizeof(*s));
}

/* Largest |entry| of the parity-mixing blocks of P, P^-1 S^-1 and A that
 * the reference's even/odd split drops, relative to the largest entry.    */
double orc_shen_parity_leak(const orc_shen *s)
{
    const int n = s->m - 2, m = s->m;
    double leak = 0.0, big = 0.0;
    /* Dirichlet pairs even rows with even (0-based) eigen-columns; the
     * Neumann split pairs even rows with odd columns (src/preshen.f90:
     * 203-287), except column 0 (the repaired constant mode).              */
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
            const int same = ((i & 1) == (j & 1));
            const int kept = (s->bound == 'd') ? same : (j == 0 ? (i == 0) : !same);
            const double a = fmax(fabs(s->P[IX(i, j, n)]), fabs(s->PSM1[IX(j, i, n)]));
            big = fmax(big, a);
            if (!kept) leak = fmax(leak, a);
        }
    for (int j = 0; j < m; ++j)
        for (int i = 0; i < m; ++i)
            if (((i + j) & 1) && s->A[IX(i, j, m)] != 0.0) leak = fmax(leak, fabs(s->A[IX(i, j, m)]));
    return leak / big;
}

/* DPTSV on a symmetric tridiagonal (d, e) of order k, right-hand side f.  */
static void ptsv(int k, double *d, double *e, double *f)
{
    int one = 1, info = 0;
    scipy_dptsv_(&k, &one, d, e, f, &k, &info);
}

/* solveshen, src/solveshen.f90:5-94 with chebleg2d, legshen2d,
 * multevenodd, solV and solevenodd (src/legendre.f90:195-660,
 * src/solveshen.f90:96-546).  The parity halves are kept together in full
 * matrices (their coupling is round-off, orc_shen_parity_leak).           */
int orc_solveshen(double *U, const orc_shen *s, double xlambda)
{
    const int m = s->m, n = m - 2;
    const double *b = s->b;
    double *G = (double *)calloc((size_t)m * m, sizeof(double));
    double *T = (double *)calloc((size_t)m * m, sizeof(double));
    double *F = (double *)calloc((size_t)n * n, sizeof(double));
    double *W = (double *)calloc((size_t)n * n, sizeof(double));
    const double one = 1.0, zero = 0.0;
    /* chebleg2d(+1): G = A U A^T */
    scipy_dgemm_("n", "n", &m, &m, &m, &one, s->A, &m, U, &m, &zero, T, &m, 1, 1);
    scipy_dgemm_("n", "t", &m, &m, &m, &one, T, &m, s->A, &m, &zero, G, &m, 1, 1);
    /* legshen2d(+1): leg2shen_sweep2d (src/legendre.f90:562-589) */
    for (int jj = 0; jj < n; ++jj) {
        const double ta = 2.0 / (double)(2 * jj + 1), tb = 2.0 * b[jj] / (double)(2 * jj + 5);
        for (int ii = 0; ii < n; ++ii) {
            const double tc = 2.0 / (double)(2 * ii + 1), td = 2.0 * b[ii] / (double)(2 * ii + 5);
            F[IX(ii, jj, n)] = ta * (G[IX(ii, jj, m)] * tc + G[IX(ii + 2, jj, m)] * td) +
                               tb * (G[IX(ii, jj + 2, m)] * tc + G[IX(ii + 2, jj + 2, m)] * td);
        }
    }
    /* multevenodd(+1): W = P^-1 S^-1 F along y */
    scipy_dgemm_("n", "n", &n, &n, &n, &one, s->PSM1, &n, F, &n, &zero, W, &n, 1, 1);
    /* solV: per y-eigen-index ip, two SPD tridiagonal systems along z */
    const int me = (n + 1) / 2, mo = n / 2;
    double *de = (double *)malloc(sizeof(double) * (size_t)me), *ee = (double *)malloc(sizeof(double) * (size_t)me);
    double *dd = (double *)malloc(sizeof(double) * (size_t)mo), *eo = (double *)malloc(sizeof(double) * (size_t)mo);
    double *fe = (double *)malloc(sizeof(double) * (size_t)me), *fo = (double *)malloc(sizeof(double) * (size_t)mo);
    const double *Md = s->M;
    for (int ip = 0; ip < n; ++ip) {
        const int neu_first = (s->bound == 'n' && ip == 0);
        const double rho = neu_first ? 0.0 : s->E[ip];
        const double ra1 = neu_first ? xlambda : rho * xlambda + 1.0;
        /* solV uses makeMS's stiffness -b_k (4k+6) (src/preshen.f90:375-379),
         * i.e. 0 for the Neumann constant mode, not precomeigen's S~ = 2.
         * Dirichlet and Neumann ip>1: rho (alpha M + S) + M;
         * Neumann ip=1: alpha M + S (src/solveshen.f90:410-421).           */
        for (int q = 0; q < me; ++q) {
            const int k = 2 * q;
            const double Mk = Md[IX(k, k, n)], Sk = -b[k] * (double)(4 * k + 6);
            de[q] = neu_first ? (xlambda * Mk + Sk) : (rho * (xlambda * Mk + Sk) + Mk);
            if (q < me - 1) ee[q] = ra1 * Md[IX(k, k + 2, n)];
            fe[q] = W[IX(ip, k, n)];
        }
        for (int q = 0; q < mo; ++q) {
            const int k = 2 * q + 1;
            const double Mk = Md[IX(k, k, n)], Sk = -b[k] * (double)(4 * k + 6);
            dd[q] = neu_first ? (xlambda * Mk + Sk) : (rho * (xlambda * Mk + Sk) + Mk);
            if (q < mo - 1) eo[q] = ra1 * Md[IX(k, k + 2, n)];
            fo[q] = W[IX(ip, k, n)];
        }
        if (neu_first && xlambda < 1.0e-10) {            /* the intended pin :424-432 */
            de[0] = 1.0;
            fe[0] = 0.0;
        }
        ptsv(me, de, ee, fe);
        ptsv(mo, dd, eo, fo);
        for (int q = 0; q < me; ++q) W[IX(ip, 2 * q, n)] = fe[q];
        for (int q = 0; q < mo; ++q) W[IX(ip, 2 * q + 1, n)] = fo[q];
    }
    free(de); free(ee); free(dd); free(eo); free(fe); free(fo);
    /* multevenodd(-1): F = P W along y */
    scipy_dgemm_("n", "n", &n, &n, &n, &one, s->P, &n, W, &n, &zero, F, &n, 1, 1);
    /* legshen2d(-1): shen2leg_sweep2d (src/legendre.f90:627-660) */
    for (int jj = 0; jj < m; ++jj)
        for (int ii = 0; ii < m; ++ii) {
            const double bi = ii >= 2 ? b[ii - 2] : 0.0, bj = jj >= 2 ? b[jj - 2] : 0.0;
            const double s00 = (ii < n && jj < n) ? F[IX(ii, jj, n)] : 0.0;
            const double s10 = (ii >= 2 && jj < n) ? F[IX(ii - 2, jj, n)] : 0.0;
            const double s01 = (ii < n && jj >= 2) ? F[IX(ii, jj - 2, n)] : 0.0;
            const double s11 = (ii >= 2 && jj >= 2) ? F[IX(ii - 2, jj - 2, n)] : 0.0;
            G[IX(ii, jj, m)] = s00 + s01 * bj + s10 * bi + bi * bj * s11;
        }
    /* chebleg2d(-1): U = B G B^T */
    scipy_dgemm_("n", "n", &m, &m, &m, &one, s->B, &m, G, &m, &zero, T, &m, 1, 1);
    scipy_dgemm_("n", "t", &m, &m, &m, &one, T, &m, s->B, &m, &zero, U, &m, 1, 1);
    free(G); free(T); free(F); free(W);
    return 0;
}

/* helm3d_shen, src/helm_shen.f90:2-85: rhs -> Chebyshev coefficients in
 * place (transyz y and z, iopt -1), int2d3d per mode (the real and the
 * imaginary part each through solveshen; mode 0 real), solution back to
 * physical space (transyz y and z, iopt +1).                              */
int orc_helm3d_shen(double *rhs, double *sol, int my, int mz, int ib, int ie,
                    const double *xalp, double alambda, const orc_shen *s, int nthreads)
{
    if (my != mz || my != s->m) return -2;
    const int nmodes = ie - ib + 1;
    const size_t plane = (size_t)my * mz;
    orc_transyz(rhs, my, mz, nmodes, 'y', -1);
    orc_transyz(rhs, my, mz, nmodes, 'z', -1);
    if (nthreads < 1) nthreads = 1;
#pragma omp parallel num_threads(nthreads)
    {
        double *U = (double *)malloc(sizeof(double) * plane);
#pragma omp for schedule(dynamic, 1)
        for (int i = 0; i < nmodes; ++i) {
            const double xl = alambda + xalp[i] * xalp[i];
            const double *r = rhs + 2 * plane * (size_t)i;
            double *so = sol + 2 * plane * (size_t)i;
            for (size_t p = 0; p < plane; ++p) U[p] = r[2 * p];
            orc_solveshen(U, s, xl);
            for (size_t p = 0; p < plane; ++p) { so[2 * p] = U[p]; so[2 * p + 1] = 0.0; }
            if (ib + i == 0) continue;
            for (size_t p = 0; p < plane; ++p) U[p] = r[2 * p + 1];
            orc_solveshen(U, s, xl);
            for (size_t p = 0; p < plane; ++p) so[2 * p + 1] += U[p];
        }
        free(U);
    }
    orc_transyz(sol, my, mz, nmodes, 'y', 1);
    orc_transyz(sol, my, mz, nmodes, 'z', 1);
    return 0;
}

/* ---- constant mass-flow-rate forcing ----------------------------------- */
/* precomp_mass_flow, src/operators.F:2205-2289 (square build): for each RK
 * index krk, solve (dyy+dzz)u - u/(alphak dtp fnu) = 1 in the interior with
 * zero walls (solvediag 'd'), store it in premassfu(:,krk) and its
 * integral (transyz_plane -1, cheb2_integral) in premassf(krk).           */
int orc_precomp_mass_flow(const orc_ops *o, double dtp, const double *alphak, int mrk,
                          double fnu, double aspect, double *premassfu, double *premassf)
{
    const int m = o->m;
    const size_t plane = (size_t)m * m;
    double *w = (double *)malloc(sizeof(double) * plane);
    for (int k = 0; k < mrk; ++k) {
        const double flambda = -1.0 / (alphak[k] * dtp * fnu);
        double *U = premassfu + plane * (size_t)k;
        for (size_t p = 0; p < plane; ++p) U[p] = 1.0;
        for (int i = 0; i < m; ++i) {
            U[IX(i, 0, m)] = U[IX(i, m - 1, m)] = 0.0;
            U[IX(0, i, m)] = U[IX(m - 1, i, m)] = 0.0;
        }
        int rc = orc_solvediag(U, o, 'd', -flambda);
        if (rc) { free(w); return rc; }
        memcpy(w, U, sizeof(double) * plane);
        orc_transyz_plane(w, m, m, -1);
        premassf[k] = orc_cheb2_integral(w, m, m, aspect);
    }
    free(w);
    return 0;
}

/* impose_mass_flow, src/operators.F:2291-2344: the mass flow of the real
 * part of mode 0 of u (complex (my,mz), first plane); iflag 0 returns it
 * in *csum, iflag 1 adds fac premassfu(:,krk) (krk 1-based) with
 * fac = (csum - sumg)/premassf(krk).  Returns sumg.                       */
double orc_impose_mass_flow(double *csum, int krk, double *u, int my, int mz, double aspect,
                            const double *premassfu, const double *premassf, int iflag)
{
    const size_t plane = (size_t)my * mz;
    double *w = (double *)malloc(sizeof(double) * plane);
    for (size_t p = 0; p < plane; ++p) w[p] = u[2 * p];
    orc_transyz_plane(w, my, mz, -1);
    const double sumg = orc_cheb2_integral(w, my, mz, aspect);
    free(w);
    if (iflag == 0) {
        *csum = sumg;
        return sumg;
    }
    const double fac = (*csum - sumg) / premassf[krk - 1];
    const double *pu = premassfu + plane * (size_t)(krk - 1);
    for (size_t p = 0; p < plane; ++p) u[2 * p] += fac * pu[p];
    return sumg;
}

/* ---- Galerkin-basis Neumann (pressure) solver -------------------------- */
/* T_n(x) and T_n''(x) at an interior node, tch0/tch2 of
 * src/pseudopois.f90:84-104 (theta = acos x).                              */
static double tch0(int n, double x) { return cos((double)n * acos(x)); }
static double tch2(int n, double x)
{
    const double a = (double)n * acos(x), t0 = cos(a), den = 1.0 - x * x;
    return (x * sin(a) - (double)n * t0 * sqrt(den)) * (double)n / pow(den, 1.5);
}

/* pseudopois(m), src/pseudopois.f90:2-82: basis phi_j = T_j - j^2/(j+2)^2
 * T_{j+2} (phi_j'(+-1) = 0), B(i,j) = phi_j(x_i) and B2 = phi_j''(x_i) on the
 * interior nodes, PNT = B^-1, D = B2 B^-1, its eigen-decomposition (dgeev),
 * PNM1, iofzero (smallest |EN|, strict update), wanted = 0.                */
int orc_pseudopois(int m, orc_pois *p)
{
    if (m < 5) return -1;
    memset(p, 0, sizeof(*p));
    const int n = m - 1, mm2 = m - 2;
    const double pi = 4.0 * atan(1.0);
    p->m = m;
    p->EN = (double *)calloc((size_t)mm2, sizeof(double));
    double *ENim = (double *)calloc((size_t)mm2, sizeof(double));
    p->PN = (double *)calloc((size_t)mm2 * mm2, sizeof(double));
    p->PNM1 = (double *)calloc((size_t)mm2 * mm2, sizeof(double));
    p->PNT = (double *)calloc((size_t)mm2 * mm2, sizeof(double));
    double *wk1 = (double *)calloc((size_t)mm2 * mm2, sizeof(double));
    double *D = (double *)calloc((size_t)mm2 * mm2, sizeof(double));
    double *x = (double *)calloc((size_t)m, sizeof(double));
    for (int j = 0; j < m; ++j) x[j] = -cos(pi * (double)j / (double)n);
    for (int i = 1; i < m - 1; ++i)
        for (int j = 0; j < mm2; ++j) {
            const double c = (double)(j * j) / (((double)j + 2.0) * ((double)j + 2.0));
            p->PNT[IX(i - 1, j, mm2)] = tch0(j, x[i]) - c * tch0(j + 2, x[i]);
            wk1[IX(i - 1, j, mm2)] = tch2(j, x[i]) - c * tch2(j + 2, x[i]);
        }
    int info = invert(mm2, p->PNT);
    if (!info) {
        const double one = 1.0, zero = 0.0;
        scipy_dgemm_("n", "n", &mm2, &mm2, &mm2, &one, wk1, &mm2, p->PNT, &mm2, &zero, D, &mm2, 1, 1);
        info = eigen(mm2, D, p->EN, ENim, p->PN);
    }
    if (!info) {
        memcpy(p->PNM1, p->PN, sizeof(double) * (size_t)mm2 * mm2);
        info = invert(mm2, p->PNM1);
    }
    double eigmin = 1.0e6;
    for (int i = 0; i < mm2; ++i) {
        const double e = fmin(eigmin, fabs(p->EN[i]));
        if (e != eigmin) { p->iofzero = i + 1; eigmin = e; }
    }
    p->wanted = 0.0;
    free(ENim); free(wk1); free(D); free(x);
    return info;
}

void orc_pois_free(orc_pois *p)
{
    free(p->EN); free(p->PN); free(p->PNM1); free(p->PNT);
    memset(p, 0, sizeof(*p));
}

/* solvepois(U,F,FT,wk1,wk2,xlambda,m), src/solvepois.f90:1-170.          */
int orc_solvepois(double *U, const orc_pois *p, double xlambda)
{
    const int m = p->m, mm2 = m - 2, io = p->iofzero - 1;
    const double one = 1.0, zero = 0.0;
    double *F = (double *)calloc((size_t)mm2 * mm2, sizeof(double));
    double *FT = (double *)calloc((size_t)mm2 * mm2, sizeof(double));
    double *w1 = (double *)calloc((size_t)mm2 * mm2, sizeof(double));
    double *w2 = (double *)calloc((size_t)mm2 * mm2, sizeof(double));
    for (int j = 0; j < mm2; ++j)
        for (int i = 0; i < mm2; ++i) F[IX(i, j, mm2)] = U[IX(i + 1, j + 1, m)];
    scipy_dgemm_("n", "n", &mm2, &mm2, &mm2, &one, p->PNM1, &mm2, F, &mm2, &zero, FT, &mm2, 1, 1);
    scipy_dgemm_("n", "t", &mm2, &mm2, &mm2, &one, FT, &mm2, p->PNM1, &mm2, &zero, F, &mm2, 1, 1);
    for (int j = 0; j < mm2; ++j)
        for (int i = 0; i < mm2; ++i)
            FT[IX(i, j, mm2)] = F[IX(i, j, mm2)] / (p->EN[i] + p->EN[j] - xlambda);
    if (!(fabs(xlambda) > 1.0e-10)) {
        /* :38-86: skip the zero eigen-coefficient, then choose it so that the
         * solution takes the value wanted at (iofzero+1, iofzero+1)         */
        FT[IX(io, io, mm2)] = 0.0;
        double valore = 0.0;
        for (int l = 0; l < mm2; ++l) {
            double val = 0.0;
            for (int k = 0; k < mm2; ++k) val += p->PN[IX(io, k, mm2)] * FT[IX(l, k, mm2)];
            valore += p->PN[IX(io, l, mm2)] * val;
        }
        FT[IX(io, io, mm2)] = (p->wanted - valore) / (p->PN[IX(io, io, mm2)] * p->PN[IX(io, io, mm2)]);
    }
    scipy_dgemm_("n", "n", &mm2, &mm2, &mm2, &one, p->PN, &mm2, FT, &mm2, &zero, F, &mm2, 1, 1);
    scipy_dgemm_("n", "t", &mm2, &mm2, &mm2, &one, F, &mm2, p->PN, &mm2, &zero, FT, &mm2, 1, 1);
    for (int j = 0; j < mm2; ++j)
        for (int i = 0; i < mm2; ++i) U[IX(i + 1, j + 1, m)] = FT[IX(i, j, mm2)];
    /* corners :104-139: basis coefficients a = B^-1 U B^-T, phi_j(+-1) */
    scipy_dgemm_("n", "n", &mm2, &mm2, &mm2, &one, p->PNT, &mm2, FT, &mm2, &zero, w1, &mm2, 1, 1);
    scipy_dgemm_("n", "t", &mm2, &mm2, &mm2, &one, w1, &mm2, p->PNT, &mm2, &zero, w2, &mm2, 1, 1);
    double vsw = 0.0, vse = 0.0, vnw = 0.0, vne = 0.0;
    for (int i = 0; i < mm2; ++i) {
        const double si = (i & 1) ? -1.0 : 1.0, vpol = (double)(i + 1) / (double)((i + 2) * (i + 2));
        double isw = 0.0, ise = 0.0, inw = 0.0, ine = 0.0;
        for (int j = 0; j < mm2; ++j) {
            const double sj = (j & 1) ? -1.0 : 1.0, coej = (double)(j + 1) / (double)((j + 2) * (j + 2));
            const double a = w2[IX(i, j, mm2)];
            isw += sj * coej * a;
            ise += sj * coej * a;
            inw += coej * a;
            ine += coej * a;
        }
        vsw += si * vpol * isw;
        vse += vpol * ise;
        vnw += si * vpol * inw;
        vne += vpol * ine;
    }
    U[IX(0, 0, m)] = 16.0 * vsw;
    U[IX(m - 1, 0, m)] = 16.0 * vse;
    U[IX(0, m - 1, m)] = 16.0 * vnw;
    U[IX(m - 1, m - 1, m)] = 16.0 * vne;
    /* edges :141-169: w1 = B^-1 U (coefficients along y), w2 = U B^-T */
    scipy_dgemm_("n", "t", &mm2, &mm2, &mm2, &one, FT, &mm2, p->PNT, &mm2, &zero, w2, &mm2, 1, 1);
    for (int j = 1; j < m - 1; ++j) {
        double vl = 0.0, vr = 0.0;
        for (int i = 0; i < mm2; ++i) {
            const double c = (double)(i + 1) / (double)((i + 2) * (i + 2)), s = (i & 1) ? -1.0 : 1.0;
            vl += s * c * w1[IX(i, j - 1, mm2)];
            vr += c * w1[IX(i, j - 1, mm2)];
        }
        U[IX(0, j, m)] = 4.0 * vl;
        U[IX(m - 1, j, m)] = 4.0 * vr;
    }
    for (int i = 1; i < m - 1; ++i) {
        double vl = 0.0, vr = 0.0;
        for (int j = 0; j < mm2; ++j) {
            const double c = (double)(j + 1) / (double)((j + 2) * (j + 2)), s = (j & 1) ? -1.0 : 1.0;
            vl += s * c * w2[IX(i - 1, j, mm2)];
            vr += c * w2[IX(i - 1, j, mm2)];
        }
        U[IX(i, 0, m)] = 4.0 * vl;
        U[IX(i, m - 1, m)] = 4.0 * vr;
    }
    free(F); free(FT); free(w1); free(w2);
    return 0;
}
