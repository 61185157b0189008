/*
 * LAPACK / Fortran stand-ins for the reference oracle build (test
 * infrastructure only).
 *
 * The reference links the system ILP64 LAPACK (Makefile:130) and calls
 * dsyevr_/dgemm_ with 64-bit integers (mathutil.c:57-98,141-162).  Here the
 * calls are forwarded to the ILP64 OpenBLAS that numpy bundles, whose
 * symbols carry the scipy_ prefix and 64_ suffix.  gfortran passes the
 * lengths of CHARACTER arguments as trailing hidden size_t arguments; the
 * reference's C callers do not, so this forwarder supplies them (each flag
 * is one character).
 *
 * dlamch_fcn_ replaces mpi_source/dlamch_fcn.f90: LAPACK dlamch('s'), the
 * safe minimum, which for IEEE binary64 is DBL_MIN.
 */
#include <float.h>
#include <stddef.h>

typedef long long i64;

extern void scipy_dsyevr_64_(const char *jobz, const char *range,
                             const char *uplo, const i64 *n, double *a,
                             const i64 *lda, const double *vl,
                             const double *vu, const i64 *il, const i64 *iu,
                             const double *abstol, i64 *m, double *w,
                             double *z, const i64 *ldz, i64 *isuppz,
                             double *work, const i64 *lwork, i64 *iwork,
                             const i64 *liwork, i64 *info, size_t l1,
                             size_t l2, size_t l3);

extern void scipy_dgemm_64_(const char *ta, const char *tb, const i64 *m,
                            const i64 *n, const i64 *k, const double *alpha,
                            const double *a, const i64 *lda, const double *b,
                            const i64 *ldb, const double *beta, double *c,
                            const i64 *ldc, size_t l1, size_t l2);

double dlamch_fcn_(void) { return DBL_MIN; }

void dsyevr_(const char *jobz, const char *range, const char *uplo,
             const i64 *n, double *a, const i64 *lda, const double *vl,
             const double *vu, const i64 *il, const i64 *iu,
             const double *abstol, i64 *m, double *w, double *z,
             const i64 *ldz, i64 *isuppz, double *work, const i64 *lwork,
             i64 *iwork, const i64 *liwork, i64 *info)
{
        scipy_dsyevr_64_(jobz, range, uplo, n, a, lda, vl, vu, il, iu, abstol,
                         m, w, z, ldz, isuppz, work, lwork, iwork, liwork,
                         info, 1, 1, 1);
}

void dgemm_(const char *ta, const char *tb, const i64 *m, const i64 *n,
            const i64 *k, const double *alpha, const double *a,
            const i64 *lda, const double *b, const i64 *ldb,
            const double *beta, double *c, const i64 *ldc)
{
        scipy_dgemm_64_(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc,
                        1, 1);
}
