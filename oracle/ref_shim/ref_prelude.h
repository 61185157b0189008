/*
 * Force-included (gcc -include) when the reference's mpi_source/*.c files
 * are compiled for the oracle.  mathutil.c calls dlamch_fcn_() without a
 * prototype (mathutil.c:24,88); declaring it here keeps the double return
 * value intact.  The LAPACK entry points are left unprototyped so the
 * reference's own argument types pass through unchanged.
 */
#ifndef ORACLE_REF_PRELUDE_H
#define ORACLE_REF_PRELUDE_H
double dlamch_fcn_(void);
void dsyevr_();
void dgemm_();
#endif
