/*
 * jci_oracle.h -- CPU restatement of the reference's determinant-CI hot path
 * (string space, excitations, Slater-rule matrix elements, sigma, Davidson).
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the parity tests, smoke()
 * and bench.py's CPU-baseline leg compare the CUDA path against; the product
 * library never links or calls it.  Each function cites the reference
 * routine (path within the reference project, file:line) it restates.
 *
 * Strings are sorted 1-based orbital lists; determinants are ordered by
 * (p,q)-group pair, then alpha string, then beta string, as in the
 * reference.  Integrals use the reference's packed layout (moindex.c).
 */
#ifndef JCI_ORACLE_H
#define JCI_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct jo_space jo_space;

/* Build the truncated string space (citruncate.c:55 citrunc). */
jo_space *jo_space_build(int ci_aelec, int ci_belec, int ci_orbs, int ndocc,
                         int nactv, int xlvl);
void jo_space_free(jo_space *s);

/* [nastr, nbstr, pegrps, qegrps, num_pq, ndets] */
void jo_space_info(const jo_space *s, long long *out);
/* Sorted orbital lists, nstr x nelec. */
void jo_strings(const jo_space *s, int spin, int *istr);
/* Per group: [docc, actv, virt, nstr, start]. */
void jo_eospaces(const jo_space *s, int spin, int *out);
/* Valid group pairs [p, q] in determinant order. */
void jo_pq(const jo_space *s, int *out);
/* Index of the string with the given sorted orbital list, or -1. */
int jo_string_index(const jo_space *s, int spin, const int *orbs);

/* Every single (nrep=1) or double (nrep=2) replacement of string istr that
 * lands in group teosp; entries [index, io0, io1, fo0, fo1, permx]. */
int jo_excitations(const jo_space *s, int spin, int nrep, int istr,
                   int teosp, int *out);

/* <i|H|i> for every determinant (action_util.c:167 hmatels_0x). */
void jo_hdiag(const jo_space *s, const double *m1, const double *m2,
              double *out);
/* <i|H|j> for two determinants by index (action_util.c:119 hmatels). */
double jo_hmatel(const jo_space *s, const double *m1, const double *m2,
                 long long i, long long j);
/* S = H V for nvec vectors stored vector-major (full-row gather). */
void jo_sigma(const jo_space *s, const double *m1, const double *m2,
              int nvec, const double *V, double *S);
/* Rows d0 <= d < d1 of the same (S holds all ndets per vector). */
void jo_sigma_range(const jo_space *s, const double *m1, const double *m2,
                    int nvec, const double *V, double *S, long long d0,
                    long long d1);

/* Sigma of one vector V (ndets) at the determinants rows[0..nrows) only:
 * out[r] = (H V)[rows[r]] (out-of-range rows give 0). */
void jo_sigma_rows(const jo_space *s, const double *m1, const double *m2,
                   const double *V, const long long *rows, long long nrows,
                   double *out);

/* Root-sequential Davidson (pdavidson.c:39).  Returns iterations taken
 * (>= 0) or a negative error.  energies[nroots] include totcore; civec is
 * nroots x ndets.  init (prediagr=3) supplies krymin start vectors. */
int jo_davidson(const jo_space *s, const double *m1, const double *m2,
                double totcore, int maxiter, int krymin, int krymax,
                int nroots, int prediagr, int refdim, double restol,
                const double *init, double *energies, double *civec);

/* Dyson orbitals between an (N+1)-electron space s0 and an N-electron
 * space s1 (run_pdycicalc.c:392-414, dysoncomp.c:103-345): for every
 * determinant of s0 and every electron of the spin whose count differs
 * (beta when nelec0 is even, else alpha), remove it; when the resulting
 * string and determinant exist in s1,
 *   dyorb[(j*nst1 + k)*norbs0 + orbital-1] += v0[state0_j][I] v1[state1_k][J]
 * with the other spin's string unchanged and no phase factor, then scale
 * by sqrt(nelec0).  states are 1-based; v0 / v1 are state-major. */
void jo_dyson(const jo_space *s0, const jo_space *s1, int nelec0, int norbs0,
              const double *v0, const double *v1, int nst0, const int *states0,
              int nst1, const int *states1, double *dyorb);

/* Cyclic Jacobi eigensolver: a (n x n, row-major, symmetric, destroyed);
 * eigenvalues ascending in w, eigenvector k in row k of z. */
void jo_symeig(int n, double *a, double *w, double *z);

#ifdef __cplusplus
}
#endif
#endif
