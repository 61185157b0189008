/*
 * ref_serial.c -- drives the reference's serial program path (jayci:
 * source/run_jayci.c:23 -> execute_ci_calculation_inpdlist,
 * source/execute_ci_calculation.c:154), compiled unchanged from source/,
 * for the cross-check of the pjayci path and for CPU timing.
 * Test infrastructure only: loaded by tests/ and make_golden.py, never by
 * the product library.
 *
 * The call sequence is the reference's: abecalc -> citrunc_rtnlist
 * (source/citruncate.c:123) -> generate_cimap (source/cimapping.c:92, the
 * O(N^2) pair map) -> compute_hdgls (source/action_util.c:106) -> dvdalg
 * (source/davidson.c:91, sigma by compute_hv, source/action_util.c:121).
 * The &dalginfo values, integrals and core energies are passed in memory
 * instead of being read from jayci.in / moints.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "abecalc.h"
#include "action_util.h"
#include "allocate_mem.h"
#include "binarystr.h"
#include "cimapping.h"
#include "citruncate.h"
#include "davidson.h"

/* The Fortran namelist, SIFS and MO-coefficient readers (readnamelist.f90,
 * readmoints.f90, readmocoef.f90) are not compiled: there is no Fortran
 * compiler here.  Only ioutil.c routines this harness never calls refer to
 * them; these definitions satisfy the linker and report misuse. */
void readnamelist_(void) { fprintf(stderr, "ref_serial: namelist reader not built\n"); }
void readmoints_(void) { fprintf(stderr, "ref_serial: SIFS reader not built\n"); }
void readmocoef_(void) { fprintf(stderr, "ref_serial: MO reader not built\n"); }

static double now(void)
{
        struct timespec t;
        clock_gettime(CLOCK_MONOTONIC, &t);
        return t.tv_sec + 1e-9 * t.tv_nsec;
}

/* Full serial solve.  energies[nroots] are the reference's cival (total
 * energies, nucrep + frzcore included); civec_out (nullable) receives
 * nroots x ndets; times[3] = {cimap, hdgls, dvdalg} wall seconds.  Returns
 * ndets (> 0) or a negative error code. */
long long ref_serial_solve(int electrons, int orbitals, int nfrzc, int ndocc,
                           int nactv, int nfrzv, int xlvl, double *m1,
                           double *m2, double nucrep, double frzcore,
                           int maxiter, int krymin, int krymax, int nroots,
                           int prediagr, int refdim, double restol, int plvl,
                           double *energies, double *civec_out, double *times)
{
        int aelec = 0, belec = 0, astr = 0, bstr = 0, ndets = 0;
        int ci_orbs = 0, ci_aelec = 0, ci_belec = 0;
        abecalc(electrons, &aelec, &belec);
        struct det *dl = citrunc_rtnlist(aelec, belec, orbitals, nfrzc, ndocc,
                                         nactv, nfrzv, xlvl, &astr, &bstr,
                                         &ndets, &ci_orbs, &ci_aelec,
                                         &ci_belec);
        if (!dl || ndets < 1) return -1;
        int ninto = ndocc + nactv;
        double totfrze = nucrep + frzcore;
        double t0 = now();
        struct rowmap *hmap = malloc(sizeof(struct rowmap) * ndets);
        int err = generate_cimap(dl, ndets, ninto, hmap);
        double t1 = now();
        if (err) {
                free(dl);
                return -2;
        }
        double *hd = malloc(sizeof(double) * ndets);
        compute_hdgls(dl, ndets, m1, m2, ci_aelec, ci_belec, hd, ninto);
        double t2 = now();
        double **civec = NULL;
        if (allocate_mem_double(&civec, ndets, nroots) != 0) return -3;
        double *cival = malloc(sizeof(double) * nroots);
        err = dvdalg(dl, ndets, m1, m2, ci_aelec, ci_belec, hd, ninto,
                     totfrze, maxiter, krymin, krymax, nroots, restol, hmap,
                     civec, cival, prediagr, plvl, ci_orbs, refdim);
        double t3 = now();
        for (int i = 0; i < nroots; i++) {
                energies[i] = cival[i];
                if (civec_out)
                        memcpy(civec_out + (size_t)i * ndets, civec[i],
                               sizeof(double) * ndets);
        }
        if (times) {
                times[0] = t1 - t0;
                times[1] = t2 - t1;
                times[2] = t3 - t2;
        }
        free(cival);
        deallocate_mem(&civec, ndets, nroots);
        free(hd);
        deallocate_cimap(hmap, ndets);
        free(dl);
        return err ? -100 - err : ndets;
}

/* The serial path's own sigma: c = H v by compute_hv over the cimap
 * (source/action_util.c:121), the diagonal included, for nvec vectors
 * (vector-major, in the serial determinant order of citrunc_rtnlist).
 * hdiag_out (nullable) receives compute_hdgls; dets_out (nullable)
 * receives each determinant's alpha and beta occupation masks (byte1).
 * Returns ndets or a negative error code. */
long long ref_serial_sigma(int electrons, int orbitals, int nfrzc, int ndocc,
                           int nactv, int nfrzv, int xlvl, double *m1,
                           double *m2, int nvec, const double *v, double *c,
                           double *hdiag_out, long long *dets_out)
{
        int aelec = 0, belec = 0, astr = 0, bstr = 0, ndets = 0;
        int ci_orbs = 0, ci_aelec = 0, ci_belec = 0;
        abecalc(electrons, &aelec, &belec);
        struct det *dl = citrunc_rtnlist(aelec, belec, orbitals, nfrzc, ndocc,
                                         nactv, nfrzv, xlvl, &astr, &bstr,
                                         &ndets, &ci_orbs, &ci_aelec,
                                         &ci_belec);
        if (!dl || ndets < 1) return -1;
        int ninto = ndocc + nactv;
        struct rowmap *hmap = malloc(sizeof(struct rowmap) * ndets);
        if (generate_cimap(dl, ndets, ninto, hmap)) return -2;
        double *vi = malloc(sizeof(double) * ndets);
        double *ci = malloc(sizeof(double) * ndets);
        for (int k = 0; k < nvec; k++) {
                memcpy(vi, v + (size_t)k * ndets, sizeof(double) * ndets);
                memset(ci, 0, sizeof(double) * ndets);
                compute_hv(dl, ndets, m1, m2, ci_aelec, ci_belec, vi, ci, ninto,
                           hmap);
                memcpy(c + (size_t)k * ndets, ci, sizeof(double) * ndets);
        }
        if (hdiag_out)
                compute_hdgls(dl, ndets, m1, m2, ci_aelec, ci_belec, hdiag_out,
                              ninto);
        if (dets_out)
                for (int i = 0; i < ndets; i++) {
                        dets_out[2 * i] = dl[i].astr.byte1;
                        dets_out[2 * i + 1] = dl[i].bstr.byte1;
                }
        free(vi);
        free(ci);
        deallocate_cimap(hmap, ndets);
        free(dl);
        return ndets;
}
