/*
 * ref_harness.c -- drives the reference's own mpi_source C code (compiled
 * unchanged against the single-process GA/MPI stand-in) for the oracle.
 * Test infrastructure only: it is loaded by tests/ and by bench.py's
 * reference/CPU-baseline leg, never by the product library.
 *
 * The call sequence mirrors execute_pjayci.c:139-222 minus the namelist and
 * SIFS readers: abecalc -> compute_stringnum -> allocate_eospace_array ->
 * citrunc, then either a single sigma application (the body of
 * perform_hvispacefast, pdavidson.c:4328-4414) or a full pdavidson
 * (pdavidson.c:39).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>
#include "mpi_utilities.h"
#include "allocate_mem.h"
#include "abecalc.h"
#include "binarystr.h"
#include "citruncate.h"
#include "combinatorial.h"
#include "moindex.h"
#include "pdavidson.h"
#include "action_util.h"
#include "ga.h"

extern double nuc_rep_e;
extern double total_core_e;
const int mpi_root = 0;

double *shim_ga_data(int g_a);
void shim_ga_reset(void);

static struct {
        int built;
        int aelec, belec, ci_aelec, ci_belec, ci_orbs;
        int ndocc, nactv, xlvl, intorb;
        int pstr_len, qstr_len, pegrps, qegrps, num_pq, ndets;
        struct occstr *pstr, *qstr;
        struct eospace *peosp, *qeosp;
        int **pq;
        int *pqdata;
} S;

static void release(void)
{
        if (!S.built) return;
        free(S.pstr);
        free(S.qstr);
        free(S.peosp);
        free(S.qeosp);
        deallocate_mem_cont_int(&S.pq, S.pqdata);
        memset(&S, 0, sizeof(S));
}

/* Build the truncated alpha/beta string space (execute_pjayci.c:139-170).
 * Returns the number of determinants, or a negative error code. */
int ref_build_space(int electrons, int orbitals, int nfrzc, int ndocc,
                    int nactv, int nfrzv, int xlvl)
{
        release();
        mpi_num_procs = 1;
        mpi_proc_rank = 0;
        abecalc(electrons, &S.aelec, &S.belec);
        compute_ci_elecs_and_orbitals(S.aelec, S.belec, orbitals, nfrzc,
                                      nfrzv, &S.ci_aelec, &S.ci_belec,
                                      &S.ci_orbs);
        if (S.ci_aelec > 20 || S.ci_belec > 20 || S.ci_orbs > 200) return -1;
        S.ndocc = ndocc;
        S.nactv = nactv;
        S.xlvl = xlvl;
        S.intorb = ndocc + nactv;
        S.pstr_len = compute_stringnum(S.ci_orbs, S.ci_aelec, ndocc, nactv,
                                       xlvl);
        S.qstr_len = compute_stringnum(S.ci_orbs, S.ci_belec, ndocc, nactv,
                                       xlvl);
        S.pstr = allocate_occstr_arrays(S.pstr_len);
        S.qstr = allocate_occstr_arrays(S.qstr_len);
        S.peosp = allocate_eospace_array(S.ci_aelec, S.ci_orbs, ndocc, nactv,
                                         xlvl, &S.pegrps);
        S.qeosp = allocate_eospace_array(S.ci_belec, S.ci_orbs, ndocc, nactv,
                                         xlvl, &S.qegrps);
        S.num_pq = S.pegrps * S.qegrps;
        S.pqdata = allocate_mem_int_cont(&S.pq, 2, S.num_pq);
        int err = citrunc(S.aelec, S.belec, orbitals, nfrzc, ndocc, nactv,
                          nfrzv, xlvl, S.pstr, S.pstr_len, S.qstr, S.qstr_len,
                          S.peosp, S.pegrps, S.qeosp, S.qegrps, &S.ndets,
                          S.pq, &S.num_pq);
        S.built = 1;
        if (err) return -err;
        return S.ndets;
}

/* Sizes: [ci_aelec, ci_belec, ci_orbs, pstr_len, qstr_len, pegrps, qegrps,
 * num_pq, ndets, intorb]. */
void ref_sizes(int *out)
{
        out[0] = S.ci_aelec; out[1] = S.ci_belec; out[2] = S.ci_orbs;
        out[3] = S.pstr_len; out[4] = S.qstr_len; out[5] = S.pegrps;
        out[6] = S.qegrps; out[7] = S.num_pq; out[8] = S.ndets;
        out[9] = S.intorb;
}

/* Orbital lists (1-based, as istr[]), byte1, virtx[2] and nvrtx for every
 * string of one spin (0 = alpha/p, 1 = beta/q). */
void ref_get_strings(int spin, int *istr, long long *byte1, int *virtx,
                     int *nvrtx)
{
        struct occstr *s = spin ? S.qstr : S.pstr;
        int n = spin ? S.qstr_len : S.pstr_len;
        int ne = spin ? S.ci_belec : S.ci_aelec;
        for (int i = 0; i < n; i++) {
                for (int e = 0; e < ne; e++) istr[i * ne + e] = s[i].istr[e];
                byte1[i] = s[i].byte1;
                virtx[2 * i] = s[i].virtx[0];
                virtx[2 * i + 1] = s[i].virtx[1];
                nvrtx[i] = s[i].nvrtx;
        }
}

/* Electron-occupation groups: per group [docc, actv, virt, nstr, start,
 * npairs, pairs[0..19]] (26 ints). */
void ref_get_eospaces(int spin, int *out)
{
        struct eospace *e = spin ? S.qeosp : S.peosp;
        int n = spin ? S.qegrps : S.pegrps;
        for (int g = 0; g < n; g++) {
                int *o = out + 26 * g;
                o[0] = e[g].docc; o[1] = e[g].actv; o[2] = e[g].virt;
                o[3] = e[g].nstr; o[4] = e[g].start; o[5] = e[g].npairs;
                for (int k = 0; k < 20; k++) o[6 + k] = e[g].pairs[k];
        }
}

void ref_get_pq(int *out)
{
        for (int i = 0; i < S.num_pq; i++) {
                out[2 * i] = S.pq[i][0];
                out[2 * i + 1] = S.pq[i][1];
        }
}

/* yij/cij tables for every string: out[(s*ne + e)*(norb+1) + o] for
 * orbital o = 1..norb (index 0 unused, set to 0). */
void ref_get_yij_cij(int spin, int *yij, int *cij)
{
        struct occstr *s = spin ? S.qstr : S.pstr;
        int n = spin ? S.qstr_len : S.pstr_len;
        int ne = spin ? S.ci_belec : S.ci_aelec;
        int w = S.ci_orbs + 1;
        for (int i = 0; i < n; i++)
                for (int e = 0; e < ne; e++)
                        for (int o = 0; o < w; o++) {
                                yij[(i * ne + e) * w + o] = o ? s[i].yij[e][o] : 0;
                                cij[(i * ne + e) * w + o] = o ? s[i].cij[e][o] : 0;
                        }
}

/* Excitation list of string istr into group teosp (generate_single/
 * double_excitations, citruncate.c:755,799).  Each entry is
 * [index, io0, io1, fo0, fo1, permx]; returns the count. */
int ref_excitations(int spin, int nrep, int istr, int teosp, int *out)
{
        struct occstr *s = spin ? S.qstr : S.pstr;
        struct eospace *e = spin ? S.qeosp : S.peosp;
        int n = spin ? S.qstr_len : S.pstr_len;
        int ne = spin ? S.ci_belec : S.ci_aelec;
        int vorbs = S.ci_orbs - S.intorb;
        struct xstr *xl = malloc(sizeof(struct xstr) * (n + 1));
        int *elecx = malloc(sizeof(int) * (ne + 1));
        int *orbsx = malloc(sizeof(int) * (S.ci_orbs + 1));
        int nx;
        if (nrep == 1)
                nx = generate_single_excitations(&s[istr], e[teosp], ne,
                                                 S.ndocc, S.nactv, S.intorb,
                                                 vorbs, xl, elecx, orbsx, s);
        else
                nx = generate_double_excitations(&s[istr], e[teosp], ne,
                                                 S.ndocc, S.nactv, S.intorb,
                                                 vorbs, xl, elecx, orbsx, s);
        for (int k = 0; k < nx; k++) {
                int *o = out + 6 * k;
                o[0] = xl[k].index; o[1] = xl[k].io[0]; o[2] = xl[k].io[1];
                o[3] = xl[k].fo[0]; o[4] = xl[k].fo[1]; o[5] = xl[k].permx;
        }
        free(xl);
        free(elecx);
        free(orbsx);
        return nx;
}

/* Determinant triples (p, q, cas) as generate_wlist writes them. */
static int make_wlist(void)
{
        int dims[2] = {S.ndets, 3};
        int chunk[2] = {-1, 3};
        int w = NGA_Create(C_INT, 2, dims, "W", chunk);
        generate_wlist(w, S.ndets, S.pq, S.num_pq, S.peosp, S.pegrps,
                       S.qeosp, S.qegrps);
        return w;
}

void ref_get_wlist(int *out)
{
        int w = make_wlist();
        int lo[2] = {0, 0}, hi[2] = {S.ndets - 1, 2}, ld[1] = {3};
        NGA_Get(w, lo, hi, out, ld);
        shim_ga_reset();
}

/* Diagonal <i|H|i> (compute_diagonal_iHi, pdavidson.c:1586). */
void ref_hdiag(double *m1, double *m2, double *out)
{
        int w = make_wlist();
        compute_diagonal_iHi(out, 0, S.ndets - 1, m1, m2, S.ci_aelec,
                             S.ci_belec, S.intorb, w, S.pstr, S.qstr);
        shim_ga_reset();
}

/* One sigma application C = H V for nvec vectors stored vector-major
 * (V[k*ndets + i]), following perform_hvispacefast (pdavidson.c:4328):
 * diagonal term via GA_Elem_multiply_patch, then compute_cblock_Hfastest
 * over the upper triangle with symmetric accumulation. */
void ref_sigma(double *m1, double *m2, int nvec, const double *V, double *C)
{
        int vd[2] = {nvec, S.ndets}, vc[2] = {nvec, -1};
        int v = NGA_Create(C_DBL, 2, vd, "V", vc);
        int c = NGA_Duplicate(v, "C");
        int nd[1] = {S.ndets}, nc[1] = {-1};
        int d = NGA_Create(C_DBL, 1, nd, "D", nc);
        int w = make_wlist();
        compute_diagonal_iHi(shim_ga_data(d), 0, S.ndets - 1, m1, m2,
                             S.ci_aelec, S.ci_belec, S.intorb, w, S.pstr,
                             S.qstr);
        memcpy(shim_ga_data(v), V, sizeof(double) * nvec * S.ndets);
        perform_hvispacefast(S.pstr, S.peosp, S.pegrps, S.qstr, S.qeosp,
                             S.qegrps, S.pq, S.num_pq, m1, m2, S.ci_aelec,
                             S.ci_belec, S.intorb, S.ndets, 0.0, nvec, nvec,
                             v, d, c, w, 0, S.ci_orbs, S.ndocc, S.nactv);
        memcpy(C, shim_ga_data(c), sizeof(double) * nvec * S.ndets);
        shim_ga_reset();
}

/* Bounded samples of the reference's sigma for CPU timing: ref_sigma_prepare
 * sets up V, C, D (<i|H|i>, compute_diagonal_iHi) and W once;
 * ref_sigma_rows_timed runs the reference's
 * row-range kernel compute_cblock_Hfastest (pdavidson.c:1296) for rows
 * [row0, row0 + nrows) of the upper triangle and returns its wall time in
 * seconds (setup excluded).  The partial C it accumulates is not a sigma. */
#include <time.h>
static int T_v, T_c, T_d, T_w, T_nvec;
static double *T_m1, *T_m2;

int ref_sigma_prepare(double *m1, double *m2, int nvec, const double *V)
{
        shim_ga_reset();
        int vd[2] = {nvec, S.ndets}, vc[2] = {nvec, -1};
        T_v = NGA_Create(C_DBL, 2, vd, "V", vc);
        T_c = NGA_Duplicate(T_v, "C");
        int nd[1] = {S.ndets}, nc[1] = {-1};
        T_d = NGA_Create(C_DBL, 1, nd, "D", nc);
        T_w = make_wlist();
        T_nvec = nvec;
        T_m1 = m1;
        T_m2 = m2;
        compute_diagonal_iHi(shim_ga_data(T_d), 0, S.ndets - 1, m1, m2,
                             S.ci_aelec, S.ci_belec, S.intorb, T_w, S.pstr,
                             S.qstr);
        memcpy(shim_ga_data(T_v), V, sizeof(double) * nvec * S.ndets);
        return 0;
}

double ref_sigma_rows_timed(int row0, int nrows)
{
        int ccols = T_nvec, crows = nrows;
        double *cdata = calloc((size_t)ccols * crows, sizeof(double));
        int **wi = NULL;
        int *widata = allocate_mem_int_cont(&wi, 3, crows);
        int lo[2] = {row0, 0}, hi[2] = {row0 + nrows - 1, 2}, ld[1] = {3};
        NGA_Get(T_w, lo, hi, widata, ld);
        int *cindx = malloc(sizeof(int) * ccols);
        for (int i = 0; i < ccols; i++) cindx[i] = i;
        struct timespec a, b;
        clock_gettime(CLOCK_MONOTONIC, &a);
        compute_cblock_Hfastest(cdata, ccols, crows, wi, T_w, T_v, T_d, 0, S.pstr,
                                S.peosp, S.pegrps, S.qstr, S.qeosp, S.qegrps, S.pq,
                                S.num_pq, T_m1, T_m2, S.ci_aelec, S.ci_belec,
                                S.intorb, S.ndets, S.ci_orbs, S.ndocc, S.nactv,
                                T_c, row0, row0 + nrows - 1, cindx);
        clock_gettime(CLOCK_MONOTONIC, &b);
        free(cindx);
        free(cdata);
        deallocate_mem_cont_int(&wi, widata);
        return (b.tv_sec - a.tv_sec) + 1e-9 * (b.tv_nsec - a.tv_nsec);
}

/* One timed step of the reference's sigma on rows [row0, row0 + nrows) of
 * every vector: the diagonal term sigma = D o v that perform_hvispacefast
 * applies first (compute_hvc_diagonal_ga, pdavidson.c:2105, whose
 * GA_Elem_multiply_patch is restricted here to the same rows), then
 * compute_cblock_Hfastest on those rows (pdavidson.c:1296).  Returns the
 * wall time of both in seconds; *diag_s receives the diagonal part. */
double ref_sigma_step_timed(int row0, int nrows, double *diag_s)
{
        struct timespec a, b;
        clock_gettime(CLOCK_MONOTONIC, &a);
        for (int k = 0; k < T_nvec; k++) {
                int d_lo[1] = {row0}, d_hi[1] = {row0 + nrows - 1};
                int p_lo[2] = {k, row0}, p_hi[2] = {k, row0 + nrows - 1};
                GA_Elem_multiply_patch(T_d, d_lo, d_hi, T_v, p_lo, p_hi, T_c, p_lo,
                                       p_hi);
        }
        clock_gettime(CLOCK_MONOTONIC, &b);
        double t_diag = (b.tv_sec - a.tv_sec) + 1e-9 * (b.tv_nsec - a.tv_nsec);
        if (diag_s) *diag_s = t_diag;
        return t_diag + ref_sigma_rows_timed(row0, nrows);
}

void ref_sigma_release(void) { shim_ga_reset(); }

/* OpenMP threads of the reference's parallel regions.  The OMP_NUM_THREADS
 * variable is read once, when the OpenMP runtime starts, which in a process
 * that already loaded it (a Python process with torch) is before this
 * library is loaded; this sets the count directly. */
#include <omp.h>
void ref_set_threads(int n)
{
        if (n > 0) omp_set_num_threads(n);
}

int ref_get_threads(void) { return omp_get_max_threads(); }

/* Full reference Davidson solve (pdavidson, pdavidson.c:39) run in
 * directory `workdir` (it writes civec / ci.restart / hvvec there).  On
 * return civec_out holds the nroots result vectors (vector-major) read back
 * from the first rows of the basis-vector array, exactly what pdavidson
 * writes to "civec" (pdavidson.c:343). */
int ref_pdavidson(double *m1, double *m2, double nucrep, double frzcore,
                  int printlvl, int maxiter, int krymin, int krymax,
                  int nroots, int prediagr, int refdim, double restol,
                  const char *workdir, double *civec_out)
{
        char cwd[4096];
        if (!getcwd(cwd, sizeof(cwd))) return -100;
        if (workdir && chdir(workdir) != 0) return -101;
        nuc_rep_e = nucrep;
        total_core_e = nucrep + frzcore;
        int err = pdavidson(S.pstr, S.peosp, S.pegrps, S.qstr, S.qeosp,
                            S.qegrps, S.pq, S.num_pq, m1, m2, S.ci_aelec,
                            S.ci_belec, S.intorb, S.ndets, nucrep, frzcore,
                            printlvl, maxiter, krymin, krymax, nroots,
                            prediagr, refdim, restol, 0, S.ci_orbs, S.ndocc,
                            S.nactv);
        fflush(stdout);
        /* The basis-vector array is the first one pdavidson creates. */
        if (civec_out)
                memcpy(civec_out, shim_ga_data(1),
                       sizeof(double) * nroots * S.ndets);
        shim_ga_reset();
        if (chdir(cwd) != 0) return -102;
        return err;
}
