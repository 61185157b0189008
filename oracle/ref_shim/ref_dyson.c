/*
 * ref_dyson.c -- drives the reference's own Dyson-orbital code
 * (mpi_source/dysoncomp.c, compiled unchanged against the single-process
 * GA/MPI stand-in) for the oracle.  Test infrastructure only.
 *
 * The call sequence mirrors run_pdycicalc.c:206-420 minus the namelist and
 * vector-file readers: both wavefunctions are built with citrunc, their
 * W lists with generate_wlist, the (N+1) -> N string removal lists with
 * generate_strcontlist on the beta strings (N+1 electrons even) or the
 * alpha strings (odd), then compute_dyson_orbital_b / _a accumulates and
 * the result is scaled by sqrt(N+1) (run_pdycicalc.c:409-414).
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "mpi_utilities.h"
#include "allocate_mem.h"
#include "abecalc.h"
#include "binarystr.h"
#include "citruncate.h"
#include "pdavidson.h"
#include "dysoncomp.h"
#include "ga.h"

void shim_ga_reset(void);

struct wf {
        int aelec, belec, ci_aelec, ci_belec, ci_orbs;
        int pstr_len, qstr_len, pegrps, qegrps, num_pq, ndets;
        struct occstr *pstr, *qstr;
        struct eospace *peosp, *qeosp;
        int **pq;
        int *pqdata;
};

static int build_wf(struct wf *w, int electrons, int orbitals, int nfrzc,
                    int ndocc, int nactv, int nfrzv, int xlvl)
{
        memset(w, 0, sizeof(*w));
        abecalc(electrons, &w->aelec, &w->belec);
        compute_ci_elecs_and_orbitals(w->aelec, w->belec, orbitals, nfrzc,
                                      nfrzv, &w->ci_aelec, &w->ci_belec,
                                      &w->ci_orbs);
        w->pstr_len = compute_stringnum(w->ci_orbs, w->ci_aelec, ndocc, nactv,
                                        xlvl);
        w->qstr_len = compute_stringnum(w->ci_orbs, w->ci_belec, ndocc, nactv,
                                        xlvl);
        w->pstr = allocate_occstr_arrays(w->pstr_len);
        w->qstr = allocate_occstr_arrays(w->qstr_len);
        w->peosp = allocate_eospace_array(w->ci_aelec, w->ci_orbs, ndocc,
                                          nactv, xlvl, &w->pegrps);
        w->qeosp = allocate_eospace_array(w->ci_belec, w->ci_orbs, ndocc,
                                          nactv, xlvl, &w->qegrps);
        w->num_pq = w->pegrps * w->qegrps;
        w->pqdata = allocate_mem_int_cont(&w->pq, 2, w->num_pq);
        return citrunc(w->aelec, w->belec, orbitals, nfrzc, ndocc, nactv,
                       nfrzv, xlvl, w->pstr, w->pstr_len, w->qstr,
                       w->qstr_len, w->peosp, w->pegrps, w->qeosp, w->qegrps,
                       &w->ndets, w->pq, &w->num_pq);
}

static void free_wf(struct wf *w)
{
        free(w->pstr);
        free(w->qstr);
        free(w->peosp);
        free(w->qeosp);
        deallocate_mem_cont_int(&w->pq, w->pqdata);
}

/*
 * g0 / g1 = {electrons, orbitals, nfrozen, ndocc, nactive, nfrzvirt,
 * xlevel} of the (N+1) and N wavefunctions; v0 (nstates0 x ndets0) and v1
 * (nstates1 x ndets1) their CI vectors; states0 / states1 the 1-based
 * states of the &dysonorbital namelist.  dyorb receives
 * (nst0 * nst1) x orbitals values.  Returns 0 or a negative error.
 */
int ref_dyson(const int *g0, const int *g1, int nstates0, const double *v0,
              int nstates1, const double *v1, int nst0, const int *states0,
              int nst1, const int *states1, double *dyorb)
{
        struct wf w0, w1;
        int dys0[5], dys1[5];
        mpi_num_procs = 1;
        mpi_proc_rank = 0;
        if (nst0 < 1 || nst0 > 5 || nst1 < 1 || nst1 > 5) return -1;
        if (build_wf(&w0, g0[0], g0[1], g0[2], g0[3], g0[4], g0[5], g0[6]))
                return -2;
        if (build_wf(&w1, g1[0], g1[1], g1[2], g1[3], g1[4], g1[5], g1[6]))
                return -3;
        for (int i = 0; i < nst0; i++) dys0[i] = states0[i] - 1;
        for (int i = 0; i < nst1; i++) dys1[i] = states1[i] - 1;
        int norbs0 = g0[1], ndocc0 = g0[3], nactv0 = g0[4];
        int nvirt0 = norbs0 - g0[2] - g0[5] - ndocc0 - nactv0;

        int wd0[2] = {w0.ndets, 3}, wc[2] = {-1, 3};
        int wd1[2] = {w1.ndets, 3};
        int h_w0 = NGA_Create(C_INT, 2, wd0, "W0", wc);
        int h_w1 = NGA_Create(C_INT, 2, wd1, "W1", wc);
        int vd0[2] = {nstates0, w0.ndets}, vc0[2] = {nstates0, -1};
        int vd1[2] = {nstates1, w1.ndets}, vc1[2] = {nstates1, -1};
        int h_v0 = NGA_Create(C_DBL, 2, vd0, "V0", vc0);
        int h_v1 = NGA_Create(C_DBL, 2, vd1, "V1", vc1);
        int lo[2] = {0, 0}, hi[2], ld[1];
        hi[0] = nstates0 - 1; hi[1] = w0.ndets - 1; ld[0] = w0.ndets;
        NGA_Put(h_v0, lo, hi, (void *)v0, ld);
        hi[0] = nstates1 - 1; hi[1] = w1.ndets - 1; ld[0] = w1.ndets;
        NGA_Put(h_v1, lo, hi, (void *)v1, ld);
        generate_wlist(h_w0, w0.ndets, w0.pq, w0.num_pq, w0.peosp, w0.pegrps,
                       w0.qeosp, w0.qegrps);
        generate_wlist(h_w1, w1.ndets, w1.pq, w1.num_pq, w1.peosp, w1.pegrps,
                       w1.qeosp, w1.qegrps);

        int ndyorbs = nst0 * nst1;
        double **dy = NULL;
        double *dydata = allocate_mem_double_cont(&dy, norbs0, ndyorbs);
        memset(dydata, 0, sizeof(double) * norbs0 * ndyorbs);
        int **strcont = NULL, **orbcont = NULL;
        int *sc1d, *oc1d;
        if (g0[0] % 2 == 0) {
                sc1d = allocate_mem_int_cont(&strcont, w0.ci_belec + 1,
                                             w0.qstr_len);
                oc1d = allocate_mem_int_cont(&orbcont, w0.ci_belec + 1,
                                             w0.qstr_len);
                generate_strcontlist(w0.qstr, w0.qstr_len, w0.qeosp,
                                     w0.qegrps, ndocc0, nactv0, nvirt0,
                                     strcont, orbcont, w1.ci_belec, w1.qeosp,
                                     w1.qegrps);
                compute_dyson_orbital_b(h_v0, h_v1, h_w0, h_w1, w0.pstr,
                                        w0.peosp, w0.pegrps, w0.qstr,
                                        w0.qeosp, w0.qegrps, w1.pstr,
                                        w1.peosp, w1.pegrps, w1.qstr,
                                        w1.qeosp, w1.qegrps, w1.pq, w1.num_pq,
                                        w1.ci_orbs, g1[3], g1[4], nst0, dys0,
                                        nst1, dys1, w0.ndets, w1.ndets,
                                        strcont, orbcont, w0.ci_belec, dy);
        } else {
                sc1d = allocate_mem_int_cont(&strcont, w0.ci_aelec + 1,
                                             w0.pstr_len);
                oc1d = allocate_mem_int_cont(&orbcont, w0.ci_aelec + 1,
                                             w0.pstr_len);
                generate_strcontlist(w0.pstr, w0.pstr_len, w0.peosp,
                                     w0.pegrps, ndocc0, nactv0, nvirt0,
                                     strcont, orbcont, w1.ci_aelec, w1.peosp,
                                     w1.pegrps);
                compute_dyson_orbital_a(h_v0, h_v1, h_w0, h_w1, w0.pstr,
                                        w0.peosp, w0.pegrps, w0.qstr,
                                        w0.qeosp, w0.qegrps, w1.pstr,
                                        w1.peosp, w1.pegrps, w1.qstr,
                                        w1.qeosp, w1.qegrps, w1.pq, w1.num_pq,
                                        w1.ci_orbs, g1[3], g1[4], nst0, dys0,
                                        nst1, dys1, w0.ndets, w1.ndets,
                                        strcont, orbcont, w0.ci_aelec, dy);
        }
        double pref = sqrt((double)g0[0]);
        for (int i = 0; i < ndyorbs * norbs0; i++) dyorb[i] = pref * dydata[i];
        deallocate_mem_cont_int(&strcont, sc1d);
        deallocate_mem_cont_int(&orbcont, oc1d);
        deallocate_mem_cont(&dy, dydata);
        free_wf(&w0);
        free_wf(&w1);
        shim_ga_reset();
        return 0;
}
