/*
 * jci_main.c -- the `jci` program: the reference's pjayci flow
 * (mpi_source/pjayci.c:25 -> execute_pjayci.c:30) on one GPU.
 *
 * Reads the namelists from ./jayci.in (&general, &dalginfo, optional
 * &gpuinfo) and the SIFS integrals from ./moints, builds the string space,
 * runs the Davidson solve and writes civec (plus ci.restart / hvvec when it
 * does not converge) to the current directory, like the reference.
 *
 * Usage: jci [jayci.in [moints]]
 */
#include <stdio.h>
#include <stdlib.h>

#include "jci.h"

static long long ix1(long long i, long long j)
{
        return i > j ? (i - 1) * i / 2 + j : (j - 1) * j / 2 + i;
}

int main(int argc, char **argv)
{
        const char *inp = argc > 1 ? argv[1] : "jayci.in";
        const char *mo = argc > 2 ? argv[2] : "moints";
        jci_general g;
        jci_dalginfo d;
        jci_gpuinfo u;
        jci_status st = jci_read_namelists(inp, &g, &d, &u);
        if (st) {
                fprintf(stderr, "jci: reading %s: %s\n", inp, jci_status_string(st));
                return 1;
        }
        if (g.ndocc + g.nactive > 64) {  /* execute_pjayci.c:96 */
                fprintf(stderr, "jci: CI-active orbital number must be < 64\n");
                return 1;
        }
        jci_space *s = NULL;
        st = jci_space_create(g.electrons, g.orbitals, g.nfrozen, g.ndocc, g.nactive,
                              g.nfrzvirt, g.xlevel, &s);
        if (st) {
                fprintf(stderr, "jci: building the string space: %s\n", jci_status_string(st));
                return 1;
        }
        long long sz[10];
        jci_space_sizes(s, sz);
        int norb = (int)sz[2];
        if (g.printlvl > 0) {
                printf("Determinants   = %15lld\n", sz[8]);
                printf(" Alpha strings = %15lld\n", sz[3]);
                printf(" Beta  strings = %15lld\n", sz[4]);
        }
        long long m1len = ix1(norb, norb), m2len = ix1(m1len, m1len);
        double *m1 = malloc(sizeof(double) * m1len);
        double *m2 = malloc(sizeof(double) * m2len);
        double enuc = 0.0, efc = 0.0;
        int nbft = 0;
        if (!m1 || !m2) {
                fprintf(stderr, "jci: out of memory\n");
                return 1;
        }
        st = jci_read_moints(mo, m1, m1len, m2, m2len, &nbft, &enuc, &efc);
        if (st || nbft != norb) {
                fprintf(stderr, "jci: reading %s: %s (nbft %d, CI orbitals %d)\n", mo,
                        st ? jci_status_string(st) : "orbital count mismatch", nbft, norb);
                return 1;
        }
        st = jci_set_integrals(s, m1, m2, norb, enuc, efc);
        if (st) {
                fprintf(stderr, "jci: uploading integrals: %s\n", jci_status_string(st));
                return 1;
        }
        jci_davidson_opts o;
        jci_davidson_defaults(&o);
        o.maxiter = d.maxiter;
        o.krymin = d.krymin;
        o.krymax = d.krymax;
        o.nroots = d.nroots;
        o.prediagr = d.prediagr;
        o.refdim = d.refdim;
        o.restol = d.restol;
        o.precision = u.precision == JCI_MIXED ? JCI_MIXED : JCI_FP64;
        o.switch_tol = u.switch_tol;
        o.block = u.block;
        o.printlvl = g.printlvl;
        o.write_files = 1;
        double *e = malloc(sizeof(double) * (d.nroots > 0 ? d.nroots : 1));
        jci_davidson_stats stats;
        st = jci_davidson(s, &o, e, NULL, &stats);
        if (st && st != JCI_ERR_NOCONV) {
                fprintf(stderr, "jci: davidson: %s\n", jci_status_string(st));
                return 1;
        }
        printf(" Davidson %s after %d iterations (%lld sigma vectors, %.3f s)\n",
               st ? "NOT converged" : "converged", stats.iterations, stats.sigma_vectors,
               stats.total_seconds);
        for (int k = 0; k < d.nroots; k++) printf("   Root #%2d  %18.10lf\n", k + 1, e[k]);
        jci_space_destroy(s);
        free(m1);
        free(m2);
        free(e);
        return 0;
}
