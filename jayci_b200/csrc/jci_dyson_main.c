/*
 * jci_dyson_main.c -- the Dyson-orbital program on one GPU, the flow of the
 * reference's pdycicalc (mpi_source/pdycicalc.c, run_pdycicalc.c:26-456)
 * without MPI / Global Arrays:
 *
 *   dycicalc.in  &wavefcn0 (N+1 electrons), &wavefcn1 (N electrons),
 *                &dysonorbital states0 / states1
 *   anion.ci     CI vectors of wavefunction 0 (unformatted, as civec)
 *   neutral.ci   CI vectors of wavefunction 1
 *   -> dysonorb.dat
 *
 * Usage: jci_dyson [directory]   (default: the current directory)
 */
#include <stdio.h>
#include <stdlib.h>
#include <unistd.h>

#include "jci.h"

static int fail(const char *what, int st)
{
        fprintf(stderr, "jci_dyson: %s: %s\n", what, jci_status_string(st));
        return st;
}

int main(int argc, char **argv)
{
        if (argc > 1 && chdir(argv[1]) != 0) {
                fprintf(stderr, "jci_dyson: cannot enter %s\n", argv[1]);
                return 1;
        }
        jci_wavefcn w0, w1;
        int st0[5], st1[5], nst0 = 0, nst1 = 0;
        int st = jci_read_dycicalc("dycicalc.in", &w0, &w1, st0, &nst0, st1, &nst1);
        if (st) return fail("dycicalc.in", st);
        printf("Wavefunction 0: %d electrons, %d orbitals, %d states\n",
               w0.electrons, w0.orbitals, w0.nstates);
        printf("Wavefunction 1: %d electrons, %d orbitals, %d states\n",
               w1.electrons, w1.orbitals, w1.nstates);
        jci_space *s0 = NULL, *s1 = NULL;
        if ((st = jci_space_create(w0.electrons, w0.orbitals, w0.nfrozen, w0.ndocc,
                                   w0.nactive, w0.nfrzvirt, w0.xlevel, &s0)))
                return fail("wavefunction 0", st);
        if ((st = jci_space_create(w1.electrons, w1.orbitals, w1.nfrozen, w1.ndocc,
                                   w1.nactive, w1.nfrzvirt, w1.xlevel, &s1)))
                return fail("wavefunction 1", st);
        long long z0[10], z1[10];
        jci_space_sizes(s0, z0);
        jci_space_sizes(s1, z1);
        printf(" Determinants  %lld / %lld\n", z0[8], z1[8]);
        double *v0 = malloc(sizeof(double) * (size_t)w0.nstates * z0[8]);
        double *v1 = malloc(sizeof(double) * (size_t)w1.nstates * z1[8]);
        int ndy = nst0 * nst1;
        double *dy = malloc(sizeof(double) * (size_t)(ndy > 0 ? ndy : 1) * w0.orbitals);
        if (!v0 || !v1 || !dy) return fail("memory", JCI_ERR_NOMEM);
        if ((st = jci_read_vectors("anion.ci", w0.nstates, (int)z0[8], v0)))
                return fail("anion.ci", st);
        if ((st = jci_read_vectors("neutral.ci", w1.nstates, (int)z1[8], v1)))
                return fail("neutral.ci", st);
        printf("Computing %d Dyson orbital(s)\n", ndy);
        if ((st = jci_dyson(s0, s1, v0, w0.nstates, v1, w1.nstates, st0, nst0, st1, nst1,
                            dy)))
                return fail("dyson", st);
        if ((st = jci_write_dysonorb("dysonorb.dat", ndy, w0.orbitals, dy, st0, nst0, st1,
                                     nst1)))
                return fail("dysonorb.dat", st);
        printf("Wrote dysonorb.dat\n");
        free(v0);
        free(v1);
        free(dy);
        jci_space_destroy(s0);
        jci_space_destroy(s1);
        return 0;
}
