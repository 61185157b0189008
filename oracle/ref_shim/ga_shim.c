/*
 * Single-process Global Arrays / MPI / MA stand-in used to run the
 * reference's own mpi_source C files on one CPU process.  This is test
 * infrastructure (the oracle's checker), never part of the product.
 *
 * Semantics follow the Global Arrays C interface as the reference uses it:
 * arrays are C row-major, patches are inclusive [lo, hi] ranges visited in
 * row-major order, buffers carry a leading dimension ld[0] for 2-D arrays.
 * GA_Sync is a no-op, NGA_Distribution gives rank 0 the whole array (the
 * single-rank case of compute_cimat_chunks, pdavidson.c:1411-1431).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "ga.h"
#include "mpi.h"
#include "macdecls.h"

#define SHIM_MAX_ARRAYS 256

struct shim_array {
        int used;
        int type;
        int ndim;
        int dims[2];
        long nelem;
        double *d;
        int *i;
};

static struct shim_array arrays[SHIM_MAX_ARRAYS];

static struct shim_array *get(int g)
{
        if (g < 1 || g > SHIM_MAX_ARRAYS || !arrays[g - 1].used) {
                fprintf(stderr, "ga_shim: bad handle %d\n", g);
                abort();
        }
        return &arrays[g - 1];
}

/* Flat offset of the element at subscript sub[] in array a. */
static long flat(struct shim_array *a, const int *sub)
{
        if (a->ndim == 1) return sub[0];
        return (long)sub[0] * a->dims[1] + sub[1];
}

/* Number of elements in the patch [lo, hi]. */
static long patch_len(struct shim_array *a, const int *lo, const int *hi)
{
        long n = hi[0] - lo[0] + 1;
        if (a->ndim == 2) n *= (hi[1] - lo[1] + 1);
        return n;
}

/* Flat offset of the k-th element (row-major order) of patch [lo, hi]. */
static long patch_off(struct shim_array *a, const int *lo, const int *hi,
                      long k)
{
        if (a->ndim == 1) return lo[0] + k;
        long w = hi[1] - lo[1] + 1;
        return (long)(lo[0] + k / w) * a->dims[1] + lo[1] + k % w;
}

void GA_Initialize(void) {}
void GA_Terminate(void) {}
void GA_Sync(void) {}
int GA_Nodeid(void) { return 0; }
int GA_Nnodes(void) { return 1; }

void GA_Error(char *msg, int code)
{
        fprintf(stderr, "GA_Error: %s (%d)\n", msg, code);
        abort();
}

int NGA_Create(int type, int ndim, int dims[], char *name, int chunk[])
{
        (void)name; (void)chunk;
        for (int g = 0; g < SHIM_MAX_ARRAYS; g++) {
                if (arrays[g].used) continue;
                struct shim_array *a = &arrays[g];
                a->used = 1;
                a->type = type;
                a->ndim = ndim;
                a->dims[0] = dims[0];
                a->dims[1] = ndim == 2 ? dims[1] : 1;
                a->nelem = (long)a->dims[0] * a->dims[1];
                a->d = NULL;
                a->i = NULL;
                if (type == C_DBL) a->d = calloc(a->nelem, sizeof(double));
                else a->i = calloc(a->nelem, sizeof(int));
                return g + 1;
        }
        return 0;
}

int NGA_Duplicate(int g_a, char *name)
{
        struct shim_array *a = get(g_a);
        int dims[2] = {a->dims[0], a->dims[1]};
        return NGA_Create(a->type, a->ndim, dims, name, NULL);
}

void NGA_Inquire(int g_a, int *type, int *ndim, int dims[])
{
        struct shim_array *a = get(g_a);
        *type = a->type;
        *ndim = a->ndim;
        dims[0] = a->dims[0];
        if (a->ndim == 2) dims[1] = a->dims[1];
}

void NGA_Distribution(int g_a, int iproc, int lo[], int hi[])
{
        struct shim_array *a = get(g_a);
        (void)iproc;
        lo[0] = 0;
        hi[0] = a->dims[0] - 1;
        if (a->ndim == 2) {
                lo[1] = 0;
                hi[1] = a->dims[1] - 1;
        }
}

/* Visit patch [lo,hi] against a local buffer with leading dimension ld. */
#define PATCH_LOOP(a, lo, hi, ld, BODY)                                     \
        do {                                                                \
                if ((a)->ndim == 1) {                                       \
                        for (long k = 0; k <= (hi)[0] - (lo)[0]; k++) {     \
                                long g = (lo)[0] + k, b = k;                \
                                BODY;                                       \
                        }                                                   \
                } else {                                                    \
                        for (long r = 0; r <= (hi)[0] - (lo)[0]; r++)       \
                        for (long c = 0; c <= (hi)[1] - (lo)[1]; c++) {     \
                                long g = ((lo)[0] + r) * (a)->dims[1]       \
                                         + (lo)[1] + c;                     \
                                long b = r * (long)(ld)[0] + c;             \
                                BODY;                                       \
                        }                                                   \
                }                                                           \
        } while (0)

void NGA_Get(int g_a, int lo[], int hi[], void *buf, int ld[])
{
        struct shim_array *a = get(g_a);
        if (a->type == C_DBL) {
                double *o = buf;
                PATCH_LOOP(a, lo, hi, ld, o[b] = a->d[g]);
        } else {
                int *o = buf;
                PATCH_LOOP(a, lo, hi, ld, o[b] = a->i[g]);
        }
}

void NGA_Put(int g_a, int lo[], int hi[], void *buf, int ld[])
{
        struct shim_array *a = get(g_a);
        if (a->type == C_DBL) {
                double *o = buf;
                PATCH_LOOP(a, lo, hi, ld, a->d[g] = o[b]);
        } else {
                int *o = buf;
                PATCH_LOOP(a, lo, hi, ld, a->i[g] = o[b]);
        }
}

void NGA_Acc(int g_a, int lo[], int hi[], void *buf, int ld[], void *alpha)
{
        struct shim_array *a = get(g_a);
        if (a->type == C_DBL) {
                double *o = buf, s = *(double *)alpha;
                PATCH_LOOP(a, lo, hi, ld, a->d[g] += s * o[b]);
        } else {
                int *o = buf, s = *(int *)alpha;
                PATCH_LOOP(a, lo, hi, ld, a->i[g] += s * o[b]);
        }
}

void NGA_Gather(int g_a, void *v, int *subs[], int n)
{
        struct shim_array *a = get(g_a);
        for (int k = 0; k < n; k++) {
                long g = flat(a, subs[k]);
                if (a->type == C_DBL) ((double *)v)[k] = a->d[g];
                else ((int *)v)[k] = a->i[g];
        }
}

void NGA_Scatter_acc(int g_a, void *v, int *subs[], int n, void *alpha)
{
        struct shim_array *a = get(g_a);
        for (int k = 0; k < n; k++) {
                long g = flat(a, subs[k]);
                if (a->type == C_DBL)
                        a->d[g] += *(double *)alpha * ((double *)v)[k];
                else
                        a->i[g] += *(int *)alpha * ((int *)v)[k];
        }
}

void NGA_Alloc_gatscat_buf(int nelems) { (void)nelems; }
void NGA_Free_gatscat_buf(void) {}

void NGA_Zero(int g_a)
{
        struct shim_array *a = get(g_a);
        if (a->type == C_DBL) memset(a->d, 0, a->nelem * sizeof(double));
        else memset(a->i, 0, a->nelem * sizeof(int));
}

void GA_Zero(int g_a) { NGA_Zero(g_a); }

void GA_Copy(int g_a, int g_b)
{
        struct shim_array *a = get(g_a), *b = get(g_b);
        if (a->nelem != b->nelem) GA_Error("GA_Copy: shape mismatch", 0);
        if (a->type == C_DBL) memcpy(b->d, a->d, a->nelem * sizeof(double));
        else memcpy(b->i, a->i, a->nelem * sizeof(int));
}

void NGA_Copy_patch(char trans, int g_a, int alo[], int ahi[], int g_b,
                    int blo[], int bhi[])
{
        struct shim_array *a = get(g_a), *b = get(g_b);
        (void)trans;
        long n = patch_len(a, alo, ahi);
        if (n != patch_len(b, blo, bhi)) GA_Error("Copy_patch: size", 0);
        for (long k = 0; k < n; k++)
                b->d[patch_off(b, blo, bhi, k)] = a->d[patch_off(a, alo, ahi, k)];
}

void GA_Scale(int g_a, void *alpha)
{
        struct shim_array *a = get(g_a);
        double s = *(double *)alpha;
        for (long k = 0; k < a->nelem; k++) a->d[k] *= s;
}

void GA_Add_constant(int g_a, void *alpha)
{
        struct shim_array *a = get(g_a);
        double s = *(double *)alpha;
        for (long k = 0; k < a->nelem; k++) a->d[k] += s;
}

void GA_Add_constant_patch(int g_a, int lo[], int hi[], void *alpha)
{
        struct shim_array *a = get(g_a);
        double s = *(double *)alpha;
        long n = patch_len(a, lo, hi);
        for (long k = 0; k < n; k++) a->d[patch_off(a, lo, hi, k)] += s;
}

void GA_Add(void *alpha, int g_a, void *beta, int g_b, int g_c)
{
        struct shim_array *a = get(g_a), *b = get(g_b), *c = get(g_c);
        double s = *(double *)alpha, t = *(double *)beta;
        for (long k = 0; k < c->nelem; k++)
                c->d[k] = s * a->d[k] + t * b->d[k];
}

void NGA_Add_patch(void *alpha, int g_a, int alo[], int ahi[], void *beta,
                   int g_b, int blo[], int bhi[], int g_c, int clo[],
                   int chi[])
{
        struct shim_array *a = get(g_a), *b = get(g_b), *c = get(g_c);
        double s = *(double *)alpha, t = *(double *)beta;
        long n = patch_len(c, clo, chi);
        for (long k = 0; k < n; k++) {
                double x = a->d[patch_off(a, alo, ahi, k)];
                double y = b->d[patch_off(b, blo, bhi, k)];
                c->d[patch_off(c, clo, chi, k)] = s * x + t * y;
        }
}

void GA_Elem_divide(int g_a, int g_b, int g_c)
{
        struct shim_array *a = get(g_a), *b = get(g_b), *c = get(g_c);
        for (long k = 0; k < c->nelem; k++) c->d[k] = a->d[k] / b->d[k];
}

void GA_Elem_multiply_patch(int g_a, int alo[], int ahi[], int g_b,
                            int blo[], int bhi[], int g_c, int clo[],
                            int chi[])
{
        struct shim_array *a = get(g_a), *b = get(g_b), *c = get(g_c);
        long n = patch_len(c, clo, chi);
        for (long k = 0; k < n; k++)
                c->d[patch_off(c, clo, chi, k)] =
                        a->d[patch_off(a, alo, ahi, k)] *
                        b->d[patch_off(b, blo, bhi, k)];
}

double GA_Ddot(int g_a, int g_b)
{
        struct shim_array *a = get(g_a), *b = get(g_b);
        double s = 0.0;
        for (long k = 0; k < a->nelem; k++) s += a->d[k] * b->d[k];
        return s;
}

double NGA_Ddot_patch(int g_a, char ta, int alo[], int ahi[], int g_b,
                      char tb, int blo[], int bhi[])
{
        struct shim_array *a = get(g_a), *b = get(g_b);
        (void)ta; (void)tb;
        long n = patch_len(a, alo, ahi);
        double s = 0.0;
        for (long k = 0; k < n; k++)
                s += a->d[patch_off(a, alo, ahi, k)] *
                     b->d[patch_off(b, blo, bhi, k)];
        return s;
}

void NGA_Print_patch(int g_a, int lo[], int hi[], int pretty)
{
        struct shim_array *a = get(g_a);
        (void)pretty;
        long n = patch_len(a, lo, hi);
        for (long k = 0; k < n; k++)
                printf("%ld %.12e\n", k, a->d[patch_off(a, lo, hi, k)]);
}

void GA_Print_file(FILE *f, int g_a)
{
        struct shim_array *a = get(g_a);
        for (long k = 0; k < a->nelem; k++)
                fprintf(f, "%ld %.12e\n", k, a->d[k]);
}

/* Direct access to an array's storage, for the oracle harness. */
double *shim_ga_data(int g_a) { return get(g_a)->d; }

/* Release every array (the reference never calls GA_Destroy). */
void shim_ga_reset(void)
{
        for (int g = 0; g < SHIM_MAX_ARRAYS; g++) {
                free(arrays[g].d);
                free(arrays[g].i);
                memset(&arrays[g], 0, sizeof(arrays[g]));
        }
}

/* --- MPI, one rank -------------------------------------------------- */

int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return 0; }
int MPI_Finalize(void) { return 0; }
int MPI_Comm_size(MPI_Comm comm, int *size) { (void)comm; *size = 1; return 0; }
int MPI_Comm_rank(MPI_Comm comm, int *rank) { (void)comm; *rank = 0; return 0; }

int MPI_Bcast(void *buf, int count, MPI_Datatype type, int root,
              MPI_Comm comm)
{
        (void)buf; (void)count; (void)type; (void)root; (void)comm;
        return 0;
}

int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count,
                  MPI_Datatype type, MPI_Op op, MPI_Comm comm)
{
        (void)op; (void)comm;
        size_t sz = type == MPI_DOUBLE ? sizeof(double)
                  : type == MPI_2INT ? 2 * sizeof(int) : sizeof(int);
        memmove(recvbuf, sendbuf, sz * count);
        return 0;
}

int MA_init(int type, long stack, long heap)
{
        (void)type; (void)stack; (void)heap;
        return 1;
}
