/*
 * Single-process Global Arrays stand-in (test infrastructure only).
 *
 * The reference's pdavidson.c keeps every vector in a Global Array
 * (pdavidson.c:111-135) and moves data with NGA_Get/Put/Acc and the GA
 * BLAS-1 patch operations.  With one rank a Global Array is one host array
 * in C row-major order: dims[0] is the slow index, dims[1] the fast one, and
 * a patch [lo, hi] (inclusive) is visited in row-major order.  The local
 * buffer of NGA_Get/Put/Acc has leading dimension ld[0] (elements of the
 * fast index per buffer row).  That is the behaviour the reference relies on
 * at pdavidson.c:1343-1395 and mpi_utilities.c:353-419.
 */
#ifndef ORACLE_SHIM_GA_H
#define ORACLE_SHIM_GA_H

#include <stdio.h>

#define C_INT 1001
#define C_DBL 1003
#define C_LONG 1002

void GA_Initialize(void);
void GA_Terminate(void);
void GA_Sync(void);
int GA_Nodeid(void);
int GA_Nnodes(void);
void GA_Error(char *msg, int code);

int NGA_Create(int type, int ndim, int dims[], char *name, int chunk[]);
int NGA_Duplicate(int g_a, char *name);
void NGA_Inquire(int g_a, int *type, int *ndim, int dims[]);
void NGA_Distribution(int g_a, int iproc, int lo[], int hi[]);

void NGA_Get(int g_a, int lo[], int hi[], void *buf, int ld[]);
void NGA_Put(int g_a, int lo[], int hi[], void *buf, int ld[]);
void NGA_Acc(int g_a, int lo[], int hi[], void *buf, int ld[], void *alpha);
void NGA_Gather(int g_a, void *v, int *subs[], int n);
void NGA_Scatter_acc(int g_a, void *v, int *subs[], int n, void *alpha);
void NGA_Alloc_gatscat_buf(int nelems);
void NGA_Free_gatscat_buf(void);

void NGA_Zero(int g_a);
void GA_Zero(int g_a);
void GA_Copy(int g_a, int g_b);
void NGA_Copy_patch(char trans, int g_a, int alo[], int ahi[], int g_b,
                    int blo[], int bhi[]);
void GA_Scale(int g_a, void *alpha);
void GA_Add_constant(int g_a, void *alpha);
void GA_Add_constant_patch(int g_a, int lo[], int hi[], void *alpha);
void GA_Add(void *alpha, int g_a, void *beta, int g_b, int g_c);
void NGA_Add_patch(void *alpha, int g_a, int alo[], int ahi[], void *beta,
                   int g_b, int blo[], int bhi[], int g_c, int clo[],
                   int chi[]);
void GA_Elem_divide(int g_a, int g_b, int g_c);
void GA_Elem_multiply_patch(int g_a, int alo[], int ahi[], int g_b,
                            int blo[], int bhi[], int g_c, int clo[],
                            int chi[]);
double GA_Ddot(int g_a, int g_b);
double NGA_Ddot_patch(int g_a, char ta, int alo[], int ahi[], int g_b,
                      char tb, int blo[], int bhi[]);
void NGA_Print_patch(int g_a, int lo[], int hi[], int pretty);
void GA_Print_file(FILE *f, int g_a);

#endif
