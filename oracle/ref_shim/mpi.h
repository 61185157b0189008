/*
 * Single-process stand-in for the handful of MPI entry points that the
 * reference's mpi_source/*.c files name (test infrastructure only).
 *
 * With one rank every collective is a local copy.  Call sites this covers:
 * execute_pjayci.c:109-137 (MPI_Bcast), mpi_utilities.c:38,40
 * (MPI_Allreduce SUM / MAXLOC), pjayci.c:34,46 (init / finalize).
 */
#ifndef ORACLE_SHIM_MPI_H
#define ORACLE_SHIM_MPI_H

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;

#define MPI_COMM_WORLD 0
#define MPI_INT        1
#define MPI_DOUBLE     2
#define MPI_2INT       3
#define MPI_SUM        1
#define MPI_MAXLOC     2

int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Bcast(void *buf, int count, MPI_Datatype type, int root,
              MPI_Comm comm);
int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count,
                  MPI_Datatype type, MPI_Op op, MPI_Comm comm);

#endif
