/*
 * Single-process stand-in for <mpi.h>, used only to compile the reference
 * CPU sources into the checker library under oracle/_ref.  Every call
 * behaves as a one-rank MPI_COMM_WORLD.  Test infrastructure, not product.
 */
#ifndef CROMA_ORACLE_SHIM_MPI_H
#define CROMA_ORACLE_SHIM_MPI_H

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_COMM_NULL (-1)
#define MPI_SUCCESS 0
#define MPI_PROC_NULL (-2)
#define MPI_UNDEFINED (-32766)
#define MPI_DOUBLE 1
#define MPI_INT 2
#define MPI_LONG 3
#define MPI_LONG_LONG 4
#define MPI_CHAR 5
#define MPI_2INT 6
#define MPI_UNSIGNED_CHAR 7
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPI_MAXLOC 4
#define MPI_IN_PLACE ((void *)1)
#define MPI_STATUS_IGNORE ((MPI_Status *)0)

int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Abort(MPI_Comm comm, int code);
int MPI_Initialized(int *flag);
int MPI_Dims_create(int nnodes, int ndims, int *dims);
int MPI_Comm_split(MPI_Comm comm, int color, int key, MPI_Comm *newcomm);
int MPI_Comm_free(MPI_Comm *comm);
int MPI_Barrier(MPI_Comm comm);
int MPI_Bcast(void *buf, int count, MPI_Datatype type, int root, MPI_Comm comm);

#endif
