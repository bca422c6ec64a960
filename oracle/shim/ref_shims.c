/*
 * Link-time stand-ins for the few external symbols that the reference CPU
 * sources reference but that are absent from this image (MPI, GNU GSL, the
 * cosmology and HDF5 translation units).  They are compiled only into the
 * checker library oracle/_ref/libcroma_ref_np*.so.  Test infrastructure:
 * nothing in the product links this file.
 *
 * - MPI: one rank, MPI_COMM_WORLD of size 1 (the tracer FP loop itself
 *   never communicates; see tracer_fp_batch.c in the reference).
 * - gsl_sf_gamma / gsl_sf_hyperg_*: only reached from PP95_analytic
 *   (src/Chang_Cooper.c:257-269), an analytic test solution that the hot
 *   path never calls.  They return NaN.
 * - gsl_sf_synchrotron_1: only reached from SYN_logFx_table
 *   (src/Synchrotron.c:31-41) when synchrotron tables are built; it returns
 *   the checker's F(x) = x int_x^inf K_5/3 restated from the integral
 *   definition (oracle/synch_fx.c), so the reference's table code runs.
 * - luminosity_distance_mpc: only used by the file writers
 *   (src/EMISSION.c:152, 250), which the checker never calls.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include "mpi.h"

int MPI_Comm_rank(MPI_Comm comm, int *rank) { (void)comm; if (rank) *rank = 0; return MPI_SUCCESS; }
int MPI_Comm_size(MPI_Comm comm, int *size) { (void)comm; if (size) *size = 1; return MPI_SUCCESS; }
int MPI_Abort(MPI_Comm comm, int code) { (void)comm; fprintf(stderr, "MPI_Abort(%d)\n", code); abort(); }
int MPI_Initialized(int *flag) { if (flag) *flag = 1; return MPI_SUCCESS; }
int MPI_Dims_create(int nnodes, int ndims, int *dims)
{
    int i;
    for (i = 0; i < ndims; i++) dims[i] = (i == 0) ? nnodes : 1;
    return MPI_SUCCESS;
}
int MPI_Comm_split(MPI_Comm comm, int color, int key, MPI_Comm *newcomm)
{
    (void)color; (void)key;
    if (newcomm) *newcomm = comm;
    return MPI_SUCCESS;
}
int MPI_Comm_free(MPI_Comm *comm) { if (comm) *comm = MPI_COMM_NULL; return MPI_SUCCESS; }
int MPI_Barrier(MPI_Comm comm) { (void)comm; return MPI_SUCCESS; }
int MPI_Bcast(void *buf, int count, MPI_Datatype type, int root, MPI_Comm comm)
{
    (void)buf; (void)count; (void)type; (void)root; (void)comm;
    return MPI_SUCCESS;
}

double gsl_sf_gamma(double x) { (void)x; return NAN; }
double gsl_sf_hyperg_1F1(double a, double b, double x) { (void)a; (void)b; (void)x; return NAN; }
double gsl_sf_hyperg_U(double a, double b, double x) { (void)a; (void)b; (void)x; return NAN; }

double oracle_synch_fx(double x);
double gsl_sf_synchrotron_1(double x) { return oracle_synch_fx(x); }

double luminosity_distance_mpc(double z) { (void)z; return NAN; }
