/* Test-infrastructure shim: the oracle links no MPI; headers that include
 * <mpi.h> only need it to parse. */
#ifndef ORACLE_SHIM_MPI_H
#define ORACLE_SHIM_MPI_H
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_File;
typedef long MPI_Offset;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;
#define MPI_COMM_WORLD 0
#define MPI_FLOAT 0
#define MPI_DOUBLE 1
#define MPI_INT 2
#define MPI_SUM 0
/* single-rank stand-ins, defined in harness_enkf.cpp (src/enfwi/Matrix.cpp
 * calls these in its parallel sums, which the oracle does not use) */
int MPI_Reduce(const void *in, void *out, int count, MPI_Datatype t, MPI_Op op, int root, MPI_Comm c);
int MPI_Gather(const void *in, int n, MPI_Datatype t, void *out, int m, MPI_Datatype u, int root,
               MPI_Comm c);
#endif
