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
#define MPI_SUM 0
#endif
