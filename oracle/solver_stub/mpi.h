/* ORACLE build only: the MPI names Apollo's headers use, for one process.
 * ref_driver.cpp defines the calls (a single rank: reductions copy). */
#ifndef APOLLO_ORACLE_MPI_STUB_H
#define APOLLO_ORACLE_MPI_STUB_H
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;
#define MPI_COMM_WORLD 1
#define MPI_COMM_SELF 2
#define MPI_INT 1
#define MPI_DOUBLE 2
#define MPI_FLOAT 3
#define MPI_UNSIGNED 4
#define MPI_CHAR 5
#define MPI_UNSIGNED_CHAR 6
#define MPI_SHORT 7
#define MPI_UNSIGNED_SHORT 8
#define MPI_LONG 9
#define MPI_UNSIGNED_LONG 10
#define MPI_LONG_DOUBLE 11
#define MPI_LONG_LONG_INT 12
#define MPI_SUM 1
#define MPI_MIN 2
#define MPI_MAX 3
int MPI_Allreduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype type, MPI_Op op, MPI_Comm comm);
int MPI_Comm_rank(MPI_Comm comm, int* rank);
int MPI_Comm_size(MPI_Comm comm, int* size);
int MPI_Barrier(MPI_Comm comm);
#endif
