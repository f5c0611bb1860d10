/*
 * Single-rank stand-in for the MPI interface, written for this project so
 * that the reference's own C sources (which include "mpi.h") can be compiled
 * and run as one process without an MPI library.
 *
 * Semantics, for exactly one rank (rank 0, size 1):
 *   - collectives (Allreduce, Reduce, Allgather, Bcast, Alltoall...) copy the
 *     send buffer to the receive buffer, or do nothing with MPI_IN_PLACE;
 *   - MPI_Cart_create remembers the periodic flags; MPI_Cart_shift returns
 *     rank 0 (self) along periodic axes and MPI_PROC_NULL along walled axes;
 *   - MPI_Sendrecv to self copies the send buffer into the receive buffer;
 *     with MPI_PROC_NULL on either side nothing is transferred;
 *   - MPI_Wtime reads CLOCK_MONOTONIC.
 * This is test infrastructure for the CPU oracle build only.
 */
#ifndef PVOF_SHIM_MPI_H
#define PVOF_SHIM_MPI_H

#include <stddef.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef int MPI_Info;
typedef long MPI_Aint;

typedef struct {
    int MPI_SOURCE;
    int MPI_TAG;
    int MPI_ERROR;
    int count_bytes;
} MPI_Status;

#define MPI_SUCCESS 0
#define MPI_COMM_WORLD 1
#define MPI_COMM_SELF 2
#define MPI_COMM_NULL 0
#define MPI_PROC_NULL (-2)
#define MPI_ANY_SOURCE (-1)
#define MPI_ANY_TAG (-1)
#define MPI_UNDEFINED (-32766)
#define MPI_INFO_NULL 0
#define MPI_COMM_TYPE_SHARED 1
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)
#define MPI_IN_PLACE ((void *)1)
#define MPI_REQUEST_NULL 0
#define MPI_MAX_PROCESSOR_NAME 64

/* built-in datatypes are negative codes; derived types index a size table */
#define MPI_DOUBLE (-1)
#define MPI_INT (-2)
#define MPI_LONG (-3)
#define MPI_BYTE (-4)
#define MPI_CHAR (-5)
#define MPI_FLOAT (-6)
#define MPI_UNSIGNED (-7)
#define MPI_LONG_LONG (-8)
#define MPI_UNSIGNED_LONG (-9)
#define MPI_SHORT (-10)
#define MPI_LONG_DOUBLE (-11)
#define MPI_C_BOOL (-12)
#define MPI_DOUBLE_INT (-13)
#define MPI_2INT (-14)

#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPI_PROD 4
#define MPI_LAND 5
#define MPI_LOR 6
#define MPI_MAXLOC 7
#define MPI_MINLOC 8
#define MPI_BOR 9

int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Initialized(int *flag);
int MPI_Abort(MPI_Comm comm, int code);
double MPI_Wtime(void);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_split(MPI_Comm comm, int color, int key, MPI_Comm *newcomm);
int MPI_Comm_split_type(MPI_Comm comm, int type, int key, MPI_Info info, MPI_Comm *newcomm);
int MPI_Comm_dup(MPI_Comm comm, MPI_Comm *newcomm);
int MPI_Comm_free(MPI_Comm *comm);
int MPI_Barrier(MPI_Comm comm);
int MPI_Bcast(void *buf, int count, MPI_Datatype t, int root, MPI_Comm comm);
int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype t, MPI_Op op, MPI_Comm comm);
int MPI_Reduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype t, MPI_Op op, int root, MPI_Comm comm);
int MPI_Allgather(const void *sendbuf, int scount, MPI_Datatype st, void *recvbuf, int rcount, MPI_Datatype rt, MPI_Comm comm);
int MPI_Allgatherv(const void *sendbuf, int scount, MPI_Datatype st, void *recvbuf, const int *rcounts, const int *displs, MPI_Datatype rt, MPI_Comm comm);
int MPI_Gather(const void *sendbuf, int scount, MPI_Datatype st, void *recvbuf, int rcount, MPI_Datatype rt, int root, MPI_Comm comm);
int MPI_Gatherv(const void *sendbuf, int scount, MPI_Datatype st, void *recvbuf, const int *rcounts, const int *displs, MPI_Datatype rt, int root, MPI_Comm comm);
int MPI_Scatter(const void *sendbuf, int scount, MPI_Datatype st, void *recvbuf, int rcount, MPI_Datatype rt, int root, MPI_Comm comm);
int MPI_Alltoall(const void *sendbuf, int scount, MPI_Datatype st, void *recvbuf, int rcount, MPI_Datatype rt, MPI_Comm comm);
int MPI_Alltoallv(const void *sendbuf, const int *scounts, const int *sdispls, MPI_Datatype st, void *recvbuf, const int *rcounts, const int *rdispls, MPI_Datatype rt, MPI_Comm comm);
int MPI_Sendrecv(const void *sendbuf, int scount, MPI_Datatype st, int dest, int stag,
                 void *recvbuf, int rcount, MPI_Datatype rt, int source, int rtag,
                 MPI_Comm comm, MPI_Status *status);
int MPI_Send(const void *buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm comm);
int MPI_Recv(void *buf, int count, MPI_Datatype t, int source, int tag, MPI_Comm comm, MPI_Status *status);
int MPI_Isend(const void *buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm comm, MPI_Request *req);
int MPI_Irecv(void *buf, int count, MPI_Datatype t, int source, int tag, MPI_Comm comm, MPI_Request *req);
int MPI_Wait(MPI_Request *req, MPI_Status *status);
int MPI_Waitall(int n, MPI_Request *reqs, MPI_Status *statuses);
int MPI_Waitany(int n, MPI_Request *reqs, int *index, MPI_Status *status);
int MPI_Get_count(const MPI_Status *status, MPI_Datatype t, int *count);
int MPI_Cart_create(MPI_Comm old, int ndims, const int *dims, const int *periods, int reorder, MPI_Comm *cart);
int MPI_Cart_get(MPI_Comm comm, int maxdims, int *dims, int *periods, int *coords);
int MPI_Cart_shift(MPI_Comm comm, int dir, int disp, int *source, int *dest);
int MPI_Cart_rank(MPI_Comm comm, const int *coords, int *rank);
int MPI_Cart_coords(MPI_Comm comm, int rank, int maxdims, int *coords);
int MPI_Dims_create(int nnodes, int ndims, int *dims);
int MPI_Type_create_struct(int count, const int *blocklens, const MPI_Aint *displs, const MPI_Datatype *types, MPI_Datatype *newtype);
int MPI_Type_contiguous(int count, MPI_Datatype old, MPI_Datatype *newtype);
int MPI_Type_commit(MPI_Datatype *t);
int MPI_Type_free(MPI_Datatype *t);
int MPI_Type_size(MPI_Datatype t, int *size);
int MPI_Get_address(const void *loc, MPI_Aint *addr);
int MPI_Info_create(MPI_Info *info);
int MPI_Info_set(MPI_Info info, const char *key, const char *value);
int MPI_Info_free(MPI_Info *info);
int MPI_Get_processor_name(char *name, int *len);

#endif
