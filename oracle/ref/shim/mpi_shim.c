/*
 * Single-rank MPI implementation for the oracle build of the reference
 * sources (see mpi.h for the semantics).  Test infrastructure only.
 */
#include "mpi.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#define SHIM_MAX_TYPES 64

static int g_periods[3] = {0, 0, 0};
static int g_type_sizes[SHIM_MAX_TYPES];
static int g_ntypes = 0;

static size_t type_size(MPI_Datatype t)
{
    switch (t) {
    case MPI_DOUBLE: return sizeof(double);
    case MPI_INT: return sizeof(int);
    case MPI_LONG: return sizeof(long);
    case MPI_BYTE: return 1;
    case MPI_CHAR: return 1;
    case MPI_FLOAT: return sizeof(float);
    case MPI_UNSIGNED: return sizeof(unsigned);
    case MPI_LONG_LONG: return sizeof(long long);
    case MPI_UNSIGNED_LONG: return sizeof(unsigned long);
    case MPI_SHORT: return sizeof(short);
    case MPI_LONG_DOUBLE: return sizeof(long double);
    case MPI_C_BOOL: return 1;
    case MPI_DOUBLE_INT: return sizeof(double) + sizeof(int) + 4;
    case MPI_2INT: return 2 * sizeof(int);
    default:
        if (t >= 0 && t < g_ntypes)
            return (size_t)g_type_sizes[t];
        fprintf(stderr, "mpi shim: unknown datatype %d\n", t);
        abort();
    }
}

static void copy_buf(const void *src, void *dst, int count, MPI_Datatype t)
{
    if (src == MPI_IN_PLACE || src == dst || count <= 0)
        return;
    memmove(dst, src, (size_t)count * type_size(t));
}

int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return 0; }
int MPI_Finalize(void) { return 0; }
int MPI_Initialized(int *flag) { *flag = 1; return 0; }
int MPI_Abort(MPI_Comm comm, int code) { (void)comm; exit(code); }

double MPI_Wtime(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

int MPI_Comm_size(MPI_Comm comm, int *size) { (void)comm; *size = 1; return 0; }
int MPI_Comm_rank(MPI_Comm comm, int *rank) { (void)comm; *rank = 0; return 0; }
int MPI_Comm_split(MPI_Comm comm, int color, int key, MPI_Comm *newcomm)
{ (void)color; (void)key; *newcomm = comm; return 0; }
int MPI_Comm_split_type(MPI_Comm comm, int type, int key, MPI_Info info, MPI_Comm *newcomm)
{ (void)type; (void)key; (void)info; *newcomm = comm; return 0; }
int MPI_Comm_dup(MPI_Comm comm, MPI_Comm *newcomm) { *newcomm = comm; return 0; }
int MPI_Comm_free(MPI_Comm *comm) { (void)comm; return 0; }
int MPI_Barrier(MPI_Comm comm) { (void)comm; return 0; }
int MPI_Bcast(void *buf, int count, MPI_Datatype t, int root, MPI_Comm comm)
{ (void)buf; (void)count; (void)t; (void)root; (void)comm; return 0; }

int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype t, MPI_Op op, MPI_Comm comm)
{ (void)op; (void)comm; copy_buf(sendbuf, recvbuf, count, t); return 0; }
int MPI_Reduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype t, MPI_Op op, int root, MPI_Comm comm)
{ (void)op; (void)root; (void)comm; copy_buf(sendbuf, recvbuf, count, t); return 0; }
int MPI_Allgather(const void *sendbuf, int scount, MPI_Datatype st, void *recvbuf, int rcount, MPI_Datatype rt, MPI_Comm comm)
{ (void)rcount; (void)rt; (void)comm; copy_buf(sendbuf, recvbuf, scount, st); return 0; }
int MPI_Allgatherv(const void *sendbuf, int scount, MPI_Datatype st, void *recvbuf, const int *rcounts, const int *displs, MPI_Datatype rt, MPI_Comm comm)
{
    (void)rcounts; (void)comm;
    if (sendbuf == MPI_IN_PLACE) return 0;
    copy_buf(sendbuf, (char *)recvbuf + (size_t)displs[0] * type_size(rt), scount, st);
    return 0;
}
int MPI_Gather(const void *sendbuf, int scount, MPI_Datatype st, void *recvbuf, int rcount, MPI_Datatype rt, int root, MPI_Comm comm)
{ (void)rcount; (void)rt; (void)root; (void)comm; copy_buf(sendbuf, recvbuf, scount, st); return 0; }
int MPI_Gatherv(const void *sendbuf, int scount, MPI_Datatype st, void *recvbuf, const int *rcounts, const int *displs, MPI_Datatype rt, int root, MPI_Comm comm)
{
    (void)rcounts; (void)root; (void)comm;
    if (sendbuf == MPI_IN_PLACE) return 0;
    copy_buf(sendbuf, (char *)recvbuf + (size_t)displs[0] * type_size(rt), scount, st);
    return 0;
}
int MPI_Scatter(const void *sendbuf, int scount, MPI_Datatype st, void *recvbuf, int rcount, MPI_Datatype rt, int root, MPI_Comm comm)
{ (void)rcount; (void)rt; (void)root; (void)comm; copy_buf(sendbuf, recvbuf, scount, st); return 0; }
int MPI_Alltoall(const void *sendbuf, int scount, MPI_Datatype st, void *recvbuf, int rcount, MPI_Datatype rt, MPI_Comm comm)
{ (void)rcount; (void)rt; (void)comm; copy_buf(sendbuf, recvbuf, scount, st); return 0; }
int MPI_Alltoallv(const void *sendbuf, const int *scounts, const int *sdispls, MPI_Datatype st, void *recvbuf, const int *rcounts, const int *rdispls, MPI_Datatype rt, MPI_Comm comm)
{
    (void)rcounts; (void)comm;
    copy_buf((const char *)sendbuf + (size_t)sdispls[0] * type_size(st),
             (char *)recvbuf + (size_t)rdispls[0] * type_size(rt), scounts[0], st);
    return 0;
}

/* A message sent to self with MPI_Send waits here until the matching receive. */
static void *g_pending = NULL;
static size_t g_pending_bytes = 0;

int MPI_Sendrecv(const void *sendbuf, int scount, MPI_Datatype st, int dest, int stag,
                 void *recvbuf, int rcount, MPI_Datatype rt, int source, int rtag,
                 MPI_Comm comm, MPI_Status *status)
{
    (void)stag; (void)rtag; (void)comm;
    if (dest != MPI_PROC_NULL && source != MPI_PROC_NULL) {
        size_t sb = (size_t)scount * type_size(st);
        size_t rb = (size_t)rcount * type_size(rt);
        memmove(recvbuf, sendbuf, sb < rb ? sb : rb);
        if (status) { status->MPI_SOURCE = 0; status->count_bytes = (int)(sb < rb ? sb : rb); }
    } else if (status) {
        status->MPI_SOURCE = MPI_PROC_NULL;
        status->count_bytes = 0;
    }
    return 0;
}

int MPI_Send(const void *buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm comm)
{
    (void)tag; (void)comm;
    if (dest == MPI_PROC_NULL) return 0;
    free(g_pending);
    g_pending_bytes = (size_t)count * type_size(t);
    g_pending = malloc(g_pending_bytes ? g_pending_bytes : 1);
    memcpy(g_pending, buf, g_pending_bytes);
    return 0;
}

int MPI_Recv(void *buf, int count, MPI_Datatype t, int source, int tag, MPI_Comm comm, MPI_Status *status)
{
    (void)tag; (void)comm;
    if (source == MPI_PROC_NULL) {
        if (status) status->count_bytes = 0;
        return 0;
    }
    size_t want = (size_t)count * type_size(t);
    size_t n = g_pending_bytes < want ? g_pending_bytes : want;
    if (g_pending) memcpy(buf, g_pending, n);
    if (status) { status->MPI_SOURCE = 0; status->count_bytes = (int)n; }
    free(g_pending);
    g_pending = NULL;
    g_pending_bytes = 0;
    return 0;
}

int MPI_Isend(const void *buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm comm, MPI_Request *req)
{ *req = 0; return MPI_Send(buf, count, t, dest, tag, comm); }
int MPI_Irecv(void *buf, int count, MPI_Datatype t, int source, int tag, MPI_Comm comm, MPI_Request *req)
{ *req = 0; return MPI_Recv(buf, count, t, source, tag, comm, NULL); }
int MPI_Wait(MPI_Request *req, MPI_Status *status) { (void)req; (void)status; return 0; }
int MPI_Waitall(int n, MPI_Request *reqs, MPI_Status *statuses) { (void)n; (void)reqs; (void)statuses; return 0; }
int MPI_Waitany(int n, MPI_Request *reqs, int *index, MPI_Status *status)
{ (void)reqs; (void)status; *index = n > 0 ? 0 : MPI_UNDEFINED; return 0; }
int MPI_Get_count(const MPI_Status *status, MPI_Datatype t, int *count)
{ *count = status ? (int)(status->count_bytes / (int)type_size(t)) : 0; return 0; }

int MPI_Cart_create(MPI_Comm old, int ndims, const int *dims, const int *periods, int reorder, MPI_Comm *cart)
{
    (void)old; (void)reorder;
    for (int d = 0; d < ndims && d < 3; d++) {
        if (dims[d] != 1) {
            fprintf(stderr, "mpi shim: only a 1x1x1 process grid is supported\n");
            abort();
        }
        g_periods[d] = periods[d];
    }
    *cart = MPI_COMM_WORLD;
    return 0;
}

int MPI_Cart_get(MPI_Comm comm, int maxdims, int *dims, int *periods, int *coords)
{
    (void)comm;
    for (int d = 0; d < maxdims && d < 3; d++) {
        dims[d] = 1;
        periods[d] = g_periods[d];
        coords[d] = 0;
    }
    return 0;
}

int MPI_Cart_shift(MPI_Comm comm, int dir, int disp, int *source, int *dest)
{
    (void)comm; (void)disp;
    int nb = (dir >= 0 && dir < 3 && g_periods[dir]) ? 0 : MPI_PROC_NULL;
    *source = nb;
    *dest = nb;
    return 0;
}

int MPI_Cart_rank(MPI_Comm comm, const int *coords, int *rank) { (void)comm; (void)coords; *rank = 0; return 0; }
int MPI_Cart_coords(MPI_Comm comm, int rank, int maxdims, int *coords)
{ (void)comm; (void)rank; for (int d = 0; d < maxdims; d++) coords[d] = 0; return 0; }
int MPI_Dims_create(int nnodes, int ndims, int *dims)
{ (void)nnodes; for (int d = 0; d < ndims; d++) if (dims[d] == 0) dims[d] = 1; return 0; }

int MPI_Type_create_struct(int count, const int *blocklens, const MPI_Aint *displs, const MPI_Datatype *types, MPI_Datatype *newtype)
{
    size_t extent = 0;
    for (int n = 0; n < count; n++) {
        size_t end = (size_t)displs[n] + (size_t)blocklens[n] * type_size(types[n]);
        if (end > extent) extent = end;
    }
    if (g_ntypes >= SHIM_MAX_TYPES) abort();
    g_type_sizes[g_ntypes] = (int)((extent + 7) & ~(size_t)7);
    *newtype = g_ntypes++;
    return 0;
}

int MPI_Type_contiguous(int count, MPI_Datatype old, MPI_Datatype *newtype)
{
    if (g_ntypes >= SHIM_MAX_TYPES) abort();
    g_type_sizes[g_ntypes] = (int)((size_t)count * type_size(old));
    *newtype = g_ntypes++;
    return 0;
}

int MPI_Type_commit(MPI_Datatype *t) { (void)t; return 0; }
int MPI_Type_free(MPI_Datatype *t) { (void)t; return 0; }
int MPI_Type_size(MPI_Datatype t, int *size) { *size = (int)type_size(t); return 0; }
int MPI_Get_address(const void *loc, MPI_Aint *addr) { *addr = (MPI_Aint)loc; return 0; }
int MPI_Info_create(MPI_Info *info) { *info = 0; return 0; }
int MPI_Info_set(MPI_Info info, const char *key, const char *value) { (void)info; (void)key; (void)value; return 0; }
int MPI_Info_free(MPI_Info *info) { (void)info; return 0; }
int MPI_Get_processor_name(char *name, int *len) { strcpy(name, "localhost"); *len = 9; return 0; }
