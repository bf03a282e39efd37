/*
 * Single-rank stand-in for the MPI interface the PittPack sources use, so that
 * the reference's CPU path compiles and runs as "mpirun -np 1" without an MPI
 * library.  TEST INFRASTRUCTURE ONLY (oracle/_ref).  Point-to-point messages
 * can only go to rank 0 (this process) and are matched by tag; collectives on
 * one rank are copies.
 */
#ifndef PP_SHIM_MPI_H
#define PP_SHIM_MPI_H
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef int MPI_Info;
typedef int MPI_Errhandler;
typedef struct {
    int MPI_SOURCE;
    int MPI_TAG;
    int MPI_ERROR;
} MPI_Status;

#define MPI_SUCCESS 0
#define MPI_ERR_OTHER 15
#define MPI_COMM_WORLD 1
#define MPI_COMM_NULL 0
#define MPI_COMM_TYPE_SHARED 1
#define MPI_CHAR 1
#define MPI_BYTE 2
#define MPI_INT 3
#define MPI_UNSIGNED 4
#define MPI_LONG 5
#define MPI_UNSIGNED_LONG 6
#define MPI_FLOAT 7
#define MPI_DOUBLE 8
#define MPI_UNSIGNED_SHORT 9
#define MPI_SHORT 10
#define MPI_LONG_LONG 11
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPI_INFO_NULL 0
#define MPI_ERRORS_RETURN 1
#define MPI_ERRORS_ARE_FATAL 2
#define MPI_MAX_PROCESSOR_NAME 256
#define MPI_UNDEFINED (-32766)
#define MPI_REQUEST_NULL (-1)
#define MPI_IN_PLACE ((void*)1)
#define MPI_UNWEIGHTED ((int*)2)
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)

int MPI_Init(int* argc, char*** argv);
int MPI_Initialized(int* flag);
int MPI_Finalized(int* flag);
int MPI_Finalize(void);
int MPI_Abort(MPI_Comm comm, int code);
double MPI_Wtime(void);
int MPI_Comm_dup(MPI_Comm comm, MPI_Comm* out);
int MPI_Comm_rank(MPI_Comm comm, int* rank);
int MPI_Comm_size(MPI_Comm comm, int* size);
int MPI_Comm_split(MPI_Comm comm, int color, int key, MPI_Comm* out);
int MPI_Comm_split_type(MPI_Comm comm, int type, int key, MPI_Info info, MPI_Comm* out);
int MPI_Comm_free(MPI_Comm* comm);
int MPI_Comm_set_errhandler(MPI_Comm comm, MPI_Errhandler h);
int MPI_Get_processor_name(char* name, int* len);
int MPI_Barrier(MPI_Comm comm);
int MPI_Isend(const void* buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm comm, MPI_Request* req);
int MPI_Irecv(void* buf, int count, MPI_Datatype t, int src, int tag, MPI_Comm comm, MPI_Request* req);
int MPI_Send(const void* buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm comm);
int MPI_Recv(void* buf, int count, MPI_Datatype t, int src, int tag, MPI_Comm comm, MPI_Status* st);
int MPI_Sendrecv(const void* sbuf, int scount, MPI_Datatype st, int dest, int stag, void* rbuf, int rcount,
                 MPI_Datatype rt, int src, int rtag, MPI_Comm comm, MPI_Status* status);
int MPI_Wait(MPI_Request* req, MPI_Status* st);
int MPI_Waitall(int n, MPI_Request* reqs, MPI_Status* sts);
int MPI_Waitany(int n, MPI_Request* reqs, int* index, MPI_Status* st);
int MPI_Allreduce(const void* s, void* r, int count, MPI_Datatype t, MPI_Op op, MPI_Comm comm);
int MPI_Reduce(const void* s, void* r, int count, MPI_Datatype t, MPI_Op op, int root, MPI_Comm comm);
int MPI_Bcast(void* buf, int count, MPI_Datatype t, int root, MPI_Comm comm);
int MPI_Gather(const void* s, int sc, MPI_Datatype st, void* r, int rc, MPI_Datatype rt, int root, MPI_Comm comm);
int MPI_Allgather(const void* s, int sc, MPI_Datatype st, void* r, int rc, MPI_Datatype rt, MPI_Comm comm);
int MPI_Dist_graph_create_adjacent(MPI_Comm comm, int indeg, const int* src, const int* sw, int outdeg,
                                   const int* dst, const int* dw, MPI_Info info, int reorder, MPI_Comm* out);
int MPI_Dist_graph_neighbors_count(MPI_Comm comm, int* indeg, int* outdeg, int* weighted);
int MPI_Dist_graph_neighbors(MPI_Comm comm, int maxin, int* src, int* sw, int maxout, int* dst, int* dw);
int MPI_Neighbor_alltoall(const void* s, int sc, MPI_Datatype st, void* r, int rc, MPI_Datatype rt, MPI_Comm comm);
int MPI_Ineighbor_alltoall(const void* s, int sc, MPI_Datatype st, void* r, int rc, MPI_Datatype rt, MPI_Comm comm,
                           MPI_Request* req);
int MPI_Neighbor_alltoallv(const void* s, const int* sc, const int* sd, MPI_Datatype st, void* r, const int* rc,
                           const int* rd, MPI_Datatype rt, MPI_Comm comm);

#ifdef __cplusplus
}
#endif
#endif
