// Single-rank MPI for the reference build.  TEST INFRASTRUCTURE ONLY
// (oracle/_ref).  Every send goes to this process and is matched with a
// receive of the same tag; collectives on one rank copy their input.
#include "mpi.h"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <vector>

namespace {
struct Op {
    bool active = false;
    bool is_send = false;
    bool done = false;
    void* buf = nullptr;
    size_t bytes = 0;
    int tag = 0;
};
std::vector<Op> g_ops;
int g_init = 0;
int g_final = 0;

size_t type_size(MPI_Datatype t)
{
    switch (t) {
    case MPI_CHAR:
    case MPI_BYTE: return 1;
    case MPI_SHORT:
    case MPI_UNSIGNED_SHORT: return 2;
    case MPI_INT:
    case MPI_UNSIGNED:
    case MPI_FLOAT: return 4;
    default: return 8;
    }
}

int new_op(bool is_send, void* buf, size_t bytes, int tag)
{
    for (size_t i = 0; i < g_ops.size(); ++i)
        if (!g_ops[i].active) {
            g_ops[i] = Op{true, is_send, false, buf, bytes, tag};
            return (int)i;
        }
    g_ops.push_back(Op{true, is_send, false, buf, bytes, tag});
    return (int)g_ops.size() - 1;
}

// match pending sends and receives of equal tag, in posting order
void progress()
{
    for (auto& r : g_ops) {
        if (!r.active || r.is_send || r.done) continue;
        for (auto& s : g_ops) {
            if (!s.active || !s.is_send || s.done || s.tag != r.tag) continue;
            size_t b = s.bytes < r.bytes ? s.bytes : r.bytes;
            std::memmove(r.buf, s.buf, b);
            s.done = r.done = true;
            break;
        }
    }
}

int complete(MPI_Request* req, MPI_Status* st)
{
    if (*req == MPI_REQUEST_NULL) return MPI_SUCCESS;
    progress();
    Op& o = g_ops[*req];
    if (!o.done) {
        std::fprintf(stderr, "mpi shim: request %d (tag %d) has no partner on a single rank\n", *req, o.tag);
        std::abort();
    }
    if (st) {
        st->MPI_SOURCE = 0;
        st->MPI_TAG = o.tag;
        st->MPI_ERROR = MPI_SUCCESS;
    }
    o.active = false;
    *req = MPI_REQUEST_NULL;
    return MPI_SUCCESS;
}

void copy_in(const void* s, void* r, int count, MPI_Datatype t)
{
    if (s != MPI_IN_PLACE && s != r) std::memmove(r, s, (size_t)count * type_size(t));
}
}  // namespace

extern "C" {
int MPI_Init(int*, char***) { g_init = 1; g_final = 0; return MPI_SUCCESS; }
int MPI_Initialized(int* flag) { *flag = g_init; return MPI_SUCCESS; }
int MPI_Finalized(int* flag) { *flag = g_final; return MPI_SUCCESS; }
int MPI_Finalize(void) { g_final = 1; g_init = 0; return MPI_SUCCESS; }
int MPI_Abort(MPI_Comm, int code) { std::exit(code); }
double MPI_Wtime(void)
{
    timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}
int MPI_Comm_dup(MPI_Comm c, MPI_Comm* o) { *o = c; return MPI_SUCCESS; }
int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return MPI_SUCCESS; }
int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return MPI_SUCCESS; }
int MPI_Comm_split(MPI_Comm c, int, int, MPI_Comm* o) { *o = c; return MPI_SUCCESS; }
int MPI_Comm_split_type(MPI_Comm c, int, int, MPI_Info, MPI_Comm* o) { *o = c; return MPI_SUCCESS; }
int MPI_Comm_free(MPI_Comm* c) { *c = MPI_COMM_NULL; return MPI_SUCCESS; }
int MPI_Comm_set_errhandler(MPI_Comm, MPI_Errhandler) { return MPI_SUCCESS; }
int MPI_Get_processor_name(char* name, int* len)
{
    std::strcpy(name, "localhost");
    *len = 9;
    return MPI_SUCCESS;
}
int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
int MPI_Isend(const void* buf, int count, MPI_Datatype t, int, int tag, MPI_Comm, MPI_Request* req)
{
    *req = new_op(true, const_cast<void*>(buf), (size_t)count * type_size(t), tag);
    progress();
    return MPI_SUCCESS;
}
int MPI_Irecv(void* buf, int count, MPI_Datatype t, int, int tag, MPI_Comm, MPI_Request* req)
{
    *req = new_op(false, buf, (size_t)count * type_size(t), tag);
    progress();
    return MPI_SUCCESS;
}
int MPI_Send(const void* buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm c)
{
    MPI_Request r;
    MPI_Isend(buf, count, t, dest, tag, c, &r);
    return MPI_SUCCESS;  // completes when the matching receive is posted
}
int MPI_Recv(void* buf, int count, MPI_Datatype t, int src, int tag, MPI_Comm c, MPI_Status* st)
{
    MPI_Request r;
    MPI_Irecv(buf, count, t, src, tag, c, &r);
    return complete(&r, st);
}
int MPI_Sendrecv(const void* sbuf, int scount, MPI_Datatype st, int dest, int stag, void* rbuf, int rcount,
                 MPI_Datatype rt, int src, int rtag, MPI_Comm comm, MPI_Status* status)
{
    MPI_Request a, b;
    MPI_Irecv(rbuf, rcount, rt, src, rtag, comm, &b);
    MPI_Isend(sbuf, scount, st, dest, stag, comm, &a);
    complete(&b, status);
    return complete(&a, nullptr);
}
int MPI_Wait(MPI_Request* req, MPI_Status* st) { return complete(req, st); }
int MPI_Waitall(int n, MPI_Request* reqs, MPI_Status* sts)
{
    for (int i = 0; i < n; ++i) complete(&reqs[i], sts ? &sts[i] : nullptr);
    return MPI_SUCCESS;
}
int MPI_Waitany(int n, MPI_Request* reqs, int* index, MPI_Status* st)
{
    progress();
    for (int i = 0; i < n; ++i)
        if (reqs[i] != MPI_REQUEST_NULL && g_ops[reqs[i]].done) {
            *index = i;
            return complete(&reqs[i], st);
        }
    for (int i = 0; i < n; ++i)
        if (reqs[i] != MPI_REQUEST_NULL) {
            *index = i;
            return complete(&reqs[i], st);
        }
    *index = MPI_UNDEFINED;
    return MPI_SUCCESS;
}
int MPI_Allreduce(const void* s, void* r, int count, MPI_Datatype t, MPI_Op, MPI_Comm)
{
    copy_in(s, r, count, t);
    return MPI_SUCCESS;
}
int MPI_Reduce(const void* s, void* r, int count, MPI_Datatype t, MPI_Op, int, MPI_Comm)
{
    copy_in(s, r, count, t);
    return MPI_SUCCESS;
}
int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }
int MPI_Gather(const void* s, int sc, MPI_Datatype st, void* r, int, MPI_Datatype, int, MPI_Comm)
{
    copy_in(s, r, sc, st);
    return MPI_SUCCESS;
}
int MPI_Allgather(const void* s, int sc, MPI_Datatype st, void* r, int, MPI_Datatype, MPI_Comm)
{
    copy_in(s, r, sc, st);
    return MPI_SUCCESS;
}
int MPI_Dist_graph_create_adjacent(MPI_Comm c, int, const int*, const int*, int, const int*, const int*, MPI_Info,
                                   int, MPI_Comm* out)
{
    *out = c;
    return MPI_SUCCESS;
}
int MPI_Dist_graph_neighbors_count(MPI_Comm, int* indeg, int* outdeg, int* weighted)
{
    *indeg = *outdeg = 1;
    *weighted = 0;
    return MPI_SUCCESS;
}
int MPI_Dist_graph_neighbors(MPI_Comm, int, int* src, int*, int, int* dst, int*)
{
    src[0] = dst[0] = 0;
    return MPI_SUCCESS;
}
int MPI_Neighbor_alltoall(const void* s, int sc, MPI_Datatype st, void* r, int, MPI_Datatype, MPI_Comm)
{
    copy_in(s, r, sc, st);
    return MPI_SUCCESS;
}
int MPI_Ineighbor_alltoall(const void* s, int sc, MPI_Datatype st, void* r, int, MPI_Datatype, MPI_Comm,
                           MPI_Request* req)
{
    copy_in(s, r, sc, st);
    *req = MPI_REQUEST_NULL;
    return MPI_SUCCESS;
}
int MPI_Neighbor_alltoallv(const void* s, const int* sc, const int* sd, MPI_Datatype st, void* r, const int*,
                           const int* rd, MPI_Datatype, MPI_Comm)
{
    size_t ts = type_size(st);
    std::memmove((char*)r + (size_t)rd[0] * ts, (const char*)s + (size_t)sd[0] * ts, (size_t)sc[0] * ts);
    return MPI_SUCCESS;
}
}
