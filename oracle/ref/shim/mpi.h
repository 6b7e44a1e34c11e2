// Single-process stand-in for the part of MPI that GHEX's set-up code calls — test
// infrastructure for compiling and running the reference's own pattern and exchange code on the
// CPU as an oracle. There is one rank: collectives copy the caller's contribution, and messages a
// rank sends to itself wait in a mailbox until a receive with the same (source, tag) takes them.
#pragma once

#include <cstddef>
#include <cstring>
#include <deque>
#include <mutex>
#include <vector>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;

struct MPI_Status
{
    int MPI_SOURCE;
    int MPI_TAG;
    int MPI_ERROR;
    int count; // bytes received
};

struct ghexref_mpi_request
{
    bool is_recv;
    void* buf;
    std::size_t capacity;
    int source;
    int tag;
    bool done;
    MPI_Status status;
};
typedef ghexref_mpi_request* MPI_Request;

#define MPI_SUCCESS 0
#define MPI_ERR_OTHER 15
#define MPI_COMM_WORLD 0
#define MPI_COMM_NULL (-1)
#define MPI_BYTE 1
#define MPI_CHAR 2
#define MPI_INT 3
#define MPI_UNSIGNED 4
#define MPI_LONG 5
#define MPI_UNSIGNED_LONG 6
#define MPI_LONG_LONG 7
#define MPI_UNSIGNED_LONG_LONG 8
#define MPI_FLOAT 9
#define MPI_DOUBLE 10
#define MPI_MAX 1
#define MPI_MIN 2
#define MPI_SUM 3
#define MPI_ANY_SOURCE (-1)
#define MPI_ANY_TAG (-1)
#define MPI_REQUEST_NULL ((MPI_Request)0)
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)
#define MPI_IN_PLACE ((void*)1)
#define MPI_THREAD_SINGLE 0
#define MPI_THREAD_FUNNELED 1
#define MPI_THREAD_SERIALIZED 2
#define MPI_THREAD_MULTIPLE 3

inline std::size_t ghexref_mpi_size(MPI_Datatype t)
{
    switch (t)
    {
        case MPI_BYTE:
        case MPI_CHAR: return 1;
        case MPI_INT:
        case MPI_UNSIGNED:
        case MPI_FLOAT: return 4;
        default: return 8;
    }
}

struct ghexref_mpi_message
{
    int source;
    int tag;
    std::vector<char> data;
};

inline std::mutex& ghexref_mpi_mutex()
{
    static std::mutex m;
    return m;
}
inline std::deque<ghexref_mpi_message>& ghexref_mpi_mailbox()
{
    static std::deque<ghexref_mpi_message> box;
    return box;
}

// takes the first queued message matching (source, tag); false if there is none
inline bool ghexref_mpi_take(void* buf, std::size_t capacity, int source, int tag, MPI_Status* st)
{
    std::lock_guard<std::mutex> lock(ghexref_mpi_mutex());
    auto& box = ghexref_mpi_mailbox();
    for (auto it = box.begin(); it != box.end(); ++it)
    {
        if ((source == MPI_ANY_SOURCE || it->source == source) && (tag == MPI_ANY_TAG || it->tag == tag))
        {
            const std::size_t n = it->data.size() < capacity ? it->data.size() : capacity;
            if (n) std::memcpy(buf, it->data.data(), n);
            if (st) *st = MPI_Status{it->source, it->tag, MPI_SUCCESS, (int)n};
            box.erase(it);
            return true;
        }
    }
    return false;
}

inline int MPI_Init(int*, char***) { return MPI_SUCCESS; }
inline int MPI_Init_thread(int*, char***, int, int* provided)
{
    *provided = MPI_THREAD_MULTIPLE;
    return MPI_SUCCESS;
}
inline int MPI_Finalize() { return MPI_SUCCESS; }
inline int MPI_Initialized(int* f)
{
    *f = 1;
    return MPI_SUCCESS;
}
inline int MPI_Finalized(int* f)
{
    *f = 0;
    return MPI_SUCCESS;
}
inline int MPI_Query_thread(int* p)
{
    *p = MPI_THREAD_MULTIPLE;
    return MPI_SUCCESS;
}
inline int MPI_Comm_rank(MPI_Comm, int* r)
{
    *r = 0;
    return MPI_SUCCESS;
}
inline int MPI_Comm_size(MPI_Comm, int* s)
{
    *s = 1;
    return MPI_SUCCESS;
}
inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
inline int MPI_Abort(MPI_Comm, int) { return MPI_SUCCESS; }

inline int MPI_Send(const void* buf, int count, MPI_Datatype t, int /*dest*/, int tag, MPI_Comm)
{
    const std::size_t n = (std::size_t)count * ghexref_mpi_size(t);
    ghexref_mpi_message m{0, tag, std::vector<char>(n)};
    if (n) std::memcpy(m.data.data(), buf, n);
    std::lock_guard<std::mutex> lock(ghexref_mpi_mutex());
    ghexref_mpi_mailbox().push_back(std::move(m));
    return MPI_SUCCESS;
}
inline int MPI_Recv(void* buf, int count, MPI_Datatype t, int source, int tag, MPI_Comm, MPI_Status* st)
{
    // a receive nothing was sent for would block forever in MPI; here it is an error
    return ghexref_mpi_take(buf, (std::size_t)count * ghexref_mpi_size(t), source, tag, st) ? MPI_SUCCESS
                                                                                             : MPI_ERR_OTHER;
}
inline int MPI_Isend(const void* buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm c, MPI_Request* r)
{
    const int e = MPI_Send(buf, count, t, dest, tag, c);
    *r = MPI_REQUEST_NULL;
    return e;
}
inline int MPI_Irecv(void* buf, int count, MPI_Datatype t, int source, int tag, MPI_Comm, MPI_Request* r)
{
    *r = new ghexref_mpi_request{true, buf, (std::size_t)count * ghexref_mpi_size(t), source, tag, false, MPI_Status{}};
    return MPI_SUCCESS;
}
inline int MPI_Test(MPI_Request* r, int* flag, MPI_Status* st)
{
    if (*r == MPI_REQUEST_NULL)
    {
        *flag = 1;
        return MPI_SUCCESS;
    }
    if (!(*r)->done) (*r)->done = ghexref_mpi_take((*r)->buf, (*r)->capacity, (*r)->source, (*r)->tag, &(*r)->status);
    *flag = (*r)->done ? 1 : 0;
    if ((*r)->done)
    {
        if (st) *st = (*r)->status;
        delete *r;
        *r = MPI_REQUEST_NULL;
    }
    return MPI_SUCCESS;
}
inline int MPI_Wait(MPI_Request* r, MPI_Status* st)
{
    int flag = 0;
    MPI_Test(r, &flag, st);
    return flag ? MPI_SUCCESS : MPI_ERR_OTHER;
}
inline int MPI_Waitall(int n, MPI_Request* r, MPI_Status* st)
{
    int e = MPI_SUCCESS;
    for (int i = 0; i < n; ++i)
        if (MPI_Wait(&r[i], st ? &st[i] : MPI_STATUS_IGNORE) != MPI_SUCCESS) e = MPI_ERR_OTHER;
    return e;
}
inline int MPI_Test_cancelled(const MPI_Status*, int* flag)
{
    *flag = 0;
    return MPI_SUCCESS;
}
inline int MPI_Get_count(const MPI_Status* st, MPI_Datatype t, int* count)
{
    *count = st->count / (int)ghexref_mpi_size(t);
    return MPI_SUCCESS;
}
inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }
inline int MPI_Allgather(const void* sb, int sc, MPI_Datatype st, void* rb, int, MPI_Datatype, MPI_Comm)
{
    std::memcpy(rb, sb, (std::size_t)sc * ghexref_mpi_size(st));
    return MPI_SUCCESS;
}
inline int MPI_Iallgather(const void* sb, int sc, MPI_Datatype st, void* rb, int rc, MPI_Datatype rt, MPI_Comm c,
    MPI_Request* r)
{
    *r = MPI_REQUEST_NULL;
    return MPI_Allgather(sb, sc, st, rb, rc, rt, c);
}
inline int MPI_Iallgatherv(const void* sb, int sc, MPI_Datatype st, void* rb, const int*, const int* displs,
    MPI_Datatype rt, MPI_Comm, MPI_Request* r)
{
    *r = MPI_REQUEST_NULL;
    std::memcpy((char*)rb + (std::size_t)displs[0] * ghexref_mpi_size(rt), sb, (std::size_t)sc * ghexref_mpi_size(st));
    return MPI_SUCCESS;
}
inline int MPI_Allreduce(const void* sb, void* rb, int count, MPI_Datatype t, MPI_Op, MPI_Comm)
{
    if (sb != MPI_IN_PLACE) std::memcpy(rb, sb, (std::size_t)count * ghexref_mpi_size(t));
    return MPI_SUCCESS;
}
inline int MPI_Reduce(const void* sb, void* rb, int count, MPI_Datatype t, MPI_Op op, int, MPI_Comm c)
{
    return MPI_Allreduce(sb, rb, count, t, op, c);
}
inline int MPI_Alltoall(const void* sb, int sc, MPI_Datatype st, void* rb, int, MPI_Datatype, MPI_Comm)
{
    std::memcpy(rb, sb, (std::size_t)sc * ghexref_mpi_size(st));
    return MPI_SUCCESS;
}
inline int MPI_Alltoallv(const void* sb, const int* sc, const int* sd, MPI_Datatype st, void* rb, const int*,
    const int* rd, MPI_Datatype rt, MPI_Comm)
{
    std::memcpy((char*)rb + (std::size_t)rd[0] * ghexref_mpi_size(rt), (const char*)sb + (std::size_t)sd[0] * ghexref_mpi_size(st),
        (std::size_t)sc[0] * ghexref_mpi_size(st));
    return MPI_SUCCESS;
}
