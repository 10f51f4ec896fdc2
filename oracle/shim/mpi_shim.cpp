// Single-rank MPI stand-in (test infrastructure for the CPU oracle).
// Collectives over one rank are copies; Isend/Irecv pairs are matched by tag
// when the receive is posted or at Wait time.
#include "mpi.h"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

namespace
{
size_t type_size(MPI_Datatype dt)
{
    switch (dt)
    {
    case MPI_BYTE:
    case MPI_CHAR:
        return 1;
    case MPI_INT:
        return sizeof(int);
    case MPI_DOUBLE:
        return sizeof(double);
    case MPI_LONG_LONG:
    case MPI_INT64_T:
        return 8;
    default:
        std::fprintf(stderr, "[mpi shim] unknown datatype %d\n", dt);
        std::abort();
    }
}

struct Message
{
    int tag;
    std::vector<char> bytes;
    bool consumed;
};

struct PendingRecv
{
    int tag;
    void *buf;
    size_t cap;
    bool done;
};

std::vector<Message> g_msgs;
std::vector<PendingRecv> g_recvs;

bool try_match(PendingRecv &r)
{
    for (auto &m : g_msgs)
    {
        if (!m.consumed && m.tag == r.tag)
        {
            if (m.bytes.size() > r.cap)
            {
                std::fprintf(stderr, "[mpi shim] message larger than receive buffer (tag %d)\n", r.tag);
                std::abort();
            }
            std::memcpy(r.buf, m.bytes.data(), m.bytes.size());
            m.consumed = true;
            r.done = true;
            return true;
        }
    }
    return false;
}
} // namespace

extern "C" {

int MPI_Init(int *, char ***) { return MPI_SUCCESS; }
int MPI_Initialized(int *flag)
{
    *flag = 1;
    return MPI_SUCCESS;
}
int MPI_Finalize(void) { return MPI_SUCCESS; }
int MPI_Comm_rank(MPI_Comm, int *rank)
{
    *rank = 0;
    return MPI_SUCCESS;
}
int MPI_Comm_size(MPI_Comm, int *size)
{
    *size = 1;
    return MPI_SUCCESS;
}
int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
int MPI_Abort(MPI_Comm, int code)
{
    std::exit(code);
}
double MPI_Wtime(void)
{
    using clk = std::chrono::steady_clock;
    return std::chrono::duration<double>(clk::now().time_since_epoch()).count();
}

int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype dt, MPI_Op, MPI_Comm)
{
    if (sendbuf != recvbuf)
        std::memmove(recvbuf, sendbuf, size_t(count) * type_size(dt));
    return MPI_SUCCESS;
}
int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }
int MPI_Gather(const void *sendbuf, int scount, MPI_Datatype sdt, void *recvbuf, int, MPI_Datatype, int, MPI_Comm)
{
    std::memmove(recvbuf, sendbuf, size_t(scount) * type_size(sdt));
    return MPI_SUCCESS;
}
int MPI_Allgather(const void *sendbuf, int scount, MPI_Datatype sdt, void *recvbuf, int, MPI_Datatype, MPI_Comm)
{
    std::memmove(recvbuf, sendbuf, size_t(scount) * type_size(sdt));
    return MPI_SUCCESS;
}
int MPI_Allgatherv(const void *sendbuf, int scount, MPI_Datatype sdt, void *recvbuf, const int *,
                   const int *displs, MPI_Datatype rdt, MPI_Comm)
{
    std::memmove(static_cast<char *>(recvbuf) + size_t(displs[0]) * type_size(rdt), sendbuf,
                 size_t(scount) * type_size(sdt));
    return MPI_SUCCESS;
}
int MPI_Alltoall(const void *sendbuf, int scount, MPI_Datatype sdt, void *recvbuf, int, MPI_Datatype, MPI_Comm)
{
    std::memmove(recvbuf, sendbuf, size_t(scount) * type_size(sdt));
    return MPI_SUCCESS;
}
int MPI_Alltoallv(const void *sendbuf, const int *scounts, const int *sdispls, MPI_Datatype sdt, void *recvbuf,
                  const int *, const int *rdispls, MPI_Datatype rdt, MPI_Comm)
{
    const size_t ss = type_size(sdt), rs = type_size(rdt);
    if (scounts[0] > 0)
        std::memmove(static_cast<char *>(recvbuf) + size_t(rdispls[0]) * rs,
                     static_cast<const char *>(sendbuf) + size_t(sdispls[0]) * ss, size_t(scounts[0]) * ss);
    return MPI_SUCCESS;
}

int MPI_Isend(const void *buf, int count, MPI_Datatype dt, int, int tag, MPI_Comm, MPI_Request *req)
{
    Message m;
    m.tag = tag;
    m.consumed = false;
    const size_t n = size_t(count) * type_size(dt);
    m.bytes.assign(static_cast<const char *>(buf), static_cast<const char *>(buf) + n);
    g_msgs.push_back(std::move(m));
    *req = MPI_REQUEST_NULL;
    return MPI_SUCCESS;
}
int MPI_Irecv(void *buf, int count, MPI_Datatype dt, int, int tag, MPI_Comm, MPI_Request *req)
{
    PendingRecv r{tag, buf, size_t(count) * type_size(dt), false};
    try_match(r);
    g_recvs.push_back(r);
    *req = int(g_recvs.size() - 1);
    return MPI_SUCCESS;
}
int MPI_Wait(MPI_Request *req, MPI_Status *)
{
    if (*req >= 0 && size_t(*req) < g_recvs.size())
    {
        PendingRecv &r = g_recvs[size_t(*req)];
        if (!r.done && !try_match(r))
        {
            std::fprintf(stderr, "[mpi shim] receive with tag %d has no matching send\n", r.tag);
            std::abort();
        }
    }
    *req = MPI_REQUEST_NULL;
    return MPI_SUCCESS;
}
int MPI_Waitall(int count, MPI_Request *reqs, MPI_Status *)
{
    for (int i = 0; i < count; ++i)
        MPI_Wait(&reqs[i], nullptr);
    bool all_done = true;
    for (auto &r : g_recvs)
        all_done = all_done && r.done;
    if (all_done)
    {
        g_recvs.clear();
        g_msgs.clear();
    }
    return MPI_SUCCESS;
}

} // extern "C"
