/* A single-process stand-in for the MPI interface, written for this
 * repository so that the reference's solve phase (which calls MPI through
 * src/comm/detail/mpi_wrapper.inl) can be compiled and run on one rank as a
 * parity pin for the CPU oracle.
 *
 * TEST INFRASTRUCTURE ONLY (oracle/_ref). Semantics of one rank: every
 * communicator has size 1 and rank 0; collectives copy their input to their
 * output; point-to-point messages to oneself are matched by tag, a receive
 * waiting for its send when it is posted first. Only the calls the reference makes exist. */
#ifndef XAMG_REF_SHIM_MPI_H_
#define XAMG_REF_SHIM_MPI_H_

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <vector>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
struct MPI_Status {
    int MPI_SOURCE, MPI_TAG, MPI_ERROR;
    int count_bytes;
};

#define MPI_COMM_NULL (-1)
#define MPI_COMM_WORLD 0
#define MPI_COMM_SELF 1
#define MPI_UNDEFINED (-32766)
#define MPI_ANY_SOURCE (-2)
#define MPI_ANY_TAG (-1)
#define MPI_SUCCESS 0
#define MPI_MAX_PROCESSOR_NAME 256
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)
#define MPI_IN_PLACE ((void *)1)
#define MPI_REQUEST_NULL 0

/* datatypes: the value is the element size in bytes times 16 plus an id */
#define MPI_CHAR (1 * 16 + 1)
#define MPI_UNSIGNED_CHAR (1 * 16 + 2)
#define MPI_BYTE (1 * 16 + 3)
#define MPI_SHORT (2 * 16 + 1)
#define MPI_UNSIGNED_SHORT (2 * 16 + 2)
#define MPI_INT (4 * 16 + 1)
#define MPI_UNSIGNED (4 * 16 + 2)
#define MPI_FLOAT (4 * 16 + 3)
#define MPI_LONG (8 * 16 + 1)
#define MPI_UNSIGNED_LONG (8 * 16 + 2)
#define MPI_DOUBLE (8 * 16 + 3)
#define MPI_LONG_LONG (8 * 16 + 4)

#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3

namespace xamg_ref_shim {
inline size_t type_size(MPI_Datatype t) { return (size_t)(t / 16); }
struct Msg {
    int tag;
    std::vector<char> data;
};
inline std::deque<Msg> &queue() {
    static std::deque<Msg> q;
    return q;
}
inline int &next_comm() {
    static int c = 2;
    return c;
}
inline void copy(const void *in, void *out, int count, MPI_Datatype t) {
    if (in != MPI_IN_PLACE && in != out && count > 0) std::memmove(out, in, count * type_size(t));
}
inline void fail(const char *what) {
    std::fprintf(stderr, "single-process MPI stand-in: %s needs another rank\n", what);
    std::abort();
}
}  // namespace xamg_ref_shim

inline int MPI_Initialized(int *flag) {
    static int init = 0;
    *flag = init;
    init = 1;
    return 0;
}
inline int MPI_Init(int *, char ***) { return 0; }
inline int MPI_Finalized(int *flag) {
    *flag = 0;
    return 0;
}
inline int MPI_Finalize() { return 0; }
inline int MPI_Abort(MPI_Comm, int code) {
    std::fprintf(stderr, "MPI_Abort(%d)\n", code);
    std::abort();
}
inline int MPI_Comm_size(MPI_Comm, int *size) {
    *size = 1;
    return 0;
}
inline int MPI_Comm_rank(MPI_Comm, int *rank) {
    *rank = 0;
    return 0;
}
inline int MPI_Comm_split(MPI_Comm, int color, int, MPI_Comm *out) {
    *out = (color == MPI_UNDEFINED) ? MPI_COMM_NULL : xamg_ref_shim::next_comm()++;
    return 0;
}
inline int MPI_Comm_dup(MPI_Comm, MPI_Comm *out) {
    *out = xamg_ref_shim::next_comm()++;
    return 0;
}
inline int MPI_Comm_free(MPI_Comm *c) {
    *c = MPI_COMM_NULL;
    return 0;
}
inline int MPI_Get_processor_name(char *name, int *len) {
    std::strcpy(name, "localhost");
    *len = 9;
    return 0;
}
inline int MPI_Barrier(MPI_Comm) { return 0; }
inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return 0; }
inline int MPI_Allreduce(const void *in, void *out, int count, MPI_Datatype t, MPI_Op, MPI_Comm) {
    xamg_ref_shim::copy(in, out, count, t);
    return 0;
}
inline int MPI_Iallreduce(const void *in, void *out, int count, MPI_Datatype t, MPI_Op, MPI_Comm,
                          MPI_Request *req) {
    xamg_ref_shim::copy(in, out, count, t);
    *req = MPI_REQUEST_NULL;
    return 0;
}
inline int MPI_Alltoall(const void *in, int count, MPI_Datatype t, void *out, int, MPI_Datatype,
                        MPI_Comm) {
    xamg_ref_shim::copy(in, out, count, t);
    return 0;
}
inline int MPI_Gather(const void *in, int count, MPI_Datatype t, void *out, int, MPI_Datatype,
                      int, MPI_Comm) {
    xamg_ref_shim::copy(in, out, count, t);
    return 0;
}
inline int MPI_Gatherv(const void *in, int count, MPI_Datatype t, void *out, const int *,
                       const int *displs, MPI_Datatype, int, MPI_Comm) {
    xamg_ref_shim::copy(in, (char *)out + (size_t)displs[0] * xamg_ref_shim::type_size(t), count,
                        t);
    return 0;
}
inline int MPI_Allgather(const void *in, int count, MPI_Datatype t, void *out, int, MPI_Datatype,
                         MPI_Comm) {
    xamg_ref_shim::copy(in, out, count, t);
    return 0;
}
inline int MPI_Allgatherv(const void *in, int count, MPI_Datatype t, void *out, const int *,
                          const int *displs, MPI_Datatype, MPI_Comm) {
    xamg_ref_shim::copy(in, (char *)out + (size_t)displs[0] * xamg_ref_shim::type_size(t), count,
                        t);
    return 0;
}
inline int MPI_Scatter(const void *in, int count, MPI_Datatype t, void *out, int, MPI_Datatype, int,
                       MPI_Comm) {
    xamg_ref_shim::copy(in, out, count, t);
    return 0;
}
/* point to point: only messages to oneself exist on one rank. A send is
 * delivered to a posted receive with its tag, or queued; a receive takes a
 * queued message with its tag, or stays posted until one arrives. A request
 * is 0 when complete, else the id of a posted receive. */
namespace xamg_ref_shim {
struct Posted {
    int id, tag;
    void *buf;
    size_t bytes;
};
inline std::deque<Posted> &posted() {
    static std::deque<Posted> p;
    return p;
}
inline int &next_req() {
    static int r = 1;
    return r;
}
inline bool take_queued(int tag, void *buf, size_t bytes, MPI_Status *st) {
    auto &q = queue();
    for (auto it = q.begin(); it != q.end(); ++it)
        if (tag == MPI_ANY_TAG || it->tag == tag) {
            const size_t n = std::min(it->data.size(), bytes);
            if (n) std::memcpy(buf, it->data.data(), n);
            if (st) {
                st->MPI_SOURCE = 0;
                st->MPI_TAG = it->tag;
                st->count_bytes = (int)n;
            }
            q.erase(it);
            return true;
        }
    return false;
}
inline bool pending(int req) {
    for (auto &p : posted())
        if (p.id == req) return true;
    return false;
}
}  // namespace xamg_ref_shim

inline int MPI_Send(const void *buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm) {
    if (dest != 0) xamg_ref_shim::fail("MPI_Send");
    const size_t bytes = count * xamg_ref_shim::type_size(t);
    auto &P = xamg_ref_shim::posted();
    for (auto it = P.begin(); it != P.end(); ++it)
        if (it->tag == tag || it->tag == MPI_ANY_TAG) {
            if (bytes) std::memcpy(it->buf, buf, std::min(bytes, it->bytes));
            P.erase(it);
            return 0;
        }
    const char *p = (const char *)buf;
    xamg_ref_shim::queue().push_back({tag, std::vector<char>(p, p + bytes)});
    return 0;
}
inline int MPI_Isend(const void *buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm c,
                     MPI_Request *req) {
    *req = MPI_REQUEST_NULL;
    return MPI_Send(buf, count, t, dest, tag, c);
}
inline int MPI_Irecv(void *buf, int count, MPI_Datatype t, int src, int tag, MPI_Comm,
                     MPI_Request *req) {
    if (src != 0 && src != MPI_ANY_SOURCE) xamg_ref_shim::fail("MPI_Irecv");
    const size_t bytes = count * xamg_ref_shim::type_size(t);
    if (xamg_ref_shim::take_queued(tag, buf, bytes, MPI_STATUS_IGNORE)) {
        *req = MPI_REQUEST_NULL;
    } else {
        *req = xamg_ref_shim::next_req()++;
        xamg_ref_shim::posted().push_back({*req, tag, buf, bytes});
    }
    return 0;
}
inline int MPI_Recv(void *buf, int count, MPI_Datatype t, int src, int tag, MPI_Comm,
                    MPI_Status *st) {
    if (src != 0 && src != MPI_ANY_SOURCE) xamg_ref_shim::fail("MPI_Recv");
    if (!xamg_ref_shim::take_queued(tag, buf, count * xamg_ref_shim::type_size(t), st))
        xamg_ref_shim::fail("MPI_Recv without a matching send");
    return 0;
}
inline int MPI_Probe(int src, int tag, MPI_Comm, MPI_Status *st) {
    if (src != 0 && src != MPI_ANY_SOURCE) xamg_ref_shim::fail("MPI_Probe");
    for (auto &m : xamg_ref_shim::queue())
        if (tag == MPI_ANY_TAG || m.tag == tag) {
            st->MPI_SOURCE = 0;
            st->MPI_TAG = m.tag;
            st->count_bytes = (int)m.data.size();
            return 0;
        }
    xamg_ref_shim::fail("MPI_Probe without a matching send");
    return 1;
}
inline int MPI_Get_count(const MPI_Status *st, MPI_Datatype t, int *count) {
    *count = st->count_bytes / (int)xamg_ref_shim::type_size(t);
    return 0;
}
inline int MPI_Wait(MPI_Request *req, MPI_Status *) {
    if (*req != MPI_REQUEST_NULL && xamg_ref_shim::pending(*req))
        xamg_ref_shim::fail("MPI_Wait on a receive that no send matches");
    *req = MPI_REQUEST_NULL;
    return 0;
}
inline int MPI_Waitall(int n, MPI_Request *reqs, MPI_Status *) {
    for (int i = 0; i < n; ++i) MPI_Wait(&reqs[i], MPI_STATUS_IGNORE);
    return 0;
}
inline int MPI_Waitany(int n, MPI_Request *reqs, int *idx, MPI_Status *) {
    *idx = MPI_UNDEFINED;
    for (int i = 0; i < n; ++i)
        if (reqs[i] != MPI_REQUEST_NULL) {
            MPI_Wait(&reqs[i], MPI_STATUS_IGNORE);
            *idx = i;
            return 0;
        }
    return 0;
}
inline int MPI_Test(MPI_Request *req, int *flag, MPI_Status *) {
    *flag = !(*req != MPI_REQUEST_NULL && xamg_ref_shim::pending(*req));
    if (*flag) *req = MPI_REQUEST_NULL;
    return 0;
}
inline int MPI_Testall(int n, MPI_Request *reqs, int *flag, MPI_Status *) {
    *flag = 1;
    for (int i = 0; i < n; ++i)
        if (reqs[i] != MPI_REQUEST_NULL && xamg_ref_shim::pending(reqs[i])) *flag = 0;
    if (*flag)
        for (int i = 0; i < n; ++i) reqs[i] = MPI_REQUEST_NULL;
    return 0;
}
inline int MPI_Testany(int n, MPI_Request *reqs, int *idx, int *flag, MPI_Status *) {
    *flag = 1;
    *idx = MPI_UNDEFINED;
    for (int i = 0; i < n; ++i)
        if (reqs[i] != MPI_REQUEST_NULL) {
            if (xamg_ref_shim::pending(reqs[i])) {
                *flag = 0;
                continue;
            }
            reqs[i] = MPI_REQUEST_NULL;
            *idx = i;
            *flag = 1;
            return 0;
        }
    return 0;
}

#endif
