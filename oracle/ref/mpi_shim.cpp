// Single-rank MPI stand-in (see mpi.h).  TEST INFRASTRUCTURE ONLY.
#include "mpi.h"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <vector>

namespace {
struct Pending {
    bool is_recv = false;
    bool done = true;
    int tag = 0;
    void *buf = nullptr;
    size_t bytes = 0;
};
std::vector<Pending> g_requests;
std::multimap<int, std::vector<char>> g_mailbox;  // tag -> payload

size_t type_size(MPI_Datatype t) { return t == MPI_DOUBLE ? sizeof(double) : sizeof(int); }
}  // namespace

int MPI_Init(int *, char ***) { return MPI_SUCCESS; }
int MPI_Finalize() { return MPI_SUCCESS; }
int MPI_Abort(MPI_Comm, int code) {
    std::fprintf(stderr, "single-rank MPI stand-in: MPI_Abort(%d)\n", code);
    std::exit(code);
}
int MPI_Comm_rank(MPI_Comm, int *rank) { *rank = 0; return MPI_SUCCESS; }
int MPI_Comm_size(MPI_Comm, int *size) { *size = 1; return MPI_SUCCESS; }
int MPI_Comm_free(MPI_Comm *) { return MPI_SUCCESS; }
int MPI_Comm_split(MPI_Comm, int, int, MPI_Comm *c) { *c = 0; return MPI_SUCCESS; }
int MPI_Cart_create(MPI_Comm, int, const int *, const int *, int, MPI_Comm *c) {
    *c = 0;
    return MPI_SUCCESS;
}
int MPI_Cart_coords(MPI_Comm, int, int maxdims, int *coords) {
    for (int d = 0; d < maxdims; ++d) coords[d] = 0;
    return MPI_SUCCESS;
}
int MPI_Cart_shift(MPI_Comm, int, int, int *src, int *dst) {
    *src = 0;  // periodic extent-1 dimension: both neighbours are this rank
    *dst = 0;
    return MPI_SUCCESS;
}
int MPI_Isend(const void *buf, int count, MPI_Datatype type, int, int tag, MPI_Comm,
              MPI_Request *req) {
    size_t bytes = type_size(type) * static_cast<size_t>(count);
    std::vector<char> payload(bytes);
    std::memcpy(payload.data(), buf, bytes);
    g_mailbox.emplace(tag, std::move(payload));
    Pending p;
    p.tag = tag;
    g_requests.push_back(p);
    *req = static_cast<int>(g_requests.size() - 1);
    return MPI_SUCCESS;
}
int MPI_Irecv(void *buf, int count, MPI_Datatype type, int, int tag, MPI_Comm,
              MPI_Request *req) {
    Pending p;
    p.is_recv = true;
    p.done = false;
    p.tag = tag;
    p.buf = buf;
    p.bytes = type_size(type) * static_cast<size_t>(count);
    g_requests.push_back(p);
    *req = static_cast<int>(g_requests.size() - 1);
    return MPI_SUCCESS;
}
int MPI_Wait(MPI_Request *req, MPI_Status *) {
    Pending &p = g_requests.at(static_cast<size_t>(*req));
    if (p.is_recv && !p.done) {
        auto it = g_mailbox.find(p.tag);
        if (it == g_mailbox.end()) {
            std::fprintf(stderr, "single-rank MPI stand-in: no message for tag %d\n", p.tag);
            std::exit(97);
        }
        if (it->second.size() != p.bytes) {
            std::fprintf(stderr, "single-rank MPI stand-in: size mismatch for tag %d\n", p.tag);
            std::exit(98);
        }
        std::memcpy(p.buf, it->second.data(), p.bytes);
        g_mailbox.erase(it);
        p.done = true;
    }
    // Requests are never reused by the reference after Wait; recycle the table
    // once every request has completed so it does not grow without bound.
    bool all_done = true;
    for (const Pending &q : g_requests) all_done = all_done && q.done;
    if (all_done) g_requests.clear();
    return MPI_SUCCESS;
}
int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype type, MPI_Op,
                  MPI_Comm) {
    std::memmove(recvbuf, sendbuf, type_size(type) * static_cast<size_t>(count));
    return MPI_SUCCESS;
}
int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
double MPI_Wtime() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}
