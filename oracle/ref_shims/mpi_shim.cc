/* Single-rank MPI implementation for the CPU oracle build (test infrastructure).
 * Messages to self are queued per tag at send time and matched at wait time. */
#include "mpi.h"
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <deque>
#include <map>
#include <vector>

namespace {

struct message {
    int tag;
    std::vector<char> bytes;
};

struct pending_recv {
    void *buf;
    size_t max_bytes;
    int tag;
    bool done;
};

std::deque<message> g_outbox;
std::map<int, pending_recv> g_recvs;
int g_next_req = 1;
int g_custom_type_size = 0;

size_t type_size(MPI_Datatype dt) {
    if (dt == MPI_DOUBLE_INT) return sizeof(double) + sizeof(int) + 4;
    if (dt > 0 && dt <= 16) return (size_t)dt;
    if (dt == 4096) return (size_t)g_custom_type_size;
    return 1;
}

bool deliver(pending_recv &r) {
    for (auto it = g_outbox.begin(); it != g_outbox.end(); ++it) {
        if (it->tag == r.tag) {
            size_t n = it->bytes.size();
            if (n > r.max_bytes) {
                fprintf(stderr, "mpi shim: message of %zu bytes for a %zu-byte buffer (tag %d)\n",
                        n, r.max_bytes, r.tag);
                abort();
            }
            if (n) memcpy(r.buf, it->bytes.data(), n);
            g_outbox.erase(it);
            r.done = true;
            return true;
        }
    }
    return false;
}

void finish(MPI_Request *req) {
    if (req == nullptr || *req <= 0) return;
    auto it = g_recvs.find(*req);
    if (it != g_recvs.end()) {
        if (!it->second.done && !deliver(it->second)) {
            fprintf(stderr, "mpi shim: receive with tag %d has no matching self-message\n",
                    it->second.tag);
            abort();
        }
        g_recvs.erase(it);
    }
    *req = MPI_REQUEST_NULL;
}

}  // namespace

int MPI_Init(int *, char ***) { return MPI_SUCCESS; }
int MPI_Finalize() { return MPI_SUCCESS; }
int MPI_Abort(MPI_Comm, int code) { exit(code == 0 ? 1 : code); }
int MPI_Comm_rank(MPI_Comm, int *rank) { *rank = 0; return MPI_SUCCESS; }
int MPI_Comm_size(MPI_Comm, int *size) { *size = 1; return MPI_SUCCESS; }
double MPI_Wtime() {
    timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}
int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }
int MPI_Allreduce(const void *s, void *r, int count, MPI_Datatype dt, MPI_Op, MPI_Comm) {
    if (s != r) memmove(r, s, count * type_size(dt));
    return MPI_SUCCESS;
}
int MPI_Reduce(const void *s, void *r, int count, MPI_Datatype dt, MPI_Op op, int, MPI_Comm c) {
    return MPI_Allreduce(s, r, count, dt, op, c);
}
int MPI_Isend(const void *buf, int count, MPI_Datatype dt, int, int tag, MPI_Comm, MPI_Request *req) {
    message m;
    m.tag = tag;
    size_t n = count * type_size(dt);
    m.bytes.resize(n);
    if (n) memcpy(m.bytes.data(), buf, n);
    g_outbox.push_back(std::move(m));
    if (req) *req = MPI_REQUEST_NULL;
    return MPI_SUCCESS;
}
int MPI_Send(const void *buf, int count, MPI_Datatype dt, int dest, int tag, MPI_Comm c) {
    return MPI_Isend(buf, count, dt, dest, tag, c, nullptr);
}
int MPI_Irecv(void *buf, int count, MPI_Datatype dt, int, int tag, MPI_Comm, MPI_Request *req) {
    int id = g_next_req++;
    g_recvs[id] = pending_recv{buf, count * type_size(dt), tag, false};
    *req = id;
    return MPI_SUCCESS;
}
int MPI_Recv(void *buf, int count, MPI_Datatype dt, int, int tag, MPI_Comm, MPI_Status *) {
    pending_recv r{buf, count * type_size(dt), tag, false};
    if (!deliver(r)) {
        fprintf(stderr, "mpi shim: blocking receive with tag %d has no matching self-message\n", tag);
        abort();
    }
    return MPI_SUCCESS;
}
int MPI_Wait(MPI_Request *req, MPI_Status *) { finish(req); return MPI_SUCCESS; }
int MPI_Waitall(int n, MPI_Request *reqs, MPI_Status *) {
    for (int i = 0; i < n; i++) finish(reqs + i);
    return MPI_SUCCESS;
}
int MPI_Cart_rank(MPI_Comm, const int *, int *rank) { *rank = 0; return MPI_SUCCESS; }
int MPI_Cart_create(MPI_Comm, int, const int *, const int *, int, MPI_Comm *cart) { *cart = 0; return MPI_SUCCESS; }
int MPI_Cart_coords(MPI_Comm, int, int maxdims, int *coords) {
    for (int i = 0; i < maxdims; i++) coords[i] = 0;
    return MPI_SUCCESS;
}
int MPI_Dims_create(int, int ndims, int *dims) {
    for (int i = 0; i < ndims; i++) dims[i] = 1;
    return MPI_SUCCESS;
}
int MPI_Type_create_struct(int n, const int *bl, const MPI_Aint *off, const MPI_Datatype *types, MPI_Datatype *nt) {
    size_t end = 0;
    for (int i = 0; i < n; i++) {
        size_t e = off[i] + bl[i] * type_size(types[i]);
        if (e > end) end = e;
    }
    g_custom_type_size = (int)((end + 7) / 8 * 8);
    *nt = 4096;
    return MPI_SUCCESS;
}
int MPI_Type_commit(MPI_Datatype *) { return MPI_SUCCESS; }
int MPI_Type_free(MPI_Datatype *) { return MPI_SUCCESS; }
int MPI_Comm_free(MPI_Comm *) { return MPI_SUCCESS; }
