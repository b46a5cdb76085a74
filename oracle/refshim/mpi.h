/* mpi.h -- a one-rank stand-in for the MPI calls the ECMC-QCB hot-path sources make, so those
 * sources compile unchanged into the reference oracle (oracle/_ref).  TEST INFRASTRUCTURE ONLY.
 *
 * Project-written, not an MPI implementation.  There is exactly one rank (rank 0, size 1) and
 * every Cartesian communicator is the periodic 1x1x1x1 grid, so every neighbour is rank 0:
 *   - MPI_Cart_create/coords/shift describe that grid (n_core_dim must be 1);
 *   - MPI_Allreduce and MPI_Reduce copy the send buffer (a sum over one rank);
 *   - MPI_Bcast and MPI_Barrier do nothing;
 *   - MPI_Sendrecv copies the send buffer into the receive buffer;
 *   - MPI_Isend/MPI_Irecv queue their buffers and MPI_Wait/MPI_Waitall pair each receive with the
 *     queued send of the same tag and copy it, which is what a periodic one-rank halo exchange
 *     (a rank sending its faces to itself) needs.
 *   - MPI-IO as the reference's ILDG code uses it: a file view of one rank's whole lattice (a
 *     subarray equal to the full array, the only view one rank can have) is one contiguous range at
 *     the view's displacement, so MPI_File_write_all / read_all are one fwrite / fread there.
 * Anything else (other collectives, other views) is not declared or refused: a source that needs
 * it does not compile or aborts.  Not thread-safe: the reference calls MPI outside its OpenMP
 * regions. */
#ifndef QCB_REFSHIM_MPI_H
#define QCB_REFSHIM_MPI_H

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct {
    int MPI_SOURCE, MPI_TAG, MPI_ERROR;
} MPI_Status;

#define MPI_SUCCESS 0
#define MPI_COMM_WORLD 0
#define MPI_COMM_NULL (-1)
#define MPI_PROC_NULL (-2)
#define MPI_REQUEST_NULL (-1)
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)

/* datatypes carry their size in bytes */
#define MPI_CHAR 1
#define MPI_INT 4
#define MPI_UNSIGNED_LONG 8
#define MPI_DOUBLE 1008
#define MPI_DOUBLE_COMPLEX 1016
#define MPI_C_DOUBLE_COMPLEX 1016

#define MPI_OFFSET 8
#define MPI_DATATYPE_NULL 0
typedef long long MPI_Offset;
typedef int MPI_Info;
#define MPI_INFO_NULL 0
#define MPI_MODE_RDONLY 2
#define MPI_MODE_WRONLY 4
#define MPI_ORDER_C 56
struct qcb_mpi_file_s {
    FILE* fp;
    MPI_Offset disp;
};
typedef qcb_mpi_file_s* MPI_File;

#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPI_LAND 4

namespace qcb_mpi_stub {
// derived datatypes (ids from kDerived): their size in bytes
constexpr int kDerived = 1 << 20;
inline std::vector<size_t>& derived_sizes() {
    static std::vector<size_t> v;
    return v;
}
inline size_t type_size(MPI_Datatype t) {
    if (t >= kDerived) return derived_sizes()[(size_t)(t - kDerived)];
    return (size_t)(t >= 1000 ? t - 1000 : t);
}
inline MPI_Datatype new_type(size_t bytes) {
    derived_sizes().push_back(bytes);
    return kDerived + (int)derived_sizes().size() - 1;
}

[[noreturn]] inline void fail(const char* what) {
    std::fprintf(stderr, "one-rank MPI stand-in: %s\n", what);
    std::abort();
}

struct Pending {
    const void* send;
    void* recv;
    size_t bytes;
    int tag;
};
inline std::vector<Pending>& sends() {
    static std::vector<Pending> v;
    return v;
}
inline std::vector<Pending>& recvs() {
    static std::vector<Pending> v;
    return v;
}
inline void check_peer(int peer) {
    if (peer != 0) fail("message to or from a rank other than 0");
}
}  // namespace qcb_mpi_stub

inline int MPI_Comm_rank(MPI_Comm, int* rank) {
    *rank = 0;
    return MPI_SUCCESS;
}
inline int MPI_Comm_size(MPI_Comm, int* size) {
    *size = 1;
    return MPI_SUCCESS;
}
inline int MPI_Cart_create(MPI_Comm comm, int ndims, const int* dims, const int*, int, MPI_Comm* cart) {
    for (int d = 0; d < ndims; d++)
        if (dims[d] != 1) qcb_mpi_stub::fail("a Cartesian grid larger than one rank");
    *cart = comm;
    return MPI_SUCCESS;
}
inline int MPI_Cart_coords(MPI_Comm, int, int maxdims, int* coords) {
    for (int d = 0; d < maxdims; d++) coords[d] = 0;
    return MPI_SUCCESS;
}
inline int MPI_Cart_shift(MPI_Comm, int, int, int* source, int* dest) {
    *source = 0;
    *dest = 0;
    return MPI_SUCCESS;
}
inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
inline int MPI_Bcast(void*, int, MPI_Datatype, int root, MPI_Comm) {
    qcb_mpi_stub::check_peer(root);
    return MPI_SUCCESS;
}
inline int MPI_Allreduce(const void* send, void* recv, int count, MPI_Datatype t, MPI_Op, MPI_Comm) {
    std::memmove(recv, send, (size_t)count * qcb_mpi_stub::type_size(t));
    return MPI_SUCCESS;
}
inline int MPI_Reduce(const void* send, void* recv, int count, MPI_Datatype t, MPI_Op, int root, MPI_Comm) {
    qcb_mpi_stub::check_peer(root);
    std::memmove(recv, send, (size_t)count * qcb_mpi_stub::type_size(t));
    return MPI_SUCCESS;
}
inline int MPI_Sendrecv(const void* send, int scount, MPI_Datatype stype, int dest, int stag, void* recv, int rcount,
                        MPI_Datatype rtype, int source, int rtag, MPI_Comm, MPI_Status*) {
    qcb_mpi_stub::check_peer(dest);
    qcb_mpi_stub::check_peer(source);
    size_t sb = (size_t)scount * qcb_mpi_stub::type_size(stype), rb = (size_t)rcount * qcb_mpi_stub::type_size(rtype);
    if (stag != rtag || sb != rb) qcb_mpi_stub::fail("MPI_Sendrecv to self with unmatched tag or size");
    std::memmove(recv, send, sb);
    return MPI_SUCCESS;
}
inline int MPI_Isend(const void* buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm, MPI_Request* req) {
    qcb_mpi_stub::check_peer(dest);
    qcb_mpi_stub::sends().push_back({buf, nullptr, (size_t)count * qcb_mpi_stub::type_size(t), tag});
    *req = 0;
    return MPI_SUCCESS;
}
inline int MPI_Irecv(void* buf, int count, MPI_Datatype t, int source, int tag, MPI_Comm, MPI_Request* req) {
    qcb_mpi_stub::check_peer(source);
    qcb_mpi_stub::recvs().push_back({nullptr, buf, (size_t)count * qcb_mpi_stub::type_size(t), tag});
    *req = 0;
    return MPI_SUCCESS;
}
/* Completes every queued message: each receive takes the first queued send of its tag. */
inline int MPI_Waitall(int, MPI_Request*, MPI_Status*) {
    auto& S = qcb_mpi_stub::sends();
    auto& R = qcb_mpi_stub::recvs();
    for (auto& r : R) {
        bool found = false;
        for (size_t k = 0; k < S.size(); k++) {
            if (S[k].tag != r.tag) continue;
            if (S[k].bytes != r.bytes) qcb_mpi_stub::fail("send and receive of one tag differ in size");
            std::memmove(r.recv, S[k].send, r.bytes);
            S.erase(S.begin() + (long)k);
            found = true;
            break;
        }
        if (!found) qcb_mpi_stub::fail("a receive with no matching send");
    }
    R.clear();
    if (!S.empty()) qcb_mpi_stub::fail("a send with no matching receive");
    return MPI_SUCCESS;
}
inline int MPI_Wait(MPI_Request* req, MPI_Status* st) { return MPI_Waitall(1, req, st); }
inline int MPI_Type_contiguous(int count, MPI_Datatype old, MPI_Datatype* t) {
    *t = qcb_mpi_stub::new_type((size_t)count * qcb_mpi_stub::type_size(old));
    return MPI_SUCCESS;
}
inline int MPI_Type_commit(MPI_Datatype*) { return MPI_SUCCESS; }
inline int MPI_Type_free(MPI_Datatype* t) {
    *t = MPI_DATATYPE_NULL;
    return MPI_SUCCESS;
}
inline int MPI_Type_create_subarray(int ndims, const int* sizes, const int* subsizes, const int* starts, int,
                                    MPI_Datatype old, MPI_Datatype* t) {
    size_t n = 1;
    for (int d = 0; d < ndims; d++) {
        if (subsizes[d] != sizes[d] || starts[d] != 0) qcb_mpi_stub::fail("a subarray other than the whole array");
        n *= (size_t)sizes[d];
    }
    *t = qcb_mpi_stub::new_type(n * qcb_mpi_stub::type_size(old));
    return MPI_SUCCESS;
}
inline int MPI_File_open(MPI_Comm, const char* path, int amode, MPI_Info, MPI_File* fh) {
    FILE* fp = std::fopen(path, (amode & MPI_MODE_WRONLY) ? "r+b" : "rb");
    if (!fp) return 1;
    *fh = new qcb_mpi_file_s{fp, 0};
    return MPI_SUCCESS;
}
inline int MPI_File_set_view(MPI_File fh, MPI_Offset disp, MPI_Datatype, MPI_Datatype, const char*, MPI_Info) {
    fh->disp = disp;
    return MPI_SUCCESS;
}
inline int MPI_File_write_all(MPI_File fh, const void* buf, int count, MPI_Datatype t, MPI_Status*) {
    const size_t n = (size_t)count * qcb_mpi_stub::type_size(t);
    if (fseeko(fh->fp, (off_t)fh->disp, SEEK_SET) || std::fwrite(buf, 1, n, fh->fp) != n)
        qcb_mpi_stub::fail("MPI_File_write_all");
    return MPI_SUCCESS;
}
inline int MPI_File_read_all(MPI_File fh, void* buf, int count, MPI_Datatype t, MPI_Status*) {
    const size_t n = (size_t)count * qcb_mpi_stub::type_size(t);
    if (fseeko(fh->fp, (off_t)fh->disp, SEEK_SET) || std::fread(buf, 1, n, fh->fp) != n)
        qcb_mpi_stub::fail("MPI_File_read_all");
    return MPI_SUCCESS;
}
inline int MPI_File_close(MPI_File* fh) {
    std::fclose((*fh)->fp);
    delete *fh;
    *fh = nullptr;
    return MPI_SUCCESS;
}
inline int MPI_Abort(MPI_Comm, int code) {
    std::fprintf(stderr, "MPI_Abort(%d)\n", code);
    std::exit(code);
}

#endif
