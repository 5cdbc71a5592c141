/*
 * Single-rank MPI shim -- TEST INFRASTRUCTURE ONLY.
 *
 * MPI is not installed on the build or GPU hosts.  The reference programs
 * (e.g. 06_transient_localization_dx1.cpp) include <mpi.h> and call a small
 * set of MPI routines.  This header implements exactly those routines with the
 * semantics of a real MPI job of size 1, so the reference sources compile and
 * run unmodified inside the oracle harness (ref_harness.cpp):
 *
 *   - MPI_Comm_size -> 1, MPI_Comm_rank -> 0, MPI_Dims_create -> {1,1,1}.
 *   - MPI_Cart_shift returns MPI_PROC_NULL on non-periodic dimensions (the
 *     family-B programs use periods {0,0,0}, 06:338) and rank 0 itself on
 *     periodic ones (family A, 01:107).
 *   - Point-to-point with MPI_PROC_NULL completes immediately and leaves the
 *     receive buffer untouched (MPI standard, section 3.11).  Self messages are
 *     matched by tag at MPI_Waitall.
 *   - Reduce/Allreduce copy the send buffer (one contributor).
 *
 * Nothing in the product library includes this file.
 */
#ifndef ORACLE_MPI_SHIM_H
#define ORACLE_MPI_SHIM_H

#include <cstddef>
#include <cstring>
#include <vector>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;
typedef int MPI_Request;

#define MPI_SUCCESS 0
#define MPI_COMM_NULL (-1)
#define MPI_COMM_WORLD 0
#define MPI_PROC_NULL (-2)
#define MPI_DOUBLE 8
#define MPI_FLOAT 4
#define MPI_INT 5
#define MPI_SUM 1
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)

namespace oracle_mpi_shim {
inline int& cart_periodic(int d) { static int p[3] = {0, 0, 0}; return p[d]; }
inline size_t type_size(MPI_Datatype t) { return t == MPI_DOUBLE ? 8 : 4; }
struct Pending { int kind; void* buf; size_t bytes; int tag; std::vector<char> data; };
inline std::vector<Pending>& pending() { static std::vector<Pending> v; return v; }
}  // namespace oracle_mpi_shim

static inline int MPI_Init(int*, char***) { return MPI_SUCCESS; }
static inline int MPI_Finalize() { return MPI_SUCCESS; }
static inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return MPI_SUCCESS; }
static inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
static inline int MPI_Dims_create(int, int nd, int* dims)
{
    for (int d = 0; d < nd; ++d) dims[d] = 1;
    return MPI_SUCCESS;
}
static inline int MPI_Cart_create(MPI_Comm, int nd, const int*, const int* periods, int, MPI_Comm* c)
{
    for (int d = 0; d < nd && d < 3; ++d) oracle_mpi_shim::cart_periodic(d) = periods[d];
    *c = 1;
    return MPI_SUCCESS;
}
static inline int MPI_Cart_coords(MPI_Comm, int, int nd, int* coords)
{
    for (int d = 0; d < nd; ++d) coords[d] = 0;
    return MPI_SUCCESS;
}
static inline int MPI_Cart_shift(MPI_Comm, int dim, int, int* src, int* dst)
{
    const int nb = oracle_mpi_shim::cart_periodic(dim) ? 0 : MPI_PROC_NULL;
    *src = nb;
    *dst = nb;
    return MPI_SUCCESS;
}
static inline int MPI_Allreduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, MPI_Comm)
{
    std::memmove(r, s, (size_t)n * oracle_mpi_shim::type_size(t));
    return MPI_SUCCESS;
}
static inline int MPI_Reduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm)
{
    if (r) std::memmove(r, s, (size_t)n * oracle_mpi_shim::type_size(t));
    return MPI_SUCCESS;
}
static inline int MPI_Isend(const void* b, int n, MPI_Datatype t, int peer, int tag, MPI_Comm, MPI_Request* req)
{
    *req = 0;
    if (peer == MPI_PROC_NULL) return MPI_SUCCESS;
    oracle_mpi_shim::Pending p{0, nullptr, (size_t)n * oracle_mpi_shim::type_size(t), tag, {}};
    p.data.assign((const char*)b, (const char*)b + p.bytes);
    oracle_mpi_shim::pending().push_back(std::move(p));
    return MPI_SUCCESS;
}
static inline int MPI_Irecv(void* b, int n, MPI_Datatype t, int peer, int tag, MPI_Comm, MPI_Request* req)
{
    *req = 0;
    if (peer == MPI_PROC_NULL) return MPI_SUCCESS;
    oracle_mpi_shim::pending().push_back({1, b, (size_t)n * oracle_mpi_shim::type_size(t), tag, {}});
    return MPI_SUCCESS;
}
static inline int MPI_Waitall(int, MPI_Request*, MPI_Status*)
{
    auto& v = oracle_mpi_shim::pending();
    for (auto& r : v)
    {
        if (r.kind != 1) continue;
        for (auto& s : v)
        {
            if (s.kind == 0 && s.tag == r.tag)
            {
                std::memcpy(r.buf, s.data.data(), r.bytes < s.bytes ? r.bytes : s.bytes);
                s.kind = 2;
                break;
            }
        }
    }
    v.clear();
    return MPI_SUCCESS;
}
static inline int MPI_Send(const void*, int, MPI_Datatype, int, int, MPI_Comm) { return MPI_SUCCESS; }
static inline int MPI_Recv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status*) { return MPI_SUCCESS; }

#endif
