/*
 * Single-process stand-in for the MPI interface, used only to compile the
 * reference's own DSMC sources (oracle test infrastructure; never linked into
 * the product library).
 *
 * Every non-null communicator is a world of one rank: rank 0, size 1.
 * Collectives copy the send buffer to the receive buffer (or do nothing for
 * MPI_IN_PLACE); point-to-point messages to self are matched by tag inside
 * MPI_Waitall. With one compute rank the reference's particle hand-off code
 * sends nothing to other ranks, so these semantics are exact for the paths it
 * exercises (src/ProcessDSMC.cpp:1842-1933, src/MessagePassing.cpp:468-531).
 */
#ifndef DSMC_ORACLE_MPI_SHIM_H
#define DSMC_ORACLE_MPI_SHIM_H

#include <chrono>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <cstdlib>
#include <vector>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef std::ptrdiff_t MPI_Aint;
typedef int MPI_Request;
struct MPI_Status { int MPI_SOURCE; int MPI_TAG; int MPI_ERROR; };

#define MPI_SUCCESS 0
#define MPI_ERR_OTHER 15
#define MPI_COMM_NULL 0
#define MPI_COMM_WORLD 1
#define MPI_UNDEFINED (-32766)
#define MPI_DATATYPE_NULL 0
#define MPI_REQUEST_NULL 0
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_IN_PLACE ((void*)1)

#define MPI_CHAR 1
#define MPI_UNSIGNED_CHAR 2
#define MPI_INT 3
#define MPI_DOUBLE 4
#define MPI_LONG 5
#define MPI_FLOAT 6
#define MPI_BYTE 7
#define MPI_UNSIGNED 8
#define MPI_LONG_LONG 9

#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPI_LOR 4

namespace dsmc_mpi_shim {
struct TypeTable {
    std::vector<MPI_Aint> extent;
    TypeTable() : extent{0, 1, 1, 4, 8, 8, 4, 1, 4, 8} {}
};
inline TypeTable& types() { static TypeTable t; return t; }
inline MPI_Aint extent(MPI_Datatype t)
{
    if (t <= 0 || (std::size_t)t >= types().extent.size()) return 0;
    return types().extent[(std::size_t)t];
}
struct Pending { bool isSend; const void* sbuf; void* rbuf; std::size_t bytes; int tag; bool done; };
inline std::vector<Pending>& pending() { static std::vector<Pending> p(1); return p; }
inline void copyBytes(const void* s, void* r, std::size_t n)
{
    if (s == MPI_IN_PLACE || s == nullptr || r == nullptr || s == r || n == 0) return;
    std::memmove(r, s, n);
}
}  // namespace dsmc_mpi_shim

inline int MPI_Init(int*, char***) { return MPI_SUCCESS; }
inline int MPI_Finalize() { return MPI_SUCCESS; }
inline int MPI_Initialized(int* flag) { *flag = 1; return MPI_SUCCESS; }
inline int MPI_Finalized(int* flag) { *flag = 0; return MPI_SUCCESS; }
inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return MPI_SUCCESS; }
inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return MPI_SUCCESS; }
inline int MPI_Comm_split(MPI_Comm, int color, int, MPI_Comm* out)
{ *out = (color == MPI_UNDEFINED) ? MPI_COMM_NULL : MPI_COMM_WORLD; return MPI_SUCCESS; }
inline int MPI_Comm_free(MPI_Comm* c) { *c = MPI_COMM_NULL; return MPI_SUCCESS; }
inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
inline double MPI_Wtime()
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
inline int MPI_Abort(MPI_Comm, int code) { std::exit(code); }

inline int MPI_Get_address(const void* p, MPI_Aint* a) { *a = (MPI_Aint)(std::intptr_t)p; return MPI_SUCCESS; }
inline int MPI_Type_create_struct(int n, const int* bl, const MPI_Aint* disp, const MPI_Datatype* ts, MPI_Datatype* out)
{
    MPI_Aint ext = 0;
    for (int i = 0; i < n; ++i) {
        const MPI_Aint end = disp[i] + (MPI_Aint)bl[i] * dsmc_mpi_shim::extent(ts[i]);
        if (end > ext) ext = end;
    }
    dsmc_mpi_shim::types().extent.push_back(ext);
    *out = (MPI_Datatype)(dsmc_mpi_shim::types().extent.size() - 1);
    return MPI_SUCCESS;
}
inline int MPI_Type_contiguous(int n, MPI_Datatype t, MPI_Datatype* out)
{
    dsmc_mpi_shim::types().extent.push_back((MPI_Aint)n * dsmc_mpi_shim::extent(t));
    *out = (MPI_Datatype)(dsmc_mpi_shim::types().extent.size() - 1);
    return MPI_SUCCESS;
}
inline int MPI_Type_create_resized(MPI_Datatype, MPI_Aint, MPI_Aint ext, MPI_Datatype* out)
{
    dsmc_mpi_shim::types().extent.push_back(ext);
    *out = (MPI_Datatype)(dsmc_mpi_shim::types().extent.size() - 1);
    return MPI_SUCCESS;
}
inline int MPI_Type_commit(MPI_Datatype*) { return MPI_SUCCESS; }
inline int MPI_Type_free(MPI_Datatype* t) { *t = MPI_DATATYPE_NULL; return MPI_SUCCESS; }

inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }
inline int MPI_Allreduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, MPI_Comm)
{ dsmc_mpi_shim::copyBytes(s, r, (std::size_t)n * dsmc_mpi_shim::extent(t)); return MPI_SUCCESS; }
inline int MPI_Reduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm)
{ dsmc_mpi_shim::copyBytes(s, r, (std::size_t)n * dsmc_mpi_shim::extent(t)); return MPI_SUCCESS; }
inline int MPI_Gather(const void* s, int sn, MPI_Datatype st, void* r, int, MPI_Datatype, int, MPI_Comm)
{ dsmc_mpi_shim::copyBytes(s, r, (std::size_t)sn * dsmc_mpi_shim::extent(st)); return MPI_SUCCESS; }
inline int MPI_Gatherv(const void* s, int sn, MPI_Datatype st, void* r, const int*, const int* displs, MPI_Datatype rt, int, MPI_Comm)
{
    char* dst = (char*)r;
    if (dst && displs) dst += (std::size_t)displs[0] * dsmc_mpi_shim::extent(rt);
    dsmc_mpi_shim::copyBytes(s, dst, (std::size_t)sn * dsmc_mpi_shim::extent(st));
    return MPI_SUCCESS;
}
inline int MPI_Allgather(const void* s, int sn, MPI_Datatype st, void* r, int, MPI_Datatype, MPI_Comm)
{ dsmc_mpi_shim::copyBytes(s, r, (std::size_t)sn * dsmc_mpi_shim::extent(st)); return MPI_SUCCESS; }
inline int MPI_Scatter(const void* s, int, MPI_Datatype, void* r, int rn, MPI_Datatype rt, int, MPI_Comm)
{ dsmc_mpi_shim::copyBytes(s, r, (std::size_t)rn * dsmc_mpi_shim::extent(rt)); return MPI_SUCCESS; }
inline int MPI_Scatterv(const void* s, const int*, const int* displs, MPI_Datatype st, void* r, int rn, MPI_Datatype rt, int, MPI_Comm)
{
    const char* src = (const char*)s;
    if (src && src != MPI_IN_PLACE && displs) src += (std::size_t)displs[0] * dsmc_mpi_shim::extent(st);
    dsmc_mpi_shim::copyBytes(src, r, (std::size_t)rn * dsmc_mpi_shim::extent(rt));
    return MPI_SUCCESS;
}
inline int MPI_Alltoall(const void* s, int sn, MPI_Datatype st, void* r, int, MPI_Datatype, MPI_Comm)
{ dsmc_mpi_shim::copyBytes(s, r, (std::size_t)sn * dsmc_mpi_shim::extent(st)); return MPI_SUCCESS; }
inline int MPI_Alltoallv(const void* s, const int* sc, const int* sd, MPI_Datatype st, void* r, const int*, const int* rd, MPI_Datatype rt, MPI_Comm)
{
    const char* src = (const char*)s + (std::size_t)sd[0] * dsmc_mpi_shim::extent(st);
    char* dst = (char*)r + (std::size_t)rd[0] * dsmc_mpi_shim::extent(rt);
    dsmc_mpi_shim::copyBytes(src, dst, (std::size_t)sc[0] * dsmc_mpi_shim::extent(st));
    return MPI_SUCCESS;
}

inline int MPI_Isend(const void* buf, int n, MPI_Datatype t, int, int tag, MPI_Comm, MPI_Request* req)
{
    dsmc_mpi_shim::pending().push_back({true, buf, nullptr, (std::size_t)n * dsmc_mpi_shim::extent(t), tag, false});
    *req = (MPI_Request)(dsmc_mpi_shim::pending().size() - 1);
    return MPI_SUCCESS;
}
inline int MPI_Irecv(void* buf, int n, MPI_Datatype t, int, int tag, MPI_Comm, MPI_Request* req)
{
    dsmc_mpi_shim::pending().push_back({false, nullptr, buf, (std::size_t)n * dsmc_mpi_shim::extent(t), tag, false});
    *req = (MPI_Request)(dsmc_mpi_shim::pending().size() - 1);
    return MPI_SUCCESS;
}
inline int MPI_Waitall(int n, MPI_Request* reqs, MPI_Status*)
{
    auto& p = dsmc_mpi_shim::pending();
    for (int i = 0; i < n; ++i) {
        const int ri = reqs[i];
        if (ri <= 0 || (std::size_t)ri >= p.size() || p[(std::size_t)ri].isSend || p[(std::size_t)ri].done) continue;
        for (std::size_t j = 1; j < p.size(); ++j) {
            if (!p[j].isSend || p[j].done || p[j].tag != p[(std::size_t)ri].tag) continue;
            const std::size_t nb = p[j].bytes < p[(std::size_t)ri].bytes ? p[j].bytes : p[(std::size_t)ri].bytes;
            dsmc_mpi_shim::copyBytes(p[j].sbuf, p[(std::size_t)ri].rbuf, nb);
            p[j].done = true;
            p[(std::size_t)ri].done = true;
            break;
        }
    }
    for (int i = 0; i < n; ++i) reqs[i] = MPI_REQUEST_NULL;
    bool anyOpen = false;
    for (std::size_t j = 1; j < p.size(); ++j) anyOpen = anyOpen || !p[j].done;
    if (!anyOpen) p.resize(1);
    return MPI_SUCCESS;
}
inline int MPI_Wait(MPI_Request* r, MPI_Status* s) { return MPI_Waitall(1, r, s); }

// Persistent requests serve only the NS solver's halo exchange between
// ranks (src/MacroSolver.cpp, src/ProcessGSIS.cpp:1493), which a world of one
// rank does not have; the harness compiles that code but never runs it, so
// they do nothing.
#define MPI_PROC_NULL (-1)
inline int MPI_Send_init(const void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request* req)
{ *req = MPI_REQUEST_NULL; return MPI_SUCCESS; }
inline int MPI_Recv_init(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request* req)
{ *req = MPI_REQUEST_NULL; return MPI_SUCCESS; }
inline int MPI_Startall(int, MPI_Request*) { return MPI_SUCCESS; }
inline int MPI_Request_free(MPI_Request* req) { *req = MPI_REQUEST_NULL; return MPI_SUCCESS; }

#endif
