// Single-rank stand-in for <mpi.h>, used only to compile the reference's own
// sources into the CPU checker under oracle/_ref/ (this machine has no MPI).
//
// With one rank every CommPlan of a LocalMesh is empty (the reference's
// Distributor builds send/recv lists only between distinct ranks), so the
// point-to-point calls below are never handed a non-empty buffer; collectives
// over one rank are copies.  Test infrastructure only: nothing in the shipped
// library includes this file.
#pragma once
#include <chrono>
#include <cstring>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_COMM_SELF 1
#define MPI_SUCCESS 0
#define MPI_IN_PLACE ((void *)1)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)
#define MPI_STATUS_IGNORE ((MPI_Status *)0)

enum { MPI_DOUBLE = 8, MPI_INT = 4, MPI_LONG_LONG = 9, MPI_LONG = 10, MPI_CHAR = 1, MPI_DOUBLE_INT = 12 };
enum { MPI_SUM = 1, MPI_MAX = 2, MPI_MIN = 3, MPI_MAXLOC = 4, MPI_MINLOC = 5 };

inline int mpistub_size(MPI_Datatype t) { return t == MPI_DOUBLE_INT ? 16 : (t == MPI_LONG ? 8 : t); }

inline int MPI_Init(int *, char ***) { return 0; }
inline int MPI_Finalize() { return 0; }
inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return 0; }
inline int MPI_Comm_size(MPI_Comm, int *s) { *s = 1; return 0; }
inline double MPI_Wtime()
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
inline int MPI_Allreduce(const void *in, void *out, int n, MPI_Datatype t, MPI_Op, MPI_Comm)
{
    if (in != MPI_IN_PLACE && n > 0) std::memcpy(out, in, static_cast<size_t>(n) * mpistub_size(t));
    return 0;
}
inline int MPI_Gather(const void *in, int n, MPI_Datatype t, void *out, int, MPI_Datatype, int, MPI_Comm)
{
    if (in != MPI_IN_PLACE && n > 0) std::memcpy(out, in, static_cast<size_t>(n) * mpistub_size(t));
    return 0;
}
inline int MPI_Gatherv(const void *in, int n, MPI_Datatype t, void *out, const int *, const int *displs, MPI_Datatype, int, MPI_Comm)
{
    if (in != MPI_IN_PLACE && n > 0)
        std::memcpy(static_cast<char *>(out) + static_cast<size_t>(displs ? displs[0] : 0) * mpistub_size(t), in,
                    static_cast<size_t>(n) * mpistub_size(t));
    return 0;
}
inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return 0; }
inline int MPI_Barrier(MPI_Comm) { return 0; }
inline int MPI_Irecv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *r) { *r = 0; return 0; }
inline int MPI_Isend(const void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *r) { *r = 0; return 0; }
inline int MPI_Waitall(int, MPI_Request *, MPI_Status *) { return 0; }
inline int MPI_Abort(MPI_Comm, int code) { return code; }
