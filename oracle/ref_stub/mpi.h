/* Single-rank stand-in for <mpi.h>, used only to compile the reference's
 * DirectPseudoSpectral and HypreFDM sources into the oracle library under oracle/_ref.
 *
 * Test infrastructure: the product never includes this header.
 *
 * With one rank (size == 1) every point-to-point call in the reference solvers
 * sits behind a `size > 1` branch, so the send/recv bodies below never run;
 * they fail loudly if they ever do.  Barrier, Bcast and Allreduce run with
 * single-rank semantics (Allreduce copies the input to the output).
 */
#ifndef ORACLE_STUB_MPI_H
#define ORACLE_STUB_MPI_H
#include <cstdio>
#include <cstdlib>
#include <cstring>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef struct { int source, tag, error; } MPI_Status;
typedef int MPI_Request;

#define MPI_COMM_WORLD 0
#define MPI_DOUBLE 1
#define MPI_INT 2
#define MPI_MAX 1
#define MPI_SUM 2
#define MPI_STATUS_IGNORE ((MPI_Status*)0)

static inline size_t oracle_mpi_type_size(MPI_Datatype t) { return t == MPI_INT ? sizeof(int) : sizeof(double); }
static inline int MPI_Init(int*, char***) { return 0; }
static inline int MPI_Finalize() { return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return 0; }
static inline int MPI_Allreduce(const void* in, void* out, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
    std::memcpy(out, in, (size_t)n * oracle_mpi_type_size(t));
    return 0;
}
static inline int MPI_Send(const void*, int, MPI_Datatype, int, int, MPI_Comm) {
    std::fprintf(stderr, "oracle stub mpi.h: MPI_Send reached with one rank\n");
    std::abort();
}
static inline int MPI_Recv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status*) {
    std::fprintf(stderr, "oracle stub mpi.h: MPI_Recv reached with one rank\n");
    std::abort();
}
/* The HypreFDM solvers: derived datatypes for their halo exchange, and
 * non-blocking halo messages that, with one rank, are never posted (a periodic
 * neighbour is the rank itself and is copied in place). */
static inline int MPI_Type_indexed(int, const int*, const int*, MPI_Datatype, MPI_Datatype* t) { *t = MPI_DOUBLE; return 0; }
static inline int MPI_Type_commit(MPI_Datatype*) { return 0; }
static inline int MPI_Isend(const void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request*) {
    std::fprintf(stderr, "oracle stub mpi.h: MPI_Isend reached with one rank\n");
    std::abort();
}
static inline int MPI_Irecv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request*) {
    std::fprintf(stderr, "oracle stub mpi.h: MPI_Irecv reached with one rank\n");
    std::abort();
}
static inline int MPI_Wait(MPI_Request*, MPI_Status*) { return 0; }
static inline int MPI_Abort(MPI_Comm, int code) {
    std::fprintf(stderr, "oracle stub mpi.h: MPI_Abort(%d)\n", code);
    std::exit(code);
}
#endif
