/*
 * mpi.h -- single-rank MPI stand-in for building the reference's own code
 * as a CPU baseline and statistical checker (test infrastructure; never part
 * of the product).  One process is rank 0 of a world of size 1: collectives
 * copy the send buffer to the receive buffer, broadcasts and barriers do
 * nothing, communicator and group calls hand back the world.  Point-to-point
 * calls are reached by the reference only with two or more ranks; here they
 * abort with a message.  Covers the MPI calls the reference's sources make
 * (src/mpiKernel.cpp, src/langevinDynamics{Single,Double}Barrier.{h,cpp}).
 */
#ifndef LDP_REFSHIM_MPI_H
#define LDP_REFSHIM_MPI_H

#include <cstdio>
#include <cstdlib>
#include <cstring>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Group;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD ((MPI_Comm)1)
#define MPI_COMM_NULL ((MPI_Comm)0)
#define MPI_SUCCESS 0
/* datatypes encode their size in bytes in the low byte */
#define MPI_INT ((MPI_Datatype)4)
#define MPI_DOUBLE ((MPI_Datatype)8)
#define MPI_UNSIGNED_LONG ((MPI_Datatype)(8 | 0x100))
#define MPI_SUM ((MPI_Op)1)
#define MPI_MAX ((MPI_Op)2)
#define MPI_MIN ((MPI_Op)3)

static inline size_t ldp_refshim_size(MPI_Datatype t) { return (size_t)(t & 0xff); }
static inline void ldp_refshim_copy(const void* src, void* dst, int count, MPI_Datatype t) {
    if (src && dst && src != dst && count > 0) std::memmove(dst, src, (size_t)count * ldp_refshim_size(t));
}
static inline void ldp_refshim_abort(const char* what) {
    std::fprintf(stderr, "single-rank MPI stand-in: %s needs two or more ranks\n", what);
    std::abort();
}

static inline int MPI_Init(int*, char***) { return MPI_SUCCESS; }
static inline int MPI_Finalize(void) { return MPI_SUCCESS; }
static inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm, int* n) { *n = 1; return MPI_SUCCESS; }
static inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
static inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }
static inline int MPI_Allreduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
    ldp_refshim_copy(s, r, n, t);
    return MPI_SUCCESS;
}
static inline int MPI_Reduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm) {
    ldp_refshim_copy(s, r, n, t);
    return MPI_SUCCESS;
}
static inline int MPI_Allgather(const void* s, int n, MPI_Datatype t, void* r, int, MPI_Datatype, MPI_Comm) {
    ldp_refshim_copy(s, r, n, t);
    return MPI_SUCCESS;
}
static inline int MPI_Allgatherv(const void* s, int n, MPI_Datatype t, void* r, const int*, const int* displs,
                                 MPI_Datatype rt, MPI_Comm) {
    ldp_refshim_copy(s, (char*)r + (size_t)displs[0] * ldp_refshim_size(rt), n, t);
    return MPI_SUCCESS;
}
static inline int MPI_Gather(const void* s, int n, MPI_Datatype t, void* r, int, MPI_Datatype, int, MPI_Comm) {
    ldp_refshim_copy(s, r, n, t);
    return MPI_SUCCESS;
}
static inline int MPI_Scatter(const void* s, int n, MPI_Datatype t, void* r, int, MPI_Datatype, int, MPI_Comm) {
    ldp_refshim_copy(s, r, n, t);
    return MPI_SUCCESS;
}
static inline int MPI_Send(const void*, int, MPI_Datatype, int, int, MPI_Comm) {
    ldp_refshim_abort("MPI_Send");
    return 1;
}
static inline int MPI_Recv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status*) {
    ldp_refshim_abort("MPI_Recv");
    return 1;
}
static inline int MPI_Comm_split(MPI_Comm c, int, int, MPI_Comm* out) { *out = c; return MPI_SUCCESS; }
static inline int MPI_Comm_group(MPI_Comm, MPI_Group* g) { *g = 1; return MPI_SUCCESS; }
static inline int MPI_Group_incl(MPI_Group g, int, const int*, MPI_Group* out) { *out = g; return MPI_SUCCESS; }
static inline int MPI_Comm_create_group(MPI_Comm c, MPI_Group, int, MPI_Comm* out) { *out = c; return MPI_SUCCESS; }
static inline int MPI_Comm_free(MPI_Comm* c) { *c = MPI_COMM_NULL; return MPI_SUCCESS; }
static inline int MPI_Group_free(MPI_Group* g) { *g = 0; return MPI_SUCCESS; }

#endif
