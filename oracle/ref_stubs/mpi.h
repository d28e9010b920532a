/* Single-process stand-in for the MPI calls the reference makes
   (src/qcs.cu:1792-1850, 2100-2256, 2497-2541, 2611, 2894). With one rank,
   collectives copy the send buffer to the receive buffer and the rest are
   no-ops, which is what MPI does at mpirun -np 1. Test infrastructure for
   building the reference only. */
#pragma once
#include <cstring>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_BYTE 1
#define MPI_C_BOOL 1
#define MPI_FLOAT 4
#define MPI_UNSIGNED 4
#define MPI_DOUBLE 8
#define MPI_SUM 0
#define MPI_MAX 1

static inline int MPI_Init(int *, char ***) { return MPI_SUCCESS; }
static inline int MPI_Finalize(void) { return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm, int *size) { *size = 1; return MPI_SUCCESS; }
static inline int MPI_Comm_rank(MPI_Comm, int *rank) { *rank = 0; return MPI_SUCCESS; }
static inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
static inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }
static inline int MPI_Allreduce(const void *send, void *recv, int count, MPI_Datatype type, MPI_Op, MPI_Comm)
{
    std::memmove(recv, send, (size_t)count * (size_t)type);
    return MPI_SUCCESS;
}
static inline int MPI_Reduce(const void *send, void *recv, int count, MPI_Datatype type, MPI_Op, int, MPI_Comm)
{
    std::memmove(recv, send, (size_t)count * (size_t)type);
    return MPI_SUCCESS;
}
static inline int MPI_Scatter(const void *send, int, MPI_Datatype, void *recv, int rcount, MPI_Datatype rtype, int, MPI_Comm)
{
    std::memmove(recv, send, (size_t)rcount * (size_t)rtype);
    return MPI_SUCCESS;
}
