// Single-rank stand-in for the MPI calls of the reference's test driver
// (Test/Test.cpp, Test/main.cpp, Test/Util/PointDistribution.cpp), for the
// oracle only: this library needs no MPI, and the driver built against it runs
// as rank 0 of 1.  Collectives copy the send buffer to the receive buffer.
#pragma once
#include <cstring>

typedef int MPI_Comm;
typedef int MPI_Op;
typedef int MPI_Datatype;  // the element size in bytes
#define MPI_COMM_WORLD 0
#define MPI_SUM 0
#define MPI_MAX 1
#define MPI_DOUBLE 8
#define MPI_INT 4
#define MPI_IN_PLACE ((void *)1)

inline int MPI_Init(int *, char ***) { return 0; }
inline int MPI_Finalize() { return 0; }
inline int MPI_Comm_rank(MPI_Comm, int *r) {
    *r = 0;
    return 0;
}
inline int MPI_Comm_size(MPI_Comm, int *n) {
    *n = 1;
    return 0;
}
inline int MPI_Barrier(MPI_Comm) { return 0; }
inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return 0; }
inline int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
    if (s != MPI_IN_PLACE && s != r) std::memcpy(r, s, (size_t)n * t);
    return 0;
}
inline int MPI_Gather(const void *s, int n, MPI_Datatype t, void *r, int, MPI_Datatype, int, MPI_Comm) {
    if (r && s != r) std::memcpy(r, s, (size_t)n * t);
    return 0;
}
inline int MPI_Gatherv(const void *s, int n, MPI_Datatype t, void *r, const int *, const int *displs, MPI_Datatype,
                       int, MPI_Comm) {
    if (r) std::memcpy((char *)r + (size_t)(displs ? displs[0] : 0) * t, s, (size_t)n * t);
    return 0;
}
