// Test infrastructure (oracle only): a single-rank subset of the MPI API so that
// the reference solver's source/parallel classes compile and run as one process
// without an MPI installation.  Every neighbour is MPI_PROC_NULL, so the halo
// exchange of source/parallel/CartesianParallel.cpp:172-427 moves nothing.
// Call sites: main.cpp:5-11, CartesianParallel.cpp:6-17,52-53,177-178,285-297.
#pragma once

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Request;
typedef struct { int source, tag, error; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_DOUBLE 1
#define MPI_INFO_NULL 0
#define MPI_PROC_NULL (-2)
#define MPI_SUCCESS 0

static inline int MPI_Init(int*, char***) { return MPI_SUCCESS; }
static inline int MPI_Finalize() { return MPI_SUCCESS; }
static inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return MPI_SUCCESS; }
static inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
static inline int MPI_Dims_create(int, int nd, int* dims) {
    for (int i = 0; i < nd; ++i) dims[i] = 1;
    return MPI_SUCCESS;
}
static inline int MPI_Cart_create(MPI_Comm, int, const int*, const int*, int, MPI_Comm* out) { *out = 1; return MPI_SUCCESS; }
static inline int MPI_Cart_coords(MPI_Comm, int, int nd, int* coords) {
    for (int i = 0; i < nd; ++i) coords[i] = 0;
    return MPI_SUCCESS;
}
static inline int MPI_Cart_shift(MPI_Comm, int, int, int* src, int* dst) {
    *src = MPI_PROC_NULL;
    *dst = MPI_PROC_NULL;
    return MPI_SUCCESS;
}
static inline int MPI_Type_contiguous(int, MPI_Datatype, MPI_Datatype* t) { *t = 2; return MPI_SUCCESS; }
static inline int MPI_Type_commit(MPI_Datatype*) { return MPI_SUCCESS; }
static inline int MPI_Type_free(MPI_Datatype*) { return MPI_SUCCESS; }
static inline int MPI_Irecv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request* r) { *r = 0; return MPI_SUCCESS; }
static inline int MPI_Isend(const void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request* r) { *r = 0; return MPI_SUCCESS; }
static inline int MPI_Waitall(int, MPI_Request*, MPI_Status*) { return MPI_SUCCESS; }
