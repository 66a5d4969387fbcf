/*
 * One-rank MPI stand-in used only to compile the reference's CPU sources for
 * the oracle (test infrastructure, never linked into the product).
 *
 * The reference calls MPI_Init/Finalize/Comm_rank/Comm_size/Bcast/Allreduce/
 * Reduce/Wtime (src/nbody.cpp:17-18, 240-246, 300-324, 346-353;
 * src/main.cpp:14, 80-84, 127-129).  With a single rank every collective is
 * the identity: a broadcast leaves the root's buffer as it is, an in-place
 * sum or max over one rank leaves the buffer as it is, and a non-in-place
 * reduce copies send to receive.
 */
#ifndef ORACLE_STUB_MPI_H
#define ORACLE_STUB_MPI_H

#include <string.h>
#include <time.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;

#define MPI_COMM_WORLD 0
#define MPI_DOUBLE 8
#define MPI_INT 4
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_IN_PLACE ((void*)1)
#define MPI_SUCCESS 0

static inline int MPI_Init(int*, char***) { return MPI_SUCCESS; }
static inline int MPI_Finalize(void) { return MPI_SUCCESS; }
static inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return MPI_SUCCESS; }
static inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }

static inline int mpi_stub_copy(const void* send, void* recv, int count, MPI_Datatype t) {
  if (send != MPI_IN_PLACE && send != nullptr && recv != nullptr && send != recv)
    memcpy(recv, send, (size_t)count * (size_t)t);
  return MPI_SUCCESS;
}
static inline int MPI_Allreduce(const void* send, void* recv, int count, MPI_Datatype t, MPI_Op,
                                MPI_Comm) {
  return mpi_stub_copy(send, recv, count, t);
}
static inline int MPI_Reduce(const void* send, void* recv, int count, MPI_Datatype t, MPI_Op, int,
                             MPI_Comm) {
  return mpi_stub_copy(send, recv, count, t);
}
static inline double MPI_Wtime(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

#endif
