/*
 * Single-process stand-in for the MPI calls the reference driver makes
 * (src/sputniPIC_CPU.cpp, src/mpi_comm.cpp), so the unmodified driver can be
 * compiled here for the drop-in integration test: world size 1, rank 0;
 * scatter/reduce copy the local buffer, broadcast does nothing.
 * TEST INFRASTRUCTURE ONLY.
 */
#ifndef SPB_TEST_MPI_STUB_H
#define SPB_TEST_MPI_STUB_H
#include <cstdlib>
#include <cstring>
#include <omp.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
#define MPI_COMM_WORLD 0
#define MPI_FLOAT 1
#define MPI_DOUBLE 2
#define MPI_C_BOOL 3
#define MPI_INT 4
#define MPI_SUM 0
#define MPI_THREAD_FUNNELED 1
#define MPI_IN_PLACE ((void *)1)

static inline size_t spb_mpi_size_of(MPI_Datatype t) {
  return t == MPI_DOUBLE ? 8 : t == MPI_C_BOOL ? 1 : 4;
}
static inline int MPI_Init_thread(int *, char ***, int required, int *provided) {
  *provided = required;
  return 0;
}
static inline int MPI_Comm_size(MPI_Comm, int *s) { *s = 1; return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return 0; }
static inline double MPI_Wtime(void) { return omp_get_wtime(); }
static inline int MPI_Abort(MPI_Comm, int code) { std::exit(code); }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Scatter(const void *s, int sc, MPI_Datatype st, void *r, int, MPI_Datatype,
                              int, MPI_Comm) {
  if (s != r) std::memmove(r, s, (size_t)sc * spb_mpi_size_of(st));
  return 0;
}
static inline int MPI_Reduce(const void *s, void *r, int c, MPI_Datatype t, MPI_Op, int,
                             MPI_Comm) {
  if (s != MPI_IN_PLACE && s != r) std::memmove(r, s, (size_t)c * spb_mpi_size_of(t));
  return 0;
}
static inline int MPI_Allreduce(const void *s, void *r, int c, MPI_Datatype t, MPI_Op o,
                                MPI_Comm m) {
  return MPI_Reduce(s, r, c, t, o, 0, m);
}
static inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return 0; }
#endif
