/* Single-process stand-in for the few MPI calls the reference's FCM file makes
 * (MPI_Barrier, MPI_Comm_rank, MPI_Reduce, MPI_Bcast), so that file can be
 * compiled and run here as one rank. Test infrastructure: only the
 * reference-pinning build in oracle/refshim uses it. */
#ifndef REFSHIM_MPI_H
#define REFSHIM_MPI_H
#include <stdlib.h>
#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
#define MPI_COMM_WORLD 0
#define MPI_DOUBLE 8
#define MPI_INT 4
#define MPI_SUM 1
#define MPI_MIN 2

static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int *rank) { *rank = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm, int *size) { *size = 1; return 0; }
/* one rank: the reduction of one contribution is the contribution */
static inline int MPI_Reduce(const void *send, void *recv, int count, MPI_Datatype type, MPI_Op, int, MPI_Comm) {
  if (send != recv) memmove(recv, send, (size_t)count * (size_t)type);
  return 0;
}
static inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return 0; }
/* one rank: the all-reduction of one contribution is the contribution */
static inline int MPI_Allreduce(const void *send, void *recv, int count, MPI_Datatype type, MPI_Op, MPI_Comm) {
  if (send != recv) memmove(recv, send, (size_t)count * (size_t)type);
  return 0;
}
static inline int MPI_Abort(MPI_Comm, int) { abort(); return 0; }
#endif
