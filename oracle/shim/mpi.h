/* TEST INFRASTRUCTURE ONLY: single-rank stand-in for <mpi.h>, used to compile
 * the reference in place as a CPU oracle.  Only the names poisson.cpp uses. */
#ifndef ORC_SHIM_MPI_H
#define ORC_SHIM_MPI_H
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef struct { int unused; } MPI_Status;
#define MPI_INT 0
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
static inline int MPI_Send(const void *, int, MPI_Datatype, int, int, MPI_Comm) { return 0; }
static inline int MPI_Recv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status *) { return 0; }
#endif
