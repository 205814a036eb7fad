/* Serial MPI stand-in for the oracle shim: one rank, reductions are copies. */
#ifndef AWSEM_ORACLE_MPI_STUB_H
#define AWSEM_ORACLE_MPI_STUB_H
#include <cstring>
#include <chrono>
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
#define MPI_COMM_WORLD 0
#define MPI_DOUBLE 1
#define MPI_INT 2
#define MPI_LMP_TAGINT 2
#define MPI_LMP_BIGINT 3
#define MPI_SUM 10
#define MPI_MAX 11
#define MPI_MIN 12
static inline int mpi_stub_size(MPI_Datatype t) { return t == MPI_DOUBLE ? 8 : (t == MPI_LMP_BIGINT ? 8 : 4); }
static inline int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op, MPI_Comm)
{ if (s != r) std::memmove(r, s, (size_t) n * mpi_stub_size(t)); return 0; }
static inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm, int *s) { *s = 1; return 0; }
static inline double MPI_Wtime()
{ return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count(); }
#endif
