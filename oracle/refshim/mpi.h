// Test infrastructure only: single-rank MPI stand-in.  The reference's EOS
// table reader is never called by the tests (tables are built in memory).
#ifndef AXREF_SHIM_MPI_H
#define AXREF_SHIM_MPI_H
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Info;
#define MPI_COMM_WORLD 0
#define MPI_INT 1
#define MPI_DOUBLE 2
#define MPI_INFO_NULL 0
inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return 0; }
inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return 0; }
#endif
