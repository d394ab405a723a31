// Single-rank stand-in for the MPI API surface that the CFDV reference headers
// touch.  It exists only so that the reference's own sources compile, unmodified,
// into the CPU oracle (oracle/_ref).  One rank: Allreduce copies, point-to-point
// calls never run (MPISwapRank returns early for rank +-1 outside [0, size)),
// Bcast/Barrier/Type_* are no-ops.
#pragma once
#include <cstring>
typedef int MPI_Datatype;
typedef int MPI_Comm;
typedef long MPI_Aint;
typedef int MPI_Op;
typedef int MPI_Status;
typedef int MPI_File;
typedef int MPI_Info;
#define MPI_COMM_WORLD 0
// datatype handles double as the element size in bytes (used by Allreduce)
#define MPI_INT 4
#define MPI_DOUBLE 8
#define MPI_C_BOOL 1
#define MPI_UB 0
#define MPI_SUM 0
#define MPI_MIN 1
#define MPI_MAX 2
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_MODE_WRONLY 0
#define MPI_MODE_CREATE 0
#define MPI_INFO_NULL 0
#define MPI_SEEK_SET 0
inline int MPI_Init(int*, char***) { return 0; }
inline int MPI_Finalize() { return 0; }
inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return 0; }
inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return 0; }
inline int MPI_Allreduce(const void* a, void* b, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
  std::memcpy(b, a, (size_t)n * (size_t)t);
  return 0;
}
inline int MPI_Barrier(MPI_Comm) { return 0; }
inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return 0; }
inline int MPI_Send(const void*, int, MPI_Datatype, int, int, MPI_Comm) { return 0; }
inline int MPI_Recv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status*) { return 0; }
inline int MPI_Type_get_extent(MPI_Datatype, MPI_Aint*, MPI_Aint*) { return 0; }
inline int MPI_Type_create_struct(int, const int*, const MPI_Aint*, const MPI_Datatype*, MPI_Datatype*) { return 0; }
inline int MPI_Type_contiguous(int, MPI_Datatype, MPI_Datatype*) { return 0; }
inline int MPI_Type_commit(MPI_Datatype*) { return 0; }
