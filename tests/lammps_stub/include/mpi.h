// TEST INFRASTRUCTURE: a single-rank stand-in for the few MPI calls of
// LAMMPS's pair_style hdnnp (handleExtrapolationWarnings).  One process is
// rank 0 of a one-rank world: gathers and reductions copy, point-to-point
// messages never occur (there is no other rank).
#pragma once
#include <cstdlib>
#include <cstring>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
struct MPI_Status { int source, tag, error; };
#define MPI_LONG 1
#define MPI_BYTE 2
#define MPI_SUM 1

inline int lmpstub_size(MPI_Datatype t) { return t == MPI_LONG ? (int)sizeof(long) : 1; }
inline int MPI_Gather(const void* s, int n, MPI_Datatype t, void* r, int, MPI_Datatype, int, MPI_Comm)
{ std::memcpy(r, s, (size_t)n * lmpstub_size(t)); return 0; }
inline int MPI_Reduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm)
{ std::memcpy(r, s, (size_t)n * lmpstub_size(t)); return 0; }
inline int MPI_Send(const void*, int, MPI_Datatype, int, int, MPI_Comm) { std::abort(); }
inline int MPI_Recv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status*) { std::abort(); }
