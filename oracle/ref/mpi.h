// Single-process stand-in for <mpi.h>, enough to compile the reference's host parser
// (src/Parameter.cpp, src/ChemData.cpp, src/gxl_lib/MyString.cpp) without MPI.
// TEST INFRASTRUCTURE ONLY: used by oracle/ref_build.py to build oracle/_ref/.
#pragma once
#include <cstdlib>
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef long long MPI_Offset;
typedef int MPI_File;
typedef struct { int s; } MPI_Status;
#define MPI_COMM_WORLD 0
#define MPI_CHAR 1
#define MPI_INT 2
#define MPI_INT32_T 3
#define MPI_DOUBLE 4
#define MPI_SUM 0
#define MPI_MIN 1
#define MPI_MAX 2
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
inline int MPI_Init(int *, char ***) { return 0; }
inline int MPI_Finalize() { return 0; }
inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return 0; }
inline int MPI_Comm_size(MPI_Comm, int *n) { *n = 1; return 0; }
inline int MPI_Abort(MPI_Comm, int c) { std::exit(c); return 0; }
inline int MPI_Barrier(MPI_Comm) { return 0; }
inline int MPI_File_read_at(MPI_File, MPI_Offset, void *, int, MPI_Datatype, MPI_Status *) { return 1; }
inline int MPI_File_write_at(MPI_File, MPI_Offset, const void *, int, MPI_Datatype, MPI_Status *) { return 1; }
inline double MPI_Wtime() { return 0.0; }
