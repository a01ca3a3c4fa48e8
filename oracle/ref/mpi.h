// Single-process stand-in for <mpi.h>, enough to compile the reference's sources without MPI:
// the host parser and chemistry (src/Parameter.cpp, src/ChemData.cpp, src/ConstVolumeReactor.cpp)
// and the CUDA hot path with its field, boundary and communication code (src/Field.cu,
// src/BoundCond.cu, src/DataCommunication.cu, src/TimeAdvanceFunc.cu, ...).
// TEST INFRASTRUCTURE ONLY: used by oracle/ref_build.py and oracle/ref_gpu_build.py to build
// oracle/_ref/.
//
// One rank, rank 0 of a world of 1.  Collectives copy the send buffer to the receive buffer (the
// result of any reduction over one rank); point-to-point calls are never made by a serial run
// (`parallel = 0`) and return an error if they are.  Files are plain stdio files addressed by
// byte offsets; of the derived datatypes only 3-D Fortran-order subarrays of doubles are supported
// (MPI_File_read of the binary grid reader, MPI_File_read_at / write_at of the flowfield reader and
// writer); other uses report an error,
// so a code path that depends on them fails loudly instead of reading garbage.
#pragma once
#include <cstdio>
#include <cstdlib>
#include <cstring>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Info;
typedef long long MPI_Offset;
typedef int MPI_Request;
typedef struct { int s; } MPI_Status;
struct cb2_mpi_file_stub { std::FILE *fp; };
typedef cb2_mpi_file_stub *MPI_File;

#define MPI_SUCCESS 0
#define MPI_ERR_OTHER 15
#define MPI_COMM_WORLD 0
#define MPI_COMM_SELF 1
#define MPI_INFO_NULL 0
#define MPI_FILE_NULL ((MPI_File)0)
#define MPI_REQUEST_NULL 0
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)

// datatypes: the code is the element size in bytes times 16 plus a distinguishing index
#define MPI_CHAR (1 * 16 + 0)
#define MPI_BYTE (1 * 16 + 1)
#define MPI_INT (4 * 16 + 0)
#define MPI_INT32_T (4 * 16 + 1)
#define MPI_FLOAT (4 * 16 + 2)
#define MPI_REAL (4 * 16 + 3)
#define MPI_DOUBLE (8 * 16 + 0)
#define MPI_OFFSET (8 * 16 + 1)
#define MPI_ORDER_C 0
#define MPI_ORDER_FORTRAN 1

#define MPI_SUM 0
#define MPI_MIN 1
#define MPI_MAX 2

#define MPI_MODE_RDONLY 2
#define MPI_MODE_WRONLY 4
#define MPI_MODE_CREATE 1
#define MPI_MODE_APPEND 128

inline int cb2_mpi_type_size(MPI_Datatype t) { return t >= 16 ? t / 16 : 1; }

inline int MPI_Init(int *, char ***) { return MPI_SUCCESS; }
inline int MPI_Finalize() { return MPI_SUCCESS; }
inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return MPI_SUCCESS; }
inline int MPI_Comm_size(MPI_Comm, int *n) { *n = 1; return MPI_SUCCESS; }
inline int MPI_Abort(MPI_Comm, int c) { std::fprintf(stderr, "MPI_Abort(%d)\n", c); std::exit(c ? c : 1); return 0; }
inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
inline double MPI_Wtime() { return 0.0; }

// ---- collectives over one rank: the receive buffer takes the send buffer ----
inline int cb2_mpi_copy(const void *s, void *r, int n, MPI_Datatype t) {
  if (s && r && s != r && n > 0) std::memmove(r, s, static_cast<size_t>(n) * cb2_mpi_type_size(t));
  return MPI_SUCCESS;
}
inline int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
  return cb2_mpi_copy(s, r, n, t);
}
inline int MPI_Reduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm) {
  return cb2_mpi_copy(s, r, n, t);
}
inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }
inline int MPI_Allgather(const void *s, int ns, MPI_Datatype ts, void *r, int, MPI_Datatype, MPI_Comm) {
  return cb2_mpi_copy(s, r, ns, ts);
}
inline int MPI_Gather(const void *s, int ns, MPI_Datatype ts, void *r, int, MPI_Datatype, int, MPI_Comm) {
  return cb2_mpi_copy(s, r, ns, ts);
}
inline int MPI_Scatter(const void *s, int ns, MPI_Datatype ts, void *r, int, MPI_Datatype, int, MPI_Comm) {
  return cb2_mpi_copy(s, r, ns, ts);
}
inline int MPI_Allgatherv(const void *s, int ns, MPI_Datatype ts, void *r, const int *, const int *displs,
                          MPI_Datatype tr, MPI_Comm) {
  return cb2_mpi_copy(s, static_cast<char *>(r) + static_cast<size_t>(displs ? displs[0] : 0) * cb2_mpi_type_size(tr),
                      ns, ts);
}
inline int MPI_Gatherv(const void *s, int ns, MPI_Datatype ts, void *r, const int *, const int *displs,
                       MPI_Datatype tr, int, MPI_Comm) {
  return cb2_mpi_copy(s, static_cast<char *>(r) + static_cast<size_t>(displs ? displs[0] : 0) * cb2_mpi_type_size(tr),
                      ns, ts);
}
inline int MPI_Scatterv(const void *s, const int *, const int *displs, MPI_Datatype ts, void *r, int nr,
                        MPI_Datatype tr, int, MPI_Comm) {
  return cb2_mpi_copy(static_cast<const char *>(s) + static_cast<size_t>(displs ? displs[0] : 0) * cb2_mpi_type_size(ts),
                      r, nr, tr);
}

// ---- point to point: a serial run never exchanges messages ----
inline int MPI_Isend(const void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) { return MPI_ERR_OTHER; }
inline int MPI_Irecv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) { return MPI_ERR_OTHER; }
inline int MPI_Waitall(int, MPI_Request *, MPI_Status *) { return MPI_SUCCESS; }

// ---- derived datatypes: contiguous ones, and 3-D Fortran-order subarrays of doubles for reads ----
inline int MPI_Type_contiguous(int n, MPI_Datatype t, MPI_Datatype *nt) {
  *nt = n * cb2_mpi_type_size(t) * 16 + 15;
  return MPI_SUCCESS;
}
// A registered subarray: its handle is a negative index into this table.
struct cb2_mpi_subarray { int sizes[3], subsizes[3], starts[3]; };
inline cb2_mpi_subarray *cb2_mpi_subarrays() {
  static cb2_mpi_subarray table[64];
  return table;
}
inline int &cb2_mpi_n_subarrays() {
  static int n = 0;
  return n;
}
inline int MPI_Type_create_subarray(int ndims, const int *sizes, const int *subsizes, const int *starts, int order,
                                    MPI_Datatype old, MPI_Datatype *nt) {
  *nt = 0;  // size 1: any file access through an unsupported type is refused below
  if (ndims != 3 || order != MPI_ORDER_FORTRAN || old != MPI_DOUBLE || cb2_mpi_n_subarrays() >= 64) return MPI_ERR_OTHER;
  cb2_mpi_subarray &d = cb2_mpi_subarrays()[cb2_mpi_n_subarrays()];
  for (int a = 0; a < 3; ++a) d.sizes[a] = sizes[a], d.subsizes[a] = subsizes[a], d.starts[a] = starts[a];
  *nt = -1 - cb2_mpi_n_subarrays()++;
  return MPI_SUCCESS;
}
inline int MPI_Type_commit(MPI_Datatype *) { return MPI_SUCCESS; }
inline int MPI_Type_free(MPI_Datatype *) { return MPI_SUCCESS; }

// ---- files ----
inline int MPI_File_open(MPI_Comm, const char *name, int mode, MPI_Info, MPI_File *fh) {
  // a write without MPI_MODE_CREATE updates the existing file in place (the flowfield writer opens
  // its file again to write the data section after the header)
  const char *m = (mode & MPI_MODE_RDONLY) ? "rb" : ((mode & MPI_MODE_APPEND) ? "ab" : "w+b");
  std::FILE *fp = nullptr;
  if (!(mode & (MPI_MODE_RDONLY | MPI_MODE_APPEND | MPI_MODE_CREATE))) fp = std::fopen(name, "r+b");
  if (!fp) fp = std::fopen(name, m);
  if (!fp) {
    *fh = MPI_FILE_NULL;
    return MPI_ERR_OTHER;
  }
  *fh = new cb2_mpi_file_stub{fp};
  return MPI_SUCCESS;
}
inline int MPI_File_close(MPI_File *fh) {
  if (fh && *fh) {
    std::fclose((*fh)->fp);
    delete *fh;
    *fh = MPI_FILE_NULL;
  }
  return MPI_SUCCESS;
}
inline int cb2_mpi_file_io(MPI_File fh, long long off, void *buf, int n, MPI_Datatype t, bool write) {
  if (!fh || t <= 0) return MPI_ERR_OTHER;
  if (off >= 0 && std::fseek(fh->fp, off, SEEK_SET) != 0) return MPI_ERR_OTHER;
  const size_t bytes = static_cast<size_t>(n) * cb2_mpi_type_size(t);
  const size_t done = write ? std::fwrite(buf, 1, bytes, fh->fp) : std::fread(buf, 1, bytes, fh->fp);
  return done == bytes ? MPI_SUCCESS : MPI_ERR_OTHER;
}
// one 3-D Fortran-order subarray of doubles at byte offset off: its elements in file order (first
// index fastest) to or from their places in the full array at buf (the flowfield writer and the
// restart reader, src/FieldIO.h, src/Initialize.cu)
inline int cb2_mpi_subarray_io(MPI_File fh, long long off, double *buf, MPI_Datatype t, bool write) {
  if (!fh || -1 - t >= cb2_mpi_n_subarrays()) return MPI_ERR_OTHER;
  if (std::fseek(fh->fp, off, SEEK_SET) != 0) return MPI_ERR_OTHER;
  const cb2_mpi_subarray &d = cb2_mpi_subarrays()[-1 - t];
  for (int k = 0; k < d.subsizes[2]; ++k)
    for (int j = 0; j < d.subsizes[1]; ++j) {
      double *row = buf + d.starts[0] + (size_t)d.sizes[0] * ((d.starts[1] + j) + (size_t)d.sizes[1] * (d.starts[2] + k));
      const size_t done = write ? std::fwrite(row, sizeof(double), d.subsizes[0], fh->fp)
                                : std::fread(row, sizeof(double), d.subsizes[0], fh->fp);
      if (done != (size_t)d.subsizes[0]) return MPI_ERR_OTHER;
    }
  return MPI_SUCCESS;
}
inline int MPI_File_read_at(MPI_File fh, MPI_Offset off, void *buf, int n, MPI_Datatype t, MPI_Status *) {
  if (t < 0 && n == 1) return cb2_mpi_subarray_io(fh, off, static_cast<double *>(buf), t, false);
  return cb2_mpi_file_io(fh, off, buf, n, t, false);
}
inline int MPI_File_write_at(MPI_File fh, MPI_Offset off, const void *buf, int n, MPI_Datatype t, MPI_Status *) {
  if (t < 0 && n == 1) return cb2_mpi_subarray_io(fh, off, static_cast<double *>(const_cast<void *>(buf)), t, true);
  return cb2_mpi_file_io(fh, off, const_cast<void *>(buf), n, t, true);
}
inline int MPI_File_read(MPI_File fh, void *buf, int n, MPI_Datatype t, MPI_Status *) {
  if (t < 0 && fh && n == 1 && -1 - t < cb2_mpi_n_subarrays()) {
    // one subarray: read its elements in file order (first index fastest) into their places in
    // the full array at buf
    const cb2_mpi_subarray &d = cb2_mpi_subarrays()[-1 - t];
    double *out = static_cast<double *>(buf);
    for (int k = 0; k < d.subsizes[2]; ++k)
      for (int j = 0; j < d.subsizes[1]; ++j) {
        double *row = out + d.starts[0] +
                      (size_t)d.sizes[0] * ((d.starts[1] + j) + (size_t)d.sizes[1] * (d.starts[2] + k));
        if (std::fread(row, sizeof(double), d.subsizes[0], fh->fp) != (size_t)d.subsizes[0]) return MPI_ERR_OTHER;
      }
    return MPI_SUCCESS;
  }
  return cb2_mpi_file_io(fh, -1, buf, n, t, false);
}
inline int MPI_File_write(MPI_File fh, const void *buf, int n, MPI_Datatype t, MPI_Status *) {
  return cb2_mpi_file_io(fh, -1, const_cast<void *>(buf), n, t, true);
}
