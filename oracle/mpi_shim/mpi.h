/*
 * Single-process MPI shim used ONLY to compile the reference's unmodified
 * CPU counting path (main.cpp + graph.hpp + utils.hpp + xxtric.hpp of
 * sg0/xxtric) into oracle/_ref/ as a test-side checker and as the CPU
 * baseline. It is test infrastructure, never linked into the product.
 *
 * Semantics: one rank (rank 0 of a communicator of size 1).
 *  - Collectives become copies (Reduce/Allreduce/Alltoall/Alltoallv) or no-ops
 *    (Barrier/Bcast), which is exactly what MPI does with one rank.
 *  - Point-to-point and Sendrecv are only ever addressed to MPI_PROC_NULL or
 *    to no peer at all with one rank; they complete immediately with no data.
 *  - MPI-IO becomes pread(2) on a plain file descriptor; read_all advances a
 *    per-file cursor as MPI's individual file pointer does.
 *  - MPI_Wtime is a monotonic clock.
 */
#ifndef XT_MPI_SHIM_H
#define XT_MPI_SHIM_H

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fcntl.h>
#include <unistd.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef int MPI_Info;
typedef long long MPI_Offset;
typedef struct { int MPI_SOURCE; int MPI_TAG; int xt_bytes; } MPI_Status;
typedef struct { int fd; long long cursor; } xt_mpi_file;
typedef xt_mpi_file *MPI_File;

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_PROC_NULL (-2)
#define MPI_ANY_SOURCE (-1)
#define MPI_ANY_TAG (-1)
#define MPI_REQUEST_NULL 0
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)
#define MPI_IN_PLACE ((void *)1)
#define MPI_THREAD_SINGLE 0
#define MPI_THREAD_MULTIPLE 3
#define MPI_MODE_RDONLY 2

/* datatype handle == element size in bytes (distinct handles for same size) */
#define MPI_BYTE ((MPI_Datatype)(1))
#define MPI_INT ((MPI_Datatype)(4 | (1 << 8)))
#define MPI_INT32_T ((MPI_Datatype)(4 | (2 << 8)))
#define MPI_FLOAT ((MPI_Datatype)(4 | (3 << 8)))
#define MPI_INT64_T ((MPI_Datatype)(8 | (4 << 8)))
#define MPI_DOUBLE ((MPI_Datatype)(8 | (5 << 8)))

#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3

static inline size_t xt_mpi_size(MPI_Datatype t) { return (size_t)(t & 0xff); }

static inline int MPI_Init(int *, char ***) { return 0; }
static inline int MPI_Init_thread(int *, char ***, int req, int *prov) { *prov = req; return 0; }
static inline int MPI_Finalize() { return 0; }
static inline int MPI_Abort(MPI_Comm, int code) { std::fflush(stdout); std::exit(code & 0xff); }
static inline int MPI_Comm_size(MPI_Comm, int *n) { *n = 1; return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline int MPI_Ibarrier(MPI_Comm, MPI_Request *r) { *r = MPI_REQUEST_NULL; return 0; }
static inline double MPI_Wtime() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}
static inline double MPI_Wtick() { return 1e-9; }

static inline void xt_mpi_copy(const void *s, void *r, size_t bytes) {
  if (s != MPI_IN_PLACE && s != r && bytes) std::memmove(r, s, bytes);
}
static inline int MPI_Reduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm) {
  xt_mpi_copy(s, r, (size_t)n * xt_mpi_size(t)); return 0;
}
static inline int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
  xt_mpi_copy(s, r, (size_t)n * xt_mpi_size(t)); return 0;
}
static inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return 0; }
static inline int MPI_Alltoall(const void *s, int n, MPI_Datatype t, void *r, int, MPI_Datatype, MPI_Comm) {
  xt_mpi_copy(s, r, (size_t)n * xt_mpi_size(t)); return 0;
}
static inline int MPI_Ialltoall(const void *s, int n, MPI_Datatype t, void *r, int, MPI_Datatype, MPI_Comm,
                                MPI_Request *q) {
  xt_mpi_copy(s, r, (size_t)n * xt_mpi_size(t)); *q = MPI_REQUEST_NULL; return 0;
}
static inline int MPI_Alltoallv(const void *s, const int *sc, const int *sd, MPI_Datatype t, void *r, const int *,
                                const int *rd, MPI_Datatype, MPI_Comm) {
  xt_mpi_copy((const char *)s + (size_t)sd[0] * xt_mpi_size(t), (char *)r + (size_t)rd[0] * xt_mpi_size(t),
              (size_t)sc[0] * xt_mpi_size(t));
  return 0;
}
static inline int MPI_Sendrecv(const void *, int, MPI_Datatype, int, int, void *, int, MPI_Datatype, int, int,
                               MPI_Comm, MPI_Status *) { return 0; }
static inline int MPI_Isend(const void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *r) {
  *r = MPI_REQUEST_NULL; return 0;
}
static inline int MPI_Irecv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *r) {
  *r = MPI_REQUEST_NULL; return 0;
}
static inline int MPI_Test(MPI_Request *, int *flag, MPI_Status *st) {
  *flag = 1;
  if (st) { st->MPI_SOURCE = MPI_ANY_SOURCE; st->MPI_TAG = MPI_ANY_TAG; st->xt_bytes = 0; }
  return 0;
}
static inline int MPI_Testsome(int, MPI_Request *, int *outcount, int *, MPI_Status *) { *outcount = 0; return 0; }
static inline int MPI_Wait(MPI_Request *, MPI_Status *) { return 0; }
static inline int MPI_Get_count(const MPI_Status *, MPI_Datatype, int *c) { *c = 0; return 0; }

static inline int MPI_Info_create(MPI_Info *i) { *i = 0; return 0; }
static inline int MPI_Info_set(MPI_Info, const char *, const char *) { return 0; }
static inline int MPI_Info_free(MPI_Info *) { return 0; }

static inline int MPI_File_open(MPI_Comm, const char *path, int, MPI_Info, MPI_File *f) {
  int fd = open(path, O_RDONLY);
  if (fd < 0) { *f = nullptr; return 1; }
  *f = new xt_mpi_file{fd, 0};
  return 0;
}
static inline int MPI_File_close(MPI_File *f) {
  if (*f) { close((*f)->fd); delete *f; *f = nullptr; }
  return 0;
}
static inline int xt_mpi_pread_full(int fd, void *buf, size_t bytes, long long off) {
  char *p = (char *)buf;
  while (bytes) {
    ssize_t k = pread(fd, p, bytes, off);
    if (k <= 0) return 1;
    p += k; bytes -= (size_t)k; off += k;
  }
  return 0;
}
static inline int MPI_File_read_all(MPI_File f, void *b, int n, MPI_Datatype t, MPI_Status *) {
  size_t bytes = (size_t)n * xt_mpi_size(t);
  int rc = xt_mpi_pread_full(f->fd, b, bytes, f->cursor);
  f->cursor += (long long)bytes;
  return rc;
}
static inline int MPI_File_read_at(MPI_File f, MPI_Offset o, void *b, int n, MPI_Datatype t, MPI_Status *) {
  return xt_mpi_pread_full(f->fd, b, (size_t)n * xt_mpi_size(t), o);
}

#endif
