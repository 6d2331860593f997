/* TEST INFRASTRUCTURE ONLY.
 *
 * A single-process stand-in for the MPI calls that the reference's
 * time-step modules make, for running them on one rank (p_row = p_col = 1)
 * without an MPI library.  Semantics are those of the MPI standard for a
 * communicator of size 1:
 *  - MPI_Sendrecv to and from MPI_PROC_NULL does nothing; a send to rank 0
 *    matched by a receive from rank 0 in the same call copies the packed
 *    elements of the send type into the receive type (the periodic halo
 *    exchange with oneself);
 *  - MPI_Allreduce on one rank leaves MPI_IN_PLACE data as it is;
 *  - derived types are vectors (MPI_Type_vector) or a struct of scalars
 *    (MPI_Type_create_struct), kept in a small table;
 *  - Cartesian communicators have every dimension of size 1; a shift along
 *    a periodic dimension finds this rank, along any other MPI_PROC_NULL;
 *  - MPI_Alltoall(v) copies this rank's block to itself.
 * Anything outside this (a send without its matching receive) aborts.
 */
#pragma once

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef long MPI_Aint;
typedef struct MPI_Status {
  int MPI_SOURCE, MPI_TAG, MPI_ERROR;
} MPI_Status;
typedef void(MPI_User_function)(void *, void *, int *, MPI_Datatype *);

#define MPI_SUCCESS 0
#define MPI_PROC_NULL (-2)
#define MPI_COMM_WORLD 0
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_IN_PLACE ((void *)1)

/* predefined types: table indices 1..5 */
#define MPI_DOUBLE 1
#define MPI_FLOAT 2
#define MPI_INT 3
#define MPI_INTEGER 4
#define MPI_CHAR 5

#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPI_LAND 4

namespace mpi_shim {

struct TypeInfo {
  int count = 0, blocklen = 0, stride = 0; /* vector: count blocks of blocklen, stride apart */
  MPI_Datatype base = 0;                   /* element type of the vector */
  long size = 0;                           /* bytes of the packed data */
  long extent = 0;
  bool used = false;
};

inline TypeInfo *table() {
  static TypeInfo t[256];
  static bool init = false;
  if (!init) {
    init = true;
    const long sz[6] = {0, 8, 4, 4, 4, 1};
    for (int i = 1; i <= 5; ++i) {
      t[i].count = 1;
      t[i].blocklen = 1;
      t[i].stride = 1;
      t[i].base = 0;
      t[i].size = sz[i];
      t[i].extent = sz[i];
      t[i].used = true;
    }
  }
  return t;
}

inline void fail(const char *what) {
  fprintf(stderr, "mpi shim: %s\n", what);
  abort();
}

inline int new_type() {
  TypeInfo *t = table();
  for (int i = 6; i < 256; ++i)
    if (!t[i].used) {
      t[i] = TypeInfo{};
      t[i].used = true;
      return i;
    }
  fail("type table full");
  return 0;
}

/* copies `count` elements of type `ty` between two buffers laid out by that type */
inline void copy_typed(const char *src, char *dst, int count, MPI_Datatype ty) {
  const TypeInfo &t = table()[ty];
  if (t.base == 0) {
    memcpy(dst, src, (size_t)(t.size * count));
    return;
  }
  const TypeInfo &b = table()[t.base];
  if (t.stride == t.blocklen) { /* contiguous vector */
    memcpy(dst, src, (size_t)((long)count * t.count * t.blocklen * b.extent));
    return;
  }
  for (int n = 0; n < count; ++n)
    for (int c = 0; c < t.count; ++c) {
      const long off = n * t.extent + (long)c * t.stride * b.extent;
      memcpy(dst + off, src + off, (size_t)(t.blocklen * b.extent));
    }
}

struct CommInfo {
  int ndims = 0;
  int periods[4] = {0, 0, 0, 0};
  bool used = false;
};

inline CommInfo *comms() {
  static CommInfo c[64];
  c[0].used = true; /* MPI_COMM_WORLD */
  return c;
}

inline int new_comm(int ndims, const int *periods) {
  CommInfo *c = comms();
  for (int i = 1; i < 64; ++i)
    if (!c[i].used) {
      c[i] = CommInfo{};
      c[i].used = true;
      c[i].ndims = ndims;
      for (int d = 0; d < ndims && d < 4; ++d) c[i].periods[d] = periods[d];
      return i;
    }
  fail("communicator table full");
  return 0;
}

}  // namespace mpi_shim

inline int MPI_Cart_create(MPI_Comm, int ndims, const int *dims, const int *periods, int,
                           MPI_Comm *cart) {
  for (int d = 0; d < ndims; ++d)
    if (dims[d] != 1) mpi_shim::fail("process grid other than 1 x 1");
  *cart = mpi_shim::new_comm(ndims, periods);
  return MPI_SUCCESS;
}
inline int MPI_Cart_coords(MPI_Comm, int, int maxdims, int *coords) {
  for (int d = 0; d < maxdims; ++d) coords[d] = 0;
  return MPI_SUCCESS;
}
inline int MPI_Cart_shift(MPI_Comm comm, int direction, int, int *source, int *dest) {
  const bool periodic = mpi_shim::comms()[comm].periods[direction] != 0;
  *source = *dest = periodic ? 0 : MPI_PROC_NULL;
  return MPI_SUCCESS;
}
inline int MPI_Cart_sub(MPI_Comm comm, const int *remain_dims, MPI_Comm *newcomm) {
  const mpi_shim::CommInfo parent = mpi_shim::comms()[comm];
  int periods[4], n = 0;
  for (int d = 0; d < parent.ndims; ++d)
    if (remain_dims[d]) periods[n++] = parent.periods[d];
  *newcomm = mpi_shim::new_comm(n, periods);
  return MPI_SUCCESS;
}
inline int MPI_Comm_free(MPI_Comm *comm) {
  if (*comm > 0) mpi_shim::comms()[*comm].used = false;
  *comm = -1;
  return MPI_SUCCESS;
}

inline int MPI_Type_vector(int count, int blocklength, int stride, MPI_Datatype oldtype,
                           MPI_Datatype *newtype) {
  using namespace mpi_shim;
  const int id = new_type();
  TypeInfo &t = table()[id];
  const TypeInfo &b = table()[oldtype];
  if (b.base != 0) fail("nested vector types");
  t.count = count;
  t.blocklen = blocklength;
  t.stride = stride;
  t.base = oldtype;
  t.size = (long)count * blocklength * b.size;
  t.extent = count > 0 ? ((long)(count - 1) * stride + blocklength) * b.extent : 0;
  *newtype = id;
  return MPI_SUCCESS;
}

inline int MPI_Type_create_struct(int count, const int *blocklengths, const MPI_Aint *displs,
                                  const MPI_Datatype *types, MPI_Datatype *newtype) {
  using namespace mpi_shim;
  const int id = new_type();
  TypeInfo &t = table()[id];
  long end = 0;
  for (int i = 0; i < count; ++i) {
    const long e = displs[i] + blocklengths[i] * table()[types[i]].extent;
    if (e > end) end = e;
  }
  t.count = 1;
  t.blocklen = 1;
  t.stride = 1;
  t.base = 0;
  t.size = end;
  t.extent = end;
  *newtype = id;
  return MPI_SUCCESS;
}

inline int MPI_Type_commit(MPI_Datatype *) { return MPI_SUCCESS; }
inline int MPI_Type_free(MPI_Datatype *t) {
  if (*t > 5) mpi_shim::table()[*t].used = false;
  *t = 0;
  return MPI_SUCCESS;
}
inline int MPI_Type_get_extent(MPI_Datatype t, MPI_Aint *lb, MPI_Aint *extent) {
  *lb = 0;
  *extent = mpi_shim::table()[t].extent;
  return MPI_SUCCESS;
}
inline int MPI_Op_create(MPI_User_function *, int, MPI_Op *op) {
  *op = 100;
  return MPI_SUCCESS;
}
inline int MPI_Op_free(MPI_Op *op) {
  *op = 0;
  return MPI_SUCCESS;
}

inline int MPI_Sendrecv(const void *sendbuf, int sendcount, MPI_Datatype sendtype, int dest,
                        int, void *recvbuf, int recvcount, MPI_Datatype recvtype, int source,
                        int, MPI_Comm, MPI_Status *) {
  if (dest == MPI_PROC_NULL && source == MPI_PROC_NULL) return MPI_SUCCESS;
  if (dest != 0 || source != 0) mpi_shim::fail("unmatched send/receive on one rank");
  if (sendtype != recvtype || sendcount != recvcount) mpi_shim::fail("type mismatch");
  mpi_shim::copy_typed(static_cast<const char *>(sendbuf), static_cast<char *>(recvbuf),
                       sendcount, sendtype);
  return MPI_SUCCESS;
}

inline int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype type,
                         MPI_Op, MPI_Comm) {
  if (sendbuf != MPI_IN_PLACE)
    memcpy(recvbuf, sendbuf, (size_t)(count * mpi_shim::table()[type].size));
  return MPI_SUCCESS;
}

inline int MPI_Alltoall(const void *sendbuf, int sendcount, MPI_Datatype sendtype, void *recvbuf,
                        int, MPI_Datatype, MPI_Comm) {
  memcpy(recvbuf, sendbuf, (size_t)(sendcount * mpi_shim::table()[sendtype].size));
  return MPI_SUCCESS;
}
inline int MPI_Alltoallv(const void *sendbuf, const int *sendcounts, const int *sdispls,
                         MPI_Datatype sendtype, void *recvbuf, const int *, const int *rdispls,
                         MPI_Datatype, MPI_Comm) {
  const long es = mpi_shim::table()[sendtype].size;
  memcpy(static_cast<char *>(recvbuf) + rdispls[0] * es,
         static_cast<const char *>(sendbuf) + sdispls[0] * es, (size_t)(sendcounts[0] * es));
  return MPI_SUCCESS;
}

inline int MPI_Comm_rank(MPI_Comm, int *rank) {
  *rank = 0;
  return MPI_SUCCESS;
}
inline int MPI_Comm_size(MPI_Comm, int *size) {
  *size = 1;
  return MPI_SUCCESS;
}
inline int MPI_Abort(MPI_Comm, int code) {
  fprintf(stderr, "mpi shim: MPI_Abort(%d)\n", code);
  abort();
  return code;
}
inline double MPI_Wtime() {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}
