/* Single-rank MPI stand-in used only to build the reference library's
 * twisted-mass path as a CPU oracle.  One process is rank 0 of a
 * 1-rank world: reductions and broadcasts are copies, barriers are no-ops,
 * and a point-to-point message can only go from the rank to itself (the
 * reference keeps every direction "parallel" and fills its own halo through
 * MPI, base/field.cpp:11-56), so sends are delivered to the receive with the
 * same tag.  Derived datatypes keep their byte size so that non-in-place
 * reductions copy the right amount. */
#ifndef ORACLE_SINGLE_RANK_MPI_H
#define ORACLE_SINGLE_RANK_MPI_H

#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <sys/time.h>
#include <unistd.h>
#include <vector>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef int MPI_Info;
typedef int MPI_File;
typedef int MPI_Fint;
typedef long long MPI_Offset;
typedef long long MPI_Count;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; size_t count; } MPI_Status;
typedef void MPI_User_function(void *, void *, int *, MPI_Datatype *);

#define MPI_SUCCESS 0
#define MPI_COMM_WORLD 1
#define MPI_COMM_NULL 0
#define MPI_COMM_TYPE_SHARED 1
#define MPI_INFO_NULL 0
#define MPI_THREAD_SINGLE 0
#define MPI_THREAD_FUNNELED 1
#define MPI_THREAD_SERIALIZED 2
#define MPI_THREAD_MULTIPLE 3
#define MPI_MAX_PROCESSOR_NAME 256
#define MPI_MAX_ERROR_STRING 256
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)
#define MPI_IN_PLACE ((void *)1)
#define MPI_PROC_NULL (-1)
#define MPI_ANY_SOURCE (-2)
#define MPI_ANY_TAG (-1)
#define MPI_UNDEFINED (-32766)

/* predefined datatypes: the handle indexes a size table */
#define MPI_DATATYPE_NULL 0
#define MPI_CHAR 1
#define MPI_BYTE 2
#define MPI_INT 3
#define MPI_UNSIGNED 4
#define MPI_LONG 5
#define MPI_FLOAT 6
#define MPI_DOUBLE 7
#define MPI_DOUBLE_COMPLEX 8
#define MPI_LONG_LONG 9
#define MPI_UNSIGNED_LONG 10
#define MPI_UNSIGNED_LONG_LONG 11
#define MPI_LONG_DOUBLE 12
#define MPI_SHORT 13
#define MPI_UNSIGNED_CHAR 14
#define MPI_C_BOOL 15
#define MPI_CXX_BOOL 15
#define MPI_UINT64_T 11
#define MPI_INT64_T 9
#define MPI_UINT32_T 4
#define MPI_INT32_T 3

#define MPI_OP_NULL 0
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPI_PROD 4
#define MPI_BXOR 5
#define MPI_LAND 6
#define MPI_LOR 7
#define MPI_BOR 8
#define MPI_BAND 9

namespace oracle_mpi
{
  inline std::vector<size_t> &type_sizes()
  {
    static std::vector<size_t> s = {0, 1, 1, sizeof(int), sizeof(unsigned), sizeof(long), sizeof(float),
                                    sizeof(double), 2 * sizeof(double), sizeof(long long),
                                    sizeof(unsigned long), sizeof(unsigned long long), sizeof(long double),
                                    sizeof(short), 1, sizeof(bool)};
    return s;
  }
  inline size_t size_of(MPI_Datatype t)
  {
    return (t >= 0 && (size_t)t < type_sizes().size()) ? type_sizes()[t] : 0;
  }
  inline MPI_Datatype new_type(size_t bytes)
  {
    type_sizes().push_back(bytes);
    return (MPI_Datatype)(type_sizes().size() - 1);
  }
  inline int &next_op()
  {
    static int n = 100;
    return n;
  }
}

inline int MPI_Init(int *, char ***) { return MPI_SUCCESS; }
inline int MPI_Init_thread(int *, char ***, int, int *provided)
{
  if (provided) *provided = MPI_THREAD_SERIALIZED;
  return MPI_SUCCESS;
}
inline int MPI_Initialized(int *flag) { *flag = 1; return MPI_SUCCESS; }
inline int MPI_Finalize() { return MPI_SUCCESS; }
inline int MPI_Abort(MPI_Comm, int code) { std::exit(code); return MPI_SUCCESS; }
inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return MPI_SUCCESS; }
inline int MPI_Comm_size(MPI_Comm, int *s) { *s = 1; return MPI_SUCCESS; }
inline int MPI_Comm_split_type(MPI_Comm c, int, int, MPI_Info, MPI_Comm *n) { *n = c; return MPI_SUCCESS; }
inline int MPI_Comm_free(MPI_Comm *) { return MPI_SUCCESS; }
inline MPI_Fint MPI_Comm_c2f(MPI_Comm c) { return c; }
inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }
inline double MPI_Wtime()
{
  struct timeval tv;
  gettimeofday(&tv, nullptr);
  return tv.tv_sec + 1e-6 * tv.tv_usec;
}
inline int MPI_Get_processor_name(char *name, int *len)
{
  gethostname(name, MPI_MAX_PROCESSOR_NAME);
  *len = (int)std::strlen(name);
  return MPI_SUCCESS;
}
inline int MPI_Error_string(int, char *s, int *len)
{
  std::strcpy(s, "single-rank stand-in");
  *len = (int)std::strlen(s);
  return MPI_SUCCESS;
}

/* one rank: a reduction is the identity on the local value */
inline int MPI_Allreduce(const void *in, void *out, int n, MPI_Datatype t, MPI_Op, MPI_Comm)
{
  if (in != MPI_IN_PLACE && in != out) std::memmove(out, in, (size_t)n * oracle_mpi::size_of(t));
  return MPI_SUCCESS;
}
inline int MPI_Reduce(const void *in, void *out, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm)
{
  if (in != MPI_IN_PLACE && in != out) std::memmove(out, in, (size_t)n * oracle_mpi::size_of(t));
  return MPI_SUCCESS;
}
inline int MPI_Op_create(MPI_User_function *, int, MPI_Op *op)
{
  *op = oracle_mpi::next_op()++;
  return MPI_SUCCESS;
}
inline int MPI_Op_free(MPI_Op *) { return MPI_SUCCESS; }

/* derived datatypes: only the byte size matters on one rank */
inline int MPI_Type_contiguous(int n, MPI_Datatype b, MPI_Datatype *t)
{
  *t = oracle_mpi::new_type((size_t)n * oracle_mpi::size_of(b));
  return MPI_SUCCESS;
}
inline int MPI_Type_vector(int n, int bl, int, MPI_Datatype b, MPI_Datatype *t)
{
  *t = oracle_mpi::new_type((size_t)n * bl * oracle_mpi::size_of(b));
  return MPI_SUCCESS;
}
inline int MPI_Type_indexed(int n, const int *bl, const int *, MPI_Datatype b, MPI_Datatype *t)
{
  size_t s = 0;
  for (int i = 0; i < n; i++) s += (size_t)bl[i];
  *t = oracle_mpi::new_type(s * oracle_mpi::size_of(b));
  return MPI_SUCCESS;
}
inline int MPI_Type_create_struct(int n, const int *bl, const long *, const MPI_Datatype *ts, MPI_Datatype *t)
{
  size_t s = 0;
  for (int i = 0; i < n; i++) s += (size_t)bl[i] * oracle_mpi::size_of(ts[i]);
  *t = oracle_mpi::new_type(s);
  return MPI_SUCCESS;
}
inline int MPI_Type_commit(MPI_Datatype *) { return MPI_SUCCESS; }
inline int MPI_Type_free(MPI_Datatype *) { return MPI_SUCCESS; }
inline int MPI_Type_size(MPI_Datatype t, int *s) { *s = (int)oracle_mpi::size_of(t); return MPI_SUCCESS; }

/* point to point on one rank can only be a message to oneself: a send is
 * recorded and delivered to the receive with the same tag when the requests
 * are completed (MPI requires the send buffer to stay untouched until then) */
namespace oracle_mpi
{
  struct pending { const void *send; void *recv; size_t bytes; int tag; };
  inline std::vector<pending> &sends() { static std::vector<pending> v; return v; }
  inline std::vector<pending> &recvs() { static std::vector<pending> v; return v; }
  inline void deliver()
  {
    for (auto &r : recvs())
      for (auto it = sends().begin(); it != sends().end(); ++it)
        if (it->tag == r.tag)
          {
            std::memmove(r.recv, it->send, r.bytes < it->bytes ? r.bytes : it->bytes);
            sends().erase(it);
            break;
          }
    recvs().clear();
  }
}
inline int MPI_Isend(const void *b, int n, MPI_Datatype t, int, int tag, MPI_Comm, MPI_Request *r)
{
  oracle_mpi::sends().push_back({b, nullptr, (size_t)n * oracle_mpi::size_of(t), tag});
  *r = 1;
  return MPI_SUCCESS;
}
inline int MPI_Irecv(void *b, int n, MPI_Datatype t, int, int tag, MPI_Comm, MPI_Request *r)
{
  oracle_mpi::recvs().push_back({nullptr, b, (size_t)n * oracle_mpi::size_of(t), tag});
  *r = 2;
  return MPI_SUCCESS;
}
inline int MPI_Send(const void *b, int n, MPI_Datatype t, int, int tag, MPI_Comm)
{
  oracle_mpi::sends().push_back({b, nullptr, (size_t)n * oracle_mpi::size_of(t), tag});
  return MPI_SUCCESS;
}
inline int MPI_Recv(void *b, int n, MPI_Datatype t, int, int tag, MPI_Comm, MPI_Status *)
{
  oracle_mpi::recvs().push_back({nullptr, b, (size_t)n * oracle_mpi::size_of(t), tag});
  oracle_mpi::deliver();
  return MPI_SUCCESS;
}
inline int MPI_Sendrecv(const void *sb, int sc, MPI_Datatype st, int, int, void *rb, int, MPI_Datatype, int, int,
                        MPI_Comm, MPI_Status *)
{
  std::memmove(rb, sb, (size_t)sc * oracle_mpi::size_of(st));
  return MPI_SUCCESS;
}
inline int MPI_Waitall(int, MPI_Request *, MPI_Status *) { oracle_mpi::deliver(); return MPI_SUCCESS; }
inline int MPI_Wait(MPI_Request *, MPI_Status *) { oracle_mpi::deliver(); return MPI_SUCCESS; }
inline int MPI_Get_count(const MPI_Status *s, MPI_Datatype t, int *c)
{
  size_t sz = oracle_mpi::size_of(t);
  *c = sz ? (int)(s->count / sz) : 0;
  return MPI_SUCCESS;
}

/* cartesian topology of a 1x1x1x1 grid */
inline int MPI_Cart_create(MPI_Comm c, int, const int *, const int *, int, MPI_Comm *n) { *n = c; return MPI_SUCCESS; }
inline int MPI_Cart_rank(MPI_Comm, const int *, int *r) { *r = 0; return MPI_SUCCESS; }
inline int MPI_Cart_coords(MPI_Comm, int, int nd, int *co)
{
  for (int i = 0; i < nd; i++) co[i] = 0;
  return MPI_SUCCESS;
}
inline int MPI_Cart_shift(MPI_Comm, int, int, int *s, int *d) { *s = 0; *d = 0; return MPI_SUCCESS; }
inline int MPI_Comm_split(MPI_Comm c, int, int, MPI_Comm *n) { *n = c; return MPI_SUCCESS; }
inline int MPI_Comm_dup(MPI_Comm c, MPI_Comm *n) { *n = c; return MPI_SUCCESS; }

#endif
