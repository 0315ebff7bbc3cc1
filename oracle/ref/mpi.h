/* Single-rank MPI stand-in used ONLY to compile the reference FP64 CPU solver
 * in place as a parity checker (test infrastructure, never shipped).
 *
 * The reference (solver/geometry_distributed.cpp:19) includes <mpi.h>; with one
 * rank every message it sends is addressed to itself (periodic faces become
 * self-messages, solver/geometry_distributed.cpp:548-569).  This header gives
 * exactly the calls the reference makes (solve.cpp:260-387,
 * geometry_distributed.cpp:291-384,592-808, time_distributed.cpp:33-34,
 * dg.cpp:27-30,138) with self-delivery: a send packs its payload into a queue
 * at post time, a receive takes the oldest queued message with the same tag and
 * unpacks it through the receiver's datatype.  Indexed + resized datatypes are
 * modelled as (base size, blocks, extent) so count>1 transfers stride by the
 * resized extent, as MPI specifies.
 */
#pragma once

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <utility>
#include <vector>

typedef int MPI_Comm;
typedef int MPI_Op;
typedef int MPI_Request;
struct MPI_Status { int MPI_SOURCE, MPI_TAG, MPI_ERROR; };

#define MPI_COMM_WORLD 0
#define MPI_COMM_NULL (-1)
#define MPI_SUM 1
#define MPI_ANY_SOURCE (-1)
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_SUCCESS 0

namespace mpishim {

struct dtype {
  size_t base;                                   // bytes of one base element
  std::vector<std::pair<long, long>> blocks;     // (displacement, length) in base elements
  long extent;                                   // bytes between consecutive items
  bool is_float, is_double;
};

inline std::vector<dtype>& types() {
  static std::vector<dtype> t;
  return t;
}

inline int make_basic(size_t sz, bool f, bool d) {
  dtype t;
  t.base = sz;
  t.blocks.push_back({0, 1});
  t.extent = (long)sz;
  t.is_float = f;
  t.is_double = d;
  types().push_back(t);
  return (int)types().size() - 1;
}

inline int t_double() { static int h = make_basic(sizeof(double), false, true); return h; }
inline int t_float() { static int h = make_basic(sizeof(float), true, false); return h; }
inline int t_int() { static int h = make_basic(sizeof(int), false, false); return h; }
inline int t_char() { static int h = make_basic(1, false, false); return h; }
inline int t_u64() { static int h = make_basic(sizeof(uint64_t), false, false); return h; }

inline std::map<int, std::deque<std::vector<char>>>& queue() {
  static std::map<int, std::deque<std::vector<char>>> q;
  return q;
}

inline void pack(const void* buf, int count, int ty, std::vector<char>& out) {
  const dtype& t = types()[ty];
  const char* b = (const char*)buf;
  for (int c = 0; c < count; ++c)
    for (auto& bl : t.blocks) {
      const char* src = b + (long)c * t.extent + bl.first * (long)t.base;
      out.insert(out.end(), src, src + bl.second * t.base);
    }
}

inline void unpack(const std::vector<char>& in, void* buf, int count, int ty) {
  const dtype& t = types()[ty];
  char* b = (char*)buf;
  size_t pos = 0;
  for (int c = 0; c < count; ++c)
    for (auto& bl : t.blocks) {
      size_t nb = bl.second * t.base;
      if (pos + nb > in.size()) { fprintf(stderr, "mpi shim: short message\n"); std::abort(); }
      memcpy(b + (long)c * t.extent + bl.first * (long)t.base, in.data() + pos, nb);
      pos += nb;
    }
}

}  // namespace mpishim

typedef int MPI_Datatype;
#define MPI_DOUBLE (mpishim::t_double())
#define MPI_FLOAT (mpishim::t_float())
#define MPI_INT (mpishim::t_int())
#define MPI_CHAR (mpishim::t_char())
#define MPI_UINT64_T (mpishim::t_u64())

inline int MPI_Init(int*, char***) { return 0; }
inline int MPI_Finalize() { return 0; }
inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return 0; }
inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return 0; }
inline int MPI_Barrier(MPI_Comm) { return 0; }
inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return 0; }

inline int MPI_Type_indexed(int n, const int* len, const int* disp, MPI_Datatype old, MPI_Datatype* nt) {
  const mpishim::dtype& o = mpishim::types()[old];
  mpishim::dtype t;
  t.base = o.base;
  t.is_float = o.is_float;
  t.is_double = o.is_double;
  long hi = 0;
  for (int i = 0; i < n; ++i) {
    t.blocks.push_back({(long)disp[i], (long)len[i]});
    if (disp[i] + len[i] > hi) hi = disp[i] + len[i];
  }
  t.extent = hi * (long)o.base;
  mpishim::types().push_back(t);
  *nt = (int)mpishim::types().size() - 1;
  return 0;
}

inline int MPI_Type_create_resized(MPI_Datatype old, long lb, long extent, MPI_Datatype* nt) {
  (void)lb;
  mpishim::dtype t = mpishim::types()[old];
  t.extent = extent;
  mpishim::types().push_back(t);
  *nt = (int)mpishim::types().size() - 1;
  return 0;
}

inline int MPI_Type_commit(MPI_Datatype*) { return 0; }
inline int MPI_Type_free(MPI_Datatype*) { return 0; }

inline int MPI_Issend(const void* buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm, MPI_Request* req) {
  if (dest != 0) { fprintf(stderr, "mpi shim: send to rank %d\n", dest); std::abort(); }
  std::vector<char> msg;
  mpishim::pack(buf, count, t, msg);
  mpishim::queue()[tag].push_back(std::move(msg));
  *req = 0;
  return 0;
}

inline int MPI_Recv(void* buf, int count, MPI_Datatype t, int src, int tag, MPI_Comm, MPI_Status*) {
  (void)src;
  auto it = mpishim::queue().find(tag);
  if (it == mpishim::queue().end() || it->second.empty()) {
    fprintf(stderr, "mpi shim: receive with tag %d has no matching send\n", tag);
    std::abort();
  }
  mpishim::unpack(it->second.front(), buf, count, t);
  it->second.pop_front();
  if (it->second.empty()) mpishim::queue().erase(it);
  return 0;
}

inline int MPI_Wait(MPI_Request*, MPI_Status*) { return 0; }

inline int MPI_Allreduce(const void* in, void* out, int count, MPI_Datatype t, MPI_Op, MPI_Comm) {
  const mpishim::dtype& d = mpishim::types()[t];
  memcpy(out, in, (size_t)count * d.base);
  return 0;
}
