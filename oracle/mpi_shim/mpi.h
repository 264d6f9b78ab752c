/*
 * Single-rank loopback MPI, header-only.  TEST INFRASTRUCTURE ONLY.
 *
 * The ORION reference solver is written against MPI (halo exchange and
 * residual reductions, HaloExchanger.cpp:70-179, ResidualMonitor.cpp:101-128).
 * No MPI is installed in this image, so the oracle build compiles the
 * reference sources against this header instead.  Semantics are those of a
 * one-process MPI_COMM_WORLD:
 *   - rank 0 of size 1; Barrier/Bcast are no-ops;
 *   - Allreduce/Reduce copy the send buffer to the receive buffer;
 *   - Isend to self enqueues a copy keyed by tag; Probe/Get_count/Recv/Irecv
 *     dequeue it (Irecv completes at Waitall if the message is not there yet);
 *   - Abort exits the process with the given code.
 * Nothing here is used by the product library.
 */
#ifndef ORION_ORACLE_MPI_SHIM_H
#define ORION_ORACLE_MPI_SHIM_H

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <vector>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;

struct MPI_Status {
  int MPI_SOURCE;
  int MPI_TAG;
  int MPI_ERROR;
  long long shim_bytes;
};

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_ANY_TAG (-1)
#define MPI_ANY_SOURCE (-2)

#define MPI_BYTE 1
#define MPI_INT 2
#define MPI_UINT 3
#define MPI_DOUBLE 4
#define MPI_LONG_LONG 5
#define MPI_UINT64_T 6
#define MPI_DOUBLE_INT 7
#define MPI_CHAR 8

#define MPI_SUM 1
#define MPI_MIN 2
#define MPI_MAX 3
#define MPI_MAXLOC 4
#define MPI_MINLOC 5

#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)
#define MPI_IN_PLACE ((void*)1)

namespace orion_mpi_shim {

inline std::size_t type_size(MPI_Datatype t) {
  switch (t) {
    case MPI_BYTE: case MPI_CHAR: return 1;
    case MPI_INT: case MPI_UINT: return 4;
    case MPI_DOUBLE: case MPI_LONG_LONG: case MPI_UINT64_T: return 8;
    case MPI_DOUBLE_INT: return 16; /* struct { double; int; } with padding */
    default: return 1;
  }
}

struct Message {
  int tag;
  std::vector<unsigned char> bytes;
};

struct PendingRecv {
  int handle;
  void* buf;
  std::size_t cap_bytes;
  int tag;
};

struct State {
  std::deque<Message> queue;
  std::vector<PendingRecv> pending;
  int next_handle = 1;
};

inline State& state() {
  static State s;
  return s;
}

inline bool take(int tag, void* buf, std::size_t cap) {
  auto& q = state().queue;
  for (auto it = q.begin(); it != q.end(); ++it) {
    if (tag == MPI_ANY_TAG || it->tag == tag) {
      std::size_t n = it->bytes.size() < cap ? it->bytes.size() : cap;
      if (n) std::memcpy(buf, it->bytes.data(), n);
      q.erase(it);
      return true;
    }
  }
  return false;
}

}  // namespace orion_mpi_shim

static inline int MPI_Init(int*, char***) { return MPI_SUCCESS; }
static inline int MPI_Finalize() { return MPI_SUCCESS; }
static inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return MPI_SUCCESS; }
static inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
static inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }
static inline int MPI_Abort(MPI_Comm, int code) {
  std::fflush(stdout);
  std::exit(code);
  return code;
}
static inline double MPI_Wtime() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

static inline int MPI_Allreduce(const void* send, void* recv, int count, MPI_Datatype t, MPI_Op, MPI_Comm) {
  if (send != MPI_IN_PLACE && send != recv)
    std::memcpy(recv, send, (std::size_t)count * orion_mpi_shim::type_size(t));
  return MPI_SUCCESS;
}
static inline int MPI_Reduce(const void* send, void* recv, int count, MPI_Datatype t, MPI_Op, int, MPI_Comm) {
  if (send != MPI_IN_PLACE && send != recv)
    std::memcpy(recv, send, (std::size_t)count * orion_mpi_shim::type_size(t));
  return MPI_SUCCESS;
}

static inline int MPI_Isend(const void* buf, int count, MPI_Datatype t, int, int tag, MPI_Comm, MPI_Request* req) {
  using namespace orion_mpi_shim;
  Message m;
  m.tag = tag;
  std::size_t n = (std::size_t)count * type_size(t);
  m.bytes.resize(n);
  if (n) std::memcpy(m.bytes.data(), buf, n);
  /* a pending Irecv with this tag takes it directly */
  auto& p = state().pending;
  for (auto it = p.begin(); it != p.end(); ++it) {
    if (it->tag == tag || it->tag == MPI_ANY_TAG) {
      std::size_t c = n < it->cap_bytes ? n : it->cap_bytes;
      if (c) std::memcpy(it->buf, m.bytes.data(), c);
      p.erase(it);
      if (req) *req = 0;
      return MPI_SUCCESS;
    }
  }
  state().queue.push_back(std::move(m));
  if (req) *req = 0;
  return MPI_SUCCESS;
}

static inline int MPI_Irecv(void* buf, int count, MPI_Datatype t, int, int tag, MPI_Comm, MPI_Request* req) {
  using namespace orion_mpi_shim;
  std::size_t cap = (std::size_t)count * type_size(t);
  if (take(tag, buf, cap)) {
    if (req) *req = 0;
    return MPI_SUCCESS;
  }
  PendingRecv pr{state().next_handle++, buf, cap, tag};
  state().pending.push_back(pr);
  if (req) *req = pr.handle;
  return MPI_SUCCESS;
}

static inline int MPI_Probe(int, int tag, MPI_Comm, MPI_Status* st) {
  using namespace orion_mpi_shim;
  for (auto& m : state().queue) {
    if (tag == MPI_ANY_TAG || m.tag == tag) {
      if (st) {
        st->MPI_SOURCE = 0;
        st->MPI_TAG = m.tag;
        st->MPI_ERROR = 0;
        st->shim_bytes = (long long)m.bytes.size();
      }
      return MPI_SUCCESS;
    }
  }
  std::fprintf(stderr, "[mpi shim] MPI_Probe: no message with tag %d (would deadlock)\n", tag);
  std::exit(3);
  return 1;
}

static inline int MPI_Get_count(const MPI_Status* st, MPI_Datatype t, int* count) {
  *count = (int)(st->shim_bytes / (long long)orion_mpi_shim::type_size(t));
  return MPI_SUCCESS;
}

static inline int MPI_Recv(void* buf, int count, MPI_Datatype t, int, int tag, MPI_Comm, MPI_Status*) {
  using namespace orion_mpi_shim;
  if (!take(tag, buf, (std::size_t)count * type_size(t))) {
    std::fprintf(stderr, "[mpi shim] MPI_Recv: no message with tag %d (would deadlock)\n", tag);
    std::exit(3);
  }
  return MPI_SUCCESS;
}

static inline int MPI_Waitall(int, MPI_Request*, MPI_Status*) {
  using namespace orion_mpi_shim;
  if (!state().pending.empty()) {
    std::fprintf(stderr, "[mpi shim] MPI_Waitall: %zu receives never matched (would deadlock)\n",
                 state().pending.size());
    std::exit(3);
  }
  return MPI_SUCCESS;
}

#endif
