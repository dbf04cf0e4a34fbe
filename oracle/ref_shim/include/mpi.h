/*
 * mpi.h — a one-rank, in-process stand-in for the MPI calls the reference's
 * engine path makes (test infrastructure for the oracle shim only).
 *
 * The reference runs its single-partition case as `mpirun -np 1`: every
 * message goes to the process itself through MPI_Isend / MPI_Irecv and every
 * collective has one participant.  This header gives exactly that behaviour
 * without an MPI library:
 *   - point to point: a send is buffered (its data copied) and completes at
 *     once; it is matched, in send order, to the oldest posted receive whose
 *     source and tag accept it, else queued until one is posted;
 *   - a receive completes when matched; MPI_Test*, MPI_Wait* poll that;
 *     MPI_Cancel withdraws a posted receive;
 *   - collectives with one rank copy send to receive buffers (nothing for
 *     MPI_IN_PLACE); MPI_Barrier and MPI_Bcast do nothing.
 * All calls hold one mutex (the reference asks for MPI_THREAD_MULTIPLE).
 */
#ifndef PLATO_ORACLE_SHIM_MPI_H
#define PLATO_ORACLE_SHIM_MPI_H

#include <sched.h>

#include <cstdint>
#include <cstring>
#include <deque>
#include <list>
#include <mutex>
#include <vector>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef long long MPI_Aint;

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_ERR_TRUNCATE 15
#define MPI_ANY_SOURCE (-1)
#define MPI_ANY_TAG (-1)
#define MPI_UNDEFINED (-32766)
#define MPI_PROC_NULL (-2)
#define MPI_MAX_PROCESSOR_NAME 256

#define MPI_THREAD_SINGLE 0
#define MPI_THREAD_FUNNELED 1
#define MPI_THREAD_SERIALIZED 2
#define MPI_THREAD_MULTIPLE 3

/* datatypes encode their size in bytes (low byte) and a kind (high bits) */
#define PLATO_SHIM_DT(size, kind) (((kind) << 8) | (size))
#define MPI_CHAR PLATO_SHIM_DT(1, 1)
#define MPI_SIGNED_CHAR PLATO_SHIM_DT(1, 2)
#define MPI_UNSIGNED_CHAR PLATO_SHIM_DT(1, 3)
#define MPI_BYTE PLATO_SHIM_DT(1, 4)
#define MPI_SHORT PLATO_SHIM_DT(2, 5)
#define MPI_UNSIGNED_SHORT PLATO_SHIM_DT(2, 6)
#define MPI_INT PLATO_SHIM_DT(4, 7)
#define MPI_UNSIGNED PLATO_SHIM_DT(4, 8)
#define MPI_LONG PLATO_SHIM_DT(8, 9)
#define MPI_UNSIGNED_LONG PLATO_SHIM_DT(8, 10)
#define MPI_LONG_LONG_INT PLATO_SHIM_DT(8, 11)
#define MPI_LONG_LONG MPI_LONG_LONG_INT
#define MPI_UNSIGNED_LONG_LONG PLATO_SHIM_DT(8, 12)
#define MPI_FLOAT PLATO_SHIM_DT(4, 13)
#define MPI_DOUBLE PLATO_SHIM_DT(8, 14)
#define MPI_LONG_DOUBLE PLATO_SHIM_DT(16, 15)
#define MPI_INT8_T PLATO_SHIM_DT(1, 16)
#define MPI_UINT8_T PLATO_SHIM_DT(1, 17)
#define MPI_INT16_T PLATO_SHIM_DT(2, 18)
#define MPI_UINT16_T PLATO_SHIM_DT(2, 19)
#define MPI_INT32_T PLATO_SHIM_DT(4, 20)
#define MPI_UINT32_T PLATO_SHIM_DT(4, 21)
#define MPI_INT64_T PLATO_SHIM_DT(8, 22)
#define MPI_UINT64_T PLATO_SHIM_DT(8, 23)
#define MPI_C_BOOL PLATO_SHIM_DT(1, 24)
#define MPI_CXX_BOOL PLATO_SHIM_DT(1, 25)
#define MPI_DATATYPE_NULL 0

#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPI_PROD 4
#define MPI_LAND 5
#define MPI_BAND 6
#define MPI_LOR 7
#define MPI_BOR 8
#define MPI_LXOR 9
#define MPI_BXOR 10
#define MPI_OP_NULL 0

#define MPI_IN_PLACE (reinterpret_cast<void*>(1))

struct MPI_Status {
  int MPI_SOURCE;
  int MPI_TAG;
  int MPI_ERROR;
  long long count_;
  int cancelled_;
};
#define MPI_STATUS_IGNORE (static_cast<MPI_Status*>(nullptr))
#define MPI_STATUSES_IGNORE (static_cast<MPI_Status*>(nullptr))

struct plato_shim_request {
  bool is_recv = false;
  bool done = false;
  void* buf = nullptr;
  long long capacity = 0;  /* bytes */
  int source = 0, tag = 0;
  MPI_Status status{};
};
typedef plato_shim_request* MPI_Request;
#define MPI_REQUEST_NULL (static_cast<MPI_Request>(nullptr))

namespace plato_shim_mpi {

struct message {
  int tag;
  std::vector<char> data;
};

struct world {
  std::mutex mu;
  std::deque<message> unmatched;        /* buffered sends, oldest first */
  std::list<plato_shim_request*> posted; /* posted receives, oldest first */
};

inline world& get() {
  static world w;
  return w;
}

inline int type_size(MPI_Datatype t) { return t & 0xFF; }

inline bool accepts(const plato_shim_request* r, int tag) {
  return (r->source == MPI_ANY_SOURCE || r->source == 0) && (r->tag == MPI_ANY_TAG || r->tag == tag);
}

/* copies a message into a receive and completes it; lock held */
inline void deliver(plato_shim_request* r, int tag, const char* data, long long bytes) {
  if (bytes > r->capacity) bytes = r->capacity;  /* MPI would flag truncation */
  if (bytes > 0) std::memcpy(r->buf, data, static_cast<size_t>(bytes));
  r->status.MPI_SOURCE = 0;
  r->status.MPI_TAG = tag;
  r->status.MPI_ERROR = MPI_SUCCESS;
  r->status.count_ = bytes;
  r->status.cancelled_ = 0;
  r->done = true;
}

inline void post_send(const void* buf, long long bytes, int tag) {
  world& w = get();
  std::lock_guard<std::mutex> lock(w.mu);
  for (auto it = w.posted.begin(); it != w.posted.end(); ++it) {
    if (accepts(*it, tag)) {
      plato_shim_request* r = *it;
      w.posted.erase(it);
      deliver(r, tag, static_cast<const char*>(buf), bytes);
      return;
    }
  }
  message m;
  m.tag = tag;
  m.data.assign(static_cast<const char*>(buf), static_cast<const char*>(buf) + bytes);
  w.unmatched.push_back(std::move(m));
}

inline void post_recv(plato_shim_request* r) {
  world& w = get();
  std::lock_guard<std::mutex> lock(w.mu);
  for (auto it = w.unmatched.begin(); it != w.unmatched.end(); ++it) {
    if (accepts(r, it->tag)) {
      deliver(r, it->tag, it->data.data(), static_cast<long long>(it->data.size()));
      w.unmatched.erase(it);
      return;
    }
  }
  w.posted.push_back(r);
}

inline bool is_done(plato_shim_request* r) {
  world& w = get();
  std::lock_guard<std::mutex> lock(w.mu);
  return r->done;
}

inline void reduce_copy(const void* send, void* recv, int count, MPI_Datatype t) {
  if (send == MPI_IN_PLACE || send == recv) return;
  std::memcpy(recv, send, static_cast<size_t>(count) * type_size(t));
}

}  // namespace plato_shim_mpi

inline int MPI_Init(int*, char***) { return MPI_SUCCESS; }
inline int MPI_Init_thread(int*, char***, int required, int* provided) {
  if (provided) *provided = required;
  return MPI_SUCCESS;
}
inline int MPI_Initialized(int* flag) {
  *flag = 1;
  return MPI_SUCCESS;
}
inline int MPI_Finalize(void) { return MPI_SUCCESS; }
inline int MPI_Abort(MPI_Comm, int code) {
  std::abort();
  return code;
}
inline int MPI_Comm_size(MPI_Comm, int* size) {
  *size = 1;
  return MPI_SUCCESS;
}
inline int MPI_Comm_rank(MPI_Comm, int* rank) {
  *rank = 0;
  return MPI_SUCCESS;
}
inline int MPI_Type_size(MPI_Datatype t, int* size) {
  *size = plato_shim_mpi::type_size(t);
  return MPI_SUCCESS;
}
inline int MPI_Get_count(const MPI_Status* s, MPI_Datatype t, int* count) {
  *count = static_cast<int>(s->count_ / plato_shim_mpi::type_size(t));
  return MPI_SUCCESS;
}
inline int MPI_Get_processor_name(char* name, int* len) {
  std::strcpy(name, "localhost");
  *len = 9;
  return MPI_SUCCESS;
}
inline double MPI_Wtime(void) { return 0.0; }

inline int MPI_Isend(const void* buf, int count, MPI_Datatype t, int, int tag, MPI_Comm, MPI_Request* req) {
  plato_shim_mpi::post_send(buf, static_cast<long long>(count) * plato_shim_mpi::type_size(t), tag);
  plato_shim_request* r = new plato_shim_request();
  r->done = true;
  *req = r;
  return MPI_SUCCESS;
}
inline int MPI_Send(const void* buf, int count, MPI_Datatype t, int, int tag, MPI_Comm) {
  plato_shim_mpi::post_send(buf, static_cast<long long>(count) * plato_shim_mpi::type_size(t), tag);
  return MPI_SUCCESS;
}
inline int MPI_Irecv(void* buf, int count, MPI_Datatype t, int source, int tag, MPI_Comm, MPI_Request* req) {
  plato_shim_request* r = new plato_shim_request();
  r->is_recv = true;
  r->buf = buf;
  r->capacity = static_cast<long long>(count) * plato_shim_mpi::type_size(t);
  r->source = source;
  r->tag = tag;
  *req = r;
  plato_shim_mpi::post_recv(r);
  return MPI_SUCCESS;
}

/* completes *req: copies its status and frees it */
inline void plato_shim_finish(MPI_Request* req, MPI_Status* status) {
  if (status) *status = (*req)->status;
  delete *req;
  *req = MPI_REQUEST_NULL;
}

inline int MPI_Test(MPI_Request* req, int* flag, MPI_Status* status) {
  if (*req == MPI_REQUEST_NULL) {
    *flag = 1;
    return MPI_SUCCESS;
  }
  *flag = plato_shim_mpi::is_done(*req) ? 1 : 0;
  if (*flag) plato_shim_finish(req, status);
  return MPI_SUCCESS;
}
inline int MPI_Wait(MPI_Request* req, MPI_Status* status) {
  int flag = 0;
  for (;;) {
    MPI_Test(req, &flag, status);
    if (flag) return MPI_SUCCESS;
    sched_yield();
  }
}
inline int MPI_Testany(int n, MPI_Request* reqs, int* index, int* flag, MPI_Status* status) {
  bool any_active = false;
  for (int i = 0; i < n; ++i) {
    if (reqs[i] == MPI_REQUEST_NULL) continue;
    any_active = true;
    if (plato_shim_mpi::is_done(reqs[i])) {
      plato_shim_finish(&reqs[i], status);
      *index = i;
      *flag = 1;
      return MPI_SUCCESS;
    }
  }
  *index = MPI_UNDEFINED;
  *flag = any_active ? 0 : 1;
  return MPI_SUCCESS;
}
inline int MPI_Testall(int n, MPI_Request* reqs, int* flag, MPI_Status* statuses) {
  for (int i = 0; i < n; ++i)
    if (reqs[i] != MPI_REQUEST_NULL && !plato_shim_mpi::is_done(reqs[i])) {
      *flag = 0;
      return MPI_SUCCESS;
    }
  for (int i = 0; i < n; ++i)
    if (reqs[i] != MPI_REQUEST_NULL) plato_shim_finish(&reqs[i], statuses ? &statuses[i] : nullptr);
  *flag = 1;
  return MPI_SUCCESS;
}
inline int MPI_Waitall(int n, MPI_Request* reqs, MPI_Status* statuses) {
  for (int i = 0; i < n; ++i) MPI_Wait(&reqs[i], statuses ? &statuses[i] : nullptr);
  return MPI_SUCCESS;
}
inline int MPI_Waitany(int n, MPI_Request* reqs, int* index, MPI_Status* status) {
  int flag = 0;
  for (;;) {
    MPI_Testany(n, reqs, index, &flag, status);
    if (flag) return MPI_SUCCESS;
    sched_yield();
  }
}
inline int MPI_Cancel(MPI_Request* req) {
  if (*req == MPI_REQUEST_NULL) return MPI_SUCCESS;
  plato_shim_mpi::world& w = plato_shim_mpi::get();
  std::lock_guard<std::mutex> lock(w.mu);
  if (!(*req)->done) {
    w.posted.remove(*req);
    (*req)->status.cancelled_ = 1;
    (*req)->done = true;
  }
  return MPI_SUCCESS;
}
inline int MPI_Test_cancelled(const MPI_Status* s, int* flag) {
  *flag = s->cancelled_;
  return MPI_SUCCESS;
}
inline int MPI_Request_free(MPI_Request* req) {
  if (*req != MPI_REQUEST_NULL && (*req)->done) delete *req;
  *req = MPI_REQUEST_NULL;
  return MPI_SUCCESS;
}

inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }
inline int MPI_Allreduce(const void* send, void* recv, int count, MPI_Datatype t, MPI_Op, MPI_Comm) {
  plato_shim_mpi::reduce_copy(send, recv, count, t);
  return MPI_SUCCESS;
}
inline int MPI_Reduce(const void* send, void* recv, int count, MPI_Datatype t, MPI_Op, int, MPI_Comm) {
  plato_shim_mpi::reduce_copy(send, recv, count, t);
  return MPI_SUCCESS;
}
inline int MPI_Allgather(const void* send, int scount, MPI_Datatype st, void* recv, int, MPI_Datatype,
                         MPI_Comm) {
  plato_shim_mpi::reduce_copy(send, recv, scount, st);
  return MPI_SUCCESS;
}
inline int MPI_Allgatherv(const void* send, int scount, MPI_Datatype st, void* recv, const int*,
                          const int* displs, MPI_Datatype rt, MPI_Comm) {
  if (send == MPI_IN_PLACE) return MPI_SUCCESS;
  std::memcpy(static_cast<char*>(recv) + static_cast<size_t>(displs[0]) * plato_shim_mpi::type_size(rt), send,
              static_cast<size_t>(scount) * plato_shim_mpi::type_size(st));
  return MPI_SUCCESS;
}
inline int MPI_Gatherv(const void* send, int scount, MPI_Datatype st, void* recv, const int*, const int* displs,
                       MPI_Datatype rt, int, MPI_Comm) {
  if (send == MPI_IN_PLACE) return MPI_SUCCESS;
  std::memcpy(static_cast<char*>(recv) + static_cast<size_t>(displs[0]) * plato_shim_mpi::type_size(rt), send,
              static_cast<size_t>(scount) * plato_shim_mpi::type_size(st));
  return MPI_SUCCESS;
}
inline int MPI_Gather(const void* send, int scount, MPI_Datatype st, void* recv, int, MPI_Datatype, int,
                      MPI_Comm) {
  plato_shim_mpi::reduce_copy(send, recv, scount, st);
  return MPI_SUCCESS;
}
inline int MPI_Alltoall(const void* send, int scount, MPI_Datatype st, void* recv, int, MPI_Datatype,
                        MPI_Comm) {
  plato_shim_mpi::reduce_copy(send, recv, scount, st);
  return MPI_SUCCESS;
}

#endif
