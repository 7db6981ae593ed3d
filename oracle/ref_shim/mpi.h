/*
 * Single-process MPI stand-in used ONLY to compile the unmodified reference
 * CPU path (suzumura/graph500 mpi/*.hpp) as a checker and CPU baseline.
 * Test infrastructure, never linked into the CUDA library.
 *
 * Semantics for a world of one rank:
 *  - size 1, rank 0; communicator split/dup hand out fresh handles;
 *  - barrier and broadcast do nothing;
 *  - every reduction / all-to-all / gather copies the rank-0 slice
 *    (honouring MPI_IN_PLACE);
 *  - derived datatypes only carry their byte size;
 *  - point-to-point messages to self go through a tag-matched queue
 *    (the bottom-up ring of the reference talks to itself);
 *  - MPI-IO is only used with TMPFILE, which this stand-in does not support.
 */
#ifndef G500_REF_SHIM_MPI_H
#define G500_REF_SHIM_MPI_H

#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <pthread.h>
#include <unistd.h>
#include <deque>
#include <vector>

#define MPI_VERSION 3
#define MPI_SUBVERSION 0
#define MPI_SUCCESS 0

struct shim_datatype { int bytes; };
typedef shim_datatype* MPI_Datatype;
typedef int MPI_Comm;
typedef int MPI_Op;
typedef int MPI_Group;
typedef int MPI_Info;
typedef int MPI_Errhandler;
typedef long MPI_Aint;
typedef long long MPI_Offset;
typedef FILE* MPI_File;

struct shim_request {
  bool is_recv;
  void* buf;
  int tag;
  bool done;
  int bytes;
};
typedef shim_request* MPI_Request;

typedef struct {
  int MPI_SOURCE;
  int MPI_TAG;
  int MPI_ERROR;
  int shim_bytes;
} MPI_Status;

inline shim_datatype shim_t1{1}, shim_t2{2}, shim_t4{4}, shim_t8{8};
#define MPI_CHAR (&shim_t1)
#define MPI_SIGNED_CHAR (&shim_t1)
#define MPI_UNSIGNED_CHAR (&shim_t1)
#define MPI_BYTE (&shim_t1)
#define MPI_INT8_T (&shim_t1)
#define MPI_UINT8_T (&shim_t1)
#define MPI_SHORT (&shim_t2)
#define MPI_UNSIGNED_SHORT (&shim_t2)
#define MPI_INT16_T (&shim_t2)
#define MPI_UINT16_T (&shim_t2)
#define MPI_INT (&shim_t4)
#define MPI_UNSIGNED (&shim_t4)
#define MPI_FLOAT (&shim_t4)
#define MPI_INT32_T (&shim_t4)
#define MPI_UINT32_T (&shim_t4)
#define MPI_LONG (&shim_t8)
#define MPI_UNSIGNED_LONG (&shim_t8)
#define MPI_LONG_LONG (&shim_t8)
#define MPI_UNSIGNED_LONG_LONG (&shim_t8)
#define MPI_DOUBLE (&shim_t8)
#define MPI_INT64_T (&shim_t8)
#define MPI_UINT64_T (&shim_t8)
#define MPI_AINT (&shim_t8)
#define MPI_DATATYPE_NULL ((MPI_Datatype)0)

#define MPI_COMM_NULL 0
#define MPI_COMM_WORLD 1
#define MPI_COMM_SELF 2
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPI_BOR 4
#define MPI_LOR 5
#define MPI_BAND 6
#define MPI_LAND 7
#define MPI_IN_PLACE ((void*)1)
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)
#define MPI_REQUEST_NULL ((MPI_Request)0)
#define MPI_UNDEFINED (-32766)
#define MPI_ANY_SOURCE (-1)
#define MPI_ANY_TAG (-1)
#define MPI_INFO_NULL 0
#define MPI_THREAD_SINGLE 0
#define MPI_THREAD_FUNNELED 1
#define MPI_THREAD_SERIALIZED 2
#define MPI_THREAD_MULTIPLE 3
#define MPI_MODE_RDWR 1
#define MPI_MODE_CREATE 2
#define MPI_MODE_DELETE_ON_CLOSE 4
#define MPI_MODE_UNIQUE_OPEN 8
#define MPI_MODE_EXCL 16
#define MPI_MODE_NOSUCCEED 32
#define MPI_MODE_NOPRECEDE 64
#define MPI_ERRORS_ARE_FATAL 0
#define MPI_FILE_NULL ((MPI_File)0)

/* ---- process and communicators ---- */
inline int shim_next_comm = 3;
inline int MPI_Init(int*, char***) { return 0; }
inline int MPI_Init_thread(int*, char***, int required, int* provided) { *provided = required; return 0; }
inline int MPI_Finalize() { return 0; }
inline int MPI_Abort(MPI_Comm, int code) { fflush(stdout); fflush(stderr); exit(code); }
inline double MPI_Wtime() {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}
inline int MPI_Comm_rank(MPI_Comm, int* rank) { *rank = 0; return 0; }
inline int MPI_Comm_size(MPI_Comm, int* size) { *size = 1; return 0; }
inline int MPI_Comm_split(MPI_Comm, int, int, MPI_Comm* out) { *out = shim_next_comm++; return 0; }
inline int MPI_Comm_dup(MPI_Comm, MPI_Comm* out) { *out = shim_next_comm++; return 0; }
inline int MPI_Comm_free(MPI_Comm* c) { *c = MPI_COMM_NULL; return 0; }
inline int MPI_Comm_group(MPI_Comm, MPI_Group* g) { *g = 1; return 0; }
inline int MPI_Group_free(MPI_Group*) { return 0; }
inline int MPI_Group_translate_ranks(MPI_Group, int n, const int* in, MPI_Group, int* out) {
  for (int i = 0; i < n; ++i) out[i] = in[i];
  return 0;
}

/* ---- collectives over one rank ---- */
inline void shim_copy(const void* src, void* dst, long count, MPI_Datatype t) {
  if (src == MPI_IN_PLACE || src == dst || count <= 0) return;
  memmove(dst, src, (size_t)count * (size_t)t->bytes);
}
inline int MPI_Barrier(MPI_Comm) { return 0; }
inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return 0; }
inline int MPI_Reduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm) { shim_copy(s, r, n, t); return 0; }
inline int MPI_Allreduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) { shim_copy(s, r, n, t); return 0; }
inline int MPI_Reduce_scatter(const void* s, void* r, const int* counts, MPI_Datatype t, MPI_Op, MPI_Comm) {
  shim_copy(s, r, counts[0], t);
  return 0;
}
inline int MPI_Alltoall(const void* s, int sc, MPI_Datatype st, void* r, int, MPI_Datatype, MPI_Comm) { shim_copy(s, r, sc, st); return 0; }
inline int MPI_Alltoallv(const void* s, const int* sc, const int* sd, MPI_Datatype st, void* r, const int*,
                         const int* rd, MPI_Datatype, MPI_Comm) {
  if (sc[0] > 0)
    memmove((char*)r + (size_t)rd[0] * st->bytes, (const char*)s + (size_t)sd[0] * st->bytes, (size_t)sc[0] * st->bytes);
  return 0;
}
inline int MPI_Allgather(const void* s, int sc, MPI_Datatype st, void* r, int, MPI_Datatype, MPI_Comm) { shim_copy(s, r, sc, st); return 0; }
inline int MPI_Allgatherv(const void* s, int sc, MPI_Datatype st, void* r, const int*, const int* rd, MPI_Datatype, MPI_Comm) {
  if (s != MPI_IN_PLACE && sc > 0) memmove((char*)r + (size_t)rd[0] * st->bytes, s, (size_t)sc * st->bytes);
  return 0;
}
inline int MPI_Scatter(const void* s, int sc, MPI_Datatype st, void* r, int, MPI_Datatype, int, MPI_Comm) { shim_copy(s, r, sc, st); return 0; }

/* ---- memory and datatypes ---- */
inline int MPI_Alloc_mem(MPI_Aint n, MPI_Info, void* out) { *(void**)out = malloc(n ? (size_t)n : 1); return 0; }
inline int MPI_Free_mem(void* p) { free(p); return 0; }
inline int MPI_Type_create_hindexed(int n, const int* lens, const MPI_Aint*, MPI_Datatype base, MPI_Datatype* out) {
  int b = 0;
  for (int i = 0; i < n; ++i) b += lens[i] * base->bytes;
  *out = new shim_datatype{b};
  return 0;
}
inline int MPI_Type_create_struct(int n, const int* lens, const MPI_Aint*, const MPI_Datatype* types, MPI_Datatype* out) {
  int b = 0;
  for (int i = 0; i < n; ++i) b += lens[i] * types[i]->bytes;
  *out = new shim_datatype{b};
  return 0;
}
inline int MPI_Type_commit(MPI_Datatype*) { return 0; }
inline int MPI_Type_free(MPI_Datatype* t) { *t = MPI_DATATYPE_NULL; return 0; }
inline int MPI_Type_size(MPI_Datatype t, int* s) { *s = t->bytes; return 0; }

/* ---- point-to-point to self ---- */
struct shim_message { std::vector<char> bytes; int tag; };
inline std::deque<shim_message>& shim_mailbox() { static std::deque<shim_message> q; return q; }
inline std::vector<shim_request*>& shim_pending() { static std::vector<shim_request*> v; return v; }
inline void shim_match() {
  std::deque<shim_message>& box = shim_mailbox();
  std::vector<shim_request*>& pend = shim_pending();
  size_t i = 0;
  while (i < pend.size()) {
    shim_request* rq = pend[i];
    bool hit = false;
    for (std::deque<shim_message>::iterator it = box.begin(); it != box.end(); ++it) {
      if (rq->tag == MPI_ANY_TAG || rq->tag == it->tag) {
        if (!it->bytes.empty()) memcpy(rq->buf, it->bytes.data(), it->bytes.size());
        rq->bytes = (int)it->bytes.size();
        rq->tag = it->tag;
        rq->done = true;
        box.erase(it);
        hit = true;
        break;
      }
    }
    if (hit) pend.erase(pend.begin() + (long)i);
    else ++i;
  }
}
inline int MPI_Isend(const void* b, int n, MPI_Datatype t, int, int tag, MPI_Comm, MPI_Request* rq) {
  shim_message msg;
  msg.bytes.assign((const char*)b, (const char*)b + (size_t)n * t->bytes);
  msg.tag = tag;
  shim_mailbox().push_back(msg);
  *rq = new shim_request{false, 0, tag, true, n * t->bytes};
  shim_match();
  return 0;
}
inline int MPI_Irecv(void* b, int, MPI_Datatype, int, int tag, MPI_Comm, MPI_Request* rq) {
  *rq = new shim_request{true, b, tag, false, 0};
  shim_pending().push_back(*rq);
  shim_match();
  return 0;
}
inline void shim_status(const shim_request* rq, MPI_Status* st) {
  if (!st) return;
  st->MPI_SOURCE = 0;
  st->MPI_TAG = rq->tag;
  st->MPI_ERROR = 0;
  st->shim_bytes = rq->bytes;
}
inline int MPI_Test(MPI_Request* rq, int* flag, MPI_Status* st) {
  shim_match();
  if (*rq == MPI_REQUEST_NULL) { *flag = 1; return 0; }
  *flag = (*rq)->done ? 1 : 0;
  if (*flag) { shim_status(*rq, st); delete *rq; *rq = MPI_REQUEST_NULL; }
  return 0;
}
inline int MPI_Wait(MPI_Request* rq, MPI_Status* st) {
  int flag;
  MPI_Test(rq, &flag, st);
  if (!flag) { fprintf(stderr, "mpi shim: wait on a receive nobody sends to\n"); abort(); }
  return 0;
}
inline int MPI_Waitall(int n, MPI_Request* rq, MPI_Status* st) {
  for (int i = 0; i < n; ++i) MPI_Wait(&rq[i], st ? &st[i] : MPI_STATUS_IGNORE);
  return 0;
}
inline int MPI_Testall(int n, MPI_Request* rq, int* flag, MPI_Status* st) {
  shim_match();
  *flag = 1;
  for (int i = 0; i < n; ++i) if (rq[i] != MPI_REQUEST_NULL && !rq[i]->done) *flag = 0;
  if (*flag)
    for (int i = 0; i < n; ++i) { int f; MPI_Test(&rq[i], &f, st ? &st[i] : MPI_STATUS_IGNORE); }
  return 0;
}
inline int MPI_Testany(int n, MPI_Request* rq, int* index, int* flag, MPI_Status* st) {
  shim_match();
  bool active = false;
  for (int i = 0; i < n; ++i) {
    if (rq[i] == MPI_REQUEST_NULL) continue;
    active = true;
    if (rq[i]->done) { *index = i; MPI_Test(&rq[i], flag, st); return 0; }
  }
  *flag = active ? 0 : 1;
  *index = MPI_UNDEFINED;
  return 0;
}
inline int MPI_Waitany(int n, MPI_Request* rq, int* index, MPI_Status* st) {
  int flag;
  MPI_Testany(n, rq, index, &flag, st);
  if (!flag) { fprintf(stderr, "mpi shim: waitany with nothing to receive\n"); abort(); }
  return 0;
}
inline int MPI_Get_count(const MPI_Status* st, MPI_Datatype t, int* count) { *count = st->shim_bytes / t->bytes; return 0; }

/* ---- MPI-IO (only reached with TMPFILE, unsupported here) ---- */
inline int MPI_File_open(MPI_Comm, const char*, int, MPI_Info, MPI_File*) {
  fprintf(stderr, "mpi shim: TMPFILE edge spill is not supported\n");
  abort();
}
inline int MPI_File_close(MPI_File*) { return 0; }
inline int MPI_File_set_atomicity(MPI_File, int) { return 0; }
inline int MPI_File_set_view(MPI_File, MPI_Offset, MPI_Datatype, MPI_Datatype, const char*, MPI_Info) { return 0; }
inline int MPI_File_set_errhandler(MPI_File, int) { return 0; }
inline int MPI_File_write_at(MPI_File, MPI_Offset, const void*, int, MPI_Datatype, MPI_Status*) { abort(); }
inline int MPI_File_iread_at(MPI_File, MPI_Offset, void*, int, MPI_Datatype, MPI_Request*) { abort(); }

#endif
