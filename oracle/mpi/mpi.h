/*
 * Test-infrastructure only: a single-node, fork-based stand-in for the subset of
 * MPI that the GIP reference sources call, so that the reference CPU path can be
 * compiled unmodified and run at 1..P ranks on one host without an MPI install.
 *
 * Calls covered (all that appear in GIP's sources):
 *   MPI_Init_thread, MPI_Comm_rank, MPI_Comm_size, MPI_Isend, MPI_Irecv, MPI_Wait,
 *   MPI_Allreduce (SUM/MIN/MAX on one double or float), MPI_Barrier, MPI_Finalize.
 *
 * Ranks: GIPSHIM_NP (default 1) processes are forked inside MPI_Init_thread; they
 * share one anonymous MAP_SHARED region.  Point-to-point messages go through one
 * mailbox per ordered (src,dst) pair of GIPSHIM_SLOT_MB megabytes (default 8).
 * MPI_Allreduce reduces in rank order 0..P-1 on every rank, so all ranks see the
 * same bits.  MPI_Comm_size returns MPI_SUCCESS (0): GIP's GIP_VectorMulticore::dot
 * assigns that return value to its size variable (GIP_VectorMulticore.cpp:97).
 *
 * This header is never linked into the product library; it is only used by the
 * oracle build recipe (oracle/Makefile) to run the reference's own CPU code.
 */
#ifndef GIPSHIM_MPI_H
#define GIPSHIM_MPI_H

#include <sched.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>
#include <sys/wait.h>
#include <unistd.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef struct { int source, tag, error; } MPI_Status;
typedef struct { int kind, peer, bytes; void* buf; } MPI_Request;

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_THREAD_SINGLE 0
#define MPI_DOUBLE 8
#define MPI_FLOAT 4
#define MPI_SUM 1
#define MPI_MIN 2
#define MPI_MAX 3

namespace gipshim {

enum { kMaxRanks = 256 };

struct Control {
  volatile int barrier_count;
  volatile int barrier_sense;
  double reduce_slot[kMaxRanks];
};

struct MailboxHeader {
  volatile long posted;    /* messages written by the sender   */
  volatile long consumed;  /* messages read by the receiver    */
  volatile int bytes;
};

struct State {
  int rank = 0;
  int size = 1;
  int local_sense = 0;
  size_t slot_bytes = 0;
  Control* ctl = nullptr;
  char* mail = nullptr;
};

inline State& st() {
  static State s;
  return s;
}

inline size_t mailbox_stride() { return sizeof(MailboxHeader) + st().slot_bytes; }

inline MailboxHeader* mailbox(int src, int dst) {
  return reinterpret_cast<MailboxHeader*>(st().mail +
                                          ((size_t)src * st().size + dst) * mailbox_stride());
}

inline void relax() { sched_yield(); }

inline void barrier() {
  State& s = st();
  if (s.size == 1) return;
  s.local_sense = !s.local_sense;
  if (__sync_add_and_fetch(&s.ctl->barrier_count, 1) == s.size) {
    s.ctl->barrier_count = 0;
    __sync_synchronize();
    s.ctl->barrier_sense = s.local_sense;
  } else {
    while (s.ctl->barrier_sense != s.local_sense) relax();
  }
  __sync_synchronize();
}

}  // namespace gipshim

inline int MPI_Init_thread(int*, char***, int, int* provided) {
  using namespace gipshim;
  State& s = st();
  const char* np = getenv("GIPSHIM_NP");
  s.size = np ? atoi(np) : 1;
  if (s.size < 1 || s.size > kMaxRanks) {
    fprintf(stderr, "gipshim: GIPSHIM_NP must be in [1,%d]\n", kMaxRanks);
    exit(2);
  }
  const char* mb = getenv("GIPSHIM_SLOT_MB");
  s.slot_bytes = (size_t)(mb ? atoi(mb) : 8) << 20;
  size_t mail_bytes = (size_t)s.size * s.size * mailbox_stride();
  size_t total = sizeof(Control) + mail_bytes;
  void* p = mmap(nullptr, total, PROT_READ | PROT_WRITE,
                 MAP_SHARED | MAP_ANONYMOUS | MAP_NORESERVE, -1, 0);
  if (p == MAP_FAILED) {
    perror("gipshim: mmap");
    exit(2);
  }
  s.ctl = reinterpret_cast<Control*>(p);
  s.mail = reinterpret_cast<char*>(p) + sizeof(Control);
  fflush(stdout);
  fflush(stderr);
  for (int r = 1; r < s.size; ++r) {
    pid_t pid = fork();
    if (pid < 0) {
      perror("gipshim: fork");
      exit(2);
    }
    if (pid == 0) {
      s.rank = r;
      break;
    }
  }
  if (provided) *provided = MPI_THREAD_SINGLE;
  return MPI_SUCCESS;
}

inline int MPI_Init(int* argc, char*** argv) {
  int prov;
  return MPI_Init_thread(argc, argv, MPI_THREAD_SINGLE, &prov);
}

inline int MPI_Comm_rank(MPI_Comm, int* r) {
  *r = gipshim::st().rank;
  return MPI_SUCCESS;
}

inline int MPI_Comm_size(MPI_Comm, int* n) {
  *n = gipshim::st().size;
  return MPI_SUCCESS;
}

inline int MPI_Isend(const void* buf, int count, MPI_Datatype type, int dest, int, MPI_Comm,
                     MPI_Request* req) {
  using namespace gipshim;
  size_t bytes = (size_t)count * (size_t)type;
  if (bytes > st().slot_bytes) {
    fprintf(stderr, "gipshim: message of %zu bytes exceeds GIPSHIM_SLOT_MB\n", bytes);
    exit(2);
  }
  MailboxHeader* m = mailbox(st().rank, dest);
  while (m->posted != m->consumed) relax();
  memcpy(reinterpret_cast<char*>(m) + sizeof(MailboxHeader), buf, bytes);
  m->bytes = (int)bytes;
  __sync_synchronize();
  m->posted = m->posted + 1;
  req->kind = 0;
  return MPI_SUCCESS;
}

inline int MPI_Irecv(void* buf, int count, MPI_Datatype type, int source, int, MPI_Comm,
                     MPI_Request* req) {
  req->kind = 1;
  req->peer = source;
  req->bytes = count * type;
  req->buf = buf;
  return MPI_SUCCESS;
}

inline int MPI_Wait(MPI_Request* req, MPI_Status*) {
  using namespace gipshim;
  if (req->kind != 1) return MPI_SUCCESS;
  MailboxHeader* m = mailbox(req->peer, st().rank);
  while (m->posted == m->consumed) relax();
  __sync_synchronize();
  memcpy(req->buf, reinterpret_cast<char*>(m) + sizeof(MailboxHeader), (size_t)req->bytes);
  __sync_synchronize();
  m->consumed = m->consumed + 1;
  return MPI_SUCCESS;
}

inline int MPI_Allreduce(const void* in, void* out, int count, MPI_Datatype type, MPI_Op op,
                         MPI_Comm) {
  using namespace gipshim;
  State& s = st();
  if (count != 1) {
    fprintf(stderr, "gipshim: MPI_Allreduce supports count==1 only\n");
    exit(2);
  }
  double v = (type == MPI_DOUBLE) ? *(const double*)in : (double)*(const float*)in;
  s.ctl->reduce_slot[s.rank] = v;
  barrier();
  double acc = s.ctl->reduce_slot[0];
  for (int r = 1; r < s.size; ++r) {
    double x = s.ctl->reduce_slot[r];
    if (op == MPI_SUM)
      acc = acc + x;
    else if (op == MPI_MIN)
      acc = (x < acc) ? x : acc;
    else
      acc = (x > acc) ? x : acc;
  }
  barrier();
  if (type == MPI_DOUBLE)
    *(double*)out = acc;
  else
    *(float*)out = (float)acc;
  return MPI_SUCCESS;
}

inline int MPI_Barrier(MPI_Comm) {
  gipshim::barrier();
  return MPI_SUCCESS;
}

inline int MPI_Finalize() {
  using namespace gipshim;
  State& s = st();
  fflush(stdout);
  fflush(stderr);
  barrier();
  if (s.rank != 0) _exit(0);
  int status = 0;
  for (int r = 1; r < s.size; ++r) wait(&status);
  return MPI_SUCCESS;
}

#endif /* GIPSHIM_MPI_H */
