// Single-rank MPI stand-in for the reference-solver oracle build (test
// infrastructure only).  Every communicator has one member, rank 0.
//   * shared windows (MPI_Win_allocate_shared) are zero-filled heap blocks and
//     MPI_Win_shared_query hands back the same block;
//   * collectives copy send to receive buffers (MPI_IN_PLACE is a no-op);
//   * point-to-point messages go to self through a small mailbox so that an
//     Irecv/Send/Wait sequence addressed to rank 0 completes;
//   * MPI_Abort prints the reference's abort code and exits with it, so the
//     test harness can map it to the reference's error conditions.
#include "mpi.h"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <vector>

namespace {

struct WinRec {
  char *base = nullptr;
  MPI_Aint size = 0;
  int disp_unit = 1;
  bool owned = false;
  bool live = false;
};

struct PendingRecv {
  void *buf;
  size_t bytes;
  int source, tag;
  MPI_Comm comm;
  bool done;
};

struct Message {
  std::vector<char> data;
  int source, tag;
  MPI_Comm comm;
};

std::vector<WinRec> &wins() {
  static std::vector<WinRec> w(1);  // handle 0 is never used
  return w;
}
std::vector<size_t> &types() {
  // index = handle; 0 null, 1 int, 2 double, 3 char, 4 byte, 5 long, 6 float
  static std::vector<size_t> t = {0, sizeof(int), sizeof(double), 1, 1, sizeof(long), sizeof(float)};
  return t;
}
std::vector<PendingRecv> &recvs() {
  static std::vector<PendingRecv> r(1);
  return r;
}
std::vector<Message> &mailbox() {
  static std::vector<Message> m;
  return m;
}

size_t tsize(MPI_Datatype t) {
  if (t <= 0 || (size_t)t >= types().size() || types()[t] == 0) {
    std::fprintf(stderr, "mpi_shim: unknown datatype handle %d\n", t);
    std::exit(90);
  }
  return types()[t];
}

bool match(int want_src, int want_tag, MPI_Comm want_comm, int src, int tag, MPI_Comm comm) {
  return (want_src == MPI_ANY_SOURCE || want_src == src) &&
         (want_tag == MPI_ANY_TAG || want_tag == tag) && want_comm == comm;
}

}  // namespace

extern "C" {

int MPI_Init(int *, char ***) { return MPI_SUCCESS; }
int MPI_Finalize(void) { return MPI_SUCCESS; }

int MPI_Abort(MPI_Comm, int errorcode) {
  std::fflush(stdout);
  std::fprintf(stderr, "MPI_Abort(%d)\n", errorcode);
  std::fflush(stderr);
  std::exit(errorcode == 0 ? 1 : (errorcode & 0xff ? errorcode & 0xff : 1));
}

double MPI_Wtime(void) {
  timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

int MPI_Comm_size(MPI_Comm, int *size) { *size = 1; return MPI_SUCCESS; }
int MPI_Comm_rank(MPI_Comm, int *rank) { *rank = 0; return MPI_SUCCESS; }

int MPI_Comm_split(MPI_Comm, int, int, MPI_Comm *newcomm) {
  static int next = 16;
  *newcomm = next++;
  return MPI_SUCCESS;
}
int MPI_Comm_split_type(MPI_Comm, int, int, MPI_Info, MPI_Comm *newcomm) {
  static int next = 1024;
  *newcomm = next++;
  return MPI_SUCCESS;
}

int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }

int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype datatype,
                  MPI_Op, MPI_Comm) {
  if (sendbuf != MPI_IN_PLACE && count > 0)
    std::memmove(recvbuf, sendbuf, (size_t)count * tsize(datatype));
  return MPI_SUCCESS;
}
int MPI_Reduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype datatype,
               MPI_Op op, int, MPI_Comm comm) {
  return MPI_Allreduce(sendbuf, recvbuf, count, datatype, op, comm);
}
int MPI_Allgather(const void *sendbuf, int sendcount, MPI_Datatype sendtype, void *recvbuf,
                  int, MPI_Datatype, MPI_Comm) {
  if (sendbuf != MPI_IN_PLACE && sendcount > 0)
    std::memmove(recvbuf, sendbuf, (size_t)sendcount * tsize(sendtype));
  return MPI_SUCCESS;
}
int MPI_Allgatherv(const void *sendbuf, int sendcount, MPI_Datatype sendtype, void *recvbuf,
                   const int[], const int displs[], MPI_Datatype recvtype, MPI_Comm) {
  if (sendbuf != MPI_IN_PLACE && sendcount > 0)
    std::memmove((char *)recvbuf + (size_t)displs[0] * tsize(recvtype), sendbuf,
                 (size_t)sendcount * tsize(sendtype));
  return MPI_SUCCESS;
}
int MPI_Scatter(const void *sendbuf, int sendcount, MPI_Datatype sendtype, void *recvbuf,
                int, MPI_Datatype, int, MPI_Comm) {
  if (recvbuf != MPI_IN_PLACE && sendcount > 0)
    std::memmove(recvbuf, sendbuf, (size_t)sendcount * tsize(sendtype));
  return MPI_SUCCESS;
}

int MPI_Irecv(void *buf, int count, MPI_Datatype datatype, int source, int tag,
              MPI_Comm comm, MPI_Request *request) {
  size_t bytes = (size_t)count * tsize(datatype);
  auto &mb = mailbox();
  for (size_t i = 0; i < mb.size(); ++i) {
    if (match(source, tag, comm, mb[i].source, mb[i].tag, mb[i].comm)) {
      std::memcpy(buf, mb[i].data.data(), bytes < mb[i].data.size() ? bytes : mb[i].data.size());
      mb.erase(mb.begin() + (long)i);
      recvs().push_back({buf, bytes, source, tag, comm, true});
      *request = (MPI_Request)(recvs().size() - 1);
      return MPI_SUCCESS;
    }
  }
  recvs().push_back({buf, bytes, source, tag, comm, false});
  *request = (MPI_Request)(recvs().size() - 1);
  return MPI_SUCCESS;
}

int MPI_Send(const void *buf, int count, MPI_Datatype datatype, int dest, int tag,
             MPI_Comm comm) {
  if (dest != 0) {
    std::fprintf(stderr, "mpi_shim: send to rank %d in a one-rank world\n", dest);
    std::exit(91);
  }
  size_t bytes = (size_t)count * tsize(datatype);
  for (auto &r : recvs()) {
    if (r.buf && !r.done && match(r.source, r.tag, r.comm, 0, tag, comm)) {
      std::memcpy(r.buf, buf, bytes < r.bytes ? bytes : r.bytes);
      r.done = true;
      return MPI_SUCCESS;
    }
  }
  Message m;
  m.data.assign((const char *)buf, (const char *)buf + bytes);
  m.source = 0;
  m.tag = tag;
  m.comm = comm;
  mailbox().push_back(std::move(m));
  return MPI_SUCCESS;
}

int MPI_Isend(const void *buf, int count, MPI_Datatype datatype, int dest, int tag,
              MPI_Comm comm, MPI_Request *request) {
  *request = MPI_REQUEST_NULL;
  return MPI_Send(buf, count, datatype, dest, tag, comm);
}

int MPI_Wait(MPI_Request *request, MPI_Status *status) {
  if (*request != MPI_REQUEST_NULL) {
    PendingRecv &r = recvs()[(size_t)*request];
    if (!r.done) {
      std::fprintf(stderr, "mpi_shim: wait on a receive nobody sends (one-rank world)\n");
      std::exit(92);
    }
    r.buf = nullptr;
    *request = MPI_REQUEST_NULL;
  }
  if (status) status->MPI_ERROR = MPI_SUCCESS;
  return MPI_SUCCESS;
}

int MPI_Waitany(int count, MPI_Request reqs[], int *index, MPI_Status *status) {
  for (int i = 0; i < count; ++i) {
    if (reqs[i] != MPI_REQUEST_NULL) {
      *index = i;
      return MPI_Wait(&reqs[i], status);
    }
  }
  *index = MPI_UNDEFINED;
  return MPI_SUCCESS;
}

int MPI_Type_contiguous(int count, MPI_Datatype oldtype, MPI_Datatype *newtype) {
  types().push_back((size_t)count * tsize(oldtype));
  *newtype = (MPI_Datatype)(types().size() - 1);
  return MPI_SUCCESS;
}
int MPI_Type_commit(MPI_Datatype *) { return MPI_SUCCESS; }
int MPI_Type_free(MPI_Datatype *datatype) { *datatype = MPI_DATATYPE_NULL; return MPI_SUCCESS; }

int MPI_Info_create(MPI_Info *info) { *info = 1; return MPI_SUCCESS; }
int MPI_Info_set(MPI_Info, const char *, const char *) { return MPI_SUCCESS; }
int MPI_Info_free(MPI_Info *info) { *info = MPI_INFO_NULL; return MPI_SUCCESS; }

int MPI_Win_allocate_shared(MPI_Aint size, int disp_unit, MPI_Info, MPI_Comm, void *baseptr,
                            MPI_Win *win) {
  WinRec w;
  w.size = size;
  w.disp_unit = disp_unit;
  w.base = (char *)std::calloc(size > 0 ? (size_t)size : 1, 1);
  if (!w.base) {
    std::fprintf(stderr, "mpi_shim: out of memory allocating %ld bytes\n", (long)size);
    std::exit(93);
  }
  w.owned = true;
  w.live = true;
  wins().push_back(w);
  *win = (MPI_Win)(wins().size() - 1);
  *(void **)baseptr = w.base;
  return MPI_SUCCESS;
}

int MPI_Win_shared_query(MPI_Win win, int, MPI_Aint *size, int *disp_unit, void *baseptr) {
  const WinRec &w = wins()[(size_t)win];
  *size = w.size;
  *disp_unit = w.disp_unit;
  *(void **)baseptr = w.base;
  return MPI_SUCCESS;
}

int MPI_Win_create(void *base, MPI_Aint size, int disp_unit, MPI_Info, MPI_Comm, MPI_Win *win) {
  WinRec w;
  w.base = (char *)base;
  w.size = size;
  w.disp_unit = disp_unit;
  w.owned = false;
  w.live = true;
  wins().push_back(w);
  *win = (MPI_Win)(wins().size() - 1);
  return MPI_SUCCESS;
}

int MPI_Win_free(MPI_Win *win) {
  if (*win > 0 && (size_t)*win < wins().size()) {
    WinRec &w = wins()[(size_t)*win];
    if (w.live && w.owned) std::free(w.base);
    w.base = nullptr;
    w.live = false;
  }
  *win = 0;
  return MPI_SUCCESS;
}

int MPI_Win_fence(int, MPI_Win) { return MPI_SUCCESS; }
int MPI_Win_lock_all(int, MPI_Win) { return MPI_SUCCESS; }
int MPI_Win_unlock_all(MPI_Win) { return MPI_SUCCESS; }
int MPI_Win_flush_all(MPI_Win) { return MPI_SUCCESS; }

int MPI_Get(void *origin_addr, int origin_count, MPI_Datatype origin_datatype, int,
            MPI_Aint target_disp, int, MPI_Datatype, MPI_Win win) {
  const WinRec &w = wins()[(size_t)win];
  std::memcpy(origin_addr, w.base + (size_t)target_disp * (size_t)w.disp_unit,
              (size_t)origin_count * tsize(origin_datatype));
  return MPI_SUCCESS;
}

}  // extern "C"
