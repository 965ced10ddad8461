// MPI stand-in for the reference-solver oracle build (test infrastructure
// only; never linked into the GPU library).
//
// One rank (the default): every communicator has one member, rank 0.
//   * shared windows (MPI_Win_allocate_shared) are zero-filled heap blocks and
//     MPI_Win_shared_query hands back the same block;
//   * collectives copy send to receive buffers (MPI_IN_PLACE is a no-op);
//   * point-to-point messages go to self through a small mailbox so that an
//     Irecv/Send/Wait sequence addressed to rank 0 completes;
//   * MPI_Abort prints the reference's abort code and exits with it, so the
//     test harness can map it to the reference's error conditions.
//
// IB_RANKS=N (N > 1): one shared-memory node of N processes, the reference's
// own intra-node MPI-3 mode (every rank in one share_comm; SHN, the ranks
// per node, is ib_shim_ranks() = N, mpiparams.cpp:68-105).  MPI_Init maps one
// shared anonymous arena and forks ranks 1..N-1 from the calling process
// (rank 0), so the arena sits at the same address in every rank.  In it:
//   * communicator records: members (world ranks in rank order) and a
//     sense-counting barrier; MPI_Comm_split gathers (color, key) pairs and
//     rank 0 of the parent lays out the new records;
//   * one staging buffer per rank: collectives copy their data through it in
//     chunks, each phase closed by a barrier, and reduce in rank order, so
//     every rank gets the same bits;
//   * shared windows: one contiguous block per window (rank r's segment at
//     the sum of the lower ranks' sizes, the layout DataArray.H indexes from
//     rank 0's base), first-fit allocated under a lock by rank 0 of the
//     window's communicator, zero-filled, pages returned on MPI_Win_free.
// Every wait spins with a bounded total time (IB_MPI_TIMEOUT seconds,
// default 1800) and gives up with exit code 96; an MPI_Abort anywhere ends
// every rank with the abort code; a rank that ends without MPI_Finalize ends
// the others (rank 0 watches its children, the children die with rank 0).
// Point-to-point messages only ever go to self: the reference sends them over
// nodecomm, one rank per node here.
#include "mpi.h"

#include <sched.h>
#include <signal.h>
#include <sys/mman.h>
#include <sys/prctl.h>
#include <sys/wait.h>
#include <unistd.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <map>
#include <vector>

namespace {

// ---------------------------------------------------------------- datatypes

struct TypeRec {
  size_t bytes;
  int base;  // predefined handle of the element type (reductions)
};

std::vector<TypeRec> &types() {
  // index = handle; 0 null, 1 int, 2 double, 3 char, 4 byte, 5 long, 6 float
  static std::vector<TypeRec> t = {{0, 0},           {sizeof(int), 1},  {sizeof(double), 2},
                                   {1, 3},           {1, 4},            {sizeof(long), 5},
                                   {sizeof(float), 6}};
  return t;
}

size_t tsize(MPI_Datatype t) {
  if (t <= 0 || (size_t)t >= types().size() || types()[t].bytes == 0) {
    std::fprintf(stderr, "mpi_shim: unknown datatype handle %d\n", t);
    std::exit(90);
  }
  return types()[t].bytes;
}

double now_s() {
  timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

// ---------------------------------------------------------- one-rank state

struct WinRec {
  char *base = nullptr;       // this rank's segment
  char *block = nullptr;      // the whole window (rank 0's segment first)
  MPI_Aint size = 0;          // this rank's segment bytes
  int disp_unit = 1;
  bool owned = false;
  bool live = false;
  MPI_Comm comm = 0;
  long long arena_off = -1;   // shared block offset (several ranks)
  std::vector<MPI_Aint> seg;  // every member's segment bytes (several ranks)
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
std::vector<PendingRecv> &recvs() {
  static std::vector<PendingRecv> r(1);
  return r;
}
std::vector<Message> &mailbox() {
  static std::vector<Message> m;
  return m;
}

bool match(int want_src, int want_tag, MPI_Comm want_comm, int src, int tag, MPI_Comm comm) {
  return (want_src == MPI_ANY_SOURCE || want_src == src) &&
         (want_tag == MPI_ANY_TAG || want_tag == tag) && want_comm == comm;
}

// ------------------------------------------------------ shared-memory node

constexpr int kMaxRanks = 256;
constexpr int kMaxComms = 256;
constexpr int kMaxBlocks = 1 << 16;
constexpr size_t kStageBytes = size_t(4) << 20;  // per rank
constexpr size_t kPage = 4096;

struct CommRec {
  int size;
  int members[kMaxRanks];        // world rank of member i
  alignas(64) unsigned count;    // barrier arrivals
  alignas(64) unsigned gen;      // barrier generation
  alignas(64) long long word;    // rank 0 -> members (split base, window offset)
};

struct Block {
  long long off, bytes;
  int used;
};

struct Node {
  int nranks;
  int abort_code;  // 0 while every rank runs
  int next_comm;
  int lock;        // allocator lock
  int nblocks;
  long long heap_off, arena_bytes;
  pid_t pids[kMaxRanks];
  Block blocks[kMaxBlocks];  // sorted by offset, covering the heap
  CommRec comms[kMaxComms];
};

Node *g_node = nullptr;  // null in the one-rank build
char *g_arena = nullptr;
int g_rank = 0;
int g_nranks = 1;
double g_timeout = 1800.0;
bool g_finalized = false;

struct LocalComm {
  int slot;  // CommRec index; -1 for MPI_COMM_SELF
  int rank;
  int size;
};
std::map<int, LocalComm> &comms() {
  static std::map<int, LocalComm> c;
  return c;
}

[[noreturn]] void die(int code, const char *why) {
  if (g_node) {
    int zero = 0;
    __atomic_compare_exchange_n(&g_node->abort_code, &zero, code, false, __ATOMIC_SEQ_CST,
                                __ATOMIC_SEQ_CST);
  }
  std::fflush(stdout);
  std::fprintf(stderr, "mpi_shim rank %d: %s\n", g_rank, why);
  std::fflush(stderr);
  _exit(code & 0xff ? code & 0xff : 1);
}

// rank 0: a child that ended before MPI_Finalize ends the node
void watch_children() {
  if (g_rank != 0 || g_finalized) return;
  for (int r = 1; r < g_nranks; ++r) {
    int st = 0;
    if (g_node->pids[r] > 0 && waitpid(g_node->pids[r], &st, WNOHANG) == g_node->pids[r]) {
      g_node->pids[r] = -1;
      char msg[96];
      std::snprintf(msg, sizeof msg, "rank %d ended before MPI_Finalize (status %d)", r, st);
      die(WIFEXITED(st) && WEXITSTATUS(st) ? WEXITSTATUS(st) : 97, msg);
    }
  }
}

template <class Pred>
void wait_until(Pred done) {
  const double t0 = now_s();
  for (long it = 0;; ++it) {
    if (done()) return;
    if ((it & 255) == 255) {
      const int code = __atomic_load_n(&g_node->abort_code, __ATOMIC_ACQUIRE);
      if (code) {
        std::fflush(stdout);
        _exit(code & 0xff ? code & 0xff : 1);
      }
      watch_children();
      if (now_s() - t0 > g_timeout) die(96, "wait timed out (IB_MPI_TIMEOUT)");
    }
    if (it < 4096) __builtin_ia32_pause();
    else sched_yield();
  }
}

const LocalComm &local(MPI_Comm c) {
  auto it = comms().find(c);
  if (it == comms().end()) {
    char msg[64];
    std::snprintf(msg, sizeof msg, "unknown communicator %d", c);
    die(90, msg);
  }
  return it->second;
}

void barrier(const LocalComm &lc) {
  if (lc.size == 1) return;
  CommRec &c = g_node->comms[lc.slot];
  const unsigned gen = __atomic_load_n(&c.gen, __ATOMIC_ACQUIRE);
  if (__atomic_add_fetch(&c.count, 1u, __ATOMIC_ACQ_REL) == (unsigned)lc.size) {
    __atomic_store_n(&c.count, 0u, __ATOMIC_RELAXED);
    __atomic_store_n(&c.gen, gen + 1, __ATOMIC_RELEASE);
  } else {
    wait_until([&] { return __atomic_load_n(&c.gen, __ATOMIC_ACQUIRE) != gen; });
  }
}

char *stage(int world_rank) {
  return g_arena + sizeof(Node) + (size_t)world_rank * kStageBytes;
}
int member(const LocalComm &lc, int r) { return g_node->comms[lc.slot].members[r]; }

// first-fit allocation of the shared heap (callers hold no lock)
void lock() {
  wait_until([] {
    int z = 0;
    return __atomic_compare_exchange_n(&g_node->lock, &z, 1, false, __ATOMIC_ACQUIRE,
                                       __ATOMIC_RELAXED);
  });
}
void unlock() { __atomic_store_n(&g_node->lock, 0, __ATOMIC_RELEASE); }

long long heap_alloc(long long bytes) {
  bytes = (long long)(((size_t)(bytes > 0 ? bytes : 1) + kPage - 1) / kPage * kPage);
  lock();
  Node &n = *g_node;
  for (int i = 0; i < n.nblocks; ++i) {
    Block &b = n.blocks[i];
    if (b.used || b.bytes < bytes) continue;
    if (b.bytes > bytes) {
      if (n.nblocks == kMaxBlocks) break;
      std::memmove(&n.blocks[i + 2], &n.blocks[i + 1], sizeof(Block) * (size_t)(n.nblocks - i - 1));
      n.blocks[i + 1] = {b.off + bytes, b.bytes - bytes, 0};
      ++n.nblocks;
      b.bytes = bytes;
    }
    b.used = 1;
    const long long off = b.off;
    unlock();
    return off;
  }
  unlock();
  die(93, "shared arena exhausted (IB_MPI_ARENA_GB)");
}

void heap_free(long long off) {
  lock();
  Node &n = *g_node;
  int i = 0;
  while (i < n.nblocks && n.blocks[i].off != off) ++i;
  if (i == n.nblocks || !n.blocks[i].used) {
    unlock();
    die(94, "free of an unknown shared block");
  }
  // hand the pages back; a later block reads zeros there
  madvise(g_arena + off, (size_t)n.blocks[i].bytes, MADV_REMOVE);
  n.blocks[i].used = 0;
  if (i + 1 < n.nblocks && !n.blocks[i + 1].used) {
    n.blocks[i].bytes += n.blocks[i + 1].bytes;
    std::memmove(&n.blocks[i + 1], &n.blocks[i + 2], sizeof(Block) * (size_t)(n.nblocks - i - 2));
    --n.nblocks;
  }
  if (i > 0 && !n.blocks[i - 1].used) {
    n.blocks[i - 1].bytes += n.blocks[i].bytes;
    std::memmove(&n.blocks[i], &n.blocks[i + 1], sizeof(Block) * (size_t)(n.nblocks - i - 1));
    --n.nblocks;
  }
  unlock();
}

// element-wise reduction of `count` elements of predefined type `base`
template <class T>
void reduce_into(T *acc, const T *v, size_t count, MPI_Op op) {
  for (size_t i = 0; i < count; ++i) {
    if (op == MPI_SUM) acc[i] = acc[i] + v[i];
    else if (op == MPI_MAX) acc[i] = v[i] > acc[i] ? v[i] : acc[i];
    else if (op == MPI_MIN) acc[i] = v[i] < acc[i] ? v[i] : acc[i];
    else die(90, "unsupported reduction op");
  }
}
void reduce_any(void *acc, const void *v, size_t bytes, MPI_Datatype t, MPI_Op op) {
  switch (types()[t].base) {
    case 1: reduce_into((int *)acc, (const int *)v, bytes / sizeof(int), op); break;
    case 2: reduce_into((double *)acc, (const double *)v, bytes / sizeof(double), op); break;
    case 5: reduce_into((long *)acc, (const long *)v, bytes / sizeof(long), op); break;
    case 6: reduce_into((float *)acc, (const float *)v, bytes / sizeof(float), op); break;
    default: die(90, "reduction over a datatype without arithmetic");
  }
}

// world size from IB_RANKS (1 when unset)
int env_ranks() {
  const char *s = std::getenv("IB_RANKS");
  const int n = (s && *s) ? std::atoi(s) : 1;
  return n < 1 ? 1 : n;
}

void start_node(int n) {
  if (n > kMaxRanks) die(90, "IB_RANKS above the shim's limit");
  if (const char *t = std::getenv("IB_MPI_TIMEOUT")) g_timeout = std::atof(t);
  size_t arena = (size_t)sysconf(_SC_PHYS_PAGES) * (size_t)sysconf(_SC_PAGE_SIZE);
  if (const char *g = std::getenv("IB_MPI_ARENA_GB")) arena = (size_t)(std::atof(g) * 1073741824.0);
  const size_t head = ((sizeof(Node) + (size_t)n * kStageBytes) + kPage - 1) / kPage * kPage;
  if (arena < head + (size_t(64) << 20)) arena = head + (size_t(64) << 20);
  void *p = mmap(nullptr, arena, PROT_READ | PROT_WRITE, MAP_SHARED | MAP_ANONYMOUS | MAP_NORESERVE,
                 -1, 0);
  if (p == MAP_FAILED) die(93, "cannot map the shared arena");
  g_arena = (char *)p;
  g_node = (Node *)p;
  g_nranks = n;
  Node &s = *g_node;
  s.nranks = n;
  s.heap_off = (long long)head;
  s.arena_bytes = (long long)arena;
  s.nblocks = 1;
  s.blocks[0] = {s.heap_off, s.arena_bytes - s.heap_off, 0};
  // record 1: MPI_COMM_WORLD
  s.comms[1].size = n;
  for (int r = 0; r < n; ++r) s.comms[1].members[r] = r;
  s.next_comm = 3;
  s.pids[0] = getpid();
  std::fflush(nullptr);
  const pid_t parent = getpid();
  for (int r = 1; r < n; ++r) {
    const pid_t pid = fork();
    if (pid < 0) die(95, "fork failed");
    if (pid == 0) {
      prctl(PR_SET_PDEATHSIG, SIGKILL);
      if (getppid() != parent) _exit(97);
      g_rank = r;
      break;
    }
    s.pids[r] = pid;
  }
}

}  // namespace

extern "C" {

int ib_shim_ranks(void) { return g_nranks; }

int MPI_Init(int *, char ***) {
  const int n = env_ranks();
  if (n > 1) start_node(n);
  comms()[MPI_COMM_WORLD] = {1, g_rank, g_nranks};
  comms()[MPI_COMM_SELF] = {-1, 0, 1};
  return MPI_SUCCESS;
}

int MPI_Finalize(void) {
  if (!g_node) return MPI_SUCCESS;
  barrier(local(MPI_COMM_WORLD));
  g_finalized = true;
  std::fflush(nullptr);
  if (g_rank == 0) {
    int worst = 0;
    for (int r = 1; r < g_nranks; ++r) {
      int st = 0;
      if (g_node->pids[r] > 0 && waitpid(g_node->pids[r], &st, 0) == g_node->pids[r]) {
        const int code = WIFEXITED(st) ? WEXITSTATUS(st) : 97;
        if (code && !worst) worst = code;
      }
    }
    if (worst) {
      std::fprintf(stderr, "mpi_shim: a rank ended with status %d\n", worst);
      std::exit(worst);
    }
  }
  return MPI_SUCCESS;
}

int MPI_Abort(MPI_Comm, int errorcode) {
  std::fflush(stdout);
  std::fprintf(stderr, "MPI_Abort(%d)\n", errorcode);
  std::fflush(stderr);
  const int code = errorcode == 0 ? 1 : (errorcode & 0xff ? errorcode & 0xff : 1);
  if (g_node) {
    int zero = 0;
    __atomic_compare_exchange_n(&g_node->abort_code, &zero, code, false, __ATOMIC_SEQ_CST,
                                __ATOMIC_SEQ_CST);
    _exit(code);
  }
  std::exit(code);
}

double MPI_Wtime(void) { return now_s(); }

int MPI_Comm_size(MPI_Comm comm, int *size) {
  *size = g_node ? local(comm).size : 1;
  return MPI_SUCCESS;
}
int MPI_Comm_rank(MPI_Comm comm, int *rank) {
  *rank = g_node ? local(comm).rank : 0;
  return MPI_SUCCESS;
}

int MPI_Comm_split(MPI_Comm comm, int color, int key, MPI_Comm *newcomm) {
  if (!g_node) {
    static int next = 16;
    *newcomm = color == MPI_UNDEFINED ? MPI_COMM_NULL : next++;
    return MPI_SUCCESS;
  }
  const LocalComm &pc = local(comm);
  if (pc.slot < 0) {  // a split of MPI_COMM_SELF
    if (color == MPI_UNDEFINED) {
      *newcomm = MPI_COMM_NULL;
      return MPI_SUCCESS;
    }
    const int slot = __atomic_fetch_add(&g_node->next_comm, 1, __ATOMIC_ACQ_REL);
    if (slot >= kMaxComms) die(90, "too many communicators");
    g_node->comms[slot].size = 1;
    g_node->comms[slot].members[0] = g_rank;
    comms()[slot] = {slot, 0, 1};
    *newcomm = slot;
    return MPI_SUCCESS;
  }
  CommRec &parent = g_node->comms[pc.slot];
  int *mine = (int *)stage(g_rank);
  mine[0] = color;
  mine[1] = key;
  barrier(pc);
  // the members' (color, key, parent rank), read by every rank alike
  std::vector<int> colors;
  std::vector<int> col(pc.size), keys(pc.size);
  for (int r = 0; r < pc.size; ++r) {
    const int *o = (const int *)stage(member(pc, r));
    col[r] = o[0];
    keys[r] = o[1];
    if (o[0] != MPI_UNDEFINED &&
        std::find(colors.begin(), colors.end(), o[0]) == colors.end())
      colors.push_back(o[0]);
  }
  std::sort(colors.begin(), colors.end());
  if (pc.rank == 0) {
    const int base = __atomic_fetch_add(&g_node->next_comm, (int)colors.size(), __ATOMIC_ACQ_REL);
    if (base + (int)colors.size() > kMaxComms) die(90, "too many communicators");
    for (size_t c = 0; c < colors.size(); ++c) {
      std::vector<int> who;
      for (int r = 0; r < pc.size; ++r)
        if (col[r] == colors[c]) who.push_back(r);
      std::stable_sort(who.begin(), who.end(), [&](int a, int b) { return keys[a] < keys[b]; });
      CommRec &nc = g_node->comms[base + (int)c];
      nc.size = (int)who.size();
      for (size_t i = 0; i < who.size(); ++i) nc.members[i] = member(pc, who[i]);
      nc.count = 0;
      nc.gen = 0;
    }
    __atomic_store_n(&parent.word, (long long)base, __ATOMIC_RELEASE);
  }
  barrier(pc);
  const int base = (int)__atomic_load_n(&parent.word, __ATOMIC_ACQUIRE);
  barrier(pc);  // every member has its (color, key) and the base read
  if (color == MPI_UNDEFINED) {
    *newcomm = MPI_COMM_NULL;
    return MPI_SUCCESS;
  }
  const int slot = base + (int)(std::find(colors.begin(), colors.end(), color) - colors.begin());
  const CommRec &nc = g_node->comms[slot];
  int me = 0;
  while (nc.members[me] != g_rank) ++me;
  comms()[slot] = {slot, me, nc.size};
  *newcomm = slot;
  return MPI_SUCCESS;
}

int MPI_Comm_split_type(MPI_Comm comm, int, int key, MPI_Info, MPI_Comm *newcomm) {
  if (!g_node) {
    static int next = 1024;
    *newcomm = next++;
    return MPI_SUCCESS;
  }
  return MPI_Comm_split(comm, 0, key, newcomm);  // one shared-memory node
}

int MPI_Barrier(MPI_Comm comm) {
  if (g_node) barrier(local(comm));
  return MPI_SUCCESS;
}

int MPI_Bcast(void *buffer, int count, MPI_Datatype datatype, int root, MPI_Comm comm) {
  if (!g_node) return MPI_SUCCESS;
  const LocalComm &lc = local(comm);
  if (lc.size == 1) return MPI_SUCCESS;
  const size_t bytes = (size_t)count * tsize(datatype);
  for (size_t o = 0; o < bytes || o == 0; o += kStageBytes) {
    const size_t n = bytes - o < kStageBytes ? bytes - o : kStageBytes;
    if (lc.rank == root && n) std::memcpy(stage(g_rank), (char *)buffer + o, n);
    barrier(lc);
    if (lc.rank != root && n) std::memcpy((char *)buffer + o, stage(member(lc, root)), n);
    barrier(lc);
    if (bytes == 0) break;
  }
  return MPI_SUCCESS;
}

int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype datatype,
                  MPI_Op op, MPI_Comm comm) {
  const size_t bytes = (size_t)count * tsize(datatype);
  if (sendbuf != MPI_IN_PLACE && bytes > 0) std::memmove(recvbuf, sendbuf, bytes);
  if (!g_node) return MPI_SUCCESS;
  const LocalComm &lc = local(comm);
  if (lc.size == 1) return MPI_SUCCESS;
  const size_t esz = tsize(types()[datatype].base);
  const size_t chunk = kStageBytes / esz * esz;
  std::vector<char> acc;
  for (size_t o = 0; o < bytes; o += chunk) {
    const size_t n = bytes - o < chunk ? bytes - o : chunk;
    std::memcpy(stage(g_rank), (char *)recvbuf + o, n);
    barrier(lc);
    // rank order: every member combines the same values the same way
    acc.assign(stage(member(lc, 0)), stage(member(lc, 0)) + n);
    for (int r = 1; r < lc.size; ++r) reduce_any(acc.data(), stage(member(lc, r)), n, datatype, op);
    barrier(lc);
    std::memcpy((char *)recvbuf + o, acc.data(), n);
  }
  return MPI_SUCCESS;
}

int MPI_Reduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype datatype,
               MPI_Op op, int root, MPI_Comm comm) {
  if (!g_node || local(comm).size == 1)
    return MPI_Allreduce(sendbuf, recvbuf, count, datatype, op, comm);
  const size_t bytes = (size_t)count * tsize(datatype);
  std::vector<char> tmp(bytes);
  if (bytes) std::memcpy(tmp.data(), sendbuf == MPI_IN_PLACE ? recvbuf : sendbuf, bytes);
  MPI_Allreduce(MPI_IN_PLACE, tmp.data(), count, datatype, op, comm);
  if (local(comm).rank == root && bytes) std::memcpy(recvbuf, tmp.data(), bytes);
  return MPI_SUCCESS;
}

int MPI_Allgatherv(const void *sendbuf, int sendcount, MPI_Datatype sendtype, void *recvbuf,
                   const int recvcounts[], const int displs[], MPI_Datatype recvtype,
                   MPI_Comm comm) {
  const size_t rsz = tsize(recvtype);
  if (!g_node || local(comm).size == 1) {
    if (sendbuf != MPI_IN_PLACE && sendcount > 0)
      std::memmove((char *)recvbuf + (size_t)displs[0] * rsz, sendbuf,
                   (size_t)sendcount * tsize(sendtype));
    return MPI_SUCCESS;
  }
  const LocalComm &lc = local(comm);
  const char *src = sendbuf == MPI_IN_PLACE ? (const char *)recvbuf + (size_t)displs[lc.rank] * rsz
                                            : (const char *)sendbuf;
  const size_t mine = sendbuf == MPI_IN_PLACE ? (size_t)recvcounts[lc.rank] * rsz
                                              : (size_t)sendcount * tsize(sendtype);
  size_t most = 0;
  for (int r = 0; r < lc.size; ++r)
    most = (size_t)recvcounts[r] * rsz > most ? (size_t)recvcounts[r] * rsz : most;
  for (size_t o = 0; o < most; o += kStageBytes) {
    if (o < mine) std::memcpy(stage(g_rank), src + o, mine - o < kStageBytes ? mine - o : kStageBytes);
    barrier(lc);
    for (int r = 0; r < lc.size; ++r) {
      const size_t have = (size_t)recvcounts[r] * rsz;
      if (r == lc.rank && sendbuf == MPI_IN_PLACE) continue;
      if (o < have)
        std::memcpy((char *)recvbuf + (size_t)displs[r] * rsz + o, stage(member(lc, r)),
                    have - o < kStageBytes ? have - o : kStageBytes);
    }
    barrier(lc);
  }
  return MPI_SUCCESS;
}

int MPI_Allgather(const void *sendbuf, int sendcount, MPI_Datatype sendtype, void *recvbuf,
                  int recvcount, MPI_Datatype recvtype, MPI_Comm comm) {
  if (!g_node || local(comm).size == 1) {
    if (sendbuf != MPI_IN_PLACE && sendcount > 0)
      std::memmove(recvbuf, sendbuf, (size_t)sendcount * tsize(sendtype));
    return MPI_SUCCESS;
  }
  const LocalComm &lc = local(comm);
  std::vector<int> counts(lc.size, recvcount), displs(lc.size);
  for (int r = 0; r < lc.size; ++r) displs[r] = r * recvcount;
  return MPI_Allgatherv(sendbuf, sendcount, sendtype, recvbuf, counts.data(), displs.data(),
                        recvtype, comm);
}

int MPI_Scatter(const void *sendbuf, int sendcount, MPI_Datatype sendtype, void *recvbuf,
                int recvcount, MPI_Datatype recvtype, int root, MPI_Comm comm) {
  if (!g_node || local(comm).size == 1) {
    if (recvbuf != MPI_IN_PLACE && sendcount > 0)
      std::memmove(recvbuf, sendbuf, (size_t)sendcount * tsize(sendtype));
    return MPI_SUCCESS;
  }
  const LocalComm &lc = local(comm);
  const size_t each = (size_t)sendcount * tsize(sendtype);
  const size_t want = (size_t)recvcount * tsize(recvtype);
  for (size_t o = 0; o < each || o == 0; o += kStageBytes) {
    const size_t n = each - o < kStageBytes ? each - o : kStageBytes;
    barrier(lc);  // every member is done with its own staging buffer
    if (lc.rank == root && n)
      for (int r = 0; r < lc.size; ++r)
        std::memcpy(stage(member(lc, r)), (const char *)sendbuf + (size_t)r * each + o, n);
    barrier(lc);
    if (recvbuf != MPI_IN_PLACE && o < want)
      std::memcpy((char *)recvbuf + o, stage(g_rank), want - o < n ? want - o : n);
    if (each == 0) break;
  }
  barrier(lc);
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
  int me = 0;
  MPI_Comm_rank(comm, &me);
  if (dest != me) {
    std::fprintf(stderr, "mpi_shim: send from rank %d to rank %d (messages only go to self)\n",
                 me, dest);
    std::exit(91);
  }
  size_t bytes = (size_t)count * tsize(datatype);
  for (auto &r : recvs()) {
    if (r.buf && !r.done && match(r.source, r.tag, r.comm, me, tag, comm)) {
      std::memcpy(r.buf, buf, bytes < r.bytes ? bytes : r.bytes);
      r.done = true;
      return MPI_SUCCESS;
    }
  }
  Message m;
  m.data.assign((const char *)buf, (const char *)buf + bytes);
  m.source = me;
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
      std::fprintf(stderr, "mpi_shim: wait on a receive nobody sends (messages only go to self)\n");
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
  types().push_back({(size_t)count * tsize(oldtype), types()[oldtype].base});
  *newtype = (MPI_Datatype)(types().size() - 1);
  return MPI_SUCCESS;
}
int MPI_Type_commit(MPI_Datatype *) { return MPI_SUCCESS; }
int MPI_Type_free(MPI_Datatype *datatype) { *datatype = MPI_DATATYPE_NULL; return MPI_SUCCESS; }

int MPI_Info_create(MPI_Info *info) { *info = 1; return MPI_SUCCESS; }
int MPI_Info_set(MPI_Info, const char *, const char *) { return MPI_SUCCESS; }
int MPI_Info_free(MPI_Info *info) { *info = MPI_INFO_NULL; return MPI_SUCCESS; }

int MPI_Win_allocate_shared(MPI_Aint size, int disp_unit, MPI_Info, MPI_Comm comm, void *baseptr,
                            MPI_Win *win) {
  WinRec w;
  w.size = size;
  w.disp_unit = disp_unit;
  w.comm = comm;
  w.owned = true;
  w.live = true;
  if (!g_node) {
    w.base = (char *)std::calloc(size > 0 ? (size_t)size : 1, 1);
    if (!w.base) {
      std::fprintf(stderr, "mpi_shim: out of memory allocating %ld bytes\n", (long)size);
      std::exit(93);
    }
    w.block = w.base;
    w.seg.assign(1, size);
  } else {
    const LocalComm &lc = local(comm);
    long long *mine = (long long *)stage(g_rank);
    mine[0] = (long long)size;
    barrier(lc);
    w.seg.resize((size_t)lc.size);
    long long total = 0, before = 0;
    for (int r = 0; r < lc.size; ++r) {
      w.seg[(size_t)r] = (MPI_Aint)((const long long *)stage(member(lc, r)))[0];
      if (r < lc.rank) before += w.seg[(size_t)r];
      total += w.seg[(size_t)r];
    }
    CommRec *c = lc.slot >= 0 ? &g_node->comms[lc.slot] : nullptr;
    if (lc.rank == 0) {
      const long long off = heap_alloc(total);
      if (c) __atomic_store_n(&c->word, off, __ATOMIC_RELEASE);
      w.arena_off = off;
    }
    barrier(lc);
    if (c) w.arena_off = __atomic_load_n(&c->word, __ATOMIC_ACQUIRE);
    w.block = g_arena + w.arena_off;
    w.base = w.block + before;
    if (size > 0) std::memset(w.base, 0, (size_t)size);  // each rank zeroes its own segment
    barrier(lc);
  }
  wins().push_back(w);
  *win = (MPI_Win)(wins().size() - 1);
  *(void **)baseptr = w.base;
  return MPI_SUCCESS;
}

int MPI_Win_shared_query(MPI_Win win, int rank, MPI_Aint *size, int *disp_unit, void *baseptr) {
  const WinRec &w = wins()[(size_t)win];
  char *p = w.block;
  for (int r = 0; r < rank && r < (int)w.seg.size(); ++r) p += w.seg[(size_t)r];
  *size = rank < (int)w.seg.size() ? w.seg[(size_t)rank] : 0;
  *disp_unit = w.disp_unit;
  *(void **)baseptr = p;
  return MPI_SUCCESS;
}

int MPI_Win_create(void *base, MPI_Aint size, int disp_unit, MPI_Info, MPI_Comm comm,
                   MPI_Win *win) {
  WinRec w;
  w.base = w.block = (char *)base;
  w.size = size;
  w.disp_unit = disp_unit;
  w.comm = comm;
  w.owned = false;
  w.live = true;
  w.seg.assign(1, size);
  wins().push_back(w);
  *win = (MPI_Win)(wins().size() - 1);
  return MPI_SUCCESS;
}

int MPI_Win_free(MPI_Win *win) {
  if (*win > 0 && (size_t)*win < wins().size()) {
    WinRec &w = wins()[(size_t)*win];
    if (w.live && w.owned) {
      if (!g_node) {
        std::free(w.base);
      } else {
        const LocalComm &lc = local(w.comm);
        barrier(lc);  // no member touches the window any more
        if (lc.rank == 0) heap_free(w.arena_off);
      }
    }
    w.base = w.block = nullptr;
    w.live = false;
  }
  *win = 0;
  return MPI_SUCCESS;
}

int MPI_Win_fence(int, MPI_Win win) {
  __atomic_thread_fence(__ATOMIC_SEQ_CST);
  if (g_node && win > 0 && (size_t)win < wins().size()) barrier(local(wins()[(size_t)win].comm));
  return MPI_SUCCESS;
}
int MPI_Win_lock_all(int, MPI_Win) { __atomic_thread_fence(__ATOMIC_SEQ_CST); return MPI_SUCCESS; }
int MPI_Win_unlock_all(MPI_Win) { __atomic_thread_fence(__ATOMIC_SEQ_CST); return MPI_SUCCESS; }
int MPI_Win_flush_all(MPI_Win) { __atomic_thread_fence(__ATOMIC_SEQ_CST); return MPI_SUCCESS; }

int MPI_Get(void *origin_addr, int origin_count, MPI_Datatype origin_datatype, int target_rank,
            MPI_Aint target_disp, int, MPI_Datatype, MPI_Win win) {
  const WinRec &w = wins()[(size_t)win];
  int me = 0;
  MPI_Comm_rank(w.comm ? w.comm : MPI_COMM_WORLD, &me);
  if (w.seg.size() == 1 && target_rank != me) {
    std::fprintf(stderr, "mpi_shim: MPI_Get from another rank's private window\n");
    std::exit(91);
  }
  char *p = nullptr;
  MPI_Aint sz = 0;
  int du = 1;
  if (w.seg.size() == 1) p = w.base;
  else MPI_Win_shared_query(win, target_rank, &sz, &du, &p);
  std::memcpy(origin_addr, p + (size_t)target_disp * (size_t)w.disp_unit,
              (size_t)origin_count * tsize(origin_datatype));
  return MPI_SUCCESS;
}

}  // extern "C"
