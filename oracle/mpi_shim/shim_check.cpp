// Self-check of the one-node MPI stand-in (test infrastructure): run with
// IB_RANKS=N.  Every rank checks what the reference relies on and rank 0
// prints SHIM_OK when all ranks agree:
//   * the node layout of mpiparams.cpp:68-105 (split_type, split by node,
//     split by shared rank) and SHN = N;
//   * Allreduce sums / max / min in rank order, Reduce, Bcast, Allgather,
//     Allgatherv (also in place and above the staging chunk), Scatter;
//   * a shared window whose segments are contiguous from rank 0's base
//     (DataArray.H indexes it that way), zero-filled, freed and re-made;
//   * self messages over the one-rank node communicator.
// Argument "abort" makes the highest rank call MPI_Abort(comm, 7) mid-run,
// "exit" makes it end without MPI_Finalize: either must end every rank.
#include <mpi.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

static int fails = 0;
#define CHECK(c)                                                            \
  do {                                                                      \
    if (!(c)) {                                                             \
      std::fprintf(stderr, "check failed line %d: %s\n", __LINE__, #c);     \
      ++fails;                                                              \
    }                                                                       \
  } while (0)

int main(int argc, char **argv) {
  MPI_Init(&argc, &argv);
  int rank, n;
  MPI_Comm_rank(MPI_COMM_WORLD, &rank);
  MPI_Comm_size(MPI_COMM_WORLD, &n);
  CHECK(SHN == n);
  const char *mode = argc > 1 ? argv[1] : "";

  MPI_Comm shm, share, nodec;
  MPI_Comm_split_type(MPI_COMM_WORLD, MPI_COMM_TYPE_SHARED, 0, MPI_INFO_NULL, &shm);
  int srank, sprocs, node;
  MPI_Comm_rank(shm, &srank);
  MPI_Comm_split(shm, srank / SHN, srank, &share);
  MPI_Comm_rank(share, &srank);
  MPI_Comm_size(share, &sprocs);
  MPI_Comm_split(MPI_COMM_WORLD, srank, rank, &nodec);
  MPI_Comm_rank(nodec, &node);
  int nsize;
  MPI_Comm_size(nodec, &nsize);
  CHECK(srank == rank && sprocs == n && node == 0 && nsize == 1);

  // reversed keys reverse the ranks; odd/even colours split in two
  MPI_Comm rev, parity;
  MPI_Comm_split(MPI_COMM_WORLD, 0, n - rank, &rev);
  int rrank;
  MPI_Comm_rank(rev, &rrank);
  CHECK(rrank == n - 1 - rank);
  MPI_Comm_split(MPI_COMM_WORLD, rank % 2, rank, &parity);
  int prank, psize;
  MPI_Comm_rank(parity, &prank);
  MPI_Comm_size(parity, &psize);
  CHECK(prank == rank / 2 && psize == (rank % 2 ? n / 2 : (n + 1) / 2));
  int psum = rank;
  MPI_Allreduce(MPI_IN_PLACE, &psum, 1, MPI_INT, MPI_SUM, parity);
  int want = 0;
  for (int r = rank % 2; r < n; r += 2) want += r;
  CHECK(psum == want);

  // reductions: doubles summed in rank order give the same bits everywhere
  double x = 0.1 * (rank + 1), sum = 0.0, mx, mn;
  MPI_Allreduce(&x, &sum, 1, MPI_DOUBLE, MPI_SUM, share);
  double ordered = 0.0;
  for (int r = 0; r < n; ++r) ordered = r ? ordered + 0.1 * (r + 1) : 0.1;
  CHECK(sum == ordered);
  MPI_Allreduce(&x, &mx, 1, MPI_DOUBLE, MPI_MAX, MPI_COMM_WORLD);
  MPI_Allreduce(&x, &mn, 1, MPI_DOUBLE, MPI_MIN, MPI_COMM_WORLD);
  CHECK(mx == 0.1 * n && mn == 0.1);
  int red = rank + 1, tot = -1;
  MPI_Reduce(&red, &tot, 1, MPI_INT, MPI_SUM, 0, share);
  if (rank == 0) CHECK(tot == n * (n + 1) / 2);
  MPI_Bcast(&tot, 1, MPI_INT, 0, share);
  CHECK(tot == n * (n + 1) / 2);
  // a long vector (several staging chunks)
  std::vector<int> big(3 << 20, rank);
  MPI_Allreduce(MPI_IN_PLACE, big.data(), (int)big.size(), MPI_INT, MPI_SUM, MPI_COMM_WORLD);
  CHECK(big.front() == n * (n - 1) / 2 && big.back() == n * (n - 1) / 2);

  // gathers
  std::vector<int> all(n, -1);
  MPI_Allgather(&rank, 1, MPI_INT, all.data(), 1, MPI_INT, share);
  for (int r = 0; r < n; ++r) CHECK(all[r] == r);
  std::vector<int> counts(n), displs(n);
  int total = 0;
  for (int r = 0; r < n; ++r) {
    counts[r] = (r + 1) * 700000;  // rank r sends (r+1) * 700000 ints
    displs[r] = total;
    total += counts[r];
  }
  std::vector<int> mine(counts[rank]);
  for (int i = 0; i < counts[rank]; ++i) mine[i] = rank * 10000000 + i;
  std::vector<int> gath(total, -1);
  MPI_Allgatherv(mine.data(), counts[rank], MPI_INT, gath.data(), counts.data(), displs.data(),
                 MPI_INT, share);
  bool ok = true;
  for (int r = 0; r < n; ++r)
    for (int i = 0; i < counts[r]; i += 9973) ok = ok && gath[displs[r] + i] == r * 10000000 + i;
  CHECK(ok && gath[total - 1] == (n - 1) * 10000000 + counts[n - 1] - 1);
  std::vector<int> inplace(total, -1);
  std::memcpy(&inplace[displs[rank]], mine.data(), sizeof(int) * counts[rank]);
  MPI_Allgatherv(MPI_IN_PLACE, 0, MPI_INT, inplace.data(), counts.data(), displs.data(), MPI_INT,
                 share);
  CHECK(inplace == gath);
  std::vector<int> sc(2 * n);
  for (int i = 0; i < 2 * n; ++i) sc[i] = 100 + i;
  int got[2] = {0, 0};
  MPI_Scatter(sc.data(), 2, MPI_INT, got, 2, MPI_INT, 0, share);
  CHECK(got[0] == 100 + 2 * rank && got[1] == 101 + 2 * rank);

  // derived type reductions by element
  MPI_Datatype pair;
  MPI_Type_contiguous(2, MPI_INT, &pair);
  MPI_Type_commit(&pair);
  int pv[2] = {rank, 1};
  MPI_Allreduce(MPI_IN_PLACE, pv, 1, pair, MPI_SUM, MPI_COMM_WORLD);
  CHECK(pv[0] == n * (n - 1) / 2 && pv[1] == n);

  // shared windows: rank r holds r + 1 doubles; contiguous from rank 0
  for (int round = 0; round < 3; ++round) {
    MPI_Info info;
    MPI_Info_create(&info);
    MPI_Info_set(info, "alloc_shared_noncontig", "true");
    double *lp = nullptr, *gp = nullptr;
    MPI_Win win;
    MPI_Win_allocate_shared((MPI_Aint)(rank + 1 + round) * (MPI_Aint)sizeof(double),
                            sizeof(double), info, share, &lp, &win);
    MPI_Aint bytes;
    int du;
    MPI_Win_shared_query(win, 0, &bytes, &du, &gp);
    MPI_Info_free(&info);
    CHECK(bytes == (MPI_Aint)((1 + round) * sizeof(double)) && du == (int)sizeof(double));
    int before = 0;
    for (int r = 0; r < rank; ++r) before += r + 1 + round;
    CHECK(lp == gp + before);
    bool zero = true;
    for (int i = 0; i < rank + 1 + round; ++i) zero = zero && lp[i] == 0.0;
    CHECK(zero);
    for (int i = 0; i < rank + 1 + round; ++i) lp[i] = rank + 0.5;
    MPI_Win_fence(0, win);
    MPI_Barrier(share);
    int at = 0;
    for (int r = 0; r < n; ++r)
      for (int i = 0; i < r + 1 + round; ++i) CHECK(gp[at++] == r + 0.5);
    MPI_Barrier(share);
    if (round == 1 && rank == n - 1) {
      if (!std::strcmp(mode, "abort")) MPI_Abort(MPI_COMM_WORLD, 7);
      if (!std::strcmp(mode, "exit")) std::exit(0);
    }
    MPI_Win_free(&win);
  }

  // self messages over the node communicator (one rank per node)
  int sendv = 40 + rank, recvv = -1;
  MPI_Request req;
  MPI_Irecv(&recvv, 1, MPI_INT, node, node, nodec, &req);
  MPI_Send(&sendv, 1, MPI_INT, node, node, nodec);
  MPI_Wait(&req, MPI_STATUS_IGNORE);
  CHECK(recvv == 40 + rank);

  int bad = fails;
  MPI_Allreduce(MPI_IN_PLACE, &bad, 1, MPI_INT, MPI_SUM, MPI_COMM_WORLD);
  if (rank == 0 && bad == 0) std::printf("SHIM_OK ranks=%d\n", n);
  MPI_Finalize();
  return bad ? 1 : 0;
}
