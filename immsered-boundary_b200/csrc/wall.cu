// Wall distances of moved bodies on the device: the per-box part of the
// reference's re-immersion (Body::RenewLevelDistance, Bodymove.cpp:127-300)
// and the block-ghost copies of Mesh::SynNormal_BlockDistance
// (Mesh.cpp:2303-2374), in three passes over every level at once:
//   walk     closest wall patch of the box's own body by the reference's
//            walk over neighbouring patches (Body::FindClosePatchtoCell,
//            Body.H:505-580), signed distance along that patch's normal;
//   junction boxes whose in-plane neighbours belong to another body try that
//            body from the neighbour's patch and take it by the reference's
//            rule (Bodymove.cpp:158-228), reading the neighbours' walked pairs;
//   finalise signed distance capped by the distance to the domain boundary,
//            solid flag, and the boxes that changed sides (the reference's
//            move lists, Bodymove.cpp:231-255); then each box's block ghosts
//            take its final pair and their solid flags;
// and, for ibgpu_wall_distance_near, the compaction of the boxes near the
// walls.
// This unit is compiled without floating-point contraction and uses the
// correctly rounded square root, so every distance is the reference's bit
// for bit (its host code evaluates the same expressions in the same order).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/ibgpu.h"
#include "host_internal.h"

namespace ibgpu {
namespace wall {

constexpr double kCriticDis = 9.5;  // Bodymove.cpp:132
constexpr double kFar = 999.0;      // the walk's starting distance (Bodymove.cpp:150, 199)

struct BodiesDev {
  int nbodies;
  const int32_t *start;  // nbodies + 1
  const double *pc, *nv;
  const int32_t *nbc, *nb;
  int periodic_y;
  double critic_y, len_y;
};

struct LevelDev {
  int64_t n, nblock;
  const double *center, *dtdm;
  const int32_t *neib;
  const uint8_t *kind;
  const int32_t *block_in, *block_out;
  // the block pairs of each origin box: pair indices blk_pair[blk_first[i]
  // .. blk_first[i + 1]) (origins' pairs in pair order)
  const int32_t *blk_first, *blk_pair;
  // pairs as handed in, after the walk, final
  const int32_t *body0, *patch0;
  const double *dist0, *sd0, *dtb0;
  int32_t *body1, *patch1;
  double *dist1, *sd1, *dtb1;
  int32_t *body2, *patch2;
  double *dist2, *sd2, *dtb2;
  uint8_t *solid, *moved, *block_moved;
};

// PeriodicLength (mpiparams.cpp:294-310): the y offset across a periodic
// domain
__device__ __forceinline__ double periodic_dy(const BodiesDev &B, double dy) {
  if (fabs(dy) > B.critic_y && B.periodic_y) {
    if (dy > B.critic_y) dy -= B.len_y;
    else if (dy < -B.critic_y) dy += B.len_y;
  }
  return dy;
}

// |centre - pc| of patch row r (Pointxyz::length, Point.H:211-214)
__device__ __forceinline__ double patch_distance(const BodiesDev &B, int r, double cx, double cy,
                                                 double cz) {
  const double dx = cx - B.pc[3 * r];
  const double dy = periodic_dy(B, cy - B.pc[3 * r + 1]);
  const double dz = cz - B.pc[3 * r + 2];
  return sqrt(dx * dx + dy * dy + dz * dz);
}

// Body::FindClosePatchtoCell from patch p of body b with the distance still
// at kFar: the walk to a patch no neighbour of which is closer (each step
// strictly closer, so it ends within the body's patch count), then the
// signed distance nv . (centre - pc).  false when the walk does not end.
__device__ __forceinline__ bool find_close(const BodiesDev &B, int b, int p, double cx, double cy,
                                           double cz, int &patch, double &dist, double &signdis) {
  const int base = B.start[b], count = B.start[b + 1] - base;
  double best = kFar;
  int bp = p;
  {
    const double d = patch_distance(B, base + p, cx, cy, cz);
    if (d < best) best = d;
  }
  int old = -1, ps0 = bp;
  for (int guard = 0; old != ps0; ++guard) {
    if (guard > count) return false;
    old = bp;
    const int row = base + ps0;
    const int nn = B.nbc[row];
    for (int k = 0; k < nn; ++k) {
      const int q = B.nb[row * IBGPU_WALL_MAX_NB + k];
      if (q < 0 || q >= count) return false;
      const double d = patch_distance(B, base + q, cx, cy, cz);
      if (d < best) {
        best = d;
        bp = q;
      }
    }
    ps0 = bp;
  }
  const int r = base + bp;
  const double dx = cx - B.pc[3 * r];
  const double dy = periodic_dy(B, cy - B.pc[3 * r + 1]);
  const double dz = cz - B.pc[3 * r + 2];
  patch = bp;
  dist = best;
  signdis = B.nv[3 * r] * dx + B.nv[3 * r + 1] * dy + B.nv[3 * r + 2] * dz;
  return true;
}

__device__ __forceinline__ bool valid_pair(const BodiesDev &B, int body, int patch) {
  return body > -1 && body < B.nbodies && patch > -1 && patch < B.start[body + 1] - B.start[body];
}

// The levels of one call as one index space, so each pass is one launch
// for every level: level l's boxes at [box0[l], box0[l] + n_l), box0[l] a
// multiple of kNearBlock (no block of the compaction straddles two
// levels).
constexpr int kNearBlock = 256;
constexpr int kMaxWallLevels = 16;
struct Span {
  int nlevels;
  int64_t box0[kMaxWallLevels + 1];
  double band[kMaxWallLevels];  // near-wall report (ibgpu_wall_distance_near)
};

__device__ __forceinline__ int level_of(const int64_t *start, int nlevels, int64_t g) {
  int l = 0;
  while (l + 1 < nlevels && g >= start[l + 1]) ++l;
  return l;
}

// box g of the span: its level and index there, false past the level's end
__device__ __forceinline__ bool span_box(const Span &sp, int64_t g, int &l, int64_t &i,
                                         const LevelDev *lv) {
  if (g >= sp.box0[sp.nlevels]) return false;
  l = level_of(sp.box0, sp.nlevels, g);
  i = g - sp.box0[l];
  return i < lv[l].n;
}

__global__ void walk_kernel(const LevelDev *lv, Span sp, BodiesDev B, int *err) {
  int l;
  int64_t i;
  if (!span_box(sp, blockIdx.x * (int64_t)blockDim.x + threadIdx.x, l, i, lv)) return;
  const LevelDev &L = lv[l];
  int body = L.body0[i], patch = L.patch0[i];
  double dist = L.dist0[i], sd = L.sd0[i], dtb = L.dtb0[i];
  if (sd < kCriticDis && L.kind[i] != IBGPU_WALL_BOX_BLOCK_GHOST) {
    if (!valid_pair(B, body, patch) ||
        !find_close(B, body, patch, L.center[3 * i], L.center[3 * i + 1], L.center[3 * i + 2],
                    patch, dist, sd)) {
      atomicExch(err, 1);
    } else {
      dtb = sd;
    }
  }
  L.body1[i] = body;
  L.patch1[i] = patch;
  L.dist1[i] = dist;
  L.sd1[i] = sd;
  L.dtb1[i] = dtb;
}

// Boxes next to another body's boxes: that body from the neighbour's patch,
// taken when it is on the fluid side where the own one is not, or closer
// without a worse side (the neighbours in Point_iterator_2d order, each
// compared with the box's pair as the earlier ones left it).
__global__ void junction_kernel(const LevelDev *lv, Span sp, BodiesDev B, int *err) {
  int l;
  int64_t i;
  if (!span_box(sp, blockIdx.x * (int64_t)blockDim.x + threadIdx.x, l, i, lv)) return;
  const LevelDev &L = lv[l];
  int body = L.body1[i], patch = L.patch1[i];
  double dist = L.dist1[i], sd = L.sd1[i], dtb = L.dtb1[i];
  if (sd < kCriticDis && L.kind[i] != IBGPU_WALL_BOX_BLOCK_GHOST) {
    const int own = L.body1[i];
    const double cx = L.center[3 * i], cy = L.center[3 * i + 1], cz = L.center[3 * i + 2];
    for (int k = 0; k < 9; ++k) {
      const int an = L.neib[9 * i + k];
      if (an < 0 || L.body1[an] == own) continue;
      const int cb = L.body1[an], cp = L.patch1[an];
      if (body == cb) continue;
      int np = 0;
      double nd = 0.0, nsd = 0.0;
      if (!valid_pair(B, cb, cp) || !find_close(B, cb, cp, cx, cy, cz, np, nd, nsd)) {
        atomicExch(err, 1);
        break;
      }
      bool change = false;
      if (nsd > 0.0 && sd < 0.0) {
        change = true;
      } else if (nd < dist) {
        if (sd * nsd > 0.0) change = true;
        else if (nsd > 0.0) change = true;
      }
      if (change) {
        body = cb;
        patch = np;
        dist = nd;
        sd = nsd;
        dtb = nsd;
      }
    }
  }
  L.body2[i] = body;
  L.patch2[i] = patch;
  L.dist2[i] = dist;
  L.sd2[i] = sd;
  L.dtb2[i] = dtb;
}

// Caps, solid flags and move lists; then the box's block ghosts take its
// final pair (Mesh::SynNormal_BlockDistance: targets are distinct and never
// origins, checked on upload, so no ghost is written twice and none is an
// input here).
__global__ void finalize_kernel(const LevelDev *lv, Span sp) {
  int l;
  int64_t i;
  if (!span_box(sp, blockIdx.x * (int64_t)blockDim.x + threadIdx.x, l, i, lv)) return;
  const LevelDev &L = lv[l];
  uint8_t mv = 0;
  const uint8_t kind = L.kind[i];
  if (kind == IBGPU_WALL_BOX_BLOCK_GHOST) {
    L.moved[i] = 0;  // its pair comes from its origin
    return;
  }
  double sd = L.sd2[i];
  uint8_t solid = L.solid[i];
  if (sd < kCriticDis) {
    const double dm = L.dtdm[i];
    sd = (dm < sd) ? dm : sd;  // std::min(signdis, distance_to_dm)
    L.sd2[i] = sd;
    if (sd < 0.0) {
      if (!solid && kind != IBGPU_WALL_BOX_DOMAIN_GHOST) mv = IBGPU_WALL_INTO_BODY;
      solid = 1;
    } else {
      if (solid && kind != IBGPU_WALL_BOX_DOMAIN_GHOST) mv = IBGPU_WALL_OUT_OF_BODY;
      solid = 0;
    }
    L.solid[i] = solid;
  }
  L.moved[i] = mv;
  const int k0 = L.blk_first[i], k1 = L.blk_first[i + 1];
  if (k0 == k1) return;
  const int body = L.body2[i], patch = L.patch2[i];
  const double dist = L.dist2[i];
  for (int q = k0; q < k1; ++q) {
    const int k = L.blk_pair[q], out = L.block_out[k];
    L.body2[out] = body;
    L.patch2[out] = patch;
    L.dist2[out] = dist;
    L.sd2[out] = sd;
    uint8_t gm = 0;
    const bool dg = L.kind[out] == IBGPU_WALL_BOX_DOMAIN_GHOST;
    if (sd < 0.0) {
      if (!L.solid[out] && !dg) gm = IBGPU_WALL_INTO_BODY;
      L.solid[out] = 1;
    } else {
      if (L.solid[out] && !dg) gm = IBGPU_WALL_OUT_OF_BODY;
      L.solid[out] = 0;
    }
    L.block_moved[k] = gm;
  }
}

// The boxes a host re-immersion reads (ibgpu_wall_distance_near): near a
// wall before or after the move, or on the other side now; compacted in
// level and box order (per-block counts, one exclusive scan, a ranked
// write).
__device__ __forceinline__ bool near_box(const LevelDev &L, int64_t i, double band) {
  return L.moved[i] != 0 || fabs(L.sd2[i]) < band || fabs(L.sd0[i]) < band;
}

__device__ __forceinline__ bool near_flag(const LevelDev *lv, const Span &sp, int64_t g, int &l,
                                          int64_t &i) {
  return span_box(sp, g, l, i, lv) && near_box(lv[l], i, sp.band[l]);
}

__global__ void near_count_kernel(const LevelDev *lv, Span sp, int *block_count) {
  int l;
  int64_t i;
  const bool f = near_flag(lv, sp, blockIdx.x * (int64_t)kNearBlock + threadIdx.x, l, i);
  const int c = __syncthreads_count(f);
  if (threadIdx.x == 0) block_count[blockIdx.x] = c;
}

// one block of 1024 threads: block_count[0..nb) becomes its exclusive
// prefix sums, block_count[nb] the sum
__global__ void near_scan_kernel(int *block_count, int nb) {
  __shared__ int wsum[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int carry = 0;
  for (int base = 0; base < nb; base += 1024) {
    const int i = base + threadIdx.x;
    const int v = i < nb ? block_count[i] : 0;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    if (warp == 0) {
      int w = wsum[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += y;
      }
      wsum[lane] = w;
    }
    __syncthreads();
    if (i < nb) block_count[i] = carry + (warp > 0 ? wsum[warp - 1] : 0) + x - v;
    carry += wsum[31];
    __syncthreads();  // wsum is rewritten by the next chunk
  }
  if (threadIdx.x == 0) block_count[nb] = carry;
}

__global__ void near_write_kernel(const LevelDev *lv, Span sp, const int *block_base,
                                  ibgpu_wall_change *out) {
  __shared__ int wcount[kNearBlock / 32];
  int l;
  int64_t i;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const bool f = near_flag(lv, sp, blockIdx.x * (int64_t)kNearBlock + threadIdx.x, l, i);
  const unsigned m = __ballot_sync(0xffffffffu, f);
  if (lane == 0) wcount[warp] = __popc(m);
  __syncthreads();
  if (!f) return;
  int pos = block_base[blockIdx.x] + __popc(m & ((1u << lane) - 1u));
  for (int w = 0; w < warp; ++w) pos += wcount[w];
  const LevelDev &L = lv[l];
  ibgpu_wall_change c;
  c.box = (int32_t)i;
  c.body = L.body2[i];
  c.patch = L.patch2[i];
  c.solid = L.solid[i];
  c.moved = L.moved[i];
  c.pad_[0] = c.pad_[1] = 0;
  c.distance = L.dist2[i];
  c.signdis = L.sd2[i];
  c.distance_to_body = L.dtb2[i];
  out[pos] = c;
}

// ---------------------------------------------------------------------------
// host side

struct Buf {
  void *p = nullptr;
  size_t bytes = 0;
  Buf() = default;
  Buf(const Buf &) = delete;
  Buf &operator=(const Buf &) = delete;
  Buf(Buf &&o) noexcept : p(o.p), bytes(o.bytes) {
    o.p = nullptr;
    o.bytes = 0;
  }
  Buf &operator=(Buf &&o) noexcept {
    if (this != &o) {
      cudaFree(p);
      p = o.p;
      bytes = o.bytes;
      o.p = nullptr;
      o.bytes = 0;
    }
    return *this;
  }
  ~Buf() { cudaFree(p); }
  // at least b bytes; a buffer that grows takes a quarter to spare, since
  // a regrid changes the box counts a little and a free + allocation
  // costs far more than the spare bytes
  cudaError_t reserve(size_t b) {
    if (b <= bytes) return cudaSuccess;
    cudaFree(p);
    p = nullptr;
    bytes = 0;
    const size_t want = b + b / 4;
    cudaError_t e = cudaMalloc(&p, want > 0 ? want : 1);
    if (e == cudaSuccess) bytes = want;
    return e;
  }
  template <typename T>
  T *as() const { return static_cast<T *>(p); }
};

struct Level {
  int64_t n = 0, nblock = 0;
  Buf center, dtdm, neib, kind, block_in, block_out, blk_first, blk_pair;
  Buf body[3], patch[3], dist[3], sd[3], dtb[3], solid, moved, block_moved;
};

struct State {
  std::vector<Level> levels;
  Buf start, pc, nv, nbc, nb, err;
  Buf lv;                     // the levels' LevelDev records of a call
  Buf block_count, changes;   // near-wall report (ibgpu_wall_distance_near)
  bool resident = false;  // every level's last results are its next inputs
};

}  // namespace wall

void wall_free(void *state) { delete static_cast<wall::State *>(state); }

}  // namespace ibgpu

using namespace ibgpu;
using namespace ibgpu::wall;

namespace {

int cuda_fail(cudaError_t e, const char *what) {
  set_last_error(std::string(what) + ": " + cudaGetErrorString(e));
  return e == cudaErrorMemoryAllocation ? IBGPU_E_NOMEM : IBGPU_E_CUDA;
}
#define WK(call)                                        \
  do {                                                  \
    cudaError_t e_ = (call);                            \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
  } while (0)

template <typename T>
int put(Buf &b, const T *h, int64_t n, cudaStream_t st) {
  WK(b.reserve((size_t)n * sizeof(T)));
  if (n > 0) WK(cudaMemcpyAsync(b.p, h, (size_t)n * sizeof(T), cudaMemcpyHostToDevice, st));
  return IBGPU_OK;
}
template <typename T>
int get(T *h, const Buf &b, int64_t n, cudaStream_t st) {
  if (n > 0) WK(cudaMemcpyAsync(h, b.p, (size_t)n * sizeof(T), cudaMemcpyDeviceToHost, st));
  return IBGPU_OK;
}

unsigned blocks(int64_t n) { return (unsigned)((n + 255) / 256); }

// Every neighbour index of a level's geometry is a box of the level or -1;
// *bad becomes 1 when one is not (grid-stride over at most four blocks per
// SM of a B200).
constexpr int64_t kCheckBlocks = 4 * 148;
__global__ void neib_check_kernel(const int32_t *neib, int64_t m, int64_t n, int *bad) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t v = neib[i];
    if (v < -1 || v >= n) *bad = 1;
  }
}

}  // namespace

extern "C" {

int ibgpu_host_register(void *ptr, size_t bytes) {
  if (!ptr || bytes == 0) return IBGPU_E_ARG;
  WK(cudaHostRegister(ptr, bytes, cudaHostRegisterDefault));
  return IBGPU_OK;
}

int ibgpu_host_unregister(void *ptr) {
  if (!ptr) return IBGPU_E_ARG;
  WK(cudaHostUnregister(ptr));
  return IBGPU_OK;
}

int ibgpu_wall_geometry(ibgpu_ctx *ctx, int nlevels, const ibgpu_wall_level_geom *levels) {
  CtxView V;
  if (!ctx || nlevels < 0 || nlevels > kMaxWallLevels || (nlevels > 0 && !levels) ||
      ctx_view(ctx, &V) != IBGPU_OK)
    return IBGPU_E_ARG;
  for (int l = 0; l < nlevels; ++l) {
    const ibgpu_wall_level_geom &g = levels[l];
    if (g.n < 0 || g.n > INT32_MAX || g.nblock < 0 ||
        (g.n > 0 && (!g.center || !g.neib || !g.kind || !g.distance_to_dm)) ||
        (g.nblock > 0 && (!g.block_in || !g.block_out)))
      return IBGPU_E_ARG;
    // (the neighbour indices are checked on the device below)
    // block pairs: distinct targets, none of them an origin
    std::vector<uint8_t> mark((size_t)g.n, 0);
    for (int64_t k = 0; k < g.nblock; ++k) {
      const int in = g.block_in[k], out = g.block_out[k];
      if (in < 0 || in >= g.n || out < 0 || out >= g.n || mark[out]) {
        set_last_error("wall geometry: block pair out of range or a ghost targeted twice");
        return IBGPU_E_ARG;
      }
      mark[out] = 1;
    }
    for (int64_t k = 0; k < g.nblock; ++k)
      if (mark[g.block_in[k]]) {
        set_last_error("wall geometry: a block ghost is the origin of another pair");
        return IBGPU_E_ARG;
      }
  }
  void **slot = ctx_wall_state(ctx);
  State *S = static_cast<State *>(*slot);
  if (!S) *slot = S = new State();
  S->levels.resize((size_t)nlevels);
  cudaStream_t st = V.stream;
  WK(S->err.reserve(sizeof(int)));
  WK(cudaMemsetAsync(S->err.p, 0, sizeof(int), st));
  for (int l = 0; l < nlevels; ++l) {
    const ibgpu_wall_level_geom &g = levels[l];
    Level &L = S->levels[(size_t)l];
    L.n = g.n;
    L.nblock = g.nblock;
    int rc;
    if ((rc = put(L.center, g.center, 3 * g.n, st)) || (rc = put(L.neib, g.neib, 9 * g.n, st)) ||
        (rc = put(L.kind, g.kind, g.n, st)) || (rc = put(L.dtdm, g.distance_to_dm, g.n, st)) ||
        (rc = put(L.block_in, g.block_in, g.nblock, st)) ||
        (rc = put(L.block_out, g.block_out, g.nblock, st))) {
      S->levels.clear();
      return rc;
    }
    if (g.n > 0)
      neib_check_kernel<<<std::min<int64_t>(blocks(9 * g.n), kCheckBlocks), 256, 0, st>>>(
          L.neib.as<int32_t>(), 9 * g.n, g.n, S->err.as<int>());
    // each origin's block pairs (a counting sort of the pairs by origin)
    std::vector<int32_t> first((size_t)g.n + 1, 0), order((size_t)std::max<int64_t>(g.nblock, 1));
    for (int64_t k = 0; k < g.nblock; ++k) ++first[(size_t)g.block_in[k] + 1];
    for (int64_t i = 0; i < g.n; ++i) first[(size_t)i + 1] += first[(size_t)i];
    {
      std::vector<int32_t> fill(first.begin(), first.end() - 1);
      for (int64_t k = 0; k < g.nblock; ++k) order[(size_t)fill[(size_t)g.block_in[k]]++] = (int32_t)k;
    }
    if ((rc = put(L.blk_first, first.data(), g.n + 1, st)) ||
        (rc = put(L.blk_pair, order.data(), std::max<int64_t>(g.nblock, 1), st)))
      return rc;
    for (int k = 0; k < 3; ++k) {
      WK(L.body[k].reserve((size_t)g.n * 4));
      WK(L.patch[k].reserve((size_t)g.n * 4));
      WK(L.dist[k].reserve((size_t)g.n * 8));
      WK(L.sd[k].reserve((size_t)g.n * 8));
      WK(L.dtb[k].reserve((size_t)g.n * 8));
    }
    WK(L.solid.reserve((size_t)g.n));
    WK(L.moved.reserve((size_t)g.n));
    WK(L.block_moved.reserve((size_t)g.nblock));
  }
  int bad = 0;
  WK(cudaMemcpyAsync(&bad, S->err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  WK(cudaStreamSynchronize(st));
  S->resident = false;
  if (bad) {
    S->levels.clear();  // no geometry: the distance calls refuse until the next upload
    set_last_error("wall geometry: neighbour index out of the level's boxes");
    return IBGPU_E_ARG;
  }
  return IBGPU_OK;
}

}  // extern "C"

namespace {

// The bodies' patch rows: checked, then on the device.
int upload_bodies(State *S, const ibgpu_wall_bodies *bodies, cudaStream_t st, BodiesDev &B) {
  const int nb = bodies->nbodies;
  if (nb < 0 || (nb > 0 && (!bodies->patch_start || !bodies->pc || !bodies->nv ||
                            !bodies->nb_count || !bodies->nb)))
    return IBGPU_E_ARG;
  const int64_t np = nb > 0 ? bodies->patch_start[nb] : 0;
  for (int b = 0; b < nb; ++b)
    if (bodies->patch_start[b] < 0 || bodies->patch_start[b + 1] < bodies->patch_start[b])
      return IBGPU_E_ARG;
  for (int64_t r = 0; r < np; ++r)
    if (bodies->nb_count[r] < 0 || bodies->nb_count[r] > IBGPU_WALL_MAX_NB) return IBGPU_E_ARG;
  int rc;
  const int32_t zero_start = 0;
  if ((rc = put(S->start, nb > 0 ? bodies->patch_start : &zero_start, nb + 1, st)) ||
      (rc = put(S->pc, bodies->pc, 3 * np, st)) || (rc = put(S->nv, bodies->nv, 3 * np, st)) ||
      (rc = put(S->nbc, bodies->nb_count, np, st)) ||
      (rc = put(S->nb, bodies->nb, (int64_t)IBGPU_WALL_MAX_NB * np, st)))
    return rc;
  B.nbodies = nb;
  B.start = S->start.as<int32_t>();
  B.pc = S->pc.as<double>();
  B.nv = S->nv.as<double>();
  B.nbc = S->nbc.as<int32_t>();
  B.nb = S->nb.as<int32_t>();
  B.periodic_y = bodies->periodic_y;
  B.critic_y = bodies->critic_ylength;
  B.len_y = bodies->dm_length_y;
  return IBGPU_OK;
}

LevelDev level_dev(Level &L) {
  LevelDev D;
  D.n = L.n;
  D.nblock = L.nblock;
  D.center = L.center.as<double>();
  D.dtdm = L.dtdm.as<double>();
  D.neib = L.neib.as<int32_t>();
  D.kind = L.kind.as<uint8_t>();
  D.block_in = L.block_in.as<int32_t>();
  D.block_out = L.block_out.as<int32_t>();
  D.blk_first = L.blk_first.as<int32_t>();
  D.blk_pair = L.blk_pair.as<int32_t>();
  D.body0 = L.body[0].as<int32_t>();
  D.patch0 = L.patch[0].as<int32_t>();
  D.dist0 = L.dist[0].as<double>();
  D.sd0 = L.sd[0].as<double>();
  D.dtb0 = L.dtb[0].as<double>();
  D.body1 = L.body[1].as<int32_t>();
  D.patch1 = L.patch[1].as<int32_t>();
  D.dist1 = L.dist[1].as<double>();
  D.sd1 = L.sd[1].as<double>();
  D.dtb1 = L.dtb[1].as<double>();
  D.body2 = L.body[2].as<int32_t>();
  D.patch2 = L.patch[2].as<int32_t>();
  D.dist2 = L.dist[2].as<double>();
  D.sd2 = L.sd[2].as<double>();
  D.dtb2 = L.dtb[2].as<double>();
  D.solid = L.solid.as<uint8_t>();
  D.moved = L.moved.as<uint8_t>();
  D.block_moved = L.block_moved.as<uint8_t>();
  return D;
}

// Every level's LevelDev record on the device and the span of the call.
int level_span(State *S, cudaStream_t st, Span &sp) {
  const int nl = (int)S->levels.size();
  std::vector<LevelDev> h((size_t)std::max(nl, 1));
  sp.nlevels = nl;
  sp.box0[0] = 0;
  for (int l = 0; l < nl; ++l) {
    Level &L = S->levels[(size_t)l];
    h[(size_t)l] = level_dev(L);
    sp.box0[l + 1] = sp.box0[l] + (L.n + kNearBlock - 1) / kNearBlock * kNearBlock;
    sp.band[l] = 0.0;
  }
  return put(S->lv, h.data(), std::max(nl, 1), st);
}

// The passes of every level (walk, junction, then caps, move lists and the
// block ghosts' copies) from the input pairs (set 0) to the new ones (set
// 2), one launch each.
int launch_passes(State *S, const Span &sp, const BodiesDev &B, cudaStream_t st) {
  const LevelDev *lv = S->lv.as<LevelDev>();
  int *err = S->err.as<int>();
  const int64_t nbox = sp.box0[sp.nlevels];
  if (nbox > 0) {
    walk_kernel<<<blocks(nbox), 256, 0, st>>>(lv, sp, B, err);
    junction_kernel<<<blocks(nbox), 256, 0, st>>>(lv, sp, B, err);
    finalize_kernel<<<blocks(nbox), 256, 0, st>>>(lv, sp);
  }
  WK(cudaGetLastError());
  return IBGPU_OK;
}

// After the copies of a call: the walk's verdict; on success the new pairs
// become the device's current ones (set 0).
int settle(State *S, int herr) {
  if (herr) {
    S->resident = false;
    set_last_error("wall distances: a box within 9.5 of a wall has no valid body or patch, "
                   "or a patch walk did not end");
    return IBGPU_E_ABORT;
  }
  for (Level &L : S->levels) {
    std::swap(L.body[0], L.body[2]);
    std::swap(L.patch[0], L.patch[2]);
    std::swap(L.dist[0], L.dist[2]);
    std::swap(L.sd[0], L.sd[2]);
    std::swap(L.dtb[0], L.dtb[2]);
  }
  S->resident = true;
  return IBGPU_OK;
}

State *wall_state(ibgpu_ctx *ctx, int nlevels) {
  State *S = static_cast<State *>(*ctx_wall_state(ctx));
  if (!S || (int)S->levels.size() != nlevels) {
    set_last_error("wall distances: upload the wall geometry of these levels first");
    return nullptr;
  }
  return S;
}

}  // namespace

extern "C" {

int ibgpu_wall_distance(ibgpu_ctx *ctx, const ibgpu_wall_bodies *bodies, int nlevels,
                        ibgpu_wall_pairs *pairs, int flags) {
  CtxView V;
  if (!ctx || !bodies || nlevels < 0 || (nlevels > 0 && !pairs) ||
      (flags & ~IBGPU_WALL_RESIDENT) || ctx_view(ctx, &V) != IBGPU_OK)
    return IBGPU_E_ARG;
  State *S = wall_state(ctx, nlevels);
  if (!S) return IBGPU_E_STATE;
  const bool resident = (flags & IBGPU_WALL_RESIDENT) != 0;
  if (resident && !S->resident) {
    set_last_error("wall distances: no pairs on the device since the geometry upload");
    return IBGPU_E_STATE;
  }
  for (int l = 0; l < nlevels; ++l) {
    const ibgpu_wall_pairs &p = pairs[l];
    const Level &L = S->levels[(size_t)l];
    if ((L.n > 0 && (!p.body || !p.patch || !p.distance || !p.signdis || !p.distance_to_body ||
                     !p.solid || !p.moved)) ||
        (L.nblock > 0 && !p.block_moved))
      return IBGPU_E_ARG;
  }
  cudaStream_t st = V.stream;
  BodiesDev B;
  int rc;
  if ((rc = upload_bodies(S, bodies, st, B))) return rc;
  WK(cudaMemsetAsync(S->err.p, 0, sizeof(int), st));
  for (int l = 0; l < nlevels && !resident; ++l) {
    Level &L = S->levels[(size_t)l];
    const ibgpu_wall_pairs &p = pairs[l];
    if ((rc = put(L.body[0], p.body, L.n, st)) || (rc = put(L.patch[0], p.patch, L.n, st)) ||
        (rc = put(L.dist[0], p.distance, L.n, st)) || (rc = put(L.sd[0], p.signdis, L.n, st)) ||
        (rc = put(L.dtb[0], p.distance_to_body, L.n, st)) || (rc = put(L.solid, p.solid, L.n, st)))
      return rc;
  }
  Span sp;
  if ((rc = level_span(S, st, sp)) || (rc = launch_passes(S, sp, B, st))) return rc;
  for (int l = 0; l < nlevels; ++l) {
    Level &L = S->levels[(size_t)l];
    ibgpu_wall_pairs &p = pairs[l];
    if ((rc = get(p.body, L.body[2], L.n, st)) || (rc = get(p.patch, L.patch[2], L.n, st)) ||
        (rc = get(p.distance, L.dist[2], L.n, st)) || (rc = get(p.signdis, L.sd[2], L.n, st)) ||
        (rc = get(p.distance_to_body, L.dtb[2], L.n, st)) || (rc = get(p.solid, L.solid, L.n, st)) ||
        (rc = get(p.moved, L.moved, L.n, st)) ||
        (rc = get(p.block_moved, L.block_moved, L.nblock, st)))
      return rc;
  }
  int herr = 0;
  WK(cudaMemcpyAsync(&herr, S->err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  WK(cudaStreamSynchronize(st));
  return settle(S, herr);
}

int ibgpu_wall_distance_near(ibgpu_ctx *ctx, const ibgpu_wall_bodies *bodies, int nlevels,
                             ibgpu_wall_near *levels) {
  CtxView V;
  if (!ctx || !bodies || nlevels < 0 || (nlevels > 0 && !levels) ||
      ctx_view(ctx, &V) != IBGPU_OK)
    return IBGPU_E_ARG;
  State *S = wall_state(ctx, nlevels);
  if (!S) return IBGPU_E_STATE;
  if (!S->resident) {
    set_last_error("wall distances: no pairs on the device since the geometry upload");
    return IBGPU_E_STATE;
  }
  for (int l = 0; l < nlevels; ++l) {
    const ibgpu_wall_near &o = levels[l];
    const Level &L = S->levels[(size_t)l];
    if (o.capacity < 0 || (o.capacity > 0 && !o.changes) || (L.nblock > 0 && !o.block_moved) ||
        !(o.band >= 0.0))
      return IBGPU_E_ARG;
  }
  cudaStream_t st = V.stream;
  BodiesDev B;
  int rc;
  if ((rc = upload_bodies(S, bodies, st, B))) return rc;
  WK(cudaMemsetAsync(S->err.p, 0, sizeof(int), st));
  Span sp;
  if ((rc = level_span(S, st, sp))) return rc;
  for (int l = 0; l < nlevels; ++l) sp.band[l] = levels[l].band;
  if ((rc = launch_passes(S, sp, B, st))) return rc;
  const int64_t nbox = sp.box0[nlevels];
  const int nb = (int)(nbox / kNearBlock);
  WK(S->block_count.reserve(sizeof(int) * ((size_t)nb + 1)));
  WK(S->changes.reserve(sizeof(ibgpu_wall_change) * (size_t)std::max<int64_t>(nbox, 1)));
  int *base = S->block_count.as<int>();
  if (nb > 0) near_count_kernel<<<nb, kNearBlock, 0, st>>>(S->lv.as<LevelDev>(), sp, base);
  near_scan_kernel<<<1, 1024, 0, st>>>(base, nb);
  if (nb > 0)
    near_write_kernel<<<nb, kNearBlock, 0, st>>>(S->lv.as<LevelDev>(), sp, base,
                                                 S->changes.as<ibgpu_wall_change>());
  WK(cudaGetLastError());
  for (int l = 0; l < nlevels; ++l)
    if ((rc = get(levels[l].block_moved, S->levels[(size_t)l].block_moved,
                  S->levels[(size_t)l].nblock, st)))
      return rc;
  // each level's first block's offset (and the total) from the scan
  std::vector<int> hbase((size_t)nb + 1, 0);
  int herr = 0;
  WK(cudaMemcpyAsync(hbase.data(), base, sizeof(int) * ((size_t)nb + 1), cudaMemcpyDeviceToHost,
                     st));
  WK(cudaMemcpyAsync(&herr, S->err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  WK(cudaStreamSynchronize(st));
  if (herr) return settle(S, herr);
  bool fits = true;
  for (int l = 0; l < nlevels; ++l) {
    ibgpu_wall_near &o = levels[l];
    const int64_t first = hbase[(size_t)(sp.box0[l] / kNearBlock)];
    o.count = hbase[(size_t)(sp.box0[l + 1] / kNearBlock)] - first;
    if (o.count > o.capacity) {
      fits = false;
      continue;
    }
    if (o.count > 0)
      WK(cudaMemcpyAsync(o.changes, S->changes.as<ibgpu_wall_change>() + first,
                         sizeof(ibgpu_wall_change) * (size_t)o.count, cudaMemcpyDeviceToHost,
                         st));
  }
  WK(cudaStreamSynchronize(st));
  rc = settle(S, 0);
  if (rc == IBGPU_OK && !fits) {
    set_last_error("wall distances: more boxes near the walls than the output holds");
    return IBGPU_E_ARG;
  }
  return rc;
}

int ibgpu_wall_fetch(ibgpu_ctx *ctx, int nlevels, ibgpu_wall_pairs *pairs) {
  CtxView V;
  if (!ctx || nlevels < 0 || (nlevels > 0 && !pairs) || ctx_view(ctx, &V) != IBGPU_OK)
    return IBGPU_E_ARG;
  State *S = wall_state(ctx, nlevels);
  if (!S) return IBGPU_E_STATE;
  if (!S->resident) {
    set_last_error("wall distances: no pairs on the device since the geometry upload");
    return IBGPU_E_STATE;
  }
  cudaStream_t st = V.stream;
  for (int l = 0; l < nlevels; ++l) {
    const Level &L = S->levels[(size_t)l];
    ibgpu_wall_pairs &p = pairs[l];
    if (L.n > 0 && (!p.body || !p.patch || !p.distance || !p.signdis || !p.distance_to_body ||
                    !p.solid))
      return IBGPU_E_ARG;
  }
  int rc;
  for (int l = 0; l < nlevels; ++l) {
    const Level &L = S->levels[(size_t)l];
    ibgpu_wall_pairs &p = pairs[l];
    if ((rc = get(p.body, L.body[0], L.n, st)) || (rc = get(p.patch, L.patch[0], L.n, st)) ||
        (rc = get(p.distance, L.dist[0], L.n, st)) || (rc = get(p.signdis, L.sd[0], L.n, st)) ||
        (rc = get(p.distance_to_body, L.dtb[0], L.n, st)) || (rc = get(p.solid, L.solid, L.n, st)))
      return rc;
  }
  WK(cudaStreamSynchronize(st));
  return IBGPU_OK;
}

}  // extern "C"
