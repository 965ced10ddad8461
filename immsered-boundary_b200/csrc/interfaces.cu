// ibgpu_build_interfaces: the coarse/fine interface lists of an AMR mesh from
// its leaf cells, built on the device.
//
// The reference rebuilds these lists incrementally in every regrid
// (AMR::PerformAdaptive, AMR.cpp:6-209): TagRefineGhost marks around each
// refined box the first restriction layer (a box with an unrefined box among
// its neighbours), the second (an unrefined box two steps away along an axis)
// and the prolongation boxes (unrefined neighbours of refined boxes)
// (AMRGhost_refine.cpp:30-98), and the pair bookkeeping of AMRLevel keeps
// f_res_ghost[0..1], f_pro_ghost and g_pro (AMRLevel.H:320-329).  On the
// finished mesh they depend on the leaf cells of every level alone:
//   refined(l)   level-l positions with sons on level l+1 (leaves or refined)
//   res(l), layer 0  refined, four leaf sons, a leaf of level l among the 8
//                    in-plane neighbours; layer 1: not layer 0, four leaf
//                    sons, a leaf of level l two steps away along x or y
//   pro(l)       leaves of level l with a refined position among their 8
//                neighbours (their four sons are the fine ghosts)
//   ghosts(l)    res(l) positions and the sons of pro(l-1)
//
// Layout: each level is a byte map over the bounding box of its leaves and
// refined positions, padded by two cells; one map holds LEAF / REF, a second
// the classes.  Every pass is a stencil over the maps; the lists come out of
// one ordered compaction of all levels' class maps (rows sorted by level,
// then y, then x).
#include <algorithm>
#include <climits>
#include <cstdint>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/ibgpu.h"
#include "host_internal.h"

using namespace ibgpu;

namespace {

enum : uint8_t { M_LEAF = 1, M_REF = 2 };
enum : uint8_t { C_RES0 = 1, C_RES1 = 2, C_PRO = 4, C_GHOST = 8 };

struct MapLevel {
  int x0, y0, w, h;
  int64_t off;
};
struct MapSet {
  int nlev;
  MapLevel lv[IBGPU_MAX_LEVELS];
};

__device__ __forceinline__ int64_t map_at(const MapLevel &L, int x, int y) {
  x -= L.x0;
  y -= L.y0;
  if (x < 0 || y < 0 || x >= L.w || y >= L.h) return -1;
  return L.off + (int64_t)y * L.w + x;
}

__device__ __forceinline__ bool has(const uint8_t *m, const MapLevel &L, int x, int y, uint8_t bits) {
  const int64_t i = map_at(L, x, y);
  return i >= 0 && (m[i] & bits);
}

constexpr int kThreads = 256;
constexpr int kPerThread = 8;
constexpr int kPerBlock = kThreads * kPerThread;

__global__ void scatter_leaves_kernel(const int32_t *lev, const int32_t *ix, const int32_t *iy,
                                      int64_t n, MapSet ms, uint8_t *map) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = map_at(ms.lv[lev[i]], ix[i], iy[i]);
    if (k >= 0) map[k] = M_LEAF;  // the maps are zeroed; only this bit is written here
  }
}

// REF on level l: a son on level l+1 is a leaf or refined
__global__ void refine_kernel(MapSet ms, int l, uint8_t *map) {
  const MapLevel &L = ms.lv[l], &F = ms.lv[l + 1];
  const int64_t n = (int64_t)L.w * L.h;
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x) {
    const int x = L.x0 + (int)(c % L.w), y = L.y0 + (int)(c / L.w);
    bool r = false;
    for (int a = 0; a < 2 && !r; ++a)
      for (int b = 0; b < 2 && !r; ++b) r = has(map, F, 2 * x + a, 2 * y + b, M_LEAF | M_REF);
    if (r) map[L.off + c] |= M_REF;
  }
}

// restriction layers and prolongation pairs of level l (l < finest)
__global__ void classify_kernel(MapSet ms, int l, const uint8_t *map, uint8_t *cls) {
  const MapLevel &L = ms.lv[l], &F = ms.lv[l + 1];
  const int64_t n = (int64_t)L.w * L.h;
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x) {
    const uint8_t f = map[L.off + c];
    if (!(f & (M_LEAF | M_REF))) continue;
    const int x = L.x0 + (int)(c % L.w), y = L.y0 + (int)(c / L.w);
    uint8_t out = 0;
    if (f & M_REF) {
      bool sons = true;
      for (int a = 0; a < 2 && sons; ++a)
        for (int b = 0; b < 2 && sons; ++b) sons = has(map, F, 2 * x + a, 2 * y + b, M_LEAF);
      if (sons) {
        bool near = false;
        for (int dy = -1; dy <= 1 && !near; ++dy)
          for (int dx = -1; dx <= 1 && !near; ++dx)
            near = (dx || dy) && has(map, L, x + dx, y + dy, M_LEAF);
        if (near) out = C_RES0;
        else if (has(map, L, x + 2, y, M_LEAF) || has(map, L, x - 2, y, M_LEAF) ||
                 has(map, L, x, y + 2, M_LEAF) || has(map, L, x, y - 2, M_LEAF))
          out = C_RES1;
      }
    }
    if (f & M_LEAF) {
      bool nb = false;
      for (int dy = -1; dy <= 1 && !nb; ++dy)
        for (int dx = -1; dx <= 1 && !nb; ++dx) nb = (dx || dy) && has(map, L, x + dx, y + dy, M_REF);
      if (nb) out |= C_PRO;
    }
    cls[L.off + c] = out;
  }
}

// interface ghosts of level l: its restriction positions and (l >= 1) the
// sons of the prolongation pairs of level l-1
__global__ void ghost_kernel(MapSet ms, int l, uint8_t *cls) {
  const MapLevel &L = ms.lv[l];
  const int64_t n = (int64_t)L.w * L.h;
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x) {
    const int x = L.x0 + (int)(c % L.w), y = L.y0 + (int)(c / L.w);
    const int64_t p = l > 0 ? map_at(ms.lv[l - 1], x >> 1, y >> 1) : -1;
    if ((cls[L.off + c] & (C_RES0 | C_RES1)) || (p >= 0 && (cls[p] & C_PRO)))
      cls[L.off + c] |= C_GHOST;
  }
}

struct Count3 {
  int res, pro, ghost;
};

__device__ __forceinline__ Count3 count_cell(uint8_t k) {
  return Count3{(k & (C_RES0 | C_RES1)) ? 1 : 0, (k & C_PRO) ? 1 : 0, (k & C_GHOST) ? 1 : 0};
}

// per block of kPerBlock cells: the three counts
__global__ void count_kernel(const uint8_t *cls, int64_t n, int3 *block_counts) {
  __shared__ int3 part[kThreads / 32];
  const int64_t base = (int64_t)blockIdx.x * kPerBlock + (int64_t)threadIdx.x * kPerThread;
  int3 t = make_int3(0, 0, 0);
  for (int k = 0; k < kPerThread; ++k)
    if (base + k < n) {
      const Count3 c = count_cell(cls[base + k]);
      t.x += c.res;
      t.y += c.pro;
      t.z += c.ghost;
    }
  for (int o = 16; o > 0; o >>= 1) {
    t.x += __shfl_down_sync(0xffffffffu, t.x, o);
    t.y += __shfl_down_sync(0xffffffffu, t.y, o);
    t.z += __shfl_down_sync(0xffffffffu, t.z, o);
  }
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = t;
  __syncthreads();
  if (threadIdx.x == 0) {
    int3 s = make_int3(0, 0, 0);
    for (int w = 0; w < kThreads / 32; ++w) {
      s.x += part[w].x;
      s.y += part[w].y;
      s.z += part[w].z;
    }
    block_counts[blockIdx.x] = s;
  }
}

// exclusive scan of the block counts in one block; totals in out[nb]
__global__ void scan_kernel(const int3 *in, int nb, int3 *out) {
  __shared__ int3 sums[1024];
  const int t = threadIdx.x, T = blockDim.x;
  const int per = (nb + T - 1) / T, lo = t * per, hi = min(nb, lo + per);
  int3 s = make_int3(0, 0, 0);
  for (int i = lo; i < hi; ++i) {
    s.x += in[i].x;
    s.y += in[i].y;
    s.z += in[i].z;
  }
  sums[t] = s;
  __syncthreads();
  if (t == 0) {
    int3 run = make_int3(0, 0, 0);
    for (int k = 0; k < T; ++k) {
      const int3 v = sums[k];
      sums[k] = run;
      run.x += v.x;
      run.y += v.y;
      run.z += v.z;
    }
    out[nb] = run;
  }
  __syncthreads();
  int3 run = sums[t];
  for (int i = lo; i < hi; ++i) {
    out[i] = run;
    run.x += in[i].x;
    run.y += in[i].y;
    run.z += in[i].z;
  }
}

__global__ void write_kernel(MapSet ms, const uint8_t *cls, int64_t n, const int3 *block_base,
                             int32_t *res, int32_t *pro, int32_t *ghost) {
  __shared__ int3 warp_tot[kThreads / 32];
  const int64_t base = (int64_t)blockIdx.x * kPerBlock + (int64_t)threadIdx.x * kPerThread;
  int3 t = make_int3(0, 0, 0);
  for (int k = 0; k < kPerThread; ++k)
    if (base + k < n) {
      const Count3 c = count_cell(cls[base + k]);
      t.x += c.res;
      t.y += c.pro;
      t.z += c.ghost;
    }
  // inclusive warp scan, then the warps' totals
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int3 inc = t;
  for (int o = 1; o < 32; o <<= 1) {
    const int a = __shfl_up_sync(0xffffffffu, inc.x, o), b = __shfl_up_sync(0xffffffffu, inc.y, o),
              c = __shfl_up_sync(0xffffffffu, inc.z, o);
    if (lane >= o) {
      inc.x += a;
      inc.y += b;
      inc.z += c;
    }
  }
  if (lane == 31) warp_tot[warp] = inc;
  __syncthreads();
  int3 off = block_base[blockIdx.x];
  for (int w = 0; w < warp; ++w) {
    off.x += warp_tot[w].x;
    off.y += warp_tot[w].y;
    off.z += warp_tot[w].z;
  }
  off.x += inc.x - t.x;
  off.y += inc.y - t.y;
  off.z += inc.z - t.z;
  for (int k = 0; k < kPerThread; ++k) {
    const int64_t i = base + k;
    if (i >= n) break;
    const uint8_t kc = cls[i];
    if (!kc) continue;
    int l = 0;
    while (l + 1 < ms.nlev && i >= ms.lv[l + 1].off) ++l;
    const MapLevel &L = ms.lv[l];
    const int64_t c = i - L.off;
    const int x = L.x0 + (int)(c % L.w), y = L.y0 + (int)(c / L.w);
    if (kc & (C_RES0 | C_RES1)) {
      int32_t *r = res + 12 * (int64_t)off.x++;
      r[0] = l;
      r[1] = (kc & C_RES0) ? 0 : 1;
      r[2] = x;
      r[3] = y;
      for (int s = 0; s < 4; ++s) {
        r[4 + 2 * s] = 2 * x + (s >> 1);
        r[5 + 2 * s] = 2 * y + (s & 1);
      }
    }
    if (kc & C_PRO) {
      int32_t *p = pro + 11 * (int64_t)off.y++;
      p[0] = l;
      p[1] = x;
      p[2] = y;
      for (int s = 0; s < 4; ++s) {
        p[3 + 2 * s] = 2 * x + (s >> 1);
        p[4 + 2 * s] = 2 * y + (s & 1);
      }
    }
    if (kc & C_GHOST) {
      int32_t *g = ghost + 3 * (int64_t)off.z++;
      g[0] = l;
      g[1] = x;
      g[2] = y;
    }
  }
}

#define IF_CK(call)                                                       \
  do {                                                                    \
    cudaError_t e_ = (call);                                              \
    if (e_ != cudaSuccess) {                                              \
      set_last_error(std::string(#call) + ": " + cudaGetErrorString(e_)); \
      rc = IBGPU_E_CUDA;                                                  \
      goto done;                                                          \
    }                                                                     \
  } while (0)

int grid_for(int64_t n, int nsm) {
  int64_t b = (n + 255) / 256;
  return (int)std::max<int64_t>(1, std::min<int64_t>(b, (int64_t)nsm * 16));
}

}  // namespace

extern "C" int ibgpu_build_interfaces(ibgpu_ctx *ctx, int nlevels, const ibgpu_cells *leaves,
                                      ibgpu_interface_lists *out) {
  if (!ctx || !leaves || !out || nlevels < 1 || nlevels > IBGPU_MAX_LEVELS || leaves->n < 0 ||
      (leaves->n > 0 && (!leaves->level || !leaves->ix || !leaves->iy)))
    return IBGPU_E_ARG;
  CtxView v;
  int rc = ctx_view(ctx, &v);
  if (rc) return rc;
  const int64_t n = leaves->n;
  // per-level boxes: the leaves, then the parents of the finer level's box
  // (its refined positions lie there), padded by two cells
  std::vector<int> bx0(nlevels, INT_MAX), by0(nlevels, INT_MAX), bx1(nlevels, INT_MIN),
      by1(nlevels, INT_MIN);
  for (int64_t i = 0; i < n; ++i) {
    const int l = leaves->level[i];
    if (l < 0 || l >= nlevels) {
      set_last_error("leaf level out of range");
      return IBGPU_E_ARG;
    }
    bx0[l] = std::min(bx0[l], leaves->ix[i]);
    bx1[l] = std::max(bx1[l], leaves->ix[i]);
    by0[l] = std::min(by0[l], leaves->iy[i]);
    by1[l] = std::max(by1[l], leaves->iy[i]);
  }
  MapSet ms;
  std::memset(&ms, 0, sizeof(ms));
  ms.nlev = nlevels;
  for (int l = nlevels - 1; l >= 0; --l) {
    int x0 = bx0[l], x1 = bx1[l], y0 = by0[l], y1 = by1[l];
    if (l + 1 < nlevels && ms.lv[l + 1].w > 0) {
      const MapLevel &F = ms.lv[l + 1];
      x0 = std::min(x0, F.x0 >> 1);
      y0 = std::min(y0, F.y0 >> 1);
      x1 = std::max(x1, (F.x0 + F.w - 1) >> 1);
      y1 = std::max(y1, (F.y0 + F.h - 1) >> 1);
    }
    if (x0 > x1 || y0 > y1) {  // a level without cells
      ms.lv[l] = MapLevel{0, 0, 0, 0, 0};
      continue;
    }
    const int64_t w = (int64_t)x1 - x0 + 5, h = (int64_t)y1 - y0 + 5;
    if (w * h > ((int64_t)1 << 31)) {
      set_last_error("level box too large for the interface builder");
      return IBGPU_E_ARG;
    }
    ms.lv[l] = MapLevel{x0 - 2, y0 - 2, (int)w, (int)h, 0};
  }
  int64_t total = 0;
  for (int l = 0; l < nlevels; ++l) {
    ms.lv[l].off = total;
    total += (int64_t)ms.lv[l].w * ms.lv[l].h;
  }
  const int nblocks = (int)std::max<int64_t>(1, (total + kPerBlock - 1) / kPerBlock);
  cudaStream_t st = v.stream;
  uint8_t *d_map = nullptr, *d_cls = nullptr;
  int32_t *d_in = nullptr, *d_res = nullptr, *d_pro = nullptr, *d_ghost = nullptr;
  int3 *d_bc = nullptr, *d_bs = nullptr;
  int3 tot = make_int3(0, 0, 0);
  IF_CK(cudaMalloc(&d_map, std::max<int64_t>(total, 1)));
  IF_CK(cudaMalloc(&d_cls, std::max<int64_t>(total, 1)));
  IF_CK(cudaMalloc(&d_in, sizeof(int32_t) * std::max<int64_t>(3 * n, 1)));
  IF_CK(cudaMalloc(&d_bc, sizeof(int3) * nblocks));
  IF_CK(cudaMalloc(&d_bs, sizeof(int3) * (nblocks + 1)));
  IF_CK(cudaMemsetAsync(d_map, 0, std::max<int64_t>(total, 1), st));
  IF_CK(cudaMemsetAsync(d_cls, 0, std::max<int64_t>(total, 1), st));
  if (n > 0) {
    IF_CK(cudaMemcpyAsync(d_in, leaves->level, sizeof(int32_t) * n, cudaMemcpyHostToDevice, st));
    IF_CK(cudaMemcpyAsync(d_in + n, leaves->ix, sizeof(int32_t) * n, cudaMemcpyHostToDevice, st));
    IF_CK(cudaMemcpyAsync(d_in + 2 * n, leaves->iy, sizeof(int32_t) * n, cudaMemcpyHostToDevice, st));
    scatter_leaves_kernel<<<grid_for(n, v.nsm), 256, 0, st>>>(d_in, d_in + n, d_in + 2 * n, n, ms,
                                                              d_map);
  }
  for (int l = nlevels - 2; l >= 0; --l) {
    const int64_t c = (int64_t)ms.lv[l].w * ms.lv[l].h;
    if (c > 0) refine_kernel<<<grid_for(c, v.nsm), 256, 0, st>>>(ms, l, d_map);
  }
  for (int l = 0; l + 1 < nlevels; ++l) {
    const int64_t c = (int64_t)ms.lv[l].w * ms.lv[l].h;
    if (c > 0) classify_kernel<<<grid_for(c, v.nsm), 256, 0, st>>>(ms, l, d_map, d_cls);
  }
  for (int l = 0; l < nlevels; ++l) {
    const int64_t c = (int64_t)ms.lv[l].w * ms.lv[l].h;
    if (c > 0) ghost_kernel<<<grid_for(c, v.nsm), 256, 0, st>>>(ms, l, d_cls);
  }
  count_kernel<<<nblocks, kThreads, 0, st>>>(d_cls, total, d_bc);
  scan_kernel<<<1, 1024, 0, st>>>(d_bc, nblocks, d_bs);
  IF_CK(cudaGetLastError());
  IF_CK(cudaMemcpyAsync(&tot, d_bs + nblocks, sizeof(int3), cudaMemcpyDeviceToHost, st));
  IF_CK(cudaStreamSynchronize(st));
  out->nres = tot.x;
  out->npro = tot.y;
  out->nghost = tot.z;
  if (out->cap_res < tot.x || out->cap_pro < tot.y || out->cap_ghost < tot.z ||
      (tot.x && !out->res) || (tot.y && !out->pro) || (tot.z && !out->ghost)) {
    set_last_error("output capacity below the counts (counts returned)");
    rc = IBGPU_E_ARG;
    goto done;
  }
  IF_CK(cudaMalloc(&d_res, sizeof(int32_t) * 12 * std::max(tot.x, 1)));
  IF_CK(cudaMalloc(&d_pro, sizeof(int32_t) * 11 * std::max(tot.y, 1)));
  IF_CK(cudaMalloc(&d_ghost, sizeof(int32_t) * 3 * std::max(tot.z, 1)));
  write_kernel<<<nblocks, kThreads, 0, st>>>(ms, d_cls, total, d_bs, d_res, d_pro, d_ghost);
  IF_CK(cudaGetLastError());
  if (tot.x) IF_CK(cudaMemcpyAsync(out->res, d_res, sizeof(int32_t) * 12 * tot.x, cudaMemcpyDeviceToHost, st));
  if (tot.y) IF_CK(cudaMemcpyAsync(out->pro, d_pro, sizeof(int32_t) * 11 * tot.y, cudaMemcpyDeviceToHost, st));
  if (tot.z) IF_CK(cudaMemcpyAsync(out->ghost, d_ghost, sizeof(int32_t) * 3 * tot.z, cudaMemcpyDeviceToHost, st));
  IF_CK(cudaStreamSynchronize(st));
done:
  cudaFree(d_map);
  cudaFree(d_cls);
  cudaFree(d_in);
  cudaFree(d_bc);
  cudaFree(d_bs);
  cudaFree(d_res);
  cudaFree(d_pro);
  cudaFree(d_ghost);
  return rc;
}
