// Host side of the ibgpu C ABI: context, tiled layout builder, state
// transfer and the per-step launch sequence.  Mirrors the call order of the
// reference main loop and NS_Solver::TimeMarching (main.cpp:84-116,
// NS_Solver.H:657-702).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <unordered_map>
#include <map>
#include <numeric>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/ibgpu.h"
#include "host_internal.h"
#include "launchers.h"
#include "layout.h"

using namespace ibgpu;

namespace {

thread_local std::string g_last_error;

int cuda_fail(cudaError_t e, const char *what) {
  g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
  return IBGPU_E_CUDA;
}

#define CK(call)                                       \
  do {                                                 \
    cudaError_t e_ = (call);                           \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
  } while (0)

inline int floordiv(int a, int b) { return (a >= 0) ? a / b : -((-a + b - 1) / b); }

inline uint64_t morton2(uint32_t x, uint32_t y) {
  auto spread = [](uint64_t v) {
    v &= 0xffffffffull;
    v = (v | (v << 16)) & 0x0000ffff0000ffffull;
    v = (v | (v << 8)) & 0x00ff00ff00ff00ffull;
    v = (v | (v << 4)) & 0x0f0f0f0f0f0f0f0full;
    v = (v | (v << 2)) & 0x3333333333333333ull;
    v = (v | (v << 1)) & 0x5555555555555555ull;
    return v;
  };
  return spread(x) | (spread(y) << 1);
}

inline uint64_t key2(int a, int b) { return ((uint64_t)(uint32_t)a << 32) | (uint32_t)b; }

template <typename T>
int dev_alloc(T **p, size_t n) {
  if (n == 0) n = 1;
  cudaError_t e = cudaMalloc((void **)p, n * sizeof(T));
  if (e != cudaSuccess) {
    g_last_error = std::string("cudaMalloc: ") + cudaGetErrorString(e);
    return IBGPU_E_NOMEM;
  }
  return IBGPU_OK;
}

}  // namespace

struct ibgpu_ctx {
  void *wall = nullptr;  // wall-distance state (csrc/wall.cu)
  ibgpu_case cs;
  CaseConst cc;
  int device = 0;
  int nsm = 148;
  int body_level = -1;  // finest level of a run with immersed bodies
  cudaStream_t own_stream = nullptr;
  cudaStream_t copy_stream = nullptr;  // asynchronous state downloads
  cudaEvent_t ev_ready = nullptr, ev_copied = nullptr;
  cudaStream_t in_stream = nullptr;  // asynchronous state uploads
  cudaEvent_t ev_in_free = nullptr, ev_in_done = nullptr;
  bool in_used = false;     // ev_in_free marks the last upload's scatter
  bool chain_open = false;  // asynchronous steps since the last ibgpu_step_result
  int chain_steps = 0;
  int64_t chain_marched = 0;
  bool download_pending = false;       // an asynchronous download may still read s0
  int row_fields = 7;                  // state rows: 7 FlowVariables or 4 (roe u v p)
  double *d_rows_out = nullptr;        // staging of asynchronous downloads
  cudaStream_t stream = nullptr;

  // layout
  bool has_topology = false, has_state = false;
  int64_t ncells = 0;       // rows of the caller's cell list
  int64_t ntiles = 0, nslots = 0;
  std::vector<int> level_tile_begin, level_tile_count;  // per level
  std::vector<int64_t> level_normal_cells;
  std::vector<int32_t> h_slot_level, h_slot_ix, h_slot_iy;  // slot -> position (abort reports)
  int32_t *d_tile_nb = nullptr, *d_tile_level = nullptr, *d_cell_slot = nullptr;
  int2 *d_tile_org = nullptr;      // (ix, iy) of each tile's first cell
  double *d_signdis = nullptr;     // per slot, after ibgpu_upload_signdis
  uint8_t *d_tags = nullptr;       // indicator output: per slot, then per cell row
  uint8_t *d_flags = nullptr, *d_cell_alias = nullptr, *d_tile_uniform = nullptr;
  // ibgpu_update_flags on the device: each row's layout bits (PRESENT /
  // NORMAL / ALIAS as uploaded), the rows' new flags, per-tile scratch and
  // the first row whose layout bits changed
  uint8_t *d_cell_layout = nullptr, *d_row_flags = nullptr, *d_tile_full = nullptr;
  int *d_layout_err = nullptr;
  // ibgpu_update_flags_rows: the rows and their flags (grown when short)
  int64_t *d_row_which = nullptr;
  uint8_t *d_row_sub = nullptr;

  // state: step state (6 fields) + two stage buffers (4 fields each)
  double *d_s0[kStateFields] = {};
  void *d_buf[2][4] = {};  // stage buffers: FP64, FP32 in the mixed build
  double *d_vsd = nullptr;
  double *d_rows = nullptr;  // staging for AoS state transfers
  DevDiag *d_diag = nullptr;
  DevDiag *h_diag = nullptr;  // pinned
  int *d_aux_err = nullptr;   // time-out flag of the indicator kernels

  // slot lookup: per level, tile (tx,ty) -> tile index
  std::vector<std::unordered_map<uint64_t, int>> tilemap;

  // coarse/fine pairs per coarse level
  struct DevPairs {
    int32_t *coarse = nullptr, *fine = nullptr, *nb = nullptr;
    int n = 0;
  };
  std::vector<DevPairs> res, pro;

  // domain ghosts: level-sorted, dependency waves [begin, end)
  int32_t *d_bc_ghost = nullptr, *d_bc_ref = nullptr, *d_bc_type = nullptr, *d_bc_face = nullptr;
  double *d_bc_nmv = nullptr, *d_facevar = nullptr;
  std::vector<std::vector<std::pair<int, int>>> bc_waves;  // per level
  double backpressure = 0.0, cos_in = 1.0, sin_in = 0.0;

  // immersed boundary
  int32_t *d_ib_cell = nullptr, *d_ib_intp = nullptr;
  double *d_ib_f = nullptr, *d_ib_out = nullptr;
  int n_ib = 0;
  int32_t *d_pat_body = nullptr, *d_pat_intp = nullptr, *d_body_begin = nullptr;
  double *d_pat_f = nullptr, *d_pat_out = nullptr, *d_body_center = nullptr, *d_force = nullptr;
  int n_pat = 0, nbodies = 0;
  // element capacities of the buffers ibgpu_upload_ib refills after every
  // move (kept between calls, grown when short), by buffer member
  std::map<const void *, size_t> cap;

  // kernel timing
  bool timing = false;
  double kms[3] = {0, 0, 0};
  int64_t klaunch[3] = {0, 0, 0};

  void free_aux() {
    for (auto *v : {&res, &pro})
      for (auto &p : *v) {
        cudaFree(p.coarse);
        cudaFree(p.fine);
        cudaFree(p.nb);
      }
    res.clear();
    pro.clear();
    for (int32_t **p : {&d_bc_ghost, &d_bc_ref, &d_bc_type, &d_bc_face, &d_ib_cell, &d_ib_intp,
                        &d_pat_body, &d_pat_intp, &d_body_begin}) {
      cudaFree(*p);
      *p = nullptr;
      cap.erase(p);
    }
    for (double **p : {&d_bc_nmv, &d_facevar, &d_ib_f, &d_ib_out, &d_pat_f, &d_pat_out,
                       &d_body_center, &d_force}) {
      cudaFree(*p);
      *p = nullptr;
      cap.erase(p);
    }
    bc_waves.clear();
    n_ib = n_pat = nbodies = 0;
  }

  // Before a new topology: the lists that belong to the old one go, and the
  // per-slot buffers made on demand (sized by the old slot count); the
  // layout's own buffers stay for the new one to reuse when large enough.
  void reset_layout() {
    free_aux();
    cudaFree(d_signdis);
    cudaFree(d_tags);
    d_signdis = nullptr;
    d_tags = nullptr;
    has_topology = has_state = false;
  }

  // slot of (level, x, y) with periodic wrap, -1 if absent
  int64_t slot_at(int l, int ix, int iy) const {
    if (l < 0 || l >= (int)tilemap.size()) return -1;
    if (cs.periodic_x) { int e = cs.domain_nx << l; ix = ((ix % e) + e) % e; }
    if (cs.periodic_y) { int e = cs.domain_ny << l; iy = ((iy % e) + e) % e; }
    int tx = floordiv(ix, kTile), ty = floordiv(iy, kTile);
    auto it = tilemap[l].find(key2(tx, ty));
    if (it == tilemap[l].end() || it->second < 0) return -1;
    int64_t s = (int64_t)it->second * kTileCells + (iy - ty * kTile) * kTile + (ix - tx * kTile);
    return h_flags_present[s] ? s : -1;
  }
  std::vector<uint8_t> h_flags_present;

  void free_layout() {
    free_aux();
    cudaFree(d_tile_nb);
    cudaFree(d_tile_level);
    cudaFree(d_cell_slot);
    cudaFree(d_flags);
    cudaFree(d_cell_alias);
    cudaFree(d_tile_uniform);
    d_tile_uniform = nullptr;
    for (uint8_t **p : {&d_cell_layout, &d_row_flags, &d_tile_full}) {
      cudaFree(*p);
      *p = nullptr;
    }
    cudaFree(d_layout_err);
    d_layout_err = nullptr;
    cudaFree(d_row_which);
    cudaFree(d_row_sub);
    d_row_which = nullptr;
    d_row_sub = nullptr;
    cap.erase(&d_row_which);
    cap.erase(&d_row_sub);
    cudaFree(d_tile_org);
    cudaFree(d_signdis);
    cudaFree(d_tags);
    d_tile_org = nullptr;
    d_signdis = nullptr;
    d_tags = nullptr;
    for (auto &p : d_s0) { cudaFree(p); p = nullptr; }
    for (auto &b : d_buf)
      for (auto &p : b) { cudaFree(p); p = nullptr; }
    cudaFree(d_vsd);
    cudaFree(d_rows);
    cudaFree(d_rows_out);
    d_rows_out = nullptr;
    d_tile_nb = d_tile_level = d_cell_slot = nullptr;
    d_flags = d_cell_alias = nullptr;
    d_vsd = d_rows = nullptr;
    has_topology = has_state = false;
    cap.clear();
  }
};

namespace {

// A context buffer of at least n elements that stays between calls (freed
// and allocated again only when it is too short).
template <typename T>
int keep_alloc(ibgpu_ctx *ctx, T **dst, size_t n) {
  size_t &c = ctx->cap[dst];
  if (*dst && n <= c) return IBGPU_OK;
  cudaFree(*dst);
  *dst = nullptr;
  c = 0;
  const int rc = dev_alloc(dst, n);
  if (rc) return rc;
  c = n > 0 ? n : 1;
  return IBGPU_OK;
}
template <typename T>
int keep_upload(ibgpu_ctx *ctx, T **dst, const std::vector<T> &v, cudaStream_t st) {
  const int rc = keep_alloc(ctx, dst, v.size());
  if (rc) return rc;
  if (!v.empty()) CK(cudaMemcpyAsync(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st));
  return IBGPU_OK;
}

}  // namespace

namespace ibgpu {
void set_last_error(const std::string &msg) { g_last_error = msg; }

int validate_case(const ibgpu_case *cs) {
  if (cs->abi_version != IBGPU_ABI_VERSION) {
    g_last_error = "ABI version mismatch";
    return IBGPU_E_ARG;
  }
  if (cs->nlevels < 1 || cs->nlevels > IBGPU_MAX_LEVELS || cs->nstages < 1 || cs->nstages > 4 ||
      cs->dt_var_step < 1 || (cs->limiter != IBGPU_LIM_VANLEER && cs->limiter != IBGPU_LIM_MINMOD) ||
      cs->precision < IBGPU_FP64 || cs->precision > IBGPU_MIXED) {
    g_last_error = "invalid case parameters";
    return IBGPU_E_ARG;
  }
  for (int l = 0; l < cs->nlevels; ++l)
    if (cs->march_step[l] < 1 || !(cs->dh[l][0] > 0) || !(cs->dh[l][1] > 0) || !(cs->dh[l][2] > 0)) {
      g_last_error = "invalid level parameters";
      return IBGPU_E_ARG;
    }
  return IBGPU_OK;
}
}  // namespace ibgpu

namespace ibgpu {
// CaseConst of a validated case (shared with the allocation-free entry point)
void fill_case_const(const ibgpu_case *cs, CaseConst &k) {
  std::memset(&k, 0, sizeof(k));
  k.gama = cs->gama;
  k.Rg = cs->Rg;
  k.Cv = cs->Cv;
  k.Ma = cs->Ma;
  k.Re = cs->Re;
  k.qk = cs->qk;
  k.s_over_t = cs->s_over_t;
  k.dt_ratio = cs->dt_ratio;
  k.gm1 = cs->gama - 1.0;
  k.gamaRg = cs->gama * cs->Rg;
  k.inv_Rg = 1.0 / cs->Rg;
  k.Cp = cs->Cp;
  k.p_ref = cs->p_ref;
  k.area_ref = cs->area_ref;
  k.shear_ref = cs->shear_ref;
  k.L_ref = cs->L_ref;
  k.mu = cs->mu;
  for (int i = 0; i < 7; ++i) k.initvar[i] = cs->initvar[i];
  for (int l = 0; l < cs->nlevels; ++l) {
    LevelConst &L = k.lev[l];
    L.dx = cs->dh[l][0];
    L.dy = cs->dh[l][1];
    L.dz = cs->dh[l][2];
    L.vol = cs->dh[l][0] * cs->dh[l][1] * cs->dh[l][2];
    L.inv_vol = 1.0 / L.vol;
    L.area_x = cs->dh[l][1] * cs->dh[l][2];
    L.area_y = cs->dh[l][2] * cs->dh[l][0];
    L.area_z = cs->dh[l][0] * cs->dh[l][1];
    L.inv_dx = 1.0 / cs->dh[l][0];
    L.inv_dy = 1.0 / cs->dh[l][1];
    L.step_num = cs->step_num[l];
    L.cfl_vol = cs->cfl * L.vol;
  }
}
}  // namespace ibgpu

namespace ibgpu {
int ctx_view(const ibgpu_ctx *ctx, CtxView *v) {
  if (!ctx || !v) return IBGPU_E_ARG;
  v->stream = ctx->stream;
  v->device = ctx->device;
  v->nsm = ctx->nsm;
  v->has_topology = ctx->has_topology;
  v->has_state = ctx->has_state;
  for (int k = 0; k < kStateFields; ++k) v->s0[k] = ctx->d_s0[k];
  v->flags = ctx->d_flags;
  v->tile_nb = ctx->d_tile_nb;
  v->tile_level = ctx->d_tile_level;
  v->tile_org = ctx->d_tile_org;
  v->cell_slot = ctx->d_cell_slot;
  v->ncells = ctx->ncells;
  v->nslots = ctx->nslots;
  v->ntiles = ctx->ntiles;
  v->aux_err = ctx->d_aux_err;
  v->cc = ctx->cc;
  return IBGPU_OK;
}
int ctx_signdis_buffer(ibgpu_ctx *ctx, double **dev, bool create) {
  if (!ctx->d_signdis && create) {
    int rc = dev_alloc(&ctx->d_signdis, (size_t)std::max<int64_t>(ctx->nslots, 1));
    if (rc) return rc;
  }
  *dev = ctx->d_signdis;
  return IBGPU_OK;
}
int ctx_tags_buffer(ibgpu_ctx *ctx, uint8_t **dev) {
  if (!ctx->d_tags) {
    // per slot, then per cell row
    int rc = dev_alloc(&ctx->d_tags, (size_t)std::max<int64_t>(ctx->nslots + ctx->ncells, 1));
    if (rc) return rc;
  }
  *dev = ctx->d_tags;
  return IBGPU_OK;
}
int64_t ctx_slot_at(const ibgpu_ctx *ctx, int l, int ix, int iy) {
  return ctx ? ctx->slot_at(l, ix, iy) : -1;
}
void **ctx_wall_state(ibgpu_ctx *ctx) { return &ctx->wall; }
}  // namespace ibgpu

namespace {

// ibgpu_update_flags on the device, over the rows' new flags in `rows`:
// the first row whose PRESENT / NORMAL / ALIAS bits differ from the
// topology upload (atomicMin into *err, which starts at INT_MAX) ...
// (with `which`, new flags rows[k] for row which[k], k < n; without, for
// every row c < n) ...
__global__ void layout_check_kernel(const uint8_t *rows, const int64_t *which,
                                    const uint8_t *layout, int64_t n, int *err) {
  constexpr uint8_t kBits = CF_PRESENT | CF_NORMAL | IBGPU_CELL_ALIAS;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = which ? which[k] : k;
    const uint8_t lay = (uint8_t)((rows[k] & kBits) | (layout[c] & IBGPU_CELL_ALIAS));
    if (lay != layout[c]) atomicMin(err, (int)k);
  }
}

// ... each non-alias row's flags into its slot (the slots no row maps to
// keep the zeros of the topology upload) ...
__global__ void flags_scatter_kernel(const uint8_t *rows, const int64_t *which,
                                     const uint8_t *layout, const int32_t *slot, int64_t n,
                                     uint8_t *flags) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = which ? which[k] : k;
    if (!(layout[c] & IBGPU_CELL_ALIAS)) flags[slot[c]] = rows[k] & 0x3f;
  }
}

// ... which tiles hold only leaf cells that update and recover their
// primitives (one warp per tile, eight slots per lane) ...
__global__ void tile_full_kernel(const uint8_t *flags, int64_t ntiles, uint8_t *full) {
  constexpr uint64_t kFull8 = 0x0101010101010101ull *
                              (uint64_t)(CF_PRESENT | CF_NORMAL | CF_UPDATE | CF_PRIM | CF_RESNORM);
  const int64_t t = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  if (t >= ntiles) return;  // whole warps
  const uint64_t w = reinterpret_cast<const uint64_t *>(flags + t * kTileCells)[threadIdx.x & 31];
  const bool all = __all_sync(0xffffffffu, w == kFull8);
  if ((threadIdx.x & 31) == 0) full[t] = all ? 1 : 0;
}

// ... and the uniform tiles: full, with four full side neighbours (the
// stage kernel then needs no presence flags and no one-sided stencils).
// The topology upload makes them with the same two kernels.
__global__ void tile_uniform_kernel(const uint8_t *full, const int32_t *nb, int64_t ntiles,
                                    uint8_t *uniform) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= ntiles) return;
  bool u = full[t] != 0;
  for (int k = 1; k < 9 && u; k += 2) {
    const int n = nb[t * 9 + k];
    u = n >= 0 && full[n] != 0;
  }
  uniform[t] = u ? 1 : 0;
}

// Every stencil a face of a leaf cell reads must exist (NS_Solver.H:738-756,
// NS_Solver.cpp:410-424), checked per slot on the device over the tile
// neighbour table (which wraps periodic directions): per face direction d
// the face neighbour (check 0), one of the two outer MUSCL neighbours
// (check 1), and with viscosity the four tangential neighbours (check 2).
// The smallest (slot, d, check) that fails goes to *first as
// slot * 16 + d * 4 + check (~0 when none fails).
__device__ __forceinline__ bool slot_present(const uint8_t *flags, const int32_t *nb, int64_t t,
                                             int lx, int ly, int dx, int dy) {
  const int nx = lx + dx, ny = ly + dy;  // |dx|, |dy| <= 2: at most the next tile
  const int ox = nx < 0 ? -1 : (nx >= kTile ? 1 : 0), oy = ny < 0 ? -1 : (ny >= kTile ? 1 : 0);
  const int64_t tile = (ox == 0 && oy == 0) ? t : nb[t * 9 + (oy + 1) * 3 + (ox + 1)];
  if (tile < 0) return false;
  return (flags[tile * kTileCells + (ny - oy * kTile) * kTile + (nx - ox * kTile)] & CF_PRESENT) != 0;
}

__global__ void stencil_check_kernel(const uint8_t *flags, const int32_t *nb, int64_t nslots,
                                     int viscous, unsigned long long *first) {
  for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < nslots;
       s += (int64_t)gridDim.x * blockDim.x) {
    if (!(flags[s] & CF_NORMAL)) continue;
    const int64_t t = s / kTileCells;
    const int lx = (int)(s % kTile), ly = (int)((s / kTile) % kTile);
    for (int d = 0; d < 4; ++d) {
      const int dx = d == 0 ? -1 : d == 1 ? 1 : 0, dy = d == 2 ? -1 : d == 3 ? 1 : 0;
      int bad = -1;
      if (!slot_present(flags, nb, t, lx, ly, dx, dy)) {
        bad = 0;
      } else if (!slot_present(flags, nb, t, lx, ly, -dx, -dy) &&
                 !slot_present(flags, nb, t, lx, ly, 2 * dx, 2 * dy)) {
        bad = 1;
      } else if (viscous) {
        const int tx = dy != 0 ? 1 : 0, ty = dx != 0 ? 1 : 0;
        if (!slot_present(flags, nb, t, lx, ly, tx, ty) ||
            !slot_present(flags, nb, t, lx, ly, -tx, -ty) ||
            !slot_present(flags, nb, t, lx, ly, dx + tx, dy + ty) ||
            !slot_present(flags, nb, t, lx, ly, dx - tx, dy - ty))
          bad = 2;
      }
      if (bad >= 0) {
        atomicMin(first, (unsigned long long)s * 16ull + (unsigned long long)(d * 4 + bad));
        break;
      }
    }
  }
}

}  // namespace

extern "C" {

const char *ibgpu_errstr(int code) {
  switch (code) {
    case IBGPU_OK: return "ok";
    case IBGPU_E_ARG: return "invalid argument";
    case IBGPU_E_CUDA: return "CUDA runtime error";
    case IBGPU_E_STATE: return "call out of order (topology/state not uploaded)";
    case IBGPU_E_ABORT: return "solver abort condition (see ibgpu_diag.abort_code)";
    case IBGPU_E_NOMEM: return "device allocation failed";
    case IBGPU_E_TOPOLOGY: return "cell list cannot be laid out on the tiled mesh";
    case IBGPU_E_TIMEOUT: return "device-side wait ran out of its time limit";
    default: return "unknown error";
  }
}

const char *ibgpu_last_error(void) { return g_last_error.c_str(); }

int ibgpu_create(const ibgpu_case *cs, ibgpu_ctx **out) {
  if (!cs || !out) return IBGPU_E_ARG;
  *out = nullptr;
  int vrc = validate_case(cs);
  if (vrc) return vrc;
  ibgpu_ctx *c = new (std::nothrow) ibgpu_ctx();
  if (!c) return IBGPU_E_NOMEM;
  c->cs = *cs;
  fill_case_const(cs, c->cc);
  cudaError_t e = cudaGetDevice(&c->device);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, c->device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_ready, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_copied, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->in_stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_in_free, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_in_done, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaMalloc((void **)&c->d_diag, sizeof(DevDiag));
  if (e == cudaSuccess) e = cudaMallocHost((void **)&c->h_diag, sizeof(DevDiag));
  if (e == cudaSuccess) e = cudaMalloc((void **)&c->d_aux_err, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(c->d_aux_err, 0, sizeof(int));
  if (e != cudaSuccess) {
    int rc = cuda_fail(e, "ibgpu_create");
    ibgpu_destroy(c);
    return rc;
  }
  c->stream = c->own_stream;
  c->body_level = cs->body_level;
  *out = c;
  return IBGPU_OK;
}

int ibgpu_set_stream(ibgpu_ctx *ctx, void *stream) {
  if (!ctx) return IBGPU_E_ARG;
  ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
  return IBGPU_OK;
}

// Cell-list bits that fix the layout: a flag update may change every other
// bit of a row, never these.
static const uint8_t kLayoutBits = IBGPU_CELL_PRESENT | IBGPU_CELL_NORMAL | IBGPU_CELL_ALIAS;

int ibgpu_upload_topology(ibgpu_ctx *ctx, const ibgpu_cells *cells) {
  if (!ctx || !cells || cells->n < 0 || (cells->n > 0 && (!cells->level || !cells->ix ||
                                                          !cells->iy || !cells->flags)))
    return IBGPU_E_ARG;
  const ibgpu_case &cs = ctx->cs;
  const int nlev = cs.nlevels;
  const int64_t n = cells->n;
  CK(cudaStreamSynchronize(ctx->stream));
  if (ctx->copy_stream) cudaStreamSynchronize(ctx->copy_stream);  // pending downloads
  if (ctx->in_stream) cudaStreamSynchronize(ctx->in_stream);      // pending uploads
  ctx->download_pending = false;
  ctx->in_used = false;
  ctx->chain_open = false;  // a new mesh ends any chain of asynchronous steps
  ctx->chain_steps = 0;
  ctx->reset_layout();

  // 1. owners vs aliases; each level's tiles in a dense index over the
  //    bounding box of its owner cells' tiles (-1: no tile)
  std::vector<uint8_t> alias(n, 0);
  struct Grid {
    int x0 = 1 << 30, y0 = 1 << 30, x1 = -(1 << 30), y1 = -(1 << 30), w = 0;
    std::vector<int> idx;
    int at(int tx, int ty) const {
      if (tx < x0 || ty < y0 || tx > x1 || ty > y1) return -1;
      return idx[(size_t)(ty - y0) * w + (tx - x0)];
    }
    int &ref(int tx, int ty) { return idx[(size_t)(ty - y0) * w + (tx - x0)]; }
  };
  std::vector<Grid> grid(nlev);
  for (int64_t c = 0; c < n; ++c) {
    int l = cells->level[c];
    if (l < 0 || l >= nlev) { g_last_error = "cell level out of range"; return IBGPU_E_ARG; }
    if (!(cells->flags[c] & IBGPU_CELL_PRESENT)) { g_last_error = "cell without PRESENT flag"; return IBGPU_E_ARG; }
    int ix = cells->ix[c], iy = cells->iy[c];
    int ex = cs.domain_nx << l, ey = cs.domain_ny << l;
    bool out_periodic = (cs.periodic_x && (ix < 0 || ix >= ex)) || (cs.periodic_y && (iy < 0 || iy >= ey));
    if ((cells->flags[c] & IBGPU_CELL_ALIAS) || out_periodic) {
      if (cells->flags[c] & IBGPU_CELL_NORMAL) { g_last_error = "normal cell outside the periodic domain"; return IBGPU_E_TOPOLOGY; }
      alias[c] = 1;
      continue;
    }
    Grid &g = grid[l];
    const int tx = floordiv(ix, kTile), ty = floordiv(iy, kTile);
    g.x0 = std::min(g.x0, tx);
    g.y0 = std::min(g.y0, ty);
    g.x1 = std::max(g.x1, tx);
    g.y1 = std::max(g.y1, ty);
  }
  for (Grid &g : grid)
    if (g.x1 >= g.x0) {
      g.w = g.x1 - g.x0 + 1;
      g.idx.assign((size_t)g.w * (g.y1 - g.y0 + 1), -1);
    }
  std::vector<std::vector<std::pair<int, int>>> tiles(nlev);
  for (int64_t c = 0; c < n; ++c) {
    if (alias[c]) continue;
    const int l = cells->level[c];
    const int tx = floordiv(cells->ix[c], kTile), ty = floordiv(cells->iy[c], kTile);
    int &e = grid[l].ref(tx, ty);
    if (e == -1) {
      e = -2;
      tiles[l].push_back({tx, ty});
    }
  }
  for (int l = 0; l < nlev; ++l) {
    bool px = cs.periodic_x && ((cs.domain_nx << l) % kTile != 0);
    bool py = cs.periodic_y && ((cs.domain_ny << l) % kTile != 0);
    if ((px || py) && !tiles[l].empty()) {
      g_last_error = "periodic extent is not a multiple of the 16-cell tile";
      return IBGPU_E_TOPOLOGY;
    }
  }
  // 2. Morton order within a level, levels concatenated
  ctx->level_tile_begin.assign(nlev, 0);
  ctx->level_tile_count.assign(nlev, 0);
  std::vector<int32_t> h_tile_level;
  std::vector<std::pair<int, int>> tile_pos;
  std::vector<std::unordered_map<uint64_t, int>> tilemap(nlev);
  for (int l = 0; l < nlev; ++l) {
    auto &tl = tiles[l];
    int mx = grid[l].x0, my = grid[l].y0;
    std::sort(tl.begin(), tl.end(), [mx, my](const std::pair<int, int> &a, const std::pair<int, int> &b) {
      return morton2((uint32_t)(a.first - mx), (uint32_t)(a.second - my)) <
             morton2((uint32_t)(b.first - mx), (uint32_t)(b.second - my));
    });
    ctx->level_tile_begin[l] = (int)h_tile_level.size();
    ctx->level_tile_count[l] = (int)tl.size();
    tilemap[l].reserve(tl.size());
    for (auto &t : tl) {
      grid[l].ref(t.first, t.second) = (int)h_tile_level.size();
      tilemap[l][key2(t.first, t.second)] = (int)h_tile_level.size();
      h_tile_level.push_back(l);
      tile_pos.push_back(t);
    }
  }
  const int64_t ntiles = (int64_t)h_tile_level.size();
  const int64_t nslots = ntiles * kTileCells;
  if (nslots > INT32_MAX) { g_last_error = "mesh too large for 32-bit slot indices"; return IBGPU_E_TOPOLOGY; }
  // 3. neighbour table (periodic wrap at tile granularity)
  std::vector<int32_t> h_nb(ntiles * 9, -1);
  for (int64_t t = 0; t < ntiles; ++t) {
    int l = h_tile_level[t];
    int ntx = (cs.domain_nx << l) / kTile, nty = (cs.domain_ny << l) / kTile;
    for (int oy = -1; oy <= 1; ++oy)
      for (int ox = -1; ox <= 1; ++ox) {
        int tx = tile_pos[t].first + ox, ty = tile_pos[t].second + oy;
        if (cs.periodic_x) tx = ((tx % ntx) + ntx) % ntx;
        if (cs.periodic_y) ty = ((ty % nty) + nty) % nty;
        h_nb[t * 9 + (oy + 1) * 3 + (ox + 1)] = grid[l].at(tx, ty);
      }
  }
  // 4. slots of owner cells, then aliases
  std::vector<uint8_t> h_flags(nslots, 0);
  std::vector<int32_t> cell_slot(n, -1);
  ctx->h_slot_level.assign(nslots, -1);
  ctx->h_slot_ix.assign(nslots, 0);
  ctx->h_slot_iy.assign(nslots, 0);
  ctx->level_normal_cells.assign(nlev, 0);
  auto slot_of = [&](int l, int ix, int iy) -> int64_t {
    int tx = floordiv(ix, kTile), ty = floordiv(iy, kTile);
    const int t = grid[l].at(tx, ty);
    if (t < 0) return -1;
    return (int64_t)t * kTileCells + (iy - ty * kTile) * kTile + (ix - tx * kTile);
  };
  for (int64_t c = 0; c < n; ++c) {
    if (alias[c]) continue;
    int l = cells->level[c];
    int64_t s = slot_of(l, cells->ix[c], cells->iy[c]);
    if (h_flags[s]) { g_last_error = "two cells at one position"; return IBGPU_E_TOPOLOGY; }
    h_flags[s] = cells->flags[c] & 0x3f;
    cell_slot[c] = (int32_t)s;
    ctx->h_slot_level[s] = l;
    ctx->h_slot_ix[s] = cells->ix[c];
    ctx->h_slot_iy[s] = cells->iy[c];
    if (cells->flags[c] & IBGPU_CELL_NORMAL) ctx->level_normal_cells[l]++;
  }
  for (int64_t c = 0; c < n; ++c) {
    if (!alias[c]) continue;
    int l = cells->level[c];
    int ex = cs.domain_nx << l, ey = cs.domain_ny << l;
    int ix = cells->ix[c], iy = cells->iy[c];
    if (cs.periodic_x) ix = ((ix % ex) + ex) % ex;
    if (cs.periodic_y) iy = ((iy % ey) + ey) % ey;
    int64_t s = slot_of(l, ix, iy);
    if (s < 0 || !h_flags[s]) { g_last_error = "periodic ghost without a source cell"; return IBGPU_E_TOPOLOGY; }
    cell_slot[c] = (int32_t)s;
  }
  // 5. (the stencils of the leaf cells and 6. the uniform tiles are made on
  //    the device below)
  // 7. device arrays (a regrid's new layout reuses the old one's buffers
  //    where they are large enough)
  int rc;
  if ((rc = keep_alloc(ctx, &ctx->d_tile_nb, h_nb.size())) ||
      (rc = keep_alloc(ctx, &ctx->d_tile_level, (size_t)ntiles)) ||
      (rc = keep_alloc(ctx, &ctx->d_flags, (size_t)nslots)) ||
      (rc = keep_alloc(ctx, &ctx->d_tile_uniform, (size_t)ntiles)) ||
      (rc = keep_alloc(ctx, &ctx->d_tile_org, (size_t)ntiles)) ||
      (rc = keep_alloc(ctx, &ctx->d_cell_slot, (size_t)n)) ||
      (rc = keep_alloc(ctx, &ctx->d_cell_alias, (size_t)n)) ||
      (rc = keep_alloc(ctx, &ctx->d_cell_layout, (size_t)n)) ||
      (rc = keep_alloc(ctx, &ctx->d_row_flags, (size_t)n)) ||
      (rc = keep_alloc(ctx, &ctx->d_tile_full, (size_t)ntiles)) ||
      (rc = keep_alloc(ctx, &ctx->d_layout_err, (size_t)2)) ||  // also the stencil check's key
      (rc = keep_alloc(ctx, &ctx->d_rows, (size_t)n * 7)) ||
      // staging of asynchronous downloads, here so that the first one in a
      // pipelined loop does not allocate (and wait for the device)
      (rc = keep_alloc(ctx, &ctx->d_rows_out, (size_t)n * 7)))
    return rc;
  for (int f = 0; f < kStateFields; ++f)
    if ((rc = keep_alloc(ctx, &ctx->d_s0[f], (size_t)nslots))) return rc;
  const size_t buf_elem = cs.precision == IBGPU_MIXED ? sizeof(float) : sizeof(double);
  for (int b = 0; b < 2; ++b)
    for (int f = 0; f < 4; ++f)
      if ((rc = keep_alloc(ctx, (unsigned char **)&ctx->d_buf[b][f], (size_t)nslots * buf_elem))) return rc;
  if (cs.viscous && (rc = keep_alloc(ctx, &ctx->d_vsd, (size_t)nslots * 8))) return rc;
  cudaStream_t st = ctx->stream;
  CK(cudaMemcpyAsync(ctx->d_tile_nb, h_nb.data(), h_nb.size() * 4, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(ctx->d_tile_level, h_tile_level.data(), ntiles * 4, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(ctx->d_flags, h_flags.data(), nslots, cudaMemcpyHostToDevice, st));
  std::vector<int2> h_org(ntiles);
  for (int64_t t = 0; t < ntiles; ++t)
    h_org[t] = make_int2(tile_pos[t].first * kTile, tile_pos[t].second * kTile);
  if (ntiles > 0)
    CK(cudaMemcpyAsync(ctx->d_tile_org, h_org.data(), ntiles * sizeof(int2), cudaMemcpyHostToDevice, st));
  // 5. every stencil a face of a leaf cell reads exists (stencil_check_kernel)
  if (nslots > 0) {
    const unsigned long long none = ~0ull;
    unsigned long long first = none;
    unsigned long long *d_first = reinterpret_cast<unsigned long long *>(ctx->d_layout_err);
    CK(cudaMemcpyAsync(d_first, &none, sizeof(none), cudaMemcpyHostToDevice, st));
    stencil_check_kernel<<<4 * ctx->nsm, 256, 0, st>>>(ctx->d_flags, ctx->d_tile_nb, nslots,
                                                       cs.viscous != 0, d_first);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(&first, d_first, sizeof(first), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (first != none) {
      const int check = (int)(first & 3);
      g_last_error = check == 0 ? "leaf cell with a missing face neighbour"
                     : check == 1 ? "face stencil with neither outer neighbour"
                                  : "viscous stencil with a missing cell";
      return IBGPU_E_TOPOLOGY;
    }
    // 6. uniform tiles: full tiles whose four side neighbours are full
    tile_full_kernel<<<(unsigned)((ntiles * 32 + 255) / 256), 256, 0, st>>>(ctx->d_flags, ntiles,
                                                                            ctx->d_tile_full);
    tile_uniform_kernel<<<(unsigned)((ntiles + 255) / 256), 256, 0, st>>>(
        ctx->d_tile_full, ctx->d_tile_nb, ntiles, ctx->d_tile_uniform);
    CK(cudaGetLastError());
  }
  if (n > 0) {
    CK(cudaMemcpyAsync(ctx->d_cell_slot, cell_slot.data(), n * 4, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(ctx->d_cell_alias, alias.data(), n, cudaMemcpyHostToDevice, st));
  }
  // absent slots hold zeros in every field (never read as a stencil value)
  for (int f = 0; f < kStateFields; ++f) CK(cudaMemsetAsync(ctx->d_s0[f], 0, nslots * 8, st));
  for (int b = 0; b < 2; ++b)
    for (int f = 0; f < 4; ++f) CK(cudaMemsetAsync(ctx->d_buf[b][f], 0, nslots * buf_elem, st));
  if (ctx->d_vsd) CK(cudaMemsetAsync(ctx->d_vsd, 0, nslots * 8 * 8, st));
  CK(cudaStreamSynchronize(st));
  ctx->tilemap = std::move(tilemap);
  // each row's layout bits, against which ibgpu_update_flags checks new flags
  std::vector<uint8_t> layout(n);
  for (int64_t c = 0; c < n; ++c)
    layout[c] = (cells->flags[c] & kLayoutBits) | (alias[c] ? IBGPU_CELL_ALIAS : 0);
  if (n > 0) {
    CK(cudaMemcpyAsync(ctx->d_cell_layout, layout.data(), n, cudaMemcpyHostToDevice, st));
    CK(cudaStreamSynchronize(st));
  }
  ctx->h_flags_present.assign(nslots, 0);
  for (int64_t s = 0; s < nslots; ++s) ctx->h_flags_present[s] = (h_flags[s] & CF_PRESENT) ? 1 : 0;
  ctx->ncells = n;
  ctx->ntiles = ntiles;
  ctx->nslots = nslots;
  ctx->has_topology = true;
  return IBGPU_OK;
}


}  // extern "C"

// New flags of n rows (all rows in order when which is null, else rows
// which[k]) into the device's slot flags, then the uniform tiles anew.
static int update_flags_on_device(ibgpu_ctx *ctx, int64_t n, const int64_t *which,
                                  const uint8_t *flags) {
  if (ctx->chain_open) {
    g_last_error = "asynchronous steps pending: call ibgpu_step_result first";
    return IBGPU_E_STATE;
  }
  if (n == 0) return IBGPU_OK;
  cudaStream_t st = ctx->stream;
  const int grid = 4 * ctx->nsm;
  const int64_t nt = ctx->ntiles;
  int rc;
  uint8_t *d_rows = ctx->d_row_flags;  // room for every row
  int64_t *d_which = nullptr;
  if (which) {
    // the previous step may still read the staging buffer of an earlier call
    if ((size_t)n > ctx->cap[&ctx->d_row_which]) CK(cudaStreamSynchronize(st));
    if ((rc = keep_alloc(ctx, &ctx->d_row_which, (size_t)n))) return rc;
    if ((rc = keep_alloc(ctx, &ctx->d_row_sub, (size_t)n))) return rc;
    d_which = ctx->d_row_which;
    d_rows = ctx->d_row_sub;
    CK(cudaMemcpyAsync(d_which, which, n * sizeof(int64_t), cudaMemcpyHostToDevice, st));
  }
  // the flags and the layout check first: nothing changes on the device
  // when a row's layout bits differ
  const int big = INT32_MAX;
  CK(cudaMemcpyAsync(d_rows, flags, n, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(ctx->d_layout_err, &big, sizeof(int), cudaMemcpyHostToDevice, st));
  layout_check_kernel<<<grid, 256, 0, st>>>(d_rows, d_which, ctx->d_cell_layout, n,
                                            ctx->d_layout_err);
  CK(cudaGetLastError());
  int bad = big;
  CK(cudaMemcpyAsync(&bad, ctx->d_layout_err, sizeof(int), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if (bad != big) {
    g_last_error = "a row changed its PRESENT, NORMAL or ALIAS bit: upload the topology";
    return IBGPU_E_TOPOLOGY;
  }
  flags_scatter_kernel<<<grid, 256, 0, st>>>(d_rows, d_which, ctx->d_cell_layout,
                                             ctx->d_cell_slot, n, ctx->d_flags);
  if (nt > 0) {
    tile_full_kernel<<<(unsigned)((nt * 32 + 255) / 256), 256, 0, st>>>(ctx->d_flags, nt,
                                                                        ctx->d_tile_full);
    tile_uniform_kernel<<<(unsigned)((nt + 255) / 256), 256, 0, st>>>(ctx->d_tile_full,
                                                                      ctx->d_tile_nb, nt,
                                                                      ctx->d_tile_uniform);
  }
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(st));
  return IBGPU_OK;
}

extern "C" {

int ibgpu_update_flags(ibgpu_ctx *ctx, const uint8_t *flags) {
  if (!ctx || (!flags && ctx->ncells > 0)) return IBGPU_E_ARG;
  if (!ctx->has_topology) return IBGPU_E_STATE;
  return update_flags_on_device(ctx, ctx->ncells, nullptr, flags);
}

int ibgpu_update_flags_rows(ibgpu_ctx *ctx, int64_t n, const int64_t *rows,
                            const uint8_t *flags) {
  if (!ctx || n < 0 || (n > 0 && (!rows || !flags))) return IBGPU_E_ARG;
  if (!ctx->has_topology) return IBGPU_E_STATE;
  for (int64_t k = 0; k < n; ++k)
    if (rows[k] < 0 || rows[k] >= ctx->ncells) {
      g_last_error = "flag update: a row index outside the topology's rows";
      return IBGPU_E_ARG;
    }
  return update_flags_on_device(ctx, n, rows, flags);
}

int ibgpu_layout_info(const ibgpu_ctx *ctx, int64_t *nslots, int64_t *ntiles) {
  if (!ctx) return IBGPU_E_ARG;
  if (nslots) *nslots = ctx->nslots;
  if (ntiles) *ntiles = ctx->ntiles;
  return IBGPU_OK;
}

// Work on the context's stream that writes the state waits for an
// asynchronous download still reading it.
static int order_after_download(ibgpu_ctx *ctx, cudaStream_t st) {
  if (ctx->download_pending) {
    CK(cudaStreamWaitEvent(st, ctx->ev_copied, 0));
    ctx->download_pending = false;
  }
  return IBGPU_OK;
}

// Scatter / gather of the staged state rows in the context's row format.
static void scatter_rows(ibgpu_ctx *ctx, const double *rows, cudaStream_t st) {
  if (ctx->row_fields == 4)
    fast::launch_scatter4(rows, ctx->d_cell_slot, ctx->d_cell_alias, ctx->ncells, ctx->cs.Rg,
                          ctx->cs.Cv, ctx->d_s0, ctx->nsm, st);
  else
    fast::launch_scatter(rows, ctx->d_cell_slot, ctx->d_cell_alias, ctx->ncells, ctx->d_s0,
                         ctx->nsm, st);
}
static void gather_rows(ibgpu_ctx *ctx, double *rows, cudaStream_t st) {
  if (ctx->row_fields == 4) fast::launch_gather4(rows, ctx->d_cell_slot, ctx->ncells, ctx->d_s0, ctx->nsm, st);
  else fast::launch_gather(rows, ctx->d_cell_slot, ctx->ncells, ctx->d_s0, ctx->nsm, st);
}

int ibgpu_set_state_rows(ibgpu_ctx *ctx, int fields) {
  if (!ctx || (fields != IBGPU_ROWS_FLOWVARS && fields != IBGPU_ROWS_COMPACT)) return IBGPU_E_ARG;
  if (ctx->chain_open || ctx->download_pending || ctx->in_used) {
    // transfers in flight use the current format's buffer layout
    CK(cudaStreamSynchronize(ctx->stream));
    CK(cudaStreamSynchronize(ctx->in_stream));
    CK(cudaStreamSynchronize(ctx->copy_stream));
    ctx->download_pending = false;
    ctx->in_used = false;
  }
  ctx->row_fields = fields;
  return IBGPU_OK;
}

int ibgpu_upload_state(ibgpu_ctx *ctx, const double *prim) {
  if (!ctx || (!prim && ctx->ncells > 0)) return IBGPU_E_ARG;
  if (!ctx->has_topology) return IBGPU_E_STATE;
  cudaStream_t st = ctx->stream;
  if (ctx->ncells > 0) {
    // the host-to-device copy may overlap a pending download (other buffer,
    // other copy direction); the scatter into the state waits for it
    CK(cudaMemcpyAsync(ctx->d_rows, prim, ctx->ncells * ctx->row_fields * sizeof(double),
                       cudaMemcpyHostToDevice, st));
    int rc = order_after_download(ctx, st);
    if (rc) return rc;
    scatter_rows(ctx, ctx->d_rows, st);
    CK(cudaGetLastError());
  }
  CK(cudaStreamSynchronize(st));
  ctx->has_state = true;
  return IBGPU_OK;
}

int ibgpu_download_state(ibgpu_ctx *ctx, double *prim) {
  if (!ctx || (!prim && ctx->ncells > 0)) return IBGPU_E_ARG;
  if (!ctx->has_state) return IBGPU_E_STATE;
  cudaStream_t st = ctx->stream;
  if (ctx->ncells > 0) {
    gather_rows(ctx, ctx->d_rows, st);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(prim, ctx->d_rows, ctx->ncells * ctx->row_fields * sizeof(double),
                       cudaMemcpyDeviceToHost, st));
  }
  CK(cudaStreamSynchronize(st));
  return IBGPU_OK;
}

int ibgpu_download_state_async(ibgpu_ctx *ctx, double *prim) {
  if (!ctx || (!prim && ctx->ncells > 0)) return IBGPU_E_ARG;
  if (!ctx->has_state) return IBGPU_E_STATE;
  if (ctx->ncells == 0) return IBGPU_OK;
  CK(cudaEventRecord(ctx->ev_ready, ctx->stream));
  CK(cudaStreamWaitEvent(ctx->copy_stream, ctx->ev_ready, 0));
  gather_rows(ctx, ctx->d_rows_out, ctx->copy_stream);
  CK(cudaGetLastError());
  CK(cudaEventRecord(ctx->ev_copied, ctx->copy_stream));
  ctx->download_pending = true;
  CK(cudaMemcpyAsync(prim, ctx->d_rows_out, ctx->ncells * ctx->row_fields * sizeof(double),
                     cudaMemcpyDeviceToHost, ctx->copy_stream));
  return IBGPU_OK;
}

int ibgpu_synchronize(ibgpu_ctx *ctx) {
  if (!ctx) return IBGPU_E_ARG;
  CK(cudaStreamSynchronize(ctx->stream));
  CK(cudaStreamSynchronize(ctx->in_stream));
  CK(cudaStreamSynchronize(ctx->copy_stream));
  ctx->download_pending = false;
  return IBGPU_OK;
}

int ibgpu_set_kernel_timing(ibgpu_ctx *ctx, int enable) {
  if (!ctx) return IBGPU_E_ARG;
  ctx->timing = enable != 0;
  for (int k = 0; k < 3; ++k) {
    ctx->kms[k] = 0.0;
    ctx->klaunch[k] = 0;
  }
  return IBGPU_OK;
}

int ibgpu_kernel_times(const ibgpu_ctx *ctx, double ms_out[3], int64_t launches_out[3]) {
  if (!ctx) return IBGPU_E_ARG;
  for (int k = 0; k < 3; ++k) {
    if (ms_out) ms_out[k] = ctx->kms[k];
    if (launches_out) launches_out[k] = ctx->klaunch[k];
  }
  return IBGPU_OK;
}

namespace {

// Event timing of the dominant kernels of one run (kind 0 stage, 1 viscous,
// 2 CFL), read back after the run's synchronisation.
struct RunTimer {
  ibgpu_ctx *ctx;
  cudaStream_t st;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> evs;
  std::vector<int> kind;
  bool off = false;  // asynchronous steps are not timed
  cudaEvent_t mark(int k) {
    if (off || !ctx->timing) return nullptr;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, st);
    evs.push_back({a, b});
    kind.push_back(k);
    return b;
  }
  void done(cudaEvent_t b) {
    if (b) cudaEventRecord(b, st);
  }
  void collect() {
    for (size_t i = 0; i < evs.size(); ++i) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, evs[i].first, evs[i].second);
      ctx->kms[kind[i]] += ms;
      ctx->klaunch[kind[i]] += 1;
      cudaEventDestroy(evs[i].first);
      cudaEventDestroy(evs[i].second);
    }
    evs.clear();
    kind.clear();
  }
};

// Device diag of a run: dt in, CFL/residual reductions reset, no abort.
int begin_diag(ibgpu_ctx *ctx, double dt, cudaStream_t st) {
  DevDiag *hd = ctx->h_diag;
  std::memset(hd, 0, sizeof(DevDiag));
  hd->dt = dt;
  double cfl_init = 10000.0;
  std::memcpy(&hd->cfl_bits, &cfl_init, sizeof(double));
  hd->err_key = ~0ull;
  std::memcpy(&hd->cfl_next_bits, &cfl_init, sizeof(double));
  CK(cudaMemcpyAsync(ctx->d_diag, hd, sizeof(DevDiag), cudaMemcpyHostToDevice, st));
  return IBGPU_OK;
}

// Whether the final stage folds in the next step's CFL pass: one level (all
// cells march every step), no immersed body (the immersed-boundary fill
// rewrites normal cells between the stages and the CFL pass) and a CFL pass
// every step.
bool folds_cfl(const ibgpu_ctx *ctx) {
  return ctx->cs.nlevels == 1 && ctx->body_level < 0 && ctx->n_ib == 0 &&
         ctx->cs.dt_var_step == 1;
}

// Everything of step ts before the stages (main.cpp:87-89 and the frozen
// part of NS_Solver::TimeMarching): reduction reset, restriction and
// prolongation on their schedules, immersed-body ghosts, CFL dt, domain
// ghosts and the viscous flux of the levels that march.
int enqueue_prestage(ibgpu_ctx *ctx, int ts, int step, cudaStream_t st, RunTimer &tm,
                     bool batched = false, bool fresh_cfl = false,
                     const int *phase_base = nullptr) {
  const ibgpu_case &cs = ctx->cs;
  const bool exact = cs.precision == IBGPU_FP64_EXACT;
  const bool mixed = cs.precision == IBGPU_MIXED;
  const int pbase = 8 * step;  // abort-order phases of this step
  // a batch resets the reductions and runs the CFL pass of all its cases in
  // merged launches (the CFL pass reads normal cells only, which the domain
  // ghosts and the viscous pass below do not write, so it may follow them)
  if (step > 0 && !batched) {
    if (exact) exact::launch_step_begin(ctx->d_diag, st);
    else fast::launch_step_begin(ctx->d_diag, st);
  }
  // AMR::InterfaceExchange (AMRInterface.cpp:3-35): restriction of every
  // scheduled pair (coarse level ascending), then prolongation
  for (int l = 0; l + 1 < cs.nlevels && l < (int)ctx->res.size(); ++l) {
    if (ts % cs.average_step[l + 1] != cs.average_left[l + 1] || ctx->res[l].n == 0) continue;
    PairArgs pa;
    pa.coarse = ctx->res[l].coarse;
    pa.fine = ctx->res[l].fine;
    pa.nb = nullptr;
    pa.n = ctx->res[l].n;
    for (int f = 0; f < kStateFields; ++f) pa.s0[f] = ctx->d_s0[f];
    if (exact) exact::launch_restrict(pa, ctx->cc, st);
    else fast::launch_restrict(pa, ctx->cc, st);
    CK(cudaGetLastError());
  }
  for (int l = 0; l + 1 < cs.nlevels && l < (int)ctx->pro.size(); ++l) {
    if (ts % cs.prolong_step[l + 1] != cs.prolong_left[l + 1] || ctx->pro[l].n == 0) continue;
    PairArgs pa;
    pa.coarse = ctx->pro[l].coarse;
    pa.fine = ctx->pro[l].fine;
    pa.nb = ctx->pro[l].nb;
    pa.n = ctx->pro[l].n;
    for (int f = 0; f < kStateFields; ++f) pa.s0[f] = ctx->d_s0[f];
    if (exact) exact::launch_prolong(pa, ctx->cc, st);
    else fast::launch_prolong(pa, ctx->cc, st);
    CK(cudaGetLastError());
  }
  // Body::IBConditions_Image (static bodies): IB ghost cells of the finest level
  if (ctx->n_ib > 0) {
    IbArgs ia;
    ia.cell = ctx->d_ib_cell;
    ia.intp = ctx->d_ib_intp;
    ia.cellf = ctx->d_ib_f;
    ia.out = ctx->d_ib_out;
    ia.n = ctx->n_ib;
    for (int f = 0; f < kStateFields; ++f) ia.s0[f] = ctx->d_s0[f];
    // the abort-order phase of this step: from the host, or (a captured
    // batch step replayed for every step) from the batch's device counter
    ia.phase = phase_base ? 0 : pbase + 0;
    ia.phase_base = phase_base;
    ia.diag = ctx->d_diag;
    if (exact) exact::launch_ib(ia, ctx->cc, st);
    else fast::launch_ib(ia, ctx->cc, st);
    CK(cudaGetLastError());
  }

  // CFL time step (TimeMarching: Comptdt when ts % dt_var_step == 0); from
  // the second step of a run that folds it into the final stage, the
  // previous step already accumulated the bound
  if (!batched && (ts % cs.dt_var_step) == 0 && step > 0 && !fresh_cfl && folds_cfl(ctx)) {
    cudaEvent_t e = tm.mark(2);
    if (exact) exact::launch_take_folded_cfl(ctx->d_diag, ctx->cc, st);
    else fast::launch_take_folded_cfl(ctx->d_diag, ctx->cc, st);
    tm.done(e);
    CK(cudaGetLastError());
  } else if (!batched && (ts % cs.dt_var_step) == 0) {
    CflArgs ca;
    ca.tile_level = ctx->d_tile_level;
    ca.flags = ctx->d_flags;
    for (int f = 0; f < kStateFields; ++f) ca.s0[f] = ctx->d_s0[f];
    ca.nslots = ctx->nslots;
    ca.phase = pbase + 1;
    ca.diag = ctx->d_diag;
    cudaEvent_t e = tm.mark(2);
    if (exact) exact::launch_cfl(ca, ctx->cc, ctx->nsm, st);
    else fast::launch_cfl(ca, ctx->cc, ctx->nsm, st);
    tm.done(e);
    CK(cudaGetLastError());
  }

  // BCValues::BCBoxTreat over the levels that march at ts, by dependency wave
  for (int l = 0; l < cs.nlevels && l < (int)ctx->bc_waves.size(); ++l) {
    if (ts % cs.march_step[l] != cs.march_left[l]) continue;
    for (auto &w : ctx->bc_waves[l]) {
      BcArgs ba;
      ba.ghost = ctx->d_bc_ghost;
      ba.ref = ctx->d_bc_ref;
      ba.type = ctx->d_bc_type;
      ba.face = ctx->d_bc_face;
      ba.nmv = ctx->d_bc_nmv;
      ba.facevar = ctx->d_facevar;
      ba.begin = w.first;
      ba.end = w.second;
      ba.backpressure = ctx->backpressure;
      ba.cos_in = ctx->cos_in;
      ba.sin_in = ctx->sin_in;
      for (int f = 0; f < kStateFields; ++f) ba.s0[f] = ctx->d_s0[f];
      if (exact) exact::launch_bc(ba, ctx->cc, st);
      else fast::launch_bc(ba, ctx->cc, st);
      CK(cudaGetLastError());
    }
  }
  // NS_Solver::ComptViscousStress, frozen for the stages
  if (cs.viscous) {
    ViscArgs va;
    va.tile_nb = ctx->d_tile_nb;
    va.tile_level = ctx->d_tile_level;
    va.flags = ctx->d_flags;
    for (int f = 0; f < kStateFields; ++f) va.s0[f] = ctx->d_s0[f];
    va.vsd = ctx->d_vsd;
    va.nslots = ctx->nslots;
    for (int l = 0; l < cs.nlevels; ++l) {
      if (ts % cs.march_step[l] != cs.march_left[l]) continue;
      va.tile_begin = ctx->level_tile_begin[l];
      cudaEvent_t e = tm.mark(1);
      if (exact) exact::launch_viscous(va, ctx->cc, ctx->level_tile_count[l], false, st);
      else fast::launch_viscous(va, ctx->cc, ctx->level_tile_count[l], mixed, st);
      tm.done(e);
      CK(cudaGetLastError());
    }
  }
  return IBGPU_OK;
}

// Stage arguments of stage k (ping-pong stage buffers; the final stage
// writes the step state).
void stage_args(const ibgpu_ctx *ctx, int k, StageArgs &sa) {
  const ibgpu_case &cs = ctx->cs;
  std::memset(&sa, 0, sizeof(sa));
  sa.tile_nb = ctx->d_tile_nb;
  sa.tile_level = ctx->d_tile_level;
  sa.tile_uniform = ctx->d_tile_uniform;
  sa.flags = ctx->d_flags;
  for (int f = 0; f < kStateFields; ++f) sa.s0[f] = ctx->d_s0[f];
  sa.vsd = ctx->d_vsd;
  sa.nslots = ctx->nslots;
  sa.diag = ctx->d_diag;
  const bool fin = (k == cs.nstages - 1);
  static const int map[4] = {F_RHO, F_U, F_V, F_P};
  for (int f = 0; f < 4; ++f) {
    sa.v.sin[f] = (k == 0) ? ctx->d_s0[map[f]] : ctx->d_buf[(k - 1) & 1][f];
    sa.v.sout[f] = fin ? nullptr : ctx->d_buf[k & 1][f];
  }
  sa.v.tp = cs.tp[k];
  // one wave of resident stage CTAs (4 per SM FP64, 6 mixed)
  sa.prefetch = ctx->nsm * (cs.precision == IBGPU_MIXED ? 6 : 4);
}

int64_t marched_cells(const ibgpu_ctx *ctx, int ts) {
  int64_t m = 0;
  for (int l = 0; l < ctx->cs.nlevels; ++l)
    if (ts % ctx->cs.march_step[l] == ctx->cs.march_left[l]) m += ctx->level_normal_cells[l];
  return m;
}

// The first abort of the run in the reference's order, dt and the
// reductions of the last step, from the device diag already copied to
// ctx->h_diag.
int decode_diag(ibgpu_ctx *ctx, int64_t marched, double *dt, ibgpu_diag *diag) {
  DevDiag *hd = ctx->h_diag;
  int abort_code = 0, abort_slot = -1, abort_step = 0;
  if (hd->err_key != ~0ull) {
    int check = (int)((hd->err_key >> 32) & 0xff);
    abort_step = (int)((hd->err_key >> 40) / 8);
    abort_slot = (int)(hd->err_key & 0xffffffffull);
    if (check == ERR_IB_NEG_T) abort_code = 1050;
    else if (check == ERR_IB_NAN) abort_code = 1076;
    else if (check == ERR_CFL_NEG_DT) abort_code = 424;
    else if (check == ERR_NEG_T) abort_code = 37;
    else {
      // UpdateConsVars: 611 on the finest level of a run with bodies, else 523
      int lvl = (abort_slot >= 0 && abort_slot < ctx->nslots) ? ctx->h_slot_level[abort_slot] : 0;
      abort_code = (ctx->body_level >= 0 && lvl == ctx->body_level) ? 611 : 523;
    }
  }
  *dt = hd->dt;
  if (diag) {
    std::memset(diag, 0, sizeof(*diag));
    diag->dt = hd->dt;
    std::memcpy(&diag->cfl_dt, &hd->cfl_bits, sizeof(double));
    for (int c = 0; c < 5; ++c) std::memcpy(&diag->res_max[c], &hd->res_bits[c], sizeof(double));
    diag->cells_marched = marched;
    diag->abort_code = abort_code;
    diag->abort_step = abort_step;
    if (abort_code && abort_slot >= 0 && abort_slot < ctx->nslots) {
      diag->abort_level = ctx->h_slot_level[abort_slot];
      diag->abort_ix = ctx->h_slot_ix[abort_slot];
      diag->abort_iy = ctx->h_slot_iy[abort_slot];
    }
  }
  if (abort_code) return IBGPU_E_ABORT;
  for (int c = 0; c < 5; ++c) {
    double v;
    std::memcpy(&v, &hd->res_bits[c], sizeof(double));
    if (v != v) {  // NaN residual (NS_Solver.H:355-361)
      if (diag) diag->abort_code = 268;
      return IBGPU_E_ABORT;
    }
  }
  return IBGPU_OK;
}

}  // namespace

// asynchronous steps between two ibgpu_step_result calls (abort-order phases
// 8 * step + p stay below 2^24)
constexpr int kMaxChainSteps = 1 << 20;

// The stages of step ts (index `step` of its run: abort-order phases) over
// the tiles of the levels that march at ts; fold_next: the final stage
// accumulates the next step's CFL bound where the case allows it.
static int enqueue_stages(ibgpu_ctx *ctx, int ts, int step, bool fold_next, cudaStream_t st,
                          RunTimer &tm) {
  const ibgpu_case &cs = ctx->cs;
  const bool exact = cs.precision == IBGPU_FP64_EXACT;
  const bool mixed = cs.precision == IBGPU_MIXED;
  for (int k = 0; k < cs.nstages; ++k) {
    StageArgs sa;
    stage_args(ctx, k, sa);
    sa.phase = 8 * step + 2 + k;
    const bool fin = (k == cs.nstages - 1);
    if (fin && fold_next && folds_cfl(ctx)) sa.v.cfl_next = 1 + 8 * (step + 1) + 1;
    for (int l = 0; l < cs.nlevels; ++l) {
      if (ts % cs.march_step[l] != cs.march_left[l]) continue;
      sa.tile_begin = ctx->level_tile_begin[l];
      cudaEvent_t e = tm.mark(0);
      if (exact) exact::launch_stage(sa, ctx->cc, ctx->level_tile_count[l], cs.limiter, cs.viscous != 0, fin, false, k, st);
      else fast::launch_stage(sa, ctx->cc, ctx->level_tile_count[l], cs.limiter, cs.viscous != 0, fin, mixed, k, st);
      tm.done(e);
      CK(cudaGetLastError());
    }
  }
  return IBGPU_OK;
}

static int run_steps(ibgpu_ctx *ctx, int ts0, int nsteps, double *dt, ibgpu_diag *diag) {
  if (!ctx || !dt || ts0 < 0 || nsteps < 1) return IBGPU_E_ARG;
  if (!ctx->has_state) return IBGPU_E_STATE;
  if (ctx->chain_open) {
    g_last_error = "asynchronous steps pending: call ibgpu_step_result first";
    return IBGPU_E_STATE;
  }
  cudaStream_t st = ctx->stream;
  int rc = order_after_download(ctx, st);
  if (rc) return rc;
  if ((rc = begin_diag(ctx, *dt, st))) return rc;
  RunTimer tm{ctx, st, {}, {}};
  int64_t marched = 0;
  for (int step = 0; step < nsteps; ++step) {
    const int ts = ts0 + step;
    if ((rc = enqueue_prestage(ctx, ts, step, st, tm))) return rc;
    marched = marched_cells(ctx, ts);
    if ((rc = enqueue_stages(ctx, ts, step, step + 1 < nsteps, st, tm))) return rc;
  }
  CK(cudaMemcpyAsync(ctx->h_diag, ctx->d_diag, sizeof(DevDiag), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  tm.collect();
  return decode_diag(ctx, marched, dt, diag);
}

int ibgpu_step(ibgpu_ctx *ctx, int ts, double *dt, ibgpu_diag *diag) {
  return run_steps(ctx, ts, 1, dt, diag);
}

int ibgpu_run(ibgpu_ctx *ctx, int ts0, int nsteps, double *dt, ibgpu_diag *diag) {
  return run_steps(ctx, ts0, nsteps, dt, diag);
}

int ibgpu_upload_state_async(ibgpu_ctx *ctx, const double *prim) {
  if (!ctx || (!prim && ctx->ncells > 0)) return IBGPU_E_ARG;
  if (!ctx->has_topology) return IBGPU_E_STATE;
  if (ctx->ncells > 0) {
    cudaStream_t st = ctx->stream;
    // the rows buffer is free once the previous upload's scatter has run
    if (ctx->in_used) CK(cudaStreamWaitEvent(ctx->in_stream, ctx->ev_in_free, 0));
    CK(cudaMemcpyAsync(ctx->d_rows, prim, ctx->ncells * ctx->row_fields * sizeof(double),
                       cudaMemcpyHostToDevice, ctx->in_stream));
    CK(cudaEventRecord(ctx->ev_in_done, ctx->in_stream));
    // the scatter follows the copy and the context's pending work, and
    // overwrites the state a pending download still reads only after it
    CK(cudaStreamWaitEvent(st, ctx->ev_in_done, 0));
    int rc = order_after_download(ctx, st);
    if (rc) return rc;
    scatter_rows(ctx, ctx->d_rows, st);
    CK(cudaGetLastError());
    CK(cudaEventRecord(ctx->ev_in_free, st));
    ctx->in_used = true;
  }
  ctx->has_state = true;
  return IBGPU_OK;
}

int ibgpu_step_async(ibgpu_ctx *ctx, int ts, double dt) {
  if (!ctx || ts < 0) return IBGPU_E_ARG;
  if (!ctx->has_state) return IBGPU_E_STATE;
  if (ctx->chain_steps >= kMaxChainSteps) {
    g_last_error = "too many asynchronous steps: call ibgpu_step_result";
    return IBGPU_E_ARG;
  }
  cudaStream_t st = ctx->stream;
  int rc = order_after_download(ctx, st);
  if (rc) return rc;
  if (!ctx->chain_open) {
    if (!(dt > 0.0)) return IBGPU_E_ARG;
    if ((rc = begin_diag(ctx, dt, st))) return rc;
    ctx->chain_open = true;
    ctx->chain_steps = 0;
  }
  RunTimer tm{ctx, st, {}, {}};
  tm.off = true;
  // a fresh CFL pass every step (the state may have been replaced since the
  // previous one), so no fold into the final stage either
  const int step = ctx->chain_steps;
  if ((rc = enqueue_prestage(ctx, ts, step, st, tm, false, true))) return rc;
  if ((rc = enqueue_stages(ctx, ts, step, false, st, tm))) return rc;
  ctx->chain_marched = marched_cells(ctx, ts);
  ctx->chain_steps = step + 1;
  return IBGPU_OK;
}

int ibgpu_step_result(ibgpu_ctx *ctx, double *dt, ibgpu_diag *diag) {
  if (!ctx || !dt) return IBGPU_E_ARG;
  if (!ctx->chain_open) return IBGPU_E_STATE;
  cudaStream_t st = ctx->stream;
  CK(cudaMemcpyAsync(ctx->h_diag, ctx->d_diag, sizeof(DevDiag), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  ctx->chain_open = false;
  ctx->chain_steps = 0;
  return decode_diag(ctx, ctx->chain_marched, dt, diag);
}

// ---------------------------------------------------------------------------
// Batched cases: the stage launches of every case merged into one persistent
// launch over a (case, tile) work list, replayed from a CUDA graph.
struct ibgpu_batch {
  std::vector<ibgpu_ctx *> cases;
  cudaStream_t stream = nullptr;
  int nsm = 148, nstages = 0, limiter = 0, period = 1;
  bool visc = false, mixed = false;
  StageArgs *d_args = nullptr;     // [case * nstages + k]
  CaseConst *d_ccs = nullptr;      // [case]
  int *d_phase_base = nullptr;
  std::vector<int2 *> d_work;      // per schedule phase r = ts % period
  std::vector<int> nwork;
  // whole-step graphs (every case's ghost fills and viscous pass on parallel
  // branches, then the merged CFL and stage launches), captured on first use
  // per (ts % full_period, CFL variant)
  std::map<int, cudaGraphExec_t> graphs;
  bool graphs_ready = false;  // every phase's graphs captured (first run after tuning)
  int full_period = 1;  // every schedule of every case repeats with it
  std::vector<cudaStream_t> fork;  // branches of the captured steps
  std::vector<cudaEvent_t> ev_fork_join;
  int2 *d_cfl_work = nullptr;      // every tile of every case
  int ncfl = 0, dt_var_step = 1;
  // cases with different CFL intervals (each dividing the schedule period):
  // per phase r the tiles and the indices of the cases whose CFL pass runs
  // when ts % period == r
  bool mixed_cfl = false;
  std::vector<int2 *> d_cfl_work_r;
  std::vector<int *> d_cfl_cases_r;
  std::vector<int> ncfl_r, ncfl_cases_r;
  bool folds = false;  // every case single-level without bodies: CFL folded into final stages
  int grid = 0;                    // CTAs of the persistent launch (0 = one per item)
  int device = 0;
  int table = -1;       // byte offset of the arguments in the constant-memory table (-1: global)
  int table_bytes = 0;  // bytes reserved there
  bool tuned = false;
  int *h_err = nullptr;  // pinned: the cases' time-out flags (batch tagging)
  std::vector<cudaEvent_t> ev_tag;  // batch tagging: per case, + the fork
  int fixed_grid = -1;  // >= 0: CTA count set by the caller (no autotuning)
  int threads = 0;        // threads per CTA of the merged stage launch (256 / 288)
  int fixed_threads = 0;  // set by the caller (0: autotuned)
  bool timing = false;
  double stage_ms = 0.0;
  int64_t stage_launches = 0;
  std::vector<int> tune_grid, tune_threads;
  std::vector<float> tune_ms;

  void drop_graphs() {
    for (auto &g : graphs)
      if (g.second) cudaGraphExecDestroy(g.second);
    graphs.clear();
    graphs_ready = false;
  }
  void release() {
    drop_graphs();
    for (auto f : fork) cudaStreamDestroy(f);
    fork.clear();
    for (auto e : ev_fork_join) cudaEventDestroy(e);
    ev_fork_join.clear();
    for (auto w : d_work) cudaFree(w);
    d_work.clear();
    cudaFree(d_cfl_work);
    d_cfl_work = nullptr;
    for (auto w : d_cfl_work_r) cudaFree(w);
    for (auto w : d_cfl_cases_r) cudaFree(w);
    d_cfl_work_r.clear();
    d_cfl_cases_r.clear();
    cudaFree(d_args);
    cudaFree(d_ccs);
    cudaFree(d_phase_base);
    d_args = nullptr;
    d_ccs = nullptr;
    d_phase_base = nullptr;
    fast::batch_table_release(device, table);
    table = -1;
    table_bytes = 0;
    if (h_err) cudaFreeHost(h_err);
    h_err = nullptr;
    for (auto e : ev_tag) cudaEventDestroy(e);
    ev_tag.clear();
  }
};

namespace {

// cfl: 0 none, 1 the CFL pass, 2 the bound folded into the previous step
int enqueue_batch_stages(ibgpu_batch *b, int r, int cfl, cudaStream_t st) {
  if (cfl == 1 && b->mixed_cfl) {
    if (b->ncfl_cases_r[r] > 0) {  // (phases without a CFL pass never take this graph)
      fast::launch_cfl_batch(b->d_args, b->d_ccs, b->d_cfl_work_r[r], b->ncfl_r[r], b->nstages,
                             b->d_phase_base, b->ncfl_cases_r[r], 0, st, b->d_cfl_cases_r[r]);
      CK(cudaGetLastError());
    }
  } else if (cfl == 1) {
    fast::launch_cfl_batch(b->d_args, b->d_ccs, b->d_cfl_work, b->ncfl, b->nstages,
                           b->d_phase_base, (int)b->cases.size(), 0, st);
    CK(cudaGetLastError());
  } else if (cfl == 2) {
    fast::launch_take_folded_batch(b->d_args, b->d_ccs, (int)b->cases.size(), b->nstages, st);
    CK(cudaGetLastError());
  }
  for (int k = 0; k < b->nstages; ++k) {
    fast::launch_stage_batch(b->d_args, b->d_ccs, b->d_work[r], b->nwork[r], k, b->nstages,
                             b->d_phase_base, b->limiter, b->visc, k == b->nstages - 1, b->mixed,
                             b->grid, b->threads, b->table, st);
    CK(cudaGetLastError());
  }
  return IBGPU_OK;
}

// Autotuner: time the first stage of the largest phase's work list at each
// candidate CTA count (one CTA per item, or 1..6 resident CTAs per SM) and
// keep the fastest.  Runs before the run's diag is initialised; it writes
// only the first stage buffer, which stage 0 of every step rewrites.
// Threads per CTA of the merged stage launch by default: 288 for FP64 (a
// ninth warp owns the tile's edge faces), 256 for the mixed build.
int default_threads(const ibgpu_batch *b) { return b->mixed ? kTileCells : kTileCells + 32; }

// The merged stage launch's shape from timed candidates on the busiest
// phase's work list: the CTA count (one CTA per work item, or 1..4 (FP64) /
// 1..6 (mixed) persistent CTAs per SM) and the block (256 or 288 threads),
// each unless the caller fixed it.
int autotune(ibgpu_batch *b) {
  int r = 0;
  for (int i = 1; i < b->period; ++i)
    if (b->nwork[i] > b->nwork[r]) r = i;
  b->tune_grid.clear();
  b->tune_threads.clear();
  b->tune_ms.clear();
  if (b->nwork[r] == 0) {
    b->grid = std::max(b->fixed_grid, 0);
    b->threads = b->fixed_threads ? b->fixed_threads : default_threads(b);
    b->tuned = true;
    return IBGPU_OK;
  }
  std::vector<int> grids, blocks;
  if (b->fixed_grid >= 0) {
    grids.push_back(b->fixed_grid);
  } else {
    grids.push_back(0);
    for (int m = 1; m <= (b->mixed ? 6 : 4); ++m)
      if (m * b->nsm < b->nwork[r]) grids.push_back(m * b->nsm);
  }
  if (b->fixed_threads) blocks.push_back(b->fixed_threads);
  else blocks = {default_threads(b), b->mixed ? kTileCells + 32 : kTileCells};
  if (grids.size() * blocks.size() == 1) {
    b->grid = grids[0];
    b->threads = blocks[0];
    b->tuned = true;
    return IBGPU_OK;
  }
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  float best = 1e30f;
  int best_grid = grids[0], best_threads = blocks[0];
  for (int nt : blocks)
    for (int g : grids) {
      float tbest = 1e30f;
      for (int rep = 0; rep < 3; ++rep) {
        CK(cudaEventRecord(e0, b->stream));
        fast::launch_stage_batch(b->d_args, b->d_ccs, b->d_work[r], b->nwork[r], 0, b->nstages,
                                 b->d_phase_base, b->limiter, b->visc, b->nstages == 1, b->mixed,
                                 g, nt, b->table, b->stream);
        CK(cudaGetLastError());
        CK(cudaEventRecord(e1, b->stream));
        CK(cudaEventSynchronize(e1));
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, e0, e1));
        if (rep > 0 && ms < tbest) tbest = ms;  // the first launch warms up
      }
      b->tune_grid.push_back(g);
      b->tune_threads.push_back(nt);
      b->tune_ms.push_back(tbest);
      if (tbest < best) {
        best = tbest;
        best_grid = g;
        best_threads = nt;
      }
    }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  b->grid = best_grid;
  b->threads = best_threads;
  b->tuned = true;
  return IBGPU_OK;
}

// The batch's stage arguments in the constant-memory table when they fit:
// a header of one int4 per case (byte offsets of the case's StageArgs up to
// its stage-dependent part, of its StageVar records, of its CaseConst), then
// per case those three, the CaseConst cut after its finest level (the stage
// kernel reads only the levels the case's tiles have).  A batch that does
// not fit keeps reading its arguments from global memory.
int write_batch_table(ibgpu_batch *b, const std::vector<StageArgs> &args,
                      const std::vector<CaseConst> &ccs) {
  const int n = (int)b->cases.size(), S = b->nstages;
  auto up16 = [](size_t x) { return (x + 15) & ~(size_t)15; };
  std::vector<size_t> rec(n);
  size_t total = up16((size_t)n * sizeof(int4));
  for (int i = 0; i < n; ++i) {
    rec[i] = total;
    const size_t cc_bytes = offsetof(CaseConst, lev) + b->cases[i]->cs.nlevels * sizeof(LevelConst);
    total += up16(kStageCommonBytes) + up16((size_t)S * sizeof(StageVar)) + up16(cc_bytes);
  }
  if (total > (size_t)INT32_MAX) return IBGPU_OK;
  const int off = fast::batch_table_reserve(b->device, (int)total);
  if (off < 0) return IBGPU_OK;  // does not fit: global-memory arguments
  std::vector<unsigned char> img(total, 0);
  for (int i = 0; i < n; ++i) {
    const size_t a_at = rec[i], v_at = a_at + up16(kStageCommonBytes),
                 c_at = v_at + up16((size_t)S * sizeof(StageVar));
    const int4 h = make_int4(off + (int)a_at, off + (int)v_at, off + (int)c_at, 0);
    std::memcpy(&img[(size_t)i * sizeof(int4)], &h, sizeof(int4));
    std::memcpy(&img[a_at], &args[(size_t)i * S], kStageCommonBytes);
    for (int k = 0; k < S; ++k)
      std::memcpy(&img[v_at + k * sizeof(StageVar)], &args[(size_t)i * S + k].v, sizeof(StageVar));
    std::memcpy(&img[c_at], &ccs[i],
                offsetof(CaseConst, lev) + b->cases[i]->cs.nlevels * sizeof(LevelConst));
  }
  cudaError_t e = fast::batch_table_write(off, img.data(), (int)total);
  if (e != cudaSuccess) {
    fast::batch_table_release(b->device, off);
    return cuda_fail(e, "batch constant table");
  }
  b->table = off;
  b->table_bytes = (int)total;
  return IBGPU_OK;
}

// One graph per schedule phase holding the nstages merged stage launches;
// without a capturable stream the launches are issued directly.
// The graph of one whole batch step at schedule phase q = ts % full_period
// with CFL variant cfl, captured on first use: the cases' ghost fills and
// viscous passes (their abort phase read from the batch's device counter)
// forked onto the batch's branch streams, joined, then the merged CFL and
// stage launches.  Nothing in it depends on the step index except through
// the device counter, so one capture serves every step of that phase.
int batch_step_graph(ibgpu_batch *b, int q, int cfl, cudaGraphExec_t *out) {
  const int key = q * 3 + cfl;
  auto it = b->graphs.find(key);
  if (it != b->graphs.end()) {
    *out = it->second;
    return IBGPU_OK;
  }
  cudaStream_t st = b->stream;
  const int nf = (int)b->fork.size();
  cudaGraph_t g = nullptr;
  CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  int rc = IBGPU_OK;
  cudaError_t e = cudaEventRecord(b->ev_fork_join[nf], st);
  for (int k = 0; k < nf && e == cudaSuccess; ++k) e = cudaStreamWaitEvent(b->fork[k], b->ev_fork_join[nf], 0);
  for (size_t i = 0; i < b->cases.size() && e == cudaSuccess && !rc; ++i) {
    RunTimer tm{b->cases[i], b->fork[i % nf], {}, {}};
    tm.off = true;
    rc = enqueue_prestage(b->cases[i], q, 1, b->fork[i % nf], tm, true, false, b->d_phase_base);
  }
  for (int k = 0; k < nf && e == cudaSuccess && !rc; ++k) {
    e = cudaEventRecord(b->ev_fork_join[k], b->fork[k]);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(st, b->ev_fork_join[k], 0);
  }
  if (e == cudaSuccess && !rc) rc = enqueue_batch_stages(b, q % b->period, cfl, st);
  cudaError_t e2 = cudaStreamEndCapture(st, &g);
  if (rc) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess) return cuda_fail(e, "batch step capture");
  if (e2 != cudaSuccess) return cuda_fail(e2, "cudaStreamEndCapture");
  cudaGraphExec_t x = nullptr;
  e = cudaGraphInstantiate(&x, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate");
  b->graphs[key] = x;
  *out = x;
  return IBGPU_OK;
}

// Capture the graphs of every schedule phase up front (the first run after
// tuning), so that later runs replay them without capturing.
int batch_prepare_graphs(ibgpu_batch *b) {
  if (b->graphs_ready) return IBGPU_OK;
  for (int q = 0; q < b->full_period; ++q) {
    const bool cfl_now = b->mixed_cfl ? b->ncfl_cases_r[q % b->period] > 0 : (q % b->dt_var_step) == 0;
    cudaGraphExec_t gx = nullptr;
    int rc = batch_step_graph(b, q, cfl_now ? 1 : 0, &gx);
    if (!rc && cfl_now && b->folds) rc = batch_step_graph(b, q, 2, &gx);
    if (rc) return rc;
  }
  b->graphs_ready = true;
  return IBGPU_OK;
}

}  // namespace

int ibgpu_batch_create(ibgpu_ctx *const *cases, int ncases, ibgpu_batch **out) {
  if (!cases || ncases < 1 || !out) return IBGPU_E_ARG;
  *out = nullptr;
  const ibgpu_case &c0 = cases[0]->cs;
  if (c0.precision == IBGPU_FP64_EXACT) {
    g_last_error = "batched cases run the FP64 or mixed builds";
    return IBGPU_E_ARG;
  }
  for (int i = 0; i < ncases; ++i) {
    const ibgpu_ctx *c = cases[i];
    if (!c) return IBGPU_E_ARG;
    if (!c->has_state) return IBGPU_E_STATE;
    const ibgpu_case &cs = c->cs;
    bool same = cs.precision == c0.precision && cs.limiter == c0.limiter &&
                (cs.viscous != 0) == (c0.viscous != 0) && cs.nstages == c0.nstages &&
                c->device == cases[0]->device;
    for (int k = 0; same && k < cs.nstages; ++k) same = cs.tp[k] == c0.tp[k];
    if (!same) {
      g_last_error = "batched cases differ in precision, limiter, viscosity, stages or device";
      return IBGPU_E_ARG;
    }
  }
  ibgpu_batch *b = new (std::nothrow) ibgpu_batch;
  if (!b) return IBGPU_E_NOMEM;
  b->cases.assign(cases, cases + ncases);
  b->stream = cases[0]->stream;
  b->nsm = cases[0]->nsm;
  b->device = cases[0]->device;
  b->nstages = c0.nstages;
  b->limiter = c0.limiter;
  b->visc = c0.viscous != 0;
  b->mixed = c0.precision == IBGPU_MIXED;
  b->dt_var_step = c0.dt_var_step;
  b->folds = true;
  // schedule period: every level's marching step divides the largest
  for (auto *c : b->cases)
    for (int l = 0; l < c->cs.nlevels; ++l) b->period = std::max(b->period, c->cs.march_step[l]);
  for (auto *c : b->cases)
    for (int l = 0; l < c->cs.nlevels; ++l)
      if (b->period % c->cs.march_step[l] != 0) {
        delete b;
        g_last_error = "marching steps of the batched cases have no common period";
        return IBGPU_E_ARG;
      }
  // every schedule (marching, restriction, prolongation, CFL) repeats with
  // the least common multiple of its steps
  {
    auto lcm = [](int a, int c) { return a / std::gcd(a, c) * c; };
    int fp = b->period;
    for (auto *c : b->cases) {
      fp = lcm(fp, c->cs.dt_var_step);
      for (int l = 0; l < c->cs.nlevels; ++l) {
        fp = lcm(fp, c->cs.march_step[l]);
        if (l >= 1) fp = lcm(lcm(fp, c->cs.average_step[l]), c->cs.prolong_step[l]);
      }
      if (fp > 4096) break;
    }
    b->full_period = fp;
  }
  // CFL intervals: all equal, or each dividing the schedule period (then the
  // cases whose pass runs depend only on ts % period)
  for (auto *c : b->cases) b->mixed_cfl = b->mixed_cfl || c->cs.dt_var_step != c0.dt_var_step;
  if (b->mixed_cfl)
    for (auto *c : b->cases)
      if (b->period % c->cs.dt_var_step != 0) {
        delete b;
        g_last_error = "batched cases with different dt_var_step need each to divide the "
                       "schedule period";
        return IBGPU_E_ARG;
      }
  const int S = b->nstages;
  std::vector<StageArgs> args((size_t)ncases * S);
  std::vector<CaseConst> ccs(ncases);
  for (int i = 0; i < ncases; ++i) {
    for (int k = 0; k < S; ++k) stage_args(b->cases[i], k, args[(size_t)i * S + k]);
    ccs[i] = b->cases[i]->cc;
    b->folds = b->folds && folds_cfl(b->cases[i]);
  }
  if (b->folds)
    for (int i = 0; i < ncases; ++i) args[(size_t)i * S + S - 1].v.cfl_next = 1;  // enabled marker
  auto fail = [&](int rc) {
    b->release();
    delete b;
    return rc;
  };
  int rc;
  if ((rc = dev_alloc(&b->d_args, args.size())) || (rc = dev_alloc(&b->d_ccs, ccs.size())) ||
      (rc = dev_alloc(&b->d_phase_base, 2)))
    return fail(rc);
  cudaError_t e = cudaMemcpy(b->d_args, args.data(), args.size() * sizeof(StageArgs), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(b->d_ccs, ccs.data(), ccs.size() * sizeof(CaseConst), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(b->d_phase_base, 0, 2 * sizeof(int));
  if (e != cudaSuccess) return fail(cuda_fail(e, "batch upload"));
  if ((rc = write_batch_table(b, args, ccs))) return fail(rc);
  // work lists: case-interleaved so the persistent CTAs mix the cases
  b->d_work.assign(b->period, nullptr);
  b->nwork.assign(b->period, 0);
  for (int r = 0; r < b->period; ++r) {
    std::vector<std::vector<int2>> per(ncases);
    size_t total = 0;
    for (int i = 0; i < ncases; ++i) {
      const ibgpu_ctx *c = b->cases[i];
      for (int l = 0; l < c->cs.nlevels; ++l) {
        if (r % c->cs.march_step[l] != c->cs.march_left[l]) continue;
        for (int t = 0; t < c->level_tile_count[l]; ++t)
          per[i].push_back(make_int2(i, c->level_tile_begin[l] + t));
      }
      total += per[i].size();
    }
    std::vector<int2> w;
    w.reserve(total);
    std::vector<double> pos(ncases, 0.0);
    // proportional interleave: case i's j-th item at key (j + 0.5) / n_i
    std::vector<std::pair<double, int2>> keyed;
    keyed.reserve(total);
    for (int i = 0; i < ncases; ++i)
      for (size_t j = 0; j < per[i].size(); ++j)
        keyed.push_back({(j + 0.5) / (double)per[i].size(), per[i][j]});
    std::stable_sort(keyed.begin(), keyed.end(),
                     [](const std::pair<double, int2> &a, const std::pair<double, int2> &b2) {
                       return a.first < b2.first;
                     });
    for (auto &kv : keyed) w.push_back(kv.second);
    if (w.size() > (size_t)INT32_MAX) return fail(IBGPU_E_ARG);
    b->nwork[r] = (int)w.size();
    if ((rc = dev_alloc(&b->d_work[r], w.size()))) return fail(rc);
    e = cudaMemcpy(b->d_work[r], w.data(), w.size() * sizeof(int2), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return fail(cuda_fail(e, "batch work list"));
  }
  {
    std::vector<int2> w;
    for (int i = 0; i < ncases; ++i)
      for (int t = 0; t < (int)b->cases[i]->ntiles; ++t) w.push_back(make_int2(i, t));
    b->ncfl = (int)w.size();
    if ((rc = dev_alloc(&b->d_cfl_work, w.size()))) return fail(rc);
    e = cudaMemcpy(b->d_cfl_work, w.data(), w.size() * sizeof(int2), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return fail(cuda_fail(e, "batch CFL work list"));
  }
  if (b->mixed_cfl) {
    b->d_cfl_work_r.assign(b->period, nullptr);
    b->d_cfl_cases_r.assign(b->period, nullptr);
    b->ncfl_r.assign(b->period, 0);
    b->ncfl_cases_r.assign(b->period, 0);
    for (int r = 0; r < b->period; ++r) {
      std::vector<int2> w;
      std::vector<int> cl;
      for (int i = 0; i < ncases; ++i) {
        if (r % b->cases[i]->cs.dt_var_step != 0) continue;
        cl.push_back(i);
        for (int t = 0; t < (int)b->cases[i]->ntiles; ++t) w.push_back(make_int2(i, t));
      }
      b->ncfl_r[r] = (int)w.size();
      b->ncfl_cases_r[r] = (int)cl.size();
      if (cl.empty()) continue;
      if ((rc = dev_alloc(&b->d_cfl_work_r[r], w.size())) ||
          (rc = dev_alloc(&b->d_cfl_cases_r[r], cl.size())))
        return fail(rc);
      e = cudaMemcpy(b->d_cfl_work_r[r], w.data(), w.size() * sizeof(int2), cudaMemcpyHostToDevice);
      if (e == cudaSuccess)
        e = cudaMemcpy(b->d_cfl_cases_r[r], cl.data(), cl.size() * sizeof(int), cudaMemcpyHostToDevice);
      if (e != cudaSuccess) return fail(cuda_fail(e, "batch CFL work list"));
    }
  }
  // branch streams of the captured steps: up to eight, cases round robin
  {
    const int nf = std::min(8, ncases);
    b->fork.assign(nf, nullptr);
    b->ev_fork_join.assign(nf + 1, nullptr);
    for (int k = 0; k < nf; ++k)
      if ((e = cudaStreamCreateWithFlags(&b->fork[k], cudaStreamNonBlocking)) != cudaSuccess)
        return fail(cuda_fail(e, "batch branch stream"));
    for (auto &ev : b->ev_fork_join)
      if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess)
        return fail(cuda_fail(e, "batch branch event"));
  }
  *out = b;
  return IBGPU_OK;
}

int ibgpu_batch_run(ibgpu_batch *b, int ts0, int nsteps, double *dt, ibgpu_diag *diag) {
  if (!b || !dt || ts0 < 0 || nsteps < 1) return IBGPU_E_ARG;
  const int n = (int)b->cases.size();
  cudaStream_t st = b->stream;
  int rc;
  if (!b->tuned) {
    if ((rc = autotune(b))) return rc;
    b->drop_graphs();  // captured with the previous launch shape
  }
  // captured whole steps, unless something asks for per-launch timing or the
  // batch runs on the legacy stream (not capturable); captured before this
  // run's first work is enqueued
  bool use_graphs = b->stream != nullptr && !b->timing && b->full_period <= 4096;
  for (int i = 0; i < n; ++i) use_graphs = use_graphs && !b->cases[i]->timing;
  if (use_graphs && (rc = batch_prepare_graphs(b))) return rc;
  for (int i = 0; i < n; ++i) {
    if (b->cases[i]->download_pending) {
      CK(cudaStreamWaitEvent(st, b->cases[i]->ev_copied, 0));
      b->cases[i]->download_pending = false;
    }
    if ((rc = begin_diag(b->cases[i], dt[i], st))) return rc;
  }
  std::vector<RunTimer> tms;
  for (int i = 0; i < n; ++i) tms.push_back(RunTimer{b->cases[i], st, {}, {}});

  cudaEvent_t e0 = nullptr, e1 = nullptr;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> sev;
  std::vector<int64_t> marched(n, 0);
  for (int step = 0; step < nsteps; ++step) {
    const int ts = ts0 + step;
    const int r = ts % b->period;
    if (step > 0) fast::launch_step_begin_batch(b->d_args, n, b->nstages, st);
    for (int i = 0; i < n; ++i) marched[i] = marched_cells(b->cases[i], ts);
    const bool cfl_now = b->mixed_cfl ? b->ncfl_cases_r[r] > 0 : (ts % b->dt_var_step) == 0;
    const int cfl = !cfl_now ? 0 : (b->folds && step > 0 ? 2 : 1);
    fast::launch_set_phase_base(b->d_phase_base, 8 * step, b->folds && step + 1 < nsteps, st);
    if (use_graphs) {
      // the whole step as one graph (the stage launches' own timing is not
      // separable then: b->timing runs without graphs)
      cudaGraphExec_t gx = nullptr;
      if ((rc = batch_step_graph(b, ts % b->full_period, cfl, &gx))) return rc;
      CK(cudaGraphLaunch(gx, st));
    } else {
      for (int i = 0; i < n; ++i)
        if ((rc = enqueue_prestage(b->cases[i], ts, step, st, tms[i], true))) return rc;
      if (b->timing) {
        CK(cudaEventCreate(&e0));
        CK(cudaEventCreate(&e1));
        CK(cudaEventRecord(e0, st));
      }
      if ((rc = enqueue_batch_stages(b, r, cfl, st))) return rc;
      if (b->timing) {
        CK(cudaEventRecord(e1, st));
        sev.push_back({e0, e1});
      }
    }
  }
  for (int i = 0; i < n; ++i)
    CK(cudaMemcpyAsync(b->cases[i]->h_diag, b->cases[i]->d_diag, sizeof(DevDiag),
                       cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  for (auto &p : sev) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, p.first, p.second);
    b->stage_ms += ms;
    b->stage_launches += b->nstages;
    cudaEventDestroy(p.first);
    cudaEventDestroy(p.second);
  }
  int result = IBGPU_OK;
  for (int i = 0; i < n; ++i) {
    tms[i].collect();
    int ri = decode_diag(b->cases[i], marched[i], &dt[i], diag ? &diag[i] : nullptr);
    if (ri != IBGPU_OK && result == IBGPU_OK) result = ri;
  }
  return result;
}

int ibgpu_batch_tag_mesh(ibgpu_batch *b, const ibgpu_tag_rule *rule, const float *d_params,
                         uint8_t *tags) {
  if (!b || !rule || !tags) return IBGPU_E_ARG;
  cudaStream_t st = b->stream;
  int rc = tag_mesh_prepare(d_params != nullptr);
  if (rc) return rc;
  // each case tags on its own stream after the batch's pending work (the
  // cases' kernels overlap, so one case's last partial wave does not idle the
  // GPU), its rows copied back behind its kernels; the batch stream then
  // waits for all of them and reads every time-out flag in one
  // synchronisation
  const size_t n = b->cases.size();
  if (b->ev_tag.size() != n + 1) {
    for (auto e : b->ev_tag) cudaEventDestroy(e);
    b->ev_tag.assign(n + 1, nullptr);
    for (auto &e : b->ev_tag) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  CK(cudaEventRecord(b->ev_tag[n], st));
  int64_t off = 0;
  for (size_t i = 0; i < n; ++i) {
    ibgpu_ctx *c = b->cases[i];
    if (c->ncells == 0) continue;
    cudaStream_t cst = c->stream;
    CK(cudaStreamWaitEvent(cst, b->ev_tag[n], 0));
    uint8_t *rows = nullptr;
    if ((rc = tag_mesh_enqueue(c, rule, d_params, cst, &rows))) return rc;
    CK(cudaMemcpyAsync(tags + off, rows, (size_t)c->ncells, cudaMemcpyDeviceToHost, cst));
    CK(cudaEventRecord(b->ev_tag[i], cst));
    CK(cudaStreamWaitEvent(st, b->ev_tag[i], 0));
    off += c->ncells;
  }
  if (d_params) {
    if (!b->h_err) CK(cudaHostAlloc((void **)&b->h_err, n * sizeof(int), cudaHostAllocDefault));
    for (size_t i = 0; i < n; ++i)
      CK(cudaMemcpyAsync(b->h_err + i, b->cases[i]->d_aux_err, sizeof(int), cudaMemcpyDeviceToHost, st));
  }
  CK(cudaStreamSynchronize(st));
  if (d_params) {
    bool timed_out = false;
    for (size_t i = 0; i < n; ++i)
      if (b->h_err[i]) {
        timed_out = true;
        CK(cudaMemsetAsync(b->cases[i]->d_aux_err, 0, sizeof(int), st));
      }
    if (timed_out) {
      CK(cudaStreamSynchronize(st));
      g_last_error = "tensor-core wait ran out of its time limit";
      return IBGPU_E_TIMEOUT;
    }
  }
  return IBGPU_OK;
}

int ibgpu_batch_set_grid(ibgpu_batch *b, int grid) {
  if (!b || grid < -1) return IBGPU_E_ARG;
  if (b->stream) CK(cudaStreamSynchronize(b->stream));  // captured graphs may be in flight
  b->drop_graphs();
  b->fixed_grid = grid;
  b->tuned = false;  // the next run tunes (grid -1) or takes the count, and recaptures
  return IBGPU_OK;
}

int ibgpu_batch_set_block(ibgpu_batch *b, int threads) {
  if (!b || (threads != 0 && threads != kTileCells && threads != kTileCells + 32))
    return IBGPU_E_ARG;
  if (b->stream) CK(cudaStreamSynchronize(b->stream));  // captured graphs may be in flight
  b->drop_graphs();
  b->fixed_threads = threads;
  b->tuned = false;
  return IBGPU_OK;
}

int ibgpu_batch_set_timing(ibgpu_batch *b, int enable) {
  if (!b) return IBGPU_E_ARG;
  b->timing = enable != 0;
  b->stage_ms = 0.0;
  b->stage_launches = 0;
  return IBGPU_OK;
}

int ibgpu_batch_info(const ibgpu_batch *b, int *grid, int *threads, int *period,
                     double *stage_ms, int64_t *stage_launches) {
  if (!b) return IBGPU_E_ARG;
  if (grid) *grid = b->grid;
  if (threads) *threads = b->threads;
  if (period) *period = b->period;
  if (stage_ms) *stage_ms = b->stage_ms;
  if (stage_launches) *stage_launches = b->stage_launches;
  return IBGPU_OK;
}

int ibgpu_batch_tuning(const ibgpu_batch *b, int max, int *grids, int *threads, float *ms) {
  if (!b || max < 0) return IBGPU_E_ARG;
  const int n = std::min<int>(max, (int)b->tune_grid.size());
  for (int i = 0; i < n; ++i) {
    if (grids) grids[i] = b->tune_grid[i];
    if (threads) threads[i] = b->tune_threads[i];
    if (ms) ms[i] = b->tune_ms[i];
  }
  return (int)b->tune_grid.size();
}

int ibgpu_batch_table_bytes(const ibgpu_batch *b) { return b ? b->table_bytes : 0; }

void ibgpu_batch_destroy(ibgpu_batch *b) {
  if (!b) return;
  if (b->stream) cudaStreamSynchronize(b->stream);
  b->release();
  delete b;
}

}  // extern "C"

namespace {

template <typename T>
int upload_vec(T **dst, const std::vector<T> &v, cudaStream_t st) {
  int rc = dev_alloc(dst, v.size());
  if (rc) return rc;
  if (!v.empty()) CK(cudaMemcpyAsync(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st));
  return IBGPU_OK;
}


}  // namespace

extern "C" {

int ibgpu_upload_interfaces(ibgpu_ctx *ctx, const ibgpu_cf_pairs *pp) {
  if (!ctx || !pp || pp->nres < 0 || pp->npro < 0 || (pp->nres && !pp->res) || (pp->npro && !pp->pro))
    return IBGPU_E_ARG;
  if (!ctx->has_topology) return IBGPU_E_STATE;
  const int nlev = ctx->cs.nlevels;
  cudaStream_t st = ctx->stream;
  CK(cudaStreamSynchronize(st));
  for (auto *v : {&ctx->res, &ctx->pro})
    for (auto &p : *v) {
      cudaFree(p.coarse);
      cudaFree(p.fine);
      cudaFree(p.nb);
    }
  ctx->res.assign(nlev, {});
  ctx->pro.assign(nlev, {});
  // restriction: per coarse level, in list order
  std::vector<std::vector<int32_t>> rc_(nlev), rf(nlev);
  for (int64_t i = 0; i < pp->nres; ++i) {
    const int32_t *r = pp->res + 11 * i;
    int l = r[0];
    if (l < 0 || l + 1 >= nlev) { g_last_error = "restriction pair level out of range"; return IBGPU_E_ARG; }
    int64_t c = ctx->slot_at(l, r[1], r[2]);
    if (c < 0) { g_last_error = "restriction coarse cell absent"; return IBGPU_E_TOPOLOGY; }
    rc_[l].push_back((int32_t)c);
    for (int k = 0; k < 4; ++k) {
      int64_t f = ctx->slot_at(l + 1, r[3 + 2 * k], r[4 + 2 * k]);
      if (f < 0) { g_last_error = "restriction son absent"; return IBGPU_E_TOPOLOGY; }
      rf[l].push_back((int32_t)f);
    }
  }
  // prolongation: duplicates of a coarse cell write identical sons; keep one
  std::vector<std::vector<int32_t>> pc(nlev), pf(nlev), pn(nlev);
  std::vector<std::unordered_map<int64_t, int64_t>> fine_owner(nlev);
  std::vector<std::unordered_map<int64_t, int>> seen(nlev);
  for (int64_t i = 0; i < pp->npro; ++i) {
    const int32_t *r = pp->pro + 11 * i;
    int l = r[0];
    if (l < 0 || l + 1 >= nlev) { g_last_error = "prolongation pair level out of range"; return IBGPU_E_ARG; }
    int64_t c = ctx->slot_at(l, r[1], r[2]);
    if (c < 0) { g_last_error = "prolongation coarse cell absent"; return IBGPU_E_TOPOLOGY; }
    int64_t sons[4];
    for (int k = 0; k < 4; ++k) {
      sons[k] = ctx->slot_at(l + 1, r[3 + 2 * k], r[4 + 2 * k]);
      if (sons[k] < 0) { g_last_error = "prolongation son absent"; return IBGPU_E_TOPOLOGY; }
      auto it = fine_owner[l].find(sons[k]);
      if (it != fine_owner[l].end() && it->second != c) {
        g_last_error = "fine ghost claimed by two coarse cells";
        return IBGPU_E_TOPOLOGY;
      }
      fine_owner[l][sons[k]] = c;
    }
    if (seen[l].count(c)) continue;
    seen[l][c] = 1;
    const int off[4][2] = {{-1, 0}, {1, 0}, {0, -1}, {0, 1}};
    for (int k = 0; k < 4; ++k) {
      int64_t nb = ctx->slot_at(l, r[1] + off[k][0], r[2] + off[k][1]);
      if (nb < 0) { g_last_error = "prolongation stencil cell absent"; return IBGPU_E_TOPOLOGY; }
      pn[l].push_back((int32_t)nb);
    }
    pc[l].push_back((int32_t)c);
    for (int k = 0; k < 4; ++k) pf[l].push_back((int32_t)sons[k]);
  }
  int e;
  for (int l = 0; l < nlev; ++l) {
    if ((e = upload_vec(&ctx->res[l].coarse, rc_[l], st)) || (e = upload_vec(&ctx->res[l].fine, rf[l], st)) ||
        (e = upload_vec(&ctx->pro[l].coarse, pc[l], st)) || (e = upload_vec(&ctx->pro[l].fine, pf[l], st)) ||
        (e = upload_vec(&ctx->pro[l].nb, pn[l], st)))
      return e;
    ctx->res[l].n = (int)rc_[l].size();
    ctx->pro[l].n = (int)pc[l].size();
  }
  CK(cudaStreamSynchronize(st));
  return IBGPU_OK;
}

int ibgpu_upload_boundaries(ibgpu_ctx *ctx, const ibgpu_bc *bc) {
  if (!ctx || !bc || bc->n < 0 || (bc->n && !bc->ghost) || bc->nfaces < 0 || (bc->nfaces && !bc->facevar))
    return IBGPU_E_ARG;
  if (!ctx->has_topology) return IBGPU_E_STATE;
  const int nlev = ctx->cs.nlevels;
  cudaStream_t st = ctx->stream;
  CK(cudaStreamSynchronize(st));
  for (int32_t **p : {&ctx->d_bc_ghost, &ctx->d_bc_ref, &ctx->d_bc_type, &ctx->d_bc_face}) {
    cudaFree(*p);
    *p = nullptr;
  }
  for (double **p : {&ctx->d_bc_nmv, &ctx->d_facevar}) {
    cudaFree(*p);
    *p = nullptr;
  }
  // entries per level in list order (periodic faces need no work)
  struct Ent { int64_t g, r; int type, face; double n[3]; int wave; };
  std::vector<std::vector<Ent>> per(nlev);
  for (int64_t i = 0; i < bc->n; ++i) {
    const int32_t *g = bc->ghost + 7 * i;
    int l = g[0], type = g[6], face = g[5];
    if (l < 0 || l >= nlev) { g_last_error = "boundary ghost level out of range"; return IBGPU_E_ARG; }
    if (type == -99 || type == -125) continue;
    if (type != -50 && type != -12 && type != -13 && type != -49 && type != -46 && type != -42 &&
        type != -51 && type != -10 && type != -45) {
      g_last_error = "unknown boundary type";
      return IBGPU_E_ARG;
    }
    if (face < 0 || face >= bc->nfaces) { g_last_error = "boundary face out of range"; return IBGPU_E_ARG; }
    if (type == -51 && !bc->nmv) { g_last_error = "slip wall without normals"; return IBGPU_E_ARG; }
    Ent en;
    en.g = ctx->slot_at(l, g[1], g[2]);
    en.r = ctx->slot_at(l, g[3], g[4]);
    if (en.g < 0 || en.r < 0) { g_last_error = "boundary ghost or reference cell absent"; return IBGPU_E_TOPOLOGY; }
    en.type = type;
    en.face = face;
    for (int k = 0; k < 3; ++k) en.n[k] = bc->nmv ? bc->nmv[3 * i + k] : 0.0;
    per[l].push_back(en);
  }
  // dependency waves: a ghost whose reference is written earlier in the list
  // runs after that write; one written later must read it before the write;
  // a cell written twice keeps the later value (BCBoxTreat is sequential)
  ctx->bc_waves.assign(nlev, {});
  std::vector<int32_t> hg, hr, ht, hf;
  std::vector<double> hn;
  for (int l = 0; l < nlev; ++l) {
    auto &E = per[l];
    std::unordered_map<int64_t, int> last_writer, max_reader_wave;
    for (size_t i = 0; i < E.size(); ++i) {
      int w = 0;
      auto it = last_writer.find(E[i].r);
      if (it != last_writer.end()) w = std::max(w, E[it->second].wave + 1);
      auto rd = max_reader_wave.find(E[i].g);
      if (rd != max_reader_wave.end()) w = std::max(w, rd->second + 1);
      auto pw = last_writer.find(E[i].g);
      if (pw != last_writer.end()) w = std::max(w, E[pw->second].wave + 1);
      E[i].wave = w;
      last_writer[E[i].g] = (int)i;
      int &mr = max_reader_wave[E[i].r];
      mr = std::max(mr, w);
    }
    std::stable_sort(E.begin(), E.end(), [](const Ent &x, const Ent &y) { return x.wave < y.wave; });
    size_t i = 0;
    while (i < E.size()) {
      size_t j = i;
      while (j < E.size() && E[j].wave == E[i].wave) ++j;
      ctx->bc_waves[l].push_back({(int)(hg.size() + i), (int)(hg.size() + j)});
      i = j;
    }
    for (auto &en : E) {
      hg.push_back((int32_t)en.g);
      hr.push_back((int32_t)en.r);
      ht.push_back(en.type);
      hf.push_back(en.face);
      hn.insert(hn.end(), en.n, en.n + 3);
    }
  }
  std::vector<double> fv(bc->facevar, bc->facevar + 7 * (size_t)bc->nfaces);
  int e;
  if ((e = upload_vec(&ctx->d_bc_ghost, hg, st)) || (e = upload_vec(&ctx->d_bc_ref, hr, st)) ||
      (e = upload_vec(&ctx->d_bc_type, ht, st)) || (e = upload_vec(&ctx->d_bc_face, hf, st)) ||
      (e = upload_vec(&ctx->d_bc_nmv, hn, st)) || (e = upload_vec(&ctx->d_facevar, fv, st)))
    return e;
  ctx->backpressure = bc->backpressure;
  ctx->cos_in = std::cos(bc->inlet_flow_angle);
  ctx->sin_in = std::sin(bc->inlet_flow_angle);
  CK(cudaStreamSynchronize(st));
  return IBGPU_OK;
}

int ibgpu_upload_ib(ibgpu_ctx *ctx, const ibgpu_ib *ib) {
  if (!ctx || !ib || ib->ncells < 0 || ib->npatches < 0 || ib->nbodies < 0 ||
      (ib->ncells && (!ib->cell || !ib->cellf)) || (ib->npatches && (!ib->patch || !ib->patchf)) ||
      (ib->nbodies && !ib->body_center))
    return IBGPU_E_ARG;
  if (!ctx->has_topology) return IBGPU_E_STATE;
  const int bl = ctx->body_level;
  if ((ib->ncells || ib->npatches) && (bl < 0 || bl >= ctx->cs.nlevels)) {
    g_last_error = "immersed-boundary records without a body level";
    return IBGPU_E_ARG;
  }
  cudaStream_t st = ctx->stream;
  std::vector<int32_t> cell, intp, pbody, pintp, begin(ib->nbodies + 1, 0);
  for (int64_t i = 0; i < ib->ncells; ++i) {
    const int32_t *c = ib->cell + 18 * i;
    int64_t s = ctx->slot_at(bl, c[0], c[1]);
    if (s < 0) { g_last_error = "IB cell absent"; return IBGPU_E_TOPOLOGY; }
    cell.push_back((int32_t)s);
    for (int k = 0; k < 8; ++k) {
      int64_t t = ctx->slot_at(bl, c[2 + 2 * k], c[3 + 2 * k]);
      if (t < 0) { g_last_error = "IB interpolation cell absent"; return IBGPU_E_TOPOLOGY; }
      intp.push_back((int32_t)t);
    }
  }
  int prev = 0;
  for (int64_t i = 0; i < ib->npatches; ++i) {
    const int32_t *p = ib->patch + 17 * i;
    if (p[0] < prev || p[0] >= ib->nbodies) { g_last_error = "patches must be grouped by body"; return IBGPU_E_ARG; }
    prev = p[0];
    pbody.push_back(p[0]);
    begin[p[0] + 1]++;
    for (int k = 0; k < 8; ++k) {
      int64_t t = ctx->slot_at(bl, p[1 + 2 * k], p[2 + 2 * k]);
      if (t < 0) { g_last_error = "patch interpolation cell absent"; return IBGPU_E_TOPOLOGY; }
      pintp.push_back((int32_t)t);
    }
  }
  for (int b = 0; b < ib->nbodies; ++b) begin[b + 1] += begin[b];
  std::vector<double> cf(ib->cellf, ib->cellf + 16 * (size_t)ib->ncells);
  std::vector<double> pf(ib->patchf, ib->patchf + 19 * (size_t)ib->npatches);
  std::vector<double> bc(ib->body_center, ib->body_center + 3 * (size_t)ib->nbodies);
  // the buffers stay between moves (the copies queue behind the last step's
  // kernels on the same stream); when one has to grow, the work that may
  // still read it finishes first
  const size_t nf = 6 * (size_t)std::max(ib->nbodies, 1);
  const std::pair<const void *, size_t> need[] = {
      {&ctx->d_ib_cell, cell.size()},       {&ctx->d_ib_intp, intp.size()},
      {&ctx->d_ib_f, cf.size()},            {&ctx->d_ib_out, 6 * cell.size()},
      {&ctx->d_pat_body, pbody.size()},     {&ctx->d_pat_intp, pintp.size()},
      {&ctx->d_pat_f, pf.size()},           {&ctx->d_pat_out, 12 * pbody.size()},
      {&ctx->d_body_center, bc.size()},     {&ctx->d_body_begin, begin.size()},
      {&ctx->d_force, nf}};
  bool grows = false;
  for (const auto &q : need) grows = grows || q.second > ctx->cap[q.first];
  if (grows) CK(cudaStreamSynchronize(st));
  int e;
  if ((e = keep_upload(ctx, &ctx->d_ib_cell, cell, st)) || (e = keep_upload(ctx, &ctx->d_ib_intp, intp, st)) ||
      (e = keep_upload(ctx, &ctx->d_ib_f, cf, st)) || (e = keep_alloc(ctx, &ctx->d_ib_out, 6 * cell.size())) ||
      (e = keep_upload(ctx, &ctx->d_pat_body, pbody, st)) || (e = keep_upload(ctx, &ctx->d_pat_intp, pintp, st)) ||
      (e = keep_upload(ctx, &ctx->d_pat_f, pf, st)) || (e = keep_alloc(ctx, &ctx->d_pat_out, 12 * pbody.size())) ||
      (e = keep_upload(ctx, &ctx->d_body_center, bc, st)) || (e = keep_upload(ctx, &ctx->d_body_begin, begin, st)) ||
      (e = keep_alloc(ctx, &ctx->d_force, nf)))
    return e;
  ctx->n_ib = (int)cell.size();
  ctx->n_pat = (int)pbody.size();
  ctx->nbodies = ib->nbodies;
  CK(cudaStreamSynchronize(st));
  return IBGPU_OK;
}

int ibgpu_wall_forces(ibgpu_ctx *ctx, double *out) {
  if (!ctx || (!out && ctx->nbodies > 0)) return IBGPU_E_ARG;
  if (!ctx->has_state) return IBGPU_E_STATE;
  if (ctx->nbodies == 0) return IBGPU_OK;
  cudaStream_t st = ctx->stream;
  ForceArgs fa;
  fa.body = ctx->d_pat_body;
  fa.intp = ctx->d_pat_intp;
  fa.patchf = ctx->d_pat_f;
  fa.body_center = ctx->d_body_center;
  fa.body_begin = ctx->d_body_begin;
  fa.n = ctx->n_pat;
  fa.nbodies = ctx->nbodies;
  fa.out = ctx->d_pat_out;
  fa.result = ctx->d_force;
  for (int f = 0; f < kStateFields; ++f) fa.s0[f] = ctx->d_s0[f];
  fast::launch_forces(fa, ctx->cc, st);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out, ctx->d_force, 6 * sizeof(double) * ctx->nbodies, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return IBGPU_OK;
}

}  // extern "C"

extern "C" {

void ibgpu_destroy(ibgpu_ctx *ctx) {
  if (!ctx) return;
  // pending uploads, steps and downloads finish before their buffers go
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->in_stream) cudaStreamSynchronize(ctx->in_stream);
  if (ctx->copy_stream) cudaStreamSynchronize(ctx->copy_stream);
  ctx->free_layout();
  ibgpu::wall_free(ctx->wall);
  cudaFree(ctx->d_diag);
  cudaFree(ctx->d_aux_err);
  cudaFreeHost(ctx->h_diag);
  if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
  if (ctx->in_stream) cudaStreamDestroy(ctx->in_stream);
  if (ctx->ev_in_free) cudaEventDestroy(ctx->ev_in_free);
  if (ctx->ev_in_done) cudaEventDestroy(ctx->ev_in_done);
  if (ctx->ev_ready) cudaEventDestroy(ctx->ev_ready);
  if (ctx->ev_copied) cudaEventDestroy(ctx->ev_copied);
  if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
  delete ctx;
}

}  // extern "C"
