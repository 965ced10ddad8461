// Host side of the ibgpu C ABI: context, tiled layout builder, state
// transfer and the per-step launch sequence.  Mirrors the call order of the
// reference main loop and NS_Solver::TimeMarching (main.cpp:84-116,
// NS_Solver.H:657-702).
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/ibgpu.h"
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
  ibgpu_case cs;
  CaseConst cc;
  int device = 0;
  int nsm = 148;
  int body_level = -1;  // finest level of a run with immersed bodies
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;

  // layout
  bool has_topology = false, has_state = false;
  int64_t ncells = 0;       // rows of the caller's cell list
  int64_t ntiles = 0, nslots = 0;
  std::vector<int> level_tile_begin, level_tile_count;  // per level
  std::vector<int64_t> level_normal_cells;
  std::vector<int32_t> h_slot_level, h_slot_ix, h_slot_iy;  // slot -> position (abort reports)
  int32_t *d_tile_nb = nullptr, *d_tile_level = nullptr, *d_cell_slot = nullptr;
  uint8_t *d_flags = nullptr, *d_cell_alias = nullptr;

  // state: step state (6 fields) + two stage buffers (4 fields each)
  double *d_s0[kStateFields] = {};
  double *d_buf[2][4] = {};
  double *d_vsd = nullptr;
  double *d_rows = nullptr;  // staging for AoS state transfers
  DevDiag *d_diag = nullptr;
  DevDiag *h_diag = nullptr;  // pinned

  // kernel timing
  bool timing = false;
  double kms[3] = {0, 0, 0};
  int64_t klaunch[3] = {0, 0, 0};

  void free_layout() {
    cudaFree(d_tile_nb);
    cudaFree(d_tile_level);
    cudaFree(d_cell_slot);
    cudaFree(d_flags);
    cudaFree(d_cell_alias);
    for (auto &p : d_s0) { cudaFree(p); p = nullptr; }
    for (auto &b : d_buf)
      for (auto &p : b) { cudaFree(p); p = nullptr; }
    cudaFree(d_vsd);
    cudaFree(d_rows);
    d_tile_nb = d_tile_level = d_cell_slot = nullptr;
    d_flags = d_cell_alias = nullptr;
    d_vsd = d_rows = nullptr;
    has_topology = has_state = false;
  }
};

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
    default: return "unknown error";
  }
}

const char *ibgpu_last_error(void) { return g_last_error.c_str(); }

int ibgpu_create(const ibgpu_case *cs, ibgpu_ctx **out) {
  if (!cs || !out) return IBGPU_E_ARG;
  *out = nullptr;
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
  ibgpu_ctx *c = new (std::nothrow) ibgpu_ctx();
  if (!c) return IBGPU_E_NOMEM;
  c->cs = *cs;
  CaseConst &k = c->cc;
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
  cudaError_t e = cudaGetDevice(&c->device);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, c->device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc((void **)&c->d_diag, sizeof(DevDiag));
  if (e == cudaSuccess) e = cudaMallocHost((void **)&c->h_diag, sizeof(DevDiag));
  if (e != cudaSuccess) {
    int rc = cuda_fail(e, "ibgpu_create");
    ibgpu_destroy(c);
    return rc;
  }
  c->stream = c->own_stream;
  *out = c;
  return IBGPU_OK;
}

int ibgpu_set_stream(ibgpu_ctx *ctx, void *stream) {
  if (!ctx) return IBGPU_E_ARG;
  ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
  return IBGPU_OK;
}

int ibgpu_upload_topology(ibgpu_ctx *ctx, const ibgpu_cells *cells) {
  if (!ctx || !cells || cells->n < 0 || (cells->n > 0 && (!cells->level || !cells->ix ||
                                                          !cells->iy || !cells->flags)))
    return IBGPU_E_ARG;
  const ibgpu_case &cs = ctx->cs;
  const int nlev = cs.nlevels;
  const int64_t n = cells->n;
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->free_layout();

  // 1. owners vs aliases; tiles per level
  std::vector<uint8_t> alias(n, 0);
  std::vector<std::unordered_map<uint64_t, int>> tilemap(nlev);
  std::vector<std::vector<std::pair<int, int>>> tiles(nlev);
  std::vector<int> minx(nlev, 1 << 30), miny(nlev, 1 << 30);
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
    int tx = floordiv(ix, kTile), ty = floordiv(iy, kTile);
    uint64_t k = key2(tx, ty);
    if (!tilemap[l].count(k)) {
      tilemap[l][k] = -1;
      tiles[l].push_back({tx, ty});
      minx[l] = std::min(minx[l], tx);
      miny[l] = std::min(miny[l], ty);
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
  for (int l = 0; l < nlev; ++l) {
    auto &tl = tiles[l];
    int mx = minx[l], my = miny[l];
    std::sort(tl.begin(), tl.end(), [mx, my](const std::pair<int, int> &a, const std::pair<int, int> &b) {
      return morton2((uint32_t)(a.first - mx), (uint32_t)(a.second - my)) <
             morton2((uint32_t)(b.first - mx), (uint32_t)(b.second - my));
    });
    ctx->level_tile_begin[l] = (int)h_tile_level.size();
    ctx->level_tile_count[l] = (int)tl.size();
    for (auto &t : tl) {
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
        auto it = tilemap[l].find(key2(tx, ty));
        h_nb[t * 9 + (oy + 1) * 3 + (ox + 1)] = (it == tilemap[l].end()) ? -1 : it->second;
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
    auto it = tilemap[l].find(key2(tx, ty));
    if (it == tilemap[l].end() || it->second < 0) return -1;
    return (int64_t)it->second * kTileCells + (iy - ty * kTile) * kTile + (ix - tx * kTile);
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
  // 5. the stencils every face of a leaf cell reads must exist
  //    (NS_Solver.H:738-756, NS_Solver.cpp:410-424)
  auto present = [&](int l, int ix, int iy) -> bool {
    int ex = cs.domain_nx << l, ey = cs.domain_ny << l;
    if (cs.periodic_x) ix = ((ix % ex) + ex) % ex;
    if (cs.periodic_y) iy = ((iy % ey) + ey) % ey;
    int64_t s = slot_of(l, ix, iy);
    return s >= 0 && (h_flags[s] & CF_PRESENT);
  };
  for (int64_t s = 0; s < nslots; ++s) {
    if (!(h_flags[s] & CF_NORMAL)) continue;
    int l = ctx->h_slot_level[s], ix = ctx->h_slot_ix[s], iy = ctx->h_slot_iy[s];
    for (int d = 0; d < 4; ++d) {
      int dx = d == 0 ? -1 : d == 1 ? 1 : 0, dy = d == 2 ? -1 : d == 3 ? 1 : 0;
      if (!present(l, ix + dx, iy + dy)) {
        g_last_error = "leaf cell with a missing face neighbour";
        return IBGPU_E_TOPOLOGY;
      }
      // MUSCL: at least one outer neighbour of the face stencil
      if (!present(l, ix - dx, iy - dy) && !present(l, ix + 2 * dx, iy + 2 * dy)) {
        g_last_error = "face stencil with neither outer neighbour";
        return IBGPU_E_TOPOLOGY;
      }
      if (cs.viscous) {
        int tx = dy != 0 ? 1 : 0, ty = dx != 0 ? 1 : 0;
        if (!present(l, ix + tx, iy + ty) || !present(l, ix - tx, iy - ty) ||
            !present(l, ix + dx + tx, iy + dy + ty) || !present(l, ix + dx - tx, iy + dy - ty)) {
          g_last_error = "viscous stencil with a missing cell";
          return IBGPU_E_TOPOLOGY;
        }
      }
    }
  }
  // 6. device arrays
  int rc;
  if ((rc = dev_alloc(&ctx->d_tile_nb, h_nb.size())) ||
      (rc = dev_alloc(&ctx->d_tile_level, (size_t)ntiles)) ||
      (rc = dev_alloc(&ctx->d_flags, (size_t)nslots)) ||
      (rc = dev_alloc(&ctx->d_cell_slot, (size_t)n)) ||
      (rc = dev_alloc(&ctx->d_cell_alias, (size_t)n)) ||
      (rc = dev_alloc(&ctx->d_rows, (size_t)n * 7)))
    return rc;
  for (int f = 0; f < kStateFields; ++f)
    if ((rc = dev_alloc(&ctx->d_s0[f], (size_t)nslots))) return rc;
  for (int b = 0; b < 2; ++b)
    for (int f = 0; f < 4; ++f)
      if ((rc = dev_alloc(&ctx->d_buf[b][f], (size_t)nslots))) return rc;
  if (cs.viscous && (rc = dev_alloc(&ctx->d_vsd, (size_t)nslots * 8))) return rc;
  cudaStream_t st = ctx->stream;
  CK(cudaMemcpyAsync(ctx->d_tile_nb, h_nb.data(), h_nb.size() * 4, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(ctx->d_tile_level, h_tile_level.data(), ntiles * 4, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(ctx->d_flags, h_flags.data(), nslots, cudaMemcpyHostToDevice, st));
  if (n > 0) {
    CK(cudaMemcpyAsync(ctx->d_cell_slot, cell_slot.data(), n * 4, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(ctx->d_cell_alias, alias.data(), n, cudaMemcpyHostToDevice, st));
  }
  // absent slots hold zeros in every field (never read as a stencil value)
  for (int f = 0; f < kStateFields; ++f) CK(cudaMemsetAsync(ctx->d_s0[f], 0, nslots * 8, st));
  for (int b = 0; b < 2; ++b)
    for (int f = 0; f < 4; ++f) CK(cudaMemsetAsync(ctx->d_buf[b][f], 0, nslots * 8, st));
  if (ctx->d_vsd) CK(cudaMemsetAsync(ctx->d_vsd, 0, nslots * 8 * 8, st));
  CK(cudaStreamSynchronize(st));
  ctx->ncells = n;
  ctx->ntiles = ntiles;
  ctx->nslots = nslots;
  ctx->has_topology = true;
  return IBGPU_OK;
}

int ibgpu_layout_info(const ibgpu_ctx *ctx, int64_t *nslots, int64_t *ntiles) {
  if (!ctx) return IBGPU_E_ARG;
  if (nslots) *nslots = ctx->nslots;
  if (ntiles) *ntiles = ctx->ntiles;
  return IBGPU_OK;
}

int ibgpu_upload_state(ibgpu_ctx *ctx, const double *prim) {
  if (!ctx || (!prim && ctx->ncells > 0)) return IBGPU_E_ARG;
  if (!ctx->has_topology) return IBGPU_E_STATE;
  cudaStream_t st = ctx->stream;
  if (ctx->ncells > 0) {
    CK(cudaMemcpyAsync(ctx->d_rows, prim, ctx->ncells * 7 * sizeof(double), cudaMemcpyHostToDevice, st));
    fast::launch_scatter(ctx->d_rows, ctx->d_cell_slot, ctx->d_cell_alias, ctx->ncells, ctx->d_s0,
                         ctx->nsm, st);
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
    fast::launch_gather(ctx->d_rows, ctx->d_cell_slot, ctx->ncells, ctx->d_s0, ctx->nsm, st);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(prim, ctx->d_rows, ctx->ncells * 7 * sizeof(double), cudaMemcpyDeviceToHost, st));
  }
  CK(cudaStreamSynchronize(st));
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

int ibgpu_step(ibgpu_ctx *ctx, int ts, double *dt, ibgpu_diag *diag) {
  if (!ctx || !dt || ts < 0) return IBGPU_E_ARG;
  if (!ctx->has_state) return IBGPU_E_STATE;
  const ibgpu_case &cs = ctx->cs;
  cudaStream_t st = ctx->stream;
  const bool exact = cs.precision == IBGPU_FP64_EXACT;
  const bool mixed = cs.precision == IBGPU_MIXED;

  DevDiag *hd = ctx->h_diag;
  std::memset(hd, 0, sizeof(DevDiag));
  hd->dt = *dt;
  double cfl_init = 10000.0;
  std::memcpy(&hd->cfl_bits, &cfl_init, sizeof(double));
  hd->err_key = ~0ull;
  CK(cudaMemcpyAsync(ctx->d_diag, hd, sizeof(DevDiag), cudaMemcpyHostToDevice, st));

  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> evs;
  std::vector<int> evkind;
  auto mark = [&](int kind) -> cudaEvent_t {
    if (!ctx->timing) return nullptr;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, st);
    evs.push_back({a, b});
    evkind.push_back(kind);
    return b;
  };
  auto done = [&](cudaEvent_t b) {
    if (b) cudaEventRecord(b, st);
  };

  // CFL time step (TimeMarching: Comptdt when ts % dt_var_step == 0)
  const bool do_cfl = (ts % cs.dt_var_step) == 0;
  if (do_cfl) {
    CflArgs ca;
    ca.tile_level = ctx->d_tile_level;
    ca.flags = ctx->d_flags;
    for (int f = 0; f < kStateFields; ++f) ca.s0[f] = ctx->d_s0[f];
    ca.nslots = ctx->nslots;
    ca.diag = ctx->d_diag;
    cudaEvent_t e = mark(2);
    if (exact) exact::launch_cfl(ca, ctx->cc, ctx->nsm, st);
    else fast::launch_cfl(ca, ctx->cc, ctx->nsm, st);
    done(e);
    CK(cudaGetLastError());
  }

  // stages over the tiles of the levels that march at ts
  int64_t marched = 0;
  StageArgs sa;
  std::memset(&sa, 0, sizeof(sa));
  sa.tile_nb = ctx->d_tile_nb;
  sa.tile_level = ctx->d_tile_level;
  sa.flags = ctx->d_flags;
  for (int f = 0; f < kStateFields; ++f) sa.s0[f] = ctx->d_s0[f];
  sa.vsd = ctx->d_vsd;
  sa.nslots = ctx->nslots;
  sa.diag = ctx->d_diag;
  const int S = cs.nstages;
  for (int k = 0; k < S; ++k) {
    const bool fin = (k == S - 1);
    for (int f = 0; f < 4; ++f) {
      static const int map[4] = {F_RHO, F_U, F_V, F_P};
      sa.sin[f] = (k == 0) ? ctx->d_s0[map[f]] : ctx->d_buf[(k - 1) & 1][f];
      sa.sout[f] = fin ? nullptr : ctx->d_buf[k & 1][f];
    }
    sa.tp = cs.tp[k];
    sa.stage = k;
    for (int l = 0; l < cs.nlevels; ++l) {
      if (ts % cs.march_step[l] != cs.march_left[l]) continue;
      if (k == 0) marched += ctx->level_normal_cells[l];
      sa.tile_begin = ctx->level_tile_begin[l];
      cudaEvent_t e = mark(0);
      if (exact) exact::launch_stage(sa, ctx->cc, ctx->level_tile_count[l], cs.limiter, cs.viscous != 0, fin, false, st);
      else fast::launch_stage(sa, ctx->cc, ctx->level_tile_count[l], cs.limiter, cs.viscous != 0, fin, mixed, st);
      done(e);
      CK(cudaGetLastError());
    }
  }
  CK(cudaMemcpyAsync(hd, ctx->d_diag, sizeof(DevDiag), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  for (size_t i = 0; i < evs.size(); ++i) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, evs[i].first, evs[i].second);
    ctx->kms[evkind[i]] += ms;
    ctx->klaunch[evkind[i]] += 1;
    cudaEventDestroy(evs[i].first);
    cudaEventDestroy(evs[i].second);
  }

  // decode the first abort in the reference's order
  int abort_code = 0, abort_slot = -1;
  if (hd->err_key != ~0ull) {
    int check = (int)((hd->err_key >> 32) & 0xff);
    abort_slot = (int)(hd->err_key & 0xffffffffull);
    if (check == ERR_CFL_NEG_DT) abort_code = 424;
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

void ibgpu_destroy(ibgpu_ctx *ctx) {
  if (!ctx) return;
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  ctx->free_layout();
  cudaFree(ctx->d_diag);
  cudaFreeHost(ctx->h_diag);
  if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
  delete ctx;
}

}  // extern "C"
