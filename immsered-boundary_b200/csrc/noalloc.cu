// ibgpu_step_periodic_noalloc: one time step of a single-level periodic
// grid without any device allocation.
//
// Who needs it: a caller that may not allocate device memory while it runs
// the solver — for instance a host application whose device memory belongs
// to another framework's pool (a multiphysics coupler that hands the solver
// buffers it owns), or a time loop that must not hit cudaMalloc/cudaFree
// because they synchronise the whole device.  Such a caller passes its own
// device buffers for the state in and out; every intermediate (the tiled
// state, the two stage buffers, the neighbour table and the step's
// diagnostics) lives in one file-scope __device__ array of fixed size, which
// each GPU that loads the library keeps until the process exits.
//
// Set-up: the first call on a device looks up the array's device address
// with cudaGetSymbolAddress (once per device, with that device current); make
// that first call before any stream capture.  All calls share the array and
// it keeps the last call's contents: calls that overlap on the GPU (two
// streams, two host threads) race and must be serialised by the caller.
#include <cstdint>
#include <cstring>
#include <mutex>

#include <cuda_runtime.h>

#include "../../include/ibgpu.h"
#include "host_internal.h"
#include "launchers.h"
#include "layout.h"

using namespace ibgpu;

namespace {

constexpr int kMaxCells = IBGPU_NOALLOC_MAX_CELLS;
constexpr int kMaxTiles = kMaxCells / kTileCells;

// byte layout of the scratch array (each part 256-byte aligned)
constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
constexpr size_t kOffDiag = 0;
constexpr size_t kOffNb = align256(kOffDiag + sizeof(DevDiag));
constexpr size_t kOffLevel = align256(kOffNb + sizeof(int32_t) * 9 * kMaxTiles);
constexpr size_t kOffFlags = align256(kOffLevel + sizeof(int32_t) * kMaxTiles);
constexpr size_t kOffS0 = align256(kOffFlags + kMaxCells);
constexpr size_t kOffBuf = kOffS0 + sizeof(double) * kStateFields * kMaxCells;
constexpr size_t kScratchBytes = kOffBuf + sizeof(double) * 8 * kMaxCells;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_mu;
void *g_scratch_addr[256] = {};

// periodic neighbour table of a row-major tile grid, all-leaf flags, and the
// step diagnostics' initial values (the array keeps the previous call's)
__global__ void noalloc_setup_kernel(int ntx, int nty, int32_t *nb, int32_t *lvl, uint8_t *flags,
                                     DevDiag *diag, double dt) {
  const int ntiles = ntx * nty;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int stride = gridDim.x * blockDim.x;
  for (int t = tid; t < ntiles; t += stride) {
    int tx = t % ntx, ty = t / ntx;
    for (int oy = -1; oy <= 1; ++oy)
      for (int ox = -1; ox <= 1; ++ox) {
        int x = (tx + ox + ntx) % ntx, y = (ty + oy + nty) % nty;
        nb[t * 9 + (oy + 1) * 3 + (ox + 1)] = y * ntx + x;
      }
    lvl[t] = 0;
  }
  for (int s = tid; s < ntiles * kTileCells; s += stride)
    flags[s] = CF_PRESENT | CF_NORMAL | CF_UPDATE | CF_PRIM | CF_RESNORM;
  if (tid == 0) {
    diag->dt = dt;
    double cfl0 = 10000.0;
    diag->cfl_bits = (unsigned long long)__double_as_longlong(cfl0);
    for (int c = 0; c < 5; ++c) diag->res_bits[c] = 0ull;
    diag->err_key = ~0ull;
  }
}

__device__ __forceinline__ int64_t tiled_slot(int ix, int iy, int ntx) {
  return ((int64_t)(iy / kTile) * ntx + ix / kTile) * kTileCells + (iy % kTile) * kTile + ix % kTile;
}

// caller rows (row-major cells, FlowVariables layout) -> tiled SoA
__global__ void noalloc_rows_in_kernel(const double *rows, int nx, int ny, double *s0) {
  const int64_t n = (int64_t)nx * ny;
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x) {
    int ix = (int)(c % nx), iy = (int)(c / nx);
    int64_t s = tiled_slot(ix, iy, nx / kTile);
    const double *r = rows + 7 * c;
    s0[F_RHO * (int64_t)kMaxCells + s] = r[0];
    s0[F_U * (int64_t)kMaxCells + s] = r[1];
    s0[F_V * (int64_t)kMaxCells + s] = r[2];
    s0[F_P * (int64_t)kMaxCells + s] = r[4];
    s0[F_E * (int64_t)kMaxCells + s] = r[6];
    s0[F_T * (int64_t)kMaxCells + s] = r[5];
  }
}

// tiled SoA -> caller rows
__global__ void noalloc_rows_out_kernel(const double *s0, int nx, int ny, double *rows) {
  const int64_t n = (int64_t)nx * ny;
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x) {
    int ix = (int)(c % nx), iy = (int)(c / nx);
    int64_t s = tiled_slot(ix, iy, nx / kTile);
    double *r = rows + 7 * c;
    r[0] = s0[F_RHO * (int64_t)kMaxCells + s];
    r[1] = s0[F_U * (int64_t)kMaxCells + s];
    r[2] = s0[F_V * (int64_t)kMaxCells + s];
    r[3] = 0.0;
    r[4] = s0[F_P * (int64_t)kMaxCells + s];
    r[5] = s0[F_T * (int64_t)kMaxCells + s];
    r[6] = s0[F_E * (int64_t)kMaxCells + s];
  }
}

#define NA_CK(call)                                                       \
  do {                                                                    \
    cudaError_t e_ = (call);                                              \
    if (e_ != cudaSuccess) {                                              \
      set_last_error(std::string(#call) + ": " + cudaGetErrorString(e_)); \
      return IBGPU_E_CUDA;                                                \
    }                                                                     \
  } while (0)

int scratch_address(unsigned char **out) {
  int dev = 0;
  NA_CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 256) {
    set_last_error("device ordinal out of range");
    return IBGPU_E_ARG;
  }
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_addr[dev]) {
    void *p = nullptr;
    NA_CK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_scratch_addr[dev] = p;
  }
  *out = (unsigned char *)g_scratch_addr[dev];
  return IBGPU_OK;
}

}  // namespace

extern "C" int ibgpu_step_periodic_noalloc(const ibgpu_case *cs, int ts, int nx, int ny,
                                           const double *d_rows_in, double *d_rows_out,
                                           double *dt, ibgpu_diag *diag, void *stream) {
  if (!cs || !dt || !d_rows_in || !d_rows_out || ts < 0) return IBGPU_E_ARG;
  int rc = validate_case(cs);
  if (rc) return rc;
  if (cs->nlevels != 1 || !cs->periodic_x || !cs->periodic_y || cs->viscous ||
      cs->domain_nx != nx || cs->domain_ny != ny || cs->march_step[0] != 1) {
    set_last_error("the allocation-free step takes one periodic inviscid level");
    return IBGPU_E_ARG;
  }
  if (nx <= 0 || ny <= 0 || nx % kTile || ny % kTile || (int64_t)nx * ny > kMaxCells) {
    set_last_error("grid must be a multiple of 16 per side and at most IBGPU_NOALLOC_MAX_CELLS cells");
    return IBGPU_E_ARG;
  }
  unsigned char *base = nullptr;
  if ((rc = scratch_address(&base))) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  CaseConst cc;
  fill_case_const(cs, cc);

  DevDiag *d_diag = (DevDiag *)(base + kOffDiag);
  int32_t *d_nb = (int32_t *)(base + kOffNb);
  int32_t *d_lvl = (int32_t *)(base + kOffLevel);
  uint8_t *d_flags = base + kOffFlags;
  double *d_s0 = (double *)(base + kOffS0);
  double *d_buf = (double *)(base + kOffBuf);
  const int ntx = nx / kTile, nty = ny / kTile, ntiles = ntx * nty;
  const int64_t nslots = (int64_t)ntiles * kTileCells;

  noalloc_setup_kernel<<<64, 256, 0, st>>>(ntx, nty, d_nb, d_lvl, d_flags, d_diag, *dt);
  noalloc_rows_in_kernel<<<(nx * ny + 255) / 256, 256, 0, st>>>(d_rows_in, nx, ny, d_s0);
  NA_CK(cudaGetLastError());

  const bool exact = cs->precision == IBGPU_FP64_EXACT;
  const bool mixed = cs->precision == IBGPU_MIXED;
  int dev = 0, nsm = 148;
  NA_CK(cudaGetDevice(&dev));
  NA_CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  if (ts % cs->dt_var_step == 0) {
    CflArgs ca;
    ca.tile_level = d_lvl;
    ca.flags = d_flags;
    for (int f = 0; f < kStateFields; ++f) ca.s0[f] = d_s0 + (int64_t)f * kMaxCells;
    ca.nslots = nslots;
    ca.phase = 1;
    ca.diag = d_diag;
    if (exact) exact::launch_cfl(ca, cc, nsm, st);
    else fast::launch_cfl(ca, cc, nsm, st);
  }
  StageArgs sa;
  std::memset(&sa, 0, sizeof(sa));
  sa.tile_nb = d_nb;
  sa.tile_level = d_lvl;
  sa.flags = d_flags;
  sa.tile_begin = 0;
  for (int f = 0; f < kStateFields; ++f) sa.s0[f] = d_s0 + (int64_t)f * kMaxCells;
  sa.vsd = nullptr;
  sa.nslots = nslots;
  sa.diag = d_diag;
  static const int map[4] = {F_RHO, F_U, F_V, F_P};
  for (int k = 0; k < cs->nstages; ++k) {
    const bool fin = k == cs->nstages - 1;
    for (int f = 0; f < 4; ++f) {
      // stage buffers (FP32 values in the mixed build, in the same regions)
      sa.v.sin[f] = (k == 0) ? (const void *)sa.s0[map[f]]
                             : (const void *)(d_buf + ((int64_t)(((k - 1) & 1) * 4 + f)) * kMaxCells);
      sa.v.sout[f] = fin ? nullptr : (void *)(d_buf + ((int64_t)((k & 1) * 4 + f)) * kMaxCells);
    }
    sa.v.tp = cs->tp[k];
    sa.phase = 2 + k;
    if (exact) exact::launch_stage(sa, cc, ntiles, cs->limiter, false, fin, false, k, st);
    else fast::launch_stage(sa, cc, ntiles, cs->limiter, false, fin, mixed, k, st);
  }
  noalloc_rows_out_kernel<<<(nx * ny + 255) / 256, 256, 0, st>>>(d_s0, nx, ny, d_rows_out);
  NA_CK(cudaGetLastError());

  DevDiag hd;
  NA_CK(cudaMemcpyAsync(&hd, d_diag, sizeof(DevDiag), cudaMemcpyDeviceToHost, st));
  NA_CK(cudaStreamSynchronize(st));
  int abort_code = 0;
  if (hd.err_key != ~0ull) {
    int check = (int)((hd.err_key >> 32) & 0xff);  // one step: phases 1 (CFL), 2+k
    abort_code = check == ERR_CFL_NEG_DT ? 424 : check == ERR_NEG_T ? 37 : 523;
  }
  for (int c = 0; c < 5; ++c) {
    double v;
    std::memcpy(&v, &hd.res_bits[c], sizeof(double));
    if (v != v && !abort_code) abort_code = 268;
  }
  *dt = hd.dt;
  if (diag) {
    std::memset(diag, 0, sizeof(*diag));
    diag->dt = hd.dt;
    std::memcpy(&diag->cfl_dt, &hd.cfl_bits, sizeof(double));
    for (int c = 0; c < 5; ++c) std::memcpy(&diag->res_max[c], &hd.res_bits[c], sizeof(double));
    diag->abort_code = abort_code;
    diag->cells_marched = (int64_t)nx * ny;
    if (abort_code && abort_code != 268) {
      int slot = (int)(hd.err_key & 0xffffffffull);
      int tile = slot / kTileCells, local = slot % kTileCells;
      diag->abort_ix = (tile % ntx) * kTile + local % kTile;
      diag->abort_iy = (tile / ntx) * kTile + local / kTile;
    }
  }
  return abort_code ? IBGPU_E_ABORT : IBGPU_OK;
}
