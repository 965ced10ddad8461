// Kernels of the explicit time step over the tiled level layout (layout.h).
//
// Included by one translation unit per arithmetic build:
//   kernels_fp64.cu   FP64 (multiply-adds contracted) and mixed precision
//   kernels_exact.cu  FP64 compiled with -fmad=false: operation-for-operation
//                     the reference's arithmetic
// Each includer defines IBGPU_KNS, the namespace its launchers live in.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "flux.cuh"
#include "layout.h"

namespace ibgpu {
namespace IBGPU_KNS {

constexpr int kHalo = 2;
constexpr int kReg = kTile + 2 * kHalo;  // 20: tile plus a 2-cell halo
constexpr int kXFaces = kTile * (kTile + 1);
constexpr int kYFaces = (kTile + 1) * kTile;

__device__ __forceinline__ void raise_error(DevDiag *d, int phase, int check, int slot) {
  unsigned long long key = ((unsigned long long)phase << 40) |
                           ((unsigned long long)check << 32) | (unsigned)slot;
  atomicMin(&d->err_key, key);
}

__device__ __forceinline__ unsigned long long warp_max_u64(unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
    v = w > v ? w : v;
  }
  return v;
}

// One stage of the multistage update for one tile per CTA (256 threads):
// NS_Solver::ComputeFaceFlux (NS_Solver.H:704-832), ComptSource
// (NS_Solver.cpp:282-363), UpdateConsVars (:844-985) and ComptNewPrimVar
// (:3-194), plus ResinDomain's max-norm (NS_Solver.H:264-378) on the final
// stage.  Every face of the tile (and of its east/north edge) is computed
// once into shared memory from a 20x20 staged stencil region; each thread
// then gathers the four faces of its cell in the reference's summation order.
template <typename R, int LIM, bool VISC, bool FINAL>
__global__ void __launch_bounds__(kTileCells) stage_kernel(StageArgs a, CaseConst cc) {
  __shared__ R sq[4][kReg * kReg];
  __shared__ uint8_t sfl[kReg * kReg];
  __shared__ R fx[4][kXFaces];  // x-face f between cells (f%17-1, f/17) and (f%17, f/17)
  __shared__ R fy[4][kYFaces];  // y-face f between cells (f%16, f/16-1) and (f%16, f/16)

  const int tid = threadIdx.x;
  const int tile = a.tile_begin + blockIdx.x;
  const int lvl = a.tile_level[tile];
  const LevelConst &L = cc.lev[lvl];

  // ---- stage the stencil region (tile + 2-cell halo, corners not needed)
  for (int r = tid; r < kReg * kReg; r += kTileCells) {
    int rx = r % kReg - kHalo, ry = r / kReg - kHalo;
    int ox = rx < 0 ? -1 : (rx >= kTile ? 1 : 0);
    int oy = ry < 0 ? -1 : (ry >= kTile ? 1 : 0);
    uint8_t f = 0;
    R q0 = R(0), q1 = R(0), q2 = R(0), q3 = R(0);
    if (!(ox && oy)) {
      int nb = a.tile_nb[tile * 9 + (oy + 1) * 3 + (ox + 1)];
      if (nb >= 0) {
        int64_t s = (int64_t)nb * kTileCells + (ry - oy * kTile) * kTile + (rx - ox * kTile);
        f = a.flags[s];
        if (f & CF_PRESENT) {
          const bool varying = (f & (CF_PRIM | CF_RESET)) != 0;
          const double *p0 = varying ? a.sin[0] : a.s0[F_RHO];
          const double *p1 = varying ? a.sin[1] : a.s0[F_U];
          const double *p2 = varying ? a.sin[2] : a.s0[F_V];
          const double *p3 = varying ? a.sin[3] : a.s0[F_P];
          q0 = (R)p0[s];
          q1 = (R)p1[s];
          q2 = (R)p2[s];
          q3 = (R)p3[s];
        }
      }
    }
    sfl[r] = f;
    sq[0][r] = q0;
    sq[1][r] = q1;
    sq[2][r] = q2;
    sq[3][r] = q3;
  }
  __syncthreads();

  Gas<R> g;
  g.gama = (R)cc.gama;
  g.Rg = (R)cc.Rg;
  g.Cv = (R)cc.Cv;
  g.Ma = (R)cc.Ma;
  g.gm1 = (R)cc.gm1;
  g.gamaRg = (R)cc.gamaRg;

  // ---- face fluxes
  for (int w = tid; w < kXFaces + kYFaces; w += kTileCells) {
    const bool xdir = w < kXFaces;
    int i, j, step;
    int rL1, rR1;
    if (xdir) {
      j = w / (kTile + 1);
      i = w % (kTile + 1);
      rR1 = (j + kHalo) * kReg + (i + kHalo);
      rL1 = rR1 - 1;
      step = 1;
    } else {
      int v = w - kXFaces;
      j = v / kTile;
      i = v % kTile;
      rR1 = (j + kHalo) * kReg + (i + kHalo);
      rL1 = rR1 - kReg;
      step = kReg;
    }
    const uint8_t fL = sfl[rL1], fR = sfl[rR1];
    R fm = R(0), fn = R(0), ft = R(0), fe = R(0);
    if ((fL & CF_PRESENT) && (fR & CF_PRESENT) && ((fL | fR) & CF_NORMAL)) {
      int rL2 = rL1 - step, rR2 = rR1 + step;
      const bool hasL2 = (sfl[rL2] & CF_PRESENT) != 0;
      const bool hasR2 = (sfl[rR2] & CF_PRESENT) != 0;
      // missing outer neighbour: use the other side's (NS_Solver.H:743-750)
      const int sL2 = hasL2 ? rL2 : rR2;
      const int sR2 = hasR2 ? rR2 : rL2;
      const int cn = xdir ? 1 : 2, ct = xdir ? 2 : 1;
      const R area = (R)(xdir ? L.area_x : L.area_y);
      roe_face_flux<LIM, R>(g, area,
                            sq[0][sL2], sq[cn][sL2], sq[ct][sL2], sq[3][sL2],
                            sq[0][rL1], sq[cn][rL1], sq[ct][rL1], sq[3][rL1],
                            sq[0][rR1], sq[cn][rR1], sq[ct][rR1], sq[3][rR1],
                            sq[0][sR2], sq[cn][sR2], sq[ct][sR2], sq[3][sR2],
                            fm, fn, ft, fe);
    }
    if (xdir) {
      fx[0][w] = fm;
      fx[1][w] = fn;
      fx[2][w] = ft;
      fx[3][w] = fe;
    } else {
      int v = w - kXFaces;
      fy[0][v] = fm;
      fy[1][v] = ft;
      fy[2][v] = fn;
      fy[3][v] = fe;
    }
  }
  __syncthreads();

  // ---- residual, update, primitive recovery for the thread's own cell
  const int lx = tid % kTile, ly = tid / kTile;
  const int64_t slot = (int64_t)tile * kTileCells + tid;
  const uint8_t fl = sfl[(ly + kHalo) * kReg + (lx + kHalo)];
  unsigned long long rb[4] = {0ull, 0ull, 0ull, 0ull};
  if ((fl & CF_NORMAL) && (fl & (CF_UPDATE | CF_RESET))) {
    const int xlo = ly * (kTile + 1) + lx, xhi = xlo + 1;
    const int ylo = ly * kTile + lx, yhi = ylo + kTile;
    double res[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      double sx = (double)fx[c][xlo] - (double)fx[c][xhi];
      double sy = (double)fy[c][ylo] - (double)fy[c][yhi];
      if (VISC) {
        sx += a.vsd[(int64_t)c * a.nslots + slot];
        sy += a.vsd[(int64_t)(4 + c) * a.nslots + slot];
      }
      res[c] = sx + sy;
    }
    const double dt = a.diag->dt;
    const double level_ts = (a.tp * dt) * L.step_num;
    double orho = a.s0[F_RHO][slot], ou = a.s0[F_U][slot], ov = a.s0[F_V][slot],
           oe = a.s0[F_E][slot];
    double nrho, nu, nv, np, ne, nT;
    bool wrote = false;
    if (fl & CF_UPDATE) {
      // ComptOldConsVar (NS_Solver.H:392-424) then UpdateConsVars
      const double un0 = orho, un1 = orho * ou, un2 = orho * ov, un3 = orho * oe;
      const double cv0 = un0 + res[0] * level_ts / L.vol;
      const double cv1 = un1 + res[1] * level_ts / L.vol;
      const double cv2 = un2 + res[2] * level_ts / L.vol;
      const double cv3 = un3 + res[3] * level_ts / L.vol;
      if (cv0 < 0.0) raise_error(a.diag, 2 + a.stage, ERR_NEG_RHO, (int)slot);
      if (fl & CF_PRIM) {
        // Get_Prim_Vars (FlowVariables.H:50-57), FP64
        nrho = cv0;
        nu = cv1 / cv0;
        nv = cv2 / cv0;
        ne = cv3 / cv0;
        np = (ne - 0.5 * (nu * nu + nv * nv)) * cc.gm1 * nrho;
        nT = np / (nrho * cc.Rg);
        wrote = true;
      }
    }
    if (!wrote && (fl & CF_RESET)) {
      nrho = cc.initvar[0];
      nu = cc.initvar[1];
      nv = cc.initvar[2];
      np = cc.initvar[4];
      nT = cc.initvar[5];
      ne = cc.initvar[6];
      wrote = true;
    }
    if (wrote) {
      if (nT < 0.0) raise_error(a.diag, 2 + a.stage, ERR_NEG_T, (int)slot);
      if (FINAL) {
        a.s0[F_RHO][slot] = nrho;
        a.s0[F_U][slot] = nu;
        a.s0[F_V][slot] = nv;
        a.s0[F_P][slot] = np;
        a.s0[F_E][slot] = ne;
        a.s0[F_T][slot] = nT;
      } else {
        a.sout[0][slot] = nrho;
        a.sout[1][slot] = nu;
        a.sout[2][slot] = nv;
        a.sout[3][slot] = np;
      }
    }
    if (FINAL && (fl & CF_RESNORM)) {
#pragma unroll
      for (int c = 0; c < 4; ++c) rb[c] = (unsigned long long)__double_as_longlong(fabs(res[c]));
    }
  }
  if (FINAL) {
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      unsigned long long m = warp_max_u64(rb[c]);
      // residual components map to res_max[0,1,2,4] (no z momentum in 2-D)
      if ((tid & 31) == 0 && m) atomicMax(&a.diag->res_bits[c == 3 ? 4 : c], m);
    }
  }
}

// Fast build of the stage (FP64 with FastMath divisions/roots, or FP32 flux
// arithmetic for the mixed mode): per-cell limited slopes computed once and
// shared by the cell's two faces in each direction, divisions replaced by
// reciprocals.  Faces whose outer stencil cell is missing use the
// reference's one-sided reconstruction (NS_Solver.H:743-750).  The residual,
// update and primitive recovery run in FP64 in every mode.
template <typename R, int LIM, bool VISC, bool FINAL>
__global__ void __launch_bounds__(kTileCells) stage_kernel_fast(StageArgs a, CaseConst cc) {
  constexpr int kSlopeX = kTile * (kTile + 2);  // x-slopes: rows 0..15, cols -1..16
  constexpr int kSlopeY = (kTile + 2) * kTile;  // y-slopes: rows -1..16, cols 0..15
  __shared__ R sq[4][kReg * kReg];
  __shared__ uint8_t sfl[kReg * kReg];
  __shared__ R slx[4][kSlopeX];
  __shared__ R sly[4][kSlopeY];
  __shared__ R fx[4][kXFaces];
  __shared__ R fy[4][kYFaces];

  const int tid = threadIdx.x;
  const int tile = a.tile_begin + blockIdx.x;
  const int lvl = a.tile_level[tile];
  const LevelConst &L = cc.lev[lvl];

  for (int r = tid; r < kReg * kReg; r += kTileCells) {
    int rx = r % kReg - kHalo, ry = r / kReg - kHalo;
    int ox = rx < 0 ? -1 : (rx >= kTile ? 1 : 0);
    int oy = ry < 0 ? -1 : (ry >= kTile ? 1 : 0);
    uint8_t f = 0;
    R q0 = R(0), q1 = R(0), q2 = R(0), q3 = R(0);
    if (!(ox && oy)) {
      int nb = a.tile_nb[tile * 9 + (oy + 1) * 3 + (ox + 1)];
      if (nb >= 0) {
        int64_t s = (int64_t)nb * kTileCells + (ry - oy * kTile) * kTile + (rx - ox * kTile);
        f = a.flags[s];
        if (f & CF_PRESENT) {
          const bool varying = (f & (CF_PRIM | CF_RESET)) != 0;
          q0 = (R)(varying ? a.sin[0] : a.s0[F_RHO])[s];
          q1 = (R)(varying ? a.sin[1] : a.s0[F_U])[s];
          q2 = (R)(varying ? a.sin[2] : a.s0[F_V])[s];
          q3 = (R)(varying ? a.sin[3] : a.s0[F_P])[s];
        }
      }
    }
    sfl[r] = f;
    sq[0][r] = q0;
    sq[1][r] = q1;
    sq[2][r] = q2;
    sq[3][r] = q3;
  }
  __syncthreads();

  // ---- per-cell limited slopes (valid where both neighbours exist)
  for (int w = tid; w < kSlopeX + kSlopeY; w += kTileCells) {
    int rc, step;
    if (w < kSlopeX) {
      int row = w / (kTile + 2), col = w % (kTile + 2) - 1;
      rc = (row + kHalo) * kReg + (col + kHalo);
      step = 1;
    } else {
      int v = w - kSlopeX;
      int row = v / kTile - 1, col = v % kTile;
      rc = (row + kHalo) * kReg + (col + kHalo);
      step = kReg;
    }
    R s0 = R(0), s1 = R(0), s2 = R(0), s3 = R(0);
    if ((sfl[rc - step] & CF_PRESENT) && (sfl[rc + step] & CF_PRESENT)) {
      s0 = limited_slope<LIM>(sq[0][rc] - sq[0][rc - step], sq[0][rc + step] - sq[0][rc]);
      s1 = limited_slope<LIM>(sq[1][rc] - sq[1][rc - step], sq[1][rc + step] - sq[1][rc]);
      s2 = limited_slope<LIM>(sq[2][rc] - sq[2][rc - step], sq[2][rc + step] - sq[2][rc]);
      s3 = limited_slope<LIM>(sq[3][rc] - sq[3][rc - step], sq[3][rc + step] - sq[3][rc]);
    }
    if (w < kSlopeX) {
      slx[0][w] = s0; slx[1][w] = s1; slx[2][w] = s2; slx[3][w] = s3;
    } else {
      int v = w - kSlopeX;
      sly[0][v] = s0; sly[1][v] = s1; sly[2][v] = s2; sly[3][v] = s3;
    }
  }
  __syncthreads();

  Gas<R> g;
  g.gama = (R)cc.gama;
  g.Rg = (R)cc.Rg;
  g.Cv = (R)cc.Cv;
  g.Ma = (R)cc.Ma;
  g.gm1 = (R)cc.gm1;
  g.gamaRg = (R)cc.gamaRg;
  g.inv_Rg = (R)(1.0 / cc.Rg);
  g.inv_gm1 = (R)(1.0 / cc.gm1);

  // ---- face fluxes
  for (int w = tid; w < kXFaces + kYFaces; w += kTileCells) {
    const bool xdir = w < kXFaces;
    int rL1, rR1, step, sL, sR;  // sL, sR: slope slots of L1 and R1
    const R(*sl)[kSlopeX];
    if (xdir) {
      int j = w / (kTile + 1), i = w % (kTile + 1);
      rR1 = (j + kHalo) * kReg + (i + kHalo);
      rL1 = rR1 - 1;
      step = 1;
      sR = j * (kTile + 2) + (i + 1);
      sL = sR - 1;
      sl = slx;
    } else {
      int v = w - kXFaces;
      int j = v / kTile, i = v % kTile;
      rR1 = (j + kHalo) * kReg + (i + kHalo);
      rL1 = rR1 - kReg;
      step = kReg;
      sR = (j + 1) * kTile + i;
      sL = sR - kTile;
      sl = sly;
    }
    const uint8_t fL = sfl[rL1], fR = sfl[rR1];
    R fm = R(0), fn = R(0), ft = R(0), fe = R(0);
    if ((fL & CF_PRESENT) && (fR & CF_PRESENT) && ((fL | fR) & CF_NORMAL)) {
      const int rL2 = rL1 - step, rR2 = rR1 + step;
      const bool hasL2 = (sfl[rL2] & CF_PRESENT) != 0;
      const bool hasR2 = (sfl[rR2] & CF_PRESENT) != 0;
      R ls[4], rs[4];
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        ls[c] = hasL2 ? sq[c][rL1] + sl[c][sL]
                      : muscl_left_fast<LIM>(sq[c][rR2], sq[c][rL1], sq[c][rR1]);
        rs[c] = hasR2 ? sq[c][rR1] - sl[c][sR]
                      : muscl_right_fast<LIM>(sq[c][rL1], sq[c][rR1], sq[c][rL2]);
      }
      const int cn = xdir ? 1 : 2, ct = xdir ? 2 : 1;
      const R area = (R)(xdir ? L.area_x : L.area_y);
      roe_flux_states<R>(g, area, ls[0], ls[cn], ls[ct], ls[3], rs[0], rs[cn], rs[ct], rs[3],
                         fm, fn, ft, fe);
    }
    if (xdir) {
      fx[0][w] = fm; fx[1][w] = fn; fx[2][w] = ft; fx[3][w] = fe;
    } else {
      int v = w - kXFaces;
      fy[0][v] = fm; fy[1][v] = ft; fy[2][v] = fn; fy[3][v] = fe;
    }
  }
  __syncthreads();

  // ---- residual, update, primitive recovery (FP64)
  const int lx = tid % kTile, ly = tid / kTile;
  const int64_t slot = (int64_t)tile * kTileCells + tid;
  const uint8_t fl = sfl[(ly + kHalo) * kReg + (lx + kHalo)];
  unsigned long long rb[4] = {0ull, 0ull, 0ull, 0ull};
  if ((fl & CF_NORMAL) && (fl & (CF_UPDATE | CF_RESET))) {
    const int xlo = ly * (kTile + 1) + lx, xhi = xlo + 1;
    const int ylo = ly * kTile + lx, yhi = ylo + kTile;
    double res[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      double sx = (double)fx[c][xlo] - (double)fx[c][xhi];
      double sy = (double)fy[c][ylo] - (double)fy[c][yhi];
      if (VISC) {
        sx += a.vsd[(int64_t)c * a.nslots + slot];
        sy += a.vsd[(int64_t)(4 + c) * a.nslots + slot];
      }
      res[c] = sx + sy;
    }
    const double dt = a.diag->dt;
    const double scale = (a.tp * dt) * L.step_num * L.inv_vol;
    double nrho, nu, nv, np, ne, nT;
    bool wrote = false;
    if (fl & CF_UPDATE) {
      const double orho = a.s0[F_RHO][slot], ou = a.s0[F_U][slot], ov = a.s0[F_V][slot],
                   oe = a.s0[F_E][slot];
      const double cv0 = orho + res[0] * scale;
      const double cv1 = orho * ou + res[1] * scale;
      const double cv2 = orho * ov + res[2] * scale;
      const double cv3 = orho * oe + res[3] * scale;
      if (cv0 < 0.0) raise_error(a.diag, 2 + a.stage, ERR_NEG_RHO, (int)slot);
      if (fl & CF_PRIM) {
        const double ir = FastMath<double>::rcp(cv0);
        nrho = cv0;
        nu = cv1 * ir;
        nv = cv2 * ir;
        ne = cv3 * ir;
        np = (ne - 0.5 * (nu * nu + nv * nv)) * cc.gm1 * nrho;
        nT = np * ir * cc.inv_Rg;
        wrote = true;
      }
    }
    if (!wrote && (fl & CF_RESET)) {
      nrho = cc.initvar[0];
      nu = cc.initvar[1];
      nv = cc.initvar[2];
      np = cc.initvar[4];
      nT = cc.initvar[5];
      ne = cc.initvar[6];
      wrote = true;
    }
    if (wrote) {
      if (nT < 0.0) raise_error(a.diag, 2 + a.stage, ERR_NEG_T, (int)slot);
      if (FINAL) {
        a.s0[F_RHO][slot] = nrho;
        a.s0[F_U][slot] = nu;
        a.s0[F_V][slot] = nv;
        a.s0[F_P][slot] = np;
        a.s0[F_E][slot] = ne;
        a.s0[F_T][slot] = nT;
      } else {
        a.sout[0][slot] = nrho;
        a.sout[1][slot] = nu;
        a.sout[2][slot] = nv;
        a.sout[3][slot] = np;
      }
    }
    if (FINAL && (fl & CF_RESNORM)) {
#pragma unroll
      for (int c = 0; c < 4; ++c) rb[c] = (unsigned long long)__double_as_longlong(fabs(res[c]));
    }
  }
  if (FINAL) {
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      unsigned long long m = warp_max_u64(rb[c]);
      if ((tid & 31) == 0 && m) atomicMax(&a.diag->res_bits[c == 3 ? 4 : c], m);
    }
  }
}

// CFL time step over the normal cells of every level, NS_Solver::Comptdt
// (NS_Solver.cpp:196-280): a per-cell bound, a warp-shuffle min and one
// atomic per warp (positive doubles order like their bit patterns).
__global__ void __launch_bounds__(256) cfl_kernel(CflArgs a, CaseConst cc) {
  double best = 10000.0;
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < a.nslots;
       s += (int64_t)gridDim.x * blockDim.x) {
    if (!(a.flags[s] & CF_NORMAL)) continue;
    const LevelConst &L = cc.lev[a.tile_level[s / kTileCells]];
    double c = sqrt(cc.gamaRg * a.s0[F_T][s]);
    double c0 = (fabs(a.s0[F_U][s]) + c) * L.area_x;
    double c1 = (fabs(a.s0[F_V][s]) + c) * L.area_y;
    double c2 = (0.0 + c) * L.area_z;
    double d0 = L.cfl_vol / (c0 + c1 + c2);
    if (d0 < 0.0) raise_error(a.diag, 1, ERR_CFL_NEG_DT, (int)s);
    best = (d0 < best) ? d0 : best;  // std::min(CFL_dt, CFL_dt0) ignores NaN
  }
  unsigned long long b = (unsigned long long)__double_as_longlong(best);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    unsigned long long w = __shfl_xor_sync(0xffffffffu, b, o);
    b = w < b ? w : b;
  }
  if ((threadIdx.x & 31) == 0) atomicMin(&a.diag->cfl_bits, b);
}

// dt = min(CFL_dt, dt*dt_ratio) (NS_Solver.cpp:263)
__global__ void finalize_dt_kernel(DevDiag *d, CaseConst cc) {
  double cdt = __longlong_as_double((long long)d->cfl_bits);
  double cand = d->dt * cc.dt_ratio;
  d->dt = (cand < cdt) ? cand : cdt;
}

// Scatter/gather between the caller's cell list (FlowVariables rows of 7
// doubles) and the slot SoA; alias rows (periodic copies) read their source
// slot on download and are skipped on upload.
__global__ void scatter_state_kernel(const double *rows, const int32_t *cell_slot,
                                     const uint8_t *cell_is_alias, int64_t n,
                                     double *s0_rho, double *s0_u, double *s0_v, double *s0_p,
                                     double *s0_e, double *s0_T) {
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x) {
    if (cell_is_alias[c]) continue;
    int64_t s = cell_slot[c];
    const double *r = rows + 7 * c;
    s0_rho[s] = r[0];
    s0_u[s] = r[1];
    s0_v[s] = r[2];
    s0_p[s] = r[4];
    s0_T[s] = r[5];
    s0_e[s] = r[6];
  }
}

__global__ void gather_state_kernel(double *rows, const int32_t *cell_slot, int64_t n,
                                    const double *s0_rho, const double *s0_u,
                                    const double *s0_v, const double *s0_p,
                                    const double *s0_e, const double *s0_T) {
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x) {
    int64_t s = cell_slot[c];
    double *r = rows + 7 * c;
    r[0] = s0_rho[s];
    r[1] = s0_u[s];
    r[2] = s0_v[s];
    r[3] = 0.0;
    r[4] = s0_p[s];
    r[5] = s0_T[s];
    r[6] = s0_e[s];
  }
}

// ---- launchers (one set per arithmetic build)
#ifdef IBGPU_FAST_BUILD
#define IBGPU_STAGE_KERNEL stage_kernel_fast
#else
#define IBGPU_STAGE_KERNEL stage_kernel
#endif

template <typename R, int LIM>
static void launch_stage_t(const StageArgs &a, const CaseConst &cc, int ntiles, bool visc,
                           bool final_stage, cudaStream_t st) {
  dim3 grid(ntiles), block(kTileCells);
  if (visc) {
    if (final_stage) IBGPU_STAGE_KERNEL<R, LIM, true, true><<<grid, block, 0, st>>>(a, cc);
    else IBGPU_STAGE_KERNEL<R, LIM, true, false><<<grid, block, 0, st>>>(a, cc);
  } else {
    if (final_stage) IBGPU_STAGE_KERNEL<R, LIM, false, true><<<grid, block, 0, st>>>(a, cc);
    else IBGPU_STAGE_KERNEL<R, LIM, false, false><<<grid, block, 0, st>>>(a, cc);
  }
}

void launch_stage(const StageArgs &a, const CaseConst &cc, int ntiles, int limiter, bool visc,
                  bool final_stage, bool mixed, cudaStream_t st) {
  if (ntiles <= 0) return;
#ifndef IBGPU_FAST_BUILD
  mixed = false;  // the exact build is FP64 only
#endif
  if (mixed) {
    if (limiter == LIM_MINMOD) launch_stage_t<float, LIM_MINMOD>(a, cc, ntiles, visc, final_stage, st);
    else launch_stage_t<float, LIM_VANLEER>(a, cc, ntiles, visc, final_stage, st);
  } else {
    if (limiter == LIM_MINMOD) launch_stage_t<double, LIM_MINMOD>(a, cc, ntiles, visc, final_stage, st);
    else launch_stage_t<double, LIM_VANLEER>(a, cc, ntiles, visc, final_stage, st);
  }
}

void launch_cfl(const CflArgs &a, const CaseConst &cc, int nsm, cudaStream_t st) {
  int64_t blocks = (a.nslots + 255) / 256;
  int64_t cap = (int64_t)nsm * 8;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  cfl_kernel<<<(unsigned)blocks, 256, 0, st>>>(a, cc);
  finalize_dt_kernel<<<1, 1, 0, st>>>(a.diag, cc);
}

void launch_scatter(const double *rows, const int32_t *cell_slot, const uint8_t *alias, int64_t n,
                    double *const s0[kStateFields], int nsm, cudaStream_t st) {
  int64_t blocks = (n + 255) / 256;
  if (blocks > (int64_t)nsm * 16) blocks = (int64_t)nsm * 16;
  if (blocks < 1) blocks = 1;
  scatter_state_kernel<<<(unsigned)blocks, 256, 0, st>>>(rows, cell_slot, alias, n, s0[F_RHO],
                                                         s0[F_U], s0[F_V], s0[F_P], s0[F_E],
                                                         s0[F_T]);
}

void launch_gather(double *rows, const int32_t *cell_slot, int64_t n,
                   double *const s0[kStateFields], int nsm, cudaStream_t st) {
  int64_t blocks = (n + 255) / 256;
  if (blocks > (int64_t)nsm * 16) blocks = (int64_t)nsm * 16;
  if (blocks < 1) blocks = 1;
  gather_state_kernel<<<(unsigned)blocks, 256, 0, st>>>(rows, cell_slot, n, s0[F_RHO], s0[F_U],
                                                        s0[F_V], s0[F_P], s0[F_E], s0[F_T]);
}

}  // namespace IBGPU_KNS
}  // namespace ibgpu
