// Kernels of the explicit time step over the tiled level layout (layout.h).
//
// Included by one translation unit per arithmetic build:
//   kernels_fp64.cu   FP64 (multiply-adds contracted) and mixed precision
//   kernels_exact.cu  FP64 compiled with -fmad=false: operation-for-operation
//                     the reference's arithmetic
// Each includer defines IBGPU_KNS, the namespace its launchers live in.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <mutex>
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

// Exact maximum / minimum of a 64-bit word over the full warp with the
// 32-bit warp reductions (redux.sync): the extreme high word first, then the
// extreme low word among the lanes that hold it.  Four instructions instead
// of five rounds of two 32-bit shuffles and a 64-bit compare.
__device__ __forceinline__ unsigned long long warp_max_u64(unsigned long long v) {
  const unsigned hi = (unsigned)(v >> 32), lo = (unsigned)v;
  const unsigned mh = __reduce_max_sync(0xffffffffu, hi);
  const unsigned ml = __reduce_max_sync(0xffffffffu, hi == mh ? lo : 0u);
  return ((unsigned long long)mh << 32) | ml;
}

__device__ __forceinline__ unsigned long long warp_min_u64(unsigned long long v) {
  const unsigned hi = (unsigned)(v >> 32), lo = (unsigned)v;
  const unsigned mh = __reduce_min_sync(0xffffffffu, hi);
  const unsigned ml = __reduce_min_sync(0xffffffffu, hi == mh ? lo : 0xffffffffu);
  return ((unsigned long long)mh << 32) | ml;
}

// Threads of a fast-build stage CTA: FP64 adds a ninth warp that owns the
// tile's east/north edge faces and outer slopes, so every warp computes two
// faces; FP32 keeps 8 warps (its face work is cheap enough).
// Whether a thread evaluates its two faces as one paired flux: FP32 yes
// (f32x2 instructions); FP64 no (interleaving two scalar chains needs
// registers that cost more occupancy than the extra independence returns).
template <typename R>
constexpr bool kPairFaces = sizeof(R) == 4;

template <typename R>
struct StageThreads {
  static constexpr int value = sizeof(R) == 8 ? 288 : kTileCells;
};

// Resident CTAs per SM the register budget is fixed for, by arithmetic and
// block shape (the batched stage tunes between 256 and 288 threads).
template <typename R, int NT>
constexpr int stage_min_blocks() {
  return sizeof(R) == 8 ? 4 : (NT > kTileCells ? 5 : 6);
}

// Residual max-norm of a block of up to 9 warps into the step's diag: warp and
// block maxima, then one atomicMax per component and block whose result
// nobody reads, so it retires as a fire-and-forget reduction (reading the
// global value first to skip it put a memory round trip on the tail of
// every CTA: 29 us per FP64 2048^2 final stage).  Components map to
// res_max[0,1,2,4] (no z momentum in 2-D).
// Every thread of the block must call it; sred is shared scratch of 32
// words that no thread reads or writes any more.
template <int NT = kTileCells>
__device__ __forceinline__ void block_resnorm(const unsigned long long (&rb)[4], DevDiag *d,
                                              unsigned long long *sred) {
  constexpr int kW = NT / 32;
  const int tid = threadIdx.x;
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const unsigned long long m = warp_max_u64(rb[c]);
    if ((tid & 31) == 0) sred[c * kW + (tid >> 5)] = m;
  }
  __syncthreads();
  if (tid < 4) {
    unsigned long long m = 0ull;
#pragma unroll
    for (int w = 0; w < kW; ++w) m = sred[tid * kW + w] > m ? sred[tid * kW + w] : m;
    unsigned long long *dst = &d->res_bits[tid == 3 ? 4 : tid];
    atomicMax(dst, m);  // result unused: a reduction the CTA does not wait for
  }
}

// CFL bound of one normal cell, NS_Solver::Comptdt (NS_Solver.cpp:196-280),
// with every operation separately rounded so the CFL pass and the final
// stages that fold it in produce the same bits in every build.
__device__ __forceinline__ double cfl_cell_bound(double T, double u, double v, const LevelConst &L,
                                                 const CaseConst &cc) {
  const double c = __dsqrt_rn(__dmul_rn(cc.gamaRg, T));
  const double c0 = __dmul_rn(__dadd_rn(fabs(u), c), L.area_x);
  const double c1 = __dmul_rn(__dadd_rn(fabs(v), c), L.area_y);
  const double c2 = __dmul_rn(__dadd_rn(0.0, c), L.area_z);
  return __ddiv_rn(L.cfl_vol, __dadd_rn(__dadd_rn(c0, c1), c2));
}

// Block minimum of one positive double per thread (as bits) into *dst, one
// atomic per block (result unused: not waited for); every thread of the
// block calls it; sred is shared scratch of NT/32 words nobody else uses
// meanwhile.
template <int NT>
__device__ __forceinline__ void block_min_bits(unsigned long long b, unsigned long long *dst,
                                               unsigned long long *sred) {
  b = warp_min_u64(b);
  if ((threadIdx.x & 31) == 0) sred[threadIdx.x >> 5] = b;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < NT / 32; ++k) b = sred[k] < b ? sred[k] : b;
    atomicMin(dst, b);  // result unused: a reduction the CTA does not wait for
  }
}

// The next step's CFL pass folded into a final stage: the bound of each
// normal cell from the state this stage wrote (cb >= 0) or, for a normal
// cell it did not write, from the step state; block minimum into
// diag->cfl_next_bits.  All threads call it (own = the thread owns a cell).
template <int NT>
__device__ __forceinline__ void fold_next_cfl(const StageArgs &a, const LevelConst &L,
                                              const CaseConst &cc, uint8_t fl, int64_t slot,
                                              double cb, unsigned long long *sred, int phase,
                                              bool own = true) {
  double best = 10000.0;
  if (own && (fl & CF_NORMAL)) {
    const double d0 =
        cb >= 0.0 ? cb : cfl_cell_bound(a.s0[F_T][slot], a.s0[F_U][slot], a.s0[F_V][slot], L, cc);
    if (d0 < 0.0) raise_error(a.diag, phase, ERR_CFL_NEG_DT, (int)slot);
    best = (d0 < best) ? d0 : best;
  }
  __syncthreads();  // sred is free again (block_resnorm read it)
  block_min_bits<NT>((unsigned long long)__double_as_longlong(best), &a.diag->cfl_next_bits,
                     sred + 64);
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
          const double *p0 = varying ? static_cast<const double *>(a.v.sin[0]) : a.s0[F_RHO];
          const double *p1 = varying ? static_cast<const double *>(a.v.sin[1]) : a.s0[F_U];
          const double *p2 = varying ? static_cast<const double *>(a.v.sin[2]) : a.s0[F_V];
          const double *p3 = varying ? static_cast<const double *>(a.v.sin[3]) : a.s0[F_P];
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
  double cb = -1.0;  // next step's CFL bound of this cell, when this stage writes it
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
    const double level_ts = (a.v.tp * dt) * L.step_num;
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
      if (cv0 < 0.0) raise_error(a.diag, a.phase, ERR_NEG_RHO, (int)slot);
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
      if (nT < 0.0) raise_error(a.diag, a.phase, ERR_NEG_T, (int)slot);
      if (FINAL) {
        a.s0[F_RHO][slot] = nrho;
        a.s0[F_U][slot] = nu;
        a.s0[F_V][slot] = nv;
        a.s0[F_P][slot] = np;
        a.s0[F_E][slot] = ne;
        a.s0[F_T][slot] = nT;
      } else {
        static_cast<double *>(a.v.sout[0])[slot] = nrho;
        static_cast<double *>(a.v.sout[1])[slot] = nu;
        static_cast<double *>(a.v.sout[2])[slot] = nv;
        static_cast<double *>(a.v.sout[3])[slot] = np;
      }
    }
    if (FINAL && (fl & CF_RESNORM)) {
#pragma unroll
      for (int c = 0; c < 4; ++c) rb[c] = (unsigned long long)__double_as_longlong(fabs(res[c]));
    }
    if (FINAL && a.v.cfl_next && wrote) cb = cfl_cell_bound(nT, nu, nv, L, cc);
  }
  if (FINAL) {
    __shared__ unsigned long long sred[64 + kTileCells / 32];
    block_resnorm(rb, a.diag, sred);
    if (a.v.cfl_next) fold_next_cfl<kTileCells>(a, L, cc, fl, slot, cb, sred, a.v.cfl_next - 1);
  }
}

// Fast build of the stage (FP64 with FastMath divisions/roots, or FP32 flux
// arithmetic for the mixed mode): per-cell limited slopes computed once and
// shared by the cell's two faces in each direction, divisions replaced by
// reciprocals.  Faces whose outer stencil cell is missing use the
// reference's one-sided reconstruction (NS_Solver.H:743-750).  The residual,
// update and primitive recovery run in FP64 in every mode.
// Four values of one cell (rho, u, v, p), one limited slope set, or one
// face flux (mass, x-momentum, y-momentum, energy).  In shared memory an FP32
// record is one float4; an FP64 record is split over two double2 planes
// (components 0-1 at [i], 2-3 at [i + n] for an array of n records), so a
// warp reading consecutive records moves 16-byte words at a 16-byte stride
// and every 128-bit access is conflict-free.
template <typename R>
struct Q4 {
  R x, y, z, w;
};

template <typename R>
struct SRec;

template <>
struct SRec<float> {
  using V = float4;
  static constexpr int kPlanes = 1;
  static __device__ __forceinline__ Q4<float> ld(const V *a, int i, int) {
    const float4 t = a[i];
    return Q4<float>{t.x, t.y, t.z, t.w};
  }
  static __device__ __forceinline__ void st(V *a, int i, int, float x, float y, float z, float w) {
    a[i] = make_float4(x, y, z, w);
  }
  static __device__ __forceinline__ float *comp(V *a, int i, int, int c) {
    return reinterpret_cast<float *>(a + i) + c;
  }
};

template <>
struct SRec<double> {
  using V = double2;
  static constexpr int kPlanes = 2;
  static __device__ __forceinline__ Q4<double> ld(const V *a, int i, int n) {
    const double2 lo = a[i], hi = a[i + n];
    return Q4<double>{lo.x, lo.y, hi.x, hi.y};
  }
  static __device__ __forceinline__ void st(V *a, int i, int n, double x, double y, double z,
                                            double w) {
    a[i] = make_double2(x, y);
    a[i + n] = make_double2(z, w);
  }
  static __device__ __forceinline__ double *comp(V *a, int i, int n, int c) {
    return reinterpret_cast<double *>(a + i + (c >> 1) * n) + (c & 1);
  }
};

// One face of the stencil region: cells rL1 | rR1 (rL2, rR2 one further
// out), slope records sL, sR; dir 0 = x (normal u), 1 = y (normal v).
// Reconstructed left/right states of one face; false (states set to a
// benign 1) when the face carries no flux.
template <typename R, int LIM, int NQ, int NS>
__device__ __forceinline__ bool face_recon(const typename SRec<R>::V *sq, const uint8_t *sfl,
                                           const typename SRec<R>::V *sl, int rL1, int rR1,
                                           int step, int sL, int sR, bool uni, R (&ls)[4],
                                           R (&rs)[4]) {
  using S = SRec<R>;
  bool active = true, hasL2 = true, hasR2 = true;
  if (!uni) {
    const uint8_t fL = sfl[rL1], fR = sfl[rR1];
    active = (fL & CF_PRESENT) && (fR & CF_PRESENT) && ((fL | fR) & CF_NORMAL);
    hasL2 = (sfl[rL1 - step] & CF_PRESENT) != 0;
    hasR2 = (sfl[rR1 + step] & CF_PRESENT) != 0;
  }
  if (!active) {
#pragma unroll
    for (int c = 0; c < 4; ++c) ls[c] = rs[c] = R(1);
    return false;
  }
  const Q4<R> cL = S::ld(sq, rL1, NQ), cR = S::ld(sq, rR1, NQ);
  if (hasL2) {
    const Q4<R> s = S::ld(sl, sL, NS);
    ls[0] = cL.x + s.x; ls[1] = cL.y + s.y; ls[2] = cL.z + s.z; ls[3] = cL.w + s.w;
  } else {
    const Q4<R> o = S::ld(sq, rR1 + step, NQ);
    ls[0] = muscl_left_fast<LIM>(o.x, cL.x, cR.x);
    ls[1] = muscl_left_fast<LIM>(o.y, cL.y, cR.y);
    ls[2] = muscl_left_fast<LIM>(o.z, cL.z, cR.z);
    ls[3] = muscl_left_fast<LIM>(o.w, cL.w, cR.w);
  }
  if (hasR2) {
    const Q4<R> s = S::ld(sl, sR, NS);
    rs[0] = cR.x - s.x; rs[1] = cR.y - s.y; rs[2] = cR.z - s.z; rs[3] = cR.w - s.w;
  } else {
    const Q4<R> o = S::ld(sq, rL1 - step, NQ);
    rs[0] = muscl_right_fast<LIM>(cL.x, cR.x, o.x);
    rs[1] = muscl_right_fast<LIM>(cL.y, cR.y, o.y);
    rs[2] = muscl_right_fast<LIM>(cL.z, cR.z, o.z);
    rs[3] = muscl_right_fast<LIM>(cL.w, cR.w, o.w);
  }
  return true;
}

template <typename R, int LIM, int NQ, int NS>
__device__ __forceinline__ Q4<R> fast_face(const typename SRec<R>::V *sq, const uint8_t *sfl,
                                           const typename SRec<R>::V *sl, int rL1, int rR1, int step,
                                           int sL, int sR, bool xdir, bool uni, const Gas<R> &g,
                                           R area, R halfarea) {
  R ls[4], rs[4];
  Q4<R> out = {R(0), R(0), R(0), R(0)};
  if (!face_recon<R, LIM, NQ, NS>(sq, sfl, sl, rL1, rR1, step, sL, sR, uni, ls, rs)) return out;
  // normal / tangential velocity by selection (one flux evaluation even
  // when the lanes of a warp mix x- and y-faces)
  R fm, fn, ft, fe;
  const R lun = xdir ? ls[1] : ls[2], lut = xdir ? ls[2] : ls[1];
  const R run = xdir ? rs[1] : rs[2], rut = xdir ? rs[2] : rs[1];
  roe_flux_states<R>(g, area, halfarea, ls[0], lun, lut, ls[3], rs[0], run, rut, rs[3], fm, fn,
                     ft, fe);
  out = Q4<R>{fm, xdir ? fn : ft, xdir ? ft : fn, fe};
  return out;
}

// Limited slopes of one cell in one direction (zero where a neighbour is
// missing; such faces take the one-sided reconstruction instead).
template <typename R, int LIM, int NQ, int NS>
__device__ __forceinline__ void fast_slope(const typename SRec<R>::V *sq, const uint8_t *sfl,
                                           typename SRec<R>::V *sl, int di, int rc, int step,
                                           bool uni) {
  using S = SRec<R>;
  R s0 = R(0), s1 = R(0), s2 = R(0), s3 = R(0);
  if (uni || ((sfl[rc - step] & CF_PRESENT) && (sfl[rc + step] & CF_PRESENT))) {
    const Q4<R> m = S::ld(sq, rc - step, NQ), c = S::ld(sq, rc, NQ), p = S::ld(sq, rc + step, NQ);
    s0 = limited_slope<LIM>(c.x - m.x, p.x - c.x);
    s1 = limited_slope<LIM>(c.y - m.y, p.y - c.y);
    s2 = limited_slope<LIM>(c.z - m.z, p.z - c.z);
    s3 = limited_slope<LIM>(c.w - m.w, p.w - c.w);
  }
  S::st(sl, di, NS, s0, s1, s2, s3);
}

// Fast build of the stage (FP64 with FastMath divisions/roots, or FP32 flux
// arithmetic for the mixed mode): per-cell limited slopes computed once and
// shared by the cell's two faces in each direction, divisions replaced by
// reciprocals, cell and face records in shared memory as 128-bit vectors,
// fixed thread-to-cell/face mapping (thread (tx, ty) owns the slopes and the
// west/south faces of cell (tx, ty); one warp adds the east/north edge).
// Faces whose outer stencil cell is missing use the reference's one-sided
// reconstruction (NS_Solver.H:743-750).  The residual, update and primitive
// recovery run in FP64 in every mode.
// NT: threads of the CTA, 256 (edge faces on the first two warps) or 288
// (a ninth warp owns them); the same arithmetic either way.
template <typename R, int LIM, bool VISC, bool FINAL, typename TI,
          int NT = StageThreads<R>::value>
__device__ __forceinline__ void stage_tile_fast(const StageArgs &a, const StageVar &v,
                                                const CaseConst &cc,
                                                const int tile, const int phase,
                                                const int fold, const int prefetch) {
  constexpr int kSX = kTile + 2;  // x-slope row length (cols -1..16)
  using S = SRec<R>;
  using V = typename S::V;
  constexpr int NQ = kReg * kReg, NS = kTile * kSX, NF = kTile * (kTile + 1);
  __shared__ V sq[S::kPlanes * NQ];
  __shared__ uint8_t sfl[NQ];
  __shared__ V slx[S::kPlanes * NS];  // rows 0..15, cols -1..16
  __shared__ V sly[S::kPlanes * NS];  // rows -1..16, cols 0..15
  __shared__ V fx[S::kPlanes * NF];   // x-face (i, j) at j*17 + i
  __shared__ V fy[S::kPlanes * NF];   // y-face (i, j) at j*16 + i

  static_assert(NT == kTileCells || NT == kTileCells + 32, "256 or 288 threads");
  const int tid = threadIdx.x;
  const int tx = tid & (kTile - 1), ty = (NT > kTileCells) ? ((tid >> 4) & (kTile - 1)) : (tid >> 4);
  // a cell of the tile (the ninth warp owns none)
  const bool own = (NT > kTileCells) ? tid < kTileCells : true;
  const int lvl = a.tile_level[tile];
  const LevelConst &L = cc.lev[lvl];
  // uniform tile: it and its four side neighbours hold only leaf cells that
  // recover their primitives, so no presence flags or one-sided stencils
  const bool uni = a.tile_uniform != nullptr && a.tile_uniform[tile] != 0;

  // side neighbours (the centre entry of the table is the tile itself),
  // loaded beside the tile's level and uniform flag so the region's loads
  // below wait for one round trip, not one per neighbour lookup
  const int32_t *nbrow = a.tile_nb + (int64_t)tile * 9;
  const int nbs = __ldg(nbrow + 1), nbw = __ldg(nbrow + 3), nbe = __ldg(nbrow + 5),
            nbn = __ldg(nbrow + 7);

  {
    // U^n of the tile's own cells, which the update phase reads after the
    // faces, into L1 now (FP64 step 0.798 -> 0.779 ms)
    if (tid < 64) {
      const int fld = tid >> 4;
      const double *un = a.s0[fld == 0 ? F_RHO : (fld == 1 ? F_U : (fld == 2 ? F_V : F_E))];
      asm volatile("prefetch.global.L1 [%0];" ::"l"(un + (int64_t)tile * kTileCells + (tid & 15) * 16));
    }
  }
  if (prefetch > 0) {
    // the CTA that starts when this one ends reads this tile's input from L2
    constexpr int kLines = kTileCells * (int)sizeof(TI) / 128;  // 128-byte lines per field
    const int64_t pt = (int64_t)(tile + prefetch) * kTileCells;
    if (tid < 4 * kLines && pt < a.nslots)
      asm volatile("prefetch.global.L2 [%0];" ::"l"(static_cast<const TI *>(v.sin[tid / kLines]) + pt +
                                                    (tid % kLines) * (128 / (int)sizeof(TI))));
  }

  if (uni) {
    // one region record per thread and pass: its four fields loaded (all
    // loads of both passes issued before the first store), then one record
    // store (no shared-memory bank conflicts); corners stay unset (a
    // uniform tile's stencils never read them)
    constexpr int NIT = (kReg * kReg + NT - 1) / NT;
    const TI *in0 = static_cast<const TI *>(v.sin[0]), *in1 = static_cast<const TI *>(v.sin[1]),
             *in2 = static_cast<const TI *>(v.sin[2]), *in3 = static_cast<const TI *>(v.sin[3]);
    R q[NIT][4];
    bool has[NIT];
#pragma unroll
    for (int it = 0; it < NIT; ++it) {
      const int r = tid + it * NT;
      const int rx = r % kReg - kHalo, ry = r / kReg - kHalo;
      const int ox = rx < 0 ? -1 : (rx >= kTile ? 1 : 0);
      const int oy = ry < 0 ? -1 : (ry >= kTile ? 1 : 0);
      has[it] = r < kReg * kReg && !(ox && oy);
      if (has[it]) {
        const int nb = ox < 0 ? nbw : (ox > 0 ? nbe : (oy < 0 ? nbs : (oy > 0 ? nbn : tile)));
        const int64_t sl = (int64_t)nb * kTileCells + (ry - oy * kTile) * kTile + (rx - ox * kTile);
        q[it][0] = (R)__ldg(in0 + sl);
        q[it][1] = (R)__ldg(in1 + sl);
        q[it][2] = (R)__ldg(in2 + sl);
        q[it][3] = (R)__ldg(in3 + sl);
      }
    }
#pragma unroll
    for (int it = 0; it < NIT; ++it)
      if (has[it]) S::st(sq, tid + it * NT, NQ, q[it][0], q[it][1], q[it][2], q[it][3]);
  } else {
    // region records: slot, then presence flags, then the state, each
    // step's loads of both records issued together
    constexpr int NIT = (kReg * kReg + NT - 1) / NT;
    int64_t sl[NIT];
    uint8_t fl[NIT];
#pragma unroll
    for (int it = 0; it < NIT; ++it) {
      const int r = tid + it * NT;
      sl[it] = -1;
      if (r < kReg * kReg) {
        const int rx = r % kReg - kHalo, ry = r / kReg - kHalo;
        const int ox = rx < 0 ? -1 : (rx >= kTile ? 1 : 0);
        const int oy = ry < 0 ? -1 : (ry >= kTile ? 1 : 0);
        if (!(ox && oy)) {
          const int nb = ox < 0 ? nbw : (ox > 0 ? nbe : (oy < 0 ? nbs : (oy > 0 ? nbn : tile)));
          if (nb >= 0) sl[it] = (int64_t)nb * kTileCells + (ry - oy * kTile) * kTile + (rx - ox * kTile);
        }
      }
    }
#pragma unroll
    for (int it = 0; it < NIT; ++it) fl[it] = sl[it] >= 0 ? a.flags[sl[it]] : uint8_t(0);
#pragma unroll
    for (int it = 0; it < NIT; ++it) {
      const int r = tid + it * NT;
      if (r < kReg * kReg) {
        R q0 = R(0), q1 = R(0), q2 = R(0), q3 = R(0);
        if (fl[it] & CF_PRESENT) {
          const int64_t s = sl[it];
          const bool varying = (fl[it] & (CF_PRIM | CF_RESET)) != 0;
          if (varying) {
            q0 = (R) static_cast<const TI *>(v.sin[0])[s];
            q1 = (R) static_cast<const TI *>(v.sin[1])[s];
            q2 = (R) static_cast<const TI *>(v.sin[2])[s];
            q3 = (R) static_cast<const TI *>(v.sin[3])[s];
          } else {
            q0 = (R)a.s0[F_RHO][s];
            q1 = (R)a.s0[F_U][s];
            q2 = (R)a.s0[F_V][s];
            q3 = (R)a.s0[F_P][s];
          }
        }
        sfl[r] = fl[it];
        S::st(sq, r, NQ, q0, q1, q2, q3);
      }
    }
  }
  __syncthreads();

  // ---- per-cell limited slopes: (tx, ty) in both directions, then the
  //      two outer columns (x) and rows (y) of the face stencils
  if (NT > kTileCells) {
    if (own) {
      const int rc = (ty + kHalo) * kReg + (tx + kHalo);
      fast_slope<R, LIM, NQ, NS>(sq, sfl, slx, ty * kSX + tx + 1, rc, 1, uni);
      fast_slope<R, LIM, NQ, NS>(sq, sfl, sly, (ty + 1) * kTile + tx, rc, kReg, uni);
    } else {
      // ninth warp: one outer x-slope (columns -1, 16) and one outer
      // y-slope (rows -1, 16) per lane
      const int e = (tid - kTileCells) & 15, hi = (tid - kTileCells) >= 16;
      const int col = hi ? kTile : -1;
      fast_slope<R, LIM, NQ, NS>(sq, sfl, slx, e * kSX + col + 1, (e + kHalo) * kReg + col + kHalo,
                                 1, uni);
      const int row = hi ? kTile : -1;
      fast_slope<R, LIM, NQ, NS>(sq, sfl, sly, (row + 1) * kTile + e,
                                 (row + kHalo) * kReg + e + kHalo, kReg, uni);
    }
  } else {
    const int rc = (ty + kHalo) * kReg + (tx + kHalo);
    fast_slope<R, LIM, NQ, NS>(sq, sfl, slx, ty * kSX + tx + 1, rc, 1, uni);
    fast_slope<R, LIM, NQ, NS>(sq, sfl, sly, (ty + 1) * kTile + tx, rc, kReg, uni);
    if (tid < 64) {
      const int e = tid & 15;
      if (tid < 32) {
        const int col = (tid < 16) ? -1 : kTile;
        fast_slope<R, LIM, NQ, NS>(sq, sfl, slx, e * kSX + col + 1, (e + kHalo) * kReg + col + kHalo,
                                   1, uni);
      } else {
        const int row = (tid < 48) ? -1 : kTile;
        fast_slope<R, LIM, NQ, NS>(sq, sfl, sly, (row + 1) * kTile + e,
                                   (row + kHalo) * kReg + e + kHalo, kReg, uni);
      }
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
  g.gam_gm1 = (R)(cc.gama / cc.gm1);
  g.two_gama = (R)(2.0 * cc.gama);
  const R ax = (R)L.area_x, ay = (R)L.area_y;
  const R hax = R(0.5) * ax, hay = R(0.5) * ay;

  // ---- face fluxes: west x-face and south y-face of cell (tx, ty), plus the
  //      east column (threads 0..15) and north row (threads 16..31)
  {
    const int rR1 = (ty + kHalo) * kReg + (tx + kHalo);
    Q4<R> o;
    if (!own) {
      // ninth warp: edge faces only (below)
    } else if constexpr (kPairFaces<R>) {
      // the cell's west and south faces as the two lanes of one paired flux
      // evaluation (f32x2 instructions in the mixed build)
      R lx[4], rx[4], ly[4], ry[4];
      const bool ax_ok = face_recon<R, LIM, NQ, NS>(sq, sfl, slx, rR1 - 1, rR1, 1, ty * kSX + tx,
                                                   ty * kSX + tx + 1, uni, lx, rx);
      const bool ay_ok = face_recon<R, LIM, NQ, NS>(sq, sfl, sly, rR1 - kReg, rR1, kReg,
                                                   ty * kTile + tx, (ty + 1) * kTile + tx, uni, ly,
                                                   ry);
      using P = decltype(pair(R(0), R(0)));
      P fm, fn, ft, fe;
      roe_flux_pair<P, R>(g, pair(ax, ay), pair(lx[0], ly[0]), pair(lx[1], ly[2]),
                          pair(lx[2], ly[1]), pair(lx[3], ly[3]), pair(rx[0], ry[0]),
                          pair(rx[1], ry[2]), pair(rx[2], ry[1]), pair(rx[3], ry[3]), fm, fn, ft,
                          fe);
      if (ax_ok) S::st(fx, ty * (kTile + 1) + tx, NF, lane0(fm), lane0(fn), lane0(ft), lane0(fe));
      else S::st(fx, ty * (kTile + 1) + tx, NF, R(0), R(0), R(0), R(0));
      if (ay_ok) S::st(fy, ty * kTile + tx, NF, lane1(fm), lane1(ft), lane1(fn), lane1(fe));
      else S::st(fy, ty * kTile + tx, NF, R(0), R(0), R(0), R(0));
    } else {
      o = fast_face<R, LIM, NQ, NS>(sq, sfl, slx, rR1 - 1, rR1, 1, ty * kSX + tx,
                                    ty * kSX + tx + 1, true, uni, g, ax, hax);
      S::st(fx, ty * (kTile + 1) + tx, NF, o.x, o.y, o.z, o.w);
      o = fast_face<R, LIM, NQ, NS>(sq, sfl, sly, rR1 - kReg, rR1, kReg, ty * kTile + tx,
                                    (ty + 1) * kTile + tx, false, uni, g, ay, hay);
      S::st(fy, ty * kTile + tx, NF, o.x, o.y, o.z, o.w);
    }
    const int et = tid - (NT > kTileCells ? kTileCells : 0);
    if (et >= 0 && et < 32) {
      // east column (lanes 0..15) and north row (lanes 16..31) through one
      // call site, so the warp evaluates the flux once
      const int e = et & 15;
      const bool xd = et < 16;
      const int r = xd ? (e + kHalo) * kReg + kTile + kHalo : (kTile + kHalo) * kReg + e + kHalo;
      const int step = xd ? 1 : kReg;
      const int sL = xd ? e * kSX + kTile : kTile * kTile + e;
      const int sR = xd ? e * kSX + kTile + 1 : (kTile + 1) * kTile + e;
      o = fast_face<R, LIM, NQ, NS>(sq, sfl, xd ? slx : sly, r - step, r, step, sL, sR, xd, uni,
                                    g, xd ? ax : ay, xd ? hax : hay);
      S::st(xd ? fx : fy, xd ? e * (kTile + 1) + kTile : kTile * kTile + e, NF, o.x, o.y, o.z, o.w);
    }
  }
  __syncthreads();

  // ---- residual, update, primitive recovery (FP64)
  const int64_t slot = (int64_t)tile * kTileCells + tid;
  const uint8_t fl = !own ? (uint8_t)0
                         : uni ? (uint8_t)(CF_PRESENT | CF_NORMAL | CF_UPDATE | CF_PRIM | CF_RESNORM)
                               : sfl[(ty + kHalo) * kReg + (tx + kHalo)];
  unsigned long long rb[4] = {0ull, 0ull, 0ull, 0ull};
  double cb = -1.0;  // next step's CFL bound of this cell, when this stage writes it
  if ((fl & CF_NORMAL) && (fl & (CF_UPDATE | CF_RESET))) {
    const Q4<R> fxl = S::ld(fx, ty * (kTile + 1) + tx, NF), fxh = S::ld(fx, ty * (kTile + 1) + tx + 1, NF);
    const Q4<R> fyl = S::ld(fy, ty * kTile + tx, NF), fyh = S::ld(fy, (ty + 1) * kTile + tx, NF);
    double res[4];
    const R sxl[4] = {fxl.x, fxl.y, fxl.z, fxl.w}, sxh[4] = {fxh.x, fxh.y, fxh.z, fxh.w};
    const R syl[4] = {fyl.x, fyl.y, fyl.z, fyl.w}, syh[4] = {fyh.x, fyh.y, fyh.z, fyh.w};
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      if (sizeof(R) == 4 && !VISC) {
        // mixed build: face differences in FP32 (the fluxes are FP32), one
        // conversion per component
        res[c] = (double)((sxl[c] - sxh[c]) + (syl[c] - syh[c]));
      } else {
        double sx = (sizeof(R) == 4) ? (double)(sxl[c] - sxh[c]) : (double)sxl[c] - (double)sxh[c];
        double sy = (sizeof(R) == 4) ? (double)(syl[c] - syh[c]) : (double)syl[c] - (double)syh[c];
        if (VISC) {
          sx += a.vsd[(int64_t)c * a.nslots + slot];
          sy += a.vsd[(int64_t)(4 + c) * a.nslots + slot];
        }
        res[c] = sx + sy;
      }
    }
    const double dt = a.diag->dt;
    const double scale = (v.tp * dt) * L.step_num * L.inv_vol;
    double nrho, nu, nv, np, ne, nT;
    bool wrote = false;
    if (fl & CF_UPDATE) {
      const double orho = a.s0[F_RHO][slot], ou = a.s0[F_U][slot], ov = a.s0[F_V][slot],
                   oe = a.s0[F_E][slot];
      const double cv0 = orho + res[0] * scale;
      const double cv1 = orho * ou + res[1] * scale;
      const double cv2 = orho * ov + res[2] * scale;
      const double cv3 = orho * oe + res[3] * scale;
      if (cv0 < 0.0) raise_error(a.diag, phase, ERR_NEG_RHO, (int)slot);
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
      if (nT < 0.0) raise_error(a.diag, phase, ERR_NEG_T, (int)slot);
      if (FINAL) {
        a.s0[F_RHO][slot] = nrho;
        a.s0[F_U][slot] = nu;
        a.s0[F_V][slot] = nv;
        a.s0[F_P][slot] = np;
        a.s0[F_E][slot] = ne;
        a.s0[F_T][slot] = nT;
      } else {
        // stage buffers in the arithmetic's precision (FP32 in the mixed build)
        typedef R TO;
        static_cast<TO *>(v.sout[0])[slot] = (TO)nrho;
        static_cast<TO *>(v.sout[1])[slot] = (TO)nu;
        static_cast<TO *>(v.sout[2])[slot] = (TO)nv;
        static_cast<TO *>(v.sout[3])[slot] = (TO)np;
      }
    }
    if (FINAL && (fl & CF_RESNORM)) {
#pragma unroll
      for (int c = 0; c < 4; ++c) rb[c] = (unsigned long long)__double_as_longlong(fabs(res[c]));
    }
    if (FINAL && fold && wrote) cb = cfl_cell_bound(nT, nu, nv, L, cc);
  }
  // the y-slope records are dead after the face phase: reuse them
  if (FINAL) {
    unsigned long long *sred = reinterpret_cast<unsigned long long *>(sly);
    block_resnorm<NT>(rb, a.diag, sred);
    if (fold) fold_next_cfl<NT>(a, L, cc, fl, slot, cb, sred, fold - 1, own);
  }
}

// TI: element type of the stage input (the FP64 step state for the first
// stage; the stage buffers, R, after it)
template <typename R, int LIM, bool VISC, bool FINAL, typename TI>
__global__ void __launch_bounds__(StageThreads<R>::value, sizeof(R) == 8 ? 4 : 6)
    stage_kernel_fast(StageArgs a, CaseConst cc) {
  stage_tile_fast<R, LIM, VISC, FINAL, TI>(a, a.v, cc, a.tile_begin + blockIdx.x, a.phase,
                                           a.v.cfl_next, a.prefetch);
}


#ifdef IBGPU_FAST_BUILD
// Constant-memory table of batched stage arguments.  A batch that fits keeps
// here, per case, its stage arguments up to the stage-dependent part
// (kStageCommonBytes), one StageVar per stage and its CaseConst up to its
// finest level, found through a per-batch header of one int4 per case
// (byte offsets of the three; w unused).  Read with a CTA-uniform index,
// these are constant-bank operands like a single-case launch's parameters,
// which keeps the batched tile body's registers, spills and argument loads
// at the single-case kernel's level.
constexpr int kBatchTableBytes = 60 * 1024;
__constant__ __align__(16) unsigned char c_batch_table[kBatchTableBytes];
#endif

// Batched stage over a work list of (case, tile) pairs of several
// independent cases (each its own mesh, state and constants).  TABLE: the
// case's arguments come from the constant-memory table, header at byte
// offset `table` (fast builds only); otherwise the stage's arguments of case
// c are args[c * nstages + stage] and its constants ccs[c] in global memory.
// phase_base holds 8 x the step's index within the run (abort ordering),
// written on the device so a captured graph can replay the launch for every
// step.  LOOP: persistent CTAs striding over the list; otherwise one CTA per
// item (no loop state, which keeps the tile body's register spills at the
// single-case kernel's level).
template <typename R, int LIM, bool VISC, bool FINAL, bool LOOP, bool TABLE, typename TI, int NT>
__global__ void __launch_bounds__(NT, stage_min_blocks<R, NT>())
    stage_kernel_batch(const StageArgs *__restrict__ args, const CaseConst *__restrict__ ccs,
                       const int2 *__restrict__ work, int nwork, int stage, int nstages,
                       const int *__restrict__ phase_base, int table) {
  // phase_base[0]: 8 x the step index; phase_base[1]: 1 when this step's
  // final stage folds in the next step's CFL pass of the cases that allow it
  const int pb = phase_base[0], fold_step = phase_base[1];
  for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
    const int2 it = work[w];
#ifdef IBGPU_FAST_BUILD
    if (TABLE) {
      const int4 h = reinterpret_cast<const int4 *>(c_batch_table + table)[it.x];
      const StageArgs &a = *reinterpret_cast<const StageArgs *>(c_batch_table + h.x);
      const StageVar &v = reinterpret_cast<const StageVar *>(c_batch_table + h.y)[stage];
      const CaseConst &cc = *reinterpret_cast<const CaseConst *>(c_batch_table + h.z);
      const int fold = (FINAL && fold_step && v.cfl_next) ? 1 + pb + 8 + 1 : 0;
      stage_tile_fast<R, LIM, VISC, FINAL, TI, NT>(a, v, cc, it.y, pb + 2 + stage, fold, 0);
    } else
#endif
    {
      const StageArgs &a = args[it.x * nstages + stage];
      const int fold = (FINAL && fold_step && a.v.cfl_next) ? 1 + pb + 8 + 1 : 0;
      stage_tile_fast<R, LIM, VISC, FINAL, TI, NT>(a, a.v, ccs[it.x], it.y, pb + 2 + stage, fold, 0);
    }
    if (!LOOP) break;
    __syncthreads();  // shared-memory reuse by the next work item
  }
}

// CFL time step over the normal cells of every level, NS_Solver::Comptdt
// (NS_Solver.cpp:196-280): a per-cell bound, a warp-shuffle and block min and
// one atomic per block (positive doubles order like their bit patterns).
__global__ void __launch_bounds__(256) cfl_kernel(CflArgs a, CaseConst cc) {
  double best = 10000.0;
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < a.nslots;
       s += (int64_t)gridDim.x * blockDim.x) {
    if (!(a.flags[s] & CF_NORMAL)) continue;
    const LevelConst &L = cc.lev[a.tile_level[s / kTileCells]];
    const double d0 = cfl_cell_bound(a.s0[F_T][s], a.s0[F_U][s], a.s0[F_V][s], L, cc);
    if (d0 < 0.0) raise_error(a.diag, a.phase, ERR_CFL_NEG_DT, (int)s);
    best = (d0 < best) ? d0 : best;  // std::min(CFL_dt, CFL_dt0) ignores NaN
  }
  unsigned long long b = warp_min_u64((unsigned long long)__double_as_longlong(best));
  // block minimum, then one atomic per block (result unused: not waited for)
  __shared__ unsigned long long sred[8];
  if ((threadIdx.x & 31) == 0) sred[threadIdx.x >> 5] = b;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) b = sred[w] < b ? sred[w] : b;
    atomicMin(&a.diag->cfl_bits, b);
  }
}

// Per-step reset of the step's reductions (the dt and any earlier abort
// carry over between the steps of one run).
__global__ void step_begin_kernel(DevDiag *d) {
  d->cfl_bits = (unsigned long long)__double_as_longlong(10000.0);
  for (int c = 0; c < 5; ++c) d->res_bits[c] = 0ull;
}

// dt = min(CFL_dt, dt*dt_ratio) (NS_Solver.cpp:263)
__global__ void finalize_dt_kernel(DevDiag *d, CaseConst cc) {
  double cdt = __longlong_as_double((long long)d->cfl_bits);
  double cand = d->dt * cc.dt_ratio;
  d->dt = (cand < cdt) ? cand : cdt;
}

// The CFL pass of a step whose bound the previous step's final stage
// accumulated (cfl_next_bits): take it, reset the accumulator for this
// step's final stage, and finalise dt.
__global__ void take_folded_cfl_kernel(DevDiag *d, CaseConst cc) {
  d->cfl_bits = d->cfl_next_bits;
  d->cfl_next_bits = (unsigned long long)__double_as_longlong(10000.0);
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

// Compact rows (roe, u, v, p): the remaining fields as the reference derives
// them from those four (Get_T_ideal_gas T = p / (roe Rg), Get_E e = Cv T +
// |u|^2 / 2 with w = 0, FlowVariables.H:19-33), rounded operation by
// operation (no contraction).
__global__ void scatter_state4_kernel(const double *rows, const int32_t *cell_slot,
                                      const uint8_t *cell_is_alias, int64_t n, double Rg,
                                      double Cv, double *s0_rho, double *s0_u, double *s0_v,
                                      double *s0_p, double *s0_e, double *s0_T) {
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x) {
    if (cell_is_alias[c]) continue;
    int64_t s = cell_slot[c];
    const double *r = rows + 4 * c;
    const double roe = r[0], u = r[1], v = r[2], p = r[3];
    const double T = __ddiv_rn(p, __dmul_rn(roe, Rg));
    const double k = __dmul_rn(0.5, __dadd_rn(__dadd_rn(__dmul_rn(u, u), __dmul_rn(v, v)), 0.0));
    s0_rho[s] = roe;
    s0_u[s] = u;
    s0_v[s] = v;
    s0_p[s] = p;
    s0_T[s] = T;
    s0_e[s] = __dadd_rn(__dmul_rn(Cv, T), k);
  }
}

__global__ void gather_state4_kernel(double *rows, const int32_t *cell_slot, int64_t n,
                                     const double *s0_rho, const double *s0_u,
                                     const double *s0_v, const double *s0_p) {
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x) {
    int64_t s = cell_slot[c];
    double *r = rows + 4 * c;
    r[0] = s0_rho[s];
    r[1] = s0_u[s];
    r[2] = s0_v[s];
    r[3] = s0_p[s];
  }
}

// ---- launchers (one set per arithmetic build)


#ifdef IBGPU_FAST_BUILD
template <typename R, int LIM, typename TI>
static void launch_stage_ti(const StageArgs &a, const CaseConst &cc, int ntiles, bool visc,
                            bool final_stage, cudaStream_t st) {
  dim3 grid(ntiles), block(StageThreads<R>::value);
  if (visc) {
    if (final_stage) stage_kernel_fast<R, LIM, true, true, TI><<<grid, block, 0, st>>>(a, cc);
    else stage_kernel_fast<R, LIM, true, false, TI><<<grid, block, 0, st>>>(a, cc);
  } else {
    if (final_stage) stage_kernel_fast<R, LIM, false, true, TI><<<grid, block, 0, st>>>(a, cc);
    else stage_kernel_fast<R, LIM, false, false, TI><<<grid, block, 0, st>>>(a, cc);
  }
}

// in32: the stage input is the mixed build's FP32 stage buffer
template <typename R, int LIM>
static void launch_stage_t(const StageArgs &a, const CaseConst &cc, int ntiles, bool visc,
                           bool final_stage, bool in32, cudaStream_t st) {
  if constexpr (sizeof(R) == 4) {
    if (in32) {
      launch_stage_ti<R, LIM, float>(a, cc, ntiles, visc, final_stage, st);
      return;
    }
  }
  launch_stage_ti<R, LIM, double>(a, cc, ntiles, visc, final_stage, st);
}
#else
template <typename R, int LIM>
static void launch_stage_t(const StageArgs &a, const CaseConst &cc, int ntiles, bool visc,
                           bool final_stage, bool, cudaStream_t st) {
  dim3 grid(ntiles), block(kTileCells);
  if (visc) {
    if (final_stage) stage_kernel<R, LIM, true, true><<<grid, block, 0, st>>>(a, cc);
    else stage_kernel<R, LIM, true, false><<<grid, block, 0, st>>>(a, cc);
  } else {
    if (final_stage) stage_kernel<R, LIM, false, true><<<grid, block, 0, st>>>(a, cc);
    else stage_kernel<R, LIM, false, false><<<grid, block, 0, st>>>(a, cc);
  }
}
#endif

void launch_stage(const StageArgs &a, const CaseConst &cc, int ntiles, int limiter, bool visc,
                  bool final_stage, bool mixed, int stage, cudaStream_t st) {
  if (ntiles <= 0) return;
#ifndef IBGPU_FAST_BUILD
  mixed = false;  // the exact build is FP64 only
#endif
  const bool in32 = mixed && stage > 0;
  if (mixed) {
    if (limiter == LIM_MINMOD) launch_stage_t<float, LIM_MINMOD>(a, cc, ntiles, visc, final_stage, in32, st);
    else launch_stage_t<float, LIM_VANLEER>(a, cc, ntiles, visc, final_stage, in32, st);
  } else {
    if (limiter == LIM_MINMOD) launch_stage_t<double, LIM_MINMOD>(a, cc, ntiles, visc, final_stage, false, st);
    else launch_stage_t<double, LIM_VANLEER>(a, cc, ntiles, visc, final_stage, false, st);
  }
}

#ifdef IBGPU_FAST_BUILD
template <typename R, int LIM, bool LOOP, bool TABLE, typename TI, int NT>
static void launch_batch_n(const StageArgs *args, const CaseConst *ccs, const int2 *work, int nwork,
                           int stage, int nstages, const int *phase_base, bool visc,
                           bool final_stage, int grid, int table, cudaStream_t st) {
  dim3 g(grid), block(NT);
  if (visc) {
    if (final_stage)
      stage_kernel_batch<R, LIM, true, true, LOOP, TABLE, TI, NT><<<g, block, 0, st>>>(args, ccs, work, nwork, stage, nstages, phase_base, table);
    else
      stage_kernel_batch<R, LIM, true, false, LOOP, TABLE, TI, NT><<<g, block, 0, st>>>(args, ccs, work, nwork, stage, nstages, phase_base, table);
  } else {
    if (final_stage)
      stage_kernel_batch<R, LIM, false, true, LOOP, TABLE, TI, NT><<<g, block, 0, st>>>(args, ccs, work, nwork, stage, nstages, phase_base, table);
    else
      stage_kernel_batch<R, LIM, false, false, LOOP, TABLE, TI, NT><<<g, block, 0, st>>>(args, ccs, work, nwork, stage, nstages, phase_base, table);
  }
}

template <typename R, int LIM, bool LOOP, bool TABLE, typename TI>
static void launch_batch_l(const StageArgs *args, const CaseConst *ccs, const int2 *work, int nwork,
                           int stage, int nstages, const int *phase_base, bool visc,
                           bool final_stage, int grid, int threads, int table, cudaStream_t st) {
  if (threads == kTileCells + 32)
    launch_batch_n<R, LIM, LOOP, TABLE, TI, kTileCells + 32>(args, ccs, work, nwork, stage, nstages, phase_base, visc, final_stage, grid, table, st);
  else
    launch_batch_n<R, LIM, LOOP, TABLE, TI, kTileCells>(args, ccs, work, nwork, stage, nstages, phase_base, visc, final_stage, grid, table, st);
}

// stage input element type: the FP64 step state for the first stage, the
// stage buffers (R) after it
template <typename R, int LIM, bool LOOP, bool TABLE>
static void launch_batch_i(const StageArgs *args, const CaseConst *ccs, const int2 *work, int nwork,
                           int stage, int nstages, const int *phase_base, bool visc,
                           bool final_stage, int grid, int threads, int table, cudaStream_t st) {
  if constexpr (sizeof(R) == 4) {
    if (stage > 0) {
      launch_batch_l<R, LIM, LOOP, TABLE, float>(args, ccs, work, nwork, stage, nstages, phase_base, visc, final_stage, grid, threads, table, st);
      return;
    }
  }
  launch_batch_l<R, LIM, LOOP, TABLE, double>(args, ccs, work, nwork, stage, nstages, phase_base, visc, final_stage, grid, threads, table, st);
}

// grid == nwork: one CTA per work item; fewer: persistent CTAs.  table >= 0:
// the arguments come from the constant-memory table.
template <typename R, int LIM>
static void launch_batch_t(const StageArgs *args, const CaseConst *ccs, const int2 *work, int nwork,
                           int stage, int nstages, const int *phase_base, bool visc,
                           bool final_stage, int grid, int threads, int table, cudaStream_t st) {
  const bool loop = grid < nwork;
  if (!loop) grid = nwork;
  if (table >= 0) {
    if (loop) launch_batch_i<R, LIM, true, true>(args, ccs, work, nwork, stage, nstages, phase_base, visc, final_stage, grid, threads, table, st);
    else launch_batch_i<R, LIM, false, true>(args, ccs, work, nwork, stage, nstages, phase_base, visc, final_stage, grid, threads, table, st);
  } else {
    if (loop) launch_batch_i<R, LIM, true, false>(args, ccs, work, nwork, stage, nstages, phase_base, visc, final_stage, grid, threads, -1, st);
    else launch_batch_i<R, LIM, false, false>(args, ccs, work, nwork, stage, nstages, phase_base, visc, final_stage, grid, threads, -1, st);
  }
}

void launch_stage_batch(const StageArgs *args, const CaseConst *ccs, const int2 *work, int nwork,
                        int stage, int nstages, const int *phase_base, int limiter, bool visc,
                        bool final_stage, bool mixed, int grid, int threads, int table,
                        cudaStream_t st) {
  if (nwork <= 0) return;
  if (grid < 1 || grid > nwork) grid = nwork;
  if (table >= kBatchTableBytes) table = -1;
  if (threads != kTileCells && threads != kTileCells + 32)
    threads = mixed ? StageThreads<float>::value : StageThreads<double>::value;
  if (mixed) {
    if (limiter == LIM_MINMOD) launch_batch_t<float, LIM_MINMOD>(args, ccs, work, nwork, stage, nstages, phase_base, visc, final_stage, grid, threads, table, st);
    else launch_batch_t<float, LIM_VANLEER>(args, ccs, work, nwork, stage, nstages, phase_base, visc, final_stage, grid, threads, table, st);
  } else {
    if (limiter == LIM_MINMOD) launch_batch_t<double, LIM_MINMOD>(args, ccs, work, nwork, stage, nstages, phase_base, visc, final_stage, grid, threads, table, st);
    else launch_batch_t<double, LIM_VANLEER>(args, ccs, work, nwork, stage, nstages, phase_base, visc, final_stage, grid, threads, table, st);
  }
}

// ---- constant-memory table: first-fit byte ranges per device
namespace {
std::mutex g_table_mu;
std::map<int, std::map<int, int>> g_table_used;  // device -> (offset -> bytes)
}  // namespace

int batch_table_reserve(int device, int bytes) {
  if (bytes <= 0 || bytes > kBatchTableBytes) return -1;
  bytes = (bytes + 15) & ~15;
  std::lock_guard<std::mutex> lk(g_table_mu);
  std::map<int, int> &used = g_table_used[device];
  int at = 0;
  for (const auto &r : used) {
    if (r.first - at >= bytes) break;
    at = r.first + r.second;
  }
  if (at + bytes > kBatchTableBytes) return -1;
  used[at] = bytes;
  return at;
}

void batch_table_release(int device, int offset) {
  if (offset < 0) return;
  std::lock_guard<std::mutex> lk(g_table_mu);
  auto d = g_table_used.find(device);
  if (d != g_table_used.end()) d->second.erase(offset);
}

cudaError_t batch_table_write(int offset, const void *src, int bytes) {
  if (offset < 0 || bytes < 0 || offset + bytes > kBatchTableBytes) return cudaErrorInvalidValue;
  return cudaMemcpyToSymbol(c_batch_table, src, (size_t)bytes, (size_t)offset,
                            cudaMemcpyHostToDevice);
}

// CFL pass of every batched case in one launch: one CTA per (case, tile)
// item of all tiles, the same per-cell bound as cfl_kernel, block minimum and
// one atomic (not waited for) into the case's diag.
__global__ void __launch_bounds__(kTileCells)
    cfl_kernel_batch(const StageArgs *__restrict__ args, const CaseConst *__restrict__ ccs,
                     const int2 *__restrict__ work, int nwork, int nstages,
                     const int *__restrict__ phase_base) {
  __shared__ unsigned long long sred[kTileCells / 32];
  const int pb = *phase_base;
  for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
    const int2 it = work[w];
    const StageArgs &a = args[it.x * nstages];
    const CaseConst &cc = ccs[it.x];
    const int64_t s = (int64_t)it.y * kTileCells + threadIdx.x;
    double best = 10000.0;
    if (a.flags[s] & CF_NORMAL) {
      const LevelConst &L = cc.lev[a.tile_level[it.y]];
      const double d0 = cfl_cell_bound(a.s0[F_T][s], a.s0[F_U][s], a.s0[F_V][s], L, cc);
      if (d0 < 0.0) raise_error(a.diag, pb + 1, ERR_CFL_NEG_DT, (int)s);
      best = (d0 < best) ? d0 : best;
    }
    unsigned long long b = warp_min_u64((unsigned long long)__double_as_longlong(best));
    if ((threadIdx.x & 31) == 0) sred[threadIdx.x >> 5] = b;
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int k = 1; k < kTileCells / 32; ++k) b = sred[k] < b ? sred[k] : b;
      atomicMin(&a.diag->cfl_bits, b);
    }
    __syncthreads();
  }
}

// dt = min(CFL_dt, dt*dt_ratio) of every batched case (one thread each)
__global__ void finalize_dt_batch(const StageArgs *__restrict__ args,
                                  const CaseConst *__restrict__ ccs, int ncases, int nstages) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncases) return;
  DevDiag *d = args[c * nstages].diag;
  double cdt = __longlong_as_double((long long)d->cfl_bits);
  double cand = d->dt * ccs[c].dt_ratio;
  d->dt = (cand < cdt) ? cand : cdt;
}

// the CFL bound each batched case's previous final stage accumulated
__global__ void take_folded_batch(const StageArgs *__restrict__ args,
                                  const CaseConst *__restrict__ ccs, int ncases, int nstages) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncases) return;
  DevDiag *d = args[c * nstages].diag;
  d->cfl_bits = d->cfl_next_bits;
  d->cfl_next_bits = (unsigned long long)__double_as_longlong(10000.0);
  double cdt = __longlong_as_double((long long)d->cfl_bits);
  double cand = d->dt * ccs[c].dt_ratio;
  d->dt = (cand < cdt) ? cand : cdt;
}
void launch_take_folded_batch(const StageArgs *args, const CaseConst *ccs, int ncases, int nstages,
                              cudaStream_t st) {
  take_folded_batch<<<(ncases + 127) / 128, 128, 0, st>>>(args, ccs, ncases, nstages);
}

// per-step reset of the reductions of every batched case
__global__ void step_begin_batch(const StageArgs *__restrict__ args, int ncases, int nstages) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncases) return;
  DevDiag *d = args[c * nstages].diag;
  d->cfl_bits = (unsigned long long)__double_as_longlong(10000.0);
  for (int k = 0; k < 5; ++k) d->res_bits[k] = 0ull;
}

// dt of the listed batched cases only (the cases whose CFL pass ran)
__global__ void finalize_dt_batch_list(const StageArgs *__restrict__ args,
                                       const CaseConst *__restrict__ ccs,
                                       const int *__restrict__ list, int n, int nstages) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int c = list[k];
  DevDiag *d = args[c * nstages].diag;
  double cdt = __longlong_as_double((long long)d->cfl_bits);
  double cand = d->dt * ccs[c].dt_ratio;
  d->dt = (cand < cdt) ? cand : cdt;
}

void launch_cfl_batch(const StageArgs *args, const CaseConst *ccs, const int2 *work, int nwork,
                      int nstages, const int *phase_base, int ncases, int grid, cudaStream_t st,
                      const int *case_list) {
  if (nwork > 0) {
    if (grid < 1 || grid > nwork) grid = nwork;
    cfl_kernel_batch<<<grid, kTileCells, 0, st>>>(args, ccs, work, nwork, nstages, phase_base);
  }
  if (case_list) {
    if (ncases > 0)
      finalize_dt_batch_list<<<(ncases + 127) / 128, 128, 0, st>>>(args, ccs, case_list, ncases,
                                                                    nstages);
  } else if (ncases > 0) {
    finalize_dt_batch<<<(ncases + 127) / 128, 128, 0, st>>>(args, ccs, ncases, nstages);
  }
}

void launch_step_begin_batch(const StageArgs *args, int ncases, int nstages, cudaStream_t st) {
  step_begin_batch<<<(ncases + 127) / 128, 128, 0, st>>>(args, ncases, nstages);
}

// set the abort-order phase base of the current step (8 x step index)
__global__ void set_phase_base_kernel(int *phase_base, int value, int fold) {
  phase_base[0] = value;
  phase_base[1] = fold;
}
void launch_set_phase_base(int *phase_base, int value, int fold, cudaStream_t st) {
  set_phase_base_kernel<<<1, 1, 0, st>>>(phase_base, value, fold);
}
#endif

void launch_cfl(const CflArgs &a, const CaseConst &cc, int nsm, cudaStream_t st) {
  int64_t blocks = (a.nslots + 255) / 256;
  int64_t cap = (int64_t)nsm * 8;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  cfl_kernel<<<(unsigned)blocks, 256, 0, st>>>(a, cc);
  finalize_dt_kernel<<<1, 1, 0, st>>>(a.diag, cc);
}

void launch_step_begin(DevDiag *d, cudaStream_t st) { step_begin_kernel<<<1, 1, 0, st>>>(d); }

void launch_take_folded_cfl(DevDiag *d, const CaseConst &cc, cudaStream_t st) {
  take_folded_cfl_kernel<<<1, 1, 0, st>>>(d, cc);
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

void launch_scatter4(const double *rows, const int32_t *cell_slot, const uint8_t *alias, int64_t n,
                     double Rg, double Cv, double *const s0[kStateFields], int nsm,
                     cudaStream_t st) {
  int64_t blocks = (n + 255) / 256;
  if (blocks > (int64_t)nsm * 16) blocks = (int64_t)nsm * 16;
  if (blocks < 1) blocks = 1;
  scatter_state4_kernel<<<(unsigned)blocks, 256, 0, st>>>(rows, cell_slot, alias, n, Rg, Cv,
                                                          s0[F_RHO], s0[F_U], s0[F_V], s0[F_P],
                                                          s0[F_E], s0[F_T]);
}

void launch_gather4(double *rows, const int32_t *cell_slot, int64_t n,
                    double *const s0[kStateFields], int nsm, cudaStream_t st) {
  int64_t blocks = (n + 255) / 256;
  if (blocks > (int64_t)nsm * 16) blocks = (int64_t)nsm * 16;
  if (blocks < 1) blocks = 1;
  gather_state4_kernel<<<(unsigned)blocks, 256, 0, st>>>(rows, cell_slot, n, s0[F_RHO], s0[F_U],
                                                         s0[F_V], s0[F_P]);
}

}  // namespace IBGPU_KNS
}  // namespace ibgpu
