// Ghost-fill, viscous-flux and wall-force kernels of the step (included by
// each arithmetic build after kernels.cuh, inside namespace
// ibgpu::IBGPU_KNS).  Ghost fills and forces are FP64 in every build and
// follow the reference expression by expression; the viscous flux follows
// the build's real type R.
#pragma once

#include "exactmath.cuh"

namespace ibgpu {
namespace IBGPU_KNS {

// ---- coarse/fine interface ----------------------------------------------

// AMR::InterfaceRestriction -> PairRestriction_2d -> AverageCell_2d
// (AMRInterface.cpp:78-110, TwoLevelOp.H:67-87, 225-231): density-weighted
// mean of the four sons written to the coarse ghost.
__global__ void restrict_kernel(PairArgs a, CaseConst cc) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  double *const *q = a.s0;
  double roe = 0.0, u = 0.0, v = 0.0, e = 0.0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    int f = a.fine[4 * i + k];
    double r = q[F_RHO][f];
    roe += r;
    u += q[F_U][f] * r;
    v += q[F_V][f] * r;
    e += q[F_E][f] * r;
  }
  u /= roe;
  v /= roe;
  e /= roe;
  roe *= 0.25;
  double p = (e - 0.5 * (u * u + v * v)) * cc.gm1 * roe;
  double T = p / (roe * cc.Rg);
  int c = a.coarse[i];
  q[F_RHO][c] = roe;
  q[F_U][c] = u;
  q[F_V][c] = v;
  q[F_P][c] = p;
  q[F_E][c] = e;
  q[F_T][c] = T;
}

// AMR::InterfaceProlongation -> PairProlongation_2d (TwoLevelOp.H:200-215,
// 16-22, 35-43): conserved variables of the coarse cell and its x/y
// neighbours, central gradients (q+ - q-)/2, sons at offsets -/+ 1/4,
// primitive recovery of each son.
__global__ void prolong_kernel(PairArgs a, CaseConst cc) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  double *const *q = a.s0;
  // neighbour order: -x, +x, -y, +y
  double U[5][4];
  int cells[5] = {a.coarse[i], a.nb[4 * i + 0], a.nb[4 * i + 1], a.nb[4 * i + 2], a.nb[4 * i + 3]};
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    int s = cells[k];
    double r = q[F_RHO][s];
    U[k][0] = r;
    U[k][1] = r * q[F_U][s];
    U[k][2] = r * q[F_V][s];
    U[k][3] = r * q[F_E][s];
  }
  double gx[4], gy[4];
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    gx[v] = (U[2][v] - U[1][v]) * 0.5;
    gy[v] = (U[4][v] - U[3][v]) * 0.5;
  }
  const double fincrem[2] = {-0.25, 0.25};
#pragma unroll
  for (int si = 0; si < 2; ++si)
#pragma unroll
    for (int sj = 0; sj < 2; ++sj) {
      double f[4];
#pragma unroll
      for (int v = 0; v < 4; ++v) f[v] = U[0][v] + fincrem[si] * gx[v] + fincrem[sj] * gy[v];
      double roe = f[0];
      double u = f[1] / f[0];
      double vv = f[2] / f[0];
      double e = f[3] / f[0];
      double p = (e - 0.5 * (u * u + vv * vv)) * cc.gm1 * roe;
      double T = p / (roe * cc.Rg);
      int s = a.fine[4 * i + si * 2 + sj];
      q[F_RHO][s] = roe;
      q[F_U][s] = u;
      q[F_V][s] = vv;
      q[F_P][s] = p;
      q[F_E][s] = e;
      q[F_T][s] = T;
    }
}

// ---- domain boundary ghosts (BCValues::BCBoxTreat, BCValues.H:51-298) ----
__global__ void bc_kernel(BcArgs a, CaseConst cc) {
  int i = a.begin + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.end) return;
  double *const *q = a.s0;
  const int g = a.ghost[i], r = a.ref[i];
  const int type = a.type[i];
  const double *fv = a.facevar + 7 * a.face[i];
  double roe = q[F_RHO][r], u = q[F_U][r], v = q[F_V][r], p = q[F_P][r], T = q[F_T][r],
         e = q[F_E][r];
  switch (type) {
    case -50:  // outflow: copy (SetBCType_50)
      break;
    case -12:  // pressure outlet (SetBCType_12)
      p = fv[4] + a.backpressure;
      roe = p / (cc.Rg * T);
      break;
    case -13: {  // pressure inlet (SetBCType_13)
      double speed0 = sqrt(u * u + v * v);
      u = speed0 * a.cos_in;
      v = speed0 * a.sin_in;
      T = fv[5] - 0.5 * (u * u + v * v) / cc.Cp;
      p = fv[4] * pow3p5_rn(T / fv[5]);
      roe = p / (cc.Rg * T);
      e = cc.Cv * T + 0.5 * (u * u + v * v);
      break;
    }
    case -49:  // no-slip wall (SetBCType_49); -46/-42 with a static frame and faces
    case -46:
    case -42:
      u = 0.0;
      v = 0.0;
      roe = p / (cc.Rg * T);
      e = cc.Cv * T + 0.0;
      break;
    case -51: {  // slip wall (SetBCType_51)
      const double *n = a.nmv + 3 * i;
      double un = u * n[0] + v * n[1];
      u = u - un * n[0];
      v = v - un * n[1];
      double w = 0.0 - un * n[2];
      roe = p / (cc.Rg * T);
      e = cc.Cv * T + 0.5 * (u * u + v * v + w * w);
      break;
    }
    case -10:  // fixed values (SetBCType_10)
      roe = fv[0];
      u = fv[1];
      v = fv[2];
      p = fv[4];
      T = fv[5];
      e = fv[6];
      break;
    case -45:  // fixed velocity, zero-gradient pressure (SetBCType_45)
      u = fv[1];
      v = fv[2];
      T = fv[5];
      roe = p / (cc.Rg * T);
      break;
    default:
      return;
  }
  q[F_RHO][g] = roe;
  q[F_U][g] = u;
  q[F_V][g] = v;
  q[F_P][g] = p;
  q[F_E][g] = e;
  q[F_T][g] = T;
}

// ---- immersed-boundary ghost cells (Body::IBConditions_Image) -----------

// Image-point state, Mesh::IntpHGgcellVar (Mesh.cpp:1532-1547)
__device__ __forceinline__ void image_point(const int32_t *cells, const double *w,
                                            double *const *q, const CaseConst &cc, double &T,
                                            double &p, double &u, double &v, double &roe) {
  T = 0.0;
  p = 0.0;
  u = 0.0;
  v = 0.0;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    int s = cells[k];
    T += w[k] * q[F_T][s];
    p += w[k] * q[F_P][s];
    u += w[k] * q[F_U][s];
    v += w[k] * q[F_V][s];
  }
  roe = p / (cc.Rg * T);
}

// Phase 1: every IB cell's new state from the current field (the reference
// computes them all before writing any, Body.cpp:1361-1488).
__global__ void ib_compute_kernel(IbArgs a, CaseConst cc) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const double *f = a.cellf + 16 * i;  // signdis, hgdis, w[8], nv[3], patv[3]
  double hT, hp, hu, hv, hroe;
  image_point(a.intp + 8 * i, f + 2, a.s0, cc, hT, hp, hu, hv, hroe);
  const double signdis = f[0], hgdis = f[1];
  const double *wv = f + 13;
  double u, v, w, p, T;
  if (signdis < 0.0) {
    u = 2.0 * wv[0] - hu;
    v = 2.0 * wv[1] - hv;
    w = 2.0 * wv[2] - 0.0;
    p = hp;
    T = hT;
  } else {
    // Body::LinearDist (Body.cpp:183-204)
    double rt = signdis + hgdis;
    double r0 = signdis / rt;
    u = wv[0] + (hu - wv[0]) * r0;
    v = wv[1] + (hv - wv[1]) * r0;
    w = wv[2] + (0.0 - wv[2]) * r0;
    p = hp;
    T = hT;
  }
  double roe = p / (cc.Rg * T);
  double e = cc.Cv * T + 0.5 * (u * u + v * v + w * w);
  double *o = a.out + 6 * i;
  o[0] = roe;
  o[1] = u;
  o[2] = v;
  o[3] = p;
  o[4] = e;
  o[5] = T;
  const int phase = a.phase + (a.phase_base ? *a.phase_base : 0);
  if (hT < 0.0) raise_error(a.diag, phase, ERR_IB_NEG_T, a.cell[i]);
  if (isnan(roe) || isnan(u) || isnan(v) || isnan(p) || isnan(T) || isnan(e))
    raise_error(a.diag, phase, ERR_IB_NAN, a.cell[i]);
}

// Phase 2: write them (Body.cpp:1490-1494)
__global__ void ib_store_kernel(IbArgs a) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const double *o = a.out + 6 * i;
  int s = a.cell[i];
  a.s0[F_RHO][s] = o[0];
  a.s0[F_U][s] = o[1];
  a.s0[F_V][s] = o[2];
  a.s0[F_P][s] = o[3];
  a.s0[F_E][s] = o[4];
  a.s0[F_T][s] = o[5];
}

// ---- wall forces (Body::ComptWallForce, Body.cpp:439-558) ----------------
// Per patch: image-point state, tangential shear mu*du_t/hgdis*area,
// pressure force -p n area, and their moments about the body centre.
__global__ void patch_force_kernel(ForceArgs a, CaseConst cc) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const double *f = a.patchf + 19 * i;  // pc[3], nv[3], area, hgdis, w[8], patv[3]
  double hT, hp, hu, hv, hroe;
  image_point(a.intp + 8 * i, f + 8, a.s0, cc, hT, hp, hu, hv, hroe);
  const double *pc = f, *nv = f + 3, *pv = f + 16;
  const double area = f[6], hgdis = f[7];
  const double *bc = a.body_center + 3 * a.body[i];
  double du0 = hu - pv[0], du1 = hv - pv[1], du2 = 0.0 - pv[2];
  double dx0 = pc[0] - bc[0], dx1 = pc[1] - bc[1], dx2 = pc[2] - bc[2];
  double dn = du0 * nv[0] + du1 * nv[1] + du2 * nv[2];
  du0 = (du0 - nv[0] * dn) / hgdis;
  du1 = (du1 - nv[1] * dn) / hgdis;
  du2 = (du2 - nv[2] * dn) / hgdis;
  double df0[3] = {du0 * cc.mu * area, du1 * cc.mu * area, du2 * cc.mu * area};
  double pa = -hp * area;
  double df1[3] = {nv[0] * pa, nv[1] * pa, nv[2] * pa};
  double *o = a.out + 12 * i;
  o[0] = df1[0];
  o[1] = df1[1];
  o[2] = df1[2];
  o[3] = df0[0];
  o[4] = df0[1];
  o[5] = df0[2];
  // dm = dxyz x df (Pointxyz::cross)
  o[6] = dx1 * df1[2] - dx2 * df1[1];
  o[7] = dx2 * df1[0] - dx0 * df1[2];
  o[8] = dx0 * df1[1] - dx1 * df1[0];
  o[9] = dx1 * df0[2] - dx2 * df0[1];
  o[10] = dx2 * df0[0] - dx0 * df0[2];
  o[11] = dx0 * df0[1] - dx1 * df0[0];
}

// Sums in patch order, then the reference's dimensional scaling.  Each of
// the 12 parts (pressure force, shear force, pressure moment, shear moment)
// is its own sequential sum from zero over the body's patches, as in the
// reference; the block stages the parts a chunk of patches at a time in
// shared memory and 12 threads run the 12 sums side by side (one thread
// reading them from global memory one patch after another spent some 800 ns
// per patch waiting on loads).
__global__ void __launch_bounds__(256) force_sum_kernel(ForceArgs a, CaseConst cc) {
  constexpr int kChunk = 256;
  __shared__ double part[12 * kChunk];
  __shared__ double sum[12];
  const int t = threadIdx.x;
  for (int b = 0; b < a.nbodies; ++b) {
    double acc = 0.0;
    const int i0 = a.body_begin[b], i1 = a.body_begin[b + 1];
    for (int c = i0; c < i1; c += kChunk) {
      const int m = min(kChunk, i1 - c);
      for (int k = t; k < 12 * m; k += blockDim.x) part[k] = a.out[12 * (int64_t)c + k];
      __syncthreads();
      if (t < 12)
        for (int i = 0; i < m; ++i) acc += part[12 * i + t];
      __syncthreads();  // the next chunk overwrites the parts
    }
    if (t < 12) sum[t] = acc;
    __syncthreads();
    if (t == 0) {
      double *r = a.result + 6 * b;
      for (int k = 0; k < 3; ++k) {
        double pfs = sum[k] * cc.p_ref * cc.area_ref;
        double pms = sum[6 + k] * cc.p_ref * cc.area_ref * cc.L_ref;
        double tfs = sum[3 + k] * cc.shear_ref * cc.area_ref;
        double tms = sum[9 + k] * cc.shear_ref * cc.area_ref * cc.L_ref;
        r[k] = pfs + tfs;
        r[3 + k] = pms + tms;
      }
    }
    __syncthreads();  // sum[] is rewritten for the next body
  }
}

// ---- viscous face flux (NS_Solver::ComptViscousStress) -------------------
// One tile per CTA: u, v, T of the tile and a one-cell halo (corners
// included), every x- and y-face viscous flux into shared memory, then each
// leaf cell's frozen residual parts vs(high) - vs(low) per direction.
template <typename R>
__global__ void __launch_bounds__(kTileCells) viscous_kernel(ViscArgs a, CaseConst cc) {
  constexpr int H = 1, G = kTile + 2 * H;  // 18
  __shared__ R su[G * G], sv[G * G], sT[G * G];
  __shared__ uint8_t sfl[G * G];
  __shared__ R vx[3][kXFaces];  // x-mom, y-mom, energy of x-faces
  __shared__ R vy[3][kYFaces];
  const int tid = threadIdx.x;
  const int tile = a.tile_begin + blockIdx.x;
  const LevelConst &L = cc.lev[a.tile_level[tile]];
  for (int r = tid; r < G * G; r += kTileCells) {
    int rx = r % G - H, ry = r / G - H;
    int ox = rx < 0 ? -1 : (rx >= kTile ? 1 : 0);
    int oy = ry < 0 ? -1 : (ry >= kTile ? 1 : 0);
    uint8_t f = 0;
    R u = R(0), v = R(0), T = R(0);
    int nb = a.tile_nb[tile * 9 + (oy + 1) * 3 + (ox + 1)];
    if (nb >= 0) {
      int64_t s = (int64_t)nb * kTileCells + (ry - oy * kTile) * kTile + (rx - ox * kTile);
      f = a.flags[s];
      if (f & CF_PRESENT) {
        u = (R)a.s0[F_U][s];
        v = (R)a.s0[F_V][s];
        T = (R)a.s0[F_T][s];
      }
    }
    sfl[r] = f;
    su[r] = u;
    sv[r] = v;
    sT[r] = T;
  }
  __syncthreads();
  const R ikx = (R)L.inv_dx, iky = (R)L.inv_dy;
  const R Re = (R)cc.Re, S = (R)cc.s_over_t, qk = (R)cc.qk;
  for (int w = tid; w < kXFaces + kYFaces; w += kTileCells) {
    const bool xdir = w < kXFaces;
    int rL, rR, tstep;
    if (xdir) {
      int j = w / (kTile + 1), i = w % (kTile + 1);
      rR = (j + H) * G + (i + H);
      rL = rR - 1;
      tstep = G;
    } else {
      int v = w - kXFaces;
      int j = v / kTile, i = v % kTile;
      rR = (j + H) * G + (i + H);
      rL = rR - G;
      tstep = 1;
    }
    R f1 = R(0), f2 = R(0), f3 = R(0);
    const uint8_t fL = sfl[rL], fR = sfl[rR];
    if ((fL & CF_PRESENT) && (fR & CF_PRESENT) && ((fL | fR) & CF_NORMAL)) {
      const int Lu = rL + tstep, Ru = rR + tstep, Ld = rL - tstep, Rd = rR - tstep;
      // normal difference and the 2x3-block tangential difference
      // (pfpkesai0 / pfpkesai1, NS_Solver.H:147-151)
      R dnu = su[rR] - su[rL], dnv = sv[rR] - sv[rL], dnT = sT[rR] - sT[rL];
      R dtu = R(0.25) * (su[Lu] + su[Ru] - su[Ld] - su[Rd]);
      R dtv = R(0.25) * (sv[Lu] + sv[Ru] - sv[Ld] - sv[Rd]);
      R dtT = R(0.25) * (sT[Lu] + sT[Ru] - sT[Ld] - sT[Rd]);
      R dux, duy, dvx, dvy, dTx, dTy;
      if (xdir) {
        dux = dnu * ikx; duy = dtu * iky; dvx = dnv * ikx; dvy = dtv * iky;
        dTx = dnT * ikx; dTy = dtT * iky;
      } else {
        dux = dtu * ikx; duy = dnu * iky; dvx = dtv * ikx; dvy = dnv * iky;
        dTx = dtT * ikx; dTy = dnT * iky;
      }
      R ftemp = (sT[rL] + sT[rR]) * R(0.5);
      R ft3;
      if (sizeof(R) == sizeof(double)) ft3 = (R)cube_rn((double)ftemp);
      else ft3 = ftemp * ftemp * ftemp;
      R mu0 = sqrt(ft3) * ((R(1) + S) / (ftemp + S));
      R qk0 = qk * mu0;
      R tauxx = R(2) * mu0 * (dux - (dux + dvy) / R(3)) / Re;
      R tauyy = R(2) * mu0 * (dvy - (dux + dvy) / R(3)) / Re;
      R tauxy = mu0 / Re * (duy + dvx);
      R qx = qk0 * dTx, qy = qk0 * dTy;
      R fv0 = (su[rL] + su[rR]) * R(0.5);
      R fv1 = (sv[rL] + sv[rR]) * R(0.5);
      if (xdir) {
        R area = (R)L.area_x;
        f1 = tauxx * area;
        f2 = tauxy * area;
        f3 = (fv0 * tauxx + fv1 * tauxy + qx) * area;
      } else {
        R area = (R)L.area_y;
        f1 = tauxy * area;
        f2 = tauyy * area;
        f3 = (fv0 * tauxy + fv1 * tauyy + qy) * area;
      }
    }
    if (xdir) {
      vx[0][w] = f1; vx[1][w] = f2; vx[2][w] = f3;
    } else {
      int v = w - kXFaces;
      vy[0][v] = f1; vy[1][v] = f2; vy[2][v] = f3;
    }
  }
  __syncthreads();
  const int lx = tid % kTile, ly = tid / kTile;
  const int64_t slot = (int64_t)tile * kTileCells + tid;
  if (sfl[(ly + H) * G + (lx + H)] & CF_NORMAL) {
    const int xlo = ly * (kTile + 1) + lx, xhi = xlo + 1;
    const int ylo = ly * kTile + lx, yhi = ylo + kTile;
    a.vsd[0 * a.nslots + slot] = 0.0 - 0.0;
    a.vsd[4 * a.nslots + slot] = 0.0 - 0.0;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      a.vsd[(int64_t)(1 + c) * a.nslots + slot] = (double)vx[c][xhi] - (double)vx[c][xlo];
      a.vsd[(int64_t)(5 + c) * a.nslots + slot] = (double)vy[c][yhi] - (double)vy[c][ylo];
    }
  }
}

// ---- launchers ---------------------------------------------------------------
void launch_restrict(const PairArgs &a, const CaseConst &cc, cudaStream_t st) {
  if (a.n > 0) restrict_kernel<<<(a.n + 127) / 128, 128, 0, st>>>(a, cc);
}
void launch_prolong(const PairArgs &a, const CaseConst &cc, cudaStream_t st) {
  if (a.n > 0) prolong_kernel<<<(a.n + 127) / 128, 128, 0, st>>>(a, cc);
}
void launch_bc(const BcArgs &a, const CaseConst &cc, cudaStream_t st) {
  int n = a.end - a.begin;
  if (n > 0) bc_kernel<<<(n + 127) / 128, 128, 0, st>>>(a, cc);
}
void launch_ib(const IbArgs &a, const CaseConst &cc, cudaStream_t st) {
  if (a.n <= 0) return;
  ib_compute_kernel<<<(a.n + 127) / 128, 128, 0, st>>>(a, cc);
  ib_store_kernel<<<(a.n + 127) / 128, 128, 0, st>>>(a);
}
void launch_forces(const ForceArgs &a, const CaseConst &cc, cudaStream_t st) {
  if (a.n > 0) patch_force_kernel<<<(a.n + 127) / 128, 128, 0, st>>>(a, cc);
  force_sum_kernel<<<1, 256, 0, st>>>(a, cc);
}
void launch_viscous(const ViscArgs &a, const CaseConst &cc, int ntiles, bool mixed,
                    cudaStream_t st) {
  if (ntiles <= 0) return;
#ifdef IBGPU_FAST_BUILD
  if (mixed) {
    viscous_kernel<float><<<ntiles, kTileCells, 0, st>>>(a, cc);
    return;
  }
#endif
  viscous_kernel<double><<<ntiles, kTileCells, 0, st>>>(a, cc);
}

}  // namespace IBGPU_KNS
}  // namespace ibgpu
