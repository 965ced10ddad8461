/*
 * CPU restatement of the reference solver's explicit time step.
 * Test infrastructure only (what the GPU path is tested against, and the timed CPU
 * port); nothing in the GPU library links or calls it.
 *
 * Every function cites the reference code it restates.  Evaluation order
 * follows the reference expressions literally; build with
 * -ffp-contract=off so no multiply-add is fused.
 */
#include "ib_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define Q_RHO 0
#define Q_U 1
#define Q_V 2
#define Q_W 3
#define Q_P 4
#define Q_T 5
#define Q_E 6

static inline int slot_of(const ibo_level *L, int ix, int iy) {
  if (ix < L->x0 || iy < L->y0 || ix >= L->x0 + L->nx || iy >= L->y0 + L->ny) return -1;
  int s = (iy - L->y0) * L->nx + (ix - L->x0);
  return (L->flags[s] & IBO_PRESENT) ? s : -1;
}

static inline int marches(const ibo_level *L, int step) {
  return step % L->march_step == L->march_left;
}

/* std::min / std::max as the reference calls them (<algorithm> semantics). */
static inline double smin(double a, double b) { return (b < a) ? b : a; }
static inline double smax(double a, double b) { return (a < b) ? b : a; }

/* Slopelimiter.H:14-20 (VanLeer, the #defined ALimiter) and :84-87 (minmod). */
static inline double limiter(int kind, double qr) {
  if (kind == IBO_LIM_MINMOD) return (qr < 1.0) ? qr : 1.0;
  return 2.0 * qr / (1 + qr);
}

/* comptqleft / SlopeCorrection_Left (NS_Solver.H:26-28, Slopelimiter.H:22-39) */
static inline double muscl_left(int lim, double q_i, double qi, double qi1) {
  double dqi = qi - q_i;
  double dqii = qi1 - qi;
  double qr = dqii / dqi;
  if (fabs(qr) > 1.0e10 || isnan(qr)) {
    if (dqii > 0.0) qr = 1000000.0;
    else qr = -1.0;
  }
  if (qr <= 0.0) qr = 0.0;
  double lv = limiter(lim, qr);
  return qi + 0.5 * dqi * lv;
}

/* comptqright / SlopeCorrection_Right (NS_Solver.H:22-24, Slopelimiter.H:41-58) */
static inline double muscl_right(int lim, double q_i, double qi, double qi1) {
  double dqi = qi - q_i;
  double dqii = qi1 - qi;
  double qr = dqi / dqii;
  if (fabs(qr) > 1.0e10 || isnan(qr)) {
    if (dqi > 0.0) qr = 1000000.0;
    else qr = -1.0;
  }
  if (qr <= 0.0) qr = 0.0;
  double lv = limiter(lim, qr);
  return qi - 0.5 * dqii * lv;
}

/*
 * Inviscid face flux for an axis-aligned face: FaceLeftRight, Get_inv_flux,
 * Roeaverage, roe0c_coef (ROE_ALLSPEED) and ComptFaceFlux
 * (NS_Solver.H:30-113, 704-832; FlowVariables.H:19-64).  With the face normal
 * a unit axis vector the reference's dot products reduce exactly to picking
 * the normal (n) or tangential (t) component; the frame velocity is zero.
 * st[k][c] is the primitive c (rho, un, ut, p) of stencil cell k (L2, L1, R1,
 * R2).  Output f = (mass, momentum n, momentum t, energy) * area.
 */
static void roe_flux(const ibo_params *P, double st[4][4], double area, double f[4]) {
  const double g = P->gama, Rg = P->Rg, Cv = P->Cv;
  double l[4], r[4];
  for (int c = 0; c < 4; ++c) {
    l[c] = muscl_left(P->limiter, st[0][c], st[1][c], st[2][c]);
    r[c] = muscl_right(P->limiter, st[1][c], st[2][c], st[3][c]);
  }
  double lroe = l[0], lun = l[1], lut = l[2], lp = l[3];
  double rroe = r[0], run = r[1], rut = r[2], rp = r[3];
  double lT = lp / (lroe * Rg);
  double le = Cv * lT + 0.5 * (lun * lun + lut * lut);
  double rT = rp / (rroe * Rg);
  double re = Cv * rT + 0.5 * (run * run + rut * rut);
  double lv = lun, rv = run;
  /* Get_inv_flux: (rho q_n, rho u_n q_n + p, rho u_t q_n, (p + rho e) q_n) */
  double pl0 = lroe * lv, pl1 = lroe * lun * lv + lp, pl2 = lroe * lut * lv, pl4 = (lp + le * lroe) * lv;
  double pr0 = rroe * rv, pr1 = rroe * run * rv + rp, pr2 = rroe * rut * rv, pr4 = (rp + re * rroe) * rv;
  double droe = rroe - lroe;
  double dp = rp - lp;
  double dut = rut - lut;
  double dubar = rv - lv;
  /* Roeaverage */
  double r2lroe = sqrt(rroe / lroe);
  double r2l0 = 1.0 / (1.0 + r2lroe);
  double h_left = le + lp / lroe;
  double h_right = re + rp / rroe;
  double a_roe = sqrt(lroe * rroe);
  double a_un = (lun + run * r2lroe) * r2l0;
  double a_ut = (lut + rut * r2lroe) * r2l0;
  double a_h = (h_left + h_right * r2lroe) * r2l0;
  double a_c = sqrt((g - 1.0) * (a_h - (a_un * a_un + a_ut * a_ut) / 2.0));
  double ubar = a_un;
  /* ComptFaceFlux */
  const double csquare = a_c * a_c;
  const double namda3 = fabs(ubar);
  const double coef12 = 1.0 / (2.0 * csquare) * area;
  const double roe0cxdubar = a_roe * a_c * dubar;
  const double faceareaxabsubar = area * namda3;
  const double halffacearea = 0.5 * area;
  double alpha0 = faceareaxabsubar * (droe - dp / csquare);
  /* roe0c_coef, all-speed scaling */
  double T_a = (lT + rT) * 0.5;
  double V_a = (lv + rv) * 0.5;
  double Ma_a = fabs(V_a / sqrt(g * Rg * T_a));
  double f_Ma = smin(smax(Ma_a, P->Ma), 1.0);
  double s0 = (1.0 - f_Ma) * (1.0 - f_Ma);
  double namda0 = sqrt(4.0 * a_c * a_c * f_Ma + s0 * ubar * ubar);
  double namda1 = fabs(0.5 * ((1.0 + f_Ma) * ubar + namda0));
  double namda2 = fabs(0.5 * ((1.0 + f_Ma) * ubar - namda0));
  double alpha1 = coef12 * namda1 * (dp + roe0cxdubar);
  double alpha2 = coef12 * namda2 * (dp - roe0cxdubar);
  double alpha3 = alpha0 + alpha1 + alpha2;
  double alpha4 = a_c * (alpha1 - alpha2);
  double alphat = faceareaxabsubar * (a_roe * dut); /* the normal one is exactly 0 */
  f[0] = -alpha3;
  f[1] = -(a_un * alpha3 + alpha4);
  f[2] = -(a_ut * alpha3 + alphat);
  f[3] = -(a_h * alpha3 + ubar * alpha4 + a_ut * alphat - (csquare / (g - 1.0)) * alpha0);
  f[0] += (pl0 + pr0) * halffacearea;
  f[1] += (pl1 + pr1) * halffacearea;
  f[2] += (pl2 + pr2) * halffacearea;
  f[3] += (pl4 + pr4) * halffacearea;
}

/* Stencil primitive of a slot in face-local (rho, u_n, u_t, p) order. */
static inline void load_nt(const ibo_level *L, int s, int dir, double out[4]) {
  out[0] = L->q[Q_RHO][s];
  out[1] = dir == 0 ? L->q[Q_U][s] : L->q[Q_V][s];
  out[2] = dir == 0 ? L->q[Q_V][s] : L->q[Q_U][s];
  out[3] = L->q[Q_P][s];
}

/* Face between slot a (low side) and b (high side) in direction dir: the
 * [L2, L1 | R1, R2] stencil with the reference's fallback when L2 or R2 is
 * missing (NS_Solver.H:738-756). */
static void face_flux(const ibo_params *P, const ibo_level *L, int dir, int ix, int iy,
                      double f[4]) {
  int dxs = dir == 0 ? 1 : 0, dys = dir == 0 ? 0 : 1;
  int sL1 = slot_of(L, ix, iy);
  int sR1 = slot_of(L, ix + dxs, iy + dys);
  int nL2 = slot_of(L, ix - dxs, iy - dys);
  int nR2 = slot_of(L, ix + 2 * dxs, iy + 2 * dys);
  int sL2 = nL2 >= 0 ? nL2 : nR2;
  int sR2 = nR2 >= 0 ? nR2 : nL2;
  double st[4][4];
  load_nt(L, sL2, dir, st[0]);
  load_nt(L, sL1, dir, st[1]);
  load_nt(L, sR1, dir, st[2]);
  load_nt(L, sR2, dir, st[3]);
  double area = dir == 0 ? L->dy * L->dz : L->dz * L->dx;
  double fn[4];
  roe_flux(P, st, area, fn);
  f[0] = fn[0];
  f[1] = dir == 0 ? fn[1] : fn[2];
  f[2] = dir == 0 ? fn[2] : fn[1];
  f[3] = fn[3];
}

/* Viscous face flux, NS_Solver::ComptViscousStress (NS_Solver.cpp:365-629):
 * normal difference R - L, tangential 0.25*(up1 + up2 - down1 - down2) over
 * the 2x3 block, Sutherland viscosity at the face mean temperature. */
static int visc_flux(const ibo_params *P, const ibo_level *L, int dir, int ix, int iy,
                     double vs[4]) {
  int dxs = dir == 0 ? 1 : 0, dys = dir == 0 ? 0 : 1;
  int tx = dys, ty = dxs; /* tangential unit offset */
  int sL = slot_of(L, ix, iy), sR = slot_of(L, ix + dxs, iy + dys);
  int sLu = slot_of(L, ix + tx, iy + ty), sRu = slot_of(L, ix + dxs + tx, iy + dys + ty);
  int sLd = slot_of(L, ix - tx, iy - ty), sRd = slot_of(L, ix + dxs - tx, iy + dys - ty);
  if (sL < 0 || sR < 0 || sLu < 0 || sRu < 0 || sLd < 0 || sRd < 0) return 425;
  double *const *q = L->q;
  double dnu = q[Q_U][sR] - q[Q_U][sL];
  double dnv = q[Q_V][sR] - q[Q_V][sL];
  double dnT = q[Q_T][sR] - q[Q_T][sL];
  double dtu = 0.25 * (q[Q_U][sLu] + q[Q_U][sRu] - q[Q_U][sLd] - q[Q_U][sRd]);
  double dtv = 0.25 * (q[Q_V][sLu] + q[Q_V][sRu] - q[Q_V][sLd] - q[Q_V][sRd]);
  double dtT = 0.25 * (q[Q_T][sLu] + q[Q_T][sRu] - q[Q_T][sLd] - q[Q_T][sRd]);
  double ikx = 1.0 / L->dx, iky = 1.0 / L->dy;
  double dux, duy, dvx, dvy, dTx, dTy;
  if (dir == 0) {
    dux = dnu * ikx; duy = dtu * iky;
    dvx = dnv * ikx; dvy = dtv * iky;
    dTx = dnT * ikx; dTy = dtT * iky;
  } else {
    dux = dtu * ikx; duy = dnu * iky;
    dvx = dtv * ikx; dvy = dnv * iky;
    dTx = dtT * ikx; dTy = dnT * iky;
  }
  double ftemp = (q[Q_T][sL] + q[Q_T][sR]) * 0.5;
  double mu0 = sqrt(pow(ftemp, 3)) * ((1.0 + P->s_over_t) / (ftemp + P->s_over_t));
  double qk0 = P->qk * mu0;
  double tauxx = 2.0 * mu0 * (dux - (dux + dvy) / 3.0) / P->Re;
  double tauyy = 2.0 * mu0 * (dvy - (dux + dvy) / 3.0) / P->Re;
  double tauxy = mu0 / P->Re * (duy + dvx);
  double qx = qk0 * dTx, qy = qk0 * dTy;
  double fv0 = (q[Q_U][sL] + q[Q_U][sR]) * 0.5;
  double fv1 = (q[Q_V][sL] + q[Q_V][sR]) * 0.5;
  double bbbx = fv0 * tauxx + fv1 * tauxy + qx;
  double bbby = fv0 * tauxy + fv1 * tauyy + qy;
  double area = dir == 0 ? L->dy * L->dz : L->dz * L->dx;
  vs[0] = 0.0;
  if (dir == 0) {
    vs[1] = tauxx * area;
    vs[2] = tauxy * area;
    vs[3] = bbbx * area;
  } else {
    vs[1] = tauxy * area;
    vs[2] = tauyy * area;
    vs[3] = bbby * area;
  }
  return 0;
}

/* Mesh::DataExchange restricted to one node: the intra-node block/periodic
 * copies (Mesh.cpp:768-780). */
static void exchange(ibo_level *L) {
  for (int i = 0; i < L->ncopy; ++i)
    for (int c = 0; c < 7; ++c) L->q[c][L->copy_dst[i]] = L->q[c][L->copy_src[i]];
}

int ibo_cfl_dt(const ibo_params *P, const ibo_level *lev, int nlev, double *cfl_dt) {
  /* NS_Solver::Comptdt (NS_Solver.cpp:196-280) */
  double cdt = 10000.0;
  for (int l = 0; l < nlev; ++l) {
    const ibo_level *L = &lev[l];
    double ax = L->dy * L->dz, ay = L->dz * L->dx, az = L->dx * L->dy;
    double v = L->dx * L->dy * L->dz;
    for (int s = 0; s < L->nx * L->ny; ++s) {
      if (!(L->flags[s] & IBO_NORMAL)) continue;
      double c = sqrt(P->gama * P->Rg * L->q[Q_T][s]);
      double c0 = (fabs(L->q[Q_U][s]) + c) * ax;
      double c1 = (fabs(L->q[Q_V][s]) + c) * ay;
      double c2 = (fabs(L->q[Q_W][s]) + c) * az;
      double d0 = P->cfl * v / (c0 + c1 + c2);
      if (d0 < 0.0) return 424;
      cdt = smin(cdt, d0);
    }
  }
  *cfl_dt = cdt;
  return 0;
}

int ibo_step(const ibo_params *P, ibo_level *lev, int nlev, int ts, double *dt,
             double *cfl_dt, double res_max[5]) {
  int rc = 0;
  if (nlev <= 0) return 0;
  /* AMR::InterfaceExchange: block-ghost refresh of the levels that march at
   * ts+1 (AMRInterface.cpp:20, Mesh.cpp:542-562). */
  for (int l = 0; l < nlev; ++l)
    if (marches(&lev[l], ts + 1)) exchange(&lev[l]);

  /* Comptdt every dt_var_step steps */
  if (ts % P->dt_var_step == 0) {
    double cdt;
    rc = ibo_cfl_dt(P, lev, nlev, &cdt);
    if (rc) return rc;
    *cfl_dt = cdt;
    *dt = smin(cdt, *dt * P->dt_ratio);
  }

  /* per-level work arrays */
  double **un = (double **)calloc((size_t)nlev, sizeof(double *));
  double **fx = (double **)calloc((size_t)nlev, sizeof(double *));
  double **fy = (double **)calloc((size_t)nlev, sizeof(double *));
  double **vx = (double **)calloc((size_t)nlev, sizeof(double *));
  double **vy = (double **)calloc((size_t)nlev, sizeof(double *));
  double **src = (double **)calloc((size_t)nlev, sizeof(double *));
  double **cvn = (double **)calloc((size_t)nlev, sizeof(double *));
  for (int l = 0; l < nlev; ++l) {
    size_t n = (size_t)lev[l].nx * (size_t)lev[l].ny;
    un[l] = (double *)calloc(4 * n, sizeof(double));
    fx[l] = (double *)calloc(4 * n, sizeof(double));
    fy[l] = (double *)calloc(4 * n, sizeof(double));
    vx[l] = (double *)calloc(4 * n, sizeof(double));
    vy[l] = (double *)calloc(4 * n, sizeof(double));
    src[l] = (double *)calloc(4 * n, sizeof(double));
    cvn[l] = (double *)calloc(4 * n, sizeof(double));
  }

  /* ComptOldConsVar (NS_Solver.H:392-424) */
  for (int l = 0; l < nlev; ++l) {
    ibo_level *L = &lev[l];
    if (!marches(L, ts)) continue;
    for (int s = 0; s < L->nx * L->ny; ++s) {
      if (!(L->flags[s] & IBO_NORMAL)) continue;
      double r = L->q[Q_RHO][s];
      un[l][4 * s + 0] = r;
      un[l][4 * s + 1] = r * L->q[Q_U][s];
      un[l][4 * s + 2] = r * L->q[Q_V][s];
      un[l][4 * s + 3] = r * L->q[Q_E][s];
    }
  }

  /* ComptViscousStress, frozen for all stages.  Face arrays are indexed by
   * the slot of the face's low-side cell. */
  if (P->viscous) {
    for (int l = 0; l < nlev && !rc; ++l) {
      ibo_level *L = &lev[l];
      if (!marches(L, ts)) continue;
      for (int s = 0; s < L->nx * L->ny && !rc; ++s) {
        if (!(L->flags[s] & IBO_PRESENT)) continue;
        int ix = L->x0 + s % L->nx, iy = L->y0 + s / L->nx;
        for (int dir = 0; dir < 2; ++dir) {
          int sb = slot_of(L, ix + (dir == 0), iy + (dir == 1));
          if (sb < 0) continue;
          if (!((L->flags[s] | L->flags[sb]) & IBO_NORMAL)) continue;
          rc = visc_flux(P, L, dir, ix, iy, dir == 0 ? &vx[l][4 * s] : &vy[l][4 * s]);
          if (rc) break;
        }
      }
    }
  }

  for (int k = 0; k < P->nstages && !rc; ++k) {
    /* ComputeFaceFlux */
    for (int l = 0; l < nlev; ++l) {
      ibo_level *L = &lev[l];
      if (!marches(L, ts)) continue;
      for (int s = 0; s < L->nx * L->ny; ++s) {
        if (!(L->flags[s] & IBO_PRESENT)) continue;
        int ix = L->x0 + s % L->nx, iy = L->y0 + s / L->nx;
        for (int dir = 0; dir < 2; ++dir) {
          int sb = slot_of(L, ix + (dir == 0), iy + (dir == 1));
          if (sb < 0) continue;
          if (!((L->flags[s] | L->flags[sb]) & IBO_NORMAL)) continue;
          face_flux(P, L, dir, ix, iy, dir == 0 ? &fx[l][4 * s] : &fy[l][4 * s]);
        }
      }
    }
    /* ComptSource (NS_Solver.cpp:282-363) */
    for (int l = 0; l < nlev; ++l) {
      ibo_level *L = &lev[l];
      if (!marches(L, ts)) continue;
      for (int s = 0; s < L->nx * L->ny; ++s) {
        if (!(L->flags[s] & IBO_NORMAL)) continue;
        int ix = L->x0 + s % L->nx, iy = L->y0 + s / L->nx;
        int xlo = slot_of(L, ix - 1, iy), ylo = slot_of(L, ix, iy - 1);
        double sx[4], sy[4];
        for (int c = 0; c < 4; ++c) {
          sx[c] = fx[l][4 * xlo + c] - fx[l][4 * s + c];
          sy[c] = fy[l][4 * ylo + c] - fy[l][4 * s + c];
          if (P->viscous) {
            sx[c] += vx[l][4 * s + c] - vx[l][4 * xlo + c];
            sy[c] += vy[l][4 * s + c] - vy[l][4 * ylo + c];
          }
          src[l][4 * s + c] = sx[c] + sy[c];
        }
      }
    }
    /* UpdateConsVars (NS_Solver.cpp:844-985): every level's cv_new and its
     * density check first (abort 523, or 611 on the body level) ... */
    double dt0 = P->tp[k] * *dt;
    for (int l = 0; l < nlev && !rc; ++l) {
      ibo_level *L = &lev[l];
      if (!marches(L, ts)) continue;
      double level_ts = dt0 * L->step_num;
      double v = L->dx * L->dy * L->dz;
      for (int s = 0; s < L->nx * L->ny; ++s) {
        uint8_t fl = L->flags[s];
        if (!(fl & IBO_NORMAL) || !(fl & IBO_UPDATE)) continue;
        for (int c = 0; c < 4; ++c) cvn[l][4 * s + c] = un[l][4 * s + c] + src[l][4 * s + c] * level_ts / v;
        if (cvn[l][4 * s] < 0.0) { rc = (l == P->body_level) ? 611 : 523; break; }
      }
    }
    /* ... then ComptNewPrimVar (NS_Solver.cpp:3-194) and its T check (37) */
    for (int l = 0; l < nlev && !rc; ++l) {
      ibo_level *L = &lev[l];
      if (!marches(L, ts)) continue;
      for (int s = 0; s < L->nx * L->ny; ++s) {
        uint8_t fl = L->flags[s];
        if (!(fl & IBO_NORMAL)) continue;
        if ((fl & IBO_PRIM) && (fl & IBO_UPDATE)) {
          const double *cv = &cvn[l][4 * s];
          double r = cv[0];
          double u = cv[1] / cv[0];
          double vv = cv[2] / cv[0];
          double e = cv[3] / cv[0];
          double p = (e - 0.5 * (u * u + vv * vv)) * (P->gama - 1.0) * r;
          double T = p / (r * P->Rg);
          L->q[Q_RHO][s] = r;
          L->q[Q_U][s] = u;
          L->q[Q_V][s] = vv;
          L->q[Q_W][s] = 0.0;
          L->q[Q_E][s] = e;
          L->q[Q_P][s] = p;
          L->q[Q_T][s] = T;
        } else if (fl & IBO_RESET) {
          for (int c = 0; c < 7; ++c) L->q[c][s] = P->initvar[c];
        } else {
          continue;
        }
        if (L->q[Q_T][s] < 0.0) { rc = 37; break; }
      }
    }
    /* inter-stage block-ghost refresh */
    if (k < P->nstages - 1)
      for (int l = 0; l < nlev; ++l)
        if (marches(&lev[l], ts)) exchange(&lev[l]);
  }

  /* ResinDomain max-norm (NS_Solver.H:264-378) */
  if (!rc) {
    for (int c = 0; c < 5; ++c) res_max[c] = 0.0;
    for (int l = 0; l < nlev; ++l) {
      ibo_level *L = &lev[l];
      if (!marches(L, ts)) continue;
      for (int s = 0; s < L->nx * L->ny; ++s) {
        if (!(L->flags[s] & IBO_RESNORM)) continue;
        res_max[0] = smax(fabs(src[l][4 * s + 0]), res_max[0]);
        res_max[1] = smax(fabs(src[l][4 * s + 1]), res_max[1]);
        res_max[2] = smax(fabs(src[l][4 * s + 2]), res_max[2]);
        res_max[4] = smax(fabs(src[l][4 * s + 3]), res_max[4]);
      }
    }
    for (int c = 0; c < 5; ++c)
      if (isnan(res_max[c])) rc = 268;
  }

  for (int l = 0; l < nlev; ++l) {
    free(un[l]); free(fx[l]); free(fy[l]); free(vx[l]); free(vy[l]); free(src[l]); free(cvn[l]);
  }
  free(un); free(fx); free(fy); free(vx); free(vy); free(src); free(cvn);
  return rc;
}
