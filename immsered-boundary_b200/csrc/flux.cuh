// Face-flux arithmetic of the explicit step, shared by the FP64, exact-FP64
// and mixed-precision kernel builds (the real type R is double or float).
//
// Each function restates one reference macro or member function for an
// axis-aligned face of the reference's Cartesian cells, in the reference's
// evaluation order.  With a unit-axis face normal the reference's dot
// products (n . u, k_x alpha_4, ...) reduce exactly to picking the normal
// (n) or tangential (t) velocity component, and every z term it evaluates in
// its one-cell-thick slab is an exact zero, so dropping them changes no
// result.  The frame velocity is zero (static reference frame).
#pragma once

#include <cuda_runtime.h>
#include <math.h>

#include "fastmath.cuh"

namespace ibgpu {

template <typename R>
struct Gas {
  R gama, Rg, Cv, Ma;
  R gm1;      // gama - 1.0
  R gamaRg;   // gama * Rg   (the reference's left-to-right "gama*Rg*T")
  R inv_Rg;   // 1 / Rg      (fast builds)
  R inv_gm1;  // 1 / (gama - 1)
  R gam_gm1;  // gama / (gama - 1)  (fast builds: h = gam_gm1 p/rho + |u|^2/2)
  R two_gama; // 2 gama              (fast builds: the all-speed Mach number)
};

enum { LIM_VANLEER = 0, LIM_MINMOD = 1 };

// Slopelimiter.H:14-20 (VanLeer, the reference's ALimiter) and :84-87 (minmod)
template <int LIM, typename R>
__device__ __forceinline__ R limiter_phi(R qr) {
  if (LIM == LIM_MINMOD) return qr < R(1) ? qr : R(1);
  return R(2) * qr / (R(1) + qr);
}

// comptqleft / SlopeCorrection_Left (NS_Solver.H:26-28, Slopelimiter.H:22-39)
template <int LIM, typename R>
__device__ __forceinline__ R muscl_left(R q_i, R qi, R qi1) {
  R dqi = qi - q_i;
  R dqii = qi1 - qi;
  R qr = dqii / dqi;
  if (fabs(qr) > R(1.0e10) || isnan(qr)) qr = (dqii > R(0)) ? R(1000000.0) : R(-1.0);
  if (qr <= R(0)) qr = R(0);
  R lv = limiter_phi<LIM>(qr);
  return qi + R(0.5) * dqi * lv;
}

// comptqright / SlopeCorrection_Right (NS_Solver.H:22-24, Slopelimiter.H:41-58)
template <int LIM, typename R>
__device__ __forceinline__ R muscl_right(R q_i, R qi, R qi1) {
  R dqi = qi - q_i;
  R dqii = qi1 - qi;
  R qr = dqi / dqii;
  if (fabs(qr) > R(1.0e10) || isnan(qr)) qr = (dqi > R(0)) ? R(1000000.0) : R(-1.0);
  if (qr <= R(0)) qr = R(0);
  R lv = limiter_phi<LIM>(qr);
  return qi - R(0.5) * dqii * lv;
}

// std::min / std::max as the reference calls them
template <typename R>
__device__ __forceinline__ R smin(R a, R b) { return (b < a) ? b : a; }
template <typename R>
__device__ __forceinline__ R smax(R a, R b) { return (a < b) ? b : a; }

// Inviscid all-speed Roe flux of one face from the 4-cell stencil
// [L2, L1 | R1, R2], each cell given as (rho, u_n, u_t, p):
// FaceLeftRight + Get_T/Get_E (NS_Solver.H:30-44), Get_inv_flux
// (FlowVariables.H:59-64), Roeaverage (NS_Solver.H:50-62), roe0c_coef with
// ROE_ALLSPEED (:66-75) and ComptFaceFlux (:87-113).
// Output (mass, momentum_n, momentum_t, energy), already multiplied by area.
template <int LIM, typename R>
__device__ __forceinline__ void roe_face_flux(const Gas<R> &g, R area,
                                              R r0, R n0, R t0, R p0,
                                              R r1, R n1, R t1, R p1,
                                              R r2, R n2, R t2, R p2,
                                              R r3, R n3, R t3, R p3,
                                              R &f_mass, R &f_n, R &f_t, R &f_e) {
  const R lroe = muscl_left<LIM>(r0, r1, r2);
  const R rroe = muscl_right<LIM>(r1, r2, r3);
  const R lun = muscl_left<LIM>(n0, n1, n2);
  const R run = muscl_right<LIM>(n1, n2, n3);
  const R lut = muscl_left<LIM>(t0, t1, t2);
  const R rut = muscl_right<LIM>(t1, t2, t3);
  const R lp = muscl_left<LIM>(p0, p1, p2);
  const R rp = muscl_right<LIM>(p1, p2, p3);

  const R lT = lp / (lroe * g.Rg);
  const R le = g.Cv * lT + R(0.5) * (lun * lun + lut * lut);
  const R rT = rp / (rroe * g.Rg);
  const R re = g.Cv * rT + R(0.5) * (run * run + rut * rut);
  const R lv = lun, rv = run;

  const R droe = rroe - lroe;
  const R dp = rp - lp;
  const R dut = rut - lut;
  const R dubar = rv - lv;

  // Roeaverage
  const R r2lroe = sqrt(rroe / lroe);
  const R r2l0 = R(1) / (R(1) + r2lroe);
  const R h_left = le + lp / lroe;
  const R h_right = re + rp / rroe;
  const R a_roe = sqrt(lroe * rroe);
  const R a_un = (lun + run * r2lroe) * r2l0;
  const R a_ut = (lut + rut * r2lroe) * r2l0;
  const R a_h = (h_left + h_right * r2lroe) * r2l0;
  const R a_c = sqrt(g.gm1 * (a_h - (a_un * a_un + a_ut * a_ut) / R(2)));
  const R ubar = a_un;

  // ComptFaceFlux
  const R csquare = a_c * a_c;
  const R namda3 = fabs(ubar);
  const R coef12 = R(1) / (R(2) * csquare) * area;
  const R roe0cxdubar = a_roe * a_c * dubar;
  const R faceareaxabsubar = area * namda3;
  const R halffacearea = R(0.5) * area;
  const R alpha0 = faceareaxabsubar * (droe - dp / csquare);
  // roe0c_coef (all-speed dissipation scaling)
  const R T_a = (lT + rT) * R(0.5);
  const R V_a = (lv + rv) * R(0.5);
  const R Ma_a = fabs(V_a / sqrt(g.gamaRg * T_a));
  const R f_Ma = smin(smax(Ma_a, g.Ma), R(1));
  const R s0 = (R(1) - f_Ma) * (R(1) - f_Ma);
  const R namda0 = sqrt(R(4) * a_c * a_c * f_Ma + s0 * ubar * ubar);
  const R namda1 = fabs(R(0.5) * ((R(1) + f_Ma) * ubar + namda0));
  const R namda2 = fabs(R(0.5) * ((R(1) + f_Ma) * ubar - namda0));
  const R alpha1 = coef12 * namda1 * (dp + roe0cxdubar);
  const R alpha2 = coef12 * namda2 * (dp - roe0cxdubar);
  const R alpha3 = alpha0 + alpha1 + alpha2;
  const R alpha4 = a_c * (alpha1 - alpha2);
  const R alphat = faceareaxabsubar * (a_roe * dut);

  // Get_inv_flux of both states
  const R pl0 = lroe * lv, pl1 = lroe * lun * lv + lp, pl2 = lroe * lut * lv;
  const R pl4 = (lp + le * lroe) * lv;
  const R pr0 = rroe * rv, pr1 = rroe * run * rv + rp, pr2 = rroe * rut * rv;
  const R pr4 = (rp + re * rroe) * rv;

  f_mass = -alpha3;
  f_n = -(a_un * alpha3 + alpha4);
  f_t = -(a_ut * alpha3 + alphat);
  f_e = -(a_h * alpha3 + ubar * alpha4 + a_ut * alphat - (csquare / g.gm1) * alpha0);
  f_mass += (pl0 + pr0) * halffacearea;
  f_n += (pl1 + pr1) * halffacearea;
  f_t += (pl2 + pr2) * halffacearea;
  f_e += (pl4 + pr4) * halffacearea;
}

// ---- fast builds ---------------------------------------------------------
// The same flux with every division and root replaced by the FastMath
// helpers and shared subexpressions hoisted (1/rho, 1/c^2); the MUSCL slopes
// come in precomputed (see limited_slope).  Not operation-for-operation the
// reference: agrees with it to a few units in the last place per face.

// Limited MUSCL slope of one cell from its backward difference a and forward
// difference b: the reference's left and right reconstructions
// (SlopeCorrection_Left/Right with VanLeer phi(r) = 2r/(1+r) or minmod
// phi(r) = min(r,1), r = b/a resp. a/b) both reduce to q +/- sigma with
//   VanLeer: sigma = a b / (a + b)            if a b > 0, else 0
//   minmod:  sigma = 0.5 * (|b| < |a| ? b : a) if a b > 0, else 0
template <int LIM, typename R>
__device__ __forceinline__ R limited_slope(R a, R b) {
  const R ab = a * b;
  if (LIM == LIM_MINMOD) return (ab > R(0)) ? R(0.5) * (fabs(b) < fabs(a) ? b : a) : R(0);
  if (sizeof(R) == 4) {
    // FP32: one MUFU reciprocal, cheaper than a branch; the select discards
    // the cases where a + b may vanish
    const R s = ab * FastMath<R>::rcp(a + b);
    return (ab > R(0)) ? s : R(0);
  }
  // FP64: the Newton-refined reciprocal is long, and uniform regions
  // (a = b = 0) skip it warp-wide
  if (!(ab > R(0))) return R(0);
  return ab * FastMath<R>::rcp1(a + b);
}

// The reference's explicit one-sided reconstructions, used for faces whose
// outer stencil cell is missing (its stencil then mixes sides).
template <int LIM, typename R>
__device__ __forceinline__ R muscl_left_fast(R q_i, R qi, R qi1) {
  R dqi = qi - q_i, dqii = qi1 - qi;
  R qr = FastMath<R>::div(dqii, dqi);
  if (fabs(qr) > R(1.0e10) || isnan(qr)) qr = (dqii > R(0)) ? R(1000000.0) : R(-1.0);
  if (qr <= R(0)) qr = R(0);
  R lv = (LIM == LIM_MINMOD) ? (qr < R(1) ? qr : R(1)) : FastMath<R>::div(R(2) * qr, R(1) + qr);
  return qi + R(0.5) * dqi * lv;
}
template <int LIM, typename R>
__device__ __forceinline__ R muscl_right_fast(R q_i, R qi, R qi1) {
  R dqi = qi - q_i, dqii = qi1 - qi;
  R qr = FastMath<R>::div(dqi, dqii);
  if (fabs(qr) > R(1.0e10) || isnan(qr)) qr = (dqi > R(0)) ? R(1000000.0) : R(-1.0);
  if (qr <= R(0)) qr = R(0);
  R lv = (LIM == LIM_MINMOD) ? (qr < R(1) ? qr : R(1)) : FastMath<R>::div(R(2) * qr, R(1) + qr);
  return qi - R(0.5) * dqii * lv;
}

// All-speed Roe flux from reconstructed left/right states (rho, u_n, u_t, p),
// restated with fewer operations than the reference's term order (same
// quantities, different rounding):
//   * one inverse root y = (rho_L rho_R)^-1/2 gives the Roe density
//     rho_L rho_R y, the ratio sqrt(rho_R / rho_L) = rho_R y, both inverse
//     densities (ratio y, rho_L y^2) and the Roe weights 1 / (1 + ratio),
//     ratio / (1 + ratio);
//   * Cv = Rg / (gama - 1) (FlowConstants.cpp), so the total enthalpy is
//     h = gama/(gama-1) p/rho + |u|^2/2, the energy flux (p + e rho) u_n is
//     rho u_n h, and Rg T = p / rho: no temperature is formed;
//   * c^2 / (gama - 1) in the energy dissipation is the bracket c^2 is made
//     from; the halves of the all-speed eigenvalues and of the central flux
//     go into the face area.
// halfarea = area / 2.
template <typename R>
__device__ __forceinline__ void roe_flux_states(const Gas<R> &g, R area, R halfarea, R lroe,
                                                R lun, R lut, R lp, R rroe, R run, R rut, R rp,
                                                R &f_mass, R &f_n, R &f_t, R &f_e) {
  typedef FastMath<R> M;
  const R prod = lroe * rroe;
  const R y = M::rsqrt(prod);
  const R a_roe = prod * y;                // sqrt(rho_L rho_R)
  const R ratio = rroe * y;                // sqrt(rho_R / rho_L)
  const R ilroe = ratio * y, irroe = (lroe * y) * y;
  const R lpr = lp * ilroe, rpr = rp * irroe;  // p / rho = Rg T
  const R lh = fma(g.gam_gm1, lpr, R(0.5) * fma(lun, lun, lut * lut));
  const R rh = fma(g.gam_gm1, rpr, R(0.5) * fma(run, run, rut * rut));
  const R droe = rroe - lroe, dp = rp - lp, dut = rut - lut, dubar = run - lun;
  // Roe averages w_L q_L + (1 - w_L) q_R = q_R - w_L (q_R - q_L): the
  // weights sum to one exactly
  const R wL = M::rcp(R(1) + ratio);
  const R a_un = fma(-wL, dubar, run);
  const R a_ut = fma(-wL, dut, rut);
  const R a_h = fma(-wL, rh - lh, rh);
  const R kin = fma(R(-0.5), fma(a_un, a_un, a_ut * a_ut), a_h);  // c^2 / (gama - 1)
  const R csquare = g.gm1 * kin;
  const R rc = M::rsqrt1(csquare);
  const R a_c = csquare * rc;
  const R icsq = rc * rc;
  const R ubar = a_un;
  const R coef12 = icsq * halfarea;
  const R roe0cxdubar = a_roe * a_c * dubar;
  const R faceareaxabsubar = area * fabs(ubar);
  const R alpha0 = faceareaxabsubar * fma(-dp, icsq, droe);
  // all-speed scaling: |V_a| / sqrt(gama Rg T_a) with V_a, T_a face means
  const R Ma_a = fabs(lun + run) * M::rsqrt1(g.two_gama * (lpr + rpr));
  const R f_Ma = smin(smax(Ma_a, g.Ma), R(1));
  const R hm = fma(R(-0.5), f_Ma, R(0.5)) * ubar;  // (1 - f) ubar / 2
  const R hp = fma(R(0.5), f_Ma, R(0.5)) * ubar;   // (1 + f) ubar / 2
  const R q = fma(hm, hm, csquare * f_Ma);          // (namda0 / 2)^2
  const R sq = q * M::rsqrt1(q);
  const R alpha1 = coef12 * fabs(hp + sq) * (dp + roe0cxdubar);
  const R alpha2 = coef12 * fabs(hp - sq) * (dp - roe0cxdubar);
  const R alpha3 = alpha0 + alpha1 + alpha2;
  const R alpha4 = a_c * (alpha1 - alpha2);
  const R alphat = faceareaxabsubar * (a_roe * dut);
  const R ml = lroe * lun, mr = rroe * run;  // mass fluxes of both states
  f_mass = fma(ml + mr, halfarea, -alpha3);
  f_n = fma(fma(ml, lun, lp) + fma(mr, run, rp), halfarea, -fma(a_un, alpha3, alpha4));
  f_t = fma(fma(ml, lut, mr * rut), halfarea, -fma(a_ut, alpha3, alphat));
  f_e = fma(fma(ml, lh, mr * rh), halfarea,
            -fma(a_h, alpha3, fma(ubar, alpha4, fma(a_ut, alphat, -kin * alpha0))));
}

// ---- paired flux: two faces per thread -----------------------------------
// The west and south faces of a cell evaluated together.  FP32 (mixed
// build): the lanes of a float2 through the sm_100 paired instructions
// (add/mul/fma .f32x2, one instruction per two operations).  FP64: two
// interleaved scalar chains, which doubles the independent work each warp
// has in flight.  Roots and reciprocals stay per lane.
struct F2 {
  float2 v;
};
struct D2 {
  double x, y;
};
__device__ __forceinline__ F2 pair(float a, float b) { return F2{make_float2(a, b)}; }
__device__ __forceinline__ D2 pair(double a, double b) { return D2{a, b}; }
__device__ __forceinline__ float lane0(F2 a) { return a.v.x; }
__device__ __forceinline__ float lane1(F2 a) { return a.v.y; }
__device__ __forceinline__ double lane0(D2 a) { return a.x; }
__device__ __forceinline__ double lane1(D2 a) { return a.y; }
__device__ __forceinline__ F2 operator+(F2 a, F2 b) { return F2{__fadd2_rn(a.v, b.v)}; }
__device__ __forceinline__ F2 operator-(F2 a, F2 b) {
  return F2{__fadd2_rn(a.v, make_float2(-b.v.x, -b.v.y))};
}
__device__ __forceinline__ F2 operator*(F2 a, F2 b) { return F2{__fmul2_rn(a.v, b.v)}; }
__device__ __forceinline__ F2 fma2(F2 a, F2 b, F2 c) { return F2{__ffma2_rn(a.v, b.v, c.v)}; }
__device__ __forceinline__ D2 operator+(D2 a, D2 b) { return D2{a.x + b.x, a.y + b.y}; }
__device__ __forceinline__ D2 operator-(D2 a, D2 b) { return D2{a.x - b.x, a.y - b.y}; }
__device__ __forceinline__ D2 operator*(D2 a, D2 b) { return D2{a.x * b.x, a.y * b.y}; }
__device__ __forceinline__ D2 fma2(D2 a, D2 b, D2 c) { return D2{fma(a.x, b.x, c.x), fma(a.y, b.y, c.y)}; }
template <typename P>
__device__ __forceinline__ P abs2(P a) {
  return pair(fabs(lane0(a)), fabs(lane1(a)));
}
template <typename P>
__device__ __forceinline__ P rsqrt2(P a) {
  typedef decltype(lane0(a)) S;
  return pair(FastMath<S>::rsqrt1(lane0(a)), FastMath<S>::rsqrt1(lane1(a)));
}
template <typename P>
__device__ __forceinline__ P rcp2(P a) {
  typedef decltype(lane0(a)) S;
  return pair(FastMath<S>::rcp1(lane0(a)), FastMath<S>::rcp1(lane1(a)));
}
template <typename P, typename S>
__device__ __forceinline__ P clamp2(P a, S lo, S hi) {
  return pair(smin(smax(lane0(a), lo), hi), smin(smax(lane1(a), lo), hi));
}

// roe_flux_states for two faces at once (same arithmetic, paired).
template <typename P, typename S>
__device__ __forceinline__ void roe_flux_pair(const Gas<S> &g, P area, P lroe, P lun, P lut, P lp,
                                              P rroe, P run, P rut, P rp, P &f_mass, P &f_n,
                                              P &f_t, P &f_e) {
  const P half = pair(S(0.5), S(0.5)), one = pair(S(1), S(1)), mhalf = pair(S(-0.5), S(-0.5));
  const P halfarea = half * area;
  const P prod = lroe * rroe;
  const P y = rsqrt2(prod);
  const P a_roe = prod * y;
  const P ratio = rroe * y;
  const P ilroe = ratio * y, irroe = (lroe * y) * y;
  const P lpr = lp * ilroe, rpr = rp * irroe;
  const P gg = pair(g.gam_gm1, g.gam_gm1);
  const P lh = fma2(gg, lpr, half * fma2(lun, lun, lut * lut));
  const P rh = fma2(gg, rpr, half * fma2(run, run, rut * rut));
  const P droe = rroe - lroe, dp = rp - lp, dut = rut - lut, dubar = run - lun;
  const P mwL = pair(S(0), S(0)) - rcp2(one + ratio);  // -w_L
  const P a_un = fma2(mwL, dubar, run);
  const P a_ut = fma2(mwL, dut, rut);
  const P a_h = fma2(mwL, rh - lh, rh);
  const P kin = fma2(mhalf, fma2(a_un, a_un, a_ut * a_ut), a_h);
  const P csquare = pair(g.gm1, g.gm1) * kin;
  const P rc = rsqrt2(csquare);
  const P a_c = csquare * rc;
  const P icsq = rc * rc;
  const P ubar = a_un;
  const P coef12 = icsq * halfarea;
  const P roe0cxdubar = a_roe * a_c * dubar;
  const P faceareaxabsubar = area * abs2(ubar);
  const P alpha0 = faceareaxabsubar * (droe - dp * icsq);
  const P Ma_a = abs2(lun + run) * rsqrt2(pair(g.two_gama, g.two_gama) * (lpr + rpr));
  const P f_Ma = clamp2(Ma_a, g.Ma, S(1));
  const P hm = fma2(mhalf, f_Ma, half) * ubar;
  const P hp = fma2(half, f_Ma, half) * ubar;
  const P q = fma2(hm, hm, csquare * f_Ma);
  const P sq = q * rsqrt2(q);
  const P alpha1 = coef12 * abs2(hp + sq) * (dp + roe0cxdubar);
  const P alpha2 = coef12 * abs2(hp - sq) * (dp - roe0cxdubar);
  const P alpha3 = alpha0 + alpha1 + alpha2;
  const P alpha4 = a_c * (alpha1 - alpha2);
  const P alphat = faceareaxabsubar * (a_roe * dut);
  const P ml = lroe * lun, mr = rroe * run;
  f_mass = (ml + mr) * halfarea - alpha3;
  f_n = (fma2(ml, lun, lp) + fma2(mr, run, rp)) * halfarea - fma2(a_un, alpha3, alpha4);
  f_t = fma2(ml, lut, mr * rut) * halfarea - fma2(a_ut, alpha3, alphat);
  f_e = fma2(ml, lh, mr * rh) * halfarea -
        (fma2(a_h, alpha3, fma2(ubar, alpha4, a_ut * alphat)) - kin * alpha0);
}

}  // namespace ibgpu
