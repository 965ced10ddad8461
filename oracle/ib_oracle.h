/*
 * CPU restatement of the reference solver's explicit time step (test
 * infrastructure only: used by tests/ to test the GPU path and by bench.py's
 * cpu_baseline leg; never linked into the GPU library).
 *
 * Data model: each AMR level is a dense (ix, iy) index box; a slot is present
 * when the reference holds a box at that position on the z = 0 plane.  The
 * reference's one-cell-thick z slab (Userfunction_cy_naca15.cpp:35-36) is
 * restated in 2-D: every z term it evaluates is multiplied by an exact zero
 * (NS_Solver.H:712-831, NS_Solver.cpp:426-583), so the 2-D restatement gives
 * the same numbers.  Arithmetic follows the reference expression by
 * expression, in the same evaluation order, in FP64 with no contraction.
 */
#ifndef IB_ORACLE_H
#define IB_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* slot flags */
enum {
  IBO_PRESENT = 1,     /* the reference holds a box here                        */
  IBO_NORMAL = 2,      /* leaf cell: in the level's normal range [0,size)       */
  IBO_UPDATE = 4,      /* UpdateConsVars computes cv_new (and checks rho < 0)    */
  IBO_PRIM = 8,        /* ComptNewPrimVar: prim <- Get_Prim_Vars(cv_new)        */
  IBO_RESET = 16,      /* ComptNewPrimVar: prim <- initvar                       */
  IBO_RESNORM = 32     /* counted by ResinDomain                                 */
};

enum { IBO_LIM_VANLEER = 0, IBO_LIM_MINMOD = 1 };

typedef struct ibo_params {
  double gama, Rg, Cv, Ma, Re, qk, s_over_t, cfl, dt_ratio;
  double tp[4];
  double initvar[7]; /* roe u v w p T e */
  int nstages;
  int limiter;
  int viscous;
  int dt_var_step;
  int body_level;    /* finest level of a run with bodies, or -1 */
} ibo_params;

typedef struct ibo_level {
  int x0, y0, nx, ny;        /* slot(ix,iy) = (iy - y0) * nx + (ix - x0)        */
  double dx, dy, dz;
  int march_step, march_left;
  double step_num;           /* dt multiplier of this level (subcycling)         */
  uint8_t *flags;
  double *q[7];              /* roe u v w p T e per slot                         */
  int ncopy;                 /* periodic/block ghost refresh: q[dst] <- q[src]   */
  const int32_t *copy_dst;
  const int32_t *copy_src;
} ibo_level;

/* One full time step of the levels in `lev` (reference call order,
 * main.cpp:87-97 and NS_Solver.H:657-702): block-ghost exchange, CFL dt
 * (every dt_var_step steps), U^n, viscous flux (frozen), S stages of
 * flux -> residual -> update -> prim recovery with an exchange between
 * stages, residual max-norm.  Returns 0, or the reference's abort code
 * (523 rho < 0, 611 rho < 0 on the body level, 37 T < 0, 424 dt < 0,
 * 268 NaN residual), checked in the reference's order. */
int ibo_step(const ibo_params *P, ibo_level *lev, int nlev, int ts, double *dt,
             double *cfl_dt, double res_max[5]);

/* CFL time step of the normal cells of all levels (NS_Solver.cpp:196-280). */
int ibo_cfl_dt(const ibo_params *P, const ibo_level *lev, int nlev, double *cfl_dt);

#ifdef __cplusplus
}
#endif

#endif
