/*
 * ibgpu — C ABI of the B200 explicit time step for the cell-based AMR
 * compressible Navier-Stokes solver (2-D, immersed bodies).
 *
 * The GPU step replaces, for one time step of the reference solver:
 *   NS_Solver::TimeMarching       (NS_Solver.H:657-702)
 *   AMR::InterfaceExchange         (AMRInterface.cpp:3-35)
 *   the per-cell part of Body::IBConditions_Image (Body.cpp:1361-1496)
 * called from the reference main loop (main.cpp:87, 89, 97).  The host keeps
 * the mesh (topology is built and regridded by the reference's Mesh/AMR
 * classes on the host); the device owns the flow state between regrids.
 *
 * Conventions
 *   - Plain C types only; every pointer is host memory unless a name says
 *     otherwise; sizes are element counts.
 *   - Every call returns IBGPU_OK (0) or a negative IBGPU_E* code; the
 *     solver's own abort conditions are reported as the reference's abort
 *     code (e.g. 523 for negative density) through ibgpu_diag.abort_code and
 *     the return value IBGPU_E_ABORT.  The library never exits the process.
 *   - One context = one CUDA stream; a context is not re-entrant.
 *   - Primitive state rows are the reference's FlowVariables layout
 *     (FlowVariables.H:235-334): roe, u, v, w, p, T, e  (7 doubles per cell).
 */
#ifndef IBGPU_H
#define IBGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define IBGPU_ABI_VERSION 1
#define IBGPU_MAX_LEVELS 16

/* return codes */
#define IBGPU_OK 0
#define IBGPU_E_ARG (-1)       /* invalid argument / inconsistent input        */
#define IBGPU_E_CUDA (-2)      /* CUDA runtime error (see ibgpu_last_error)     */
#define IBGPU_E_STATE (-3)     /* call order (e.g. step before upload)         */
#define IBGPU_E_ABORT (-4)     /* solver abort condition, see ibgpu_diag        */
#define IBGPU_E_NOMEM (-5)     /* device allocation failed                     */
#define IBGPU_E_TOPOLOGY (-6)  /* cell list cannot be laid out (e.g. periodic
                                  extent not a multiple of the tile edge)      */
#define IBGPU_E_TIMEOUT (-7)   /* a device-side wait ran out of its time limit;
                                  the kernel released its resources and the
                                  context stays usable                         */

/* limiter (Slopelimiter.H): VanLeer is the reference's active ALimiter */
#define IBGPU_LIM_VANLEER 0
#define IBGPU_LIM_MINMOD 1

/* arithmetic of the flux/limiter/viscous kernels */
#define IBGPU_FP64 0        /* FP64 throughout (contracted multiply-adds)       */
#define IBGPU_FP64_EXACT 1  /* FP64, no contraction: reproduces the reference
                               operation by operation                            */
#define IBGPU_MIXED 2       /* FP32 flux/limiter/viscous; FP64 accumulation of
                               conserved variables, pressure recovery, dt,
                               residual and forces                               */

/* per-cell flags of the canonical cell list (same meaning as the reference
 * code paths they select; see ibgpu_cells) */
#define IBGPU_CELL_PRESENT 1  /* a box of the level exists at (ix, iy)          */
#define IBGPU_CELL_NORMAL 2   /* leaf cell (the level's normal range [0,size))  */
#define IBGPU_CELL_UPDATE 4   /* UpdateConsVars computes cv_new (rho<0 check)   */
#define IBGPU_CELL_PRIM 8     /* ComptNewPrimVar: prim <- Get_Prim_Vars(cv_new)*/
#define IBGPU_CELL_RESET 16   /* ComptNewPrimVar: prim <- initvar              */
#define IBGPU_CELL_RESNORM 32 /* counted by ResinDomain                         */
#define IBGPU_CELL_ALIAS 64   /* periodic/block ghost: a copy of the cell at the
                                 wrapped position (Mesh::DataExchange); it gets
                                 no storage of its own                         */

typedef struct ibgpu_case {
  int abi_version; /* IBGPU_ABI_VERSION */
  /* non-dimensional gas constants (FlowConstants.cpp:5-44) */
  double gama, Rg, Cv, Cp, Ma, Re, Pr, qk, s_over_t;
  /* time step control (NS_Solver.cpp:196-280; case globals) */
  double cfl, dt_ratio;
  int dt_var_step;
  /* multistage scheme U^(k) = U^n + tp[k] dt R(U^(k-1)) (NS_Solver.H:200-231) */
  int nstages;
  double tp[4];
  int limiter;   /* IBGPU_LIM_* */
  int viscous;   /* 1: ComptViscousStress terms (frozen per step)      */
  int precision; /* IBGPU_FP64 / IBGPU_FP64_EXACT / IBGPU_MIXED        */
  double initvar[7];
  /* levels (AMRSpaceTime.H, mpiparams.cpp:134-212) */
  int nlevels;
  double dh[IBGPU_MAX_LEVELS][3];
  int march_step[IBGPU_MAX_LEVELS], march_left[IBGPU_MAX_LEVELS];
  double step_num[IBGPU_MAX_LEVELS];
  /* domain: level-0 cell counts and periodicity; level l spans n*2^l */
  int domain_nx, domain_ny;
  int periodic_x, periodic_y;
  /* coarse/fine schedule of the pair (l-1, l), indexed by the fine level l
   * (AMRInterface.cpp:8-30, mpiparams.cpp:186-212): restriction when
   * ts % average_step[l] == average_left[l], prolongation likewise */
  int average_step[IBGPU_MAX_LEVELS], average_left[IBGPU_MAX_LEVELS];
  int prolong_step[IBGPU_MAX_LEVELS], prolong_left[IBGPU_MAX_LEVELS];
  /* finest level of a run with immersed bodies (its leaf-cell branches and
   * abort code 611 differ, NS_Solver.cpp:146-190, 946-984), -1 without */
  int body_level;
  /* reference scales of the wall-force output (Body.cpp:546-552) and the
   * viscosity mu of the wall shear (FlowConstants.cpp) */
  double p_ref, area_ref, shear_ref, L_ref, mu;
} ibgpu_case;

/* Canonical cell list: one row per box of the z = 0 plane of each level
 * (normal cells and 2-D ghosts), keyed by (level, ix, iy).  Replaces the
 * reference's per-level AoS arrays Meshlevel::m_box / m_data
 * (Meshlevel.H:688-872, Box.H:113-300) as the device's input. */
typedef struct ibgpu_cells {
  int64_t n;
  const int32_t *level;
  const int32_t *ix;
  const int32_t *iy;
  const uint8_t *flags; /* IBGPU_CELL_* */
} ibgpu_cells;

/* Coarse/fine pairs.  Restriction pair (AMRLevel::f_res_ghost): the coarse
 * ghost at (cx, cy) on level `level` takes the density-weighted average of
 * its four sons on level+1 (TwoLevelOp.H:67-87, 225-231).  Prolongation pair
 * (AMRLevel::f_pro_ghost, g_pro): the four sons of the coarse leaf cell are
 * fine ghosts reconstructed from its conserved variables and central
 * gradients (TwoLevelOp.H:16-22, 35-43, 200-215).  Sons are given explicitly,
 * in the order (0,0), (0,1), (1,0), (1,1) of (x, y) offsets. */
typedef struct ibgpu_cf_pairs {
  int64_t nres;
  const int32_t *res; /* nres x 11: level, cx, cy, then 4 x (fx, fy) */
  int64_t npro;
  const int32_t *pro; /* npro x 11: same layout */
} ibgpu_cf_pairs;

/* Domain ghosts in the reference's processing order per level
 * (BCValues::BCBoxTreat, BCValues.H:51-188).  type is the face's boundary
 * type (-99 periodic, -50 outflow copy, -51 slip wall, -49/-46/-42 no-slip,
 * -45 fixed velocity, -13 pressure inlet, -12 pressure outlet, -10 fixed). */
typedef struct ibgpu_bc {
  int64_t n;
  const int32_t *ghost; /* n x 7: level, x, y, ref_x, ref_y, face, type */
  const double *nmv;    /* n x 3: wall normal of type -51 ghosts (or NULL) */
  int nfaces;
  const double *facevar; /* nfaces x 7: BCValues::facevar rows */
  double backpressure;
  double inlet_flow_angle;
} ibgpu_bc;

/* Immersed-boundary ghost cells of the finest level (IBCell,
 * Body::IBConditions_Image, Body.cpp:1361-1496) and wall patches
 * (Surfpatch, Body::ComptWallForce, Body.cpp:439-558).  The eight
 * interpolation cells and weights are the reference's [2][2][2] image-point
 * stencil in its order; in the one-cell-thick slab the z neighbours are the
 * same 2-D cells. */
typedef struct ibgpu_ib {
  int64_t ncells;
  const int32_t *cell;  /* ncells x 18: x, y, then 8 x (x, y) of the stencil */
  const double *cellf;  /* ncells x 16: signdis, hgdis, 8 weights, normal(3),
                           wall velocity(3) */
  int64_t npatches;
  const int32_t *patch; /* npatches x 17: body, then 8 x (x, y) */
  const double *patchf; /* npatches x 19: centre(3), normal(3), area, hgdis,
                           8 weights, wall velocity(3) */
  int nbodies;
  const double *body_center; /* nbodies x 3 */
} ibgpu_ib;

typedef struct ibgpu_diag {
  double dt;          /* dt used by this step                                */
  double cfl_dt;      /* CFL time step (NS_Solver.cpp:262), when evaluated   */
  double res_max[5];  /* ResinDomain max-norm of the residual (unnormalised) */
  int abort_code;     /* reference abort code, 0 if none                     */
  int abort_level, abort_ix, abort_iy;
  int abort_step;     /* index of the aborting step within an ibgpu_run      */
  int64_t cells_marched; /* leaf cells of the levels that marched           */
} ibgpu_diag;

typedef struct ibgpu_ctx ibgpu_ctx;

/* Create a context on the current CUDA device.  Replaces the NS_Solver
 * constructor (NS_Solver.H:192-236) plus the case globals it reads. */
int ibgpu_create(const ibgpu_case *cs, ibgpu_ctx **out);

/* Run the context's work on an existing CUDA stream (cudaStream_t passed as
 * a pointer); NULL restores the context's own stream. */
int ibgpu_set_stream(ibgpu_ctx *ctx, void *stream);

/* Upload the mesh as a cell list; lays the levels out as Morton-ordered
 * 16x16 tiles.  Call again after every regrid (AMR::PerformAdaptive). */
int ibgpu_upload_topology(ibgpu_ctx *ctx, const ibgpu_cells *cells);

/* Coarse/fine pairs, domain ghosts and immersed-boundary records; call after
 * ibgpu_upload_topology (each replaces the previous upload of its kind). */
int ibgpu_upload_interfaces(ibgpu_ctx *ctx, const ibgpu_cf_pairs *pairs);
int ibgpu_upload_boundaries(ibgpu_ctx *ctx, const ibgpu_bc *bc);
int ibgpu_upload_ib(ibgpu_ctx *ctx, const ibgpu_ib *ib);

/* ---------------------------------------------------------------------------
 * Wall distances of moved bodies, on the device: the first part of the
 * reference's re-immersion (Body::RenewLevelDistance, Bodymove.cpp:127-300),
 * with the block-ghost copies of Mesh::SynNormal_BlockDistance
 * (Mesh.cpp:2303-2374).  For every box of a level closer than 9.5 to a wall
 * (and not a block ghost): the closest wall patch of its body by the
 * reference's walk over neighbouring patches from the box's current patch
 * (Body::FindClosePatchtoCell, Body.H:505-580), the hand-over to another
 * body where a neighbour box is paired with it, the signed distance capped
 * by the distance to the domain boundary, and the solid flag with the boxes
 * that changed sides; then every block ghost takes its origin box's pair.
 * The same IEEE operations in the same order as the reference (no
 * contractions, correctly rounded roots): results equal the reference's bit
 * for bit.  The geometry is uploaded after every regrid, the pairs go in and
 * out with every call.
 * ------------------------------------------------------------------------- */
#define IBGPU_WALL_BOX_OTHER 0        /* normal cells and other ghosts */
#define IBGPU_WALL_BOX_DOMAIN_GHOST 1 /* Boxtype Dmghost */
#define IBGPU_WALL_BOX_BLOCK_GHOST 2  /* Boxtype Blockghost */
#define IBGPU_WALL_MAX_NB 15          /* neighbours per wall patch (PatchNeib) */
#define IBGPU_WALL_INTO_BODY 1        /* the box joined the body (solid)      */
#define IBGPU_WALL_OUT_OF_BODY 2      /* the box left it                       */

typedef struct ibgpu_wall_level_geom {
  int64_t n;                    /* boxes of the level, in its array order    */
  const double *center;         /* 3 per box (Meshlevel m_geom boxcenter)    */
  const int32_t *neib;          /* 9 per box: Box::neib[i][j][1], i-major    */
  const uint8_t *kind;          /* IBGPU_WALL_BOX_*                          */
  const double *distance_to_dm; /* BoxtoWall::distance_to_dm                 */
  int64_t nblock;               /* block pairs (Meshlevel blockpair)         */
  const int32_t *block_in;      /* origin box of pair k (innode)             */
  const int32_t *block_out;     /* block ghost of pair k (outnode.index)     */
} ibgpu_wall_level_geom;

/* After every regrid: the boxes of every level.  IBGPU_E_ARG when a block
 * ghost is the target of two pairs or the origin of one (the geometry held
 * before stays), or when a neighbour index lies outside its level's boxes
 * (checked on the device after the copies: the context then holds no wall
 * geometry until the next call). */
int ibgpu_wall_geometry(ibgpu_ctx *ctx, int nlevels, const ibgpu_wall_level_geom *levels);

typedef struct ibgpu_wall_bodies {
  int nbodies;
  const int32_t *patch_start; /* nbodies + 1: body b's patches are rows
                                 patch_start[b] .. patch_start[b+1]-1       */
  const double *pc;           /* 3 per patch row: centre                    */
  const double *nv;           /* 3 per patch row: unit outward normal       */
  const int32_t *nb_count;    /* per patch row                              */
  const int32_t *nb;          /* IBGPU_WALL_MAX_NB per patch row: the body's
                                 neighbouring patches (indices within the body) */
  int periodic_y;             /* PeriodicLength (mpiparams.cpp:294-310)     */
  double critic_ylength, dm_length_y;
} ibgpu_wall_bodies;

typedef struct ibgpu_wall_pairs {  /* one level; in and out (BoxtoWall, Box::solid) */
  int32_t *body, *patch;
  double *distance, *signdis, *distance_to_body;
  uint8_t *solid;
  uint8_t *moved;        /* out, per box: IBGPU_WALL_INTO_BODY / _OUT_OF_BODY / 0,
                            the reference's move lists of its distance loop */
  uint8_t *block_moved;  /* out, per block pair: the same for block_out[k] */
} ibgpu_wall_pairs;

/* Pin (and release) a host buffer that ibgpu calls copy from or to, e.g. the
 * shared windows the binding exchanges wall distances through
 * (cudaHostRegister / cudaHostUnregister on the current device): its
 * transfers then run at the bus rate instead of through staging. */
int ibgpu_host_register(void *ptr, size_t bytes);
int ibgpu_host_unregister(void *ptr);

/* The bodies where they are now and every level's pairs as the last move
 * left them; on return the new pairs.  The device keeps the new pairs: with
 * IBGPU_WALL_RESIDENT in flags the call starts from them (the previous
 * call's results) and reads none of the arrays, only writes them, which
 * saves the upload when nothing else changed the pairs since.
 * IBGPU_E_ABORT when a box within 9.5 of a wall has no valid body or patch
 * (the reference's assertion, Bodymove.cpp:146-147); IBGPU_E_STATE before
 * ibgpu_wall_geometry, or with IBGPU_WALL_RESIDENT before a first call
 * after it. */
#define IBGPU_WALL_RESIDENT 1
int ibgpu_wall_distance(ibgpu_ctx *ctx, const ibgpu_wall_bodies *bodies, int nlevels,
                        ibgpu_wall_pairs *pairs, int flags);

/* One box of a level in the output of ibgpu_wall_distance_near. */
typedef struct ibgpu_wall_change {
  int32_t box;           /* index of the box in its level */
  int32_t body, patch;
  uint8_t solid;
  uint8_t moved;         /* IBGPU_WALL_INTO_BODY / _OUT_OF_BODY / 0 */
  uint8_t pad_[2];
  double distance, signdis, distance_to_body;
} ibgpu_wall_change;     /* 40 bytes */

typedef struct ibgpu_wall_near { /* one level */
  double band;                 /* in: a box is reported when |signdis| < band
                                  before or after the move, or it changed sides */
  int64_t capacity;            /* in: entries `changes` holds */
  ibgpu_wall_change *changes;  /* out: the reported boxes, in box order */
  int64_t count;               /* out: the number reported */
  uint8_t *block_moved;        /* out, per block pair, as in ibgpu_wall_pairs */
} ibgpu_wall_near;

/* ibgpu_wall_distance from the pairs the device holds (as with
 * IBGPU_WALL_RESIDENT), returning per level only the boxes near a wall
 * before or after the move and those that changed sides (what a host
 * re-immersion reads before the next move: a small part of the level)
 * instead of every box.  The device keeps every new pair either way.
 * IBGPU_E_ARG when a level reports more boxes than its capacity (count
 * then says how many; the pairs have moved on: ibgpu_wall_fetch has them
 * all); the other codes as ibgpu_wall_distance. */
int ibgpu_wall_distance_near(ibgpu_ctx *ctx, const ibgpu_wall_bodies *bodies, int nlevels,
                             ibgpu_wall_near *levels);

/* Every level's pairs and solid flags as the device holds them after its
 * last wall-distance call (the moved and block_moved arrays are not
 * written).  IBGPU_E_STATE when there are none since the geometry upload. */
int ibgpu_wall_fetch(ibgpu_ctx *ctx, int nlevels, ibgpu_wall_pairs *pairs);

/* Wall force and moment of every body from the current state
 * (Body::ComptWallForce): out[6*b + 0..2] force, out[6*b + 3..5] moment,
 * in the reference's dimensional scaling. */
int ibgpu_wall_forces(ibgpu_ctx *ctx, double *out);

/* New per-cell flags for the rows of the last topology upload (same rows,
 * same order), for a body that moved without a regrid: the moved body
 * changes which cells lie inside it, which are immersed-boundary cells and
 * which update (the branches IBGPU_CELL_UPDATE / PRIM / RESET / RESNORM
 * select), while the mesh stays.  Replaces the flag part of the
 * re-immersion in Body::MovingBody_Image (Bodymove.cpp:37-125: wall
 * distances, removed and newly infected immersed-boundary cells); the new
 * immersed-boundary records go through ibgpu_upload_ib.  A row whose
 * PRESENT, NORMAL or ALIAS bit differs from the topology upload gives
 * IBGPU_E_TOPOLOGY (that needs ibgpu_upload_topology).  The state stays. */
int ibgpu_update_flags(ibgpu_ctx *ctx, const uint8_t *flags);

/* The same for some of the rows: row rows[k] (an index into the rows of the
 * last topology upload) gets flags[k], every other row keeps its flags.  A
 * move changes the flags of the rows near the walls only, so a caller that
 * knows them sends those (a row may appear twice with the same flags).
 * IBGPU_E_ARG for a row index out of range; the other codes as
 * ibgpu_update_flags, and nothing changes on the device when one fails. */
int ibgpu_update_flags_rows(ibgpu_ctx *ctx, int64_t n, const int64_t *rows,
                            const uint8_t *flags);

/* Coarse/fine interface lists of an AMR mesh from its leaf cells, built on
 * the device: the part of the regrid's list rebuild (AMR::PerformAdaptive,
 * AMR.cpp:6-209; TagRefineGhost, AMRGhost_refine.cpp:30-98; the pair lists
 * f_res_ghost, f_pro_ghost and g_pro of AMRLevel.H:320-329) that follows
 * from which cells are leaves.  With refined(l) the level-l positions whose
 * sons are leaves or refined:
 *   restriction pair of level l, layer 0: a refined position whose four sons
 *     are leaves and with a leaf of level l among its 8 neighbours; layer 1:
 *     not layer 0, four leaf sons, a leaf of level l two steps away along x
 *     or y (rows: level, layer, cx, cy, 4 x (fx, fy));
 *   prolongation pair of level l: a leaf of level l with a refined position
 *     among its 8 neighbours (rows: level, cx, cy, 4 x (fx, fy));
 *   interface ghost cells (rows: level, ix, iy): the restriction positions of
 *     each level and the sons of the prolongation pairs of the level below;
 * sons in the order (0,0), (0,1), (1,0), (1,1) of (x, y) offsets, rows sorted
 * by level, then y, then x.  leaves->flags is not read.  The counts are
 * always set; when a capacity is below its count (a first call with zero
 * capacities asks for the counts) nothing is written and the call returns
 * IBGPU_E_ARG.  ctx supplies the stream (no topology needed). */
typedef struct ibgpu_interface_lists {
  int64_t nres, npro, nghost;          /* counts, set by the call            */
  int64_t cap_res, cap_pro, cap_ghost; /* rows the arrays below can hold     */
  int32_t *res;   /* cap_res x 12   */
  int32_t *pro;   /* cap_pro x 11   */
  int32_t *ghost; /* cap_ghost x 3  */
} ibgpu_interface_lists;
int ibgpu_build_interfaces(ibgpu_ctx *ctx, int nlevels, const ibgpu_cells *leaves,
                           ibgpu_interface_lists *out);

/* Number of device cell slots and tiles after the last topology upload. */
int ibgpu_layout_info(const ibgpu_ctx *ctx, int64_t *nslots, int64_t *ntiles);

/* State in cell-list order, 7 doubles per cell (FlowVariables layout).
 * Upload replaces NS_Solver::InitFlow (NS_Solver.H:432-446) / a restart;
 * alias rows are ignored on upload and filled from their source on
 * download. */
int ibgpu_upload_state(ibgpu_ctx *ctx, const double *prim);
int ibgpu_download_state(ibgpu_ctx *ctx, double *prim);

/* Row format of every state transfer of the context (ibgpu_upload_state,
 * ibgpu_download_state and their asynchronous forms) from the next call on:
 * IBGPU_ROWS_FLOWVARS (the default) moves the 7 doubles above per cell;
 * IBGPU_ROWS_COMPACT moves 4, (roe, u, v, p), 43 % fewer bytes for a caller
 * that hands the state over every step.  A compact upload derives T and e as
 * the reference derives them from those four (Get_T_ideal_gas,
 * Get_E, FlowVariables.H:19-33); a compact download leaves them out.  Waits
 * for transfers in flight. */
#define IBGPU_ROWS_FLOWVARS 7
#define IBGPU_ROWS_COMPACT 4
int ibgpu_set_state_rows(ibgpu_ctx *ctx, int fields);

/* Download without waiting: the copy runs on the context's copy stream after
 * the work enqueued so far, so it overlaps later uploads and steps (work
 * that writes the state waits for it on the device).  prim (pinned host
 * memory for real overlap) holds the state once ibgpu_synchronize returns. */
int ibgpu_download_state_async(ibgpu_ctx *ctx, double *prim);
/* Wait for all work and copies of the context. */
int ibgpu_synchronize(ibgpu_ctx *ctx);

/* One full time step at step index ts (main.cpp:87-97): C/F ghost fill,
 * immersed-body ghost fill, CFL dt every dt_var_step steps, U^n, domain
 * ghosts, frozen viscous flux, nstages stages, residual max-norm.
 * *dt is the current dt on entry and the dt used on return (dt =
 * min(CFL_dt, dt*dt_ratio), NS_Solver.cpp:263).  diag may be NULL. */
int ibgpu_step(ibgpu_ctx *ctx, int ts, double *dt, ibgpu_diag *diag);

/* nsteps consecutive steps ts0, ts0+1, ... enqueued back to back with one
 * host synchronisation at the end: dt stays on the device between steps,
 * diag reports the last step's reductions and the first abort (with its
 * step index; the steps after an abort run on but their state is invalid). */
int ibgpu_run(ibgpu_ctx *ctx, int ts0, int nsteps, double *dt, ibgpu_diag *diag);

/* Pipelined stepping for callers that hand the state over every step (a host
 * that keeps the authoritative copy, a coupling loop): nothing here waits on
 * the host, so the copies of one step overlap the compute of its neighbours.
 *   ibgpu_upload_state_async: ibgpu_upload_state without waiting; the copy
 *     runs on the context's upload stream, the scatter into the state after
 *     the work enqueued so far.  prim (pinned for real overlap) must stay
 *     unchanged until the next ibgpu_synchronize or ibgpu_step_result.
 *   ibgpu_step_async: one ibgpu_step of step index ts enqueued; the first one
 *     after a result (or ever) starts from *dt = dt, later ones continue
 *     from the dt the device computed (CFL pass every step, as ibgpu_step).
 *   ibgpu_step_result: waits for the context's stream and reports the last
 *     asynchronous step's dt and diag, with the first abort of the chain (its
 *     step counted from the chain's first step).
 * The results equal those of the synchronous calls bit for bit.  ibgpu_step
 * and ibgpu_run return IBGPU_E_STATE while a chain is open; at most 2^20
 * asynchronous steps per result. */
int ibgpu_upload_state_async(ibgpu_ctx *ctx, const double *prim);
int ibgpu_step_async(ibgpu_ctx *ctx, int ts, double dt);
int ibgpu_step_result(ibgpu_ctx *ctx, double *dt, ibgpu_diag *diag);

/* Event timing of the dominant kernels, accumulated while enabled:
 * kernel 0 = stage update (flux + residual + update + prim recovery),
 * 1 = viscous flux, 2 = CFL dt.  ms_out[k] total milliseconds,
 * launches_out[k] launch count. */
int ibgpu_set_kernel_timing(ibgpu_ctx *ctx, int enable);
int ibgpu_kernel_times(const ibgpu_ctx *ctx, double ms_out[3], int64_t launches_out[3]);

void ibgpu_destroy(ibgpu_ctx *ctx);

/* ---------------------------------------------------------------------------
 * Batched independent cases (no counterpart in the reference, which runs one
 * case per process): several contexts, each with its own mesh, state and
 * case constants, advance together.  Every step runs each case's ghost
 * fills and viscous pass, one CFL launch over the cases whose pass is due,
 * then ONE persistent launch per stage covering the marching tiles of all
 * cases (a work list of (case, tile) pairs per subcycling phase, cases
 * interleaved).  The whole step is captured once per schedule phase in a
 * CUDA graph (the cases' ghost fills on parallel branches) and replayed;
 * the captures happen at the start of the first run.  On the first run an
 * autotuner times the candidate shapes of the merged stage launch (CTA
 * count: one CTA per work item or 1-4 / 1-6 persistent CTAs per SM; block:
 * 256 or 288 threads) and keeps the fastest.  The cases must agree on precision (IBGPU_FP64 or
 * IBGPU_MIXED), limiter, viscosity, stage count and coefficients; their CFL
 * intervals (dt_var_step) may differ when each divides the longest marching
 * step of the batch (each case then takes its CFL pass on its own steps, as
 * meshes of different depths do); the batch runs on the first context's
 * stream.  Uploads to a context (topology,
 * lists) invalidate a batch that holds it: destroy and recreate it.  A batch
 * is destroyed before any context it holds.
 * ------------------------------------------------------------------------- */
typedef struct ibgpu_batch ibgpu_batch;
int ibgpu_batch_create(ibgpu_ctx *const *cases, int ncases, ibgpu_batch **out);
/* nsteps steps of every case from step index ts0; dt[i] and diag[i] (diag
 * may be NULL) as in ibgpu_run for case i.  Returns the first case's
 * non-OK code, IBGPU_OK when every case ran clean. */
int ibgpu_batch_run(ibgpu_batch *b, int ts0, int nsteps, double *dt, ibgpu_diag *diag);
/* CTA count of the merged stage launches from the next run on: 0 = one CTA
 * per work item, > 0 = that many persistent CTAs, -1 = chosen by the
 * autotuner at the next run (the default). */
int ibgpu_batch_set_grid(ibgpu_batch *b, int grid);
/* Threads per CTA of the merged stage launches from the next run on: 256
 * (the tile's edge faces on its first two warps) or 288 (a ninth warp owns
 * them), 0 = chosen by the autotuner at the next run (the default; it times
 * both with every CTA count it tries).  The same results either way. */
int ibgpu_batch_set_block(ibgpu_batch *b, int threads);
/* Event timing of the merged stage launches (total ms, launch count); a
 * batch with timing enabled runs its steps as direct launches, not graphs. */
int ibgpu_batch_set_timing(ibgpu_batch *b, int enable);
/* Chosen CTA count (0 = one CTA per work item) and threads per CTA,
 * subcycling period, timing. */
int ibgpu_batch_info(const ibgpu_batch *b, int *grid, int *threads, int *period,
                     double *stage_ms, int64_t *stage_launches);
/* Autotuner record: up to max (CTA count, threads per CTA, ms) candidates;
 * returns the number of candidates timed. */
int ibgpu_batch_tuning(const ibgpu_batch *b, int max, int *grids, int *threads, float *ms);
/* Bytes of the device's constant-memory argument table this batch holds
 * (its stage kernels read their arguments from there); 0 when the batch did
 * not fit and its stage kernels read the arguments from global memory.  The
 * table (60 KiB per device) is shared by the live batches of the device;
 * destroying a batch returns its part.  Creation assumes the cases' device
 * is the current one. */
int ibgpu_batch_table_bytes(const ibgpu_batch *b);
void ibgpu_batch_destroy(ibgpu_batch *b);

/* Allocation-free variant of ibgpu_step for one periodic, inviscid,
 * single-level grid of nx x ny cells (this entry point has no counterpart in
 * the reference).  For callers that must not allocate device memory while
 * they run, e.g. a coupler whose device memory belongs to another
 * framework's pool, or a time loop that cannot afford cudaMalloc/cudaFree's
 * device-wide synchronisation.  The caller passes device buffers of
 * FlowVariables rows in row-major cell order (iy * nx + ix), 7 doubles per
 * cell; d_rows_in may equal d_rows_out.  Every intermediate lives in one
 * fixed file-scope device array sized for IBGPU_NOALLOC_MAX_CELLS cells
 * (about 7.4 MB, held by each GPU that loads the library until exit); no
 * cudaMalloc, cudaFree or allocating library routine is called.  nx and ny
 * must be multiples of 16 with nx * ny <= IBGPU_NOALLOC_MAX_CELLS, else
 * IBGPU_E_ARG.  The first call on a device looks up that array's address
 * (once per device, with the device current): make it before any stream
 * capture.  All calls share the array, which keeps the last call's contents;
 * calls that overlap on the GPU race, so the caller serialises them.  The
 * call synchronises `stream` (a cudaStream_t, NULL for the legacy stream)
 * to return dt and diag. */
#define IBGPU_NOALLOC_MAX_CELLS 65536
int ibgpu_step_periodic_noalloc(const ibgpu_case *cs, int ts, int nx, int ny,
                                const double *d_rows_in, double *d_rows_out, double *dt,
                                ibgpu_diag *diag, void *stream);

/* ---------------------------------------------------------------------------
 * AMR refinement indicator: the plain (geometric) tag criterion and a learned
 * replacement for its per-box refine / coarsen / keep decision.
 * ------------------------------------------------------------------------- */

#define IBGPU_TAG_MAX_LEVELS 16
#define IBGPU_TAG_REFINE 1  /* rftag::tag   == 0 (AMR::TagtheBox givetag)   */
#define IBGPU_TAG_COARSEN 2 /* rftag::detag == 0 (AMR::TagtheBox givedetag) */

/* The case hook AMR::TagtheBox (Userfunction_cy_naca15.cpp:533-650) as data.
 * A box of level l is tagged for refinement when torefine[l] and it lies in
 * region(l); it is tagged for coarsening when toderefine[l], l >= 1 and it
 * lies outside the coarsening region of level l-1.  region(k) is, for
 * k < n_rect, the rectangle
 *     x - body_left_x > -rect_up[k] && x - body_right_x < rect_down[k] &&
 *     |y - body_center_y| < rect_half[k]
 * and otherwise the signed-distance band band_lo[k] < signdis < band_hi[k]
 * (the shipped case, :560-611), optionally also requiring the centre inside
 * the body box grown by near_margin[k] when near_margin[k] > 0.  The
 * coarsening regions use the de* arrays with n_rect_coarsen (:612-635). */
typedef struct ibgpu_tag_rule {
  double body_left_x, body_right_x, body_center_y, body_half_height;
  int n_rect, n_rect_coarsen;
  int torefine[IBGPU_TAG_MAX_LEVELS], toderefine[IBGPU_TAG_MAX_LEVELS];
  double rect_up[IBGPU_TAG_MAX_LEVELS], rect_down[IBGPU_TAG_MAX_LEVELS],
      rect_half[IBGPU_TAG_MAX_LEVELS];
  double band_lo[IBGPU_TAG_MAX_LEVELS], band_hi[IBGPU_TAG_MAX_LEVELS],
      near_margin[IBGPU_TAG_MAX_LEVELS];
  double derect_up[IBGPU_TAG_MAX_LEVELS], derect_down[IBGPU_TAG_MAX_LEVELS],
      derect_half[IBGPU_TAG_MAX_LEVELS];
  double deband_lo[IBGPU_TAG_MAX_LEVELS], deband_hi[IBGPU_TAG_MAX_LEVELS],
      denear_margin[IBGPU_TAG_MAX_LEVELS];
} ibgpu_tag_rule;

/* Boxes to judge: level and integer position (the learned indicator reads
 * the 5x5 same-level stencil around (ix, iy) from the context's state), the
 * box centre as the host mesh holds it (Mesh::bc) and the signed wall
 * distance (Box::pair.signdis). */
typedef struct ibgpu_tag_cells {
  int64_t n;
  const int32_t *level, *ix, *iy;
  const double *xc, *yc, *signdis;
} ibgpu_tag_cells;

/* Plain criterion on the GPU: out[i] = IBGPU_TAG_REFINE | IBGPU_TAG_COARSEN
 * bits of box i, the (tag, detag) pair AMR::TagtheBox's loops leave in
 * m_tag.  Host arrays in and out; ctx supplies the stream (may be any
 * context, no topology needed). */
int ibgpu_tag_plain(ibgpu_ctx *ctx, const ibgpu_tag_rule *rule, const ibgpu_tag_cells *cells,
                    uint8_t *out);

/* Learned indicator: an MLP with IBGPU_MLP_IN inputs, two hidden layers of
 * IBGPU_MLP_HIDDEN with GELU (tanh form) and IBGPU_MLP_CLASSES logits
 * (0 refine, 1 coarsen, 2 keep), BF16 operands on the tensor cores with FP32
 * accumulation.  Inputs per box: the 5x5 same-level stencil of (rho, u, v,
 * p) normalised by the freestream (rho/rho_inf - 1, u/c_inf, v/c_inf,
 * p/p_inf - 1; an absent stencil cell takes the centre's value), then
 * signdis/dh clipped to [-8, 8] / 8, signdis/chord clipped to [-4, 4] / 4,
 * (x - body_left_x)/chord/8, (y - body_center_y)/chord/8, |y -
 * body_center_y|/chord/8 and a one-hot level (0..6, deeper levels as 6).
 * Parameters: one FP32 device array of IBGPU_MLP_PARAMS floats, W1[64][112],
 * b1[64], W2[64][64], b2[64], W3[3][64], b3[3]; weights are rounded to BF16
 * (nearest even) when a kernel loads them. */
#define IBGPU_MLP_IN 112
#define IBGPU_MLP_STENCIL 100
#define IBGPU_MLP_HIDDEN 64
#define IBGPU_MLP_CLASSES 3
#define IBGPU_MLP_PARAMS 11587

/* Feature rows of the boxes (device output, n x IBGPU_MLP_IN BF16 bit
 * patterns, row-major) from the context's current state; every box must be
 * a cell of the uploaded topology (else IBGPU_E_ARG). */
int ibgpu_indicator_features(ibgpu_ctx *ctx, const ibgpu_tag_rule *rule,
                             const ibgpu_tag_cells *cells, uint16_t *d_feat);

/* Inference on device feature rows: d_class[i] = argmax logit (0 refine,
 * 1 coarsen, 2 keep); d_logits (n x 3 FP32) may be NULL. */
int ibgpu_mlp_forward(ibgpu_ctx *ctx, const float *d_params, int64_t n, const uint16_t *d_feat,
                      uint8_t *d_class, float *d_logits);

/* Gradient of the class-weighted cross entropy
 *     L = (1/n) * sum_i w[y_i] * -log softmax(z_i)[y_i]
 * over the n device rows (labels 0..2; a label outside 0..2 contributes
 * nothing), ADDED to d_grad (IBGPU_MLP_PARAMS floats); d_stats[0] += L,
 * d_stats[1] += number of rows whose argmax equals the label.  The backward
 * pass rounds each layer's output gradient to BF16 before its products. */
int ibgpu_mlp_grad(ibgpu_ctx *ctx, const float *d_params, int64_t n, const uint16_t *d_feat,
                   const uint8_t *d_label, const float class_weight[3], float *d_grad,
                   float *d_stats);

/* One Adam step (beta1 0.9, beta2 0.999, eps 1e-8, bias-corrected) of the
 * FP32 parameters with moments d_m, d_v, step >= 1. */
int ibgpu_mlp_adam(ibgpu_ctx *ctx, float *d_params, const float *d_grad, float *d_m, float *d_v,
                   int step, float lr);

/* One training step: d_grad (IBGPU_MLP_PARAMS floats of scratch) is zeroed,
 * filled with the minibatch gradient (as ibgpu_mlp_grad) and applied by
 * ibgpu_mlp_adam at the given step; d_stats as in ibgpu_mlp_grad. */
int ibgpu_mlp_train_step(ibgpu_ctx *ctx, float *d_params, float *d_m, float *d_v, float *d_grad,
                         int step, float lr, int64_t n, const uint16_t *d_feat,
                         const uint8_t *d_label, const float class_weight[3], float *d_stats);

/* Learned tags: the features of the boxes, the MLP and the class mapped to
 * the plain criterion's bits (refine -> IBGPU_TAG_REFINE, coarsen ->
 * IBGPU_TAG_COARSEN, keep -> 0); host output.  Like the plain criterion it
 * refines only on levels whose rule->torefine is set and coarsens only on
 * levels >= 1 whose rule->toderefine is set (AMR::TagtheBox acts only on
 * the requests of AMRLevel::torefine / toderefine). */
int ibgpu_tag_learned(ibgpu_ctx *ctx, const ibgpu_tag_rule *rule, const ibgpu_tag_cells *cells,
                      const float *d_params, uint8_t *out);

/* Signed wall distance of every uploaded cell row (Box::pair.signdis), kept
 * on the device per cell until the next topology upload; cells without it
 * count as far from any wall. */
int ibgpu_upload_signdis(ibgpu_ctx *ctx, const double *signdis);

/* Tags of every row of the uploaded cell list (0 for rows that are not
 * normal cells): the learned indicator when d_params is non-NULL (features
 * gathered from the device state inside the tensor-core kernel, no feature
 * matrix; centres from the cell positions), else the plain criterion. */
int ibgpu_tag_mesh(ibgpu_ctx *ctx, const ibgpu_tag_rule *rule, const float *d_params,
                   uint8_t *tags);

/* ibgpu_tag_mesh of every case of a batch with one synchronisation: each
 * case tags on its own context stream (ordered after the batch stream's
 * pending work; the cases' kernels overlap) and the batch stream waits for
 * all of them; tags holds the cases' row tags one after another (case
 * order, each case's cell-list order).  Use pinned host memory for tags. */
int ibgpu_batch_tag_mesh(ibgpu_batch *b, const ibgpu_tag_rule *rule, const float *d_params,
                         uint8_t *tags);

const char *ibgpu_errstr(int code);
/* Last CUDA error string seen by this thread's most recent failing call. */
const char *ibgpu_last_error(void);

#ifdef __cplusplus
}
#endif

#endif
