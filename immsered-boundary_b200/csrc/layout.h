// Device data layout shared by the host tile builder and the kernels.
//
// Each AMR level is stored as Morton-ordered 16 x 16 tiles of cell slots;
// every field is a structure-of-arrays over slots, slot = tile * 256 +
// ly * 16 + lx, so one tile of one field is 2 KB of contiguous FP64.  A slot
// holds a leaf cell or a 2-D ghost cell of the reference mesh (domain ghost,
// coarse/fine ghost); periodic/block ghosts are not stored, the tile
// neighbour table wraps around instead.  Absent slots have flags == 0.
#pragma once

#include <stddef.h>
#include <stdint.h>

namespace ibgpu {

constexpr int kTile = 16;
constexpr int kTileCells = kTile * kTile;
constexpr int kMaxLevels = 16;

// state field indices of the step-state buffer (FP64 SoA)
enum { F_RHO = 0, F_U = 1, F_V = 2, F_P = 3, F_E = 4, F_T = 5, kStateFields = 6 };

// slot flags (identical bit values to IBGPU_CELL_*)
enum : uint8_t {
  CF_PRESENT = 1,
  CF_NORMAL = 2,
  CF_UPDATE = 4,
  CF_PRIM = 8,
  CF_RESET = 16,
  CF_RESNORM = 32,
};

struct LevelConst {
  double dx, dy, dz;
  double vol;      // dh0*dh1*dh2 (m_geom.v)
  double inv_vol;  // 1 / vol (fast builds)
  double area_x;   // dh1*dh2 (x-face area)
  double area_y;   // dh2*dh0 (y-face area)
  double area_z;   // dh0*dh1 (z-face area; enters the CFL sum)
  double inv_dx, inv_dy;  // 1.0/dh (m_geom.keisa)
  double step_num;
  double cfl_vol;  // CFL * vol
};

struct CaseConst {
  double gama, Rg, Cv, Ma, Re, qk, s_over_t, dt_ratio;
  double gm1, gamaRg, inv_Rg, Cp;
  double p_ref, area_ref, shear_ref, L_ref, mu;
  double initvar[7];
  LevelConst lev[kMaxLevels];
};

// Device-side abort record.  The reference aborts at the first failing
// check in its sequential order: the immersed-boundary fill (Body.cpp:1428,
// 1476), the CFL pass (NS_Solver.cpp:253), then per stage all density checks
// (UpdateConsVars) before all temperature checks (ComptNewPrimVar).
// err_key = (phase << 40) | (check << 32) | slot, phase = 8 * step + p with
// p = 0 for the IB fill, 1 for the CFL pass and 2 + k for stage k; the
// smallest key is the reference's abort.
enum : int {
  ERR_IB_NEG_T = 0,    // phase 0: Body::IBConditions_Image, image point T < 0 (1050)
  ERR_IB_NAN = 1,      //          IB cell state NaN (1076)
  ERR_CFL_NEG_DT = 2,  // phase 1: Comptdt (424)
  ERR_NEG_RHO = 3,     // phase 2+k: UpdateConsVars (523 / 611)
  ERR_NEG_T = 4        //            ComptNewPrimVar (37)
};

struct DevDiag {
  double dt;
  unsigned long long cfl_bits;
  unsigned long long res_bits[5];
  unsigned long long err_key;  // ~0ull: no error
  // CFL bound of the next step, accumulated by a final stage that computes
  // it (StageArgs::cfl_next) for single-level runs without bodies
  unsigned long long cfl_next_bits;
};

constexpr int kHaloStage = 2;

// Stage-dependent part of the stage arguments.  Stage input and output of
// the varying cells (rho u v p): the first stage reads the FP64 step state;
// the stage buffers between stages hold FP64 values in the FP64 builds and
// FP32 values in the mixed build, whose flux reads its inputs as FP32 (the
// rounding happens at the store instead of the load: same values).
struct StageVar {
  const void *sin[4];  // stage input of varying cells
  void *sout[4];       // stage output (non-final stages)
  double tp;             // stage coefficient tp[k]
  // final stage only: 1 + the abort-order phase of the next step's CFL pass
  // to fold that pass into this stage (0: off).  The next step's CFL reads
  // the normal cells this stage writes, and nothing else writes them in
  // between when the run has one level and no immersed body.
  int cfl_next;
  int pad_;
};

struct StageArgs {
  const int32_t *tile_nb;  // 9 neighbour tiles per tile, (oy+1)*3+(ox+1); -1 absent
  const int32_t *tile_level;
  const uint8_t *tile_uniform;  // 1: tile and side neighbours all recovering leaf cells
  const uint8_t *flags;
  double *s0[kStateFields];  // step state rho u v p e T
  const double *vsd;         // frozen viscous residual parts [8][nslots] or null
  int64_t nslots;
  DevDiag *diag;
  int tile_begin;
  int phase;  // abort-order phase of this stage (see DevDiag)
  // single-case fast stage: warm L2 with the stage input of tile + prefetch,
  // about one wave of resident CTAs ahead (0: off)
  int prefetch;
  // last member: the batched stage's constant-memory table keeps each case's
  // arguments up to here once and its StageVar records per stage
  StageVar v;
};

// bytes of StageArgs before the stage-dependent part
constexpr int kStageCommonBytes = (int)offsetof(StageArgs, v);
static_assert(kStageCommonBytes % 8 == 0, "StageVar starts 8-byte aligned");
static_assert(sizeof(StageVar) % 8 == 0, "StageVar keeps 8-byte alignment");

struct CflArgs {
  const int32_t *tile_level;
  const uint8_t *flags;
  const double *s0[kStateFields];
  int64_t nslots;
  int phase;
  DevDiag *diag;
};

// Coarse/fine pairs of one level: coarse slot, four son slots and (for
// prolongation) the coarse cell's -x, +x, -y, +y neighbour slots.
struct PairArgs {
  const int32_t *coarse;
  const int32_t *fine;  // 4 per pair
  const int32_t *nb;    // 4 per pair (prolongation only)
  int n;
  double *s0[kStateFields];
};

// One dependency wave [begin, end) of the domain-ghost list.
struct BcArgs {
  const int32_t *ghost, *ref, *type, *face;
  const double *nmv;      // 3 per ghost
  const double *facevar;  // 7 per face
  int begin, end;
  double backpressure, cos_in, sin_in;
  double *s0[kStateFields];
};

struct IbArgs {
  const int32_t *cell;   // slot per IB cell
  const int32_t *intp;   // 8 slots per IB cell
  const double *cellf;   // 16 per IB cell
  double *out;           // 6 per IB cell (rho u v p e T)
  int n;
  double *s0[kStateFields];
  int phase;
  DevDiag *diag;
  // when set, the abort-order phase is *phase_base + phase (a batch replays
  // one captured launch for every step and keeps the step's base on the device)
  const int *phase_base;
};

struct ForceArgs {
  const int32_t *body;   // per patch
  const int32_t *intp;   // 8 slots per patch
  const double *patchf;  // 19 per patch
  const double *body_center;
  const int32_t *body_begin;  // nbodies + 1 (patches sorted by body, reference order)
  int n, nbodies;
  double *out;     // 12 per patch
  double *result;  // 6 per body
  double *s0[kStateFields];
};

struct ViscArgs {
  const int32_t *tile_nb;
  const int32_t *tile_level;
  const uint8_t *flags;
  int tile_begin;
  const double *s0[kStateFields];
  double *vsd;
  int64_t nslots;
};

}  // namespace ibgpu
