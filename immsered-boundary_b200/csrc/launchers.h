// Launchers of the kernels in kernels.cuh, one set per arithmetic build:
// ibgpu::fast (kernels_fp64.cu: FP64 with contracted multiply-adds, and the
// mixed FP32-flux path) and ibgpu::exact (kernels_exact.cu, -fmad=false).
#pragma once

#include <cuda_runtime.h>

#include "layout.h"

namespace ibgpu {

#define IBGPU_DECLARE_LAUNCHERS(NS)                                                           \
  namespace NS {                                                                              \
  void launch_stage(const StageArgs &a, const CaseConst &cc, int ntiles, int limiter,         \
                    bool visc, bool final_stage, bool mixed, int stage, cudaStream_t st);     \
  void launch_cfl(const CflArgs &a, const CaseConst &cc, int nsm, cudaStream_t st);           \
  void launch_step_begin(DevDiag *d, cudaStream_t st);                                         \
  void launch_take_folded_cfl(DevDiag *d, const CaseConst &cc, cudaStream_t st);              \
  void launch_scatter(const double *rows, const int32_t *cell_slot, const uint8_t *alias,     \
                      int64_t n, double *const s0[kStateFields], int nsm, cudaStream_t st);   \
  void launch_gather(double *rows, const int32_t *cell_slot, int64_t n,                       \
                     double *const s0[kStateFields], int nsm, cudaStream_t st);               \
  void launch_scatter4(const double *rows, const int32_t *cell_slot, const uint8_t *alias,    \
                       int64_t n, double Rg, double Cv, double *const s0[kStateFields],       \
                       int nsm, cudaStream_t st);                                             \
  void launch_gather4(double *rows, const int32_t *cell_slot, int64_t n,                      \
                      double *const s0[kStateFields], int nsm, cudaStream_t st);              \
  void launch_restrict(const PairArgs &a, const CaseConst &cc, cudaStream_t st);               \
  void launch_prolong(const PairArgs &a, const CaseConst &cc, cudaStream_t st);                \
  void launch_bc(const BcArgs &a, const CaseConst &cc, cudaStream_t st);                       \
  void launch_ib(const IbArgs &a, const CaseConst &cc, cudaStream_t st);                       \
  void launch_forces(const ForceArgs &a, const CaseConst &cc, cudaStream_t st);                \
  void launch_viscous(const ViscArgs &a, const CaseConst &cc, int ntiles, bool mixed,          \
                      cudaStream_t st);                                                        \
  }

IBGPU_DECLARE_LAUNCHERS(fast)
IBGPU_DECLARE_LAUNCHERS(exact)

// batched stage over several cases (fast builds only): work = (case, tile)
// pairs, args[case * nstages + stage], ccs[case]; grid 0 = one CTA per item;
// threads 256 or 288 per CTA (others: the precision's default); table >= 0:
// byte offset of the batch's header in the constant-memory table (the
// arguments are read from there instead)
namespace fast {
void launch_stage_batch(const StageArgs *args, const CaseConst *ccs, const int2 *work, int nwork,
                        int stage, int nstages, const int *phase_base, int limiter, bool visc,
                        bool final_stage, bool mixed, int grid, int threads, int table,
                        cudaStream_t st);
// constant-memory table of batched stage arguments: reserve a byte range on
// a device (16-byte aligned offset, -1 when it does not fit), release it,
// write bytes at an offset (current device; blocking)
int batch_table_reserve(int device, int bytes);
void batch_table_release(int device, int offset);
cudaError_t batch_table_write(int offset, const void *src, int bytes);
void launch_set_phase_base(int *phase_base, int value, int fold, cudaStream_t st);
void launch_take_folded_batch(const StageArgs *args, const CaseConst *ccs, int ncases, int nstages,
                              cudaStream_t st);
// CFL pass over the work list's tiles, then dt of the first ncases cases, or
// with case_list of the ncases cases it lists
void launch_cfl_batch(const StageArgs *args, const CaseConst *ccs, const int2 *work, int nwork,
                      int nstages, const int *phase_base, int ncases, int grid, cudaStream_t st,
                      const int *case_list = nullptr);
void launch_step_begin_batch(const StageArgs *args, int ncases, int nstages, cudaStream_t st);
}  // namespace fast

#undef IBGPU_DECLARE_LAUNCHERS

}  // namespace ibgpu
