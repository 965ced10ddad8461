// Host-side helpers shared by the C ABI translation units.
#pragma once

#include <string>

#include "../../include/ibgpu.h"
#include "layout.h"

#include <cuda_runtime.h>

namespace ibgpu {
// Read-only view of a context's device state for the indicator entry points.
struct CtxView {
  cudaStream_t stream;
  int device, nsm;
  bool has_topology, has_state;
  const double *s0[kStateFields];
  const uint8_t *flags;
  const int32_t *tile_nb;
  const int32_t *tile_level;
  const int2 *tile_org;
  const int32_t *cell_slot;
  int64_t ncells, nslots, ntiles;
  int *aux_err;  // device word: set by a kernel whose wait ran out of time
  CaseConst cc;
};
int ctx_view(const ibgpu_ctx *ctx, CtxView *v);
// per-slot signed wall distance (created on demand); tag buffer of nslots
// per-slot bytes followed by ncells per-row bytes
int ctx_signdis_buffer(ibgpu_ctx *ctx, double **dev, bool create);
int ctx_tags_buffer(ibgpu_ctx *ctx, uint8_t **dev);
// slot of box (l, ix, iy) of the uploaded topology (periodic wrap), -1 if absent
int64_t ctx_slot_at(const ibgpu_ctx *ctx, int l, int ix, int iy);
// the context's wall-distance state (csrc/wall.cu), freed with the context
void **ctx_wall_state(ibgpu_ctx *ctx);
void wall_free(void *state);

// indicator entry points shared with the batched runner (csrc/indicator.cu)
int tag_mesh_enqueue(ibgpu_ctx *ctx, const ibgpu_tag_rule *rule, const float *d_params,
                     cudaStream_t st, uint8_t **rows_out);
int tag_mesh_prepare(bool learned);

int validate_case(const ibgpu_case *cs);
void fill_case_const(const ibgpu_case *cs, CaseConst &k);
void set_last_error(const std::string &msg);
}  // namespace ibgpu
