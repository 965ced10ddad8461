// AMR refinement indicator on the GPU: the plain geometric tag criterion of
// the case hook AMR::TagtheBox (Userfunction_cy_naca15.cpp:533-650, rftag in
// Box.H:11-61) and a learned replacement for its per-box decision, a small
// MLP whose forward and backward passes run on the sm_100a tensor cores
// (tcgen05.mma, BF16 operands staged in shared memory, FP32 accumulators in
// Tensor Memory).
//
// MLP shapes: X[rows x 112] -> 64 -> 64 -> 3.  Tiles of 128 rows; tile row t
// is Tensor Memory lane t of every M = 128 accumulator.  The two hidden
// layers (and in training every backward and weight-gradient product but
// the 3-row last layer's) are tensor-core MMAs; the 3-row last layer runs
// on the CUDA cores from bf16-rounded operands (3 FMAs per hidden unit, no
// MMA round trip).  Inference kernels: one thread per row, 128 threads.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "../../include/ibgpu.h"
#include "host_internal.h"
#include "layout.h"
#include "tcgen05.cuh"

namespace ibgpu {
namespace ind {

constexpr int kIn = IBGPU_MLP_IN;         // 112 inputs
constexpr int kHid = IBGPU_MLP_HIDDEN;    // 64
constexpr int kOut = IBGPU_MLP_CLASSES;   // 3
constexpr int kRows = 128;                // rows per tile = M of every MMA
constexpr int kThreads = 128;
constexpr int kOnesRow = kIn;             // feature held at 1 in the training tiles (bias gradients)

// parameter array offsets (floats)
constexpr int P_W1 = 0;
constexpr int P_B1 = P_W1 + kHid * kIn;
constexpr int P_W2 = P_B1 + kHid;
constexpr int P_B2 = P_W2 + kHid * kHid;
constexpr int P_W3 = P_B2 + kHid;
constexpr int P_B3 = P_W3 + kOut * kHid;
constexpr int P_COUNT = P_B3 + kOut;
static_assert(P_COUNT == IBGPU_MLP_PARAMS, "parameter layout");

// Tensor Memory columns of the forward kernels (f32, lanes = tile rows)
constexpr uint32_t T_D1 = 0;      // layer-1 pre-activation   (64)
constexpr uint32_t T_D2 = 64;     // layer-2 pre-activation   (64)
constexpr uint32_t T_COLS_TRAIN = 512;
constexpr uint32_t T_COLS_FWD = 256;

constexpr long long kWaitCycles = 2000000000ll;  // ~1 s at the boost clock

__device__ __forceinline__ uint16_t bf16_bits(float x) {
  return __bfloat16_as_ushort(__float2bfloat16_rn(x));
}
__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);  // .x = lo (low half)
  return *reinterpret_cast<const uint32_t *>(&h);
}
__device__ __forceinline__ float bf16_round(float x) {
  return __bfloat162float(__float2bfloat16_rn(x));
}

// GELU, tanh form (Hendrycks & Gimpel): 0.5 z (1 + tanh(sqrt(2/pi)(z + 0.044715 z^3)))
constexpr float kGeluA = 0.7978845608028654f;
constexpr float kGeluB = 0.044715f;
// tanh comes from the SFU's tanh.approx.f32 (one instruction; its error
// stays well below the BF16 rounding that every activation and every
// back-propagated gradient goes through next).  The training kernel takes
// GELU and its derivative from the same tanh in its forward pass.
__device__ __forceinline__ float tanh_sfu(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float gelu(float z) {
  const float u = kGeluA * (z + kGeluB * z * z * z);
  return 0.5f * z * (1.0f + tanh_sfu(u));
}
// GELU and its derivative d/dz [0.5 z (1 + tanh u)], u = a (z + b z^3)
__device__ __forceinline__ void gelu_and_grad(float z, float &g, float &gp) {
  const float u = kGeluA * (z + kGeluB * z * z * z);
  const float th = tanh_sfu(u);
  g = 0.5f * z * (1.0f + th);
  gp = 0.5f * (1.0f + th) + 0.5f * z * (1.0f - th * th) * kGeluA * (1.0f + 3.0f * kGeluB * z * z);
}

__device__ __forceinline__ void st_bf16(uint8_t *base, int off, float v) {
  *reinterpret_cast<uint16_t *>(base + off) = bf16_bits(v);
}

// ---------------------------------------------------------------------------
// Training kernel: 256 threads, two per tile row.  Warp w reads Tensor
// Memory lane quarter w % 4 (tile rows 32 (w % 4) ..) and owns accumulator
// columns [32 (w / 4), +32) of the 64-wide layers.  Every activation and
// gradient tile is stored once, row-major in the K-major layout (8-column
// slabs of 2048 bytes); the weight-gradient products read those same tiles
// as MN-major operands of their transposes, so nothing is transposed in
// shared memory.  Shared memory (bytes):
constexpr int kThreadsTrain = 256;
constexpr int kSlab = kRows * 16;  // 8 bf16 columns of a 128-row tile
struct TrainSmem {
  // X of two tiles (the next one is stored while the weight gradients of
  // the current one still read it): 16 slabs, features 112 = 1 (bias rows
  // of the weight gradients) and 113..127 = 0
  static constexpr int X0 = 0;
  static constexpr int X1 = X0 + 16 * kSlab;
  static constexpr int H = X1 + 16 * kSlab;    // [h1 | h2], 16 slabs
  static constexpr int DZ = H + 16 * kSlab;    // [dz1 | dz2 | dz3 (16 columns)], 18 slabs
  static constexpr int W1 = DZ + 18 * kSlab;   // [64 x 112] B of layer 1
  static constexpr int W2 = W1 + kHid * kIn * 2;       // [64 x 64]  B of layer 2
  static constexpr int W2T = W2 + kHid * kHid * 2;     // [64 x 64]  B of dh1
  static constexpr int BIAS = W2T + kHid * kHid * 2;   // b1, b2, b3 (f32)
  static constexpr int W3F = BIAS + 1024;              // W3 rounded to bf16, as f32 [3 x 64]
  static constexpr int XCH = W3F + 1024;               // row exchange between column halves [128 x 4] f32
  static constexpr int BYTES = XCH + kRows * 16;
};
static_assert(TrainSmem::BYTES <= 227 * 1024, "shared memory budget");

// Tensor Memory columns of the training kernel (f32, lanes = tile rows)
constexpr uint32_t TT_D1 = 0;      // z1, then gelu'(z1)                       (64)
constexpr uint32_t TT_D2 = 64;     // z2, then dL/dh1                          (64)
constexpr uint32_t TT_GCAT = 128;  // [h1|h2]^T [dz2|dz3], accumulated         (80)
constexpr uint32_t TT_G1 = 208;    // [x|1]^T [dz1|dz2|dz3], accumulated      (144)
static_assert(TT_G1 + 144 <= T_COLS_TRAIN, "tensor memory budget");

struct FwdSmem {
  static constexpr int X = 0;
  static constexpr int H1 = X + kRows * kIn * 2;
  static constexpr int W1 = H1 + kRows * kHid * 2;
  static constexpr int W2 = W1 + kHid * kIn * 2;
  static constexpr int BIAS = W2 + kHid * kHid * 2;
  static constexpr int W3F = BIAS + 1024;  // W3 rounded to bf16, as f32 [3 x 64]
  static constexpr int BYTES = W3F + 1024;
};

// Weights (rounded to bf16) into their B-operand tiles; W3 (3 rows, used
// on the CUDA cores) rounded to bf16 and kept as f32; biases as f32.
__device__ void load_weights(const float *__restrict__ P, uint8_t *sW1, uint8_t *sW2,
                             uint8_t *sW2T, float *sB, float *sW3f) {
  using tc::kmajor_off;
  for (int i = threadIdx.x; i < kHid * kIn; i += blockDim.x) {
    const int o = i / kIn, k = i % kIn;
    st_bf16(sW1, kmajor_off(kHid, o, k), P[P_W1 + i]);
  }
  for (int i = threadIdx.x; i < kHid * kHid; i += blockDim.x) {
    const int o = i / kHid, k = i % kHid;
    const float w = P[P_W2 + i];
    st_bf16(sW2, kmajor_off(kHid, o, k), w);
    if (sW2T) st_bf16(sW2T, kmajor_off(kHid, k, o), w);
  }
  for (int i = threadIdx.x; i < kOut * kHid; i += blockDim.x) sW3f[i] = bf16_round(P[P_W3 + i]);
  for (int i = threadIdx.x; i < 2 * kHid + 4; i += blockDim.x) {
    float b = 0.0f;
    if (i < kHid) b = P[P_B1 + i];
    else if (i < 2 * kHid) b = P[P_B2 + i - kHid];
    else if (i - 2 * kHid < kOut) b = P[P_B3 + i - 2 * kHid];
    sB[i] = b;
  }
}

// Issue `ksteps` MMAs of K = 16 over tiles whose K-slab strides are a_lbo /
// b_lbo bytes (two slabs per step), into Tensor Memory column `col`.
__device__ __forceinline__ void mma_chain(uint32_t tmem, uint32_t col, const uint8_t *A,
                                          uint32_t a_lbo, const uint8_t *B, uint32_t b_lbo,
                                          int ksteps, uint32_t idesc, bool accumulate) {
  for (int s = 0; s < ksteps; ++s) {
    const uint64_t ad = tc::smem_desc(A + 2 * s * a_lbo, a_lbo, 128);
    const uint64_t bd = tc::smem_desc(B + 2 * s * b_lbo, b_lbo, 128);
    tc::mma_bf16(tmem + col, ad, bd, idesc, (accumulate || s > 0) ? 1u : 0u);
  }
}

// Block-wide barrier that also orders tensor-core work across it.
__device__ __forceinline__ void tc_sync() {
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
}

// Commit the issuing thread's MMAs to the mbarrier and wait for them from
// every thread; false (uniformly) when the wait ran out of time.
__device__ __forceinline__ bool commit_and_wait(uint64_t *bar, uint32_t &phase, int *abort_flag) {
  if (threadIdx.x == 0) tc::mma_commit(bar);
  const bool ok = tc::mbar_wait_bounded(bar, phase, kWaitCycles);
  phase ^= 1u;
  if (!ok) atomicExch(abort_flag, 1);
  tc_sync();
  return *(volatile int *)abort_flag == 0;
}

// 64 f32 columns of this thread's lane starting at `col`, plus bias.
// (the four loads issued back to back, one wait)
__device__ __forceinline__ void tmem_row64(uint32_t taddr, const float *bias, float (&v)[64]) {
  uint32_t r[4][16];
#pragma unroll
  for (int q = 0; q < 4; ++q) tc::tmem_ld16(taddr + 16 * q, r[q]);
  tc::tmem_wait_ld16(r[0]);
#pragma unroll
  for (int q = 1; q < 4; ++q) tc::tmem_tie16(r[q]);
#pragma unroll
  for (int q = 0; q < 4; ++q)
#pragma unroll
    for (int e = 0; e < 16; ++e) v[16 * q + e] = __uint_as_float(r[q][e]) + (bias ? bias[16 * q + e] : 0.0f);
}

// Row-major [rows x 64] bf16 A tile: this thread's row from 64 values.
__device__ __forceinline__ void store_row64(uint8_t *tile, int t, const float (&v)[64]) {
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    uint4 w;
    w.x = pack_bf16(v[8 * c + 0], v[8 * c + 1]);
    w.y = pack_bf16(v[8 * c + 2], v[8 * c + 3]);
    w.z = pack_bf16(v[8 * c + 4], v[8 * c + 5]);
    w.w = pack_bf16(v[8 * c + 6], v[8 * c + 7]);
    *reinterpret_cast<uint4 *>(tile + c * (kRows * 16) + t * 16) = w;
  }
}

// Feature row -> X (row-major A tile).
__device__ __forceinline__ void load_x_row(const uint16_t *__restrict__ feat, int64_t row, bool valid,
                                           int t, uint8_t *sX) {
  const uint4 *src = reinterpret_cast<const uint4 *>(feat + row * kIn);
#pragma unroll 2
  for (int c = 0; c < kIn / 8; ++c) {
    uint4 w = make_uint4(0u, 0u, 0u, 0u);
    if (valid) w = __ldg(src + c);
    *reinterpret_cast<uint4 *>(sX + c * (kRows * 16) + t * 16) = w;
  }
}

// ---------------------------------------------------------------------------
// Gradient of the class-weighted cross entropy, accumulated over the tiles
// this CTA processes and added to grad once at the end.
//
// Per tile (thread 0 issues every MMA; one commit is outstanding at a time):
//   L1  D1 = X W1^T  -> h1 = gelu(z1) to smem, gelu'(z1) back into D1
//   L2  D2 = h1 W2^T -> h2 = gelu(z2); the next tile's X into registers;
//                       logits h2 W3^T, softmax, dz3 and dh2 = dz3 W3 on
//                       the CUDA cores (W3 has 3 rows: 3 FMAs per element,
//                       the two column halves of a row summed through
//                       shared memory), dz2 = dh2 gelu'(z2)
//   dh1 = dz2 W2     -> dz1 = dh1 gelu'(z1); the next tile's X to smem
//   with dh1, unwaited: [dW2 | dW3]^T += [h1 | h2]^T [dz2 | dz3]
//   with the next tile's L1, unwaited: [dW1 | b]^T += [x | 1]^T [dz1 | dz2 | dz3]
// The unwaited weight-gradient MMAs overlap the next epilogue; the tile
// buffers they read are rewritten only after a later commit covers them.
// Products on the CUDA cores take bf16-rounded operands and accumulate in
// f32, as the tensor core does.  (Two tiles in flight, alternating steps in
// the same warps, measured slower: 116 us against 91 us for 262,144 rows.)
__device__ __forceinline__ bool wait_phase(uint64_t *bar, uint32_t &phase, int *abort_flag) {
  const bool ok = tc::mbar_wait_bounded(bar, phase, kWaitCycles);
  if (ok) phase ^= 1u;
  else atomicExch(abort_flag, 1);
  tc_sync();
  return *(volatile int *)abort_flag == 0;
}

// 32 f32 columns of this thread's lane (two loads, one wait)
__device__ __forceinline__ void tmem_row32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[2][16];
  tc::tmem_ld16(taddr, r[0]);
  tc::tmem_ld16(taddr + 16, r[1]);
  tc::tmem_wait_ld16(r[0]);
  tc::tmem_tie16(r[1]);
#pragma unroll
  for (int e = 0; e < 32; ++e) v[e] = __uint_as_float(r[e >> 4][e & 15]);
}
__device__ __forceinline__ void tmem_store32(uint32_t taddr, const float (&v)[32]) {
  uint32_t r[2][16];
#pragma unroll
  for (int e = 0; e < 32; ++e) r[e >> 4][e & 15] = __float_as_uint(v[e]);
  tc::tmem_st16(taddr, r[0]);
  tc::tmem_st16(taddr + 16, r[1]);
}
// 32 values into slabs s0..s0+3 of a row-major tile, row t
__device__ __forceinline__ void store_row32(uint8_t *tile, int t, int s0, const float (&v)[32]) {
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    uint4 w;
    w.x = pack_bf16(v[8 * c + 0], v[8 * c + 1]);
    w.y = pack_bf16(v[8 * c + 2], v[8 * c + 3]);
    w.z = pack_bf16(v[8 * c + 4], v[8 * c + 5]);
    w.w = pack_bf16(v[8 * c + 6], v[8 * c + 7]);
    *reinterpret_cast<uint4 *>(tile + (s0 + c) * kSlab + t * 16) = w;
  }
}

__global__ void __launch_bounds__(kThreadsTrain, 1)
    mlp_grad_kernel(const float *__restrict__ P, const uint16_t *__restrict__ feat,
                    const uint8_t *__restrict__ label, int64_t n, float cw0, float cw1, float cw2,
                    float inv_n, float *__restrict__ grad, float *__restrict__ stats,
                    int *__restrict__ err) {
  extern __shared__ __align__(1024) uint8_t smem[];
  __shared__ uint64_t bar;
  __shared__ uint32_t tbase;
  __shared__ int abort_flag;
  using S = TrainSmem;
  uint8_t *const sX[2] = {smem + S::X0, smem + S::X1};
  uint8_t *sH = smem + S::H, *sH2 = sH + 8 * kSlab, *sDZ = smem + S::DZ, *sDZ2 = sDZ + 8 * kSlab,
          *sDZ3 = sDZ + 16 * kSlab, *sW1 = smem + S::W1, *sW2 = smem + S::W2,
          *sW2T = smem + S::W2T;
  float *sB = reinterpret_cast<float *>(smem + S::BIAS);
  const float *sW3f = reinterpret_cast<const float *>(smem + S::W3F);
  float4 *sXch = reinterpret_cast<float4 *>(smem + S::XCH);
  const int tid = threadIdx.x, warp = tid >> 5;
  const int t = ((warp & 3) << 5) | (tid & 31);  // tile row = Tensor Memory lane
  const int hh = warp >> 2;                      // column half of the 64-wide layers
  const int c0 = 32 * hh;
  const int pair_bar = 1 + (warp & 3);  // named barrier of warps w and w + 4 (one row each)

  load_weights(P, sW1, sW2, sW2T, sB, reinterpret_cast<float *>(smem + S::W3F));
  if (tid < kRows) {
    const uint4 zero = make_uint4(0u, 0u, 0u, 0u);
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      *reinterpret_cast<uint4 *>(sX[b] + 14 * kSlab + tid * 16) = make_uint4(0x3F80u, 0u, 0u, 0u);
      *reinterpret_cast<uint4 *>(sX[b] + 15 * kSlab + tid * 16) = zero;
    }
    *reinterpret_cast<uint4 *>(sDZ3 + kSlab + tid * 16) = zero;  // dz3 columns 8..15
  }
  if (tid == 0) {
    tc::mbar_init(&bar, 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    tc::tmem_alloc(&tbase, T_COLS_TRAIN);
    tc::tmem_relinquish();
  }

  // X rows of a tile: thread tid holds row tid % 128, slab pairs
  // (tid / 128) + 2k (one aligned 32-byte sector of the row each)
  uint4 xr[4][2];
  int ylab = -1, ycur = -1;  // labels of row tid (threads < 128)
  auto load_tile = [&](int64_t tile) {
    const int64_t row = tile * kRows + (tid & (kRows - 1));
    const bool valid = row < n;
    const uint4 *src = reinterpret_cast<const uint4 *>(feat + (valid ? row : 0) * kIn);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int p = (tid >> 7) + 2 * k;
      if (p < kIn / 16) {
        xr[k][0] = valid ? __ldg(src + 2 * p) : make_uint4(0u, 0u, 0u, 0u);
        xr[k][1] = valid ? __ldg(src + 2 * p + 1) : make_uint4(0u, 0u, 0u, 0u);
      }
    }
    if (tid < kRows) ylab = valid ? (int)label[row] : -1;
  };
  auto store_tile = [&](uint8_t *dst) {
    const int r = tid & (kRows - 1);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int p = (tid >> 7) + 2 * k;
      if (p < kIn / 16) {
        *reinterpret_cast<uint4 *>(dst + (2 * p) * kSlab + r * 16) = xr[k][0];
        *reinterpret_cast<uint4 *>(dst + (2 * p + 1) * kSlab + r * 16) = xr[k][1];
      }
    }
  };

  const int64_t ntiles = (n + kRows - 1) / kRows;
  int64_t tile = blockIdx.x;
  if (tile < ntiles) {
    load_tile(tile);
    store_tile(sX[0]);
    ycur = ylab;
  }
  tc::fence_async_smem();
  tc_sync();
  const uint32_t tm = tbase;
  const uint32_t lane = tm + (uint32_t)((warp & 3) << 21);  // this warp's lane quarter
  const uint32_t id64 = tc::idesc_bf16_f32(128, kHid), id_gcat = tc::idesc_bf16_f32_mn(128, 80),
                 id_g1 = tc::idesc_bf16_f32_mn(128, 144);
  uint32_t phase = 0;
  bool ok = true, any = false;
  int b = 0;
  float loss = 0.0f, correct = 0.0f;
  const float cw[3] = {cw0, cw1, cw2};

  if (tile < ntiles && tid == 0) {
    mma_chain(tm, TT_D1, sX[0], kSlab, sW1, kHid * 16, kIn / 16, id64, false);
    tc::mma_commit(&bar);
  }
  for (; tile < ntiles; tile += gridDim.x) {
    const int64_t next = tile + gridDim.x;
    const bool has_next = next < ntiles;
    // ---- layer 1 done: h1, gelu'(z1)
    if (!(ok = wait_phase(&bar, phase, &abort_flag))) break;
    {
      float v[32], gp[32];
      tmem_row32(lane + TT_D1 + c0, v);
#pragma unroll
      for (int j = 0; j < 32; ++j) gelu_and_grad(v[j] + sB[c0 + j], v[j], gp[j]);
      store_row32(sH, t, 4 * hh, v);
      tmem_store32(lane + TT_D1 + c0, gp);
      tc::tmem_wait_st();
    }
    tc::fence_async_smem();
    tc_sync();
    if (tid == 0) {
      mma_chain(tm, TT_D2, sH, kSlab, sW2, kHid * 16, kHid / 16, id64, false);
      tc::mma_commit(&bar);
    }
    // ---- layer 2 done (and the previous tile's weight gradients): the
    //      next tile's rows into registers; h2, logits, softmax, dz3, dz2
    if (!(ok = wait_phase(&bar, phase, &abort_flag))) break;
    if (has_next) load_tile(next);
    {
      float h[32], gp[32];
      tmem_row32(lane + TT_D2 + c0, h);
#pragma unroll
      for (int j = 0; j < 32; ++j) {
        gelu_and_grad(h[j] + sB[kHid + c0 + j], h[j], gp[j]);
        h[j] = bf16_round(h[j]);  // the value the tile holds
      }
      store_row32(sH2, t, 4 * hh, h);
      // logits: this half's partial sums, the other half's through smem
      float zp[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
      for (int j = 0; j < 32; ++j)
#pragma unroll
        for (int o = 0; o < kOut; ++o) zp[o] = fmaf(h[j], sW3f[o * kHid + c0 + j], zp[o]);
      if (hh == 1) sXch[t] = make_float4(zp[0], zp[1], zp[2], 0.0f);
      asm volatile("bar.sync %0, 64;" ::"r"(pair_bar) : "memory");
      if (hh == 0) {
        const float4 q = sXch[t];
        const int y = ycur;
        const float wy = (y >= 0 && y < kOut) ? cw[y] * inv_n : 0.0f;
        const float z[3] = {zp[0] + q.x + sB[2 * kHid + 0], zp[1] + q.y + sB[2 * kHid + 1],
                            zp[2] + q.z + sB[2 * kHid + 2]};
        const float m = fmaxf(z[0], fmaxf(z[1], z[2]));
        float e[3], se = 0.0f;
#pragma unroll
        for (int o = 0; o < kOut; ++o) { e[o] = expf(z[o] - m); se += e[o]; }
        const float inv = 1.0f / se;
        int am = 0;
        if (z[1] > z[am]) am = 1;
        if (z[2] > z[am]) am = 2;
        float dz[3] = {0.0f, 0.0f, 0.0f};
        if (wy != 0.0f) {
          loss += wy * (logf(se) + m - z[y]);
#pragma unroll
          for (int o = 0; o < kOut; ++o) dz[o] = bf16_round(wy * (e[o] * inv - (o == y ? 1.0f : 0.0f)));
        }
        if (y >= 0 && y < kOut && am == y) correct += 1.0f;
        *reinterpret_cast<uint4 *>(sDZ3 + t * 16) =
            make_uint4(pack_bf16(dz[0], dz[1]), pack_bf16(dz[2], 0.0f), 0u, 0u);
        sXch[t] = make_float4(dz[0], dz[1], dz[2], 0.0f);
      }
      asm volatile("bar.sync %0, 64;" ::"r"(pair_bar) : "memory");
      // dz2 = (dz3 W3) gelu'(z2) over this half's columns
      const float4 d3 = sXch[t];
#pragma unroll
      for (int j = 0; j < 32; ++j) {
        const float dh = fmaf(d3.x, sW3f[c0 + j],
                              fmaf(d3.y, sW3f[kHid + c0 + j], d3.z * sW3f[2 * kHid + c0 + j]));
        gp[j] *= dh;
      }
      store_row32(sDZ2, t, 4 * hh, gp);
    }
    tc::fence_async_smem();
    tc_sync();
    if (tid == 0) {
      mma_chain(tm, TT_D2, sDZ2, kSlab, sW2T, kHid * 16, kHid / 16, id64, false);
      tc::mma_commit(&bar);
      // [dW2 | dW3]^T += [h1 | h2]^T [dz2 | dz3] (K = the tile's rows)
      for (int s = 0; s < kRows / 16; ++s)
        tc::mma_bf16(tm + TT_GCAT, tc::smem_desc(sH + 256 * s, 128, kSlab),
                     tc::smem_desc(sDZ2 + 256 * s, 128, kSlab), id_gcat, (any || s > 0) ? 1u : 0u);
    }
    // ---- dz1 = dh1 gelu'(z1); the next tile's rows into the other buffer
    if (!(ok = wait_phase(&bar, phase, &abort_flag))) break;
    {
      float dh[32], gp[32];
      tmem_row32(lane + TT_D2 + c0, dh);
      tmem_row32(lane + TT_D1 + c0, gp);
#pragma unroll
      for (int j = 0; j < 32; ++j) dh[j] *= gp[j];
      store_row32(sDZ, t, 4 * hh, dh);
    }
    if (has_next) store_tile(sX[b ^ 1]);
    ycur = ylab;
    tc::fence_async_smem();
    tc_sync();
    if (tid == 0) {
      if (has_next) {
        mma_chain(tm, TT_D1, sX[b ^ 1], kSlab, sW1, kHid * 16, kIn / 16, id64, false);
        tc::mma_commit(&bar);
      }
      // [dW1 | db1 db2 db3]^T += [x | 1]^T [dz1 | dz2 | dz3]
      for (int s = 0; s < kRows / 16; ++s)
        tc::mma_bf16(tm + TT_G1, tc::smem_desc(sX[b] + 256 * s, 128, kSlab),
                     tc::smem_desc(sDZ + 256 * s, 128, kSlab), id_g1, (any || s > 0) ? 1u : 0u);
      if (!has_next) tc::mma_commit(&bar);
    }
    any = true;
    b ^= 1;
  }
  if (ok && any) ok = wait_phase(&bar, phase, &abort_flag);

  if (ok && any) {
    // lanes of [h1|h2]^T [dz2|dz3]: hidden unit t of h1 (t < 64) or h2
    if (t < kHid) {
      float c[32];
      tmem_row32(lane + TT_GCAT + c0, c);
      for (int o = 0; o < 32; ++o) atomicAdd(&grad[P_W2 + (c0 + o) * kHid + t], c[o]);
    } else if (hh == 0) {
      uint32_t r[16];
      tc::tmem_ld16(lane + TT_GCAT + kHid, r);
      tc::tmem_wait_ld16(r);
      for (int o = 0; o < kOut; ++o) atomicAdd(&grad[P_W3 + o * kHid + (t - kHid)], __uint_as_float(r[o]));
    }
    // lanes of [x|1]^T [dz1|dz2|dz3]: input feature t, or the ones row
    {
      float c[32];
      tmem_row32(lane + TT_G1 + c0, c);
      if (t < kIn) {
        for (int o = 0; o < 32; ++o) atomicAdd(&grad[P_W1 + (c0 + o) * kIn + t], c[o]);
      } else if (t == kOnesRow) {
        for (int o = 0; o < 32; ++o) atomicAdd(&grad[P_B1 + c0 + o], c[o]);
      }
    }
    if ((warp & 3) == (kOnesRow >> 5)) {
      // the ones row's dz2 and dz3 columns: db2 and db3
      float c[32];
      tmem_row32(lane + TT_G1 + kHid + c0, c);
      if (t == kOnesRow)
        for (int o = 0; o < 32; ++o) atomicAdd(&grad[P_B2 + c0 + o], c[o]);
      if (hh == 0) {
        uint32_t r[16];
        tc::tmem_ld16(lane + TT_G1 + 2 * kHid, r);
        tc::tmem_wait_ld16(r);
        if (t == kOnesRow)
          for (int o = 0; o < kOut; ++o) atomicAdd(&grad[P_B3 + o], __uint_as_float(r[o]));
      }
    }
  }
  if (hh == 0) {
    for (int off = 16; off > 0; off >>= 1) {
      loss += __shfl_xor_sync(0xffffffffu, loss, off);
      correct += __shfl_xor_sync(0xffffffffu, correct, off);
    }
    if ((tid & 31) == 0) {
      atomicAdd(&stats[0], loss);
      atomicAdd(&stats[1], correct);
    }
  }
  if (!ok) {
    if (tid == 0) {
      atomicExch(err, 1);
      tc::mma_commit(&bar);
    }
    // let the MMAs already issued finish (bounded) before freeing their memory
    tc::mbar_wait_bounded(&bar, phase, kWaitCycles);
  }
  tc_sync();
  if (warp == 0) tc::tmem_dealloc(tm, T_COLS_TRAIN);
}

// Layer 2's activations and the logits of this thread's row (one thread per
// row): h2 = gelu(z2 + b2) rounded to bf16, z3 = h2 W3^T + b3 accumulated
// in f32 on the CUDA cores (W3 has 3 rows: no third MMA round trip).
__device__ __forceinline__ void logits_row(uint32_t taddr_d2, const float *sB, const float *sW3f,
                                           float (&z)[3]) {
  float h[64];
  tmem_row64(taddr_d2, sB + kHid, h);
#pragma unroll
  for (int o = 0; o < kOut; ++o) z[o] = sB[2 * kHid + o];
#pragma unroll
  for (int j = 0; j < kHid; ++j) {
    const float g = bf16_round(gelu(h[j]));
#pragma unroll
    for (int o = 0; o < kOut; ++o) z[o] = fmaf(g, sW3f[o * kHid + j], z[o]);
  }
}

// ---------------------------------------------------------------------------
// Inference: logits and argmax class per row.
__global__ void __launch_bounds__(kThreads)
    mlp_forward_kernel(const float *__restrict__ P, const uint16_t *__restrict__ feat, int64_t n,
                       uint8_t *__restrict__ cls, float *__restrict__ logits, int *__restrict__ err) {
  extern __shared__ __align__(1024) uint8_t smem[];
  __shared__ uint64_t bar;
  __shared__ uint32_t tbase;
  __shared__ int abort_flag;
  using S = FwdSmem;
  uint8_t *sX = smem + S::X, *sH1 = smem + S::H1, *sW1 = smem + S::W1, *sW2 = smem + S::W2;
  float *sB = reinterpret_cast<float *>(smem + S::BIAS);
  float *sW3f = reinterpret_cast<float *>(smem + S::W3F);
  const int t = threadIdx.x;
  load_weights(P, sW1, sW2, nullptr, sB, sW3f);
  if (t == 0) {
    tc::mbar_init(&bar, 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if ((t >> 5) == 0) {
    tc::tmem_alloc(&tbase, T_COLS_FWD);
    tc::tmem_relinquish();
  }
  tc::fence_async_smem();
  tc_sync();
  const uint32_t tm = tbase;
  const uint32_t lane_off = (uint32_t)((t & ~31) << 16);
  const uint32_t id64 = tc::idesc_bf16_f32(128, kHid);
  uint32_t phase = 0;
  bool ok = true;
  for (int64_t tile = blockIdx.x; ok && tile * kRows < n; tile += gridDim.x) {
    const int64_t row = tile * kRows + t;
    const bool valid = row < n;
    load_x_row(feat, row, valid, t, sX);
    tc::fence_async_smem();
    tc_sync();
    if (t == 0) mma_chain(tm, T_D1, sX, kRows * 16, sW1, kHid * 16, kIn / 16, id64, false);
    if (!(ok = commit_and_wait(&bar, phase, &abort_flag))) break;
    {
      float v[64];
      tmem_row64(tm + lane_off + T_D1, sB, v);
#pragma unroll
      for (int j = 0; j < kHid; ++j) v[j] = gelu(v[j]);
      store_row64(sH1, t, v);
    }
    tc::fence_async_smem();
    tc_sync();
    if (t == 0) mma_chain(tm, T_D2, sH1, kRows * 16, sW2, kHid * 16, kHid / 16, id64, false);
    if (!(ok = commit_and_wait(&bar, phase, &abort_flag))) break;
    {
      float z[3];
      logits_row(tm + lane_off + T_D2, sB, sW3f, z);
      int am = 0;
      if (z[1] > z[am]) am = 1;
      if (z[2] > z[am]) am = 2;
      if (valid) {
        cls[row] = (uint8_t)am;
        if (logits) {
          logits[row * 3 + 0] = z[0];
          logits[row * 3 + 1] = z[1];
          logits[row * 3 + 2] = z[2];
        }
      }
    }
    // the next tile's layer-1 MMA overwrites D1 only after every thread's
    // loads above (tc_sync at the top of the loop)
  }
  if (!ok) {
    if (t == 0) atomicExch(err, 1);
    tc::mbar_wait_bounded(&bar, phase, kWaitCycles);
  }
  tc_sync();
  if ((t >> 5) == 0) tc::tmem_dealloc(tm, T_COLS_FWD);
}

__global__ void adam_kernel(float *__restrict__ P, const float *__restrict__ g, float *__restrict__ m,
                            float *__restrict__ v, int n, float lr, float c1, float c2) {
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    P[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
  }
}

// ---------------------------------------------------------------------------
// Plain criterion and features.

struct RuleDev {
  double left, right, yc, half_h;
  int n_rect, n_rect_c;
  int torefine[IBGPU_TAG_MAX_LEVELS], toderefine[IBGPU_TAG_MAX_LEVELS];
  double ru[IBGPU_TAG_MAX_LEVELS], rd[IBGPU_TAG_MAX_LEVELS], rh[IBGPU_TAG_MAX_LEVELS];
  double bl[IBGPU_TAG_MAX_LEVELS], bh[IBGPU_TAG_MAX_LEVELS], nm[IBGPU_TAG_MAX_LEVELS];
  double dru[IBGPU_TAG_MAX_LEVELS], drd[IBGPU_TAG_MAX_LEVELS], drh[IBGPU_TAG_MAX_LEVELS];
  double dbl[IBGPU_TAG_MAX_LEVELS], dbh[IBGPU_TAG_MAX_LEVELS], dnm[IBGPU_TAG_MAX_LEVELS];
};

__device__ __forceinline__ bool in_region(double x, double y, double sd, int k, int nrect,
                                          const RuleDev &R, const double *ru, const double *rd,
                                          const double *rh, const double *bl, const double *bh,
                                          const double *nm) {
  if (k < nrect) return x - R.left > -ru[k] && x - R.right < rd[k] && fabs(y - R.yc) < rh[k];
  bool near = true;
  if (nm[k] > 0.0) {
    const double m = nm[k];
    near = x > R.left - m && x < R.right + m && fabs(y - R.yc) < R.half_h + m;
  }
  return near && sd > bl[k] && sd < bh[k];
}

__global__ void tag_plain_kernel(RuleDev R, int64_t n, const int32_t *__restrict__ lvl,
                                 const double *__restrict__ xc, const double *__restrict__ yc,
                                 const double *__restrict__ sd, uint8_t *__restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int l = lvl[i];
    const double x = xc[i], y = yc[i], s = sd[i];
    uint8_t b = 0;
    if (R.torefine[l] && in_region(x, y, s, l, R.n_rect, R, R.ru, R.rd, R.rh, R.bl, R.bh, R.nm))
      b |= IBGPU_TAG_REFINE;
    if (l >= 1 && R.toderefine[l] &&
        !in_region(x, y, s, l - 1, R.n_rect_c, R, R.dru, R.drd, R.drh, R.dbl, R.dbh, R.dnm))
      b |= IBGPU_TAG_COARSEN;
    out[i] = b;
  }
}

struct FeatConst {
  double inv_rho, inv_c, inv_p;  // freestream scales
  double left, yc, inv_chord;
  double dh[IBGPU_TAG_MAX_LEVELS];
};

__global__ void features_kernel(FeatConst F, int64_t n, const int64_t *__restrict__ slot,
                                const int32_t *__restrict__ lvl, const double *__restrict__ xc,
                                const double *__restrict__ yc, const double *__restrict__ sd,
                                const int32_t *__restrict__ tile_nb,
                                const uint8_t *__restrict__ flags, const double *__restrict__ rho,
                                const double *__restrict__ u, const double *__restrict__ v,
                                const double *__restrict__ p, uint16_t *__restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t s0 = slot[i];
    const int tile = (int)(s0 >> 8), lx = (int)(s0 & 15), ly = (int)((s0 >> 4) & 15);
    uint16_t *o = out + i * kIn;
    const double cr = rho[s0], cu = u[s0], cv = v[s0], cp = p[s0];
    for (int dy = -2; dy <= 2; ++dy) {
      for (int dx = -2; dx <= 2; ++dx) {
        const int nx = lx + dx, ny = ly + dy;
        const int ox = nx < 0 ? -1 : (nx >= kTile ? 1 : 0);
        const int oy = ny < 0 ? -1 : (ny >= kTile ? 1 : 0);
        const int nb = tile_nb[tile * 9 + (oy + 1) * 3 + (ox + 1)];
        double qr = cr, qu = cu, qv = cv, qp = cp;
        if (nb >= 0) {
          const int64_t s = (int64_t)nb * kTileCells + (ny - oy * kTile) * kTile + (nx - ox * kTile);
          if (flags[s] & CF_PRESENT) {
            qr = rho[s];
            qu = u[s];
            qv = v[s];
            qp = p[s];
          }
        }
        // separately rounded products and sums (no contraction), so the
        // features are reproducible on the host
        const int k = (dy + 2) * 5 + (dx + 2);
        o[k] = bf16_bits((float)__dadd_rn(__dmul_rn(qr, F.inv_rho), -1.0));
        o[25 + k] = bf16_bits((float)__dmul_rn(qu, F.inv_c));
        o[50 + k] = bf16_bits((float)__dmul_rn(qv, F.inv_c));
        o[75 + k] = bf16_bits((float)__dadd_rn(__dmul_rn(qp, F.inv_p), -1.0));
      }
    }
    const int l = lvl[i];
    const double s = sd[i];
    const double a = fmin(fmax(s / F.dh[l], -8.0), 8.0) * 0.125;
    const double b = fmin(fmax(__dmul_rn(s, F.inv_chord), -4.0), 4.0) * 0.25;
    const double rx = __dmul_rn(__dmul_rn(__dsub_rn(xc[i], F.left), F.inv_chord), 0.125);
    const double ry = __dmul_rn(__dmul_rn(__dsub_rn(yc[i], F.yc), F.inv_chord), 0.125);
    o[100] = bf16_bits((float)a);
    o[101] = bf16_bits((float)b);
    o[102] = bf16_bits((float)rx);
    o[103] = bf16_bits((float)ry);
    o[104] = bf16_bits((float)fabs(ry));
    const int lc = l < 6 ? l : 6;
    for (int e = 0; e < 7; ++e) o[105 + e] = (e == lc) ? (uint16_t)0x3F80u : (uint16_t)0u;
  }
}



// ---------------------------------------------------------------------------
// Deployment on the mesh: every normal cell of the context, features
// gathered straight from the state into the A tile (no feature matrix in
// HBM; each thread assembles its row's 112 values in registers and stores
// them as 14 16-byte words), the two hidden layers on the tensor cores, the
// logits and their argmax on the CUDA cores, mapped to tag bits.  Shared
// memory: X, h1, weights; Tensor Memory: 128 columns (D1 0..63, D2
// 64..127) so several CTAs share an SM.
struct MeshSmem {
  static constexpr int X = 0;
  static constexpr int H1 = X + kRows * kIn * 2;
  static constexpr int W1 = H1 + kRows * kHid * 2;
  static constexpr int W2 = W1 + kHid * kIn * 2;
  static constexpr int BIAS = W2 + kHid * kHid * 2;
  static constexpr int W3F = BIAS + 1024;  // W3 rounded to bf16, as f32 [3 x 64]
  static constexpr int BYTES = W3F + 1024;
};
constexpr uint32_t T_COLS_MESH = 128;

struct MeshArgs {
  const int32_t *tile_nb, *tile_level;
  const int2 *tile_org;
  const uint8_t *flags;
  const double *rho, *u, *v, *p;
  const double *signdis;  // per slot or null (far from any wall)
  uint8_t *tags;          // per slot
  int64_t nslots;
};

struct FeatScale {
  double inv_rho, inv_c, inv_p, left, yc, inv_chord;
  double dx[IBGPU_TAG_MAX_LEVELS], dy[IBGPU_TAG_MAX_LEVELS];
  // levels on which the rule requests refinement / coarsening (bit l); the
  // learned decision, like the plain one, only acts where requested
  unsigned refine_levels, coarsen_levels;
};

// The rule's request masks over the levels (coarsening never on level 0).
inline void request_masks(const ibgpu_tag_rule *rule, unsigned &refine, unsigned &coarsen) {
  refine = coarsen = 0u;
  for (int k = 0; k < IBGPU_TAG_MAX_LEVELS; ++k) {
    if (rule->torefine[k]) refine |= 1u << k;
    if (k >= 1 && rule->toderefine[k]) coarsen |= 1u << k;
  }
}

// Class (0 refine, 1 coarsen, 2 keep) -> tag bits on level l under the masks.
__host__ __device__ __forceinline__ uint8_t masked_tag(int c, int l, unsigned refine,
                                                       unsigned coarsen) {
  if (c == 0 && ((refine >> l) & 1u)) return (uint8_t)IBGPU_TAG_REFINE;
  if (c == 1 && ((coarsen >> l) & 1u)) return (uint8_t)IBGPU_TAG_COARSEN;
  return 0;
}

__global__ void class_to_tag_kernel(const uint8_t *__restrict__ cls, int64_t n,
                                    const int32_t *__restrict__ lvl, unsigned refine,
                                    unsigned coarsen, uint8_t *__restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = masked_tag(cls[i], lvl[i], refine, coarsen);
}

__global__ void __launch_bounds__(kThreads)
    mlp_tag_mesh_kernel(const float *__restrict__ P, MeshArgs m, FeatScale F, int *__restrict__ err) {
  extern __shared__ __align__(1024) uint8_t smem[];
  __shared__ uint64_t bar;
  __shared__ uint32_t tbase;
  __shared__ int abort_flag;
  constexpr int kSW = kTile + 4, kSH = 8 + 4;  // staged region of a half tile
  __shared__ float4 sn[kSH * kSW];
  __shared__ uint8_t sp[kSH * kSW];
  using S = MeshSmem;
  uint8_t *sX = smem + S::X, *sH1 = smem + S::H1, *sW1 = smem + S::W1, *sW2 = smem + S::W2;
  float *sB = reinterpret_cast<float *>(smem + S::BIAS);
  float *sW3f = reinterpret_cast<float *>(smem + S::W3F);
  const int t = threadIdx.x;
  load_weights(P, sW1, sW2, nullptr, sB, sW3f);
  if (t == 0) {
    tc::mbar_init(&bar, 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if ((t >> 5) == 0) {
    tc::tmem_alloc(&tbase, T_COLS_MESH);
    tc::tmem_relinquish();
  }
  tc::fence_async_smem();
  tc_sync();
  const uint32_t tm = tbase;
  const uint32_t lane_off = (uint32_t)((t & ~31) << 16);
  const uint32_t id64 = tc::idesc_bf16_f32(128, kHid);
  uint32_t phase = 0;
  bool ok = true;
  const int64_t nitems = m.nslots / kRows;  // half tiles
  for (int64_t item = blockIdx.x; ok && item < nitems; item += gridDim.x) {
    const int64_t slot = item * kRows + t;
    const bool normal = (m.flags[slot] & CF_NORMAL) != 0;
    // stage the freestream-normalised (rho, u, v, p) of the 12 x 20 region
    // around this half tile (rows -2..9 of the half, columns -2..17)
    const int half = (int)(item & 1);
    {
      const int tile = (int)(item >> 1);
      for (int r = t; r < kSH * kSW; r += kThreads) {
        const int rx = r % kSW - 2, ry = r / kSW - 2 + 8 * half;
        const int ox = rx < 0 ? -1 : (rx >= kTile ? 1 : 0);
        const int oy = ry < 0 ? -1 : (ry >= kTile ? 1 : 0);
        const int nb = m.tile_nb[tile * 9 + (oy + 1) * 3 + (ox + 1)];
        uint8_t pres = 0;
        float4 q = make_float4(0.f, 0.f, 0.f, 0.f);
        if (nb >= 0) {
          const int64_t s = (int64_t)nb * kTileCells + (ry - oy * kTile) * kTile + (rx - ox * kTile);
          if (m.flags[s] & CF_PRESENT) {
            pres = 1;
            q = make_float4((float)(m.rho[s] * F.inv_rho - 1.0), (float)(m.u[s] * F.inv_c),
                            (float)(m.v[s] * F.inv_c), (float)(m.p[s] * F.inv_p - 1.0));
          }
        }
        sn[r] = q;
        sp[r] = pres;
      }
    }
    __syncthreads();
    {
      // feature row of this thread's cell (zeros for other slots), built in
      // registers and stored as 14 16-byte words of the A tile
      float fv[kIn];
#pragma unroll
      for (int k = 0; k < kIn; ++k) fv[k] = 0.0f;
      if (normal) {
        const int tile = (int)(slot >> 8), lx = (int)(slot & 15), ly = (int)((slot >> 4) & 15);
        const int rc = ((ly - 8 * half) + 2) * kSW + (lx + 2);  // centre in the staged region
        const float4 c = sn[rc];
#pragma unroll
        for (int dy = -2; dy <= 2; ++dy) {
#pragma unroll
          for (int dx = -2; dx <= 2; ++dx) {
            const int r = rc + dy * kSW + dx;
            const float4 q = sp[r] ? sn[r] : c;
            const int k = (dy + 2) * 5 + (dx + 2);
            fv[k] = q.x;
            fv[25 + k] = q.y;
            fv[50 + k] = q.z;
            fv[75 + k] = q.w;
          }
        }
        const int l = m.tile_level[tile];
        const int2 org = m.tile_org[tile];
        const double xc = (org.x + lx + 0.5) * F.dx[l], yc = (org.y + ly + 0.5) * F.dy[l];
        const double sd = m.signdis ? m.signdis[slot] : 1e30;
        fv[100] = (float)(fmin(fmax(sd / F.dx[l], -8.0), 8.0) * 0.125);
        fv[101] = (float)(fmin(fmax(sd * F.inv_chord, -4.0), 4.0) * 0.25);
        const double ry = (yc - F.yc) * F.inv_chord * 0.125;
        fv[102] = (float)((xc - F.left) * F.inv_chord * 0.125);
        fv[103] = (float)ry;
        fv[104] = (float)fabs(ry);
        const int lc = l < 6 ? l : 6;
#pragma unroll
        for (int e = 0; e < 7; ++e) fv[105 + e] = e == lc ? 1.0f : 0.0f;
      }
#pragma unroll
      for (int c = 0; c < kIn / 8; ++c) {
        uint4 w;
        w.x = pack_bf16(fv[8 * c + 0], fv[8 * c + 1]);
        w.y = pack_bf16(fv[8 * c + 2], fv[8 * c + 3]);
        w.z = pack_bf16(fv[8 * c + 4], fv[8 * c + 5]);
        w.w = pack_bf16(fv[8 * c + 6], fv[8 * c + 7]);
        *reinterpret_cast<uint4 *>(sX + c * (kRows * 16) + t * 16) = w;
      }
    }
    tc::fence_async_smem();
    tc_sync();
    if (t == 0) mma_chain(tm, 0, sX, kRows * 16, sW1, kHid * 16, kIn / 16, id64, false);
    if (!(ok = commit_and_wait(&bar, phase, &abort_flag))) break;
    {
      float h[64];
      tmem_row64(tm + lane_off + 0, sB, h);
#pragma unroll
      for (int j = 0; j < kHid; ++j) h[j] = gelu(h[j]);
      store_row64(sH1, t, h);
    }
    tc::fence_async_smem();
    tc_sync();
    if (t == 0) mma_chain(tm, 64, sH1, kRows * 16, sW2, kHid * 16, kHid / 16, id64, false);
    if (!(ok = commit_and_wait(&bar, phase, &abort_flag))) break;
    {
      float z[3];
      logits_row(tm + lane_off + 64, sB, sW3f, z);
      int am = 0;
      if (z[1] > z[am]) am = 1;
      if (z[2] > z[am]) am = 2;
      m.tags[slot] = normal ? masked_tag(am, m.tile_level[slot >> 8], F.refine_levels,
                                         F.coarsen_levels)
                            : (uint8_t)0;
    }
    // the next item's MMAs overwrite D1 and D2 only after the tc_sync that
    // follows its staging (every lane read above by then)
  }
  if (!ok) {
    if (t == 0) atomicExch(err, 1);
    tc::mbar_wait_bounded(&bar, phase, kWaitCycles);
  }
  tc_sync();
  if ((t >> 5) == 0) tc::tmem_dealloc(tm, T_COLS_MESH);
}

// Plain criterion over every normal cell of the context (centres from the
// tile origins, signed distance per slot or far from any wall).
__global__ void tag_plain_mesh_kernel(RuleDev R, MeshArgs m, FeatScale F) {
  for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < m.nslots;
       s += (int64_t)gridDim.x * blockDim.x) {
    uint8_t b = 0;
    if (m.flags[s] & CF_NORMAL) {
      const int tile = (int)(s >> 8), lx = (int)(s & 15), ly = (int)((s >> 4) & 15);
      const int l = m.tile_level[tile];
      const int2 org = m.tile_org[tile];
      const double x = (org.x + lx + 0.5) * F.dx[l], y = (org.y + ly + 0.5) * F.dy[l];
      const double sd = m.signdis ? m.signdis[s] : 1e30;
      if (R.torefine[l] && in_region(x, y, sd, l, R.n_rect, R, R.ru, R.rd, R.rh, R.bl, R.bh, R.nm))
        b |= IBGPU_TAG_REFINE;
      if (l >= 1 && R.toderefine[l] &&
          !in_region(x, y, sd, l - 1, R.n_rect_c, R, R.dru, R.drd, R.drh, R.dbl, R.dbh, R.dnm))
        b |= IBGPU_TAG_COARSEN;
    }
    m.tags[s] = b;
  }
}

__global__ void gather_rows_u8(const uint8_t *__restrict__ per_slot, const int32_t *__restrict__ cell_slot,
                               int64_t n, uint8_t *__restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = per_slot[cell_slot[i]];
}

__global__ void scatter_rows_f64(const double *__restrict__ rows, const int32_t *__restrict__ cell_slot,
                                 int64_t n, double *__restrict__ per_slot) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    per_slot[cell_slot[i]] = rows[i];
}

}  // namespace ind
}  // namespace ibgpu

// ===========================================================================
// C ABI
using namespace ibgpu;
using namespace ibgpu::ind;

namespace {

int cuda_err(cudaError_t e, const char *what) {
  set_last_error(std::string(what) + ": " + cudaGetErrorString(e));
  return IBGPU_E_CUDA;
}
#define CKI(call)                                      \
  do {                                                 \
    cudaError_t e_ = (call);                           \
    if (e_ != cudaSuccess) return cuda_err(e_, #call); \
  } while (0)

// Device scratch freed at scope exit.
struct DevBuf {
  void *p = nullptr;
  ~DevBuf() { cudaFree(p); }
  template <typename T>
  T *as() { return static_cast<T *>(p); }
};

int grid_for(int64_t n, int nsm, int threads) {
  int64_t g = (n + threads - 1) / threads;
  const int64_t cap = (int64_t)nsm * 8;
  return (int)(g < 1 ? 1 : (g > cap ? cap : g));
}

RuleDev to_dev(const ibgpu_tag_rule *r) {
  RuleDev R;
  R.left = r->body_left_x;
  R.right = r->body_right_x;
  R.yc = r->body_center_y;
  R.half_h = r->body_half_height;
  R.n_rect = r->n_rect;
  R.n_rect_c = r->n_rect_coarsen;
  for (int k = 0; k < IBGPU_TAG_MAX_LEVELS; ++k) {
    R.torefine[k] = r->torefine[k];
    R.toderefine[k] = r->toderefine[k];
    R.ru[k] = r->rect_up[k];
    R.rd[k] = r->rect_down[k];
    R.rh[k] = r->rect_half[k];
    R.bl[k] = r->band_lo[k];
    R.bh[k] = r->band_hi[k];
    R.nm[k] = r->near_margin[k];
    R.dru[k] = r->derect_up[k];
    R.drd[k] = r->derect_down[k];
    R.drh[k] = r->derect_half[k];
    R.dbl[k] = r->deband_lo[k];
    R.dbh[k] = r->deband_hi[k];
    R.dnm[k] = r->denear_margin[k];
  }
  return R;
}

int check_cells(const ibgpu_tag_cells *c) {
  if (!c || c->n < 0) return IBGPU_E_ARG;
  if (c->n == 0) return IBGPU_OK;
  if (!c->level || !c->xc || !c->yc || !c->signdis) return IBGPU_E_ARG;
  for (int64_t i = 0; i < c->n; ++i)
    if (c->level[i] < 0 || c->level[i] >= IBGPU_TAG_MAX_LEVELS) return IBGPU_E_ARG;
  return IBGPU_OK;
}

template <typename T>
int upload(DevBuf &b, const T *h, int64_t n, cudaStream_t st) {
  CKI(cudaMalloc(&b.p, (size_t)(n > 0 ? n : 1) * sizeof(T)));
  if (n > 0) CKI(cudaMemcpyAsync(b.p, h, (size_t)n * sizeof(T), cudaMemcpyHostToDevice, st));
  return IBGPU_OK;
}

int kernel_error_check(int *d_err, cudaStream_t st) {
  int h = 0;
  CKI(cudaMemcpyAsync(&h, d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
  CKI(cudaStreamSynchronize(st));
  if (h) {
    CKI(cudaMemsetAsync(d_err, 0, sizeof(int), st));
    CKI(cudaStreamSynchronize(st));
    set_last_error("tensor-core wait ran out of its time limit");
    return IBGPU_E_TIMEOUT;
  }
  return IBGPU_OK;
}

// opt in to the large dynamic shared-memory carve-out (per device, cheap)
int configure_smem() {
  CKI(cudaFuncSetAttribute(mlp_tag_mesh_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           MeshSmem::BYTES));
  CKI(cudaFuncSetAttribute(mlp_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           TrainSmem::BYTES));
  CKI(cudaFuncSetAttribute(mlp_forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           FwdSmem::BYTES));
  return IBGPU_OK;
}

int features_impl(const CtxView &V, const ibgpu_ctx *ctx, const ibgpu_tag_rule *rule,
                  const ibgpu_tag_cells *cells, uint16_t *d_feat) {
  const int64_t n = cells->n;
  if (n == 0) return IBGPU_OK;
  if (!cells->ix || !cells->iy || !d_feat) return IBGPU_E_ARG;
  if (!V.has_topology || !V.has_state) return IBGPU_E_STATE;
  std::vector<int64_t> slots((size_t)n);
  for (int64_t i = 0; i < n; ++i) {
    slots[i] = ctx_slot_at(ctx, cells->level[i], cells->ix[i], cells->iy[i]);
    if (slots[i] < 0) {
      set_last_error("indicator box is not a cell of the uploaded topology");
      return IBGPU_E_ARG;
    }
  }
  FeatConst F;
  const double rho_inf = V.cc.initvar[0], p_inf = V.cc.initvar[4];
  F.inv_rho = 1.0 / rho_inf;
  F.inv_p = 1.0 / p_inf;
  F.inv_c = 1.0 / std::sqrt(V.cc.gama * p_inf / rho_inf);
  F.left = rule->body_left_x;
  F.yc = rule->body_center_y;
  F.inv_chord = 1.0 / (rule->body_right_x - rule->body_left_x);
  for (int k = 0; k < IBGPU_TAG_MAX_LEVELS; ++k) F.dh[k] = V.cc.lev[k].dx > 0 ? V.cc.lev[k].dx : 1.0;
  cudaStream_t st = V.stream;
  DevBuf ds, dl, dx, dy, dsd;
  int rc;
  if ((rc = upload(ds, slots.data(), n, st)) || (rc = upload(dl, cells->level, n, st)) ||
      (rc = upload(dx, cells->xc, n, st)) || (rc = upload(dy, cells->yc, n, st)) ||
      (rc = upload(dsd, cells->signdis, n, st)))
    return rc;
  features_kernel<<<grid_for(n, V.nsm, 128), 128, 0, st>>>(
      F, n, ds.as<int64_t>(), dl.as<int32_t>(), dx.as<double>(), dy.as<double>(), dsd.as<double>(),
      V.tile_nb, V.flags, V.s0[F_RHO], V.s0[F_U], V.s0[F_V], V.s0[F_P], d_feat);
  CKI(cudaGetLastError());
  CKI(cudaStreamSynchronize(st));
  return IBGPU_OK;
}

int launch_grad(const CtxView &V, const float *d_params, int64_t n, const uint16_t *d_feat,
                const uint8_t *d_label, const float class_weight[3], float *d_grad,
                float *d_stats) {
  const int64_t tiles = (n + kRows - 1) / kRows;
  const int grid = (int)std::min<int64_t>(tiles, (int64_t)V.nsm);
  mlp_grad_kernel<<<grid, kThreadsTrain, TrainSmem::BYTES, V.stream>>>(
      d_params, d_feat, d_label, n, class_weight[0], class_weight[1], class_weight[2],
      (float)(1.0 / (double)n), d_grad, d_stats, V.aux_err);
  CKI(cudaGetLastError());
  return IBGPU_OK;
}

int launch_adam(const CtxView &V, float *d_params, const float *d_grad, float *d_m, float *d_v,
                int step, float lr) {
  const float c1 = (float)(1.0 / (1.0 - std::pow(0.9, step)));
  const float c2 = (float)(1.0 / (1.0 - std::pow(0.999, step)));
  adam_kernel<<<grid_for(P_COUNT, V.nsm, 256), 256, 0, V.stream>>>(d_params, d_grad, d_m, d_v,
                                                                   P_COUNT, lr, c1, c2);
  CKI(cudaGetLastError());
  return IBGPU_OK;
}

int forward_impl(const CtxView &V, const float *d_params, int64_t n, const uint16_t *d_feat,
                 uint8_t *d_class, float *d_logits) {
  int rc = configure_smem();
  if (rc) return rc;
  const int64_t tiles = (n + kRows - 1) / kRows;
  const int grid = (int)std::min<int64_t>(tiles, (int64_t)V.nsm * 2);
  mlp_forward_kernel<<<grid, kThreads, FwdSmem::BYTES, V.stream>>>(d_params, d_feat, n, d_class,
                                                                   d_logits, V.aux_err);
  CKI(cudaGetLastError());
  return kernel_error_check(V.aux_err, V.stream);
}

}  // namespace

namespace ibgpu {
// Tags of every row of ctx's cell list enqueued on st (no synchronisation):
// the learned decision with d_params, else the plain criterion; *rows_out
// is the device array of the row tags (valid once st reaches it).
int tag_mesh_enqueue(ibgpu_ctx *ctx, const ibgpu_tag_rule *rule, const float *d_params,
                     cudaStream_t st, uint8_t **rows_out) {
  CtxView V;
  if (ctx_view(ctx, &V) != IBGPU_OK) return IBGPU_E_ARG;
  uint8_t *dtags = nullptr;
  double *dsd = nullptr;
  int rc;
  if ((rc = ctx_tags_buffer(ctx, &dtags)) || (rc = ctx_signdis_buffer(ctx, &dsd, false))) return rc;
  MeshArgs m;
  m.tile_nb = V.tile_nb;
  m.tile_level = V.tile_level;
  m.tile_org = V.tile_org;
  m.flags = V.flags;
  m.rho = V.s0[F_RHO];
  m.u = V.s0[F_U];
  m.v = V.s0[F_V];
  m.p = V.s0[F_P];
  m.signdis = dsd;
  m.tags = dtags;
  m.nslots = V.nslots;
  FeatScale F;
  const double rho_inf = V.cc.initvar[0], p_inf = V.cc.initvar[4];
  F.inv_rho = 1.0 / rho_inf;
  F.inv_p = 1.0 / p_inf;
  F.inv_c = 1.0 / std::sqrt(V.cc.gama * p_inf / rho_inf);
  F.left = rule->body_left_x;
  F.yc = rule->body_center_y;
  F.inv_chord = 1.0 / (rule->body_right_x - rule->body_left_x);
  for (int k = 0; k < IBGPU_TAG_MAX_LEVELS; ++k) {
    F.dx[k] = V.cc.lev[k].dx > 0 ? V.cc.lev[k].dx : 1.0;
    F.dy[k] = V.cc.lev[k].dy > 0 ? V.cc.lev[k].dy : 1.0;
  }
  request_masks(rule, F.refine_levels, F.coarsen_levels);
  if (d_params) {
    const int64_t items = V.nslots / kRows;
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(items, (int64_t)V.nsm * 3));
    mlp_tag_mesh_kernel<<<grid, kThreads, MeshSmem::BYTES, st>>>(d_params, m, F, V.aux_err);
  } else {
    tag_plain_mesh_kernel<<<grid_for(V.nslots, V.nsm, 256), 256, 0, st>>>(to_dev(rule), m, F);
  }
  CKI(cudaGetLastError());
  uint8_t *rows = dtags + V.nslots;
  gather_rows_u8<<<grid_for(V.ncells, V.nsm, 256), 256, 0, st>>>(dtags, V.cell_slot, V.ncells, rows);
  CKI(cudaGetLastError());
  *rows_out = rows;
  return IBGPU_OK;
}

int tag_mesh_prepare(bool learned) { return learned ? configure_smem() : IBGPU_OK; }

}  // namespace ibgpu

extern "C" {

int ibgpu_tag_plain(ibgpu_ctx *ctx, const ibgpu_tag_rule *rule, const ibgpu_tag_cells *cells,
                    uint8_t *out) {
  CtxView V;
  if (!rule || ctx_view(ctx, &V) != IBGPU_OK) return IBGPU_E_ARG;
  int rc = check_cells(cells);
  if (rc) return rc;
  const int64_t n = cells->n;
  if (n == 0) return IBGPU_OK;
  if (!out) return IBGPU_E_ARG;
  cudaStream_t st = V.stream;
  DevBuf dl, dx, dy, dsd, dout;
  if ((rc = upload(dl, cells->level, n, st)) || (rc = upload(dx, cells->xc, n, st)) ||
      (rc = upload(dy, cells->yc, n, st)) || (rc = upload(dsd, cells->signdis, n, st)))
    return rc;
  CKI(cudaMalloc(&dout.p, (size_t)n));
  tag_plain_kernel<<<grid_for(n, V.nsm, 256), 256, 0, st>>>(to_dev(rule), n, dl.as<int32_t>(),
                                                            dx.as<double>(), dy.as<double>(),
                                                            dsd.as<double>(), dout.as<uint8_t>());
  CKI(cudaGetLastError());
  CKI(cudaMemcpyAsync(out, dout.p, (size_t)n, cudaMemcpyDeviceToHost, st));
  CKI(cudaStreamSynchronize(st));
  return IBGPU_OK;
}

int ibgpu_indicator_features(ibgpu_ctx *ctx, const ibgpu_tag_rule *rule,
                             const ibgpu_tag_cells *cells, uint16_t *d_feat) {
  CtxView V;
  if (!rule || ctx_view(ctx, &V) != IBGPU_OK) return IBGPU_E_ARG;
  int rc = check_cells(cells);
  if (rc) return rc;
  return features_impl(V, ctx, rule, cells, d_feat);
}

int ibgpu_mlp_forward(ibgpu_ctx *ctx, const float *d_params, int64_t n, const uint16_t *d_feat,
                      uint8_t *d_class, float *d_logits) {
  CtxView V;
  if (ctx_view(ctx, &V) != IBGPU_OK || n < 0) return IBGPU_E_ARG;
  if (n == 0) return IBGPU_OK;
  if (!d_params || !d_feat || !d_class) return IBGPU_E_ARG;
  if ((reinterpret_cast<uintptr_t>(d_feat) & 15u) != 0) return IBGPU_E_ARG;
  return forward_impl(V, d_params, n, d_feat, d_class, d_logits);
}

int ibgpu_mlp_grad(ibgpu_ctx *ctx, const float *d_params, int64_t n, const uint16_t *d_feat,
                   const uint8_t *d_label, const float class_weight[3], float *d_grad,
                   float *d_stats) {
  CtxView V;
  if (ctx_view(ctx, &V) != IBGPU_OK || n < 0) return IBGPU_E_ARG;
  if (n == 0) return IBGPU_OK;
  if (!d_params || !d_feat || !d_label || !class_weight || !d_grad || !d_stats) return IBGPU_E_ARG;
  if ((reinterpret_cast<uintptr_t>(d_feat) & 15u) != 0) return IBGPU_E_ARG;
  int rc = configure_smem();
  if (rc) return rc;
  rc = launch_grad(V, d_params, n, d_feat, d_label, class_weight, d_grad, d_stats);
  if (rc) return rc;
  return kernel_error_check(V.aux_err, V.stream);
}

int ibgpu_mlp_train_step(ibgpu_ctx *ctx, float *d_params, float *d_m, float *d_v, float *d_grad,
                         int step, float lr, int64_t n, const uint16_t *d_feat,
                         const uint8_t *d_label, const float class_weight[3], float *d_stats) {
  CtxView V;
  if (ctx_view(ctx, &V) != IBGPU_OK || n <= 0 || step < 1) return IBGPU_E_ARG;
  if (!d_params || !d_m || !d_v || !d_grad || !d_feat || !d_label || !class_weight || !d_stats)
    return IBGPU_E_ARG;
  if ((reinterpret_cast<uintptr_t>(d_feat) & 15u) != 0) return IBGPU_E_ARG;
  int rc = configure_smem();
  if (rc) return rc;
  CKI(cudaMemsetAsync(d_grad, 0, (size_t)P_COUNT * sizeof(float), V.stream));
  rc = launch_grad(V, d_params, n, d_feat, d_label, class_weight, d_grad, d_stats);
  if (rc) return rc;
  rc = launch_adam(V, d_params, d_grad, d_m, d_v, step, lr);
  if (rc) return rc;
  return kernel_error_check(V.aux_err, V.stream);
}

int ibgpu_mlp_adam(ibgpu_ctx *ctx, float *d_params, const float *d_grad, float *d_m, float *d_v,
                   int step, float lr) {
  CtxView V;
  if (ctx_view(ctx, &V) != IBGPU_OK || step < 1 || !d_params || !d_grad || !d_m || !d_v)
    return IBGPU_E_ARG;
  return launch_adam(V, d_params, d_grad, d_m, d_v, step, lr);
}

int ibgpu_tag_learned(ibgpu_ctx *ctx, const ibgpu_tag_rule *rule, const ibgpu_tag_cells *cells,
                      const float *d_params, uint8_t *out) {
  CtxView V;
  if (!rule || ctx_view(ctx, &V) != IBGPU_OK) return IBGPU_E_ARG;
  int rc = check_cells(cells);
  if (rc) return rc;
  const int64_t n = cells->n;
  if (n == 0) return IBGPU_OK;
  if (!out || !d_params) return IBGPU_E_ARG;
  DevBuf feat, cls, tags, lvl;
  CKI(cudaMalloc(&feat.p, (size_t)n * kIn * sizeof(uint16_t)));
  CKI(cudaMalloc(&cls.p, (size_t)n));
  CKI(cudaMalloc(&tags.p, (size_t)n));
  if ((rc = upload(lvl, cells->level, n, V.stream))) return rc;
  if ((rc = features_impl(V, ctx, rule, cells, feat.as<uint16_t>()))) return rc;
  if ((rc = forward_impl(V, d_params, n, feat.as<uint16_t>(), cls.as<uint8_t>(), nullptr))) return rc;
  unsigned refine, coarsen;
  request_masks(rule, refine, coarsen);
  class_to_tag_kernel<<<grid_for(n, V.nsm, 256), 256, 0, V.stream>>>(
      cls.as<uint8_t>(), n, lvl.as<int32_t>(), refine, coarsen, tags.as<uint8_t>());
  CKI(cudaGetLastError());
  CKI(cudaMemcpyAsync(out, tags.p, (size_t)n, cudaMemcpyDeviceToHost, V.stream));
  CKI(cudaStreamSynchronize(V.stream));
  return IBGPU_OK;
}

int ibgpu_upload_signdis(ibgpu_ctx *ctx, const double *signdis) {
  CtxView V;
  if (ctx_view(ctx, &V) != IBGPU_OK) return IBGPU_E_ARG;
  if (!V.has_topology) return IBGPU_E_STATE;
  if (V.ncells == 0) return IBGPU_OK;
  if (!signdis) return IBGPU_E_ARG;
  double *dsd = nullptr;
  int rc = ctx_signdis_buffer(ctx, &dsd, true);
  if (rc) return rc;
  DevBuf rows;
  if ((rc = upload(rows, signdis, V.ncells, V.stream))) return rc;
  // slots that no row names (absent cells) are far from any wall
  std::vector<double> far((size_t)V.nslots, 1e30);
  CKI(cudaMemcpyAsync(dsd, far.data(), far.size() * sizeof(double), cudaMemcpyHostToDevice, V.stream));
  scatter_rows_f64<<<grid_for(V.ncells, V.nsm, 256), 256, 0, V.stream>>>(rows.as<double>(), V.cell_slot,
                                                                         V.ncells, dsd);
  CKI(cudaGetLastError());
  CKI(cudaStreamSynchronize(V.stream));
  return IBGPU_OK;
}

int ibgpu_tag_mesh(ibgpu_ctx *ctx, const ibgpu_tag_rule *rule, const float *d_params,
                   uint8_t *tags) {
  CtxView V;
  if (!rule || ctx_view(ctx, &V) != IBGPU_OK) return IBGPU_E_ARG;
  if (!V.has_topology || (d_params && !V.has_state)) return IBGPU_E_STATE;
  if (V.ncells == 0) return IBGPU_OK;
  if (!tags) return IBGPU_E_ARG;
  int rc;
  if (d_params && (rc = configure_smem())) return rc;
  uint8_t *rows = nullptr;
  if ((rc = tag_mesh_enqueue(ctx, rule, d_params, V.stream, &rows))) return rc;
  CKI(cudaMemcpyAsync(tags, rows, (size_t)V.ncells, cudaMemcpyDeviceToHost, V.stream));
  if (d_params) return kernel_error_check(V.aux_err, V.stream);
  CKI(cudaStreamSynchronize(V.stream));
  return IBGPU_OK;
}

}  // extern "C"
