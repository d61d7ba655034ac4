// aco_prior.cu -- learned heuristic prior for the candidate edges.
//
// The plain path weighs candidate c of node i by eta^beta = d(i,c)^-beta,
// entered as integer levels L (16 per octave) in the selection weights
// (k_weights).  The learned prior replaces those levels with
//     L_t = round(gamma * (s_max - s_t) * 16 / ln 2),   s = MLP(features),
// i.e. a weight proportional to exp(gamma * s), so the construction stays
// the same exact integer roulette; the plain levels remain the fallback.
//
//   features  k_prior_features: 8 values per candidate edge, computed in
//             FP32 and stored as BF16 ([row][32 slots][8], 16 bytes/edge)
//   MLP       8 -> 64 -> 64 -> 1, ReLU, BF16 operands, FP32 accumulation on
//             the tcgen05 tensor cores (k_prior_mlp): a 128-edge tile
//             (4 rows x 32 slots) per step; forward for inference, forward
//             + backward for training
//   loss      softmax cross-entropy over each row's valid slots against the
//             successor taken by an elite route
//   optimiser Adam (k_prior_adam)
//
// Layer 1 carries its bias as the weight of a constant-one input (input 8
// of the 16-wide K of the first MMA), so one GEMM
//     [dZ2^T ; dZ1^T] (128 x E) * [H1^T ; X^T]^T (E x 80)
// accumulated in tensor memory over a block's tiles yields dW2 (rows 0-63,
// columns 0-63), db2 (column 72), dW1 and db1 (rows 64-127, columns 64-72).
#include "aco_internal.cuh"
#include "aco_prior_internal.h"
#include "umma.cuh"

#include <cuda_bf16.h>

extern "C" {
#include "aco.h"
#include "aco_b200.h"
}

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <random>
#include <vector>

namespace acob200 {
namespace prior {

// Parameter vector (FP32): W1[64][8], b1[64], W2[64][64], b2[64], w3[64], b3.
constexpr int kW1 = 0, kB1 = 512, kW2 = 576, kB2 = 4672, kW3 = 4736, kB3 = 4800;
constexpr int kParams = 4801;
constexpr int kGradStride = 4808;  // partial-gradient row: kParams values, then the loss
static_assert(kParams == ACO_B200_PRIOR_PARAMS, "parameter count");

constexpr int kSlots = 32;      // candidate slots per row (k <= 32); a tile is 4 rows
constexpr uint32_t kPolls = 1u << 24;

// Shared-memory layout of k_prior_mlp (bytes, K-major operand tiles).
constexpr uint32_t kSB1 = 0;                         // W1|b1   64 x 16
constexpr uint32_t kSB2 = kSB1 + 64 * 16 * 2;         // W2      64 x 64 [o][j]
constexpr uint32_t kSB2T = kSB2 + 64 * 64 * 2;        // W2^T    64 x 64 [j][o]
constexpr uint32_t kSA1 = kSB2T + 64 * 64 * 2;        // X       128 x 16
constexpr uint32_t kSA2 = kSA1 + 128 * 16 * 2;        // H1, then dZ2  128 x 64
constexpr uint32_t kSAdw = kSA2 + 128 * 64 * 2;       // [dZ2^T; dZ1^T] 128 x 128
constexpr uint32_t kSBdw = kSAdw + 128 * 128 * 2;     // [H1^T; X^T]   80 x 128
constexpr uint32_t kSF32 = kSBdw + 80 * 128 * 2;      // b2[64], w3[64]
constexpr uint32_t kSRed = kSF32 + 128 * 4;           // 4 warps x 65 partial sums
constexpr uint32_t kSBar = kSRed + 4 * 65 * 4 + 48;    // mbarrier, TMEM base
constexpr uint32_t kSmemTrain = kSBar + 64;
constexpr uint32_t kSmemForward = kSmemTrain;         // same layout, training parts unused

// Tensor-memory columns: Z1 0-63, Z2 64-127, dW 128-207.  dH1 goes into
// Z2's columns: Z2 is read for the last time (the dZ2 epilogue) before the
// dH1 MMA is issued.  Training thus fits 256 columns, half of an SM's
// tensor memory, and two training blocks share an SM.
constexpr uint32_t kColZ1 = 0, kColZ2 = 64, kColDH1 = 64, kColDW = 128;

__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(kFull, v, o));
  return v;
}
__device__ __forceinline__ float warp_min(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(kFull, v, o));
  return v;
}
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

__device__ __forceinline__ void st_bf16(unsigned char *base, uint32_t off, float v) {
  *reinterpret_cast<__nv_bfloat16 *>(base + off) = __float2bfloat16_rn(v);
}

// --------------------------------------------------------------------------
// Instance-level helpers and features
// --------------------------------------------------------------------------

// Largest depot distance of the instance (feature scale).
__global__ void __launch_bounds__(256) k_depot_radius(const float2 *coords, int n, float *out) {
  __shared__ float s[8];
  const float2 p0 = coords[0];
  float r = 0.f;
  for (int j = 1 + threadIdx.x; j <= n; j += blockDim.x) {
    const float dx = coords[j].x - p0.x, dy = coords[j].y - p0.y;
    r = fmaxf(r, sqrtf(dx * dx + dy * dy));
  }
  r = warp_max(r);
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = r;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) r = fmaxf(r, s[w]);
    *out = r;
  }
}

// k-nearest candidate lists (k <= 32, empty slots 0), the same lists as the
// solver's (ties to the lower index).
__global__ void __launch_bounds__(256) k_prior_knn(const float2 *coords, int n, int k,
                                                   uint16_t *cand) {
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * (blockDim.x >> 5);
  for (int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i <= n; i += warps) {
    const unsigned long long key = warp_knn(coords, n, k, i, lane);
    if (lane < k) cand[(size_t)i * k + lane] = (uint16_t)((key == ~0ull) ? 0 : (key & 0xffffffffu));
  }
}

// Features of candidate slot t (lane) of row i, c = cand[i][t]:
//   0  d(i,c) / largest candidate distance of the row
//   1  nearest candidate distance of the row / d(i,c)
//   2  t / 31 (rank in the row)
//   3  d(c,0) / R      (R = largest depot distance of the instance)
//   4  d(i,0) / R
//   5  demand(c) / capacity
//   6  cos of the angle between c - i and 0 - i (0 for the depot row)
//   7  1 if i is among c's candidates, else 0
// Empty slots get zeros; kv[i] = number of non-empty slots (a prefix).
__global__ void __launch_bounds__(256) k_prior_features(const float2 *coords, const int *demand,
                                                        float inv_cap, int n, int k,
                                                        const uint16_t *cand, const float *radius,
                                                        uint4 *feat, uint8_t *kv) {
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * (blockDim.x >> 5);
  const float2 p0 = coords[0];
  const float inv_r = 1.0f / fmaxf(*radius, 1e-6f);
  for (int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i <= n; i += warps) {
    const float2 pi = coords[i];
    const int c = (lane < k) ? (int)cand[(size_t)i * k + lane] : 0;
    const bool valid = c > 0;
    const float2 pc = valid ? coords[c] : pi;
    const float dx = pc.x - pi.x, dy = pc.y - pi.y;
    const float d = sqrtf(dx * dx + dy * dy);
    const float dmin = warp_min(valid ? d : FLT_MAX);
    const float dmax = warp_max(valid ? d : 0.f);
    const float ax = p0.x - pi.x, ay = p0.y - pi.y;
    const float di0 = sqrtf(ax * ax + ay * ay);
    const float bx = p0.x - pc.x, by = p0.y - pc.y;
    const float dc0 = sqrtf(bx * bx + by * by);
    float f[8];
    f[0] = d / fmaxf(dmax, 1e-6f);
    f[1] = dmin / fmaxf(d, 1e-6f);
    f[2] = (float)lane * (1.0f / 31.0f);
    f[3] = dc0 * inv_r;
    f[4] = di0 * inv_r;
    f[5] = (float)(valid ? demand[c] : 0) * inv_cap;
    f[6] = (i == 0) ? 0.f : (dx * ax + dy * ay) / fmaxf(d * di0, 1e-6f);
    int mutual = 0;
    if (valid)
      for (int s = 0; s < k; ++s) mutual |= (cand[(size_t)c * k + s] == i) ? 1 : 0;
    f[7] = (float)mutual;
    uint4 out = make_uint4(0u, 0u, 0u, 0u);
    if (valid) {
      uint32_t w[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const uint32_t lo = __bfloat16_as_ushort(__float2bfloat16_rn(f[2 * q]));
        const uint32_t hi = __bfloat16_as_ushort(__float2bfloat16_rn(f[2 * q + 1]));
        w[q] = lo | (hi << 16);
      }
      out = make_uint4(w[0], w[1], w[2], w[3]);
    }
    feat[(size_t)i * kSlots + lane] = out;
    const unsigned vm = __ballot_sync(kFull, valid);
    if (lane == 0) kv[i] = (uint8_t)__popc(vm);
  }
}

// Slot of each elite successor in its row's candidate list (-1: absent).
__global__ void k_prior_slots(const int2 *pairs, long long count, const uint16_t *cand, int k,
                              int *slot) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= count) return;
  const int2 pr = pairs[p];
  int s = -1;
  for (int t = 0; t < k; ++t)
    if ((int)cand[(size_t)pr.x * k + t] == pr.y) {
      s = t;
      break;
    }
  slot[p] = s;
}

// --------------------------------------------------------------------------
// MLP on the tensor cores
// --------------------------------------------------------------------------

struct MlpArgs {
  const float *params;   // kParams FP32
  const uint4 *feat;     // [rows][32] edges, 8 BF16 each
  const uint8_t *kv;     // non-empty slots per row
  int tiles;
  // forward
  long long rows;
  float *scores;         // [rows][32]
  // training
  const int2 *examples;  // {feature row, target slot}
  const int *order;      // example ids of this minibatch
  int count;
  float inv_count;
  float *gpart;          // [grid][kGradStride] per-block partial gradients
  int *error;
};

template <bool TRAIN>
__global__ void __launch_bounds__(128, 2) k_prior_mlp(MlpArgs a) {
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char *sB1 = smem + kSB1, *sB2 = smem + kSB2, *sB2T = smem + kSB2T;
  unsigned char *sA1 = smem + kSA1, *sA2 = smem + kSA2, *sAdw = smem + kSAdw, *sBdw = smem + kSBdw;
  float *s_b2 = reinterpret_cast<float *>(smem + kSF32);
  float *s_w3 = s_b2 + 64;
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem + kSBar);
  uint32_t *s_tmem = reinterpret_cast<uint32_t *>(smem + kSBar + 8);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  constexpr uint32_t kCols = TRAIN ? 256u : 128u;

  if (warp == 0) {
    umma::tmem_alloc(s_tmem, kCols);
    umma::tmem_relinquish();
  }
  if (tid == 0) {
    mbar_init(bar, 1);
    fence_mbar_init();
  }
  // Weights into their operand layouts (BF16), biases of layers 2-3 in FP32.
  const float *P = a.params;
  for (int e = tid; e < 64 * 16; e += 128) {
    const int o = e >> 4, f = e & 15;
    const float w = f < 8 ? P[kW1 + o * 8 + f] : (f == 8 ? P[kB1 + o] : 0.f);
    st_bf16(sB1, umma::kmajor_offset(o, f, 64), w);
  }
  for (int e = tid; e < 64 * 64; e += 128) {
    const int o = e >> 6, j = e & 63;
    const float w = P[kW2 + e];
    st_bf16(sB2, umma::kmajor_offset(o, j, 64), w);
    if (TRAIN) st_bf16(sB2T, umma::kmajor_offset(j, o, 64), w);
  }
  if (tid < 64) {
    s_b2[tid] = P[kB2 + tid];
    s_w3[tid] = P[kW3 + tid];
  }
  const float b3 = P[kB3];
  // Constant input 8 = 1 (layer-1 bias), inputs 9-15 = 0, for every edge.
  *reinterpret_cast<uint4 *>(sA1 + umma::kmajor_offset(tid, 8, 128)) =
      make_uint4(0x3F80u, 0u, 0u, 0u);
  if (TRAIN) {
    for (int e = tid; e < 8 * 128; e += 128) {
      const int f = 8 + (e >> 7), col = e & 127;
      st_bf16(sBdw, umma::kmajor_offset(64 + f, col, 80), f == 8 ? 1.f : 0.f);
    }
  }
  umma::fence_async_smem();
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tm = *s_tmem;
  const uint32_t tl = tm + ((uint32_t)(warp * 32) << 16);  // this warp's lanes

  const uint32_t lbo128 = umma::kmajor_lbo(128), lbo64 = umma::kmajor_lbo(64),
                 lbo80 = umma::kmajor_lbo(80);
  const uint32_t idesc64 = umma::idesc_bf16_f32(128, 64);
  const uint32_t idesc80 = umma::idesc_bf16_f32(128, 80);
  const uint32_t aA1 = umma::smem_u32(sA1), aA2 = umma::smem_u32(sA2),
                 aAdw = umma::smem_u32(sAdw), aBdw = umma::smem_u32(sBdw),
                 aB1 = umma::smem_u32(sB1), aB2 = umma::smem_u32(sB2),
                 aB2T = umma::smem_u32(sB2T);

  float acc_w3[64];
#pragma unroll
  for (int j = 0; j < 64; ++j) acc_w3[j] = 0.f;
  float acc_loss = 0.f;
  uint32_t phase = 0;
  bool ok = true;
  int done = 0;

  for (int tile = blockIdx.x; tile < a.tiles; tile += gridDim.x) {
    long long row;
    int tgt = -1;
    bool live;
    if (TRAIN) {
      const int ex = tile * 4 + warp;
      live = ex < a.count;
      const int2 e2 = live ? a.examples[a.order[ex]] : make_int2(0, -1);
      row = e2.x;
      tgt = e2.y;
    } else {
      row = (long long)tile * 4 + warp;
      live = row < a.rows;
    }
    const int kvr = live ? (int)a.kv[row] : 0;
    const bool valid = live && lane < kvr;
    const uint4 fv = valid ? a.feat[row * kSlots + lane] : make_uint4(0u, 0u, 0u, 0u);
    *reinterpret_cast<uint4 *>(sA1 + umma::kmajor_offset(tid, 0, 128)) = fv;
    if (TRAIN) {
      const __nv_bfloat16 *fb = reinterpret_cast<const __nv_bfloat16 *>(&fv);
#pragma unroll
      for (int f = 0; f < 8; ++f)
        *reinterpret_cast<__nv_bfloat16 *>(sBdw + umma::kmajor_offset(64 + f, tid, 80)) = fb[f];
    }
    umma::fence_async_smem();
    umma::fence_before_sync();
    __syncthreads();
    // Z1 = X W1^T (+ b1 through the constant input)
    if (tid == 0) {
      umma::fence_after_sync();
      umma::mma_bf16(tm + kColZ1, umma::smem_desc(aA1, lbo128, 128),
                     umma::smem_desc(aB1, lbo64, 128), idesc64, 0u);
      umma::commit(bar);
    }
    ok = __syncthreads_and(mbar_wait_bounded(bar, phase, kPolls));
    phase ^= 1u;
    if (!ok) break;
    umma::fence_after_sync();
    // H1 = relu(Z1) -> BF16 operand (and its transpose for dW2)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      float z[16];
      umma::tmem_ld16(tl + kColZ1 + 16 * q, z);
      umma::tmem_wait_ld();
      uint32_t w[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const __nv_bfloat16 lo = __float2bfloat16_rn(fmaxf(z[2 * i], 0.f));
        const __nv_bfloat16 hi = __float2bfloat16_rn(fmaxf(z[2 * i + 1], 0.f));
        w[i] = (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
        if (TRAIN) {
          *reinterpret_cast<__nv_bfloat16 *>(sBdw + umma::kmajor_offset(16 * q + 2 * i, tid, 80)) = lo;
          *reinterpret_cast<__nv_bfloat16 *>(sBdw + umma::kmajor_offset(16 * q + 2 * i + 1, tid, 80)) = hi;
        }
      }
      *reinterpret_cast<uint4 *>(sA2 + umma::kmajor_offset(tid, 16 * q, 128)) =
          make_uint4(w[0], w[1], w[2], w[3]);
      *reinterpret_cast<uint4 *>(sA2 + umma::kmajor_offset(tid, 16 * q + 8, 128)) =
          make_uint4(w[4], w[5], w[6], w[7]);
    }
    umma::fence_async_smem();
    umma::fence_before_sync();
    __syncthreads();
    // Z2 = H1 W2^T
    if (tid == 0) {
      umma::fence_after_sync();
#pragma unroll
      for (int s = 0; s < 4; ++s)
        umma::mma_bf16(tm + kColZ2, umma::smem_desc(aA2 + 2 * s * lbo128, lbo128, 128),
                       umma::smem_desc(aB2 + 2 * s * lbo64, lbo64, 128), idesc64, s > 0 ? 1u : 0u);
      umma::commit(bar);
    }
    ok = __syncthreads_and(mbar_wait_bounded(bar, phase, kPolls));
    phase ^= 1u;
    if (!ok) break;
    umma::fence_after_sync();
    // s = b3 + w3 . relu(Z2 + b2)
    float sc = b3;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      float z[16];
      umma::tmem_ld16(tl + kColZ2 + 16 * q, z);
      umma::tmem_wait_ld();
#pragma unroll
      for (int i = 0; i < 16; ++i) sc += s_w3[16 * q + i] * fmaxf(z[i] + s_b2[16 * q + i], 0.f);
    }
    if (!TRAIN) {
      if (live) a.scores[row * kSlots + lane] = sc;
    } else {
      // Softmax cross-entropy over the row's non-empty slots (one warp).
      const float mx = warp_max(valid ? sc : -FLT_MAX);
      const float ex = valid ? expf(sc - mx) : 0.f;
      const float sum = warp_sum(ex);
      float g = 0.f;
      if (valid && tgt >= 0) {
        g = (ex / sum - (lane == tgt ? 1.f : 0.f)) * a.inv_count;
        if (lane == tgt) acc_loss += (mx + logf(sum) - sc) * a.inv_count;
      }
      // dZ2 = g w3 relu'(Z2 + b2): operand of dH1 (rows = edges) and of dW2
      // (rows = units).
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        float z[16];
        umma::tmem_ld16(tl + kColZ2 + 16 * q, z);
        umma::tmem_wait_ld();
        uint32_t w[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          float d2[2];
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int j = 16 * q + 2 * i + h;
            const float h2 = z[2 * i + h] + s_b2[j];
            acc_w3[j] += g * fmaxf(h2, 0.f);
            d2[h] = h2 > 0.f ? g * s_w3[j] : 0.f;
          }
          const __nv_bfloat16 lo = __float2bfloat16_rn(d2[0]);
          const __nv_bfloat16 hi = __float2bfloat16_rn(d2[1]);
          w[i] = (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
          *reinterpret_cast<__nv_bfloat16 *>(sAdw + umma::kmajor_offset(16 * q + 2 * i, tid, 128)) = lo;
          *reinterpret_cast<__nv_bfloat16 *>(sAdw + umma::kmajor_offset(16 * q + 2 * i + 1, tid, 128)) = hi;
        }
        *reinterpret_cast<uint4 *>(sA2 + umma::kmajor_offset(tid, 16 * q, 128)) =
            make_uint4(w[0], w[1], w[2], w[3]);
        *reinterpret_cast<uint4 *>(sA2 + umma::kmajor_offset(tid, 16 * q + 8, 128)) =
            make_uint4(w[4], w[5], w[6], w[7]);
      }
      umma::fence_async_smem();
      umma::fence_before_sync();
      __syncthreads();
      // dH1 = dZ2 W2
      if (tid == 0) {
        umma::fence_after_sync();
#pragma unroll
        for (int s = 0; s < 4; ++s)
          umma::mma_bf16(tm + kColDH1, umma::smem_desc(aA2 + 2 * s * lbo128, lbo128, 128),
                         umma::smem_desc(aB2T + 2 * s * lbo64, lbo64, 128), idesc64,
                         s > 0 ? 1u : 0u);
        umma::commit(bar);
      }
      ok = __syncthreads_and(mbar_wait_bounded(bar, phase, kPolls));
      phase ^= 1u;
      if (!ok) break;
      umma::fence_after_sync();
      // dZ1 = dH1 relu'(Z1) into rows 64-127 of the weight-gradient operand
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        float dh[16], z[16];
        umma::tmem_ld16(tl + kColDH1 + 16 * q, dh);
        umma::tmem_ld16(tl + kColZ1 + 16 * q, z);
        umma::tmem_wait_ld();
#pragma unroll
        for (int i = 0; i < 16; ++i)
          st_bf16(sAdw, umma::kmajor_offset(64 + 16 * q + i, tid, 128), z[i] > 0.f ? dh[i] : 0.f);
      }
      umma::fence_async_smem();
      umma::fence_before_sync();
      __syncthreads();
      // dW += [dZ2^T; dZ1^T] [H1^T; X^T]^T, accumulated over this block's tiles
      if (tid == 0) {
        umma::fence_after_sync();
#pragma unroll
        for (int s = 0; s < 8; ++s)
          umma::mma_bf16(tm + kColDW, umma::smem_desc(aAdw + 2 * s * lbo128, lbo128, 128),
                         umma::smem_desc(aBdw + 2 * s * lbo80, lbo80, 128), idesc80,
                         (done > 0 || s > 0) ? 1u : 0u);
        umma::commit(bar);
      }
      ok = __syncthreads_and(mbar_wait_bounded(bar, phase, kPolls));
      phase ^= 1u;
      if (!ok) break;
      umma::fence_after_sync();
    }
    ++done;
    umma::fence_before_sync();
    __syncthreads();
  }

  if (!ok) {
    // A wait gave up: wait (bounded) for the group still in flight before
    // the tensor memory is released.
    mbar_wait_bounded(bar, phase ^ 1u, kPolls);
    if (tid == 0) atomicOr(a.error, kErrStageTimeout);
  } else if (TRAIN && done > 0) {
    // This block's partial gradient, row blockIdx.x of gpart (summed in a
    // fixed order by k_prior_reduce: training is bit-reproducible).
    float *out = a.gpart + (size_t)blockIdx.x * kGradStride;
    // W2, b2 (rows 0-63) and W1, b1 (rows 64-127) from tensor memory.
#pragma unroll
    for (int q = 0; q < 5; ++q) {
      float d[16];
      umma::tmem_ld16(tl + kColDW + 16 * q, d);
      umma::tmem_wait_ld();
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const int col = 16 * q + i;
        if (warp < 2) {
          if (col < 64) out[kW2 + tid * 64 + col] = d[i];
          else if (col == 72) out[kB2 + tid] = d[i];
        } else {
          const int j = tid - 64;
          if (col >= 64 && col < 72) out[kW1 + j * 8 + (col - 64)] = d[i];
          else if (col == 72) out[kB1 + j] = d[i];
        }
      }
    }
    // w3 and the loss: warp sums, then the four warps in order.
    float *s_red = reinterpret_cast<float *>(smem + kSRed);
#pragma unroll
    for (int j = 0; j < 64; ++j) {
      const float v = warp_sum(acc_w3[j]);
      if (lane == 0) s_red[warp * 65 + j] = v;
    }
    const float vl = warp_sum(acc_loss);
    if (lane == 0) s_red[warp * 65 + 64] = vl;
    __syncthreads();
    if (tid < 65) {
      const float v = s_red[tid] + s_red[65 + tid] + s_red[130 + tid] + s_red[195 + tid];
      if (tid < 64) out[kW3 + tid] = v;
      else out[kParams] = v;  // loss
    }
    // b3 is not trained: a constant added to every score of a row changes
    // neither the softmax nor the levels, and its gradient is identically 0.
    if (tid == 0) out[kB3] = 0.f;
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tm, kCols);
}

// Sum of the blocks' partial gradients in block order; the loss goes to
// *loss (accumulated over a training epoch).
__global__ void k_prior_reduce(const float *gpart, int blocks, float *grad, float *loss) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i > kParams) return;
  float v = 0.f;
  for (int r = 0; r < blocks; ++r) v += gpart[(size_t)r * kGradStride + i];
  if (i < kParams) grad[i] = v;
  else *loss += v;
}

__global__ void k_prior_adam(float *params, float *m, float *v, float *grad, int count, float lr,
                             float bc1, float bc2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const float g = grad[i];
  const float mi = 0.9f * m[i] + 0.1f * g;
  const float vi = 0.999f * v[i] + 0.001f * g * g;
  m[i] = mi;
  v[i] = vi;
  params[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + 1e-8f);
}

// Levels from scores: warp per row, L = min(4095, round(scale (s_max - s))).
// residual: the learned level is added to the plain level already in lvl
// (weights proportional to eta^beta exp(gamma s)).
__global__ void k_prior_levels(const float *scores, const uint8_t *kv, int rows, int k,
                               float scale, int residual, uint16_t *lvl) {
  const int lane = threadIdx.x & 31;
  const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (row >= rows) return;
  const bool valid = lane < (int)kv[row];
  const float s = scores[(size_t)row * kSlots + lane];
  const float mx = warp_max(valid ? s : -FLT_MAX);
  if (lane < k) {
    int L = kThresholds;
    if (valid) {
      L = (int)fminf((float)kThresholds, rintf(scale * (mx - s)));
      if (residual) L = min(kThresholds, L + (int)lvl[(size_t)row * k + lane]);
    }
    lvl[(size_t)row * k + lane] = (uint16_t)L;
  }
}

// --------------------------------------------------------------------------
// Host side
// --------------------------------------------------------------------------

bool configure_mlp() {
  static int state = 0;  // 0 unknown, 1 ok, -1 failed
  if (state == 0) {
    cudaError_t e1 = cudaFuncSetAttribute(k_prior_mlp<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)kSmemTrain);
    cudaError_t e2 = cudaFuncSetAttribute(k_prior_mlp<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)kSmemForward);
    state = (e1 == cudaSuccess && e2 == cudaSuccess) ? 1 : -1;
  }
  return state == 1;
}

}  // namespace prior
}  // namespace acob200

using namespace acob200;
using namespace acob200::prior;

struct aco_b200_prior {
  int device = 0;
  int num_sms = 148;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  float *d_params = nullptr, *d_m = nullptr, *d_v = nullptr, *d_grad = nullptr, *d_loss = nullptr;
  float *d_gpart = nullptr;  // [2 num_sms][kGradStride] partial gradients
  int *d_error = nullptr;
  int adam_step = 0;
  // training set
  long long rows = 0;
  uint4 *d_feat = nullptr;
  uint8_t *d_kv = nullptr;
  int2 *d_examples = nullptr;
  long long n_examples = 0;
  int *d_order = nullptr;
  // scratch of apply (one instance)
  long long s_rows = 0;
  uint4 *d_sfeat = nullptr;
  uint8_t *d_skv = nullptr;
  float *d_sscores = nullptr;
  float *d_radius = nullptr;

  void free_dataset() {
    cudaFree(d_feat);
    cudaFree(d_kv);
    cudaFree(d_examples);
    cudaFree(d_order);
    d_feat = nullptr;
    d_kv = nullptr;
    d_examples = nullptr;
    d_order = nullptr;
    rows = n_examples = 0;
  }
  void free_scratch() {
    cudaFree(d_sfeat);
    cudaFree(d_skv);
    cudaFree(d_sscores);
    d_sfeat = nullptr;
    d_skv = nullptr;
    d_sscores = nullptr;
    s_rows = 0;
  }
  ~aco_b200_prior() {
    cudaSetDevice(device);
    free_dataset();
    free_scratch();
    void *p[] = {d_params, d_m, d_v, d_grad, d_loss, d_error, d_radius, d_gpart};
    for (void *q : p)
      if (q) cudaFree(q);
    if (own_stream && stream) cudaStreamDestroy(stream);
  }
};

#define PTRY(call)                                                           \
  do {                                                                       \
    cudaError_t err__ = (call);                                              \
    if (err__ != cudaSuccess) {                                              \
      fprintf(stderr, "aco_b200 prior: CUDA error %s at %s:%d\n",            \
              cudaGetErrorString(err__), __FILE__, __LINE__);                \
      return err__ == cudaErrorMemoryAllocation ? ACO_ERR_ALLOCATION         \
                                                : ACO_ERR_BACKEND;           \
    }                                                                        \
  } while (0)

namespace acob200 {
namespace prior {

static int ensure_scratch(aco_b200_prior *p, long long rows) {
  if (rows <= p->s_rows) return ACO_OK;
  p->free_scratch();
  PTRY(cudaMalloc(&p->d_sfeat, (size_t)rows * kSlots * sizeof(uint4)));
  PTRY(cudaMalloc(&p->d_skv, (size_t)rows));
  PTRY(cudaMalloc(&p->d_sscores, (size_t)rows * kSlots * sizeof(float)));
  p->s_rows = rows;
  return ACO_OK;
}

static int launch_forward(aco_b200_prior *p, const uint4 *feat, const uint8_t *kv, long long rows,
                          float *scores, cudaStream_t s) {
  if (!configure_mlp()) return ACO_ERR_BACKEND;
  MlpArgs a = {};
  a.params = p->d_params;
  a.feat = feat;
  a.kv = kv;
  a.rows = rows;
  a.scores = scores;
  a.tiles = (int)((rows + 3) / 4);
  a.error = p->d_error;
  const int grid = std::max(1, std::min(a.tiles, p->num_sms * 2));
  k_prior_mlp<false><<<grid, 128, kSmemForward, s>>>(a);
  PTRY(cudaGetLastError());
  return ACO_OK;
}

static int launch_features(aco_b200_prior *p, const float2 *coords, const int *demand,
                           long long cap, int n, int k, const uint16_t *cand, uint4 *feat,
                           uint8_t *kv, cudaStream_t s) {
  k_depot_radius<<<1, 256, 0, s>>>(coords, n, p->d_radius);
  PTRY(cudaGetLastError());
  const int rows = n + 1;
  int blocks = (rows + 7) / 8;
  if (blocks > p->num_sms * 8) blocks = p->num_sms * 8;
  k_prior_features<<<blocks, 256, 0, s>>>(coords, demand, 1.0f / (float)cap, n, k, cand,
                                          p->d_radius, feat, kv);
  PTRY(cudaGetLastError());
  return ACO_OK;
}

int learned_levels(aco_b200_prior *p, const float2 *coords, const int *demand, long long cap,
                   int n, int k, const uint16_t *cand, uint16_t *lvl, float gamma,
                   int residual, cudaStream_t s) {
  if (!p || k < 1 || k > kSlots || n < 1) return ACO_ERR_INVALID_INPUT;
  const long long rows = (long long)n + 1;
  int rc = ensure_scratch(p, rows);
  if (rc) return rc;
  rc = launch_features(p, coords, demand, cap, n, k, cand, p->d_sfeat, p->d_skv, s);
  if (rc) return rc;
  rc = launch_forward(p, p->d_sfeat, p->d_skv, rows, p->d_sscores, s);
  if (rc) return rc;
  const float scale = gamma * (float)kLevelsPerOctave / logf(2.0f);
  k_prior_levels<<<(unsigned)((rows + 7) / 8), 256, 0, s>>>(p->d_sscores, p->d_skv, (int)rows, k,
                                                           scale, residual, lvl);
  PTRY(cudaGetLastError());
  return ACO_OK;
}

}  // namespace prior
}  // namespace acob200

extern "C" {

int aco_b200_prior_create(aco_b200_prior **out, int device) {
  if (!out) return ACO_ERR_INVALID_INPUT;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
    fprintf(stderr, "aco_b200 prior: no CUDA device %d\n", device);
    return ACO_ERR_BACKEND;
  }
  aco_b200_prior *p = new aco_b200_prior();
  p->device = device;
  cudaSetDevice(device);
  cudaDeviceGetAttribute(&p->num_sms, cudaDevAttrMultiProcessorCount, device);
  if (cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete p;
    return ACO_ERR_BACKEND;
  }
  p->own_stream = true;
  const size_t pb = (kParams + 3) / 4 * 16;
  if (cudaMalloc(&p->d_params, pb) != cudaSuccess || cudaMalloc(&p->d_m, pb) != cudaSuccess ||
      cudaMalloc(&p->d_v, pb) != cudaSuccess || cudaMalloc(&p->d_grad, pb) != cudaSuccess ||
      cudaMalloc(&p->d_loss, 16) != cudaSuccess || cudaMalloc(&p->d_error, 16) != cudaSuccess ||
      cudaMalloc(&p->d_radius, 16) != cudaSuccess ||
      cudaMalloc(&p->d_gpart, (size_t)2 * p->num_sms * kGradStride * sizeof(float)) !=
          cudaSuccess) {
    delete p;
    return ACO_ERR_ALLOCATION;
  }
  cudaMemset(p->d_params, 0, pb);
  cudaMemset(p->d_m, 0, pb);
  cudaMemset(p->d_v, 0, pb);
  cudaMemset(p->d_grad, 0, pb);
  cudaMemset(p->d_loss, 0, 16);
  cudaMemset(p->d_error, 0, 16);
  if (!configure_mlp()) {
    fprintf(stderr, "aco_b200 prior: cannot configure the MLP kernels\n");
    delete p;
    return ACO_ERR_BACKEND;
  }
  *out = p;
  return ACO_OK;
}

int aco_b200_prior_destroy(aco_b200_prior *p) {
  delete p;
  return ACO_OK;
}

int aco_b200_prior_set_stream(aco_b200_prior *p, void *stream) {
  if (!p) return ACO_ERR_INVALID_INPUT;
  cudaSetDevice(p->device);
  if (p->own_stream && p->stream) cudaStreamDestroy(p->stream);
  p->own_stream = false;
  p->stream = (cudaStream_t)stream;
  if (!p->stream) {
    if (cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking) != cudaSuccess)
      return ACO_ERR_BACKEND;
    p->own_stream = true;
  }
  return ACO_OK;
}

int aco_b200_prior_init(aco_b200_prior *p, unsigned int seed) {
  if (!p) return ACO_ERR_INVALID_INPUT;
  // He-normal weights, zero biases (std::mt19937 + Box-Muller, so the
  // values are the same on every platform).
  std::mt19937 rng(seed);
  auto normal = [&rng]() {
    const double u1 = (rng() + 1.0) / 4294967297.0, u2 = (rng() + 1.0) / 4294967297.0;
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
  };
  std::vector<float> h(kParams, 0.f);
  for (int i = 0; i < 512; ++i) h[kW1 + i] = (float)(normal() * std::sqrt(2.0 / 8.0));
  for (int i = 0; i < 4096; ++i) h[kW2 + i] = (float)(normal() * std::sqrt(2.0 / 64.0));
  for (int i = 0; i < 64; ++i) h[kW3 + i] = (float)(normal() * std::sqrt(1.0 / 64.0));
  return aco_b200_prior_set_params(p, h.data(), kParams);
}

int aco_b200_prior_set_params(aco_b200_prior *p, const float *params, int count) {
  if (!p || !params || count != kParams) return ACO_ERR_INVALID_INPUT;
  cudaSetDevice(p->device);
  const size_t pb = (size_t)kParams * sizeof(float);
  PTRY(cudaMemcpy(p->d_params, params, pb, cudaMemcpyHostToDevice));
  PTRY(cudaMemset(p->d_m, 0, pb));
  PTRY(cudaMemset(p->d_v, 0, pb));
  PTRY(cudaMemset(p->d_grad, 0, pb));
  p->adam_step = 0;
  return ACO_OK;
}

int aco_b200_prior_get_params(aco_b200_prior *p, float *params, int count) {
  if (!p || !params || count != kParams) return ACO_ERR_INVALID_INPUT;
  cudaSetDevice(p->device);
  PTRY(cudaStreamSynchronize(p->stream));
  PTRY(cudaMemcpy(params, p->d_params, (size_t)kParams * sizeof(float), cudaMemcpyDeviceToHost));
  return ACO_OK;
}

int aco_b200_prior_load(aco_b200_prior *p, const char *path) {
  if (!p || !path) return ACO_ERR_INVALID_INPUT;
  FILE *f = fopen(path, "rb");
  if (!f) return ACO_ERR_INVALID_INPUT;
  std::vector<float> h(kParams);
  const size_t got = fread(h.data(), sizeof(float), kParams, f);
  const bool extra = fgetc(f) != EOF;
  fclose(f);
  if (got != (size_t)kParams || extra) return ACO_ERR_INVALID_INPUT;
  return aco_b200_prior_set_params(p, h.data(), kParams);
}

int aco_b200_prior_save(aco_b200_prior *p, const char *path) {
  if (!p || !path) return ACO_ERR_INVALID_INPUT;
  std::vector<float> h(kParams);
  int rc = aco_b200_prior_get_params(p, h.data(), kParams);
  if (rc) return rc;
  FILE *f = fopen(path, "wb");
  if (!f) return ACO_ERR_INVALID_INPUT;
  const size_t put = fwrite(h.data(), sizeof(float), kParams, f);
  fclose(f);
  return put == (size_t)kParams ? ACO_OK : ACO_ERR_BACKEND;
}

int aco_b200_prior_set_dataset(aco_b200_prior *p, const aco_b200_prior_dataset *d,
                               long long *n_examples) {
  if (!p || !d || d->count < 1 || !d->n || !d->K || !d->capacity || !d->x || !d->y || !d->nodes ||
      !d->lens)
    return ACO_ERR_INVALID_INPUT;
  const int k = d->cand_k > 0 ? d->cand_k : kSlots;
  if (k > kSlots) return ACO_ERR_INVALID_INPUT;
  cudaSetDevice(p->device);
  cudaStream_t s = p->stream;
  // Offsets and validation.
  std::vector<long long> node_off(d->count + 1, 0), route_off(d->count + 1, 0),
      len_off(d->count + 1, 0);
  for (int i = 0; i < d->count; ++i) {
    const int n = d->n[i], K = d->K[i];
    if (n < 2 || n > 65534 || K < 1 || d->capacity[i] < 1) return ACO_ERR_INVALID_INPUT;
    node_off[i + 1] = node_off[i] + n + 1;
    len_off[i + 1] = len_off[i] + K;
    long long tot = 0;
    for (int v = 0; v < K; ++v) {
      const int L = d->lens[len_off[i] + v];
      if (L < 2) return ACO_ERR_INVALID_INPUT;
      tot += L;
    }
    route_off[i + 1] = route_off[i] + tot;
  }
  const long long rows = node_off[d->count];
  // Elite successor pairs (row, successor): depot -> first customer, and
  // both directions of every customer-customer arc.
  std::vector<int2> pairs;
  for (int i = 0; i < d->count; ++i) {
    const int n = d->n[i];
    long long off = route_off[i];
    for (int v = 0; v < d->K[i]; ++v) {
      const int L = d->lens[len_off[i] + v];
      const int *r = d->nodes + off;
      if (r[0] != 0 || r[L - 1] != 0) return ACO_ERR_INVALID_INPUT;
      for (int t = 1; t + 1 < L; ++t)
        if (r[t] < 1 || r[t] > n) return ACO_ERR_INVALID_INPUT;
      if (L > 2) pairs.push_back(make_int2((int)(node_off[i] + 0), r[1]));
      for (int t = 1; t + 2 < L; ++t) {
        pairs.push_back(make_int2((int)(node_off[i] + r[t]), r[t + 1]));
        pairs.push_back(make_int2((int)(node_off[i] + r[t + 1]), r[t]));
      }
      off += L;
    }
  }
  if (rows > 0x7fffffffLL) return ACO_ERR_INVALID_INPUT;
  p->free_dataset();
  // Per-instance device work: coordinates, candidate lists, features.
  float2 *d_xy = nullptr;
  int *d_dem = nullptr;
  uint16_t *d_cand = nullptr;
  int2 *d_pairs = nullptr;
  int *d_slot = nullptr;
  int rc = ACO_OK;
  auto fail = [&](int code) {
    cudaFree(d_xy);
    cudaFree(d_dem);
    cudaFree(d_cand);
    cudaFree(d_pairs);
    cudaFree(d_slot);
    return code;
  };
  std::vector<float2> xy(rows);
  std::vector<int> dem(rows);
  for (int i = 0; i < d->count; ++i)
    for (long long j = node_off[i]; j < node_off[i + 1]; ++j) {
      xy[j] = make_float2(d->x[j], d->y[j]);
      dem[j] = d->demand ? d->demand[j] : (j == node_off[i] ? 0 : 1);
    }
  if (cudaMalloc(&d_xy, rows * sizeof(float2)) != cudaSuccess ||
      cudaMalloc(&d_dem, rows * sizeof(int)) != cudaSuccess ||
      cudaMalloc(&d_cand, rows * k * sizeof(uint16_t)) != cudaSuccess ||
      cudaMalloc(&p->d_feat, rows * kSlots * sizeof(uint4)) != cudaSuccess ||
      cudaMalloc(&p->d_kv, rows) != cudaSuccess)
    return fail(ACO_ERR_ALLOCATION);
  if (cudaMemcpyAsync(d_xy, xy.data(), rows * sizeof(float2), cudaMemcpyHostToDevice, s) ||
      cudaMemcpyAsync(d_dem, dem.data(), rows * sizeof(int), cudaMemcpyHostToDevice, s))
    return fail(ACO_ERR_BACKEND);
  for (int i = 0; i < d->count && rc == ACO_OK; ++i) {
    const int n = d->n[i];
    const int ki = std::min(k, n);
    // Candidate lists of length k (the instance's own list is shorter
    // only when n < k; empty slots stay 0).
    if (ki < k) cudaMemsetAsync(d_cand + node_off[i] * k, 0, (size_t)(n + 1) * k * sizeof(uint16_t), s);
    int blocks = std::min((n + 1 + 7) / 8, p->num_sms * 16);
    k_prior_knn<<<blocks, 256, 0, s>>>(d_xy + node_off[i], n, k, d_cand + node_off[i] * k);
    if (cudaGetLastError() != cudaSuccess) rc = ACO_ERR_BACKEND;
    if (rc == ACO_OK)
      rc = launch_features(p, d_xy + node_off[i], d_dem + node_off[i], d->capacity[i], n, k,
                           d_cand + node_off[i] * k, p->d_feat + node_off[i] * kSlots,
                           p->d_kv + node_off[i], s);
  }
  if (rc) return fail(rc);
  // Slots of the successors; pairs whose successor is not a candidate drop.
  const long long np = (long long)pairs.size();
  std::vector<int> slot(np);
  if (np > 0) {
    if (cudaMalloc(&d_pairs, np * sizeof(int2)) != cudaSuccess ||
        cudaMalloc(&d_slot, np * sizeof(int)) != cudaSuccess)
      return fail(ACO_ERR_ALLOCATION);
    if (cudaMemcpyAsync(d_pairs, pairs.data(), np * sizeof(int2), cudaMemcpyHostToDevice, s))
      return fail(ACO_ERR_BACKEND);
    k_prior_slots<<<(unsigned)((np + 255) / 256), 256, 0, s>>>(d_pairs, np, d_cand, k, d_slot);
    if (cudaGetLastError() != cudaSuccess ||
        cudaMemcpyAsync(slot.data(), d_slot, np * sizeof(int), cudaMemcpyDeviceToHost, s) ||
        cudaStreamSynchronize(s))
      return fail(ACO_ERR_BACKEND);
  } else if (cudaStreamSynchronize(s)) {
    return fail(ACO_ERR_BACKEND);
  }
  std::vector<int2> ex;
  ex.reserve(np);
  for (long long q = 0; q < np; ++q)
    if (slot[q] >= 0) ex.push_back(make_int2(pairs[q].x, slot[q]));
  fail(ACO_OK);  // frees the temporaries
  p->rows = rows;
  p->n_examples = (long long)ex.size();
  if (p->n_examples > 0) {
    PTRY(cudaMalloc(&p->d_examples, ex.size() * sizeof(int2)));
    PTRY(cudaMalloc(&p->d_order, ex.size() * sizeof(int)));
    PTRY(cudaMemcpy(p->d_examples, ex.data(), ex.size() * sizeof(int2), cudaMemcpyHostToDevice));
  }
  if (n_examples) *n_examples = p->n_examples;
  return ACO_OK;
}

// Gradient of the mean loss over `count` examples listed at order: the
// tensor-core kernel writes one partial row per block, k_prior_reduce sums
// them into d_grad in block order and adds the loss to *d_loss.
static int run_gradient(aco_b200_prior *p, const int *order, int count, cudaStream_t s) {
  MlpArgs a = {};
  a.params = p->d_params;
  a.feat = p->d_feat;
  a.kv = p->d_kv;
  a.examples = p->d_examples;
  a.order = order;
  a.count = count;
  a.inv_count = 1.0f / (float)count;
  a.gpart = p->d_gpart;
  a.error = p->d_error;
  a.tiles = (count + 3) / 4;
  // Two training blocks per SM (256 tensor-memory columns and 94 KB of shared
  // memory each): one block's MMA runs while the other's epilogue does.
  const int grid = std::max(1, std::min(a.tiles, p->num_sms * 2));
  k_prior_mlp<true><<<grid, 128, kSmemTrain, s>>>(a);
  PTRY(cudaGetLastError());
  k_prior_reduce<<<(kParams + 1 + 255) / 256, 256, 0, s>>>(p->d_gpart, grid, p->d_grad, p->d_loss);
  PTRY(cudaGetLastError());
  return ACO_OK;
}

static int check_error(aco_b200_prior *p) {
  int err = 0;
  PTRY(cudaMemcpy(&err, p->d_error, sizeof(int), cudaMemcpyDeviceToHost));
  if (err) {
    fprintf(stderr, "aco_b200 prior: device error flag 0x%x\n", err);
    return ACO_ERR_BACKEND;
  }
  return ACO_OK;
}

int aco_b200_prior_gradient(aco_b200_prior *p, const int *examples, int count, float *grad,
                            float *loss) {
  if (!p || !examples || count < 1 || !grad || p->n_examples < 1) return ACO_ERR_INVALID_INPUT;
  for (int i = 0; i < count; ++i)
    if (examples[i] < 0 || examples[i] >= p->n_examples) return ACO_ERR_INVALID_INPUT;
  if (count > p->n_examples) return ACO_ERR_INVALID_INPUT;
  cudaSetDevice(p->device);
  cudaStream_t s = p->stream;
  PTRY(cudaMemcpyAsync(p->d_order, examples, count * sizeof(int), cudaMemcpyHostToDevice, s));
  PTRY(cudaMemsetAsync(p->d_loss, 0, sizeof(float), s));
  int rc = run_gradient(p, p->d_order, count, s);
  if (rc) return rc;
  PTRY(cudaStreamSynchronize(s));
  rc = check_error(p);
  if (rc) return rc;
  PTRY(cudaMemcpy(grad, p->d_grad, kParams * sizeof(float), cudaMemcpyDeviceToHost));
  if (loss) PTRY(cudaMemcpy(loss, p->d_loss, sizeof(float), cudaMemcpyDeviceToHost));
  return ACO_OK;
}

int aco_b200_prior_train(aco_b200_prior *p, int epochs, int batch, float lr, unsigned int seed,
                         float *epoch_loss) {
  if (!p || epochs < 0 || batch < 4 || !(lr >= 0.f) || p->n_examples < 1)
    return ACO_ERR_INVALID_INPUT;
  cudaSetDevice(p->device);
  cudaStream_t s = p->stream;
  const long long N = p->n_examples;
  std::vector<int> order(N);
  std::mt19937 rng(seed);
  for (int e = 0; e < epochs; ++e) {
    for (long long i = 0; i < N; ++i) order[i] = (int)i;
    for (long long i = N - 1; i > 0; --i) {
      const long long j = (long long)(rng() % (unsigned long long)(i + 1));
      std::swap(order[i], order[j]);
    }
    PTRY(cudaMemcpyAsync(p->d_order, order.data(), N * sizeof(int), cudaMemcpyHostToDevice, s));
    PTRY(cudaMemsetAsync(p->d_loss, 0, sizeof(float), s));
    int steps = 0;
    for (long long b0 = 0; b0 < N; b0 += batch, ++steps) {
      const int cnt = (int)std::min<long long>(batch, N - b0);
      int rc = run_gradient(p, p->d_order + b0, cnt, s);
      if (rc) return rc;
      p->adam_step += 1;
      const float bc1 = 1.0f - powf(0.9f, (float)p->adam_step);
      const float bc2 = 1.0f - powf(0.999f, (float)p->adam_step);
      k_prior_adam<<<(kParams + 255) / 256, 256, 0, s>>>(p->d_params, p->d_m, p->d_v, p->d_grad,
                                                         kParams, lr, bc1, bc2);
      PTRY(cudaGetLastError());
    }
    float l = 0.f;
    PTRY(cudaMemcpyAsync(&l, p->d_loss, sizeof(float), cudaMemcpyDeviceToHost, s));
    PTRY(cudaStreamSynchronize(s));
    int rc = check_error(p);
    if (rc) return rc;
    if (epoch_loss) epoch_loss[e] = steps > 0 ? l / (float)steps : 0.f;
  }
  return ACO_OK;
}

long long aco_b200_prior_num_examples(aco_b200_prior *p) { return p ? p->n_examples : -1; }

int aco_b200_prior_get_examples(aco_b200_prior *p, int *rows_slots, long long count) {
  if (!p || !rows_slots || count < 0 || count > p->n_examples) return ACO_ERR_INVALID_INPUT;
  cudaSetDevice(p->device);
  if (count == 0) return ACO_OK;
  PTRY(cudaMemcpy(rows_slots, p->d_examples, count * sizeof(int2), cudaMemcpyDeviceToHost));
  return ACO_OK;
}

int aco_b200_prior_get_rows(aco_b200_prior *p, long long first, int count, uint16_t *features,
                            uint8_t *kv, float *scores) {
  if (!p || first < 0 || count < 1 || first + count > p->rows) return ACO_ERR_INVALID_INPUT;
  cudaSetDevice(p->device);
  cudaStream_t s = p->stream;
  if (features)
    PTRY(cudaMemcpy(features, p->d_feat + first * kSlots, (size_t)count * kSlots * sizeof(uint4),
                    cudaMemcpyDeviceToHost));
  if (kv) PTRY(cudaMemcpy(kv, p->d_kv + first, (size_t)count, cudaMemcpyDeviceToHost));
  if (scores) {
    int rc = ensure_scratch(p, count);
    if (rc) return rc;
    rc = launch_forward(p, p->d_feat + first * kSlots, p->d_kv + first, count, p->d_sscores, s);
    if (rc) return rc;
    PTRY(cudaStreamSynchronize(s));
    rc = check_error(p);
    if (rc) return rc;
    PTRY(cudaMemcpy(scores, p->d_sscores, (size_t)count * kSlots * sizeof(float),
                    cudaMemcpyDeviceToHost));
  }
  return ACO_OK;
}

}  // extern "C"
