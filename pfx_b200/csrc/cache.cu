// Kernels and host side of the neural radiance cache (cache.h).
//
// Inference and training run the MLP on the 5th-generation tensor cores:
// a CTA of 128 threads owns a tile of 128 rows (one per thread and per TMEM
// lane), one thread issues tcgen05.mma (M = 128, K = 16 per instruction)
// with the FP32 accumulator in TMEM, and the epilogue reads each row back
// with tcgen05.ld, applies ReLU and writes the next layer's operand into
// shared memory.  Inference gathers the hash grid in a kernel of its own
// (k_encode, four threads per query), which writes the tiles' inputs in the
// operand layout; k_mlp copies them into shared memory in bulk.  Training fuses forward, loss, backward
// and the hash-grid gradient scatter in one kernel; the weight gradients of
// all the CTA's tiles accumulate in TMEM (dW = dH^T x H, the batch rows as
// the K dimension, with the activation tiles read MN-major) and are added
// to the global FP32 gradient once per CTA.  Adam then updates the FP32
// master copies and rewrites the BF16 weights and the FP16 table.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "cache.h"
#include "pfxt_internal.h"
#include "tracer.h"
#include "umma.cuh"

namespace pfxt {

namespace {

// A wait for the tensor cores that runs out of CacheGrid::wait_limit polls sets
// ERR_WAIT; the kernel then drains the MMAs it issued with a wait of DRAIN_LIMIT
// polls (MMAs in flight finish on working hardware, in far less), and frees its
// TMEM only once they have.  If even the drain wait runs out, ERR_DRAIN is set
// and the TMEM stays allocated: freeing columns that an unfinished MMA still
// writes could corrupt another CTA's accumulator without any sign.
constexpr uint32_t DRAIN_LIMIT = 1u << 26;
constexpr uint32_t ERR_WAIT = 1u;
constexpr uint32_t ERR_DRAIN = 2u;

// Shared memory of the training kernel.  dY, dH2 and dH1 are read as M = 128
// MN-major operands whose rows 64..127 (16..127 for dY) are not data: the
// 32 KB the descriptor spans from each of them stays inside the allocation,
// and the accumulator rows they produce are never read.
constexpr uint32_t T_DY = 0, T_DH2 = 4096, T_DH1 = 20480, T_X = 36864, T_H1 = 53248, T_H2 = 69632, T_W = 86016,
                   T_CTRL = T_W + 18432;
constexpr uint32_t T_SMEM = 120 * 1024;  // one CTA (512 TMEM columns) per SM
static_assert(T_DH1 + 32768 <= T_CTRL, "padded MN-major reads stay inside shared memory");
// Weight tiles inside the W block: W1 (64 rows), W2 (64 rows), W3 (16 rows).
constexpr uint32_t W_1 = 0, W_2 = 8192, W_3 = 16384;

constexpr uint32_t ID_F64 = umma::idesc(128, 64, false, false);   // X x W^T, N = 64
constexpr uint32_t ID_F16 = umma::idesc(128, 16, false, false);   // H2 x W3^T
constexpr uint32_t ID_B64 = umma::idesc(128, 64, false, true);    // dH x W (B MN-major)
constexpr uint32_t ID_B32 = umma::idesc(128, 32, false, true);    // dH1 x W1[:, :32]
constexpr uint32_t ID_DW = umma::idesc(128, 64, true, true);      // dH^T x H

__device__ __forceinline__ uint32_t pack2(float a, float b) {
  return (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(a)) |
         ((uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(b)) << 16);
}
__device__ __forceinline__ float lo_bf(uint32_t w) { return __uint_as_float(w << 16); }
__device__ __forceinline__ float hi_bf(uint32_t w) { return __uint_as_float(w & 0xffff0000u); }

// Row r of an R-row tile, `n` columns (a multiple of 8), as BF16.
template <int N>
__device__ __forceinline__ void store_row(uint8_t* tile, uint32_t r, uint32_t R, const float* x) {
#pragma unroll
  for (int g = 0; g < N / 8; ++g) {
    uint4 v = make_uint4(pack2(x[8 * g], x[8 * g + 1]), pack2(x[8 * g + 2], x[8 * g + 3]),
                         pack2(x[8 * g + 4], x[8 * g + 5]), pack2(x[8 * g + 6], x[8 * g + 7]));
    *reinterpret_cast<uint4*>(tile + ((uint32_t)g * (R >> 3) + (r >> 3)) * 128u + (r & 7u) * 16u) = v;
  }
}
// Zeroes x[c] where column 16 s + c of row r of the 128-row, 64-column tile
// `act` is not positive (ReLU'), for c in 0..15.
__device__ __forceinline__ void relu_mask16(const uint8_t* act, uint32_t r, uint32_t s, float* x) {
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const uint32_t g = 2u * s + (uint32_t)h;
    uint4 v = *reinterpret_cast<const uint4*>(act + (g * 16u + (r >> 3)) * 128u + (r & 7u) * 16u);
    uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      if (!(lo_bf(w[j]) > 0.0f)) x[8 * h + 2 * j] = 0.0f;
      if (!(hi_bf(w[j]) > 0.0f)) x[8 * h + 2 * j + 1] = 0.0f;
    }
  }
}

__device__ __forceinline__ float unit_coord(float p, float lo, float inv) {
  float u = (p - lo) * inv;
  return u > 0.0f ? (u < 1.0f ? u : 1.0f) : 0.0f;  // NaN -> 0
}

__device__ __forceinline__ uint32_t grid_index(const CacheGrid& g, uint32_t l, uint32_t x, uint32_t y, uint32_t z) {
  uint32_t res = g.resolution[l];
  uint32_t i = ((g.dense >> l) & 1u) ? x + y * res + z * res * res : (x * 1u) ^ (y * 2654435761u) ^ (z * 805459861u);
  return i & (g.entries - 1u);
}

struct Corners {
  uint32_t ix, iy, iz;
  float wx, wy, wz;
};
__device__ __forceinline__ Corners corners(const CacheGrid& g, uint32_t l, const float u[3]) {
  float s = g.scale[l];
  float px = u[0] * s + 0.5f, py = u[1] * s + 0.5f, pz = u[2] * s + 0.5f;
  float fx = floorf(px), fy = floorf(py), fz = floorf(pz);
  return Corners{(uint32_t)fx, (uint32_t)fy, (uint32_t)fz, px - fx, py - fy, pz - fz};
}
__device__ __forceinline__ float corner_weight(const Corners& c, uint32_t k) {
  float a = (k & 1u) ? c.wx : 1.0f - c.wx;
  float b = (k & 2u) ? c.wy : 1.0f - c.wy;
  float d = (k & 4u) ? c.wz : 1.0f - c.wz;
  return a * b * d;
}

// Hat-function one-blob encoding of a unit vector, 4 bins per component.
__device__ __forceinline__ void one_blob(float v, float* out) {
  float t = (v + 1.0f) * 0.5f * 4.0f;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    float h = 1.0f - fabsf(t - ((float)i + 0.5f));
    out[i] = h > 0.0f ? h : 0.0f;
  }
}

__device__ __forceinline__ uint32_t pick4(const uint4& w, uint32_t j) {
  return j == 0u ? w.x : j == 1u ? w.y : j == 2u ? w.z : w.w;
}
__device__ __forceinline__ float2 entry(uint32_t bits) {
  return __half22float2(*reinterpret_cast<const __half2*>(&bits));
}

// The two features of level l at unit position u: the trilinear blend of
// the cell's 8 corner entries.  Corners 2p and 2p + 1 differ in x only, and
// their entries share an aligned group of four (16 bytes, one sector) unless
// the x + 1 entry carries out of it (dense index i + 1, or hashed index
// (x + 1) ^ h): one 16-byte load fetches the group of the x entry, and a
// second, 4-byte load runs only for the lanes whose x + 1 entry lies outside.
__device__ __forceinline__ void level_features(const CacheGrid& g, const __half2* __restrict__ table, uint32_t l,
                                               const float u[3], float& f0, float& f1) {
  Corners cn = corners(g, l, u);
  const uint32_t* level = reinterpret_cast<const uint32_t*>(table) + (size_t)l * g.entries;
  float2 f[8];
#pragma unroll
  for (uint32_t p = 0; p < 4; ++p) {
    const uint32_t y = cn.iy + (p & 1u), z = cn.iz + (p >> 1);
    const uint32_t i0 = grid_index(g, l, cn.ix, y, z), i1 = grid_index(g, l, cn.ix + 1u, y, z);
    const uint4 w = __ldg(reinterpret_cast<const uint4*>(level + (i0 & ~3u)));
    uint32_t e1;
    if ((i1 & ~3u) == (i0 & ~3u))
      e1 = pick4(w, i1 & 3u);
    else
      e1 = __ldg(level + i1);
    f[2 * p] = entry(pick4(w, i0 & 3u));
    f[2 * p + 1] = entry(e1);
  }
  f0 = 0.0f;
  f1 = 0.0f;
#pragma unroll
  for (uint32_t k = 0; k < 8; ++k) {
    float w = corner_weight(cn, k);
    f0 = f0 + w * f[k].x;
    f1 = f1 + w * f[k].y;
  }
}

// A quarter of one query's 64 network inputs (5 float4: position +
// roughness, direction + transmission, normal, diffuse, specular): quarter q
// gathers levels 4q..4q+3 of the hash grid into v[0..7] (inputs 8q..8q+7) and
// writes inputs 32 + 8q .. 39 + 8q into v[8..15]: one-blob codes of the
// direction (q 0, 1) and normal (q 1, 2), then roughness, diffuse,
// specular and transmission (q 3).
__device__ __forceinline__ void encode_quad(const CacheGrid& g, const __half2* __restrict__ table, const float4* qp,
                                            uint32_t q, float v[16]) {
  const float4 a = __ldg(qp);
  const float u[3] = {unit_coord(a.x, g.lo[0], g.inv_extent[0]), unit_coord(a.y, g.lo[1], g.inv_extent[1]),
                      unit_coord(a.z, g.lo[2], g.inv_extent[2])};
#pragma unroll
  for (uint32_t j = 0; j < 4; ++j) level_features(g, table, 4u * q + j, u, v[2 * j], v[2 * j + 1]);
  if (q == 0u) {
    const float4 b = __ldg(qp + 1);
    one_blob(b.x, v + 8);
    one_blob(b.y, v + 12);
  } else if (q == 1u) {
    const float4 b = __ldg(qp + 1), c = __ldg(qp + 2);
    one_blob(b.z, v + 8);
    one_blob(c.x, v + 12);
  } else if (q == 2u) {
    const float4 c = __ldg(qp + 2);
    one_blob(c.y, v + 8);
    one_blob(c.z, v + 12);
  } else {
    const float4 b = __ldg(qp + 1), d = __ldg(qp + 3), e = __ldg(qp + 4);
    v[8] = a.w > 0.0f ? (a.w < 1.0f ? a.w : 1.0f) : 0.0f;
    v[9] = d.x;
    v[10] = d.y;
    v[11] = d.z;
    v[12] = e.x;
    v[13] = e.y;
    v[14] = e.z;
    v[15] = b.w;
  }
}

// Eight values into row r of column group `group` of an R-row BF16 operand tile.
__device__ __forceinline__ void store_group(uint8_t* tile, uint32_t r, uint32_t R, uint32_t group, const float* v) {
  *reinterpret_cast<uint4*>(tile + (group * (R >> 3) + (r >> 3)) * 128u + (r & 7u) * 16u) =
      make_uint4(pack2(v[0], v[1]), pack2(v[2], v[3]), pack2(v[4], v[5]), pack2(v[6], v[7]));
}

// Gradient of grid features 8q..8q+7 of one query (levels 4q..4q+3) into
// the FP32 table gradient.
__device__ __forceinline__ void scatter_quad(const CacheGrid& g, float* __restrict__ table_g, const float4* q,
                                             uint32_t quad, const float dx[8]) {
  float4 a = __ldg(q);
  float u[3] = {unit_coord(a.x, g.lo[0], g.inv_extent[0]), unit_coord(a.y, g.lo[1], g.inv_extent[1]),
                unit_coord(a.z, g.lo[2], g.inv_extent[2])};
#pragma unroll
  for (uint32_t j = 0; j < 4; ++j) {
    const uint32_t l = 4u * quad + j;
    float g0 = dx[2 * j], g1 = dx[2 * j + 1];
    if (g0 == 0.0f && g1 == 0.0f) continue;
    Corners cn = corners(g, l, u);
    float2* level = reinterpret_cast<float2*>(table_g) + (size_t)l * g.entries;
#pragma unroll
    for (uint32_t k = 0; k < 8; ++k) {
      float w = corner_weight(cn, k);
      uint32_t idx = grid_index(g, l, cn.ix + (k & 1u), cn.iy + ((k >> 1) & 1u), cn.iz + (k >> 2));
      atomicAdd(level + idx, make_float2(w * g0, w * g1));
    }
  }
}

__device__ __forceinline__ void sync_tc() {
  umma::fence_before();
  __syncthreads();
  umma::fence_after();
}

// The 18 KB of BF16 weights into shared memory with one bulk copy (TMA), the
// barrier `wbar` initialised for one arrival: thread 0 expects the bytes and
// issues the copy, every thread waits.  False when the wait ran out (the copy
// then counts as not finished; the kernel reports it and stops).
constexpr uint32_t WEIGHT_BYTES = 18432;
__device__ __forceinline__ bool load_weights(uint8_t* sw, const uint16_t* __restrict__ weights, uint32_t wbar) {
  if (threadIdx.x == 0) {
    umma::mbar_expect_tx(wbar, WEIGHT_BYTES);
    umma::bulk_load(umma::smem_addr(sw), weights, WEIGHT_BYTES, wbar);
  }
  return __syncthreads_and(umma::mbar_wait(wbar, 0u, DRAIN_LIMIT));
}

// End of a tensor-core kernel: after a wait that ran out, flag the error and
// drain the MMAs in flight (the commit of phase `phase ^ 1`) before the TMEM
// is freed; a drain that runs out too leaves the TMEM allocated.
__device__ __forceinline__ void finish(bool failed, uint32_t mb, uint32_t phase, uint32_t* error, uint32_t tbase,
                                       uint32_t cols) {
  bool drained = true;
  if (failed) {
    if (threadIdx.x == 0) atomicOr(error, ERR_WAIT);
    drained = umma::mbar_wait(mb, phase ^ 1u, DRAIN_LIMIT);
    if (!drained && threadIdx.x == 0) atomicOr(error, ERR_DRAIN);
  }
  umma::fence_before();
  drained = __syncthreads_and(drained);
  umma::fence_after();
  if (drained && (threadIdx.x >> 5) == 0) umma::tmem_free(tbase, cols);
}

// Four TMEM loads of 16 columns: this thread's row, columns col..col+63.
__device__ __forceinline__ void ld64(uint32_t tbase, uint32_t warp, uint32_t col, float x[64]) {
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    float v[16];
    umma::ld16(umma::taddr(tbase, 32u * warp, col + 16u * j), v);
#pragma unroll
    for (int k = 0; k < 16; ++k) x[16 * j + k] = v[k];
  }
}

// ------------------------------------------------------------------ inference
// The gather and the MLP as two kernels: k_encode gathers the hash grid with
// four threads per query (all the warps an SM holds, no shared memory or
// TMEM to limit them) and writes each 128-query tile's inputs in the MMA's
// operand layout; k_mlp streams those tiles into shared memory with bulk
// copies, two in flight per CTA, and runs the three layers on the tensor
// cores.  The tiles cross HBM once each way (128 bytes per query).
constexpr uint32_t X_TILE = NRC_ROWS * NRC_IN * 2u;  // 16 KB: one tile's inputs, BF16

// Lane (q, r) of a warp encodes row 8w + r of the queries (w the warp):
// levels 4q..4q+3 (32 corner entries) into column group q, and the extras of
// column group 4 + q; each is one 16-byte store, and the 8 lanes of a q
// write one 128-byte line of the tile.  Rows from the count up to the end
// of the last tile are written as zeros.
__global__ void __launch_bounds__(256)
    k_encode(CacheGrid g, const __half2* __restrict__ table, const float4* __restrict__ queries,
             const uint32_t* __restrict__ n_dev, uint32_t n_max, uint8_t* __restrict__ x) {
  const uint32_t lane = threadIdx.x & 31u, q = lane >> 3;
  const uint32_t row = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 8u + (lane & 7u);
  const uint32_t count = n_dev ? min(*n_dev, n_max) : n_max;
  if (row >= ((count + NRC_ROWS - 1u) & ~(NRC_ROWS - 1u))) return;
  float v[16];
  if (row < count) {
    encode_quad(g, table, queries + (size_t)row * 5u, q, v);
  } else {
#pragma unroll
    for (int k = 0; k < 16; ++k) v[k] = 0.0f;
  }
  uint8_t* tile = x + (size_t)(row / NRC_ROWS) * X_TILE;
  store_group(tile, row % NRC_ROWS, NRC_ROWS, q, v);
  store_group(tile, row % NRC_ROWS, NRC_ROWS, 4u + q, v + 8);
}

// Shared memory of k_mlp: the weights, two input stages and one hidden
// operand (the second hidden layer's overwrites the first's once the MMA
// that read it has completed).
constexpr uint32_t M_W = 0, M_X = WEIGHT_BYTES, M_H = M_X + 2u * X_TILE, M_CTRL = M_H + X_TILE;
constexpr uint32_t M_SMEM = M_CTRL + 64u;  // three CTAs (3 x 128 TMEM columns) per SM
constexpr uint32_t M_TMEM = 128;
static_assert(3u * (M_SMEM + 1024u) <= 228u * 1024u, "three CTAs per SM");

__global__ void __launch_bounds__(128, 3)
    k_mlp(const uint16_t* __restrict__ weights, const uint8_t* __restrict__ x, const uint32_t* __restrict__ n_dev,
          uint32_t n_max, const uint32_t* __restrict__ scatter, float4* __restrict__ out, uint32_t wait_limit,
          uint32_t* error) {
  extern __shared__ __align__(1024) uint8_t smem[];
  const uint32_t tid = threadIdx.x, warp = tid >> 5;
  uint32_t* slot = reinterpret_cast<uint32_t*>(smem + M_CTRL + 32);
  const uint32_t a_w = umma::smem_addr(smem + M_W), a_h = umma::smem_addr(smem + M_H);
  const uint32_t mb = umma::smem_addr(smem + M_CTRL), wb = mb + 8u, xb0 = mb + 16u;  // xb0, xb0 + 8: the stages
  if (tid == 0) {
    umma::mbar_init(mb, 1);
    umma::mbar_init(wb, 1);
    umma::mbar_init(xb0, 1);
    umma::mbar_init(xb0 + 8u, 1);
  }
  __syncthreads();
  if (!load_weights(smem + M_W, weights, wb)) {
    if (tid == 0) atomicOr(error, ERR_WAIT | ERR_DRAIN);
    return;  // no TMEM allocated yet
  }
  const uint32_t count = n_dev ? min(*n_dev, n_max) : n_max;
  const uint32_t tiles = (count + NRC_ROWS - 1u) / NRC_ROWS;
  // thread 0's record of the stages with a copy in flight (drained before the CTA leaves)
  uint32_t pending = 0;
  auto fetch = [&](uint32_t stage, uint32_t tile) {
    if (tile >= tiles) return;
    const uint32_t bar = xb0 + 8u * stage;
    umma::mbar_expect_tx(bar, X_TILE);
    umma::bulk_load(umma::smem_addr(smem + M_X + stage * X_TILE), x + (size_t)tile * X_TILE, X_TILE, bar);
    pending |= 1u << stage;
  };
  if (tid == 0) {
    fetch(0u, blockIdx.x);
    fetch(1u, blockIdx.x + gridDim.x);
  }
  if (warp == 0) umma::tmem_alloc(slot, M_TMEM);
  sync_tc();
  const uint32_t tbase = *slot;
  const uint32_t T0 = tbase, T1 = tbase + 64;
  uint32_t phase = 0, xphase = 0;  // xphase bit s: the parity of stage s's next fill
  bool late = false, mma_pending = false;
  uint32_t i = 0;
  for (uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x, ++i) {
    const uint32_t s = i & 1u, a_x = umma::smem_addr(smem + M_X + s * X_TILE);
    late = !umma::mbar_wait(xb0 + 8u * s, (xphase >> s) & 1u, wait_limit);
    if (__syncthreads_or(late)) break;  // no MMA in flight; the stage's copy is drained below
    xphase ^= 1u << s;
    mma_pending = true;  // from the commit until its wait completes
    if (tid == 0) {
      pending &= ~(1u << s);
#pragma unroll
      for (uint32_t k = 0; k < 4; ++k)
        umma::mma(T0, umma::desc_k(a_x, 128, k), umma::desc_k(a_w + W_1, 64, k), ID_F64, k);
      umma::commit(mb);
    }
    late = !umma::mbar_wait(mb, phase, wait_limit);
    phase ^= 1u;
    if (__syncthreads_or(late)) break;
    umma::fence_after();
    if (tid == 0) fetch(s, tile + 2u * gridDim.x);  // the stage's MMA has read it
    float v[64];
    ld64(tbase, warp, 0, v);
#pragma unroll
    for (int k = 0; k < 64; ++k) v[k] = v[k] > 0.0f ? v[k] : 0.0f;
    store_row<64>(smem + M_H, tid, 128, v);
    umma::fence_async_smem();
    sync_tc();
    if (tid == 0) {
#pragma unroll
      for (uint32_t k = 0; k < 4; ++k)
        umma::mma(T1, umma::desc_k(a_h, 128, k), umma::desc_k(a_w + W_2, 64, k), ID_F64, k);
      umma::commit(mb);
    }
    late = !umma::mbar_wait(mb, phase, wait_limit);
    phase ^= 1u;
    if (__syncthreads_or(late)) break;
    umma::fence_after();
    ld64(tbase, warp, 64, v);
#pragma unroll
    for (int k = 0; k < 64; ++k) v[k] = v[k] > 0.0f ? v[k] : 0.0f;
    store_row<64>(smem + M_H, tid, 128, v);
    umma::fence_async_smem();
    sync_tc();
    if (tid == 0) {
#pragma unroll
      for (uint32_t k = 0; k < 4; ++k)
        umma::mma(T0, umma::desc_k(a_h, 128, k), umma::desc_k(a_w + W_3, 16, k), ID_F16, k);
      umma::commit(mb);
    }
    late = !umma::mbar_wait(mb, phase, wait_limit);
    phase ^= 1u;
    if (__syncthreads_or(late)) break;
    mma_pending = false;
    umma::fence_after();
    float y[16];
    umma::ld16(umma::taddr(tbase, 32u * warp, 0), y);
    const uint32_t row = tile * NRC_ROWS + tid;
    if (row < count) out[scatter ? scatter[row] : row] = make_float4(y[0], y[1], y[2], 0.0f);
    sync_tc();
  }
  // Copies still in flight land before the shared memory is released: each
  // waits on the phase of its own fill, which completes.
  bool landed = true;
  if (tid == 0) {
    for (uint32_t st = 0; st < 2u; ++st)
      if (((pending >> st) & 1u) && !umma::mbar_wait(xb0 + 8u * st, (xphase >> st) & 1u, DRAIN_LIMIT)) landed = false;
  }
  if (!landed) atomicOr(error, ERR_DRAIN);
  if (late && !mma_pending) {
    // the wait that ran out was a copy's: no MMA in flight writes the TMEM
    if (tid == 0) atomicOr(error, ERR_WAIT);
    umma::fence_before();
    __syncthreads();
    if (warp == 0) umma::tmem_free(tbase, M_TMEM);
    return;
  }
  finish(late, mb, phase, error, tbase, M_TMEM);
}

// ------------------------------------------------------------------ training
// Records: 6 float4 (the query's 5, then target rgb + weight).  dY rows are
// the gradient of mean_rows,channels (y - t)^2 / (y^2 + 0.01) (the
// denominator held constant), the relative L2 loss of neural radiance caching.
//
// Four threads share each row: warp w serves TMEM lane quarter w % 4 (rows
// 32 (w % 4)..) and slice s = w / 4 of every row.  Slice s gathers and
// scatters hash-grid levels 4s..4s+3, and moves columns 16s..16s+15 of each
// 64-wide layer between TMEM and shared memory; slice 0 takes the output
// layer and the loss.
constexpr uint32_t TRAIN_THREADS = 512;
__global__ void __launch_bounds__(TRAIN_THREADS, 1)
    k_train(CacheGrid g, const __half2* __restrict__ table, const uint16_t* __restrict__ weights,
            const float4* __restrict__ records, uint32_t first, uint32_t batch, const uint32_t* __restrict__ ran,
            float* __restrict__ mlp_g, float* __restrict__ table_g, float* __restrict__ loss,
            float* __restrict__ cell_stats, uint32_t* error) {
  if (*ran == 0u) return;
  extern __shared__ __align__(1024) uint8_t smem[];
  const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31u;
  const uint32_t quarter = warp & 3u, sl = warp >> 2, row = 32u * quarter + lane;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + T_CTRL);
  uint32_t* slot = reinterpret_cast<uint32_t*>(smem + T_CTRL + 8);
  const uint32_t a_dy = umma::smem_addr(smem + T_DY), a_dh2 = umma::smem_addr(smem + T_DH2),
                 a_dh1 = umma::smem_addr(smem + T_DH1), a_x = umma::smem_addr(smem + T_X),
                 a_h1 = umma::smem_addr(smem + T_H1), a_h2 = umma::smem_addr(smem + T_H2),
                 a_w = umma::smem_addr(smem + T_W);
  const uint32_t mb = umma::smem_addr(mbar), wb = umma::smem_addr(smem + T_CTRL + 16);
  if (tid == 0) {
    umma::mbar_init(mb, 1);
    umma::mbar_init(wb, 1);
  }
  __syncthreads();
  if (!load_weights(smem + T_W, weights, wb)) {
    if (tid == 0) atomicOr(error, ERR_WAIT | ERR_DRAIN);
    return;  // no TMEM allocated yet
  }
  if (warp == 0) umma::tmem_alloc(slot, 512);
  umma::fence_async_smem();
  sync_tc();
  const uint32_t tbase = *slot, tlane = tbase + ((32u * quarter) << 16);
  const uint32_t T0 = 0, T1 = 64, T2 = 128, DW1 = tbase + 192, DW2 = tbase + 256, DW3 = tbase + 320;
  const float scale = 1.0f / (3.0f * (float)batch);
  const uint32_t tiles = batch / NRC_ROWS;
  uint32_t phase = 0, done = 0;
  bool failed = false;
  float loss_sum = 0.0f;
  // the MMAs of one step, then the bounded wait for them (false: it ran out)
  auto wait_mma = [&]() {
    failed = !umma::mbar_wait(mb, phase, g.wait_limit);
    phase ^= 1u;
    failed = __syncthreads_or(failed);
    if (!failed) umma::fence_after();
    return !failed;
  };
  float v[16];
  for (uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x, ++done) {
    const float4* rec = records + ((size_t)first + (size_t)tile * NRC_ROWS + row) * 6u;
    encode_quad(g, table, rec, sl, v);
    store_group(smem + T_X, row, 128, sl, v);
    store_group(smem + T_X, row, 128, 4u + sl, v + 8);
    umma::fence_async_smem();
    sync_tc();
    // forward
    if (tid == 0) {
#pragma unroll
      for (uint32_t s = 0; s < 4; ++s)
        umma::mma(tbase + T0, umma::desc_k(a_x, 128, s), umma::desc_k(a_w + W_1, 64, s), ID_F64, s);
      umma::commit(mb);
    }
    if (!wait_mma()) break;
    umma::ld16(tlane + T0 + 16u * sl, v);
#pragma unroll
    for (int k = 0; k < 16; ++k) v[k] = v[k] > 0.0f ? v[k] : 0.0f;
    store_group(smem + T_H1, row, 128, 2u * sl, v);
    store_group(smem + T_H1, row, 128, 2u * sl + 1u, v + 8);
    umma::fence_async_smem();
    sync_tc();
    if (tid == 0) {
#pragma unroll
      for (uint32_t s = 0; s < 4; ++s)
        umma::mma(tbase + T1, umma::desc_k(a_h1, 128, s), umma::desc_k(a_w + W_2, 64, s), ID_F64, s);
      umma::commit(mb);
    }
    if (!wait_mma()) break;
    umma::ld16(tlane + T1 + 16u * sl, v);
#pragma unroll
    for (int k = 0; k < 16; ++k) v[k] = v[k] > 0.0f ? v[k] : 0.0f;
    store_group(smem + T_H2, row, 128, 2u * sl, v);
    store_group(smem + T_H2, row, 128, 2u * sl + 1u, v + 8);
    umma::fence_async_smem();
    sync_tc();
    if (tid == 0) {
#pragma unroll
      for (uint32_t s = 0; s < 4; ++s)
        umma::mma(tbase + T2, umma::desc_k(a_h2, 128, s), umma::desc_k(a_w + W_3, 16, s), ID_F16, s);
      umma::commit(mb);
    }
    if (!wait_mma()) break;
    if (sl == 0u) {
      // loss and dY
      float y[16];
      umma::ld16(tlane + T2, y);
      float4 t = __ldg(rec + 5);
      float target[3] = {t.x, t.y, t.z};
      float dy[16];
#pragma unroll
      for (int k = 0; k < 16; ++k) dy[k] = 0.0f;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        float d = y[c] - target[c];
        float den = y[c] * y[c] + 0.01f;
        loss_sum = loss_sum + d * d / den;
        dy[c] = 2.0f * d / den * scale;
      }
      if (cell_stats) {
        float4 p = __ldg(rec);
        uint32_t cx = min((uint32_t)(unit_coord(p.x, g.lo[0], g.inv_extent[0]) * (float)NRC_CELLS), NRC_CELLS - 1u);
        uint32_t cy = min((uint32_t)(unit_coord(p.y, g.lo[1], g.inv_extent[1]) * (float)NRC_CELLS), NRC_CELLS - 1u);
        uint32_t cz = min((uint32_t)(unit_coord(p.z, g.lo[2], g.inv_extent[2]) * (float)NRC_CELLS), NRC_CELLS - 1u);
        float* cs = cell_stats + 4u * ((cz * NRC_CELLS + cy) * NRC_CELLS + cx);
        float py = 0.2126f * fmaxf(y[0], 0.0f) + 0.7152f * fmaxf(y[1], 0.0f) + 0.0722f * fmaxf(y[2], 0.0f);
        float ty = 0.2126f * target[0] + 0.7152f * target[1] + 0.0722f * target[2];
        atomicAdd(cs + 0, py - ty);
        atomicAdd(cs + 1, ty);
        atomicAdd(cs + 2, 1.0f);
      }
      store_group(smem + T_DY, row, 128, 0u, dy);
      store_group(smem + T_DY, row, 128, 1u, dy + 8);
    }
    umma::fence_async_smem();
    sync_tc();
    // dW3 += dY^T H2 ; dH2 = dY W3
    if (tid == 0) {
#pragma unroll
      for (uint32_t s = 0; s < 8; ++s)
        umma::mma(DW3, umma::desc_mn(a_dy, 128, s), umma::desc_mn(a_h2, 128, s), ID_DW, (done | s) ? 1u : 0u);
      umma::mma(tbase + T0, umma::desc_k(a_dy, 128, 0), umma::desc_mn(a_w + W_3, 16, 0), ID_B64, 0u);
      umma::commit(mb);
    }
    if (!wait_mma()) break;
    umma::ld16(tlane + T0 + 16u * sl, v);
    relu_mask16(smem + T_H2, row, sl, v);
    store_group(smem + T_DH2, row, 128, 2u * sl, v);
    store_group(smem + T_DH2, row, 128, 2u * sl + 1u, v + 8);
    umma::fence_async_smem();
    sync_tc();
    // dW2 += dH2^T H1 ; dH1 = dH2 W2
    if (tid == 0) {
#pragma unroll
      for (uint32_t s = 0; s < 8; ++s)
        umma::mma(DW2, umma::desc_mn(a_dh2, 128, s), umma::desc_mn(a_h1, 128, s), ID_DW, (done | s) ? 1u : 0u);
#pragma unroll
      for (uint32_t s = 0; s < 4; ++s)
        umma::mma(tbase + T1, umma::desc_k(a_dh2, 128, s), umma::desc_mn(a_w + W_2, 64, s), ID_B64, s);
      umma::commit(mb);
    }
    if (!wait_mma()) break;
    umma::ld16(tlane + T1 + 16u * sl, v);
    relu_mask16(smem + T_H1, row, sl, v);
    store_group(smem + T_DH1, row, 128, 2u * sl, v);
    store_group(smem + T_DH1, row, 128, 2u * sl + 1u, v + 8);
    umma::fence_async_smem();
    sync_tc();
    // dW1 += dH1^T X ; dX = dH1 W1 (grid features only: 32 columns)
    if (tid == 0) {
#pragma unroll
      for (uint32_t s = 0; s < 8; ++s)
        umma::mma(DW1, umma::desc_mn(a_dh1, 128, s), umma::desc_mn(a_x, 128, s), ID_DW, (done | s) ? 1u : 0u);
#pragma unroll
      for (uint32_t s = 0; s < 4; ++s)
        umma::mma(tbase + T2, umma::desc_k(a_dh1, 128, s), umma::desc_mn(a_w + W_1, 64, s), ID_B32, s);
      umma::commit(mb);
    }
    if (!wait_mma()) break;
    // this slice's levels: dX columns 8 sl .. 8 sl + 7 (the load's other 8 columns are not used)
    umma::ld16(tlane + T2 + 8u * sl, v);
    scatter_quad(g, table_g, rec, sl, v);
    sync_tc();
  }
  // loss: warp sums, one atomic per warp
  for (int o = 16; o > 0; o >>= 1) loss_sum += __shfl_xor_sync(0xffffffffu, loss_sum, o);
  if (lane == 0u && loss_sum != 0.0f) atomicAdd(loss, loss_sum);
  if (!failed && done > 0u && quarter < 2u) {
    // weight gradients: TMEM lanes 0..63 hold the rows of dW1 and dW2 (dW3: lanes 0..2); slice sl adds
    // columns 16 sl .. 16 sl + 15 of each
    const uint32_t m = row;  // output feature
    umma::ld16(tlane + 192u + 16u * sl, v);
    for (int k = 0; k < 16; ++k) atomicAdd(mlp_g + NRC_W1 + m * 64u + 16u * sl + k, v[k]);
    umma::ld16(tlane + 256u + 16u * sl, v);
    for (int k = 0; k < 16; ++k) atomicAdd(mlp_g + NRC_W2 + m * 64u + 16u * sl + k, v[k]);
    umma::ld16(tlane + 320u + 16u * sl, v);
    if (m < 3u)
      for (int k = 0; k < 16; ++k) atomicAdd(mlp_g + NRC_W3 + m * 64u + 16u * sl + k, v[k]);
  }
  finish(failed, mb, phase, error, tbase, 512);
}

// ------------------------------------------------------------------ Adam
// step[0]: steps taken, step[1]: this step ran; beta_pow: beta1^t, beta2^t.
__global__ void k_step(const uint32_t* count_dev, uint32_t count, uint32_t need, uint32_t* step, float* beta_pow,
                       float b1, float b2, uint32_t advance, float* loss) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  uint32_t total = count_dev ? *count_dev : count;
  uint32_t run = need <= total ? 1u : 0u;
  step[1] = run;
  loss[0] = 0.0f;
  if (run && advance) {
    step[0] += 1u;
    beta_pow[0] = beta_pow[0] * b1;
    beta_pow[1] = beta_pow[1] * b2;
  }
}

// Lazy Adam: parameters with a zero gradient keep their value and moments.
__global__ void k_adam(float* __restrict__ p, float* __restrict__ m, float* __restrict__ v, float* __restrict__ g,
                       uint32_t n, uint32_t mlp, uint16_t* __restrict__ weights, __half* __restrict__ table16,
                       const uint32_t* __restrict__ step, const float* __restrict__ beta_pow, float lr, float b1,
                       float b2, float eps) {
  if (step[1] == 0u) return;
  const float c1 = 1.0f - beta_pow[0], c2 = 1.0f - beta_pow[1];
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float gi = g[i];
    if (gi == 0.0f) continue;
    g[i] = 0.0f;
    float mi = b1 * m[i] + (1.0f - b1) * gi;
    float vi = b2 * v[i] + (1.0f - b2) * (gi * gi);
    m[i] = mi;
    v[i] = vi;
    float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    p[i] = pi;
    if (mlp) {
      uint32_t base = i < NRC_W2 ? 0u : (i < NRC_W3 ? 4096u : 8192u);
      uint32_t R = i < NRC_W3 ? 64u : 16u;
      uint32_t j = i - (i < NRC_W2 ? NRC_W1 : (i < NRC_W3 ? NRC_W2 : NRC_W3));
      uint32_t off = base + ((j & 63u) >> 3) * (R >> 3) * 64u + ((j >> 6) >> 3) * 64u + ((j >> 6) & 7u) * 8u + (j & 7u);
      weights[off] = __bfloat16_as_ushort(__float2bfloat16_rn(pi));
    } else {
      table16[i] = __float2half_rn(pi);
    }
  }
}

// Rewrites the BF16 weights and the FP16 table from the FP32 masters.
__global__ void k_copies(const float* __restrict__ mlp, uint16_t* __restrict__ weights, const float* __restrict__ table,
                         __half* __restrict__ table16, uint32_t table_n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < NRC_MLP + table_n; i += gridDim.x * blockDim.x) {
    if (i < NRC_MLP) {
      uint32_t base = i < NRC_W2 ? 0u : (i < NRC_W3 ? 4096u : 8192u);
      uint32_t R = i < NRC_W3 ? 64u : 16u;
      uint32_t j = i - (i < NRC_W2 ? NRC_W1 : (i < NRC_W3 ? NRC_W2 : NRC_W3));
      uint32_t off = base + ((j & 63u) >> 3) * (R >> 3) * 64u + ((j >> 6) >> 3) * 64u + ((j >> 6) & 7u) * 8u + (j & 7u);
      weights[off] = __bfloat16_as_ushort(__float2bfloat16_rn(mlp[i]));
    } else {
      uint32_t k = i - NRC_MLP;
      table16[k] = __float2half_rn(table[k]);
    }
  }
}

// A cell lets paths end into the cache once it has seen 32 records and the
// measured relative bias |sum(pred - target)| / sum(target) of the current
// window is within the bound; the window decays by a quarter each pass.
__global__ void k_cells(float* __restrict__ stats, uint8_t* __restrict__ ok, float bound) {
  uint32_t n = NRC_CELLS * NRC_CELLS * NRC_CELLS;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float4 s = reinterpret_cast<float4*>(stats)[i];
    bool good = s.z >= 32.0f && fabsf(s.x) <= bound * (s.y + 1e-3f * s.z);
    ok[i] = good ? 1u : 0u;
    reinterpret_cast<float4*>(stats)[i] = make_float4(s.x * 0.75f, s.y * 0.75f, s.z * 0.75f, 0.0f);
  }
}

void check(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return;
  cudaGetLastError();
  if (e == cudaErrorMemoryAllocation) throw Refused(std::string(what) + ": out of device memory");
  throw DeviceError(std::string(what) + ": " + cudaGetErrorString(e));
}

int sm_count() {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms > 0 ? sms : 1;
}

void attributes() {
  static bool done = false;
  if (done) return;
  check(cudaFuncSetAttribute(k_mlp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)M_SMEM), "cache inference");
  check(cudaFuncSetAttribute(k_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)T_SMEM), "cache training");
  done = true;
}

// PCG32 (O'Neill 2014) for the parameter initialisation.
struct Pcg {
  uint64_t state;
  explicit Pcg(uint64_t seed) : state(seed * 6364136223846793005ull + 1442695040888963407ull) {}
  uint32_t next() {
    uint64_t old = state;
    state = old * 6364136223846793005ull + 1442695040888963407ull;
    uint32_t xorshifted = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    uint32_t rot = (uint32_t)(old >> 59u);
    return (xorshifted >> rot) | (xorshifted << ((32u - rot) & 31u));
  }
  float uniform(float a) { return ((float)(next() >> 8) * (1.0f / 16777216.0f) * 2.0f - 1.0f) * a; }
};

// Beta powers live after the step words.
float* beta_pow(pfxt_cache& c) { return reinterpret_cast<float*>(c.d_step + 2); }

}  // namespace

void cache_validate(const pfxt_cache_settings& s) {
  if (s.log2_entries < 10 || s.log2_entries > 22) throw Invalid("cache: log2_entries must be in 10..22");
  if (s.base_resolution < 2 || s.max_resolution < s.base_resolution || s.max_resolution > (1u << 16))
    throw Invalid("cache: resolutions must satisfy 2 <= base <= max <= 65536");
  if (s.batch == 0 || s.batch % NRC_ROWS != 0 || s.batch > (1u << 22))
    throw Invalid("cache: batch must be a positive multiple of 128, at most 2^22");
  if (s.steps > 64) throw Invalid("cache: at most 64 steps per pass");
  if (!(s.learning_rate > 0.0f) || !(s.beta1 >= 0.0f && s.beta1 < 1.0f) || !(s.beta2 >= 0.0f && s.beta2 < 1.0f) ||
      !(s.epsilon >= 0.0f))
    throw Invalid("cache: Adam hyper-parameters out of range");
  if (!(s.train_fraction >= 0.0f && s.train_fraction <= 1.0f)) throw Invalid("cache: train_fraction must be in [0, 1]");
  if (!(s.error_bound >= 0.0f)) throw Invalid("cache: error_bound must be >= 0");
  if (!(s.min_roughness >= 0.0f)) throw Invalid("cache: min_roughness must be >= 0");
  if (s.delay_bounces > 4) throw Invalid("cache: delay_bounces above 4");
  if (s.record_bounces > 15 || s.query_bounce > 15) throw Invalid("cache: bounces above 15");
  for (int k = 0; k < 3; ++k)
    if (!(s.hi[k] > s.lo[k]) || !std::isfinite(s.lo[k]) || !std::isfinite(s.hi[k]))
      throw Invalid("cache: bounds must be finite with hi > lo");
}

void cache_create(pfxt_cache& c, const pfxt_cache_settings& s) {
  cache_validate(s);
  c.s = s;
  cudaGetDevice(&c.device);
  attributes();
  const uint32_t T = 1u << s.log2_entries;
  c.grid.entries = T;
  c.grid.dense = 0;
  c.grid.wait_limit = NRC_WAIT_LIMIT;
  double growth = std::exp(std::log((double)s.max_resolution / (double)s.base_resolution) / (double)(NRC_LEVELS - 1));
  for (uint32_t l = 0; l < NRC_LEVELS; ++l) {
    double scale = (double)s.base_resolution * std::pow(growth, (double)l) - 1.0;
    c.grid.scale[l] = (float)scale;
    uint32_t res = (uint32_t)std::ceil((double)c.grid.scale[l]) + 2u;
    c.grid.resolution[l] = res;
    if ((uint64_t)res * res * res <= T) c.grid.dense |= 1u << l;
  }
  cache_set_bounds(c, s.lo, s.hi);
  const size_t table_n = (size_t)NRC_LEVELS * T * 2u;
  auto alloc = [&](void** p, size_t bytes, const char* what) { check(cudaMalloc(p, bytes), what); };
  alloc((void**)&c.d_mlp, NRC_MLP * 4u, "cache parameters");
  alloc((void**)&c.d_mlp_m, NRC_MLP * 4u, "cache parameters");
  alloc((void**)&c.d_mlp_v, NRC_MLP * 4u, "cache parameters");
  alloc((void**)&c.d_mlp_g, NRC_MLP * 4u, "cache parameters");
  alloc((void**)&c.d_weights, 18432u, "cache weights");
  alloc((void**)&c.d_table, table_n * 4u, "cache table");
  alloc((void**)&c.d_table_m, table_n * 4u, "cache table");
  alloc((void**)&c.d_table_v, table_n * 4u, "cache table");
  alloc((void**)&c.d_table_g, table_n * 4u, "cache table");
  alloc((void**)&c.d_table16, table_n * 2u, "cache table");
  const uint32_t cells = NRC_CELLS * NRC_CELLS * NRC_CELLS;
  alloc((void**)&c.d_cell_ok, cells, "cache cells");
  alloc((void**)&c.d_cell_stats, cells * 16u, "cache cells");
  alloc((void**)&c.d_loss, 16, "cache loss");
  alloc((void**)&c.d_step, 16, "cache step");
  alloc((void**)&c.d_error, 4, "cache error word");
  check(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking), "cache stream");
  for (float* p : {c.d_mlp_m, c.d_mlp_v, c.d_mlp_g}) check(cudaMemset(p, 0, NRC_MLP * 4u), "cache reset");
  for (float* p : {c.d_table_m, c.d_table_v, c.d_table_g}) check(cudaMemset(p, 0, table_n * 4u), "cache reset");
  check(cudaMemset(c.d_cell_ok, 0, cells), "cache reset");
  check(cudaMemset(c.d_cell_stats, 0, cells * 16u), "cache reset");
  check(cudaMemset(c.d_loss, 0, 16), "cache reset");
  check(cudaMemset(c.d_error, 0, 4), "cache reset");
  uint32_t step_init[4];
  float one = 1.0f;
  step_init[0] = 0;
  step_init[1] = 0;
  std::memcpy(&step_init[2], &one, 4);
  std::memcpy(&step_init[3], &one, 4);
  check(cudaMemcpy(c.d_step, step_init, 16, cudaMemcpyHostToDevice), "cache step");
  // Glorot-uniform weights (W3 rows 3..15 stay zero) and a small uniform table.
  std::vector<float> mlp(NRC_MLP, 0.0f);
  Pcg rng(0x9e3779b97f4a7c15ull ^ (uint64_t)s.seed);
  float a_hidden = std::sqrt(6.0f / 128.0f), a_out = std::sqrt(6.0f / 67.0f);
  for (uint32_t i = 0; i < NRC_W3; ++i) mlp[i] = rng.uniform(a_hidden);
  for (uint32_t i = 0; i < 3u * NRC_HIDDEN; ++i) mlp[NRC_W3 + i] = rng.uniform(a_out);
  std::vector<float> table(table_n);
  for (size_t i = 0; i < table_n; ++i) table[i] = rng.uniform(1e-4f);
  check(cudaMemcpy(c.d_mlp, mlp.data(), NRC_MLP * 4u, cudaMemcpyHostToDevice), "cache parameters");
  check(cudaMemcpy(c.d_table, table.data(), table_n * 4u, cudaMemcpyHostToDevice), "cache table");
  k_copies<<<sm_count() * 4, 256, 0, c.stream>>>(c.d_mlp, c.d_weights, c.d_table, (__half*)c.d_table16,
                                                  (uint32_t)table_n);
  check(cudaGetLastError(), "cache copies");
  check(cudaStreamSynchronize(c.stream), "cache create");
}

void cache_release(pfxt_cache& c) {
  for (void* p : {(void*)c.d_mlp, (void*)c.d_mlp_m, (void*)c.d_mlp_v, (void*)c.d_mlp_g, (void*)c.d_weights,
                  (void*)c.d_table, (void*)c.d_table_m, (void*)c.d_table_v, (void*)c.d_table_g, (void*)c.d_table16,
                  (void*)c.d_cell_ok, (void*)c.d_cell_stats, (void*)c.d_loss, (void*)c.d_step, (void*)c.d_error,
                  c.d_stage})
    if (p) cudaFree(p);
  if (c.stream) cudaStreamDestroy(c.stream);
  c.stream = nullptr;
  c.d_stage = nullptr;
  c.stage_bytes = 0;
}

void cache_set_bounds(pfxt_cache& c, const float lo[3], const float hi[3]) {
  for (int k = 0; k < 3; ++k) {
    if (!(hi[k] > lo[k]) || !std::isfinite(lo[k]) || !std::isfinite(hi[k]))
      throw Invalid("cache: bounds must be finite with hi > lo");
    c.grid.lo[k] = lo[k];
    c.grid.inv_extent[k] = 1.0f / (hi[k] - lo[k]);
    c.s.lo[k] = lo[k];
    c.s.hi[k] = hi[k];
  }
}

CacheView cache_view(pfxt_cache& c) {
  CacheView v;
  v.grid = c.grid;
  v.table = c.d_table16;
  v.weights = c.d_weights;
  v.cell_ok = c.d_cell_ok;
  v.cell_stats = c.d_cell_stats;
  return v;
}

size_t cache_x_bytes(uint32_t n) { return (size_t)((n + NRC_ROWS - 1) / NRC_ROWS) * X_TILE; }

void cache_infer_launch(pfxt_cache& c, const float4* queries, const uint32_t* n_dev, uint32_t n,
                        const uint32_t* scatter, float4* out, uint8_t* x, cudaStream_t stream) {
  if (n == 0) return;
  if (c.broken) throw DeviceError("cache: unusable after an undrained tensor-core wait");
  const uint32_t tiles = (n + NRC_ROWS - 1) / NRC_ROWS;
  // 8 rows per warp, 64 per block of 256 threads, over whole tiles
  k_encode<<<(tiles * NRC_ROWS + 63u) / 64u, 256, 0, stream>>>(c.grid, c.d_table16, queries, n_dev, n, x);
  const uint32_t grid = std::min<uint32_t>(tiles, (uint32_t)sm_count() * 3u);
  k_mlp<<<grid, 128, M_SMEM, stream>>>(c.d_weights, x, n_dev, n, scatter, out, c.grid.wait_limit, c.d_error);
  check(cudaGetLastError(), "cache inference");
}

void cache_train_launch(pfxt_cache& c, const float4* records, const uint32_t* count_dev, uint32_t count,
                        uint32_t first, cudaStream_t stream, bool adam, uint32_t batch) {
  if (batch == 0) batch = c.s.batch;
  if (c.broken) throw DeviceError("cache: unusable after an undrained tensor-core wait");
  const uint32_t table_n = NRC_LEVELS * c.grid.entries * 2u;
  k_step<<<1, 32, 0, stream>>>(count_dev, count, first + batch, c.d_step, beta_pow(c), c.s.beta1, c.s.beta2,
                               adam ? 1u : 0u, c.d_loss);
  uint32_t grid = std::min<uint32_t>(batch / NRC_ROWS, (uint32_t)sm_count());
  k_train<<<grid, TRAIN_THREADS, T_SMEM, stream>>>(c.grid, c.d_table16, c.d_weights, records, first, batch, c.d_step + 1,
                                         c.d_mlp_g, c.d_table_g, c.d_loss, adam ? c.d_cell_stats : nullptr,
                                         c.d_error);
  check(cudaGetLastError(), "cache training");
  if (!adam) return;
  int sms = sm_count();
  k_adam<<<sms, 256, 0, stream>>>(c.d_mlp, c.d_mlp_m, c.d_mlp_v, c.d_mlp_g, NRC_MLP, 1u, c.d_weights, nullptr,
                                  c.d_step, beta_pow(c), c.s.learning_rate, c.s.beta1, c.s.beta2, c.s.epsilon);
  k_adam<<<sms * 8, 256, 0, stream>>>(c.d_table, c.d_table_m, c.d_table_v, c.d_table_g, table_n, 0u, nullptr,
                                      (__half*)c.d_table16, c.d_step, beta_pow(c), c.s.learning_rate, c.s.beta1,
                                      c.s.beta2, c.s.epsilon);
  check(cudaGetLastError(), "cache Adam");
}

void cache_cells_launch(pfxt_cache& c, cudaStream_t stream) {
  k_cells<<<16, 256, 0, stream>>>(c.d_cell_stats, c.d_cell_ok, c.s.error_bound);
  check(cudaGetLastError(), "cache cells");
}

void cache_check_error(pfxt_cache& c) {
  uint32_t e = 0;
  check(cudaMemcpy(&e, c.d_error, 4, cudaMemcpyDeviceToHost), "cache error word");
  if (e != 0u) {
    cudaMemset(c.d_error, 0, 4);
    if (e & ERR_DRAIN) {
      c.broken = true;
      throw DeviceError("cache: the tensor cores did not finish the MMAs in flight; the cache is unusable");
    }
    throw DeviceError("cache: a tensor-core wait ran out of its limit");
  }
}

void cache_copies(pfxt_cache& c) {
  const uint32_t table_n = NRC_LEVELS * c.grid.entries * 2u;
  k_copies<<<sm_count() * 4, 256, 0, c.stream>>>(c.d_mlp, c.d_weights, c.d_table, (__half*)c.d_table16, table_n);
  check(cudaGetLastError(), "cache copies");
}

}  // namespace pfxt
