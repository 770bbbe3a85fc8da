// The binned-SAH BVH build of bvh.rs:95-266 on the GPU, byte for byte the
// host build's (build.cpp BvhBuilder): the same nodes in the same preorder and
// the same triangle order.
//
// The host build is a depth-first recursion; this one goes level by level.
// Every decision the recursion makes per node is order-free or sequential in
// a way that can be reproduced in parallel:
//  * a node's box and centroid box, and each bin's box and count, are minima,
//    maxima and counts (order-free when no coordinate is -0.0, whose min/max
//    against +0.0 would depend on the order; such inputs stay on the host);
//  * the SAH sweep over 16 bins per axis runs on one thread per node with the
//    host's arithmetic, operation for operation (-fmad=false);
//  * the in-place partition of bvh.rs:232-249 (left pointer tests, a failing
//    element is swapped with the last unexamined one) is a fixed permutation
//    of the node's range given each element's side.  Reading the elements from
//    the front while they pass and from the back while they fail, the examined
//    sequence alternates front runs ending in a failing element and back runs
//    ending in a passing one; passing elements fill the range from the front
//    and failing ones from the back, both in examination order.  Each
//    element's place follows from prefix counts of failing elements from the
//    front and passing elements from the back (k_place below), so the
//    permutation is computed by scans instead of a sequential loop;
//  * node indices are preorder (a node, its left subtree, its right subtree):
//    subtree sizes are summed bottom-up over the levels, then each node's index
//    is its parent's + 1 (left) or + 1 + the left subtree's size (right).
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "pfxt_internal.h"
#include "pfxt_types.h"

namespace pfxt {

namespace {

constexpr int BINS = 16;
constexpr uint32_t NONE = 0xffffffffu;
constexpr int BLOCK = 256;

// A float's position in the total order of non-NaN floats as an unsigned key,
// for atomic minima and maxima.
__device__ __forceinline__ uint32_t fkey(float f) {
  uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float unkey(uint32_t k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}
constexpr uint32_t KEY_POS_INF = 0xff800000u;  // fkey(+inf)
constexpr uint32_t KEY_NEG_INF = 0x007fffffu;  // fkey(-inf)

// Rust's f32::min/max for non-NaN operands.
__device__ __forceinline__ float rmin(float a, float b) { return b < a ? b : a; }
__device__ __forceinline__ float rmax(float a, float b) { return b > a ? b : a; }

// bvh.rs:268-270
__device__ __forceinline__ uint32_t bin_of(float value, float lo, float extent) {
  float x = ((value - lo) / extent) * (float)BINS;
  x = rmin(rmax(x, 0.0f), (float)(BINS - 1));
  if (x != x) return 0u;
  return (uint32_t)x;
}

__device__ __forceinline__ float area_of(const float lo[3], const float hi[3]) {  // bvh.rs:64-71
  float d0 = hi[0] - lo[0], d1 = hi[1] - lo[1], d2 = hi[2] - lo[2];
  if (d0 < 0.0f) return 0.0f;
  return 2.0f * (d0 * d1 + d1 * d2 + d2 * d0);
}

// One node of the level being built.
struct LNode {
  uint32_t start, end;
  uint32_t parent;  // index of the parent in the previous level, NONE for the root
  uint32_t side;    // 0 left child, 1 right child
};

// Per level node: accumulated boxes (keys), the decision and the children.
struct Acc {
  uint32_t lo[3], hi[3], clo[3], chi[3];  // node box and centroid box as keys
};
struct Decision {
  uint32_t leaf;         // 1: a leaf
  uint32_t partition;    // 1: the range is partitioned on (axis, bin)
  uint32_t axis, bin;
  uint32_t mid;          // absolute split position (inner nodes)
  uint32_t left, right;  // indices of the children in the next level
  float lo[3], hi[3];
};
// Bins of a node: per axis and bin, box keys and count.
struct BinAcc {
  uint32_t lo[3][BINS][3], hi[3][BINS][3], count[3][BINS];
};

__global__ void k_prepare(const float* __restrict__ boxes, uint32_t n, float* __restrict__ cen,
                          uint32_t* __restrict__ order, uint32_t* __restrict__ seg) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    for (int k = 0; k < 3; ++k) cen[3 * i + k] = (boxes[6 * i + k] + boxes[6 * i + 3 + k]) * 0.5f;
    order[i] = i;
    seg[i] = 0u;
  }
}

__global__ void k_init_level(Acc* __restrict__ acc, BinAcc* __restrict__ bins, uint32_t count) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    for (int k = 0; k < 3; ++k) {
      acc[i].lo[k] = KEY_POS_INF;
      acc[i].hi[k] = KEY_NEG_INF;
      acc[i].clo[k] = KEY_POS_INF;
      acc[i].chi[k] = KEY_NEG_INF;
    }
    BinAcc& b = bins[i];
    for (int a = 0; a < 3; ++a)
      for (int j = 0; j < BINS; ++j) {
        for (int k = 0; k < 3; ++k) {
          b.lo[a][j][k] = KEY_POS_INF;
          b.hi[a][j][k] = KEY_NEG_INF;
        }
        b.count[a][j] = 0u;
      }
  }
}

// Node boxes and centroid boxes: warps whose elements share a node reduce
// first, then one atomic per key.
__global__ void k_bounds(const float* __restrict__ boxes, const float* __restrict__ cen,
                         const uint32_t* __restrict__ order, const uint32_t* __restrict__ seg, uint32_t n,
                         Acc* __restrict__ acc) {
  const unsigned FULL = 0xffffffffu;
  for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    uint32_t p = base + threadIdx.x;
    uint32_t node = p < n ? seg[p] : NONE;
    uint32_t key[12];
    if (node != NONE) {
      uint32_t e = order[p];
      for (int k = 0; k < 3; ++k) {
        float lo = boxes[6 * e + k], hi = boxes[6 * e + 3 + k];
        key[k] = fkey(lo);     // grow: min over lo and hi is the min over lo
        key[3 + k] = fkey(hi);
        key[6 + k] = fkey(cen[3 * e + k]);
        key[9 + k] = key[6 + k];
      }
    } else {
      for (int k = 0; k < 3; ++k) {
        key[k] = KEY_POS_INF;
        key[3 + k] = KEY_NEG_INF;
        key[6 + k] = KEY_POS_INF;
        key[9 + k] = KEY_NEG_INF;
      }
    }
    uint32_t first = __shfl_sync(FULL, node, 0);
    if (__all_sync(FULL, node == first)) {
      for (int o = 16; o > 0; o >>= 1)
        for (int k = 0; k < 3; ++k) {
          key[k] = min(key[k], __shfl_xor_sync(FULL, key[k], o));
          key[3 + k] = max(key[3 + k], __shfl_xor_sync(FULL, key[3 + k], o));
          key[6 + k] = min(key[6 + k], __shfl_xor_sync(FULL, key[6 + k], o));
          key[9 + k] = max(key[9 + k], __shfl_xor_sync(FULL, key[9 + k], o));
        }
      if ((threadIdx.x & 31) == 0 && first != NONE) {
        for (int k = 0; k < 3; ++k) {
          atomicMin(&acc[first].lo[k], key[k]);
          atomicMax(&acc[first].hi[k], key[3 + k]);
          atomicMin(&acc[first].clo[k], key[6 + k]);
          atomicMax(&acc[first].chi[k], key[9 + k]);
        }
      }
    } else if (node != NONE) {
      for (int k = 0; k < 3; ++k) {
        atomicMin(&acc[node].lo[k], key[k]);
        atomicMax(&acc[node].hi[k], key[3 + k]);
        atomicMin(&acc[node].clo[k], key[6 + k]);
        atomicMax(&acc[node].chi[k], key[9 + k]);
      }
    }
  }
}

// Per-axis bins of the nodes that have more than `leaf` elements.  A block
// whose elements all belong to one node accumulates in shared memory first.
__global__ void __launch_bounds__(BLOCK) k_bins(const float* __restrict__ boxes, const float* __restrict__ cen,
                                                const uint32_t* __restrict__ order, const uint32_t* __restrict__ seg,
                                                const LNode* __restrict__ level, const Acc* __restrict__ acc,
                                                uint32_t n, uint32_t leaf, BinAcc* __restrict__ bins) {
  __shared__ BinAcc local;
  __shared__ uint32_t shared_node;
  const uint32_t per = BLOCK * 4;
  for (uint32_t base = blockIdx.x * per; base < n; base += gridDim.x * per) {
    uint32_t last = min(base + per, n) - 1u;
    if (threadIdx.x == 0) shared_node = (seg[base] == seg[last]) ? seg[base] : NONE;
    __syncthreads();
    const uint32_t one = shared_node;
    bool use_shared = false;
    if (one != NONE) {
      const LNode& L = level[one];
      use_shared = L.end - L.start > leaf;
    }
    if (use_shared) {
      uint32_t* w = reinterpret_cast<uint32_t*>(&local);
      for (uint32_t k = threadIdx.x; k < sizeof(BinAcc) / 4; k += BLOCK) {
        // lo keys, hi keys, counts
        uint32_t slot = k;
        w[k] = slot < 3 * BINS * 3 ? KEY_POS_INF : (slot < 6 * BINS * 3 ? KEY_NEG_INF : 0u);
      }
      __syncthreads();
    }
    for (uint32_t p = base + threadIdx.x; p <= last; p += BLOCK) {
      uint32_t node = seg[p];
      if (node == NONE) continue;
      const LNode& L = level[node];
      if (L.end - L.start <= leaf) continue;
      const Acc& a = acc[node];
      uint32_t e = order[p];
      BinAcc* target = use_shared ? &local : &bins[node];
      for (int axis = 0; axis < 3; ++axis) {
        float clo = unkey(a.clo[axis]), chi = unkey(a.chi[axis]);
        float extent = chi - clo;
        if (extent <= 1e-9f) continue;
        uint32_t b = bin_of(cen[3 * e + axis], clo, extent);
        for (int k = 0; k < 3; ++k) {
          atomicMin(&target->lo[axis][b][k], fkey(boxes[6 * e + k]));
          atomicMax(&target->hi[axis][b][k], fkey(boxes[6 * e + 3 + k]));
        }
        atomicAdd(&target->count[axis][b], 1u);
      }
    }
    if (use_shared) {
      __syncthreads();
      const uint32_t* w = reinterpret_cast<const uint32_t*>(&local);
      uint32_t* g = reinterpret_cast<uint32_t*>(&bins[one]);
      for (uint32_t k = threadIdx.x; k < sizeof(BinAcc) / 4; k += BLOCK) {
        if (k < 3 * BINS * 3) {
          if (w[k] != KEY_POS_INF) atomicMin(&g[k], w[k]);
        } else if (k < 6 * BINS * 3) {
          if (w[k] != KEY_NEG_INF) atomicMax(&g[k], w[k]);
        } else if (w[k]) {
          atomicAdd(&g[k], w[k]);
        }
      }
    }
    __syncthreads();
  }
}

// bvh.rs:167-266 per node: leaf or split, and the split.
__global__ void k_decide(const LNode* __restrict__ level, const Acc* __restrict__ acc,
                         const BinAcc* __restrict__ bins, uint32_t count, uint32_t leaf, uint32_t most,
                         Decision* __restrict__ out, uint32_t* __restrict__ next_count) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    const LNode& L = level[i];
    const Acc& a = acc[i];
    Decision d;
    float blo[3], bhi[3];
    for (int k = 0; k < 3; ++k) {
      blo[k] = unkey(a.lo[k]);
      bhi[k] = unkey(a.hi[k]);
      d.lo[k] = blo[k];
      d.hi[k] = bhi[k];
    }
    uint32_t len = L.end - L.start;
    d.leaf = 1u;
    d.partition = 0u;
    d.axis = 0u;
    d.bin = 0u;
    d.mid = 0u;
    d.left = d.right = NONE;
    if (len > leaf) {
      const BinAcc& B = bins[i];
      float best_cost = INFINITY;
      uint32_t best_axis = 0, best_bin = 0;
      for (int axis = 0; axis < 3; ++axis) {
        float extent = unkey(a.chi[axis]) - unkey(a.clo[axis]);
        if (extent <= 1e-9f) continue;
        float areas[BINS];
        uint32_t counts[BINS];
        float glo[3] = {INFINITY, INFINITY, INFINITY}, ghi[3] = {-INFINITY, -INFINITY, -INFINITY};
        uint32_t c = 0;
        for (int b = 0; b < BINS; ++b) {
          if (B.count[axis][b] > 0)
            for (int k = 0; k < 3; ++k) {
              glo[k] = rmin(glo[k], unkey(B.lo[axis][b][k]));
              ghi[k] = rmax(ghi[k], unkey(B.hi[axis][b][k]));
            }
          c += B.count[axis][b];
          areas[b] = area_of(glo, ghi);
          counts[b] = c;
        }
        for (int k = 0; k < 3; ++k) {
          glo[k] = INFINITY;
          ghi[k] = -INFINITY;
        }
        c = 0;
        for (int b = BINS - 1; b >= 1; --b) {
          if (B.count[axis][b] > 0)
            for (int k = 0; k < 3; ++k) {
              glo[k] = rmin(glo[k], unkey(B.lo[axis][b][k]));
              ghi[k] = rmax(ghi[k], unkey(B.hi[axis][b][k]));
            }
          c += B.count[axis][b];
          float cost = areas[b - 1] * (float)counts[b - 1] + area_of(glo, ghi) * (float)c;
          if (counts[b - 1] > 0 && c > 0 && cost < best_cost) {
            best_cost = cost;
            best_axis = (uint32_t)axis;
            best_bin = (uint32_t)b;
          }
        }
      }
      if (!(best_cost >= area_of(blo, bhi) * (float)len && len <= most)) {
        d.leaf = 0u;
        if (isfinite(best_cost)) {
          d.partition = 1u;
          d.axis = best_axis;
          d.bin = best_bin;
        } else {
          d.mid = L.start + len / 2u;
        }
        uint32_t first = atomicAdd(next_count, 2u);
        d.left = first;
        d.right = first + 1u;
      }
    }
    out[i] = d;
  }
}

// Side flags of the partitioned ranges: pass[p] = 1 when the element's bin is
// below the split bin (bvh.rs:236).
__global__ void k_flags(const float* __restrict__ cen, const uint32_t* __restrict__ order,
                        const uint32_t* __restrict__ seg, const Acc* __restrict__ acc,
                        const Decision* __restrict__ dec, uint32_t n, uint32_t* __restrict__ pass,
                        uint32_t* __restrict__ fail) {
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    uint32_t node = seg[p];
    uint32_t t = 0u, f = 0u;
    if (node != NONE && dec[node].partition) {
      const Decision& d = dec[node];
      float clo = unkey(acc[node].clo[d.axis]), chi = unkey(acc[node].chi[d.axis]);
      uint32_t b = bin_of(cen[3 * order[p] + d.axis], clo, chi - clo);
      t = b < d.bin ? 1u : 0u;
      f = 1u - t;
    }
    pass[p] = t;
    fail[p] = f;
  }
}

// Exclusive scans of the flags: sums of 1024-element tiles, then the tiles'
// offsets, then the scan within each tile.
constexpr uint32_t TILE = 1024;
__global__ void k_tile_sums(const uint32_t* __restrict__ in, uint32_t n, uint32_t* __restrict__ sums) {
  __shared__ uint32_t warp_sum[TILE / 32];
  uint32_t base = blockIdx.x * TILE;
  uint32_t v = 0;
  for (uint32_t k = threadIdx.x; k < TILE; k += blockDim.x) {
    uint32_t p = base + k;
    v += p < n ? in[p] : 0u;
  }
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) warp_sum[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t s = 0;
    for (uint32_t w = 0; w < blockDim.x / 32; ++w) s += warp_sum[w];
    sums[blockIdx.x] = s;
  }
}
// One block of TILE threads: exclusive scan of a tile in place (its offset added).
__global__ void __launch_bounds__(TILE) k_tile_scan(uint32_t* __restrict__ data, uint32_t n,
                                                    const uint32_t* __restrict__ offsets, uint32_t* __restrict__ out) {
  __shared__ uint32_t warp_sum[TILE / 32];
  uint32_t p = blockIdx.x * TILE + threadIdx.x;
  uint32_t v = p < n ? data[p] : 0u;
  uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = v;
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= (uint32_t)o) x += y;
  }
  if (lane == 31) warp_sum[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t s = warp_sum[lane];
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= (uint32_t)o) s += y;
    }
    warp_sum[lane] = s;
  }
  __syncthreads();
  uint32_t before = (warp > 0 ? warp_sum[warp - 1] : 0u) + (offsets ? offsets[blockIdx.x] : 0u);
  if (p < n) out[p] = before + x - v;
}

// Where each element of a partitioned range goes.  For the node's range
// [s, e) with L passing elements: front element i (position s + i) and back
// element j (position e - 1 - j) are the two ways an element can be reached;
// exactly one of them is examined.  cf: failing elements before front i; ct:
// passing elements before back j; P[k]: front index of the (k+1)-th failing
// element; Q[k]: back index of the (k+1)-th passing element.
__global__ void k_ranks(const uint32_t* __restrict__ seg, const Decision* __restrict__ dec,
                        const LNode* __restrict__ level, const uint32_t* __restrict__ pass,
                        const uint32_t* __restrict__ pass_scan, const uint32_t* __restrict__ fail_scan, uint32_t n,
                        uint32_t* __restrict__ P, uint32_t* __restrict__ Q) {
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    uint32_t node = seg[p];
    if (node == NONE || !dec[node].partition) continue;
    const LNode& L = level[node];
    if (pass[p]) {
      // passing elements after p in the node = its rank from the back
      uint32_t after = (pass_scan[L.end - 1] + pass[L.end - 1]) - (pass_scan[p] + 1u);
      Q[L.start + after] = L.end - 1u - p;
    } else {
      P[L.start + (fail_scan[p] - fail_scan[L.start])] = p - L.start;
    }
  }
}

__global__ void k_place(const uint32_t* __restrict__ seg, Decision* dec,
                        const LNode* __restrict__ level, const uint32_t* __restrict__ pass,
                        const uint32_t* __restrict__ pass_scan, const uint32_t* __restrict__ fail_scan,
                        const uint32_t* __restrict__ P, const uint32_t* __restrict__ Q,
                        const uint32_t* __restrict__ order, uint32_t n, uint32_t* __restrict__ placed,
                        uint32_t* __restrict__ error) {
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    uint32_t node = seg[p];
    if (node == NONE || !dec[node].partition) continue;
    const LNode& L = level[node];
    const uint32_t s = L.start, e = L.end, len = e - s;
    const uint32_t total_pass = (pass_scan[e - 1] + pass[e - 1]) - pass_scan[s];
    const uint32_t i = p - s;          // as a front element
    const uint32_t j = e - 1u - p;     // as a back element
    const bool t = pass[p] != 0u;
    // failing elements before front i; passing elements before back j
    const uint32_t cf = fail_scan[p] - fail_scan[s];
    const uint32_t ct = (pass_scan[e - 1] + pass[e - 1]) - (pass_scan[p] + pass[p]);
    // front role: round k = cf + 1; back elements examined before round k: QB
    uint32_t k = cf + 1u;
    bool front = false;
    uint32_t QB = 0;
    if (k == 1u) {
      front = i < len;
    } else if (k - 2u < total_pass) {
      QB = Q[s + (k - 2u)] + 1u;
      front = i + QB < len;
    }
    uint32_t dest;
    if (front) {
      dest = t ? (i - cf) + (k - 1u) : len - 1u - (cf + (QB - (k - 1u)));
    } else {
      uint32_t kb = ct + 1u;  // back role: round kb, needs the kb-th failing front element
      if (kb - 1u >= len - total_pass) {  // cannot happen: every element is examined in one role
        atomicOr(error, 1u);
        continue;
      }
      uint32_t pk = P[s + (kb - 1u)];
      dest = t ? (pk + 1u - kb) + ct : len - 1u - (kb + (j - ct));
    }
    if (dest >= len) {  // cannot happen either; checked rather than written out of range
      atomicOr(error, 2u);
      continue;
    }
    placed[s + dest] = order[p];
    if (p == s) {
      // the split position: the passing count, or the middle when one side is empty
      uint32_t left = total_pass;
      dec[node].mid = (left == 0u || left == len) ? s + len / 2u : s + left;
    }
  }
}

__global__ void k_copy_placed(const uint32_t* __restrict__ seg, const Decision* __restrict__ dec,
                              const uint32_t* __restrict__ placed, uint32_t n, uint32_t* __restrict__ order) {
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    uint32_t node = seg[p];
    if (node != NONE && dec[node].partition) order[p] = placed[p];
  }
}

// The next level's nodes and every element's node in it.
__global__ void k_children(const LNode* __restrict__ level, const Decision* __restrict__ dec, uint32_t count,
                           LNode* __restrict__ next) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    const Decision& d = dec[i];
    if (d.leaf) continue;
    next[d.left] = LNode{level[i].start, d.mid, i, 0u};
    next[d.right] = LNode{d.mid, level[i].end, i, 1u};
  }
}
__global__ void k_segments(uint32_t* __restrict__ seg, const Decision* __restrict__ dec, uint32_t n) {
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    uint32_t node = seg[p];
    if (node == NONE) continue;
    const Decision& d = dec[node];
    seg[p] = d.leaf ? NONE : (p < d.mid ? d.left : d.right);
  }
}

void cu(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return;
  cudaGetLastError();
  throw std::runtime_error(std::string("GPU BVH build: ") + what + ": " + cudaGetErrorString(e));
}

uint32_t grid_for(uint64_t items, uint32_t per_block) {
  uint64_t g = (items + per_block - 1) / per_block;
  return (uint32_t)std::min<uint64_t>(std::max<uint64_t>(g, 1), 148ull * 32ull);
}

// Exclusive scan of n flags into `out` (tile sums recursed until one tile).
void scan(uint32_t* in, uint32_t n, uint32_t* out, std::vector<uint32_t*>& scratch, size_t depth,
          cudaStream_t st) {
  uint32_t tiles = (n + TILE - 1) / TILE;
  if (tiles <= 1) {
    k_tile_scan<<<1, TILE, 0, st>>>(in, n, nullptr, out);
    return;
  }
  uint32_t* sums = scratch[2 * depth];
  uint32_t* offsets = scratch[2 * depth + 1];
  k_tile_sums<<<tiles, BLOCK, 0, st>>>(in, n, sums);
  scan(sums, tiles, offsets, scratch, depth + 1, st);
  k_tile_scan<<<tiles, TILE, 0, st>>>(in, n, offsets, out);
}

}  // namespace

bool gpu_bvh_available() {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) {
    cudaGetLastError();
    return false;
  }
  return true;
}

// Builds the BVH of `n` boxes (lo xyz, hi xyz each) with leaves of at most
// `leaf` boxes (at most `most` when the SAH keeps them), on the current device.
// Writes the nodes in preorder and the box order; the caller has checked that no
// coordinate is NaN or -0.0.
void gpu_bvh_build(const float* host_boxes, uint32_t n, uint32_t leaf, uint32_t most, std::vector<GpuNode>& nodes,
                   std::vector<uint32_t>& order_out) {
  nodes.clear();
  order_out.assign(n, 0u);
  if (n == 0) return;
  cudaStream_t st = nullptr;
  cu(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "stream");
  std::vector<void*> owned;
  auto alloc = [&](size_t bytes) {
    void* p = nullptr;
    cu(cudaMalloc(&p, bytes < 16 ? 16 : bytes), "allocation");
    owned.push_back(p);
    return p;
  };
  try {
    float* boxes = static_cast<float*>(alloc((size_t)n * 24));
    float* cen = static_cast<float*>(alloc((size_t)n * 12));
    uint32_t* order = static_cast<uint32_t*>(alloc((size_t)n * 4));
    uint32_t* placed = static_cast<uint32_t*>(alloc((size_t)n * 4));
    uint32_t* seg = static_cast<uint32_t*>(alloc((size_t)n * 4));
    uint32_t* pass = static_cast<uint32_t*>(alloc((size_t)n * 4));
    uint32_t* fail = static_cast<uint32_t*>(alloc((size_t)n * 4));
    uint32_t* pass_scan = static_cast<uint32_t*>(alloc((size_t)n * 4));
    uint32_t* fail_scan = static_cast<uint32_t*>(alloc((size_t)n * 4));
    uint32_t* P = static_cast<uint32_t*>(alloc((size_t)n * 4));
    uint32_t* Q = static_cast<uint32_t*>(alloc((size_t)n * 4));
    uint32_t* counter = static_cast<uint32_t*>(alloc(16));
    std::vector<uint32_t*> scratch;
    for (uint32_t m = (n + TILE - 1) / TILE; ; m = (m + TILE - 1) / TILE) {
      scratch.push_back(static_cast<uint32_t*>(alloc((size_t)m * 4)));
      scratch.push_back(static_cast<uint32_t*>(alloc((size_t)m * 4)));
      if (m <= 1) break;
    }
    // a level never holds more nodes than elements; the first holds the root
    size_t most_nodes = n;
    LNode* level_a = static_cast<LNode*>(alloc(most_nodes * sizeof(LNode)));
    LNode* level_b = static_cast<LNode*>(alloc(most_nodes * sizeof(LNode)));
    Acc* acc = static_cast<Acc*>(alloc(most_nodes * sizeof(Acc)));
    cu(cudaMemcpyAsync(boxes, host_boxes, (size_t)n * 24, cudaMemcpyHostToDevice, st), "upload");
    k_prepare<<<grid_for(n, BLOCK), BLOCK, 0, st>>>(boxes, n, cen, order, seg);
    LNode root{0u, n, NONE, 0u};
    cu(cudaMemcpyAsync(level_a, &root, sizeof(root), cudaMemcpyHostToDevice, st), "root");
    cu(cudaMemsetAsync(counter, 0, 16, st), "counters");
    // every level's decisions, kept for the preorder numbering
    std::vector<Decision*> decisions;
    std::vector<uint32_t> counts;
    uint32_t count = 1;
    LNode* level = level_a;
    LNode* next = level_b;
    BinAcc* bins = nullptr;
    size_t bins_cap = 0;
    while (count > 0) {
      if (count > bins_cap) {
        bins_cap = std::max<size_t>(count, 2 * bins_cap);
        bins = static_cast<BinAcc*>(alloc(bins_cap * sizeof(BinAcc)));
      }
      Decision* dec = static_cast<Decision*>(alloc((size_t)count * sizeof(Decision)));
      decisions.push_back(dec);
      counts.push_back(count);
      k_init_level<<<grid_for(count, BLOCK), BLOCK, 0, st>>>(acc, bins, count);
      k_bounds<<<grid_for(n, BLOCK), BLOCK, 0, st>>>(boxes, cen, order, seg, n, acc);
      k_bins<<<grid_for(n, BLOCK * 4), BLOCK, 0, st>>>(boxes, cen, order, seg, level, acc, n, leaf, bins);
      cu(cudaMemsetAsync(counter, 0, 4, st), "counter");  // counter[1]: the error word, kept across levels
      k_decide<<<grid_for(count, 128), 128, 0, st>>>(level, acc, bins, count, leaf, most, dec, counter);
      k_flags<<<grid_for(n, BLOCK), BLOCK, 0, st>>>(cen, order, seg, acc, dec, n, pass, fail);
      scan(pass, n, pass_scan, scratch, 0, st);
      scan(fail, n, fail_scan, scratch, 0, st);
      k_ranks<<<grid_for(n, BLOCK), BLOCK, 0, st>>>(seg, dec, level, pass, pass_scan, fail_scan, n, P, Q);
      k_place<<<grid_for(n, BLOCK), BLOCK, 0, st>>>(seg, dec, level, pass, pass_scan, fail_scan, P, Q, order, n,
                                                     placed, counter + 1);
      k_copy_placed<<<grid_for(n, BLOCK), BLOCK, 0, st>>>(seg, dec, placed, n, order);
      k_children<<<grid_for(count, BLOCK), BLOCK, 0, st>>>(level, dec, count, next);
      k_segments<<<grid_for(n, BLOCK), BLOCK, 0, st>>>(seg, dec, n);
      cu(cudaGetLastError(), "level");
      uint32_t words[2] = {0, 0};
      cu(cudaMemcpyAsync(words, counter, 8, cudaMemcpyDeviceToHost, st), "level count");
      cu(cudaStreamSynchronize(st), "level");
      if (words[1] != 0u) throw std::runtime_error("GPU BVH build: a partition placed an element out of range");
      uint32_t next_count = words[0];
      std::swap(level, next);
      count = next_count;
    }
    // preorder numbering on the host from the decisions (a few bytes per node)
    size_t levels = decisions.size();
    std::vector<std::vector<Decision>> dec_host(levels);
    for (size_t l = 0; l < levels; ++l) {
      dec_host[l].resize(counts[l]);
      cu(cudaMemcpyAsync(dec_host[l].data(), decisions[l], counts[l] * sizeof(Decision), cudaMemcpyDeviceToHost, st),
         "decisions");
    }
    cu(cudaMemcpyAsync(order_out.data(), order, (size_t)n * 4, cudaMemcpyDeviceToHost, st), "order");
    cu(cudaStreamSynchronize(st), "readback");
    // subtree sizes, bottom-up
    std::vector<std::vector<uint32_t>> size(levels);
    for (size_t l = levels; l-- > 0;) {
      size[l].assign(counts[l], 1u);
      for (uint32_t i = 0; i < counts[l]; ++i) {
        const Decision& d = dec_host[l][i];
        if (!d.leaf) size[l][i] = 1u + size[l + 1][d.left] + size[l + 1][d.right];
      }
    }
    // preorder indices, top-down; ranges follow from the splits
    std::vector<std::vector<uint32_t>> pre(levels), start(levels), end(levels);
    pre[0] = {0u};
    start[0] = {0u};
    end[0] = {n};
    for (size_t l = 0; l + 1 < levels; ++l) {
      pre[l + 1].assign(counts[l + 1], 0u);
      start[l + 1].assign(counts[l + 1], 0u);
      end[l + 1].assign(counts[l + 1], 0u);
      for (uint32_t i = 0; i < counts[l]; ++i) {
        const Decision& d = dec_host[l][i];
        if (d.leaf) continue;
        pre[l + 1][d.left] = pre[l][i] + 1u;
        pre[l + 1][d.right] = pre[l][i] + 1u + size[l + 1][d.left];
        start[l + 1][d.left] = start[l][i];
        end[l + 1][d.left] = d.mid;
        start[l + 1][d.right] = d.mid;
        end[l + 1][d.right] = end[l][i];
      }
    }
    nodes.assign(size[0][0], GpuNode{});
    for (size_t l = 0; l < levels; ++l)
      for (uint32_t i = 0; i < counts[l]; ++i) {
        const Decision& d = dec_host[l][i];
        GpuNode g{};
        for (int k = 0; k < 3; ++k) {
          g.lo[k] = d.lo[k];
          g.hi[k] = d.hi[k];
        }
        if (d.leaf) {
          g.first = start[l][i];
          g.count = end[l][i] - start[l][i];
        } else {
          g.first = pre[l + 1][d.right];
          g.count = 0u;
        }
        nodes[pre[l][i]] = g;
      }
  } catch (...) {
    for (void* p : owned) cudaFree(p);
    cudaStreamDestroy(st);
    throw;
  }
  for (void* p : owned) cudaFree(p);
  cudaStreamDestroy(st);
}

}  // namespace pfxt
