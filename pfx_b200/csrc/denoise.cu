// The denoiser on sm_100a: OIDN's RT filter as the reference's crates/denoise
// runs it (lib.rs, net.rs, tile.rs, process.wgsl, wgsl.rs), with the U-Net's
// 3x3 convolutions as implicit GEMMs on the 5th-generation tensor cores.
//
// Layout.  A tensor of the U-Net is FP32, channels last, [y][x][C] with C
// padded to a multiple of 16, at its level's size (the tile's size >> level).
// A convolution is a GEMM per tile of R = 4 output rows x 128 pixels: M = the
// 128 pixels of a row, N = the output channels, K = 9 taps x the input
// channels, walked in chunks of 16 input channels.  For a chunk, the R + 2
// input rows x 130 pixels (one pixel of border each side) are staged in shared
// memory in the no-swizzle K-major canonical layout, pixel after pixel
// (16 bytes = 8 channels per row of a core matrix), so the A operand of tap
// (ky, kx) for output row r is the same bytes at a start address moved by
// (r + ky) rows and kx pixels: no data moves per tap.  The chunk's weights
// (9 taps x 16 channels x N) are one contiguous block, staged by one bulk
// copy (TMA, no multicast).  One thread issues tcgen05.mma.kind::f16 (M =
// 128, K = 16) into R accumulators in TMEM (columns 128 r), and the next
// chunk is staged while those MMAs run (two stages).
//
// Precision.  The reference computes in FP32 (weights are FP16 in the blob,
// exact in FP32).  Each staged activation is split into hi = fp16(a) and lo =
// fp16(a - hi), and both are multiplied by the FP16 weights with FP32
// accumulation, so an activation keeps ~22 significant bits; the products
// are exact, and the sums round in FP32 as the reference's do (in another
// order).  Weights that are not exact in FP16 are refused.
//
// Epilogue.  tcgen05.ld per 16 columns, bias, ReLU; a pooling layer takes the
// max of its two rows in the thread and of the neighbouring pixel's lane by
// a shuffle (max pooling after ReLU = ReLU after max pooling).  Upsampling and
// concatenation are in the staging: channels of the first source are read at
// (y / 2, x / 2) of the half-size tensor, the skip source's at (y, x).
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <thread>

#include "denoise.h"
#include "pfxt_internal.h"
#include "tracer.h"
#include "umma.cuh"

namespace pfxt {

namespace {

void dcheck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw DeviceError(std::string(what) + ": " + cudaGetErrorString(e));
}

// ------------------------------------------------------------------ weights blob
constexpr const char* CORRUPT = "invalid or corrupted weights blob";

struct Tensor {
  std::vector<uint32_t> dims;
  std::vector<float> data;
  std::vector<uint16_t> half;  // the FP16 bits of every value (exact)
  bool exact_half = true;
};

struct Reader {
  const uint8_t* bytes;
  size_t size, at;
  const uint8_t* take(size_t count) {
    if (at > size || count > size - at) throw Invalid(CORRUPT);
    const uint8_t* p = bytes + at;
    at += count;
    return p;
  }
  template <class T>
  T get() {
    T v;
    memcpy(&v, take(sizeof(T)), sizeof(T));
    return v;
  }
};

float half_bits_to_float(uint16_t h) { return __half2float(__ushort_as_half(h)); }

// OIDN's tensor archive, version 2 (tza.rs:51-118; OIDN core/tza.cpp): magic
// 0x41D7, major version 2, the table's offset; per tensor its name, dims,
// layout ("x" or "oihw"), type ('f' or 'h') and data offset.
std::map<std::string, Tensor> parse_tza(const uint8_t* bytes, size_t size) {
  Reader head{bytes, size, 0};
  if (head.get<uint16_t>() != 0x41D7u) throw Invalid(CORRUPT);
  uint8_t major = head.get<uint8_t>();
  head.get<uint8_t>();
  if (major != 2) throw Invalid("unsupported weights blob version");
  uint64_t table = head.get<uint64_t>();
  if (table > size) throw Invalid(CORRUPT);
  Reader in{bytes, size, (size_t)table};
  uint32_t count = in.get<uint32_t>();
  std::map<std::string, Tensor> out;
  for (uint32_t i = 0; i < count; ++i) {
    uint16_t name_len = in.get<uint16_t>();
    const uint8_t* name = in.take(name_len);
    uint8_t rank = in.get<uint8_t>();
    Tensor t;
    uint64_t elements = 1;
    for (uint8_t r = 0; r < rank; ++r) {
      uint32_t dim = in.get<uint32_t>();
      if (dim == 0 || dim > (1u << 30)) throw Invalid("invalid tensor dimension");
      t.dims.push_back(dim);
      elements *= dim;
      if (elements > (1ull << 32)) throw Invalid(CORRUPT);
    }
    const uint8_t* layout = in.take(rank);
    bool x = rank == 1 && layout[0] == 'x';
    bool oihw = rank == 4 && memcmp(layout, "oihw", 4) == 0;
    if (!x && !oihw) throw Invalid("invalid tensor layout");
    uint8_t type = in.get<uint8_t>();
    if (type != 'f' && type != 'h') throw Invalid("invalid tensor data type");
    uint64_t offset = in.get<uint64_t>();
    Reader data{bytes, size, (size_t)offset};
    if (offset > size) throw Invalid(CORRUPT);
    const uint8_t* raw = data.take((size_t)(elements * (type == 'f' ? 4 : 2)));
    t.data.resize(elements);
    t.half.resize(elements);
    for (uint64_t e = 0; e < elements; ++e) {
      if (type == 'h') {
        uint16_t h;
        memcpy(&h, raw + 2 * e, 2);
        t.half[e] = h;
        t.data[e] = half_bits_to_float(h);
      } else {
        float f;
        memcpy(&f, raw + 4 * e, 4);
        t.data[e] = f;
        uint16_t h = __half_as_ushort(__float2half_rn(f));
        t.half[e] = h;
        if (!(half_bits_to_float(h) == f)) t.exact_half = false;
      }
    }
    out.emplace(std::string(reinterpret_cast<const char*>(name), name_len), std::move(t));
  }
  return out;
}

uint32_t pad16(uint32_t c) { return (c + 15u) / 16u * 16u; }

// The weights of one layer as conv kernels stage them: for each chunk of 16
// padded input channels (the first source's padded channels, then the skip
// source's), 9 taps x 2 groups of 8 channels x n output rows x 8 halves,
//   index = (((chunk * 9 + tap) * 2 + group) * n + o) * 8 + j,
// the K-major canonical layout of the B operand of one tap (rows = output
// channels, 16-byte rows of 8 input channels).  Padding is zero.
std::vector<uint16_t> conv_chunks(const DenoiseLayer& L, const Tensor& w) {
  const uint32_t chunks = (L.c0 + L.c1) / 16u, inputs = L.in0 + L.in1;
  std::vector<uint16_t> out((size_t)chunks * 9u * 2u * L.n * 8u, 0u);
  for (uint32_t k = 0; k < chunks; ++k)
    for (uint32_t t = 0; t < 9; ++t)
      for (uint32_t g = 0; g < 2; ++g)
        for (uint32_t o = 0; o < L.out; ++o)
          for (uint32_t j = 0; j < 8; ++j) {
            uint32_t pc = k * 16u + g * 8u + j;
            int64_t ch = -1;
            if (pc < L.c0) {
              if (pc < L.in0) ch = pc;
            } else if (pc - L.c0 < L.in1) {
              ch = L.in0 + (pc - L.c0);
            }
            if (ch < 0) continue;
            out[((((size_t)k * 9u + t) * 2u + g) * L.n + o) * 8u + j] = w.half[((size_t)o * inputs + ch) * 9u + t];
          }
  return out;
}

}  // namespace

// ------------------------------------------------------------------ kernels
namespace {

__host__ __device__ constexpr uint32_t div_ceil(uint32_t a, uint32_t b) { return (a + b - 1u) / b; }

constexpr uint32_t CONV_THREADS = 128;               // 4 warps: the epilogue by TMEM lane quarter
constexpr uint32_t CONV_PIX = 128;                   // pixels per output row (M of the MMA)
constexpr uint32_t PATCH_W = CONV_PIX + 2;           // staged pixels per input row
constexpr uint32_t A_PLANE = PATCH_W * 16u;          // bytes of one (row, group of 8 channels) plane

// The shape of a conv CTA: ROWS output rows (one TMEM accumulator each, NMAX
// columns), STAGES shared-memory stages, CTAS resident CTAs per SM.  In
// k_conv, two CTAs per SM overlap one CTA's epilogue (TMEM to registers to
// HBM) with the other's copies and MMAs, and more stages in one CTA overlap
// only the copies; the persistent k_conv_ws overlaps all three in one CTA.
// The 4K frame (two tiles of 2016x2160), forcing one shape wherever it fits
// (the wide layers, above 64 channels, otherwise on Wide):
//  * k_conv, Tall:   8 rows, up to 64 channels, two stages, one CTA: 10.13 ms;
//  * k_conv, Quad:   4 rows, up to 64 channels, three stages, one CTA: 11.08 ms;
//  * k_conv, Wide:   4 rows, up to 128 channels, two stages, one CTA: 11.07 ms;
//  * k_conv, Paired: 4 rows, up to 64 channels, one stage, two CTAs: 8.82 ms;
//  * k_conv, Tall2:  8 rows, up to 32 channels, one stage, two CTAs (with
//    Paired on the 48 and 64 channel layers): 8.45 ms;
//  * k_conv, Wide2:  2 rows, up to 128 channels, one stage, two CTAs: 10.40 ms;
//  * k_conv_ws, Persist64:  4 rows, up to 64 channels, three stages (then):
//    7.66 ms;
//  * k_conv_ws, Persist32:  8 rows, up to 32 channels, two stages (with
//    Paired on the 48 and 64 channel layers): 7.98 ms;
//  * k_conv_ws, Persist128: 2 rows, up to 128 channels, three stages (then):
//    8.49 ms.
// Layer by layer the persistent shapes are the fastest: Persist32 up to 32
// channels, Persist64 up to 64, Persist128 above (the default), 7.30 ms.
// With the upsampled sources stored at their own size and widened in the
// CTA (EXPAND): 6.66 ms with one raw buffer beside three stages, 6.52 ms
// with two raw buffers beside two stages (the copies of the next chunk's raw
// rows no longer wait for the widening of the last).  Persist32 as 4 rows and
// three stages instead: 6.66 ms against 6.54; as 6 rows and three stages
// (384 of 512 TMEM columns): 6.62 ms, the same image bit for bit.
template <uint32_t ROWS_, uint32_t NMAX_, uint32_t STAGES_, uint32_t CTAS_, bool EXPAND_ = false,
          uint32_t RAWS_ = 1>
struct ConvShape {
  static constexpr uint32_t ROWS = ROWS_, N_MAX = NMAX_, STAGES = STAGES_, CTAS = CTAS_;
  // EXPAND (persistent kernel only): a first source stored at half size is
  // copied into one of RAWS raw buffers of ROWS / 2 + 2 rows x 66 pixels and
  // widened 2x2 into the stage by four more warps.
  static constexpr bool EXPAND = EXPAND_;
  static constexpr uint32_t RAWS = RAWS_;
  static constexpr uint32_t RAW_ROWS = ROWS / 2u + 2u, RAW_W = CONV_PIX / 2u + 2u;
  static constexpr uint32_t RAW_BOX = RAW_ROWS * 2u * RAW_W * 16u;   // one half (hi or lo) as copied
  static constexpr uint32_t RAW_PLANE = (RAW_BOX + 127u) / 128u * 128u;  // its place in shared memory
  static constexpr uint32_t RAW = EXPAND ? RAWS * 2u * RAW_PLANE : 0u;
  static constexpr uint32_t TMEM_COLS = ROWS * N_MAX;            // a power of two of at least 32
  static constexpr uint32_t PATCH_ROWS = ROWS + 2u;              // staged input rows
  static constexpr uint32_t A_BYTES = PATCH_ROWS * 2u * A_PLANE;   // one chunk of one half (hi or lo)
  static constexpr uint32_t W_MAX = 9u * 2u * N_MAX * 16u;         // one chunk of weights at N_MAX
  static constexpr uint32_t STAGE = 2u * A_BYTES + W_MAX;
  static constexpr uint32_t RAW_AT = STAGES * STAGE;               // the raw buffer
  static constexpr uint32_t CTRL = RAW_AT + RAW;                   // mbarriers, TMEM slot, flags
  static constexpr uint32_t SMEM = CTRL + 256u;
  static_assert(SMEM * CTAS <= 228u * 1024u - CTAS * 1024u, "shared memory per SM");
  static_assert(TMEM_COLS * CTAS <= 512u && (TMEM_COLS & (TMEM_COLS - 1u)) == 0u, "TMEM per SM");
  static_assert(STAGES >= 1u && STAGES <= 4u && RAWS >= 1u && RAWS <= 2u, "one to four stages, one or two raw buffers");
  // a tensor copy's shared-memory destination is 128-byte aligned
  static_assert(STAGE % 128u == 0u && A_BYTES % 128u == 0u && RAW_AT % 128u == 0u && RAW_PLANE % 128u == 0u,
                "copy destinations");
};
using Wide = ConvShape<4, 128, 2, 1>;
using Tall = ConvShape<8, 64, 2, 1>;
using Quad = ConvShape<4, 64, 3, 1>;
using Paired = ConvShape<4, 64, 1, 2>;
using Tall2 = ConvShape<8, 32, 1, 2>;
using Wide2 = ConvShape<2, 128, 1, 2>;
// the persistent kernel's shapes (two accumulators: 2 x ROWS x N_MAX TMEM columns)
using Persist64 = ConvShape<4, 64, 2, 1, true, 2>;
using Persist32 = ConvShape<8, 32, 2, 1>;
using Persist128 = ConvShape<2, 128, 2, 1, true, 2>;
constexpr uint32_t ERR_CONV_WAIT = 1u, ERR_CONV_DRAIN = 2u;
// Polls of the waits that drain a CTA's own work in flight (its MMAs and
// copies) before it frees its TMEM and leaves, whatever the main loop's
// limit: work this kernel issued itself always completes.
constexpr uint32_t DRAIN_LIMIT = 1u << 26;

// Instruction descriptor of kind::f16 with FP16 A and B and an FP32 accumulator, K-major operands.
__host__ __device__ constexpr uint32_t idesc_f16(uint32_t M, uint32_t N) {
  return (1u << 4) | ((N >> 3) << 17) | ((M >> 4) << 24);
}

// A tensor of the U-Net: two FP16 planes, hi = fp16(v) and lo = fp16(v - hi),
// each [y][channel group of 8][x][8 halves] at its stored size; the planes
// are the operand layout of the convolutions (16 bytes = 8 channels of one
// pixel, pixels contiguous), so a chunk's rows reach shared memory as they are.
struct ConvArgs {
  CUtensorMap a0_hi, a0_lo;   // the first source (at this layer's level, or at half of it when half0)
  CUtensorMap a1_hi, a1_lo;   // the skip source (c1 = 0: none)
  const uint16_t* weights;    // conv_chunks() layout
  const float* bias;          // n
  uint16_t* dst_hi;           // the output planes
  uint16_t* dst_lo;
  uint32_t H, W, c0, c1, n, pool;
  uint32_t up;                // the output is stored at twice its size (its consumer upsamples it)
  uint32_t half0;             // the first source is stored at half this layer's size: the CTA widens it
                              // (k_conv_ws with an EXPAND shape; its maps' boxes are RAW_ROWS x RAW_W)
  uint32_t* error;
  uint32_t wait_limit;        // polls of a bounded mbarrier wait
};

__device__ __forceinline__ uint32_t pack_half2(__half a, __half b) {
  return (uint32_t)__half_as_ushort(a) | ((uint32_t)__half_as_ushort(b) << 16);
}

// Eight channel values of one pixel into the two planes at `at` (halves).
__device__ __forceinline__ void store_split8(uint16_t* hi, uint16_t* lo, size_t at, const float* v) {
  uint32_t h[4], l[4];
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    __half h0 = __float2half_rn(v[2 * c]), h1 = __float2half_rn(v[2 * c + 1]);
    __half l0 = __float2half_rn(v[2 * c] - __half2float(h0)), l1 = __float2half_rn(v[2 * c + 1] - __half2float(h1));
    h[c] = pack_half2(h0, h1);
    l[c] = pack_half2(l0, l1);
  }
  *reinterpret_cast<uint4*>(hi + at) = make_uint4(h[0], h[1], h[2], h[3]);
  *reinterpret_cast<uint4*>(lo + at) = make_uint4(l[0], l[1], l[2], l[3]);
}

// The epilogue: warp w reads TMEM lanes 32 w.. (pixels x0 + 32 w + lane) of
// every accumulator, 16 columns at a time; bias and ReLU; a pooling layer
// takes the max of its row pair in the thread and of the neighbouring lane
// (max pooling after ReLU = ReLU after max pooling); the result is written as
// its hi/lo planes, four times over (2x2) when the output is stored upsampled.
template <class S>
__device__ __forceinline__ void conv_epilogue(const ConvArgs& a, uint32_t tmem, uint32_t warp, uint32_t lane,
                                              uint32_t x0, uint32_t y0) {
  const uint32_t x = x0 + warp * 32u + lane;
  const uint32_t G = a.n >> 3;
#pragma unroll 1
  for (uint32_t r0 = 0; r0 < S::ROWS; r0 += 2u) {
#pragma unroll 1
    for (uint32_t j = 0; j < a.n; j += 16u) {
      float v0[16], v1[16];
      umma::ld16(umma::taddr(tmem, warp * 32u, r0 * S::N_MAX + j), v0);
      umma::ld16(umma::taddr(tmem, warp * 32u, (r0 + 1u) * S::N_MAX + j), v1);
      float b[16];
#pragma unroll
      for (int c = 0; c < 16; ++c) b[c] = __ldg(a.bias + j + c);
      if (a.pool) {
        float m[16];
#pragma unroll
        for (int c = 0; c < 16; ++c) {
          m[c] = fmaxf(v0[c], v1[c]);
          m[c] = fmaxf(m[c], __shfl_xor_sync(0xffffffffu, m[c], 1));
          m[c] = fmaxf(m[c] + b[c], 0.0f);
        }
        const uint32_t oy = (y0 + r0) >> 1, ox = x >> 1, OH = a.H >> 1, OW = a.W >> 1;
        if ((lane & 1u) == 0u && oy < OH && ox < OW) {
          store_split8(a.dst_hi, a.dst_lo, (((size_t)oy * G + (j >> 3)) * OW + ox) * 8u, m);
          store_split8(a.dst_hi, a.dst_lo, (((size_t)oy * G + (j >> 3) + 1u) * OW + ox) * 8u, m + 8);
        }
      } else {
#pragma unroll
        for (uint32_t rr = 0; rr < 2; ++rr) {
          const uint32_t y = y0 + r0 + rr;
          float v[16];
#pragma unroll
          for (int c = 0; c < 16; ++c) v[c] = fmaxf((rr ? v1[c] : v0[c]) + b[c], 0.0f);
          if (y < a.H && x < a.W) {
            if (!a.up) {
              store_split8(a.dst_hi, a.dst_lo, (((size_t)y * G + (j >> 3)) * a.W + x) * 8u, v);
              store_split8(a.dst_hi, a.dst_lo, (((size_t)y * G + (j >> 3) + 1u) * a.W + x) * 8u, v + 8);
            } else {
              const uint32_t W2 = 2u * a.W;
#pragma unroll
              for (uint32_t q = 0; q < 4; ++q) {
                const size_t Y = 2u * y + (q >> 1), X = 2u * x + (q & 1u);
                store_split8(a.dst_hi, a.dst_lo, ((Y * G + (j >> 3)) * W2 + X) * 8u, v);
                store_split8(a.dst_hi, a.dst_lo, ((Y * G + (j >> 3) + 1u) * W2 + X) * 8u, v + 8);
              }
            }
          }
        }
      }
    }
  }
}

// One 3x3 convolution (+ bias, ReLU, and 2x2 max pooling when a.pool) of a
// tile of ROWS rows x 128 pixels.  Grid: (ceil(W / 128), ceil(H / ROWS)).
// Lane 0 of warp 0 copies each chunk of 16 input channels into a stage: the
// hi and lo planes' boxes of 8 halves x 130 pixels x 2 groups x (ROWS + 2)
// rows from the source's tensor maps (zeros outside the tensor: the
// convolution's padding), and the chunk's weights by a bulk copy, all on the
// stage's `full` barrier; lane 0 of warp 1 issues the chunk's MMAs once it is
// full, and their commit frees the stage.  Every wait is bounded: a wait that
// runs out stops the CTA's pipeline (the other lane's waits then run out too),
// the CTA drains what it issued and reports it in a.error.
template <class S>
__global__ void __launch_bounds__(CONV_THREADS, S::CTAS) k_conv(const __grid_constant__ ConvArgs a) {
  constexpr uint32_t STAGE = S::STAGE, A_BYTES = S::A_BYTES, CTRL = S::CTRL, N_MAX = S::N_MAX, ROWS = S::ROWS;
  constexpr uint32_t NS = S::STAGES, TMEM_COLS = S::TMEM_COLS;
  extern __shared__ __align__(1024) uint8_t smem[];
  const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31u;
  const uint32_t x0 = blockIdx.x * CONV_PIX, y0 = blockIdx.y * ROWS;
  const uint32_t base = umma::smem_addr(smem);
  const uint32_t full0 = base + CTRL, done0 = base + CTRL + 32u;  // NS barriers of 8 bytes each
  uint32_t* slot = reinterpret_cast<uint32_t*>(smem + CTRL + 64u);
  volatile uint32_t* abort_flag = reinterpret_cast<volatile uint32_t*>(smem + CTRL + 68u);
  uint32_t* counts = reinterpret_cast<uint32_t*>(smem + CTRL + 72u);  // [0] chunks committed, [1] chunks loaded
  if (tid == 0) {
    for (uint32_t s = 0; s < NS; ++s) {
      umma::mbar_init(full0 + 8u * s, 1);
      umma::mbar_init(done0 + 8u * s, 1);
    }
    *abort_flag = 0u;
    counts[0] = counts[1] = 0u;
  }
  if (warp == 0) umma::tmem_alloc(slot, TMEM_COLS);
  umma::fence_before();
  __syncthreads();
  umma::fence_after();
  const uint32_t tmem = *slot;
  const uint32_t chunks = (a.c0 + a.c1) >> 4, chunks0 = a.c0 >> 4;
  const uint32_t wbytes = 9u * 2u * a.n * 16u;
  if (tid == 0) {  // the copies
    uint32_t loads = 0;
    for (uint32_t k = 0; k < chunks; ++k) {
      const uint32_t s = k % NS;
      if (k >= NS && !umma::mbar_wait(done0 + 8u * s, ((k - NS) / NS) & 1u, a.wait_limit)) {
        *abort_flag = 1u;
        break;
      }
      if (*abort_flag) break;
      const uint32_t st = base + s * STAGE, full = full0 + 8u * s;
      umma::mbar_expect_tx(full, 2u * A_BYTES + wbytes);
      const bool first = k < chunks0;
      const int g = (int)(2u * (first ? k : k - chunks0));
      umma::tensor_load_4d(st, first ? &a.a0_hi : &a.a1_hi, 0, (int)x0 - 1, g, (int)y0 - 1, full);
      umma::tensor_load_4d(st + A_BYTES, first ? &a.a0_lo : &a.a1_lo, 0, (int)x0 - 1, g, (int)y0 - 1, full);
      umma::bulk_load(st + 2u * A_BYTES, a.weights + (size_t)k * (wbytes / 2u), wbytes, full);
      loads = k + 1u;
    }
    counts[1] = loads;
  } else if (tid == 32) {  // the MMAs
    const uint32_t id = idesc_f16(128, a.n);
    uint32_t issued = 0;
    for (uint32_t k = 0; k < chunks; ++k) {
      const uint32_t s = k % NS;
      if (!umma::mbar_wait(full0 + 8u * s, (k / NS) & 1u, a.wait_limit) || *abort_flag) {
        *abort_flag = 1u;
        break;
      }
      umma::fence_after();
      // Descriptors move with their start address (bits 0-13, address / 16; a
      // shared-memory address stays below 2^18, so adding to it never carries
      // into the other fields): one base descriptor per operand, offsets known
      // at compile time, so the lane issues ROWS x 18 MMAs back to back.
      const uint64_t hi_desc = umma::desc(base + s * STAGE, A_PLANE, 128u);
      const uint64_t lo_desc = umma::desc(base + s * STAGE + A_BYTES, A_PLANE, 128u);
      const uint64_t w_desc = umma::desc(base + s * STAGE + 2u * A_BYTES, a.n * 16u, 128u);
      const uint32_t w_step = (2u * a.n * 16u) >> 4;
      const uint32_t first = k == 0 ? 0u : 1u;
#pragma unroll
      for (uint32_t r = 0; r < ROWS; ++r) {
#pragma unroll
        for (uint32_t tap = 0; tap < 9; ++tap) {
          const uint32_t off = ((r + tap / 3u) * 2u * A_PLANE + (tap % 3u) * 16u) / 16u;
          const uint64_t bd = w_desc + tap * w_step;
          umma::mma(tmem + r * N_MAX, hi_desc + off, bd, id, tap > 0 ? 1u : first);
          umma::mma(tmem + r * N_MAX, lo_desc + off, bd, id, 1u);
        }
      }
      umma::commit(done0 + 8u * s);
      issued = k + 1u;
    }
    counts[0] = issued;
  }
  __syncthreads();
  const uint32_t issued = counts[0], loads = counts[1];
  const bool late = *abort_flag != 0u;
  // every MMA issued is done when the last commit's phase completes; copies
  // whose MMAs were never issued land before the CTA leaves
  bool drained = true;
  if (issued > 0) drained = umma::mbar_wait(done0 + 8u * ((issued - 1u) % NS), ((issued - 1u) / NS) & 1u, DRAIN_LIMIT);
  for (uint32_t k = issued; k < loads; ++k)
    drained = umma::mbar_wait(full0 + 8u * (k % NS), (k / NS) & 1u, DRAIN_LIMIT) && drained;
  drained = __syncthreads_and(drained);
  umma::fence_after();
  if (late || !drained) {
    if (tid == 0) atomicOr(a.error, (late ? ERR_CONV_WAIT : 0u) | (drained ? 0u : ERR_CONV_DRAIN));
  } else {
    conv_epilogue<S>(a, tmem, warp, lane, x0, y0);
  }
  umma::fence_before();
  __syncthreads();
  if (drained && warp == 0) umma::tmem_free(tmem, TMEM_COLS);
}

// The persistent form of k_conv: one CTA per SM walks the layer's tiles
// (tile t: pixels 128 (t % gx).., rows ROWS (t / gx)..) in steps of gridDim.x.
// Lane 0 of warp 0 streams every tile's chunks through the NS-stage ring;
// lane 0 of warp 1 issues each tile's MMAs into one of two TMEM accumulators
// (tiles alternate) and commits it to the accumulator's `full` barrier; warps
// 2-5 (TMEM lane quarters 2, 3, 0, 1) run the epilogue of one accumulator while
// the MMAs of the next tile fill the other, and free it on its `empty`
// barrier (one arrival per warp).  With an EXPAND shape and a first source
// stored at half size (a.half0), that source's chunks are copied into a raw
// buffer of RAW_ROWS x RAW_W pixels, and warps 6-9 widen it 2x2 into the
// stage (patch pixel p of row r reads raw pixel floor((x0 - 1 + p) / 2) -
// floor((x0 - 1) / 2) of raw row floor((y0 - 1 + r) / 2) - floor((y0 - 1) / 2)),
// then release the raw buffer (`raw empty`) and tell the MMA lane (the
// stage's `widened` barrier).  The stage's own `full` barrier then counts the
// weights alone.  Waits are bounded as in k_conv.
template <class S>
constexpr uint32_t ws_threads() {
  return S::EXPAND ? 320u : 192u;
}
template <class S>
__global__ void __launch_bounds__(ws_threads<S>(), 1) k_conv_ws(const __grid_constant__ ConvArgs a) {
  constexpr uint32_t STAGE = S::STAGE, A_BYTES = S::A_BYTES, CTRL = S::CTRL, N_MAX = S::N_MAX, ROWS = S::ROWS;
  constexpr uint32_t NS = S::STAGES, ACC = ROWS * N_MAX, TMEM_COLS = 2u * ACC;
  constexpr uint32_t RAW_PLANE = S::RAW_PLANE, RAW_W = S::RAW_W;
  static_assert(TMEM_COLS <= 512u, "two accumulators in the TMEM of one SM");
  extern __shared__ __align__(1024) uint8_t smem[];
  const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31u;
  const uint32_t base = umma::smem_addr(smem);
  const uint32_t full0 = base + CTRL, empty0 = base + CTRL + 32u;  // NS barriers each
  const uint32_t accf0 = base + CTRL + 64u, acce0 = base + CTRL + 80u;  // two each
  uint32_t* slot = reinterpret_cast<uint32_t*>(smem + CTRL + 96u);
  volatile uint32_t* abort_flag = reinterpret_cast<volatile uint32_t*>(smem + CTRL + 100u);
  // [0] chunks loaded, [1] chunks committed, [2] raw copies issued, [3] raw copies widened
  uint32_t* counts = reinterpret_cast<uint32_t*>(smem + CTRL + 104u);
  const uint32_t wide0 = base + CTRL + 128u;  // NS barriers: the stage's widened source
  const uint32_t raw_full0 = base + CTRL + 160u, raw_empty0 = base + CTRL + 176u;  // RAWS barriers each
  constexpr uint32_t RAWS = S::RAWS;
  const bool half0 = S::EXPAND && a.half0 != 0u;
  if (tid == 0) {
    for (uint32_t s = 0; s < NS; ++s) {
      umma::mbar_init(full0 + 8u * s, 1);
      umma::mbar_init(empty0 + 8u * s, 1);
      umma::mbar_init(wide0 + 8u * s, 4);
    }
    for (uint32_t b = 0; b < 2u; ++b) {
      umma::mbar_init(accf0 + 8u * b, 1);
      umma::mbar_init(acce0 + 8u * b, 4);
    }
    for (uint32_t j = 0; j < RAWS; ++j) {
      umma::mbar_init(raw_full0 + 8u * j, 1);
      umma::mbar_init(raw_empty0 + 8u * j, 4);
    }
    *abort_flag = 0u;
    counts[0] = counts[1] = counts[2] = counts[3] = 0u;
  }
  if (warp == 0) umma::tmem_alloc(slot, TMEM_COLS);
  umma::fence_before();
  __syncthreads();
  umma::fence_after();
  const uint32_t tmem = *slot;
  const uint32_t gx = div_ceil(a.W, CONV_PIX), tiles = gx * div_ceil(a.H, ROWS);
  const uint32_t chunks = (a.c0 + a.c1) >> 4, chunks0 = a.c0 >> 4;
  const uint32_t wbytes = 9u * 2u * a.n * 16u;
  if (tid == 0) {  // the copies
    uint32_t c = 0, u = 0;  // chunks, raw copies
    for (uint32_t t = blockIdx.x; t < tiles && !*abort_flag; t += gridDim.x) {
      const int x0 = (int)((t % gx) * CONV_PIX), y0 = (int)((t / gx) * ROWS);
      for (uint32_t k = 0; k < chunks; ++k, ++c) {
        const uint32_t s = c % NS;
        if (c >= NS && !umma::mbar_wait(empty0 + 8u * s, ((c - NS) / NS) & 1u, a.wait_limit)) *abort_flag = 1u;
        if (*abort_flag) break;
        const uint32_t st = base + s * STAGE, full = full0 + 8u * s;
        const bool first = k < chunks0;
        const int g = (int)(2u * (first ? k : k - chunks0));
        if (half0 && first) {
          // raw buffer u % RAWS is free once the widening warps are done with copy u - RAWS
          const uint32_t j = u % RAWS, raw_full = raw_full0 + 8u * j;
          if (u >= RAWS && !umma::mbar_wait(raw_empty0 + 8u * j, ((u - RAWS) / RAWS) & 1u, a.wait_limit))
            *abort_flag = 1u;
          if (*abort_flag) break;
          umma::mbar_expect_tx(full, wbytes);
          umma::mbar_expect_tx(raw_full, 2u * S::RAW_BOX);
          const uint32_t raw = base + S::RAW_AT + j * 2u * RAW_PLANE;
          umma::tensor_load_4d(raw, &a.a0_hi, 0, (x0 >> 1) - 1, g, (y0 >> 1) - 1, raw_full);
          umma::tensor_load_4d(raw + RAW_PLANE, &a.a0_lo, 0, (x0 >> 1) - 1, g, (y0 >> 1) - 1, raw_full);
          counts[2] = ++u;
        } else {
          umma::mbar_expect_tx(full, 2u * A_BYTES + wbytes);
          umma::tensor_load_4d(st, first ? &a.a0_hi : &a.a1_hi, 0, x0 - 1, g, y0 - 1, full);
          umma::tensor_load_4d(st + A_BYTES, first ? &a.a0_lo : &a.a1_lo, 0, x0 - 1, g, y0 - 1, full);
        }
        umma::bulk_load(st + 2u * A_BYTES, a.weights + (size_t)k * (wbytes / 2u), wbytes, full);
        counts[0] = c + 1u;
      }
    }
  } else if (tid == 32) {  // the MMAs
    const uint32_t id = idesc_f16(128, a.n);
    const uint32_t w_step = (2u * a.n * 16u) >> 4;
    uint32_t c = 0, i = 0, wph = 0;  // wph bit s: the parity of stage s's next widening
    for (uint32_t t = blockIdx.x; t < tiles && !*abort_flag; t += gridDim.x, ++i) {
      const uint32_t b = i & 1u, acc = tmem + b * ACC;
      if (i >= 2u && !umma::mbar_wait(acce0 + 8u * b, ((i - 2u) >> 1) & 1u, a.wait_limit)) *abort_flag = 1u;
      if (*abort_flag) break;
      umma::fence_after();
      for (uint32_t k = 0; k < chunks; ++k, ++c) {
        const uint32_t s = c % NS;
        if (!umma::mbar_wait(full0 + 8u * s, (c / NS) & 1u, a.wait_limit)) *abort_flag = 1u;
        if (half0 && k < chunks0 && !*abort_flag) {
          if (!umma::mbar_wait(wide0 + 8u * s, (wph >> s) & 1u, a.wait_limit)) *abort_flag = 1u;
          wph ^= 1u << s;
        }
        if (*abort_flag) break;
        umma::fence_after();
        const uint64_t hi_desc = umma::desc(base + s * STAGE, A_PLANE, 128u);
        const uint64_t lo_desc = umma::desc(base + s * STAGE + A_BYTES, A_PLANE, 128u);
        const uint64_t w_desc = umma::desc(base + s * STAGE + 2u * A_BYTES, a.n * 16u, 128u);
        const uint32_t first = k == 0 ? 0u : 1u;
#pragma unroll
        for (uint32_t r = 0; r < ROWS; ++r) {
#pragma unroll
          for (uint32_t tap = 0; tap < 9; ++tap) {
            const uint32_t off = ((r + tap / 3u) * 2u * A_PLANE + (tap % 3u) * 16u) / 16u;
            const uint64_t bd = w_desc + tap * w_step;
            umma::mma(acc + r * N_MAX, hi_desc + off, bd, id, tap > 0 ? 1u : first);
            umma::mma(acc + r * N_MAX, lo_desc + off, bd, id, 1u);
          }
        }
        umma::commit(empty0 + 8u * s);
        counts[1] = c + 1u;
      }
      if (*abort_flag) break;
      umma::commit(accf0 + 8u * b);
    }
  } else if (warp >= 2u && warp < 6u) {  // the epilogue
    const uint32_t quarter = warp & 3u;
    uint32_t i = 0;
    for (uint32_t t = blockIdx.x; t < tiles; t += gridDim.x, ++i) {
      const uint32_t b = i & 1u;
      const bool ok = umma::mbar_wait(accf0 + 8u * b, (i >> 1) & 1u, a.wait_limit);
      if (__any_sync(0xffffffffu, !ok || *abort_flag)) {
        *abort_flag = 1u;
        break;
      }
      umma::fence_after();
      conv_epilogue<S>(a, tmem + b * ACC, quarter, lane, (t % gx) * CONV_PIX, (t / gx) * ROWS);
      umma::fence_before();
      __syncwarp();
      if (lane == 0) umma::mbar_arrive(acce0 + 8u * b);
    }
  } else if (S::EXPAND && warp >= 6u && half0) {  // the widening of a half-size first source
    constexpr uint32_t ITEMS = 2u * S::PATCH_ROWS * 2u * PATCH_W;  // planes x rows x groups x pixels
    const uint32_t e = tid - 192u;
    uint32_t c = 0, u = 0;
    bool stop = false;
    for (uint32_t t = blockIdx.x; t < tiles && !stop; t += gridDim.x) {
      const int x0 = (int)((t % gx) * CONV_PIX), y0 = (int)((t / gx) * ROWS);
      const int xl = (x0 - 1) >> 1, yl = (y0 - 1) >> 1;  // the raw buffer's first pixel and row
      for (uint32_t k = 0; k < chunks; ++k, ++c) {
        if (k >= chunks0) continue;
        const uint32_t s = c % NS, j = u % RAWS;
        const bool ok = umma::mbar_wait(raw_full0 + 8u * j, (u / RAWS) & 1u, a.wait_limit);
        if (__any_sync(0xffffffffu, !ok || *abort_flag)) {
          *abort_flag = 1u;
          stop = true;
          break;
        }
        uint8_t* st = smem + s * STAGE;
        const uint8_t* raw = smem + S::RAW_AT + j * 2u * RAW_PLANE;
        for (uint32_t item = e; item < ITEMS; item += 128u) {
          const uint32_t p = item % PATCH_W, rest = item / PATCH_W;  // rest = (plane x rows + r) x 2 + group
          const uint32_t grp = rest & 1u, r = (rest >> 1) % S::PATCH_ROWS, plane = (rest >> 1) / S::PATCH_ROWS;
          const uint32_t rl = (uint32_t)(((y0 - 1 + (int)r) >> 1) - yl), pl = (uint32_t)(((x0 - 1 + (int)p) >> 1) - xl);
          const uint4 v = *reinterpret_cast<const uint4*>(raw + plane * RAW_PLANE + ((rl * 2u + grp) * RAW_W + pl) * 16u);
          *reinterpret_cast<uint4*>(st + plane * A_BYTES + (r * 2u + grp) * A_PLANE + p * 16u) = v;
        }
        umma::fence_async_smem();
        __syncwarp();
        if (lane == 0) {
          umma::mbar_arrive(raw_empty0 + 8u * j);
          umma::mbar_arrive(wide0 + 8u * s);
        }
        ++u;
        if (e == 0u) counts[3] = u;
      }
    }
  }
  __syncthreads();
  const uint32_t loads = counts[0], issued = counts[1], raws = counts[2], widened = counts[3];
  const bool late = *abort_flag != 0u;
  // every MMA issued is done when the last chunk's commit completes; copies
  // whose MMAs were never issued land before the CTA leaves (a widened
  // chunk's `full` barrier counts its weights alone), and so does a raw copy
  // that was not widened
  bool drained = true;
  if (issued > 0)
    drained = umma::mbar_wait(empty0 + 8u * ((issued - 1u) % NS), ((issued - 1u) / NS) & 1u, DRAIN_LIMIT);
  for (uint32_t k = issued; k < loads; ++k)
    drained = umma::mbar_wait(full0 + 8u * (k % NS), (k / NS) & 1u, DRAIN_LIMIT) && drained;
  for (uint32_t k = widened; k < raws; ++k)
    drained = umma::mbar_wait(raw_full0 + 8u * (k % RAWS), (k / RAWS) & 1u, DRAIN_LIMIT) && drained;
  drained = __syncthreads_and(drained);
  if ((late || !drained) && tid == 0)
    atomicOr(a.error, (late ? ERR_CONV_WAIT : 0u) | (drained ? 0u : ERR_CONV_DRAIN));
  umma::fence_after();
  if (drained && warp == 0) umma::tmem_free(tmem, TMEM_COLS);
}

// ------------------------------------------------------------------ image processing
constexpr float DN_FLT_MAX = 3.4028234663852886e38f;

__device__ __forceinline__ float nan_to_zero(float v) { return isnan(v) ? 0.0f : v; }

// OIDN's PU transfer function (process.wgsl:45-63; OIDN devices/gpu/gpu_input_process.h).
__device__ __forceinline__ float pu_forward(float y) {
  if (y <= 1.57945760e-06f) return 1.41283765e+03f * y;
  if (y <= 3.22087631e-02f) return 1.64593172e+00f * powf(y, 4.31384981e-01f) + -2.94139609e-03f;
  return 1.92653254e-01f * logf(y + 6.26026094e-03f) + 9.98620152e-01f;
}
__device__ __forceinline__ float pu_inverse(float x) {
  if (x <= 2.23151711e-03f) return x / 1.41283765e+03f;
  if (x <= 3.70974749e-01f) return powf((x - -2.94139609e-03f) / 1.64593172e+00f, 1.0f / 4.31384981e-01f);
  return expf((x - 9.98620152e-01f) / 1.92653254e-01f) - 6.26026094e-03f;
}

__device__ __forceinline__ float luminance(float4 c) {
  float r = fminf(fmaxf(nan_to_zero(c.x), 0.0f), DN_FLT_MAX), g = fminf(fmaxf(nan_to_zero(c.y), 0.0f), DN_FLT_MAX),
        b = fminf(fmaxf(nan_to_zero(c.z), 0.0f), DN_FLT_MAX);
  return 0.212671f * r + 0.715160f * g + 0.072169f * b;
}

// Autoexposure, step 1 (process.wgsl:108-134): the mean luminance of bin
// (blockIdx.x, blockIdx.y) of a ceil(W/16) x ceil(H/16) split of the image.
__global__ void __launch_bounds__(256) k_exposure_bins(const float4* __restrict__ color, uint32_t W, uint32_t H,
                                                       float* __restrict__ bins) {
  __shared__ float sums[256];
  const uint32_t gx = gridDim.x, gy = gridDim.y;
  const uint32_t bh = blockIdx.y * H / gy, eh = (blockIdx.y + 1u) * H / gy;
  const uint32_t bw = blockIdx.x * W / gx, ew = (blockIdx.x + 1u) * W / gx;
  const uint32_t h = bh + (threadIdx.x >> 4), w = bw + (threadIdx.x & 15u);
  sums[threadIdx.x] = (h < eh && w < ew) ? luminance(color[(size_t)h * W + w]) : 0.0f;
  for (uint32_t i = 128; i > 0; i >>= 1) {
    __syncthreads();
    if (threadIdx.x < i) sums[threadIdx.x] += sums[threadIdx.x + i];
  }
  if (threadIdx.x == 0) bins[blockIdx.y * gx + blockIdx.x] = sums[0] / (float)((eh - bh) * (ew - bw));
}

// Autoexposure, step 2 (process.wgsl:136-157): 0.18 over the geometric mean
// of the bins above 1e-8 (1 when there are none).  One block of 256.
__global__ void __launch_bounds__(256) k_exposure_reduce(const float* __restrict__ bins, uint32_t count,
                                                         float* __restrict__ scale) {
  __shared__ float sums[256];
  __shared__ uint32_t counts[256];
  float sum = 0.0f;
  uint32_t n = 0;
  for (uint32_t i = threadIdx.x; i < count; i += 256u) {
    float l = bins[i];
    if (l > 1e-8f) {
      sum += log2f(l);
      n += 1u;
    }
  }
  sums[threadIdx.x] = sum;
  counts[threadIdx.x] = n;
  for (uint32_t i = 128; i > 0; i >>= 1) {
    __syncthreads();
    if (threadIdx.x < i) {
      sums[threadIdx.x] += sums[threadIdx.x + i];
      counts[threadIdx.x] += counts[threadIdx.x + i];
    }
  }
  if (threadIdx.x == 0) scale[0] = counts[0] > 0u ? 0.18f / exp2f(sums[0] / (float)counts[0]) : 1.0f;
}

struct TileArgs {
  uint32_t src[2], dst[2], size[2], out_src[2], out_dst[2], out_size[2];
  uint32_t tile_h, tile_w, width;
  float norm, rcp_norm;
};

// The tile's input tensor (process.wgsl:65-86): colour times the exposure,
// NaN to 0, clamped, through the PU curve and normalised; albedo clamped to
// [0, 1]; normal clamped to [-1, 1] and mapped to [0, 1]; 9 channels of 16,
// written as the hi/lo planes of the U-Net's tensors (out: hi, out + plane: lo).
__global__ void __launch_bounds__(256) k_input(const __grid_constant__ TileArgs t, const float4* __restrict__ color,
                                               const float4* __restrict__ albedo, const float4* __restrict__ normal,
                                               const float* __restrict__ scale, uint16_t* __restrict__ out) {
  const uint32_t n = t.tile_h * t.tile_w;
  const size_t plane = (size_t)n * 16u;
  const float s = scale[0];
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t y = i / t.tile_w, x = i - y * t.tile_w;
    float v[16] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    const int ix = (int)x - (int)t.dst[1], iy = (int)y - (int)t.dst[0];
    if (ix >= 0 && ix < (int)t.size[1] && iy >= 0 && iy < (int)t.size[0]) {
      const size_t at = (size_t)(iy + t.src[0]) * t.width + (ix + t.src[1]);
      const float4 c = color[at], a = albedo[at], m = normal[at];
      const float cs[3] = {c.x * s, c.y * s, c.z * s}, as[3] = {a.x, a.y, a.z}, ms[3] = {m.x, m.y, m.z};
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        v[k] = pu_forward(fminf(fmaxf(nan_to_zero(cs[k]), 0.0f), DN_FLT_MAX)) * t.norm;
        v[3 + k] = fminf(fmaxf(nan_to_zero(as[k]), 0.0f), 1.0f);
        v[6 + k] = fminf(fmaxf(nan_to_zero(ms[k]), -1.0f), 1.0f) * 0.5f + 0.5f;
      }
    }
    store_split8(out, out + plane, (((size_t)y * 2u) * t.tile_w + x) * 8u, v);
    store_split8(out, out + plane, (((size_t)y * 2u + 1u) * t.tile_w + x) * 8u, v + 8);
  }
}

// The kept part of a tile back into the image (process.wgsl:88-101): the
// network's three channels (hi + lo of its output's first group), NaN to 0,
// clamped, denormalised, through the inverse PU curve and divided by the
// exposure; alpha from the colour.
__global__ void __launch_bounds__(256) k_output(const __grid_constant__ TileArgs t, const uint16_t* __restrict__ net,
                                                uint32_t net_channels, const float4* __restrict__ color,
                                                const float* __restrict__ scale, float4* __restrict__ out) {
  const uint32_t n = t.out_size[0] * t.out_size[1];
  const size_t plane = (size_t)t.tile_h * t.tile_w * net_channels;
  const float s = scale[0];
  const float inv = s != 0.0f ? 1.0f / s : 0.0f;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t gy = i / t.out_size[1], gx = i - gy * t.out_size[1];
    const size_t at = ((size_t)(gy + t.out_src[0]) * (net_channels >> 3) * t.tile_w + gx + t.out_src[1]) * 8u;
    float r[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const float v = __half2float(__ushort_as_half(net[at + k])) + __half2float(__ushort_as_half(net[plane + at + k]));
      r[k] = pu_inverse(fminf(fmaxf(nan_to_zero(v), 0.0f), DN_FLT_MAX) * t.rcp_norm) * inv;
    }
    const size_t o = (size_t)(gy + t.out_dst[0]) * t.width + gx + t.out_dst[1];
    out[o] = make_float4(r[0], r[1], r[2], color[o].w);
  }
}

}  // namespace

// ------------------------------------------------------------------ tiling
// OIDN's tile split (tile.rs:30-95, from UNetFilter::init): the same
// arithmetic, so a frame splits into the reference's tiles.
namespace {
uint32_t round_up(uint32_t a, uint32_t b) { return (a + b - 1u) / b * b; }
uint32_t round_up_rem(uint32_t a, uint32_t b, uint32_t c) { return (a + b - c - 1u) / b * b + c; }
constexpr uint32_t ALIGN = 16, RECEPTIVE_FIELD = 174;
}  // namespace

DenoisePlan denoise_plan(uint32_t h, uint32_t w, uint64_t max_tile_pixels) {
  DenoisePlan p;
  const uint32_t overlap = round_up(RECEPTIVE_FIELD / 2u, ALIGN);
  uint32_t tile_h = round_up(h, ALIGN), tile_w = round_up(w, ALIGN);
  const uint32_t pad_h = tile_h % ALIGN, pad_w = tile_w % ALIGN;
  uint32_t count_h = 1, count_w = 1;
  const uint32_t min_dim = std::max(4u * overlap, 768u);
  const uint32_t min_tile_h = round_up_rem(min_dim, ALIGN, pad_h), min_tile_w = round_up_rem(min_dim, ALIGN, pad_w);
  const uint32_t span_h = 2u * overlap + pad_h, span_w = 2u * overlap + pad_w;
  while ((uint64_t)tile_h * tile_w > max_tile_pixels) {
    if (tile_h > min_tile_h && tile_h > tile_w) {
      uint32_t next = div_ceil(h + span_h * count_h, count_h + 1u);
      tile_h = std::min(std::max(round_up_rem(next, ALIGN, pad_h), min_tile_h), tile_h - ALIGN);
      count_h = std::max(div_ceil(h > span_h ? h - span_h : 0u, tile_h - span_h), 1u);
    } else if (tile_w > min_tile_w) {
      uint32_t next = div_ceil(w + span_w * count_w, count_w + 1u);
      tile_w = std::min(std::max(round_up_rem(next, ALIGN, pad_w), min_tile_w), tile_w - ALIGN);
      count_w = std::max(div_ceil(w > span_w ? w - span_w : 0u, tile_w - span_w), 1u);
    } else {
      break;
    }
  }
  p.tile_h = tile_h;
  p.tile_w = tile_w;
  p.overlap = overlap;
  for (uint32_t i = 0; i < count_h; ++i) {
    uint32_t y = i * (tile_h > span_h ? tile_h - span_h : 0u);
    uint32_t begin_h = i > 0 ? overlap : 0u, end_h = i < count_h - 1u ? overlap + pad_h : 0u;
    uint32_t th1 = std::min(h - y, tile_h), th2 = th1 - begin_h - end_h;
    uint32_t align_h = tile_h - round_up(th1, ALIGN);
    for (uint32_t j = 0; j < count_w; ++j) {
      uint32_t x = j * (tile_w > span_w ? tile_w - span_w : 0u);
      uint32_t begin_w = j > 0 ? overlap : 0u, end_w = j < count_w - 1u ? overlap + pad_w : 0u;
      uint32_t tw1 = std::min(w - x, tile_w), tw2 = tw1 - begin_w - end_w;
      uint32_t align_w = tile_w - round_up(tw1, ALIGN);
      p.tiles.push_back(DenoiseTile{{y, x},
                                    {align_h, align_w},
                                    {th1, tw1},
                                    {align_h + begin_h, align_w + begin_w},
                                    {y + begin_h, x + begin_w},
                                    {th2, tw2}});
    }
  }
  return p;
}

// ------------------------------------------------------------------ host
Denoiser::~Denoiser() {
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(device);
  for (auto& L : layers) {
    if (L.d_weights) cudaFree(L.d_weights);
    if (L.d_bias) cudaFree(L.d_bias);
  }
  for (uint16_t* t : tensors)
    if (t) cudaFree(t);
  if (d_scale) cudaFree(d_scale);
  if (d_bins) cudaFree(d_bins);
  if (d_error) cudaFree(d_error);
  if (ev0) cudaEventDestroy(ev0);
  if (ev1) cudaEventDestroy(ev1);
  if (d_images) cudaFree(d_images);
  if (stream) cudaStreamSynchronize(stream);
  if (h_stage) cudaFreeHost(h_stage);
  for (cudaEvent_t e : stage_ev)
    if (e) cudaEventDestroy(e);
  if (stream) cudaStreamDestroy(stream);
  if (prev >= 0) cudaSetDevice(prev);
}

// The U-Net of net.rs:193-232 over the parsed tensors, its weights uploaded.
Denoiser* denoiser_create(const void* blob, size_t bytes) {
  if (!blob || bytes == 0) throw Invalid(CORRUPT);
  auto tensors = parse_tza(static_cast<const uint8_t*>(blob), bytes);
  std::unique_ptr<Denoiser> d(new Denoiser());
  const uint32_t input_channels = 9;
  auto channels = [&](int src) { return src == -1 ? input_channels : d->layers[src].out; };
  auto padded = [&](int src) { return src == -1 ? pad16(input_channels) : d->layers[src].n; };
  auto level = [&](int src) { return src == -1 ? 0u : d->layers[src].out_level(); };
  auto push = [&](const char* name, int src0, int src1, bool pool) {
    auto w = tensors.find(std::string(name) + ".weight");
    auto b = tensors.find(std::string(name) + ".bias");
    if (w == tensors.end() || b == tensors.end()) throw Invalid(CORRUPT);
    DenoiseLayer L;
    L.name = name;
    L.src0 = src0;
    L.src1 = src1;
    L.pool = pool;
    L.upsample = src1 != -2;
    L.in0 = channels(src0);
    L.in1 = src1 != -2 ? channels(src1) : 0u;
    L.level = src1 != -2 ? level(src1) : level(src0);
    if (L.upsample && level(src0) != L.level + 1u)
      throw Invalid(std::string(name) + ": the upsampled source is not one level down");
    if (w->second.dims.size() != 4 || b->second.dims.size() != 1) throw Invalid("invalid convolution weight/bias");
    L.out = w->second.dims[0];
    if (w->second.dims[1] != L.in0 + L.in1 || w->second.dims[2] != 3 || w->second.dims[3] != 3 ||
        b->second.dims[0] != L.out)
      throw Invalid(std::string(name) + ": the weights do not match the network");
    if (!w->second.exact_half) throw Invalid(std::string(name) + ": weights not exact in half precision");
    L.c0 = padded(src0);
    L.c1 = src1 != -2 ? padded(src1) : 0u;
    L.n = pad16(L.out);
    if (L.n > Wide::N_MAX) throw Invalid(std::string(name) + ": more than 128 output channels");
    L.weights = conv_chunks(L, w->second);
    L.bias.assign(L.n, 0.0f);
    std::copy(b->second.data.begin(), b->second.data.end(), L.bias.begin());
    d->layers.push_back(std::move(L));
    return (int)d->layers.size() - 1;
  };
  int x = push("enc_conv0", -1, -2, false);
  int pool1 = push("enc_conv1", x, -2, true);
  int pool2 = push("enc_conv2", pool1, -2, true);
  int pool3 = push("enc_conv3", pool2, -2, true);
  int pool4 = push("enc_conv4", pool3, -2, true);
  x = push("enc_conv5a", pool4, -2, false);
  x = push("enc_conv5b", x, -2, false);
  x = push("dec_conv4a", x, pool3, false);
  x = push("dec_conv4b", x, -2, false);
  x = push("dec_conv3a", x, pool2, false);
  x = push("dec_conv3b", x, -2, false);
  x = push("dec_conv2a", x, pool1, false);
  x = push("dec_conv2b", x, -2, false);
  x = push("dec_conv1a", x, -1, false);
  x = push("dec_conv1b", x, -2, false);
  push("dec_conv0", x, -2, false);
  if (d->layers.back().out != 3) throw Invalid("the network does not end in three channels");
  // the blob is valid: now the device
  int devices = 0;
  if (cudaGetDeviceCount(&devices) != cudaSuccess || devices == 0) {
    cudaGetLastError();
    throw Refused("no CUDA device");
  }
  dcheck(cudaGetDevice(&d->device), "denoiser device");
  for (auto& L : d->layers) {
    dcheck(cudaMalloc(&L.d_weights, L.weights.size() * 2u), "denoiser weights");
    dcheck(cudaMemcpy(L.d_weights, L.weights.data(), L.weights.size() * 2u, cudaMemcpyHostToDevice),
           "denoiser weights");
    dcheck(cudaMalloc(&L.d_bias, L.bias.size() * 4u), "denoiser bias");
    dcheck(cudaMemcpy(L.d_bias, L.bias.data(), L.bias.size() * 4u, cudaMemcpyHostToDevice), "denoiser bias");
  }
  dcheck(cudaMalloc(&d->d_scale, 16), "denoiser exposure");
  dcheck(cudaMalloc(&d->d_error, 4), "denoiser error word");
  dcheck(cudaMemset(d->d_error, 0, 4), "denoiser error word");
  dcheck(cudaEventCreate(&d->ev0), "denoiser events");
  dcheck(cudaEventCreate(&d->ev1), "denoiser events");
  dcheck(cudaFuncSetAttribute(k_conv<Wide>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Wide::SMEM),
         "convolution shared memory");
  dcheck(cudaFuncSetAttribute(k_conv<Tall>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Tall::SMEM),
         "convolution shared memory");
  dcheck(cudaFuncSetAttribute(k_conv<Quad>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Quad::SMEM),
         "convolution shared memory");
  dcheck(cudaFuncSetAttribute(k_conv<Paired>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Paired::SMEM),
         "convolution shared memory");
  dcheck(cudaFuncSetAttribute(k_conv<Tall2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Tall2::SMEM),
         "convolution shared memory");
  dcheck(cudaFuncSetAttribute(k_conv<Wide2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Wide2::SMEM),
         "convolution shared memory");
  dcheck(cudaFuncSetAttribute(k_conv_ws<Persist64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Persist64::SMEM),
         "convolution shared memory");
  dcheck(cudaFuncSetAttribute(k_conv_ws<Persist32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Persist32::SMEM),
         "convolution shared memory");
  dcheck(cudaFuncSetAttribute(k_conv_ws<Persist128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)Persist128::SMEM),
         "convolution shared memory");
  return d.release();
}

// The plan and the tile tensors for a width x height image (setup.rs:82-156;
// every tensor of a tile has its own buffer).
namespace {
PFN_cuTensorMapEncodeTiled_v12000 encode_tiled() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    dcheck(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q), "tensor map entry point");
    if (q != cudaDriverEntryPointSuccess || !p) throw DeviceError("cuTensorMapEncodeTiled is not available");
    fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

// The tensor map of one plane of a U-Net tensor ([H][C/8][W][8] halves) for
// boxes of 8 halves x 130 pixels x 2 groups x `rows` rows.
CUtensorMap plane_map(const uint16_t* plane, uint32_t H, uint32_t W, uint32_t C, uint32_t rows, bool half = false) {
  CUtensorMap m;
  const cuuint64_t dims[4] = {8u, W, C / 8u, H};
  const cuuint64_t strides[3] = {16u, (cuuint64_t)W * 16u, (cuuint64_t)(C / 8u) * W * 16u};
  // a half-size source is read as the raw box that k_conv_ws widens: RAW_W pixels, rows / 2 + 2 rows
  const cuuint32_t box[4] = {8u, half ? CONV_PIX / 2u + 2u : PATCH_W, 2u, half ? rows / 2u + 2u : rows + 2u};
  const cuuint32_t elem[4] = {1u, 1u, 1u, 1u};
  CUresult r = encode_tiled()(&m, CU_TENSOR_MAP_DATA_TYPE_UINT16, 4, const_cast<uint16_t*>(plane), dims, strides, box,
                              elem, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) throw DeviceError("denoiser tensor map: error " + std::to_string((int)r));
  return m;
}

// The shapes by number (the measurement hook's values): 1 Tall, 2 Quad,
// 3 Wide, 4 Paired, 5 Tall2, 6 Wide2; 7-9 the persistent kernel with
// Persist64, Persist32, Persist128.
constexpr uint32_t SHAPES = 10;
constexpr uint32_t SHAPE_ROWS[SHAPES] = {0,           Tall::ROWS,      Quad::ROWS,      Wide::ROWS,     Paired::ROWS,
                                         Tall2::ROWS, Wide2::ROWS,     Persist64::ROWS, Persist32::ROWS, Persist128::ROWS};
constexpr uint32_t SHAPE_NMAX[SHAPES] = {0,            Tall::N_MAX,      Quad::N_MAX,      Wide::N_MAX,
                                         Paired::N_MAX, Tall2::N_MAX,     Wide2::N_MAX,     Persist64::N_MAX,
                                         Persist32::N_MAX, Persist128::N_MAX};

// Which conv shape a layer runs: the one set for measurement where the
// layer's outputs fit it, else the fastest measured for its output count.
uint32_t shape_of(const Denoiser& d, const DenoiseLayer& L) {
  if (d.conv_shape && d.conv_shape < SHAPES && L.n <= SHAPE_NMAX[d.conv_shape]) return d.conv_shape;
  if (L.n <= Persist32::N_MAX) return 8u;
  if (L.n <= Persist64::N_MAX) return 7u;
  return 9u;
}
uint32_t rows_of(uint32_t shape) { return SHAPE_ROWS[shape]; }
// Whether a shape widens a half-size first source itself (k_conv_ws with an EXPAND shape).
bool widens(uint32_t shape) { return (shape == 7u && Persist64::EXPAND) || (shape == 9u && Persist128::EXPAND); }

struct Launches {
  std::vector<ConvArgs> args;
  std::vector<uint32_t> shapes;
};
}  // namespace

// The plan, the tile tensors and every convolution's arguments for a width x
// height image (setup.rs:82-156; every tensor of a tile has its own buffer).
void denoiser_prepare(Denoiser& d, uint32_t width, uint32_t height) {
  if (width == 0 || height == 0) throw Invalid("image dimensions must be nonzero");
  if (d.width == width && d.height == height) return;
  for (uint16_t* t : d.tensors)
    if (t) cudaFree(t);
  d.tensors.clear();
  d.stored_level.clear();
  d.launches.reset();
  d.width = d.height = 0;
  d.plan = denoise_plan(height, width, d.max_tile_pixels);
  const uint32_t TH = d.plan.tile_h, TW = d.plan.tile_w;
  auto alloc = [&](uint32_t level, uint32_t channels) {
    uint16_t* p = nullptr;
    size_t bytes = 2u * (size_t)(TH >> level) * (TW >> level) * channels * 2u;
    dcheck(cudaMalloc(&p, std::max<size_t>(bytes, 16)), "denoiser tensors");
    d.tensors.push_back(p);
    d.stored_level.push_back(level);
  };
  alloc(0, 16);
  for (size_t i = 0; i < d.layers.size(); ++i) {
    const DenoiseLayer& L = d.layers[i];
    // the first source of an upsampling layer is stored at that layer's size, unless the layer widens it
    bool upsampled = false;
    for (const auto& M : d.layers) upsampled = upsampled || (M.upsample && M.src0 == (int)i && !widens(shape_of(d, M)));
    if (upsampled && L.pool) throw Invalid("a pooled output cannot feed an upsampling layer");
    alloc(upsampled ? L.out_level() - 1u : L.out_level(), L.n);
  }
  auto plane = [&](int src, bool lo) {
    const uint32_t t = (uint32_t)(src + 1);
    const uint32_t lv = d.stored_level[t];
    const uint32_t C = src == -1 ? 16u : d.layers[src].n;
    return d.tensors[t] + (lo ? (size_t)(TH >> lv) * (TW >> lv) * C : 0u);
  };
  auto launches = std::make_shared<Launches>();
  for (size_t i = 0; i < d.layers.size(); ++i) {
    const DenoiseLayer& L = d.layers[i];
    ConvArgs a;
    memset(&a, 0, sizeof(a));
    a.H = TH >> L.level;
    a.W = TW >> L.level;
    const uint32_t shape = shape_of(d, L), rows = rows_of(shape);
    a.half0 = L.upsample && widens(shape) ? 1u : 0u;
    const uint32_t h0 = a.half0 ? a.H / 2u : a.H, w0 = a.half0 ? a.W / 2u : a.W;
    a.a0_hi = plane_map(plane(L.src0, false), h0, w0, L.c0, rows, a.half0 != 0u);
    a.a0_lo = plane_map(plane(L.src0, true), h0, w0, L.c0, rows, a.half0 != 0u);
    if (L.src1 != -2) {
      a.a1_hi = plane_map(plane(L.src1, false), a.H, a.W, L.c1, rows);
      a.a1_lo = plane_map(plane(L.src1, true), a.H, a.W, L.c1, rows);
    }
    a.weights = L.d_weights;
    a.bias = L.d_bias;
    a.dst_hi = plane((int)i, false);
    a.dst_lo = plane((int)i, true);
    a.c0 = L.c0;
    a.c1 = L.c1;
    a.n = L.n;
    a.pool = L.pool ? 1u : 0u;
    a.up = d.stored_level[i + 1] + 1u == L.out_level() ? 1u : 0u;
    a.error = d.d_error;
    launches->args.push_back(a);
    launches->shapes.push_back(shape);
  }
  d.launches = launches;
  size_t bins = (size_t)div_ceil(width, 16) * div_ceil(height, 16);
  if (bins > d.bins_capacity) {
    if (d.d_bins) cudaFree(d.d_bins);
    d.d_bins = nullptr;
    dcheck(cudaMalloc(&d.d_bins, bins * 4u), "denoiser exposure bins");
    d.bins_capacity = bins;
  }
  d.width = width;
  d.height = height;
}

// norm_scales (lib.rs:75-78): the PU value of 65504 and its reciprocal.
static void norm_scales(float& norm, float& rcp_norm) {
  const float max = 1.926'532'5e-1f * std::log(65504.0f + 6.260'261e-3f) + 9.986'201'5e-1f;
  norm = (float)(1.0 / (double)max);
  rcp_norm = max;
}

void denoise_device(Denoiser& d, uint32_t width, uint32_t height, const float4* color, const float4* albedo,
                    const float4* normal, float4* out, cudaStream_t st) {
  if (!color || !albedo || !normal || !out) throw Invalid("null argument");
  dcheck(cudaSetDevice(d.device), "denoiser device");
  denoiser_prepare(d, width, height);
  const DenoisePlan& p = d.plan;
  const Launches& launches = *static_cast<const Launches*>(d.launches.get());
  float norm, rcp_norm;
  norm_scales(norm, rcp_norm);
  int sms = 0;
  dcheck(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, d.device), "device");
  // the persistent kernel's grid: one CTA per SM, or per tile when there are fewer
  auto persistent = [&](const ConvArgs& a, uint32_t rows) {
    return std::min<uint32_t>(div_ceil(a.W, CONV_PIX) * div_ceil(a.H, rows), (uint32_t)sms);
  };
  dcheck(cudaEventRecord(d.ev0, st), "denoiser timing");
  const uint32_t gx = div_ceil(width, 16), gy = div_ceil(height, 16);
  k_exposure_bins<<<dim3(gx, gy), 256, 0, st>>>(color, width, height, d.d_bins);
  k_exposure_reduce<<<1, 256, 0, st>>>(d.d_bins, gx * gy, d.d_scale);
  uint64_t macs = 0;
  for (const DenoiseTile& tile : p.tiles) {
    TileArgs t;
    for (int k = 0; k < 2; ++k) {
      t.src[k] = tile.src[k];
      t.dst[k] = tile.dst[k];
      t.size[k] = tile.size[k];
      t.out_src[k] = tile.out_src[k];
      t.out_dst[k] = tile.out_dst[k];
      t.out_size[k] = tile.out_size[k];
    }
    t.tile_h = p.tile_h;
    t.tile_w = p.tile_w;
    t.width = width;
    t.norm = norm;
    t.rcp_norm = rcp_norm;
    k_input<<<sms * 8, 256, 0, st>>>(t, color, albedo, normal, d.d_scale, d.tensors[0]);
    for (size_t i = 0; i < d.layers.size(); ++i) {
      ConvArgs a = launches.args[i];
      a.wait_limit = d.wait_limit;
      const uint32_t shape = launches.shapes[i];
      if (shape == 1u) {
        k_conv<Tall><<<dim3(div_ceil(a.W, CONV_PIX), div_ceil(a.H, Tall::ROWS)), CONV_THREADS, Tall::SMEM, st>>>(a);
      } else if (shape == 2u) {
        k_conv<Quad><<<dim3(div_ceil(a.W, CONV_PIX), div_ceil(a.H, Quad::ROWS)), CONV_THREADS, Quad::SMEM, st>>>(a);
      } else if (shape == 4u) {
        k_conv<Paired>
            <<<dim3(div_ceil(a.W, CONV_PIX), div_ceil(a.H, Paired::ROWS)), CONV_THREADS, Paired::SMEM, st>>>(a);
      } else if (shape == 5u) {
        k_conv<Tall2><<<dim3(div_ceil(a.W, CONV_PIX), div_ceil(a.H, Tall2::ROWS)), CONV_THREADS, Tall2::SMEM, st>>>(a);
      } else if (shape == 6u) {
        k_conv<Wide2><<<dim3(div_ceil(a.W, CONV_PIX), div_ceil(a.H, Wide2::ROWS)), CONV_THREADS, Wide2::SMEM, st>>>(a);
      } else if (shape == 7u) {
        k_conv_ws<Persist64><<<persistent(a, Persist64::ROWS), ws_threads<Persist64>(), Persist64::SMEM, st>>>(a);
      } else if (shape == 8u) {
        k_conv_ws<Persist32><<<persistent(a, Persist32::ROWS), ws_threads<Persist32>(), Persist32::SMEM, st>>>(a);
      } else if (shape == 9u) {
        k_conv_ws<Persist128><<<persistent(a, Persist128::ROWS), ws_threads<Persist128>(), Persist128::SMEM, st>>>(a);
      } else {
        k_conv<Wide><<<dim3(div_ceil(a.W, CONV_PIX), div_ceil(a.H, Wide::ROWS)), CONV_THREADS, Wide::SMEM, st>>>(a);
      }
      macs += (uint64_t)a.H * a.W * 9u * (a.c0 + a.c1) * a.n;
    }
    k_output<<<sms * 8, 256, 0, st>>>(t, d.tensors.back(), d.layers.back().n, color, d.d_scale, out);
  }
  dcheck(cudaGetLastError(), "denoiser launch");
  dcheck(cudaEventRecord(d.ev1, st), "denoiser timing");
  d.last_macs = macs;
}

// Device time of the last denoise (waits for it) and its error word.
float denoiser_finish(Denoiser& d) {
  dcheck(cudaEventSynchronize(d.ev1), "denoise");
  uint32_t error = 0;
  dcheck(cudaMemcpy(&error, d.d_error, 4, cudaMemcpyDeviceToHost), "denoiser error word");
  if (error) {
    cudaMemset(d.d_error, 0, 4);
    throw DeviceError("a denoiser convolution's wait for the tensor cores ran out");
  }
  float ms = 0.0f;
  dcheck(cudaEventElapsedTime(&ms, d.ev0, d.ev1), "denoiser timing");
  d.last_ms = ms;
  return ms;
}

namespace {
// memcpy split over up to four host threads (pageable memory is copied by the
// CPU either way; one thread does not reach the device copies' rate).
void copy_parallel(char* dst, const char* src, size_t bytes) {
  constexpr size_t PART_MIN = 1u << 20;
  const size_t parts = std::min<size_t>(4, std::max<size_t>(1, bytes / PART_MIN));
  if (parts == 1) {
    memcpy(dst, src, bytes);
    return;
  }
  const size_t part = (bytes / parts + 63u) & ~size_t(63);
  std::vector<std::thread> helpers;
  for (size_t i = 1; i < parts && i * part < bytes; ++i)
    helpers.emplace_back([=]() { memcpy(dst + i * part, src + i * part, std::min(part, bytes - i * part)); });
  memcpy(dst, src, std::min(part, bytes));
  for (std::thread& t : helpers) t.join();
}
}  // namespace

void denoise_host(Denoiser& d, uint32_t width, uint32_t height, const float* color, const float* albedo,
                  const float* normal, float* out) {
  if (!color || !albedo || !normal || !out) throw Invalid("null argument");
  if (width == 0 || height == 0) throw Invalid("image dimensions must be nonzero");
  dcheck(cudaSetDevice(d.device), "denoiser device");
  if (!d.stream) dcheck(cudaStreamCreateWithFlags(&d.stream, cudaStreamNonBlocking), "denoiser stream");
  if (!d.h_stage) {
    dcheck(cudaHostAlloc(reinterpret_cast<void**>(&d.h_stage), 2u * DENOISE_STAGE_BYTES, cudaHostAllocDefault),
           "denoiser staging");
    for (cudaEvent_t& e : d.stage_ev) dcheck(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "denoiser staging");
  }
  const size_t pixels = (size_t)width * height, image = pixels * sizeof(float4);
  if (pixels > d.images_pixels) {
    if (d.d_images) cudaFree(d.d_images);
    d.d_images = nullptr;
    d.images_pixels = 0;
    dcheck(cudaMalloc(&d.d_images, pixels * 4u * sizeof(float4)), "denoiser images");
    d.images_pixels = pixels;
  }
  char* dev = reinterpret_cast<char*>(d.d_images);
  const char* in[3] = {reinterpret_cast<const char*>(color), reinterpret_cast<const char*>(albedo),
                       reinterpret_cast<const char*>(normal)};
  // up: half j & 1 takes piece j once the device copy out of it (piece j - 2) is done
  uint32_t j = 0;
  for (int k = 0; k < 3; ++k)
    for (size_t off = 0; off < image; off += DENOISE_STAGE_BYTES, ++j) {
      const size_t len = std::min(DENOISE_STAGE_BYTES, image - off);
      char* half = d.h_stage + (j & 1u) * DENOISE_STAGE_BYTES;
      if (j >= 2u) dcheck(cudaEventSynchronize(d.stage_ev[j & 1u]), "denoiser upload");
      copy_parallel(half, in[k] + off, len);
      dcheck(cudaMemcpyAsync(dev + k * image + off, half, len, cudaMemcpyHostToDevice, d.stream), "denoiser upload");
      dcheck(cudaEventRecord(d.stage_ev[j & 1u], d.stream), "denoiser upload");
    }
  float4* img = d.d_images;
  denoise_device(d, width, height, img, img + pixels, img + 2 * pixels, img + 3 * pixels, d.stream);
  // down: the device copy of piece i + 1 runs while the host copies piece i out
  const size_t pieces = (image + DENOISE_STAGE_BYTES - 1u) / DENOISE_STAGE_BYTES;
  auto fetch = [&](size_t i) {
    const size_t off = i * DENOISE_STAGE_BYTES, len = std::min(DENOISE_STAGE_BYTES, image - off);
    dcheck(cudaMemcpyAsync(d.h_stage + (i & 1u) * DENOISE_STAGE_BYTES, dev + 3 * image + off, len,
                           cudaMemcpyDeviceToHost, d.stream),
           "denoiser readback");
    dcheck(cudaEventRecord(d.stage_ev[i & 1u], d.stream), "denoiser readback");
  };
  fetch(0);
  for (size_t i = 0; i < pieces; ++i) {
    if (i + 1u < pieces) fetch(i + 1u);
    dcheck(cudaEventSynchronize(d.stage_ev[i & 1u]), "denoiser readback");
    const size_t off = i * DENOISE_STAGE_BYTES;
    copy_parallel(reinterpret_cast<char*>(out) + off, d.h_stage + (i & 1u) * DENOISE_STAGE_BYTES,
                  std::min(DENOISE_STAGE_BYTES, image - off));
  }
  denoiser_finish(d);
}

}  // namespace pfxt
