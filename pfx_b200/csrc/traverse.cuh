// BVH traversal on the B200 layout (pfxt_types.h: WideNode, TravTri, InstRec).
//
// Closest hit restates scene() (crates/trace/src/trace.wgsl:999-1075, with
// tri_hit :780-804 and box_hit :453-468); any hit restates occluded()
// (:1096-1168, tri_blocks :1076-1095).  Both walk the reference's tree in the
// reference's order (left child first, right child when the left subtree is
// done), test the same fp32 boxes with the same slab arithmetic (the quotients
// (lo - o)/d are correctly rounded, so they equal the reference's divisions
// bit for bit), and run the same Moller-Trumbore test
// with the same operation order, so the hit slot, record and distance are
// bit-identical to the CPU oracle's.  Clip planes, cutouts, alpha, sprites,
// motion and analytic shapes are outside this library's scope; the scenes it
// accepts have none.
//
// The per-ray stack holds (entry, near) pairs.  `near` is the entry distance
// of the child box computed when its parent was opened; box_hit(node, hit.t)
// at pop time is exactly "geometry passes && near <= hit.t", so re-checking
// near against the current hit distance on pop reproduces the reference's
// pruning.  The stack never holds more entries than the reference's 64-entry
// stack holds at the same point; scenes that would overflow that stack are
// refused when they are created.
//
// Work accounting (COUNT): the reference tests a node's box when it pops the
// node, and it pushes both children of every inner node it opens.  The
// counting variant therefore charges the left child when its parent is opened
// (the reference pops it next) and the right child when it is popped, pushing
// failed right children with near = +inf so they are charged, not visited.
#pragma once
#include "pfxt_math.h"
#include "pfxt_types.h"

namespace pfxt {

constexpr uint32_t STACK_SENTINEL = 0xfffffffeu;

struct SceneView {
  const WideNode* __restrict__ wide;
  const TravTri* __restrict__ tris;
  const InstRec* __restrict__ insts;
  uint32_t root;
  uint32_t small;  // 1 when every box coordinate is 0 or in [BOUNDED_TINY, BOUNDED_COORD] in magnitude
};

struct TraceHit {
  float t;
  uint32_t slot;
  uint32_t record;
  uint32_t hit;
  float u, v;  // barycentrics of the closest hit (tri_fill's u, v)
};

// Box and triangle tests one query did, counted as the reference counts them.
struct TraceCounts {
  uint32_t boxes;
  uint32_t tris;
};

// The Markstein quotients of the box test below are the correctly rounded
// (lo - o)/d whenever nothing in them underflows or overflows.  That holds for
// every box of a "bounded" ray, with no check per quotient:
//  * box coordinates and ray origin components are 0 or of magnitude in
//    [2^-70, 2^79], so a numerator x = lo - o is 0 (exact) or of magnitude in
//    [2^-93, 2^80] (a nonzero difference of two such values is a multiple of
//    the smaller one's ulp, at least 2^-93);
//  * direction components are degenerate (below 1e-12, never divided by) or of
//    magnitude in [1e-12, 2^20], so a nonzero quotient lies in [2^-113, 2^120]
//    (normal, with margin), and the residual x - q d, a multiple of
//    ulp(q) ulp(d) >= 2^-141 (q d is within a few ulps of x), is exact.
// Box coordinates are checked once per scene (SceneView::small); origins and
// directions per ray, in world space and in every instance's space.
constexpr float BOUNDED_COORD = 0x1p+79f;
constexpr float BOUNDED_TINY = 0x1p-70f;
constexpr float BOUNDED_DIR = 0x1p+20f;

// A ray in the space it is being traversed in, with the per-axis reciprocal
// used by the quotients (only read on axes with |d| >= 1e-12).  The boxes of
// a ray that is not `bounded` are all tested with IEEE division.
struct TRay {
  v3 o, d, r;
  bool bounded;
};

__device__ __forceinline__ bool bounded_axis(float o, float d) {
  float ao = fabsf(o), ad = fabsf(d);
  return (ao == 0.0f || (ao >= BOUNDED_TINY && ao <= BOUNDED_COORD)) && (ad <= BOUNDED_DIR || ad < 1e-12f);
}

__device__ __forceinline__ TRay make_tray(v3 o, v3 d, uint32_t small) {
  TRay t;
  t.o = o;
  t.d = d;
  t.r = mk3(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
  t.bounded = small != 0u && bounded_axis(o.x, d.x) && bounded_axis(o.y, d.y) && bounded_axis(o.z, d.z);
  return t;
}

// Slab test of one box with IEEE division throughout, for rays that are not
// bounded (see above).
__device__ __forceinline__ bool box_geometry_ieee_inline(float lx, float ly, float lz, float hx, float hy, float hz,
                                                         const TRay& ray, float& near) {
  float n = 0.0f, f = INFINITY;
  if (fabsf(ray.d.x) < 1e-12f) {
    if (ray.o.x < lx || ray.o.x > hx) return false;
  } else {
    float a = (lx - ray.o.x) / ray.d.x, b = (hx - ray.o.x) / ray.d.x;
    n = fmaxf(n, fminf(a, b));
    f = fminf(f, fmaxf(a, b));
  }
  if (fabsf(ray.d.y) < 1e-12f) {
    if (ray.o.y < ly || ray.o.y > hy) return false;
  } else {
    float a = (ly - ray.o.y) / ray.d.y, b = (hy - ray.o.y) / ray.d.y;
    n = fmaxf(n, fminf(a, b));
    f = fminf(f, fmaxf(a, b));
  }
  if (fabsf(ray.d.z) < 1e-12f) {
    if (ray.o.z < lz || ray.o.z > hz) return false;
  } else {
    float a = (lz - ray.o.z) / ray.d.z, b = (hz - ray.o.z) / ray.d.z;
    n = fmaxf(n, fminf(a, b));
    f = fminf(f, fmaxf(a, b));
  }
  near = n;
  return !(n > f);
}

// The same test out of line, for walks that take both kinds of ray (the work
// counting variant).
static __device__ __noinline__ bool box_geometry_ieee(float lx, float ly, float lz, float hx, float hy, float hz,
                                                      const TRay& ray, float& near) {
  return box_geometry_ieee_inline(lx, ly, lz, hx, hy, hz, ray, near);
}

// x / d by Markstein's correction from r = RN(1/d) (Markstein 1990; Cornea,
// Harrison and Tang, "Scientific Computing on Itanium-based Systems", 2002,
// ch. 8): with q = RN(x r) the residual fma(-q, d, x) is exact and
// RN(q + e r) is the correctly rounded quotient, provided nothing underflows
// or overflows, which a bounded ray guarantees.
__device__ __forceinline__ float quotient(float x, float d, float r) {
  float q = x * r;
  float e = fmaf(-q, d, x);
  return fmaf(e, r, q);
}

// Slab test of one box for a bounded ray: true when the ray's geometry passes
// (degenerate axes inside the slab, entry <= exit); `near` receives
// max(0, entries).  The six quotients equal IEEE division's (the reference
// divides).
__device__ __forceinline__ bool box_geometry_bounded(float lx, float ly, float lz, float hx, float hy, float hz,
                                                     const TRay& ray, float& near) {
  float n = 0.0f, f = INFINITY;
  if (fabsf(ray.d.x) < 1e-12f) {
    if (ray.o.x < lx || ray.o.x > hx) return false;
  } else {
    float a = quotient(lx - ray.o.x, ray.d.x, ray.r.x), b = quotient(hx - ray.o.x, ray.d.x, ray.r.x);
    n = fmaxf(n, fminf(a, b));
    f = fminf(f, fmaxf(a, b));
  }
  if (fabsf(ray.d.y) < 1e-12f) {
    if (ray.o.y < ly || ray.o.y > hy) return false;
  } else {
    float a = quotient(ly - ray.o.y, ray.d.y, ray.r.y), b = quotient(hy - ray.o.y, ray.d.y, ray.r.y);
    n = fmaxf(n, fminf(a, b));
    f = fminf(f, fmaxf(a, b));
  }
  if (fabsf(ray.d.z) < 1e-12f) {
    if (ray.o.z < lz || ray.o.z > hz) return false;
  } else {
    float a = quotient(lz - ray.o.z, ray.d.z, ray.r.z), b = quotient(hz - ray.o.z, ray.d.z, ray.r.z);
    n = fmaxf(n, fminf(a, b));
    f = fminf(f, fmaxf(a, b));
  }
  near = n;
  return !(n > f);
}

// Two fp32 lanes in one 64-bit register and the sm_100 paired instructions on
// them: each lane is one IEEE round-to-nearest add, multiply or fused
// multiply-add, the same operation as the scalar instruction, two per issue.
typedef unsigned long long f32x2;
__device__ __forceinline__ f32x2 pair(float lo, float hi) {
  f32x2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ void unpair(f32x2 v, float& lo, float& hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ f32x2 sub2(f32x2 a, f32x2 b) {
  f32x2 r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ f32x2 mul2(f32x2 a, f32x2 b) {
  f32x2 r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ f32x2 fma2(f32x2 a, f32x2 b, f32x2 c) {
  f32x2 r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
  return r;
}

// A bounded ray whose direction has no degenerate axis, paired the way a
// child box's six coordinates lie in a node, (lx, ly), (lz, hx), (hy, hz):
// origins (ox, oy), (oz, ox), (oy, oz), reciprocals and negated directions
// likewise.
struct PRay {
  f32x2 o[3], r[3], nd[3];
};
__device__ __forceinline__ PRay make_pray(const TRay& t) {
  PRay p;
  p.o[0] = pair(t.o.x, t.o.y);
  p.o[1] = pair(t.o.z, t.o.x);
  p.o[2] = pair(t.o.y, t.o.z);
  p.r[0] = pair(t.r.x, t.r.y);
  p.r[1] = pair(t.r.z, t.r.x);
  p.r[2] = pair(t.r.y, t.r.z);
  p.nd[0] = pair(-t.d.x, -t.d.y);
  p.nd[1] = pair(-t.d.z, -t.d.x);
  p.nd[2] = pair(-t.d.y, -t.d.z);
  return p;
}
__device__ __forceinline__ bool packable(const TRay& t) {
  return t.bounded && fabsf(t.d.x) >= 1e-12f && fabsf(t.d.y) >= 1e-12f && fabsf(t.d.z) >= 1e-12f;
}

// Markstein quotients of a pair: (x0/d0, x1/d1) correctly rounded, as quotient().
__device__ __forceinline__ f32x2 quotient2(f32x2 x, f32x2 nd, f32x2 r) {
  f32x2 q = mul2(x, r);
  f32x2 e = fma2(q, nd, x);  // q * (-d) + x = fma(-q, d, x) exactly
  return fma2(e, r, q);
}

// The sm_100 three-input minimum and maximum: the same value as two two-input
// ones (no NaN reaches them here; a signed zero only ever meets comparisons).
__device__ __forceinline__ float min3f(float a, float b, float c) {
  float r;
  asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
}
__device__ __forceinline__ float max3f(float a, float b, float c) {
  float r;
  asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
}

// box_geometry_bounded for a ray with no degenerate axis, the box given as
// the three coordinate pairs of its node: (lx, ly), (lz, hx), (hy, hz).
__device__ __forceinline__ bool box_geometry_paired(f32x2 b0, f32x2 b1, f32x2 b2, const PRay& p, float& near) {
  float lx, ly, lz, hx, hy, hz;
  unpair(quotient2(sub2(b0, p.o[0]), p.nd[0], p.r[0]), lx, ly);
  unpair(quotient2(sub2(b1, p.o[1]), p.nd[1], p.r[1]), lz, hx);
  unpair(quotient2(sub2(b2, p.o[2]), p.nd[2], p.r[2]), hy, hz);
  // max(0, entries) and min(exits), as box_geometry_bounded's chains
  float n = fmaxf(max3f(fminf(lx, hx), fminf(ly, hy), fminf(lz, hz)), 0.0f);
  float f = min3f(fmaxf(lx, hx), fmaxf(ly, hy), fmaxf(lz, hz));
  near = n;
  return !(n > f);
}

// How a walk tests boxes.
//  BOX_EITHER:  bounded rays with the Markstein quotients, other rays with the
//               out-of-line IEEE test (one walk for every ray; the call costs
//               the walk loop spills, so only the counting variant uses it);
//  BOX_BOUNDED: Markstein quotients only; a ray that is not bounded (in world
//               space or in an instance's space) stops at once with `retry`
//               set, and a second kernel walks it again from the start with
//               BOX_IEEE, so the walk loop has no call;
//  BOX_IEEE:    IEEE division throughout, inline;
//  BOX_PAIRED:  BOX_BOUNDED with the quotients in paired instructions; a ray
//               with a degenerate axis is handed over like an unbounded one.
// All four give the same bits for every box they test.
constexpr int BOX_EITHER = 0, BOX_BOUNDED = 1, BOX_IEEE = 2, BOX_PAIRED = 3;
// The flavour of the batch and queue traversal kernels (their retry kernels walk with BOX_IEEE) and
// whether they set leaves aside (Walker's SPEC).  On the 4K room's pass mix (closest hit, 2^22 rays):
// bounded 1023 Mrays/s, paired 1151, bounded with leaves set aside 1258, paired with leaves set aside
// 1551; the plain 4K pass 133.3, 125.4, 105.0 and 95.2 ms.
#ifndef TRACE_BOX
#define TRACE_BOX BOX_PAIRED
#endif
#ifndef TRACE_SPEC
#define TRACE_SPEC true
#endif
// Whether any-hit walks open the nearer child first (their result does not depend on the order).
// Measured on the plain 4K pass: 94.6 ms nearer first against 92.4 ms left first.
#ifndef TRACE_ANY_NEAR
#define TRACE_ANY_NEAR false
#endif
// Whether a leaf set aside has its triangles prefetched: 0 no, 1 into L1 (prefetch.global.L1 per
// line), 2 into L2 by one bulk prefetch (cp.async.bulk.prefetch.L2, the TMA unit).  Measured on the
// pass mix (closest hit, 2^22 rays) and the plain 4K pass: none 1550 Mrays/s and 91.4 ms, L1 1470 and
// 100.6 ms, L2 bulk 1489 and 94.5 ms.  The scene's nodes and triangles mostly sit in L2 already, and
// the extra instructions cost more than the latency they hide.
#ifndef TRACE_LEAF_PREFETCH
#define TRACE_LEAF_PREFETCH 0
#endif

template <int BOX>
__device__ __forceinline__ bool box_test(float lx, float ly, float lz, float hx, float hy, float hz, const TRay& ray,
                                         float& near) {
  if (BOX == BOX_IEEE) return box_geometry_ieee_inline(lx, ly, lz, hx, hy, hz, ray, near);
  if (BOX == BOX_EITHER && !ray.bounded) return box_geometry_ieee(lx, ly, lz, hx, hy, hz, ray, near);
  return box_geometry_bounded(lx, ly, lz, hx, hy, hz, ray, near);
}

// to_object (trace.wgsl:449-452): (dot(lo,q), dot(hi,q), dot(rows2,q)), q=(p,w).
__device__ __forceinline__ v3 to_object(const float4& r0, const float4& r1, const float4& r2, v3 p, float w) {
  v3 o;
  o.x = ((r0.x * p.x + r0.y * p.y) + r0.z * p.z) + r0.w * w;
  o.y = ((r1.x * p.x + r1.y * p.y) + r1.z * p.z) + r1.w * w;
  o.z = ((r2.x * p.x + r2.y * p.y) + r2.z * p.z) + r2.w * w;
  return o;
}

// The traversal stack of one lane.  With SHORT > 0 its first SHORT entries
// live in shared memory, one column per lane (entry k of lane t at word
// k * lanes + t, so a warp's accesses fall in distinct banks), and the rest
// in local memory; with SHORT == 0 all of it is local.  Only where entries
// are kept differs: the walk pushes and pops exactly the same entries.
constexpr int SHORT_STACK = 16;

// Resident warps per SM the traversal kernels are compiled for: it sets their
// register budget.  32 warps (64 registers, a few bytes of spill) measured
// faster than 24 (72 registers) and 36 (56 registers, more spills).
#ifndef TRACE_WARPS_PER_SM
#define TRACE_WARPS_PER_SM 32
#endif

template <int SHORT>
struct LaneStack {
  uint32_t* sh_ref;
  float* sh_near;
  uint32_t lanes;
  uint2 entry[REF_STACK - SHORT];  // (ref, near bits) pairs past the shared-memory top
  __device__ __forceinline__ void put(int k, uint32_t r, float n) {
    if (k < SHORT) {
      sh_ref[k * lanes] = r;
      sh_near[k * lanes] = n;
    } else {
      entry[k - SHORT] = make_uint2(r, __float_as_uint(n));
    }
  }
  __device__ __forceinline__ void get(int k, uint32_t& r, float& n) const {
    if (k < SHORT) {
      r = sh_ref[k * lanes];
      n = sh_near[k * lanes];
    } else {
      uint2 e = entry[k - SHORT];
      r = e.x;
      n = __uint_as_float(e.y);
    }
  }
};

// Entries as (ref, near bits) pairs: one 8-byte store per push and one 8-byte
// load per pop (measured 1037 against 1011 Mrays/s with two 4-byte arrays).
template <>
struct LaneStack<0> {
  uint2 entry[REF_STACK];
  __device__ __forceinline__ void put(int k, uint32_t r, float n) { entry[k] = make_uint2(r, __float_as_uint(n)); }
  __device__ __forceinline__ void get(int k, uint32_t& r, float& n) const {
    uint2 e = entry[k];
    r = e.x;
    n = __uint_as_float(e.y);
  }
};

// One query's traversal state; the stack is the caller's.
// SPEC: a lane that reaches a leaf while other lanes of its warp still walk
// inner nodes sets the leaf aside (`held`) and walks on, so that the warp's
// leaf tests run with more lanes at once (Aila and Laine, "Understanding the
// efficiency of ray traversal on GPUs", 2009).  It tests the leaves the
// reference tests, in the reference's order, with the same hit distance at
// each: the held leaf is the next one in the reference's order and is tested
// before any other; everything walked past it was decided against the hit
// distance from before its test, which is not smaller than the reference's, so
// the walk only keeps more entries; and each of those is checked again
// against the current distance before it is opened or tested (a node's entry
// distance is at least its ancestors' in the same space, as a box holds its
// children's).  A held leaf is tested before the walk enters or leaves an
// instance, so it is tested in its own space.  Entries are right siblings of
// the current path, as in the reference, so the stack is no deeper.
template <bool ANY, bool COUNT, int BOX = BOX_EITHER, bool SPEC = false>
struct Walker {
  TRay ray;     // ray in the current space (the world ray itself is the caller's: see inner_phase)
  PRay pr;      // BOX_PAIRED: `ray` paired for the box test
  float limit;
  uint32_t base, record, word;
  float inv_det;
  uint32_t ref;
  float near_cur;
  int top;
  uint32_t held;  // SPEC: the leaf set aside, REF_NONE when none
  bool done;
  bool retry;  // BOX_BOUNDED, BOX_PAIRED: the ray is not bounded (or, paired, has a degenerate axis); walk
               // it again with BOX_IEEE
  TraceHit hit;
  TraceCounts counts;

  __device__ __forceinline__ void start(const SceneView& s, v3 wo, v3 wd, float lim) {
    ray = make_tray(wo, wd, s.small);
    limit = lim;
    base = record = word = 0u;
    inv_det = 1.0f;
    ref = s.root;
    near_cur = -INFINITY;
    top = 0;
    held = REF_NONE;
    done = (s.root == REF_NONE);
    retry = false;
    if (BOX == BOX_BOUNDED && !done && !ray.bounded) {
      retry = true;
      done = true;
    }
    if (BOX == BOX_PAIRED && !done) {
      if (!packable(ray)) {
        retry = true;
        done = true;
      } else {
        pr = make_pray(ray);
      }
    }
    hit.t = lim;
    hit.slot = hit.record = hit.hit = 0u;
    hit.u = hit.v = 0.0f;
    counts.boxes = counts.tris = 0u;
  }

  template <class Stack>
  __device__ __forceinline__ void pop(const Stack& st) {
    if (top == 0) {
      done = true;
      return;
    }
    --top;
    st.get(top, ref, near_cur);
    if (COUNT && ref != STACK_SENTINEL) counts.boxes += 1u;
  }

  // Walk inner nodes until the current entry is a leaf that passes its
  // near check, or the traversal is finished.  world(o, d) gives the world
  // ray again where an instance is entered or left (the walk keeps only the
  // ray of the current space; callers read it back from where it came from).
  template <class Stack, class World>
  __device__ __forceinline__ void inner_phase(const SceneView& s, Stack& st, const World& world) {
    while (!done) {
      if constexpr (SPEC) {
        // a lane holding a leaf walks on only while another lane of the warp still looks for one
        if (held != REF_NONE && !__any_sync(__activemask(), held == REF_NONE)) return;
      }
      if (ref == STACK_SENTINEL) {
        if (SPEC && held != REF_NONE) return;  // the held leaf is tested in its own space
        v3 o, d;
        world(o, d);
        ray = make_tray(o, d, s.small);
        if (BOX == BOX_PAIRED) pr = make_pray(ray);
        base = record = word = 0u;
        inv_det = 1.0f;
        pop(st);
        continue;
      }
      if (!(near_cur <= hit.t)) {
        pop(st);
        continue;
      }
      if ((ref & REF_LEAF) == 0u) {
        const float4* p = reinterpret_cast<const float4*>(s.wide + ref);
        uint4 q3 = __ldg(reinterpret_cast<const uint4*>(p + 3));
        float n0 = 0.0f, n1 = 0.0f;
        bool ok0, ok1;
        bool has1 = q3.y != REF_NONE;
        if constexpr (BOX == BOX_PAIRED) {
          // the node's twelve coordinates as six pairs: (lx, ly), (lz, hx), (hy, hz) of each child
          const ulonglong2* pp = reinterpret_cast<const ulonglong2*>(p);
          ulonglong2 a = __ldg(pp + 0), b = __ldg(pp + 1), c = __ldg(pp + 2);
          ok0 = box_geometry_paired(a.x, a.y, b.x, pr, n0) && n0 <= hit.t;
          ok1 = has1 && box_geometry_paired(b.y, c.x, c.y, pr, n1) && n1 <= hit.t;
        } else {
          float4 q0 = __ldg(p + 0), q1 = __ldg(p + 1), q2 = __ldg(p + 2);
          ok0 = box_test<BOX>(q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, ray, n0) && n0 <= hit.t;
          ok1 = has1 && box_test<BOX>(q1.z, q1.w, q2.x, q2.y, q2.z, q2.w, ray, n1) && n1 <= hit.t;
        }
        if (COUNT) counts.boxes += 1u;  // the left child, popped next by the reference
        uint32_t r0 = q3.x, r1 = q3.y;
        if constexpr (ANY && !COUNT && TRACE_ANY_NEAR) {
          // any hit: whether the ray is blocked does not depend on the order,
          // so the nearer child goes first
          if (ok0 && ok1 && n1 < n0) {
            r0 = q3.y;
            r1 = q3.x;
            float t = n0;
            n0 = n1;
            n1 = t;
          }
        }
        if ((ok1 || (COUNT && has1)) && top < (int)REF_STACK) {
          st.put(top, r1, ok1 ? n1 : INFINITY);
          ++top;
        }
        if (ok0) {
          ref = r0;
          near_cur = n0;
        } else {
          pop(st);
        }
        continue;
      }
      if ((ref & REF_INST) == REF_INST) {
        if (SPEC && held != REF_NONE) return;  // the held leaf is tested in its own space
        if (top >= (int)REF_STACK) {  // refused at creation; never taken
          pop(st);
          continue;
        }
        const float4* p = reinterpret_cast<const float4*>(s.insts + (ref & 0x3fffffffu));
        float4 r0 = __ldg(p + 0), r1 = __ldg(p + 1), r2 = __ldg(p + 2);
        uint4 m = __ldg(reinterpret_cast<const uint4*>(p + 3));
        float4 m2 = __ldg(p + 4);
        st.put(top, STACK_SENTINEL, -INFINITY);
        ++top;
        base = m.y;
        record = m.z;
        word = m.w;
        inv_det = m2.x;
        if (__float_as_uint(m2.y) != 0u) {
          v3 o, d;
          world(o, d);
          ray = make_tray(to_object(r0, r1, r2, o, 1.0f), to_object(r0, r1, r2, d, 0.0f), s.small);
          if (BOX == BOX_BOUNDED && !ray.bounded) {
            retry = true;
            done = true;
            return;
          }
          if (BOX == BOX_PAIRED) {
            if (!packable(ray)) {
              retry = true;
              done = true;
              return;
            }
            pr = make_pray(ray);
          }
        }
        ref = m.x;
        near_cur = -INFINITY;
        continue;
      }
      // a leaf that passed its near check
      if constexpr (SPEC) {
        if (held == REF_NONE) {
          held = ref;
          prefetch_leaf(s, ref);
          pop(st);
          continue;
        }
      }
      return;
    }
  }

  // A leaf set aside is tested later: its triangles (contiguous TravTri
  // records, 48 bytes each) may be fetched meanwhile.
  __device__ __forceinline__ void prefetch_leaf(const SceneView& s, uint32_t leaf) const {
#if TRACE_LEAF_PREFETCH
    const uint32_t n = ((leaf >> LEAF_FIRST_BITS) & 15u) + 1u;
    const char* p = reinterpret_cast<const char*>(s.tris + base + (leaf & LEAF_FIRST_MASK));
#if TRACE_LEAF_PREFETCH == 1
    for (uint32_t b = 0; b < n * 48u; b += 128u) asm volatile("prefetch.global.L1 [%0];" ::"l"(p + b));
    asm volatile("prefetch.global.L1 [%0];" ::"l"(p + n * 48u - 1u));
#else
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(n * 48u) : "memory");
#endif
#else
    (void)s;
    (void)leaf;
#endif
  }

  // SPEC: is there a leaf to test (the held one, or the current entry)?
  __device__ __forceinline__ bool leaf_ready() const { return SPEC ? (held != REF_NONE || !done) : !done; }

  // Test the triangles of the held leaf, then move to the next entry.
  template <class Stack>
  __device__ __forceinline__ void leaf_phase(const SceneView& s, Stack& st) {
    // SPEC: the held leaf first; the current entry stays, to be checked again
    const bool from_held = SPEC && held != REF_NONE;
    const uint32_t leaf = from_held ? held : ref;
    if (SPEC) held = REF_NONE;
    uint32_t first = leaf & LEAF_FIRST_MASK;
    uint32_t n = ((leaf >> LEAF_FIRST_BITS) & 15u) + 1u;
    bool skip = ANY ? ((word & CASTS_NO_SHADOW) != 0u) : ((word & SHADOW_ONLY) != 0u);
    if (COUNT && skip) counts.tris += n;
    if (!skip) {
      for (uint32_t j = 0; j < n; ++j) {
        if (COUNT) counts.tris += 1u;  // the reference stops counting at an any-hit blocker
        uint32_t i = base + first + j;
        const float4* tp = reinterpret_cast<const float4*>(s.tris + i);
        float4 ta = __ldg(tp + 0), te1 = __ldg(tp + 1), te2 = __ldg(tp + 2);
        v3 a = mk3(ta.x, ta.y, ta.z), e1 = mk3(te1.x, te1.y, te1.z), e2 = mk3(te2.x, te2.y, te2.z);
        float u, v, t;
        if constexpr (BOX == BOX_PAIRED) {
          // The same test on the negated direction n = -d the paired ray
          // holds: pv, det and inv change sign exactly (round-to-nearest is
          // symmetric), so u and v are the same bits and t = -(e2.qv * inv).
          v3 rn, ro;
          float spare;
          unpair(pr.nd[0], rn.x, rn.y);
          unpair(pr.nd[1], rn.z, spare);
          unpair(pr.o[0], ro.x, ro.y);
          unpair(pr.o[1], ro.z, spare);
          v3 pv = cross3(rn, e2);
          float det = dot3(e1, pv);
          float seen = det * inv_det;
          if (fabsf(seen) < 1e-9f) continue;
          if (!ANY && (word & ONE_SIDED) != 0u && seen > 0.0f) continue;
          float inv = 1.0f / det;
          v3 sv = sub3(ro, a);
          u = dot3(sv, pv) * inv;
          if (u < 0.0f || u > 1.0f) continue;
          v3 qv = cross3(sv, e1);
          v = dot3(rn, qv) * inv;
          if (v < 0.0f || u + v > 1.0f) continue;
          t = -(dot3(e2, qv) * inv);
        } else {
          v3 pv = cross3(ray.d, e2);
          float det = dot3(e1, pv);
          float seen = det * inv_det;
          if (fabsf(seen) < 1e-9f) continue;
          if (!ANY && (word & ONE_SIDED) != 0u && seen < 0.0f) continue;
          float inv = 1.0f / det;
          v3 sv = sub3(ray.o, a);
          u = dot3(sv, pv) * inv;
          if (u < 0.0f || u > 1.0f) continue;
          v3 qv = cross3(sv, e1);
          v = dot3(ray.d, qv) * inv;
          if (v < 0.0f || u + v > 1.0f) continue;
          t = dot3(e2, qv) * inv;
        }
        if (ANY) {
          if (t <= 0.0001f || t >= limit) continue;
          hit.hit = 1u;
          hit.t = t;
          hit.slot = i;
          hit.record = record;
          done = true;
          return;
        } else if (t > 0.0001f && t < hit.t) {
          hit.t = t;
          hit.slot = i;
          hit.record = record;
          hit.hit = 1u;
          hit.u = u;
          hit.v = v;
        }
      }
    }
    if (!from_held) pop(st);
  }

  // Run to completion (one query, no work sharing).
  template <class Stack, class World>
  __device__ __forceinline__ void run(const SceneView& s, Stack& st, const World& world) {
    while (leaf_ready()) {
      inner_phase(s, st, world);
      if (!leaf_ready()) break;
      leaf_phase(s, st);
    }
  }
};

// Single-query helpers used by shading code.
template <bool ANY>
__device__ __forceinline__ TraceHit traverse(const SceneView& s, v3 o, v3 d, float limit) {
  LaneStack<0> st;
  Walker<ANY, false, BOX_EITHER> w;
  w.start(s, o, d, limit);
  w.run(s, st, [&](v3& wo, v3& wd) {
    wo = o;
    wd = d;
  });
  return w.hit;
}

}  // namespace pfxt
