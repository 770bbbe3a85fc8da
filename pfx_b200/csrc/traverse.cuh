// BVH traversal on the B200 layout (pfxt_types.h: WideNode, TravTri, InstRec).
//
// Closest hit restates scene() (crates/trace/src/trace.wgsl:999-1075, with
// tri_hit :780-804 and box_hit :453-468); any hit restates occluded()
// (:1096-1168, tri_blocks :1076-1095).  Both walk the reference's tree in the
// reference's order (left child first, right child when the left subtree is
// done), test the same fp32 boxes with the same division-based slab arithmetic,
// and run the same Moller-Trumbore test with the same operation order, so the
// hit slot, record and distance are bit-identical to the CPU oracle's.  The
// parts of the reference not in this library's scope (clip planes, cutouts,
// alpha, sprites, motion, analytic shapes) are absent from the scenes it
// accepts and are not tested here.
//
// The per-ray stack holds (entry, near) pairs.  `near` is the entry distance
// of the child box computed when its parent was opened; box_hit(node, hit.t)
// at pop time is exactly "geometry passes && near <= hit.t", so re-checking
// near against the current hit distance on pop reproduces the reference's
// pruning.  The stack never holds more entries than the reference's 64-entry
// stack holds at the same point; scenes that would overflow that stack are
// refused when they are created.
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
};

struct TraceHit {
  float t;
  uint32_t slot;
  uint32_t record;
  uint32_t hit;
};

// Counters of the work one query did (node box tests and triangle tests, as
// the reference counts them: one box test per popped node).
struct TraceCounts {
  uint32_t boxes;
  uint32_t tris;
};

// Slab test of one box: true when the ray's geometry passes (degenerate axes
// inside the slab, entry <= exit); `near` receives max(0, entries).
__device__ __forceinline__ bool box_geometry(float lx, float ly, float lz, float hx, float hy, float hz, v3 o, v3 d,
                                             float& near) {
  float n = 0.0f, f = INFINITY;
  if (fabsf(d.x) < 1e-12f) {
    if (o.x < lx || o.x > hx) return false;
  } else {
    float a = (lx - o.x) / d.x, b = (hx - o.x) / d.x;
    n = fmaxf(n, fminf(a, b));
    f = fminf(f, fmaxf(a, b));
  }
  if (fabsf(d.y) < 1e-12f) {
    if (o.y < ly || o.y > hy) return false;
  } else {
    float a = (ly - o.y) / d.y, b = (hy - o.y) / d.y;
    n = fmaxf(n, fminf(a, b));
    f = fminf(f, fmaxf(a, b));
  }
  if (fabsf(d.z) < 1e-12f) {
    if (o.z < lz || o.z > hz) return false;
  } else {
    float a = (lz - o.z) / d.z, b = (hz - o.z) / d.z;
    n = fmaxf(n, fminf(a, b));
    f = fminf(f, fmaxf(a, b));
  }
  near = n;
  return !(n > f);
}

// to_object (trace.wgsl:449-452): (dot(lo,q), dot(hi,q), dot(rows2,q)), q=(p,w).
__device__ __forceinline__ v3 to_object(const InstRec& r, v3 p, float w) {
  v3 o;
  o.x = ((r.inv[0][0] * p.x + r.inv[0][1] * p.y) + r.inv[0][2] * p.z) + r.inv[0][3] * w;
  o.y = ((r.inv[1][0] * p.x + r.inv[1][1] * p.y) + r.inv[1][2] * p.z) + r.inv[1][3] * w;
  o.z = ((r.inv[2][0] * p.x + r.inv[2][1] * p.y) + r.inv[2][2] * p.z) + r.inv[2][3] * w;
  return o;
}

__device__ __forceinline__ void load_inst(const InstRec* __restrict__ insts, uint32_t i, InstRec& r) {
  const float4* p = reinterpret_cast<const float4*>(insts + i);
  float4 q0 = __ldg(p + 0), q1 = __ldg(p + 1), q2 = __ldg(p + 2), q3 = __ldg(p + 3), q4 = __ldg(p + 4);
  r.inv[0][0] = q0.x; r.inv[0][1] = q0.y; r.inv[0][2] = q0.z; r.inv[0][3] = q0.w;
  r.inv[1][0] = q1.x; r.inv[1][1] = q1.y; r.inv[1][2] = q1.z; r.inv[1][3] = q1.w;
  r.inv[2][0] = q2.x; r.inv[2][1] = q2.y; r.inv[2][2] = q2.z; r.inv[2][3] = q2.w;
  r.root = __float_as_uint(q3.x);
  r.base = __float_as_uint(q3.y);
  r.record = __float_as_uint(q3.z);
  r.word = __float_as_uint(q3.w);
  r.inv_det = q4.x;
  r.transformed = __float_as_uint(q4.y);
}

// Closest hit (ANY = false) or any hit (ANY = true).  `limit` is the
// reference's limit argument (1e20 for camera and bounce rays).
template <bool ANY, bool COUNT>
__device__ __forceinline__ TraceHit traverse(const SceneView& s, v3 o, v3 d, float limit, TraceCounts* counts) {
  TraceHit hit;
  hit.t = limit;
  hit.slot = 0u;
  hit.record = 0u;
  hit.hit = 0u;
  if (s.root == REF_NONE) return hit;
  uint32_t stack_ref[REF_STACK];
  float stack_near[REF_STACK];
  int top = 0;
  v3 ro = o, rd = d;
  uint32_t base = 0u, record = 0u, word = 0u;
  float inv_det = 1.0f;
  uint32_t ref = s.root;  // current entry: a wide node whose children are tested
  float near_cur = -INFINITY;
  for (;;) {
    if (ref == STACK_SENTINEL) {
      ro = o;
      rd = d;
      base = 0u;
      record = 0u;
      word = 0u;
      inv_det = 1.0f;
    } else if (near_cur <= hit.t) {
      if ((ref & REF_LEAF) == 0u) {
        const float4* p = reinterpret_cast<const float4*>(s.wide + ref);
        float4 q0 = __ldg(p + 0), q1 = __ldg(p + 1), q2 = __ldg(p + 2);
        uint4 q3 = __ldg(reinterpret_cast<const uint4*>(p + 3));
        float n0 = 0.0f, n1 = 0.0f;
        bool ok0 = box_geometry(q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, ro, rd, n0);
        bool ok1 = (q3.y != REF_NONE) && box_geometry(q1.z, q1.w, q2.x, q2.y, q2.z, q2.w, ro, rd, n1);
        if (COUNT) counts->boxes += (q3.y != REF_NONE) ? 2u : 1u;
        ok0 = ok0 && n0 <= hit.t;
        ok1 = ok1 && n1 <= hit.t;
        if (ok1 && top < (int)REF_STACK) {
          stack_ref[top] = q3.y;
          stack_near[top] = n1;
          ++top;
        }
        if (ok0) {
          ref = q3.x;
          near_cur = n0;
          continue;
        }
      } else if ((ref & REF_INST) == REF_INST) {
        if (top >= (int)REF_STACK) goto pop;  // refused at creation; never taken
        InstRec r;
        load_inst(s.insts, ref & 0x3fffffffu, r);
        stack_ref[top] = STACK_SENTINEL;
        stack_near[top] = -INFINITY;
        ++top;
        base = r.base;
        record = r.record;
        word = r.word;
        inv_det = r.inv_det;
        if (r.transformed) {
          ro = to_object(r, o, 1.0f);
          rd = to_object(r, d, 0.0f);
        }
        ref = r.root;
        near_cur = -INFINITY;
        continue;
      } else {
        uint32_t first = ref & LEAF_FIRST_MASK;
        uint32_t n = ((ref >> LEAF_FIRST_BITS) & 15u) + 1u;
        if (COUNT) counts->tris += n;
        bool skip = ANY ? ((word & CASTS_NO_SHADOW) != 0u) : ((word & SHADOW_ONLY) != 0u);
        if (!skip) {
          for (uint32_t j = 0; j < n; ++j) {
            uint32_t i = base + first + j;
            const float4* tp = reinterpret_cast<const float4*>(s.tris + i);
            float4 ta = __ldg(tp + 0), te1 = __ldg(tp + 1), te2 = __ldg(tp + 2);
            v3 a = mk3(ta.x, ta.y, ta.z), e1 = mk3(te1.x, te1.y, te1.z), e2 = mk3(te2.x, te2.y, te2.z);
            v3 pv = cross3(rd, e2);
            float det = dot3(e1, pv);
            float seen = det * inv_det;
            if (fabsf(seen) < 1e-9f) continue;
            if (!ANY && (word & ONE_SIDED) != 0u && seen < 0.0f) continue;
            float inv = 1.0f / det;
            v3 sv = sub3(ro, a);
            float u = dot3(sv, pv) * inv;
            if (u < 0.0f || u > 1.0f) continue;
            v3 qv = cross3(sv, e1);
            float v = dot3(rd, qv) * inv;
            if (v < 0.0f || u + v > 1.0f) continue;
            float t = dot3(e2, qv) * inv;
            if (ANY) {
              if (t <= 0.0001f || t >= limit) continue;
              hit.hit = 1u;
              hit.t = t;
              hit.slot = i;
              hit.record = record;
              return hit;
            } else {
              if (t > 0.0001f && t < hit.t) {
                hit.t = t;
                hit.slot = i;
                hit.record = record;
                hit.hit = 1u;
              }
            }
          }
        }
      }
    }
  pop:
    if (top == 0) break;
    --top;
    ref = stack_ref[top];
    near_cur = stack_near[top];
  }
  return hit;
}

}  // namespace pfxt
