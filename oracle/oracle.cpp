// TEST INFRASTRUCTURE ONLY - the CPU oracle of the B200 tracer.
//
// A scalar C++ restatement of the reference tracer (gmrdad82/pfx,
// crates/trace) used by tests/ and by bench.py's CPU-baseline leg as the
// checker.  Nothing in the product (pfx_b200/) links, imports or calls it.
//
// It works on the reference's own packed layouts (SceneBuffers: 48-byte BVH2
// nodes in preorder, 96-byte triangles in slot order, 176-byte instance
// surfaces) and walks them the way the WGSL does, transliterated function by
// function; each function cites the reference lines it follows.  Transcendental
// functions come from pfx_b200/csrc/pfxt_math.h, the one implementation shared
// with the kernels (written from published methods), so that both sides round
// the same way.
//
// Parity pins: the restatement is checked against the reference's own tests
// (bvh.rs:330-381 brute force on the LCG fixture, sobol.rs known answers,
// adaptive.rs known answers, lights.rs and tree.rs properties) in
// tests/test_oracle.py.
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <cfloat>
#include <climits>
#include <atomic>
#include <thread>
#include <vector>

#include "pfxt_math.h"

using namespace pfxt;

namespace {

// Work-sharing loop over [0, n) on all host threads (chunks of `grain`).
template <typename F>
void parallel_for(int64_t n, int64_t grain, F&& fn) {
  unsigned threads = std::max(1u, std::thread::hardware_concurrency());
  if (n <= grain || threads == 1) {
    for (int64_t i = 0; i < n; ++i) fn(i, 0u);
    return;
  }
  std::atomic<int64_t> next{0};
  std::vector<std::thread> pool;
  for (unsigned t = 0; t < threads; ++t) {
    pool.emplace_back([&, t]() {
      for (;;) {
        int64_t start = next.fetch_add(grain);
        if (start >= n) break;
        int64_t end = std::min(n, start + grain);
        for (int64_t i = start; i < end; ++i) fn(i, t);
      }
    });
  }
  for (auto& th : pool) th.join();
}

struct Node {  // bvh.rs:7-13
  float lo[4], hi[4];
  uint32_t first, count, pad[2];
};
struct Tri {  // gpu.rs:19-26
  float a[4], b[4], c[4], na[4], nb[4], nc[4];
};
struct Surface {  // gpu.rs:29-38
  float clip0[4], clip1[4], transform[4], crop[4];
  uint32_t info[4];
  float forward[3][4], inverse[3][4];
};
struct RayIn {
  float o[3], tmax, d[3];
  uint32_t pad;
};
struct HitOut {
  float t;
  uint32_t slot, record, hit;
};

const uint32_t ENTRYPOINT_SENTINEL = 0x76543210u;  // trace.wgsl:447
const uint32_t INSTANCE_LEAF = 1u;

struct Scene {
  const Node* nodes;
  uint32_t node_count;
  const Tri* tris;
  uint32_t tri_count;
  const Surface* surfaces;
};

// ------------------------------------------------------------------ bvh.rs
// bvh.rs:294-324, triangle_hit of the CPU builder's own walk.
bool bvh_triangle_hit(const float v[9], v3 o, v3 d, float limit, float* dist) {
  v3 a = mk3(v[0], v[1], v[2]), b = mk3(v[3], v[4], v[5]), c = mk3(v[6], v[7], v[8]);
  v3 e1 = sub3(b, a), e2 = sub3(c, a);
  v3 p = cross3(d, e2);
  float det = dot3(e1, p);
  if (fabsf(det) < 1e-9f) return false;
  float inv = 1.0f / det;
  v3 s = sub3(o, a);
  float u = dot3(s, p) * inv;
  if (!(u >= 0.0f && u <= 1.0f)) return false;
  v3 q = cross3(s, e1);
  float vv = dot3(d, q) * inv;
  if (vv < 0.0f || u + vv > 1.0f) return false;
  float t = dot3(e2, q) * inv;
  if (t <= 1e-5f || t >= limit) return false;
  *dist = t;
  return true;
}

// bvh.rs:272-292
bool bvh_box_hit(const Node& n, v3 o, v3 d, float limit) {
  float near_ = 0.0f, far_ = limit;
  float oo[3] = {o.x, o.y, o.z}, dd[3] = {d.x, d.y, d.z};
  for (int axis = 0; axis < 3; ++axis) {
    if (fabsf(dd[axis]) < 1e-12f) {
      if (oo[axis] < n.lo[axis] || oo[axis] > n.hi[axis]) return false;
    } else {
      float a = (n.lo[axis] - oo[axis]) / dd[axis];
      float b = (n.hi[axis] - oo[axis]) / dd[axis];
      near_ = fmaxf(near_, fminf(a, b));
      far_ = fminf(far_, fmaxf(a, b));
      if (near_ > far_) return false;
    }
  }
  return true;
}

// ------------------------------------------------------------ trace.wgsl
// box_hit (trace.wgsl:453-468)
bool box_hit(const Node& node, v3 o, v3 d, float limit) {
  float near_ = 0.0f, far_ = limit;
  float oo[3] = {o.x, o.y, o.z}, dd[3] = {d.x, d.y, d.z};
  for (int axis = 0; axis < 3; ++axis) {
    if (fabsf(dd[axis]) < 1e-12f) {
      if (oo[axis] < node.lo[axis] || oo[axis] > node.hi[axis]) return false;
    } else {
      float a = (node.lo[axis] - oo[axis]) / dd[axis];
      float b = (node.hi[axis] - oo[axis]) / dd[axis];
      near_ = fmaxf(near_, fminf(a, b));
      far_ = fminf(far_, fmaxf(a, b));
      if (near_ > far_) return false;
    }
  }
  return true;
}

// to_object (trace.wgsl:449-452)
v3 to_object(const Node& m, v3 p, float w) {
  float r2[4] = {bits2f(m.first), bits2f(m.count), bits2f(m.pad[0]), bits2f(m.pad[1])};
  v3 out;
  out.x = ((m.lo[0] * p.x + m.lo[1] * p.y) + m.lo[2] * p.z) + m.lo[3] * w;
  out.y = ((m.hi[0] * p.x + m.hi[1] * p.y) + m.hi[2] * p.z) + m.hi[3] * w;
  out.z = ((r2[0] * p.x + r2[1] * p.y) + r2[2] * p.z) + r2[3] * w;
  return out;
}

// clipped_at (trace.wgsl:678-681)
bool clipped_at(const Surface& s, v3 point) {
  bool c0 = (s.clip0[0] != 0.0f || s.clip0[1] != 0.0f || s.clip0[2] != 0.0f) &&
            dot3(mk3(s.clip0[0], s.clip0[1], s.clip0[2]), point) > s.clip0[3];
  bool c1 = (s.clip1[0] != 0.0f || s.clip1[1] != 0.0f || s.clip1[2] != 0.0f) &&
            dot3(mk3(s.clip1[0], s.clip1[1], s.clip1[2]), point) > s.clip1[3];
  return c0 || c1;
}

struct Walk {
  float t;
  uint32_t surface, record;
  bool hit;
  float u, v;
};

// tri_hit (trace.wgsl:780-804); cut_out is false for the scenes in scope
// (no cutout word, no alpha materials, no sprites).
void tri_hit(const Scene& s, uint32_t i, uint32_t record, uint32_t word, float inv_det, v3 o, v3 d, v3 wo, v3 wd,
             bool shadow_ray, Walk* hit) {
  const Tri& tri = s.tris[i];
  if ((word & 1u) != 0u && !shadow_ray) return;
  if ((word & 2u) != 0u && shadow_ray) return;
  v3 a = mk3(tri.a[0], tri.a[1], tri.a[2]);
  v3 e1 = sub3(mk3(tri.b[0], tri.b[1], tri.b[2]), a);
  v3 e2 = sub3(mk3(tri.c[0], tri.c[1], tri.c[2]), a);
  v3 p = cross3(d, e2);
  float det = dot3(e1, p);
  float seen = det * inv_det;
  if (fabsf(seen) < 1e-9f) return;
  if (!shadow_ray && (word & (1u << 23)) != 0u && seen < 0.0f) return;
  float inv = 1.0f / det;
  v3 sv = sub3(o, a);
  float u = dot3(sv, p) * inv;
  if (u < 0.0f || u > 1.0f) return;
  v3 q = cross3(sv, e1);
  float v = dot3(d, q) * inv;
  if (v < 0.0f || u + v > 1.0f) return;
  float t = dot3(e2, q) * inv;
  if (t > 0.0001f && t < hit->t) {
    if (clipped_at(s.surfaces[record], add3(wo, scl3(wd, t)))) return;
    hit->t = t;
    hit->surface = i;
    hit->record = record;
    hit->hit = true;
    hit->u = u;
    hit->v = v;
  }
}

// tri_blocks (trace.wgsl:1076-1095)
bool tri_blocks(const Scene& s, uint32_t i, uint32_t record, uint32_t word, float inv_det, v3 o, v3 d, v3 wo, v3 wd,
                float limit) {
  const Tri& tri = s.tris[i];
  if ((word & 2u) != 0u) return false;
  v3 a = mk3(tri.a[0], tri.a[1], tri.a[2]);
  v3 e1 = sub3(mk3(tri.b[0], tri.b[1], tri.b[2]), a);
  v3 e2 = sub3(mk3(tri.c[0], tri.c[1], tri.c[2]), a);
  v3 p = cross3(d, e2);
  float det = dot3(e1, p);
  if (fabsf(det * inv_det) < 1e-9f) return false;
  float inv = 1.0f / det;
  v3 sv = sub3(o, a);
  float u = dot3(sv, p) * inv;
  if (u < 0.0f || u > 1.0f) return false;
  v3 q = cross3(sv, e1);
  float v = dot3(d, q) * inv;
  if (v < 0.0f || u + v > 1.0f) return false;
  float t = dot3(e2, q) * inv;
  if (t <= 0.0001f || t >= limit) return false;
  if (clipped_at(s.surfaces[record], add3(wo, scl3(wd, t)))) return false;
  return true;
}

// scene() (trace.wgsl:999-1075) and occluded() (:1096-1168) share the walk;
// `any` selects occluded().  Counts: one box test per popped node, one
// triangle test per leaf slot visited.
Walk walk(const Scene& s, v3 o, v3 d, float limit, bool any, uint32_t* boxes, uint32_t* tris, uint32_t* overflow) {
  Walk hit{limit, 0u, 0u, false, 0.0f, 0.0f};
  if (s.tri_count == 0 || s.node_count == 0) return hit;
  uint32_t stack[64];
  uint32_t top = 1u;
  stack[0] = 0u;
  v3 ro = o, rd = d;
  uint32_t base = 0u, record = 0u, word = 0u;
  float inv_det = 1.0f;
  while (top > 0u) {
    top -= 1u;
    uint32_t index = stack[top];
    if (index == ENTRYPOINT_SENTINEL) {
      ro = o;
      rd = d;
      base = 0u;
      record = 0u;
      word = 0u;
      inv_det = 1.0f;
      continue;
    }
    const Node& node = s.nodes[index];
    if (boxes) *boxes += 1u;
    if (!box_hit(node, ro, rd, any ? limit : hit.t)) continue;
    if (node.pad[0] == INSTANCE_LEAF) {
      if (top + 2u <= 64u) {
        stack[top] = ENTRYPOINT_SENTINEL;
        stack[top + 1u] = node.first;
        top += 2u;
        base = node.count;
        record = f2bits(node.lo[3]);
        const Surface& surf = s.surfaces[record];
        word = surf.info[0];
        inv_det = bits2f(surf.info[3]);
        if (node.pad[1] > 0u) {
          const Node& m = s.nodes[node.pad[1]];
          ro = to_object(m, o, 1.0f);
          rd = to_object(m, d, 0.0f);
        }
      } else if (overflow) {
        *overflow += 1u;
      }
    } else if (node.count == 0u) {
      if (top + 2u <= 64u) {
        stack[top] = node.first;
        stack[top + 1u] = index + 1u;
        top += 2u;
      } else if (overflow) {
        *overflow += 1u;
      }
    } else {
      for (uint32_t j = 0u; j < node.count; ++j) {
        if (tris) *tris += 1u;
        uint32_t i = base + node.first + j;
        if (any) {
          if (tri_blocks(s, i, record, word, inv_det, ro, rd, o, d, limit)) {
            hit.hit = true;
            hit.t = limit;
            hit.surface = i;
            hit.record = record;
            return hit;
          }
        } else {
          tri_hit(s, i, record, word, inv_det, ro, rd, o, d, false, &hit);
        }
      }
    }
  }
  return hit;
}

}  // namespace

// Shared with render.cpp (the path integrator restatement).
Walk orc_walk(const Scene& s, v3 o, v3 d, float limit, bool any) { return walk(s, o, d, limit, any, nullptr, nullptr, nullptr); }

extern "C" {

int orc_version(void) { return 1; }

// ---------------------------------------------------------------- bvh.rs
// Bvh::build restated (bvh.rs:95-266): triangles as 9 floats each; writes up
// to 2n nodes and n order entries, returns the node count.
static void orc_bounds_point(float lo[3], float hi[3], const float* p) {
  for (int k = 0; k < 3; ++k) {
    lo[k] = fminf(lo[k], p[k]);
    hi[k] = fmaxf(hi[k], p[k]);
  }
}
static float orc_area(const float lo[3], const float hi[3]) {
  float d0 = hi[0] - lo[0], d1 = hi[1] - lo[1], d2 = hi[2] - lo[2];
  if (d0 < 0.0f) return 0.0f;
  return 2.0f * (d0 * d1 + d1 * d2 + d2 * d0);
}
static size_t orc_bin(float value, float lo, float extent) {
  float x = ((value - lo) / extent) * 16.0f;
  x = fminf(fmaxf(x, 0.0f), 15.0f);
  return (size_t)x;
}

struct OrcBuild {
  std::vector<float> blo, bhi, cen;  // per primitive: box lo/hi, centre
  std::vector<uint32_t> order;
  std::vector<Node> nodes;
  size_t leaf, most;
  void split(size_t start, size_t end) {
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    float clo[3] = {INFINITY, INFINITY, INFINITY}, chi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (size_t i = start; i < end; ++i) {
      uint32_t k = order[i];
      orc_bounds_point(lo, hi, &blo[3 * k]);
      orc_bounds_point(lo, hi, &bhi[3 * k]);
      orc_bounds_point(clo, chi, &cen[3 * k]);
    }
    size_t here = nodes.size();
    Node n{};
    for (int k = 0; k < 3; ++k) {
      n.lo[k] = lo[k];
      n.hi[k] = hi[k];
    }
    n.first = (uint32_t)start;
    n.count = (uint32_t)(end - start);
    nodes.push_back(n);
    size_t len = end - start;
    if (len <= leaf) return;
    float best = INFINITY;
    int baxis = 0;
    size_t bbin = 0;
    for (int axis = 0; axis < 3; ++axis) {
      float extent = chi[axis] - clo[axis];
      if (extent <= 1e-9f) continue;
      float bl[16][3], bh[16][3];
      size_t bc[16] = {0};
      for (int b = 0; b < 16; ++b)
        for (int k = 0; k < 3; ++k) {
          bl[b][k] = INFINITY;
          bh[b][k] = -INFINITY;
        }
      for (size_t i = start; i < end; ++i) {
        uint32_t k = order[i];
        size_t b = orc_bin(cen[3 * k + axis], clo[axis], extent);
        orc_bounds_point(bl[b], bh[b], &blo[3 * k]);
        orc_bounds_point(bl[b], bh[b], &bhi[3 * k]);
        bc[b] += 1;
      }
      float areas[16];
      size_t counts[16];
      float gl[3] = {INFINITY, INFINITY, INFINITY}, gh[3] = {-INFINITY, -INFINITY, -INFINITY};
      size_t count = 0;
      for (int b = 0; b < 16; ++b) {
        if (bc[b] > 0) {
          orc_bounds_point(gl, gh, bl[b]);
          orc_bounds_point(gl, gh, bh[b]);
        }
        count += bc[b];
        areas[b] = orc_area(gl, gh);
        counts[b] = count;
      }
      for (int k = 0; k < 3; ++k) {
        gl[k] = INFINITY;
        gh[k] = -INFINITY;
      }
      count = 0;
      for (int b = 15; b >= 1; --b) {
        if (bc[b] > 0) {
          orc_bounds_point(gl, gh, bl[b]);
          orc_bounds_point(gl, gh, bh[b]);
        }
        count += bc[b];
        float cost = areas[b - 1] * (float)counts[b - 1] + orc_area(gl, gh) * (float)count;
        if (counts[b - 1] > 0 && count > 0 && cost < best) {
          best = cost;
          baxis = axis;
          bbin = (size_t)b;
        }
      }
    }
    if (best >= orc_area(lo, hi) * (float)len && len <= most) return;
    size_t mid;
    if (isfinite(best)) {
      float extent = chi[baxis] - clo[baxis];
      size_t l = 0, r = len;
      uint32_t* sl = order.data() + start;
      while (l < r) {
        if (orc_bin(cen[3 * sl[l] + baxis], clo[baxis], extent) < bbin) {
          l += 1;
        } else {
          r -= 1;
          std::swap(sl[l], sl[r]);
        }
      }
      mid = (l == 0 || l == len) ? start + len / 2 : start + l;
    } else {
      mid = start + len / 2;
    }
    split(start, mid);
    size_t right = nodes.size();
    split(mid, end);
    nodes[here].first = (uint32_t)right;
    nodes[here].count = 0;
  }
};

uint32_t orc_bvh_build(const float* vertices, uint32_t n, void* nodes_out, uint32_t* order_out) {
  OrcBuild b;
  b.leaf = 4;
  b.most = 16;
  b.blo.resize(3 * (size_t)n);
  b.bhi.resize(3 * (size_t)n);
  b.cen.resize(3 * (size_t)n);
  for (uint32_t i = 0; i < n; ++i) {
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int c = 0; c < 3; ++c) orc_bounds_point(lo, hi, &vertices[9 * (size_t)i + 3 * c]);
    for (int k = 0; k < 3; ++k) {
      b.blo[3 * i + k] = lo[k];
      b.bhi[3 * i + k] = hi[k];
      b.cen[3 * i + k] = (lo[k] + hi[k]) * 0.5f;
    }
  }
  b.order.resize(n);
  for (uint32_t i = 0; i < n; ++i) b.order[i] = i;
  if (n) b.split(0, n);
  memcpy(nodes_out, b.nodes.data(), b.nodes.size() * sizeof(Node));
  memcpy(order_out, b.order.data(), (size_t)n * 4);
  return (uint32_t)b.nodes.size();
}

// Bvh::intersect (bvh.rs:135-164) over triangles in input order; returns the
// triangle index or -1.
int32_t orc_bvh_intersect(const void* nodes_in, uint32_t node_count, const uint32_t* order, const float* vertices,
                          const float* o, const float* d, float limit) {
  const Node* nodes = (const Node*)nodes_in;
  if (node_count == 0) return -1;
  v3 ro = mk3(o[0], o[1], o[2]), rd = mk3(d[0], d[1], d[2]);
  std::vector<uint32_t> stack{0u};
  bool found = false;
  float best = limit;
  int32_t index_out = -1;
  while (!stack.empty()) {
    uint32_t index = stack.back();
    stack.pop_back();
    const Node& node = nodes[index];
    float max = found ? best : limit;
    if (!bvh_box_hit(node, ro, rd, max)) continue;
    if (node.count == 0) {
      stack.push_back(node.first);
      stack.push_back(index + 1);
    } else {
      for (uint32_t k = node.first; k < node.first + node.count; ++k) {
        uint32_t i = order[k];
        float dist;
        if (bvh_triangle_hit(&vertices[9 * (size_t)i], ro, rd, found ? best : limit, &dist)) {
          best = dist;
          found = true;
          index_out = (int32_t)i;
        }
      }
    }
  }
  return index_out;
}

// Brute force with the same triangle test (the reference test's baseline):
// the smallest distance wins; ties keep the lowest index (min_by keeps the
// first of equal minima).
int32_t orc_brute_intersect(const float* vertices, uint32_t n, const float* o, const float* d, float limit) {
  v3 ro = mk3(o[0], o[1], o[2]), rd = mk3(d[0], d[1], d[2]);
  int32_t best_i = -1;
  float best = 0.0f;
  for (uint32_t i = 0; i < n; ++i) {
    float dist;
    if (bvh_triangle_hit(&vertices[9 * (size_t)i], ro, rd, limit, &dist)) {
      if (best_i < 0 || dist < best) {
        best = dist;
        best_i = (int32_t)i;
      }
    }
  }
  return best_i;
}

// ------------------------------------------------------------ traversal
// scene() / occluded() over ray batches on the SceneBuffers layouts.
// counts (optional): 2 u32 per ray (box tests, triangle tests).
int orc_trace(const void* nodes, uint32_t node_count, const void* tris, uint32_t tri_count, const void* surfaces,
              const void* rays_in, uint32_t n, int any, void* hits_out, uint32_t* counts, uint32_t* overflow) {
  Scene s{(const Node*)nodes, node_count, (const Tri*)tris, tri_count, (const Surface*)surfaces};
  const RayIn* rays = (const RayIn*)rays_in;
  HitOut* hits = (HitOut*)hits_out;
  std::atomic<uint32_t> of{0};
  parallel_for((int64_t)n, 256, [&](int64_t i, unsigned) {
    const RayIn& r = rays[i];
    uint32_t b = 0, t = 0, o_ = 0;
    Walk w = walk(s, mk3(r.o[0], r.o[1], r.o[2]), mk3(r.d[0], r.d[1], r.d[2]), r.tmax, any != 0, &b, &t, &o_);
    if (o_) of += o_;
    hits[i].t = w.t;
    hits[i].slot = w.surface;
    hits[i].record = w.record;
    hits[i].hit = w.hit ? 1u : 0u;
    if (counts) {
      counts[2 * i] = b;
      counts[2 * i + 1] = t;
    }
  });
  if (overflow) *overflow = of.load();
  return 0;
}

}  // extern "C"

// ================================================================ sobol.rs
namespace {
const uint32_t ORC_XORS[4][32] = {
    {0},
    {0x00000000, 0x00000001, 0x00000001, 0x00000007, 0x00000001, 0x00000013, 0x00000015, 0x0000007f,
     0x00000001, 0x00000103, 0x00000105, 0x0000070f, 0x00000111, 0x00001333, 0x00001555, 0x00007fff,
     0x00000001, 0x00010003, 0x00010005, 0x0007000f, 0x00010011, 0x00130033, 0x00150055, 0x007f00ff,
     0x00010101, 0x01030303, 0x01050505, 0x070f0f0f, 0x01111111, 0x13333333, 0x15555555, 0x7fffffff},
    {0x00000000, 0x00000001, 0x00000003, 0x00000001, 0x00000005, 0x0000001f, 0x0000002b, 0x0000003d,
     0x00000011, 0x00000133, 0x00000377, 0x00000199, 0x00000445, 0x00001ccf, 0x00002ddb, 0x0000366d,
     0x00000101, 0x00010303, 0x00030707, 0x00010909, 0x00051515, 0x001f3f3f, 0x002b6b6b, 0x003dbdbd,
     0x00101011, 0x01303033, 0x03707077, 0x01909099, 0x04515145, 0x1cf3f3cf, 0x2db6b6db, 0x36dbdb6d},
    {0x00000000, 0x00000001, 0x00000000, 0x00000003, 0x0000000d, 0x0000000c, 0x00000005, 0x0000004f,
     0x00000014, 0x000000e7, 0x00000329, 0x0000039c, 0x00000011, 0x00001033, 0x00000044, 0x000030bb,
     0x0000d1cd, 0x0000c2ec, 0x00005415, 0x0004fc3f, 0x00015054, 0x000e5c97, 0x0032e5b9, 0x0039725c,
     0x00000101, 0x01000303, 0x00000404, 0x03000b0b, 0x0d001d1d, 0x0c002c2c, 0x05004545, 0x4f00cfcf},
};
uint32_t rotl(uint32_t x, int k) { return (x << k) | (x >> (32 - k)); }
uint32_t orc_hash_hp(uint32_t i) {  // sobol.rs:66-73
  i ^= i >> 16;
  i *= 0x21f0aaadu;
  i ^= i >> 15;
  i *= 0xd35a2d97u;
  i ^= i >> 15;
  return i ^ 0xe6fe3bebu;
}
}  // namespace

extern "C" {

// sobol.rs:84-103 (Cycles lookup3 hash of two words)
uint32_t orc_hash_uint2(uint32_t kx, uint32_t ky) {
  uint32_t a = 0xdeadbeefu + ((2u << 2) + 13u);
  uint32_t b = a + ky;
  uint32_t c = a;
  a += kx;
  c ^= b;
  c -= rotl(b, 14);
  a ^= c;
  a -= rotl(c, 11);
  b ^= a;
  b -= rotl(a, 25);
  c ^= b;
  c -= rotl(b, 16);
  a ^= c;
  a -= rotl(c, 4);
  b ^= a;
  b -= rotl(a, 14);
  c ^= b;
  return c - rotl(b, 24);
}

uint32_t orc_animated_seed(uint32_t seed, uint32_t frame) { return orc_hash_uint2(frame, seed); }

// sobol.rs:33-39
uint32_t orc_sequence_size(uint32_t samples) {
  uint64_t s = samples ? samples : 1u;
  uint64_t p = 1;
  while (p < s) p <<= 1;
  if (p > 0xffffffffull) p = 8192;
  return (uint32_t)std::min<uint64_t>(std::max<uint64_t>(p, 256), 8192);
}

// sobol.rs:109-136
void orc_generate_4d(float* points, uint32_t size, uint32_t seed) {
  if (size == 0) return;
  uint32_t s19 = 0x44605a73u;
  s19 ^= s19 << 19;
  uint32_t rng = orc_hash_hp(seed ^ s19);
  auto next = [&]() {
    float v = (float)orc_hash_hp(rng) * (1.0f / 4294967808.0f);
    rng += 1u;
    return v;
  };
  for (int k = 0; k < 4; ++k) points[k] = next();
  uint32_t log_n = 0, n = 1;
  while (n < size) {
    float strata = (float)(n * 2);
    for (uint32_t i = 0; i < n && n + i < size; ++i) {
      for (int axis = 0; axis < 4; ++axis) {
        float src = points[(size_t)(i ^ ORC_XORS[axis][log_n]) * 4 + axis];
        uint32_t occupied = f2u(src * strata);
        points[(size_t)(n + i) * 4 + axis] = ((float)(occupied ^ 1u) + next()) / strata;
      }
    }
    log_n += 1;
    n *= 2;
  }
}

// ============================================================= adaptive.rs
// Adaptive::automatic_min_samples (adaptive.rs:38-40) with powf(0.3) from the
// host libm, as the reference's Rust does.
uint32_t orc_automatic_min_samples(float threshold) {
  float v = ceilf(16.0f / powf(threshold, 0.3f));
  uint32_t n = f2u(v);
  return n > 4u ? n : 4u;
}

// error (adaptive.rs:375-385)
float orc_adaptive_error(const float* prior, float prior_count, const float* now, float count) {
  if (prior_count <= 0.0f || count <= prior_count) return 1e9f;
  float scale = sqrtf(1.0f / count) / sqrtf(1.0f / prior_count + 1.0f / (count - prior_count));
  float gap[4];
  for (int k = 0; k < 4; ++k) {
    float rest = (now[k] * count - prior[k] * prior_count) / (count - prior_count);
    gap[k] = fabsf(prior[k] - rest) * scale;
  }
  return (gap[0] + gap[1] + gap[2]) / (1e-4f + sqrtf(fmaxf(now[0] + now[1] + now[2], 0.0f))) + gap[3];
}

// LocalLight::falloff (lights.rs:155-163)
float orc_falloff(float intensity, float radius, float range, float distance) {
  if (distance >= range || distance <= 1e-6f) return 0.0f;
  float ratio = distance / range;
  float r2 = ratio * ratio;
  float window = fminf(fmaxf(1.0f - r2 * r2, 0.0f), 1.0f);
  float reach = fmaxf(distance, radius);
  return intensity * window * window / (reach * reach);
}

}  // extern "C"

// ======================================================= division identity
namespace {
uint64_t splitmix(uint64_t& s) {
  uint64_t z = (s += 0x9e3779b97f4a7c15ull);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}
}  // namespace

extern "C" {
// Number of (x, d) pairs, over four input families, where the shared
// div_rn (pfxt_math.h) differs from IEEE division.  The kernels compute every
// slab quotient with div_rn; the oracle divides.
uint64_t orc_check_div(uint64_t per_family, uint64_t seed) {
  uint64_t bad = 0;
  for (int fam = 0; fam < 4; ++fam) {
    uint64_t s = seed * 4 + fam;
    for (uint64_t i = 0; i < per_family; ++i) {
      uint64_t r = splitmix(s);
      float x, d;
      if (fam == 0) {
        x = bits2f((uint32_t)r);
        d = bits2f((uint32_t)(r >> 32));
        if (!isfinite(x) || !isfinite(d) || fabsf(d) < 1e-12f) continue;
      } else if (fam == 1) {
        x = ((float)(uint32_t)r * 0x1p-32f - 0.5f) * 2000.0f - ((float)(uint32_t)(r >> 32) * 0x1p-32f) * 1000.0f;
        d = (float)(uint32_t)(r >> 16) * 0x1p-32f * 2.0f - 1.0f;
        if (fabsf(d) < 1e-12f) continue;
      } else if (fam == 2) {
        x = bits2f(0x3f800000u | ((uint32_t)r & 0x7fffffu));
        d = bits2f(0x3f800000u | ((uint32_t)(r >> 32) & 0x7fffffu));
      } else {
        x = ((float)(uint32_t)r * 0x1p-32f - 0.5f) * 100.0f;
        d = bits2f(0x2b8cbcccu + (uint32_t)((r >> 32) % 0x14000000u));
        if (r & 1) d = -d;
      }
      float a = x / d, b = div_rn(x, d, 1.0f / d);
      if (f2bits(a) != f2bits(b) && !(a == 0.0f && b == 0.0f)) ++bad;
    }
  }
  return bad;
}

// The shared transcendentals over an array, for their accuracy test:
// fn 0 sin, 1 cos, 2 asin, 3 acos, 4 atan2(x, y), 5 exp, 6 log, 7 pow(x, y).
void orc_math(int fn, const float* x, const float* y, float* out, uint64_t n) {
  for (uint64_t i = 0; i < n; ++i) {
    float a = x[i], b = y ? y[i] : 0.0f, r = 0.0f;
    switch (fn) {
      case 0: r = sin_(a); break;
      case 1: r = cos_(a); break;
      case 2: r = asin_(a); break;
      case 3: r = acos_(a); break;
      case 4: r = atan2_(a, b); break;
      case 5: r = exp_(a); break;
      case 6: r = log_(a); break;
      case 7: r = pow_(a, b); break;
      default: break;
    }
    out[i] = r;
  }
}
}  // extern "C"

// The path integrator restatement and the scene packing share this
// translation unit.
#include "render.cpp"
#include "pack.cpp"
