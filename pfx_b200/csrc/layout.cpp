// Reference node array (bvh.rs Node, 48 B) -> B200 traversal layout.
//
// Every inner node X of the reference BVH2 becomes one 64-byte WideNode that
// holds the fp32 boxes of both children (X+1 and X.first).  The box arithmetic
// that the reference runs when it pops a child (trace.wgsl:453-468 box_hit) is
// run on the same fp32 numbers when the parent is opened, so one 4 x 16 B load
// feeds two box tests.  The visiting order stays the reference's left-first
// depth-first order, and the part of box_hit that depends on the current hit
// distance (near <= hit.t) is re-checked when an entry is popped, so the set and
// the order of triangle tests equal the reference's.
//
// The scene root and every bottom-level root get a "pseudo-parent" wide node
// whose child 0 is the root, so that the root box is tested exactly as the
// reference tests it after popping index 0 (or after entering an instance).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <unordered_map>

#include "pfxt_internal.h"

namespace pfxt {

namespace {

struct Builder {
  const GpuNode* nodes;
  size_t node_count;
  const GpuSurface* surfaces;
  size_t surface_count;
  uint64_t tri_count;
  TraversalLayout out;
  std::unordered_map<uint32_t, uint32_t> pseudo_of;  // reference root -> pseudo-parent wide index

  void set_box(WideNode& w, int child, const GpuNode& n) {
    float* f = &w.b0[0];  // b0, b1, b2 are contiguous: 12 floats
    for (int k = 0; k < 3; ++k) {
      f[child * 6 + k] = n.lo[k];
      f[child * 6 + 3 + k] = n.hi[k];
    }
  }

  // Largest leaf end (first + count) under each pseudo-parent, so that every
  // slot a kernel can reach is checked against the triangle count.
  std::unordered_map<uint32_t, uint64_t> reach_of;
  uint64_t reach = 0;  // running maximum while one subtree is laid out

  uint32_t leaf_ref(const GpuNode& n) {
    if (n.count == 0 || n.count > 16) throw Invalid("BVH leaf holds more than 16 triangles");
    if (n.first > LEAF_FIRST_MASK) throw Invalid("BVH leaf offset exceeds the traversal encoding");
    reach = std::max<uint64_t>(reach, (uint64_t)n.first + n.count);
    return REF_LEAF | ((n.count - 1u) << LEAF_FIRST_BITS) | n.first;
  }

  uint32_t inst_ref(const GpuNode& n) {
    InstRec r{};
    uint32_t record = f2bits(n.lo[3]);
    if (record >= surface_count) throw Invalid("instance record out of range");
    const GpuSurface& s = surfaces[record];
    r.record = record;
    r.base = n.count;
    r.word = s.info[0];
    r.inv_det = bits2f(s.info[3]);
    r.transformed = n.pad[1] > 0 ? 1u : 0u;
    if (r.transformed) {
      if (n.pad[1] >= node_count) throw Invalid("instance rows out of range");
      const GpuNode& m = nodes[n.pad[1]];
      for (int k = 0; k < 4; ++k) {
        r.inv[0][k] = m.lo[k];
        r.inv[1][k] = m.hi[k];
      }
      r.inv[2][0] = bits2f(m.first);
      r.inv[2][1] = bits2f(m.count);
      r.inv[2][2] = bits2f(m.pad[0]);
      r.inv[2][3] = bits2f(m.pad[1]);
    }
    if (n.first >= node_count) throw Invalid("instance root out of range");
    uint64_t outer = reach;
    reach = 0;
    r.root = pseudo(n.first);
    uint64_t inner = reach_of[r.root];
    reach = outer;
    if ((uint64_t)r.base + inner > tri_count) throw Invalid("an instance leaf reaches past the triangles");
    uint32_t index = (uint32_t)out.insts.size();
    if (index >= (1u << 30)) throw Invalid("too many instances");
    out.insts.push_back(r);
    return REF_INST | index;
  }

  // Reference of child node `i` as seen from its parent.
  uint32_t child_ref(uint32_t i) {
    const GpuNode& n = nodes[i];
    if (n.pad[0] == INSTANCE_LEAF) return inst_ref(n);
    if (n.count == 0) return wide_of(i);
    return leaf_ref(n);
  }

  uint32_t pseudo(uint32_t root) {
    auto it = pseudo_of.find(root);
    if (it != pseudo_of.end()) return it->second;
    uint32_t w = (uint32_t)out.wide.size();
    out.wide.push_back(WideNode{});
    pseudo_of[root] = w;
    uint64_t outer = reach;
    reach = 0;
    WideNode node{};
    set_box(node, 0, nodes[root]);
    node.child[0] = child_ref(root);
    node.child[1] = REF_NONE;
    out.wide[w] = node;
    reach_of[w] = reach;
    reach = outer;
    return w;
  }

  // Wide node of inner node `i`; children are laid out depth first, left first.
  uint32_t wide_of(uint32_t i) {
    const GpuNode& n = nodes[i];
    uint32_t left = i + 1, right = n.first;
    if (left >= node_count || right >= node_count) throw Invalid("BVH child out of range");
    uint32_t w = (uint32_t)out.wide.size();
    out.wide.push_back(WideNode{});
    WideNode node{};
    set_box(node, 0, nodes[left]);
    set_box(node, 1, nodes[right]);
    node.child[0] = child_ref(left);
    node.child[1] = child_ref(right);
    out.wide[w] = node;
    return w;
  }
};

}  // namespace

TraversalLayout make_layout(const pfxt_buffers& b) {
  Builder builder;
  builder.nodes = (const GpuNode*)b.nodes;
  builder.node_count = b.nodes_bytes / sizeof(GpuNode);
  builder.surfaces = (const GpuSurface*)b.surfaces;
  builder.surface_count = b.surfaces_bytes / sizeof(GpuSurface);
  builder.tri_count = b.triangles_bytes / sizeof(GpuTriangle);
  if (b.triangle_count != builder.tri_count) throw Invalid("triangle count does not match the triangle buffer");
  if (builder.node_count > 0 && b.triangle_count > 0) {
    builder.out.wide.reserve(builder.node_count / 2 + 16);
    builder.out.root = builder.pseudo(0);
    // the top level itself: world leaves (base 0) must stay inside the triangles
    if (builder.reach_of[builder.out.root] > builder.tri_count)
      throw Invalid("a BVH leaf reaches past the triangles");
  }
  // The box test needs no range check on its quotients when every box
  // coordinate is 0 or of magnitude in [2^-70, 2^79] (traverse.cuh,
  // BOUNDED_TINY and BOUNDED_COORD); NaN coordinates fail this too.
  builder.out.small = true;
  for (const WideNode& w : builder.out.wide) {
    const float* f = &w.b0[0];
    for (int k = 0; k < 12; ++k) {
      float a = std::fabs(f[k]);
      if (!(a == 0.0f || (a >= 0x1p-70f && a <= 0x1p+79f))) builder.out.small = false;
    }
  }
  const GpuTriangle* tris = (const GpuTriangle*)b.triangles;
  size_t count = b.triangles_bytes / sizeof(GpuTriangle);
  builder.out.tris.resize(count);
  for (size_t i = 0; i < count; ++i) {
    const GpuTriangle& t = tris[i];
    TravTri& o = builder.out.tris[i];
    for (int k = 0; k < 3; ++k) {
      o.a[k] = t.a[k];
      o.e1[k] = t.b[k] - t.a[k];  // tri_hit: e1 = tri.b.xyz - tri.a.xyz
      o.e2[k] = t.c[k] - t.a[k];  // e2 = tri.c.xyz - tri.a.xyz
    }
    o.a[3] = 0.0f;
    o.e1[3] = 0.0f;
    o.e2[3] = 0.0f;
  }
  return std::move(builder.out);
}

}  // namespace pfxt
