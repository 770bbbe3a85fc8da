// Packed scene layouts.
//
// Two families live here:
//  * the reference's SceneBuffers records (crates/trace/src/gpu.rs:19-26
//    GpuTriangle 96 B, bvh.rs:7-13 Node 48 B, lights.rs:247-252 GpuLight 64 B,
//    lights.rs:256-261 GpuEmitter 64 B, gpu.rs:29-38 GpuSurface 176 B,
//    record.rs:18-27 Hot 128 B).  They are the drop-in seam: a host that already
//    packs SceneBuffers hands these bytes over unchanged;
//  * the B200 traversal layout derived from them on upload: 64-byte two-box
//    nodes (both children's fp32 boxes in the parent, one 4 x 16 B fetch per
//    pair of box tests), 48-byte triangles (vertex a and the two edges,
//    precomputed with the same fp32 subtraction the reference does per test) and
//    64-byte instance records.
#pragma once
#include <stdint.h>

namespace pfxt {

// ------------------------------------------------ reference SceneBuffers rows
struct alignas(16) GpuTriangle {  // gpu.rs:19-26
  float a[4];  // a.w = material
  float b[4];  // b.w = flag word (0 in SceneBuffers::build)
  float c[4];  // c.w = 1-based emitter index, 0 = not sampled
  float na[4], nb[4], nc[4];  // normals, w = u coordinate of the vertex
};
static_assert(sizeof(GpuTriangle) == 96, "GpuTriangle");

struct alignas(16) GpuNode {  // bvh.rs:7-13
  float lo[4];  // lo.w = instance record bits on top-level instance leaves
  float hi[4];
  uint32_t first, count;  // count 0: inner node, right child = first, left = index+1
  uint32_t pad[2];        // pad.x = 1 on instance leaves, pad.y = inverse-rows node
};
static_assert(sizeof(GpuNode) == 48, "GpuNode");

struct alignas(16) GpuLight {  // lights.rs:247-252
  float a[4], b[4], c[4], d[4];
};
static_assert(sizeof(GpuLight) == 64, "GpuLight");

struct alignas(16) GpuEmitter {  // lights.rs:256-261
  float a[4], b[4], c[4], emission[4];
};
static_assert(sizeof(GpuEmitter) == 64, "GpuEmitter");

struct alignas(16) GpuSurface {  // gpu.rs:29-38
  float clip0[4], clip1[4], transform[4], crop[4];
  uint32_t info[4];  // word, material (NO_MATERIAL = all), alpha cutoff bits, inverse det bits
  float forward[3][4];
  float inverse[3][4];
};
static_assert(sizeof(GpuSurface) == 176, "GpuSurface");

struct alignas(16) GpuHot {  // record.rs:18-27
  float base_roughness[4];
  float metal_spec_coat[4];
  float sheen_trans_ior_disp[4];
  float thick_sub_film[4];
  float tint_absorption[4];
  float emission_film[4];
  float extension[4];  // fresnel power, flag bits, first extension row, uvs1
  float wet[4];
};
static_assert(sizeof(GpuHot) == 128, "GpuHot");

// Instance word bits (gpu.rs:125-133).
constexpr uint32_t SHADOW_ONLY = 1u;
constexpr uint32_t CASTS_NO_SHADOW = 2u;
constexpr uint32_t CUTOUT = 4u;
constexpr uint32_t ONE_SIDED = 1u << 23;
constexpr uint32_t NO_MATERIAL = 0xffffffffu;
constexpr uint32_t INSTANCE_LEAF = 1u;

// ------------------------------------------------- B200 traversal layout
// Child reference inside a wide node.
//   bit31 = 0            : inner node, index into the wide-node array
//   bit31 = 1, bit30 = 0 : triangle leaf, bits 0..25 first slot (before the
//                          instance base is added), bits 26..29 count-1
//   bit31 = 1, bit30 = 1 : instance leaf, bits 0..29 instance record
//   0xffffffff           : no child
constexpr uint32_t REF_NONE = 0xffffffffu;
constexpr uint32_t REF_LEAF = 0x80000000u;
constexpr uint32_t REF_INST = 0xc0000000u;
constexpr uint32_t LEAF_FIRST_BITS = 26u;
constexpr uint32_t LEAF_FIRST_MASK = (1u << LEAF_FIRST_BITS) - 1u;

struct alignas(16) WideNode {
  // child 0 box: lo(x,y,z) hi(x,y,z); child 1 box likewise
  float b0[4];  // l.lo.x l.lo.y l.lo.z l.hi.x
  float b1[4];  // l.hi.y l.hi.z r.lo.x r.lo.y
  float b2[4];  // r.lo.z r.hi.x r.hi.y r.hi.z
  uint32_t child[2];
  uint32_t pad[2];
};
static_assert(sizeof(WideNode) == 64, "WideNode");

struct alignas(16) TravTri {
  float a[4];   // a.xyz
  float e1[4];  // b - a
  float e2[4];  // c - a
};
static_assert(sizeof(TravTri) == 48, "TravTri");

struct alignas(16) InstRec {
  float inv[3][4];     // inverse rows (world -> object), levels.rs:457-467
  uint32_t root;       // wide node whose child 0 is the bottom-level root
  uint32_t base;       // triangle slot base of the mesh
  uint32_t record;     // instance surface record (1-based; 0 = world)
  uint32_t word;       // instance word
  float inv_det;       // inverse determinant (object-space det sign/scale)
  uint32_t transformed;  // 0: the ray stays in world space (the world group)
  uint32_t pad[2];
};
static_assert(sizeof(InstRec) == 80, "InstRec");

// Stack bound of the reference traversal (trace.wgsl:1003, 64 entries).
constexpr uint32_t REF_STACK = 64u;

}  // namespace pfxt
