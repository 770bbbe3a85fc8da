// Host-side scene packing: the C++ restatement of SceneBuffers::build
// (crates/trace/src/gpu.rs:566-1061) for the scope this library covers
// (triangles, instances, materials, local lights, emissive triangles, a uniform
// environment and the Sobol table).  Everything is integer or fp32/fp64 host
// arithmetic in the reference's own order, so the packed bytes are the ones the
// reference would upload for the same scene.
#include <algorithm>
#include <atomic>
#include <array>
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "pfxt.h"
#include "pfxt_internal.h"
#include "pfxt_types.h"

namespace pfxt {

namespace {

constexpr float F32_INF = std::numeric_limits<float>::infinity();
constexpr float F32_MAX = std::numeric_limits<float>::max();

// Rust's f32::min/max: a NaN operand loses.
inline float rmin(float a, float b) { return std::isnan(a) ? b : (std::isnan(b) ? a : (b < a ? b : a)); }
inline float rmax(float a, float b) { return std::isnan(a) ? b : (std::isnan(b) ? a : (b > a ? b : a)); }

struct V3 {
  float v[3];
  float& operator[](int i) { return v[i]; }
  float operator[](int i) const { return v[i]; }
};
inline V3 vsub(const V3& a, const V3& b) { return {{a[0] - b[0], a[1] - b[1], a[2] - b[2]}}; }
inline V3 vadd(const V3& a, const V3& b) { return {{a[0] + b[0], a[1] + b[1], a[2] + b[2]}}; }
inline V3 vscale(const V3& a, float s) { return {{a[0] * s, a[1] * s, a[2] * s}}; }
inline float vdot(const V3& a, const V3& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
inline V3 vcross(const V3& a, const V3& b) {
  return {{a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]}};
}
inline float vlength(const V3& a) { return std::sqrt(vdot(a, a)); }
// math.rs:29-36
inline V3 vnormalize(const V3& a) {
  float len = vlength(a);
  if (len <= 1e-12f) return {{0.0f, 0.0f, 1.0f}};
  return vscale(a, 1.0f / len);
}
inline V3 v3of(const float* p) { return {{p[0], p[1], p[2]}}; }

// ------------------------------------------------------------------ bvh.rs
struct Bounds {
  float lo[3], hi[3];
  static Bounds empty() {
    Bounds b;
    for (int k = 0; k < 3; ++k) {
      b.lo[k] = F32_INF;
      b.hi[k] = -F32_INF;
    }
    return b;
  }
  void point(const float* p) {  // bvh.rs:54-59
    for (int k = 0; k < 3; ++k) {
      lo[k] = rmin(lo[k], p[k]);
      hi[k] = rmax(hi[k], p[k]);
    }
  }
  void grow(const Bounds& o) {  // bvh.rs:60-63
    point(o.lo);
    point(o.hi);
  }
  float area() const {  // bvh.rs:64-71
    float d0 = hi[0] - lo[0], d1 = hi[1] - lo[1], d2 = hi[2] - lo[2];
    if (d0 < 0.0f) return 0.0f;
    return 2.0f * (d0 * d1 + d1 * d2 + d2 * d0);
  }
};

constexpr int BINS = 16;  // bvh.rs:74-76
struct Leaves {
  size_t size, most;
};
constexpr Leaves TRIANGLE_LEAVES{4, 16};
constexpr Leaves INSTANCE_LEAVES{1, 0};

inline size_t bin_of(float value, float lo, float extent) {  // bvh.rs:268-270
  float x = ((value - lo) / extent) * (float)BINS;
  x = rmin(rmax(x, 0.0f), (float)(BINS - 1));
  if (std::isnan(x)) return 0;
  return (size_t)x;
}

struct BvhBuilder {
  const std::vector<Bounds>& boxes;
  std::vector<std::array<float, 3>> centers;
  std::vector<uint32_t> order;
  std::vector<GpuNode> nodes;
  Leaves leaves;

  BvhBuilder(const std::vector<Bounds>& b, Leaves l) : boxes(b), leaves(l) {
    centers.resize(b.size());
    for (size_t i = 0; i < b.size(); ++i)
      for (int k = 0; k < 3; ++k) centers[i][k] = (b[i].lo[k] + b[i].hi[k]) * 0.5f;
    order.resize(b.size());
    for (size_t i = 0; i < b.size(); ++i) order[i] = (uint32_t)i;
    nodes.reserve(2 * b.size());
    if (!b.empty()) split(0, b.size());
  }

  // bvh.rs:167-266
  void split(size_t start, size_t end) {
    Bounds bounds = Bounds::empty(), centroids = Bounds::empty();
    for (size_t i = start; i < end; ++i) {
      bounds.grow(boxes[order[i]]);
      centroids.point(centers[order[i]].data());
    }
    size_t here = nodes.size();
    GpuNode node{};
    for (int k = 0; k < 3; ++k) {
      node.lo[k] = bounds.lo[k];
      node.hi[k] = bounds.hi[k];
    }
    node.first = (uint32_t)start;
    node.count = (uint32_t)(end - start);
    nodes.push_back(node);
    size_t len = end - start;
    if (len <= leaves.size) return;
    float best_cost = F32_INF;
    int best_axis = 0;
    size_t best_bin = 0;
    for (int axis = 0; axis < 3; ++axis) {
      float extent = centroids.hi[axis] - centroids.lo[axis];
      if (extent <= 1e-9f) continue;
      Bounds bin_box[BINS];
      size_t bin_count[BINS];
      for (int b = 0; b < BINS; ++b) {
        bin_box[b] = Bounds::empty();
        bin_count[b] = 0;
      }
      for (size_t i = start; i < end; ++i) {
        uint32_t idx = order[i];
        size_t b = bin_of(centers[idx][axis], centroids.lo[axis], extent);
        bin_box[b].grow(boxes[idx]);
        bin_count[b] += 1;
      }
      float areas[BINS];
      size_t counts[BINS];
      Bounds bound = Bounds::empty();
      size_t count = 0;
      for (int b = 0; b < BINS; ++b) {
        if (bin_count[b] > 0) bound.grow(bin_box[b]);
        count += bin_count[b];
        areas[b] = bound.area();
        counts[b] = count;
      }
      bound = Bounds::empty();
      count = 0;
      for (int b = BINS - 1; b >= 1; --b) {
        if (bin_count[b] > 0) bound.grow(bin_box[b]);
        count += bin_count[b];
        float cost = areas[b - 1] * (float)counts[b - 1] + bound.area() * (float)count;
        if (counts[b - 1] > 0 && count > 0 && cost < best_cost) {
          best_cost = cost;
          best_axis = axis;
          best_bin = (size_t)b;
        }
      }
    }
    if (best_cost >= bounds.area() * (float)len && len <= leaves.most) return;
    size_t mid;
    if (std::isfinite(best_cost)) {
      int axis = best_axis;
      float extent = centroids.hi[axis] - centroids.lo[axis];
      size_t left = 0, right = len;
      uint32_t* slice = order.data() + start;
      while (left < right) {
        if (bin_of(centers[slice[left]][axis], centroids.lo[axis], extent) < best_bin) {
          left += 1;
        } else {
          right -= 1;
          std::swap(slice[left], slice[right]);
        }
      }
      mid = (left == 0 || left == len) ? start + len / 2 : start + left;
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

struct Bvh {
  std::vector<GpuNode> nodes;
  std::vector<uint32_t> order;
  bool gpu = false;  // built on the GPU
};

Bvh bvh_over(const std::vector<Bounds>& boxes, Leaves leaves) {
  BvhBuilder b(boxes, leaves);
  return Bvh{std::move(b.nodes), std::move(b.order), false};
}

// Triangle BVHs of at least this many triangles are built on the GPU when one
// is present; smaller ones take longer to launch than to build on the host.
constexpr size_t GPU_BVH_MIN = 1u << 16;
std::atomic<int> g_gpu_bvh{1};

Bvh bvh_triangles(const pfxt_triangle* tris, size_t n) {  // bvh.rs:95-105
  std::vector<Bounds> boxes(n);
  // no -0.0 and no NaN: the GPU's minima and maxima are then order-free
  auto plain_value = [](float v) { return !std::isnan(v) && !(v == 0.0f && std::signbit(v)); };
  bool plain = true;
  for (size_t i = 0; i < n; ++i) {
    Bounds b = Bounds::empty();
    for (int c = 0; c < 3; ++c) b.point(tris[i].v[c]);
    boxes[i] = b;
    for (int k = 0; k < 3; ++k) plain = plain && plain_value(b.lo[k]) && plain_value(b.hi[k]);
  }
  if (plain && n >= GPU_BVH_MIN && n <= 0xffffffffu && g_gpu_bvh.load() && gpu_bvh_available()) {
    try {
      std::vector<float> flat(6 * n);
      for (size_t i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) {
          flat[6 * i + k] = boxes[i].lo[k];
          flat[6 * i + 3 + k] = boxes[i].hi[k];
        }
      Bvh out;
      gpu_bvh_build(flat.data(), (uint32_t)n, (uint32_t)TRIANGLE_LEAVES.size, (uint32_t)TRIANGLE_LEAVES.most,
                    out.nodes, out.order);
      out.gpu = true;
      return out;
    } catch (const std::exception&) {
      // the host build gives the same bytes
    }
  }
  return bvh_over(boxes, TRIANGLE_LEAVES);
}

// ------------------------------------------------------------ detail.rs Pose
// Transform is column-major: m[column][row] = t[column*4 + row].
struct Pose {
  float m[4][4];
};

bool pose_new(const float* t, Pose* out, std::string* error) {  // detail.rs:190-221
  for (int i = 0; i < 16; ++i)
    if (!std::isfinite(t[i])) {
      *error = "instance transform is not finite";
      return false;
    }
  for (int c = 0; c < 4; ++c)
    for (int r = 0; r < 4; ++r) out->m[c][r] = t[c * 4 + r];
  const float(*m)[4] = out->m;
  if (m[0][3] != 0.0f || m[1][3] != 0.0f || m[2][3] != 0.0f || m[3][3] != 1.0f) {
    *error = "instance transform is not affine";
    return false;
  }
  auto a = [&](int row, int column) { return (double)m[column][row]; };
  auto cofactor = [&](int row, int column) {
    int r0 = (row + 1) % 3, r1 = (row + 2) % 3, c0 = (column + 1) % 3, c1 = (column + 2) % 3;
    return a(r0, c0) * a(r1, c1) - a(r0, c1) * a(r1, c0);
  };
  double determinant = 0.0;
  for (int c = 0; c < 3; ++c) determinant += a(0, c) * cofactor(0, c);
  double volume = 1.0;
  for (int c = 0; c < 3; ++c) {
    double s = 0.0;
    for (int r = 0; r < 3; ++r) s += a(r, c) * a(r, c);
    volume *= std::sqrt(s);
  }
  if (std::fabs(determinant) <= volume * 1e-6) {
    *error = "instance transform is singular";
    return false;
  }
  return true;
}

// Pose::point (detail.rs:232-240): m[3][row] + sum over columns.
inline V3 pose_point(const Pose& p, const float* q) {
  V3 r;
  for (int row = 0; row < 3; ++row) {
    float s = (p.m[0][row] * q[0] + p.m[1][row] * q[1]) + p.m[2][row] * q[2];
    r[row] = p.m[3][row] + s;
  }
  return r;
}

// Pose::rows (detail.rs:254-260)
void pose_rows(const Pose& p, float out[12]) {
  const float(*m)[4] = p.m;
  float r[12] = {m[0][0], m[1][0], m[2][0], m[3][0], m[0][1], m[1][1],
                 m[2][1], m[3][1], m[0][2], m[1][2], m[2][2], m[3][2]};
  memcpy(out, r, sizeof(r));
}

// Pose::inverse_rows (detail.rs:262-287)
void pose_inverse_rows(const Pose& p, float out[12]) {
  auto a = [&](int row, int column) { return (double)p.m[column][row]; };
  auto cofactor = [&](int row, int column) {
    int r0 = (row + 1) % 3, r1 = (row + 2) % 3, c0 = (column + 1) % 3, c1 = (column + 2) % 3;
    return a(r0, c0) * a(r1, c1) - a(r0, c1) * a(r1, c0);
  };
  double determinant = 0.0;
  for (int c = 0; c < 3; ++c) determinant += a(0, c) * cofactor(0, c);
  double inverse[3][3];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) inverse[r][c] = cofactor(c, r) / determinant;
  double translation[3] = {(double)p.m[3][0], (double)p.m[3][1], (double)p.m[3][2]};
  for (int r = 0; r < 3; ++r) {
    double shift = 0.0;
    for (int k = 0; k < 3; ++k) shift += inverse[r][k] * translation[k];
    for (int c = 0; c < 3; ++c) out[r * 4 + c] = (float)inverse[r][c];
    out[r * 4 + 3] = (float)(-shift);
  }
}

// Pose::inverse_determinant (detail.rs:223-230)
float pose_inverse_determinant(const Pose& p) {
  auto a = [&](int row, int column) { return (double)p.m[column][row]; };
  double det = a(0, 0) * (a(1, 1) * a(2, 2) - a(1, 2) * a(2, 1)) -
               a(0, 1) * (a(1, 0) * a(2, 2) - a(1, 2) * a(2, 0)) +
               a(0, 2) * (a(1, 0) * a(2, 1) - a(1, 1) * a(2, 0));
  return (float)(1.0 / det);
}

// levels.rs:114-127
Bounds placed_bounds(const Pose& pose, const Bounds& local) {
  Bounds b = Bounds::empty();
  for (int corner = 0; corner < 8; ++corner) {
    float q[3];
    for (int axis = 0; axis < 3; ++axis) q[axis] = ((corner >> axis) & 1) == 0 ? local.lo[axis] : local.hi[axis];
    V3 w = pose_point(pose, q);
    b.point(w.v);
  }
  return b;
}

// levels.rs:58-73, FNV-1a over the f32 bits of vertices, normals and uvs
// (the second uv set is zero here).
uint64_t geometry_hash(const pfxt_triangle* tris, size_t n) {
  uint64_t hash = 0xcbf29ce484222325ull;
  auto mix = [&](float v) {
    uint32_t bits;
    memcpy(&bits, &v, 4);
    hash = (hash ^ (uint64_t)bits) * 0x00000100000001b3ull;
  };
  for (size_t i = 0; i < n; ++i) {
    for (int c = 0; c < 3; ++c)
      for (int k = 0; k < 3; ++k) mix(tris[i].v[c][k]);
    for (int c = 0; c < 3; ++c)
      for (int k = 0; k < 3; ++k) mix(tris[i].n[c][k]);
    for (int c = 0; c < 3; ++c)
      for (int k = 0; k < 2; ++k) mix(tris[i].uv[c][k]);
    for (int c = 0; c < 6; ++c) mix(0.0f);
  }
  return hash;
}

bool same_geometry(const pfxt_triangle& a, const pfxt_triangle& b) {
  return memcmp(a.v, b.v, sizeof(a.v)) == 0 && memcmp(a.n, b.n, sizeof(a.n)) == 0 &&
         memcmp(a.uv, b.uv, sizeof(a.uv)) == 0;
}

// ---------------------------------------------------------------- lights.rs
inline float luminance(const float* v) { return 0.2126f * v[0] + 0.7152f * v[1] + 0.0722f * v[2]; }

bool emits(const float* e) {  // lights.rs:293-298
  for (int k = 0; k < 3; ++k)
    if (!std::isfinite(e[k]) || !(e[k] >= 0.0f)) return false;
  return luminance(e) > 0.0f;
}

float triangle_area(const float v[3][3]) {  // lights.rs:300-305
  V3 a = v3of(v[0]), b = v3of(v[1]), c = v3of(v[2]);
  return 0.5f * vlength(vcross(vsub(b, a), vsub(c, a)));
}

float light_area(const pfxt_light& l) {  // lights.rs:147-153
  if (l.shape == PFXT_LIGHT_RECT) return 4.0f * vlength(vcross(v3of(l.half_u), v3of(l.half_v)));
  if (l.shape == PFXT_LIGHT_DISC) return PFXT_PI_F * l.disc_radius * l.disc_radius;
  return 0.0f;
}

bool light_valid(const pfxt_light& l) {  // lights.rs:102-145
  const float* scal[] = {l.position, l.colour};
  for (auto p : scal)
    for (int k = 0; k < 3; ++k)
      if (!std::isfinite(p[k])) return false;
  if (!std::isfinite(l.intensity) || !std::isfinite(l.radius) || !std::isfinite(l.range)) return false;
  for (int k = 0; k < 3; ++k)
    if (!(l.colour[k] >= 0.0f)) return false;
  if (!(l.intensity >= 0.0f) || !(l.radius >= 0.0f) || !(l.range >= 0.0f)) return false;
  switch (l.shape) {
    case PFXT_LIGHT_POINT:
      return true;
    case PFXT_LIGHT_SPOT: {
      for (int k = 0; k < 3; ++k)
        if (!std::isfinite(l.direction[k])) return false;
      return vlength(v3of(l.direction)) > 1e-6f && std::isfinite(l.inner_deg) && std::isfinite(l.outer_deg) &&
             0.0f <= l.inner_deg && l.inner_deg <= l.outer_deg && l.outer_deg > 0.0f && l.outer_deg <= 90.0f;
    }
    case PFXT_LIGHT_RECT: {
      for (int k = 0; k < 3; ++k)
        if (!std::isfinite(l.half_u[k]) || !std::isfinite(l.half_v[k])) return false;
      float lu = vlength(v3of(l.half_u)), lv = vlength(v3of(l.half_v));
      return lu > 1e-6f && lv > 1e-6f && std::fabs(vdot(v3of(l.half_u), v3of(l.half_v))) <= 1e-4f * lu * lv;
    }
    case PFXT_LIGHT_DISC: {
      for (int k = 0; k < 3; ++k)
        if (!std::isfinite(l.direction[k])) return false;
      return vlength(v3of(l.direction)) > 1e-6f && std::isfinite(l.disc_radius) && l.disc_radius > 1e-6f;
    }
    default:
      return false;
  }
}

bool light_lit(const pfxt_light& l) {  // lights.rs:98-100
  return l.intensity > 0.0f && l.range > 0.0f && (l.colour[0] > 0.0f || l.colour[1] > 0.0f || l.colour[2] > 0.0f);
}

// f32::to_radians: self * (PI / 180) with the constant folded in f32.
inline float to_radians(float deg) { return deg * (PFXT_PI_F / 180.0f); }

void spot_terms(float inner_deg, float outer_deg, float* scale, float* offset) {  // lights.rs:238-243
  float inner = std::cos(to_radians(inner_deg));
  float outer = std::cos(to_radians(outer_deg));
  float s = 1.0f / rmax(inner - outer, 0.001f);
  *scale = s;
  *offset = -outer * s;
}

GpuLight light_pack(const pfxt_light& l) {  // lights.rs:182-235
  GpuLight g{};
  float colour[3];
  for (int k = 0; k < 3; ++k) colour[k] = l.colour[k] * l.intensity;
  float shadow = l.shadow ? 1.0f : 0.0f;
  switch (l.shape) {
    case PFXT_LIGHT_POINT:
      g = GpuLight{{l.position[0], l.position[1], l.position[2], 0.0f},
                   {colour[0], colour[1], colour[2], l.range},
                   {0.0f, 0.0f, 0.0f, l.radius},
                   {0.0f, 0.0f, 0.0f, shadow}};
      break;
    case PFXT_LIGHT_SPOT: {
      float s, o;
      spot_terms(l.inner_deg, l.outer_deg, &s, &o);
      V3 d = vnormalize(v3of(l.direction));
      g = GpuLight{{l.position[0], l.position[1], l.position[2], 1.0f},
                   {colour[0], colour[1], colour[2], l.range},
                   {d[0], d[1], d[2], l.radius},
                   {s, o, 0.0f, shadow}};
      break;
    }
    case PFXT_LIGHT_RECT: {
      float area = light_area(l);
      g = GpuLight{{l.position[0], l.position[1], l.position[2], 2.0f},
                   {colour[0] / area, colour[1] / area, colour[2] / area, F32_MAX},
                   {l.half_u[0], l.half_u[1], l.half_u[2], l.two_sided ? 1.0f : 0.0f},
                   {l.half_v[0], l.half_v[1], l.half_v[2], shadow}};
      break;
    }
    default: {  // disc
      float area = light_area(l);
      V3 n = vnormalize(v3of(l.direction));
      g = GpuLight{{l.position[0], l.position[1], l.position[2], 3.0f},
                   {colour[0] / area, colour[1] / area, colour[2] / area, F32_MAX},
                   {n[0], n[1], n[2], l.two_sided ? 1.0f : 0.0f},
                   {l.disc_radius, 0.0f, 0.0f, shadow}};
      break;
    }
  }
  return g;
}

// ------------------------------------------------------------------ tree.rs
constexpr size_t TREE_LOOPED = 4;  // tree.rs:6-8
constexpr size_t TREE_LEAF = 8;
constexpr int BUCKETS = 12;
constexpr float TAU_F = 2.0f * PFXT_PI_F;
constexpr float FRAC_PI_2_F = PFXT_PI_F / 2.0f;

struct Cone {
  float axis[3];
  float theta_o, theta_e;
  bool is_empty() const { return axis[0] == 0.0f && axis[1] == 0.0f && axis[2] == 0.0f; }
  float measure() const {  // tree.rs:28-41
    if (is_empty()) return 0.0f;
    float theta_w = rmin(theta_o + theta_e, PFXT_PI_F);
    float cos_o = std::cos(theta_o), sin_o = std::sin(theta_o);
    return TAU_F * (1.0f - cos_o) +
           FRAC_PI_2_F * (((2.0f * theta_w * sin_o - std::cos(theta_o - 2.0f * theta_w)) - 2.0f * theta_o * sin_o) + cos_o);
  }
};
const Cone CONE_EMPTY{{0.0f, 0.0f, 0.0f}, std::numeric_limits<float>::min(), std::numeric_limits<float>::min()};

V3 orthogonal(const V3& n) {  // tree.rs:84-91
  V3 helper = std::fabs(n[0]) > 0.1f ? V3{{0.0f, 1.0f, 0.0f}} : V3{{1.0f, 0.0f, 0.0f}};
  return vnormalize(vcross(n, helper));
}

Cone cone_merge(const Cone& self, const Cone& other) {  // tree.rs:43-81
  if (self.is_empty()) return other;
  if (other.is_empty()) return self;
  Cone a = self, b = other;
  if (other.theta_o > self.theta_o) {
    a = other;
    b = self;
  }
  V3 aa = v3of(a.axis), ba = v3of(b.axis);
  float cos_a_b = vdot(aa, ba);
  float theta_d = std::acos(rmin(rmax(cos_a_b, -1.0f), 1.0f));
  float theta_e = rmax(a.theta_e, b.theta_e);
  if (a.theta_o + 5e-4f >= rmin(PFXT_PI_F, theta_d + b.theta_o)) {
    Cone r = a;
    r.theta_e = theta_e;
    return r;
  }
  float theta_o = (theta_d + a.theta_o + b.theta_o) * 0.5f;
  if (theta_o >= PFXT_PI_F) return Cone{{aa[0], aa[1], aa[2]}, PFXT_PI_F, theta_e};
  V3 axis;
  if (cos_a_b < -0.9995f) {
    axis = orthogonal(aa);
  } else {
    float theta_r = theta_o - a.theta_o;
    V3 ortho = vnormalize(vsub(ba, vscale(aa, cos_a_b)));
    axis = vadd(vscale(aa, std::cos(theta_r)), vscale(ortho, std::sin(theta_r)));
  }
  return Cone{{axis[0], axis[1], axis[2]}, theta_o, theta_e};
}

struct Measure {
  float min[3], max[3];
  Cone cone;
  float energy, range;
  static Measure empty() {
    Measure m;
    for (int k = 0; k < 3; ++k) {
      m.min[k] = F32_MAX;
      m.max[k] = -F32_MAX;
    }
    m.cone = CONE_EMPTY;
    m.energy = 0.0f;
    m.range = 0.0f;
    return m;
  }
  void add(const Measure& o) {  // tree.rs:111-122
    if (o.energy == 0.0f) return;
    for (int k = 0; k < 3; ++k) {
      min[k] = rmin(min[k], o.min[k]);
      max[k] = rmax(max[k], o.max[k]);
    }
    cone = cone_merge(cone, o.cone);
    energy += o.energy;
    range = rmax(range, o.range);
  }
  float calculate() const {  // tree.rs:124-132
    if (energy == 0.0f) return 0.0f;
    float s0 = max[0] - min[0], s1 = max[1] - min[1], s2 = max[2] - min[2];
    float area = 2.0f * (s0 * s1 + s1 * s2 + s2 * s0);
    float area_measure = area == 0.0f ? vlength(V3{{s0, s1, s2}}) : area;
    return energy * area_measure * cone.measure();
  }
};

struct TreeEmitter {
  size_t index;
  float centroid[3];
  Measure measure;
};

TreeEmitter tree_emitter(size_t index, const pfxt_light& l) {  // tree.rs:143-174
  Cone cone;
  if (l.shape == PFXT_LIGHT_SPOT) {
    V3 a = vnormalize(v3of(l.direction));
    cone = Cone{{a[0], a[1], a[2]}, 0.0f, rmin(to_radians(l.outer_deg), FRAC_PI_2_F)};
  } else {
    cone = Cone{{0.0f, 0.0f, -1.0f}, PFXT_PI_F, FRAC_PI_2_F};
  }
  float strength[3];
  for (int k = 0; k < 3; ++k) strength[k] = std::fabs(l.colour[k] * l.intensity);
  TreeEmitter e;
  e.index = index;
  for (int k = 0; k < 3; ++k) {
    e.centroid[k] = l.position[k];
    e.measure.min[k] = l.position[k] - l.radius;
    e.measure.max[k] = l.position[k] + l.radius;
  }
  e.measure.cone = cone;
  e.measure.energy = (strength[0] + strength[1] + strength[2]) / 3.0f;
  e.measure.range = l.range;
  return e;
}

struct Bucket {
  bool has = false;
  Measure measure = Measure::empty();
  size_t count = 0;
  void add(const Measure& m) {
    if (!has) {
      has = true;
      measure = Measure::empty();
    }
    measure.add(m);
    count += 1;
  }
  Bucket plus(const Bucket& o) const {  // tree.rs:189-198
    Bucket r;
    r.has = true;
    r.measure = has ? measure : Measure::empty();
    if (o.has) r.measure.add(o.measure);
    r.count = count + o.count;
    return r;
  }
  float cost() const { return has ? measure.calculate() : 0.0f; }
};

bool treed(const pfxt_light& l) {  // tree.rs:205-207
  return light_lit(l) && (l.shape == PFXT_LIGHT_POINT || l.shape == PFXT_LIGHT_SPOT);
}

GpuLight tree_row(const Measure& m, size_t count, size_t link) {  // tree.rs:295-317
  return GpuLight{{m.min[0], m.min[1], m.min[2], m.energy},
                  {m.max[0], m.max[1], m.max[2], m.range},
                  {m.cone.axis[0], m.cone.axis[1], m.cone.axis[2], m.cone.theta_o},
                  {m.cone.theta_e, (float)count, (float)link, 0.0f}};
}

// tree.rs:319-395. Returns false for "no split".
bool should_split(const std::vector<TreeEmitter>& em, size_t lo, size_t hi, Measure* out_measure, size_t* middle,
                  int* dim_out) {
  size_t count = hi - lo;
  if (count < 2) {
    *out_measure = em[lo].measure;
    return false;
  }
  size_t mid = count / 2;
  float low[3] = {F32_MAX, F32_MAX, F32_MAX}, high[3] = {-F32_MAX, -F32_MAX, -F32_MAX};
  for (size_t i = lo; i < hi; ++i)
    for (int k = 0; k < 3; ++k) {
      low[k] = rmin(low[k], em[i].centroid[k]);
      high[k] = rmax(high[k], em[i].centroid[k]);
    }
  float extent[3] = {high[0] - low[0], high[1] - low[1], high[2] - low[2]};
  float max_extent = rmax(rmax(rmax(extent[0], extent[1]), extent[2]), 0.0f);
  Measure measure = Measure::empty();
  float total_cost = 0.0f, min_cost = F32_MAX;
  int split_dim = -1;
  for (int dim = 0; dim < 3; ++dim) {
    Bucket buckets[BUCKETS];
    float inv_extent;
    if (extent[dim] == 0.0f) {
      if (dim != 0) continue;
      inv_extent = F32_MAX;
      for (size_t i = lo; i < hi; ++i) buckets[0].add(em[i].measure);
    } else {
      inv_extent = 1.0f / extent[dim];
      for (size_t i = lo; i < hi; ++i) {
        float x = (float)BUCKETS * (em[i].centroid[dim] - low[dim]) * inv_extent;
        int64_t at = std::isnan(x) ? 0 : (x >= 9.2e18f ? INT64_MAX : (x <= -9.2e18f ? INT64_MIN : (int64_t)x));
        at = std::min<int64_t>(std::max<int64_t>(at, 0), BUCKETS - 1);
        buckets[at].add(em[i].measure);
      }
    }
    Bucket left[BUCKETS - 1];
    left[0] = buckets[0];
    for (int i = 1; i < BUCKETS - 1; ++i) left[i] = left[i - 1].plus(buckets[i]);
    if (dim == 0) {
      Bucket all = left[BUCKETS - 2].plus(buckets[BUCKETS - 1]);
      measure = all.has ? all.measure : Measure::empty();
      if (extent[0] == 0.0f && extent[1] == 0.0f && extent[2] == 0.0f) break;
      total_cost = measure.calculate();
      if (total_cost == 0.0f) break;
      if (extent[dim] == 0.0f) continue;
    }
    Bucket right[BUCKETS - 1];
    right[BUCKETS - 2] = buckets[BUCKETS - 1];
    for (int i = BUCKETS - 3; i >= 0; --i) right[i] = right[i + 1].plus(buckets[i + 1]);
    float regularization = max_extent * inv_extent;
    for (int s = 0; s < BUCKETS - 1; ++s) {
      float cost = regularization * (left[s].cost() + right[s].cost());
      if (cost < total_cost && cost < min_cost && left[s].count >= 1 && left[s].count < count) {
        min_cost = cost;
        split_dim = dim;
        mid = left[s].count;
      }
    }
  }
  *out_measure = measure;
  *middle = mid;
  *dim_out = split_dim;
  return min_cost < total_cost || count > TREE_LEAF;
}

// f32::total_cmp as a signed-integer key: -0 < +0, NaNs at the ends.
inline int32_t total_order_key(float f) {
  int32_t i;
  memcpy(&i, &f, 4);
  return i ^ (int32_t)(((uint32_t)(i >> 31)) >> 1);
}

// ------------------------------------------------- Rust's select_nth_unstable
// The reference splits a light-tree node with slice::select_nth_unstable_by
// (tree.rs:281).  The order it leaves on each side is the leaf's light order
// (which tree_leaf's reservoir walk consumes) and the order the next split
// sums its buckets in, so the exact permutation is part of the tree's bytes.
// Restated from the selection algorithm of Rust's core library (core::slice::
// select, Rust 1.81 and later): introselect over the partition of ipnsort
// (Bergdoll and Peters): at most 16 rounds of median-of-3 (a recursive
// pseudo-median from 64 elements) pivots and branchless cyclic Lomuto
// partitions, insertion sort from 16 elements down, Alexandrescu's median of
// medians with ninthers after 16 rounds, and the min/max shortcuts for the
// first and last index.  `less` is a strict weak order.
template <class T, class Less>
struct RustSelect {
  Less less;
  int rounds = 16;  // partition rounds before the deterministic fallback

  static constexpr size_t SMALL = 16;            // insertion sort at or below
  static constexpr size_t PSEUDO_MEDIAN = 64;    // recursive pivot choice from here

  void insertion_sort(T* v, size_t n) {
    for (size_t i = 1; i < n; ++i) {
      if (!less(v[i], v[i - 1])) continue;
      T tail = v[i];
      size_t j = i;
      do {
        v[j] = v[j - 1];
        --j;
      } while (j > 0 && less(tail, v[j - 1]));
      v[j] = tail;
    }
  }
  size_t median3(const T* v, size_t a, size_t b, size_t c) {
    bool x = less(v[a], v[b]), y = less(v[a], v[c]);
    if (x == y) return (less(v[b], v[c]) != x) ? c : b;
    return a;
  }
  size_t median3_rec(const T* v, size_t a, size_t b, size_t c, size_t n) {
    if (n * 8 >= PSEUDO_MEDIAN) {
      size_t n8 = n / 8;
      a = median3_rec(v, a, a + n8 * 4, a + n8 * 7, n8);
      b = median3_rec(v, b, b + n8 * 4, b + n8 * 7, n8);
      c = median3_rec(v, c, c + n8 * 4, c + n8 * 7, n8);
    }
    return median3(v, a, b, c);
  }
  size_t choose_pivot(const T* v, size_t n) {  // n >= 8
    size_t n8 = n / 8;
    if (n < PSEUDO_MEDIAN) return median3(v, 0, n8 * 4, n8 * 7);
    return median3_rec(v, 0, n8 * 4, n8 * 7, n8);
  }
  // Branchless cyclic Lomuto partition of w[0, m) around `pivot`: the first
  // element is lifted out, every later one is written to the front when it
  // is less, and the lifted one is placed last.  Returns the count of less.
  template <class L>
  size_t lomuto_cyclic(T* w, size_t m, const T& pivot, L& lt) {
    if (m == 0) return 0;
    T lifted = w[0];
    size_t gap = 0, num_lt = 0;
    for (size_t right = 1; right < m; ++right) {
      T r = w[right];
      bool is_lt = lt(r, pivot);
      w[gap] = w[num_lt];
      w[num_lt] = r;
      gap = right;
      num_lt += is_lt ? 1 : 0;
    }
    bool is_lt = lt(lifted, pivot);
    w[gap] = w[num_lt];
    w[num_lt] = lifted;
    return num_lt + (is_lt ? 1 : 0);
  }
  // Pivot to the front, partition the rest, pivot between the two sides.
  template <class L>
  size_t partition(T* v, size_t n, size_t pivot, L& lt) {
    std::swap(v[0], v[pivot]);
    const T p = v[0];
    size_t num_lt = lomuto_cyclic(v + 1, n - 1, p, lt);
    std::swap(v[0], v[num_lt]);
    return num_lt;
  }
  size_t min_index(const T* v, size_t n) {
    size_t best = 0;
    for (size_t i = 1; i < n; ++i)
      if (less(v[i], v[best])) best = i;
    return best;
  }
  size_t max_index(const T* v, size_t n) {
    size_t best = 0;
    for (size_t i = 1; i < n; ++i)
      if (less(v[best], v[i])) best = i;
    return best;
  }
  size_t median_idx(const T* v, size_t a, size_t b, size_t c) {
    if (less(v[c], v[a])) std::swap(a, c);
    if (less(v[c], v[b])) return c;
    if (less(v[b], v[a])) return a;
    return b;
  }
  void ninther(T* v, size_t a, size_t b, size_t c, size_t d, size_t e, size_t f, size_t g, size_t h, size_t i) {
    b = median_idx(v, a, b, c);
    h = median_idx(v, g, h, i);
    if (less(v[h], v[b])) std::swap(b, h);
    if (less(v[f], v[d])) std::swap(d, f);
    if (less(v[e], v[d])) {
      // d stays
    } else if (less(v[f], v[e])) {
      d = f;
    } else {
      if (less(v[e], v[b]))
        std::swap(v[e], v[b]);
      else if (less(v[h], v[e]))
        std::swap(v[e], v[h]);
      return;
    }
    if (less(v[d], v[b]))
      d = b;
    else if (less(v[h], v[d]))
      d = h;
    std::swap(v[d], v[e]);
  }
  size_t median_of_ninthers(T* v, size_t n) {
    size_t frac = n <= 1024 ? n / 12 : (n <= 128 * 1024 ? n / 64 : n / 1024);
    size_t pivot = frac / 2;
    size_t lo = n / 2 - pivot, hi = frac + lo;
    size_t gap = (n - 9 * frac) / 4;
    size_t a = lo - 4 * frac - gap, b = hi + gap;
    for (size_t i = lo; i < hi; ++i, a += 3, b += 3) ninther(v, a, i - frac, b, a + 1, i, b + 1, a + 2, i + frac, b + 2);
    median_of_medians(v + lo, frac, pivot);
    return partition(v, n, lo + pivot, less);
  }
  void median_of_medians(T* v, size_t n, size_t k) {
    for (;;) {
      if (n <= SMALL) {
        if (n >= 2) insertion_sort(v, n);
        return;
      }
      if (k == n - 1) {
        std::swap(v[max_index(v, n)], v[k]);
        return;
      }
      if (k == 0) {
        std::swap(v[min_index(v, n)], v[0]);
        return;
      }
      size_t p = median_of_ninthers(v, n);
      if (p == k) return;
      if (p > k) {
        n = p;
      } else {
        v += p + 1;
        n -= p + 1;
        k -= p + 1;
      }
    }
  }
  void select_loop(T* v, size_t n, size_t index) {
    int limit = rounds;
    bool has_ancestor = false;
    T ancestor{};
    for (;;) {
      if (n <= SMALL) {
        if (n >= 2) insertion_sort(v, n);
        return;
      }
      if (limit == 0) {
        median_of_medians(v, n, index);
        return;
      }
      --limit;
      size_t pivot = choose_pivot(v, n);
      // A pivot equal to the left neighbour's (the previous round's) is the
      // smallest value here: split off everything equal to it instead.
      if (has_ancestor && !less(ancestor, v[pivot])) {
        auto not_greater = [this](const T& a, const T& b) { return !less(b, a); };
        size_t mid = partition(v, n, pivot, not_greater) + 1;
        if (mid > index) return;
        v += mid;
        n -= mid;
        index -= mid;
        has_ancestor = false;
        continue;
      }
      size_t mid = partition(v, n, pivot, less);
      if (mid < index) {
        ancestor = v[mid];
        has_ancestor = true;
        v += mid + 1;
        n -= mid + 1;
        index -= mid + 1;
      } else if (mid > index) {
        n = mid;
      } else {
        return;
      }
    }
  }
  void select_nth(T* v, size_t n, size_t index) {
    if (index >= n) throw Invalid("select_nth: index out of range");
    if (index == n - 1)
      std::swap(v[max_index(v, n)], v[index]);
    else if (index == 0)
      std::swap(v[min_index(v, n)], v[0]);
    else
      select_loop(v, n, index);
  }
};

void grow(std::vector<TreeEmitter>& em, size_t lo, size_t hi, size_t start, size_t base, size_t root,
          std::vector<GpuLight>& nodes) {  // tree.rs:263-293
  size_t at = nodes.size();
  nodes.push_back(GpuLight{});
  Measure measure;
  size_t middle = 0;
  int dim = -1;
  bool split = should_split(em, lo, hi, &measure, &middle, &dim);
  if (split) {
    if (dim >= 0) {
      auto by_axis = [dim](const TreeEmitter& l, const TreeEmitter& r) {
        return total_order_key(l.centroid[dim]) < total_order_key(r.centroid[dim]);
      };
      RustSelect<TreeEmitter, decltype(by_axis)> select{by_axis};
      select.select_nth(em.data() + lo, hi - lo, middle);
    }
    grow(em, lo, lo + middle, start, base, root, nodes);
    size_t right_at = root + nodes.size();
    grow(em, lo + middle, hi, start + middle, base, root, nodes);
    nodes[at] = tree_row(measure, 0, right_at);
  } else {
    nodes[at] = tree_row(measure, hi - lo, base + start);
  }
}

struct TreeLaid {
  std::vector<GpuLight> rows;
  size_t looped, tree;
};

TreeLaid tree_lay(const pfxt_light* lights, size_t n) {  // tree.rs:220-261
  size_t treed_count = 0;
  for (size_t i = 0; i < n; ++i) treed_count += treed(lights[i]) ? 1 : 0;
  TreeLaid laid;
  if (treed_count <= TREE_LOOPED) {
    for (size_t i = 0; i < n; ++i) laid.rows.push_back(light_pack(lights[i]));
    laid.looped = n;
    laid.tree = 0;
    return laid;
  }
  for (size_t i = 0; i < n; ++i)
    if (!treed(lights[i])) laid.rows.push_back(light_pack(lights[i]));
  size_t looped = laid.rows.size();
  std::vector<TreeEmitter> em;
  for (size_t i = 0; i < n; ++i)
    if (treed(lights[i])) em.push_back(tree_emitter(i, lights[i]));
  std::vector<GpuLight> nodes;
  size_t count = em.size();
  if (count > 0) grow(em, 0, count, 0, looped, looped + count, nodes);
  for (auto& e : em) laid.rows.push_back(light_pack(lights[e.index]));
  laid.rows.insert(laid.rows.end(), nodes.begin(), nodes.end());
  laid.looped = looped;
  laid.tree = treed_count;
  return laid;
}

// ------------------------------------------------------------ emitter list
struct Candidate {
  float vertices[3][3];
  uint32_t slot, record;
  float emission[3];
};

void build_emitters(const std::vector<Candidate>& cands, size_t lights, size_t tree, std::vector<GpuEmitter>& entries,
                    std::vector<float>& cdf) {  // lights.rs:391-440
  std::vector<double> powers;
  for (auto& c : cands) powers.push_back((double)triangle_area(c.vertices) * (double)luminance(c.emission));
  // Rust's f64 Iterator::sum starts from -0.0 (the additive identity): an
  // empty list's total is -0.0
  double total = -0.0;
  for (double p : powers) total += p;
  entries.clear();
  cdf.clear();
  entries.push_back(GpuEmitter{{(float)cands.size(), (float)lights, (float)total, (float)tree}, {}, {}, {}});
  double running = 0.0;
  for (size_t i = 0; i < cands.size(); ++i) {
    running += powers[i];
    cdf.push_back((float)(running / total));
    float probability = (float)(powers[i] / total);
    const Candidate& c = cands[i];
    entries.push_back(GpuEmitter{{c.vertices[0][0], c.vertices[0][1], c.vertices[0][2], 0.0f},
                                 {c.vertices[1][0], c.vertices[1][1], c.vertices[1][2], (float)c.record},
                                 {c.vertices[2][0], c.vertices[2][1], c.vertices[2][2], triangle_area(c.vertices)},
                                 {c.emission[0], c.emission[1], c.emission[2], probability}});
  }
  if (!cdf.empty()) cdf.back() = 1.0f;
}

// -------------------------------------------------------------- sobol.rs
const uint32_t XORS[4][32] = {
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

inline uint32_t hash_hp_uint(uint32_t i) {  // sobol.rs:66-73
  i ^= i >> 16;
  i *= 0x21f0aaadu;
  i ^= i >> 15;
  i *= 0xd35a2d97u;
  i ^= i >> 15;
  return i ^ 0xe6fe3bebu;
}
inline uint32_t hash_hp_seeded_uint(uint32_t i, uint32_t seed) {
  seed ^= seed << 19;
  return hash_hp_uint(i ^ seed);
}
inline float hash_hp_float(uint32_t i) { return (float)hash_hp_uint(i) * (1.0f / 4294967808.0f); }

void generate_4d(float* points, size_t size, uint32_t seed) {  // sobol.rs:109-136
  if (size == 0) return;
  uint32_t rng = hash_hp_seeded_uint(seed, 0x44605a73u);
  auto next = [&]() {
    float v = hash_hp_float(rng);
    rng += 1u;
    return v;
  };
  for (int k = 0; k < 4; ++k) points[k] = next();
  size_t log_n = 0, n = 1;
  while (n < size) {
    float strata = (float)(n * 2);
    for (size_t i = 0; i < n && n + i < size; ++i) {
      for (int axis = 0; axis < 4; ++axis) {
        float src = points[(i ^ (size_t)XORS[axis][log_n]) * 4 + axis];
        uint32_t occupied = pfxt::f2u(src * strata);
        points[(n + i) * 4 + axis] = ((float)(occupied ^ 1u) + next()) / strata;
      }
    }
    log_n += 1;
    n *= 2;
  }
}

// -------------------------------------------------------------- sky.rs
void sky_cdf_uniform(const float radiance[3], uint32_t width, uint32_t height, std::vector<float>& rows,
                     std::vector<float>& columns, float* total_out) {  // sky.rs:212-275 (diffuse = radiance)
  width = std::max(width, 1u);
  height = std::max(height, 1u);
  rows.assign(height, 0.0f);
  columns.assign((size_t)width * height, 0.0f);
  double total = 0.0;
  float lum = rmax(luminance(radiance), 0.0f);
  for (uint32_t row = 0; row < height; ++row) {
    float theta = PFXT_PI_F * ((float)row + 0.5f) / (float)height;
    float sine = std::sin(theta);
    double row_total = 0.0;
    for (uint32_t col = 0; col < width; ++col) {
      row_total += (double)lum * (double)sine;
      columns[(size_t)row * width + col] = (float)row_total;
    }
    if (row_total > 0.0) {
      for (uint32_t col = 0; col < width; ++col) columns[(size_t)row * width + col] /= (float)row_total;
    } else {
      for (uint32_t col = 0; col < width; ++col) columns[(size_t)row * width + col] = (float)(col + 1) / (float)width;
    }
    total += row_total;
    rows[row] = (float)total;
  }
  if (total > 0.0) {
    for (auto& v : rows) v /= (float)total;
  } else {
    for (uint32_t i = 0; i < height; ++i) rows[i] = (float)(i + 1) / (float)height;
  }
  *total_out = (float)total;
}

// Deepest occupancy the reference's traversal stack can reach on `nodes`
// (trace.wgsl:1003-1060): popping an inner node pushes both children, popping
// an instance leaf pushes a sentinel and the bottom-level root.
uint32_t stack_need(const std::vector<GpuNode>& nodes, uint32_t index, int guard) {
  if (guard > 4096) return 1u << 20;
  const GpuNode& n = nodes[index];
  if (n.pad[0] == INSTANCE_LEAF) {
    uint32_t inner = stack_need(nodes, n.first, guard + 1);
    return std::max<uint32_t>(2u, 1u + inner);
  }
  if (n.count != 0) return 0u;
  uint32_t l = stack_need(nodes, index + 1, guard + 1);
  uint32_t r = stack_need(nodes, n.first, guard + 1);
  return std::max<uint32_t>(std::max<uint32_t>(2u, 1u + l), r);
}

}  // namespace

// Levels::meshes / placed / world (levels.rs:11-48) and the emitter candidates
// with the light counts (gpu.rs:530-540): what moving an instance rewrites.
struct Placing {
  struct Mesh {
    std::vector<pfxt_triangle> triangles;  // local space, BVH order: slot first + j
    uint32_t root, first;
    Bounds bounds;
  };
  struct Placed {
    uint32_t mesh, base, record;
    float transform[16];
    Bounds bounds;
    float inverse[12];
  };
  std::vector<Mesh> meshes;
  std::vector<int> placed_index;  // per instance: index into `placed`, -1 for an empty mesh
  std::vector<Placed> placed;
  bool world = false;
  Bounds world_bounds;
  uint32_t world_root = 0;
  uint32_t top_len = 0;
  std::vector<Candidate> candidates;
  size_t looped = 0, tree = 0;
};

namespace {

// Levels::top (levels.rs:393-470) with `room` = 0, written over nodes
// [0, top_len): the instance BVH over the world and every placed instance,
// leaves patched to enter their group, then one inverse-rows node per group.
void lay_top(const Placing& s, GpuNode* out) {
  struct Group {
    Bounds bounds;
    uint32_t root, base, record;
    const float* inverse;  // null for the world group
  };
  std::vector<Group> groups;
  if (s.world) groups.push_back(Group{s.world_bounds, s.world_root, 0u, 0u, nullptr});
  for (const auto& p : s.placed) groups.push_back(Group{p.bounds, s.meshes[p.mesh].root, p.base, p.record, p.inverse});
  if (groups.empty()) return;
  std::vector<Bounds> boxes;
  for (auto& g : groups) boxes.push_back(g.bounds);
  Bvh top = bvh_over(boxes, INSTANCE_LEAVES);
  uint32_t tree = (uint32_t)top.nodes.size();
  if ((size_t)tree + groups.size() != s.top_len) throw Invalid("the instance BVH does not fill its nodes");
  size_t at = 0;
  for (auto node : top.nodes) {
    if (node.count > 0) {
      uint32_t index = top.order[node.first];
      const Group& g = groups[index];
      node.first = g.root;
      node.count = g.base;
      node.lo[3] = bits2f(g.record);
      node.pad[0] = INSTANCE_LEAF;
      node.pad[1] = g.inverse ? tree + index : 0u;
    }
    out[at++] = node;
  }
  for (auto& g : groups) {
    static const float identity[12] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0};
    const float* r = g.inverse ? g.inverse : identity;
    GpuNode n{};
    for (int k = 0; k < 4; ++k) {
      n.lo[k] = r[k];
      n.hi[k] = r[4 + k];
    }
    n.first = f2bits(r[8]);
    n.count = f2bits(r[9]);
    n.pad[0] = f2bits(r[10]);
    n.pad[1] = f2bits(r[11]);
    out[at++] = n;
  }
}

}  // namespace

// ======================================================================
SceneBlobs* build_scene(const pfxt_scene& scene, const pfxt_settings& settings) {
  auto out = std::make_unique<SceneBlobs>();
  if (scene.light_count > (1u << 16)) throw Invalid("invalid trace light");
  for (uint32_t i = 0; i < scene.light_count; ++i)
    if (!light_valid(scene.lights[i])) throw Invalid("invalid trace light");
  if (scene.material_count == 0 || !scene.materials) throw Invalid("invalid trace scene detail");
  for (uint32_t i = 0; i < 4; ++i)
    if (settings.bounces[i] > 64) throw Invalid("bounces above 64");
  auto finite3 = [](const float* p) { return std::isfinite(p[0]) && std::isfinite(p[1]) && std::isfinite(p[2]); };
  auto broken = [&](const pfxt_triangle& t) {
    for (int c = 0; c < 3; ++c) {
      if (!finite3(t.v[c]) || !finite3(t.n[c]) || !std::isfinite(t.uv[c][0]) || !std::isfinite(t.uv[c][1]))
        return true;
    }
    return t.material >= scene.material_count;
  };
  for (uint32_t i = 0; i < scene.triangle_count; ++i)
    if (broken(scene.triangles[i])) throw Invalid("invalid trace geometry");
  for (uint32_t m = 0; m < scene.mesh_count; ++m)
    for (uint32_t i = 0; i < scene.meshes[m].count; ++i)
      if (broken(scene.meshes[m].triangles[i])) throw Invalid("invalid trace geometry");
  for (uint32_t i = 0; i < scene.instance_count; ++i)
    if (scene.instances[i].mesh >= scene.mesh_count) throw Invalid("instance mesh out of range");

  // ---- material records (record.rs:57-180; no extension rows in this scope)
  std::vector<GpuHot> hot(scene.material_count + 1);
  memset(hot.data(), 0, hot.size() * sizeof(GpuHot));
  for (uint32_t m = 0; m < scene.material_count; ++m) {
    const pfxt_material& s = scene.materials[m];
    GpuHot& h = hot[m + 1];
    float rows[7][4] = {
        {s.base[0], s.base[1], s.base[2], s.roughness},
        {s.metalness, s.specular, s.clearcoat, s.clearcoat_roughness},
        {s.sheen, s.transmission, s.ior, s.dispersion},
        {s.thickness, s.subsurface, s.thin_film, s.thin_film_ior},
        {s.subsurface_tint[0], s.subsurface_tint[1], s.subsurface_tint[2], s.absorption},
        {s.emission[0], s.emission[1], s.emission[2], s.thin_film_amount},
        {s.fresnel_power, 0.0f, 0.0f, 0.0f},
    };
    memcpy(&h, rows, sizeof(rows));
  }
  std::vector<bool> emitting(scene.material_count);
  for (uint32_t m = 0; m < scene.material_count; ++m) emitting[m] = emits(scene.materials[m].emission);

  // ---- instance words and uniqueness (gpu.rs:451-472, 745-759)
  std::vector<uint32_t> words(scene.instance_count);
  std::vector<bool> unique(scene.instance_count);
  for (uint32_t i = 0; i < scene.instance_count; ++i) {
    const pfxt_instance& in = scene.instances[i];
    uint32_t w = 0;
    if (in.shadow_only) w |= SHADOW_ONLY;
    if (!in.casts_shadow) w |= CASTS_NO_SHADOW;
    if (!in.two_sided) w |= ONE_SIDED;
    words[i] = w;
    const pfxt_mesh& mesh = scene.meshes[in.mesh];
    bool emissive = false;
    for (uint32_t t = 0; t < mesh.count && !emissive; ++t) emissive = emitting[mesh.triangles[t].material];
    unique[i] = (w & (SHADOW_ONLY | CUTOUT)) == 0 && emissive;
  }

  // ---- levels::lay (levels.rs:225-383)
  Bvh world_bvh = bvh_triangles(scene.triangles, scene.triangle_count);
  if (world_bvh.gpu) out->gpu_builds += 1;
  struct Mesh {
    uint32_t source;
    std::vector<pfxt_triangle> triangles;  // BVH order
    std::vector<uint32_t> order;
    std::vector<GpuNode> nodes;
    uint32_t root, first;
    Bounds bounds;
    uint64_t hash;
  };
  struct Placed {
    uint32_t mesh, base, record, word;
    bool has_material;
    uint32_t material;
    Bounds bounds;
    float inverse[12];
    Pose pose;
  };
  std::vector<Mesh> meshes;
  std::vector<int> placed_index(scene.instance_count, -1);
  std::vector<Placed> placed;
  std::vector<GpuNode> nodes;
  uint32_t slots = scene.triangle_count;
  if (scene.instance_count == 0) {
    nodes = world_bvh.nodes;
  } else {
    uint32_t next = scene.triangle_count, record = 0;
    struct Known {
      uint32_t source;
      uint64_t hash;
      size_t mesh;
    };
    std::vector<Known> known;
    for (uint32_t i = 0; i < scene.instance_count; ++i) {
      const pfxt_instance& in = scene.instances[i];
      const pfxt_mesh& src = scene.meshes[in.mesh];
      if (src.count == 0) continue;
      Pose pose;
      std::string err;
      if (!pose_new(in.transform, &pose, &err)) throw Invalid(err);
      bool alone = unique[i];
      bool one = true;
      for (uint32_t t = 1; t < src.count; ++t) one = one && src.triangles[t].material == src.triangles[0].material;
      auto fits = [&](const Mesh& mesh) {
        if (one) return true;
        for (size_t k = 0; k < mesh.order.size(); ++k)
          if (src.triangles[mesh.order[k]].material != mesh.triangles[k].material) return false;
        return true;
      };
      bool shared = false;
      for (auto& k : known) shared = shared || k.source == in.mesh;
      long found = -1;
      uint64_t hash = 0;
      bool hashed = false;
      if (!alone) {
        for (auto& k : known)
          if (k.source == in.mesh && fits(meshes[k.mesh])) {
            found = (long)k.mesh;
            break;
          }
        if (found < 0) {
          hash = geometry_hash(src.triangles, src.count);
          hashed = true;
          for (auto& k : known) {
            const Mesh& mesh = meshes[k.mesh];
            if (k.hash != hash || mesh.order.size() != src.count || !fits(mesh)) continue;
            bool same = true;
            for (size_t j = 0; j < mesh.order.size() && same; ++j)
              same = same_geometry(src.triangles[mesh.order[j]], mesh.triangles[j]);
            if (same) {
              found = (long)k.mesh;
              break;
            }
          }
        }
      }
      size_t mesh_index;
      if (found >= 0) {
        mesh_index = (size_t)found;
      } else {
        Bvh bvh = bvh_triangles(src.triangles, src.count);
        if (bvh.gpu) out->gpu_builds += 1;
        Mesh mesh;
        mesh.source = in.mesh;
        mesh.bounds = Bounds::empty();
        if (!bvh.nodes.empty()) {
          for (int k = 0; k < 3; ++k) {
            mesh.bounds.lo[k] = bvh.nodes[0].lo[k];
            mesh.bounds.hi[k] = bvh.nodes[0].hi[k];
          }
        }
        for (uint32_t j : bvh.order) mesh.triangles.push_back(src.triangles[j]);
        mesh.order = std::move(bvh.order);
        mesh.nodes = std::move(bvh.nodes);
        mesh.root = 0;
        mesh.first = next;
        if ((uint64_t)next + src.count > 0xffffffffull) throw Invalid("trace scene has too many triangles");
        next += src.count;
        meshes.push_back(std::move(mesh));
        mesh_index = meshes.size() - 1;
      }
      if (!alone && !shared) {
        if (!hashed) hash = geometry_hash(src.triangles, src.count);
        known.push_back(Known{in.mesh, hash, mesh_index});
      }
      record += 1;
      Placed p;
      p.mesh = (uint32_t)mesh_index;
      p.base = meshes[mesh_index].first;
      p.record = record;
      p.word = words[i];
      p.has_material = one;
      p.material = src.triangles[0].material;
      p.bounds = placed_bounds(pose, meshes[mesh_index].bounds);
      pose_inverse_rows(pose, p.inverse);
      p.pose = pose;
      placed_index[i] = (int)placed.size();
      placed.push_back(p);
    }
    slots = next;
    // Node offsets of the world and mesh BVHs after the top (levels.rs:361-375).
    auto state = std::make_shared<Placing>();
    Placing& s = *state;
    s.world = !world_bvh.nodes.empty();
    size_t group_count = (s.world ? 1 : 0) + placed.size();
    s.top_len = group_count == 0 ? 0u : (uint32_t)(3 * group_count - 1);
    uint32_t offset = s.top_len;
    if (s.world) {
      s.world_root = offset;
      for (int k = 0; k < 3; ++k) {
        s.world_bounds.lo[k] = world_bvh.nodes[0].lo[k];
        s.world_bounds.hi[k] = world_bvh.nodes[0].hi[k];
      }
      offset += (uint32_t)world_bvh.nodes.size();
    }
    for (auto& mesh : meshes) {
      mesh.root = offset;
      offset += (uint32_t)mesh.nodes.size();
      s.meshes.push_back(Placing::Mesh{mesh.triangles, mesh.root, mesh.first, mesh.bounds});
    }
    s.placed_index = placed_index;
    for (uint32_t i = 0; i < scene.instance_count; ++i) {
      if (placed_index[i] < 0) continue;
      const Placed& p = placed[placed_index[i]];
      Placing::Placed q;
      q.mesh = p.mesh;
      q.base = p.base;
      q.record = p.record;
      memcpy(q.transform, scene.instances[i].transform, sizeof(q.transform));
      q.bounds = p.bounds;
      memcpy(q.inverse, p.inverse, sizeof(q.inverse));
      s.placed.push_back(q);
    }
    nodes.resize(s.top_len);
    lay_top(s, nodes.data());
    out->placing = std::move(state);
    out->top_builds = 1;
    auto shifted = [&](const std::vector<GpuNode>& src, uint32_t off) {
      for (auto n : src) {
        if (n.count == 0) n.first += off;
        nodes.push_back(n);
      }
    };
    if (s.world) shifted(world_bvh.nodes, s.world_root);
    for (auto& mesh : meshes) shifted(mesh.nodes, mesh.root);
  }

  // ---- triangles in slot order (gpu.rs:765-780)
  out->triangles.resize(slots);
  out->uv.resize(slots);
  auto put = [&](size_t slot, const pfxt_triangle& t) {
    GpuTriangle g{};
    for (int k = 0; k < 3; ++k) {
      g.a[k] = t.v[0][k];
      g.b[k] = t.v[1][k];
      g.c[k] = t.v[2][k];
      g.na[k] = t.n[0][k];
      g.nb[k] = t.n[1][k];
      g.nc[k] = t.n[2][k];
    }
    g.a[3] = (float)t.material;
    g.b[3] = 0.0f;
    g.c[3] = 0.0f;
    g.na[3] = t.uv[0][0];
    g.nb[3] = t.uv[1][0];
    g.nc[3] = t.uv[2][0];
    out->triangles[slot] = g;
    out->uv[slot] = {t.uv[0][1], t.uv[1][1], t.uv[2][1], 0.0f};
  };
  for (uint32_t s = 0; s < scene.triangle_count; ++s) put(s, scene.triangles[world_bvh.order[s]]);
  for (auto& mesh : meshes)
    for (size_t j = 0; j < mesh.triangles.size(); ++j) put(mesh.first + j, mesh.triangles[j]);

  // ---- instance surface records (gpu.rs:782-805)
  // GpuSurface::of over InstanceSurface::default (gpu.rs:40-88, detail.rs:123-138):
  // uv offset 0, uv scale 1, crop [0, 0, 1, 1]
  GpuSurface world_surface{};
  world_surface.transform[2] = 1.0f;
  world_surface.transform[3] = 1.0f;
  world_surface.crop[2] = 1.0f;
  world_surface.crop[3] = 1.0f;
  world_surface.info[0] = 0;
  world_surface.info[1] = NO_MATERIAL;
  world_surface.info[2] = 0;
  world_surface.info[3] = f2bits(1.0f);
  {
    static const float identity[12] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0};
    memcpy(world_surface.forward, identity, sizeof(identity));
    memcpy(world_surface.inverse, identity, sizeof(identity));
  }
  out->surfaces.push_back(world_surface);
  for (uint32_t i = 0; i < scene.instance_count; ++i) {
    if (placed_index[i] < 0) continue;
    const Placed& p = placed[placed_index[i]];
    GpuSurface s = world_surface;
    s.info[0] = p.word;
    s.info[1] = p.has_material ? p.material : NO_MATERIAL;
    s.info[2] = f2bits(0.5f);
    s.info[3] = f2bits(pose_inverse_determinant(p.pose));
    float rows[12];
    pose_rows(p.pose, rows);
    memcpy(s.forward, rows, sizeof(rows));
    memcpy(s.inverse, p.inverse, sizeof(p.inverse));
    out->surfaces.push_back(s);
  }

  // ---- emitter candidates (gpu.rs:826-877)
  std::vector<Candidate> cands;
  auto mark = [&](size_t slot, size_t value) { out->triangles[slot].c[3] = (float)value; };
  for (uint32_t s = 0; s < scene.triangle_count; ++s) {
    const pfxt_triangle& t = scene.triangles[world_bvh.order[s]];
    if (emitting[t.material] && triangle_area(t.v) > 1e-12f) {
      Candidate c;
      memcpy(c.vertices, t.v, sizeof(c.vertices));
      c.slot = s;
      c.record = 0;
      memcpy(c.emission, scene.materials[t.material].emission, sizeof(c.emission));
      cands.push_back(c);
      mark(s, cands.size());
    }
  }
  for (uint32_t i = 0; i < scene.instance_count; ++i) {
    if (placed_index[i] < 0 || !unique[i]) continue;
    const Placed& p = placed[placed_index[i]];
    const Mesh& mesh = meshes[p.mesh];
    for (size_t j = 0; j < mesh.triangles.size(); ++j) {
      const pfxt_triangle& t = mesh.triangles[j];
      uint32_t material = p.has_material ? p.material : t.material;
      float v[3][3];
      for (int c = 0; c < 3; ++c) {
        V3 w = pose_point(p.pose, t.v[c]);
        for (int k = 0; k < 3; ++k) v[c][k] = w[k];
      }
      if (emitting[material] && triangle_area(v) > 1e-12f) {
        Candidate c;
        memcpy(c.vertices, v, sizeof(v));
        c.slot = (uint32_t)(mesh.first + j);
        c.record = p.record;
        memcpy(c.emission, scene.materials[material].emission, sizeof(c.emission));
        cands.push_back(c);
        mark(mesh.first + j, cands.size());
      }
    }
  }
  if (cands.size() > (1u << 24)) throw Invalid("trace scene has too many emitters");

  // ---- lights and the emitter list (gpu.rs:1011-1013)
  TreeLaid laid = tree_lay(scene.lights, scene.light_count);
  build_emitters(cands, laid.looped, laid.tree, out->emitters, out->emitter_cdf);
  if (out->placing) {
    out->placing->candidates = cands;
    out->placing->looped = laid.looped;
    out->placing->tree = laid.tree;
  }
  out->lights = std::move(laid.rows);
  out->materials = std::move(hot);
  out->nodes = std::move(nodes);
  out->order = std::move(world_bvh.order);

  // ---- environment
  out->sky_width = std::max(scene.sky_width, 1u);
  out->sky_height = std::max(scene.sky_height, 1u);
  memcpy(out->sky_radiance, scene.sky, sizeof(out->sky_radiance));
  float total = 0.0f;
  sky_cdf_uniform(scene.sky, out->sky_width, out->sky_height, out->sky_rows, out->sky_columns, &total);

  // ---- Sobol table (sobol.rs:33-39, 138-153)
  out->sobol_length = 0;
  if (settings.sampler == PFXT_SAMPLER_SOBOL) {
    uint32_t samples = std::max(settings.sobol_samples, 1u);
    uint32_t length = 1;
    while (length < samples && length < (1u << 31)) length <<= 1;
    if (length < samples) length = 8192;
    length = std::min(std::max(length, 256u), 8192u);
    out->sobol_length = length;
    out->sobol.assign((size_t)length * 256 * 4, 0.0f);
    unsigned threads = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < threads; ++t) {
      pool.emplace_back([&, t]() {
        for (uint32_t pattern = t; pattern < 256; pattern += threads)
          generate_4d(out->sobol.data() + (size_t)pattern * length * 4, length, pattern);
      });
    }
    for (auto& th : pool) th.join();
  }

  out->triangle_count = slots;
  out->bottom_builds = (uint32_t)meshes.size() + (scene.triangle_count > 0 ? 1u : 0u);
  out->light_count = scene.light_count;
  out->emitter_count = (uint32_t)cands.size();
  out->max_depth = out->nodes.empty() ? 0 : std::max<uint32_t>(1u, stack_need(out->nodes, 0, 0));
  return out.release();
}

int set_gpu_bvh(int on) { return g_gpu_bvh.exchange(on ? 1 : 0); }

// The light tree's selection on its own, for tests: sorts (key, index) pairs
// as select_nth_unstable_by(index, total_cmp on the key) leaves them and
// writes the original indices in their final order.  `rounds` < 16 reaches
// the deterministic fallback sooner.
void select_nth_for_test(const float* keys, uint32_t n, uint32_t index, int rounds, uint32_t* order) {
  struct Item {
    float key;
    uint32_t at;
  };
  std::vector<Item> v(n);
  for (uint32_t i = 0; i < n; ++i) v[i] = Item{keys[i], i};
  auto by_key = [](const Item& a, const Item& b) { return total_order_key(a.key) < total_order_key(b.key); };
  RustSelect<Item, decltype(by_key)> select{by_key};
  select.rounds = rounds;
  select.select_nth(v.data(), n, index);
  for (uint32_t i = 0; i < n; ++i) order[i] = v[i].at;
}

// Trace::move_instances (gpu.rs:2433-2530).  Every transform is checked first;
// an instance moves when any of its 16 floats differs bit for bit.  A moved
// instance gets its inverse rows and world box (levels.rs:114-127), its
// surface record's forward and inverse rows and inverse determinant, and its
// emitter candidates' world vertices; the candidate list itself stays as built,
// so the emitter list is rebuilt from it when one of them moved.  The top-level
// BVH is then laid again over the new boxes, as finish_tops writes it
// (gpu.rs:2533-2540).
bool move_instances(SceneBlobs& b, const float* transforms, size_t count) {
  Placing* s = b.placing.get();
  if (!s) {
    if (count == 0) return false;
    throw Invalid("this trace has no instances to move");
  }
  if (count > s->placed_index.size())
    throw Invalid("the trace has " + std::to_string(s->placed_index.size()) + " instances and " +
                  std::to_string(count) + " transforms were given");
  if (count > 0 && !transforms) throw Invalid("null argument");
  std::vector<Pose> poses(count);
  for (size_t i = 0; i < count; ++i) {
    std::string err;
    if (!pose_new(transforms + 16 * i, &poses[i], &err)) throw Invalid(err);
  }
  auto moved = [&](const Placing::Placed& p, const float* t) {
    for (int k = 0; k < 16; ++k)
      if (f2bits(p.transform[k]) != f2bits(t[k])) return true;
    return false;
  };
  bool any = false;
  for (size_t i = 0; i < count && !any; ++i)
    any = s->placed_index[i] >= 0 && moved(s->placed[s->placed_index[i]], transforms + 16 * i);
  if (!any) return false;
  bool emitters_moved = false;
  for (size_t i = 0; i < count; ++i) {
    if (s->placed_index[i] < 0) continue;
    Placing::Placed& p = s->placed[s->placed_index[i]];
    const float* t = transforms + 16 * i;
    if (!moved(p, t)) continue;
    const Pose& pose = poses[i];
    const Placing::Mesh& mesh = s->meshes[p.mesh];
    memcpy(p.transform, t, sizeof(p.transform));
    pose_inverse_rows(pose, p.inverse);
    p.bounds = placed_bounds(pose, mesh.bounds);
    for (auto& c : s->candidates) {
      if (c.record != p.record) continue;
      const pfxt_triangle& local = mesh.triangles[c.slot - mesh.first];
      for (int v = 0; v < 3; ++v) {
        V3 w = pose_point(pose, local.v[v]);
        for (int k = 0; k < 3; ++k) c.vertices[v][k] = w[k];
      }
      emitters_moved = true;
    }
    GpuSurface& sf = b.surfaces[p.record];
    sf.info[3] = f2bits(pose_inverse_determinant(pose));
    float rows[12];
    pose_rows(pose, rows);
    memcpy(sf.forward, rows, sizeof(rows));
    memcpy(sf.inverse, p.inverse, sizeof(p.inverse));
  }
  if (emitters_moved) {
    std::vector<GpuEmitter> entries;
    std::vector<float> cdf;
    build_emitters(s->candidates, s->looped, s->tree, entries, cdf);
    if (entries.size() != b.emitters.size() || cdf.size() != b.emitter_cdf.size())
      throw Invalid("the emitter list changed size");
    // in place: the buffers handed out by pfxt_scene_buffers keep pointing here
    std::copy(entries.begin(), entries.end(), b.emitters.begin());
    std::copy(cdf.begin(), cdf.end(), b.emitter_cdf.begin());
  }
  lay_top(*s, b.nodes.data());
  b.max_depth = std::max<uint32_t>(1u, stack_need(b.nodes, 0, 0));
  b.top_builds += 1;
  return true;
}

}  // namespace pfxt
