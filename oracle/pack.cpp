// TEST INFRASTRUCTURE ONLY - the oracle's own scene packing.
//
// An independent C++ restatement of the reference's SceneBuffers::build
// (crates/trace/src/gpu.rs:566-1061) for the scope the tracer covers: world
// triangles, instanced meshes, materials, local lights through the light
// tree, emissive triangles, a uniform environment and the Sobol table.  It
// produces the byte blobs the reference would upload, so the tests can hold
// the product's packing to them byte for byte and the oracle's tracer can run
// on buffers that the product did not make.  Each function cites the
// reference lines it follows.  Included by oracle.cpp (after the BVH builder
// and the Sobol generator it reuses).

namespace orcpack {

// ------------------------------------------------------------ input layouts
struct InTri {  // detail.rs TriangleDetail without uvs1
  float v[3][3];
  float n[3][3];
  float uv[3][2];
  uint32_t material;
};
static_assert(sizeof(InTri) == 100, "triangle input");
struct InMesh {
  const InTri* tris;
  uint32_t count;
};
struct InInstance {  // detail.rs:53-60 (with the surface's casts_shadow)
  uint32_t mesh, shadow_only, two_sided, casts_shadow;
  float transform[16];  // column-major: transform[column * 4 + row]
};
static_assert(sizeof(InInstance) == 80, "instance input");
struct InMaterial {  // the material fields the hot record packs (material.rs:827-866)
  float base[3], roughness;
  float metalness, specular, clearcoat, clearcoat_roughness;
  float sheen, transmission, ior, dispersion;
  float thickness, subsurface, thin_film, thin_film_ior;
  float subsurface_tint[3], absorption;
  float emission[3], thin_film_amount;
  float fresnel_power, pad[3];
};
static_assert(sizeof(InMaterial) == 112, "material input");
struct InLight {  // lights.rs:11-39
  uint32_t shape, shadow, two_sided, pad;
  float position[3], colour[3];
  float intensity, radius, range;
  float direction[3];
  float inner_deg, outer_deg;
  float half_u[3], half_v[3];
  float disc_radius;
};
static_assert(sizeof(InLight) == 100, "light input");
struct InScene {
  const InTri* world;
  uint32_t world_count;
  const InMesh* meshes;
  uint32_t mesh_count;
  const InInstance* instances;
  uint32_t instance_count;
  const InMaterial* materials;
  uint32_t material_count;
  const InLight* lights;
  uint32_t light_count;
  float sky[3];
  uint32_t sky_width, sky_height;
  uint32_t sobol, sobol_samples;
};

// ------------------------------------------------------------ output layouts
struct F4 {
  float v[4];
};
struct GpuTri {  // gpu.rs:19-26
  float a[4], b[4], c[4], na[4], nb[4], nc[4];
};
struct GpuSurf {  // gpu.rs:29-38
  float clip0[4], clip1[4], transform[4], crop[4];
  uint32_t info[4];
  float forward[12], inverse[12];
};
static_assert(sizeof(GpuSurf) == 176, "surface record");
struct Row4 {  // GpuLight / GpuEmitter (lights.rs): four vec4
  float a[4], b[4], c[4], d[4];
};
struct Hot {  // record.rs:18-27
  float rows[8][4];
};

struct Blobs {
  std::vector<Node> nodes;
  std::vector<uint32_t> order;
  std::vector<GpuTri> triangles;
  std::vector<F4> uv;
  std::vector<GpuSurf> surfaces;
  std::vector<Hot> materials;
  std::vector<Row4> emitters;
  std::vector<float> emitter_cdf;
  std::vector<Row4> lights;
  std::vector<float> sky_rows, sky_columns;
  std::vector<float> sobol;
  uint32_t sobol_length = 0;
  uint32_t triangle_count = 0, emitter_count = 0, light_count = 0, sky_width = 1, sky_height = 1;
  uint32_t bottom_builds = 0;
  float sky_radiance[3] = {0, 0, 0};
};

// --------------------------------------------------------------- math.rs
inline float fmin_r(float a, float b) { return fminf(a, b); }  // f32::min: a NaN loses, as fminf
inline float fmax_r(float a, float b) { return fmaxf(a, b); }
struct P3 {
  float x, y, z;
};
inline P3 p3(const float* p) { return P3{p[0], p[1], p[2]}; }
inline P3 psub(P3 a, P3 b) { return P3{a.x - b.x, a.y - b.y, a.z - b.z}; }
inline P3 padd(P3 a, P3 b) { return P3{a.x + b.x, a.y + b.y, a.z + b.z}; }
inline P3 pscale(P3 a, float s) { return P3{a.x * s, a.y * s, a.z * s}; }
inline float pdot(P3 a, P3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline P3 pcross(P3 a, P3 b) { return P3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline float plength(P3 a) { return sqrtf(pdot(a, a)); }
inline P3 pnormalize(P3 a) {  // math.rs:29-36
  float len = plength(a);
  if (len <= 1e-12f) return P3{0.0f, 0.0f, 1.0f};
  return pscale(a, 1.0f / len);
}
inline uint32_t fbits(float f) {
  uint32_t u;
  memcpy(&u, &f, 4);
  return u;
}
inline float bitsf(uint32_t u) {
  float f;
  memcpy(&f, &u, 4);
  return f;
}
const float PI_F = 3.14159265358979323846f;

// ----------------------------------------------------------- lights.rs
inline float luminance(const float* v) { return 0.2126f * v[0] + 0.7152f * v[1] + 0.0722f * v[2]; }
// lights.rs:293-298
bool emits(const float* e) {
  for (int k = 0; k < 3; ++k)
    if (!isfinite(e[k]) || !(e[k] >= 0.0f)) return false;
  return luminance(e) > 0.0f;
}
// lights.rs:300-305
float triangle_area(const float v[3][3]) {
  return 0.5f * plength(pcross(psub(p3(v[1]), p3(v[0])), psub(p3(v[2]), p3(v[0]))));
}
// lights.rs:98-100
bool lit(const InLight& l) {
  return l.intensity > 0.0f && l.range > 0.0f && (l.colour[0] > 0.0f || l.colour[1] > 0.0f || l.colour[2] > 0.0f);
}
// lights.rs:147-153
float light_area(const InLight& l) {
  if (l.shape == 2) return 4.0f * plength(pcross(p3(l.half_u), p3(l.half_v)));
  if (l.shape == 3) return PI_F * l.disc_radius * l.disc_radius;
  return 0.0f;
}
inline float radians(float deg) { return deg * (PI_F / 180.0f); }
// lights.rs:238-243
void spot_terms(float inner_deg, float outer_deg, float* scale, float* offset) {
  float inner = cosf(radians(inner_deg)), outer = cosf(radians(outer_deg));
  *scale = 1.0f / fmax_r(inner - outer, 0.001f);
  *offset = -outer * *scale;
}
// LocalLight::pack (lights.rs:182-235)
Row4 pack_light(const InLight& l) {
  float c[3] = {l.colour[0] * l.intensity, l.colour[1] * l.intensity, l.colour[2] * l.intensity};
  float shadow = l.shadow ? 1.0f : 0.0f;
  Row4 r{};
  auto set = [](float* dst, float x, float y, float z, float w) {
    dst[0] = x;
    dst[1] = y;
    dst[2] = z;
    dst[3] = w;
  };
  if (l.shape == 0) {
    set(r.a, l.position[0], l.position[1], l.position[2], 0.0f);
    set(r.b, c[0], c[1], c[2], l.range);
    set(r.c, 0.0f, 0.0f, 0.0f, l.radius);
    set(r.d, 0.0f, 0.0f, 0.0f, shadow);
  } else if (l.shape == 1) {
    float scale, offset;
    spot_terms(l.inner_deg, l.outer_deg, &scale, &offset);
    P3 d = pnormalize(p3(l.direction));
    set(r.a, l.position[0], l.position[1], l.position[2], 1.0f);
    set(r.b, c[0], c[1], c[2], l.range);
    set(r.c, d.x, d.y, d.z, l.radius);
    set(r.d, scale, offset, 0.0f, shadow);
  } else if (l.shape == 2) {
    float area = light_area(l);
    set(r.a, l.position[0], l.position[1], l.position[2], 2.0f);
    set(r.b, c[0] / area, c[1] / area, c[2] / area, FLT_MAX);
    set(r.c, l.half_u[0], l.half_u[1], l.half_u[2], l.two_sided ? 1.0f : 0.0f);
    set(r.d, l.half_v[0], l.half_v[1], l.half_v[2], shadow);
  } else {
    float area = light_area(l);
    P3 n = pnormalize(p3(l.direction));
    set(r.a, l.position[0], l.position[1], l.position[2], 3.0f);
    set(r.b, c[0] / area, c[1] / area, c[2] / area, FLT_MAX);
    set(r.c, n.x, n.y, n.z, l.two_sided ? 1.0f : 0.0f);
    set(r.d, l.disc_radius, 0.0f, 0.0f, shadow);
  }
  return r;
}

// Candidate + build_emitters (lights.rs:391-440).  Rust's f64 Iterator::sum
// folds from -0.0, the additive identity, so an empty list's total is -0.0.
struct Candidate {
  float v[3][3];
  uint32_t record;
  float emission[3];
};
void build_emitters(const std::vector<Candidate>& cands, size_t looped, size_t tree, Blobs& out) {
  std::vector<double> powers(cands.size());
  for (size_t i = 0; i < cands.size(); ++i)
    powers[i] = (double)triangle_area(cands[i].v) * (double)luminance(cands[i].emission);
  double total = -0.0;
  for (double p : powers) total += p;
  Row4 head{};
  head.a[0] = (float)cands.size();
  head.a[1] = (float)looped;
  head.a[2] = (float)total;
  head.a[3] = (float)tree;
  out.emitters.assign(1, head);
  out.emitter_cdf.clear();
  double running = 0.0;
  for (size_t i = 0; i < cands.size(); ++i) {
    running += powers[i];
    out.emitter_cdf.push_back((float)(running / total));
    const Candidate& c = cands[i];
    Row4 e{};
    for (int k = 0; k < 3; ++k) {
      e.a[k] = c.v[0][k];
      e.b[k] = c.v[1][k];
      e.c[k] = c.v[2][k];
      e.d[k] = c.emission[k];
    }
    e.a[3] = 0.0f;
    e.b[3] = (float)c.record;
    e.c[3] = triangle_area(c.v);
    e.d[3] = (float)(powers[i] / total);
    out.emitters.push_back(e);
  }
  if (!out.emitter_cdf.empty()) out.emitter_cdf.back() = 1.0f;
}

// -------------------------------------------------------------- tree.rs
const size_t LOOPED = 4, LEAF = 8, BUCKETS = 12;  // tree.rs:6-8

struct Cone {  // tree.rs:10-82
  float axis[3], theta_o, theta_e;
};
const Cone CONE_EMPTY = {{0.0f, 0.0f, 0.0f}, FLT_MIN, FLT_MIN};
bool cone_empty(const Cone& c) { return c.axis[0] == 0.0f && c.axis[1] == 0.0f && c.axis[2] == 0.0f; }
float cone_measure(const Cone& c) {  // tree.rs:28-41
  if (cone_empty(c)) return 0.0f;
  float theta_w = fmin_r(c.theta_o + c.theta_e, PI_F);
  float cos_o = cosf(c.theta_o), sin_o = sinf(c.theta_o);
  float inner = 2.0f * theta_w * sin_o - cosf(c.theta_o - 2.0f * theta_w) - 2.0f * c.theta_o * sin_o + cos_o;
  return 2.0f * PI_F * (1.0f - cos_o) + (PI_F / 2.0f) * inner;
}
P3 orthogonal(P3 n) {  // tree.rs:84-91
  P3 helper = fabsf(n.x) > 0.1f ? P3{0.0f, 1.0f, 0.0f} : P3{1.0f, 0.0f, 0.0f};
  return pnormalize(pcross(n, helper));
}
Cone cone_merge(const Cone& self, const Cone& other) {  // tree.rs:43-81
  if (cone_empty(self)) return other;
  if (cone_empty(other)) return self;
  const Cone& a = other.theta_o > self.theta_o ? other : self;
  const Cone& b = other.theta_o > self.theta_o ? self : other;
  P3 aa = p3(a.axis), ba = p3(b.axis);
  float cos_ab = pdot(aa, ba);
  float theta_d = acosf(fmin_r(fmax_r(cos_ab, -1.0f), 1.0f));
  float theta_e = fmax_r(a.theta_e, b.theta_e);
  if (a.theta_o + 5e-4f >= fmin_r(PI_F, theta_d + b.theta_o)) {
    Cone r = a;
    r.theta_e = theta_e;
    return r;
  }
  float theta_o = (theta_d + a.theta_o + b.theta_o) * 0.5f;
  if (theta_o >= PI_F) return Cone{{a.axis[0], a.axis[1], a.axis[2]}, PI_F, theta_e};
  P3 axis;
  if (cos_ab < -0.9995f) {
    axis = orthogonal(aa);
  } else {
    float theta_r = theta_o - a.theta_o;
    P3 ortho = pnormalize(psub(ba, pscale(aa, cos_ab)));
    axis = padd(pscale(aa, cosf(theta_r)), pscale(ortho, sinf(theta_r)));
  }
  return Cone{{axis.x, axis.y, axis.z}, theta_o, theta_e};
}

struct Measure {  // tree.rs:93-133
  float lo[3], hi[3];
  Cone cone;
  float energy, range;
};
const Measure MEASURE_EMPTY = {{FLT_MAX, FLT_MAX, FLT_MAX}, {-FLT_MAX, -FLT_MAX, -FLT_MAX}, CONE_EMPTY, 0.0f, 0.0f};
void measure_add(Measure& m, const Measure& o) {
  if (o.energy == 0.0f) return;
  for (int k = 0; k < 3; ++k) {
    m.lo[k] = fmin_r(m.lo[k], o.lo[k]);
    m.hi[k] = fmax_r(m.hi[k], o.hi[k]);
  }
  m.cone = cone_merge(m.cone, o.cone);
  m.energy += o.energy;
  m.range = fmax_r(m.range, o.range);
}
float measure_cost(const Measure& m) {
  if (m.energy == 0.0f) return 0.0f;
  float s[3] = {m.hi[0] - m.lo[0], m.hi[1] - m.lo[1], m.hi[2] - m.lo[2]};
  float area = 2.0f * (s[0] * s[1] + s[1] * s[2] + s[2] * s[0]);
  float am = area == 0.0f ? plength(P3{s[0], s[1], s[2]}) : area;
  return m.energy * am * cone_measure(m.cone);
}

struct TreeLight {  // tree.rs:135-175 Emitter
  size_t index;
  float centroid[3];
  Measure measure;
};
TreeLight tree_light(size_t index, const InLight& l) {
  Cone cone;
  if (l.shape == 1) {
    P3 a = pnormalize(p3(l.direction));
    cone = Cone{{a.x, a.y, a.z}, 0.0f, fmin_r(radians(l.outer_deg), PI_F / 2.0f)};
  } else {
    cone = Cone{{0.0f, 0.0f, -1.0f}, PI_F, PI_F / 2.0f};
  }
  TreeLight t;
  t.index = index;
  float sum = 0.0f;
  for (int k = 0; k < 3; ++k) {
    t.centroid[k] = l.position[k];
    t.measure.lo[k] = l.position[k] - l.radius;
    t.measure.hi[k] = l.position[k] + l.radius;
  }
  float st[3] = {fabsf(l.colour[0] * l.intensity), fabsf(l.colour[1] * l.intensity),
                 fabsf(l.colour[2] * l.intensity)};
  sum = (st[0] + st[1] + st[2]) / 3.0f;
  t.measure.cone = cone;
  t.measure.energy = sum;
  t.measure.range = l.range;
  return t;
}

struct Bucket {  // tree.rs:177-203: measure is an Option
  bool some = false;
  Measure m = MEASURE_EMPTY;
  size_t count = 0;
};
void bucket_add(Bucket& b, const Measure& m) {
  if (!b.some) {
    b.some = true;
    b.m = MEASURE_EMPTY;
  }
  measure_add(b.m, m);
  b.count += 1;
}
Bucket bucket_plus(const Bucket& a, const Bucket& o) {
  Bucket r;
  r.some = true;
  r.m = a.some ? a.m : MEASURE_EMPTY;
  if (o.some) measure_add(r.m, o.m);
  r.count = a.count + o.count;
  return r;
}
float bucket_cost(const Bucket& b) { return b.some ? measure_cost(b.m) : 0.0f; }

// ---- slice::select_nth_unstable_by as Rust's core library runs it
// (core::slice::select, Rust 1.81 and later): introselect over ipnsort's
// partition (Lukas Bergdoll and Orson Peters).  Written here over an index
// range of a vector, separately from the product's version.
template <class Item>
struct SelectOf {
  std::vector<Item>& v;
  int dim;
  int rounds_cap = 16;  // partition rounds before the deterministic fallback
  bool lt(const Item& a, const Item& b) const {  // f32::total_cmp == Less
    auto key = [](float f) {
      int32_t i = (int32_t)fbits(f);
      return i ^ (int32_t)((uint32_t)(i >> 31) >> 1);
    };
    return key(a.centroid[dim]) < key(b.centroid[dim]);
  }
  void sort_small(size_t lo, size_t hi) {  // insertion sort (stable)
    for (size_t i = lo + 1; i < hi; ++i) {
      Item x = v[i];
      size_t j = i;
      while (j > lo && lt(x, v[j - 1])) {
        v[j] = v[j - 1];
        --j;
      }
      v[j] = x;
    }
  }
  size_t med3(size_t a, size_t b, size_t c) const {
    bool ab = lt(v[a], v[b]), ac = lt(v[a], v[c]);
    if (ab != ac) return a;
    bool bc = lt(v[b], v[c]);
    return (bc != ab) ? c : b;
  }
  size_t pseudo_median(size_t a, size_t b, size_t c, size_t n) const {
    if (n * 8 >= 64) {
      size_t s = n / 8;
      a = pseudo_median(a, a + 4 * s, a + 7 * s, s);
      b = pseudo_median(b, b + 4 * s, b + 7 * s, s);
      c = pseudo_median(c, c + 4 * s, c + 7 * s, s);
    }
    return med3(a, b, c);
  }
  size_t pivot_of(size_t lo, size_t hi) const {
    size_t n = hi - lo, s = n / 8;
    return n < 64 ? med3(lo, lo + 4 * s, lo + 7 * s) : pseudo_median(lo, lo + 4 * s, lo + 7 * s, s);
  }
  // Pivot first; cyclic branchless Lomuto over the rest; pivot placed between.
  // `le` switches the comparison to "not greater than".  Returns the
  // pivot's final position (relative to lo).
  size_t split(size_t lo, size_t hi, size_t p, bool le) {
    std::swap(v[lo], v[p]);
    Item pivot = v[lo];
    auto below = [&](const Item& x) { return le ? !lt(pivot, x) : lt(x, pivot); };
    size_t base = lo + 1, m = hi - base, count = 0;
    if (m > 0) {
      Item held = v[base];
      size_t hole = base;
      for (size_t r = base + 1; r < hi; ++r) {
        Item x = v[r];
        bool b = below(x);
        v[hole] = v[base + count];
        v[base + count] = x;
        hole = r;
        count += b ? 1 : 0;
      }
      bool b = below(held);
      v[hole] = v[base + count];
      v[base + count] = held;
      count += b ? 1 : 0;
    }
    std::swap(v[lo], v[lo + count]);
    return count;
  }
  size_t first_min(size_t lo, size_t hi) const {
    size_t k = lo;
    for (size_t i = lo + 1; i < hi; ++i)
      if (lt(v[i], v[k])) k = i;
    return k;
  }
  size_t first_max(size_t lo, size_t hi) const {
    size_t k = lo;
    for (size_t i = lo + 1; i < hi; ++i)
      if (lt(v[k], v[i])) k = i;
    return k;
  }
  size_t median_index(size_t a, size_t b, size_t c) const {
    if (lt(v[c], v[a])) std::swap(a, c);
    if (lt(v[c], v[b])) return c;
    if (lt(v[b], v[a])) return a;
    return b;
  }
  void ninther(size_t a, size_t b, size_t c, size_t d, size_t e, size_t f, size_t g, size_t h, size_t i) {
    b = median_index(a, b, c);
    h = median_index(g, h, i);
    if (lt(v[h], v[b])) std::swap(b, h);
    if (lt(v[f], v[d])) std::swap(d, f);
    if (lt(v[e], v[d])) {
    } else if (lt(v[f], v[e])) {
      d = f;
    } else {
      if (lt(v[e], v[b]))
        std::swap(v[e], v[b]);
      else if (lt(v[h], v[e]))
        std::swap(v[e], v[h]);
      return;
    }
    if (lt(v[d], v[b]))
      d = b;
    else if (lt(v[h], v[d]))
      d = h;
    std::swap(v[d], v[e]);
  }
  // Alexandrescu's deterministic selection ("Fast deterministic selection").
  void deterministic(size_t lo, size_t hi, size_t k) {
    while (true) {
      size_t n = hi - lo;
      if (n <= 16) {
        sort_small(lo, hi);
        return;
      }
      if (k == n - 1) {
        std::swap(v[first_max(lo, hi)], v[lo + k]);
        return;
      }
      if (k == 0) {
        std::swap(v[first_min(lo, hi)], v[lo]);
        return;
      }
      size_t frac = n <= 1024 ? n / 12 : (n <= 131072 ? n / 64 : n / 1024);
      size_t pivot = frac / 2, a_lo = n / 2 - pivot, a_hi = frac + a_lo, gap = (n - 9 * frac) / 4;
      size_t a = a_lo - 4 * frac - gap, b = a_hi + gap;
      for (size_t i = a_lo; i < a_hi; ++i) {
        ninther(lo + a, lo + i - frac, lo + b, lo + a + 1, lo + i, lo + b + 1, lo + a + 2, lo + i + frac, lo + b + 2);
        a += 3;
        b += 3;
      }
      deterministic(lo + a_lo, lo + a_hi, pivot);
      size_t p = split(lo, hi, lo + a_lo + pivot, false);
      if (p == k) return;
      if (p > k) {
        hi = lo + p;
      } else {
        lo = lo + p + 1;
        k -= p + 1;
      }
    }
  }
  void run(size_t lo, size_t hi, size_t k) {
    size_t n = hi - lo;
    if (k == n - 1) {
      std::swap(v[first_max(lo, hi)], v[lo + k]);
      return;
    }
    if (k == 0) {
      std::swap(v[first_min(lo, hi)], v[lo]);
      return;
    }
    int rounds = rounds_cap;
    bool ancestor = false;
    Item previous{};
    while (true) {
      n = hi - lo;
      if (n <= 16) {
        sort_small(lo, hi);
        return;
      }
      if (rounds == 0) {
        deterministic(lo, hi, k);
        return;
      }
      --rounds;
      size_t p = pivot_of(lo, hi);
      if (ancestor && !lt(previous, v[p])) {
        size_t mid = split(lo, hi, p, true) + 1;
        if (mid > k) return;
        lo += mid;
        k -= mid;
        ancestor = false;
        continue;
      }
      size_t mid = split(lo, hi, p, false);
      if (mid == k) return;
      if (mid < k) {
        previous = v[lo + mid];
        ancestor = true;
        lo += mid + 1;
        k -= mid + 1;
      } else {
        hi = lo + mid;
      }
    }
  }
};

// should_split (tree.rs:319-395) over v[lo, hi): returns whether to split,
// with the node's measure, the middle and the axis (-1: none).
bool should_split(const std::vector<TreeLight>& v, size_t lo, size_t hi, Measure* node, size_t* middle, int* axis) {
  size_t count = hi - lo;
  if (count < 2) {
    *node = v[lo].measure;
    return false;
  }
  size_t mid = count / 2;
  float low[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, high[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
  for (size_t i = lo; i < hi; ++i)
    for (int k = 0; k < 3; ++k) {
      low[k] = fmin_r(low[k], v[i].centroid[k]);
      high[k] = fmax_r(high[k], v[i].centroid[k]);
    }
  float extent[3] = {high[0] - low[0], high[1] - low[1], high[2] - low[2]};
  float max_extent = fmax_r(fmax_r(fmax_r(extent[0], extent[1]), extent[2]), 0.0f);
  Measure measure = MEASURE_EMPTY;
  float total = 0.0f, best = FLT_MAX;
  int dim_best = -1;
  for (int dim = 0; dim < 3; ++dim) {
    Bucket b[BUCKETS];
    float inv;
    if (extent[dim] == 0.0f) {
      if (dim != 0) continue;
      inv = FLT_MAX;
      for (size_t i = lo; i < hi; ++i) bucket_add(b[0], v[i].measure);
    } else {
      inv = 1.0f / extent[dim];
      for (size_t i = lo; i < hi; ++i) {
        float x = (float)BUCKETS * (v[i].centroid[dim] - low[dim]) * inv;
        // `as i64` saturates and maps NaN to 0; then clamp(0, 11)
        long long at = isnan(x) ? 0 : (x >= 9.2233720e18f ? LLONG_MAX : (x <= -9.2233720e18f ? LLONG_MIN : (long long)x));
        at = at < 0 ? 0 : (at > (long long)BUCKETS - 1 ? (long long)BUCKETS - 1 : at);
        bucket_add(b[at], v[i].measure);
      }
    }
    Bucket left[BUCKETS - 1];
    left[0] = b[0];
    for (size_t i = 1; i < BUCKETS - 1; ++i) left[i] = bucket_plus(left[i - 1], b[i]);
    if (dim == 0) {
      Bucket all = bucket_plus(left[BUCKETS - 2], b[BUCKETS - 1]);
      measure = all.some ? all.m : MEASURE_EMPTY;
      if (extent[0] == 0.0f && extent[1] == 0.0f && extent[2] == 0.0f) break;
      total = measure_cost(measure);
      if (total == 0.0f) break;
      if (extent[0] == 0.0f) continue;
    }
    Bucket right[BUCKETS - 1];
    right[BUCKETS - 2] = b[BUCKETS - 1];
    for (size_t i = BUCKETS - 2; i-- > 0;) right[i] = bucket_plus(right[i + 1], b[i + 1]);
    float reg = max_extent * inv;
    for (size_t s = 0; s < BUCKETS - 1; ++s) {
      float cost = reg * (bucket_cost(left[s]) + bucket_cost(right[s]));
      if (cost < total && cost < best && left[s].count >= 1 && left[s].count < count) {
        best = cost;
        dim_best = dim;
        mid = left[s].count;
      }
    }
  }
  *node = measure;
  *middle = mid;
  *axis = dim_best;
  return best < total || count > LEAF;
}

Row4 tree_row(const Measure& m, size_t count, size_t link) {  // tree.rs:295-317
  Row4 r;
  float a[4] = {m.lo[0], m.lo[1], m.lo[2], m.energy};
  float b[4] = {m.hi[0], m.hi[1], m.hi[2], m.range};
  float c[4] = {m.cone.axis[0], m.cone.axis[1], m.cone.axis[2], m.cone.theta_o};
  float d[4] = {m.cone.theta_e, (float)count, (float)link, 0.0f};
  memcpy(r.a, a, 16);
  memcpy(r.b, b, 16);
  memcpy(r.c, c, 16);
  memcpy(r.d, d, 16);
  return r;
}

// grow (tree.rs:263-293)
void grow(std::vector<TreeLight>& v, size_t lo, size_t hi, size_t start, size_t base, size_t root,
          std::vector<Row4>& nodes) {
  size_t at = nodes.size();
  nodes.push_back(Row4{});
  Measure measure;
  size_t middle = 0;
  int axis = -1;
  if (should_split(v, lo, hi, &measure, &middle, &axis)) {
    if (axis >= 0) {
      SelectOf<TreeLight> sel{v, axis};
      sel.run(lo, hi, middle);
    }
    grow(v, lo, lo + middle, start, base, root, nodes);
    size_t right_at = root + nodes.size();
    grow(v, lo + middle, hi, start + middle, base, root, nodes);
    nodes[at] = tree_row(measure, 0, right_at);
  } else {
    nodes[at] = tree_row(measure, hi - lo, base + start);
  }
}

// tree::lay (tree.rs:220-261): looped lights first, then the tree's lights in
// leaf order, then its nodes.
void lay_lights(const InLight* lights, size_t n, Blobs& out, size_t* looped, size_t* tree) {
  auto treed = [](const InLight& l) { return lit(l) && (l.shape == 0 || l.shape == 1); };
  size_t treed_count = 0;
  for (size_t i = 0; i < n; ++i) treed_count += treed(lights[i]) ? 1 : 0;
  out.lights.clear();
  if (treed_count <= LOOPED) {
    for (size_t i = 0; i < n; ++i) out.lights.push_back(pack_light(lights[i]));
    *looped = n;
    *tree = 0;
    return;
  }
  for (size_t i = 0; i < n; ++i)
    if (!treed(lights[i])) out.lights.push_back(pack_light(lights[i]));
  *looped = out.lights.size();
  std::vector<TreeLight> v;
  for (size_t i = 0; i < n; ++i)
    if (treed(lights[i])) v.push_back(tree_light(i, lights[i]));
  std::vector<Row4> nodes;
  if (!v.empty()) grow(v, 0, v.size(), 0, *looped, *looped + v.size(), nodes);
  for (auto& t : v) out.lights.push_back(pack_light(lights[t.index]));
  out.lights.insert(out.lights.end(), nodes.begin(), nodes.end());
  *tree = treed_count;
}

// ------------------------------------------------------------ detail.rs Pose
struct Pose {
  float m[4][4];  // m[column][row]
};
Pose pose_of(const float* t) {
  Pose p;
  for (int c = 0; c < 4; ++c)
    for (int r = 0; r < 4; ++r) p.m[c][r] = t[c * 4 + r];
  return p;
}
// Pose::point (detail.rs:232-240): m[3][row] + the sum over columns
P3 pose_point(const Pose& p, const float* q) {
  float out[3];
  for (int row = 0; row < 3; ++row) {
    float s = -0.0f;  // Rust's f32 Iterator::sum starts at -0.0
    for (int c = 0; c < 3; ++c) s += p.m[c][row] * q[c];
    out[row] = p.m[3][row] + s;
  }
  return P3{out[0], out[1], out[2]};
}
// Pose::rows (detail.rs:254-260)
void pose_rows(const Pose& p, float r[12]) {
  for (int row = 0; row < 3; ++row)
    for (int c = 0; c < 4; ++c) r[row * 4 + c] = p.m[c][row];
}
double pose_cofactor(const Pose& p, int row, int column) {
  auto a = [&](int r, int c) { return (double)p.m[c][r]; };
  int r0 = (row + 1) % 3, r1 = (row + 2) % 3, c0 = (column + 1) % 3, c1 = (column + 2) % 3;
  return a(r0, c0) * a(r1, c1) - a(r0, c1) * a(r1, c0);
}
// Pose::inverse_rows (detail.rs:262-287)
void pose_inverse_rows(const Pose& p, float r[12]) {
  double det = -0.0;
  for (int c = 0; c < 3; ++c) det += (double)p.m[c][0] * pose_cofactor(p, 0, c);
  double inv[3][3];
  for (int row = 0; row < 3; ++row)
    for (int c = 0; c < 3; ++c) inv[row][c] = pose_cofactor(p, c, row) / det;
  double tr[3] = {(double)p.m[3][0], (double)p.m[3][1], (double)p.m[3][2]};
  for (int row = 0; row < 3; ++row) {
    double shift = -0.0;
    for (int k = 0; k < 3; ++k) shift += inv[row][k] * tr[k];
    for (int c = 0; c < 3; ++c) r[row * 4 + c] = (float)inv[row][c];
    r[row * 4 + 3] = (float)(-shift);
  }
}
// Pose::inverse_determinant (detail.rs:223-230)
float pose_inverse_determinant(const Pose& p) {
  auto a = [&](int r, int c) { return (double)p.m[c][r]; };
  double det = a(0, 0) * (a(1, 1) * a(2, 2) - a(1, 2) * a(2, 1)) - a(0, 1) * (a(1, 0) * a(2, 2) - a(1, 2) * a(2, 0)) +
               a(0, 2) * (a(1, 0) * a(2, 1) - a(1, 1) * a(2, 0));
  return (float)(1.0 / det);
}

// ------------------------------------------------------------ levels.rs
struct Box3 {
  float lo[3], hi[3];
};
Box3 box_empty() { return Box3{{INFINITY, INFINITY, INFINITY}, {-INFINITY, -INFINITY, -INFINITY}}; }
void box_point(Box3& b, P3 p) {
  float q[3] = {p.x, p.y, p.z};
  for (int k = 0; k < 3; ++k) {
    b.lo[k] = fmin_r(b.lo[k], q[k]);
    b.hi[k] = fmax_r(b.hi[k], q[k]);
  }
}
// placed_bounds (levels.rs:114-127)
Box3 placed_bounds(const Pose& pose, const Box3& local) {
  Box3 b = box_empty();
  for (int corner = 0; corner < 8; ++corner) {
    float q[3];
    for (int k = 0; k < 3; ++k) q[k] = ((corner >> k) & 1) ? local.hi[k] : local.lo[k];
    box_point(b, pose_point(pose, q));
  }
  return b;
}
// geometry_hash / same_geometry (levels.rs:58-95): FNV-1a over the bits of
// vertices, normals, uvs and the (zero) second uv set
uint64_t geometry_hash(const InTri* t, size_t n) {
  uint64_t h = 0xcbf29ce484222325ull;
  auto mix = [&](float f) { h = (h ^ (uint64_t)fbits(f)) * 0x100000001b3ull; };
  for (size_t i = 0; i < n; ++i) {
    for (int c = 0; c < 3; ++c)
      for (int k = 0; k < 3; ++k) mix(t[i].v[c][k]);
    for (int c = 0; c < 3; ++c)
      for (int k = 0; k < 3; ++k) mix(t[i].n[c][k]);
    for (int c = 0; c < 3; ++c)
      for (int k = 0; k < 2; ++k) mix(t[i].uv[c][k]);
    for (int k = 0; k < 6; ++k) mix(0.0f);
  }
  return h;
}
bool same_geometry(const InTri& a, const InTri& b) {
  for (int c = 0; c < 3; ++c) {
    for (int k = 0; k < 3; ++k)
      if (fbits(a.v[c][k]) != fbits(b.v[c][k]) || fbits(a.n[c][k]) != fbits(b.n[c][k])) return false;
    for (int k = 0; k < 2; ++k)
      if (fbits(a.uv[c][k]) != fbits(b.uv[c][k])) return false;
  }
  return true;
}

// Bvh::over (bvh.rs:95-130) on boxes with the given leaf sizes.
void bvh_over(const std::vector<Box3>& boxes, size_t leaf, size_t most, std::vector<Node>& nodes,
              std::vector<uint32_t>& order) {
  OrcBuild b;
  b.leaf = leaf;
  b.most = most;
  size_t n = boxes.size();
  b.blo.resize(3 * n);
  b.bhi.resize(3 * n);
  b.cen.resize(3 * n);
  for (size_t i = 0; i < n; ++i)
    for (int k = 0; k < 3; ++k) {
      b.blo[3 * i + k] = boxes[i].lo[k];
      b.bhi[3 * i + k] = boxes[i].hi[k];
      b.cen[3 * i + k] = (boxes[i].lo[k] + boxes[i].hi[k]) * 0.5f;
    }
  b.order.resize(n);
  for (size_t i = 0; i < n; ++i) b.order[i] = (uint32_t)i;
  if (n) b.split(0, n);
  nodes = std::move(b.nodes);
  order = std::move(b.order);
}
void bvh_triangles(const InTri* t, size_t n, std::vector<Node>& nodes, std::vector<uint32_t>& order) {
  std::vector<Box3> boxes(n);
  for (size_t i = 0; i < n; ++i) {
    boxes[i] = box_empty();
    for (int c = 0; c < 3; ++c) box_point(boxes[i], p3(t[i].v[c]));
  }
  bvh_over(boxes, 4, 16, nodes, order);
}

const uint32_t SHADOW_ONLY = 1, CASTS_NO_SHADOW = 2, CUTOUT = 4, ONE_SIDED = 1u << 23;  // gpu.rs:127-132
const uint32_t NO_MATERIAL = 0xffffffffu;

// pack_triangle (gpu.rs:539-563) with word 0
GpuTri pack_triangle(const InTri& t) {
  GpuTri g;
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
  return g;
}

// GpuSurface::of over InstanceSurface::default (gpu.rs:40-88, detail.rs:123-138)
GpuSurf surface_of(const uint32_t info[4], const float forward[12], const float inverse[12]) {
  GpuSurf s;
  memset(&s, 0, sizeof(s));
  s.transform[0] = 0.0f;  // uv offset
  s.transform[1] = 0.0f;
  s.transform[2] = 1.0f;  // uv scale
  s.transform[3] = 1.0f;
  s.crop[0] = 0.0f;
  s.crop[1] = 0.0f;
  s.crop[2] = 1.0f;
  s.crop[3] = 1.0f;
  memcpy(s.info, info, 16);
  memcpy(s.forward, forward, 48);
  memcpy(s.inverse, inverse, 48);
  return s;
}
const float IDENTITY_ROWS[12] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0};

struct MeshOut {
  std::vector<InTri> tris;  // BVH order
  std::vector<uint32_t> order;
  std::vector<Node> nodes;
  uint32_t first = 0, root = 0;
  Box3 bounds;
};
struct PlacedOut {
  size_t mesh;
  uint32_t base, record, word;
  bool one;
  uint32_t material;
  Pose pose;
  Box3 bounds;
  float inverse[12];
};

// SceneBuffers::build (gpu.rs:566-1061) restricted to this scope.
void build(const InScene& s, Blobs& out) {
  // material records: Records::split (record.rs:57-77) with zero effects and
  // no extension rows (no maps, lobes, thin walls, layers, alpha or flakes)
  out.materials.assign(s.material_count + 1, Hot{});
  memset(out.materials.data(), 0, out.materials.size() * sizeof(Hot));
  for (uint32_t m = 0; m < s.material_count; ++m) {
    const InMaterial& x = s.materials[m];
    float rows[8][4] = {{x.base[0], x.base[1], x.base[2], x.roughness},
                        {x.metalness, x.specular, x.clearcoat, x.clearcoat_roughness},
                        {x.sheen, x.transmission, x.ior, x.dispersion},
                        {x.thickness, x.subsurface, x.thin_film, x.thin_film_ior},
                        {x.subsurface_tint[0], x.subsurface_tint[1], x.subsurface_tint[2], x.absorption},
                        {x.emission[0], x.emission[1], x.emission[2], x.thin_film_amount},
                        {x.fresnel_power, bitsf(0u), bitsf(0u), 0.0f},
                        {0.0f, 0.0f, 0.0f, 0.0f}};
    memcpy(out.materials[m + 1].rows, rows, sizeof(rows));
  }
  std::vector<bool> emitting(s.material_count);
  for (uint32_t m = 0; m < s.material_count; ++m) emitting[m] = emits(out.materials[m + 1].rows[5]);

  // instance words (gpu.rs:451-472) and which instances carry their own
  // emitters (gpu.rs:746-758)
  std::vector<uint32_t> words(s.instance_count);
  std::vector<bool> unique(s.instance_count);
  for (uint32_t i = 0; i < s.instance_count; ++i) {
    const InInstance& in = s.instances[i];
    uint32_t w = 0;
    if (in.shadow_only) w |= SHADOW_ONLY;
    if (!in.casts_shadow) w |= CASTS_NO_SHADOW;
    if (!in.two_sided) w |= ONE_SIDED;
    words[i] = w;
    const InMesh& mesh = s.meshes[in.mesh];
    bool any = false;
    for (uint32_t t = 0; t < mesh.count; ++t) any = any || emitting[mesh.tris[t].material];
    unique[i] = (w & (SHADOW_ONLY | CUTOUT)) == 0 && any;
  }

  // levels::lay (levels.rs:225-385)
  std::vector<Node> world_nodes;
  std::vector<uint32_t> world_order;
  bvh_triangles(s.world, s.world_count, world_nodes, world_order);
  std::vector<MeshOut> meshes;
  std::vector<int> placed_of(s.instance_count, -1);
  std::vector<PlacedOut> placed;
  uint32_t slots = s.world_count;
  out.bottom_builds = s.world_count > 0 ? 1 : 0;
  if (s.instance_count == 0) {
    out.nodes = world_nodes;
  } else {
    struct Known {
      uint32_t source;
      uint64_t hash;
      size_t mesh;
    };
    std::vector<Known> known;
    uint32_t next = s.world_count, record = 0;
    for (uint32_t i = 0; i < s.instance_count; ++i) {
      const InInstance& in = s.instances[i];
      const InMesh& src = s.meshes[in.mesh];
      if (src.count == 0) continue;
      bool alone = unique[i];
      bool one = true;
      for (uint32_t t = 1; t < src.count; ++t) one = one && src.tris[t].material == src.tris[0].material;
      auto fits = [&](const MeshOut& m) {
        if (one) return true;
        for (size_t k = 0; k < m.order.size(); ++k)
          if (src.tris[m.order[k]].material != m.tris[k].material) return false;
        return true;
      };
      bool shared = false;
      for (auto& k : known) shared = shared || k.source == in.mesh;
      bool hashed = false;
      uint64_t hash = 0;
      long found = -1;
      if (!alone) {
        for (auto& k : known)
          if (k.source == in.mesh && fits(meshes[k.mesh])) {
            found = (long)k.mesh;
            break;
          }
        if (found < 0) {
          hash = geometry_hash(src.tris, src.count);
          hashed = true;
          for (auto& k : known) {
            const MeshOut& m = meshes[k.mesh];
            if (k.hash != hash || m.order.size() != src.count || !fits(m)) continue;
            bool same = true;
            for (size_t j = 0; j < m.order.size() && same; ++j) same = same_geometry(src.tris[m.order[j]], m.tris[j]);
            if (same) {
              found = (long)k.mesh;
              break;
            }
          }
        }
      }
      size_t mi;
      if (found >= 0) {
        mi = (size_t)found;
      } else {
        MeshOut m;
        bvh_triangles(src.tris, src.count, m.nodes, m.order);
        out.bottom_builds += 1;
        m.bounds = box_empty();
        if (!m.nodes.empty())
          for (int k = 0; k < 3; ++k) {
            m.bounds.lo[k] = m.nodes[0].lo[k];
            m.bounds.hi[k] = m.nodes[0].hi[k];
          }
        for (uint32_t j : m.order) m.tris.push_back(src.tris[j]);
        m.first = next;
        next += src.count;
        meshes.push_back(std::move(m));
        mi = meshes.size() - 1;
      }
      if (!alone && !shared) known.push_back(Known{in.mesh, hashed ? hash : geometry_hash(src.tris, src.count), mi});
      record += 1;
      // place (levels.rs:188-222)
      PlacedOut p;
      p.mesh = mi;
      p.base = meshes[mi].first;
      p.record = record;
      p.word = words[i];
      p.one = one;
      p.material = src.tris[0].material;
      p.pose = pose_of(in.transform);
      p.bounds = placed_bounds(p.pose, meshes[mi].bounds);
      pose_inverse_rows(p.pose, p.inverse);
      placed_of[i] = (int)placed.size();
      placed.push_back(p);
    }
    slots = next;
    bool world = !world_nodes.empty();
    size_t groups_n = (world ? 1 : 0) + placed.size();
    uint32_t top_len = groups_n == 0 ? 0 : (uint32_t)(3 * groups_n - 1);  // Levels::top_len, room 0
    uint32_t offset = top_len, world_root = 0;
    if (world) {
      world_root = offset;
      offset += (uint32_t)world_nodes.size();
    }
    for (auto& m : meshes) {
      m.root = offset;
      offset += (uint32_t)m.nodes.size();
    }
    // Levels::top (levels.rs:393-470)
    struct Group {
      Box3 bounds;
      uint32_t root, base, record;
      const float* inverse;
    };
    std::vector<Group> groups;
    if (world) {
      Group g;
      for (int k = 0; k < 3; ++k) {
        g.bounds.lo[k] = world_nodes[0].lo[k];
        g.bounds.hi[k] = world_nodes[0].hi[k];
      }
      g.root = world_root;
      g.base = 0;
      g.record = 0;
      g.inverse = nullptr;
      groups.push_back(g);
    }
    for (auto& p : placed) groups.push_back(Group{p.bounds, meshes[p.mesh].root, p.base, p.record, p.inverse});
    std::vector<Box3> boxes;
    for (auto& g : groups) boxes.push_back(g.bounds);
    std::vector<Node> top;
    std::vector<uint32_t> top_order;
    bvh_over(boxes, 1, 0, top, top_order);
    uint32_t tree = (uint32_t)top.size();
    for (auto node : top) {
      if (node.count > 0) {
        uint32_t index = top_order[node.first];
        const Group& g = groups[index];
        node.first = g.root;
        node.count = g.base;
        node.lo[3] = bitsf(g.record);
        node.pad[0] = 1;  // INSTANCE_LEAF
        node.pad[1] = g.inverse ? tree + index : 0u;
      }
      out.nodes.push_back(node);
    }
    for (auto& g : groups) {
      const float* r = g.inverse ? g.inverse : IDENTITY_ROWS;
      Node n;
      memcpy(n.lo, r, 16);
      memcpy(n.hi, r + 4, 16);
      n.first = fbits(r[8]);
      n.count = fbits(r[9]);
      n.pad[0] = fbits(r[10]);
      n.pad[1] = fbits(r[11]);
      out.nodes.push_back(n);
    }
    out.nodes.resize(top_len);
    auto shifted = [&](const std::vector<Node>& src, uint32_t off) {  // levels.rs:97-108
      for (Node n : src) {
        if (n.count == 0) n.first += off;
        out.nodes.push_back(n);
      }
    };
    if (world) shifted(world_nodes, world_root);
    for (auto& m : meshes) shifted(m.nodes, m.root);
  }
  out.order = world_order;

  // triangles in slot order (gpu.rs:765-780)
  for (uint32_t k = 0; k < s.world_count; ++k) {
    const InTri& t = s.world[world_order[k]];
    out.triangles.push_back(pack_triangle(t));
    out.uv.push_back(F4{{t.uv[0][1], t.uv[1][1], t.uv[2][1], 0.0f}});
  }
  for (auto& m : meshes)
    for (auto& t : m.tris) {
      out.triangles.push_back(pack_triangle(t));
      out.uv.push_back(F4{{t.uv[0][1], t.uv[1][1], t.uv[2][1], 0.0f}});
    }

  // surface records (gpu.rs:781-805)
  {
    uint32_t info[4] = {0u, NO_MATERIAL, 0u, fbits(1.0f)};
    out.surfaces.push_back(surface_of(info, IDENTITY_ROWS, IDENTITY_ROWS));
  }
  for (uint32_t i = 0; i < s.instance_count; ++i) {
    if (placed_of[i] < 0) continue;
    const PlacedOut& p = placed[placed_of[i]];
    uint32_t info[4] = {p.word, p.one ? p.material : NO_MATERIAL, fbits(0.5f),
                        fbits(pose_inverse_determinant(p.pose))};
    float fwd[12];
    pose_rows(p.pose, fwd);
    out.surfaces.push_back(surface_of(info, fwd, p.inverse));
  }

  // emitter candidates: world triangles in slot order, then the triangles of
  // instances that carry their own (gpu.rs:826-910)
  std::vector<Candidate> cands;
  auto mark = [&](size_t slot) { out.triangles[slot].c[3] = (float)cands.size(); };
  for (uint32_t k = 0; k < s.world_count; ++k) {
    const InTri& t = s.world[world_order[k]];
    if (emitting[t.material] && triangle_area(t.v) > 1e-12f) {
      Candidate c;
      memcpy(c.v, t.v, sizeof(c.v));
      c.record = 0;
      memcpy(c.emission, out.materials[t.material + 1].rows[5], 12);
      cands.push_back(c);
      mark(k);
    }
  }
  for (uint32_t i = 0; i < s.instance_count; ++i) {
    if (placed_of[i] < 0 || !unique[i]) continue;
    const PlacedOut& p = placed[placed_of[i]];
    const MeshOut& m = meshes[p.mesh];
    for (size_t j = 0; j < m.tris.size(); ++j) {
      uint32_t material = p.one ? p.material : m.tris[j].material;
      float v[3][3];
      for (int c = 0; c < 3; ++c) {
        P3 w = pose_point(p.pose, m.tris[j].v[c]);
        v[c][0] = w.x;
        v[c][1] = w.y;
        v[c][2] = w.z;
      }
      if (emitting[material] && triangle_area(v) > 1e-12f) {
        Candidate c;
        memcpy(c.v, v, sizeof(v));
        c.record = p.record;
        memcpy(c.emission, out.materials[material + 1].rows[5], 12);
        cands.push_back(c);
        mark(m.first + j);
      }
    }
  }

  // lights and the emitter list (gpu.rs:1011-1013)
  size_t looped = 0, tree = 0;
  lay_lights(s.lights, s.light_count, out, &looped, &tree);
  build_emitters(cands, looped, tree, out);

  // uniform environment: SkyCdf::build (sky.rs:212-275) without a sun
  uint32_t w = s.sky_width > 1 ? s.sky_width : 1, h = s.sky_height > 1 ? s.sky_height : 1;
  out.sky_width = w;
  out.sky_height = h;
  memcpy(out.sky_radiance, s.sky, 12);
  out.sky_rows.assign(h, 0.0f);
  out.sky_columns.assign((size_t)w * h, 0.0f);
  double total = 0.0;
  float lum = fmax_r(luminance(s.sky), 0.0f);
  for (uint32_t row = 0; row < h; ++row) {
    float theta = PI_F * ((float)row + 0.5f) / (float)h;
    float sine = sinf(theta);
    double row_total = 0.0;
    for (uint32_t col = 0; col < w; ++col) {
      row_total += (double)lum * (double)sine;
      out.sky_columns[(size_t)row * w + col] = (float)row_total;
    }
    for (uint32_t col = 0; col < w; ++col) {
      float& c = out.sky_columns[(size_t)row * w + col];
      c = row_total > 0.0 ? c / (float)row_total : (float)(col + 1) / (float)w;
    }
    total += row_total;
    out.sky_rows[row] = (float)total;
  }
  for (uint32_t row = 0; row < h; ++row)
    out.sky_rows[row] = total > 0.0 ? out.sky_rows[row] / (float)total : (float)(row + 1) / (float)h;

  // the Sobol table (sobol.rs:33-39, 138-153): 256 patterns of `length` points
  if (s.sobol) {
    uint32_t length = orc_sequence_size(s.sobol_samples);
    out.sobol_length = length;
    out.sobol.assign((size_t)length * 256 * 4, 0.0f);
    parallel_for(256, 1, [&](int64_t pattern, unsigned) {
      orc_generate_4d(out.sobol.data() + (size_t)pattern * length * 4, length, (uint32_t)pattern);
    });
  }
  out.triangle_count = slots;
  out.emitter_count = (uint32_t)cands.size();
  out.light_count = s.light_count;
}

}  // namespace orcpack

extern "C" {

void* orc_scene_build(const void* scene) {
  auto* b = new orcpack::Blobs();
  orcpack::build(*static_cast<const orcpack::InScene*>(scene), *b);
  return b;
}

void orc_scene_free(void* blobs) { delete static_cast<orcpack::Blobs*>(blobs); }

// The tree's selection on bare keys (tests): the keys' original indices in the
// order select_nth_unstable_by(index, total_cmp) leaves them.
void orc_select_nth(const float* keys, uint32_t n, uint32_t index, int32_t rounds, uint32_t* order) {
  struct Keyed {
    float centroid[1];
    uint32_t at;
  };
  std::vector<Keyed> v(n);
  for (uint32_t i = 0; i < n; ++i) v[i] = Keyed{{keys[i]}, i};
  orcpack::SelectOf<Keyed> sel{v, 0, rounds};
  sel.run(0, n, index);
  for (uint32_t i = 0; i < n; ++i) order[i] = v[i].at;
}

// Blob `which` of a built scene: 0 nodes, 1 triangles, 2 uv, 3 surfaces,
// 4 materials, 5 emitters, 6 emitter_cdf, 7 lights, 8 order, 9 sky rows,
// 10 sky columns, 11 sobol.  Returns its byte size and sets *data.
uint64_t orc_scene_blob(void* blobs, int which, const void** data) {
  auto& b = *static_cast<orcpack::Blobs*>(blobs);
  auto give = [&](const void* p, size_t bytes) {
    *data = p;
    return (uint64_t)bytes;
  };
  switch (which) {
    case 0: return give(b.nodes.data(), b.nodes.size() * sizeof(Node));
    case 1: return give(b.triangles.data(), b.triangles.size() * sizeof(orcpack::GpuTri));
    case 2: return give(b.uv.data(), b.uv.size() * 16);
    case 3: return give(b.surfaces.data(), b.surfaces.size() * sizeof(orcpack::GpuSurf));
    case 4: return give(b.materials.data(), b.materials.size() * sizeof(orcpack::Hot));
    case 5: return give(b.emitters.data(), b.emitters.size() * sizeof(orcpack::Row4));
    case 6: return give(b.emitter_cdf.data(), b.emitter_cdf.size() * 4);
    case 7: return give(b.lights.data(), b.lights.size() * sizeof(orcpack::Row4));
    case 8: return give(b.order.data(), b.order.size() * 4);
    case 9: return give(b.sky_rows.data(), b.sky_rows.size() * 4);
    case 10: return give(b.sky_columns.data(), b.sky_columns.size() * 4);
    case 11: return give(b.sobol.data(), b.sobol.size() * 4);
    default: *data = nullptr; return 0;
  }
}

// Counts of a built scene: triangle slots, emitters, lights, sky width and
// height, Sobol length, bottom-level builds.
void orc_scene_counts(void* blobs, uint32_t out[7]) {
  auto& b = *static_cast<orcpack::Blobs*>(blobs);
  uint32_t v[7] = {b.triangle_count, b.emitter_count, b.light_count, b.sky_width, b.sky_height, b.sobol_length,
                   b.bottom_builds};
  memcpy(out, v, sizeof(v));
}

}  // extern "C"
