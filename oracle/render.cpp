// TEST INFRASTRUCTURE ONLY - included at the end of oracle.cpp (one
// translation unit).  The CPU restatement of the reference's path integrator:
// main() and radiance() of crates/trace/src/trace.wgsl, the light sampling of
// lights.wgsl, the BSDF of crates/materials/src/wgsl/brdf.wgsl, the Sobol
// lookup of sobol.wgsl and the sky sampling of sky.rs (SKY_SAMPLING_WGSL),
// for the feature set the B200 tracer covers (no fog, sprites, steam, matte
// catcher, content layers, texture maps, lobes, wet, flakes, thin film,
// motion, analytic shapes, transmissive shadows).  Expressions keep the
// reference's operand order: WGSL evaluates a*b*c as (a*b)*c.
//
// Scope rules checked by the restatement: a material with thin film (both
// thin_film and thin_film_amount > 0) is outside the scope and is rejected by
// the product when the scene is packed.

namespace orc {

struct Light {
  float a[4], b[4], c[4], d[4];
};
struct Emitter {
  float a[4], b[4], c[4], e[4];
};

struct Shaded {  // brdf.wgsl:9-30
  v3 base;
  float roughness, metalness, specular, clearcoat, clearcoat_roughness, sheen, transmission, ior, dispersion,
      thickness, subsurface;
  v3 subsurface_tint;
  float absorption, thin_film, thin_film_ior, thin_film_amount;
  v3 emission;
  float fresnel_power;
};

}  // namespace orc

extern "C" {

// Everything a pass reads: the SceneBuffers bytes, the sky CDF, the Sobol
// table, the Frame fields and the pipeline constants.
struct OrcScene {
  const void* nodes;
  uint32_t node_count;
  const void* tris;
  uint32_t tri_count;
  const void* surfaces;
  const float* materials;  // rows of 4 floats
  uint32_t material_rows;
  const void* emitters;
  const float* emitter_cdf;
  const void* lights;
  const float* sky_rows;
  const float* sky_columns;
  uint32_t sky_width, sky_height;
  float sky_radiance[3];
  float sky_sun_probability;
  const float* sobol;  // RGBA per texel
  uint32_t sobol_length;
  uint32_t sobol_on;
  uint32_t bounces[4];  // total, diffuse, glossy, transmission
  float clamp_indirect, filter_glossy;
};

struct OrcFrame {  // Frame (trace.wgsl:1-16) fields the integrator reads
  uint32_t size[4];
  uint32_t counts[4];
  float origin[4], forward[4], right[4], up[4], sun_dir[4], sun_color[4], lens[4];
  uint32_t window[4];
};

}  // extern "C"

namespace orc {

const float PI = 0x1.921fb6p+1f;  // brdf.wgsl:1 `const PI: f32 = 3.141592653589793`
const uint32_t NO_MATERIAL = 0xffffffffu;

struct Ctx {
  const OrcScene* sc;
  const OrcFrame* fr;
  Scene geo;
  // private per-invocation state (var<private> rng, trace.wgsl:427)
  uint32_t rng[3];
};

// ------------------------------------------------------------------ random
// pcg (trace.wgsl:168-172)
uint32_t pcg(uint32_t v) {
  uint32_t s = v * 747796405u + 2891336453u;
  uint32_t w = ((s >> ((s >> 28u) + 4u)) ^ s) * 277803737u;
  return (w >> 22u) ^ w;
}
// random (trace.wgsl:423-426)
float random(uint32_t* state) {
  *state = pcg(*state);
  return (float)(*state >> 8u) / 16777216.0f;
}
// hash_iqnt2d (trace.wgsl:428-432)
uint32_t hash_iqnt2d(uint32_t x, uint32_t y) {
  uint32_t qx = 1103515245u * ((x >> 1u) ^ y);
  uint32_t qy = 1103515245u * ((y >> 1u) ^ x);
  return 1103515245u * (qx ^ (qy >> 3u));
}
// sobol.wgsl:2-46
uint32_t reversed_bit_owen(uint32_t n, uint32_t seed) {
  n ^= n * 0x3d20adeau;
  n += seed;
  n *= (seed >> 16u) | 1u;
  n ^= n * 0x05526c56u;
  n ^= n * 0x53a22864u;
  return n;
}
uint32_t nested_uniform_scramble(uint32_t i, uint32_t seed) { return brev_(reversed_bit_owen(brev_(i), seed)); }
uint32_t hash_wang_seeded_uint(uint32_t i0, uint32_t seed) {
  uint32_t i = (i0 ^ 61u) ^ seed;
  i += i << 3u;
  i ^= i >> 4u;
  i *= 0x27d4eb2du;
  return i;
}
uint32_t hash_shuffle_uint(uint32_t i0, uint32_t length, uint32_t seed) {
  uint32_t i = i0 % length;
  uint32_t mask = (1u << (32u - clz_(length - 1u))) - 1u;
  for (;;) {
    i ^= seed;
    i *= 0xe170893du;
    i ^= seed >> 16u;
    i ^= (i & mask) >> 4u;
    i ^= seed >> 8u;
    i *= 0x0929eb3fu;
    i ^= seed >> 23u;
    i ^= (i & mask) >> 1u;
    i *= 1u | (seed >> 27u);
    i *= 0x6935fa69u;
    i ^= (i & mask) >> 11u;
    i *= 0x74dcb303u;
    i ^= (i & mask) >> 2u;
    i *= 0x9e501cc3u;
    i ^= (i & mask) >> 2u;
    i *= 0xc860a3dfu;
    i &= mask;
    i ^= i >> 5u;
    if (i < length) break;
  }
  return i;
}
struct V4 {
  float x, y, z, w;
};
// sobol (sobol.wgsl:47-58)
V4 sobol(Ctx& c, uint32_t dimension) {
  if (!c.sc->sobol_on) return V4{0, 0, 0, 0};
  uint32_t L = c.sc->sobol_length;
  uint32_t seed = c.rng[0];
  uint32_t dim = c.rng[2] + dimension;
  uint32_t pattern = hash_shuffle_uint(dim, 256u, seed);
  uint32_t mask = L - 1u;
  uint32_t shuffled = nested_uniform_scramble(c.rng[1], hash_wang_seeded_uint(dim, seed));
  uint32_t sample = (c.rng[1] & ~mask) | (shuffled & mask);
  uint32_t index = (pattern * L + sample) % (L * 256u);
  const float* t = c.sc->sobol + 4 * (size_t)index;
  float sh[4] = {(float)hash_wang_seeded_uint(dim, seed), (float)hash_wang_seeded_uint(dim, seed ^ 0xca0e1151u),
                 (float)hash_wang_seeded_uint(dim, seed ^ 0xbf604c5au),
                 (float)hash_wang_seeded_uint(dim, seed ^ 0x99634d1du)};
  float out[4];
  for (int k = 0; k < 4; ++k) out[k] = fmin_(fract_(t[k] + sh[k] * 2.3283064e-10f), 0.99999994f);
  return V4{out[0], out[1], out[2], out[3]};
}
// rnd (trace.wgsl:440-443)
float rnd(Ctx& c, uint32_t* state, float value) {
  if (c.sc->sobol_on) return value;
  return random(state);
}
// light_dim (trace.wgsl:444-448)
uint32_t light_dim(uint32_t k) {
  if (k == 0u) return 1u;
  if (k < 13u) return 3u + k;
  return k << 16u;
}

// ------------------------------------------------------------------ records
const float* mat_row(const Ctx& c, uint32_t material, uint32_t row) {
  return c.sc->materials + 4 * ((size_t)(material + 1u) * 8u + row);
}
Shaded surface(const Ctx& c, uint32_t material) {  // trace.wgsl:1274-1282
  const float* r0 = mat_row(c, material, 0);
  const float* r1 = mat_row(c, material, 1);
  const float* r2 = mat_row(c, material, 2);
  const float* r3 = mat_row(c, material, 3);
  const float* r4 = mat_row(c, material, 4);
  const float* r5 = mat_row(c, material, 5);
  const float* r6 = mat_row(c, material, 6);
  Shaded s;
  s.base = mk3(r0[0], r0[1], r0[2]);
  s.roughness = r0[3];
  s.metalness = r1[0];
  s.specular = r1[1];
  s.clearcoat = r1[2];
  s.clearcoat_roughness = r1[3];
  s.sheen = r2[0];
  s.transmission = r2[1];
  s.ior = r2[2];
  s.dispersion = r2[3];
  s.thickness = r3[0];
  s.subsurface = r3[1];
  s.subsurface_tint = mk3(r4[0], r4[1], r4[2]);
  s.absorption = r4[3];
  s.thin_film = r3[2];
  s.thin_film_ior = r3[3];
  s.thin_film_amount = r5[3];
  s.emission = mk3(r5[0], r5[1], r5[2]);
  s.fresnel_power = r6[0];
  return s;
}
const Light& light_at(const Ctx& c, uint32_t i) { return ((const Light*)c.sc->lights)[i]; }
const Emitter& emitter_at(const Ctx& c, uint32_t i) { return ((const Emitter*)c.sc->emitters)[i]; }
const Surface& surface_at(const Ctx& c, uint32_t r) { return ((const Surface*)c.sc->surfaces)[r]; }
v3 xyz(const float* p) { return mk3(p[0], p[1], p[2]); }

// ------------------------------------------------------------------ brdf.wgsl
float dielectric_f0(float ior) {
  float r = (ior - 1.0f) / (ior + 1.0f);
  return r * r;
}
v3 dispersed_ior(float ior, float dispersion) {
  return mk3(ior + -0.016f * dispersion, ior, ior + 0.022f * dispersion);
}
v3 schlick(v3 f0, float cos_theta, float power) {
  float k = pow_(1.0f - clamp_(cos_theta, 0.0f, 1.0f), power);
  return mix3(f0, splat3(1.0f), k);
}
float fresnel_dielectric(float cos_theta, float eta_in) {
  float c = clamp_(cos_theta, 0.0f, 1.0f);
  float eta = eta_in;
  if (abs_(eta) < 1e-4f) eta = 1.0f;
  float s2 = 1.0f - c * c;
  float t2 = 1.0f - s2 / (eta * eta);
  if (t2 <= 0.0f) return 1.0f;
  float ct = sqrtf(t2);
  float rs = (c - eta * ct) / (c + eta * ct);
  float rp = (eta * c - ct) / (eta * c + ct);
  return 0.5f * (rs * rs + rp * rp);
}
float ggx_d(float nh, float a2) {
  float n = fmax_(nh, 0.0f);
  float k = n * n * (a2 - 1.0f) + 1.0f;
  return a2 / (PI * k * k);
}
float smith_g1(float ndot, float a2) {
  float n = fmax_(ndot, 0.0f);
  return 2.0f * n / (n + sqrtf(a2 + (1.0f - a2) * n * n));
}
float smith_g(float ndv, float ndl, float a2) { return smith_g1(ndv, a2) * smith_g1(ndl, a2); }
float alpha_rough(float roughness) {
  float rough = clamp_(roughness, 0.02f, 1.0f);
  return rough * rough;
}
v3 beer(float distance, v3 tint, float absorption) {
  if (distance <= 0.0f || absorption <= 0.0f) return splat3(1.0f);
  return mk3(exp_(-distance * absorption * fmax_(1.0f - tint.x, 0.0f)),
             exp_(-distance * absorption * fmax_(1.0f - tint.y, 0.0f)),
             exp_(-distance * absorption * fmax_(1.0f - tint.z, 0.0f)));
}
v3 refract_dir(v3 incident, v3 normal, float eta, float* w) {
  float cos_i = dot3(normal, incident);
  float k = 1.0f - eta * eta * (1.0f - cos_i * cos_i);
  if (k < 0.0f) {
    *w = 0.0f;
    return splat3(0.0f);
  }
  float t = eta * cos_i + sqrtf(k);
  *w = 1.0f;
  return sub3(scl3(incident, eta), scl3(normal, t));
}
float fresnel_exponent(const Shaded& s) { return s.fresnel_power <= 0.0f ? 5.0f : s.fresnel_power; }
// reflection_filmed without film (brdf.wgsl:206-228)
v3 reflection(const Shaded& s, float ndh_cos) {
  float power = fresnel_exponent(s);
  v3 f0 = mix3(splat3(s.specular), s.base, clamp_(s.metalness, 0.0f, 1.0f));
  v3 plain;
  if (s.transmission > 0.0f || s.dispersion != 0.0f) {
    v3 iors = dispersed_ior(s.ior, s.dispersion);
    v3 metal = schlick(s.base, ndh_cos, power);
    v3 diel = mk3(fresnel_dielectric(ndh_cos, iors.x), fresnel_dielectric(ndh_cos, iors.y),
                  fresnel_dielectric(ndh_cos, iors.z));
    plain = mix3(diel, metal, clamp_(s.metalness, 0.0f, 1.0f));
  } else if (f0.x <= 0.0f && f0.y <= 0.0f && f0.z <= 0.0f) {
    plain = splat3(0.0f);
  } else {
    plain = schlick(f0, ndh_cos, power);
  }
  return plain;
}
v3 ggx_spec(float ndv, float ndl, float ndh, float a2, v3 fresnel) {
  return divs3(scl3(scl3(fresnel, ggx_d(ndh, a2)), smith_g(ndv, ndl, a2)), 4.0f * ndv * ndl);
}
// eval_filmed without film (brdf.wgsl:242-283)
v3 eval(const Shaded& s, v3 wo, v3 wi) {
  float ndv = wo.z;
  if (ndv <= 1e-5f) return splat3(0.0f);
  float ndl = wi.z;
  if (abs_(ndl) <= 1e-8f) return splat3(0.0f);
  float metal = clamp_(s.metalness, 0.0f, 1.0f);
  float trans = clamp_(s.transmission, 0.0f, 1.0f);
  float sss = clamp_(s.subsurface, 0.0f, 1.0f) * (1.0f - trans);
  float sheen = clamp_(s.sheen, 0.0f, 1.0f);
  float sheen_cover = sheen * pow_(1.0f - ndv, 4.0f);
  float view = clamp_(ndv, 0.0f, 1.0f);
  if (ndl < 0.0f) {
    v3 fresnel = reflection(s, view);
    v3 transmitted = sub3(splat3(1.0f), fresnel);
    float back = (1.0f - metal) * sss + trans * (1.0f - metal);
    v3 tint = beer(s.thickness, s.subsurface_tint, s.absorption);
    return divs3(scl3(mul3(mul3(s.base, tint), transmitted), back), PI);
  }
  v3 h = normalize3(add3(wo, wi));
  float ndh = fmax_(h.z, 0.0f);
  float vdh = fmax_(dot3(wo, h), 0.0f);
  v3 fresnel = reflection(s, vdh);
  float a = alpha_rough(s.roughness);
  v3 spec = ggx_spec(ndv, ndl, ndh, a * a, fresnel);
  v3 transmitted = sub3(splat3(1.0f), fresnel);
  float body = (1.0f - metal) * (1.0f - trans) * (1.0f - sss);
  float diffuse_w = body * (1.0f - sheen_cover);
  float sheen_w = body * sheen_cover * pow_(1.0f - ndh, 5.0f);
  v3 colour = add3(spec, divs3(scl3(mul3(s.base, transmitted), diffuse_w + sheen_w), PI));
  float coat = clamp_(s.clearcoat, 0.0f, 1.0f);
  if (coat > 0.0f) {
    float coat_a = alpha_rough(s.clearcoat_roughness);
    v3 coat_f = schlick(splat3(0.04f), vdh, fresnel_exponent(s));
    v3 coat_spec = ggx_spec(ndv, ndl, ndh, coat_a * coat_a, coat_f);
    float fc = schlick(splat3(0.04f), view, fresnel_exponent(s)).x;
    colour = add3(scl3(coat_spec, coat), scl3(colour, 1.0f - coat * fc));
  }
  return colour;
}

// ----------------------------------------------------- trace.wgsl BSDF use
float glossy_share(const Shaded& s) {  // trace.wgsl:1713-1715
  return 1.0f - clamp_(s.transmission, 0.0f, 1.0f) * (1.0f - clamp_(s.metalness, 0.0f, 1.0f));
}
v3 channel_mask(uint32_t ch) {
  return mk3(ch == 0u ? 1.0f : 0.0f, ch == 1u ? 1.0f : 0.0f, ch == 2u ? 1.0f : 0.0f);
}
float channel_ior(const Shaded& s, uint32_t ch) {
  if (ch > 2u) return fmax_(s.ior, 1.01f);
  return fmax_(get3(dispersed_ior(s.ior, s.dispersion), (int)ch), 1.01f);
}
float coat_weight_of(const Shaded& s, v3 wo) {
  return clamp_(s.clearcoat * (0.12f + 0.88f * (0.04f + 0.96f * pow_(1.0f - fmax_(wo.z, 0.0f), 5.0f))), 0.0f, 0.9f);
}
// bsdf_pdf (trace.wgsl:1774-1788)
float bsdf_pdf(const Shaded& s, v3 wo, v3 wi) {
  if (wi.z <= 0.0f) return 0.0f;
  float trans = clamp_(s.transmission, 0.0f, 1.0f) * (1.0f - clamp_(s.metalness, 0.0f, 1.0f));
  float coat = coat_weight_of(s, wo);
  float spec = (1.0f - coat) * clamp_(s.metalness + s.specular, 0.0f, 0.9f);
  v3 h = normalize3(add3(wo, wi));
  float a = alpha_rough(s.roughness);
  float ca = alpha_rough(s.clearcoat_roughness);
  float denom = fmax_(4.0f * abs_(dot3(wi, h)), 1e-8f);
  float base_pdf = ggx_d(fmax_(h.z, 0.0f), a * a) * fmax_(h.z, 0.0f) / denom;
  float coat_pdf = ggx_d(fmax_(h.z, 0.0f), ca * ca) * fmax_(h.z, 0.0f) / denom;
  return (1.0f - trans) * (coat * coat_pdf + spec * base_pdf + (1.0f - coat - spec) * wi.z / PI);
}
struct LightSample {
  v3 dir;
  float pdf;
  uint32_t channel;
  v3 weight;
  uint32_t lobe;
};
// sample_bsdf (trace.wgsl:1716-1773) without thin walls, lobes and flakes
LightSample sample_bsdf(Ctx& c, const Shaded& s, v3 wo, bool entering, uint32_t carried, uint32_t* state, V4 u) {
  float transmission = clamp_(s.transmission, 0.0f, 1.0f) * (1.0f - clamp_(s.metalness, 0.0f, 1.0f));
  if (rnd(c, state, u.w) < transmission) {
    v3 iors = dispersed_ior(s.ior, s.dispersion);
    uint32_t channel = carried;
    v3 weight = splat3(1.0f);
    if (channel > 2u && fmax_(abs_(iors.x - iors.y), abs_(iors.z - iors.y)) > 1e-4f) {
      uint32_t ch = f2u(rnd(c, state, u.z) * 3.0f);
      channel = ch < 2u ? ch : 2u;
      weight = scl3(channel_mask(channel), 3.0f);
    }
    float ior = channel_ior(s, channel);
    float ratio = entering ? ior : 1.0f / ior;
    v3 live = channel > 2u ? splat3(1.0f) : channel_mask(channel);
    v3 fresnel = mul3(splat3(fresnel_dielectric(fmax_(wo.z, 0.0f), ratio)), live);
    float chance = dot3(fresnel, splat3(1.0f)) / dot3(live, splat3(1.0f));
    v3 incident = neg3(wo);
    v3 mirrored = reflect3(incident, mk3(0.0f, 0.0f, 1.0f));
    if (rnd(c, state, u.x) < chance) return LightSample{mirrored, -1.0f, channel, divs3(mul3(weight, fresnel), chance), 1u};
    float rw;
    v3 refracted = refract_dir(incident, mk3(0.0f, 0.0f, 1.0f), 1.0f / ratio, &rw);
    if (rw > 0.0f)
      return LightSample{normalize3(refracted), -2.0f, channel, divs3(mul3(weight, sub3(live, fresnel)), 1.0f - chance),
                         2u};
    return LightSample{mirrored, -1.0f, channel, mul3(weight, live), 1u};
  }
  float coat_weight = coat_weight_of(s, wo);
  float spec_weight = (1.0f - coat_weight) * clamp_(s.metalness + s.specular, 0.0f, 0.9f);
  float pick = rnd(c, state, u.z);
  if (pick < coat_weight + spec_weight) {
    bool coat = pick < coat_weight;
    float alpha = alpha_rough(coat ? s.clearcoat_roughness : s.roughness);
    float u1 = rnd(c, state, u.x);
    float u2 = rnd(c, state, u.y);
    float phi = 2.0f * PI * u1;
    float cos_theta = sqrtf((1.0f - u2) / (1.0f + (alpha * alpha - 1.0f) * u2));
    float st = sqrtf(fmax_(0.0f, 1.0f - cos_theta * cos_theta));
    v3 h = mk3(cos_(phi) * st, sin_(phi) * st, cos_theta);
    v3 wi = reflect3(neg3(wo), h);
    return LightSample{wi, bsdf_pdf(s, wo, wi), 3u, splat3(1.0f), 1u};
  }
  float u1 = rnd(c, state, u.x);
  float u2 = rnd(c, state, u.y);
  float phi = 2.0f * PI * u1;
  float r = sqrtf(u2);
  v3 wi = mk3(cos_(phi) * r, sin_(phi) * r, sqrtf(1.0f - u2));
  return LightSample{wi, bsdf_pdf(s, wo, wi), 3u, splat3(1.0f), 0u};
}

// ------------------------------------------------------------------ sky
struct SkySample {
  v3 direction;
  v3 radiance;
  float pdf;
};
uint32_t sky_find(const float* cdf, uint32_t count, float needle) {
  uint32_t low = 0u, high = count;
  for (;;) {
    if (low >= high) break;
    uint32_t mid = (low + high) / 2u;
    if (cdf[mid] <= needle)
      low = mid + 1u;
    else
      high = mid;
  }
  return low < count - 1u ? low : count - 1u;
}
v3 sky_radiance(const Ctx& c) { return xyz(c.sc->sky_radiance); }
// sky_pdf (sky.rs SKY_SAMPLING_WGSL)
float sky_pdf(const Ctx& c, v3 direction) {
  const OrcScene& s = *c.sc;
  v3 d = normalize3(direction);
  float theta = acos_(clamp_(d.y, -1.0f, 1.0f));
  float phi = fmod_wgsl(atan2_(d.z, d.x) + 6.28318531f, 6.28318531f);
  uint32_t row = f2u(theta / 3.14159265f * (float)s.sky_height);
  row = row < s.sky_height - 1u ? row : s.sky_height - 1u;
  uint32_t col = f2u(phi / 6.28318531f * (float)s.sky_width);
  col = col < s.sky_width - 1u ? col : s.sky_width - 1u;
  float row_before = row > 0u ? s.sky_rows[(row > 1u ? row : 1u) - 1u] : 0.0f;
  float col_before = col > 0u ? s.sky_columns[row * s.sky_width + (col > 1u ? col : 1u) - 1u] : 0.0f;
  float mass = (s.sky_rows[row] - row_before) * (s.sky_columns[row * s.sky_width + col] - col_before);
  float area = 6.28318531f / (float)s.sky_width * 3.14159265f / (float)s.sky_height * fmax_(sin_(theta), 0.00001f);
  float sun_pdf = 0.0f;  // sun sampling is off (SkyCdf::without_sun)
  return (1.0f - s.sky_sun_probability) * mass / area + sun_pdf;
}
SkySample sky_sample(const Ctx& c, float rx, float ry) {
  const OrcScene& s = *c.sc;
  float u = clamp_(rx, 0.0f, 0.99999994f);
  float v = clamp_(ry, 0.0f, 0.99999994f);
  uint32_t row = sky_find(s.sky_rows, s.sky_height, v);
  float row_before = row > 0u ? s.sky_rows[(row > 1u ? row : 1u) - 1u] : 0.0f;
  float fy = (v - row_before) / fmax_(s.sky_rows[row] - row_before, 0.000001f);
  float needle = fmax_(u - s.sky_sun_probability, 0.0f) / fmax_(1.0f - s.sky_sun_probability, 0.000001f);
  const float* cols = s.sky_columns + (size_t)row * s.sky_width;
  uint32_t col = sky_find(cols, s.sky_width, needle);
  float col_before = col > 0u ? cols[(col > 1u ? col : 1u) - 1u] : 0.0f;
  float fx = (needle - col_before) / fmax_(cols[col] - col_before, 0.000001f);
  float theta = 3.14159265f * ((float)row + fy) / (float)s.sky_height;
  float phi = 6.28318531f * ((float)col + fx) / (float)s.sky_width;
  v3 direction = mk3(sin_(theta) * cos_(phi), cos_(theta), sin_(theta) * sin_(phi));
  float area = 6.28318531f / (float)s.sky_width * 3.14159265f / (float)s.sky_height * fmax_(sin_(theta), 0.00001f);
  float mass = (s.sky_rows[row] - row_before) * (cols[col] - col_before);
  float sun_pdf = 0.0f;
  return SkySample{direction, sky_radiance(c), (1.0f - s.sky_sun_probability) * mass / area + sun_pdf};
}

// ------------------------------------------------------------- offsets
// trace.wgsl:1257-1269
float offset_axis(float position, float normal) {
  if (abs_(position) < 1.0f / 32.0f) return position + normal / 65536.0f;
  int32_t bits = (int32_t)f2bits(position);
  int32_t shift = f2i(normal * 256.0f);
  return bits2f((uint32_t)(bits + (position < 0.0f ? -shift : shift)));
}
v3 offset_ray(v3 p, v3 n) { return mk3(offset_axis(p.x, n.x), offset_axis(p.y, n.y), offset_axis(p.z, n.z)); }
v3 spawn_point(v3 p, v3 dir, v3 origin, float t) {
  float err = 4e-7f * (fmax_(abs_(origin.x), fmax_(abs_(origin.y), abs_(origin.z))) + t);
  return add3(offset_ray(p, dir), scl3(dir, err));
}

// ------------------------------------------------------------------ lights.wgsl
float mis_power(float chosen, float other) {
  if (chosen <= 0.0f) return 0.0f;
  float ratio = other / chosen;
  return 1.0f / (1.0f + ratio * ratio);
}
uint32_t find_emitter(const Ctx& c, uint32_t count, float u) {
  uint32_t low = 0u, high = count;
  for (;;) {
    if (low >= high) break;
    uint32_t mid = (low + high) / 2u;
    if (c.sc->emitter_cdf[mid] <= u)
      low = mid + 1u;
    else
      high = mid;
  }
  return low < count - 1u ? low : count - 1u;
}
float cone_pdf(v3 apex, v3 center, float radius) {
  v3 to = sub3(center, apex);
  float distance2 = dot3(to, to);
  float r2 = radius * radius;
  if (distance2 <= r2) return 1.0f / (4.0f * PI);
  float cos_max = sqrtf(fmax_(1.0f - r2 / distance2, 0.0f));
  float open = (r2 / distance2) / (1.0f + cos_max);
  return 1.0f / (2.0f * PI * open);
}
float emitter_pdf(const Emitter& e, v3 x, v3 apex, v3 normal) {
  if (e.a[3] > 0.5f) return e.e[3] * cone_pdf(apex, xyz(e.a), e.c[0]);
  v3 to = sub3(x, apex);
  float distance2 = dot3(to, to);
  float cosine = abs_(dot3(normal, to)) / sqrtf(fmax_(distance2, 1e-30f));
  return e.e[3] / fmax_(e.c[3], 1e-30f) * distance2 / fmax_(cosine, 1e-7f);
}
struct HitInfo {
  float t;
  v3 n, geometric;
  uint32_t material, surface, shape, record;
};
float emitter_weight(const Ctx& c, const HitInfo& hit, v3 p, v3 previous_point, float previous_pdf) {
  const float* em = mat_row(c, hit.material, 5);
  if (previous_pdf <= 0.0f || (em[0] <= 0.0f && em[1] <= 0.0f && em[2] <= 0.0f)) return 1.0f;
  const Tri& tri = c.geo.tris[hit.surface];
  uint32_t index = f2u(tri.c[3]);
  if (index == 0u) return 1.0f;
  return mis_power(previous_pdf, emitter_pdf(emitter_at(c, index), p, previous_point, hit.geometric));
}
struct Frame4 {
  v3 n;
  float area;
};
Frame4 rect_frame(const Light& l) {
  v3 spanned = scl3(cross3(xyz(l.c), xyz(l.d)), 4.0f);
  float area = length3(spanned);
  return Frame4{divs3(spanned, area), area};
}
Frame4 area_frame(const Light& l) {
  if (f2u(l.a[3]) == 3u) return Frame4{xyz(l.c), PI * l.d[0] * l.d[0]};
  return rect_frame(l);
}
v3 light_hits(const Ctx& c, v3 o, v3 d, float limit, v3 previous_point, float previous_pdf) {
  uint32_t count = f2u(emitter_at(c, 0).a[1]);
  v3 total = splat3(0.0f);
  for (uint32_t i = 0u; i < count; ++i) {
    const Light& light = light_at(c, i);
    uint32_t kind = f2u(light.a[3]);
    if ((kind != 2u && kind != 3u) || light.d[3] < 0.5f) continue;
    Frame4 plane = area_frame(light);
    float facing = dot3(d, plane.n);
    if (abs_(facing) < 1e-9f || (light.c[3] < 0.5f && facing >= 0.0f)) continue;
    float t = dot3(sub3(xyz(light.a), o), plane.n) / facing;
    if (t <= 0.0001f || t >= limit) continue;
    v3 x = add3(o, scl3(d, t));
    v3 q = sub3(x, xyz(light.a));
    if (kind == 3u) {
      if (dot3(q, q) > light.d[0] * light.d[0]) continue;
    } else if (abs_(dot3(q, xyz(light.c))) > dot3(xyz(light.c), xyz(light.c)) ||
               abs_(dot3(q, xyz(light.d))) > dot3(xyz(light.d), xyz(light.d))) {
      continue;
    }
    float weight = 1.0f;
    if (previous_pdf > 0.0f) {
      v3 to = sub3(x, previous_point);
      float distance2 = dot3(to, to);
      float cosine = abs_(dot3(plane.n, to)) / sqrtf(fmax_(distance2, 1e-30f));
      weight = mis_power(previous_pdf, distance2 / (plane.area * fmax_(cosine, 1e-7f)));
    }
    total = add3(total, scl3(xyz(light.b), weight));
  }
  return total;
}
struct Candidate {
  v3 wi, scale;
  float pdf, roughness;
  v3 direction;
  float limit;
  uint32_t shape;
};
Candidate candidate_none() {
  return Candidate{mk3(0, 0, 1), splat3(0.0f), 0.0f, 0.0f, mk3(0, 0, 1), -1.0f, 0u};
}
struct ShadowRay {
  v3 dir;
  float limit;
};
ShadowRay shadow_ray(v3 origin, v3 aim, bool shadow) {
  if (!shadow) return ShadowRay{mk3(0, 0, 1), 0.0f};
  v3 ray = sub3(aim, origin);
  float distance = length3(ray);
  float limit = distance * 0.9999f - 0.0002f;
  if (limit <= 0.0f) return ShadowRay{mk3(0, 0, 1), 0.0f};
  return ShadowRay{divs3(ray, distance), limit};
}
Candidate emitter_candidate(Ctx& c, const m3& transform, v3 p, v3 origin, uint32_t* state, V4 u) {
  uint32_t count = f2u(emitter_at(c, 0).a[0]);
  const Emitter& e = emitter_at(c, find_emitter(c, count, rnd(c, state, u.z)) + 1u);
  Candidate out = candidate_none();
  if (e.a[3] > 0.5f) return out;  // analytic shape emitters: none in scope
  float r1 = sqrtf(rnd(c, state, u.x));
  float r2 = rnd(c, state, u.y);
  v3 x = add3(add3(scl3(xyz(e.a), 1.0f - r1), scl3(xyz(e.b), r1 * (1.0f - r2))), scl3(xyz(e.c), r1 * r2));
  if (clipped_at(surface_at(c, f2u(e.b[3])), x)) return out;
  v3 to = sub3(x, p);
  float distance2 = dot3(to, to);
  v3 direction = divs3(to, sqrtf(fmax_(distance2, 1e-30f)));
  v3 local = mulmtv(transform, direction);
  if (local.z <= 0.0f) return out;
  v3 normal = normalize3(cross3(sub3(xyz(e.b), xyz(e.a)), sub3(xyz(e.c), xyz(e.a))));
  if (abs_(dot3(normal, sub3(p, xyz(e.a)))) <= 1e-5f) return out;
  float cosine = abs_(dot3(normal, direction));
  if (cosine <= 1e-7f) return out;
  ShadowRay ray = shadow_ray(origin, x, true);
  return Candidate{local, xyz(e.e), e.e[3] / e.c[3] * distance2 / cosine, 0.0f, ray.dir, ray.limit, 0u};
}
Candidate light_candidate(Ctx& c, const Light& light, const m3& transform, v3 p, v3 origin, v3 geometric,
                          uint32_t* state, V4 u) {
  Candidate out = candidate_none();
  bool shadow = light.d[3] > 0.5f;
  uint32_t kind = f2u(light.a[3]);
  if (kind == 2u || kind == 3u) {
    float u1 = rnd(c, state, u.x);
    float u2 = rnd(c, state, u.y);
    Frame4 plane = area_frame(light);
    v3 x = add3(add3(xyz(light.a), scl3(xyz(light.c), 2.0f * u1 - 1.0f)), scl3(xyz(light.d), 2.0f * u2 - 1.0f));
    if (kind == 3u) {
      m3 disc = basis(xyz(light.c));
      float r = light.d[0] * sqrtf(u1);
      float phi = 2.0f * PI * u2;
      x = add3(add3(xyz(light.a), scl3(disc.c0, r * cos_(phi))), scl3(disc.c1, r * sin_(phi)));
    }
    v3 to = sub3(x, p);
    float distance2 = dot3(to, to);
    v3 direction = divs3(to, sqrtf(fmax_(distance2, 1e-30f)));
    v3 local = mulmtv(transform, direction);
    if (local.z <= 0.0f) return out;
    float facing = -dot3(plane.n, direction);
    float cosine = light.c[3] > 0.5f ? abs_(facing) : facing;
    if (cosine <= 1e-7f) return out;
    float pdf = distance2 / (plane.area * cosine);
    ShadowRay ray = shadow_ray(origin, x, shadow);
    if (!shadow) return Candidate{local, divs3(xyz(light.b), pdf), 0.0f, 0.0f, ray.dir, ray.limit, 0u};
    return Candidate{local, xyz(light.b), pdf, 0.0f, ray.dir, ray.limit, 0u};
  }
  v3 to = sub3(xyz(light.a), p);
  float distance = length3(to);
  float range = light.b[3];
  if (distance >= range || distance <= 1e-6f) return out;
  v3 l = divs3(to, distance);
  v3 local = mulmtv(transform, l);
  if (local.z <= 0.0f || dot3(geometric, l) <= 0.0f) return out;
  float cone = 1.0f;
  if (f2u(light.a[3]) == 1u) {
    float along = clamp_(dot3(neg3(l), xyz(light.c)) * light.d[0] + light.d[1], 0.0f, 1.0f);
    cone = along * along;
    if (cone <= 0.0f) return out;
  }
  float radius = light.c[3];
  v3 aim = xyz(light.a);
  if (shadow && radius > 0.0f) {
    m3 disc = basis(l);
    float r = radius * sqrtf(rnd(c, state, u.x));
    float phi = 2.0f * PI * rnd(c, state, u.y);
    aim = add3(aim, add3(scl3(disc.c0, r * cos_(phi)), scl3(disc.c1, r * sin_(phi))));
  }
  float ratio = distance / range;
  float window = clamp_(1.0f - ratio * ratio * ratio * ratio, 0.0f, 1.0f);
  float reach = fmax_(distance, radius);
  ShadowRay ray = shadow_ray(origin, aim, shadow);
  float roughness = sqrtf(clamp_(radius / (2.0f * distance), 0.0f, 1.0f));
  return Candidate{local, scl3(xyz(light.b), window * window * cone / (reach * reach)), 0.0f, roughness, ray.dir,
                   ray.limit, 0u};
}
float sin_from_cos(float c) { return sqrtf(fmax_(1.0f - c * c, 0.0f)); }
struct V2 {
  float x, y;
};
V2 tree_importance(v3 n, v3 to, float cos_u, v3 axis, float theta_o, float theta_e, float far, float near,
                   float energy) {
  float sin_u = sin_from_cos(cos_u);
  float cos_i = dot3(to, n);
  float sin_i = sin_from_cos(cos_i);
  float cos_min_i = cos_i >= cos_u ? 1.0f : cos_i * cos_u + sin_i * sin_u;
  if (cos_min_i < 0.0f) return V2{0.0f, 0.0f};
  float cos_max_i = fmax_(cos_i * cos_u - sin_i * sin_u, 0.0f);
  float cos_t = 1.0f, sin_t = 0.0f;
  v3 nt = neg3(to);
  if (axis.x != nt.x || axis.y != nt.y || axis.z != nt.z) {
    cos_t = dot3(axis, nt);
    sin_t = sin_from_cos(cos_t);
  }
  float cos_t_minus_u = cos_t * cos_u + sin_t * sin_u;
  float cos_o = cos_(theta_o);
  float sin_o = sin_(theta_o);
  float cos_min_out = 1.0f;
  if (cos_t >= cos_u || cos_t_minus_u >= cos_o) {
    cos_min_out = 1.0f;
  } else if (theta_o + theta_e > PI || cos_t_minus_u > cos_(theta_o + theta_e)) {
    cos_min_out = cos_t_minus_u * cos_o + sin_from_cos(cos_t_minus_u) * sin_o;
  } else {
    return V2{0.0f, 0.0f};
  }
  float most = abs_(cos_min_i * energy * cos_min_out / (near * near));
  float cos_t_plus_u = cos_t * cos_u - sin_t * sin_u;
  if (theta_e - theta_o < 0.0f || cos_t < 0.0f || cos_u < 0.0f || cos_t_plus_u < cos_(theta_e - theta_o))
    return V2{most, 0.0f};
  float cos_max_out = cos_t_plus_u * cos_o - sin_from_cos(cos_t_plus_u) * sin_o;
  return V2{most, abs_(cos_max_i * energy * cos_max_out / (far * far))};
}
V2 node_importance(const Light& node, v3 p, v3 n) {
  v3 centroid = scl3(add3(xyz(node.a), xyz(node.b)), 0.5f);
  v3 extent = sub3(xyz(node.b), centroid);
  if (dot3(n, sub3(centroid, p)) + dot3(abs3(n), abs3(extent)) <= 0.0f) return V2{0.0f, 0.0f};
  if (length3(sub3(p, clamp3(p, xyz(node.a), xyz(node.b)))) >= node.b[3]) return V2{0.0f, 0.0f};
  v3 to = sub3(centroid, p);
  float reach = length3(to);
  float radius2 = dot3(extent, extent);
  float cos_u = -1.0f;
  if (reach * reach > radius2) cos_u = sqrtf(fmax_(1.0f - radius2 / (reach * reach), 0.0f));
  float distance = fmax_(fmax_(0.5f * sqrtf(radius2), reach), 1e-6f);
  return tree_importance(n, divs3(to, fmax_(reach, 1e-30f)), cos_u, xyz(node.c), node.c[3], node.d[0], distance,
                         distance, node.a[3]);
}
float spot_cone(const Light& light, float cosine) {
  float along = clamp_(cosine * light.d[0] + light.d[1], 0.0f, 1.0f);
  return along * along;
}
V2 emitter_importance(const Light& light, v3 p, v3 n) {
  v3 to = sub3(xyz(light.a), p);
  float near = length3(to);
  if (near >= light.b[3] || near <= 1e-6f) return V2{0.0f, 0.0f};
  v3 toward = divs3(to, near);
  float radius = light.c[3];
  float far = sqrtf(radius * radius + near * near);
  float cos_u = near / far;
  float energy = (light.b[0] + light.b[1] + light.b[2]) / 3.0f;
  if (f2u(light.a[3]) == 1u) {
    float theta_e = acos_(clamp_(-light.d[1] / light.d[0], -1.0f, 1.0f));
    float cos_min_out =
        cos_(fmax_(0.0f, acos_(clamp_(dot3(xyz(light.c), neg3(toward)), -1.0f, 1.0f)) - acos_(cos_u)));
    energy = energy * spot_cone(light, cos_min_out);
    return tree_importance(n, toward, cos_u, xyz(light.c), 0.0f, theta_e, far, near, energy);
  }
  return tree_importance(n, toward, cos_u, neg3(toward), 0.0f, PI / 2.0f, far, near, energy);
}
V2 child_importance(const Ctx& c, const Light& node, v3 p, v3 n) {
  if (f2u(node.d[1]) == 1u) return emitter_importance(light_at(c, f2u(node.d[2])), p, n);
  return node_importance(node, p, n);
}
// tree_leaf (lights.wgsl:276-349) -> (selected, pmf)
V2 tree_leaf(const Ctx& c, uint32_t first, uint32_t count, v3 p, v3 n, float start) {
  float rand = start;
  bool sample_max = rand > 0.5f;
  if (count > 1u) rand = rand * 2.0f - (sample_max ? 1.0f : 0.0f);
  int32_t selected = -1;
  float chosen = 0.0f, chosen_other = 0.0f, total = 0.0f, total_other = 0.0f;
  uint32_t has = 0u;
  for (uint32_t i = 0u; i < count; ++i) {
    int32_t index = (int32_t)(first + i);
    V2 importance = emitter_importance(light_at(c, first + i), p, n);
    float weight = sample_max ? importance.x : importance.y;
    float other = sample_max ? importance.y : importance.x;
    if (weight > 0.0f) {
      total += weight;
      if (selected < 0) {
        selected = index;
        chosen = weight;
      } else {
        float thresh = weight / total;
        if (rand <= thresh) {
          selected = index;
          chosen = weight;
          rand = rand / thresh;
        } else {
          rand = (rand - thresh) / (1.0f - thresh);
        }
        rand = clamp_(rand, 0.0f, 1.0f);
      }
    }
    if (selected == index) chosen_other = other;
    total_other += other;
    has |= (importance.x > 0.0f ? 1u : 0u) << i;
  }
  if (has == 0u) return V2{0.0f, 0.0f};
  float chosen_max = sample_max ? chosen : chosen_other;
  float total_max = sample_max ? total : total_other;
  float chosen_min = sample_max ? chosen_other : chosen;
  float total_min = sample_max ? total_other : total;
  if (total_min == 0.0f) {
    if (sample_max) {
      chosen_min = 1.0f;
      total_min = (float)popc_(has);
    } else {
      selected = -1;
      float valid = 0.0f;
      uint32_t bits = has;
      for (uint32_t i = 0u; i < count; ++i) {
        if ((bits & 1u) != 0u) {
          valid += 1.0f;
          if (selected < 0) {
            selected = (int32_t)(first + i);
          } else {
            float thresh = 1.0f / valid;
            if (rand <= thresh) {
              selected = (int32_t)(first + i);
              rand = rand / thresh;
            } else {
              rand = (rand - thresh) / (1.0f - thresh);
            }
            rand = clamp_(rand, 0.0f, 1.0f);
          }
        }
        bits >>= 1u;
      }
      chosen_min = 1.0f;
      total_min = valid;
      chosen_max = emitter_importance(light_at(c, (uint32_t)selected), p, n).x;
    }
  }
  return V2{(float)selected, 0.5f * (chosen_max / total_max + chosen_min / total_min)};
}
// tree_pick (lights.wgsl:350-386) -> (light index, pmf); also reports the leaf row
V2 tree_pick(const Ctx& c, v3 p, v3 n, float start, uint32_t* leaf_row) {
  const Emitter& head = emitter_at(c, 0);
  uint32_t at = f2u(head.a[1] + head.a[3]);
  float rand = start;
  float pdf = 1.0f;
  for (int guard = 0; guard < 4096; ++guard) {
    const Light& node = light_at(c, at);
    uint32_t count = f2u(node.d[1]);
    if (count > 0u) {
      if (leaf_row) *leaf_row = at;
      V2 leaf = tree_leaf(c, f2u(node.d[2]), count, p, n, rand);
      return V2{leaf.x, leaf.y * pdf};
    }
    uint32_t left = at + 1u;
    uint32_t right = f2u(node.d[2]);
    V2 l = child_importance(c, light_at(c, left), p, n);
    V2 r = child_importance(c, light_at(c, right), p, n);
    float total_max = l.x + r.x;
    if (total_max == 0.0f) return V2{0.0f, 0.0f};
    float total_min = l.y + r.y;
    float probability_min = 0.5f * ((l.x > 0.0f ? 1.0f : 0.0f) + (r.x == 0.0f ? 1.0f : 0.0f));
    if (total_min > 0.0f) probability_min = l.y / total_min;
    float left_probability = 0.5f * (l.x / total_max + probability_min);
    float right_weight = 1.0f - left_probability;
    at = left;
    if (right_weight > 0.0f) {
      float thresh = right_weight / (left_probability + right_weight);
      if (rand <= thresh) {
        at = right;
        rand = rand / thresh;
      } else {
        rand = (rand - thresh) / (1.0f - thresh);
      }
      rand = clamp_(rand, 0.0f, 1.0f);
    }
    pdf = pdf * (at == left ? left_probability : 1.0f - left_probability);
  }
  return V2{0.0f, 0.0f};
}
Candidate tree_light(Ctx& c, const m3& transform, v3 p, v3 origin, v3 geometric, uint32_t* state, V4 u) {
  V2 picked = tree_pick(c, p, transform.c2, rnd(c, state, u.z), nullptr);
  if (!(picked.y > 0.0f)) return candidate_none();
  Candidate cand = light_candidate(c, light_at(c, f2u(picked.x)), transform, p, origin, geometric, state, u);
  cand.scale = divs3(cand.scale, picked.y);
  return cand;
}
uint32_t light_slots(const Ctx& c) {
  const Emitter& h = emitter_at(c, 0);
  return 1u + f2u(h.a[1]) + (h.a[3] > 0.5f ? 1u : 0u);
}
Candidate direct_light(Ctx& c, uint32_t slot, const m3& transform, v3 p, v3 origin, v3 geometric, uint32_t* state,
                       V4 u) {
  const Emitter& h = emitter_at(c, 0);
  uint32_t looped = f2u(h.a[1]);
  if (slot > looped) return tree_light(c, transform, p, origin, geometric, state, u);
  if (slot > 0u) return light_candidate(c, light_at(c, slot - 1u), transform, p, origin, geometric, state, u);
  if (h.a[0] < 0.5f) return candidate_none();
  return emitter_candidate(c, transform, p, origin, state, u);
}

// ------------------------------------------------------------- scene hit
// Closest-hit and any-hit queries traced (for the CPU baseline's rays/s).
std::atomic<uint64_t> g_closest{0}, g_any{0};

// scene() result with tri_fill (trace.wgsl:754-779) and world_hit (:682-694)
HitInfo scene_hit(const Ctx& c, v3 o, v3 d, float limit) {
  g_closest.fetch_add(1, std::memory_order_relaxed);
  Walk w = orc_walk(c.geo, o, d, limit, false);
  HitInfo h;
  h.t = w.t;
  h.n = splat3(0.0f);
  h.geometric = splat3(0.0f);
  h.material = 0u;
  h.surface = 0u;
  h.shape = 0u;
  h.record = 0u;
  if (!w.hit) return h;
  const Tri& tri = c.geo.tris[w.surface];
  float u = w.u, v = w.v;
  v3 a = xyz(tri.a);
  v3 e1 = sub3(xyz(tri.b), a);
  v3 e2 = sub3(xyz(tri.c), a);
  h.surface = w.surface;
  h.record = w.record;
  v3 geometric = normalize3(cross3(e1, e2));
  h.geometric = geometric;
  v3 shaded = add3(add3(scl3(xyz(tri.na), 1.0f - u - v), scl3(xyz(tri.nb), u)), scl3(xyz(tri.nc), v));
  v3 fallback = w.record > 0u ? splat3(0.0f) : geometric;
  h.n = dot3(shaded, shaded) > 1e-12f ? normalize3(shaded) : fallback;
  const Surface& s = surface_at(c, w.record);
  h.material = s.info[1] == NO_MATERIAL ? f2u(tri.a[3]) : s.info[1];
  if (h.record == 0u) return h;
  // world_hit
  float mirror = bits2f(s.info[3]) < 0.0f ? -1.0f : 1.0f;
  v3 i0 = xyz(s.inverse[0]), i1 = xyz(s.inverse[1]), i2 = xyz(s.inverse[2]);
  v3 g = add3(add3(scl3(i0, h.geometric.x), scl3(i1, h.geometric.y)), scl3(i2, h.geometric.z));
  v3 wg = scl3(normalize3(g), mirror);
  v3 sh = add3(add3(scl3(i0, h.n.x), scl3(i1, h.n.y)), scl3(i2, h.n.z));
  bool zero = h.n.x == 0.0f && h.n.y == 0.0f && h.n.z == 0.0f;
  h.n = zero ? wg : normalize3(sh);
  h.geometric = wg;
  return h;
}
bool occluded(const Ctx& c, v3 o, v3 d, float limit) {
  g_any.fetch_add(1, std::memory_order_relaxed);
  return orc_walk(c.geo, o, d, limit, true).hit;
}

v3 indirect_capped(const Ctx& c, v3 value, bool deep) {
  float cap = c.sc->clamp_indirect;
  if (!(cap > 0.0f) || !deep) return value;
  float luma = dot3(value, mk3(0.2126f, 0.7152f, 0.0722f));
  if (!(luma > cap)) return value;
  return scl3(value, cap / luma);
}

// radiance (trace.wgsl:2153-2502) for the features in scope
v3 radiance(Ctx& c, v3 o0, v3 d0, uint32_t* state, float first_albedo[4], float first_normal[4]) {
  const OrcScene& sc = *c.sc;
  const OrcFrame& fr = *c.fr;
  const uint32_t TOTAL = sc.bounces[0], DIFFUSE = sc.bounces[1], GLOSSY = sc.bounces[2], TRANSMISSION = sc.bounces[3];
  v3 o = o0, d = d0;
  v3 throughput = splat3(1.0f);
  v3 result = splat3(0.0f);
  float previous_pdf = 0.0f;
  uint32_t carried = 3u;
  uint32_t lobes[3] = {0u, 0u, 0u};
  bool last = false, lit_vertex = false, through = false, diffused = false, medium = false;
  for (uint32_t bounce = 0u; bounce <= TOTAL + 1u; ++bounce) {
    if (sc.sobol_on) c.rng[2] = 16u * (bounce + 1u);
    HitInfo hit = scene_hit(c, o, d, 1e20f);
    float reach = hit.t;
    v3 origin_point = medium ? o : spawn_point(o, neg3(d), o, 0.0f);
    result = add3(result, indirect_capped(c, mul3(throughput, light_hits(c, o, d, reach, origin_point, previous_pdf)),
                                          bounce > 1u));
    if (hit.t >= 1e19f) {
      if (bounce == 0u && fr.forward[3] > 0.0f) break;
      float pdf = sky_pdf(c, d);
      float weight = (bounce > 0u && previous_pdf > 0.0f) ? previous_pdf / (previous_pdf + pdf) : 1.0f;
      v3 environment = sky_radiance(c);  // sky_seen with the plain look = the radiance
      result = add3(result, indirect_capped(c, scl3(mul3(throughput, environment), weight), bounce > 1u));
      break;
    }
    v3 p = add3(o, scl3(d, hit.t));
    v3 n = dot3(hit.n, d) > 0.0f ? neg3(hit.n) : hit.n;
    Shaded s = surface(c, hit.material);
    v3 geometric = dot3(hit.geometric, d) > 0.0f ? neg3(hit.geometric) : hit.geometric;
    if (dot3(n, geometric) < 0.05f) n = normalize3(add3(n, scl3(geometric, 0.1f)));
    s.roughness = fmax_(s.roughness, 0.05f);
    s.clearcoat_roughness = fmax_(s.clearcoat_roughness, 0.05f);
    if (sc.filter_glossy > 0.0f && diffused) {
      s.roughness = fmax_(s.roughness, sc.filter_glossy);
      s.clearcoat_roughness = fmax_(s.clearcoat_roughness, sc.filter_glossy);
    }
    if (bounce == 0u) {
      first_albedo[0] = s.base.x;
      first_albedo[1] = s.base.y;
      first_albedo[2] = s.base.z;
      first_albedo[3] = 1.0f;
      first_normal[0] = n.x;
      first_normal[1] = n.y;
      first_normal[2] = n.z;
      first_normal[3] = 1.0f;
    }
    s.emission = scl3(s.emission, emitter_weight(c, hit, p, origin_point, previous_pdf));
    result = add3(result, indirect_capped(c, mul3(throughput, s.emission), bounce > 1u));
    if (last) break;
    m3 transform = basis(n);
    v3 wo = mulmtv(transform, neg3(d));
    v3 origin = spawn_point(p, n, o, hit.t);
    bool entering = dot3(hit.n, d) < 0.0f;
    uint32_t slots = 2u + light_slots(c);
    for (uint32_t k = 0u; k < slots; ++k) {
      V4 u = sobol(c, light_dim(k));
      v3 local = mk3(0, 0, 1), direction = mk3(0, 0, 1), strength = splat3(0.0f);
      float limit = 1e19f;
      uint32_t shape = 0u;
      float pdf = 0.0f;
      Shaded lit = s;
      if (k == 0u) {
        if (fr.sun_color[3] <= 0.0f) continue;
        direction = normalize3(xyz(fr.sun_dir));
        if (fr.sun_dir[3] < 1.0f) {
          float height = 1.0f - rnd(c, state, u.x) * (1.0f - fr.sun_dir[3]);
          float radius = sqrtf(fmax_(0.0f, 1.0f - height * height));
          float phi = 2.0f * PI * rnd(c, state, u.y);
          m3 orient = basis(direction);
          direction = normalize3(mulmv(orient, mk3(radius * cos_(phi), radius * sin_(phi), height)));
        }
        local = mulmtv(transform, direction);
        if (local.z <= 0.0f) continue;  // scatter_reach() is 0 without lobes
        strength = scl3(xyz(fr.sun_color), fr.sun_color[3] * 1.0f);
      } else if (k == 1u) {
        if (sc.sky_width == 0u) continue;
        float ux = rnd(c, state, u.x);
        float uy = rnd(c, state, u.y);
        SkySample light = sky_sample(c, ux, uy);
        direction = light.direction;
        local = mulmtv(transform, direction);
        if (local.z <= 0.0f) continue;
        strength = scl3(sky_radiance(c), 1.0f);
        pdf = light.pdf;
        if (!(pdf > 0.0f)) continue;
      } else {
        Candidate picked = direct_light(c, k - 2u, transform, p, origin, geometric, state, u);
        if (picked.limit < 0.0f) continue;
        local = picked.wi;
        direction = picked.direction;
        strength = picked.scale;
        pdf = picked.pdf;
        limit = picked.limit;
        shape = picked.shape;
        lit.roughness = fmax_(s.roughness, picked.roughness);
      }
      if (pdf > 0.0f) {
        float bsdf = bsdf_pdf(s, wo, local);
        if (k == 1u) {
          strength = divs3(strength, pdf + bsdf);
        } else {
          float ratio = bsdf / pdf;
          strength = divs3(strength, pdf * (1.0f + ratio * ratio));
        }
      }
      (void)shape;
      if (limit > 0.0f) {
        if (occluded(c, origin, direction, limit)) continue;
      }
      v3 term = mul3(scl3(scl3(mul3(throughput, eval(lit, wo, local)), pdf > 0.0f ? glossy_share(s) : 1.0f), local.z),
                     strength);
      result = add3(result, indirect_capped(c, term, bounce > 0u));
    }
    LightSample sample = sample_bsdf(c, s, wo, entering, carried, state, sobol(c, 3u));
    v3 wi = sample.dir;
    diffused = diffused || sample.lobe == 0u;
    lobes[0] += sample.lobe == 0u ? 1u : 0u;
    lobes[1] += sample.lobe == 1u ? 1u : 0u;
    lobes[2] += sample.lobe == 2u ? 1u : 0u;
    last = bounce >= TOTAL || lobes[0] > DIFFUSE || lobes[1] > GLOSSY || lobes[2] > TRANSMISSION;
    through = sample.pdf < -1.5f && lit_vertex;
    lit_vertex = sample.pdf > 0.0f || through;
    if (sample.pdf < 0.0f) {
      throughput = mul3(throughput, sample.weight);
      carried = sample.channel;
      if (sample.pdf < -1.5f)
        throughput = mul3(throughput, mul3(mk3(sqrtf(clamp_(s.base.x, 0.0f, 1.0f)), sqrtf(clamp_(s.base.y, 0.0f, 1.0f)),
                                               sqrtf(clamp_(s.base.z, 0.0f, 1.0f))),
                                           beer(s.thickness, s.subsurface_tint, s.absorption)));
      d = normalize3(mulmv(transform, wi));
      previous_pdf = 0.0f;
    } else {
      if (wi.z <= 0.0f || sample.pdf <= 0.0f) break;
      throughput = mul3(throughput, scl3(divs3(scl3(scl3(eval(s, wo, wi), glossy_share(s)), wi.z), sample.pdf), 1.0f));
      d = normalize3(mulmv(transform, wi));
      previous_pdf = sample.pdf;
    }
    o = spawn_point(p, d, o, hit.t);
    medium = false;
    if (bounce >= 3u) {
      float keep = clamp_(fmax_(throughput.x, fmax_(throughput.y, throughput.z)), 0.05f, 0.95f);
      if (rnd(c, state, sobol(c, 0u).x) > keep) break;
      throughput = divs3(throughput, keep);
    }
  }
  (void)through;
  return result;
}

}  // namespace orc

extern "C" {

// One sampling pass of main() (trace.wgsl:2503-2579) over the whole film:
// `accum` holds 12 floats per pixel (Accum) and is read and updated; the three
// films (4 floats per pixel each) are written.  frame->size.z must hold the
// samples already accumulated and size.w the samples of this pass.
int orc_render_masked(const OrcScene* sc, const OrcFrame* fr, float* accum, float* color, float* albedo, float* normal,
                      const uint8_t* mask);
int orc_render(const OrcScene* sc, const OrcFrame* fr, float* accum, float* color, float* albedo, float* normal) {
  return orc_render_masked(sc, fr, accum, color, albedo, normal, nullptr);
}

// The same pass over the pixels whose `mask` byte is non-zero (all of them when
// `mask` is null); the others are neither reset nor sampled.  A pixel's samples
// depend only on the pixel, so a masked pass gives the masked pixels exactly
// the values a full pass gives them.
int orc_render_masked(const OrcScene* sc, const OrcFrame* fr, float* accum, float* color, float* albedo, float* normal,
                      const uint8_t* mask) {
  uint32_t W = fr->size[0], H = fr->size[1];
  orc::Ctx base;
  base.sc = sc;
  base.fr = fr;
  base.geo = Scene{(const Node*)sc->nodes, sc->node_count, (const Tri*)sc->tris, sc->tri_count,
                   (const Surface*)sc->surfaces};
  parallel_for((int64_t)W * H, 64, [&](int64_t index, unsigned) {
    orc::Ctx c = base;
    uint32_t gx = (uint32_t)(index % W), gy = (uint32_t)(index / W);
    uint32_t px = gx + fr->window[2], py = gy + fr->window[3];
    uint32_t stream = py * fr->window[0] + px;
    float* sum = accum + 12 * (size_t)index;
    if (mask && !mask[index]) return;
    if (fr->size[2] == 0u)
      for (int k = 0; k < 12; ++k) sum[k] = 0.0f;
    if (sum[3] < 0.0f) return;
    for (uint32_t sample = 0u; sample < fr->size[3]; ++sample) {
      float fa[4] = {0, 0, 0, 0}, fn[4] = {0, 0, 0, 0};
      uint32_t state = orc::pcg(stream * 1973u + orc::pcg(fr->counts[2] * 9277u + (fr->size[2] + sample) * 7919u + 26699u));
      if (sc->sobol_on) {
        c.rng[0] = orc::hash_iqnt2d(px, py) ^ fr->counts[2];
        c.rng[1] = fr->size[2] + sample;
        c.rng[2] = 0u;
      }
      orc::V4 pf = orc::sobol(c, 0u);
      float jx = orc::rnd(c, &state, pf.x);
      float jy = orc::rnd(c, &state, pf.y);
      float ndc_x = ((float)px + jx) / (float)fr->window[0] * 2.0f - 1.0f;
      float ndc_y = ((float)py + jy) / (float)fr->window[1] * 2.0f - 1.0f;
      uint32_t kind = f2u(rint_(fr->origin[3]));
      v3 cam_origin = orc::xyz(fr->origin), cam_forward = orc::xyz(fr->forward), cam_right = orc::xyz(fr->right),
         cam_up = orc::xyz(fr->up);
      v3 direction = normalize3(add3(add3(cam_forward, scl3(cam_right, ndc_x + fr->lens[0])),
                                     scl3(cam_up, -ndc_y + fr->lens[1])));
      v3 origin = cam_origin;
      if (kind == 1u) {
        direction = normalize3(cam_forward);
        origin = add3(origin, add3(scl3(normalize3(cam_right), (ndc_x + fr->lens[0]) * fr->right[3]),
                                   scl3(normalize3(cam_up), (-ndc_y + fr->lens[1]) * fr->up[3])));
      } else if (kind == 2u) {
        float phi = (ndc_x * 0.5f) * 2.0f * orc::PI;
        float theta = (ndc_y * 0.5f + 0.5f) * orc::PI;
        v3 local = mk3(sin_(theta) * sin_(phi), cos_(theta), -sin_(theta) * cos_(phi));
        direction = normalize3(sub3(add3(scl3(normalize3(cam_right), local.x), scl3(normalize3(cam_up), local.y)),
                                    scl3(normalize3(cam_forward), local.z)));
      } else if (fr->lens[2] > 0.0f) {
        v3 focus = add3(origin, scl3(direction, fr->lens[3] / dot3(direction, normalize3(cam_forward))));
        orc::V4 aperture = orc::sobol(c, 1u);
        float radius = sqrtf(orc::rnd(c, &state, aperture.x)) * fr->lens[2];
        float phi = 2.0f * orc::PI * orc::rnd(c, &state, aperture.y);
        origin = add3(origin, add3(scl3(normalize3(cam_right), radius * cos_(phi)),
                                   scl3(normalize3(cam_up), radius * sin_(phi))));
        direction = normalize3(sub3(focus, origin));
      }
      v3 value = orc::radiance(c, origin, direction, &state, fa, fn);
      sum[0] = sum[0] + value.x;
      sum[1] = sum[1] + value.y;
      sum[2] = sum[2] + value.z;
      for (int k = 0; k < 4; ++k) {
        sum[4 + k] = sum[4 + k] + fa[k];
        sum[8 + k] = sum[8 + k] + fn[k];
      }
    }
    sum[3] = (float)(fr->size[2] + fr->size[3]);
    float count = fmax_(sum[3], 1.0f);
    v3 nn = divs3(mk3(sum[8], sum[9], sum[10]), count);
    float* co = color + 4 * (size_t)index;
    co[0] = sum[0] / count;
    co[1] = sum[1] / count;
    co[2] = sum[2] / count;
    co[3] = fr->forward[3] > 0.0f ? sum[7] / count : 1.0f;
    float* al = albedo + 4 * (size_t)index;
    for (int k = 0; k < 4; ++k) al[k] = sum[4 + k] / count;
    float* no = normal + 4 * (size_t)index;
    v3 nv = length3(nn) > 1e-6f ? normalize3(nn) : splat3(0.0f);
    no[0] = nv.x;
    no[1] = nv.y;
    no[2] = nv.z;
    no[3] = sum[11] / count;
  });
  return 0;
}

// Adaptive convergence (converge.wgsl:9-51): measure then, when `mark_on`,
// mark; returns the running count (pixels still sampling).
uint32_t orc_converge(float* accum, float* snaps, uint32_t W, uint32_t H, uint32_t min_samples, float threshold,
                      int mark_on) {
  // mark_on: 0 measure only, 1 measure then mark, 2 mark only (the snapshots'
  // errors were measured, and neighbours' errors filled in, by the caller)
  size_t n = (size_t)W * H;
  for (size_t index = 0; index < (mark_on == 2 ? 0 : n); ++index) {
    float* sum = accum + 12 * index;
    float* snap = snaps + 8 * index;
    float count = sum[3];
    if (count <= 0.0f) {
      snap[5] = 0.0f;
      continue;
    }
    float now[4] = {sum[0] / count, sum[1] / count, sum[2] / count, sum[7] / count};
    float prior = snap[4];
    float error = 1e9f;
    if (prior > 0.0f && count > prior) {
      float scale = sqrtf(1.0f / count) / sqrtf(1.0f / prior + 1.0f / (count - prior));
      float gap[4];
      for (int k = 0; k < 4; ++k) {
        float rest = (now[k] * count - snap[k] * prior) / (count - prior);
        gap[k] = abs_(snap[k] - rest) * scale;
      }
      error = (gap[0] + gap[1] + gap[2]) / (1e-4f + sqrtf(fmax_(now[0] + now[1] + now[2], 0.0f))) + gap[3];
    }
    for (int k = 0; k < 4; ++k) snap[k] = now[k];
    snap[4] = count;
    snap[5] = error;
    snap[6] = 0.0f;
    snap[7] = 0.0f;
  }
  if (!mark_on) return (uint32_t)n;
  uint32_t running = 0;
  for (size_t index = 0; index < n; ++index) {
    uint32_t gx = (uint32_t)(index % W), gy = (uint32_t)(index / W);
    float count = accum[12 * index + 3];
    if (count <= 0.0f) continue;
    float worst = 0.0f;
    for (int dy = -1; dy <= 1; ++dy)
      for (int dx = -1; dx <= 1; ++dx) {
        int x = std::min(std::max((int)gx + dx, 0), (int)W - 1);
        int y = std::min(std::max((int)gy + dy, 0), (int)H - 1);
        worst = fmax_(worst, snaps[8 * ((size_t)y * W + x) + 5]);
      }
    if (count >= (float)min_samples && worst < threshold)
      accum[12 * index + 3] = -count;
    else
      running += 1;
  }
  return running;
}

// Closest-hit and any-hit queries traced by orc_render since the last call.
void orc_ray_counts(uint64_t* out) {
  out[0] = orc::g_closest.exchange(0);
  out[1] = orc::g_any.exchange(0);
}

// One light-tree pick (tree_pick, lights.wgsl:350-386) per query point:
// returns the picked light row, the pmf and the leaf row reached.
void orc_tree_pick(const OrcScene* sc, const float* points, const float* normals, const float* rands, uint32_t n,
                   int32_t* light, float* pmf, uint32_t* leaf) {
  orc::Ctx c;
  c.sc = sc;
  c.fr = nullptr;
  for (uint32_t i = 0; i < n; ++i) {
    uint32_t row = 0;
    orc::V2 r = orc::tree_pick(c, mk3(points[3 * i], points[3 * i + 1], points[3 * i + 2]),
                               mk3(normals[3 * i], normals[3 * i + 1], normals[3 * i + 2]), rands[i], &row);
    light[i] = r.y > 0.0f ? (int32_t)f2u(r.x) : -1;
    pmf[i] = r.y;
    leaf[i] = row;
  }
}

}  // extern "C"
