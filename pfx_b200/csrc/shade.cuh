// Device-side shading of the wavefront tracer: the samplers, BSDF, light
// sampling and sky sampling of the reference tracer, in the reference's
// operation order (WGSL evaluates a*b*c as (a*b)*c), for the feature set this
// library covers.
//
//   pcg / random / hash_iqnt2d / rnd / light_dim   trace.wgsl:168-172, 423-448
//   sobol                                          sobol.wgsl:1-58
//   eval (without film) / reflection               materials/src/wgsl/brdf.wgsl:32-283
//   sample_bsdf / bsdf_pdf / glossy_share          trace.wgsl:1705-1788
//   light_hits / light_candidate / emitter_*       lights.wgsl:1-200
//   tree_importance / tree_leaf / tree_pick        lights.wgsl:201-393
//   direct_light / light_slots                     lights.wgsl:394-409
//   sky_pdf / sky_sample                           sky.rs (SKY_SAMPLING_WGSL)
//   offset_axis / offset_ray / spawn_point         trace.wgsl:1257-1269
#pragma once
#include "pfxt_math.h"
#include "pfxt_types.h"
#include "tracer.h"

namespace pfxt {

constexpr float SH_PI = 0x1.921fb6p+1f;

// Heavy helpers are kept out of line (one copy each in the shading kernel).
#ifndef SH_CALL
#define SH_CALL static __device__ __noinline__
#endif
// Small helpers: out of line as well unless a build inlines them.
#ifndef SH_SMALL
#define SH_SMALL SH_CALL
#endif  // brdf.wgsl:1 `const PI: f32 = 3.141592653589793`
// The light-tree descent, its leaf and the light candidate: out of line unless
// a build inlines them.
#ifndef SH_TREE
#define SH_TREE SH_CALL
#endif

// ------------------------------------------------------------------ random
__device__ __forceinline__ uint32_t pcg(uint32_t v) {
  uint32_t s = v * 747796405u + 2891336453u;
  uint32_t w = ((s >> ((s >> 28u) + 4u)) ^ s) * 277803737u;
  return (w >> 22u) ^ w;
}
__device__ __forceinline__ float random01(uint32_t& state) {
  state = pcg(state);
  return (float)(state >> 8u) / 16777216.0f;
}
__device__ __forceinline__ uint32_t hash_iqnt2d(uint32_t x, uint32_t y) {
  uint32_t qx = 1103515245u * ((x >> 1u) ^ y);
  uint32_t qy = 1103515245u * ((y >> 1u) ^ x);
  return 1103515245u * (qx ^ (qy >> 3u));
}
__device__ __forceinline__ uint32_t light_dim(uint32_t k) {
  if (k == 0u) return 1u;
  if (k < 13u) return 3u + k;
  return k << 16u;
}

// Sobol lookup state (var<private> rng of trace.wgsl:427): x = pixel hash ^
// seed, y = sample index, z = dimension base.
struct Rng {
  uint32_t x, y, z;
};

__device__ __forceinline__ uint32_t reversed_bit_owen(uint32_t n, uint32_t seed) {
  n ^= n * 0x3d20adeau;
  n += seed;
  n *= (seed >> 16u) | 1u;
  n ^= n * 0x05526c56u;
  n ^= n * 0x53a22864u;
  return n;
}
__device__ __forceinline__ uint32_t hash_wang_seeded(uint32_t i0, uint32_t seed) {
  uint32_t i = (i0 ^ 61u) ^ seed;
  i += i << 3u;
  i ^= i >> 4u;
  i *= 0x27d4eb2du;
  return i;
}
__device__ __forceinline__ uint32_t hash_shuffle_256(uint32_t i0, uint32_t seed) {
  const uint32_t length = 256u, mask = 255u;
  uint32_t i = i0 % length;
  for (int guard = 0; guard < 1024; ++guard) {  // the permutation is bijective: ends within a few rounds
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
SH_SMALL float4 sobol4(const ShadeView& v, const Specialise& sp, const Rng& r, uint32_t dimension) {
  if (!sp.sobol) return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  uint32_t L = sp.sobol_length;
  uint32_t seed = r.x;
  uint32_t dim = r.z + dimension;
  uint32_t pattern = hash_shuffle_256(dim, seed);
  uint32_t mask = L - 1u;
  uint32_t shuffled = brev_(reversed_bit_owen(brev_(r.y), hash_wang_seeded(dim, seed)));
  uint32_t sample = (r.y & ~mask) | (shuffled & mask);
  uint32_t index = (pattern * L + sample) % (L * 256u);
  float4 t = __ldg(v.sobol + index);
  float s0 = (float)hash_wang_seeded(dim, seed) * 2.3283064e-10f;
  float s1 = (float)hash_wang_seeded(dim, seed ^ 0xca0e1151u) * 2.3283064e-10f;
  float s2 = (float)hash_wang_seeded(dim, seed ^ 0xbf604c5au) * 2.3283064e-10f;
  float s3 = (float)hash_wang_seeded(dim, seed ^ 0x99634d1du) * 2.3283064e-10f;
  return make_float4(fmin_(fract_(t.x + s0), 0.99999994f), fmin_(fract_(t.y + s1), 0.99999994f),
                     fmin_(fract_(t.z + s2), 0.99999994f), fmin_(fract_(t.w + s3), 0.99999994f));
}
__device__ __forceinline__ float rnd(const Specialise& sp, uint32_t& state, float value) {
  if (sp.sobol) return value;
  return random01(state);
}

// ------------------------------------------------------------------ material
struct Shaded {
  v3 base;
  float roughness, metalness, specular, clearcoat, clearcoat_roughness, sheen, transmission, ior, dispersion,
      thickness, subsurface;
  v3 subsurface_tint;
  float absorption;
  v3 emission;
  float fresnel_power;
};

__device__ __forceinline__ Shaded load_surface(const ShadeView& v, uint32_t material) {
  const float4* r = v.materials + (size_t)(material + 1u) * 8u;
  float4 r0 = __ldg(r + 0), r1 = __ldg(r + 1), r2 = __ldg(r + 2), r3 = __ldg(r + 3), r4 = __ldg(r + 4),
         r5 = __ldg(r + 5), r6 = __ldg(r + 6);
  Shaded s;
  s.base = mk3(r0.x, r0.y, r0.z);
  s.roughness = r0.w;
  s.metalness = r1.x;
  s.specular = r1.y;
  s.clearcoat = r1.z;
  s.clearcoat_roughness = r1.w;
  s.sheen = r2.x;
  s.transmission = r2.y;
  s.ior = r2.z;
  s.dispersion = r2.w;
  s.thickness = r3.x;
  s.subsurface = r3.y;
  s.subsurface_tint = mk3(r4.x, r4.y, r4.z);
  s.absorption = r4.w;
  s.emission = mk3(r5.x, r5.y, r5.z);
  s.fresnel_power = r6.x;
  return s;
}

// ------------------------------------------------------------------ brdf.wgsl
__device__ __forceinline__ v3 dispersed_ior(float ior, float dispersion) {
  return mk3(ior + -0.016f * dispersion, ior, ior + 0.022f * dispersion);
}
__device__ __forceinline__ v3 schlick(v3 f0, float cos_theta, float power) {
  float k = pow_(1.0f - clamp_(cos_theta, 0.0f, 1.0f), power);
  return mix3(f0, splat3(1.0f), k);
}
__device__ __forceinline__ float fresnel_dielectric(float cos_theta, float eta_in) {
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
__device__ __forceinline__ float ggx_d(float nh, float a2) {
  float n = fmax_(nh, 0.0f);
  float k = n * n * (a2 - 1.0f) + 1.0f;
  return a2 / (SH_PI * k * k);
}
__device__ __forceinline__ float smith_g1(float ndot, float a2) {
  float n = fmax_(ndot, 0.0f);
  return 2.0f * n / (n + sqrtf(a2 + (1.0f - a2) * n * n));
}
__device__ __forceinline__ float alpha_rough(float roughness) {
  float r = clamp_(roughness, 0.02f, 1.0f);
  return r * r;
}
__device__ __forceinline__ v3 beer(float distance, v3 tint, float absorption) {
  if (distance <= 0.0f || absorption <= 0.0f) return splat3(1.0f);
  return mk3(exp_(-distance * absorption * fmax_(1.0f - tint.x, 0.0f)),
             exp_(-distance * absorption * fmax_(1.0f - tint.y, 0.0f)),
             exp_(-distance * absorption * fmax_(1.0f - tint.z, 0.0f)));
}
__device__ __forceinline__ float fresnel_exponent(const Shaded& s) {
  return s.fresnel_power <= 0.0f ? 5.0f : s.fresnel_power;
}
SH_SMALL v3 reflection(const Shaded& s, float ndh_cos) {
  float power = fresnel_exponent(s);
  v3 f0 = mix3(splat3(s.specular), s.base, clamp_(s.metalness, 0.0f, 1.0f));
  if (s.transmission > 0.0f || s.dispersion != 0.0f) {
    v3 iors = dispersed_ior(s.ior, s.dispersion);
    v3 metal = schlick(s.base, ndh_cos, power);
    v3 diel = mk3(fresnel_dielectric(ndh_cos, iors.x), fresnel_dielectric(ndh_cos, iors.y),
                  fresnel_dielectric(ndh_cos, iors.z));
    return mix3(diel, metal, clamp_(s.metalness, 0.0f, 1.0f));
  }
  if (f0.x <= 0.0f && f0.y <= 0.0f && f0.z <= 0.0f) return splat3(0.0f);
  return schlick(f0, ndh_cos, power);
}
__device__ __forceinline__ v3 ggx_spec(float ndv, float ndl, float ndh, float a2, v3 fresnel) {
  float g = smith_g1(ndv, a2) * smith_g1(ndl, a2);
  return divs3(scl3(scl3(fresnel, ggx_d(ndh, a2)), g), 4.0f * ndv * ndl);
}
// `roughness` stands for s.roughness: a light slot evaluates the lobe widened
// to the light's own roughness without copying the whole Shaded record.
SH_CALL v3 bsdf_eval(const Shaded& s, v3 wo, v3 wi, float roughness) {
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
    return divs3(scl3(mul3(mul3(s.base, tint), transmitted), back), SH_PI);
  }
  v3 h = normalize3(add3(wo, wi));
  float ndh = fmax_(h.z, 0.0f);
  float vdh = fmax_(dot3(wo, h), 0.0f);
  v3 fresnel = reflection(s, vdh);
  float a = alpha_rough(roughness);
  v3 spec = ggx_spec(ndv, ndl, ndh, a * a, fresnel);
  v3 transmitted = sub3(splat3(1.0f), fresnel);
  float body = (1.0f - metal) * (1.0f - trans) * (1.0f - sss);
  float diffuse_w = body * (1.0f - sheen_cover);
  float sheen_w = body * sheen_cover * pow_(1.0f - ndh, 5.0f);
  v3 colour = add3(spec, divs3(scl3(mul3(s.base, transmitted), diffuse_w + sheen_w), SH_PI));
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
__device__ __forceinline__ float glossy_share(const Shaded& s) {
  return 1.0f - clamp_(s.transmission, 0.0f, 1.0f) * (1.0f - clamp_(s.metalness, 0.0f, 1.0f));
}
__device__ __forceinline__ float coat_weight_of(const Shaded& s, v3 wo) {
  return clamp_(s.clearcoat * (0.12f + 0.88f * (0.04f + 0.96f * pow_(1.0f - fmax_(wo.z, 0.0f), 5.0f))), 0.0f, 0.9f);
}
SH_SMALL float bsdf_pdf(const Shaded& s, v3 wo, v3 wi) {
  if (wi.z <= 0.0f) return 0.0f;
  float trans = clamp_(s.transmission, 0.0f, 1.0f) * (1.0f - clamp_(s.metalness, 0.0f, 1.0f));
  float coat = coat_weight_of(s, wo);
  float spec = (1.0f - coat) * clamp_(s.metalness + s.specular, 0.0f, 0.9f);
  v3 h = normalize3(add3(wo, wi));
  float a = alpha_rough(s.roughness);
  float ca = alpha_rough(s.clearcoat_roughness);
  float denom = fmax_(4.0f * abs_(dot3(wi, h)), 1e-8f);
  float hz = fmax_(h.z, 0.0f);
  float base_pdf = ggx_d(hz, a * a) * hz / denom;
  float coat_pdf = ggx_d(hz, ca * ca) * hz / denom;
  return (1.0f - trans) * (coat * coat_pdf + spec * base_pdf + (1.0f - coat - spec) * wi.z / SH_PI);
}
__device__ __forceinline__ v3 channel_mask(uint32_t ch) {
  return mk3(ch == 0u ? 1.0f : 0.0f, ch == 1u ? 1.0f : 0.0f, ch == 2u ? 1.0f : 0.0f);
}

struct BsdfSample {
  v3 dir;
  float pdf;
  uint32_t channel;
  v3 weight;
  uint32_t lobe;
};

SH_CALL BsdfSample sample_bsdf(const Specialise& sp, const Shaded& s, v3 wo, bool entering,
                                                  uint32_t carried, uint32_t& state, float4 u) {
  BsdfSample out;
  float transmission = clamp_(s.transmission, 0.0f, 1.0f) * (1.0f - clamp_(s.metalness, 0.0f, 1.0f));
  if (rnd(sp, state, u.w) < transmission) {
    v3 iors = dispersed_ior(s.ior, s.dispersion);
    uint32_t channel = carried;
    v3 weight = splat3(1.0f);
    if (channel > 2u && fmax_(abs_(iors.x - iors.y), abs_(iors.z - iors.y)) > 1e-4f) {
      uint32_t ch = f2u(rnd(sp, state, u.z) * 3.0f);
      channel = ch < 2u ? ch : 2u;
      weight = scl3(channel_mask(channel), 3.0f);
    }
    float ior = channel > 2u ? fmax_(s.ior, 1.01f) : fmax_(get3(iors, (int)channel), 1.01f);
    float ratio = entering ? ior : 1.0f / ior;
    v3 live = channel > 2u ? splat3(1.0f) : channel_mask(channel);
    v3 fresnel = mul3(splat3(fresnel_dielectric(fmax_(wo.z, 0.0f), ratio)), live);
    float chance = dot3(fresnel, splat3(1.0f)) / dot3(live, splat3(1.0f));
    v3 incident = neg3(wo);
    v3 mirrored = reflect3(incident, mk3(0.0f, 0.0f, 1.0f));
    out.channel = channel;
    out.lobe = 1u;
    out.pdf = -1.0f;
    if (rnd(sp, state, u.x) < chance) {
      out.dir = mirrored;
      out.weight = divs3(mul3(weight, fresnel), chance);
      return out;
    }
    float eta = 1.0f / ratio;
    float cos_i = incident.z;  // dot((0,0,1), incident)
    float k = 1.0f - eta * eta * (1.0f - cos_i * cos_i);
    if (!(k < 0.0f)) {
      float t = eta * cos_i + sqrtf(k);
      v3 refracted = sub3(scl3(incident, eta), scl3(mk3(0.0f, 0.0f, 1.0f), t));
      out.dir = normalize3(refracted);
      out.pdf = -2.0f;
      out.weight = divs3(mul3(weight, sub3(live, fresnel)), 1.0f - chance);
      out.lobe = 2u;
      return out;
    }
    out.dir = mirrored;
    out.weight = mul3(weight, live);
    return out;
  }
  float coat_weight = coat_weight_of(s, wo);
  float spec_weight = (1.0f - coat_weight) * clamp_(s.metalness + s.specular, 0.0f, 0.9f);
  float pick = rnd(sp, state, u.z);
  out.channel = 3u;
  out.weight = splat3(1.0f);
  if (pick < coat_weight + spec_weight) {
    bool coat = pick < coat_weight;
    float alpha = alpha_rough(coat ? s.clearcoat_roughness : s.roughness);
    float u1 = rnd(sp, state, u.x);
    float u2 = rnd(sp, state, u.y);
    float phi = 2.0f * SH_PI * u1;
    float cos_theta = sqrtf((1.0f - u2) / (1.0f + (alpha * alpha - 1.0f) * u2));
    float st = sqrtf(fmax_(0.0f, 1.0f - cos_theta * cos_theta));
    v3 h = mk3(cos_(phi) * st, sin_(phi) * st, cos_theta);
    out.dir = reflect3(neg3(wo), h);
    out.pdf = bsdf_pdf(s, wo, out.dir);
    out.lobe = 1u;
    return out;
  }
  float u1 = rnd(sp, state, u.x);
  float u2 = rnd(sp, state, u.y);
  float phi = 2.0f * SH_PI * u1;
  float r = sqrtf(u2);
  out.dir = mk3(cos_(phi) * r, sin_(phi) * r, sqrtf(1.0f - u2));
  out.pdf = bsdf_pdf(s, wo, out.dir);
  out.lobe = 0u;
  return out;
}

// ------------------------------------------------------------------ sky
__device__ __forceinline__ uint32_t cdf_find(const float* __restrict__ cdf, uint32_t count, float needle) {
  uint32_t low = 0u, high = count;
  while (low < high) {
    uint32_t mid = (low + high) / 2u;
    if (__ldg(cdf + mid) <= needle)
      low = mid + 1u;
    else
      high = mid;
  }
  return low < count - 1u ? low : count - 1u;
}
__device__ __forceinline__ v3 sky_radiance(const ShadeView& v) {
  return mk3(v.sky_radiance[0], v.sky_radiance[1], v.sky_radiance[2]);
}
SH_SMALL float sky_pdf(const ShadeView& v, v3 direction) {
  v3 d = normalize3(direction);
  float theta = acos_(clamp_(d.y, -1.0f, 1.0f));
  float phi = fmod_wgsl(atan2_(d.z, d.x) + 6.28318531f, 6.28318531f);
  uint32_t row = f2u(theta / 3.14159265f * (float)v.sky_height);
  row = row < v.sky_height - 1u ? row : v.sky_height - 1u;
  uint32_t col = f2u(phi / 6.28318531f * (float)v.sky_width);
  col = col < v.sky_width - 1u ? col : v.sky_width - 1u;
  float row_before = row > 0u ? __ldg(v.sky_rows + (row > 1u ? row : 1u) - 1u) : 0.0f;
  const float* cols = v.sky_columns + (size_t)row * v.sky_width;
  float col_before = col > 0u ? __ldg(cols + (col > 1u ? col : 1u) - 1u) : 0.0f;
  float mass = (__ldg(v.sky_rows + row) - row_before) * (__ldg(cols + col) - col_before);
  float area = 6.28318531f / (float)v.sky_width * 3.14159265f / (float)v.sky_height * fmax_(sin_(theta), 0.00001f);
  return (1.0f - v.sky_sun_probability) * mass / area + 0.0f;
}
struct SkySample {
  v3 direction;
  float pdf;
};
SH_CALL SkySample sky_sample(const ShadeView& v, float rx, float ry) {
  float u = clamp_(rx, 0.0f, 0.99999994f);
  float w = clamp_(ry, 0.0f, 0.99999994f);
  uint32_t row = cdf_find(v.sky_rows, v.sky_height, w);
  float row_before = row > 0u ? __ldg(v.sky_rows + (row > 1u ? row : 1u) - 1u) : 0.0f;
  float fy = (w - row_before) / fmax_(__ldg(v.sky_rows + row) - row_before, 0.000001f);
  float needle = fmax_(u - v.sky_sun_probability, 0.0f) / fmax_(1.0f - v.sky_sun_probability, 0.000001f);
  const float* cols = v.sky_columns + (size_t)row * v.sky_width;
  uint32_t col = cdf_find(cols, v.sky_width, needle);
  float col_before = col > 0u ? __ldg(cols + (col > 1u ? col : 1u) - 1u) : 0.0f;
  float fx = (needle - col_before) / fmax_(__ldg(cols + col) - col_before, 0.000001f);
  float theta = 3.14159265f * ((float)row + fy) / (float)v.sky_height;
  float phi = 6.28318531f * ((float)col + fx) / (float)v.sky_width;
  SkySample s;
  s.direction = mk3(sin_(theta) * cos_(phi), cos_(theta), sin_(theta) * sin_(phi));
  float area = 6.28318531f / (float)v.sky_width * 3.14159265f / (float)v.sky_height * fmax_(sin_(theta), 0.00001f);
  float mass = (__ldg(v.sky_rows + row) - row_before) * (__ldg(cols + col) - col_before);
  s.pdf = (1.0f - v.sky_sun_probability) * mass / area + 0.0f;
  return s;
}

// ------------------------------------------------------------------ offsets
__device__ __forceinline__ float offset_axis(float position, float normal) {
  if (abs_(position) < 1.0f / 32.0f) return position + normal / 65536.0f;
  int32_t bits = (int32_t)f2bits(position);
  int32_t shift = f2i(normal * 256.0f);
  return bits2f((uint32_t)(bits + (position < 0.0f ? -shift : shift)));
}
__device__ __forceinline__ v3 spawn_point(v3 p, v3 dir, v3 origin, float t) {
  float err = 4e-7f * (fmax_(abs_(origin.x), fmax_(abs_(origin.y), abs_(origin.z))) + t);
  v3 moved = mk3(offset_axis(p.x, dir.x), offset_axis(p.y, dir.y), offset_axis(p.z, dir.z));
  return add3(moved, scl3(dir, err));
}

// ------------------------------------------------------------------ lights
struct LightRow {
  float4 a, b, c, d;
};
__device__ __forceinline__ LightRow load_light(const ShadeView& v, uint32_t i) {
  const float4* p = reinterpret_cast<const float4*>(v.lights + i);
  LightRow l;
  l.a = __ldg(p);
  l.b = __ldg(p + 1);
  l.c = __ldg(p + 2);
  l.d = __ldg(p + 3);
  return l;
}
// The trigonometry of a light-tree row's cones, which its importance needs at
// every visit, computed once per row by the same functions (k_light_trig):
// node  = (cos theta_o, sin theta_o, cos(theta_o + theta_e), cos(theta_e - theta_o))
//         of a tree node (theta_o = c.w, theta_e = d.x);
// light = (theta_e, cos theta_e, cos 0, sin 0) of a light (theta_o = 0; a
//         spot's theta_e = acos(-d.y / d.x), otherwise pi / 2).
struct RowTrig {
  float4 node, light;
};
__device__ __forceinline__ RowTrig load_trig(const ShadeView& v, uint32_t i) {
  return RowTrig{__ldg(v.light_trig + 2u * i), __ldg(v.light_trig + 2u * i + 1u)};
}

__device__ __forceinline__ v3 f3of(float4 q) { return mk3(q.x, q.y, q.z); }
__device__ __forceinline__ float mis_power(float chosen, float other) {
  if (chosen <= 0.0f) return 0.0f;
  float ratio = other / chosen;
  return 1.0f / (1.0f + ratio * ratio);
}
struct Plane {
  v3 n;
  float area;
};
__device__ __forceinline__ Plane area_frame(const LightRow& l) {
  if (f2u(l.a.w) == 3u) return Plane{f3of(l.c), SH_PI * l.d.x * l.d.x};
  v3 spanned = scl3(cross3(f3of(l.c), f3of(l.d)), 4.0f);
  float area = length3(spanned);
  return Plane{divs3(spanned, area), area};
}

// light_hits (lights.wgsl:64-91)
SH_CALL v3 light_hits(const ShadeView& v, v3 o, v3 d, float limit, v3 previous_point,
                                         float previous_pdf) {
  v3 total = splat3(0.0f);
  for (uint32_t i = 0u; i < v.looped; ++i) {
    LightRow light = load_light(v, i);
    uint32_t kind = f2u(light.a.w);
    if ((kind != 2u && kind != 3u) || light.d.w < 0.5f) continue;
    Plane plane = area_frame(light);
    float facing = dot3(d, plane.n);
    if (abs_(facing) < 1e-9f || (light.c.w < 0.5f && facing >= 0.0f)) continue;
    float t = dot3(sub3(f3of(light.a), o), plane.n) / facing;
    if (t <= 0.0001f || t >= limit) continue;
    v3 x = add3(o, scl3(d, t));
    v3 q = sub3(x, f3of(light.a));
    if (kind == 3u) {
      if (dot3(q, q) > light.d.x * light.d.x) continue;
    } else if (abs_(dot3(q, f3of(light.c))) > dot3(f3of(light.c), f3of(light.c)) ||
               abs_(dot3(q, f3of(light.d))) > dot3(f3of(light.d), f3of(light.d))) {
      continue;
    }
    float weight = 1.0f;
    if (previous_pdf > 0.0f) {
      v3 to = sub3(x, previous_point);
      float distance2 = dot3(to, to);
      float cosine = abs_(dot3(plane.n, to)) / sqrtf(fmax_(distance2, 1e-30f));
      weight = mis_power(previous_pdf, distance2 / (plane.area * fmax_(cosine, 1e-7f)));
    }
    total = add3(total, scl3(f3of(light.b), weight));
  }
  return total;
}

struct Candidate {
  v3 wi, scale;
  float pdf, roughness;
  v3 direction;
  float limit;
};
__device__ __forceinline__ Candidate candidate_none() {
  Candidate c;
  c.wi = mk3(0.0f, 0.0f, 1.0f);
  c.scale = splat3(0.0f);
  c.pdf = 0.0f;
  c.roughness = 0.0f;
  c.direction = mk3(0.0f, 0.0f, 1.0f);
  c.limit = -1.0f;
  return c;
}
__device__ __forceinline__ void shadow_ray(v3 origin, v3 aim, bool shadow, v3& dir, float& limit) {
  dir = mk3(0.0f, 0.0f, 1.0f);
  limit = 0.0f;
  if (!shadow) return;
  v3 ray = sub3(aim, origin);
  float distance = length3(ray);
  float l = distance * 0.9999f - 0.0002f;
  if (l <= 0.0f) return;
  dir = divs3(ray, distance);
  limit = l;
}

// light_candidate (lights.wgsl:145-200) of light row `row`, loaded here so that
// the caller holds no copy of the row in memory across the call.
SH_TREE Candidate light_candidate(const Specialise& sp, const ShadeView& v, uint32_t row, const m3& transform,
                                  v3 p, v3 origin, v3 geometric, uint32_t& state, float4 u) {
  const LightRow light = load_light(v, row);
  Candidate out = candidate_none();
  bool shadow = light.d.w > 0.5f;
  uint32_t kind = f2u(light.a.w);
  if (kind == 2u || kind == 3u) {
    float u1 = rnd(sp, state, u.x);
    float u2 = rnd(sp, state, u.y);
    Plane plane = area_frame(light);
    v3 x = add3(add3(f3of(light.a), scl3(f3of(light.c), 2.0f * u1 - 1.0f)), scl3(f3of(light.d), 2.0f * u2 - 1.0f));
    if (kind == 3u) {
      m3 disc = basis(f3of(light.c));
      float r = light.d.x * sqrtf(u1);
      float phi = 2.0f * SH_PI * u2;
      x = add3(add3(f3of(light.a), scl3(disc.c0, r * cos_(phi))), scl3(disc.c1, r * sin_(phi)));
    }
    v3 to = sub3(x, p);
    float distance2 = dot3(to, to);
    v3 direction = divs3(to, sqrtf(fmax_(distance2, 1e-30f)));
    v3 local = mulmtv(transform, direction);
    if (local.z <= 0.0f) return out;
    float facing = -dot3(plane.n, direction);
    float cosine = light.c.w > 0.5f ? abs_(facing) : facing;
    if (cosine <= 1e-7f) return out;
    float pdf = distance2 / (plane.area * cosine);
    v3 dir;
    float limit;
    shadow_ray(origin, x, shadow, dir, limit);
    out.wi = local;
    out.direction = dir;
    out.limit = limit;
    out.roughness = 0.0f;
    if (!shadow) {
      out.scale = divs3(f3of(light.b), pdf);
      out.pdf = 0.0f;
    } else {
      out.scale = f3of(light.b);
      out.pdf = pdf;
    }
    return out;
  }
  v3 to = sub3(f3of(light.a), p);
  float distance = length3(to);
  float range = light.b.w;
  if (distance >= range || distance <= 1e-6f) return out;
  v3 l = divs3(to, distance);
  v3 local = mulmtv(transform, l);
  if (local.z <= 0.0f || dot3(geometric, l) <= 0.0f) return out;
  float cone = 1.0f;
  if (f2u(light.a.w) == 1u) {
    float along = clamp_(dot3(neg3(l), f3of(light.c)) * light.d.x + light.d.y, 0.0f, 1.0f);
    cone = along * along;
    if (cone <= 0.0f) return out;
  }
  float radius = light.c.w;
  v3 aim = f3of(light.a);
  if (shadow && radius > 0.0f) {
    m3 disc = basis(l);
    float r = radius * sqrtf(rnd(sp, state, u.x));
    float phi = 2.0f * SH_PI * rnd(sp, state, u.y);
    aim = add3(aim, add3(scl3(disc.c0, r * cos_(phi)), scl3(disc.c1, r * sin_(phi))));
  }
  float ratio = distance / range;
  float window = clamp_(1.0f - ratio * ratio * ratio * ratio, 0.0f, 1.0f);
  float reach = fmax_(distance, radius);
  v3 dir;
  float limit;
  shadow_ray(origin, aim, shadow, dir, limit);
  out.wi = local;
  out.scale = scl3(f3of(light.b), window * window * cone / (reach * reach));
  out.pdf = 0.0f;
  out.roughness = sqrtf(clamp_(radius / (2.0f * distance), 0.0f, 1.0f));
  out.direction = dir;
  out.limit = limit;
  return out;
}

__device__ __forceinline__ float sin_from_cos(float c) { return sqrtf(fmax_(1.0f - c * c, 0.0f)); }

// tree_importance (lights.wgsl:204-237) -> (max, min)
// trig = (cos theta_o, sin theta_o, cos(theta_o + theta_e), cos(theta_e - theta_o)).
// The light-tree functions are written once as inline bodies (`*_b`); IN
// selects whether a body calls the next ones inline (the descent kernel) or
// through their out-of-line copies (the kernels that keep them out of line).
__device__ __forceinline__ float2 tree_importance_b(v3 n, v3 to, float cos_u, v3 axis, float theta_o, float theta_e,
                                                    float far, float near, float energy, float4 trig) {
  float sin_u = sin_from_cos(cos_u);
  float cos_i = dot3(to, n);
  float sin_i = sin_from_cos(cos_i);
  float cos_min_i = cos_i >= cos_u ? 1.0f : cos_i * cos_u + sin_i * sin_u;
  if (cos_min_i < 0.0f) return make_float2(0.0f, 0.0f);
  float cos_max_i = fmax_(cos_i * cos_u - sin_i * sin_u, 0.0f);
  float cos_t = 1.0f, sin_t = 0.0f;
  v3 nt = neg3(to);
  if (axis.x != nt.x || axis.y != nt.y || axis.z != nt.z) {
    cos_t = dot3(axis, nt);
    sin_t = sin_from_cos(cos_t);
  }
  float cos_t_minus_u = cos_t * cos_u + sin_t * sin_u;
  float cos_o = trig.x;
  float sin_o = trig.y;
  float cos_min_out;
  if (cos_t >= cos_u || cos_t_minus_u >= cos_o) {
    cos_min_out = 1.0f;
  } else if (theta_o + theta_e > SH_PI || cos_t_minus_u > trig.z) {
    cos_min_out = cos_t_minus_u * cos_o + sin_from_cos(cos_t_minus_u) * sin_o;
  } else {
    return make_float2(0.0f, 0.0f);
  }
  float most = abs_(cos_min_i * energy * cos_min_out / (near * near));
  float cos_t_plus_u = cos_t * cos_u - sin_t * sin_u;
  if (theta_e - theta_o < 0.0f || cos_t < 0.0f || cos_u < 0.0f || cos_t_plus_u < trig.w)
    return make_float2(most, 0.0f);
  float cos_max_out = cos_t_plus_u * cos_o - sin_from_cos(cos_t_plus_u) * sin_o;
  return make_float2(most, abs_(cos_max_i * energy * cos_max_out / (far * far)));
}
SH_SMALL float2 tree_importance(v3 n, v3 to, float cos_u, v3 axis, float theta_o, float theta_e, float far,
                                float near, float energy, float4 trig) {
  return tree_importance_b(n, to, cos_u, axis, theta_o, theta_e, far, near, energy, trig);
}
template <bool IN>
__device__ __forceinline__ float2 tree_importance_to(v3 n, v3 to, float cos_u, v3 axis, float theta_o, float theta_e,
                                                     float far, float near, float energy, float4 trig) {
  if constexpr (IN) return tree_importance_b(n, to, cos_u, axis, theta_o, theta_e, far, near, energy, trig);
  return tree_importance(n, to, cos_u, axis, theta_o, theta_e, far, near, energy, trig);
}
template <bool IN>
__device__ __forceinline__ float2 node_importance_b(const LightRow& node, float4 trig, v3 p, v3 n) {
  v3 lo = f3of(node.a), hi = f3of(node.b);
  v3 centroid = scl3(add3(lo, hi), 0.5f);
  v3 extent = sub3(hi, centroid);
  if (dot3(n, sub3(centroid, p)) + dot3(abs3(n), abs3(extent)) <= 0.0f) return make_float2(0.0f, 0.0f);
  if (length3(sub3(p, clamp3(p, lo, hi))) >= node.b.w) return make_float2(0.0f, 0.0f);
  v3 to = sub3(centroid, p);
  float reach = length3(to);
  float radius2 = dot3(extent, extent);
  float cos_u = -1.0f;
  if (reach * reach > radius2) cos_u = sqrtf(fmax_(1.0f - radius2 / (reach * reach), 0.0f));
  float distance = fmax_(fmax_(0.5f * sqrtf(radius2), reach), 1e-6f);
  return tree_importance_to<IN>(n, divs3(to, fmax_(reach, 1e-30f)), cos_u, f3of(node.c), node.c.w, node.d.x,
                                distance, distance, node.a.w, trig);
}
SH_SMALL float2 node_importance(const LightRow& node, float4 trig, v3 p, v3 n) {
  return node_importance_b<false>(node, trig, p, n);
}
// trig: the light's RowTrig::light.
template <bool IN>
__device__ __forceinline__ float2 emitter_importance_b(const LightRow& light, float4 trig, v3 p, v3 n) {
  v3 to = sub3(f3of(light.a), p);
  float near = length3(to);
  if (near >= light.b.w || near <= 1e-6f) return make_float2(0.0f, 0.0f);
  v3 toward = divs3(to, near);
  float radius = light.c.w;
  float far = sqrtf(radius * radius + near * near);
  float cos_u = near / far;
  float energy = (light.b.x + light.b.y + light.b.z) / 3.0f;
  const float4 cones = make_float4(trig.z, trig.w, trig.y, trig.y);  // theta_o = 0
  if (f2u(light.a.w) == 1u) {
    float theta_e = trig.x;
    float cos_min_out = cos_(fmax_(0.0f, acos_(clamp_(dot3(f3of(light.c), neg3(toward)), -1.0f, 1.0f)) - acos_(cos_u)));
    float along = clamp_(cos_min_out * light.d.x + light.d.y, 0.0f, 1.0f);
    energy = energy * (along * along);
    return tree_importance_to<IN>(n, toward, cos_u, f3of(light.c), 0.0f, theta_e, far, near, energy, cones);
  }
  return tree_importance_to<IN>(n, toward, cos_u, neg3(toward), 0.0f, trig.x, far, near, energy, cones);
}
SH_SMALL float2 emitter_importance(const LightRow& light, float4 trig, v3 p, v3 n) {
  return emitter_importance_b<false>(light, trig, p, n);
}
template <bool IN>
__device__ __forceinline__ float2 emitter_importance_to(const LightRow& light, float4 trig, v3 p, v3 n) {
  if constexpr (IN) return emitter_importance_b<true>(light, trig, p, n);
  return emitter_importance(light, trig, p, n);
}
template <bool IN>
__device__ __forceinline__ float2 child_importance(const ShadeView& v, uint32_t row, v3 p, v3 n) {
  LightRow node = load_light(v, row);
  if (f2u(node.d.y) == 1u) {
    uint32_t light = f2u(node.d.z);
    return emitter_importance_to<IN>(load_light(v, light), load_trig(v, light).light, p, n);
  }
  if constexpr (IN) return node_importance_b<true>(node, load_trig(v, row).node, p, n);
  return node_importance(node, load_trig(v, row).node, p, n);
}

// tree_leaf (lights.wgsl:276-349): (selected row, pmf).  `use_known`: the
// leaf holds one light whose importance the descent has already evaluated
// (child_importance of that leaf: emitter_importance of the same light row
// at the same point), passed as `known` instead of being evaluated again.
template <bool IN>
__device__ __forceinline__ float2 tree_leaf_b(const ShadeView& v, uint32_t first, uint32_t count, v3 p, v3 n,
                                              float start, float2 known, bool use_known) {
  float rand = start;
  bool sample_max = rand > 0.5f;
  if (count > 1u) rand = rand * 2.0f - (sample_max ? 1.0f : 0.0f);
  int32_t selected = -1;
  float chosen = 0.0f, chosen_other = 0.0f, total = 0.0f, total_other = 0.0f;
  uint32_t has = 0u;
  for (uint32_t i = 0u; i < count; ++i) {
    int32_t index = (int32_t)(first + i);
    float2 importance = (use_known && i == 0u)
                            ? known
                            : emitter_importance_to<IN>(load_light(v, first + i), load_trig(v, first + i).light, p, n);
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
  if (has == 0u) return make_float2(0.0f, 0.0f);
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
      chosen_max = (use_known && (uint32_t)selected == first)
                       ? known.x
                       : emitter_importance_to<IN>(load_light(v, (uint32_t)selected),
                                                   load_trig(v, (uint32_t)selected).light, p, n).x;
    }
  }
  return make_float2((float)selected, 0.5f * (chosen_max / total_max + chosen_min / total_min));
}

// tree_pick (lights.wgsl:350-386): (light row, pmf).  The descent is bounded
// by the number of tree rows; a malformed tree ends the descent with pmf 0.
SH_TREE float2 tree_leaf(const ShadeView& v, uint32_t first, uint32_t count, v3 p, v3 n, float start, float2 known,
                         bool use_known) {
  return tree_leaf_b<false>(v, first, count, p, n, start, known, use_known);
}
template <bool IN>
__device__ __forceinline__ float2 tree_pick_b(const ShadeView& v, uint32_t rows, v3 p, v3 n, float start,
                                              uint32_t* leaf_row) {
  uint32_t at = f2u((float)v.looped + (float)v.tree);
  float rand = start;
  float pdf = 1.0f;
  float2 known = make_float2(0.0f, 0.0f);  // the importance of `at`, once the descent has evaluated it
  bool evaluated = false;
  for (uint32_t guard = 0u; guard < rows; ++guard) {
    if (at >= rows) break;
    LightRow node = load_light(v, at);
    uint32_t count = f2u(node.d.y);
    if (count > 0u) {
      if (leaf_row) *leaf_row = at;
      const bool use_known = evaluated && count == 1u;
      float2 leaf = IN ? tree_leaf_b<true>(v, f2u(node.d.z), count, p, n, rand, known, use_known)
                       : tree_leaf(v, f2u(node.d.z), count, p, n, rand, known, use_known);
      return make_float2(leaf.x, leaf.y * pdf);
    }
    uint32_t left = at + 1u;
    uint32_t right = f2u(node.d.z);
    if (right >= rows) break;
    float2 l = child_importance<IN>(v, left, p, n);
    float2 r = child_importance<IN>(v, right, p, n);
    float total_max = l.x + r.x;
    if (total_max == 0.0f) return make_float2(0.0f, 0.0f);
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
    known = at == left ? l : r;
    evaluated = true;
  }
  return make_float2(0.0f, 0.0f);
}
SH_TREE float2 tree_pick(const ShadeView& v, uint32_t rows, v3 p, v3 n, float start, uint32_t* leaf_row) {
  return tree_pick_b<false>(v, rows, p, n, start, leaf_row);
}

// ------------------------------------------------------------ emitters
__device__ __forceinline__ float cone_pdf(v3 apex, v3 center, float radius) {
  v3 to = sub3(center, apex);
  float distance2 = dot3(to, to);
  float r2 = radius * radius;
  if (distance2 <= r2) return 1.0f / (4.0f * SH_PI);
  float cos_max = sqrtf(fmax_(1.0f - r2 / distance2, 0.0f));
  float open = (r2 / distance2) / (1.0f + cos_max);
  return 1.0f / (2.0f * SH_PI * open);
}
struct EmitterRow {
  float4 a, b, c, e;
};
__device__ __forceinline__ EmitterRow load_emitter(const ShadeView& v, uint32_t i) {
  const float4* p = reinterpret_cast<const float4*>(v.emitters + i);
  EmitterRow r;
  r.a = __ldg(p);
  r.b = __ldg(p + 1);
  r.c = __ldg(p + 2);
  r.e = __ldg(p + 3);
  return r;
}
// emitter_pdf (lights.wgsl:31-37)
__device__ __forceinline__ float emitter_pdf(const EmitterRow& e, v3 x, v3 apex, v3 normal) {
  if (e.a.w > 0.5f) return e.e.w * cone_pdf(apex, f3of(e.a), e.c.x);
  v3 to = sub3(x, apex);
  float distance2 = dot3(to, to);
  float cosine = abs_(dot3(normal, to)) / sqrtf(fmax_(distance2, 1e-30f));
  return e.e.w / fmax_(e.c.w, 1e-30f) * distance2 / fmax_(cosine, 1e-7f);
}
__device__ __forceinline__ uint32_t find_emitter(const ShadeView& v, uint32_t count, float u) {
  uint32_t low = 0u, high = count;
  while (low < high) {
    uint32_t mid = (low + high) / 2u;
    if (__ldg(v.emitter_cdf + mid) <= u)
      low = mid + 1u;
    else
      high = mid;
  }
  return low < count - 1u ? low : count - 1u;
}
__device__ __forceinline__ bool clipped_at(const GpuSurface* __restrict__ surfaces, uint32_t record, v3 point) {
  const float4* s = reinterpret_cast<const float4*>(surfaces + record);
  float4 c0 = __ldg(s), c1 = __ldg(s + 1);
  bool a = (c0.x != 0.0f || c0.y != 0.0f || c0.z != 0.0f) && dot3(f3of(c0), point) > c0.w;
  bool b = (c1.x != 0.0f || c1.y != 0.0f || c1.z != 0.0f) && dot3(f3of(c1), point) > c1.w;
  return a || b;
}
// emitter_candidate (lights.wgsl:103-144) for triangle emitters
SH_CALL Candidate emitter_candidate(const ShadeView& v, const Specialise& sp, const m3& transform,
                                                       v3 p, v3 origin, uint32_t& state, float4 u) {
  EmitterRow e = load_emitter(v, find_emitter(v, v.emitter_count, rnd(sp, state, u.z)) + 1u);
  Candidate out = candidate_none();
  if (e.a.w > 0.5f) return out;  // analytic shape emitters are outside this tracer
  float r1 = sqrtf(rnd(sp, state, u.x));
  float r2 = rnd(sp, state, u.y);
  v3 x = add3(add3(scl3(f3of(e.a), 1.0f - r1), scl3(f3of(e.b), r1 * (1.0f - r2))), scl3(f3of(e.c), r1 * r2));
  if (clipped_at(v.surfaces, f2u(e.b.w), x)) return out;
  v3 to = sub3(x, p);
  float distance2 = dot3(to, to);
  v3 direction = divs3(to, sqrtf(fmax_(distance2, 1e-30f)));
  v3 local = mulmtv(transform, direction);
  if (local.z <= 0.0f) return out;
  v3 normal = normalize3(cross3(sub3(f3of(e.b), f3of(e.a)), sub3(f3of(e.c), f3of(e.a))));
  if (abs_(dot3(normal, sub3(p, f3of(e.a)))) <= 1e-5f) return out;
  float cosine = abs_(dot3(normal, direction));
  if (cosine <= 1e-7f) return out;
  v3 dir;
  float limit;
  shadow_ray(origin, x, true, dir, limit);
  out.wi = local;
  out.scale = f3of(e.e);
  out.pdf = e.e.w / e.c.w * distance2 / cosine;
  out.roughness = 0.0f;
  out.direction = dir;
  out.limit = limit;
  return out;
}

}  // namespace pfxt
