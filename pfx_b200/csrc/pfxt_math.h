// Exact-arithmetic primitives shared by the sm_100a kernels and the host code.
//
// Every function here uses only IEEE-754 single-precision +, -, *, /, sqrt,
// floor, trunc, rint, comparisons and integer bit operations.  Compiled with
// FMA contraction off (nvcc -fmad=false, gcc -ffp-contract=off) and IEEE
// division/square root, a function returns the same bits on the GPU and on the
// CPU.  That is what makes the per-pixel parity of the tracer possible: a path
// that takes one different rounding turns into a different path.
//
// The transcendental functions are this project's own, written from published
// methods, not copied from any math library:
//   * argument reduction: W. J. Cody and W. Waite, "Software Manual for the
//     Elementary Functions" (1980): x - k*C1 - k*C2 - k*C3 with C1, C2 holding
//     few significant bits so that k*C1 and k*C2 are exact; the split
//     constants below are pi/2 and ln 2 cut at 12 trailing mantissa bits;
//   * kernels: truncated Taylor series (coefficients 1/n!, 1/(2n+1), and the
//     arcsine series (2n)!/(4^n (n!)^2 (2n+1))), evaluated by Horner's rule;
//   * arctangent: the half-angle identity atan t = 2 atan(t / (1 + sqrt(1+t^2)))
//     applied twice before the series;
//   * logarithm: log m = 2 atanh((m-1)/(m+1)) for m in [sqrt(1/2), sqrt(2)).
// Accuracy (checked against the host libm in tests/test_math.py): a few ulp.
//
// The WGSL built-ins of the reference tracer (crates/trace/src/trace.wgsl,
// crates/materials/src/wgsl/brdf.wgsl) map onto the helpers here: dot/cross
// evaluate left to right, mix(a,b,t) = a*(1-t) + b*t, clamp = min(max()),
// normalize(v) = v * (1/sqrt(dot(v,v))), fract(x) = x - floor(x), and the float
// modulo is x - y*trunc(x/y).
#pragma once

#include <stdint.h>
#include <string.h>
#include <math.h>

#if defined(__CUDACC__)
#define PFXT_HD __host__ __device__ __forceinline__
// Out-of-line on the device: the transcendentals are called from many sites of
// the shading kernel, and one shared copy keeps its code in the instruction
// cache.
#ifndef PFXT_HDN
#define PFXT_HDN static __host__ __device__ __noinline__
#endif
#else
#define PFXT_HD static inline
#define PFXT_HDN static inline
#endif

namespace pfxt {

// ---------------------------------------------------------------- bit casts
PFXT_HD uint32_t f2bits(float f) {
#if defined(__CUDA_ARCH__)
  return __float_as_uint(f);
#else
  uint32_t u;
  memcpy(&u, &f, 4);
  return u;
#endif
}
PFXT_HD float bits2f(uint32_t u) {
#if defined(__CUDA_ARCH__)
  return __uint_as_float(u);
#else
  float f;
  memcpy(&f, &u, 4);
  return f;
#endif
}
PFXT_HD bool isnan_(float x) { return x != x; }

// min/max with the NaN rule of fminf/fmaxf (a NaN operand loses) and a fixed
// choice for signed zeros (the first operand wins a tie), identical on both
// sides.
PFXT_HD float fmin_(float a, float b) {
  if (isnan_(a)) return b;
  if (isnan_(b)) return a;
  return (b < a) ? b : a;
}
PFXT_HD float fmax_(float a, float b) {
  if (isnan_(a)) return b;
  if (isnan_(b)) return a;
  return (b > a) ? b : a;
}
PFXT_HD float clamp_(float x, float lo, float hi) { return fmin_(fmax_(x, lo), hi); }
PFXT_HD float abs_(float x) { return bits2f(f2bits(x) & 0x7fffffffu); }
PFXT_HD float sqrt_(float x) { return sqrtf(x); }
PFXT_HD float floor_(float x) { return floorf(x); }
PFXT_HD float trunc_(float x) { return truncf(x); }
PFXT_HD float rint_(float x) { return rintf(x); }
PFXT_HD float fract_(float x) { return x - floorf(x); }
PFXT_HD float mix_(float a, float b, float t) { return a * (1.0f - t) + b * t; }
PFXT_HD float select_(float f, float t, bool c) { return c ? t : f; }
PFXT_HD float fmod_wgsl(float x, float y) { return x - y * truncf(x / y); }

// x / d, correctly rounded, given r = x-independent RN(1/d): one product and
// one fused correction (P. Markstein, "Computation of elementary functions on
// the IBM RISC System/6000 processor", IBM J. Res. Dev. 34(1), 1990: with r
// the correctly rounded reciprocal and q within an ulp of x/d, the fused
// residual x - q*d is exact and q + residual*r rounds to RN(x/d)).  The
// theorem assumes no underflow or overflow, so tiny numerators or quotients
// and huge quotients take the plain division.  fmaf is exact on both sides.
PFXT_HD float div_rn(float x, float d, float r) {
  float q = x * r;
  float e = fmaf(-q, d, x);
  float q2 = fmaf(e, r, q);
  if (!(abs_(x) >= 0x1p-96f) || !(abs_(q2) >= 0x1p-100f) || !(abs_(q2) <= 0x1p+120f)) return x / d;
  return q2;
}
PFXT_HD float smoothstep_(float e0, float e1, float x) {
  float t = clamp_((x - e0) / (e1 - e0), 0.0f, 1.0f);
  return t * t * (3.0f - 2.0f * t);
}

// WGSL u32(f32): round toward zero, saturating; NaN gives 0.
PFXT_HD uint32_t f2u(float x) {
  if (!(x > 0.0f)) return 0u;
  if (x >= 4294967296.0f) return 0xffffffffu;
  return (uint32_t)x;
}
// WGSL i32(f32): round toward zero, saturating; NaN gives 0.
PFXT_HD int32_t f2i(float x) {
  if (isnan_(x)) return 0;
  if (x >= 2147483648.0f) return 2147483647;
  if (x <= -2147483648.0f) return (-2147483647 - 1);
  return (int32_t)x;
}
PFXT_HD float u2f(uint32_t u) { return (float)u; }

PFXT_HD uint32_t popc_(uint32_t x) {
#if defined(__CUDA_ARCH__)
  return (uint32_t)__popc(x);
#else
  return (uint32_t)__builtin_popcount(x);
#endif
}
PFXT_HD uint32_t brev_(uint32_t x) {
#if defined(__CUDA_ARCH__)
  return __brev(x);
#else
  x = ((x >> 1) & 0x55555555u) | ((x & 0x55555555u) << 1);
  x = ((x >> 2) & 0x33333333u) | ((x & 0x33333333u) << 2);
  x = ((x >> 4) & 0x0f0f0f0fu) | ((x & 0x0f0f0f0fu) << 4);
  x = ((x >> 8) & 0x00ff00ffu) | ((x & 0x00ff00ffu) << 8);
  return (x >> 16) | (x << 16);
#endif
}
PFXT_HD uint32_t clz_(uint32_t x) {
#if defined(__CUDA_ARCH__)
  return (uint32_t)__clz(x);
#else
  return x == 0u ? 32u : (uint32_t)__builtin_clz(x);
#endif
}

// ---------------------------------------------------------------- constants
// f32 nearest to pi, as the reference's `const PI: f32 = 3.141592653589793`.
#define PFXT_PI 0x1.921fb6p+1f
#define PFXT_HALF_PI 0x1.921fb6p+0f
// Cody-Waite split of pi/2 (12 trailing mantissa bits cleared in C1, C2).
#define PFXT_PIO2_C1 0x1.92p+0f
#define PFXT_PIO2_C2 0x1.fb4p-12f
#define PFXT_PIO2_C3 0x1.4442d2p-24f
#define PFXT_TWO_OVER_PI 0x1.45f306p-1f
// Cody-Waite split of ln 2.
#define PFXT_LN2_C1 0x1.62ep-1f
#define PFXT_LN2_C2 0x1.0bfbe8p-15f
#define PFXT_LOG2E 0x1.715476p+0f
#define PFXT_LN2 0x1.62e430p-1f
#define PFXT_SQRT_HALF 0x1.6a09e6p-1f

// --------------------------------------------------------- sine and cosine
// Reduced argument r in [-pi/4, pi/4]; quadrant q = k mod 4.
PFXT_HD float sin_kernel(float r) {
  float r2 = r * r;
  float p = -0x1.ae6456p-26f;
  p = p * r2 + 0x1.71de3ap-19f;
  p = p * r2 + -0x1.a01a02p-13f;
  p = p * r2 + 0x1.111112p-7f;
  p = p * r2 + -0x1.555556p-3f;
  return r + (r * r2) * p;
}
PFXT_HD float cos_kernel(float r) {
  float r2 = r * r;
  float p = 0x1.1eed8ep-29f;
  p = p * r2 + -0x1.27e4fcp-22f;
  p = p * r2 + 0x1.a01a02p-16f;
  p = p * r2 + -0x1.6c16c2p-10f;
  p = p * r2 + 0x1.555556p-5f;
  // 1 - r2/2 + r2^2 * p
  return 1.0f - 0.5f * r2 + (r2 * r2) * p;
}
PFXT_HD void reduce_pio2(float x, float* r, int* q) {
  float k = floorf(x * PFXT_TWO_OVER_PI + 0.5f);
  float y = x - k * PFXT_PIO2_C1;
  y = y - k * PFXT_PIO2_C2;
  y = y - k * PFXT_PIO2_C3;
  *r = y;
  int ki = (int)k;
  *q = ki & 3;
}
PFXT_HDN float sin_(float x) {
  if (isnan_(x) || abs_(x) == INFINITY) return NAN;
  float r;
  int q;
  reduce_pio2(x, &r, &q);
  float v = (q & 1) ? cos_kernel(r) : sin_kernel(r);
  return (q & 2) ? -v : v;
}
PFXT_HDN float cos_(float x) {
  if (isnan_(x) || abs_(x) == INFINITY) return NAN;
  float r;
  int q;
  reduce_pio2(x, &r, &q);
  float v = (q & 1) ? sin_kernel(r) : cos_kernel(r);
  return (q == 1 || q == 2) ? -v : v;
}

// ------------------------------------------------------ arcsine / arccosine
// Odd series for |z| <= 0.5.
PFXT_HD float asin_series(float z) {
  float z2 = z * z;
  float p = 0x1.df3bd4p-8f;
  p = p * z2 + 0x1.12ef3cp-7f;
  p = p * z2 + 0x1.3fde50p-7f;
  p = p * z2 + 0x1.7a8788p-7f;
  p = p * z2 + 0x1.c9999ap-7f;
  p = p * z2 + 0x1.1c4ec4p-6f;
  p = p * z2 + 0x1.6e8ba2p-6f;
  p = p * z2 + 0x1.f1c71cp-6f;
  p = p * z2 + 0x1.6db6dcp-5f;
  p = p * z2 + 0x1.333334p-4f;
  p = p * z2 + 0x1.555556p-3f;
  return z + (z * z2) * p;
}
PFXT_HDN float asin_(float x) {
  if (isnan_(x) || x > 1.0f || x < -1.0f) return NAN;
  float ax = abs_(x);
  float a;
  if (ax <= 0.5f) {
    a = asin_series(ax);
  } else {
    float s = sqrtf((1.0f - ax) * 0.5f);
    a = PFXT_HALF_PI - 2.0f * asin_series(s);
  }
  return x < 0.0f ? -a : a;
}
PFXT_HDN float acos_(float x) {
  if (isnan_(x) || x > 1.0f || x < -1.0f) return NAN;
  float ax = abs_(x);
  if (ax <= 0.5f) return PFXT_HALF_PI - asin_series(x);
  float s = sqrtf((1.0f - ax) * 0.5f);
  float a = 2.0f * asin_series(s);
  return x > 0.0f ? a : PFXT_PI - a;
}

// --------------------------------------------------------------- arctangent
PFXT_HD float atan_unit(float t) {  // t in [0, 1]
  float t1 = t / (1.0f + sqrtf(1.0f + t * t));
  float t2 = t1 / (1.0f + sqrtf(1.0f + t1 * t1));
  float s = t2 * t2;
  float p = -0x1.111112p-4f;
  p = p * s + 0x1.3b13b2p-4f;
  p = p * s + -0x1.745d18p-4f;
  p = p * s + 0x1.c71c72p-4f;
  p = p * s + -0x1.24924ap-3f;
  p = p * s + 0x1.99999ap-3f;
  p = p * s + -0x1.555556p-2f;
  return 4.0f * (t2 + (t2 * s) * p);
}
PFXT_HDN float atan2_(float y, float x) {
  if (isnan_(x) || isnan_(y)) return NAN;
  float ax = abs_(x), ay = abs_(y);
  if (ax == 0.0f && ay == 0.0f) return 0.0f;
  float a;
  if (ay > ax) {
    a = PFXT_HALF_PI - atan_unit(ax / ay);
  } else {
    a = atan_unit(ay / ax);
  }
  if (x < 0.0f) a = PFXT_PI - a;
  return y < 0.0f ? -a : a;
}

// ------------------------------------------------- exponential / logarithm
PFXT_HD float ldexp_(float x, int k) {  // x * 2^k, k in [-252, 254]
  while (k > 127) {
    x = x * 0x1.p+127f;
    k -= 127;
  }
  while (k < -126) {
    x = x * 0x1.p-126f;
    k += 126;
  }
  return x * bits2f((uint32_t)(k + 127) << 23);
}
PFXT_HDN float exp_(float x) {
  if (isnan_(x)) return NAN;
  if (x > 88.7228f) return INFINITY;
  if (x < -103.973f) return 0.0f;
  float k = floorf(x * PFXT_LOG2E + 0.5f);
  float r = x - k * PFXT_LN2_C1;
  r = r - k * PFXT_LN2_C2;
  float p = 0x1.71de3ap-19f;
  p = p * r + 0x1.a01a02p-16f;
  p = p * r + 0x1.a01a02p-13f;
  p = p * r + 0x1.6c16c2p-10f;
  p = p * r + 0x1.111112p-7f;
  p = p * r + 0x1.555556p-5f;
  p = p * r + 0x1.555556p-3f;
  p = p * r + 0x1.p-1f;
  float e = 1.0f + (r + (r * r) * p);
  return ldexp_(e, (int)k);
}
PFXT_HDN float log_(float x) {
  if (isnan_(x) || x < 0.0f) return NAN;
  if (x == 0.0f) return -INFINITY;
  if (x == INFINITY) return INFINITY;
  int e = 0;
  if (x < 0x1.p-126f) {  // subnormal: scale into the normal range
    x = x * 0x1.p+24f;
    e = -24;
  }
  uint32_t b = f2bits(x);
  e += (int)((b >> 23) & 0xffu) - 127;
  float m = bits2f((b & 0x007fffffu) | 0x3f800000u);  // [1, 2)
  if (m > 0x1.6a09e6p+0f) {  // > sqrt(2): use m/2, e+1
    m = m * 0.5f;
    e += 1;
  }
  float s = (m - 1.0f) / (m + 1.0f);
  float s2 = s * s;
  float p = 0x1.3b13b2p-4f;
  p = p * s2 + 0x1.745d18p-4f;
  p = p * s2 + 0x1.c71c72p-4f;
  p = p * s2 + 0x1.24924ap-3f;
  p = p * s2 + 0x1.99999ap-3f;
  p = p * s2 + 0x1.555556p-2f;
  float lm = 2.0f * s + (2.0f * s * s2) * p;
  float ef = (float)e;
  return (ef * PFXT_LN2_C2 + lm) + ef * PFXT_LN2_C1;
}
// pow(x, y): small non-negative integer exponents by repeated multiplication
// (the common Fresnel and falloff powers), else exp(y log x).
PFXT_HD float pow_(float x, float y) {
  if (y == 0.0f) return 1.0f;
  if (y > 0.0f && y <= 16.0f && floorf(y) == y) {
    int n = (int)y;
    float r = 1.0f, b = x;
    while (n) {
      if (n & 1) r = r * b;
      n >>= 1;
      if (n) b = b * b;
    }
    return r;
  }
  if (x == 0.0f) return y > 0.0f ? 0.0f : INFINITY;
  if (x < 0.0f) return NAN;
  return exp_(y * log_(x));
}

// ------------------------------------------------------------------ vectors
struct v3 {
  float x, y, z;
};
PFXT_HD v3 mk3(float x, float y, float z) {
  v3 r;
  r.x = x;
  r.y = y;
  r.z = z;
  return r;
}
PFXT_HD v3 add3(v3 a, v3 b) { return mk3(a.x + b.x, a.y + b.y, a.z + b.z); }
PFXT_HD v3 sub3(v3 a, v3 b) { return mk3(a.x - b.x, a.y - b.y, a.z - b.z); }
PFXT_HD v3 mul3(v3 a, v3 b) { return mk3(a.x * b.x, a.y * b.y, a.z * b.z); }
PFXT_HD v3 div3(v3 a, v3 b) { return mk3(a.x / b.x, a.y / b.y, a.z / b.z); }
PFXT_HD v3 scl3(v3 a, float s) { return mk3(a.x * s, a.y * s, a.z * s); }
PFXT_HD v3 divs3(v3 a, float s) { return mk3(a.x / s, a.y / s, a.z / s); }
PFXT_HD v3 neg3(v3 a) { return mk3(-a.x, -a.y, -a.z); }
PFXT_HD float dot3(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
PFXT_HD v3 cross3(v3 a, v3 b) {
  return mk3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
PFXT_HD float length3(v3 a) { return sqrtf(dot3(a, a)); }
PFXT_HD v3 normalize3(v3 a) { return scl3(a, 1.0f / sqrtf(dot3(a, a))); }
PFXT_HD v3 abs3(v3 a) { return mk3(abs_(a.x), abs_(a.y), abs_(a.z)); }
PFXT_HD v3 min3(v3 a, v3 b) { return mk3(fmin_(a.x, b.x), fmin_(a.y, b.y), fmin_(a.z, b.z)); }
PFXT_HD v3 max3(v3 a, v3 b) { return mk3(fmax_(a.x, b.x), fmax_(a.y, b.y), fmax_(a.z, b.z)); }
PFXT_HD v3 clamp3(v3 a, v3 lo, v3 hi) { return min3(max3(a, lo), hi); }
PFXT_HD v3 splat3(float s) { return mk3(s, s, s); }
PFXT_HD v3 mix3(v3 a, v3 b, float t) {
  return mk3(mix_(a.x, b.x, t), mix_(a.y, b.y, t), mix_(a.z, b.z, t));
}
PFXT_HD v3 mixv3(v3 a, v3 b, v3 t) {
  return mk3(mix_(a.x, b.x, t.x), mix_(a.y, b.y, t.y), mix_(a.z, b.z, t.z));
}
PFXT_HD v3 sel3(v3 f, v3 t, bool c) { return c ? t : f; }
PFXT_HD float maxc3(v3 a) { return fmax_(a.x, fmax_(a.y, a.z)); }
PFXT_HD float get3(v3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
// reflect(i, n) = i - 2 dot(n, i) n
PFXT_HD v3 reflect3(v3 i, v3 n) { return sub3(i, scl3(n, 2.0f * dot3(n, i))); }

// 3x3 matrix stored as three columns (WGSL mat3x3f layout).
struct m3 {
  v3 c0, c1, c2;
};
// M * v = c0*v.x + c1*v.y + c2*v.z, summed left to right per component.
PFXT_HD v3 mulmv(m3 m, v3 v) {
  return add3(add3(scl3(m.c0, v.x), scl3(m.c1, v.y)), scl3(m.c2, v.z));
}
// transpose(M) * v = (dot(c0,v), dot(c1,v), dot(c2,v))
PFXT_HD v3 mulmtv(m3 m, v3 v) { return mk3(dot3(m.c0, v), dot3(m.c1, v), dot3(m.c2, v)); }

// Orthonormal basis around n (trace.wgsl:1270-1273 `basis`).
PFXT_HD m3 basis(v3 n) {
  v3 helper = abs_(n.y) > 0.9f ? mk3(1.0f, 0.0f, 0.0f) : mk3(0.0f, 1.0f, 0.0f);
  v3 t = normalize3(cross3(helper, n));
  m3 m;
  m.c0 = t;
  m.c1 = cross3(n, t);
  m.c2 = n;
  return m;
}

}  // namespace pfxt
