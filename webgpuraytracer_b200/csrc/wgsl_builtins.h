// WGSL built-in functions restated in single precision so that the CUDA kernels (device) and the
// CPU restatement of the shaders (host) produce bit-identical results for the same sequence of
// operations.
//
// Why this layer exists: WGSL leaves the precision of its transcendental built-ins
// implementation-defined (sin/cos within 2^-11 absolute on [-pi, pi], exp/log within 3+2|x| ULP,
// pow inherited from exp2(y*log2(x))).  The reference shaders (shader.wgsl, denoiser.wgsl,
// scale.wgsl) therefore have no single "true" output.  We pin one: every built-in below is
// computed from +, -, *, /, sqrt and integer bit manipulation only, each of which is correctly
// rounded IEEE-754 binary32 on both the GPU (nvcc -fmad=false -prec-div=true -prec-sqrt=true
// -ftz=false) and the CPU (g++ -ffp-contract=off, SSE).  Accuracy against float64 is checked by
// tests/test_builtins.py (a few ULP; see the per-function notes).
//
// Methods (all published, coefficients derived here from the mathematics):
//   exp   : Cody & Waite (1980) argument reduction x = n*ln2 + r with a two-part ln2, then the
//           degree-7 Taylor polynomial of e^r on |r| <= ln2/2.
//   exp2  : x = n + f, |f| <= 1/2, Taylor polynomial of e^(f ln2) in f (coefficients ln2^k/k!).
//   log   : x = m * 2^e with m in [sqrt(1/2), sqrt(2)), log m = 2 atanh(s), s = (m-1)/(m+1),
//           odd atanh series to s^11.
//   sin/cos: Cody & Waite reduction by pi/2 with a three-part pi/2, Taylor polynomials on
//           |r| <= pi/4 (sin to r^11, cos to r^12).
//   atan  : reduction to |t| <= tan(pi/8) by atan(x) = pi/4 + atan((x-1)/(x+1)) and
//           atan(x) = pi/2 - atan(1/x), then the Gregory series to t^21.
//   asin/acos: through atan2 and sqrt((1-x)(1+x)).
// Semantics follow the WGSL specification (min/max ignore a NaN operand, mix(a,b,t) =
// a*(1-t) + b*t, select(f,t,c) = c ? t : f, sign(0) = 0, pow(x,y) = exp2(y*log2(x))).
#pragma once
#include <stdint.h>
#include <math.h>
#include <string.h>

#if defined(__CUDACC__)
#define WB_HD __host__ __device__ __forceinline__
#else
#define WB_HD static inline
#endif

namespace wb {

// ------------------------------------------------------------------ bit casts
WB_HD uint32_t as_u32(float f) {
#if defined(__CUDA_ARCH__)
  return __float_as_uint(f);
#else
  uint32_t u; memcpy(&u, &f, 4); return u;
#endif
}
WB_HD float as_f32(uint32_t u) {
#if defined(__CUDA_ARCH__)
  return __uint_as_float(u);
#else
  float f; memcpy(&f, &u, 4); return f;
#endif
}
WB_HD int32_t as_i32(float f) { return (int32_t)as_u32(f); }

WB_HD bool isnan_(float x) { return x != x; }

// ------------------------------------------------------------------ scalar WGSL built-ins
// min/max: WGSL returns the non-NaN operand; for equal operands (incl. +0/-0) the first one.
WB_HD float wmin(float a, float b) { return (b < a || a != a) ? b : a; }
WB_HD float wmax(float a, float b) { return (b > a || a != a) ? b : a; }
WB_HD float clamp(float x, float lo, float hi) { return wmin(wmax(x, lo), hi); }
WB_HD float mix(float a, float b, float t) { return a * (1.0f - t) + b * t; }
WB_HD float sel(float f, float t, bool c) { return c ? t : f; }
WB_HD float sign(float x) { return x > 0.0f ? 1.0f : (x < 0.0f ? -1.0f : 0.0f); }
WB_HD float absf(float x) { return as_f32(as_u32(x) & 0x7fffffffu); }
WB_HD float fract(float x) { return x - floorf(x); }
WB_HD float sqrt_(float x) { return sqrtf(x); }

constexpr float kPI = 3.141592741e+00f;      // float(pi)
constexpr float kPIO2 = 1.570796371e+00f;    // float(pi/2)
constexpr float kPIO4 = 7.853981853e-01f;    // float(pi/4)

WB_HD float inf_() { return as_f32(0x7f800000u); }
WB_HD float nan_() { return as_f32(0x7fc00000u); }

// 2^n for integer n in [-126, 127] as an exact float.
WB_HD float pow2i(int n) { return as_f32((uint32_t)(n + 127) << 23); }

// p * 2^n with a single rounding (p normal, |log2 p| < 1).
WB_HD float scale2(float p, int n) {
  if (n > 127) return (p * pow2i(127)) * pow2i(n - 127);
  if (n >= -126) return p * pow2i(n);
  // result is subnormal or zero: the first product is exact, the second rounds once
  return (p * pow2i(n + 64)) * pow2i(-64);
}

// e^x (Cody-Waite reduction, degree-7 Taylor).
WB_HD float exp_(float x) {
  if (x != x) return x;
  if (x > 88.72284f) return inf_();
  if (x < -103.97209f) return 0.0f;
  const float kLog2e = 1.442695022e+00f;
  const float kLn2Hi = 0.693115234375f;       // 12 significant bits: n*kLn2Hi is exact
  const float kLn2Lo = 3.194618330e-05f;
  float n = floorf(x * kLog2e + 0.5f);
  float r = (x - n * kLn2Hi) - n * kLn2Lo;
  float p = 1.984127011e-04f;                 // 1/7!
  p = p * r + 1.388888923e-03f;               // 1/6!
  p = p * r + 8.333333768e-03f;               // 1/5!
  p = p * r + 4.166666791e-02f;               // 1/4!
  p = p * r + 1.666666716e-01f;               // 1/3!
  p = p * r + 5.000000000e-01f;
  p = p * r + 1.0f;
  p = p * r + 1.0f;
  return scale2(p, (int)n);
}

// 2^x (integer/fraction split, Taylor polynomial of e^(f ln2)).
WB_HD float exp2_(float x) {
  if (x != x) return x;
  if (x >= 128.0f) return inf_();
  if (x < -150.0f) return 0.0f;
  float n = floorf(x + 0.5f);
  float f = x - n;                             // exact, |f| <= 1/2 (+1 ulp)
  float p = 1.525273365e-05f;                  // ln2^7/7!
  p = p * f + 1.540352969e-04f;
  p = p * f + 1.333355787e-03f;
  p = p * f + 9.618128650e-03f;
  p = p * f + 5.550410971e-02f;
  p = p * f + 2.402265072e-01f;
  p = p * f + 6.931471825e-01f;
  p = p * f + 1.0f;
  return scale2(p, (int)n);
}

// Splits x > 0 (finite) into m in [sqrt(1/2), sqrt(2)) and e with x = m * 2^e.
WB_HD float frexp_m(float x, int* e) {
  uint32_t u = as_u32(x);
  int ex = (int)((u >> 23) & 0xffu);
  int bias = 127;
  if (ex == 0) {                               // subnormal: normalise by 2^23 (exact)
    x = x * 8388608.0f;
    u = as_u32(x);
    ex = (int)((u >> 23) & 0xffu);
    bias = 127 + 23;
  }
  float m = as_f32((u & 0x007fffffu) | 0x3f800000u);   // [1, 2)
  int k = ex - bias;
  if (m > 1.414213538e+00f) { m = m * 0.5f; k += 1; }
  *e = k;
  return m;
}

// log(m) for m in [sqrt(1/2), sqrt(2)): 2*atanh(s).
WB_HD float log_m(float m) {
  float s = (m - 1.0f) / (m + 1.0f);
  float z = s * s;
  float p = 9.090909362e-02f;                  // 1/11
  p = p * z + 1.111111119e-01f;                // 1/9
  p = p * z + 1.428571492e-01f;                // 1/7
  p = p * z + 2.000000030e-01f;                // 1/5
  p = p * z + 3.333333433e-01f;                // 1/3
  p = p * z;
  float t = s + s;
  return t + t * p;
}

WB_HD float log_(float x) {
  if (x != x) return x;
  if (x < 0.0f) return nan_();
  if (x == 0.0f) return -inf_();
  if (x == inf_()) return x;
  int e;
  float m = frexp_m(x, &e);
  float lm = log_m(m);
  float fe = (float)e;
  return fe * 0.693115234375f + (lm + fe * 3.194618330e-05f);
}

WB_HD float log2_(float x) {
  if (x != x) return x;
  if (x < 0.0f) return nan_();
  if (x == 0.0f) return -inf_();
  if (x == inf_()) return x;
  int e;
  float m = frexp_m(x, &e);
  return (float)e + log_m(m) * 1.442695022e+00f;
}

// WGSL pow: exp2(y * log2(x)).  pow(0, y>0) = 0; negative bases give NaN as the specification's
// definition implies.
WB_HD float pow_(float x, float y) { return exp2_(y * log2_(x)); }

// Square with a constant exponent of 2: WGSL pow(x, 2.0) on a negative base has no defined value;
// shader compilers fold the constant exponent into x*x, which is what the reference relies on for
// its Fresnel F0 term.
WB_HD float pow2c(float x) { return x * x; }

// sin/cos of the reduced argument r, |r| <= pi/4 (+ulp)
WB_HD float sin_poly(float r) {
  float z = r * r;
  float p = -2.505210794e-08f;                 // -1/11!
  p = p * z + 2.755731884e-06f;                // 1/9!
  p = p * z - 1.984127011e-04f;                // -1/7!
  p = p * z + 8.333333768e-03f;                // 1/5!
  p = p * z - 1.666666716e-01f;                // -1/3!
  return r + (r * z) * p;
}
WB_HD float cos_poly(float r) {
  float z = r * r;
  float p = 2.087675588e-09f;                  // 1/12!
  p = p * z - 2.755731998e-07f;                // -1/10!
  p = p * z + 2.480158764e-05f;                // 1/8!
  p = p * z - 1.388888923e-03f;                // -1/6!
  p = p * z + 4.166666791e-02f;                // 1/4!
  p = p * z - 5.000000000e-01f;
  return 1.0f + z * p;
}

// Reduction by pi/2 (three-part Cody-Waite split; exact products for |k| < 2^12).
WB_HD float reduce_pio2(float x, int* q) {
  float k = floorf(x * 6.366197467e-01f + 0.5f);
  float r = ((x - k * 1.5703125f) - k * 4.837512969970703e-04f) - k * 7.549790126e-08f;
  *q = (int)k;
  return r;
}

WB_HD float sin_(float x) {
  if (x != x || absf(x) == inf_()) return nan_();
  int q;
  float r = reduce_pio2(x, &q);
  float s;
  switch (q & 3) {
    case 0: s = sin_poly(r); break;
    case 1: s = cos_poly(r); break;
    case 2: s = -sin_poly(r); break;
    default: s = -cos_poly(r); break;
  }
  return s;
}

WB_HD float cos_(float x) {
  if (x != x || absf(x) == inf_()) return nan_();
  int q;
  float r = reduce_pio2(x, &q);
  float c;
  switch (q & 3) {
    case 0: c = cos_poly(r); break;
    case 1: c = -sin_poly(r); break;
    case 2: c = -cos_poly(r); break;
    default: c = sin_poly(r); break;
  }
  return c;
}

// atan(t) for |t| <= tan(pi/8) (+ulp): Gregory series to t^21.
WB_HD float atan_series(float t) {
  float z = t * t;
  float p = 4.761904851e-02f;                  // 1/21
  p = p * z - 5.263157934e-02f;                // -1/19
  p = p * z + 5.882352963e-02f;                // 1/17
  p = p * z - 6.666667014e-02f;                // -1/15
  p = p * z + 7.692307979e-02f;                // 1/13
  p = p * z - 9.090909362e-02f;                // -1/11
  p = p * z + 1.111111119e-01f;                // 1/9
  p = p * z - 1.428571492e-01f;                // -1/7
  p = p * z + 2.000000030e-01f;                // 1/5
  p = p * z - 3.333333433e-01f;                // -1/3
  return t + (t * z) * p;
}

// atan(a) for a >= 0 (finite or +inf).
WB_HD float atan_pos(float a) {
  if (a > 2.414213657e+00f) {                  // tan(3pi/8)
    if (a == inf_()) return kPIO2;
    return kPIO2 - atan_series(1.0f / a);
  }
  if (a > 4.142135680e-01f) {                  // tan(pi/8)
    return kPIO4 + atan_series((a - 1.0f) / (a + 1.0f));
  }
  return atan_series(a);
}

WB_HD float atan_(float x) {
  if (x != x) return x;
  float a = atan_pos(absf(x));
  return x < 0.0f ? -a : a;
}

// atan2 with C99 conventions for signed zeros.
WB_HD float atan2_(float y, float x) {
  if (x != x || y != y) return nan_();
  float ax = absf(x), ay = absf(y);
  bool xneg = (as_u32(x) >> 31) != 0u;
  bool yneg = (as_u32(y) >> 31) != 0u;
  float a;
  if (ay == 0.0f) {
    a = xneg ? kPI : 0.0f;
  } else if (ax == 0.0f) {
    a = kPIO2;
  } else if (ax == inf_() && ay == inf_()) {
    a = xneg ? 2.356194496e+00f : kPIO4;
  } else {
    if (ay <= ax) {
      a = atan_pos(ay / ax);
    } else {
      a = kPIO2 - atan_pos(ax / ay);
    }
    if (xneg) a = kPI - a;
  }
  return yneg ? -a : a;
}

WB_HD float asin_(float x) { return atan2_(x, sqrtf((1.0f - x) * (1.0f + x))); }
WB_HD float acos_(float x) { return atan2_(sqrtf((1.0f - x) * (1.0f + x)), x); }

// f32 -> unorm8 conversion of a storage-texture write: clamp to [0,1], scale, round half up.
WB_HD uint32_t unorm8(float x) {
  if (!(x > 0.0f)) return 0u;
  if (x >= 1.0f) return 255u;
  return (uint32_t)floorf(x * 255.0f + 0.5f);
}

// IEEE binary16 -> binary32 (exact).
WB_HD float half_to_float(uint16_t h) {
  uint32_t s = (uint32_t)(h & 0x8000u) << 16;
  uint32_t e = (h >> 10) & 0x1fu;
  uint32_t m = h & 0x3ffu;
  if (e == 0u) {
    if (m == 0u) return as_f32(s);
    // subnormal half: m * 2^-24 (exact in float)
    float v = (float)m * 5.960464478e-08f;
    return (s != 0u) ? -v : v;
  }
  if (e == 31u) return as_f32(s | 0x7f800000u | (m << 13));
  return as_f32(s | ((e + 112u) << 23) | (m << 13));
}

// ------------------------------------------------------------------ vectors
struct v2 { float x, y; };
struct v3 { float x, y, z; };
struct v4 { float x, y, z, w; };

WB_HD v2 mk2(float x, float y) { v2 r; r.x = x; r.y = y; return r; }
WB_HD v3 mk3(float x, float y, float z) { v3 r; r.x = x; r.y = y; r.z = z; return r; }
WB_HD v3 mk3s(float s) { return mk3(s, s, s); }
WB_HD v4 mk4(float x, float y, float z, float w) { v4 r; r.x = x; r.y = y; r.z = z; r.w = w; return r; }
WB_HD v4 mk4(v3 a, float w) { return mk4(a.x, a.y, a.z, w); }
WB_HD v3 xyz(v4 a) { return mk3(a.x, a.y, a.z); }

WB_HD v2 operator+(v2 a, v2 b) { return mk2(a.x + b.x, a.y + b.y); }
WB_HD v2 operator-(v2 a, v2 b) { return mk2(a.x - b.x, a.y - b.y); }
WB_HD v2 operator*(v2 a, float s) { return mk2(a.x * s, a.y * s); }
WB_HD v2 operator*(v2 a, v2 b) { return mk2(a.x * b.x, a.y * b.y); }
WB_HD v2 operator/(v2 a, v2 b) { return mk2(a.x / b.x, a.y / b.y); }

WB_HD v3 operator+(v3 a, v3 b) { return mk3(a.x + b.x, a.y + b.y, a.z + b.z); }
WB_HD v3 operator-(v3 a, v3 b) { return mk3(a.x - b.x, a.y - b.y, a.z - b.z); }
WB_HD v3 operator-(v3 a) { return mk3(-a.x, -a.y, -a.z); }
WB_HD v3 operator*(v3 a, v3 b) { return mk3(a.x * b.x, a.y * b.y, a.z * b.z); }
WB_HD v3 operator*(v3 a, float s) { return mk3(a.x * s, a.y * s, a.z * s); }
WB_HD v3 operator*(float s, v3 a) { return mk3(s * a.x, s * a.y, s * a.z); }
WB_HD v3 operator/(v3 a, v3 b) { return mk3(a.x / b.x, a.y / b.y, a.z / b.z); }
WB_HD v3 operator/(v3 a, float s) { return mk3(a.x / s, a.y / s, a.z / s); }
WB_HD v3 operator/(float s, v3 a) { return mk3(s / a.x, s / a.y, s / a.z); }
WB_HD v3 operator+(v3 a, float s) { return mk3(a.x + s, a.y + s, a.z + s); }
WB_HD v3 operator-(v3 a, float s) { return mk3(a.x - s, a.y - s, a.z - s); }
WB_HD v3 operator-(float s, v3 a) { return mk3(s - a.x, s - a.y, s - a.z); }

WB_HD v4 operator+(v4 a, v4 b) { return mk4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
WB_HD v4 operator-(v4 a, v4 b) { return mk4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w); }
WB_HD v4 operator*(v4 a, float s) { return mk4(a.x * s, a.y * s, a.z * s, a.w * s); }
WB_HD v4 operator/(v4 a, float s) { return mk4(a.x / s, a.y / s, a.z / s, a.w / s); }

WB_HD float dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
WB_HD float dot2(v2 a, v2 b) { return a.x * b.x + a.y * b.y; }
WB_HD v3 cross(v3 a, v3 b) {
  return mk3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
WB_HD float length(v3 a) { return sqrtf(dot(a, a)); }
WB_HD float length(v2 a) { return sqrtf(a.x * a.x + a.y * a.y); }
WB_HD float length2(v2 a) { return sqrtf(dot2(a, a)); }
// WGSL normalize(e) = e / length(e); one reciprocal keeps the two IEEE ops correctly rounded.
WB_HD v3 normalize(v3 a) { float inv = 1.0f / sqrtf(dot(a, a)); return a * inv; }
WB_HD v3 vmin(v3 a, v3 b) { return mk3(wmin(a.x, b.x), wmin(a.y, b.y), wmin(a.z, b.z)); }
WB_HD v3 vmax(v3 a, v3 b) { return mk3(wmax(a.x, b.x), wmax(a.y, b.y), wmax(a.z, b.z)); }
WB_HD v3 vabs(v3 a) { return mk3(absf(a.x), absf(a.y), absf(a.z)); }
WB_HD v3 vmix(v3 a, v3 b, float t) { return mk3(mix(a.x, b.x, t), mix(a.y, b.y, t), mix(a.z, b.z, t)); }
WB_HD v3 vmix3(v3 a, v3 b, v3 t) { return mk3(mix(a.x, b.x, t.x), mix(a.y, b.y, t.y), mix(a.z, b.z, t.z)); }
WB_HD v4 vmix4(v4 a, v4 b, float t) {
  return mk4(mix(a.x, b.x, t), mix(a.y, b.y, t), mix(a.z, b.z, t), mix(a.w, b.w, t));
}
WB_HD v3 vsel(v3 f, v3 t, bool c) { return c ? t : f; }
WB_HD v3 vclamp(v3 x, float lo, float hi) { return mk3(clamp(x.x, lo, hi), clamp(x.y, lo, hi), clamp(x.z, lo, hi)); }
WB_HD float max_component(v3 v) { return wmax(wmax(v.x, v.y), v.z); }
WB_HD float min_component(v3 v) { return wmin(wmin(v.x, v.y), v.z); }
WB_HD v3 vpow(v3 a, float y) { return mk3(pow_(a.x, y), pow_(a.y, y), pow_(a.z, y)); }
WB_HD v3 vexp(v3 a) { return mk3(exp_(a.x), exp_(a.y), exp_(a.z)); }
WB_HD v3 vlog(v3 a) { return mk3(log_(a.x), log_(a.y), log_(a.z)); }
// reflect(e1, e2) = e1 - 2 * dot(e2, e1) * e2
WB_HD v3 reflect(v3 e1, v3 e2) { return e1 - (2.0f * dot(e2, e1)) * e2; }
// refract(e1, e2, e3): k = 1 - e3^2 (1 - dot(e2,e1)^2); 0 if k < 0 else e3 e1 - (e3 dot + sqrt k) e2
WB_HD v3 refract(v3 e1, v3 e2, float e3) {
  float d = dot(e2, e1);
  float k = 1.0f - e3 * e3 * (1.0f - d * d);
  if (k < 0.0f) return mk3s(0.0f);
  return e3 * e1 - (e3 * d + sqrtf(k)) * e2;
}

// Column-major 4x4 matrix as WGSL mat4x4f (c[i] is column i).
struct m4 { v4 c[4]; };
struct m3 { v3 c[3]; };

// m * vec4(v, w) with w in {0, 1}: sum of columns, left to right.
WB_HD v3 mul_point(const m4& m, v3 p) {
  return mk3(((m.c[0].x * p.x + m.c[1].x * p.y) + m.c[2].x * p.z) + m.c[3].x * 1.0f,
             ((m.c[0].y * p.x + m.c[1].y * p.y) + m.c[2].y * p.z) + m.c[3].y * 1.0f,
             ((m.c[0].z * p.x + m.c[1].z * p.y) + m.c[2].z * p.z) + m.c[3].z * 1.0f);
}
WB_HD v3 mul_dir(const m4& m, v3 d) {
  return mk3(((m.c[0].x * d.x + m.c[1].x * d.y) + m.c[2].x * d.z) + m.c[3].x * 0.0f,
             ((m.c[0].y * d.x + m.c[1].y * d.y) + m.c[2].y * d.z) + m.c[3].y * 0.0f,
             ((m.c[0].z * d.x + m.c[1].z * d.y) + m.c[2].z * d.z) + m.c[3].z * 0.0f);
}
// transpose(m) * vec4(v, 0): row i of the result is dot(column i, (v, 0)).
WB_HD v3 mul_transpose_dir(const m4& m, v3 d) {
  return mk3(((m.c[0].x * d.x + m.c[0].y * d.y) + m.c[0].z * d.z) + m.c[0].w * 0.0f,
             ((m.c[1].x * d.x + m.c[1].y * d.y) + m.c[1].z * d.z) + m.c[1].w * 0.0f,
             ((m.c[2].x * d.x + m.c[2].y * d.y) + m.c[2].z * d.z) + m.c[2].w * 0.0f);
}
// mat3x3f(a, b, c) * v = a*v.x + b*v.y + c*v.z
WB_HD v3 mul3(const m3& m, v3 v) {
  return mk3((m.c[0].x * v.x + m.c[1].x * v.y) + m.c[2].x * v.z,
             (m.c[0].y * v.x + m.c[1].y * v.y) + m.c[2].y * v.z,
             (m.c[0].z * v.x + m.c[1].z * v.y) + m.c[2].z * v.z);
}
// transpose(mat3x3f(a, b, c)) * v = (dot(a,v), dot(b,v), dot(c,v))
WB_HD v3 mul3t(const m3& m, v3 v) { return mk3(dot(m.c[0], v), dot(m.c[1], v), dot(m.c[2], v)); }
WB_HD m3 upper3(const m4& m) {
  m3 r; r.c[0] = xyz(m.c[0]); r.c[1] = xyz(m.c[1]); r.c[2] = xyz(m.c[2]); return r;
}
WB_HD m3 transpose3(const m3& m) {
  m3 r;
  r.c[0] = mk3(m.c[0].x, m.c[1].x, m.c[2].x);
  r.c[1] = mk3(m.c[0].y, m.c[1].y, m.c[2].y);
  r.c[2] = mk3(m.c[0].z, m.c[1].z, m.c[2].z);
  return r;
}

// PCG-RXS-M-XS 32 step of the reference's rand_pcg (shader.wgsl:146-154).
WB_HD float rand_pcg(uint32_t& state) {
  uint32_t s = state;
  state = s * 747796405u + 2891336453u;
  uint32_t word = ((s >> ((s >> 28u) + 4u)) ^ s) * 277803737u;
  word = (word >> 22u) ^ word;
  return (float)word * 2.3283064365386963e-10f;
}

// textureSampleLevel(texture_2d_array<f32>, sampler, uv, layer, 0.0) for an rgba8unorm array with
// the reference's sampler (linear min/mag filter, repeat addressing; tracer.js:1965-1968), pinned
// to FP32 arithmetic like the sky: texel (c / 255), centres at uv * size - 0.5, the two integer
// neighbours wrapped modulo the size, weights the fractional part, mixed along x then y.  A
// non-finite coordinate samples as coordinate 0 (hardware behaviour is undefined there).
// `fetch(x, y)` returns the packed rgba8 texel of the layer.
WB_HD v4 unorm8x4(uint32_t t) {
  return mk4((float)(t & 255u) / 255.0f, (float)((t >> 8) & 255u) / 255.0f, (float)((t >> 16) & 255u) / 255.0f,
             (float)(t >> 24) / 255.0f);
}
template <class Fetch>
WB_HD v4 sample_rgba8_repeat(const Fetch& fetch, uint32_t w, uint32_t h, v2 uv) {
  float fx = uv.x * (float)w - 0.5f;
  float fy = uv.y * (float)h - 0.5f;
  if (!(fx == fx) || fx > 3.0e38f || fx < -3.0e38f) fx = 0.0f;
  if (!(fy == fy) || fy > 3.0e38f || fy < -3.0e38f) fy = 0.0f;
  float x0f = floorf(fx), y0f = floorf(fy);
  float tx = fx - x0f, ty = fy - y0f;
  float mx = fmodf(x0f, (float)w), my = fmodf(y0f, (float)h);
  if (mx < 0.0f) mx += (float)w;
  if (my < 0.0f) my += (float)h;
  uint32_t xa = (uint32_t)mx, ya = (uint32_t)my;
  uint32_t xb = xa + 1u == w ? 0u : xa + 1u, yb = ya + 1u == h ? 0u : ya + 1u;
  v4 t00 = unorm8x4(fetch(xa, ya)), t10 = unorm8x4(fetch(xb, ya));
  v4 t01 = unorm8x4(fetch(xa, yb)), t11 = unorm8x4(fetch(xb, yb));
  return vmix4(vmix4(t00, t10, tx), vmix4(t01, t11, tx), ty);
}

}  // namespace wb
