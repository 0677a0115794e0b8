// Device-side path tracing for the progressive renderer: scene access, closest-hit and shadow
// traversal of the two-level BVH, analytic primitives, the Disney-style BSDF, light and
// environment sampling, and one full camera path.  Semantics follow shader.wgsl (file:line given
// per function); the arithmetic of every expression is kept in the reference's order so that
// results are reproducible bit for bit on the CPU.
//
// GPU-specific structure (all exact re-arrangements of the reference's work):
//  * hit attributes (normal, material) are evaluated once for the winning primitive instead of at
//    every closer candidate (the reference recomputes them on each update);
//  * eval_surface and pdf_surface are evaluated together, sharing their common terms;
//  * node, object and triangle records are fetched as 16-byte read-only vector loads.
#pragma once
#include <stdint.h>
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include "wgsl_builtins.h"
#include "../../include/wgpt_layout.h"
#include "wgpt_internal.h"

namespace pt {

using namespace wb;

constexpr float PI = 3.14159265359f;
constexpr float TWO_PI = 6.28318530718f;
constexpr float INFINITY_ = 65504.0f;
constexpr int STACK_SIZE = 64;

// Error bits reported through the context's device status word.
enum : uint32_t { ERR_STACK = 1u };

// Counter slots of algorithmic work (match the oracle's).
enum {
  C_PATHS = 0, C_RAYS_EXT, C_RAYS_SHADOW, C_NODES, C_CHILD_TESTS, C_TRI_TESTS, C_OBJ_VISITS,
  C_SHADE, C_ENV_NEE, C_CDF_PROBES, C_SKY_TEXELS, C_HIT_ATTR, C_NCOUNTERS = 16
};

struct DScene {
  const float4* mats; uint32_t n_mats;     // 9 x float4
  const float4* objs; uint32_t n_objs;     // 6 x float4
  const float4* tlas; uint32_t n_tlas;     // 2 x float4
  const float4* meshes; uint32_t n_meshes; // read at 80 B = 5 x float4
  const float4* bvh; uint32_t n_bvh;       // 2 x float4
  const float4* tris; uint32_t n_tris;     // 8 x float4
  const float4* planes; uint32_t n_planes; // 2 x float4
  const float4* lights; uint32_t n_lights; // 5 x float4
  const uint2* sky; uint32_t sky_w, sky_h; // rgba16f texel = 8 bytes
  const float* cdf; uint32_t n_cdf;
  const uint32_t* tex; uint32_t tex_w, tex_h;   // rgba8 texture array, one 32-bit texel per entry
  const uint2* alias;                           // sky alias table: (prob bits, alias) per texel
  int32_t bounce_limit;
  uint32_t flags;   // WGPT_HAS_* plus the wgpt::SCENE_* bits derived from the materials
};

struct DParams {
  v3 eye; uint32_t sample_number;
  v3 ray00; uint32_t width;
  v3 ray10; uint32_t height;
  v3 ray01; float exposure;
  v3 ray11; uint32_t seed;
  uint32_t sky_width, sky_height;
  float sky_total_lum, total_light_power;
  uint32_t sec_x, sec_y, sky_cdf_index;
};

template <bool COUNT>
struct Counters {
  uint32_t v[C_NCOUNTERS];
  __device__ __forceinline__ void init() {
    if (COUNT) {
#pragma unroll
      for (int i = 0; i < C_NCOUNTERS; ++i) v[i] = 0;
    }
  }
  __device__ __forceinline__ void add(int k, uint32_t n = 1) { if (COUNT) v[k] += n; }
};

static __device__ __forceinline__ bool HAS(const DScene& s, uint32_t f) { return (s.flags & f) != 0u; }
// A texture feature bit (wgpt::SCENE_*) in code instantiated with texture support (TEX); the
// untextured instantiations compile the texture paths out.
template <bool TEX>
static __device__ __forceinline__ bool HAS_TEX(const DScene& s, uint32_t f) { return TEX && HAS(s, f); }
static __device__ __forceinline__ float4 ld4(const float4* p) { return __ldg(p); }
static __device__ __forceinline__ v3 f3(float4 a) { return mk3(a.x, a.y, a.z); }
static __device__ __forceinline__ int32_t bi(float f) { return __float_as_int(f); }
static __device__ __forceinline__ uint32_t bu(float f) { return __float_as_uint(f); }

static __device__ __forceinline__ m4 load_m4(const float4* p) {
  m4 m;
  float4 a = ld4(p), b = ld4(p + 1), c = ld4(p + 2), d = ld4(p + 3);
  m.c[0] = mk4(a.x, a.y, a.z, a.w); m.c[1] = mk4(b.x, b.y, b.z, b.w);
  m.c[2] = mk4(c.x, c.y, c.z, c.w); m.c[3] = mk4(d.x, d.y, d.z, d.w);
  return m;
}

// ------------------------------------------------------------------------ materials
struct DMat {
  v3 color; float metallic, roughness, ior, specular_tint, anisotropic, aniso_rotation, sheen,
      sheen_tint, clearcoat, clearcoat_gloss, clearcoat_ior, transmission, concentration;
  v3 subsurface_tint; float subsurface; v3 emittance;
};
static __device__ __forceinline__ DMat load_mat(const DScene& s, int32_t i) {
  const float4* p = s.mats + (size_t)i * 9;
  float4 a = ld4(p), b = ld4(p + 1), c = ld4(p + 2), d = ld4(p + 3), e = ld4(p + 4), f = ld4(p + 5);
  DMat m;
  m.color = mk3(a.x, a.y, a.z); m.metallic = a.w;
  m.roughness = b.x; m.ior = b.y; m.specular_tint = b.z; m.anisotropic = b.w;
  m.aniso_rotation = c.x; m.sheen = c.y; m.sheen_tint = c.z; m.clearcoat = c.w;
  m.clearcoat_gloss = d.x; m.clearcoat_ior = d.y; m.transmission = d.z; m.concentration = d.w;
  m.subsurface_tint = mk3(e.x, e.y, e.z); m.subsurface = e.w;
  m.emittance = mk3(f.x, f.y, f.z);
  return m;
}
static __device__ __forceinline__ v3 load_mat_emittance(const DScene& s, int32_t i) {
  return f3(ld4(s.mats + (size_t)i * 9 + 5));
}

// Texture fields of a material record (words 23-35 of the 144-byte record); hp = height_params
// (normal multiplier, height multiplier, layer count, offset).
struct DMatTex { int32_t emissive, albedo, normal, height, roughness, metallic; v2 uv_scale; v4 hp; };
static __device__ __forceinline__ DMatTex load_mat_tex(const DScene& s, int32_t i) {
  const float4* p = s.mats + (size_t)i * 9;
  float4 f = ld4(p + 5), g = ld4(p + 6), h = ld4(p + 7), k = ld4(p + 8);
  DMatTex t;
  t.emissive = bi(f.w); t.albedo = bi(g.x); t.normal = bi(g.y); t.height = bi(g.z); t.roughness = bi(g.w);
  t.metallic = bi(h.x);
  t.uv_scale = mk2(h.z, h.w); t.hp = mk4(k.x, k.y, k.z, k.w);
  return t;
}

// sample_texture (shader.wgsl:170-173): layer idx of the material texture array sampled with the
// linear, repeating sampler; vec4(1) for a negative index.
static __device__ __forceinline__ v4 sample_texture(const DScene& s, int32_t idx, v2 uv) {
  if (idx < 0) return mk4(1.0f, 1.0f, 1.0f, 1.0f);
  const uint32_t w = s.tex_w;
  const uint32_t* base = s.tex + (size_t)idx * w * s.tex_h;
  auto fetch = [&](uint32_t x, uint32_t y) { return __ldg(base + (size_t)y * w + x); };
  return sample_rgba8_repeat(fetch, w, s.tex_h, uv);
}

// ------------------------------------------------------------------------ sky and env CDF
static __device__ __forceinline__ v4 sky_texel(const DScene& s, int x, int y) {
  uint2 t = __ldg(s.sky + (size_t)y * s.sky_w + x);
  __half2 lo = *reinterpret_cast<__half2*>(&t.x);
  __half2 hi = *reinterpret_cast<__half2*>(&t.y);
  float2 a = __half22float2(lo), b = __half22float2(hi);
  return mk4(a.x, a.y, b.x, b.y);
}
// Linear filter with clamp-to-edge addressing, in FP32.
template <bool COUNT>
static __device__ v3 sky_bilinear(const DScene& s, v2 uv, Counters<COUNT>& cn) {
  cn.add(C_SKY_TEXELS, 4);
  float fx = uv.x * (float)s.sky_w - 0.5f;
  float fy = uv.y * (float)s.sky_h - 0.5f;
  float x0f = floorf(fx), y0f = floorf(fy);
  float tx = fx - x0f, ty = fy - y0f;
  int x0 = (int)x0f, y0 = (int)y0f;
  int W = (int)s.sky_w, H = (int)s.sky_h;
  int xa = min(max(x0, 0), W - 1), xb = min(max(x0 + 1, 0), W - 1);
  int ya = min(max(y0, 0), H - 1), yb = min(max(y0 + 1, 0), H - 1);
  v4 t00 = sky_texel(s, xa, ya), t10 = sky_texel(s, xb, ya);
  v4 t01 = sky_texel(s, xa, yb), t11 = sky_texel(s, xb, yb);
  return xyz(vmix4(vmix4(t00, t10, tx), vmix4(t01, t11, tx), ty));
}

// shader.wgsl:176-188
template <bool COUNT>
static __device__ __noinline__ v3 sample_sky(const DScene& s, v3 dir, Counters<COUNT>& cn) {
  float phi = atan2_(dir.z, dir.x);
  float theta = asin_(clamp(dir.y, -1.0f, 1.0f));
  return sky_bilinear(s, mk2(0.5f + phi / TWO_PI, 0.5f - theta / PI), cn);
}

// shader.wgsl:192-206
template <bool COUNT>
static __device__ __forceinline__ uint32_t binary_search_cdf(const DScene& s, uint32_t offset, uint32_t size, float targ, Counters<COUNT>& cn) {
  uint32_t low = 0u, high = size;
  while (low < high) {
    uint32_t mid = low + (high - low) / 2u;
    cn.add(C_CDF_PROBES);
    float val = __ldg(s.cdf + offset + mid);
    if (val < targ) low = mid + 1u; else high = mid;
  }
  return max(1u, low) - 1u;
}

// shader.wgsl:208-229
template <bool COUNT>
static __device__ __noinline__ float get_sky_pdf(const DScene& s, const DParams& p, v3 dir, Counters<COUNT>& cn) {
  float phi = atan2_(dir.z, dir.x);
  float theta = acos_(clamp(dir.y, -1.0f, 1.0f));
  float u = (phi + PI) / (2.0f * PI);
  float v = theta / PI;
  v3 sky_color = sky_bilinear(s, mk2(u, v), cn);
  float lum = dot(sky_color, mk3(0.2126f, 0.7152f, 0.0722f));
  float sin_theta = sin_(theta);
  if (p.sky_total_lum <= 0.0f || sin_theta <= 0.0f) return 1.0f / (4.0f * PI);
  return (lum * (float)p.sky_width * (float)p.sky_height) / (p.sky_total_lum * 2.0f * PI * PI);
}

struct LightSample { v3 dir; v3 color; float dist; float pdf; };

// shader.wgsl:231-254
template <bool COUNT>
static __device__ __noinline__ LightSample sample_env_cdf(const DScene& s, const DParams& p, float ux, float uy, Counters<COUNT>& cn) {
  LightSample samp;
  uint32_t v_idx, u_idx;
  if (HAS(s, wgpt::SCENE_ENV_ALIAS)) {
    // alias table over the same texel weights: the first number picks a bin, the second keeps
    // it or takes its alias (validated on upload: probabilities in [0, 1], aliases in range)
    const uint32_t n = s.sky_w * s.sky_h;
    const uint32_t i = min((uint32_t)(ux * (float)n), n - 1u);
    const uint2 e = __ldg(s.alias + i);
    const uint32_t t = uy < __uint_as_float(e.x) ? i : e.y;
    v_idx = t / s.sky_w;
    u_idx = t - v_idx * s.sky_w;
  } else {
    v_idx = binary_search_cdf(s, 0u, p.sky_height, uy, cn);
    uint32_t row_offset = p.sky_cdf_index + (v_idx * (p.sky_width + 1u));
    u_idx = binary_search_cdf(s, row_offset, p.sky_width, ux, cn);
  }
  float u_coord = ((float)u_idx + 0.5f) / (float)p.sky_width;
  float v_coord = ((float)v_idx + 0.5f) / (float)p.sky_height;
  float theta = PI * v_coord;
  float phi = 2.0f * PI * u_coord - PI;
  float sin_theta = sin_(theta);
  samp.dir = mk3(sin_theta * cos_(phi), cos_(theta), sin_theta * sin_(phi));
  samp.color = sky_bilinear(s, mk2(u_coord, v_coord), cn);
  samp.pdf = get_sky_pdf(s, p, samp.dir, cn);
  samp.dist = INFINITY_;
  return samp;
}

// ------------------------------------------------------------------------ intersection
struct Ray { v3 origin, direction; };

// Closest hit record.  kind: 0 none, 1 plane (id = plane), 2 TLAS mesh triangle (id = triangle),
// 3 analytic TLAS object, 4 list-mesh triangle (id = triangle, aux = list index).
// tsrc/tsrc_t: the last plane (-2 - plane), sphere or cube (object index) accepted as the closest
// candidate and its distance, -1 when none was: the source of the tangent frame the reference
// leaves in SurfaceHit (triangles, cylinders and tori do not write one).
struct HitRec {
  float t; int32_t m_idx; int32_t o_idx;
  int32_t kind; int32_t id; int32_t aux;
  float bu, bv;   // barycentrics (u, v) of a triangle hit
  int32_t tsrc; float tsrc_t;
};

// shader.wgsl:256-265.  IEEE fminf/fmaxf: the sign of a zero result can differ from WGSL's
// min/max, but every consumer only compares the result, where +0 == -0.
static __device__ __forceinline__ float intersect_aabb(v3 o, v3 inv, float4 lo, float4 hi) {
  float t0x = (lo.x - o.x) * inv.x, t0y = (lo.y - o.y) * inv.y, t0z = (lo.z - o.z) * inv.z;
  float t1x = (hi.x - o.x) * inv.x, t1y = (hi.y - o.y) * inv.y, t1z = (hi.z - o.z) * inv.z;
  float t_near = fmaxf(fmaxf(fminf(t0x, t1x), fminf(t0y, t1y)), fminf(t0z, t1z));
  float t_far = fminf(fminf(fmaxf(t0x, t1x), fmaxf(t0y, t1y)), fmaxf(t0z, t1z));
  if (t_near > t_far || t_far < 0.0f) return -1.0f;
  return t_near < 0.0f ? 0.0f : t_near;
}

// shader.wgsl:267-288 (hit distance and barycentrics only)
static __device__ __forceinline__ bool intersect_triangle(const Ray& r, float4 a, float4 b, float4 c, float* t_out, float* u_out, float* v_out) {
  v3 v0 = f3(a);
  v3 edge1 = f3(b) - v0;
  v3 edge2 = f3(c) - v0;
  v3 h = cross(r.direction, edge2);
  float det = dot(edge1, h);
  if (absf(det) < 0.000001f) return false;
  float f = 1.0f / det;
  v3 sv = r.origin - v0;
  float u = f * dot(sv, h);
  if (u < 0.0f || u > 1.0f) return false;
  v3 q = cross(sv, edge1);
  float v = f * dot(r.direction, q);
  if (v < 0.0f || u + v > 1.0f) return false;
  float t = f * dot(edge2, q);
  if (t > 0.000001f) { *t_out = t; *u_out = u; *v_out = v; return true; }
  return false;
}

// shader.wgsl:290-300
static __device__ __forceinline__ float hit_unit_sphere(const Ray& r) {
  float a = dot(r.direction, r.direction);
  float half_b = dot(r.origin, r.direction);
  float cc = dot(r.origin, r.origin) - 1.0f;
  float disc = half_b * half_b - a * cc;
  if (disc < 0.0f) return -1.0f;
  float sqrtd = sqrtf(disc);
  float root = (-half_b - sqrtd) / a;
  if (root < 0.001f) root = (-half_b + sqrtd) / a;
  return root >= 0.001f ? root : -1.0f;
}

// shader.wgsl:302-312
static __device__ __forceinline__ float hit_unit_cube(const Ray& r) {
  v3 inv = 1.0f / r.direction;
  float t0x = (-1.0f - r.origin.x) * inv.x, t0y = (-1.0f - r.origin.y) * inv.y, t0z = (-1.0f - r.origin.z) * inv.z;
  float t1x = (1.0f - r.origin.x) * inv.x, t1y = (1.0f - r.origin.y) * inv.y, t1z = (1.0f - r.origin.z) * inv.z;
  float tnear = fmaxf(fmaxf(fminf(t0x, t1x), fminf(t0y, t1y)), fminf(t0z, t1z));
  float tfar = fminf(fminf(fmaxf(t0x, t1x), fmaxf(t0y, t1y)), fmaxf(t0z, t1z));
  if (tnear < tfar && tfar > 0.0f) return tnear > 0.001f ? tnear : tfar;
  return -1.0f;
}

// shader.wgsl:323-379; UV also returns the texture coordinate of the hit (side: angle and
// height, caps: planar in units of the larger diameter).
template <bool UV>
static __device__ __noinline__ bool hit_cylinder(const Ray& r, float r0, float r1, float* t_out, v3* n_out,
                                                 v2* uv_out) {
  float h = 1.0f;
  float dr = r1 - r0;
  float k = dr / h;
  float origin_eff_radius = r0 + k * r.origin.y;
  float A = r.direction.x * r.direction.x + r.direction.z * r.direction.z - k * k * r.direction.y * r.direction.y;
  float B = 2.0f * (r.origin.x * r.direction.x + r.origin.z * r.direction.z - origin_eff_radius * k * r.direction.y);
  float C = r.origin.x * r.origin.x + r.origin.z * r.origin.z - origin_eff_radius * origin_eff_radius;
  float t_min = 1e10f;
  bool hit = false;
  float disc = B * B - 4.0f * A * C;
  if (disc > 0.0f) {
    float sqrt_d = sqrtf(disc);
    float t0 = (-B - sqrt_d) / (2.0f * A);
    float t1 = (-B + sqrt_d) / (2.0f * A);
#pragma unroll
    for (int i = 0; i < 2; i++) {
      float t = i == 0 ? t0 : t1;
      float y = r.origin.y + t * r.direction.y;
      if (t > 0.001f && t < t_min && y >= 0.0f && y <= h) {
        t_min = t;
        v3 p = r.origin + t * r.direction;
        float slant = -k * (r0 + k * y);
        *n_out = normalize(mk3(p.x, slant, p.z));
        if (UV) *uv_out = mk2(atan2_(p.z, p.x) / TWO_PI + 0.5f, y);
        hit = true;
      }
    }
  }
#pragma unroll
  for (int i = 0; i < 2; i++) {
    float py = i == 0 ? 0.0f : 1.0f;
    float rad = i == 0 ? r0 : r1;
    float t = (py - r.origin.y) / r.direction.y;
    if (t > 0.001f && t < t_min) {
      v3 p = r.origin + t * r.direction;
      if (p.x * p.x + p.z * p.z <= rad * rad) {
        t_min = t;
        *n_out = mk3(0.0f, (float)i * 2.0f - 1.0f, 0.0f);
        if (UV) {
          float den = wmax(r0, r1) * 2.0f;
          *uv_out = mk2(p.x / den + 0.5f, p.z / den + 0.5f);
        }
        hit = true;
      }
    }
  }
  if (hit) *t_out = t_min;
  return hit;
}

// shader.wgsl:381-471
static __device__ __noinline__ float hit_torus(const Ray& r, float Ra, float ra) {
  float po = 1.0f;
  float Ra2 = Ra * Ra;
  float ra2 = ra * ra;
  float m = dot(r.origin, r.origin);
  float n = dot(r.origin, r.direction);
  float bounds_radius = Ra + ra;
  float h_bound = n * n - m + bounds_radius * bounds_radius;
  if (h_bound < 0.0f) return -1.0f;
  float k = (m - ra2 - Ra2) / 2.0f;
  float k3 = n;
  float k2 = n * n + Ra2 * r.direction.y * r.direction.y + k;
  float k1 = k * n + Ra2 * r.origin.y * r.direction.y;
  float k0 = k * k + Ra2 * r.origin.y * r.origin.y - Ra2 * ra2;
  float K3 = k3, K2 = k2, K1 = k1, K0 = k0;
  if (absf(k3 * (k3 * k3 - k2) + k1) < 0.01f) {
    po = -1.0f;
    float inv_k0 = 1.0f / k0;
    K1 = k3 * inv_k0;
    K2 = k2 * inv_k0;
    K3 = k1 * inv_k0;
    K0 = inv_k0;
  }
  float c2 = (2.0f * K2 - 3.0f * K3 * K3) / 3.0f;
  float c1 = 2.0f * (K3 * (K3 * K3 - K2) + K1);
  float c0 = (K3 * (K3 * (-3.0f * K3 * K3 + 4.0f * K2) - 8.0f * K1) + 4.0f * K0) / 3.0f;
  float Q = c2 * c2 + c0;
  float R = 3.0f * c0 * c2 - c2 * c2 * c2 - c1 * c1;
  float h = R * R - Q * Q * Q;
  float z;
  if (h < 0.0f) {
    float sQ = sqrtf(Q);
    z = 2.0f * sQ * cos_(acos_(clamp(R / (sQ * Q), -1.0f, 1.0f)) / 3.0f);
  } else {
    float sQ = pow_(sqrtf(h) + absf(R), 1.0f / 3.0f);
    z = sign(R) * absf(sQ + Q / sQ);
  }
  z = c2 - z;
  float d1 = z - 3.0f * c2;
  float d2 = z * z - 3.0f * c0;
  if (absf(d1) < 1.0e-4f) {
    if (d2 < 0.0f) return -1.0f;
    d2 = sqrtf(d2);
  } else {
    if (d1 < 0.0f) return -1.0f;
    d1 = sqrtf(d1 / 2.0f);
    d2 = c1 / d1;
  }
  float result = 1e20f;
  float h1 = d1 * d1 - z + d2;
  if (h1 > 0.0f) {
    h1 = sqrtf(h1);
    float t1 = -d1 - h1 - K3; if (po < 0.0f) t1 = 2.0f / t1;
    float t2 = -d1 + h1 - K3; if (po < 0.0f) t2 = 2.0f / t2;
    if (t1 > 0.001f) result = t1;
    if (t2 > 0.001f) result = wmin(result, t2);
  }
  float h2 = d1 * d1 - z - d2;
  if (h2 > 0.0f) {
    h2 = sqrtf(h2);
    float t3 = d1 - h2 - K3; if (po < 0.0f) t3 = 2.0f / t3;
    float t4 = d1 + h2 - K3; if (po < 0.0f) t4 = 2.0f / t4;
    if (t3 > 0.001f) result = wmin(result, t3);
    if (t4 > 0.001f) result = wmin(result, t4);
  }
  return result > 1e10f ? -1.0f : result;
}

// Local-space ray of an object (m * (o,1), m * (d,0)).
static __device__ __forceinline__ Ray to_local(const m4& m, const Ray& r) {
  Ray l; l.origin = mul_point(m, r.origin); l.direction = mul_dir(m, r.direction); return l;
}

// Object record fields used by traversal: inverse matrix rows and the fourth/fifth vectors.
struct ObjHdr { int32_t material_idx, light_idx, type; float param0; v3 world_position; float param1; };
static __device__ __forceinline__ ObjHdr load_obj_hdr(const DScene& s, uint32_t i) {
  float4 a = ld4(s.objs + (size_t)i * 6 + 4), b = ld4(s.objs + (size_t)i * 6 + 5);
  ObjHdr h;
  h.material_idx = bi(a.x); h.light_idx = bi(a.y); h.type = bi(a.z); h.param0 = a.w;
  h.world_position = mk3(b.x, b.y, b.z); h.param1 = b.w;
  return h;
}

// BLAS closest hit: shader.wgsl:473-542.  Updates hit if a closer triangle is found.
template <bool COUNT>
static __device__ __forceinline__ void trace_mesh(const DScene& s, const Ray& rw, const m4& inv_m, uint32_t node_offset,
                                           uint32_t tri_offset, int32_t material_idx, int32_t idx, int32_t kind,
                                           int32_t aux, HitRec& hit, uint32_t& err, Counters<COUNT>& cn) {
  Ray rl = to_local(inv_m, rw);
  v3 inv_dir = 1.0f / rl.direction;
  uint32_t stack[STACK_SIZE];
  int sp = 0;
  stack[sp++] = node_offset;
  cn.add(C_CHILD_TESTS);
  {
    const float4* rn = s.bvh + (size_t)node_offset * 2;
    float base_t = intersect_aabb(rl.origin, inv_dir, ld4(rn), ld4(rn + 1));
    if (base_t < 0.0f || base_t >= hit.t) return;
  }
  while (sp > 0) {
    cn.add(C_NODES);
    uint32_t node_idx = stack[--sp];
    const float4* np = s.bvh + (size_t)node_idx * 2;
    float4 lo = ld4(np), hi = ld4(np + 1);
    uint32_t ntri = bu(lo.w), next = bu(hi.w);
    if (ntri > 0u) {
      uint32_t start = tri_offset + next;
      uint32_t end = start + ntri;
      for (uint32_t i = start; i < end; i++) {
        const float4* tp = s.tris + (size_t)i * 8;
        float t_tri, u, v;
        cn.add(C_TRI_TESTS);
        if (intersect_triangle(rl, ld4(tp), ld4(tp + 1), ld4(tp + 2), &t_tri, &u, &v)) {
          if (t_tri >= 0.0f && t_tri < hit.t) {
            hit.t = t_tri; hit.m_idx = material_idx; hit.o_idx = idx;
            hit.kind = kind; hit.id = (int32_t)i; hit.aux = aux; hit.bu = u; hit.bv = v;
          }
        }
      }
    } else {
      uint32_t left_idx = node_idx + 1u;
      uint32_t right_idx = node_offset + next;
      const float4* lp = s.bvh + (size_t)left_idx * 2;
      const float4* rp = s.bvh + (size_t)right_idx * 2;
      cn.add(C_CHILD_TESTS, 2);
      float left_t = intersect_aabb(rl.origin, inv_dir, ld4(lp), ld4(lp + 1));
      float right_t = intersect_aabb(rl.origin, inv_dir, ld4(rp), ld4(rp + 1));
      bool push_l = left_t >= 0.0f && left_t < hit.t;
      bool push_r = right_t >= 0.0f && right_t < hit.t;
      uint32_t first = right_idx, second = left_idx;
      bool pf = push_r, ps = push_l;
      if (!(left_t < right_t)) { first = left_idx; second = right_idx; pf = push_l; ps = push_r; }
      if (pf) { if (sp < STACK_SIZE) stack[sp++] = first; else err |= ERR_STACK; }
      if (ps) { if (sp < STACK_SIZE) stack[sp++] = second; else err |= ERR_STACK; }
    }
  }
}

// Analytic TLAS objects: shader.wgsl:544-692 (hit distance only; attributes are deferred).
// Returns true when the reference would accept the candidate at world distance *t_out before the
// comparison with the current closest hit.
static __device__ __forceinline__ bool analytic_t(const m4& inv, const ObjHdr& h, const Ray& rw, float* t_out) {
  Ray rl = to_local(inv, rw);
  if (h.type == 1) { float t = hit_unit_sphere(rl); *t_out = t; return t > 0.001f; }
  if (h.type == 2) { float t = hit_unit_cube(rl); *t_out = t; return t > 0.001f; }
  if (h.type == 3) {
    float t; v3 n;
    if (hit_cylinder<false>(rl, 1.0f, h.param0, &t, &n, nullptr)) { *t_out = t; return true; }
    return false;
  }
  float ray_scale = length(rl.direction);
  rl.direction = rl.direction / ray_scale;
  float t = hit_torus(rl, 1.0f, h.param0 * 1.0f);
  if (t > 0.0f) { *t_out = t / ray_scale; return true; }
  return false;
}

// shader.wgsl:694-752 (+ trace_scene planes and list meshes, :754-774)
template <bool COUNT>
static __device__ HitRec trace_scene(const DScene& s, const Ray& ray, uint32_t& err, Counters<COUNT>& cn) {
  cn.add(C_RAYS_EXT);
  HitRec hit;
  hit.t = 1e10f; hit.m_idx = -1; hit.o_idx = -1; hit.kind = 0; hit.id = -1; hit.aux = -1; hit.bu = 0.0f; hit.bv = 0.0f;
  hit.tsrc = -1; hit.tsrc_t = 0.0f;
  if (HAS(s, WGPT_HAS_PLANES)) {
    for (uint32_t i = 0; i < s.n_planes; i++) {
      float4 a = ld4(s.planes + (size_t)i * 2);
      float4 b = ld4(s.planes + (size_t)i * 2 + 1);
      v3 pn = f3(a);
      float denom = dot(pn, ray.direction);
      float t = -1.0f;
      if (absf(denom) > 1e-6f) {
        float tt = (a.w - dot(pn, ray.origin)) / denom;
        if (tt > 0.001f) t = tt;
      }
      if (t > 0.001f && t < hit.t) {
        hit.t = t; hit.m_idx = bi(b.x); hit.kind = 1; hit.id = (int32_t)i;
        hit.tsrc = -2 - (int32_t)i; hit.tsrc_t = t;
      }
    }
  }
  if (HAS(s, WGPT_HAS_SPHERES | WGPT_HAS_CUBES | WGPT_HAS_CYLINDERS | WGPT_HAS_TORI | WGPT_HAS_MESHES)) {
    v3 inv_dir = 1.0f / ray.direction;
    uint32_t stack[STACK_SIZE];
    int sp = 0;
    stack[sp++] = 0;
    cn.add(C_CHILD_TESTS);
    float base_t = intersect_aabb(ray.origin, inv_dir, ld4(s.tlas), ld4(s.tlas + 1));
    if (!(base_t < 0.0f || base_t >= hit.t)) {
      while (sp > 0) {
        cn.add(C_NODES);
        uint32_t node_idx = stack[--sp];
        const float4* np = s.tlas + (size_t)node_idx * 2;
        float4 lo = ld4(np), hi = ld4(np + 1);
        uint32_t nobj = bu(lo.w), next = bu(hi.w);
        if (nobj > 0u) {
          for (uint32_t i = next; i < next + nobj; i++) {
            ObjHdr h = load_obj_hdr(s, i);
            cn.add(C_OBJ_VISITS);
            bool on = (h.type == 0 && HAS(s, WGPT_HAS_MESHES)) || (h.type == 1 && HAS(s, WGPT_HAS_SPHERES)) ||
                      (h.type == 2 && HAS(s, WGPT_HAS_CUBES)) || (h.type == 3 && HAS(s, WGPT_HAS_CYLINDERS)) ||
                      (h.type == 4 && HAS(s, WGPT_HAS_TORI));
            if (!on) continue;
            m4 inv = load_m4(s.objs + (size_t)i * 6);
            if (h.type == 0) {
              trace_mesh<COUNT>(s, ray, inv, bu(h.param0), bu(h.param1), h.material_idx, (int32_t)i, 2, -1, hit, err, cn);
            } else {
              float t = 0.0f;
              if (analytic_t(inv, h, ray, &t) && t < hit.t) {
                hit.t = t; hit.m_idx = h.material_idx; hit.o_idx = (int32_t)i; hit.kind = 3; hit.id = (int32_t)i;
                if (h.type <= 2) { hit.tsrc = (int32_t)i; hit.tsrc_t = t; }
              }
            }
          }
        } else {
          uint32_t left_idx = node_idx + 1u;
          uint32_t right_idx = next;
          const float4* lp = s.tlas + (size_t)left_idx * 2;
          const float4* rp = s.tlas + (size_t)right_idx * 2;
          cn.add(C_CHILD_TESTS, 2);
          float left_t = intersect_aabb(ray.origin, inv_dir, ld4(lp), ld4(lp + 1));
          float right_t = intersect_aabb(ray.origin, inv_dir, ld4(rp), ld4(rp + 1));
          bool push_l = left_t >= 0.0f && left_t < hit.t;
          bool push_r = right_t >= 0.0f && right_t < hit.t;
          uint32_t first = right_idx, second = left_idx;
          bool pf = push_r, ps = push_l;
          if (!(left_t < right_t)) { first = left_idx; second = right_idx; pf = push_l; ps = push_r; }
          if (pf) { if (sp < STACK_SIZE) stack[sp++] = first; else err |= ERR_STACK; }
          if (ps) { if (sp < STACK_SIZE) stack[sp++] = second; else err |= ERR_STACK; }
        }
      }
    }
  }
  if (HAS(s, WGPT_HAS_LIST_MESHES)) {
    for (uint32_t i = 0; i < s.n_meshes; i++) {
      const float4* mp = s.meshes + (size_t)i * 5;
      m4 inv = load_m4(mp);
      float4 e = ld4(mp + 4);
      trace_mesh<COUNT>(s, ray, inv, bu(e.z), bu(e.w), bi(e.x), -1, 4, (int32_t)i, hit, err, cn);
    }
  }
  return hit;
}

// World-space normal of the winning primitive (the hit_n the reference leaves in SurfaceHit).
static __device__ __noinline__ v3 hit_normal(const DScene& s, const Ray& rw, const HitRec& hit) {
  if (hit.kind == 1) return f3(ld4(s.planes + (size_t)hit.id * 2));
  if (hit.kind == 2 || hit.kind == 4) {
    m4 inv = hit.kind == 2 ? load_m4(s.objs + (size_t)hit.o_idx * 6) : load_m4(s.meshes + (size_t)hit.aux * 5);
    const float4* tp = s.tris + (size_t)hit.id * 8;
    float u = hit.bu, v = hit.bv;
    v3 bary = mk3(1.0f - u - v, u, v);
    v3 n0 = f3(ld4(tp + 3)), n1 = f3(ld4(tp + 4)), n2 = f3(ld4(tp + 5));
    v3 local_norm = normalize((n0 * bary.x + n1 * bary.y) + n2 * bary.z);
    return normalize(mul_transpose_dir(inv, local_norm));
  }
  // analytic object
  ObjHdr h = load_obj_hdr(s, (uint32_t)hit.o_idx);
  m4 inv = load_m4(s.objs + (size_t)hit.o_idx * 6);
  Ray rl = to_local(inv, rw);
  m3 n_mat = transpose3(upper3(inv));
  if (h.type == 1) {
    v3 local_normal = rl.origin + rl.direction * hit.t;
    return normalize(mul3(n_mat, local_normal));
  }
  if (h.type == 2) {
    v3 lh = rl.origin + rl.direction * hit.t;
    v3 d = vabs(lh);
    float max_d = max_component(d);
    v3 ln;
    if (max_d == d.x) ln = mk3(sign(lh.x), 0.0f, 0.0f);
    else if (max_d == d.y) ln = mk3(0.0f, sign(lh.y), 0.0f);
    else ln = mk3(0.0f, 0.0f, sign(lh.z));
    return normalize(mul3(n_mat, ln));
  }
  if (h.type == 3) {
    float t; v3 n = mk3s(0.0f);
    hit_cylinder<false>(rl, 1.0f, h.param0, &t, &n, nullptr);
    return normalize(mul3(n_mat, n));
  }
  // torus: the reference multiplies by mat3(inv) without the transpose (shader.wgsl:681)
  float ray_scale = length(rl.direction);
  rl.direction = rl.direction / ray_scale;
  float tl = hit_torus(rl, 1.0f, h.param0 * 1.0f);
  v3 p = rl.origin + rl.direction * tl;
  v3 ring_p = normalize(mk3(p.x, 0.0f, p.z));
  v3 local_n = normalize(p - ring_p);
  return normalize(mul3(upper3(inv), local_n));
}

// ------------------------------------------------------------------------ texture coordinates
// Tangent and bitangent of a plane with normal pn (shader.wgsl:630-633 with thresh 0.9 for the
// closest hit; 1197-1200 with 0.9999 for shadow rays).
static __device__ __forceinline__ void plane_frame(v3 pn, float thresh, v3* T, v3* B) {
  v3 tangent = absf(pn.x) > thresh ? mk3(0.0f, 0.0f, 1.0f) : mk3(1.0f, 0.0f, 0.0f);
  *T = normalize(cross(pn, tangent));
  *B = normalize(cross(pn, *T));
}

// Face frame and texture coordinate of a point on the unit cube (shader.wgsl:590-608, 907-924).
static __device__ __forceinline__ void cube_face(v3 lh, v3* lt, v3* lb, v2* uv) {
  v3 d = vabs(lh);
  float max_d = max_component(d);
  if (max_d == d.x) {
    float sg = sign(lh.x);
    *lt = mk3(0.0f, 0.0f, -sg); *lb = mk3(0.0f, 1.0f, 0.0f);
    *uv = mk2((-sg * lh.z) * 0.5f + 0.5f, lh.y * 0.5f + 0.5f);
  } else if (max_d == d.y) {
    float sg = sign(lh.y);
    *lt = mk3(1.0f, 0.0f, 0.0f); *lb = mk3(0.0f, 0.0f, sg);
    *uv = mk2(lh.x * 0.5f + 0.5f, (sg * lh.z) * 0.5f + 0.5f);
  } else {
    float sg = sign(lh.z);
    *lt = mk3(sg, 0.0f, 0.0f); *lb = mk3(0.0f, 1.0f, 0.0f);
    *uv = mk2((sg * lh.x) * 0.5f + 0.5f, lh.y * 0.5f + 0.5f);
  }
}

// Texture coordinate of a point on the unit sphere (shader.wgsl:556-558, 893-899).
static __device__ __forceinline__ v2 sphere_uv(v3 p) {
  return mk2(0.5f + atan2_(p.z, p.x) / TWO_PI, 0.5f + asin_(clamp(p.y, -1.0f, 1.0f)) / PI);
}

// Texture coordinate of a point on the torus (shader.wgsl:684-686, 1090-1094).
static __device__ __forceinline__ v2 torus_uv(v3 p) {
  float u = (atan2_(p.z, p.x) / TWO_PI) + 0.5f;
  float v = (atan2_(p.y, length2(mk2(p.x, p.z)) - 1.0f) / TWO_PI) + 0.5f;
  return mk2(u, v);
}

// The closest hit's texture coordinate (SurfaceHit.hit_uv, before the material's uv scale) and
// the tangent frame the reference leaves beside it: the frame of the candidate hit.tsrc names,
// recomputed at its distance, or zero vectors.
struct UvFrame { v2 uv; v3 T, B; };
static __device__ __noinline__ UvFrame hit_uv_frame(const DScene& s, const Ray& rw, const HitRec& hit) {
  UvFrame f;
  f.uv = mk2(0.0f, 0.0f);
  if (hit.kind == 1) {
    v3 pn = f3(ld4(s.planes + (size_t)hit.id * 2));
    v3 T, B;
    plane_frame(pn, 0.9f, &T, &B);
    v3 hp = rw.origin + rw.direction * hit.t;
    f.uv = mk2(dot(hp, T), dot(hp, B));
  } else if (hit.kind == 2 || hit.kind == 4) {
    const float4* tp = s.tris + (size_t)hit.id * 8;
    float4 a = ld4(tp + 6), b = ld4(tp + 7);
    float u = hit.bu, v = hit.bv;
    v3 bary = mk3(1.0f - u - v, u, v);
    f.uv = (mk2(a.x, a.y) * bary.x + mk2(a.z, a.w) * bary.y) + mk2(b.x, b.y) * bary.z;
  } else if (hit.kind == 3) {
    ObjHdr h = load_obj_hdr(s, (uint32_t)hit.o_idx);
    m4 inv = load_m4(s.objs + (size_t)hit.o_idx * 6);
    Ray rl = to_local(inv, rw);
    if (h.type == 1) {
      f.uv = sphere_uv(rl.origin + rl.direction * hit.t);
    } else if (h.type == 2) {
      v3 lt, lb;
      cube_face(rl.origin + rl.direction * hit.t, &lt, &lb, &f.uv);
    } else if (h.type == 3) {
      float t; v3 n;
      hit_cylinder<true>(rl, 1.0f, h.param0, &t, &n, &f.uv);
    } else {
      float ray_scale = length(rl.direction);
      rl.direction = rl.direction / ray_scale;
      float tl = hit_torus(rl, 1.0f, h.param0 * 1.0f);
      f.uv = torus_uv(rl.origin + rl.direction * tl);
    }
  }
  f.T = mk3s(0.0f);
  f.B = mk3s(0.0f);
  if (hit.tsrc <= -2) {
    plane_frame(f3(ld4(s.planes + (size_t)(-2 - hit.tsrc) * 2)), 0.9f, &f.T, &f.B);
  } else if (hit.tsrc >= 0) {
    ObjHdr h = load_obj_hdr(s, (uint32_t)hit.tsrc);
    m4 inv = load_m4(s.objs + (size_t)hit.tsrc * 6);
    Ray rl = to_local(inv, rw);
    v3 lp = rl.origin + rl.direction * hit.tsrc_t;
    v3 lt, lb;
    if (h.type == 1) {
      lt = absf(lp.y) > 0.9999f ? mk3(1.0f, 0.0f, 0.0f) : mk3(-lp.z, 0.0f, lp.x);
      lt = normalize(lt);
      lb = cross(lp, lt);
    } else {
      v2 uv;
      cube_face(lp, &lt, &lb, &uv);
    }
    m3 n_mat = transpose3(upper3(inv));
    f.T = normalize(mul3(n_mat, lt));
    f.B = normalize(mul3(n_mat, lb));
  }
  return f;
}

// ------------------------------------------------------------------------ shadow rays
// Shadow rays carry a transmittance: a surface without an albedo texture blocks completely; one
// with it lets (1 - alpha) through at every crossing and blocks once alpha exceeds 0.9999
// (evaluate_shadow_attenuation, shader.wgsl:777-811).  The crossings are taken in the
// reference's order (planes, TLAS traversal, list meshes; entry before exit), so the product
// is rounded the same way.  Without albedo textures in the scene every crossing blocks and no
// material or texture coordinate is read.
struct OccMat { int32_t albedo; v2 uv_scale; };
template <bool TEX>
static __device__ __forceinline__ OccMat occ_mat(const DScene& s, int32_t m) {
  OccMat o;
  o.albedo = -1;
  o.uv_scale = mk2(0.0f, 0.0f);
  if (HAS_TEX<TEX>(s, wgpt::SCENE_ALPHA_SHADOWS) && m >= 0) {
    float4 g = ld4(s.mats + (size_t)m * 9 + 6), h = ld4(s.mats + (size_t)m * 9 + 7);
    o.albedo = bi(g.x);
    o.uv_scale = mk2(h.z, h.w);
  }
  return o;
}
// One crossing of a textured occluder at texture coordinate uv (before the uv scale); true when
// it blocks.
static __device__ __forceinline__ bool attenuate(const DScene& s, const OccMat& m, v2 uv, float& trans) {
  v4 c = sample_texture(s, m.albedo, uv * m.uv_scale);
  trans = trans * (1.0f - c.w);
  return c.w > 0.9999f;
}
// Crossing of triangle tp at barycentrics (u, v) (trace_mesh_shadow, shader.wgsl:846-852).
static __device__ __forceinline__ bool tri_blocks(const DScene& s, const OccMat& m, const float4* tp, float u,
                                                  float v, float& trans) {
  if (m.albedo < 0) return true;
  float4 a = ld4(tp + 6), b = ld4(tp + 7);
  v3 bary = mk3(1.0f - u - v, u, v);
  v2 uv = (mk2(a.x, a.y) * bary.x + mk2(a.z, a.w) * bary.y) + mk2(b.x, b.y) * bary.z;
  return attenuate(s, m, uv, trans);
}
// Crossing of plane i (normal pn) at distance t (trace_plane_shadow, shader.wgsl:1190-1201).
template <bool TEX>
static __device__ __forceinline__ bool plane_blocks(const DScene& s, uint32_t i, v3 pn, const Ray& ray, float t,
                                                    float& trans) {
  if (!HAS_TEX<TEX>(s, wgpt::SCENE_ALPHA_SHADOWS)) return true;
  OccMat m = occ_mat<TEX>(s, bi(ld4(s.planes + (size_t)i * 2 + 1).x));
  if (m.albedo < 0) return true;
  v3 hit_pos = ray.origin + ray.direction * t;
  v3 T, B;
  plane_frame(pn, 0.9999f, &T, &B);
  return attenuate(s, m, mk2(dot(hit_pos, T), dot(hit_pos, B)), trans);
}

// BLAS shadow traversal (trace_mesh_shadow, shader.wgsl:813-872); true when blocked.
template <bool COUNT, bool TEX>
static __device__ bool mesh_shadow(const DScene& s, const Ray& rw, const m4& inv_m, uint32_t node_offset,
                                   uint32_t tri_offset, int32_t material, float target_dist, float& trans,
                                   uint32_t& err, Counters<COUNT>& cn) {
  Ray rl = to_local(inv_m, rw);
  v3 inv_dir = 1.0f / rl.direction;
  uint32_t stack[STACK_SIZE];
  int sp = 0;
  stack[sp++] = node_offset;
  cn.add(C_CHILD_TESTS);
  {
    const float4* rn = s.bvh + (size_t)node_offset * 2;
    float base_t = intersect_aabb(rl.origin, inv_dir, ld4(rn), ld4(rn + 1));
    if (base_t < 0.0f || base_t >= target_dist) return false;
  }
  const OccMat om = occ_mat<TEX>(s, material);
  while (sp > 0) {
    cn.add(C_NODES);
    uint32_t node_idx = stack[--sp];
    const float4* np = s.bvh + (size_t)node_idx * 2;
    float4 lo = ld4(np), hi = ld4(np + 1);
    uint32_t ntri = bu(lo.w), next = bu(hi.w);
    if (ntri > 0u) {
      uint32_t start = tri_offset + next;
      for (uint32_t i = start; i < start + ntri; i++) {
        const float4* tp = s.tris + (size_t)i * 8;
        float t_tri, u, v;
        cn.add(C_TRI_TESTS);
        if (intersect_triangle(rl, ld4(tp), ld4(tp + 1), ld4(tp + 2), &t_tri, &u, &v)) {
          if (t_tri >= 0.0f && t_tri < target_dist && tri_blocks(s, om, tp, u, v, trans)) return true;
        }
      }
    } else {
      uint32_t left_idx = node_idx + 1u;
      uint32_t right_idx = node_offset + next;
      const float4* lp = s.bvh + (size_t)left_idx * 2;
      const float4* rp = s.bvh + (size_t)right_idx * 2;
      cn.add(C_CHILD_TESTS, 2);
      float left_t = intersect_aabb(rl.origin, inv_dir, ld4(lp), ld4(lp + 1));
      float right_t = intersect_aabb(rl.origin, inv_dir, ld4(rp), ld4(rp + 1));
      bool push_l = left_t >= 0.0f && left_t < target_dist;
      bool push_r = right_t >= 0.0f && right_t < target_dist;
      uint32_t first = right_idx, second = left_idx;
      bool pf = push_r, ps = push_l;
      if (!(left_t < right_t)) { first = left_idx; second = right_idx; pf = push_l; ps = push_r; }
      if (pf) { if (sp < STACK_SIZE) stack[sp++] = first; else err |= ERR_STACK; }
      if (ps) { if (sp < STACK_SIZE) stack[sp++] = second; else err |= ERR_STACK; }
    }
  }
  return false;
}

// shader.wgsl:1019-1034
static __device__ __noinline__ float solve_cubic_real(float a, float b, float cc) {
  float q = (a * a - 3.0f * b) / 9.0f;
  float r = (2.0f * a * a * a - 9.0f * a * b + 27.0f * cc) / 54.0f;
  float r2 = r * r;
  float q3 = q * q * q;
  if (r2 < q3) {
    float theta = acos_(clamp(r / sqrtf(q3), -1.0f, 1.0f));
    return -2.0f * sqrtf(q) * cos_(theta / 3.0f) - a / 3.0f;
  }
  float aa = -sign(r) * pow_(absf(r) + sqrtf(r2 - q3), 1.0f / 3.0f);
  float bb = 0.0f;
  if (aa != 0.0f) bb = q / aa;
  return (aa + bb) - a / 3.0f;
}

// shader.wgsl:1037-1087
static __device__ __noinline__ void solve_quartic_real(float a, float b, float cc, float d, float roots[4]) {
  roots[0] = roots[1] = roots[2] = roots[3] = -1.0f;
  float a2 = a * a;
  float y = solve_cubic_real(-b, a * cc - 4.0f * d, 4.0f * b * d - a2 * d - cc * cc);
  float R2 = 0.25f * a2 - b + y;
  if (R2 < 0.0f) return;
  float R = sqrtf(R2);
  float D2, E2;
  if (R < 1e-6f) {
    D2 = 0.75f * a2 - 2.0f * b + 2.0f * sqrtf(y * y - 4.0f * d);
    E2 = 0.75f * a2 - 2.0f * b - 2.0f * sqrtf(y * y - 4.0f * d);
  } else {
    D2 = 0.75f * a2 - R2 - 2.0f * b + (4.0f * a * b - 8.0f * cc - a2 * a) / (4.0f * R);
    E2 = 0.75f * a2 - R2 - 2.0f * b - (4.0f * a * b - 8.0f * cc - a2 * a) / (4.0f * R);
  }
  int count = 0;
  if (D2 >= 0.0f) {
    float D = sqrtf(D2);
    roots[0] = -0.25f * a + 0.5f * R + 0.5f * D;
    roots[1] = -0.25f * a + 0.5f * R - 0.5f * D;
    count = 2;
  }
  if (E2 >= 0.0f) {
    float E = sqrtf(E2);
    float e0 = -0.25f * a - 0.5f * R + 0.5f * E;
    float e1 = -0.25f * a - 0.5f * R - 0.5f * E;
    if (count == 0) { roots[0] = e0; roots[1] = e1; } else { roots[2] = e0; roots[3] = e1; }
  }
#pragma unroll
  for (int i = 0; i < 3; i++) {
#pragma unroll
    for (int j = i + 1; j < 4; j++) {
      if (roots[i] > roots[j]) { float tmp = roots[i]; roots[i] = roots[j]; roots[j] = tmp; }
    }
  }
}

// Texture coordinate of a point on the cylinder or frustum (shader.wgsl:958-962).
static __device__ __forceinline__ v2 frustum_uv(v3 p, float r0, float r1) {
  if (p.y > 0.999f) return mk2(p.x / (r1 * 2.0f) + 0.5f, p.z / (r1 * 2.0f) + 0.5f);
  if (p.y < 0.001f) return mk2(p.x / (r0 * 2.0f) + 0.5f, p.z / (r0 * 2.0f) + 0.5f);
  return mk2(atan2_(p.z, p.x) / TWO_PI + 0.5f, p.y);
}

// Analytic shadow tests: shader.wgsl:874-905 (sphere), 926-956 (cube), 964-1016 (cylinder),
// 1096-1132 (torus).  An overlap of the object's interval with (0.001, target_dist) crosses it
// at the interval's entry and exit; true when blocked.
template <bool TEX>
static __device__ __noinline__ bool analytic_shadow(const DScene& s, const m4& inv, const ObjHdr& h, const Ray& rw,
                                                    float target_dist, float& trans) {
  Ray lr = to_local(inv, rw);
  if (h.type == 1 || h.type == 2) {
    float t1, t2;
    if (h.type == 1) {
      float a = dot(lr.direction, lr.direction);
      float half_b = dot(lr.origin, lr.direction);
      float cc = dot(lr.origin, lr.origin) - 1.0f;
      float disc = half_b * half_b - a * cc;
      if (disc < 0.0f) return false;
      float sqrtd = sqrtf(disc);
      t1 = (-half_b - sqrtd) / a;
      t2 = (-half_b + sqrtd) / a;
    } else {
      v3 inv_dir = 1.0f / lr.direction;
      v3 tn = (-1.0f - lr.origin) * inv_dir;
      v3 tf = (1.0f - lr.origin) * inv_dir;
      t1 = max_component(vmin(tn, tf));
      t2 = min_component(vmax(tn, tf));
    }
    float h1 = wmax(0.001f, t1), h2 = wmin(target_dist, t2);
    if (!(h1 < h2)) return false;
    OccMat om = occ_mat<TEX>(s, h.material_idx);
    if (om.albedo < 0) return true;
    v3 p1 = lr.origin + lr.direction * h1, p2 = lr.origin + lr.direction * h2;
    v2 uv1, uv2;
    if (h.type == 1) {
      uv1 = sphere_uv(p1);
      uv2 = sphere_uv(p2);
    } else {
      v3 lt, lb;
      cube_face(p1, &lt, &lb, &uv1);
      cube_face(p2, &lt, &lb, &uv2);
    }
    if (attenuate(s, om, uv1, trans)) return true;
    return attenuate(s, om, uv2, trans);
  }
  if (h.type == 3) {
    const Ray& r = lr;
    float top_radius = h.param0;
    float k = (top_radius - 1.0f) / 1.0f;
    float origin_eff_r = 1.0f + k * r.origin.y;
    float A = r.direction.x * r.direction.x + r.direction.z * r.direction.z - k * k * r.direction.y * r.direction.y;
    float B = 2.0f * (r.origin.x * r.direction.x + r.origin.z * r.direction.z - origin_eff_r * k * r.direction.y);
    float C = r.origin.x * r.origin.x + r.origin.z * r.origin.z - origin_eff_r * origin_eff_r;
    float h1 = 1e10f, h2 = -1e10f;
    uint32_t hit_count = 0u;
    float disc = B * B - 4.0f * A * C;
    if (disc >= 0.0f) {
      float sqrt_d = sqrtf(disc);
      float ts0 = (-B - sqrt_d) / (2.0f * A), ts1 = (-B + sqrt_d) / (2.0f * A);
#pragma unroll
      for (int i = 0; i < 2; i++) {
        float t = i == 0 ? ts0 : ts1;
        float y = r.origin.y + t * r.direction.y;
        if (y >= 0.0f && y <= 1.0f) { h1 = wmin(h1, t); h2 = wmax(h2, t); hit_count++; }
      }
    }
#pragma unroll
    for (int i = 0; i < 2; i++) {
      float cap = i == 0 ? 0.0f : 1.0f;
      float rad = i == 0 ? 1.0f : top_radius;
      float t = (cap - r.origin.y) / r.direction.y;
      v3 p = r.origin + t * r.direction;
      if (p.x * p.x + p.z * p.z <= rad * rad) { h1 = wmin(h1, t); h2 = wmax(h2, t); hit_count++; }
    }
    if (hit_count < 2u) return false;
    float final_h1 = wmax(0.001f, h1);
    float final_h2 = wmin(target_dist, h2);
    if (!(final_h1 < final_h2)) return false;
    OccMat om = occ_mat<TEX>(s, h.material_idx);
    if (om.albedo < 0) return true;
    if (attenuate(s, om, frustum_uv(r.origin + r.direction * final_h1, 1.0f, top_radius), trans)) return true;
    return attenuate(s, om, frustum_uv(r.origin + r.direction * final_h2, 1.0f, top_radius), trans);
  }
  // torus
  float ray_scale = length(lr.direction);
  lr.direction = lr.direction / ray_scale;
  float R = 1.0f, r = h.param0;
  float K = dot(lr.origin, lr.origin) + R * R - r * r;
  float G = dot(lr.origin, lr.direction);
  float B = 4.0f * G;
  float C = 2.0f * K + 4.0f * G * G - 4.0f * R * R * (1.0f - lr.direction.y * lr.direction.y);
  float D = 4.0f * K * G - 8.0f * R * R * lr.origin.y * lr.direction.y;
  float E = K * K - 4.0f * R * R * (lr.origin.x * lr.origin.x + lr.origin.z * lr.origin.z);
  float roots[4];
  solve_quartic_real(B, C, D, E, roots);
#pragma unroll
  for (int i = 0; i < 4; i += 2) {
    float t_near = roots[i], t_far = roots[i + 1];
    if (t_near < 0.0f || t_near > target_dist * ray_scale) continue;
    float h1 = wmax(0.001f, t_near) / ray_scale;
    float h2 = wmin(target_dist * ray_scale, t_far) / ray_scale;
    if (h1 < h2) {
      OccMat om = occ_mat<TEX>(s, h.material_idx);
      if (om.albedo < 0) return true;
      if (attenuate(s, om, torus_uv(lr.origin + lr.direction * (h1 * ray_scale)), trans)) return true;
      if (attenuate(s, om, torus_uv(lr.origin + lr.direction * (h2 * ray_scale)), trans)) return true;
    }
  }
  return false;
}

// shader.wgsl:1206-1229: the shadow ray's transmittance (one component of trace_scene_shadow's
// equal-component result), 0 when blocked.
template <bool COUNT, bool TEX>
static __device__ float scene_shadow(const DScene& s, const Ray& ray, int32_t target_idx, float target_dist,
                                     uint32_t& err, Counters<COUNT>& cn) {
  cn.add(C_RAYS_SHADOW);
  float trans = 1.0f;
  if (HAS(s, WGPT_HAS_PLANES)) {
    for (uint32_t i = 0; i < s.n_planes; i++) {
      float4 a = ld4(s.planes + (size_t)i * 2);
      v3 pn = f3(a);
      float denom = dot(pn, ray.direction);
      if (absf(denom) > 1e-6f) {
        float t = (a.w - dot(pn, ray.origin)) / denom;
        if (t > 0.001f && t < target_dist && plane_blocks<TEX>(s, i, pn, ray, t, trans)) return 0.0f;
      }
    }
  }
  if (HAS(s, WGPT_HAS_SPHERES | WGPT_HAS_CUBES | WGPT_HAS_CYLINDERS | WGPT_HAS_TORI | WGPT_HAS_MESHES)) {
    v3 inv_dir = 1.0f / ray.direction;
    uint32_t stack[STACK_SIZE];
    int sp = 0;
    stack[sp++] = 0u;
    while (sp > 0) {
      cn.add(C_NODES);
      uint32_t node_idx = stack[--sp];
      const float4* np = s.tlas + (size_t)node_idx * 2;
      float4 lo = ld4(np), hi = ld4(np + 1);
      uint32_t nobj = bu(lo.w), next = bu(hi.w);
      if (nobj > 0u) {
        for (uint32_t i = next; i < next + nobj; i++) {
          if ((int32_t)i == target_idx) continue;
          ObjHdr h = load_obj_hdr(s, i);
          cn.add(C_OBJ_VISITS);
          bool on = (h.type == 0 && HAS(s, WGPT_HAS_MESHES)) || (h.type == 1 && HAS(s, WGPT_HAS_SPHERES)) ||
                    (h.type == 2 && HAS(s, WGPT_HAS_CUBES)) || (h.type == 3 && HAS(s, WGPT_HAS_CYLINDERS)) ||
                    (h.type == 4 && HAS(s, WGPT_HAS_TORI));
          if (!on) continue;
          m4 inv = load_m4(s.objs + (size_t)i * 6);
          if (h.type == 0) {
            if (mesh_shadow<COUNT, TEX>(s, ray, inv, bu(h.param0), bu(h.param1), h.material_idx, target_dist, trans,
                                        err, cn))
              return 0.0f;
          } else if (analytic_shadow<TEX>(s, inv, h, ray, target_dist, trans)) {
            return 0.0f;
          }
        }
      } else {
        uint32_t left_idx = node_idx + 1u;
        uint32_t right_idx = next;
        const float4* lp = s.tlas + (size_t)left_idx * 2;
        const float4* rp = s.tlas + (size_t)right_idx * 2;
        cn.add(C_CHILD_TESTS, 2);
        float left_t = intersect_aabb(ray.origin, inv_dir, ld4(lp), ld4(lp + 1));
        float right_t = intersect_aabb(ray.origin, inv_dir, ld4(rp), ld4(rp + 1));
        bool push_l = left_t >= 0.0f && left_t < target_dist;
        bool push_r = right_t >= 0.0f && right_t < target_dist;
        uint32_t first = right_idx, second = left_idx;
        bool pf = push_r, ps = push_l;
        if (!(left_t < right_t)) { first = left_idx; second = right_idx; pf = push_l; ps = push_r; }
        if (pf) { if (sp < STACK_SIZE) stack[sp++] = first; else err |= ERR_STACK; }
        if (ps) { if (sp < STACK_SIZE) stack[sp++] = second; else err |= ERR_STACK; }
      }
    }
  }
  if (HAS(s, WGPT_HAS_LIST_MESHES)) {
    for (uint32_t i = 0; i < s.n_meshes; i++) {
      const float4* mp = s.meshes + (size_t)i * 5;
      m4 inv = load_m4(mp);
      float4 e = ld4(mp + 4);
      if (mesh_shadow<COUNT, TEX>(s, ray, inv, bu(e.z), bu(e.w), bi(e.x), target_dist, trans, err, cn)) return 0.0f;
    }
  }
  return trans;
}

// ------------------------------------------------------------------------ BSDF
struct Medium { float ior; v3 sigma; v3 emission; };
struct MediumStack { Medium media[4]; int32_t count; };
static __device__ __forceinline__ Medium air() { Medium m; m.ior = 1.0f; m.sigma = mk3s(0.0f); m.emission = mk3s(0.0f); return m; }
static __device__ __forceinline__ Medium peek_medium(const MediumStack& st) { return st.count > 0 ? st.media[st.count - 1] : air(); }
static __device__ __forceinline__ float peek_ior(const MediumStack& st) { return st.count > 0 ? st.media[st.count - 1].ior : 1.0f; }
static __device__ __forceinline__ float peek_outer_ior(const MediumStack& st) { return st.count > 1 ? st.media[st.count - 2].ior : 1.0f; }
static __device__ __forceinline__ void push_medium(MediumStack& st, const Medium& m) { if (st.count < 4) { st.media[st.count] = m; st.count += 1; } }
static __device__ __forceinline__ void pop_medium(MediumStack& st) { if (st.count > 0) st.count -= 1; }

// SurfaceContext of shader.wgsl:1393-1440: shading normal, geometric normal, albedo, alpha ...
struct SurfCtx { v3 normal; v3 surface_normal; v3 albedo; float roughness, metallic; v3 emittance; float alpha; };

// The context of an untextured material.
static __device__ __forceinline__ SurfCtx plain_context(const DMat& mat, v3 hit_n) {
  SurfCtx c;
  c.normal = hit_n; c.surface_normal = hit_n;
  c.albedo = mat.color; c.roughness = mat.roughness; c.metallic = mat.metallic; c.emittance = mat.emittance;
  c.alpha = 1.0f;
  return c;
}

// Texture state of a shading point: the material's texture fields, the frame (tangent,
// bitangent, hit normal), the texture coordinate after the uv scale and parallax shift, and the
// depth parallax mapping found (currentheight of main).
struct TexPoint { DMatTex mt; m3 tbn; v2 uv; float height; };

// calculate_pom (shader.wgsl:1237-1278).  A result that leaves through the early return keeps
// WGSL's zero initialisation (uv (0, 0), height 0), which main then uses as the coordinate.
struct PomResult { v2 uv; float height; bool hit; };
static __device__ __forceinline__ float height_depth(const DScene& s, int32_t idx, v2 uv, bool is_height_map) {
  float v = sample_texture(s, idx, uv).x;
  return is_height_map ? 1.0f - v : v;
}
static __device__ __noinline__ PomResult calculate_pom(const DScene& s, v2 initial_uv, v3 view_ts, float start_depth,
                                                       const DMatTex& mt) {
  PomResult res;
  res.uv = mk2(0.0f, 0.0f); res.height = 0.0f; res.hit = false;
  const bool is_height_map = mt.hp.y < 0.0f;
  const float scale = absf(mt.hp.y);
  const float num_layers = mt.hp.z;
  const float layer_depth = 1.0f / num_layers;
  float cur_layer = clamp(start_depth, 0.0f, 1.0f);
  v2 P = mk2(-(view_ts.x / view_ts.z), -(view_ts.y / view_ts.z)) * scale;
  v2 delta = mk2(P.x / num_layers, P.y / num_layers);
  v2 cur_uv = initial_uv - P * mt.hp.w;
  float cur_depth = height_depth(s, mt.height, cur_uv, is_height_map);
  for (int i = 0; i < 64; i++) {
    if ((float)i >= num_layers || cur_layer >= cur_depth) break;
    if (cur_layer > 1.0f || cur_layer < 0.0f) return res;
    cur_uv = cur_uv + delta;
    cur_depth = height_depth(s, mt.height, cur_uv, is_height_map);
    cur_layer += layer_depth;
  }
  v2 prev_uv = cur_uv - delta;
  float prev_depth = height_depth(s, mt.height, prev_uv, is_height_map);
  float after = cur_depth - cur_layer;
  float before = prev_depth - cur_layer + layer_depth;
  float weight = after / (after - before);
  res.uv = mk2(mix(cur_uv.x, prev_uv.x, weight), mix(cur_uv.y, prev_uv.y, weight));
  res.height = mix(cur_layer, cur_layer - layer_depth, weight);
  res.hit = true;
  return res;
}

// calculate_shadow_pom (shader.wgsl:1280-1328): marches from the parallax point toward the
// surface along light_ts; hit when the height field is above the ray (or the light is behind).
static __device__ __noinline__ PomResult calculate_shadow_pom(const DScene& s, v2 current_uv, float current_height,
                                                              v3 light_ts, const DMatTex& mt) {
  PomResult res;
  res.hit = false; res.uv = current_uv; res.height = current_height;
  if (light_ts.z <= 0.0f) { res.hit = true; return res; }
  const bool is_height_map = mt.hp.y < 0.0f;
  const float scale = absf(mt.hp.y);
  const float num_layers = mt.hp.z;
  const float layer_depth = 1.0f / num_layers;
  v2 p = (mk2(light_ts.x / light_ts.z, light_ts.y / light_ts.z) * scale) * layer_depth;
  v2 shadow_uv = current_uv;
  float shadow_depth = current_height;
  for (int i = 0; i < 32; i++) {
    if ((float)i / 2.0f >= num_layers || shadow_depth <= 0.0f) break;
    shadow_uv = shadow_uv + p;
    shadow_depth -= layer_depth;
    float map_depth = height_depth(s, mt.height, shadow_uv, is_height_map);
    if (map_depth < shadow_depth) {
      res.hit = true; res.uv = shadow_uv; res.height = map_depth;
      return res;
    }
  }
  return res;
}

// get_surface_context (shader.wgsl:1393-1440): normal map in the frame tp.tbn, albedo
// (sRGB-decoded, alpha from its fourth channel), roughness (second channel), metallic (third
// channel) and emissive maps at the coordinate uv.
static __device__ __noinline__ SurfCtx surface_context(const DScene& s, const DMat& mat, v3 hit_n, const TexPoint& tp,
                                                      v2 uv) {
  const DMatTex& mt = tp.mt;
  SurfCtx c;
  c.normal = hit_n;
  c.surface_normal = hit_n;
  if (mt.normal >= 0) {
    v4 t = sample_texture(s, mt.normal, uv);
    v3 n_map = mk3(t.x, t.y, t.z) * 2.0f - mk3s(1.0f);
    n_map = normalize(n_map * mk3(mt.hp.x, mt.hp.x, 1.0f));
    c.normal = normalize(mul3(tp.tbn, n_map));
  }
  c.albedo = mat.color;
  c.alpha = 1.0f;
  if (mt.albedo >= 0) {
    v4 t = sample_texture(s, mt.albedo, uv);
    c.alpha = t.w;
    c.albedo = c.albedo * vpow(mk3(t.x, t.y, t.z), 2.2f);
  }
  c.metallic = mat.metallic;
  c.roughness = mat.roughness;
  if (mt.roughness >= 0) c.roughness *= sample_texture(s, mt.roughness, uv).y;
  if (mt.metallic >= 0) c.metallic *= sample_texture(s, mt.metallic, uv).z;
  c.emittance = mat.emittance;
  if (mt.emissive >= 0) {
    v4 e = sample_texture(s, mt.emissive, uv);
    c.emittance = c.emittance * vpow(mk3(e.x, e.y, e.z), 2.2f);
  }
  return c;
}

// The surface context of the closest hit hn = hit_normal(...) of material hit.m_idx
// (shader.wgsl:2361-2375): texture coordinate, tangent frame and (with `parallax`, which main
// applies and gbuf_main does not) the parallax shift into *tp.
template <bool TEX>
static __device__ __forceinline__ SurfCtx hit_context(const DScene& s, const Ray& rw, const HitRec& hit,
                                                      const DMat& mat, v3 hn, TexPoint* tp, bool parallax) {
  if (!HAS_TEX<TEX>(s, wgpt::SCENE_TEXTURED)) return plain_context(mat, hn);
  UvFrame f = hit_uv_frame(s, rw, hit);
  tp->mt = load_mat_tex(s, hit.m_idx);
  tp->tbn.c[0] = f.T; tp->tbn.c[1] = f.B; tp->tbn.c[2] = hn;
  tp->uv = f.uv * tp->mt.uv_scale;
  tp->height = 0.0f;
  if (parallax && HAS(s, WGPT_HAS_HEIGHTMAPS) && tp->mt.height >= 0) {
    v3 view_ts = normalize(mul3t(tp->tbn, -rw.direction));
    if (view_ts.z > 0.0f) {
      PomResult pom = calculate_pom(s, tp->uv, view_ts, 0.0f, tp->mt);
      tp->uv = pom.uv;
      tp->height = pom.height;
    }
  }
  return surface_context(s, mat, hn, *tp, tp->uv);
}

// True when the point's height field shadows direction dir (evaluate_nee's parallax test and
// main's after sample_surface, shader.wgsl:2254-2257, 2459-2461); *uv receives the result's
// coordinate.
template <bool TEX>
static __device__ __forceinline__ bool pom_shadowed(const DScene& s, const TexPoint& tp, v3 dir, v2* uv) {
  if (!(HAS_TEX<TEX>(s, WGPT_HAS_HEIGHTMAPS) && tp.mt.height >= 0)) return false;
  PomResult r = calculate_shadow_pom(s, tp.uv, tp.height, normalize(mul3t(tp.tbn, dir)), tp.mt);
  *uv = r.uv;
  return r.hit;
}

// shader.wgsl:1700-1704
static __device__ __forceinline__ float D_GGX(float NdotH, float alpha2) {
  float denom = (NdotH * NdotH * (alpha2 - 1.0f) + 1.0f);
  return alpha2 / (PI * denom * denom + 1e-10f);
}
// shader.wgsl:1721-1733
static __device__ __forceinline__ float fresnel_dielectric(float cosThetaI, float etai, float etat) {
  float cosi = clamp(absf(cosThetaI), 0.0f, 1.0f);
  float sint = (etai / etat) * sqrtf(wmax(0.0f, 1.0f - cosi * cosi));
  if (sint >= 1.0f) return 1.0f;
  float cost = sqrtf(wmax(0.0f, 1.0f - sint * sint));
  float Rs = ((etat * cosi) - (etai * cost)) / ((etat * cosi) + (etai * cost));
  float Rp = ((etai * cosi) - (etat * cost)) / ((etai * cosi) + (etat * cost));
  return (Rs * Rs + Rp * Rp) / 2.0f;
}
// shader.wgsl:1787-1803
static __device__ __forceinline__ float G_Smith_GGX_div_NV(float NdotV, float NdotL, float alpha2) {
  float sqrt_v = sqrtf(wmax(0.0f, alpha2 + NdotV * NdotV * (1.0f - alpha2)));
  float sqrt_l = sqrtf(wmax(0.0f, alpha2 + NdotL * NdotL * (1.0f - alpha2)));
  return (2.0f * NdotL) / (NdotL * sqrt_v + NdotV * sqrt_l + 1e-10f);
}
static __device__ __forceinline__ float G_Smith_GGX_Uncorrelated_div_NV(float NdotV, float NdotL, float alpha2) {
  float lambda_v = NdotV + sqrtf(wmax(0.0f, alpha2 + NdotV * NdotV * (1.0f - alpha2)));
  float lambda_l = NdotL + sqrtf(wmax(0.0f, alpha2 + NdotL * NdotL * (1.0f - alpha2)));
  return (4.0f * NdotL) / (lambda_v * lambda_l + 1e-7f);
}
static __device__ __forceinline__ float G1_GGX_div_NV(float NdotV, float alpha2) {
  return 2.0f / (NdotV + sqrtf(wmax(0.0f, alpha2 + (1.0f - alpha2) * NdotV * NdotV)) + 1e-7f);
}

// eval_surface and pdf_surface of shader.wgsl:1831-2047 evaluated together.  Untextured
// instantiations (TEX false) have alpha 1, where the final "* ctx.alpha" is exact.
template <bool TEX>
static __device__ __noinline__ void bsdf_eval_pdf(v3 V, v3 L, const DMat& mat, const SurfCtx& ctx, const MediumStack& stack, v3* f_out, float* pdf_out) {
  bool entering = dot(ctx.normal, V) > 0.0f;
  v3 n_orient = entering ? ctx.normal : -ctx.normal;
  float dotNV = dot(n_orient, V);
  float dotNL = dot(n_orient, L);
  if (dotNV <= 0.0f) { *f_out = mk3s(0.0f); *pdf_out = 1e-7f; return; }
  float roughness_val = clamp(ctx.roughness, 0.01f, 1.0f);
  float alpha = roughness_val * roughness_val;
  float alpha2 = wmax(alpha * alpha, 1e-6f);
  float etai = peek_ior(stack);
  float etat = entering ? mat.ior : peek_outer_ior(stack);
  // shared macro-Fresnel terms (eval: F_macro_*, pdf: F_est/F_metal/F_actual)
  float F_cc = fresnel_dielectric(dotNV, 1.0f, mat.clearcoat_ior);
  float p_cc = entering ? mat.clearcoat * F_cc : 0.0f;
  float F_est_raw = fresnel_dielectric(dotNV, etai, etat);
  float F0_d = pow2c((etai - etat) / (etai + etat));
  float F_est = mix(F_est_raw, F0_d, roughness_val);
  float pw5_nv = pow_(wmax(0.0f, 1.0f - dotNV), 5.0f);
  v3 F_metal = ctx.albedo + (mk3s(1.0f) - ctx.albedo) * pw5_nv;
  v3 F_actual_m = vmix3(mk3s(F_est), F_metal, mk3s(ctx.metallic));
  float f_avg = clamp((F_actual_m.x + F_actual_m.y + F_actual_m.z) / 3.0f, 0.0f, 1.0f);
  float p_spec = (1.0f - p_cc) * f_avg;
  float p_trans = (1.0f - p_cc) * (1.0f - f_avg) * mat.transmission * (1.0f - ctx.metallic);
  float p_diff = (1.0f - p_cc) * (1.0f - f_avg) * (1.0f - mat.transmission) * (1.0f - ctx.metallic);
  v3 f = mk3s(0.0f);
  float pdf = 0.0f;
  if (dotNL > 0.0f) {
    v3 H_vec = V + L;
    v3 H = dot(H_vec, H_vec) > 1e-6f ? normalize(H_vec) : n_orient;
    float dotNH = wmax(dot(n_orient, H), 0.0f);
    float dotVH = wmax(dot(V, H), 0.0f);
    float D = D_GGX(dotNH, alpha2);
    // ---- eval
    v3 diff_col = ctx.albedo;
    if (mat.sheen > 0.0f) diff_col = diff_col + (vmix(mk3s(1.0f), ctx.albedo, mat.sheen_tint) * pw5_nv) * mat.sheen;
    if (mat.subsurface > 0.0f) diff_col = vmix(diff_col, mat.subsurface_tint, mat.subsurface);
    v3 diffuse = ((diff_col / PI) * (1.0f - ctx.metallic)) * (1.0f - mat.transmission);
    float G2_div_NV = G_Smith_GGX_div_NV(dotNV, dotNL, alpha2);
    float F_dielectric = fresnel_dielectric(dotVH, etai, etat);
    float lum = dot(ctx.albedo, mk3(0.2126f, 0.7152f, 0.0722f));
    v3 tint = lum <= 0.0f ? mk3s(1.0f) : ctx.albedo / wmax(lum, 0.0001f);
    v3 F_dielectric_tinted = vmix3(mk3s(F_dielectric), mk3s(F_dielectric) * tint, mk3s(mat.specular_tint));
    v3 F90_metal = vmix3(mk3s(1.0f), tint, mk3s(mat.specular_tint));
    v3 F_metal_h = ctx.albedo + (F90_metal - ctx.albedo) * pow_(wmax(0.0f, 1.0f - dotVH), 5.0f);
    v3 F_actual = vmix3(F_dielectric_tinted, F_metal_h, mk3s(ctx.metallic));
    v3 diffuse_cos = (diffuse * dotNL) * (mk3s(1.0f) - F_actual_m);
    float ms_factor = 1.0f + alpha * 0.4f;
    v3 specular_cos = (((F_actual * D) * G2_div_NV) / 4.0f) * ms_factor;
    v3 clearcoat_cos = mk3s(0.0f);
    float cc_attenuation = 1.0f;
    float cc_D = 0.0f, cc_alpha2 = 0.0f;
    bool need_cc = (mat.clearcoat > 0.0f && entering) || p_cc > 0.0f;
    if (need_cc) {
      float cc_roughness = clamp(1.0f - mat.clearcoat_gloss, 0.01f, 1.0f);
      float cc_alpha = cc_roughness * cc_roughness;
      cc_alpha2 = wmax(cc_alpha * cc_alpha, 1e-6f);
      cc_D = D_GGX(dotNH, cc_alpha2);
    }
    if (mat.clearcoat > 0.0f && entering) {
      float cc_G2_div_NV = G_Smith_GGX_div_NV(dotNV, dotNL, cc_alpha2);
      float cc_F = fresnel_dielectric(dotVH, 1.0f, mat.clearcoat_ior);
      clearcoat_cos = (mk3s(cc_F) * ((mat.clearcoat * cc_D) * cc_G2_div_NV)) / 4.0f;
      cc_attenuation = 1.0f - (mat.clearcoat * F_cc);
    }
    f = (diffuse_cos + specular_cos) * cc_attenuation + clearcoat_cos;
    // ---- pdf
    if (p_diff > 0.0f) pdf += p_diff * (dotNL / PI);
    if (p_spec > 0.0f) {
      float G1_div_NV = G1_GGX_div_NV(dotNV, alpha2);
      float spec_weight = p_spec;
      if (p_trans > 0.0f) {
        float cosi = clamp(dotVH, 0.0f, 1.0f);
        float sint = (etai / etat) * sqrtf(wmax(0.0f, 1.0f - cosi * cosi));
        if (sint >= 1.0f) spec_weight += p_trans;
      }
      float pdf_H = G1_div_NV * D * wmax(0.0f, dotVH);
      pdf += spec_weight * pdf_H / wmax(4.0f * dotVH, 1e-7f);
    }
    if (p_cc > 0.0f) {
      float cc_G1_div_NV = G1_GGX_div_NV(dotNV, cc_alpha2);
      float pdf_H_cc = cc_G1_div_NV * cc_D * wmax(0.0f, dotVH);
      pdf += p_cc * pdf_H_cc / wmax(4.0f * dotVH, 1e-7f);
    }
  } else if (dotNL < 0.0f && (mat.transmission > 0.0f || p_trans > 0.0f)) {
    v3 H_vec = -(etai * V + etat * L);
    v3 H = normalize(H_vec);
    if (dot(H, n_orient) < 0.0f) H = -H;
    float dotNH = wmax(dot(n_orient, H), 0.0f);
    float dotVH = dot(V, H);
    float dotLH = dot(L, H);
    if (dotVH * dotLH < 0.0f) {
      float D = D_GGX(dotNH, alpha2);
      float denom = etai * dotVH + etat * dotLH;
      if (mat.transmission > 0.0f) {
        float G2_unc_div_NV = G_Smith_GGX_Uncorrelated_div_NV(dotNV, absf(dotNL), alpha2);
        float F_dielectric = fresnel_dielectric(dotVH, etai, etat);
        float denom2 = wmax(denom * denom, 1e-7f);
        float ms_factor = 1.0f + alpha * 0.25f;
        float btdf_cos = (absf(dotVH) * absf(dotLH) * etat * etat * (1.0f - F_dielectric) * D * G2_unc_div_NV) / denom2 * ms_factor;
        float cc_attenuation = 1.0f;
        if (mat.clearcoat > 0.0f && entering) cc_attenuation = 1.0f - (mat.clearcoat * F_cc);
        v3 trans_color = mk3s(mat.transmission * (1.0f - ctx.metallic));
        f = (trans_color * btdf_cos) * cc_attenuation;
      }
      if (p_trans > 0.0f) {
        float G1_div_NV = G1_GGX_div_NV(dotNV, alpha2);
        float pdf_H = G1_div_NV * D * wmax(0.0f, dotVH);
        float dwh_dwi = (etat * etat * absf(dotLH)) / wmax(denom * denom, 1e-7f);
        pdf += p_trans * pdf_H * dwh_dwi;
      }
    }
  }
  const float alpha_c = TEX ? ctx.alpha : 1.0f;
  *f_out = f * alpha_c;
  *pdf_out = wmax(pdf, 1e-7f) * alpha_c;
}

// shader.wgsl:1806-1829
static __device__ __noinline__ v3 ImportanceSampleVNDF_GGX(float xi0, float xi1, v3 V, v3 N, float alpha_ggx) {
  v3 up = absf(N.y) > 0.999f ? mk3(0.0f, 0.0f, 1.0f) : mk3(0.0f, 1.0f, 0.0f);
  v3 T = normalize(cross(up, N));
  v3 B = cross(N, T);
  v3 V_local = mk3(dot(V, T), dot(V, B), dot(V, N));
  v3 Vh = normalize(mk3(alpha_ggx * V_local.x, alpha_ggx * V_local.y, wmax(V_local.z, 0.0f)));
  float lensq = Vh.x * Vh.x + Vh.y * Vh.y;
  v3 T1 = lensq > 0.0f ? mk3(-Vh.y, Vh.x, 0.0f) / sqrtf(wmax(lensq, 1e-7f)) : mk3(1.0f, 0.0f, 0.0f);
  v3 T2 = cross(Vh, T1);
  float r = sqrtf(xi0);
  float phi = 2.0f * PI * xi1;
  float t1 = r * cos_(phi);
  float t2 = r * sin_(phi);
  float s = 0.5f * (1.0f + Vh.z);
  float t2_mod = mix(sqrtf(wmax(0.0f, 1.0f - t1 * t1)), t2, s);
  v3 Nh_local = (t1 * T1 + t2_mod * T2) + sqrtf(wmax(0.0f, 1.0f - t1 * t1 - t2_mod * t2_mod)) * Vh;
  v3 Ne_local = normalize(mk3(alpha_ggx * Nh_local.x, alpha_ggx * Nh_local.y, wmax(0.0f, Nh_local.z)));
  return normalize((T * Ne_local.x + B * Ne_local.y) + N * Ne_local.z);
}

// shader.wgsl:1751-1763
static __device__ __noinline__ v3 ImportanceSampleCosine(float xi0, float xi1, v3 N) {
  float phi = TWO_PI * xi0;
  float cosTheta = sqrtf(clamp(xi1, 0.0f, 1.0f));
  float sinTheta = sqrtf(wmax(0.0f, 1.0f - xi1));
  v3 L_local = mk3(cos_(phi) * sinTheta, sin_(phi) * sinTheta, cosTheta);
  v3 up = absf(N.y) > 0.999f ? mk3(0.0f, 0.0f, 1.0f) : mk3(0.0f, 1.0f, 0.0f);
  v3 tangent = normalize(cross(up, N));
  v3 bitangent = cross(N, tangent);
  return normalize((tangent * L_local.x + bitangent * L_local.y) + N * L_local.z);
}

// shader.wgsl:1648-1659
static __device__ __forceinline__ float mis_weight(float pdf_a, float pdf_b) {
  if (pdf_a <= 0.0f) return 0.0f;
  float max_pdf = wmax(pdf_a, pdf_b);
  float a = pdf_a / max_pdf;
  float b = pdf_b / max_pdf;
  float a2 = a * a;
  float b2 = b * b;
  float sum = a2 + b2;
  if (sum <= 0.0f) return 0.0f;
  return a2 / sum;
}

// shader.wgsl:2177-2189
static __device__ __forceinline__ v3 clamp_firefly(v3 rad, int bounce) {
  if (bounce == 0) return rad;
  float lum = dot(rad, mk3(0.2126f, 0.7152f, 0.0722f));
  if (lum > 20.0f) return rad * (20.0f / lum);
  return rad;
}

// ------------------------------------------------------------------------ analytic lights
// shader.wgsl:1459-1464
static __device__ __forceinline__ m3 build_tangent_space(v3 N) {
  v3 a = absf(N.y) > 0.99999f ? mk3(0.0f, 0.0f, 1.0f) : mk3(0.0f, 1.0f, 0.0f);
  v3 T = normalize(cross(N, a));
  v3 B = cross(T, N);
  m3 r; r.c[0] = T; r.c[1] = B; r.c[2] = N; return r;
}

struct DLight { int32_t obj_idx; float area, power, scale; m4 matrix; };
static __device__ __forceinline__ DLight load_light(const DScene& s, uint32_t i) {
  const float4* p = s.lights + (size_t)i * 5;
  float4 a = ld4(p);
  DLight l; l.obj_idx = bi(a.x); l.area = a.y; l.power = a.z; l.scale = a.w;
  l.matrix = load_m4(p + 1);
  return l;
}

struct BoxAreas { v3 v1, v2, v3_, cen; float s1, s2, s3, a1, a2, a3, total; };
static __device__ __noinline__ BoxAreas box_areas(const DLight& light, v3 hit_pos) {
  BoxAreas b;
  b.v1 = xyz(light.matrix.c[0]); b.v2 = xyz(light.matrix.c[1]); b.v3_ = xyz(light.matrix.c[2]); b.cen = xyz(light.matrix.c[3]);
  v3 d = b.cen - hit_pos;
  b.s1 = dot(d, b.v1) < 0.0f ? 1.0f : -1.0f;
  b.s2 = dot(d, b.v2) < 0.0f ? 1.0f : -1.0f;
  b.s3 = dot(d, b.v3_) < 0.0f ? 1.0f : -1.0f;
  b.a1 = length(cross(b.v2 * 2.0f, b.v3_ * 2.0f)) * wmax(dot(normalize(-d), normalize(b.v1 * b.s1)), 0.01f);
  b.a2 = length(cross(b.v1 * 2.0f, b.v3_ * 2.0f)) * wmax(dot(normalize(-d), normalize(b.v2 * b.s2)), 0.01f);
  b.a3 = length(cross(b.v1 * 2.0f, b.v2 * 2.0f)) * wmax(dot(normalize(-d), normalize(b.v3_ * b.s3)), 0.01f);
  b.total = b.a1 + b.a2 + b.a3;
  return b;
}

// shader.wgsl:1473-1499
static __device__ __noinline__ float light_sphere_pdf(const DLight& light, v3 light_pos, v3 hit_pos, v3 dir) {
  v3 d = light_pos - hit_pos;
  float d2 = dot(d, d);
  float r2 = light.scale * light.scale;
  if (d2 <= r2) return 1.0f / (4.0f * PI);
  float tc = dot(d, dir);
  if (tc <= 0.0f) return 0.0f;
  float d_perp_sq = d2 - tc * tc;
  if (d_perp_sq > r2) return 0.0f;
  float sin_theta_max_sq = r2 / d2;
  float cos_theta_max = sqrtf(wmax(0.0f, 1.0f - sin_theta_max_sq));
  float solid_angle = TWO_PI * (1.0f - cos_theta_max);
  return 1.0f / wmax(solid_angle, 0.0001f);
}

// shader.wgsl:1501-1549
static __device__ __noinline__ LightSample sample_light_sphere(const DLight& light, v3 light_pos, v3 emit, v3 hit_pos, float xi0, float xi1) {
  v3 d = light_pos - hit_pos;
  float d2 = dot(d, d);
  float r2 = light.scale * light.scale;
  LightSample ls;
  ls.color = emit;
  if (d2 <= r2) {
    float z = 1.0f - 2.0f * xi0;
    float sin_theta = sqrtf(wmax(0.0f, 1.0f - z * z));
    float phi = TWO_PI * xi1;
    ls.dir = mk3(sin_theta * cos_(phi), sin_theta * sin_(phi), z);
    ls.dist = 0.0f;
    ls.pdf = 1.0f / (4.0f * PI);
    return ls;
  }
  float sin_theta_max_sq = r2 / d2;
  float cos_theta_max = sqrtf(wmax(0.0f, 1.0f - sin_theta_max_sq));
  float cos_theta = 1.0f - xi0 * (1.0f - cos_theta_max);
  float sin_theta = sqrtf(wmax(0.0f, 1.0f - cos_theta * cos_theta));
  float phi = TWO_PI * xi1;
  v3 local_dir = mk3(sin_theta * cos_(phi), sin_theta * sin_(phi), cos_theta);
  v3 w = normalize(d);
  m3 tbn = build_tangent_space(w);
  ls.dir = normalize(mul3(tbn, local_dir));
  float tc = dot(d, ls.dir);
  float d_perp_sq = d2 - tc * tc;
  float t_c = sqrtf(wmax(0.0f, r2 - d_perp_sq));
  ls.dist = tc - t_c;
  float solid_angle = TWO_PI * (1.0f - cos_theta_max);
  ls.pdf = 1.0f / wmax(solid_angle, 0.0001f);
  return ls;
}

// shader.wgsl:1575-1624 (the face pick draws one more random number)
static __device__ __noinline__ LightSample sample_light_box(const DLight& light, v3 emit, v3 hit_pos, float xi0, float xi1, uint32_t& rng) {
  BoxAreas b = box_areas(light, hit_pos);
  v3 p = b.cen;
  v3 n;
  float u = xi0 * 2.0f - 1.0f;
  float v = xi1 * 2.0f - 1.0f;
  float pick = rand_pcg(rng) * b.total;
  if (pick < b.a1) { p = p + ((b.v1 * b.s1 + b.v2 * u) + b.v3_ * v); n = normalize(b.v1 * b.s1); }
  else if (pick < b.a1 + b.a2) { p = p + ((b.v2 * b.s2 + b.v1 * u) + b.v3_ * v); n = normalize(b.v2 * b.s2); }
  else { p = p + ((b.v3_ * b.s3 + b.v1 * u) + b.v2 * v); n = normalize(b.v3_ * b.s3); }
  LightSample ls;
  v3 delta = p - hit_pos;
  float dist_sq = dot(delta, delta);
  ls.dist = sqrtf(dist_sq);
  ls.dir = delta / ls.dist;
  float cos_l = wmax(dot(-ls.dir, n), 1e-6f);
  ls.pdf = dist_sq / (b.total * cos_l);
  ls.color = emit;
  return ls;
}

}  // namespace pt
