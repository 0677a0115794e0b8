// ORACLE -- test infrastructure only.  A scalar CPU restatement of the reference's WGSL shaders,
// used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as the checker for the
// CUDA path.  It is never part of the product: the library under webgpuraytracer_b200/ does not
// link, load or call it.
//
// Follows, function by function:
//   shader.wgsl   main (2273-2492), gbuf_main (2510-2603) and every helper they reach (14-2271)
//   denoiser.wgsl prepass_main (55-112), atrous_main (117-189), composite_main (194-213)
//   scale.wgsl    main (6-35)
// Built-in functions (sin, exp, pow, normalize, mix, ...) come from wgsl_builtins.h, the shared
// single-precision restatement of WGSL's built-ins, so that this file and the CUDA kernels agree
// bit for bit; everything above the built-ins is written here independently of the kernels.
// Parity is unpinned by the reference itself (it ships no tests, golden images or known-answer
// vectors and its WGSL cannot run without a graphics stack).
//
// Textures (bindings 11/12) are sampled by wgsl_builtins.h's pinned FP32 bilinear, repeating
// sampler (the WebGPU sampler's precision is implementation-defined).
#include <stdint.h>
#include <string.h>
#include <math.h>
#include <vector>
#include <atomic>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/wgpt_layout.h"
#include "../webgpuraytracer_b200/csrc/wgsl_builtins.h"

using namespace wb;

namespace {

const float PI = 3.14159265359f;     // shader.wgsl:14
const float TWO_PI = 6.28318530718f; // shader.wgsl:15
const float INFINITY_ = 65504.0f;    // shader.wgsl:16
const int STACK_SIZE = 64;           // shader.wgsl:17

struct Scene {
  const wgpt_material* mats; uint32_t n_mats;
  const wgpt_object* objs; uint32_t n_objs;
  const wgpt_bvh_node* tlas; uint32_t n_tlas;
  const uint8_t* meshes; uint32_t n_meshes;      // read at the 80-byte WGSL stride
  const wgpt_bvh_node* bvh; uint32_t n_bvh;
  const wgpt_triangle* tris; uint32_t n_tris;
  const wgpt_plane* planes; uint32_t n_planes;
  const wgpt_light* lights; uint32_t n_lights;
  const uint16_t* sky; uint32_t sky_w, sky_h;    // rgba16float texels
  const float* cdf; uint32_t n_cdf;
  const uint8_t* tex; uint32_t tex_w, tex_h, tex_layers;   // texture_list, rgba8, layer-major
  int32_t bounce_limit;
  uint32_t flags;
};

// Counters of algorithmic work (the units of the roofline numerator).
enum {
  C_PATHS = 0, C_RAYS_EXT, C_RAYS_SHADOW, C_NODES, C_CHILD_TESTS, C_TRI_TESTS, C_OBJ_VISITS,
  C_SHADE, C_ENV_NEE, C_CDF_PROBES, C_SKY_TEXELS, C_HIT_ATTR, C_NCOUNTERS = 16
};

struct Ctx {
  const Scene* s;
  const wgpt_scene_params* p;
  uint32_t rng;
  uint64_t* cnt;   // per-thread counters or null
  int err;
  double* acc64 = nullptr;   // per-pixel FP64 Welford records (8 doubles) or null
  inline void count(int k, uint64_t v = 1) { if (cnt) cnt[k] += v; }
};

inline bool HAS(const Scene* s, uint32_t f) { return (s->flags & f) != 0u; }

// --------------------------------------------------------------------------------- data access
struct Mat4 { m4 m; };
inline m4 load_m4(const float* f) {
  m4 r;
  for (int c = 0; c < 4; ++c) r.c[c] = mk4(f[c * 4 + 0], f[c * 4 + 1], f[c * 4 + 2], f[c * 4 + 3]);
  return r;
}
inline v3 L3(const float* f) { return mk3(f[0], f[1], f[2]); }
inline v2 L2(const float* f) { return mk2(f[0], f[1]); }

struct MeshInstance { m4 inv_matrix; int32_t material_idx; uint32_t node_offset, tri_offset; };

inline MeshInstance mesh_from_object(const wgpt_object& o) {
  MeshInstance m;
  m.inv_matrix = load_m4(o.inv_matrix);
  m.material_idx = o.material_idx;
  m.node_offset = as_u32(o.param0);
  m.tri_offset = as_u32(o.param1);
  return m;
}
inline MeshInstance mesh_from_list(const Scene* s, uint32_t i) {
  wgpt_mesh_instance mi;
  memcpy(&mi, s->meshes + (size_t)i * WGPT_STRIDE_MESH_READ, sizeof(mi));
  MeshInstance m;
  m.inv_matrix = load_m4(mi.inv_matrix);
  m.material_idx = mi.material_idx;
  m.node_offset = mi.node_offset;
  m.tri_offset = mi.tri_offset;
  return m;
}

// ------------------------------------------------------------------------ textures and sky
// textureSampleLevel(skyTex, linear, clamp-to-edge) restated as an FP32 bilinear filter.
v4 sky_texel(const Scene* s, int x, int y) {
  const uint16_t* t = s->sky + ((size_t)y * s->sky_w + (size_t)x) * 4;
  return mk4(half_to_float(t[0]), half_to_float(t[1]), half_to_float(t[2]), half_to_float(t[3]));
}
v3 sky_bilinear(Ctx& c, v2 uv) {
  const Scene* s = c.s;
  c.count(C_SKY_TEXELS, 4);
  float fx = uv.x * (float)s->sky_w - 0.5f;
  float fy = uv.y * (float)s->sky_h - 0.5f;
  float x0f = floorf(fx), y0f = floorf(fy);
  float tx = fx - x0f, ty = fy - y0f;
  int x0 = (int)x0f, y0 = (int)y0f;
  int W = (int)s->sky_w, H = (int)s->sky_h;
  int xa = x0 < 0 ? 0 : (x0 > W - 1 ? W - 1 : x0);
  int xb = x0 + 1 < 0 ? 0 : (x0 + 1 > W - 1 ? W - 1 : x0 + 1);
  int ya = y0 < 0 ? 0 : (y0 > H - 1 ? H - 1 : y0);
  int yb = y0 + 1 < 0 ? 0 : (y0 + 1 > H - 1 ? H - 1 : y0 + 1);
  v4 t00 = sky_texel(s, xa, ya), t10 = sky_texel(s, xb, ya);
  v4 t01 = sky_texel(s, xa, yb), t11 = sky_texel(s, xb, yb);
  v4 r = vmix4(vmix4(t00, t10, tx), vmix4(t01, t11, tx), ty);
  return xyz(r);
}

// shader.wgsl:176-188
// sample_texture (shader.wgsl:170-173): layer idx of texture_list, vec4(1) for a negative index.
v4 sample_texture(const Scene* s, int32_t idx, v2 uv) {
  if (idx < 0) return mk4(1.0f, 1.0f, 1.0f, 1.0f);
  const uint8_t* base = s->tex + (size_t)idx * s->tex_w * s->tex_h * 4;
  const uint32_t w = s->tex_w;
  auto fetch = [&](uint32_t x, uint32_t y) {
    const uint8_t* t = base + ((size_t)y * w + x) * 4;
    return (uint32_t)t[0] | ((uint32_t)t[1] << 8) | ((uint32_t)t[2] << 16) | ((uint32_t)t[3] << 24);
  };
  return sample_rgba8_repeat(fetch, s->tex_w, s->tex_h, uv);
}

v3 sample_sky(Ctx& c, v3 dir) {
  float phi = atan2_(dir.z, dir.x);
  float theta = asin_(clamp(dir.y, -1.0f, 1.0f));
  float u = 0.5f + phi / TWO_PI;
  float v = 0.5f - theta / PI;
  return sky_bilinear(c, mk2(u, v));
}

// shader.wgsl:192-206
uint32_t binary_search_cdf(Ctx& c, uint32_t offset, uint32_t size, float targ) {
  uint32_t low = 0u, high = size;
  while (low < high) {
    uint32_t mid = low + (high - low) / 2u;
    c.count(C_CDF_PROBES);
    float val = c.s->cdf[offset + mid];
    if (val < targ) low = mid + 1u; else high = mid;
  }
  return (low > 1u ? low : 1u) - 1u;
}

// shader.wgsl:208-229
float get_sky_pdf(Ctx& c, v3 dir) {
  float phi = atan2_(dir.z, dir.x);
  float theta = acos_(clamp(dir.y, -1.0f, 1.0f));
  float u = (phi + PI) / (2.0f * PI);
  float v = theta / PI;
  v3 sky_color = sky_bilinear(c, mk2(u, v));
  float lum = dot(sky_color, mk3(0.2126f, 0.7152f, 0.0722f));
  float sin_theta = sin_(theta);
  if (c.p->sky_total_lum <= 0.0f || sin_theta <= 0.0f) return 1.0f / (4.0f * PI);
  float pdf = (lum * (float)c.p->sky_width * (float)c.p->sky_height) /
              (c.p->sky_total_lum * 2.0f * PI * PI);
  return pdf;
}

struct LightSample { v3 dir; v3 color; float dist; float pdf; };

// shader.wgsl:231-254
LightSample sample_env_cdf(Ctx& c, v2 u) {
  LightSample samp;
  uint32_t v_idx = binary_search_cdf(c, 0u, c.p->sky_height, u.y);
  uint32_t row_offset = c.p->sky_cdf_index + (v_idx * (c.p->sky_width + 1u));
  uint32_t u_idx = binary_search_cdf(c, row_offset, c.p->sky_width, u.x);
  float u_coord = ((float)u_idx + 0.5f) / (float)c.p->sky_width;
  float v_coord = ((float)v_idx + 0.5f) / (float)c.p->sky_height;
  float theta = PI * v_coord;
  float phi = 2.0f * PI * u_coord - PI;
  float sin_theta = sin_(theta);
  samp.dir = mk3(sin_theta * cos_(phi), cos_(theta), sin_theta * sin_(phi));
  samp.color = sky_bilinear(c, mk2(u_coord, v_coord));
  samp.pdf = get_sky_pdf(c, samp.dir);
  samp.dist = INFINITY_;
  return samp;
}

// ------------------------------------------------------------------------ intersection
struct Ray { v3 origin, direction; };

struct SurfaceHit {
  float t; int32_t m_idx;
  v3 hit_p, hit_n; v2 hit_uv;
  v3 tangent, bitangent;
  int32_t o_idx; int32_t count;
  int32_t prim;   // global triangle index of a mesh hit (-1 otherwise); not part of the WGSL
};

// shader.wgsl:256-265
float intersect_aabb(v3 origin, v3 inv_dir, v3 mn, v3 mx) {
  v3 t0 = (mn - origin) * inv_dir;
  v3 t1 = (mx - origin) * inv_dir;
  v3 tmin = vmin(t0, t1);
  v3 tmax = vmax(t0, t1);
  float t_near = max_component(tmin);
  float t_far = min_component(tmax);
  if (t_near > t_far || t_far < 0.0f) return -1.0f;
  return sel(t_near, 0.0f, t_near < 0.0f);
}

// shader.wgsl:267-288
bool intersect_triangle(const Ray& ray, const wgpt_triangle& tri, float* hit_t, v2* hit_uv, v3* bary) {
  v3 v0 = L3(tri.v0), v1 = L3(tri.v1), v2_ = L3(tri.v2);
  v3 edge1 = v1 - v0;
  v3 edge2 = v2_ - v0;
  v3 h = cross(ray.direction, edge2);
  float a = dot(edge1, h);
  if (absf(a) < 0.000001f) return false;
  float f = 1.0f / a;
  v3 s = ray.origin - v0;
  float u = f * dot(s, h);
  if (u < 0.0f || u > 1.0f) return false;
  v3 q = cross(s, edge1);
  float v = f * dot(ray.direction, q);
  if (v < 0.0f || u + v > 1.0f) return false;
  float t = f * dot(edge2, q);
  if (t > 0.000001f) {
    *hit_t = t;
    *bary = mk3(1.0f - u - v, u, v);
    v2 uv0 = mk2(tri.uv0[0], tri.uv0[1]), uv1 = mk2(tri.uv1[0], tri.uv1[1]), uv2 = mk2(tri.uv2[0], tri.uv2[1]);
    *hit_uv = (uv0 * bary->x + uv1 * bary->y) + uv2 * bary->z;
    return true;
  }
  return false;
}

// shader.wgsl:290-300
float hit_unit_sphere(const Ray& r) {
  float a = dot(r.direction, r.direction);
  float half_b = dot(r.origin, r.direction);
  float cc = dot(r.origin, r.origin) - 1.0f;
  float discriminant = half_b * half_b - a * cc;
  if (discriminant < 0.0f) return -1.0f;
  float sqrtd = sqrtf(discriminant);
  float root = (-half_b - sqrtd) / a;
  if (root < 0.001f) root = (-half_b + sqrtd) / a;
  return sel(-1.0f, root, root >= 0.001f);
}

// shader.wgsl:302-312
float hit_unit_cube(const Ray& r) {
  v3 inv_dir = 1.0f / r.direction;
  v3 t0 = (-1.0f - r.origin) * inv_dir;
  v3 t1 = (1.0f - r.origin) * inv_dir;
  v3 tmin = vmin(t0, t1);
  v3 tmax = vmax(t0, t1);
  float tnear = max_component(tmin);
  float tfar = min_component(tmax);
  if (tnear < tfar && tfar > 0.0f) return sel(tfar, tnear, tnear > 0.001f);
  return -1.0f;
}

// shader.wgsl:314-321
float hit_plane(v3 normal, float d, const Ray& r) {
  float denom = dot(normal, r.direction);
  if (absf(denom) > 1e-6f) {
    float t = (d - dot(normal, r.origin)) / denom;
    if (t > 0.001f) return t;
  }
  return -1.0f;
}

// shader.wgsl:323-379
bool hit_cylinder(const Ray& r, float r0, float r1, float* t_out, v3* n_out, v2* uv_out) {
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
    float ts[2] = {(-B - sqrt_d) / (2.0f * A), (-B + sqrt_d) / (2.0f * A)};
    for (int i = 0; i < 2; i++) {
      float t = ts[i];
      float y = r.origin.y + t * r.direction.y;
      if (t > 0.001f && t < t_min && y >= 0.0f && y <= h) {
        t_min = t;
        v3 p = r.origin + t * r.direction;
        float slant = -k * (r0 + k * y);
        *n_out = normalize(mk3(p.x, slant, p.z));
        *uv_out = mk2(atan2_(p.z, p.x) / TWO_PI + 0.5f, y);
        hit = true;
      }
    }
  }
  const float caps[2] = {0.0f, 1.0f};
  const float radii[2] = {r0, r1};
  for (int i = 0; i < 2; i++) {
    float py = caps[i];
    float t = (py - r.origin.y) / r.direction.y;
    if (t > 0.001f && t < t_min) {
      v3 p = r.origin + t * r.direction;
      if (p.x * p.x + p.z * p.z <= radii[i] * radii[i]) {
        t_min = t;
        *n_out = mk3(0.0f, (float)i * 2.0f - 1.0f, 0.0f);
        float den = wmax(r0, r1) * 2.0f;
        *uv_out = mk2(p.x / den + 0.5f, p.z / den + 0.5f);
        hit = true;
      }
    }
  }
  if (hit) *t_out = t_min;
  return hit;
}

// shader.wgsl:381-471
float hit_torus(const Ray& r, float Ra, float ra) {
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
  float z = 0.0f;
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
  return sel(result, -1.0f, result > 1e10f);
}

// shader.wgsl:473-542
void trace_mesh(Ctx& c, const Ray& ray_world, const MeshInstance& mesh, SurfaceHit* hit, int32_t idx) {
  const Scene* s = c.s;
  Ray ray_local;
  ray_local.origin = mul_point(mesh.inv_matrix, ray_world.origin);
  ray_local.direction = mul_dir(mesh.inv_matrix, ray_world.direction);
  v3 inv_dir = 1.0f / ray_local.direction;
  uint32_t stack[STACK_SIZE];
  int32_t stack_ptr = 0;
  stack[0] = mesh.node_offset;
  stack_ptr++;
  const wgpt_bvh_node& root = s->bvh[mesh.node_offset];
  c.count(C_CHILD_TESTS);
  float base_t = intersect_aabb(ray_local.origin, inv_dir, L3(root.aabb_min), L3(root.aabb_max));
  if (base_t < 0.0f || base_t >= hit->t) return;
  while (stack_ptr > 0) {
    hit->count++;
    c.count(C_NODES);
    stack_ptr--;
    uint32_t node_idx = stack[stack_ptr];
    const wgpt_bvh_node& node = s->bvh[node_idx];
    if (node.num_triangles > 0u) {
      uint32_t start = mesh.tri_offset + node.next;
      uint32_t end = start + node.num_triangles;
      for (uint32_t i = start; i < end; i++) {
        const wgpt_triangle& tri = s->tris[i];
        float t_tri = 0.0f; v2 uv_tri = mk2(0.0f, 0.0f); v3 bary = mk3s(0.0f);
        c.count(C_TRI_TESTS);
        if (intersect_triangle(ray_local, tri, &t_tri, &uv_tri, &bary)) {
          if (t_tri >= 0.0f && t_tri < hit->t) {
            hit->t = t_tri;
            hit->m_idx = mesh.material_idx;
            v3 local_norm = normalize((L3(tri.n0) * bary.x + L3(tri.n1) * bary.y) + L3(tri.n2) * bary.z);
            hit->hit_p = ray_world.origin + ray_world.direction * t_tri;
            v3 world_norm = mul_transpose_dir(mesh.inv_matrix, local_norm);
            hit->hit_n = normalize(world_norm);
            hit->hit_uv = uv_tri;
            hit->o_idx = idx;
            hit->prim = (int32_t)i;
          }
        }
      }
    } else {
      uint32_t left_idx = node_idx + 1u;
      uint32_t right_idx = mesh.node_offset + node.next;
      const wgpt_bvh_node& ln = s->bvh[left_idx];
      const wgpt_bvh_node& rn = s->bvh[right_idx];
      c.count(C_CHILD_TESTS, 2);
      float left_t = intersect_aabb(ray_local.origin, inv_dir, L3(ln.aabb_min), L3(ln.aabb_max));
      float right_t = intersect_aabb(ray_local.origin, inv_dir, L3(rn.aabb_min), L3(rn.aabb_max));
      if (left_t < right_t) {
        if (right_t >= 0.0f && right_t < hit->t && stack_ptr < STACK_SIZE) stack[stack_ptr++] = right_idx; else if (right_t >= 0.0f && right_t < hit->t) c.err |= 1;
        if (left_t >= 0.0f && left_t < hit->t && stack_ptr < STACK_SIZE) stack[stack_ptr++] = left_idx; else if (left_t >= 0.0f && left_t < hit->t) c.err |= 1;
      } else {
        if (left_t >= 0.0f && left_t < hit->t && stack_ptr < STACK_SIZE) stack[stack_ptr++] = left_idx; else if (left_t >= 0.0f && left_t < hit->t) c.err |= 1;
        if (right_t >= 0.0f && right_t < hit->t && stack_ptr < STACK_SIZE) stack[stack_ptr++] = right_idx; else if (right_t >= 0.0f && right_t < hit->t) c.err |= 1;
      }
    }
  }
}

// shader.wgsl:544-575
void trace_sphere(const Ray& ray_world, const wgpt_object& so, SurfaceHit* hit, int32_t idx) {
  m4 inv = load_m4(so.inv_matrix);
  Ray local_ray;
  local_ray.origin = mul_point(inv, ray_world.origin);
  local_ray.direction = mul_dir(inv, ray_world.direction);
  float t = hit_unit_sphere(local_ray);
  if (t > 0.001f && t < hit->t) {
    hit->t = t;
    hit->m_idx = so.material_idx;
    v3 local_normal = local_ray.origin + local_ray.direction * t;
    float phi = atan2_(local_normal.z, local_normal.x);
    float theta = asin_(clamp(local_normal.y, -1.0f, 1.0f));
    hit->hit_uv = mk2(0.5f + phi / TWO_PI, 0.5f + theta / PI);
    v3 local_t = mk3(-local_normal.z, 0.0f, local_normal.x);
    if (absf(local_normal.y) > 0.9999f) local_t = mk3(1.0f, 0.0f, 0.0f);
    local_t = normalize(local_t);
    v3 local_b = cross(local_normal, local_t);
    m3 n_mat = transpose3(upper3(inv));
    hit->hit_n = normalize(mul3(n_mat, local_normal));
    hit->tangent = normalize(mul3(n_mat, local_t));
    hit->bitangent = normalize(mul3(n_mat, local_b));
    hit->hit_p = ray_world.origin + ray_world.direction * t;
    hit->o_idx = idx;
    hit->prim = -1;
  }
}

// shader.wgsl:577-620
void trace_cube(const Ray& ray_world, const wgpt_object& co, SurfaceHit* hit, int32_t idx) {
  m4 inv = load_m4(co.inv_matrix);
  Ray local_ray;
  local_ray.origin = mul_point(inv, ray_world.origin);
  local_ray.direction = mul_dir(inv, ray_world.direction);
  float t = hit_unit_cube(local_ray);
  if (t > 0.001f && t < hit->t) {
    hit->t = t;
    hit->m_idx = co.material_idx;
    v3 local_hit = local_ray.origin + local_ray.direction * t;
    v3 d = vabs(local_hit);
    float max_d = max_component(d);
    v3 local_n, local_t, local_b;
    if (max_d == d.x) {
      float s = sign(local_hit.x);
      local_n = mk3(s, 0.0f, 0.0f); local_t = mk3(0.0f, 0.0f, -s); local_b = mk3(0.0f, 1.0f, 0.0f);
      hit->hit_uv = mk2((-s * local_hit.z) * 0.5f + 0.5f, local_hit.y * 0.5f + 0.5f);
    } else if (max_d == d.y) {
      float s = sign(local_hit.y);
      local_n = mk3(0.0f, s, 0.0f); local_t = mk3(1.0f, 0.0f, 0.0f); local_b = mk3(0.0f, 0.0f, s);
      hit->hit_uv = mk2(local_hit.x * 0.5f + 0.5f, (s * local_hit.z) * 0.5f + 0.5f);
    } else {
      float s = sign(local_hit.z);
      local_n = mk3(0.0f, 0.0f, s); local_t = mk3(s, 0.0f, 0.0f); local_b = mk3(0.0f, 1.0f, 0.0f);
      hit->hit_uv = mk2((s * local_hit.x) * 0.5f + 0.5f, local_hit.y * 0.5f + 0.5f);
    }
    m3 n_mat = transpose3(upper3(inv));
    hit->hit_n = normalize(mul3(n_mat, local_n));
    hit->tangent = normalize(mul3(n_mat, local_t));
    hit->bitangent = normalize(mul3(n_mat, local_b));
    hit->hit_p = ray_world.origin + ray_world.direction * t;
    hit->o_idx = idx;
    hit->prim = -1;
  }
}

// shader.wgsl:622-636
void trace_plane(const Ray& ray_world, const wgpt_plane& p, SurfaceHit* hit) {
  v3 pn = L3(p.normal);
  float t = hit_plane(pn, p.d, ray_world);
  if (t > 0.001f && t < hit->t) {
    hit->t = t;
    hit->m_idx = p.material_idx;
    hit->hit_n = pn;
    hit->hit_p = ray_world.origin + ray_world.direction * t;
    v3 tangent = mk3(1.0f, 0.0f, 0.0f);
    if (absf(hit->hit_n.x) > 0.9f) tangent = mk3(0.0f, 0.0f, 1.0f);
    hit->tangent = normalize(cross(hit->hit_n, tangent));
    hit->bitangent = normalize(cross(hit->hit_n, hit->tangent));
    hit->hit_uv = mk2(dot(hit->hit_p, hit->tangent), dot(hit->hit_p, hit->bitangent));
    hit->prim = -1;
    // o_idx is not written by trace_plane (shader.wgsl:622-636)
  }
}

// shader.wgsl:638-656
void trace_cylinder(const Ray& ray_world, const wgpt_object& f, SurfaceHit* hit, int32_t idx) {
  m4 inv = load_m4(f.inv_matrix);
  Ray local_ray;
  local_ray.origin = mul_point(inv, ray_world.origin);
  local_ray.direction = mul_dir(inv, ray_world.direction);
  float t = 0.0f; v3 n = mk3s(0.0f); v2 uv = mk2(0.0f, 0.0f);
  if (hit_cylinder(local_ray, 1.0f, f.param0, &t, &n, &uv)) {
    if (t < hit->t) {
      hit->t = t;
      hit->m_idx = f.material_idx;
      hit->hit_uv = uv;
      m3 n_mat = transpose3(upper3(inv));
      hit->hit_n = normalize(mul3(n_mat, n));
      hit->hit_p = ray_world.origin + ray_world.direction * t;
      hit->o_idx = idx;
      hit->prim = -1;
    }
  }
}

// shader.wgsl:658-692
void trace_torus(const Ray& ray, const wgpt_object& tor, SurfaceHit* hit, int32_t idx) {
  m4 inv = load_m4(tor.inv_matrix);
  Ray l_ray;
  l_ray.origin = mul_point(inv, ray.origin);
  l_ray.direction = mul_dir(inv, ray.direction);
  float ray_scale = length(l_ray.direction);
  l_ray.direction = l_ray.direction / ray_scale;
  float t = hit_torus(l_ray, 1.0f, tor.param0 * 1.0f);
  if (t > 0.0f) {
    float world_t = t / ray_scale;
    if (world_t < hit->t) {
      hit->t = world_t;
      hit->m_idx = tor.material_idx;
      v3 p = l_ray.origin + l_ray.direction * t;
      v3 ring_p = normalize(mk3(p.x, 0.0f, p.z));
      v3 local_n = normalize(p - ring_p);
      m3 n_mat = upper3(inv);   // no transpose (reference quirk, shader.wgsl:681)
      hit->hit_n = normalize(mul3(n_mat, local_n));
      float u = (atan2_(p.z, p.x) / TWO_PI) + 0.5f;
      float v = (atan2_(p.y, length2(mk2(p.x, p.z)) - 1.0f) / TWO_PI) + 0.5f;
      hit->hit_uv = mk2(u, v);
      hit->o_idx = idx;
      hit->prim = -1;
    }
  }
}

// shader.wgsl:694-752
void trace_tlas(Ctx& c, const Ray& ray, SurfaceHit* hit) {
  const Scene* s = c.s;
  v3 inv_dir = 1.0f / ray.direction;
  uint32_t stack[STACK_SIZE];
  int32_t stack_ptr = 0;
  stack[0] = 0;
  stack_ptr++;
  c.count(C_CHILD_TESTS);
  float base_t = intersect_aabb(ray.origin, inv_dir, L3(s->tlas[0].aabb_min), L3(s->tlas[0].aabb_max));
  if (base_t < 0.0f || base_t >= hit->t) return;
  while (stack_ptr > 0) {
    hit->count++;
    c.count(C_NODES);
    stack_ptr--;
    uint32_t node_idx = stack[stack_ptr];
    const wgpt_bvh_node& node = s->tlas[node_idx];
    if (node.num_triangles > 0u) {
      uint32_t start = node.next;
      uint32_t end = start + node.num_triangles;
      for (uint32_t i = start; i < end; i++) {
        const wgpt_object& obj = s->objs[i];
        int32_t otype = obj.object_type;
        int32_t idx = (int32_t)i;
        c.count(C_OBJ_VISITS);
        if (HAS(s, WGPT_HAS_MESHES) && otype == 0) {
          MeshInstance mesh = mesh_from_object(obj);
          trace_mesh(c, ray, mesh, hit, idx);
        } else if (HAS(s, WGPT_HAS_SPHERES) && otype == 1) {
          trace_sphere(ray, obj, hit, idx);
        } else if (HAS(s, WGPT_HAS_CUBES) && otype == 2) {
          trace_cube(ray, obj, hit, idx);
        } else if (HAS(s, WGPT_HAS_CYLINDERS) && otype == 3) {
          trace_cylinder(ray, obj, hit, idx);
        } else if (HAS(s, WGPT_HAS_TORI) && otype == 4) {
          trace_torus(ray, obj, hit, idx);
        }
      }
    } else {
      uint32_t left_idx = node_idx + 1u;
      uint32_t right_idx = node.next;
      c.count(C_CHILD_TESTS, 2);
      float left_t = intersect_aabb(ray.origin, inv_dir, L3(s->tlas[left_idx].aabb_min), L3(s->tlas[left_idx].aabb_max));
      float right_t = intersect_aabb(ray.origin, inv_dir, L3(s->tlas[right_idx].aabb_min), L3(s->tlas[right_idx].aabb_max));
      if (left_t < right_t) {
        if (right_t >= 0.0f && right_t < hit->t) { if (stack_ptr < STACK_SIZE) stack[stack_ptr++] = right_idx; else c.err |= 1; }
        if (left_t >= 0.0f && left_t < hit->t) { if (stack_ptr < STACK_SIZE) stack[stack_ptr++] = left_idx; else c.err |= 1; }
      } else {
        if (left_t >= 0.0f && left_t < hit->t) { if (stack_ptr < STACK_SIZE) stack[stack_ptr++] = left_idx; else c.err |= 1; }
        if (right_t >= 0.0f && right_t < hit->t) { if (stack_ptr < STACK_SIZE) stack[stack_ptr++] = right_idx; else c.err |= 1; }
      }
    }
  }
}

// shader.wgsl:754-774
SurfaceHit trace_scene(Ctx& c, const Ray& ray) {
  const Scene* s = c.s;
  c.count(C_RAYS_EXT);
  SurfaceHit hit;
  hit.t = 1e10f; hit.m_idx = -1;
  hit.hit_p = mk3s(0.0f); hit.hit_n = mk3s(0.0f); hit.hit_uv = mk2(0.0f, 0.0f);
  hit.tangent = mk3s(0.0f); hit.bitangent = mk3s(0.0f);
  hit.o_idx = -1; hit.count = 0; hit.prim = -1;
  if (HAS(s, WGPT_HAS_PLANES)) {
    for (uint32_t i = 0; i < s->n_planes; i++) trace_plane(ray, s->planes[i], &hit);
  }
  if (HAS(s, WGPT_HAS_SPHERES | WGPT_HAS_CUBES | WGPT_HAS_CYLINDERS | WGPT_HAS_TORI | WGPT_HAS_MESHES)) {
    trace_tlas(c, ray, &hit);
  }
  if (HAS(s, WGPT_HAS_LIST_MESHES)) {
    for (uint32_t i = 0; i < s->n_meshes; i++) {
      MeshInstance m = mesh_from_list(s, i);
      trace_mesh(c, ray, m, &hit, -1);
    }
  }
  return hit;
}

// ------------------------------------------------------------------------ shadow rays
// shader.wgsl:777-811: a surface without an albedo texture blocks fully; one with it lets
// (1 - alpha) through and blocks once alpha exceeds 0.9999 (the distance is unused).
// An occluder with material index -1 (read out of bounds by the WGSL, where the value is not
// pinned) blocks like an untextured one.
const wgpt_material* occluder_material(const Scene* s, int32_t idx) { return idx >= 0 ? &s->mats[idx] : nullptr; }

bool evaluate_shadow_attenuation(const Scene* s, const wgpt_material* mat, v2 uv, float /*dist*/, v3* shadow) {
  if (mat && mat->albedo_idx >= 0) {
    v4 tex_color = sample_texture(s, mat->albedo_idx, uv * L2(mat->uv_scale));
    *shadow = *shadow * (1.0f - tex_color.w);
    if (tex_color.w > 0.9999f) return true;
  } else {
    return true;
  }
  return false;
}

// shader.wgsl:1090-1094
v2 get_torus_uv(v3 p) {
  float u = (atan2_(p.z, p.x) / TWO_PI) + 0.5f;
  float v = (atan2_(p.y, length(mk2(p.x, p.z)) - 1.0f) / TWO_PI) + 0.5f;
  return mk2(u, v);
}

// shader.wgsl:907-924
v2 get_cube_uv(v3 local_hit) {
  v3 d = vabs(local_hit);
  float max_d = max_component(d);
  if (max_d == d.x) {
    float sg = sign(local_hit.x);
    return mk2((-sg * local_hit.z) * 0.5f + 0.5f, local_hit.y * 0.5f + 0.5f);
  } else if (max_d == d.y) {
    float sg = sign(local_hit.y);
    return mk2(local_hit.x * 0.5f + 0.5f, (sg * local_hit.z) * 0.5f + 0.5f);
  }
  float sg = sign(local_hit.z);
  return mk2((sg * local_hit.x) * 0.5f + 0.5f, local_hit.y * 0.5f + 0.5f);
}

// shader.wgsl:958-962
v2 get_frustum_uv(v3 p, float r0, float r1) {
  if (p.y > 0.999f) return mk2(p.x / (r1 * 2.0f) + 0.5f, p.z / (r1 * 2.0f) + 0.5f);
  if (p.y < 0.001f) return mk2(p.x / (r0 * 2.0f) + 0.5f, p.z / (r0 * 2.0f) + 0.5f);
  return mk2(atan2_(p.z, p.x) / TWO_PI + 0.5f, p.y);
}

v2 sphere_uv(v3 p) {
  return mk2(0.5f + atan2_(p.z, p.x) / TWO_PI, 0.5f + asin_(clamp(p.y, -1.0f, 1.0f)) / PI);
}

// shader.wgsl:813-872
bool trace_mesh_shadow(Ctx& c, const Ray& ray_world, const MeshInstance& mesh, float target_dist, v3* shadow) {
  const Scene* s = c.s;
  Ray ray_local;
  ray_local.origin = mul_point(mesh.inv_matrix, ray_world.origin);
  ray_local.direction = mul_dir(mesh.inv_matrix, ray_world.direction);
  v3 inv_dir = 1.0f / ray_local.direction;
  uint32_t stack[STACK_SIZE];
  int32_t stack_ptr = 0;
  stack[0] = mesh.node_offset;
  stack_ptr++;
  c.count(C_CHILD_TESTS);
  float base_t = intersect_aabb(ray_local.origin, inv_dir, L3(s->bvh[mesh.node_offset].aabb_min), L3(s->bvh[mesh.node_offset].aabb_max));
  if (base_t < 0.0f || base_t >= target_dist) return false;
  float last_t = 0.0f;
  bool is_inside = false;
  const wgpt_material* mat = occluder_material(s, mesh.material_idx);
  while (stack_ptr > 0) {
    stack_ptr--;
    c.count(C_NODES);
    uint32_t node_idx = stack[stack_ptr];
    const wgpt_bvh_node& node = s->bvh[node_idx];
    if (node.num_triangles > 0u) {
      uint32_t start = mesh.tri_offset + node.next;
      uint32_t end = start + node.num_triangles;
      for (uint32_t i = start; i < end; i++) {
        const wgpt_triangle& tri = s->tris[i];
        float t_tri = 0.0f; v2 uv_tri = mk2(0.0f, 0.0f); v3 bary = mk3s(0.0f);
        c.count(C_TRI_TESTS);
        if (intersect_triangle(ray_local, tri, &t_tri, &uv_tri, &bary)) {
          if (t_tri >= 0.0f && t_tri < target_dist) {
            float volume_dist = sel(0.0f, t_tri - last_t, is_inside);
            if (evaluate_shadow_attenuation(s, mat, uv_tri, volume_dist, shadow)) return true;
            last_t = t_tri;
            is_inside = !is_inside;
          }
        }
      }
    } else {
      uint32_t left_idx = node_idx + 1u;
      uint32_t right_idx = mesh.node_offset + node.next;
      c.count(C_CHILD_TESTS, 2);
      float left_t = intersect_aabb(ray_local.origin, inv_dir, L3(s->bvh[left_idx].aabb_min), L3(s->bvh[left_idx].aabb_max));
      float right_t = intersect_aabb(ray_local.origin, inv_dir, L3(s->bvh[right_idx].aabb_min), L3(s->bvh[right_idx].aabb_max));
      if (left_t < right_t) {
        if (right_t >= 0.0f && right_t < target_dist) { if (stack_ptr < STACK_SIZE) stack[stack_ptr++] = right_idx; else c.err |= 1; }
        if (left_t >= 0.0f && left_t < target_dist) { if (stack_ptr < STACK_SIZE) stack[stack_ptr++] = left_idx; else c.err |= 1; }
      } else {
        if (left_t >= 0.0f && left_t < target_dist) { if (stack_ptr < STACK_SIZE) stack[stack_ptr++] = left_idx; else c.err |= 1; }
        if (right_t >= 0.0f && right_t < target_dist) { if (stack_ptr < STACK_SIZE) stack[stack_ptr++] = right_idx; else c.err |= 1; }
      }
    }
  }
  return false;
}

// shader.wgsl:874-905
bool trace_sphere_shadow(Ctx& c, const Ray& ray_world, const wgpt_object& so, float target_dist, v3* shadow) {
  m4 inv = load_m4(so.inv_matrix);
  Ray local_ray;
  local_ray.origin = mul_point(inv, ray_world.origin);
  local_ray.direction = mul_dir(inv, ray_world.direction);
  float a = dot(local_ray.direction, local_ray.direction);
  float half_b = dot(local_ray.origin, local_ray.direction);
  float cc = dot(local_ray.origin, local_ray.origin) - 1.0f;
  float disc = half_b * half_b - a * cc;
  if (disc < 0.0f) return false;
  float sqrtd = sqrtf(disc);
  float t1 = (-half_b - sqrtd) / a;
  float t2 = (-half_b + sqrtd) / a;
  float h1 = wmax(0.001f, t1);
  float h2 = wmin(target_dist, t2);
  if (h1 < h2) {
    const wgpt_material* mat = occluder_material(c.s, so.material_idx);
    v3 p1 = local_ray.origin + local_ray.direction * h1;
    if (evaluate_shadow_attenuation(c.s, mat, sphere_uv(p1), 0.0f, shadow)) return true;
    v3 p2 = local_ray.origin + local_ray.direction * h2;
    return evaluate_shadow_attenuation(c.s, mat, sphere_uv(p2), h2 - h1, shadow);
  }
  return false;
}

// shader.wgsl:926-956
bool trace_cube_shadow(Ctx& c, const Ray& ray_world, const wgpt_object& co, float target_dist, v3* shadow) {
  m4 inv = load_m4(co.inv_matrix);
  Ray local_ray;
  local_ray.origin = mul_point(inv, ray_world.origin);
  local_ray.direction = mul_dir(inv, ray_world.direction);
  v3 inv_dir = 1.0f / local_ray.direction;
  v3 t_near_xyz = (-1.0f - local_ray.origin) * inv_dir;
  v3 t_far_xyz = (1.0f - local_ray.origin) * inv_dir;
  v3 t_min = vmin(t_near_xyz, t_far_xyz);
  v3 t_max = vmax(t_near_xyz, t_far_xyz);
  float t1 = max_component(t_min);
  float t2 = min_component(t_max);
  float h1 = wmax(0.001f, t1);
  float h2 = wmin(target_dist, t2);
  if (h1 < h2) {
    const wgpt_material* mat = occluder_material(c.s, co.material_idx);
    v3 p1 = local_ray.origin + local_ray.direction * h1;
    if (evaluate_shadow_attenuation(c.s, mat, get_cube_uv(p1), 0.0f, shadow)) return true;
    v3 p2 = local_ray.origin + local_ray.direction * h2;
    return evaluate_shadow_attenuation(c.s, mat, get_cube_uv(p2), h2 - h1, shadow);
  }
  return false;
}

// shader.wgsl:964-1016
bool trace_cylinder_shadow(Ctx& c, const Ray& ray_world, const wgpt_object& f, float target_dist, v3* shadow) {
  m4 inv = load_m4(f.inv_matrix);
  Ray r;
  r.origin = mul_point(inv, ray_world.origin);
  r.direction = mul_dir(inv, ray_world.direction);
  float top_radius = f.param0;
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
    float ts[2] = {(-B - sqrt_d) / (2.0f * A), (-B + sqrt_d) / (2.0f * A)};
    for (int i = 0; i < 2; i++) {
      float t = ts[i];
      float y = r.origin.y + t * r.direction.y;
      if (y >= 0.0f && y <= 1.0f) { h1 = wmin(h1, t); h2 = wmax(h2, t); hit_count++; }
    }
  }
  const float caps[2] = {0.0f, 1.0f};
  const float radii[2] = {1.0f, top_radius};
  for (int i = 0; i < 2; i++) {
    float t = (caps[i] - r.origin.y) / r.direction.y;
    v3 p = r.origin + t * r.direction;
    if (p.x * p.x + p.z * p.z <= radii[i] * radii[i]) { h1 = wmin(h1, t); h2 = wmax(h2, t); hit_count++; }
  }
  if (hit_count >= 2u) {
    float final_h1 = wmax(0.001f, h1);
    float final_h2 = wmin(target_dist, h2);
    if (final_h1 < final_h2) {
      const wgpt_material* mat = occluder_material(c.s, f.material_idx);
      v2 uv1 = get_frustum_uv(r.origin + r.direction * final_h1, 1.0f, top_radius);
      if (evaluate_shadow_attenuation(c.s, mat, uv1, 0.0f, shadow)) return true;
      v2 uv2 = get_frustum_uv(r.origin + r.direction * final_h2, 1.0f, top_radius);
      return evaluate_shadow_attenuation(c.s, mat, uv2, final_h2 - final_h1, shadow);
    }
  }
  return false;
}

// shader.wgsl:1019-1034
float solve_cubic_real(float a, float b, float cc) {
  float q = (a * a - 3.0f * b) / 9.0f;
  float r = (2.0f * a * a * a - 9.0f * a * b + 27.0f * cc) / 54.0f;
  float r2 = r * r;
  float q3 = q * q * q;
  if (r2 < q3) {
    float theta = acos_(clamp(r / sqrtf(q3), -1.0f, 1.0f));
    return -2.0f * sqrtf(q) * cos_(theta / 3.0f) - a / 3.0f;
  } else {
    float aa = -sign(r) * pow_(absf(r) + sqrtf(r2 - q3), 1.0f / 3.0f);
    float bb = 0.0f;
    if (aa != 0.0f) bb = q / aa;
    return (aa + bb) - a / 3.0f;
  }
}

// shader.wgsl:1037-1087
void solve_quartic_real(float a, float b, float cc, float d, float roots[4]) {
  roots[0] = roots[1] = roots[2] = roots[3] = -1.0f;
  uint32_t count = 0u;
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
  if (D2 >= 0.0f) {
    float D = sqrtf(D2);
    roots[0] = -0.25f * a + 0.5f * R + 0.5f * D;
    roots[1] = -0.25f * a + 0.5f * R - 0.5f * D;
    count += 2u;
  }
  if (E2 >= 0.0f) {
    float E = sqrtf(E2);
    roots[count] = -0.25f * a - 0.5f * R + 0.5f * E;
    roots[count + 1u] = -0.25f * a - 0.5f * R - 0.5f * E;
    count += 2u;
  }
  for (uint32_t i = 0u; i < 3u; i++) {
    for (uint32_t j = i + 1u; j < 4u; j++) {
      if (roots[i] > roots[j]) { float tmp = roots[i]; roots[i] = roots[j]; roots[j] = tmp; }
    }
  }
}

// shader.wgsl:1096-1132
bool trace_torus_shadow(Ctx& c, const Ray& ray_world, const wgpt_object& tor, float target_dist, v3* shadow) {
  m4 inv = load_m4(tor.inv_matrix);
  Ray l_r;
  l_r.origin = mul_point(inv, ray_world.origin);
  l_r.direction = mul_dir(inv, ray_world.direction);
  float ray_scale = length(l_r.direction);
  l_r.direction = l_r.direction / ray_scale;
  float R = 1.0f; float r = tor.param0;
  float K = dot(l_r.origin, l_r.origin) + R * R - r * r;
  float G = dot(l_r.origin, l_r.direction);
  float B = 4.0f * G;
  float C = 2.0f * K + 4.0f * G * G - 4.0f * R * R * (1.0f - l_r.direction.y * l_r.direction.y);
  float D = 4.0f * K * G - 8.0f * R * R * l_r.origin.y * l_r.direction.y;
  float E = K * K - 4.0f * R * R * (l_r.origin.x * l_r.origin.x + l_r.origin.z * l_r.origin.z);
  float roots[4];
  solve_quartic_real(B, C, D, E, roots);
  const wgpt_material* mat = occluder_material(c.s, tor.material_idx);
  for (int i = 0; i < 4; i += 2) {
    float t_near = roots[i]; float t_far = roots[i + 1];
    if (t_near < 0.0f || t_near > target_dist * ray_scale) continue;
    float h1 = wmax(0.001f, t_near) / ray_scale;
    float h2 = wmin(target_dist * ray_scale, t_far) / ray_scale;
    if (h1 < h2) {
      v2 uv1 = get_torus_uv(l_r.origin + l_r.direction * (h1 * ray_scale));
      if (evaluate_shadow_attenuation(c.s, mat, uv1, 0.0f, shadow)) return true;
      v2 uv2 = get_torus_uv(l_r.origin + l_r.direction * (h2 * ray_scale));
      if (evaluate_shadow_attenuation(c.s, mat, uv2, h2 - h1, shadow)) return true;
    }
  }
  return false;
}

// shader.wgsl:1134-1184
bool trace_tlas_shadow(Ctx& c, const Ray& ray, int32_t target_idx, float target_dist, v3* shadow) {
  const Scene* s = c.s;
  v3 inv_dir = 1.0f / ray.direction;
  uint32_t stack[STACK_SIZE];
  int32_t stack_ptr = 0;
  stack[stack_ptr] = 0u;
  stack_ptr++;
  while (stack_ptr > 0) {
    stack_ptr--;
    c.count(C_NODES);
    uint32_t node_idx = stack[stack_ptr];
    const wgpt_bvh_node& node = s->tlas[node_idx];
    if (node.num_triangles > 0u) {
      uint32_t start = node.next;
      uint32_t end = start + node.num_triangles;
      for (uint32_t i = start; i < end; i++) {
        if ((int32_t)i == target_idx) continue;
        const wgpt_object& obj = s->objs[i];
        int32_t otype = obj.object_type;
        c.count(C_OBJ_VISITS);
        if (HAS(s, WGPT_HAS_MESHES) && otype == 0) {
          MeshInstance mesh = mesh_from_object(obj);
          if (trace_mesh_shadow(c, ray, mesh, target_dist, shadow)) return true;
        } else if (HAS(s, WGPT_HAS_SPHERES) && otype == 1) {
          if (trace_sphere_shadow(c, ray, obj, target_dist, shadow)) return true;
        } else if (HAS(s, WGPT_HAS_CUBES) && otype == 2) {
          if (trace_cube_shadow(c, ray, obj, target_dist, shadow)) return true;
        } else if (HAS(s, WGPT_HAS_CYLINDERS) && otype == 3) {
          if (trace_cylinder_shadow(c, ray, obj, target_dist, shadow)) return true;
        } else if (HAS(s, WGPT_HAS_TORI) && otype == 4) {
          if (trace_torus_shadow(c, ray, obj, target_dist, shadow)) return true;
        }
      }
    } else {
      uint32_t left_idx = node_idx + 1u;
      uint32_t right_idx = node.next;
      c.count(C_CHILD_TESTS, 2);
      float left_t = intersect_aabb(ray.origin, inv_dir, L3(s->tlas[left_idx].aabb_min), L3(s->tlas[left_idx].aabb_max));
      float right_t = intersect_aabb(ray.origin, inv_dir, L3(s->tlas[right_idx].aabb_min), L3(s->tlas[right_idx].aabb_max));
      if (left_t < right_t) {
        if (right_t >= 0.0f && right_t < target_dist) { if (stack_ptr < STACK_SIZE) stack[stack_ptr++] = right_idx; else c.err |= 1; }
        if (left_t >= 0.0f && left_t < target_dist) { if (stack_ptr < STACK_SIZE) stack[stack_ptr++] = left_idx; else c.err |= 1; }
      } else {
        if (left_t >= 0.0f && left_t < target_dist) { if (stack_ptr < STACK_SIZE) stack[stack_ptr++] = left_idx; else c.err |= 1; }
        if (right_t >= 0.0f && right_t < target_dist) { if (stack_ptr < STACK_SIZE) stack[stack_ptr++] = right_idx; else c.err |= 1; }
      }
    }
  }
  return false;
}

// shader.wgsl:1186-1204
bool trace_plane_shadow(Ctx& c, const Ray& ray, const wgpt_plane& p, float target_dist, v3* shadow) {
  v3 pn = L3(p.normal);
  float denom = dot(pn, ray.direction);
  if (absf(denom) > 1e-6f) {
    float t = (p.d - dot(pn, ray.origin)) / denom;
    if (t > 0.001f && t < target_dist) {
      v3 hit_pos = ray.origin + ray.direction * t;
      const wgpt_material* mat = occluder_material(c.s, p.material_idx);
      v3 tangent = mk3(1.0f, 0.0f, 0.0f);
      if (absf(pn.x) > 0.9999f) tangent = mk3(0.0f, 0.0f, 1.0f);
      tangent = normalize(cross(pn, tangent));
      v3 bitangent = normalize(cross(pn, tangent));
      v2 uv = mk2(dot(hit_pos, tangent), dot(hit_pos, bitangent));
      return evaluate_shadow_attenuation(c.s, mat, uv, length(ray.origin - hit_pos), shadow);
    }
  }
  return false;
}

// shader.wgsl:1206-1229
v3 trace_scene_shadow(Ctx& c, const Ray& ray, int32_t target_idx, float target_dist) {
  const Scene* s = c.s;
  c.count(C_RAYS_SHADOW);
  v3 shadow = mk3s(1.0f);
  if (HAS(s, WGPT_HAS_PLANES)) {
    for (uint32_t i = 0; i < s->n_planes; i++)
      if (trace_plane_shadow(c, ray, s->planes[i], target_dist, &shadow)) return mk3s(0.0f);
  }
  if (HAS(s, WGPT_HAS_SPHERES | WGPT_HAS_CUBES | WGPT_HAS_CYLINDERS | WGPT_HAS_TORI | WGPT_HAS_MESHES)) {
    if (trace_tlas_shadow(c, ray, target_idx, target_dist, &shadow)) return mk3s(0.0f);
  }
  if (HAS(s, WGPT_HAS_LIST_MESHES)) {
    for (uint32_t i = 0; i < s->n_meshes; i++) {
      MeshInstance m = mesh_from_list(s, i);
      if (trace_mesh_shadow(c, ray, m, target_dist, &shadow)) return mk3s(0.0f);
    }
  }
  return shadow;
}

// ------------------------------------------------------------------------ shading
struct SurfaceContext { v3 normal, surface_normal, albedo; float roughness, metallic; v3 emittance; float alpha; };

// shader.wgsl:1393-1440
SurfaceContext get_surface_context(const Scene* s, const SurfaceHit& hit, const wgpt_material& mat, const m3& tbn,
                                   v2 uv) {
  SurfaceContext ctx;
  ctx.normal = hit.hit_n;
  ctx.surface_normal = hit.hit_n;
  if (mat.normal_idx >= 0) {
    v4 t = sample_texture(s, mat.normal_idx, uv);
    v3 n_map = mk3(t.x, t.y, t.z) * 2.0f - mk3s(1.0f);
    n_map = normalize(n_map * mk3(mat.height_params[0], mat.height_params[0], 1.0f));
    ctx.normal = normalize(mul3(tbn, n_map));
  }
  ctx.albedo = L3(mat.color);
  ctx.alpha = 1.0f;
  if (mat.albedo_idx >= 0) {
    v4 tex_color = sample_texture(s, mat.albedo_idx, uv);
    ctx.alpha = tex_color.w;
    ctx.albedo = ctx.albedo * vpow(mk3(tex_color.x, tex_color.y, tex_color.z), 2.2f);
  }
  ctx.metallic = mat.metallic;
  ctx.roughness = mat.roughness;
  if (mat.roughness_idx >= 0) ctx.roughness *= sample_texture(s, mat.roughness_idx, uv).y;
  if (mat.metallic_idx >= 0) ctx.metallic *= sample_texture(s, mat.metallic_idx, uv).z;
  ctx.emittance = L3(mat.emittance);
  if (mat.emissive_idx >= 0) {
    v4 e = sample_texture(s, mat.emissive_idx, uv);
    ctx.emittance = ctx.emittance * vpow(mk3(e.x, e.y, e.z), 2.2f);
  }
  return ctx;
}

// shader.wgsl:1230-1278.  A result that leaves through the early return keeps WGSL's zero
// initialisation (uv (0, 0), height 0), which main then uses as the texture coordinate.
struct PomResult { v2 uv; float height; bool hit; };
float height_depth(const Scene* s, int32_t height_idx, v2 uv, bool is_height_map) {
  float v = sample_texture(s, height_idx, uv).x;
  return is_height_map ? 1.0f - v : v;
}
PomResult calculate_pom(const Scene* s, v2 initial_uv, v3 view_ts, float start_depth, const wgpt_material& mat,
                        int32_t height_idx) {
  PomResult res;
  res.uv = mk2(0.0f, 0.0f); res.height = 0.0f; res.hit = false;
  float hm = mat.height_params[1];
  bool is_height_map = hm < 0.0f;
  float scale = absf(hm);
  float num_layers = mat.height_params[2];
  float layer_depth = 1.0f / num_layers;
  float cur_layer = clamp(start_depth, 0.0f, 1.0f);
  v2 P = mk2(-(view_ts.x / view_ts.z), -(view_ts.y / view_ts.z)) * scale;
  v2 delta = mk2(P.x / num_layers, P.y / num_layers);
  v2 cur_uv = initial_uv - P * mat.height_params[3];
  float cur_depth = height_depth(s, height_idx, cur_uv, is_height_map);
  for (int i = 0; i < 64; i++) {
    if ((float)i >= num_layers || cur_layer >= cur_depth) break;
    if (cur_layer > 1.0f || cur_layer < 0.0f) return res;
    cur_uv = cur_uv + delta;
    cur_depth = height_depth(s, height_idx, cur_uv, is_height_map);
    cur_layer += layer_depth;
  }
  v2 prev_uv = cur_uv - delta;
  float prev_depth = height_depth(s, height_idx, prev_uv, is_height_map);
  float after = cur_depth - cur_layer;
  float before = prev_depth - cur_layer + layer_depth;
  float weight = after / (after - before);
  res.uv = mk2(mix(cur_uv.x, prev_uv.x, weight), mix(cur_uv.y, prev_uv.y, weight));
  res.height = mix(cur_layer, cur_layer - layer_depth, weight);
  res.hit = true;
  return res;
}

// shader.wgsl:1280-1328
PomResult calculate_shadow_pom(const Scene* s, v2 current_uv, float current_height, v3 light_ts,
                               const wgpt_material& mat, int32_t height_idx) {
  PomResult res;
  res.hit = false; res.uv = current_uv; res.height = current_height;
  if (light_ts.z <= 0.0f) { res.hit = true; return res; }
  float hm = mat.height_params[1];
  bool is_height_map = hm < 0.0f;
  float scale = absf(hm);
  float num_layers = mat.height_params[2];
  float layer_depth = 1.0f / num_layers;
  v2 p = (mk2(light_ts.x / light_ts.z, light_ts.y / light_ts.z) * scale) * layer_depth;
  v2 shadow_uv = current_uv;
  float shadow_depth = current_height;
  for (int i = 0; i < 32; i++) {
    if ((float)i / 2.0f >= num_layers || shadow_depth <= 0.0f) break;
    shadow_uv = shadow_uv + p;
    shadow_depth -= layer_depth;
    float map_depth = height_depth(s, height_idx, shadow_uv, is_height_map);
    if (map_depth < shadow_depth) {
      res.hit = true; res.uv = shadow_uv; res.height = map_depth;
      return res;
    }
  }
  return res;
}

// shader.wgsl:1459-1464
m3 build_tangent_space(v3 N) {
  v3 a = vsel(mk3(0.0f, 1.0f, 0.0f), mk3(0.0f, 0.0f, 1.0f), absf(N.y) > 0.99999f);
  v3 T = normalize(cross(N, a));
  v3 B = cross(T, N);
  m3 r; r.c[0] = T; r.c[1] = B; r.c[2] = N; return r;
}

// shader.wgsl:1473-1499
float light_sphere_pdf(const wgpt_light& light, const wgpt_object& sphere, v3 hit_pos, v3 dir) {
  v3 light_pos = L3(sphere.world_position);
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
LightSample sample_light_sphere(Ctx& c, const wgpt_light& light, const wgpt_object& sphere, v3 hit_pos, v2 xi) {
  v3 light_pos = L3(sphere.world_position);
  const wgpt_material& mat = c.s->mats[sphere.material_idx];
  v3 d = light_pos - hit_pos;
  float d2 = dot(d, d);
  float r2 = light.scale * light.scale;
  LightSample ls;
  ls.color = L3(mat.emittance);
  if (d2 <= r2) {
    float z = 1.0f - 2.0f * xi.x;
    float sin_theta = sqrtf(wmax(0.0f, 1.0f - z * z));
    float phi = TWO_PI * xi.y;
    ls.dir = mk3(sin_theta * cos_(phi), sin_theta * sin_(phi), z);
    ls.dist = 0.0f;
    ls.pdf = 1.0f / (4.0f * PI);
    return ls;
  }
  float sin_theta_max_sq = r2 / d2;
  float cos_theta_max = sqrtf(wmax(0.0f, 1.0f - sin_theta_max_sq));
  float cos_theta = 1.0f - xi.x * (1.0f - cos_theta_max);
  float sin_theta = sqrtf(wmax(0.0f, 1.0f - cos_theta * cos_theta));
  float phi = TWO_PI * xi.y;
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

struct BoxAreas { v3 v1, v2, v3_, cen; float s1, s2, s3, a1, a2, a3, total; };
BoxAreas box_areas(const wgpt_light& light, v3 hit_pos) {
  BoxAreas b;
  m4 m = load_m4(light.matrix);
  b.v1 = xyz(m.c[0]); b.v2 = xyz(m.c[1]); b.v3_ = xyz(m.c[2]); b.cen = xyz(m.c[3]);
  v3 d = b.cen - hit_pos;
  b.s1 = sel(-1.0f, 1.0f, dot(d, b.v1) < 0.0f);
  b.s2 = sel(-1.0f, 1.0f, dot(d, b.v2) < 0.0f);
  b.s3 = sel(-1.0f, 1.0f, dot(d, b.v3_) < 0.0f);
  b.a1 = length(cross(b.v2 * 2.0f, b.v3_ * 2.0f)) * wmax(dot(normalize(-d), normalize(b.v1 * b.s1)), 0.01f);
  b.a2 = length(cross(b.v1 * 2.0f, b.v3_ * 2.0f)) * wmax(dot(normalize(-d), normalize(b.v2 * b.s2)), 0.01f);
  b.a3 = length(cross(b.v1 * 2.0f, b.v2 * 2.0f)) * wmax(dot(normalize(-d), normalize(b.v3_ * b.s3)), 0.01f);
  b.total = b.a1 + b.a2 + b.a3;
  return b;
}

// shader.wgsl:1551-1573
float light_box_pdf(const wgpt_light& light, v3 hit_pos, v3 ray_dir, const SurfaceHit& hit) {
  BoxAreas b = box_areas(light, hit_pos);
  float cos_l = wmax(dot(-ray_dir, hit.hit_n), 1e-6f);
  float dist_sq = hit.t * hit.t;
  return dist_sq / (b.total * cos_l);
}

// shader.wgsl:1575-1624
LightSample sample_light_box(Ctx& c, const wgpt_light& light, const wgpt_object& obj, v3 hit_pos, v2 xi) {
  BoxAreas b = box_areas(light, hit_pos);
  v3 p = b.cen;
  v3 n = mk3s(0.0f);
  float u = xi.x * 2.0f - 1.0f;
  float v = xi.y * 2.0f - 1.0f;
  float pick = rand_pcg(c.rng) * b.total;
  if (pick < b.a1) {
    p = p + ((b.v1 * b.s1 + b.v2 * u) + b.v3_ * v);
    n = normalize(b.v1 * b.s1);
  } else if (pick < b.a1 + b.a2) {
    p = p + ((b.v2 * b.s2 + b.v1 * u) + b.v3_ * v);
    n = normalize(b.v2 * b.s2);
  } else {
    p = p + ((b.v3_ * b.s3 + b.v1 * u) + b.v2 * v);
    n = normalize(b.v3_ * b.s3);
  }
  LightSample ls;
  v3 delta = p - hit_pos;
  float dist_sq = dot(delta, delta);
  ls.dist = sqrtf(dist_sq);
  ls.dir = delta / ls.dist;
  float cos_l = wmax(dot(-ls.dir, n), 1e-6f);
  ls.pdf = dist_sq / (b.total * cos_l);
  ls.color = L3(c.s->mats[obj.material_idx].emittance);
  return ls;
}

// shader.wgsl:1626-1633
float get_light_pdf(const Scene* s, const wgpt_light& light, const wgpt_object& obj, v3 hit_pos, v3 dir, const SurfaceHit& hit) {
  if (HAS(s, WGPT_HAS_SPHERES) && obj.object_type == 1) return light_sphere_pdf(light, obj, hit_pos, dir);
  if (HAS(s, WGPT_HAS_CUBES) && obj.object_type == 2) return light_box_pdf(light, hit_pos, dir, hit);
  return 0.0f;
}

// shader.wgsl:1636-1646
LightSample sample_light(Ctx& c, const wgpt_light& light, const wgpt_object& obj, v3 hit_pos) {
  LightSample samp;
  samp.dir = mk3s(0.0f); samp.color = mk3s(0.0f); samp.dist = 0.0f; samp.pdf = 0.0f;
  if (HAS(c.s, WGPT_HAS_SPHERES) && obj.object_type == 1) {
    float x0 = rand_pcg(c.rng); float x1 = rand_pcg(c.rng);
    samp = sample_light_sphere(c, light, obj, hit_pos, mk2(x0, x1));
  } else if (HAS(c.s, WGPT_HAS_CUBES) && obj.object_type == 2) {
    float x0 = rand_pcg(c.rng); float x1 = rand_pcg(c.rng);
    samp = sample_light_box(c, light, obj, hit_pos, mk2(x0, x1));
  }
  return samp;
}

// shader.wgsl:1648-1659
float mis_weight(float pdf_a, float pdf_b) {
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

// shader.wgsl:1661-1697
struct Medium { float ior; v3 sigma; v3 emission; };
struct MediumStack { Medium media[4]; int32_t count; };
Medium air() { Medium m; m.ior = 1.0f; m.sigma = mk3s(0.0f); m.emission = mk3s(0.0f); return m; }
Medium peek_medium(const MediumStack* st) { return st->count > 0 ? st->media[st->count - 1] : air(); }
Medium peek_outer_medium(const MediumStack* st) { return st->count > 1 ? st->media[st->count - 2] : air(); }
void push_medium(MediumStack* st, Medium m) { if (st->count < 4) { st->media[st->count] = m; st->count += 1; } }
void pop_medium(MediumStack* st) { if (st->count > 0) st->count -= 1; }

// shader.wgsl:1700-1704
float D_GGX(float NdotH, float alpha2) {
  float denom = (NdotH * NdotH * (alpha2 - 1.0f) + 1.0f);
  return alpha2 / (PI * denom * denom + 1e-10f);
}
// shader.wgsl:1721-1733
float fresnel_dielectric(float cosThetaI, float etai, float etat) {
  float cosi = clamp(absf(cosThetaI), 0.0f, 1.0f);
  float sint = (etai / etat) * sqrtf(wmax(0.0f, 1.0f - cosi * cosi));
  if (sint >= 1.0f) return 1.0f;
  float cost = sqrtf(wmax(0.0f, 1.0f - sint * sint));
  float Rs = ((etat * cosi) - (etai * cost)) / ((etat * cosi) + (etai * cost));
  float Rp = ((etai * cosi) - (etat * cost)) / ((etai * cosi) + (etat * cost));
  return (Rs * Rs + Rp * Rp) / 2.0f;
}
// shader.wgsl:1751-1763
v3 ImportanceSampleCosine(v2 xi, v3 N) {
  float phi = TWO_PI * xi.x;
  float cosTheta = sqrtf(clamp(xi.y, 0.0f, 1.0f));
  float sinTheta = sqrtf(wmax(0.0f, 1.0f - xi.y));
  v3 L_local = mk3(cos_(phi) * sinTheta, sin_(phi) * sinTheta, cosTheta);
  v3 up = vsel(mk3(0.0f, 1.0f, 0.0f), mk3(0.0f, 0.0f, 1.0f), absf(N.y) > 0.999f);
  v3 tangent = normalize(cross(up, N));
  v3 bitangent = cross(N, tangent);
  return normalize((tangent * L_local.x + bitangent * L_local.y) + N * L_local.z);
}
// shader.wgsl:1787-1791
float G_Smith_GGX_div_NV(float NdotV, float NdotL, float alpha2) {
  float sqrt_v = sqrtf(wmax(0.0f, alpha2 + NdotV * NdotV * (1.0f - alpha2)));
  float sqrt_l = sqrtf(wmax(0.0f, alpha2 + NdotL * NdotL * (1.0f - alpha2)));
  return (2.0f * NdotL) / (NdotL * sqrt_v + NdotV * sqrt_l + 1e-10f);
}
// shader.wgsl:1794-1798
float G_Smith_GGX_Uncorrelated_div_NV(float NdotV, float NdotL, float alpha2) {
  float lambda_v = NdotV + sqrtf(wmax(0.0f, alpha2 + NdotV * NdotV * (1.0f - alpha2)));
  float lambda_l = NdotL + sqrtf(wmax(0.0f, alpha2 + NdotL * NdotL * (1.0f - alpha2)));
  return (4.0f * NdotL) / (lambda_v * lambda_l + 1e-7f);
}
// shader.wgsl:1801-1803
float G1_GGX_div_NV(float NdotV, float alpha2) {
  return 2.0f / (NdotV + sqrtf(wmax(0.0f, alpha2 + (1.0f - alpha2) * NdotV * NdotV)) + 1e-7f);
}
// shader.wgsl:1806-1829
v3 ImportanceSampleVNDF_GGX(v2 xi, v3 V, v3 N, float alpha_ggx) {
  v3 up = vsel(mk3(0.0f, 1.0f, 0.0f), mk3(0.0f, 0.0f, 1.0f), absf(N.y) > 0.999f);
  v3 T = normalize(cross(up, N));
  v3 B = cross(N, T);
  v3 V_local = mk3(dot(V, T), dot(V, B), dot(V, N));
  v3 Vh = normalize(mk3(alpha_ggx * V_local.x, alpha_ggx * V_local.y, wmax(V_local.z, 0.0f)));
  float lensq = Vh.x * Vh.x + Vh.y * Vh.y;
  v3 T1 = lensq > 0.0f ? mk3(-Vh.y, Vh.x, 0.0f) / sqrtf(wmax(lensq, 1e-7f)) : mk3(1.0f, 0.0f, 0.0f);
  v3 T2 = cross(Vh, T1);
  float r = sqrtf(xi.x);
  float phi = 2.0f * PI * xi.y;
  float t1 = r * cos_(phi);
  float t2 = r * sin_(phi);
  float s = 0.5f * (1.0f + Vh.z);
  float t2_mod = mix(sqrtf(wmax(0.0f, 1.0f - t1 * t1)), t2, s);
  v3 Nh_local = (t1 * T1 + t2_mod * T2) + sqrtf(wmax(0.0f, 1.0f - t1 * t1 - t2_mod * t2_mod)) * Vh;
  v3 Ne_local = normalize(mk3(alpha_ggx * Nh_local.x, alpha_ggx * Nh_local.y, wmax(0.0f, Nh_local.z)));
  return normalize((T * Ne_local.x + B * Ne_local.y) + N * Ne_local.z);
}

struct Etas { float etai, etat; };
Etas etas_for(bool entering, const wgpt_material& mat, const MediumStack* stack) {
  Etas e;
  if (entering) { e.etai = peek_medium(stack).ior; e.etat = mat.ior; }
  else { e.etai = peek_medium(stack).ior; e.etat = peek_outer_medium(stack).ior; }
  return e;
}

// shader.wgsl:1831-1947
v3 eval_surface(v3 V, v3 L, const wgpt_material& mat, const SurfaceContext& ctx, const MediumStack* stack) {
  bool entering = dot(ctx.normal, V) > 0.0f;
  v3 n_orient = vsel(-ctx.normal, ctx.normal, entering);
  float dotNV = dot(n_orient, V);
  float dotNL = dot(n_orient, L);
  if (dotNV <= 0.0f) return mk3s(0.0f);
  float roughness_val = clamp(ctx.roughness, 0.01f, 1.0f);
  float alpha = roughness_val * roughness_val;
  float alpha2 = wmax(alpha * alpha, 1e-6f);
  Etas e = etas_for(entering, mat, stack);
  float etai = e.etai, etat = e.etat;
  if (dotNL > 0.0f) {
    v3 H_vec = V + L;
    v3 H = dot(H_vec, H_vec) > 1e-6f ? normalize(H_vec) : n_orient;
    float dotNH = wmax(dot(n_orient, H), 0.0f);
    float dotVH = wmax(dot(V, H), 0.0f);
    v3 diff_col = ctx.albedo;
    if (mat.sheen > 0.0f) diff_col = diff_col + (vmix(mk3s(1.0f), ctx.albedo, mat.sheen_tint) * pow_(wmax(0.0f, 1.0f - dotNV), 5.0f)) * mat.sheen;
    if (mat.subsurface > 0.0f) diff_col = vmix(diff_col, L3(mat.subsurface_tint), mat.subsurface);
    v3 diffuse = ((diff_col / PI) * (1.0f - ctx.metallic)) * (1.0f - mat.transmission);
    float D = D_GGX(dotNH, alpha2);
    float G2_div_NV = G_Smith_GGX_div_NV(dotNV, dotNL, alpha2);
    float F_dielectric = fresnel_dielectric(dotVH, etai, etat);
    float lum = dot(ctx.albedo, mk3(0.2126f, 0.7152f, 0.0722f));
    v3 tint = lum <= 0.0f ? mk3s(1.0f) : ctx.albedo / wmax(lum, 0.0001f);
    v3 F_dielectric_tinted = vmix3(mk3s(F_dielectric), mk3s(F_dielectric) * tint, mk3s(mat.specular_tint));
    v3 F0_metal = ctx.albedo;
    v3 F90_metal = vmix3(mk3s(1.0f), tint, mk3s(mat.specular_tint));
    v3 F_metal = F0_metal + (F90_metal - F0_metal) * pow_(wmax(0.0f, 1.0f - dotVH), 5.0f);
    v3 F_actual = vmix3(F_dielectric_tinted, F_metal, mk3s(ctx.metallic));
    float F_macro_raw = fresnel_dielectric(dotNV, etai, etat);
    float F0_macro_d = pow2c((etai - etat) / (etai + etat));
    float F_macro_est = mix(F_macro_raw, F0_macro_d, roughness_val);
    v3 F_macro_metal = ctx.albedo + (mk3s(1.0f) - ctx.albedo) * pow_(wmax(0.0f, 1.0f - dotNV), 5.0f);
    v3 F_macro_actual = vmix3(mk3s(F_macro_est), F_macro_metal, mk3s(ctx.metallic));
    v3 diffuse_cos = (diffuse * dotNL) * (mk3s(1.0f) - F_macro_actual);
    float ms_factor = 1.0f + alpha * 0.4f;
    v3 specular_cos = ((((F_actual * D) * G2_div_NV) / 4.0f) * ms_factor);
    v3 clearcoat_cos = mk3s(0.0f);
    float cc_attenuation = 1.0f;
    if (mat.clearcoat > 0.0f && entering) {
      float cc_roughness = clamp(1.0f - mat.clearcoat_gloss, 0.01f, 1.0f);
      float cc_alpha = cc_roughness * cc_roughness;
      float cc_alpha2 = wmax(cc_alpha * cc_alpha, 1e-6f);
      float cc_D = D_GGX(dotNH, cc_alpha2);
      float cc_G2_div_NV = G_Smith_GGX_div_NV(dotNV, dotNL, cc_alpha2);
      float cc_F = fresnel_dielectric(dotVH, 1.0f, mat.clearcoat_ior);
      clearcoat_cos = (mk3s(cc_F) * ((mat.clearcoat * cc_D) * cc_G2_div_NV)) / 4.0f;
      float cc_F_macro = fresnel_dielectric(dotNV, 1.0f, mat.clearcoat_ior);
      cc_attenuation = 1.0f - (mat.clearcoat * cc_F_macro);
    }
    return ((diffuse_cos + specular_cos) * cc_attenuation + clearcoat_cos) * ctx.alpha;
  } else if (dotNL < 0.0f && mat.transmission > 0.0f) {
    v3 H_vec = -(etai * V + etat * L);
    v3 H = normalize(H_vec);
    if (dot(H, n_orient) < 0.0f) H = -H;
    float dotNH = wmax(dot(n_orient, H), 0.0f);
    float dotVH = dot(V, H);
    float dotLH = dot(L, H);
    if (dotVH * dotLH >= 0.0f) return mk3s(0.0f);
    float D = D_GGX(dotNH, alpha2);
    float G2_unc_div_NV = G_Smith_GGX_Uncorrelated_div_NV(dotNV, absf(dotNL), alpha2);
    float F_dielectric = fresnel_dielectric(dotVH, etai, etat);
    float denom = etai * dotVH + etat * dotLH;
    float denom2 = wmax(denom * denom, 1e-7f);
    float ms_factor = 1.0f + alpha * 0.25f;
    float btdf_cos = (absf(dotVH) * absf(dotLH) * etat * etat * (1.0f - F_dielectric) * D * G2_unc_div_NV) / denom2 * ms_factor;
    float cc_attenuation = 1.0f;
    if (mat.clearcoat > 0.0f && entering) {
      float cc_F_macro = fresnel_dielectric(dotNV, 1.0f, mat.clearcoat_ior);
      cc_attenuation = 1.0f - (mat.clearcoat * cc_F_macro);
    }
    v3 trans_color = mk3s(mat.transmission * (1.0f - ctx.metallic));
    return ((trans_color * btdf_cos) * cc_attenuation) * ctx.alpha;
  }
  return mk3s(0.0f);
}

// shader.wgsl:1952-2047
float pdf_surface(v3 V, v3 L, const wgpt_material& mat, const SurfaceContext& ctx, const MediumStack* stack) {
  bool entering = dot(ctx.normal, V) > 0.0f;
  v3 n_orient = vsel(-ctx.normal, ctx.normal, entering);
  float dotNV = dot(n_orient, V);
  float dotNL = dot(n_orient, L);
  if (dotNV <= 0.0f) return 1e-7f;
  float roughness_val = clamp(ctx.roughness, 0.01f, 1.0f);
  float alpha = roughness_val * roughness_val;
  float alpha2 = wmax(alpha * alpha, 1e-6f);
  Etas e = etas_for(entering, mat, stack);
  float etai = e.etai, etat = e.etat;
  float F_cc = fresnel_dielectric(dotNV, 1.0f, mat.clearcoat_ior);
  float p_cc = sel(0.0f, mat.clearcoat * F_cc, entering);
  float F_est_raw = fresnel_dielectric(dotNV, etai, etat);
  float F0_d = pow2c((etai - etat) / (etai + etat));
  float F_est = mix(F_est_raw, F0_d, roughness_val);
  v3 F_metal = ctx.albedo + (mk3s(1.0f) - ctx.albedo) * pow_(wmax(0.0f, 1.0f - dotNV), 5.0f);
  v3 F_actual = vmix3(mk3s(F_est), F_metal, mk3s(ctx.metallic));
  float f_avg = clamp((F_actual.x + F_actual.y + F_actual.z) / 3.0f, 0.0f, 1.0f);
  float p_spec = (1.0f - p_cc) * f_avg;
  float p_trans = (1.0f - p_cc) * (1.0f - f_avg) * mat.transmission * (1.0f - ctx.metallic);
  float p_diff = (1.0f - p_cc) * (1.0f - f_avg) * (1.0f - mat.transmission) * (1.0f - ctx.metallic);
  float pdf = 0.0f;
  if (dotNL > 0.0f) {
    v3 H_vec = V + L;
    v3 H = dot(H_vec, H_vec) > 1e-6f ? normalize(H_vec) : n_orient;
    float dotNH = wmax(dot(n_orient, H), 0.0f);
    float dotVH = wmax(dot(V, H), 0.0f);
    if (p_diff > 0.0f) pdf += p_diff * (dotNL / PI);
    if (p_spec > 0.0f) {
      float D = D_GGX(dotNH, alpha2);
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
      float cc_roughness = clamp(1.0f - mat.clearcoat_gloss, 0.01f, 1.0f);
      float cc_alpha = cc_roughness * cc_roughness;
      float cc_alpha2 = wmax(cc_alpha * cc_alpha, 1e-6f);
      float cc_D = D_GGX(dotNH, cc_alpha2);
      float cc_G1_div_NV = G1_GGX_div_NV(dotNV, cc_alpha2);
      float pdf_H_cc = cc_G1_div_NV * cc_D * wmax(0.0f, dotVH);
      pdf += p_cc * pdf_H_cc / wmax(4.0f * dotVH, 1e-7f);
    }
  } else if (dotNL < 0.0f && p_trans > 0.0f) {
    v3 H_vec = -(etai * V + etat * L);
    v3 H = normalize(H_vec);
    if (dot(H, n_orient) < 0.0f) H = -H;
    float dotNH = wmax(dot(n_orient, H), 0.0f);
    float dotVH = dot(V, H);
    float dotLH = dot(L, H);
    if (dotVH * dotLH < 0.0f) {
      float D = D_GGX(dotNH, alpha2);
      float G1_div_NV = G1_GGX_div_NV(dotNV, alpha2);
      float pdf_H = G1_div_NV * D * wmax(0.0f, dotVH);
      float denom = etai * dotVH + etat * dotLH;
      float dwh_dwi = (etat * etat * absf(dotLH)) / wmax(denom * denom, 1e-7f);
      pdf += p_trans * pdf_H * dwh_dwi;
    }
  }
  return wmax(pdf, 1e-7f) * ctx.alpha;
}

// shader.wgsl:2052-2175
bool sample_surface(Ctx& c, Ray* ray, v3* throughput, v3 hit_pos, const wgpt_material& mat,
                    const SurfaceContext& ctx, MediumStack* stack, float* last_surface_pdf) {
  v3 V = -ray->direction;
  bool entering = dot(ctx.normal, V) > 0.0f;
  v3 n_orient = vsel(-ctx.normal, ctx.normal, entering);
  v3 sn_orient = vsel(-ctx.surface_normal, ctx.surface_normal, entering);
  float dotSNV = wmax(dot(sn_orient, V), 1e-6f);
  float roughness_val = clamp(ctx.roughness, 0.01f, 1.0f);
  float alpha = roughness_val * roughness_val;
  float cc_roughness = clamp(1.0f - mat.clearcoat_gloss, 0.01f, 1.0f);
  float cc_alpha = cc_roughness * cc_roughness;
  Etas e = etas_for(entering, mat, stack);
  float etai = e.etai, etat = e.etat;
  float cc_F_est = fresnel_dielectric(dotSNV, 1.0f, mat.clearcoat_ior);
  float w_cc = sel(0.0f, mat.clearcoat * cc_F_est, entering);
  float F_est_raw = fresnel_dielectric(dotSNV, etai, etat);
  float F0_d = pow2c((etai - etat) / (etai + etat));
  float F_est = mix(F_est_raw, F0_d, roughness_val);
  v3 F_metal = ctx.albedo + (mk3s(1.0f) - ctx.albedo) * pow_(wmax(0.0f, 1.0f - dotSNV), 5.0f);
  v3 F_actual = vmix3(mk3s(F_est), F_metal, mk3s(ctx.metallic));
  float f_avg = clamp((F_actual.x + F_actual.y + F_actual.z) / 3.0f, 0.0f, 1.0f);
  float p_cc = w_cc;
  float p_spec = (1.0f - p_cc) * f_avg;
  float p_trans = (1.0f - p_cc) * (1.0f - f_avg) * mat.transmission * (1.0f - ctx.metallic);
  float p_diff = (1.0f - p_cc) * (1.0f - f_avg) * (1.0f - mat.transmission) * (1.0f - ctx.metallic);
  float total_p = p_cc + p_spec + p_trans + p_diff;

  if (rand_pcg(c.rng) > ctx.alpha) {
    ray->origin = hit_pos - n_orient * 0.005f;
    return true;
  }
  float rng = rand_pcg(c.rng);
  float xi0 = rand_pcg(c.rng);
  float xi1 = rand_pcg(c.rng);
  v2 xi = mk2(xi0, xi1);
  v3 L = mk3s(0.0f);
  bool is_transmission = false;
  if (rng < p_cc) {
    v3 H = ImportanceSampleVNDF_GGX(xi, V, sn_orient, cc_alpha);
    L = reflect(-V, H);
  } else if (rng < p_cc + p_spec) {
    v3 N_spec = n_orient;
    if (mat.anisotropic > 0.0f) {
      v3 up = vsel(mk3(0.0f, 1.0f, 0.0f), mk3(0.0f, 0.0f, 1.0f), absf(n_orient.y) > 0.99999f);
      v3 T = normalize(cross(up, n_orient));
      v3 B = cross(n_orient, T);
      float angle = mat.aniso_rotation * TWO_PI;
      T = T * cos_(angle) + B * sin_(angle);
      N_spec = normalize(vmix(n_orient, cross(cross(V, T), T), mat.anisotropic));
    }
    v3 H = ImportanceSampleVNDF_GGX(xi, V, N_spec, alpha);
    L = reflect(-V, H);
  } else if (rng < p_cc + p_spec + p_trans) {
    if (absf(etai - etat) < 1e-4f) {
      ray->direction = -V;
      ray->origin = hit_pos - n_orient * 0.001f;
      *throughput = *throughput * mk3s(mat.transmission * (1.0f - ctx.metallic));
      *last_surface_pdf = p_trans;
      if (entering) {
        v3 sigma = (-vlog(vmax(ctx.albedo, mk3s(0.0001f)))) * mat.concentration;
        Medium m; m.ior = mat.ior; m.sigma = sigma; m.emission = L3(mat.emittance);
        push_medium(stack, m);
      } else {
        pop_medium(stack);
      }
      return true;
    }
    v3 H = ImportanceSampleVNDF_GGX(xi, V, n_orient, alpha);
    float eta_ratio = etai / etat;
    L = refract(-V, H, eta_ratio);
    if (length(L) < 0.1f) L = reflect(-V, H);
    else is_transmission = true;
  } else if (rng < total_p) {
    L = ImportanceSampleCosine(xi, n_orient);
  } else {
    return false;
  }
  float dotNL = dot(n_orient, L);
  if (is_transmission) {
    if (dotNL >= 0.0f) return false;
    ray->origin = hit_pos - n_orient * 0.001f;
  } else {
    if (dotNL <= 0.0f) return false;
    ray->origin = hit_pos + n_orient * 0.001f;
  }
  ray->direction = L;
  v3 bsdf_val = eval_surface(V, L, mat, ctx, stack);
  float pdf_val = pdf_surface(V, L, mat, ctx, stack);
  if (pdf_val > 0.0f) *throughput = *throughput * (bsdf_val / pdf_val);
  else return false;
  *last_surface_pdf = pdf_val;
  if (is_transmission) {
    if (entering) {
      v3 sigma = (-vlog(vmax(ctx.albedo, mk3s(0.0001f)))) * mat.concentration;
      Medium m; m.ior = mat.ior; m.sigma = sigma; m.emission = L3(mat.emittance);
      push_medium(stack, m);
    } else {
      pop_medium(stack);
    }
  }
  return true;
}

// shader.wgsl:2177-2189
v3 clamp_firefly(v3 rad, int bounce) {
  if (bounce == 0) return rad;
  float lum = dot(rad, mk3(0.2126f, 0.7152f, 0.0722f));
  if (lum > 20.0f) return rad * (20.0f / lum);
  return rad;
}

// shader.wgsl:2226-2271
v3 evaluate_nee(Ctx& c, const LightSample& ls, v3 hit_pos, v3 n_orient, v3 V, const wgpt_material& mat,
                const SurfaceContext& ctx, const m3& tbn, float currentheight, v2 final_uv,
                const MediumStack* stack, int32_t ignore_obj_idx) {
  if (ls.pdf <= 0.0f) return mk3s(0.0f);
  float dotNL = dot(n_orient, ls.dir);
  if (dotNL <= 0.0f && mat.transmission <= 0.0f) return mk3s(0.0f);
  float bsdf_pdf = pdf_surface(V, ls.dir, mat, ctx, stack);
  float weight = mis_weight(ls.pdf, bsdf_pdf);
  v3 bsdf_val = eval_surface(V, ls.dir, mat, ctx, stack);
  v3 sample_color = ls.color;
  v3 c_weight = (bsdf_val * weight) / wmax(ls.pdf, 1e-6f);
  if (max_component(sample_color * c_weight) < 1e-5f) return mk3s(0.0f);
  v3 ray_offset = dotNL < 0.0f ? -n_orient * 0.001f : n_orient * 0.001f;
  Ray shadow_ray; shadow_ray.origin = hit_pos + ray_offset; shadow_ray.direction = ls.dir;
  bool in_shadow = false;
  if (HAS(c.s, WGPT_HAS_HEIGHTMAPS) && mat.height_idx >= 0) {
    v3 light_ts = normalize(mul3t(tbn, ls.dir));
    if (calculate_shadow_pom(c.s, final_uv, currentheight, light_ts, mat, mat.height_idx).hit) in_shadow = true;
  }
  if (!in_shadow) {
    v3 shadow_hit = trace_scene_shadow(c, shadow_ray, ignore_obj_idx, ls.dist);
    sample_color = sample_color * shadow_hit;
    if (max_component(shadow_hit) < 0.001f) in_shadow = true;
  }
  if (!in_shadow) return sample_color * c_weight;
  return mk3s(0.0f);
}

// shader.wgsl:2273-2492: one invocation of main
void main_pixel(Ctx& c, uint32_t ix, uint32_t iy, float* accum, uint8_t* out) {
  const Scene* s = c.s;
  const wgpt_scene_params* p = c.p;
  uint32_t idx = iy * p->width + ix;
  c.rng = (idx * 1973u + p->sample_number * 9277u + p->seed * 26699u) | 1u;
  rand_pcg(c.rng);
  c.count(C_PATHS);
  float j0 = rand_pcg(c.rng);
  float j1 = rand_pcg(c.rng);
  v2 screen_uv = mk2(((float)ix + j0) / (float)p->width, ((float)iy + j1) / (float)p->height);
  v3 r00 = L3(p->ray00), r10 = L3(p->ray10), r01 = L3(p->ray01), r11 = L3(p->ray11);
  v3 ray_dir = normalize(vmix(vmix(r00, r10, screen_uv.x), vmix(r01, r11, screen_uv.x), 1.0f - screen_uv.y));
  Ray ray; ray.origin = L3(p->eye); ray.direction = ray_dir;
  v3 throughput = mk3s(1.0f);
  v3 radiance = mk3s(0.0f);
  float last_surface_pdf = 1.0f;
  float last_weight_sum = 0.0f;
  MediumStack stack; stack.count = 0;
  for (int m = 0; m < 4; ++m) stack.media[m] = air();

  for (int bounce = 0; bounce < s->bounce_limit; bounce++) {
    SurfaceHit hit = trace_scene(c, ray);
    wgpt_object obj; memset(&obj, 0, sizeof(obj));
    if (hit.o_idx >= 0) obj = s->objs[hit.o_idx];
    Medium current_med = peek_medium(&stack);
    if (current_med.ior > 1.0f || length(current_med.sigma) > 0.0f) {
      float dist = sel(hit.t, 1000.0f, hit.m_idx == -1);
      v3 attenuation = vexp(-current_med.sigma * dist);
      v3 sigma = current_med.sigma;
      float emit_x = sigma.x > 1e-4f ? current_med.emission.x * (1.0f - attenuation.x) / sigma.x : current_med.emission.x * dist;
      float emit_y = sigma.y > 1e-4f ? current_med.emission.y * (1.0f - attenuation.y) / sigma.y : current_med.emission.y * dist;
      float emit_z = sigma.z > 1e-4f ? current_med.emission.z * (1.0f - attenuation.z) / sigma.z : current_med.emission.z * dist;
      v3 incoming = mk3(emit_x, emit_y, emit_z);
      radiance = radiance + throughput * clamp_firefly(incoming, bounce);
      throughput = throughput * attenuation;
    }
    if (hit.m_idx == -1) {
      if (HAS(s, WGPT_HAS_SKYBOX)) {
        v3 sky_color = sample_sky(c, ray.direction);
        float weight = 1.0f;
        if (bounce > 0 && HAS(s, WGPT_MIS_SKYBOX)) {
          float sky_pdf = get_sky_pdf(c, ray.direction);
          weight = mis_weight(last_surface_pdf, sky_pdf);
        }
        v3 incoming = sky_color * weight;
        radiance = radiance + throughput * clamp_firefly(incoming, bounce);
      } else {
        radiance = radiance + throughput * clamp_firefly(mk3(0.02f, 0.03f, 0.05f), bounce);
      }
      break;
    }
    c.count(C_SHADE);
    const wgpt_material& mat = s->mats[hit.m_idx];
    // shader.wgsl:2361-2375
    v2 final_uv = hit.hit_uv * L2(mat.uv_scale);
    m3 tbn; tbn.c[0] = hit.tangent; tbn.c[1] = hit.bitangent; tbn.c[2] = hit.hit_n;
    float currentheight = 0.0f;
    if (HAS(s, WGPT_HAS_HEIGHTMAPS) && mat.height_idx >= 0) {
      v3 view_ts = normalize(mul3t(tbn, -ray.direction));
      if (view_ts.z > 0.0f) {
        PomResult pom = calculate_pom(s, final_uv, view_ts, 0.0f, mat, mat.height_idx);
        final_uv = pom.uv;
        currentheight = pom.height;
      }
    }
    SurfaceContext ctx = get_surface_context(s, hit, mat, tbn, final_uv);
    if (length(ctx.emittance) > 0.0f) {
      float weight = 1.0f;
      if (HAS(s, WGPT_HAS_LIGHTS) && bounce > 0 && hit.o_idx >= 0 && obj.light_idx >= 0) {
        const wgpt_light& light = s->lights[obj.light_idx];
        float raw_light_pdf = get_light_pdf(s, light, obj, ray.origin, ray.direction, hit);
        v3 to_light = L3(obj.world_position) - ray.origin;
        float d2 = wmax(dot(to_light, to_light), 0.001f);
        float light_importance = light.power / d2;
        float selection_pdf = last_weight_sum > 0.0f ? light_importance / last_weight_sum : 0.0f;
        float total_light_pdf = raw_light_pdf * selection_pdf;
        weight = mis_weight(last_surface_pdf, total_light_pdf);
      }
      v3 incoming = ctx.emittance * weight;
      radiance = radiance + throughput * clamp_firefly(incoming, bounce);
      if (length(ctx.emittance) > 1.0f) break;
    }
    v3 hit_pos = ray.origin + ray.direction * hit.t;
    v3 V = -ray.direction;
    v3 n_orient = vsel(-ctx.normal, ctx.normal, dot(ctx.normal, V) > 0.0f);

    if (HAS(s, WGPT_HAS_LIGHTS)) {
      int32_t selected_light_idx = -1;
      float weight_sum = 0.0f;
      float selected_weight = 0.0f;
      uint32_t num_lights = s->n_lights;
      for (uint32_t i = 0u; i < num_lights; i++) {
        const wgpt_light& light = s->lights[i];
        if (light.obj_idx < 0) continue;
        const wgpt_object& l_obj = s->objs[light.obj_idx];
        v3 to_light = L3(l_obj.world_position) - hit_pos;
        float d2 = wmax(dot(to_light, to_light), 0.001f);
        float w = light.power / d2;
        weight_sum += w;
        if (rand_pcg(c.rng) < (w / weight_sum)) { selected_light_idx = (int32_t)i; selected_weight = w; }
      }
      if (selected_light_idx >= 0 && weight_sum > 0.0f) {
        const wgpt_light& light = s->lights[selected_light_idx];
        const wgpt_object& l_obj = s->objs[light.obj_idx];
        LightSample light_sample = sample_light(c, light, l_obj, hit_pos);
        if (light_sample.pdf > 0.0f) {
          float selection_pdf = selected_weight / weight_sum;
          light_sample.pdf *= selection_pdf;
          v3 incoming = evaluate_nee(c, light_sample, hit_pos, n_orient, V, mat, ctx, tbn, currentheight, final_uv,
                                     &stack, light.obj_idx);
          radiance = radiance + throughput * clamp_firefly(incoming, bounce);
        }
      }
      last_weight_sum = weight_sum;
    }
    if (HAS(s, WGPT_HAS_SKYBOX) && HAS(s, WGPT_MIS_SKYBOX)) {
      c.count(C_ENV_NEE);
      float u0 = rand_pcg(c.rng);
      float u1 = rand_pcg(c.rng);
      LightSample env_sample = sample_env_cdf(c, mk2(u0, u1));
      v3 incoming = evaluate_nee(c, env_sample, hit_pos, n_orient, V, mat, ctx, tbn, currentheight, final_uv, &stack,
                                 -1);
      radiance = radiance + throughput * clamp_firefly(incoming, bounce);
    }
    if (!sample_surface(c, &ray, &throughput, hit_pos, mat, ctx, &stack, &last_surface_pdf)) break;
    // shader.wgsl:2458-2472: self-shadowing of the height field along the sampled direction
    if (HAS(s, WGPT_HAS_HEIGHTMAPS) && mat.height_idx >= 0) {
      v3 light_ts = normalize(mul3t(tbn, ray.direction));
      PomResult sh = calculate_shadow_pom(s, final_uv, currentheight, light_ts, mat, mat.height_idx);
      if (sh.hit) {
        final_uv = sh.uv;
        SurfaceContext ctx_pom = get_surface_context(s, hit, mat, tbn, final_uv);
        radiance = radiance + throughput * clamp_firefly(ctx_pom.emittance, bounce);
        if (length(ctx_pom.emittance) > 1.0f) break;
        if (!sample_surface(c, &ray, &throughput, hit_pos, mat, ctx_pom, &stack, &last_surface_pdf)) break;
      }
    }
    if (bounce < 2) continue;
    float pmax = max_component(throughput);
    float survival_prob = clamp(pmax, 0.05f, 0.95f);
    if (rand_pcg(c.rng) > survival_prob) break;
    throughput = throughput / survival_prob;
  }
  if (c.acc64) {   // FP64 Welford record of every sample: mean rgb, M2 rgb, count
    double* w = c.acc64 + (size_t)idx * 8;
    const double n = w[6] + 1.0;
    const double x[3] = {radiance.x, radiance.y, radiance.z};
    for (int k = 0; k < 3; ++k) {
      const double d = x[k] - w[k];
      w[k] += d / n;
      w[3 + k] += d * (x[k] - w[k]);
    }
    w[6] = n;
  }
  float weight = 1.0f / (float)(p->sample_number + 1u);
  float* a = accum + (size_t)idx * 4;
  v3 old_c = mk3(a[0], a[1], a[2]);
  v3 final_c = vmix(old_c, radiance, weight);
  a[0] = final_c.x; a[1] = final_c.y; a[2] = final_c.z; a[3] = 1.0f;
  final_c = final_c * mk3s(p->exposure);
  final_c = final_c / (final_c + mk3s(0.3f));
  final_c = vpow(final_c, 0.4545f);
  uint8_t* o = out + (size_t)idx * 4;
  o[0] = (uint8_t)unorm8(final_c.x); o[1] = (uint8_t)unorm8(final_c.y);
  o[2] = (uint8_t)unorm8(final_c.z); o[3] = 255;
}

// shader.wgsl:2510-2603: one invocation of gbuf_main
void gbuf_pixel(Ctx& c, uint32_t ix, uint32_t iy, float* gbuf, uint8_t* out) {
  const Scene* s = c.s;
  const wgpt_scene_params* p = c.p;
  uint32_t idx = iy * p->width + ix;
  c.rng = (idx * 1973u + p->sample_number * 9277u + p->seed * 26699u) | 1u;
  rand_pcg(c.rng);
  v2 screen_uv = mk2(((float)ix + 0.5f) / (float)p->width, ((float)iy + 0.5f) / (float)p->height);
  v3 r00 = L3(p->ray00), r10 = L3(p->ray10), r01 = L3(p->ray01), r11 = L3(p->ray11);
  v3 ray_dir = normalize(vmix(vmix(r00, r10, screen_uv.x), vmix(r01, r11, screen_uv.x), 1.0f - screen_uv.y));
  Ray ray; ray.origin = L3(p->eye); ray.direction = ray_dir;
  SurfaceContext ctx;
  memset(&ctx, 0, sizeof(ctx));
  wgpt_material mat; memset(&mat, 0, sizeof(mat));
  float dist = 0.0f;
  v3 tint = mk3s(1.0f);
  for (int bounce = 0; bounce < s->bounce_limit; bounce++) {
    SurfaceHit hit = trace_scene(c, ray);
    if (hit.m_idx == -1) {
      ctx.normal = mk3s(0.0f);
      ctx.emittance = sample_sky(c, ray.direction);
      ctx.albedo = mk3s(0.0f);
      break;
    }
    mat = s->mats[hit.m_idx];
    m3 tbn; tbn.c[0] = hit.tangent; tbn.c[1] = hit.bitangent; tbn.c[2] = hit.hit_n;
    v2 final_uv = hit.hit_uv * L2(mat.uv_scale);
    ctx = get_surface_context(s, hit, mat, tbn, final_uv);
    ctx.normal = vsel(-ctx.normal, ctx.normal, dot(ctx.normal, -ray.direction) > 0.0f);
    dist += hit.t;
    if (ctx.alpha < 1.0f) {
      tint = tint * vmix(mk3s(1.0f), ctx.albedo, ctx.alpha);
      ray.origin = (ray.origin + ray.direction * hit.t) - ctx.normal * 0.001f;
      continue;
    }
    if (mat.metallic >= 0.99f && mat.roughness <= 0.01f) {
      tint = tint * ctx.albedo;
      ray.origin = (ray.origin + ray.direction * hit.t) + ctx.normal * 0.001f;
      ray.direction = reflect(ray.direction, ctx.normal);
      continue;
    }
    break;
  }
  v3 color = (ctx.albedo + ctx.emittance) * tint;
  float* g = gbuf + (size_t)idx * 12;
  g[0] = ctx.normal.x; g[1] = ctx.normal.y; g[2] = ctx.normal.z;
  g[3] = ctx.roughness;
  g[4] = color.x; g[5] = color.y; g[6] = color.z;
  g[7] = ctx.metallic;
  // motion (8, 9) is never written by gbuf_main
  g[10] = mat.transmission;
  g[11] = dist;
  v3 o3;
  if (ix < p->width * 1u / 4u) {
    float dd = dist / (dist + 3.0f);
    o3 = mk3s(dd);
  } else if (ix < p->width * 2u / 4u) {
    o3 = ctx.normal * 0.5f + mk3s(0.5f);
  } else if (ix < p->width * 3u / 4u) {
    color = color * mk3s(p->exposure);
    color = color / (color + mk3s(0.3f));
    o3 = vpow(color, 0.4545f);
  } else {
    o3 = mk3(mat.transmission, ctx.roughness, ctx.metallic);
  }
  uint8_t* o = out + (size_t)idx * 4;
  o[0] = (uint8_t)unorm8(o3.x); o[1] = (uint8_t)unorm8(o3.y); o[2] = (uint8_t)unorm8(o3.z); o[3] = 255;
}

void fill_scene(Scene* s, const void* const* bufs, const uint64_t* sizes, const uint32_t* meta) {
  s->mats = (const wgpt_material*)bufs[0]; s->n_mats = (uint32_t)(sizes[0] / WGPT_STRIDE_MATERIAL);
  s->objs = (const wgpt_object*)bufs[1]; s->n_objs = (uint32_t)(sizes[1] / WGPT_STRIDE_OBJECT);
  s->tlas = (const wgpt_bvh_node*)bufs[2]; s->n_tlas = (uint32_t)(sizes[2] / WGPT_STRIDE_NODE);
  s->meshes = (const uint8_t*)bufs[3]; s->n_meshes = (uint32_t)(sizes[3] / WGPT_STRIDE_MESH_READ);
  s->bvh = (const wgpt_bvh_node*)bufs[4]; s->n_bvh = (uint32_t)(sizes[4] / WGPT_STRIDE_NODE);
  s->tris = (const wgpt_triangle*)bufs[5]; s->n_tris = (uint32_t)(sizes[5] / WGPT_STRIDE_TRIANGLE);
  s->planes = (const wgpt_plane*)bufs[6]; s->n_planes = (uint32_t)(sizes[6] / WGPT_STRIDE_PLANE);
  s->lights = (const wgpt_light*)bufs[7]; s->n_lights = (uint32_t)(sizes[7] / WGPT_STRIDE_LIGHT);
  s->cdf = (const float*)bufs[8]; s->n_cdf = (uint32_t)(sizes[8] / 4);
  s->sky = (const uint16_t*)bufs[9];
  s->sky_w = meta[0]; s->sky_h = meta[1];
  s->bounce_limit = (int32_t)meta[2];
  s->flags = meta[3];
  s->tex = (const uint8_t*)bufs[10];
  s->tex_w = meta[4]; s->tex_h = meta[5]; s->tex_layers = meta[6];
}

// denoiser.wgsl:41-50
float lum_dn(v3 c) { return dot(c, mk3(0.299f, 0.587f, 0.114f)); }
v3 tonemap_dn(v3 c, float exposure) {
  v3 color = c * exposure;
  color = color / (color + mk3s(0.3f));
  return vpow(color, 0.4545f);
}
bool is_valid(v3 c) {
  return (c.x >= 0.0f && c.y >= 0.0f && c.z >= 0.0f) && (c.x <= 10000.0f && c.y <= 10000.0f && c.z <= 10000.0f);
}
inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

}  // namespace

extern "C" {

// Renders `reps` dispatches of main over the section [sx, sx+sw) x [sy, sy+sh) with
// sample_number = first_frame + i.  bufs/sizes: materials, objects, tlas, meshes, bvh, triangles,
// planes, lights, sky_cdf, sky texels (rgba16f).  meta: sky_w, sky_h, bounce_limit, flags.
// counters (16 x u64, nullable) receive the algorithmic work counted per category.
int oracle_render(const void* const* bufs, const uint64_t* sizes, const uint32_t* meta,
                  const void* params112, uint32_t first_frame, uint32_t reps,
                  uint32_t sx, uint32_t sy, uint32_t sw, uint32_t sh,
                  float* accum, uint8_t* out, int nthreads, uint64_t* counters) {
  Scene s; fill_scene(&s, bufs, sizes, meta);
  wgpt_scene_params p0; memcpy(&p0, params112, sizeof(p0));
  if (sx + sw > p0.width || sy + sh > p0.height) return 1;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
  int err = 0;
  for (uint32_t r = 0; r < reps; ++r) {
    wgpt_scene_params p = p0;
    p.sample_number = first_frame + r;
    const long long npix = (long long)sw * sh;
#pragma omp parallel reduction(| : err)
    {
      uint64_t local[C_NCOUNTERS] = {0};
      Ctx c; c.s = &s; c.p = &p; c.rng = 0; c.cnt = counters ? local : nullptr; c.err = 0;
#pragma omp for schedule(dynamic, 64)
      for (long long k = 0; k < npix; ++k) {
        uint32_t ix = sx + (uint32_t)(k % sw), iy = sy + (uint32_t)(k / sw);
        main_pixel(c, ix, iy, accum, out);
      }
      err |= c.err;
      if (counters) {
#pragma omp critical
        for (int i = 0; i < C_NCOUNTERS; ++i) counters[i] += local[i];
      }
    }
  }
  return err ? 2 : 0;
}

// oracle_render with every sample also folded into a per-pixel FP64 Welford record (acc8: 8
// doubles per pixel of the params' image: mean r g b, sum of squared deviations r g b, count,
// unused; zero it before the first call).  The paths run in FP32 as in the reference; only the
// accumulation over samples is FP64.  The FP32 running mean goes into a scratch image.
int oracle_render_f64(const void* const* bufs, const uint64_t* sizes, const uint32_t* meta,
                      const void* params112, uint32_t first_frame, uint32_t reps,
                      uint32_t sx, uint32_t sy, uint32_t sw, uint32_t sh, double* acc8, int nthreads) {
  Scene s; fill_scene(&s, bufs, sizes, meta);
  wgpt_scene_params p0; memcpy(&p0, params112, sizeof(p0));
  if (sx + sw > p0.width || sy + sh > p0.height) return 1;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
  std::vector<float> accum((size_t)p0.width * p0.height * 4, 0.0f);
  std::vector<uint8_t> out((size_t)p0.width * p0.height * 4, 0);
  int err = 0;
  const long long npix = (long long)sw * sh;
#pragma omp parallel reduction(| : err)
  {
    // pixels are split over the threads and each thread runs all samples of its pixels, so
    // every Welford record is updated by one thread in sample order
#pragma omp for schedule(dynamic, 4)
    for (long long k = 0; k < npix; ++k) {
      uint32_t ix = sx + (uint32_t)(k % sw), iy = sy + (uint32_t)(k / sw);
      for (uint32_t r = 0; r < reps; ++r) {
        wgpt_scene_params p = p0;
        p.sample_number = first_frame + r;
        Ctx c; c.s = &s; c.p = &p; c.rng = 0; c.cnt = nullptr; c.err = 0; c.acc64 = acc8;
        main_pixel(c, ix, iy, accum.data(), out.data());
        err |= c.err;
      }
    }
  }
  return err ? 2 : 0;
}

// One dispatch of gbuf_main.  gbuf receives 12 floats (48 bytes) per pixel.
int oracle_gbuffer(const void* const* bufs, const uint64_t* sizes, const uint32_t* meta,
                   const void* params112, uint32_t sx, uint32_t sy, uint32_t sw, uint32_t sh,
                   float* gbuf, uint8_t* out, int nthreads) {
  Scene s; fill_scene(&s, bufs, sizes, meta);
  wgpt_scene_params p; memcpy(&p, params112, sizeof(p));
  if (sx + sw > p.width || sy + sh > p.height) return 1;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
  int err = 0;
  const long long npix = (long long)sw * sh;
#pragma omp parallel reduction(| : err)
  {
    Ctx c; c.s = &s; c.p = &p; c.rng = 0; c.cnt = nullptr; c.err = 0;
#pragma omp for schedule(dynamic, 64)
    for (long long k = 0; k < npix; ++k) {
      uint32_t ix = sx + (uint32_t)(k % sw), iy = sy + (uint32_t)(k / sw);
      gbuf_pixel(c, ix, iy, gbuf, out);
    }
    err |= c.err;
  }
  return err ? 2 : 0;
}

// Closest hit of arbitrary rays (trace_scene, shader.wgsl:754-774).  rays: n x 6 floats
// (origin, direction).  Outputs per ray: object index (-1 plane/miss), material index (-1 miss),
// global triangle index (-1 if not a mesh hit), t (1e10 on a miss), world normal (3 floats).
int oracle_trace_closest(const void* const* bufs, const uint64_t* sizes, const uint32_t* meta,
                         const float* rays, uint32_t n, int32_t* o_idx, int32_t* m_idx,
                         int32_t* prim, float* t, float* normal, int nthreads) {
  Scene s; fill_scene(&s, bufs, sizes, meta);
  wgpt_scene_params p; memset(&p, 0, sizeof(p));
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
#pragma omp parallel for schedule(dynamic, 256)
  for (long long i = 0; i < (long long)n; ++i) {
    Ctx c; c.s = &s; c.p = &p; c.rng = 0; c.cnt = nullptr; c.err = 0;
    Ray r; r.origin = mk3(rays[i * 6 + 0], rays[i * 6 + 1], rays[i * 6 + 2]);
    r.direction = mk3(rays[i * 6 + 3], rays[i * 6 + 4], rays[i * 6 + 5]);
    SurfaceHit h = trace_scene(c, r);
    o_idx[i] = h.o_idx; m_idx[i] = h.m_idx; prim[i] = h.prim; t[i] = h.t;
    normal[i * 3 + 0] = h.hit_n.x; normal[i * 3 + 1] = h.hit_n.y; normal[i * 3 + 2] = h.hit_n.z;
  }
  return 0;
}

// BSDF tables: eval_surface / pdf_surface (shader.wgsl:1831-2047) for n (V, L) pairs against one
// material and a surface normal, with an empty medium stack (air outside).
int oracle_bsdf(const void* material144, const float* normal3, float roughness, float metallic,
                const float* albedo3, const float* vl, uint32_t n, float* f_out, float* pdf_out) {
  wgpt_material mat; memcpy(&mat, material144, sizeof(mat));
  SurfaceContext ctx;
  ctx.normal = mk3(normal3[0], normal3[1], normal3[2]);
  ctx.surface_normal = ctx.normal;
  ctx.albedo = mk3(albedo3[0], albedo3[1], albedo3[2]);
  ctx.roughness = roughness; ctx.metallic = metallic;
  ctx.emittance = L3(mat.emittance); ctx.alpha = 1.0f;
  MediumStack st; st.count = 0;
  for (uint32_t i = 0; i < n; ++i) {
    v3 V = mk3(vl[i * 6 + 0], vl[i * 6 + 1], vl[i * 6 + 2]);
    v3 L = mk3(vl[i * 6 + 3], vl[i * 6 + 4], vl[i * 6 + 5]);
    v3 f = eval_surface(V, L, mat, ctx, &st);
    f_out[i * 3 + 0] = f.x; f_out[i * 3 + 1] = f.y; f_out[i * 3 + 2] = f.z;
    pdf_out[i] = pdf_surface(V, L, mat, ctx, &st);
  }
  return 0;
}

// Environment samples (sample_env_cdf, shader.wgsl:231-254) of n random pairs: the texel the two
// CDF searches pick, as (x, y), and the sample's pdf.  params: the 112-byte SceneParams.
int oracle_sample_env(const void* const* bufs, const uint64_t* sizes, const uint32_t* meta, const void* params112,
                      const float* u2, uint32_t n, uint32_t* texel_xy, float* pdf) {
  Scene s; fill_scene(&s, bufs, sizes, meta);
  wgpt_scene_params p; memcpy(&p, params112, sizeof(p));
  for (uint32_t i = 0; i < n; ++i) {
    Ctx c; c.s = &s; c.p = &p; c.rng = 0; c.cnt = nullptr; c.err = 0;
    const v2 u = mk2(u2[2 * i], u2[2 * i + 1]);
    const uint32_t v_idx = binary_search_cdf(c, 0u, p.sky_height, u.y);
    const uint32_t u_idx = binary_search_cdf(c, p.sky_cdf_index + v_idx * (p.sky_width + 1u), p.sky_width, u.x);
    texel_xy[2 * i] = u_idx;
    texel_xy[2 * i + 1] = v_idx;
    pdf[i] = sample_env_cdf(c, u).pdf;
  }
  return 0;
}

// One call of sample_surface (shader.wgsl:2052-2175) for a ray arriving along -V at a surface
// with the given normal, material and context, in air with an empty medium stack, the random
// stream starting at `rng_state`.  Writes the new ray direction, the throughput it carries
// (starting from 1) and the return value (1 = the path continues).
int oracle_sample_surface(const void* material144, const float* normal3, float roughness, float metallic,
                          const float* albedo3, const float* V3, uint32_t rng_state, float* dir_out,
                          float* throughput_out) {
  wgpt_material mat; memcpy(&mat, material144, sizeof(mat));
  SurfaceContext ctx;
  ctx.normal = mk3(normal3[0], normal3[1], normal3[2]);
  ctx.surface_normal = ctx.normal;
  ctx.albedo = mk3(albedo3[0], albedo3[1], albedo3[2]);
  ctx.roughness = roughness; ctx.metallic = metallic;
  ctx.emittance = L3(mat.emittance); ctx.alpha = 1.0f;
  MediumStack st; st.count = 0;
  Scene s; memset(&s, 0, sizeof(s));
  wgpt_scene_params p; memset(&p, 0, sizeof(p));
  Ctx c; c.s = &s; c.p = &p; c.rng = rng_state; c.cnt = nullptr; c.err = 0;
  Ray ray; ray.origin = mk3s(0.0f); ray.direction = -mk3(V3[0], V3[1], V3[2]);
  v3 tp = mk3s(1.0f);
  float last_pdf = 0.0f;
  const bool cont = sample_surface(c, &ray, &tp, mk3s(0.0f), mat, ctx, &st, &last_pdf);
  dir_out[0] = ray.direction.x; dir_out[1] = ray.direction.y; dir_out[2] = ray.direction.z;
  throughput_out[0] = tp.x; throughput_out[1] = tp.y; throughput_out[2] = tp.z;
  return cont ? 1 : 0;
}

// The PCG stream of one pixel (shader.wgsl:146-154, 2280-2282) after the seeding discard.
void oracle_rng_stream(uint32_t idx, uint32_t sample_number, uint32_t seed, uint32_t n, float* out) {
  uint32_t st = (idx * 1973u + sample_number * 9277u + seed * 26699u) | 1u;
  rand_pcg(st);
  for (uint32_t i = 0; i < n; ++i) out[i] = rand_pcg(st);
}

// Denoiser: prepass_main, atrous_main x passes (step widths from `steps`), composite_main.
// color: W*H*4 f32 (the accumulation buffer), gbuf: W*H*12 f32, uniforms: 48 bytes.
// filtered: W*H*4 f32 receives the buffer composite_main reads; composited: W*H*4 f32 the
// composited colour before conversion; out: W*H*4 rgba8.
int oracle_denoise(const float* color, const float* gbuf, const void* uniforms48,
                   const uint32_t* steps, uint32_t passes, float* filtered, float* composited,
                   uint8_t* out, int nthreads) {
  wgpt_denoise_uniforms u; memcpy(&u, uniforms48, sizeof(u));
  const int W = (int)u.width, H = (int)u.height;
  const size_t npix = (size_t)W * H;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
  std::vector<float> A(npix * 4), B(npix * 4);
  auto G = [&](size_t i) { return gbuf + i * 12; };
  // denoiser.wgsl:55-112
#pragma omp parallel for schedule(static)
  for (long long k = 0; k < (long long)npix; ++k) {
    int x = (int)(k % W), y = (int)(k / W);
    size_t idx = (size_t)y * W + x;
    v4 center_c;
    bool use_median = (u.flags & 1u) != 0u;
    if (use_median) {
      v4 colors[9]; float lums[9]; int kk = 0;
      for (int dy = -1; dy <= 1; dy++) {
        for (int dx = -1; dx <= 1; dx++) {
          int cx = clampi(x + dx, 0, W - 1), cy = clampi(y + dy, 0, H - 1);
          const float* cp = color + ((size_t)cy * W + cx) * 4;
          colors[kk] = mk4(cp[0], cp[1], cp[2], cp[3]);
          lums[kk] = lum_dn(xyz(colors[kk]));
          kk++;
        }
      }
      for (int i = 0; i < 5; i++) {
        for (int j = i + 1; j < 9; j++) {
          if (lums[j] < lums[i]) {
            float tl = lums[i]; lums[i] = lums[j]; lums[j] = tl;
            v4 tc = colors[i]; colors[i] = colors[j]; colors[j] = tc;
          }
        }
      }
      center_c = colors[4];
    } else {
      const float* cp = color + idx * 4;
      center_c = mk4(cp[0], cp[1], cp[2], cp[3]);
    }
    if (!is_valid(xyz(center_c))) center_c = mk4(0.0f, 0.0f, 0.0f, center_c.w);
    v3 mapped_c = tonemap_dn(xyz(center_c), u.exposure);
    bool demodulate = (u.flags & 2u) != 0u;
    const float* g = G(idx);
    bool is_sky = length(mk3(g[0], g[1], g[2])) < 0.1f;
    if (demodulate && !is_sky) {
      v3 mapped_albedo = vmax(tonemap_dn(mk3(g[4], g[5], g[6]), u.exposure), mk3s(0.001f));
      mapped_c = mapped_c / mapped_albedo;
      mapped_c = vmin(vmax(mapped_c, mk3s(0.0f)), mk3s(10.0f));
    }
    float* o = &A[idx * 4];
    o[0] = mapped_c.x; o[1] = mapped_c.y; o[2] = mapped_c.z; o[3] = center_c.w;
  }
  // denoiser.wgsl:117-189
  const float kernel[5] = {0.0625f, 0.25f, 0.375f, 0.25f, 0.0625f};
  float* in = A.data();
  float* outb = B.data();
  for (uint32_t pass = 0; pass < passes; ++pass) {
    const int step = (int)steps[pass];
#pragma omp parallel for schedule(static)
    for (long long k = 0; k < (long long)npix; ++k) {
      int x = (int)(k % W), y = (int)(k / W);
      size_t ci = (size_t)y * W + x;
      const float* cc = in + ci * 4;
      v4 c_color = mk4(cc[0], cc[1], cc[2], cc[3]);
      const float* cg = G(ci);
      v3 c_n = mk3(cg[0], cg[1], cg[2]);
      float c_rough = cg[3], c_metal = cg[7], c_trans = cg[10], c_dist = cg[11];
      v3 c_alb = mk3(cg[4], cg[5], cg[6]);
      v4 sum_color = mk4(0.0f, 0.0f, 0.0f, 0.0f);
      float sum_weight = 0.0f;
      float preserve = (1.0f - c_rough) * wmax(c_metal, c_trans);
      float attenuation = mix(1.0f, 0.0f, preserve * u.glossy_protect);
      for (int dy = -2; dy <= 2; dy++) {
        for (int dx = -2; dx <= 2; dx++) {
          int sxp = clampi(x + dx * step, 0, W - 1), syp = clampi(y + dy * step, 0, H - 1);
          size_t si = (size_t)syp * W + sxp;
          const float* sc = in + si * 4;
          v4 s_color = mk4(sc[0], sc[1], sc[2], sc[3]);
          const float* sg = G(si);
          float h = kernel[dx + 2] * kernel[dy + 2];
          v3 c_diff = xyz(c_color) - xyz(s_color);
          float w_color = exp_(-dot(c_diff, c_diff) / (u.sigma_color * u.sigma_color + 1e-5f));
          float w_normal = 1.0f;
          v3 s_n = mk3(sg[0], sg[1], sg[2]);
          float c_n_len = length(c_n);
          float s_n_len = length(s_n);
          if (c_n_len > 0.1f || s_n_len > 0.1f) {
            float n_dot = wmax(0.0f, dot(c_n, s_n));
            w_normal = pow_(n_dot, u.sigma_normal);
          }
          float c_d_mapped = c_dist / (c_dist + 3.0f);
          float s_d_mapped = sg[11] / (sg[11] + 3.0f);
          float d_diff = c_d_mapped - s_d_mapped;
          float w_depth = exp_(-(d_diff * d_diff) / (u.sigma_depth * u.sigma_depth + 1e-5f));
          v3 c_a_mapped = tonemap_dn(c_alb, u.exposure);
          v3 s_a_mapped = tonemap_dn(mk3(sg[4], sg[5], sg[6]), u.exposure);
          v3 a_diff = c_a_mapped - s_a_mapped;
          float w_albedo = exp_(-dot(a_diff, a_diff) / (u.sigma_albedo * u.sigma_albedo + 1e-5f));
          v3 c_mat = mk3(c_trans, c_rough, c_metal);
          v3 s_mat = mk3(sg[10], sg[3], sg[7]);
          v3 m_diff = c_mat - s_mat;
          float w_material = exp_(-dot(m_diff, m_diff) / (u.sigma_material * u.sigma_material + 1e-5f));
          float weight = h * w_color * w_normal * w_depth * w_albedo * w_material;
          if (dx != 0 || dy != 0) weight *= attenuation;
          sum_color = sum_color + s_color * weight;
          sum_weight += weight;
        }
      }
      v4 r = sum_color / (sum_weight + 1e-5f);
      float* o = outb + ci * 4;
      o[0] = r.x; o[1] = r.y; o[2] = r.z; o[3] = r.w;
    }
    float* tmp = in; in = outb; outb = tmp;
  }
  // denoiser.wgsl:194-213
  memcpy(filtered, in, npix * 4 * sizeof(float));
#pragma omp parallel for schedule(static)
  for (long long k = 0; k < (long long)npix; ++k) {
    const float* fc = in + (size_t)k * 4;
    v4 final_c = mk4(fc[0], fc[1], fc[2], fc[3]);
    const float* g = G((size_t)k);
    bool demodulate = (u.flags & 2u) != 0u;
    bool is_sky = length(mk3(g[0], g[1], g[2])) < 0.1f;
    if (demodulate && !is_sky) {
      v3 mapped_albedo = vmax(tonemap_dn(mk3(g[4], g[5], g[6]), u.exposure), mk3s(0.001f));
      v3 rgb = xyz(final_c) * mapped_albedo;
      final_c = mk4(rgb, final_c.w);
    }
    float* cp = composited + (size_t)k * 4;
    cp[0] = final_c.x; cp[1] = final_c.y; cp[2] = final_c.z; cp[3] = final_c.w;
    uint8_t* o = out + (size_t)k * 4;
    o[0] = (uint8_t)unorm8(final_c.x); o[1] = (uint8_t)unorm8(final_c.y);
    o[2] = (uint8_t)unorm8(final_c.z); o[3] = (uint8_t)unorm8(final_c.w);
  }
  return 0;
}

// scale.wgsl:6-35.  src: src_w x src_h rgba8, dst: dst_w x dst_h rgba8.
int oracle_resample(const uint8_t* src, uint32_t src_w, uint32_t src_h, uint8_t* dst,
                    uint32_t dst_w, uint32_t dst_h, float ratio_x, float ratio_y) {
  for (uint32_t y = 0; y < dst_h; ++y) {
    for (uint32_t x = 0; x < dst_w; ++x) {
      v2 uv = mk2((float)x / (float)dst_w, (float)y / (float)dst_h);
      v2 sp = mk2(uv.x * ratio_x * (float)src_w - 0.5f, uv.y * ratio_y * (float)src_h - 0.5f);
      v2 f = mk2(fract(sp.x), fract(sp.y));
      int bx = (int)floorf(sp.x), by = (int)floorf(sp.y);
      int mx = (int)src_w - 1, my = (int)src_h - 1;
      auto tl = [&](int tx, int ty) {
        tx = clampi(tx, 0, mx); ty = clampi(ty, 0, my);
        const uint8_t* t = src + ((size_t)ty * src_w + tx) * 4;
        return mk4((float)t[0] / 255.0f, (float)t[1] / 255.0f, (float)t[2] / 255.0f, (float)t[3] / 255.0f);
      };
      v4 t00 = tl(bx, by), t10 = tl(bx + 1, by), t01 = tl(bx, by + 1), t11 = tl(bx + 1, by + 1);
      v4 col = vmix4(vmix4(t00, t10, f.x), vmix4(t01, t11, f.x), f.y);
      uint8_t* o = dst + ((size_t)y * dst_w + x) * 4;
      o[0] = (uint8_t)unorm8(col.x); o[1] = (uint8_t)unorm8(col.y); o[2] = (uint8_t)unorm8(col.z); o[3] = 255;
    }
  }
  return 0;
}

// Elementary-function probe for the accuracy tests: op 0 sin, 1 cos, 2 exp, 3 log, 4 exp2, 5 log2,
// 6 atan2(x, y2), 7 asin, 8 acos, 9 pow(x, y2).
// textureSampleLevel of layer `layer` of an rgba8 array (w x h x layers) at n texture
// coordinates uv (2 floats each); out: 4 floats each.
void oracle_sample_texture(const uint8_t* tex, uint32_t w, uint32_t h, uint32_t layers, int32_t layer,
                           const float* uv, uint32_t n, float* out) {
  Scene s;
  memset(&s, 0, sizeof s);
  s.tex = tex; s.tex_w = w; s.tex_h = h; s.tex_layers = layers;
  for (uint32_t i = 0; i < n; ++i) {
    v4 c = sample_texture(&s, layer, mk2(uv[2 * i], uv[2 * i + 1]));
    out[4 * i] = c.x; out[4 * i + 1] = c.y; out[4 * i + 2] = c.z; out[4 * i + 3] = c.w;
  }
}

void oracle_builtin(int op, const float* x, const float* y2, uint32_t n, float* out) {
  for (uint32_t i = 0; i < n; ++i) {
    float v = x[i];
    float r = 0.0f;
    switch (op) {
      case 0: r = sin_(v); break;
      case 1: r = cos_(v); break;
      case 2: r = exp_(v); break;
      case 3: r = log_(v); break;
      case 4: r = exp2_(v); break;
      case 5: r = log2_(v); break;
      case 6: r = atan2_(v, y2[i]); break;
      case 7: r = asin_(v); break;
      case 8: r = acos_(v); break;
      case 9: r = pow_(v, y2[i]); break;
      default: r = 0.0f;
    }
    out[i] = r;
  }
}

}  // extern "C"
