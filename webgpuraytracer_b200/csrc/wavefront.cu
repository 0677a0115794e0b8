// Wavefront form of the progressive renderer's path tracing (shader.wgsl main, 2273-2492).
//
// A sample of a section is rendered by a sequence of small kernels over compacted path queues
// instead of one thread running a whole path:
//   k_wf_raygen       per pixel: RNG seed and discard, jittered camera ray, path state
//   per bounce b:
//     k_wf_extend     closest hit of every live path (two-level BVH, planes, list meshes)
//     k_wf_shade_miss walks the live queue in order: queues surface hits, shades paths that left
//                     the scene (media and the sky term)
//     k_wf_shade      surface hits: media, emission, light and environment NEE set-up, BSDF
//                     sampling, Russian roulette; appends surviving paths to the next queue and
//                     records up to two next-event contributions with their shadow rays
//     k_wf_shadow     traces the recorded shadow rays (their own compacted queue, fetched
//                     dynamically by warps) and stores one visibility byte per record
//     k_wf_resolve    adds the next-event contributions (light first, then environment, as main
//                     does), then accumulates finished paths into the running mean and the rgba8
//                     image
// Each stage keeps only its own code and registers resident, so warps stay converged on one
// code path and the instruction cache holds the stage (the single-kernel form stalls on
// instruction fetch).  Every floating-point operation and random draw happens in the order of
// the reference; only the place where it happens changes, so results equal the single-kernel
// form and the CPU restatement bit for bit.
#include <algorithm>
#include "pt_device.cuh"
#include "traverse.cuh"
#include "wgpt_internal.h"

namespace pt {

struct WfBuffers {
  float4* ray_o;     // origin.xyz
  float4* ray_d;     // direction.xyz
  float4* tp;        // throughput.xyz, last_surface_pdf
  float4* rad;       // radiance.xyz, last_weight_sum
  uint4* meta;       // rng, flags, bounce of the pending records, medium count
  float4* med;       // 8 per path: (ior, sigma.xyz), (emission.xyz, -) for media 0..3
  uint4* hit;        // 2 per path: (t, m_idx, o_idx, kind), (id, aux, bu, bv)
  float4* nee;       // 4 per path: (tp.xyz, -), (incoming.xyz, -) for the light and env records
  float4* shadow;    // 4 per path: (origin.xyz, target_dist), (direction.xyz, ignore_idx) x 2
  uint8_t* vis;      // 2 per path: 1 if the record's shadow ray reached its light
  uint32_t* queue[2];
  uint32_t* shq;     // shadow-ray queue: slot * 2 + record
  uint32_t* hitq;    // paths of the current bounce that hit a surface
  uint32_t* missq;   // paths of the current bounce that left the scene
  uint32_t* counts;  // counts[c * 256 + b] for bounce b and counter c (see enum Cnt)
};

enum Cnt : int { CNT_LIVE = 0, CNT_EXT_CURSOR = 1, CNT_HIT = 2, CNT_MISS = 3, CNT_SHADOW = 4, CNT_SH_CURSOR = 5,
                 CNT_KINDS = 6 };

// meta.y flags
enum : uint32_t {
  F_ALIVE = 1u,          // continues to the next bounce
  F_NEE_LIGHT = 2u,      // a light NEE contribution was recorded this bounce
  F_NEE_ENV = 4u,        // an environment NEE contribution was recorded this bounce
  F_SHADOW_LIGHT = 8u,   // ... and it needs its shadow ray traced
  F_SHADOW_ENV = 16u
};

struct WfArgs {
  DScene s;
  DPairs P;
  DParams p;
  WfBuffers b;
  uint32_t sec_w, sec_h;
  uint32_t sample_number;
  float4* accum;
  uchar4* out;
  uint32_t out_pitch;
  uint32_t* status;
  unsigned long long* counters;
};

__device__ __forceinline__ void px_of(const WfArgs& a, uint32_t slot, uint32_t& ix, uint32_t& iy) {
  ix = a.p.sec_x + slot % a.sec_w;
  iy = a.p.sec_y + slot / a.sec_w;
}

template <bool COUNT>
__device__ __forceinline__ void flush_wf(Counters<COUNT>& cn, unsigned long long* counters, bool lane_active) {
  if (!COUNT) return;
  (void)lane_active;
#pragma unroll
  for (int k = 0; k < C_NCOUNTERS; ++k) {
    unsigned long long v = cn.v[k];
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(counters + k, v);
  }
}

// Warp-aggregated append of `slot` to a queue.
__device__ __forceinline__ void queue_push(uint32_t* q, uint32_t* count, uint32_t slot, bool push) {
  unsigned mask = __ballot_sync(0xffffffffu, push);
  if (!mask) return;
  int lane = threadIdx.x & 31;
  int leader = __ffs(mask) - 1;
  uint32_t base = 0;
  if (lane == leader) base = atomicAdd(count, (uint32_t)__popc(mask));
  base = __shfl_sync(0xffffffffu, base, leader);
  if (push) q[base + __popc(mask & ((1u << lane) - 1u))] = slot;
}

// ---------------------------------------------------------------------------- raygen
template <bool COUNT>
__global__ void __launch_bounds__(256) k_wf_raygen(WfArgs a) {
  Counters<COUNT> cn; cn.init();
  uint32_t n = a.sec_w * a.sec_h;
  for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    uint32_t slot = base + threadIdx.x;
    if (slot < n) {
      uint32_t ix, iy;
      px_of(a, slot, ix, iy);
      uint32_t idx = iy * a.p.width + ix;
      uint32_t rng = (idx * 1973u + a.sample_number * 9277u + a.p.seed * 26699u) | 1u;
      rand_pcg(rng);
      cn.add(C_PATHS);
      float j0 = rand_pcg(rng);
      float j1 = rand_pcg(rng);
      float su = ((float)ix + j0) / (float)a.p.width;
      float sv = ((float)iy + j1) / (float)a.p.height;
      v3 d = normalize(vmix(vmix(a.p.ray00, a.p.ray10, su), vmix(a.p.ray01, a.p.ray11, su), 1.0f - sv));
      a.b.ray_o[slot] = make_float4(a.p.eye.x, a.p.eye.y, a.p.eye.z, 0.0f);
      a.b.ray_d[slot] = make_float4(d.x, d.y, d.z, 0.0f);
      a.b.tp[slot] = make_float4(1.0f, 1.0f, 1.0f, 1.0f);
      a.b.rad[slot] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      a.b.meta[slot] = make_uint4(rng, 0u, 0u, 0u);
      a.b.queue[0][slot] = slot;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) a.b.counts[CNT_LIVE * 256] = n;
  flush_wf<COUNT>(cn, a.counters, true);
}

// ---------------------------------------------------------------------------- extend
constexpr unsigned FULL = 0xffffffffu;

// Hands queue entries to the lanes of a warp that have no ray, from a shared cursor; returns the
// entry index for this lane (>= n when there is none).  `exhausted` becomes true (warp-uniform)
// once the queue has been handed out completely.
__device__ __forceinline__ uint32_t refill(bool have, uint32_t* cursor, uint32_t n, bool& exhausted) {
  uint32_t qi = 0xffffffffu;
  unsigned need = __ballot_sync(FULL, !have);
  if (need) {
    int lane = threadIdx.x & 31;
    int leader = __ffs(need) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(cursor, (uint32_t)__popc(need));
    base = __shfl_sync(FULL, base, leader);
    if (!have) qi = base + (uint32_t)__popc(need & ((1u << lane) - 1u));
    if (base + (uint32_t)__popc(need) >= n) exhausted = true;
  }
  return qi;
}

template <bool COUNT>
__global__ void __launch_bounds__(256) k_wf_extend(WfArgs a, const uint32_t* __restrict__ q, const uint32_t* count_ptr,
                                                   uint32_t* cursor) {
  Counters<COUNT> cn; cn.init();
  uint32_t err = 0;
  const uint32_t n = *count_ptr;
  ClosestTrav t;
  bool have = false, exhausted = false;
  uint32_t slot = 0;
  while (true) {
    if (!exhausted) {
      uint32_t qi = refill(have, cursor, n, exhausted);
      if (!have && qi < n) {
        slot = q[qi];
        float4 o = a.b.ray_o[slot], d = a.b.ray_d[slot];
        t.rw.origin = mk3(o.x, o.y, o.z);
        t.rw.direction = mk3(d.x, d.y, d.z);
        closest_init<COUNT>(a.s, t, cn);
        have = true;
      }
    }
    if (!__any_sync(FULL, have)) break;
    if (have && closest_step<COUNT>(a.s, a.P, t, err, cn)) {
      closest_finish<COUNT>(a.s, t, err, cn);
      const HitRec& h = t.hit;
      a.b.hit[slot * 2 + 0] = make_uint4(__float_as_uint(h.t), (uint32_t)h.m_idx, (uint32_t)h.o_idx, (uint32_t)h.kind);
      a.b.hit[slot * 2 + 1] = make_uint4((uint32_t)h.id, (uint32_t)h.aux, __float_as_uint(h.bu), __float_as_uint(h.bv));
      have = false;
    }
  }
  flush_wf<COUNT>(cn, a.counters, true);
  if (err) atomicOr(a.status, err);
}

// ---------------------------------------------------------------------------- shade
__device__ __forceinline__ void load_stack(const WfArgs& a, uint32_t slot, uint32_t count, MediumStack& st) {
  st.count = (int32_t)count;
  for (uint32_t m = 0; m < count; ++m) {
    float4 x = a.b.med[slot * 8 + m * 2], y = a.b.med[slot * 8 + m * 2 + 1];
    st.media[m].ior = x.x; st.media[m].sigma = mk3(x.y, x.z, x.w); st.media[m].emission = mk3(y.x, y.y, y.z);
  }
}
__device__ __forceinline__ void store_medium(const WfArgs& a, uint32_t slot, uint32_t m, const Medium& md) {
  a.b.med[slot * 8 + m * 2] = make_float4(md.ior, md.sigma.x, md.sigma.y, md.sigma.z);
  a.b.med[slot * 8 + m * 2 + 1] = make_float4(md.emission.x, md.emission.y, md.emission.z, 0.0f);
}

// Beer-Lambert attenuation and emission of the medium the path travels in (shader.wgsl:2327-2342).
__device__ __forceinline__ void apply_medium(const MediumStack& stack, const HitRec& hit, int bounce, v3& throughput,
                                             v3& radiance) {
  if (stack.count > 0) {
    Medium cm = peek_medium(stack);
    if (cm.ior > 1.0f || length(cm.sigma) > 0.0f) {
      float dist = hit.m_idx == -1 ? 1000.0f : hit.t;
      v3 attenuation = vexp(-cm.sigma * dist);
      float ex = cm.sigma.x > 1e-4f ? cm.emission.x * (1.0f - attenuation.x) / cm.sigma.x : cm.emission.x * dist;
      float ey = cm.sigma.y > 1e-4f ? cm.emission.y * (1.0f - attenuation.y) / cm.sigma.y : cm.emission.y * dist;
      float ez = cm.sigma.z > 1e-4f ? cm.emission.z * (1.0f - attenuation.z) / cm.sigma.z : cm.emission.z * dist;
      radiance = radiance + throughput * clamp_firefly(mk3(ex, ey, ez), bounce);
      throughput = throughput * attenuation;
    }
  }
}

// Walks the bounce's live queue in order: paths that hit a surface go to the hit queue (kept in
// queue order within each warp, so the surface stage and the next bounce see rays as coherent as
// the camera's); paths that left the scene are shaded here: medium, then the sky (MIS-weighted
// after the first bounce) or the background colour (shader.wgsl:2344-2358).  They end here.
template <bool COUNT>
__global__ void __launch_bounds__(256) k_wf_shade_miss(WfArgs a, int bounce, const uint32_t* __restrict__ q,
                                                       const uint32_t* count_ptr, uint32_t* hit_count) {
  Counters<COUNT> cn; cn.init();
  const DScene& s = a.s;
  uint32_t n = *count_ptr;
  for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    uint32_t i = base + threadIdx.x;
    bool is_hit = false;
    uint32_t slot = 0;
    if (i < n) {
      slot = q[i];
      is_hit = (int32_t)a.b.hit[slot * 2].y != -1;
    }
    queue_push(a.b.hitq, hit_count, slot, is_hit);
    if (i < n && !is_hit) {
      float4 d4 = a.b.ray_d[slot], tp4 = a.b.tp[slot], rd4 = a.b.rad[slot];
      uint4 meta = a.b.meta[slot];
      HitRec hit;
      hit.m_idx = -1; hit.t = __uint_as_float(a.b.hit[slot * 2].x);
      v3 dir = mk3(d4.x, d4.y, d4.z);
      v3 throughput = mk3(tp4.x, tp4.y, tp4.z);
      v3 radiance = mk3(rd4.x, rd4.y, rd4.z);
      if (meta.w > 0u) {
        MediumStack stack;
        load_stack(a, slot, meta.w, stack);
        apply_medium(stack, hit, bounce, throughput, radiance);
      }
      if (HAS(s, WGPT_HAS_SKYBOX)) {
        v3 sky_color = sample_sky(s, dir, cn);
        float weight = 1.0f;
        if (bounce > 0 && HAS(s, WGPT_MIS_SKYBOX)) {
          float sky_pdf = get_sky_pdf(s, a.p, dir, cn);
          weight = mis_weight(tp4.w, sky_pdf);
        }
        radiance = radiance + throughput * clamp_firefly(sky_color * weight, bounce);
      } else {
        radiance = radiance + throughput * clamp_firefly(mk3(0.02f, 0.03f, 0.05f), bounce);
      }
      a.b.rad[slot] = make_float4(radiance.x, radiance.y, radiance.z, rd4.w);
      a.b.meta[slot] = make_uint4(meta.x, 0u, (uint32_t)bounce, meta.w);
    }
  }
  flush_wf<COUNT>(cn, a.counters, true);
}

// Records one next-event contribution: the throughput it is weighted by, the incoming
// radiance if the light is visible, and the shadow ray to test (when evaluate_nee reaches it).
template <bool COUNT>
__device__ void record_nee(const WfArgs& a, uint32_t slot, int rec, const LightSample& ls, v3 hit_pos, v3 n_orient,
                           v3 V, const DMat& mat, const SurfCtx& ctx, const MediumStack& stack, int32_t ignore_idx,
                           v3 throughput, uint32_t& flags) {
  v3 incoming = mk3s(0.0f);
  bool shadow = false;
  v3 so = mk3s(0.0f);
  // shader.wgsl:2226-2271 up to the shadow ray
  if (ls.pdf > 0.0f) {
    float dotNL = dot(n_orient, ls.dir);
    if (!(dotNL <= 0.0f && mat.transmission <= 0.0f)) {
      v3 bsdf_val; float bsdf_pdf;
      bsdf_eval_pdf(V, ls.dir, mat, ctx, stack, &bsdf_val, &bsdf_pdf);
      float weight = mis_weight(ls.pdf, bsdf_pdf);
      v3 c_weight = (bsdf_val * weight) / wmax(ls.pdf, 1e-6f);
      if (!(max_component(ls.color * c_weight) < 1e-5f)) {
        v3 ray_offset = dotNL < 0.0f ? -n_orient * 0.001f : n_orient * 0.001f;
        so = hit_pos + ray_offset;
        incoming = (ls.color * mk3s(1.0f)) * c_weight;
        shadow = true;
      }
    }
  }
  a.b.nee[slot * 4 + rec * 2] = make_float4(throughput.x, throughput.y, throughput.z, 0.0f);
  a.b.nee[slot * 4 + rec * 2 + 1] = make_float4(incoming.x, incoming.y, incoming.z, 0.0f);
  flags |= rec == 0 ? F_NEE_LIGHT : F_NEE_ENV;
  if (shadow) {
    flags |= rec == 0 ? F_SHADOW_LIGHT : F_SHADOW_ENV;   // queued after the shading body
    a.b.shadow[slot * 4 + rec * 2] = make_float4(so.x, so.y, so.z, ls.dist);
    a.b.shadow[slot * 4 + rec * 2 + 1] = make_float4(ls.dir.x, ls.dir.y, ls.dir.z, __int_as_float(ignore_idx));
  }
}

template <bool COUNT>
__global__ void __launch_bounds__(256) k_wf_shade(WfArgs a, int bounce, const uint32_t* __restrict__ q,
                                                  const uint32_t* count_ptr, uint32_t* __restrict__ q_next,
                                                  uint32_t* count_next, uint32_t* sh_count) {
  Counters<COUNT> cn; cn.init();
  const DScene& s = a.s;
  const DParams& p = a.p;
  uint32_t n = *count_ptr;
  for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    uint32_t i = base + threadIdx.x;
    bool alive = false, sh_light = false, sh_env = false;
    uint32_t slot = 0;
    if (i < n) {
      slot = q[i];
      float4 o4 = a.b.ray_o[slot], d4 = a.b.ray_d[slot], tp4 = a.b.tp[slot], rd4 = a.b.rad[slot];
      uint4 meta = a.b.meta[slot];
      uint4 h0 = a.b.hit[slot * 2], h1 = a.b.hit[slot * 2 + 1];
      HitRec hit;
      hit.t = __uint_as_float(h0.x); hit.m_idx = (int32_t)h0.y; hit.o_idx = (int32_t)h0.z; hit.kind = (int32_t)h0.w;
      hit.id = (int32_t)h1.x; hit.aux = (int32_t)h1.y; hit.bu = __uint_as_float(h1.z); hit.bv = __uint_as_float(h1.w);
      Ray ray; ray.origin = mk3(o4.x, o4.y, o4.z); ray.direction = mk3(d4.x, d4.y, d4.z);
      v3 throughput = mk3(tp4.x, tp4.y, tp4.z);
      float last_surface_pdf = tp4.w;
      v3 radiance = mk3(rd4.x, rd4.y, rd4.z);
      float last_weight_sum = rd4.w;
      uint32_t rng = meta.x;
      uint32_t mcount = meta.w;
      uint32_t flags = 0u;
      MediumStack stack;
      load_stack(a, slot, mcount, stack);
      do {
        apply_medium(stack, hit, bounce, throughput, radiance);
        cn.add(C_SHADE);
        cn.add(C_HIT_ATTR);
        DMat mat = load_mat(s, hit.m_idx);
        SurfCtx ctx;
        ctx.normal = hit_normal(s, ray, hit);
        ctx.albedo = mat.color; ctx.roughness = mat.roughness; ctx.metallic = mat.metallic; ctx.emittance = mat.emittance;
        float em_len = length(ctx.emittance);
        if (em_len > 0.0f) {
          float weight = 1.0f;
          if (HAS(s, WGPT_HAS_LIGHTS) && bounce > 0 && hit.o_idx >= 0) {
            ObjHdr oh = load_obj_hdr(s, (uint32_t)hit.o_idx);
            if (oh.light_idx >= 0) {
              DLight light = load_light(s, (uint32_t)oh.light_idx);
              float raw_light_pdf = 0.0f;
              if (HAS(s, WGPT_HAS_SPHERES) && oh.type == 1) {
                raw_light_pdf = light_sphere_pdf(light, oh.world_position, ray.origin, ray.direction);
              } else if (HAS(s, WGPT_HAS_CUBES) && oh.type == 2) {
                BoxAreas bx = box_areas(light, ray.origin);
                float cos_l = wmax(dot(-ray.direction, ctx.normal), 1e-6f);
                raw_light_pdf = (hit.t * hit.t) / (bx.total * cos_l);
              }
              v3 to_light = oh.world_position - ray.origin;
              float d2 = wmax(dot(to_light, to_light), 0.001f);
              float light_importance = light.power / d2;
              float selection_pdf = last_weight_sum > 0.0f ? light_importance / last_weight_sum : 0.0f;
              weight = mis_weight(last_surface_pdf, raw_light_pdf * selection_pdf);
            }
          }
          radiance = radiance + throughput * clamp_firefly(ctx.emittance * weight, bounce);
          if (em_len > 1.0f) break;
        }
        v3 hit_pos = ray.origin + ray.direction * hit.t;
        v3 V = -ray.direction;
        v3 n_orient = dot(ctx.normal, V) > 0.0f ? ctx.normal : -ctx.normal;
        if (HAS(s, WGPT_HAS_LIGHTS)) {
          int32_t selected = -1;
          float weight_sum = 0.0f, selected_weight = 0.0f;
          for (uint32_t li = 0u; li < s.n_lights; li++) {
            float4 lp = ld4(s.lights + (size_t)li * 5);
            int32_t lo = __float_as_int(lp.x);
            if (lo < 0) continue;
            v3 wp = load_obj_hdr(s, (uint32_t)lo).world_position;
            v3 to_light = wp - hit_pos;
            float d2 = wmax(dot(to_light, to_light), 0.001f);
            float w = lp.z / d2;
            weight_sum += w;
            if (rand_pcg(rng) < (w / weight_sum)) { selected = (int32_t)li; selected_weight = w; }
          }
          if (selected >= 0 && weight_sum > 0.0f) {
            DLight light = load_light(s, (uint32_t)selected);
            ObjHdr lh = load_obj_hdr(s, (uint32_t)light.obj_idx);
            v3 emit = load_mat_emittance(s, lh.material_idx);
            LightSample ls; ls.dir = mk3s(0.0f); ls.color = mk3s(0.0f); ls.dist = 0.0f; ls.pdf = 0.0f;
            if (HAS(s, WGPT_HAS_SPHERES) && lh.type == 1) {
              float x0 = rand_pcg(rng), x1 = rand_pcg(rng);
              ls = sample_light_sphere(light, lh.world_position, emit, hit_pos, x0, x1);
            } else if (HAS(s, WGPT_HAS_CUBES) && lh.type == 2) {
              float x0 = rand_pcg(rng), x1 = rand_pcg(rng);
              ls = sample_light_box(light, emit, hit_pos, x0, x1, rng);
            }
            if (ls.pdf > 0.0f) {
              ls.pdf *= selected_weight / weight_sum;
              record_nee<COUNT>(a, slot, 0, ls, hit_pos, n_orient, V, mat, ctx, stack, light.obj_idx, throughput, flags);
            }
          }
          last_weight_sum = weight_sum;
        }
        if (HAS(s, WGPT_HAS_SKYBOX) && HAS(s, WGPT_MIS_SKYBOX)) {
          cn.add(C_ENV_NEE);
          float u0 = rand_pcg(rng);
          float u1 = rand_pcg(rng);
          LightSample env = sample_env_cdf(s, p, u0, u1, cn);
          record_nee<COUNT>(a, slot, 1, env, hit_pos, n_orient, V, mat, ctx, stack, -1, throughput, flags);
        }
        // shader.wgsl:2052-2175 (alpha == 1) -- the same arithmetic as the single-kernel form
        int32_t count_before = stack.count;
        {
          bool entering = dot(ctx.normal, V) > 0.0f;
          v3 sn_orient = n_orient;
          float dotSNV = wmax(dot(sn_orient, V), 1e-6f);
          float roughness_val = clamp(ctx.roughness, 0.01f, 1.0f);
          float alpha = roughness_val * roughness_val;
          float cc_roughness = clamp(1.0f - mat.clearcoat_gloss, 0.01f, 1.0f);
          float cc_alpha = cc_roughness * cc_roughness;
          float etai = peek_ior(stack);
          float etat = entering ? mat.ior : peek_outer_ior(stack);
          float cc_F_est = fresnel_dielectric(dotSNV, 1.0f, mat.clearcoat_ior);
          float w_cc = entering ? mat.clearcoat * cc_F_est : 0.0f;
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
          if (rand_pcg(rng) > 1.0f) {   // alpha test draw (alpha == 1)
            ray.origin = hit_pos - n_orient * 0.005f;
            alive = true;
          } else {
            float rsel = rand_pcg(rng);
            float xi0 = rand_pcg(rng);
            float xi1 = rand_pcg(rng);
            v3 L = mk3s(0.0f);
            bool is_transmission = false;
            bool done = false, ok = true;
            // lobe choice; the VNDF sampler has one call site for the three microfacet lobes
            int lobe = -1;
            v3 Nv = n_orient;
            float av = alpha;
            if (rsel < p_cc) {
              lobe = 0; Nv = sn_orient; av = cc_alpha;
            } else if (rsel < p_cc + p_spec) {
              lobe = 1;
              if (mat.anisotropic > 0.0f) {
                v3 up = absf(n_orient.y) > 0.99999f ? mk3(0.0f, 0.0f, 1.0f) : mk3(0.0f, 1.0f, 0.0f);
                v3 T = normalize(cross(up, n_orient));
                v3 B = cross(n_orient, T);
                float angle = mat.aniso_rotation * TWO_PI;
                T = T * cos_(angle) + B * sin_(angle);
                Nv = normalize(vmix(n_orient, cross(cross(V, T), T), mat.anisotropic));
              }
            } else if (rsel < p_cc + p_spec + p_trans) {
              if (absf(etai - etat) < 1e-4f) {
                ray.direction = -V;
                ray.origin = hit_pos - n_orient * 0.001f;
                throughput = throughput * mk3s(mat.transmission * (1.0f - ctx.metallic));
                last_surface_pdf = p_trans;
                if (entering) {
                  Medium m; m.ior = mat.ior;
                  m.sigma = (-vlog(vmax(ctx.albedo, mk3s(0.0001f)))) * mat.concentration;
                  m.emission = mat.emittance;
                  push_medium(stack, m);
                } else {
                  pop_medium(stack);
                }
                done = true;
              } else {
                lobe = 2;
              }
            } else if (rsel < total_p) {
              lobe = 3;
            } else {
              ok = false;
            }
            if (lobe >= 0 && lobe <= 2) {
              v3 H = ImportanceSampleVNDF_GGX(xi0, xi1, V, Nv, av);
              if (lobe == 2) {
                float eta_ratio = etai / etat;
                L = refract(-V, H, eta_ratio);
                if (length(L) < 0.1f) L = reflect(-V, H);
                else is_transmission = true;
              } else {
                L = reflect(-V, H);
              }
            } else if (lobe == 3) {
              L = ImportanceSampleCosine(xi0, xi1, n_orient);
            }
            if (ok && !done) {
              float dotNL = dot(n_orient, L);
              if (is_transmission) {
                if (dotNL >= 0.0f) ok = false;
                else ray.origin = hit_pos - n_orient * 0.001f;
              } else {
                if (dotNL <= 0.0f) ok = false;
                else ray.origin = hit_pos + n_orient * 0.001f;
              }
              if (ok) {
                ray.direction = L;
                v3 bsdf_val; float pdf_val;
                bsdf_eval_pdf(V, L, mat, ctx, stack, &bsdf_val, &pdf_val);
                if (pdf_val > 0.0f) throughput = throughput * (bsdf_val / pdf_val);
                else ok = false;
                if (ok) {
                  last_surface_pdf = pdf_val;
                  if (is_transmission) {
                    if (entering) {
                      Medium m; m.ior = mat.ior;
                      m.sigma = (-vlog(vmax(ctx.albedo, mk3s(0.0001f)))) * mat.concentration;
                      m.emission = mat.emittance;
                      push_medium(stack, m);
                    } else {
                      pop_medium(stack);
                    }
                  }
                }
              }
            }
            alive = ok;
          }
        }
        if (!alive) break;
        if (stack.count > count_before) store_medium(a, slot, (uint32_t)(stack.count - 1), stack.media[stack.count - 1]);
        if (bounce < 2) break;
        float survival_prob = clamp(max_component(throughput), 0.05f, 0.95f);
        if (rand_pcg(rng) > survival_prob) { alive = false; break; }
        throughput = throughput / survival_prob;
      } while (false);
      if (bounce + 1 >= s.bounce_limit) alive = false;
      if (alive) flags |= F_ALIVE;
      sh_light = (flags & F_SHADOW_LIGHT) != 0u;
      sh_env = (flags & F_SHADOW_ENV) != 0u;
      a.b.ray_o[slot] = make_float4(ray.origin.x, ray.origin.y, ray.origin.z, 0.0f);
      a.b.ray_d[slot] = make_float4(ray.direction.x, ray.direction.y, ray.direction.z, 0.0f);
      a.b.tp[slot] = make_float4(throughput.x, throughput.y, throughput.z, last_surface_pdf);
      a.b.rad[slot] = make_float4(radiance.x, radiance.y, radiance.z, last_weight_sum);
      a.b.meta[slot] = make_uint4(rng, flags, (uint32_t)bounce, (uint32_t)stack.count);
    }
    queue_push(q_next, count_next, slot, alive);
    queue_push(a.b.shq, sh_count, slot * 2u, sh_light);
    queue_push(a.b.shq, sh_count, slot * 2u + 1u, sh_env);
  }
  flush_wf<COUNT>(cn, a.counters, true);
}

// ---------------------------------------------------------------------------- shadow
template <bool COUNT>
__global__ void __launch_bounds__(256) k_wf_shadow(WfArgs a, const uint32_t* count_ptr, uint32_t* cursor) {
  Counters<COUNT> cn; cn.init();
  uint32_t err = 0;
  const uint32_t n = *count_ptr;
  ShadowTrav t;
  bool have = false, exhausted = false;
  uint32_t e = 0;
  while (true) {
    if (!exhausted) {
      uint32_t qi = refill(have, cursor, n, exhausted);
      if (!have && qi < n) {
        e = a.b.shq[qi];
        float4 so = a.b.shadow[(e >> 1) * 4 + (e & 1u) * 2], sd = a.b.shadow[(e >> 1) * 4 + (e & 1u) * 2 + 1];
        t.rw.origin = mk3(so.x, so.y, so.z);
        t.rw.direction = mk3(sd.x, sd.y, sd.z);
        t.target_dist = so.w;
        t.target_idx = __float_as_int(sd.w);
        shadow_init<COUNT>(a.s, t, cn);
        have = true;
      }
    }
    if (!__any_sync(FULL, have)) break;
    if (have && shadow_step<COUNT>(a.s, a.P, t, err, cn)) {
      shadow_finish<COUNT>(a.s, t, err, cn);
      a.b.vis[e] = t.occluded ? 0u : 1u;
      have = false;
    }
  }
  flush_wf<COUNT>(cn, a.counters, true);
  if (err) atomicOr(a.status, err);
}

// ---------------------------------------------------------------------------- resolve
template <bool COUNT>
__global__ void __launch_bounds__(256) k_wf_resolve(WfArgs a, const uint32_t* __restrict__ q, const uint32_t* count_ptr) {
  Counters<COUNT> cn; cn.init();
  uint32_t n = *count_ptr;
  for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    uint32_t i = base + threadIdx.x;
    if (i < n) {
      uint32_t slot = q[i];
      uint4 meta = a.b.meta[slot];
      uint32_t flags = meta.y;
      int bounce = (int)meta.z;
      float4 rd4 = a.b.rad[slot];
      v3 radiance = mk3(rd4.x, rd4.y, rd4.z);
      if (flags & (F_NEE_LIGHT | F_NEE_ENV)) {
#pragma unroll
        for (int rec = 0; rec < 2; ++rec) {
          uint32_t has = rec == 0 ? F_NEE_LIGHT : F_NEE_ENV;
          uint32_t needs = rec == 0 ? F_SHADOW_LIGHT : F_SHADOW_ENV;
          if (!(flags & has)) continue;
          float4 t4 = a.b.nee[slot * 4 + rec * 2], c4 = a.b.nee[slot * 4 + rec * 2 + 1];
          v3 incoming = mk3(c4.x, c4.y, c4.z);
          if ((flags & needs) && a.b.vis[slot * 2 + rec] == 0u) incoming = mk3s(0.0f);
          radiance = radiance + mk3(t4.x, t4.y, t4.z) * clamp_firefly(incoming, bounce);
        }
        a.b.rad[slot] = make_float4(radiance.x, radiance.y, radiance.z, rd4.w);
      }
      if (!(flags & F_ALIVE)) {
        uint32_t ix, iy;
        px_of(a, slot, ix, iy);
        size_t idx = (size_t)iy * a.p.width + ix;
        float4 acc4 = a.accum[idx];
        float weight = 1.0f / (float)(a.sample_number + 1u);
        v3 acc = vmix(mk3(acc4.x, acc4.y, acc4.z), radiance, weight);
        a.accum[idx] = make_float4(acc.x, acc.y, acc.z, 1.0f);
        v3 c = acc * mk3s(a.p.exposure);
        c = c / (c + mk3s(0.3f));
        c = vpow(c, 0.4545f);
        a.out[(size_t)iy * a.out_pitch + ix] =
            make_uchar4((unsigned char)unorm8(c.x), (unsigned char)unorm8(c.y), (unsigned char)unorm8(c.z), 255);
      }
    }
  }
  flush_wf<COUNT>(cn, a.counters, true);
}

}  // namespace pt

namespace wgpt {

using namespace pt;

static DScene to_dscene_wf(const DeviceScene& d) {
  DScene s;
  s.mats = (const float4*)d.mats; s.n_mats = d.n_mats;
  s.objs = (const float4*)d.objs; s.n_objs = d.n_objs;
  s.tlas = (const float4*)d.tlas; s.n_tlas = d.n_tlas;
  s.meshes = (const float4*)d.meshes; s.n_meshes = d.n_meshes;
  s.bvh = (const float4*)d.bvh; s.n_bvh = d.n_bvh;
  s.tris = (const float4*)d.tris; s.n_tris = d.n_tris;
  s.planes = (const float4*)d.planes; s.n_planes = d.n_planes;
  s.lights = (const float4*)d.lights; s.n_lights = d.n_lights;
  s.sky = (const uint2*)d.sky; s.sky_w = d.sky_w; s.sky_h = d.sky_h;
  s.cdf = (const float*)d.cdf; s.n_cdf = d.n_cdf;
  s.bounce_limit = d.bounce_limit; s.flags = d.flags;
  return s;
}

static DParams to_dparams_wf(const wgpt_scene_params& q, uint32_t sec_x, uint32_t sec_y) {
  DParams p;
  p.eye = mk3(q.eye[0], q.eye[1], q.eye[2]); p.sample_number = q.sample_number;
  p.ray00 = mk3(q.ray00[0], q.ray00[1], q.ray00[2]); p.width = q.width;
  p.ray10 = mk3(q.ray10[0], q.ray10[1], q.ray10[2]); p.height = q.height;
  p.ray01 = mk3(q.ray01[0], q.ray01[1], q.ray01[2]); p.exposure = q.exposure;
  p.ray11 = mk3(q.ray11[0], q.ray11[1], q.ray11[2]); p.seed = q.seed;
  p.sky_width = q.sky_width; p.sky_height = q.sky_height;
  p.sky_total_lum = q.sky_total_lum; p.total_light_power = q.total_light_power;
  p.sec_x = sec_x; p.sec_y = sec_y; p.sky_cdf_index = q.sky_cdf_index;
  return p;
}

size_t wavefront_bytes_per_path() {
  // ray 32 + tp 16 + rad 16 + meta 16 + media 128 + hit 32 + nee 64 + shadow 64 + vis 2 +
  // 2 path queues 8 + shadow queue 8 + hit and miss queues 8
  return 32 + 16 + 16 + 16 + 128 + 32 + 64 + 64 + 2 + 8 + 8 + 8;
}

// Carves the path-state arrays out of one scratch allocation of wavefront_bytes_per_path() *
// capacity + 256 * 16 bytes (256-byte aligned base).
static WfBuffers carve(void* scratch, uint32_t capacity) {
  char* p = (char*)scratch;
  auto take = [&](size_t bytes) { char* r = p; p += (bytes + 255) & ~(size_t)255; return (void*)r; };
  WfBuffers b;
  size_t n = capacity;
  b.ray_o = (float4*)take(n * 16);
  b.ray_d = (float4*)take(n * 16);
  b.tp = (float4*)take(n * 16);
  b.rad = (float4*)take(n * 16);
  b.meta = (uint4*)take(n * 16);
  b.med = (float4*)take(n * 128);
  b.hit = (uint4*)take(n * 32);
  b.nee = (float4*)take(n * 64);
  b.shadow = (float4*)take(n * 64);
  b.vis = (uint8_t*)take(n * 2);
  b.queue[0] = (uint32_t*)take(n * 4);
  b.queue[1] = (uint32_t*)take(n * 4);
  b.shq = (uint32_t*)take(n * 8);
  b.hitq = (uint32_t*)take(n * 4);
  b.missq = (uint32_t*)take(n * 4);
  b.counts = (uint32_t*)take(CNT_KINDS * 256 * 4);
  return b;
}

size_t wavefront_scratch_bytes(uint32_t capacity) {
  size_t n = capacity, s = 0;
  size_t parts[15] = {n * 16, n * 16, n * 16, n * 16, n * 16, n * 128, n * 32, n * 64, n * 64, n * 2, n * 4, n * 4,
                      n * 8, n * 4, n * 4};
  for (size_t x : parts) s += (x + 255) & ~(size_t)255;
  return s + CNT_KINDS * 256 * 4;
}

static int g_grid[8] = {0, 0, 0, 0, 0, 0, 0, 0};   // persistent grid size per stage (computed once)

template <typename K>
static int grid_for(K kernel, int stage) {
  if (g_grid[stage] == 0) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 256, 0);
    g_grid[stage] = sms * (per_sm > 0 ? per_sm : 1);
  }
  return g_grid[stage];
}

template <bool COUNT>
static cudaError_t render_wf(const WfArgs& a0, uint32_t first_frame, uint32_t reps, uint32_t n, cudaStream_t st,
                            StageTimer* timer) {
  WfArgs a = a0;
  unsigned long long* cbase = a0.counters;
  auto stage_args = [&](int stage) {
    WfArgs x = a;
    x.counters = cbase ? cbase + 16 * stage : nullptr;
    return x;
  };
  int bl = a.s.bounce_limit;
  if (bl > 255) return cudaErrorInvalidValue;
  int g_ray = grid_for(k_wf_raygen<COUNT>, 0);
  int g_ext = grid_for(k_wf_extend<COUNT>, 1);
  int g_sh = grid_for(k_wf_shade<COUNT>, 2);
  int g_shw = grid_for(k_wf_shadow<COUNT>, 3);
  int g_res = grid_for(k_wf_resolve<COUNT>, 4);
  int need = (int)((n + 255) / 256);
  int g_miss = grid_for(k_wf_shade_miss<COUNT>, 5);
  uint32_t* C = a.b.counts;
  auto cnt = [&](int kind, int b) { return C + kind * 256 + b; };
  for (uint32_t r = 0; r < reps; ++r) {
    a.sample_number = first_frame + r;
    cudaMemsetAsync(C, 0, CNT_KINDS * 256 * 4, st);
    if (timer) timer->begin(0, st);
    k_wf_raygen<COUNT><<<std::min(g_ray, need), 256, 0, st>>>(stage_args(0));
    if (timer) timer->end(0, st);
    for (int b = 0; b < bl; ++b) {
      uint32_t* qin = a.b.queue[b & 1];
      uint32_t* qout = a.b.queue[(b + 1) & 1];
      if (timer) timer->begin(1, st);
      k_wf_extend<COUNT><<<std::min(g_ext, need), 256, 0, st>>>(stage_args(1), qin, cnt(CNT_LIVE, b),
                                                                cnt(CNT_EXT_CURSOR, b));
      if (timer) timer->end(1, st);
      if (timer) timer->begin(5, st);
      k_wf_shade_miss<COUNT><<<std::min(g_miss, need), 256, 0, st>>>(stage_args(5), b, qin, cnt(CNT_LIVE, b),
                                                                     cnt(CNT_HIT, b));
      if (timer) timer->end(5, st);
      if (timer) timer->begin(2, st);
      k_wf_shade<COUNT><<<std::min(g_sh, need), 256, 0, st>>>(stage_args(2), b, a.b.hitq, cnt(CNT_HIT, b), qout,
                                                               cnt(CNT_LIVE, b + 1), cnt(CNT_SHADOW, b));
      if (timer) timer->end(2, st);
      if (timer) timer->begin(3, st);
      k_wf_shadow<COUNT><<<std::min(g_shw, 2 * need), 256, 0, st>>>(stage_args(3), cnt(CNT_SHADOW, b),
                                                                   cnt(CNT_SH_CURSOR, b));
      if (timer) timer->end(3, st);
      if (timer) timer->begin(4, st);
      k_wf_resolve<COUNT><<<std::min(g_res, need), 256, 0, st>>>(stage_args(4), qin, cnt(CNT_LIVE, b));
      if (timer) timer->end(4, st);
    }
  }
  return cudaGetLastError();
}

cudaError_t launch_render_wavefront(const DeviceScene& d, const wgpt_scene_params& q, uint32_t first_frame,
                                    uint32_t reps, uint32_t sx, uint32_t sy, uint32_t sw, uint32_t sh, float* accum,
                                    uint8_t* out, uint32_t out_pitch, void* scratch, uint32_t capacity,
                                    uint32_t* status, unsigned long long* counters, cudaStream_t st,
                                    StageTimer* timer, const void* pairs_tlas, const void* pairs_bvh) {
  uint32_t n = sw * sh;
  if (n == 0) return cudaSuccess;
  if (n > capacity || !scratch) return cudaErrorInvalidValue;
  WfArgs a;
  a.s = to_dscene_wf(d);
  a.P.tlas = (const float4*)pairs_tlas;
  a.P.bvh = (const float4*)pairs_bvh;
  a.p = to_dparams_wf(q, sx, sy);
  a.b = carve(scratch, capacity);
  a.sec_w = sw; a.sec_h = sh;
  a.sample_number = first_frame;
  a.accum = (float4*)accum;
  a.out = (uchar4*)out;
  a.out_pitch = out_pitch;
  a.status = status;
  a.counters = counters;
  if (counters) return render_wf<true>(a, first_frame, reps, n, st, timer);
  return render_wf<false>(a, first_frame, reps, n, st, timer);
}

}  // namespace wgpt
