// Path-tracing kernels of the progressive renderer:
//   k_render      one camera path per pixel and repetition, running-mean accumulation and the
//                 tonemapped rgba8 store (shader.wgsl main, 2273-2492);
//   k_gbuffer     the denoiser's guide buffer (shader.wgsl gbuf_main, 2510-2603);
//   k_trace_rays  closest hit of caller-supplied rays (trace_scene, shader.wgsl:754-774).
// A launch covers one section (tile) of the image like one reference dispatch; all `reps`
// samples of a pixel run in the same thread, so the pixel's accumulator stays in registers
// between samples (the reference re-reads and re-writes it per dispatch; the arithmetic is the
// same).
#include "pt_device.cuh"
#include "wgpt_internal.h"

namespace pt {

template <bool COUNT>
struct PathState {
  uint32_t rng;
  uint32_t err;
  Counters<COUNT> cn;
};

// shader.wgsl:2226-2271
template <bool COUNT, bool TEX>
__device__ v3 evaluate_nee(const DScene& s, const LightSample& ls, v3 hit_pos, v3 n_orient, v3 V, const DMat& mat,
                           const SurfCtx& ctx, const TexPoint& tp, const MediumStack& stack, int32_t ignore_obj_idx,
                           PathState<COUNT>& ps) {
  if (ls.pdf <= 0.0f) return mk3s(0.0f);
  float dotNL = dot(n_orient, ls.dir);
  if (dotNL <= 0.0f && mat.transmission <= 0.0f) return mk3s(0.0f);
  v3 bsdf_val; float bsdf_pdf;
  bsdf_eval_pdf<TEX>(V, ls.dir, mat, ctx, stack, &bsdf_val, &bsdf_pdf);
  float weight = mis_weight(ls.pdf, bsdf_pdf);
  v3 c_weight = (bsdf_val * weight) / wmax(ls.pdf, 1e-6f);
  if (max_component(ls.color * c_weight) < 1e-5f) return mk3s(0.0f);
  v3 ray_offset = dotNL < 0.0f ? -n_orient * 0.001f : n_orient * 0.001f;
  Ray sr; sr.origin = hit_pos + ray_offset; sr.direction = ls.dir;
  v2 pom_uv;
  if (pom_shadowed<TEX>(s, tp, ls.dir, &pom_uv)) return mk3s(0.0f);
  float shadow = scene_shadow<COUNT, TEX>(s, sr, ignore_obj_idx, ls.dist, ps.err, ps.cn);
  if (shadow < 0.001f) return mk3s(0.0f);
  return (ls.color * shadow) * c_weight;
}

// shader.wgsl:2052-2175
template <bool COUNT, bool TEX>
__device__ bool sample_surface(Ray& ray, v3& throughput, v3 hit_pos, const DMat& mat, const SurfCtx& ctx,
                               MediumStack& stack, float& last_surface_pdf, PathState<COUNT>& ps) {
  v3 V = -ray.direction;
  bool entering = dot(ctx.normal, V) > 0.0f;
  v3 n_orient = entering ? ctx.normal : -ctx.normal;
  v3 sn_orient = entering ? ctx.surface_normal : -ctx.surface_normal;
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

  if (rand_pcg(ps.rng) > ctx.alpha) {   // alpha cut-out: the path passes through
    ray.origin = hit_pos - n_orient * 0.005f;
    return true;
  }
  float rng = rand_pcg(ps.rng);
  float xi0 = rand_pcg(ps.rng);
  float xi1 = rand_pcg(ps.rng);
  v3 L = mk3s(0.0f);
  bool is_transmission = false;
  if (rng < p_cc) {
    v3 H = ImportanceSampleVNDF_GGX(xi0, xi1, V, sn_orient, cc_alpha);
    L = reflect(-V, H);
  } else if (rng < p_cc + p_spec) {
    v3 N_spec = n_orient;
    if (mat.anisotropic > 0.0f) {
      v3 up = absf(n_orient.y) > 0.99999f ? mk3(0.0f, 0.0f, 1.0f) : mk3(0.0f, 1.0f, 0.0f);
      v3 T = normalize(cross(up, n_orient));
      v3 B = cross(n_orient, T);
      float angle = mat.aniso_rotation * TWO_PI;
      T = T * cos_(angle) + B * sin_(angle);
      N_spec = normalize(vmix(n_orient, cross(cross(V, T), T), mat.anisotropic));
    }
    v3 H = ImportanceSampleVNDF_GGX(xi0, xi1, V, N_spec, alpha);
    L = reflect(-V, H);
  } else if (rng < p_cc + p_spec + p_trans) {
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
      return true;
    }
    v3 H = ImportanceSampleVNDF_GGX(xi0, xi1, V, n_orient, alpha);
    float eta_ratio = etai / etat;
    L = refract(-V, H, eta_ratio);
    if (length(L) < 0.1f) L = reflect(-V, H);
    else is_transmission = true;
  } else if (rng < total_p) {
    L = ImportanceSampleCosine(xi0, xi1, n_orient);
  } else {
    return false;
  }
  float dotNL = dot(n_orient, L);
  if (is_transmission) {
    if (dotNL >= 0.0f) return false;
    ray.origin = hit_pos - n_orient * 0.001f;
  } else {
    if (dotNL <= 0.0f) return false;
    ray.origin = hit_pos + n_orient * 0.001f;
  }
  ray.direction = L;
  v3 bsdf_val; float pdf_val;
  bsdf_eval_pdf<TEX>(V, L, mat, ctx, stack, &bsdf_val, &pdf_val);
  if (pdf_val > 0.0f) throughput = throughput * (bsdf_val / pdf_val);
  else return false;
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
  return true;
}

// One camera path of main (shader.wgsl:2280-2480); returns the path's radiance.
template <bool COUNT, bool TEX>
__device__ v3 trace_path(const DScene& s, const DParams& p, uint32_t ix, uint32_t iy, uint32_t sample_number, PathState<COUNT>& ps) {
  uint32_t idx = iy * p.width + ix;
  ps.rng = (idx * 1973u + sample_number * 9277u + p.seed * 26699u) | 1u;
  rand_pcg(ps.rng);
  ps.cn.add(C_PATHS);
  float j0 = rand_pcg(ps.rng);
  float j1 = rand_pcg(ps.rng);
  float su = ((float)ix + j0) / (float)p.width;
  float sv = ((float)iy + j1) / (float)p.height;
  Ray ray;
  ray.origin = p.eye;
  ray.direction = normalize(vmix(vmix(p.ray00, p.ray10, su), vmix(p.ray01, p.ray11, su), 1.0f - sv));
  v3 throughput = mk3s(1.0f);
  v3 radiance = mk3s(0.0f);
  float last_surface_pdf = 1.0f;
  float last_weight_sum = 0.0f;
  MediumStack stack; stack.count = 0;

  for (int bounce = 0; bounce < s.bounce_limit; bounce++) {
    HitRec hit = trace_scene<COUNT>(s, ray, ps.err, ps.cn);
    // shader.wgsl:2327-2342 Beer-Lambert attenuation and emission of the current medium
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
    if (hit.m_idx == -1) {
      if (HAS(s, WGPT_HAS_SKYBOX)) {
        v3 sky_color = sample_sky(s, ray.direction, ps.cn);
        float weight = 1.0f;
        if (bounce > 0 && HAS(s, WGPT_MIS_SKYBOX)) {
          float sky_pdf = get_sky_pdf(s, p, ray.direction, ps.cn);
          weight = mis_weight(last_surface_pdf, sky_pdf);
        }
        radiance = radiance + throughput * clamp_firefly(sky_color * weight, bounce);
      } else {
        radiance = radiance + throughput * clamp_firefly(mk3(0.02f, 0.03f, 0.05f), bounce);
      }
      break;
    }
    ps.cn.add(C_SHADE);
    ps.cn.add(C_HIT_ATTR);
    DMat mat = load_mat(s, hit.m_idx);
    v3 hn = hit_normal(s, ray, hit);
    TexPoint tp;
    SurfCtx ctx = hit_context<TEX>(s, ray, hit, mat, hn, &tp, true);

    // shader.wgsl:2378-2395 implicit light hit
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
            BoxAreas b = box_areas(light, ray.origin);
            float cos_l = wmax(dot(-ray.direction, hn), 1e-6f);
            raw_light_pdf = (hit.t * hit.t) / (b.total * cos_l);
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

    // shader.wgsl:2402-2446 light NEE by reservoir selection
    if (HAS(s, WGPT_HAS_LIGHTS)) {
      int32_t selected = -1;
      float weight_sum = 0.0f, selected_weight = 0.0f;
      for (uint32_t i = 0u; i < s.n_lights; i++) {
        int32_t lo = bi(ld4(s.lights + (size_t)i * 5).x);
        if (lo < 0) continue;
        float4 lp = ld4(s.lights + (size_t)i * 5);
        v3 wp = load_obj_hdr(s, (uint32_t)lo).world_position;
        v3 to_light = wp - hit_pos;
        float d2 = wmax(dot(to_light, to_light), 0.001f);
        float w = lp.z / d2;
        weight_sum += w;
        if (rand_pcg(ps.rng) < (w / weight_sum)) { selected = (int32_t)i; selected_weight = w; }
      }
      if (selected >= 0 && weight_sum > 0.0f) {
        DLight light = load_light(s, (uint32_t)selected);
        ObjHdr lh = load_obj_hdr(s, (uint32_t)light.obj_idx);
        v3 emit = load_mat_emittance(s, lh.material_idx);
        LightSample ls; ls.dir = mk3s(0.0f); ls.color = mk3s(0.0f); ls.dist = 0.0f; ls.pdf = 0.0f;
        if (HAS(s, WGPT_HAS_SPHERES) && lh.type == 1) {
          float x0 = rand_pcg(ps.rng), x1 = rand_pcg(ps.rng);
          ls = sample_light_sphere(light, lh.world_position, emit, hit_pos, x0, x1);
        } else if (HAS(s, WGPT_HAS_CUBES) && lh.type == 2) {
          float x0 = rand_pcg(ps.rng), x1 = rand_pcg(ps.rng);
          ls = sample_light_box(light, emit, hit_pos, x0, x1, ps.rng);
        }
        if (ls.pdf > 0.0f) {
          ls.pdf *= selected_weight / weight_sum;
          v3 incoming = evaluate_nee<COUNT, TEX>(s, ls, hit_pos, n_orient, V, mat, ctx, tp, stack, light.obj_idx, ps);
          radiance = radiance + throughput * clamp_firefly(incoming, bounce);
        }
      }
      last_weight_sum = weight_sum;
    }
    // shader.wgsl:2449-2453 environment NEE
    if (HAS(s, WGPT_HAS_SKYBOX) && HAS(s, WGPT_MIS_SKYBOX)) {
      ps.cn.add(C_ENV_NEE);
      float u0 = rand_pcg(ps.rng);
      float u1 = rand_pcg(ps.rng);
      LightSample env = sample_env_cdf(s, p, u0, u1, ps.cn);
      v3 incoming = evaluate_nee<COUNT, TEX>(s, env, hit_pos, n_orient, V, mat, ctx, tp, stack, -1, ps);
      radiance = radiance + throughput * clamp_firefly(incoming, bounce);
    }
    if (!sample_surface<COUNT, TEX>(ray, throughput, hit_pos, mat, ctx, stack, last_surface_pdf, ps)) break;
    // shader.wgsl:2458-2472: the height field shadows the sampled direction: shade the occluding
    // texel and sample again from it
    v2 pom_uv;
    if (pom_shadowed<TEX>(s, tp, ray.direction, &pom_uv)) {
      SurfCtx cp = surface_context(s, mat, hn, tp, pom_uv);
      radiance = radiance + throughput * clamp_firefly(cp.emittance, bounce);
      if (length(cp.emittance) > 1.0f) break;
      if (!sample_surface<COUNT, TEX>(ray, throughput, hit_pos, mat, cp, stack, last_surface_pdf, ps)) break;
    }
    if (bounce < 2) continue;
    float survival_prob = clamp(max_component(throughput), 0.05f, 0.95f);
    if (rand_pcg(ps.rng) > survival_prob) break;
    throughput = throughput / survival_prob;
  }
  return radiance;
}

template <bool COUNT>
__device__ __forceinline__ void flush_counters(PathState<COUNT>& ps, unsigned long long* counters) {
  if (!COUNT) return;
#pragma unroll
  for (int k = 0; k < C_NCOUNTERS; ++k) {
    unsigned long long v = ps.cn.v[k];
    // warp-level reduction, one atomic per warp and counter
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(counters + k, v);
  }
}

template <bool COUNT, bool TEX>
__global__ void __launch_bounds__(128)
k_render(DScene s, DParams p, uint32_t first_frame, uint32_t reps, uint32_t sec_w, uint32_t sec_h,
         float4* __restrict__ accum, uchar4* __restrict__ out, uint32_t out_pitch, uint32_t* status,
         unsigned long long* counters) {
  // 8x16 pixel tile per block; a warp covers 8x4 pixels.
  uint32_t lx = threadIdx.x & 7u, ly = threadIdx.x >> 3;
  uint32_t x = blockIdx.x * 8u + lx, y = blockIdx.y * 16u + ly;
  bool active = x < sec_w && y < sec_h;
  PathState<COUNT> ps;
  ps.err = 0u;
  ps.cn.init();
  if (active) {
    uint32_t ix = p.sec_x + x, iy = p.sec_y + y;
    size_t idx = (size_t)iy * p.width + ix;
    float4 a = accum[idx];
    v3 acc = mk3(a.x, a.y, a.z);
    for (uint32_t r = 0; r < reps; ++r) {
      uint32_t sn = first_frame + r;
      v3 radiance = trace_path<COUNT, TEX>(s, p, ix, iy, sn, ps);
      float weight = 1.0f / (float)(sn + 1u);
      acc = vmix(acc, radiance, weight);
    }
    accum[idx] = make_float4(acc.x, acc.y, acc.z, 1.0f);
    v3 c = acc * mk3s(p.exposure);
    c = c / (c + mk3s(0.3f));
    c = vpow(c, 0.4545f);
    out[(size_t)iy * out_pitch + ix] =
        make_uchar4((unsigned char)unorm8(c.x), (unsigned char)unorm8(c.y), (unsigned char)unorm8(c.z), 255);
  }
  flush_counters<COUNT>(ps, counters);
  if (ps.err) atomicOr(status, ps.err);
}

// shader.wgsl:2510-2603
template <bool TEX>
__global__ void __launch_bounds__(128)
k_gbuffer(DScene s, DParams p, uint32_t sec_w, uint32_t sec_h, float* __restrict__ gbuf, uchar4* __restrict__ out,
          uint32_t out_pitch, uint32_t* status) {
  uint32_t lx = threadIdx.x & 7u, ly = threadIdx.x >> 3;
  uint32_t x = blockIdx.x * 8u + lx, y = blockIdx.y * 16u + ly;
  if (x >= sec_w || y >= sec_h) return;
  uint32_t ix = p.sec_x + x, iy = p.sec_y + y;
  size_t idx = (size_t)iy * p.width + ix;
  PathState<false> ps; ps.err = 0u;
  float su = ((float)ix + 0.5f) / (float)p.width;
  float sv = ((float)iy + 0.5f) / (float)p.height;
  Ray ray;
  ray.origin = p.eye;
  ray.direction = normalize(vmix(vmix(p.ray00, p.ray10, su), vmix(p.ray01, p.ray11, su), 1.0f - sv));
  v3 c_normal = mk3s(0.0f), c_albedo = mk3s(0.0f), c_emit = mk3s(0.0f);
  float c_rough = 0.0f, c_metal = 0.0f, m_trans = 0.0f;
  float dist = 0.0f;
  v3 tint = mk3s(1.0f);
  for (int bounce = 0; bounce < s.bounce_limit; bounce++) {
    HitRec hit = trace_scene<false>(s, ray, ps.err, ps.cn);
    if (hit.m_idx == -1) {
      c_normal = mk3s(0.0f);
      c_emit = sample_sky(s, ray.direction, ps.cn);
      c_albedo = mk3s(0.0f);
      break;
    }
    DMat mat = load_mat(s, hit.m_idx);
    TexPoint tp;
    SurfCtx ctx = hit_context<TEX>(s, ray, hit, mat, hit_normal(s, ray, hit), &tp, false);
    c_albedo = ctx.albedo; c_rough = ctx.roughness; c_metal = ctx.metallic; c_emit = ctx.emittance;
    m_trans = mat.transmission;
    c_normal = dot(ctx.normal, -ray.direction) > 0.0f ? ctx.normal : -ctx.normal;
    dist += hit.t;
    if (ctx.alpha < 1.0f) {   // cut-out: tint by the albedo's coverage and continue behind the surface
      tint = tint * vmix(mk3s(1.0f), c_albedo, ctx.alpha);
      ray.origin = (ray.origin + ray.direction * hit.t) - c_normal * 0.001f;
      continue;
    }
    if (mat.metallic >= 0.99f && mat.roughness <= 0.01f) {
      tint = tint * c_albedo;
      ray.origin = (ray.origin + ray.direction * hit.t) + c_normal * 0.001f;
      ray.direction = reflect(ray.direction, c_normal);
      continue;
    }
    break;
  }
  v3 color = (c_albedo + c_emit) * tint;
  float* g = gbuf + idx * 12;
  g[0] = c_normal.x; g[1] = c_normal.y; g[2] = c_normal.z; g[3] = c_rough;
  g[4] = color.x; g[5] = color.y; g[6] = color.z; g[7] = c_metal;
  g[10] = m_trans; g[11] = dist;
  v3 o3;
  if (ix < p.width * 1u / 4u) {
    o3 = mk3s(dist / (dist + 3.0f));
  } else if (ix < p.width * 2u / 4u) {
    o3 = c_normal * 0.5f + mk3s(0.5f);
  } else if (ix < p.width * 3u / 4u) {
    v3 cc = color * mk3s(p.exposure);
    cc = cc / (cc + mk3s(0.3f));
    o3 = vpow(cc, 0.4545f);
  } else {
    o3 = mk3(m_trans, c_rough, c_metal);
  }
  out[(size_t)iy * out_pitch + ix] =
      make_uchar4((unsigned char)unorm8(o3.x), (unsigned char)unorm8(o3.y), (unsigned char)unorm8(o3.z), 255);
  if (ps.err) atomicOr(status, ps.err);
}

__global__ void k_trace_rays(DScene s, const float* __restrict__ rays, uint32_t n, int32_t* o_idx, int32_t* m_idx,
                             int32_t* prim, float* t, float* normal, uint32_t* status) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  PathState<false> ps; ps.err = 0u;
  Ray r;
  r.origin = mk3(rays[i * 6 + 0], rays[i * 6 + 1], rays[i * 6 + 2]);
  r.direction = mk3(rays[i * 6 + 3], rays[i * 6 + 4], rays[i * 6 + 5]);
  HitRec h = trace_scene<false>(s, r, ps.err, ps.cn);
  o_idx[i] = h.o_idx; m_idx[i] = h.m_idx;
  prim[i] = (h.kind == 2 || h.kind == 4) ? h.id : -1;
  t[i] = h.t;
  v3 nn = h.kind == 0 ? mk3s(0.0f) : hit_normal(s, r, h);
  normal[i * 3 + 0] = nn.x; normal[i * 3 + 1] = nn.y; normal[i * 3 + 2] = nn.z;
  if (ps.err) atomicOr(status, ps.err);
}

// Environment light samples of caller random pairs through sample_env_cdf (shader.wgsl:231-254):
// the chosen texel (x, y) and the sample's pdf, for known-answer tests of the CDF search.
__global__ void k_sample_env(DScene s, DParams p, const float* __restrict__ u2, uint32_t n, uint32_t* texel,
                             float* pdf) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  Counters<false> cn;
  const float ux = u2[2 * i], uy = u2[2 * i + 1];
  // the two searches sample_env_cdf makes, for the texel indices it turns into a direction
  const uint32_t v_idx = binary_search_cdf(s, 0u, p.sky_height, uy, cn);
  const uint32_t u_idx = binary_search_cdf(s, p.sky_cdf_index + v_idx * (p.sky_width + 1u), p.sky_width, ux, cn);
  texel[2 * i] = u_idx;
  texel[2 * i + 1] = v_idx;
  pdf[i] = sample_env_cdf(s, p, ux, uy, cn).pdf;
}

// The per-pixel random stream of main (shader.wgsl:146-154, seeding 2280-2282): draws 1..n after
// the discarded first one.
__global__ void k_rng_stream(uint32_t idx, uint32_t sample_number, uint32_t seed, uint32_t n, float* out) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  uint32_t st = (idx * 1973u + sample_number * 9277u + seed * 26699u) | 1u;
  rand_pcg(st);
  for (uint32_t i = 0; i < n; ++i) out[i] = rand_pcg(st);
}

}  // namespace pt

using namespace pt;

static DScene to_dscene(const wgpt::DeviceScene& d) {
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
  s.tex = (const uint32_t*)d.tex; s.tex_w = d.tex_w; s.tex_h = d.tex_h;
  s.alias = (const uint2*)d.alias;
  s.bounce_limit = d.bounce_limit; s.flags = d.flags;
  return s;
}

static DParams to_dparams(const wgpt_scene_params& q, uint32_t sec_x, uint32_t sec_y) {
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

namespace wgpt {

cudaError_t launch_render(const DeviceScene& d, const wgpt_scene_params& q, uint32_t first_frame, uint32_t reps,
                          uint32_t sx, uint32_t sy, uint32_t sw, uint32_t sh, float* accum, uint8_t* out,
                          uint32_t out_pitch, uint32_t* status, unsigned long long* counters, cudaStream_t st) {
  DScene s = to_dscene(d);
  DParams p = to_dparams(q, sx, sy);
  dim3 grid((sw + 7) / 8, (sh + 15) / 16);
  auto launch = [&](auto kernel, unsigned long long* c) {
    kernel<<<grid, 128, 0, st>>>(s, p, first_frame, reps, sw, sh, (float4*)accum, (uchar4*)out, out_pitch, status, c);
  };
  const bool tex = (s.flags & wgpt::SCENE_TEXTURED) != 0u;
  if (counters) {
    if (tex) launch(k_render<true, true>, counters); else launch(k_render<true, false>, counters);
  } else {
    if (tex) launch(k_render<false, true>, nullptr); else launch(k_render<false, false>, nullptr);
  }
  return cudaGetLastError();
}

cudaError_t launch_gbuffer(const DeviceScene& d, const wgpt_scene_params& q, uint32_t sx, uint32_t sy, uint32_t sw,
                           uint32_t sh, float* gbuf, uint8_t* out, uint32_t out_pitch, uint32_t* status,
                           cudaStream_t st) {
  DScene s = to_dscene(d);
  DParams p = to_dparams(q, sx, sy);
  dim3 grid((sw + 7) / 8, (sh + 15) / 16);
  if (s.flags & wgpt::SCENE_TEXTURED)
    k_gbuffer<true><<<grid, 128, 0, st>>>(s, p, sw, sh, gbuf, (uchar4*)out, out_pitch, status);
  else
    k_gbuffer<false><<<grid, 128, 0, st>>>(s, p, sw, sh, gbuf, (uchar4*)out, out_pitch, status);
  return cudaGetLastError();
}

cudaError_t launch_trace_rays(const DeviceScene& d, const float* rays, uint32_t n, int32_t* o_idx, int32_t* m_idx,
                              int32_t* prim, float* t, float* normal, uint32_t* status, cudaStream_t st) {
  DScene s = to_dscene(d);
  k_trace_rays<<<(n + 127) / 128, 128, 0, st>>>(s, rays, n, o_idx, m_idx, prim, t, normal, status);
  return cudaGetLastError();
}

cudaError_t launch_sample_env(const DeviceScene& d, const wgpt_scene_params& q, const float* u2, uint32_t n,
                              uint32_t* texel, float* pdf, cudaStream_t st) {
  DScene s = to_dscene(d);
  DParams p = to_dparams(q, 0, 0);
  k_sample_env<<<(n + 127) / 128, 128, 0, st>>>(s, p, u2, n, texel, pdf);
  return cudaGetLastError();
}

cudaError_t launch_rng_stream(uint32_t idx, uint32_t sample_number, uint32_t seed, uint32_t n, float* out,
                              cudaStream_t st) {
  k_rng_stream<<<1, 32, 0, st>>>(idx, sample_number, seed, n, out);
  return cudaGetLastError();
}

}  // namespace wgpt
