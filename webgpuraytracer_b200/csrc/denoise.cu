// Edge-aware a-trous denoiser (denoiser.wgsl) and the preview resample blit (scale.wgsl).
//   k_prepass    3x3 luminance median, NaN/Inf sanitising, tonemap, albedo demodulation
//                (denoiser.wgsl:55-112); also writes the per-pixel guide record that every
//                a-trous pass reads instead of re-deriving it from the G-buffer 25 times;
//   k_atrous     one 5x5 B3-spline a-trous pass with colour/normal/depth/albedo/material edge
//                stops (denoiser.wgsl:117-189);
//   k_composite  remodulation and the rgba8 store (denoiser.wgsl:194-213), fused into the last
//                a-trous pass (a launch of its own only when there are no passes);
//   k_resample   bilinear resample of an rgba8 image (scale.wgsl:6-35).
// The guide record holds, per pixel, values the reference computes identically for every tap:
// normal (3), normal length, depth mapped by d/(d+3), tonemapped albedo (3),
// and (transmission, roughness, metallic) -- 12 floats, so the per-tap arithmetic is unchanged.
#include <stdint.h>
#include <string.h>
#include <mutex>
#include <cuda_runtime.h>
#include "wgsl_builtins.h"
#include "wgpt_internal.h"
#include "../../include/wgpt.h"

using namespace wb;

namespace {

__device__ __forceinline__ v3 tonemap_dn(v3 c, float exposure) {
  v3 color = c * exposure;
  color = color / (color + mk3s(0.3f));
  return vpow(color, 0.4545f);
}
__device__ __forceinline__ float lum_dn(float4 c) { return dot(mk3(c.x, c.y, c.z), mk3(0.299f, 0.587f, 0.114f)); }

struct GuidePix { float4 a, b, c; };   // (n.xyz, |n|) (dmap, alb.rgb) (trans, rough, metal, -)

__global__ void __launch_bounds__(256)
k_prepass(const float4* __restrict__ color, const float* __restrict__ gbuf, wgpt_denoise_uniforms u,
          float4* __restrict__ out, float4* __restrict__ guide) {
  int x = blockIdx.x * 16 + (threadIdx.x & 15), y = blockIdx.y * 16 + (threadIdx.x >> 4);
  int W = (int)u.width, H = (int)u.height;
  if (x >= W || y >= H) return;
  size_t idx = (size_t)y * W + x;
  float4 center;
  if (u.flags & 1u) {
    float4 cols[9]; float lums[9];
    int k = 0;
#pragma unroll
    for (int dy = -1; dy <= 1; dy++) {
#pragma unroll
      for (int dx = -1; dx <= 1; dx++) {
        int cx = min(max(x + dx, 0), W - 1), cy = min(max(y + dy, 0), H - 1);
        cols[k] = __ldg(color + (size_t)cy * W + cx);
        lums[k] = lum_dn(cols[k]);
        k++;
      }
    }
#pragma unroll
    for (int i = 0; i < 5; i++) {
#pragma unroll
      for (int j = i + 1; j < 9; j++) {
        if (lums[j] < lums[i]) {
          float tl = lums[i]; lums[i] = lums[j]; lums[j] = tl;
          float4 tc = cols[i]; cols[i] = cols[j]; cols[j] = tc;
        }
      }
    }
    center = cols[4];
  } else {
    center = color[idx];
  }
  bool valid = (center.x >= 0.0f && center.y >= 0.0f && center.z >= 0.0f) &&
               (center.x <= 10000.0f && center.y <= 10000.0f && center.z <= 10000.0f);
  if (!valid) center = make_float4(0.0f, 0.0f, 0.0f, center.w);
  v3 mapped = tonemap_dn(mk3(center.x, center.y, center.z), u.exposure);
  const float* g = gbuf + idx * 12;
  v3 n = mk3(g[0], g[1], g[2]);
  float nlen = length(n);
  bool is_sky = nlen < 0.1f;
  v3 alb_map = tonemap_dn(mk3(g[4], g[5], g[6]), u.exposure);
  if ((u.flags & 2u) && !is_sky) {
    v3 ma = vmax(alb_map, mk3s(0.001f));
    mapped = mapped / ma;
    mapped = vmin(vmax(mapped, mk3s(0.0f)), mk3s(10.0f));
  }
  out[idx] = make_float4(mapped.x, mapped.y, mapped.z, center.w);
  float dist = g[11];
  GuidePix gp;
  gp.a = make_float4(n.x, n.y, n.z, nlen);
  gp.b = make_float4(dist / (dist + 3.0f), alb_map.x, alb_map.y, alb_map.z);
  gp.c = make_float4(g[10], g[3], g[7], 0.0f);
  guide[idx * 3 + 0] = gp.a; guide[idx * 3 + 1] = gp.b; guide[idx * 3 + 2] = gp.c;
}

// One a-trous pass over a lattice tile.  The 25 taps of a pixel lie on the lattice of spacing
// `step` through it, so a CTA takes the 16 x 16 pixels (rx + step*(16*tx + i), ry + step*(16*ty + j))
// of one residue class (rx, ry) and stages the 20 x 20 lattice points they read (each clamped to
// the image like the reference's taps) in shared memory once: colour and the three guide
// vectors, 64 bytes a point, 25.6 KB a CTA.  Every tap then reads shared memory.  The per-tap
// arithmetic and its order are denoiser.wgsl:117-189's, so results are bit-identical to a
// direct gather.  The edge-stop weight of a tap pair is the same seen from either end, so the
// exact passes evaluate each unordered pair of the tile once (3,570 pairs instead of 6,144
// directed taps, 14.3 KB more shared memory) and each pixel then reads its 24 weights back in
// the reference's tap order.  FAST (opt-in, not bit-exact) evaluates the four exponential edge
// stops as one hardware exponential of their summed arguments and the normal stop with the
// hardware power, with fused multiply-adds; its results stay within 1e-5 relative of the exact
// ones.
// With COMPOSITE the last pass also remodulates and stores the rgba8 image
// (composite_main, denoiser.wgsl:194-213), which then needs no pass of its own.
constexpr int kTile = 16, kApron = 2, kPts = kTile + 2 * kApron;   // 20 x 20 lattice points

struct AtrousSmem {
  float4 col[kPts * kPts];
  float4 ga[kPts * kPts], gb[kPts * kPts], gc[kPts * kPts];
};

struct EdgeSigmas { float sc, sd, sa, sm, sn; };

__device__ __forceinline__ bool same_normal(float4 a, float4 b) {
  return __float_as_uint(a.x) == __float_as_uint(b.x) && __float_as_uint(a.y) == __float_as_uint(b.y) &&
         __float_as_uint(a.z) == __float_as_uint(b.z);
}

// Edge-stop weight of the taps p (centre) and q, staged points, before the centre's attenuation:
// denoiser.wgsl:140-170's factors and their order.  Each factor is symmetric in p and q bit for
// bit (squared differences, products that commute, the normal test on either pixel), so the
// weight of p's tap on q equals that of q's tap on p.  npow[i] is the normal stop of staged point
// i with itself, pow_(max(0, n.n), sigma_normal) (1 when its normal is too short), which every
// pair of bitwise-equal normals (a flat face) shares; stops whose argument is exactly zero skip
// the series, since exp_(-0 / s) is exactly 1 (s > 0).
__device__ __forceinline__ float pair_weight(const AtrousSmem& sm, const float* npow, int p, int q, float h,
                                             const EdgeSigmas& e) {
  const float4 cc = sm.col[p], ga = sm.ga[p], gb = sm.gb[p], gc = sm.gc[p];
  const float4 s = sm.col[q], sa4 = sm.ga[q], sb4 = sm.gb[q], sc4 = sm.gc[q];
  v3 c_diff = mk3(cc.x, cc.y, cc.z) - mk3(s.x, s.y, s.z);
  const float c2 = dot(c_diff, c_diff);
  float w_color = c2 == 0.0f ? 1.0f : exp_(-c2 / e.sc);
  float w_normal = 1.0f;
  if (ga.w > 0.1f || sa4.w > 0.1f) {
    if (same_normal(ga, sa4)) {
      w_normal = npow[p];
    } else {
      float n_dot = wmax(0.0f, dot(mk3(ga.x, ga.y, ga.z), mk3(sa4.x, sa4.y, sa4.z)));
      w_normal = pow_(n_dot, e.sn);
    }
  }
  float d_diff = gb.x - sb4.x;
  const float d2 = d_diff * d_diff;
  float w_depth = d2 == 0.0f ? 1.0f : exp_(-d2 / e.sd);
  // neighbours of the same material usually have identical albedo and material records
  v3 a_diff = mk3(gb.y, gb.z, gb.w) - mk3(sb4.y, sb4.z, sb4.w);
  const float a2 = dot(a_diff, a_diff);
  float w_albedo = a2 == 0.0f ? 1.0f : exp_(-a2 / e.sa);
  v3 m_diff = mk3(gc.x, gc.y, gc.z) - mk3(sc4.x, sc4.y, sc4.z);
  const float m2 = dot(m_diff, m_diff);
  float w_material = m2 == 0.0f ? 1.0f : exp_(-m2 / e.sm);
  return h * w_color * w_normal * w_depth * w_albedo * w_material;
}

// The 12 tap offsets of one half of the 5x5 footprint (dy > 0, or dy == 0 and dx > 0); offset k
// pairs the staged points a and a + (dx, dy) for the (16 + |dx|) x (16 + dy) points a whose pair
// touches the tile's pixels, stored from pair_base(k) on, row-major, a relative to
// (min(0, -dx), -dy).
__host__ __device__ constexpr int pair_dy(int k) { return k < 2 ? 0 : (k < 7 ? 1 : 2); }
__host__ __device__ constexpr int pair_dx(int k) { return k < 2 ? k + 1 : (k < 7 ? k - 4 : k - 9); }
__host__ __device__ constexpr int pair_w(int k) { return kTile + (pair_dx(k) < 0 ? -pair_dx(k) : pair_dx(k)); }
__host__ __device__ constexpr int pair_base(int k) {
  return k == 0 ? 0 : pair_base(k - 1) + pair_w(k - 1) * (kTile + pair_dy(k - 1));
}
__host__ __device__ constexpr int pair_index(int dx, int dy) { return dy == 0 ? dx - 1 : (dy == 1 ? dx + 4 : dx + 9); }
constexpr int kPairSlots = pair_base(12);
static_assert(kPairSlots == 3570, "pair table size");
__device__ __forceinline__ float kern_w(int d) { return d == 0 ? 0.375f : ((d == 1 || d == -1) ? 0.25f : 0.0625f); }

template <bool FAST, bool COMPOSITE>
__global__ void __launch_bounds__(256)
k_atrous(const float4* __restrict__ in, const float4* __restrict__ guide, wgpt_denoise_uniforms u, int step,
         float4* __restrict__ out, float4* __restrict__ composited, uchar4* __restrict__ rgba) {
  __shared__ AtrousSmem sm;
  __shared__ float pw[FAST ? 1 : kPairSlots];
  __shared__ float npow[FAST ? 1 : kPts * kPts];
  const int W = (int)u.width, H = (int)u.height;
  const int rx = (int)(blockIdx.x % (unsigned)step), tx = (int)(blockIdx.x / (unsigned)step);
  const int ry = (int)(blockIdx.y % (unsigned)step), ty = (int)(blockIdx.y / (unsigned)step);
  const int lx0 = tx * kTile - kApron, ly0 = ty * kTile - kApron;   // first staged lattice index
  for (int p = threadIdx.x; p < kPts * kPts; p += blockDim.x) {
    const int px = p % kPts, py = p / kPts;
    const int sx = min(max(rx + step * (lx0 + px), 0), W - 1);
    const int sy = min(max(ry + step * (ly0 + py), 0), H - 1);
    const size_t si = (size_t)sy * W + sx;
    sm.col[p] = __ldg(in + si);
    sm.ga[p] = __ldg(guide + si * 3);
    sm.gb[p] = __ldg(guide + si * 3 + 1);
    sm.gc[p] = __ldg(guide + si * 3 + 2);
    if (!FAST) {
      const float4 g = sm.ga[p];
      npow[p] = g.w > 0.1f ? pow_(wmax(0.0f, dot(mk3(g.x, g.y, g.z), mk3(g.x, g.y, g.z))), u.sigma_normal) : 1.0f;
    }
  }
  __syncthreads();
  EdgeSigmas es;
  es.sc = u.sigma_color * u.sigma_color + 1e-5f;
  es.sd = u.sigma_depth * u.sigma_depth + 1e-5f;
  es.sa = u.sigma_albedo * u.sigma_albedo + 1e-5f;
  es.sm = u.sigma_material * u.sigma_material + 1e-5f;
  es.sn = u.sigma_normal;
  if (!FAST) {
    // every unordered tap pair of the tile once (the tile's pixels reach 2 lattice points out)
    for (int t = threadIdx.x; t < kPairSlots; t += blockDim.x) {
      int odx = pair_dx(0), ody = pair_dy(0), ow = pair_w(0), ob = 0;
#pragma unroll
      for (int k = 1; k < 12; ++k)
        if (t >= pair_base(k)) { odx = pair_dx(k); ody = pair_dy(k); ow = pair_w(k); ob = pair_base(k); }
      const int r = t - ob, ay = r / ow - ody, ax = r - (r / ow) * ow + min(0, -odx);
      const int pa = (ay + kApron) * kPts + (ax + kApron);
      pw[t] = pair_weight(sm, npow, pa, pa + ody * kPts + odx, kern_w(odx) * kern_w(ody), es);
    }
    __syncthreads();
  }
  const int i = (int)(threadIdx.x & 15), j = (int)(threadIdx.x >> 4);
  const int x = rx + step * (tx * kTile + i), y = ry + step * (ty * kTile + j);
  if (x >= W || y >= H) return;
  const int cp = (j + kApron) * kPts + (i + kApron);
  const float4 cc = sm.col[cp], ga = sm.ga[cp], gb = sm.gb[cp], gc = sm.gc[cp];
  v3 c_n = mk3(ga.x, ga.y, ga.z);
  bool c_nflag = ga.w > 0.1f;
  float preserve = (1.0f - gc.y) * wmax(gc.z, gc.x);
  float attenuation = mix(1.0f, 0.0f, preserve * u.glossy_protect);
  const float inv_sc = __frcp_rn(es.sc), inv_sd = __frcp_rn(es.sd), inv_sa = __frcp_rn(es.sa),
              inv_sm = __frcp_rn(es.sm);
  const float kern[5] = {0.0625f, 0.25f, 0.375f, 0.25f, 0.0625f};
  float4 sum = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  float sum_w = 0.0f;
#pragma unroll
  for (int dy = -2; dy <= 2; dy++) {
#pragma unroll
    for (int dx = -2; dx <= 2; dx++) {
      const int q = cp + dy * kPts + dx;
      const float4 s = sm.col[q];
      float weight;
      if (FAST) {
        const float4 sa4 = sm.ga[q], sb4 = sm.gb[q], sc4 = sm.gc[q];
        float h = kern[dx + 2] * kern[dy + 2];
        const float cx = cc.x - s.x, cy = cc.y - s.y, cz = cc.z - s.z;
        const float dd = gb.x - sb4.x;
        const float ax = gb.y - sb4.y, ay = gb.z - sb4.z, az = gb.w - sb4.w;
        const float mx = gc.x - sc4.x, my = gc.y - sc4.y, mz = gc.z - sc4.z;
        float e = __fmul_rn(__fmaf_rn(cx, cx, __fmaf_rn(cy, cy, cz * cz)), inv_sc);
        e = __fmaf_rn(__fmul_rn(dd, dd), inv_sd, e);
        e = __fmaf_rn(__fmaf_rn(ax, ax, __fmaf_rn(ay, ay, az * az)), inv_sa, e);
        e = __fmaf_rn(__fmaf_rn(mx, mx, __fmaf_rn(my, my, mz * mz)), inv_sm, e);
        float w_normal = 1.0f;
        if (c_nflag || sa4.w > 0.1f) {
          float n_dot = fmaxf(0.0f, __fmaf_rn(c_n.x, sa4.x, __fmaf_rn(c_n.y, sa4.y, c_n.z * sa4.z)));
          w_normal = n_dot > 0.0f ? __powf(n_dot, u.sigma_normal) : (u.sigma_normal > 0.0f ? 0.0f : 1.0f);
        }
        weight = h * __expf(-e) * w_normal;
      } else if (dx == 0 && dy == 0) {
        weight = pair_weight(sm, npow, cp, cp, kern[2] * kern[2], es);
      } else if (dy > 0 || (dy == 0 && dx > 0)) {
        // the pair (this pixel, its neighbour): slot of a = this pixel
        const int k = pair_index(dx, dy);
        weight = pw[pair_base(k) + (j + dy) * pair_w(k) + (i - min(0, -dx))];
      } else {
        // the pair (neighbour, this pixel) under the opposite offset: slot of a = the neighbour
        const int k = pair_index(-dx, -dy);
        weight = pw[pair_base(k) + j * pair_w(k) + (i + dx - min(0, dx))];
      }
      if (dx != 0 || dy != 0) weight *= attenuation;
      sum.x = sum.x + s.x * weight; sum.y = sum.y + s.y * weight;
      sum.z = sum.z + s.z * weight; sum.w = sum.w + s.w * weight;
      sum_w += weight;
    }
  }
  float d = sum_w + 1e-5f;
  float4 c = make_float4(sum.x / d, sum.y / d, sum.z / d, sum.w / d);
  const size_t ci = (size_t)y * W + x;
  out[ci] = c;
  if (COMPOSITE) {
    // composite_main on this pass's result (the guide of the centre pixel is already staged)
    bool is_sky = ga.w < 0.1f;
    if ((u.flags & 2u) && !is_sky) {
      v3 ma = vmax(mk3(gb.y, gb.z, gb.w), mk3s(0.001f));
      c = make_float4(c.x * ma.x, c.y * ma.y, c.z * ma.z, c.w);
    }
    if (composited) composited[ci] = c;
    rgba[ci] = make_uchar4((unsigned char)unorm8(c.x), (unsigned char)unorm8(c.y), (unsigned char)unorm8(c.z),
                           (unsigned char)unorm8(c.w));
  }
}

__global__ void __launch_bounds__(256)
k_composite(const float4* __restrict__ in, const float4* __restrict__ guide, wgpt_denoise_uniforms u,
            float4* __restrict__ composited, uchar4* __restrict__ out) {
  int x = blockIdx.x * 16 + (threadIdx.x & 15), y = blockIdx.y * 16 + (threadIdx.x >> 4);
  int W = (int)u.width, H = (int)u.height;
  if (x >= W || y >= H) return;
  size_t idx = (size_t)y * W + x;
  float4 c = in[idx];
  float4 ga = guide[idx * 3], gb = guide[idx * 3 + 1];
  bool is_sky = ga.w < 0.1f;
  if ((u.flags & 2u) && !is_sky) {
    v3 ma = vmax(mk3(gb.y, gb.z, gb.w), mk3s(0.001f));
    c = make_float4(c.x * ma.x, c.y * ma.y, c.z * ma.z, c.w);
  }
  if (composited) composited[idx] = c;
  out[idx] = make_uchar4((unsigned char)unorm8(c.x), (unsigned char)unorm8(c.y), (unsigned char)unorm8(c.z),
                         (unsigned char)unorm8(c.w));
}

__global__ void __launch_bounds__(256)
k_resample(const uchar4* __restrict__ src, uint32_t sw, uint32_t sh, uchar4* __restrict__ dst, uint32_t dw,
           uint32_t dh, float rx, float ry) {
  uint32_t x = blockIdx.x * 16 + (threadIdx.x & 15), y = blockIdx.y * 16 + (threadIdx.x >> 4);
  if (x >= dw || y >= dh) return;
  float ux = (float)x / (float)dw, uy = (float)y / (float)dh;
  float spx = ux * rx * (float)sw - 0.5f, spy = uy * ry * (float)sh - 0.5f;
  float fx = fract(spx), fy = fract(spy);
  int bx = (int)floorf(spx), by = (int)floorf(spy);
  int mx = (int)sw - 1, my = (int)sh - 1;
  auto tl = [&](int tx, int ty) {
    tx = min(max(tx, 0), mx); ty = min(max(ty, 0), my);
    uchar4 t = __ldg(src + (size_t)ty * sw + tx);
    return mk4((float)t.x / 255.0f, (float)t.y / 255.0f, (float)t.z / 255.0f, (float)t.w / 255.0f);
  };
  v4 t00 = tl(bx, by), t10 = tl(bx + 1, by), t01 = tl(bx, by + 1), t11 = tl(bx + 1, by + 1);
  v4 col = vmix4(vmix4(t00, t10, fx), vmix4(t01, t11, fx), fy);
  dst[(size_t)y * dw + x] = make_uchar4((unsigned char)unorm8(col.x), (unsigned char)unorm8(col.y),
                                        (unsigned char)unorm8(col.z), 255);
}

}  // namespace

namespace wgpt {

static inline dim3 grid16(uint32_t w, uint32_t h) { return dim3((w + 15) / 16, (h + 15) / 16); }

cudaError_t launch_denoise(const float* color, const float* gbuf, const wgpt_denoise_uniforms& u,
                           const uint32_t* steps, uint32_t passes, float* buf_a, float* buf_b, float* guide,
                           float* composited, uint8_t* out, const float** final_buf, cudaStream_t st,
                           bool fast) {
  dim3 g = grid16(u.width, u.height);
  k_prepass<<<g, 256, 0, st>>>((const float4*)color, gbuf, u, (float4*)buf_a, (float4*)guide);
  float* in = buf_a;
  float* ob = buf_b;
  for (uint32_t i = 0; i < passes; ++i) {
    const uint32_t step = steps[i];
    // lattice tiles: per residue class, ceil(ceil(W / step) / 16) x ceil(ceil(H / step) / 16)
    const uint32_t lw = (u.width + step - 1) / step, lh = (u.height + step - 1) / step;
    dim3 ga(((lw + kTile - 1) / kTile) * step, ((lh + kTile - 1) / kTile) * step);
    const bool last = i + 1 == passes;
    auto kern = fast ? (last ? k_atrous<true, true> : k_atrous<true, false>)
                     : (last ? k_atrous<false, true> : k_atrous<false, false>);
    kern<<<ga, 256, 0, st>>>((const float4*)in, (const float4*)guide, u, (int)step, (float4*)ob,
                             (float4*)composited, (uchar4*)out);
    float* t = in; in = ob; ob = t;
  }
  if (passes == 0)
    k_composite<<<g, 256, 0, st>>>((const float4*)in, (const float4*)guide, u, (float4*)composited, (uchar4*)out);
  if (final_buf) *final_buf = in;
  return cudaGetLastError();
}

cudaError_t launch_resample(const uint8_t* src, uint32_t sw, uint32_t sh, uint8_t* dst, uint32_t dw, uint32_t dh,
                            float rx, float ry, cudaStream_t st) {
  k_resample<<<grid16(dw, dh), 256, 0, st>>>((const uchar4*)src, sw, sh, (uchar4*)dst, dw, dh, rx, ry);
  return cudaGetLastError();
}

}  // namespace wgpt

// ---------------------------------------------------------------------------------------------
// Allocation-free denoiser entry point.
//
// The ping-pong buffers (16 B/pixel each) and the guide record (48 B/pixel) of the denoiser
// live in one file-scope device array of WGPT_NOALLOC_MAX_PIXELS * 80 bytes (10 MiB) that every
// GPU loading this library holds until the process exits.  Host code cannot use the array's
// name as a device address (it is a host-side stand-in), so the first call on each device looks
// the address up with cudaGetSymbolAddress while that device is current and keeps it.
static __device__ __align__(256) float4 g_noalloc_scratch[(size_t)WGPT_NOALLOC_MAX_PIXELS * 5];

namespace {
constexpr int kMaxDevices = 64;
float4* g_noalloc_addr[kMaxDevices] = {nullptr};
std::mutex g_noalloc_mu;
}  // namespace

extern "C" int wgpt_denoise_noalloc(const float* color, const void* gbuf, const void* uniforms_48,
                                    const uint32_t* steps, uint32_t passes, uint8_t* out_rgba8,
                                    float* out_composited, void* stream) {
  if (!color || !gbuf || !uniforms_48 || !out_rgba8 || (passes && !steps)) return WGPT_E_INVALID;
  // the kernels read color and gbuf and write out_composited as float4, out_rgba8 as uchar4
  if (((uintptr_t)color | (uintptr_t)gbuf | (uintptr_t)out_composited) & 15u) return WGPT_E_INVALID;
  if ((uintptr_t)out_rgba8 & 3u) return WGPT_E_INVALID;
  wgpt_denoise_uniforms u;
  memcpy(&u, uniforms_48, sizeof u);
  if (u.width == 0 || u.height == 0) return WGPT_E_INVALID;
  if ((uint64_t)u.width * u.height > WGPT_NOALLOC_MAX_PIXELS) return WGPT_E_TOO_LARGE;
  if (passes > 64) return WGPT_E_INVALID;
  for (uint32_t i = 0; i < passes; ++i)
    if (steps[i] == 0 || steps[i] > (1u << 20)) return WGPT_E_INVALID;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return WGPT_E_CUDA;
  (void)cudaGetLastError();   // a stale non-sticky error from other code is not this call's
  float4* base = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
      void* p = nullptr;
      if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return WGPT_E_CUDA;
      g_noalloc_addr[dev] = (float4*)p;
    }
    base = g_noalloc_addr[dev];
  }
  // Nothing in the scratch has to start at zero: the prepass writes every pixel of the first
  // buffer and of the guide, and every pass writes each pixel it later reads.
  const size_t npix = (size_t)u.width * u.height;
  float* buf_a = (float*)base;
  float* buf_b = (float*)(base + npix);
  float* guide = (float*)(base + 2 * npix);
  cudaError_t e = wgpt::launch_denoise(color, (const float*)gbuf, u, steps, passes, buf_a, buf_b, guide,
                                       out_composited, out_rgba8, nullptr, (cudaStream_t)stream);
  return e == cudaSuccess ? WGPT_OK : WGPT_E_CUDA;
}
