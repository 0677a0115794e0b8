// Wavefront form of the progressive renderer's path tracing (shader.wgsl main, 2273-2492).
//
// The samples of one render call -- every (view, sample, pixel) of a batch of camera views --
// are work units, numbered view by view, sample-major inside a view.  A fixed pool of path slots
// traces them; a slot whose path ends takes the next unit at once (path regeneration), so the
// queues stay full until the last units drain instead of shrinking bounce after bounce.
// One iteration runs each stage once over the slots that hold a path:
//   k_wf_extend     closest hit of every queued path (two-level BVH, planes, list meshes)
//   k_wf_shade_miss walks the queue in order: queues surface hits, shades paths that left the
//                   scene (media and the sky term)
//   k_wf_shade      surface hits: media, emission, light and environment NEE set-up, BSDF
//                   sampling, Russian roulette; records up to two next-event contributions with
//                   their shadow rays
//   k_wf_shadow     traces the recorded shadow rays (their own compacted queue, fetched
//                   dynamically by warps) and stores one visibility byte per record
//   k_wf_resolve    adds the next-event contributions (light first, then environment, as main
//                   does); a path that continues is queued for the next iteration, a finished
//                   path stores its radiance under its unit and the slot starts the next unit
//   k_wf_control    advances the iteration and decides whether another one runs
// The loop is a WHILE node of a CUDA graph (the control kernel sets its condition), so a render
// call is one graph launch.  k_wf_accumulate then folds each pixel's samples into the running
// mean in sample order, so the accumulation buffer and the rgba8 image equal the reference's
// frame-by-frame result bit for bit, whatever order the paths finished in.  Every
// floating-point operation and random draw of a path happens in the order of the reference;
// only the place where it happens changes, so results equal the single-kernel form and the CPU
// restatement bit for bit.
#include <algorithm>
#include <cstring>
#include <vector>
#include "pt_device.cuh"
#include "traverse.cuh"
#include "wgpt_internal.h"

namespace pt {

struct WfBuffers {
  float4* ray;       // 2 per path (one 32-byte sector): origin.xyz, direction.xyz
  float4* tr;        // 2 per path: (throughput.xyz, last_surface_pdf), (radiance.xyz, last_weight_sum)
  uint4* meta;       // rng, flags, bounce of the current segment, medium count
  uint32_t* unit;    // work unit of the slot's path
  float4* med;       // 8 per path: (ior, sigma.xyz), (emission.xyz, -) for media 0..3
  uint4* hit;        // 2 per path: (t, m_idx, o_idx, kind), (id, aux, bu, bv)
  uint2* tsrc;       // 1 per path: tangent-frame source of the hit (tsrc, tsrc_t), with normal maps
  float4* nee;       // 4 per path: (tp.xyz, -), (incoming.xyz, -) for the light and env records;
                     // with alpha-textured shadows `incoming` holds the BSDF weight alone
  float4* necol;     // 2 per path: the records' light colour (alpha-textured shadows only)
  float4* shadow;    // 4 per path: (origin.xyz, target_dist), (direction.xyz, ignore_idx) x 2
  float* vis;        // 2 per path: transmittance of the record's shadow ray (0 when blocked)
  uint32_t* qcont[2];  // paths continuing into the iteration (ping-pong by iteration parity)
  uint32_t* qnew[2];   // slots that started a new unit for the iteration
  uint32_t* hitq;    // paths of the iteration that hit a surface
  uint32_t* shq;     // shadow-ray queue: slot * 2 + record
};

// Per-iteration counters, a ring of four sets indexed by iteration & 3.
enum Cnt : int { K_CONT = 0, K_NEW = 1, K_EXT_CURSOR = 2, K_HIT = 3, K_SHADOW = 4, K_SH_CURSOR = 5, K_NKINDS = 8 };

// meta.y flags
enum : uint32_t {
  F_ALIVE = 1u,          // continues to the next bounce
  F_NEE_LIGHT = 2u,      // a light NEE contribution was recorded this bounce
  F_NEE_ENV = 4u,        // an environment NEE contribution was recorded this bounce
  F_SHADOW_LIGHT = 8u,   // ... and it needs its shadow ray traced
  F_SHADOW_ENV = 16u
};

}  // namespace pt

namespace wgpt {

// One camera view of a pass: its parameters, its section and the samples it gets.
struct WfView {
  pt::DParams p;          // the view's 112-byte parameters; sec_x/sec_y = section origin
  uint32_t sec_w, npix;   // section width, section pixel count
  uint32_t first_frame;   // sample_number of the pass's first sample of the view
  uint32_t spp;           // samples of the view in the pass
  uint32_t unit_base;     // unit = unit_base + sample * npix + pixel
  uint32_t pix_base;      // first pixel of the view in the pass's pixel numbering
  uint32_t out_pitch;     // pixels per row of the view's images
  uint32_t job;           // index of the view in the caller's list (completion tracking)
  float4* accum;
  uchar4* out;
  double* acc64;          // optional FP64 Welford records (8 doubles per pixel)
  uint64_t pad2;
};

// Device control block of a pass.
struct WfCtl {
  uint32_t iter;          // current iteration
  uint32_t unit_next;     // next unit to hand out
  uint32_t n_units;       // units of the pass
  uint32_t max_iter;      // bound on the iterations (host-computed; the loop stops there)
  uint32_t n_views, n_pixels, fill_count, cond;
  uint32_t track;         // record when each view's last sample finishes
  uint32_t first_pass;    // the fill kernel records the start time
  uint32_t pad[2];
  uint32_t counts[4][pt::K_NKINDS];
  pt::DParams sp;         // scene-level parameters (sky size, luminance, CDF offset) of the pass
};

}  // namespace wgpt

namespace pt {

using wgpt::WfCtl;
using wgpt::WfView;

enum : uint32_t { ERR_ITER = 2u };   // the iteration bound was reached with paths left

struct WfArgs {
  DScene s;
  DPairs P;
  WfBuffers b;
  const WfView* views;
  WfCtl* ctl;
  float4* samples;        // radiance of every unit of the pass
  uint32_t* remaining;    // per view of the call: samples still being traced
  unsigned long long* done_ns;   // per view: global timer when its last sample finished
  unsigned long long* t0_ns;     // global timer at the start of the call's first pass
  uint32_t* status;
  unsigned long long* counters;
  uint32_t refill_closest;       // lanes a warp lets go idle before it refills (closest hit)
  uint32_t refill_shadow;        // the same for the shadow kernel
};

// The iteration's input queue: continuing paths, then the slots that started a new unit.
struct QIn {
  const uint32_t* qc;
  const uint32_t* qn;
  uint32_t nc, n;
  __device__ __forceinline__ uint32_t at(uint32_t i) const { return i < nc ? qc[i] : qn[i - nc]; }
};
__device__ __forceinline__ QIn queue_in(const WfArgs& a, uint32_t iter) {
  QIn q;
  uint32_t r = iter & 3u, p = iter & 1u;
  q.qc = a.b.qcont[p];
  q.qn = a.b.qnew[p];
  q.nc = a.ctl->counts[r][K_CONT];
  q.n = q.nc + a.ctl->counts[r][K_NEW];
  return q;
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

// Block-wide allocation of `k` entries per thread from one atomicAdd on `count`; returns the
// thread's first entry.  Every thread of the block calls it at the same point (the kernels'
// loops run the same number of times in all threads of a block).  One atomic per block instead
// of one per warp: all the block's pushes to a queue share a single counter, and same-address
// atomics are serialised in L2.  `sh` is a __shared__ array of blockDim.x / 32 + 1 words.
__device__ __forceinline__ uint32_t block_alloc(uint32_t* count, uint32_t k, uint32_t* sh) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  uint32_t x = k;   // inclusive scan over the warp
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sh[warp] = x;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t tot = 0;
    for (int w = 0; w < nw; ++w) {
      uint32_t c = sh[w];
      sh[w] = tot;
      tot += c;
    }
    sh[nw] = tot ? atomicAdd(count, tot) : 0u;
  }
  __syncthreads();
  const uint32_t r = sh[nw] + sh[warp] + x - k;
  __syncthreads();   // sh is reused by the next call
  return r;
}

// The view a unit belongs to (views are ordered by unit_base).
__device__ __forceinline__ const WfView* find_view(const WfArgs& a, uint32_t n_views, uint32_t u) {
  uint32_t lo = 0, hi = n_views;
  while (hi - lo > 1u) {
    uint32_t mid = (lo + hi) >> 1;
    if (a.views[mid].unit_base <= u) lo = mid; else hi = mid;
  }
  return a.views + lo;
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Pixel of ordinal `pix` within a section of sec_w x (npix / sec_w) pixels.  The section is cut
// into bands of kTileH rows and each band into blocks kTileW wide (the last band and each band's
// last block may be smaller), numbered block by block and row-major inside a block, so the 32
// consecutive units a warp starts are camera rays through a 4 x 8 block rather than a 32 x 1
// strip.  Only the order in which pixels are started changes: each pixel keeps its own RNG seed
// and sample numbers, and the accumulation folds its samples in sample order.  Measured on the
// flagship (M paths/s, one box): rows 624.6, 16 x 2 623.6, 8 x 4 628.0, 4 x 8 629.7.
constexpr uint32_t kTileW = 4u, kTileH = 8u;
__device__ __forceinline__ void section_pixel(uint32_t pix, uint32_t sec_w, uint32_t npix, uint32_t& dx,
                                              uint32_t& dy) {
  const uint32_t band_px = kTileH * sec_w;
  const uint32_t band = pix / band_px;
  const uint32_t r = pix - band * band_px;
  const uint32_t bh = min(kTileH, npix / sec_w - band * kTileH);   // rows of this band
  const uint32_t blk_px = kTileW * bh;
  const uint32_t full = sec_w / kTileW;                             // blocks kTileW wide
  const uint32_t blk = r / blk_px;
  uint32_t x0, bw, k;
  if (blk < full) {
    x0 = blk * kTileW; bw = kTileW; k = r - blk * blk_px;
  } else {
    x0 = full * kTileW; bw = sec_w - x0; k = r - full * blk_px;
  }
  dx = x0 + k % bw;
  dy = band * kTileH + k / bw;
}

// Starts unit `u` in path slot `slot`: RNG seeding and discard, jittered camera ray
// (shader.wgsl:2276-2287 with sample_number = the unit's sample).
template <bool COUNT>
__device__ __forceinline__ void spawn(const WfArgs& a, uint32_t n_views, uint32_t slot, uint32_t u,
                                      Counters<COUNT>& cn) {
  const WfView* v = find_view(a, n_views, u);
  uint32_t l = u - v->unit_base;
  uint32_t k = l / v->npix;
  uint32_t pix = l - k * v->npix;
  uint32_t dx, dy;
  section_pixel(pix, v->sec_w, v->npix, dx, dy);
  uint32_t ix = v->p.sec_x + dx;
  uint32_t iy = v->p.sec_y + dy;
  uint32_t width = v->p.width, height = v->p.height;
  uint32_t idx = iy * width + ix;
  uint32_t sample_number = v->first_frame + k;
  uint32_t rng = (idx * 1973u + sample_number * 9277u + v->p.seed * 26699u) | 1u;
  rand_pcg(rng);
  cn.add(C_PATHS);
  float j0 = rand_pcg(rng);
  float j1 = rand_pcg(rng);
  float su = ((float)ix + j0) / (float)width;
  float sv = ((float)iy + j1) / (float)height;
  v3 d = normalize(vmix(vmix(v->p.ray00, v->p.ray10, su), vmix(v->p.ray01, v->p.ray11, su), 1.0f - sv));
  v3 eye = v->p.eye;
  a.b.ray[slot * 2] = make_float4(eye.x, eye.y, eye.z, 0.0f);
  a.b.ray[slot * 2 + 1] = make_float4(d.x, d.y, d.z, 0.0f);
  a.b.tr[slot * 2] = make_float4(1.0f, 1.0f, 1.0f, 1.0f);
  a.b.tr[slot * 2 + 1] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  a.b.meta[slot] = make_uint4(rng, 0u, 0u, 0u);
  a.b.unit[slot] = u;
}

// ---------------------------------------------------------------------------- fill
// Starts the pass: slot i takes unit i for the first fill_count units.
template <bool COUNT>
__global__ void __launch_bounds__(256) k_wf_fill(WfArgs a) {
  Counters<COUNT> cn; cn.init();
  const uint32_t n = a.ctl->fill_count, n_views = a.ctl->n_views;
  if (a.ctl->track && a.ctl->first_pass && blockIdx.x == 0 && threadIdx.x == 0) *a.t0_ns = global_ns();
  for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    uint32_t slot = base + threadIdx.x;
    if (slot < n) {
      spawn<COUNT>(a, n_views, slot, slot, cn);
      a.b.qnew[0][slot] = slot;
    }
  }
  flush_wf<COUNT>(cn, a.counters, true);
}

// ---------------------------------------------------------------------------- extend
constexpr unsigned FULL = 0xffffffffu;

// Hands queue entries to the lanes of a warp that have no ray, from a shared cursor; returns the
// entry index for this lane (>= n when there is none).  `exhausted` becomes true (warp-uniform)
// once the queue has been handed out completely.  A warp refills only when at least MIN lanes
// are idle (or all are): a refill runs the ray set-up for the idle lanes while the others wait,
// so taking several at once costs less than refilling lane by lane.  Measured on the flagship
// (M paths/s, one box, one threshold for both traversal kernels): 1: 658.0, 4: 665.8, 8: 674.2,
// 16: 680.6, 20: 682.3, 24: 682.4, 28: 678.5, 32: 663.5; the shadow kernel alone is fastest at 8
// or below (47.7 ms per step at 8, 49.0 at 24, 52.2 at 32).
// The thresholds are arguments (WfArgs::refill_closest / refill_shadow; defaults 24 and 8, set by
// the wavefront tuning) so the autotuner can choose them per scene.
constexpr uint32_t kRefillMinClosest = 24;
constexpr uint32_t kRefillMinShadow = 8;
__device__ __forceinline__ uint32_t refill(uint32_t min_idle, bool have, uint32_t* cursor, uint32_t n, bool& exhausted) {
  uint32_t qi = 0xffffffffu;
  unsigned need = __ballot_sync(FULL, !have);
  if (need && ((uint32_t)__popc(need) >= min_idle || need == FULL)) {
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

// Traversal kernels are latency bound; their block shape trades registers for resident warps.
// Measured on one box (flagship / batch, M paths/s): 256 x 4 per SM at 64 registers 569 / 691;
// 256 x 5 at 48 (spilling) 597 / 732; 192 x 6 at 56 (closest hit without spills) 627 / 748;
// 128 x 9 at 56 625 / 748; 128 x 10 at 48 596 / 734.  Three shapes are compiled and the
// wavefront tuning picks one: 0 = 192 x 6 (default), 1 = 128 x 9, 2 = 256 x 4.
constexpr int kTravShapes = 3;
__host__ __device__ constexpr int trav_threads(int shape) { return shape == 1 ? 128 : shape == 2 ? 256 : 192; }
__host__ __device__ constexpr int trav_blocks(int shape) { return shape == 1 ? 9 : shape == 2 ? 4 : 6; }

template <bool COUNT, int SHAPE>
__global__ void __launch_bounds__(trav_threads(SHAPE), trav_blocks(SHAPE)) k_wf_extend(WfArgs a) {
  Counters<COUNT> cn; cn.init();
  uint32_t err = 0;
  const uint32_t iter = a.ctl->iter;
  const QIn q = queue_in(a, iter);
  const uint32_t n = q.n;
  uint32_t* cursor = &a.ctl->counts[iter & 3u][K_EXT_CURSOR];
  ClosestTrav t;
  bool have = false, exhausted = false;
  uint32_t slot = 0;
  while (true) {
    if (!exhausted) {
      uint32_t qi = refill(a.refill_closest, have, cursor, n, exhausted);
      if (!have && qi < n) {
        slot = q.at(qi);
        float4 o = a.b.ray[slot * 2], d = a.b.ray[slot * 2 + 1];
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
      if (HAS(a.s, wgpt::SCENE_TANGENTS)) a.b.tsrc[slot] = make_uint2((uint32_t)h.tsrc, __float_as_uint(h.tsrc_t));
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

// Walks the iteration's queue in order: paths that hit a surface go to the hit queue (kept in
// queue order within each block, so the surface stage sees rays as coherent as the queue); paths
// that left the scene are shaded here: medium, then the sky (MIS-weighted after the first
// bounce) or the background colour (shader.wgsl:2344-2358).  They end here.
template <bool COUNT>
__global__ void __launch_bounds__(256) k_wf_shade_miss(WfArgs a) {
  Counters<COUNT> cn; cn.init();
  const DScene& s = a.s;
  const uint32_t iter = a.ctl->iter;
  const QIn q = queue_in(a, iter);
  const uint32_t n = q.n;
  uint32_t* hit_count = &a.ctl->counts[iter & 3u][K_HIT];
  const DParams& sp = a.ctl->sp;
  __shared__ uint32_t sh[9];
  for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    uint32_t i = base + threadIdx.x;
    bool is_hit = false;
    uint32_t slot = 0;
    if (i < n) {
      slot = q.at(i);
      is_hit = (int32_t)a.b.hit[slot * 2].y != -1;
    }
    const uint32_t at = block_alloc(hit_count, is_hit ? 1u : 0u, sh);
    if (is_hit) a.b.hitq[at] = slot;
    if (i < n && !is_hit) {
      float4 d4 = a.b.ray[slot * 2 + 1], tp4 = a.b.tr[slot * 2], rd4 = a.b.tr[slot * 2 + 1];
      uint4 meta = a.b.meta[slot];
      const int bounce = (int)meta.z;
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
          float sky_pdf = get_sky_pdf(s, sp, dir, cn);
          weight = mis_weight(tp4.w, sky_pdf);
        }
        radiance = radiance + throughput * clamp_firefly(sky_color * weight, bounce);
      } else {
        radiance = radiance + throughput * clamp_firefly(mk3(0.02f, 0.03f, 0.05f), bounce);
      }
      a.b.tr[slot * 2 + 1] = make_float4(radiance.x, radiance.y, radiance.z, rd4.w);
      a.b.meta[slot] = make_uint4(meta.x, 0u, meta.z, meta.w);
    }
  }
  flush_wf<COUNT>(cn, a.counters, true);
}

// Records one next-event contribution: the throughput it is weighted by, the incoming
// radiance if the light is visible, and the shadow ray to test (when evaluate_nee reaches it).
template <bool COUNT, bool TEX>
__device__ void record_nee(const WfArgs& a, uint32_t slot, int rec, const LightSample& ls, v3 hit_pos, v3 n_orient,
                           v3 V, const DMat& mat, const SurfCtx& ctx, const TexPoint& tp, const MediumStack& stack,
                           int32_t ignore_idx, v3 throughput, uint32_t& flags) {
  v3 incoming = mk3s(0.0f);
  bool shadow = false;
  v3 so = mk3s(0.0f);
  // shader.wgsl:2226-2271 up to the shadow ray
  if (ls.pdf > 0.0f) {
    float dotNL = dot(n_orient, ls.dir);
    if (!(dotNL <= 0.0f && mat.transmission <= 0.0f)) {
      v3 bsdf_val; float bsdf_pdf;
      bsdf_eval_pdf<TEX>(V, ls.dir, mat, ctx, stack, &bsdf_val, &bsdf_pdf);
      float weight = mis_weight(ls.pdf, bsdf_pdf);
      v3 c_weight = (bsdf_val * weight) / wmax(ls.pdf, 1e-6f);
      v2 pom_uv;
      if (!(max_component(ls.color * c_weight) < 1e-5f) && !pom_shadowed<TEX>(a.s, tp, ls.dir, &pom_uv)) {
        v3 ray_offset = dotNL < 0.0f ? -n_orient * 0.001f : n_orient * 0.001f;
        so = hit_pos + ray_offset;
        if (HAS_TEX<TEX>(a.s, wgpt::SCENE_ALPHA_SHADOWS)) {
          // (colour * transmittance) * weight once the shadow ray is traced
          incoming = c_weight;
          a.b.necol[slot * 2 + rec] = make_float4(ls.color.x, ls.color.y, ls.color.z, 0.0f);
        } else {
          incoming = ls.color * c_weight;   // transmittance 1 or 0
        }
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

// sample_surface (shader.wgsl:2052-2175) with the single-kernel form's arithmetic; the VNDF
// sampler has one call site for the three microfacet lobes.  False when the path ends.
template <bool TEX>
__device__ __forceinline__ bool wf_sample_surface(Ray& ray, v3& throughput, v3 hit_pos, const DMat& mat,
                                                  const SurfCtx& ctx, MediumStack& stack, float& last_surface_pdf,
                                                  uint32_t& rng) {
  const v3 V = -ray.direction;
  const v3 n_orient = dot(ctx.normal, V) > 0.0f ? ctx.normal : -ctx.normal;
  bool alive = false;
  {
    bool entering = dot(ctx.normal, V) > 0.0f;
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
    if (rand_pcg(rng) > ctx.alpha) {   // alpha cut-out: the path passes through
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
          bsdf_eval_pdf<TEX>(V, L, mat, ctx, stack, &bsdf_val, &pdf_val);
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
  return alive;
}

// Surface shading blocks: one 512-thread block per SM at 128 registers; textured scenes need
// ~200 registers and keep 256-thread blocks.  Measured on the flagship (M paths/s, one box):
// 128 threads 868.6, 256 threads 916.0, 512 threads 957.4 (shading 40.8 / 33.2 / 27.1 ms per
// step): the larger the block, the fewer block-wide queue allocations and blocks to schedule.
// The wavefront tuning can also choose 256-thread blocks for untextured scenes.
template <bool TEX>
constexpr int shade_threads() { return TEX ? 256 : 512; }

template <bool COUNT, bool TEX, int THREADS>
__global__ void __launch_bounds__(THREADS) k_wf_shade(WfArgs a) {
  Counters<COUNT> cn; cn.init();
  const DScene& s = a.s;
  const uint32_t iter = a.ctl->iter;
  const uint32_t* __restrict__ q = a.b.hitq;
  const uint32_t n = a.ctl->counts[iter & 3u][K_HIT];
  uint32_t* sh_count = &a.ctl->counts[iter & 3u][K_SHADOW];
  const DParams& p = a.ctl->sp;
  __shared__ uint32_t shq[512 / 32 + 1];
  for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    uint32_t i = base + threadIdx.x;
    bool alive = false, sh_light = false, sh_env = false;
    uint32_t slot = 0;
    if (i < n) {
      slot = q[i];
      float4 o4 = a.b.ray[slot * 2], d4 = a.b.ray[slot * 2 + 1], tp4 = a.b.tr[slot * 2], rd4 = a.b.tr[slot * 2 + 1];
      uint4 meta = a.b.meta[slot];
      const int bounce = (int)meta.z;
      uint4 h0 = a.b.hit[slot * 2], h1 = a.b.hit[slot * 2 + 1];
      HitRec hit;
      hit.t = __uint_as_float(h0.x); hit.m_idx = (int32_t)h0.y; hit.o_idx = (int32_t)h0.z; hit.kind = (int32_t)h0.w;
      hit.id = (int32_t)h1.x; hit.aux = (int32_t)h1.y; hit.bu = __uint_as_float(h1.z); hit.bv = __uint_as_float(h1.w);
      hit.tsrc = -1; hit.tsrc_t = 0.0f;
      if (HAS_TEX<TEX>(s, wgpt::SCENE_TANGENTS)) {
        uint2 ts = a.b.tsrc[slot];
        hit.tsrc = (int32_t)ts.x; hit.tsrc_t = __uint_as_float(ts.y);
      }
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
        v3 hn = hit_normal(s, ray, hit);
        TexPoint tp;
        SurfCtx ctx = hit_context<TEX>(s, ray, hit, mat, hn, &tp, true);
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
                float cos_l = wmax(dot(-ray.direction, hn), 1e-6f);
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
              record_nee<COUNT, TEX>(a, slot, 0, ls, hit_pos, n_orient, V, mat, ctx, tp, stack, light.obj_idx, throughput,
                                     flags);
            }
          }
          last_weight_sum = weight_sum;
        }
        if (HAS(s, WGPT_HAS_SKYBOX) && HAS(s, WGPT_MIS_SKYBOX)) {
          cn.add(C_ENV_NEE);
          float u0 = rand_pcg(rng);
          float u1 = rand_pcg(rng);
          LightSample env = sample_env_cdf(s, p, u0, u1, cn);
          record_nee<COUNT, TEX>(a, slot, 1, env, hit_pos, n_orient, V, mat, ctx, tp, stack, -1, throughput, flags);
        }
        // shader.wgsl:2052-2175 -- the same arithmetic as the single-kernel form
        int32_t count_before = stack.count;
        alive = wf_sample_surface<TEX>(ray, throughput, hit_pos, mat, ctx, stack, last_surface_pdf, rng);
        if (!alive) break;
        const int32_t low = count_before < stack.count ? count_before : stack.count;
        // shader.wgsl:2458-2472: the height field shadows the sampled direction: shade the
        // occluding texel and sample again from it
        v2 pom_uv;
        if (pom_shadowed<TEX>(s, tp, ray.direction, &pom_uv)) {
          SurfCtx cp = surface_context(s, mat, hn, tp, pom_uv);
          radiance = radiance + throughput * clamp_firefly(cp.emittance, bounce);
          if (length(cp.emittance) > 1.0f) { alive = false; break; }
          alive = wf_sample_surface<TEX>(ray, throughput, hit_pos, mat, cp, stack, last_surface_pdf, rng);
          if (!alive) break;
        }
        if (TEX) {
          for (int32_t m = low; m < stack.count; ++m) store_medium(a, slot, (uint32_t)m, stack.media[m]);
        } else if (stack.count > count_before) {
          store_medium(a, slot, (uint32_t)(stack.count - 1), stack.media[stack.count - 1]);
        }
        if (bounce < 2) break;
        float survival_prob = clamp(max_component(throughput), 0.05f, 0.95f);
        if (rand_pcg(rng) > survival_prob) { alive = false; break; }
        throughput = throughput / survival_prob;
      } while (false);
      if (bounce + 1 >= s.bounce_limit) alive = false;
      if (alive) flags |= F_ALIVE;
      sh_light = (flags & F_SHADOW_LIGHT) != 0u;
      sh_env = (flags & F_SHADOW_ENV) != 0u;
      a.b.ray[slot * 2] = make_float4(ray.origin.x, ray.origin.y, ray.origin.z, 0.0f);
      a.b.ray[slot * 2 + 1] = make_float4(ray.direction.x, ray.direction.y, ray.direction.z, 0.0f);
      a.b.tr[slot * 2] = make_float4(throughput.x, throughput.y, throughput.z, last_surface_pdf);
      a.b.tr[slot * 2 + 1] = make_float4(radiance.x, radiance.y, radiance.z, last_weight_sum);
      a.b.meta[slot] = make_uint4(rng, flags, (uint32_t)bounce, (uint32_t)stack.count);
    }
    const uint32_t at = block_alloc(sh_count, (sh_light ? 1u : 0u) + (sh_env ? 1u : 0u), shq);
    if (sh_light) a.b.shq[at] = slot * 2u;
    if (sh_env) a.b.shq[at + (sh_light ? 1u : 0u)] = slot * 2u + 1u;
  }
  flush_wf<COUNT>(cn, a.counters, true);
}

// ---------------------------------------------------------------------------- shadow
// WIDE: the 4-wide any-hit walk over the quad records (untextured scenes, no counting).
template <bool COUNT, bool TEX, int SHAPE, bool WIDE = false>
__global__ void __launch_bounds__(trav_threads(SHAPE), TEX ? 3 * 256 / trav_threads(SHAPE) : trav_blocks(SHAPE))
k_wf_shadow(WfArgs a) {
  Counters<COUNT> cn; cn.init();
  uint32_t err = 0;
  const uint32_t iter = a.ctl->iter;
  const uint32_t n = a.ctl->counts[iter & 3u][K_SHADOW];
  uint32_t* cursor = &a.ctl->counts[iter & 3u][K_SH_CURSOR];
  ShadowTrav t;
  bool have = false, exhausted = false;
  uint32_t e = 0;
  while (true) {
    if (!exhausted) {
      uint32_t qi = refill(a.refill_shadow, have, cursor, n, exhausted);
      if (!have && qi < n) {
        e = a.b.shq[qi];
        float4 so = a.b.shadow[(e >> 1) * 4 + (e & 1u) * 2], sd = a.b.shadow[(e >> 1) * 4 + (e & 1u) * 2 + 1];
        t.rw.origin = mk3(so.x, so.y, so.z);
        t.rw.direction = mk3(sd.x, sd.y, sd.z);
        t.target_dist = so.w;
        t.target_idx = __float_as_int(sd.w);
        shadow_init<COUNT, TEX>(a.s, t, cn);
        have = true;
      }
    }
    if (!__any_sync(FULL, have)) break;
    if (have && shadow_step<COUNT, TEX, WIDE>(a.s, a.P, t, err, cn)) {
      shadow_finish<COUNT, TEX>(a.s, t, err, cn);
      a.b.vis[e] = t.occluded ? 0.0f : t.trans;
      have = false;
    }
  }
  flush_wf<COUNT>(cn, a.counters, true);
  if (err) atomicOr(a.status, err);
}

// ---------------------------------------------------------------------------- resolve
// Adds the recorded next-event contributions (shader.wgsl:2271 with the shadow result), queues
// continuing paths for the next iteration, stores the radiance of finished paths under their
// unit and starts the next units in the freed slots (handed out in queue order within a block).
template <bool COUNT>
__global__ void __launch_bounds__(256) k_wf_resolve(WfArgs a) {
  Counters<COUNT> cn; cn.init();
  const uint32_t iter = a.ctl->iter;
  const QIn q = queue_in(a, iter);
  const uint32_t n = q.n;
  const uint32_t r1 = (iter + 1u) & 3u, p1 = (iter + 1u) & 1u;
  uint32_t* cont_count = &a.ctl->counts[r1][K_CONT];
  uint32_t* new_count = &a.ctl->counts[r1][K_NEW];
  const uint32_t n_units = a.ctl->n_units, n_views = a.ctl->n_views;
  const bool track = a.ctl->track != 0u;
  __shared__ uint32_t sh[9];
  for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    uint32_t i = base + threadIdx.x;
    bool alive = false, ended = false;
    uint32_t slot = 0, unit = 0;
    if (i < n) {
      slot = q.at(i);
      uint4 meta = a.b.meta[slot];
      uint32_t flags = meta.y;
      int bounce = (int)meta.z;
      float4 rd4 = a.b.tr[slot * 2 + 1];
      v3 radiance = mk3(rd4.x, rd4.y, rd4.z);
      if (flags & (F_NEE_LIGHT | F_NEE_ENV)) {
#pragma unroll
        for (int rec = 0; rec < 2; ++rec) {
          uint32_t has = rec == 0 ? F_NEE_LIGHT : F_NEE_ENV;
          uint32_t needs = rec == 0 ? F_SHADOW_LIGHT : F_SHADOW_ENV;
          if (!(flags & has)) continue;
          float4 t4 = a.b.nee[slot * 4 + rec * 2], c4 = a.b.nee[slot * 4 + rec * 2 + 1];
          v3 incoming = mk3(c4.x, c4.y, c4.z);
          if (flags & needs) {
            float sh = a.b.vis[slot * 2 + rec];
            if (sh < 0.001f) {
              incoming = mk3s(0.0f);
            } else if (HAS(a.s, wgpt::SCENE_ALPHA_SHADOWS)) {
              float4 col = a.b.necol[slot * 2 + rec];
              incoming = (mk3(col.x, col.y, col.z) * sh) * incoming;
            }
          }
          radiance = radiance + mk3(t4.x, t4.y, t4.z) * clamp_firefly(incoming, bounce);
        }
      }
      if (flags & F_ALIVE) {
        alive = true;
        if (flags & (F_NEE_LIGHT | F_NEE_ENV)) a.b.tr[slot * 2 + 1] = make_float4(radiance.x, radiance.y, radiance.z, rd4.w);
        a.b.meta[slot] = make_uint4(meta.x, 0u, meta.z + 1u, meta.w);
      } else {
        unit = a.b.unit[slot];
        a.samples[unit] = make_float4(radiance.x, radiance.y, radiance.z, 0.0f);
        ended = true;
      }
    }
    const uint32_t at = block_alloc(cont_count, alive ? 1u : 0u, sh);
    if (alive) a.b.qcont[p1][at] = slot;
    unsigned em = __ballot_sync(0xffffffffu, ended);
    if (track && ended) {
      // one atomic per view per warp; the lane that takes a view's count to zero stamps it
      uint32_t job = find_view(a, n_views, unit)->job;
      unsigned peers = __match_any_sync(em, job);
      if ((int)(threadIdx.x & 31) == __ffs(peers) - 1) {
        uint32_t k = (uint32_t)__popc(peers);
        if (atomicSub(&a.remaining[job], k) == k) a.done_ns[job] = global_ns();
      }
    }
    bool started = false;
    const uint32_t u = block_alloc(&a.ctl->unit_next, ended ? 1u : 0u, sh);
    if (ended && u < n_units) {
      spawn<COUNT>(a, n_views, slot, u, cn);
      started = true;
    }
    const uint32_t at_new = block_alloc(new_count, started ? 1u : 0u, sh);
    if (started) a.b.qnew[p1][at_new] = slot;
  }
  flush_wf<COUNT>(cn, a.counters, true);
}

// ---------------------------------------------------------------------------- control
// Ends an iteration: clears the counter set the next iteration writes into, advances the
// iteration and continues the loop while paths are queued (and the iteration bound is not hit).
template <bool GRAPH>
__global__ void k_wf_control(WfArgs a, cudaGraphConditionalHandle h) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  WfCtl* c = a.ctl;
  const uint32_t iter = c->iter;
  const uint32_t r1 = (iter + 1u) & 3u, r2 = (iter + 2u) & 3u;
  for (int k = 0; k < K_NKINDS; ++k) c->counts[r2][k] = 0u;
  uint32_t next = c->counts[r1][K_CONT] + c->counts[r1][K_NEW];
  uint32_t go = next > 0u ? 1u : 0u;
  if (go && iter + 1u >= c->max_iter) {
    go = 0u;
    atomicOr(a.status, ERR_ITER);
  }
  c->iter = iter + 1u;
  c->cond = go;
  if (GRAPH) cudaGraphSetConditional(h, go);
}

// ---------------------------------------------------------------------------- accumulate
// Folds each pixel's samples into the running mean in sample order (shader.wgsl:2482-2491 once
// per sample: accum = mix(accum, L, 1/(sample_number+1)), alpha 1) and writes the rgba8 image of
// the last sample.
__global__ void __launch_bounds__(256) k_wf_accumulate(WfArgs a) {
  const uint32_t n = a.ctl->n_pixels, n_views = a.ctl->n_views;
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < n; g += gridDim.x * blockDim.x) {
    uint32_t lo = 0, hi = n_views;
    while (hi - lo > 1u) {
      uint32_t mid = (lo + hi) >> 1;
      if (a.views[mid].pix_base <= g) lo = mid; else hi = mid;
    }
    const WfView* v = a.views + lo;
    uint32_t pix = g - v->pix_base;
    uint32_t dx, dy;
    section_pixel(pix, v->sec_w, v->npix, dx, dy);
    uint32_t ix = v->p.sec_x + dx;
    uint32_t iy = v->p.sec_y + dy;
    size_t idx = (size_t)iy * v->p.width + ix;
    float4 acc4 = v->accum[idx];
    v3 acc = mk3(acc4.x, acc4.y, acc4.z);
    const float4* smp = a.samples + v->unit_base + pix;
    for (uint32_t k = 0; k < v->spp; ++k) {
      float4 L = smp[(size_t)k * v->npix];
      float weight = 1.0f / (float)(v->first_frame + k + 1u);
      acc = vmix(acc, mk3(L.x, L.y, L.z), weight);
    }
    v->accum[idx] = make_float4(acc.x, acc.y, acc.z, 1.0f);
    if (v->acc64) {
      // the same samples, in the same order, into an FP64 mean and sum of squared deviations
      double* r = v->acc64 + idx * 8;
      double m0 = r[0], m1 = r[1], m2 = r[2], q0 = r[3], q1 = r[4], q2 = r[5], cnt = r[6];
      for (uint32_t k = 0; k < v->spp; ++k) {
        float4 L = smp[(size_t)k * v->npix];
        cnt += 1.0;
        double d0 = (double)L.x - m0, d1 = (double)L.y - m1, d2 = (double)L.z - m2;
        m0 += d0 / cnt; m1 += d1 / cnt; m2 += d2 / cnt;
        q0 += d0 * ((double)L.x - m0); q1 += d1 * ((double)L.y - m1); q2 += d2 * ((double)L.z - m2);
      }
      r[0] = m0; r[1] = m1; r[2] = m2; r[3] = q0; r[4] = q1; r[5] = q2; r[6] = cnt;
    }
    v3 c = acc * mk3s(v->p.exposure);
    c = c / (c + mk3s(0.3f));
    c = vpow(c, 0.4545f);
    v->out[(size_t)iy * v->out_pitch + ix] =
        make_uchar4((unsigned char)unorm8(c.x), (unsigned char)unorm8(c.y), (unsigned char)unorm8(c.z), 255);
  }
}

}  // namespace pt

namespace wgpt {

using namespace pt;

static void fill_dscene(DScene& s, const DeviceScene& d) {
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
}

static void fill_dparams(DParams& p, const wgpt_scene_params& q, uint32_t sec_x, uint32_t sec_y) {
  p.eye = mk3(q.eye[0], q.eye[1], q.eye[2]); p.sample_number = q.sample_number;
  p.ray00 = mk3(q.ray00[0], q.ray00[1], q.ray00[2]); p.width = q.width;
  p.ray10 = mk3(q.ray10[0], q.ray10[1], q.ray10[2]); p.height = q.height;
  p.ray01 = mk3(q.ray01[0], q.ray01[1], q.ray01[2]); p.exposure = q.exposure;
  p.ray11 = mk3(q.ray11[0], q.ray11[1], q.ray11[2]); p.seed = q.seed;
  p.sky_width = q.sky_width; p.sky_height = q.sky_height;
  p.sky_total_lum = q.sky_total_lum; p.total_light_power = q.total_light_power;
  p.sec_x = sec_x; p.sec_y = sec_y; p.sky_cdf_index = q.sky_cdf_index;
}

// Path-slot state, in carving order: ray 32 + throughput/radiance 32 + meta 16 + unit 4 +
// media 128 + hit 32 + tangent source 8 + nee 64 + light colour 32 + shadow 64 + vis 8 +
// continuing and new queues 16 + hit queue 4 + shadow queue 8.
static constexpr int kParts = 17;
static const uint32_t kPartBytes[kParts] = {32, 32, 16, 4, 128, 32, 8, 64, 32, 64, 8, 4, 4, 4, 4, 4, 8};
size_t wavefront_bytes_per_path() {
  size_t s = 0;
  for (uint32_t x : kPartBytes) s += x;
  return s;
}

static size_t pool_bytes(uint32_t capacity) {
  size_t s = 0;
  for (uint32_t x : kPartBytes) s += ((size_t)capacity * x + 255) & ~(size_t)255;
  return s;
}

static WfBuffers carve(void* scratch, uint32_t capacity) {
  char* p = (char*)scratch;
  auto take = [&](size_t bytes) { char* r = p; p += (bytes + 255) & ~(size_t)255; return (void*)r; };
  WfBuffers b;
  size_t n = capacity;
  b.ray = (float4*)take(n * 32);
  b.tr = (float4*)take(n * 32);
  b.meta = (uint4*)take(n * 16);
  b.unit = (uint32_t*)take(n * 4);
  b.med = (float4*)take(n * 128);
  b.hit = (uint4*)take(n * 32);
  b.tsrc = (uint2*)take(n * 8);
  b.nee = (float4*)take(n * 64);
  b.necol = (float4*)take(n * 32);
  b.shadow = (float4*)take(n * 64);
  b.vis = (float*)take(n * 8);
  b.qcont[0] = (uint32_t*)take(n * 4);
  b.qcont[1] = (uint32_t*)take(n * 4);
  b.qnew[0] = (uint32_t*)take(n * 4);
  b.qnew[1] = (uint32_t*)take(n * 4);
  b.hitq = (uint32_t*)take(n * 4);
  b.shq = (uint32_t*)take(n * 8);
  return b;
}

struct WfEngine {
  // path slots of the pool (upper bound; a pass uses at most its units, and a new allocation at
  // most a quarter of the device's free memory).  Larger pools need fewer iterations per call,
  // so less of each stage's time is its tail: flagship 1080p x 64 spp, M paths/s by pool size
  // 2 M 687, 4 M 742, 8 M 800, 16 M 854, 32 M 895, 64 M 914 (448 bytes per slot: 30 GB).
  uint32_t pool_paths = 1u << 26;
  uint64_t units_per_pass = 1ull << 27;    // samples held before they are folded into the images
  void* pool = nullptr;
  uint32_t pool_cap = 0;
  float4* samples = nullptr;
  uint64_t samples_cap = 0;
  WfView* d_views = nullptr;
  uint32_t views_cap = 0;
  WfCtl* d_ctl = nullptr;
  uint32_t* d_remaining = nullptr;         // per-view completion tracking
  unsigned long long* d_done = nullptr;    // track_cap stamps, then the start stamp
  uint32_t track_cap = 0;
  uint32_t* h_cond = nullptr;              // pinned copy of the loop condition (host-driven loop)
  int grids[8][8] = {{0}};                 // launch grid per stage, per (counting, textured, wide) variant
  int* grid = grids[0];
  // kernel variants and thresholds chosen by the wavefront tuning (wgpt_set_wavefront_tuning)
  int trav_shape = 2;                      // traversal block shape (trav_threads / trav_blocks)
  int shade_block = 512;                   // surface-shading block of untextured scenes: 512 or 256
  uint32_t refill_closest = kRefillMinClosest;
  uint32_t refill_shadow = kRefillMinShadow;
  int shadow_wide = 0;                     // 4-wide any-hit walk for untextured scenes
  bool wide_now = false;                   // this call uses it (tuning, scene, not counting)
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  WfArgs key;
  bool key_count = false;
  bool has_graph = false;
};

WfEngine* wf_engine_create() { return new WfEngine(); }

static void drop_graph(WfEngine* e) {
  if (e->exec) cudaGraphExecDestroy(e->exec);
  if (e->graph) cudaGraphDestroy(e->graph);
  e->exec = nullptr;
  e->graph = nullptr;
  e->has_graph = false;
}

void wf_engine_destroy(WfEngine* e) {
  if (!e) return;
  drop_graph(e);
  if (e->pool) cudaFree(e->pool);
  if (e->samples) cudaFree(e->samples);
  if (e->d_views) cudaFree(e->d_views);
  if (e->d_ctl) cudaFree(e->d_ctl);
  if (e->d_remaining) cudaFree(e->d_remaining);
  if (e->d_done) cudaFree(e->d_done);
  if (e->h_cond) cudaFreeHost(e->h_cond);
  delete e;
}

int wf_engine_tune(WfEngine* e, int trav_shape, int shade_block, uint32_t refill_closest, uint32_t refill_shadow,
                   int shadow_wide) {
  if (trav_shape < 0 || trav_shape >= kTravShapes) return 1;
  if (shade_block != 256 && shade_block != 512) return 1;
  if (refill_closest < 1 || refill_closest > 32 || refill_shadow < 1 || refill_shadow > 32) return 1;
  if (shadow_wide != 0 && shadow_wide != 1) return 1;
  if (trav_shape != e->trav_shape || shade_block != e->shade_block || shadow_wide != e->shadow_wide) {
    memset(e->grids, 0, sizeof e->grids);   // new variants: new occupancy grids and a new graph
    drop_graph(e);
  }
  e->trav_shape = trav_shape;
  e->shade_block = shade_block;
  e->refill_closest = refill_closest;
  e->refill_shadow = refill_shadow;
  e->shadow_wide = shadow_wide;
  return 0;
}

void wf_engine_tuning(const WfEngine* e, int* trav_shape, int* shade_block, uint32_t* refill_closest,
                      uint32_t* refill_shadow, int* shadow_wide) {
  *trav_shape = e->trav_shape;
  *shade_block = e->shade_block;
  *refill_closest = e->refill_closest;
  *refill_shadow = e->refill_shadow;
  *shadow_wide = e->shadow_wide;
}

int wf_engine_configure(WfEngine* e, uint32_t pool_paths, uint64_t units_per_pass) {
  if (pool_paths < 1024u || pool_paths > (1u << 26)) return 1;
  if (units_per_pass < (1ull << 16) || units_per_pass > (1ull << 30)) return 1;
  e->pool_paths = pool_paths;
  e->units_per_pass = units_per_pass;
  return 0;
}

void wf_engine_get(const WfEngine* e, uint32_t* pool_paths, uint64_t* units_per_pass) {
  *pool_paths = e->pool_paths;
  *units_per_pass = e->units_per_pass;
}

template <typename K>
static int occupancy_grid(K kernel, int threads = 256) {
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0);
  return sms * (per_sm > 0 ? per_sm : 1);
}

// The tuned variants of the three kernels that have them.  Textured scenes keep the default
// traversal shape for shadow rays and 256-thread shading blocks (their register counts).
using KFn = void (*)(WfArgs);
struct KernSet {
  KFn extend, shade, shadow;
  int t_extend, t_shade, t_shadow;
};

template <bool COUNT, bool TEX>
static KernSet kernel_set(const WfEngine* e) {
  KernSet k;
  const int sh = e->trav_shape;
  k.extend = sh == 1 ? k_wf_extend<COUNT, 1> : sh == 2 ? k_wf_extend<COUNT, 2> : k_wf_extend<COUNT, 0>;
  k.t_extend = trav_threads(sh);
  if (TEX) {
    k.shadow = k_wf_shadow<COUNT, true, 0>;
    k.t_shadow = trav_threads(0);
    k.shade = k_wf_shade<COUNT, true, shade_threads<true>()>;
    k.t_shade = shade_threads<true>();
  } else {
    if (!COUNT && e->wide_now)
      k.shadow = sh == 1 ? k_wf_shadow<false, false, 1, true> : sh == 2 ? k_wf_shadow<false, false, 2, true>
                                                                      : k_wf_shadow<false, false, 0, true>;
    else
      k.shadow = sh == 1 ? k_wf_shadow<COUNT, false, 1> : sh == 2 ? k_wf_shadow<COUNT, false, 2> : k_wf_shadow<COUNT, false, 0>;
    k.t_shadow = trav_threads(sh);
    k.shade = e->shade_block == 256 ? k_wf_shade<COUNT, false, 256> : k_wf_shade<COUNT, false, 512>;
    k.t_shade = e->shade_block == 256 ? 256 : 512;
  }
  return k;
}

template <bool COUNT, bool TEX>
static void compute_grids(WfEngine* e) {
  e->grid = e->grids[(COUNT ? 2 : 0) + (TEX ? 1 : 0) + (e->wide_now ? 4 : 0)];
  if (e->grid[0]) return;
  const KernSet k = kernel_set<COUNT, TEX>(e);
  e->grid[0] = occupancy_grid(k_wf_fill<COUNT>);
  e->grid[1] = occupancy_grid(k.extend, k.t_extend);
  e->grid[2] = occupancy_grid(k.shade, k.t_shade);
  e->grid[3] = occupancy_grid(k.shadow, k.t_shadow);
  e->grid[4] = occupancy_grid(k_wf_resolve<COUNT>);
  e->grid[5] = occupancy_grid(k_wf_shade_miss<COUNT>);
  e->grid[6] = occupancy_grid(k_wf_accumulate);
  e->grid[7] = 1;
}

static WfArgs stage_args(const WfArgs& a, int stage) {
  WfArgs x = a;
  x.counters = a.counters ? a.counters + 16 * stage : nullptr;
  return x;
}

// The whole pass as one graph: fill -> WHILE(extend, shade_miss, shade, shadow, resolve,
// control) -> accumulate.  Arguments live in device memory (views, control block), so the graph
// only changes when buffers move.
template <bool COUNT, bool TEX>
static cudaError_t build_graph(WfEngine* e, const WfArgs& a) {
  drop_graph(e);
  cudaError_t err;
  cudaGraph_t g = nullptr;
  if ((err = cudaGraphCreate(&g, 0)) != cudaSuccess) return err;
  e->graph = g;
  cudaGraphConditionalHandle h;
  if ((err = cudaGraphConditionalHandleCreate(&h, g, 1u, cudaGraphCondAssignDefault)) != cudaSuccess) return err;
  WfArgs sa[8];
  for (int st = 0; st < 8; ++st) sa[st] = stage_args(a, st);
  const KernSet ks = kernel_set<COUNT, TEX>(e);
  auto add_kernel = [&](cudaGraph_t gr, const void* fn, int grid, void** args, const cudaGraphNode_t* dep,
                        cudaGraphNode_t* out, int threads = 256) -> cudaError_t {
    cudaKernelNodeParams kp;
    memset(&kp, 0, sizeof kp);
    kp.func = const_cast<void*>(fn);
    kp.gridDim = dim3((unsigned)grid);
    kp.blockDim = dim3(grid == 1 ? 32u : (unsigned)threads);
    kp.sharedMemBytes = 0;
    kp.kernelParams = args;
    return cudaGraphAddKernelNode(out, gr, dep, dep ? 1 : 0, &kp);
  };
  cudaGraphNode_t n_fill, n_loop, n_acc;
  void* a_fill[] = {&sa[0]};
  if ((err = add_kernel(g, (const void*)k_wf_fill<COUNT>, e->grid[0], a_fill, nullptr, &n_fill)) != cudaSuccess)
    return err;
  cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};   // the rest zero, as the API requires
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  if ((err = cudaGraphAddNode(&n_loop, g, &n_fill, 1, &cp)) != cudaSuccess) return err;
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  cudaGraphNode_t prev, cur;
  void* a1[] = {&sa[1]};
  void* a5[] = {&sa[5]};
  void* a2[] = {&sa[2]};
  void* a3[] = {&sa[3]};
  void* a4[] = {&sa[4]};
  void* a7[] = {&sa[7], &h};
  if ((err = add_kernel(body, (const void*)ks.extend, e->grid[1], a1, nullptr, &prev, ks.t_extend)) != cudaSuccess)
    return err;
  if ((err = add_kernel(body, (const void*)k_wf_shade_miss<COUNT>, e->grid[5], a5, &prev, &cur)) != cudaSuccess) return err;
  prev = cur;
  if ((err = add_kernel(body, (const void*)ks.shade, e->grid[2], a2, &prev, &cur, ks.t_shade)) != cudaSuccess) return err;
  prev = cur;
  if ((err = add_kernel(body, (const void*)ks.shadow, e->grid[3], a3, &prev, &cur, ks.t_shadow)) != cudaSuccess)
    return err;
  prev = cur;
  if ((err = add_kernel(body, (const void*)k_wf_resolve<COUNT>, e->grid[4], a4, &prev, &cur)) != cudaSuccess) return err;
  prev = cur;
  if ((err = add_kernel(body, (const void*)k_wf_control<true>, 1, a7, &prev, &cur)) != cudaSuccess) return err;
  void* a6[] = {&sa[6]};
  if ((err = add_kernel(g, (const void*)k_wf_accumulate, e->grid[6], a6, &n_loop, &n_acc)) != cudaSuccess) return err;
  if ((err = cudaGraphInstantiate(&e->exec, g, 0)) != cudaSuccess) return err;
  e->key = a;
  e->key_count = COUNT;
  e->has_graph = true;
  return cudaSuccess;
}

// The same pass launched from the host, one event pair per stage launch (stage timing).
template <bool COUNT, bool TEX>
static cudaError_t run_pass_host(WfEngine* e, const WfArgs& a, uint32_t max_iter, cudaStream_t st,
                                 StageTimer* timer) {
  auto T0 = [&](int k) { if (timer) timer->begin(k, st); };
  auto T1 = [&](int k) { if (timer) timer->end(k, st); };
  const KernSet ks = kernel_set<COUNT, TEX>(e);
  T0(0); k_wf_fill<COUNT><<<e->grid[0], 256, 0, st>>>(stage_args(a, 0)); T1(0);
  for (uint32_t it = 0; it <= max_iter; ++it) {
    T0(1); ks.extend<<<e->grid[1], ks.t_extend, 0, st>>>(stage_args(a, 1)); T1(1);
    T0(5); k_wf_shade_miss<COUNT><<<e->grid[5], 256, 0, st>>>(stage_args(a, 5)); T1(5);
    T0(2); ks.shade<<<e->grid[2], ks.t_shade, 0, st>>>(stage_args(a, 2)); T1(2);
    T0(3); ks.shadow<<<e->grid[3], ks.t_shadow, 0, st>>>(stage_args(a, 3)); T1(3);
    T0(4); k_wf_resolve<COUNT><<<e->grid[4], 256, 0, st>>>(stage_args(a, 4)); T1(4);
    T0(7); k_wf_control<false><<<1, 32, 0, st>>>(stage_args(a, 7), cudaGraphConditionalHandle{}); T1(7);
    cudaError_t err = cudaMemcpyAsync(e->h_cond, &a.ctl->cond, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
    if (err == cudaSuccess) err = cudaStreamSynchronize(st);
    if (err != cudaSuccess) return err;
    if (*e->h_cond == 0u) break;
  }
  T0(6); k_wf_accumulate<<<e->grid[6], 256, 0, st>>>(stage_args(a, 6)); T1(6);
  return cudaGetLastError();
}

template <bool COUNT>
static cudaError_t render_views(WfEngine* e, const DeviceScene& d, const void* pairs_tlas, const void* pairs_bvh,
                                const WfJobView* jv, uint32_t nv, uint32_t* status, unsigned long long* counters,
                                cudaStream_t st, StageTimer* timer, float* done_ms) {
  cudaError_t err;
  const bool tex = (d.flags & SCENE_TEXTURED) != 0u;
  // shadow rays over the quad records: untextured scenes whose trees are shallow enough for the
  // 4-wide walk's stack (SCENE_WIDE_OK, set on upload), when not counting work
  e->wide_now = !COUNT && !tex && e->shadow_wide && (d.flags & SCENE_WIDE_OK) != 0u;
  if (tex) compute_grids<COUNT, true>(e); else compute_grids<COUNT, false>(e);
  const bool track = done_ms != nullptr;
  uint64_t total_npix = 0;
  for (uint32_t v = 0; v < nv; ++v) total_npix += (uint64_t)jv[v].sw * jv[v].sh;
  if (total_npix == 0) return cudaSuccess;
  if (total_npix > (1ull << 30)) return cudaErrorInvalidValue;
  const int bl = d.bounce_limit;
  if (!e->d_ctl) {
    if ((err = cudaMalloc(&e->d_ctl, sizeof(WfCtl))) != cudaSuccess) return err;
    if ((err = cudaMallocHost(&e->h_cond, sizeof(uint32_t))) != cudaSuccess) return err;
  }
  if (e->views_cap < nv) {
    cudaStreamSynchronize(st);
    if (e->d_views) cudaFree(e->d_views);
    e->d_views = nullptr;
    e->views_cap = 0;
    if ((err = cudaMalloc(&e->d_views, sizeof(WfView) * nv)) != cudaSuccess) return err;
    e->views_cap = nv;
  }
  if (e->track_cap < nv) {
    cudaStreamSynchronize(st);
    drop_graph(e);
    if (e->d_remaining) cudaFree(e->d_remaining);
    if (e->d_done) cudaFree(e->d_done);
    e->d_remaining = nullptr;
    e->d_done = nullptr;
    e->track_cap = 0;
    if ((err = cudaMalloc(&e->d_remaining, sizeof(uint32_t) * nv)) != cudaSuccess) return err;
    if ((err = cudaMalloc(&e->d_done, sizeof(unsigned long long) * (nv + 1))) != cudaSuccess) return err;
    e->track_cap = nv;
  }
  if (track) {
    std::vector<uint32_t> rem(nv);
    for (uint32_t v = 0; v < nv; ++v) rem[v] = jv[v].sw * jv[v].sh * jv[v].spp;
    if ((err = cudaMemcpyAsync(e->d_remaining, rem.data(), sizeof(uint32_t) * nv, cudaMemcpyHostToDevice, st)) !=
        cudaSuccess)
      return err;
    if ((err = cudaMemsetAsync(e->d_done, 0, sizeof(unsigned long long) * (nv + 1), st)) != cudaSuccess) return err;
  }
  // views in ascending order of work: the unit numbering decides which views finish first, and
  // shortest-first minimises the mean completion time; results do not depend on the order
  std::vector<uint32_t> order(nv);
  for (uint32_t v = 0; v < nv; ++v) order[v] = v;
  std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) {
    return (uint64_t)jv[x].sw * jv[x].sh * jv[x].spp < (uint64_t)jv[y].sw * jv[y].sh * jv[y].spp;
  });
  std::vector<uint32_t> done(nv, 0u);
  std::vector<WfView> hv;
  hv.reserve(nv);
  bool first_pass = true;
  while (true) {
    // samples per view in this pass: the largest count whose units fit units_per_pass (at least 1)
    auto units_at = [&](uint64_t s_) {
      uint64_t u = 0;
      for (uint32_t v = 0; v < nv; ++v) u += (uint64_t)jv[v].sw * jv[v].sh * std::min<uint64_t>(jv[v].spp - done[v], s_);
      return u;
    };
    uint64_t lo = 1, hi = 1;
    for (uint32_t v = 0; v < nv; ++v) hi = std::max<uint64_t>(hi, jv[v].spp - done[v]);
    while (lo < hi) {
      uint64_t mid = (lo + hi + 1) / 2;
      if (units_at(mid) <= e->units_per_pass) lo = mid; else hi = mid - 1;
    }
    const uint64_t per = lo;
    hv.clear();
    uint64_t units = 0, pixels = 0;
    std::vector<uint32_t> take(nv, 0u);
    for (uint32_t v : order) {
      uint32_t rem = jv[v].spp - done[v];
      uint32_t npix = jv[v].sw * jv[v].sh;
      if (rem == 0 || npix == 0) continue;
      take[v] = (uint32_t)std::min<uint64_t>(rem, per);
      WfView w;
      memset(&w, 0, sizeof w);
      fill_dparams(w.p, jv[v].q, jv[v].sx, jv[v].sy);
      w.sec_w = jv[v].sw;
      w.npix = npix;
      w.first_frame = jv[v].first_frame + done[v];
      w.spp = take[v];
      w.unit_base = (uint32_t)units;
      w.pix_base = (uint32_t)pixels;
      w.out_pitch = jv[v].out_pitch;
      w.accum = (float4*)jv[v].accum;
      w.out = (uchar4*)jv[v].out;
      w.acc64 = jv[v].acc64;
      w.job = v;
      hv.push_back(w);
      units += (uint64_t)npix * take[v];
      pixels += npix;
    }
    if (hv.empty()) break;
    if (units >= (1ull << 31)) return cudaErrorInvalidValue;
    // buffers: the pool never exceeds the pass's units; samples hold the pass
    uint32_t want_pool = (uint32_t)std::min<uint64_t>(e->pool_paths, units);
    if (e->pool_cap < want_pool) {
      size_t free_b = 0, total_b = 0;
      if ((err = cudaMemGetInfo(&free_b, &total_b)) != cudaSuccess) return err;
      const uint64_t budget = (free_b + (e->pool ? pool_bytes(e->pool_cap) : 0)) / 4 / wavefront_bytes_per_path();
      want_pool = (uint32_t)std::max<uint64_t>(std::min<uint64_t>(want_pool, budget), std::min<uint64_t>(units, 1024));
      if (e->pool_cap >= want_pool) want_pool = std::min<uint32_t>(e->pool_cap, (uint32_t)std::min<uint64_t>(e->pool_paths, units));
    }
    if (e->pool_cap < want_pool || e->samples_cap < units) {
      cudaStreamSynchronize(st);
      drop_graph(e);
      if (e->pool_cap < want_pool) {
        if (e->pool) cudaFree(e->pool);
        e->pool = nullptr;
        e->pool_cap = 0;
        if ((err = cudaMalloc(&e->pool, pool_bytes(want_pool))) != cudaSuccess) return err;
        e->pool_cap = want_pool;
      }
      if (e->samples_cap < units) {
        if (e->samples) cudaFree(e->samples);
        e->samples = nullptr;
        e->samples_cap = 0;
        if ((err = cudaMalloc(&e->samples, units * sizeof(float4))) != cudaSuccess) return err;
        e->samples_cap = units;
      }
    }
    uint32_t fill = want_pool;   // active slots of the pass (the allocation may be larger)
    WfCtl c;
    memset(&c, 0, sizeof c);
    c.iter = 0;
    c.unit_next = fill;
    c.n_units = (uint32_t)units;
    uint64_t bound = (units * (uint64_t)std::max(bl, 0) + fill - 1) / fill + (uint64_t)std::max(bl, 0) + 4;
    c.max_iter = (uint32_t)std::min<uint64_t>(bound, 1u << 22);
    c.n_views = (uint32_t)hv.size();
    c.n_pixels = (uint32_t)pixels;
    c.fill_count = fill;
    c.counts[0][K_NEW] = fill;
    c.sp = hv[0].p;
    c.track = track ? 1u : 0u;
    c.first_pass = first_pass ? 1u : 0u;
    if ((err = cudaMemcpyAsync(e->d_views, hv.data(), sizeof(WfView) * hv.size(), cudaMemcpyHostToDevice, st)) !=
        cudaSuccess)
      return err;
    if ((err = cudaMemcpyAsync(e->d_ctl, &c, sizeof c, cudaMemcpyHostToDevice, st)) != cudaSuccess) return err;
    WfArgs a;
    memset(&a, 0, sizeof a);
    fill_dscene(a.s, d);
    a.P.tlas = (const float4*)pairs_tlas;
    a.P.bvh = (const float4*)pairs_bvh;
    a.P.tlas4 = a.P.tlas + (size_t)(d.n_tlas > 0u ? d.n_tlas : 1u) * 4;   // quads follow the pairs
    a.P.bvh4 = a.P.bvh + (size_t)(d.n_bvh > 0u ? d.n_bvh : 1u) * 4;
    a.b = carve(e->pool, e->pool_cap);
    a.views = e->d_views;
    a.ctl = e->d_ctl;
    a.samples = e->samples;
    a.remaining = e->d_remaining;
    a.done_ns = e->d_done;
    a.t0_ns = e->d_done + e->track_cap;
    a.status = status;
    a.counters = counters;
    a.refill_closest = e->refill_closest;
    a.refill_shadow = e->refill_shadow;
    if (bl <= 0) {
      // no bounce runs: every sample's radiance is zero
      if ((err = cudaMemsetAsync(e->samples, 0, units * sizeof(float4), st)) != cudaSuccess) return err;
      if (timer) timer->begin(6, st);
      k_wf_accumulate<<<e->grid[6], 256, 0, st>>>(stage_args(a, 6));
      if (timer) timer->end(6, st);
      if ((err = cudaGetLastError()) != cudaSuccess) return err;
    } else if (timer) {
      err = tex ? run_pass_host<COUNT, true>(e, a, c.max_iter, st, timer)
                : run_pass_host<COUNT, false>(e, a, c.max_iter, st, timer);
      if (err != cudaSuccess) return err;
    } else {
      if (!e->has_graph || e->key_count != COUNT || memcmp(&e->key, &a, sizeof a) != 0) {
        err = tex ? build_graph<COUNT, true>(e, a) : build_graph<COUNT, false>(e, a);
        if (err != cudaSuccess) {
          drop_graph(e);
          return err;
        }
      }
      if ((err = cudaGraphLaunch(e->exec, st)) != cudaSuccess) return err;
    }
    for (uint32_t v = 0; v < nv; ++v) done[v] += take[v];
    first_pass = false;
  }
  if (track) {
    std::vector<unsigned long long> ns(nv + 1);
    if ((err = cudaMemcpyAsync(ns.data(), e->d_done, sizeof(unsigned long long) * nv, cudaMemcpyDeviceToHost, st)) !=
        cudaSuccess)
      return err;
    if ((err = cudaMemcpyAsync(&ns[nv], e->d_done + e->track_cap, sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                               st)) != cudaSuccess)
      return err;
    if ((err = cudaStreamSynchronize(st)) != cudaSuccess) return err;
    for (uint32_t v = 0; v < nv; ++v)
      done_ms[v] = ns[v] >= ns[nv] && ns[v] != 0ull ? (float)((double)(ns[v] - ns[nv]) * 1e-6) : -1.0f;
  }
  return cudaSuccess;
}

cudaError_t wf_render(WfEngine* e, const DeviceScene& d, const void* pairs_tlas, const void* pairs_bvh,
                      const WfJobView* views, uint32_t n_views, uint32_t* status, unsigned long long* counters,
                      cudaStream_t st, StageTimer* timer, float* done_ms) {
  if (!e || n_views == 0) return cudaErrorInvalidValue;
  if (counters)
    return render_views<true>(e, d, pairs_tlas, pairs_bvh, views, n_views, status, counters, st, timer, done_ms);
  return render_views<false>(e, d, pairs_tlas, pairs_bvh, views, n_views, status, counters, st, timer, done_ms);
}

}  // namespace wgpt
