// Internal interfaces between the C ABI (api.cu) and the kernel translation units.
#pragma once
#include <stdint.h>
#include <cuda_runtime.h>
#include "../../include/wgpt_layout.h"

struct wgpt_ctx;

namespace wgpt {

// Selects the device and drops a non-sticky error left in this thread's runtime state by code
// outside this library, so that the cudaGetLastError() after each of the library's launches
// reports that launch alone (a sticky error is returned again by the next runtime call).
inline cudaError_t select_device(int device) {
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) (void)cudaGetLastError();
  return e;
}

// The images of a context (for the learned denoiser, which reads the accumulation and the
// G-buffer and writes the rgba8 image).
struct CtxImages {
  int device;
  uint32_t w, h;
  float* accum;
  float* gbuf;
  uint8_t* out;
  cudaStream_t stream;
};
bool ctx_images(::wgpt_ctx* ctx, int view, CtxImages* out);   // view -1: the main image

// Scene flag bits derived from the materials on upload (above the WGPT_HAS_* bits): some
// material samples a texture; some has an albedo texture (shadow rays then attenuate through
// it); some reads the tangent frame, through a normal map or a height field (closest hits then
// carry their tangent-frame source).
enum : uint32_t { SCENE_TEXTURED = 1u << 24, SCENE_ALPHA_SHADOWS = 1u << 25, SCENE_TANGENTS = 1u << 26,
                  SCENE_ENV_ALIAS = 1u << 27,    // environment NEE from the alias table
                  SCENE_WIDE_OK = 1u << 28 };    // TLAS + BLAS depths fit the 4-wide walk's stack

// Device copies of the scene buffers, in the reference's packed layouts.
struct DeviceScene {
  const void* mats; uint32_t n_mats;
  const void* objs; uint32_t n_objs;
  const void* tlas; uint32_t n_tlas;
  const void* meshes; uint32_t n_meshes;   // count at the 80-byte read stride
  const void* bvh; uint32_t n_bvh;
  const void* tris; uint32_t n_tris;
  const void* planes; uint32_t n_planes;
  const void* lights; uint32_t n_lights;
  const void* sky; uint32_t sky_w, sky_h;
  const void* cdf; uint32_t n_cdf;
  const void* tex; uint32_t tex_w, tex_h, tex_layers;   // rgba8 texture array
  const void* alias;                                    // sky alias table (8 bytes per texel)
  int32_t bounce_limit;
  uint32_t flags;
};

cudaError_t launch_render(const DeviceScene& d, const wgpt_scene_params& q, uint32_t first_frame, uint32_t reps,
                          uint32_t sx, uint32_t sy, uint32_t sw, uint32_t sh, float* accum, uint8_t* out,
                          uint32_t out_pitch, uint32_t* status, unsigned long long* counters, cudaStream_t st);
// CUDA-event timing of the renderer's stages on the launching stream: 0 path start (single
// kernel in megakernel mode), 1 closest hit, 2 surface shading, 3 shadow rays, 4 resolve and
// regeneration, 5 miss shading, 6 accumulation, 7 loop control.
struct StageTimer {
  static constexpr int kMaxEvents = 8192;
  cudaEvent_t ev[kMaxEvents];
  int stage_of[kMaxEvents / 2];
  int used = 0;
  bool ready = false;
  int open_stage = -1;
  void begin(int stage, cudaStream_t st) {
    if (!ready || used + 2 > kMaxEvents) return;
    cudaEventRecord(ev[used], st);
    stage_of[used / 2] = stage;
    open_stage = stage;
  }
  void end(int stage, cudaStream_t st) {
    if (!ready || open_stage != stage || used + 2 > kMaxEvents) return;
    cudaEventRecord(ev[used + 1], st);
    used += 2;
    open_stage = -1;
  }
};

// Wavefront renderer with path regeneration (wavefront.cu).  A job is a list of camera views,
// each with its section, first sample number, sample count and images.
struct WfJobView {
  wgpt_scene_params q;
  uint32_t sx, sy, sw, sh;
  uint32_t first_frame, spp;
  float* accum;          // float4 per pixel, row pitch q.width
  uint8_t* out;          // rgba8, row pitch out_pitch
  uint32_t out_pitch;
  double* acc64 = nullptr;   // optional FP64 Welford record per pixel (mean.rgb, m2.rgb, n, -), row pitch q.width
};
struct WfEngine;
WfEngine* wf_engine_create();
void wf_engine_destroy(WfEngine* e);
int wf_engine_configure(WfEngine* e, uint32_t pool_paths, uint64_t units_per_pass);
void wf_engine_get(const WfEngine* e, uint32_t* pool_paths, uint64_t* units_per_pass);
int wf_engine_tune(WfEngine* e, int trav_shape, int shade_block, uint32_t refill_closest, uint32_t refill_shadow,
                   int shadow_wide);
void wf_engine_tuning(const WfEngine* e, int* trav_shape, int* shade_block, uint32_t* refill_closest,
                      uint32_t* refill_shadow, int* shadow_wide);
size_t wavefront_bytes_per_path();
cudaError_t wf_render(WfEngine* e, const DeviceScene& d, const void* pairs_tlas, const void* pairs_bvh,
                      const WfJobView* views, uint32_t n_views, uint32_t* status, unsigned long long* counters,
                      cudaStream_t st, StageTimer* timer, float* done_ms = nullptr);
cudaError_t launch_gbuffer(const DeviceScene& d, const wgpt_scene_params& q, uint32_t sx, uint32_t sy, uint32_t sw,
                           uint32_t sh, float* gbuf, uint8_t* out, uint32_t out_pitch, uint32_t* status,
                           cudaStream_t st);
cudaError_t launch_trace_rays(const DeviceScene& d, const float* rays, uint32_t n, int32_t* o_idx, int32_t* m_idx,
                              int32_t* prim, float* t, float* normal, uint32_t* status, cudaStream_t st);
cudaError_t launch_sample_env(const DeviceScene& d, const wgpt_scene_params& q, const float* u2, uint32_t n,
                              uint32_t* texel, float* pdf, cudaStream_t st);
cudaError_t launch_rng_stream(uint32_t idx, uint32_t sample_number, uint32_t seed, uint32_t n, float* out,
                              cudaStream_t st);
cudaError_t launch_denoise(const float* color, const float* gbuf, const wgpt_denoise_uniforms& u,
                           const uint32_t* steps, uint32_t passes, float* buf_a, float* buf_b, float* guide,
                           float* composited, uint8_t* out, const float** final_buf, cudaStream_t st,
                           bool fast = false);
cudaError_t launch_resample(const uint8_t* src, uint32_t sw, uint32_t sh, uint8_t* dst, uint32_t dw, uint32_t dh,
                            float rx, float ry, cudaStream_t st);

}  // namespace wgpt
