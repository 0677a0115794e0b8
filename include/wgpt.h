/*
 * wgpt -- C ABI of the B200 progressive path tracer, a drop-in for the WebGPU device, buffers and
 * dispatch loop of DragonFireGames/WebGPURaytracer's Renderer / Denoiser (tracer.js).
 *
 * Buffers are accepted in the reference's own packed layouts (see wgpt_layout.h).  All functions
 * return WGPT_OK (0) or an error code; wgpt_last_error() gives a message.  No function aborts.
 * The library owns all device memory; callers own every host pointer they pass.  One context is
 * used by one thread at a time.  Work is queued on the context's CUDA stream; functions that
 * hand data back to the host synchronise that stream first.
 */
#ifndef WGPT_H
#define WGPT_H

#include <stddef.h>
#include <stdint.h>
#include "wgpt_layout.h"

#ifdef __cplusplus
extern "C" {
#endif

#define WGPT_ABI_VERSION 1

enum wgpt_status {
  WGPT_OK = 0,
  WGPT_E_INVALID = 1,     /* bad argument (null pointer, zero size, out-of-range section) */
  WGPT_E_LAYOUT = 2,      /* a buffer's size or an index inside it breaks the layout contract */
  WGPT_E_CUDA = 3,        /* a CUDA runtime call failed */
  WGPT_E_NOMEM = 4,       /* device allocation failed */
  WGPT_E_STATE = 5,       /* call out of order (no scene, no size, no G-buffer) */
  WGPT_E_UNSUPPORTED = 6, /* a combination this build does not run (e.g. FP64 accumulation in the single-kernel mode) */
  WGPT_E_REBUILD = 7,     /* wgpt_update_scene / wgpt_update_objects: upload the scene again */
  WGPT_E_DEVICE = 8,      /* a kernel reported an error (traversal stack overflow) */
  WGPT_E_TOO_LARGE = 9,   /* wgpt_denoise_noalloc: more than WGPT_NOALLOC_MAX_PIXELS pixels */
  WGPT_E_TIMEOUT = 10     /* wgpt_synchronize_timeout: the work did not finish in time */
};

typedef struct wgpt_ctx wgpt_ctx;

typedef struct wgpt_buffer {
  const void* ptr;
  size_t bytes;
} wgpt_buffer;

/* Scene buffers of Renderer.setScene (tracer.js:1955-2102); binding numbers of shader.wgsl. */
typedef struct wgpt_scene_desc {
  wgpt_buffer materials;    /* binding 3,  wgpt_material[]      (144 B) */
  wgpt_buffer objects;      /* binding 4,  wgpt_object[]        (96 B)  */
  wgpt_buffer tlas;         /* binding 5,  wgpt_bvh_node[]      (32 B)  */
  wgpt_buffer meshes;       /* binding 6,  list meshes, packed at 96 B and read at 80 B */
  wgpt_buffer bvh;          /* binding 7,  wgpt_bvh_node[]      (32 B)  */
  wgpt_buffer triangles;    /* binding 8,  wgpt_triangle[]      (128 B) */
  wgpt_buffer planes;       /* binding 9,  wgpt_plane[]         (32 B)  */
  wgpt_buffer lights;       /* binding 10, wgpt_light[]         (80 B)  */
  wgpt_buffer sky_cdf;      /* binding 15, float[] (buildHDRCDF, tracer.js:135-204) */
  const uint16_t* sky_rgba16f; /* binding 13, sky_width*sky_height texels of 4 IEEE halves */
  uint32_t sky_width;
  uint32_t sky_height;
  int32_t bounce_limit;     /* override constant 0 (BOUNCE_LIMIT) */
  uint32_t feature_flags;   /* override constants 1..11 as WGPT_HAS_* bits */
  /* binding 11, texture_list (prepareTextureArray, tracer.js:1919-1953): tex_layers images of
     tex_width x tex_height rgba8 texels, layer after layer (the reference resizes every texture
     to 512 x 512); NULL / 0 when no material references a texture.  Sampled bilinearly with
     repeat addressing (sampler of tracer.js:1965-1968) in FP32. */
  const uint8_t* textures_rgba8;
  uint32_t tex_width;
  uint32_t tex_height;
  uint32_t tex_layers;
  /* optional (no reference counterpart): alias table of the sky, sky_width * sky_height entries
     of {float prob; uint32_t alias;} from wgpt_build_env_alias, for wgpt_set_env_sampling */
  const void* sky_alias;
} wgpt_scene_desc;

/* Renderer constructor + init() (tracer.js:1720-1770): binds CUDA device `device`. */
int wgpt_create(int device, wgpt_ctx** out);
int wgpt_destroy(wgpt_ctx* ctx);
const char* wgpt_last_error(const wgpt_ctx* ctx);
int wgpt_abi_version(void);

/* setScene buffer creation + writeBuffer (tracer.js:2015-2036) and the pipeline constants
   (tracer.js:2062-2082).  Validates strides, indices and tree structure (WGPT_E_LAYOUT). */
int wgpt_upload_scene(wgpt_ctx* ctx, const wgpt_scene_desc* desc);

/* The upload checks alone, on the host (no device needed): 0 or the status wgpt_upload_scene
   would return; msg (nullable) receives the reason. */
int wgpt_validate_scene(const wgpt_scene_desc* desc, char* msg, size_t msg_len);

/* Rewrites every buffer of the scene in place (validated like wgpt_upload_scene) when each
   fits its resident buffer and the pipeline constants are unchanged, else WGPT_E_REBUILD.  No
   reference counterpart: a full setScene without reallocation. */
int wgpt_update_scene(wgpt_ctx* ctx, const wgpt_scene_desc* desc);

/* updateObjects fast path (tracer.js:2132-2164): reads only desc->objects, tlas, planes, meshes
   and materials (tracer.js:2151-2155), writes each at offset 0 of its resident buffer (the
   buffer keeps the length wgpt_upload_scene gave it, as a WebGPU writeBuffer does), rebuilds
   the TLAS node pairs, and leaves lights, BLAS, triangles, sky, CDF and textures as they are.
   WGPT_E_REBUILD when the flags differ, a buffer does not fit, or a mesh instance names a BLAS
   that was not uploaded (the caller then uploads the scene again, as setScene does);
   WGPT_E_LAYOUT for an out-of-range index in the new records. */
int wgpt_update_objects(wgpt_ctx* ctx, const wgpt_scene_desc* desc);

/* resize (tracer.js:2166-2205): accumulation (16 B/px), rgba8 output and, with want_gbuf, the
   48 B/px G-buffer; all zero-filled. */
int wgpt_resize(wgpt_ctx* ctx, uint32_t width, uint32_t height, int want_gbuf);

/* updateUniforms (tracer.js:2207-2240): the 112-byte SceneParams, taken verbatim (the seed is
   the caller's; the reference draws it with Math.random). */
int wgpt_set_params(wgpt_ctx* ctx, const void* scene_params_112);

/* render / renderSection (tracer.js:2242-2309): `reps` samples of main over the section, sample
   k using sample_number = first_frame + k.  Queued on the context stream (asynchronous). */
int wgpt_render(wgpt_ctx* ctx, uint32_t first_frame, uint32_t reps, uint32_t sec_x, uint32_t sec_y,
                uint32_t sec_w, uint32_t sec_h);

/* How wgpt_render runs its samples: WGPT_MODE_WAVEFRONT (default) treats every (sample, pixel)
   of the call as a work unit traced by a pool of path slots through closest-hit, shading,
   shadow and resolve kernels over compacted queues; a slot whose path ends starts the next unit
   at once (path regeneration), the iteration loop is one CUDA-graph launch, and each pixel's
   samples are folded into the running mean in sample order at the end.  WGPT_MODE_MEGAKERNEL
   runs one thread per pixel through all bounces and samples, like the reference's single
   compute entry point.  Both produce identical results. */
enum { WGPT_MODE_WAVEFRONT = 0, WGPT_MODE_MEGAKERNEL = 1 };
int wgpt_set_render_mode(wgpt_ctx* ctx, int mode);

/* Environment light sampling for next-event estimation: WGPT_ENV_CDF (default) inverts the
   reference's CDF by binary search (shader.wgsl:192-254) and reproduces its sample stream;
   WGPT_ENV_ALIAS draws the texel from the uploaded alias table in O(1) with the same per-texel
   probabilities (FP64 weights; same random numbers consumed, same pdf), so images agree
   statistically, not bit for bit.  WGPT_E_STATE when no alias table was uploaded.  The mode
   stays set across uploads; a scene uploaded without sky_alias samples by CDF. */
enum { WGPT_ENV_CDF = 0, WGPT_ENV_ALIAS = 1 };
int wgpt_set_env_sampling(wgpt_ctx* ctx, int mode);

/* FP64 accumulation (no counterpart in the reference): with it on, the wavefront mode also
   folds every sample, in sample order, into a per-pixel FP64 Welford record of 8 doubles
   (mean r, g, b; sum of squared deviations r, g, b; sample count; unused) alongside the FP32
   running mean; cleared when switched on and by wgpt_resize.  Used for converged reference
   images and per-pixel confidence intervals.  The megakernel mode rejects it. */
int wgpt_set_accum_f64(wgpt_ctx* ctx, int on);
int wgpt_read_accum_f64(wgpt_ctx* ctx, double* dst_8_per_px);
int wgpt_write_accum_f64(wgpt_ctx* ctx, const double* src_8_per_px);   /* checkpoint resume */

/* Wavefront sizing (no counterpart in the reference, whose dispatch has no path pool):
   pool_paths path slots (1,024 .. 67,108,864; default 67,108,864; 448 bytes each; a pass uses
   no more than its samples, and a new pool takes at most a quarter of the free device memory) and at
   most units_per_pass samples held (65,536 .. 2^30; default 2^27; 16 bytes each) before they are
   folded into the images; a call with more samples runs in several passes.  Results do not
   depend on either.  0 keeps the current value. */
int wgpt_set_wavefront_config(wgpt_ctx* ctx, uint32_t pool_paths, uint64_t units_per_pass);
int wgpt_get_wavefront_config(wgpt_ctx* ctx, uint32_t* pool_paths, uint64_t* units_per_pass);

/* Kernel variants and thresholds of the wavefront renderer, for the autotuner (no counterpart
   in the reference).  trav_shape: block shape of the closest-hit and shadow traversal kernels,
   0 = 192 threads x 6 blocks per SM, 1 = 128 x 9, 2 = 256 x 4 (default; textured scenes keep 0
   for shadow rays); shade_block: surface-shading block of untextured scenes, 512 (default) or 256;
   refill_closest / refill_shadow: idle lanes (1..32) a traversal warp accumulates before it takes
   new rays from the queue (defaults 24 and 8); shadow_wide: 1 walks shadow rays of
   scenes without alpha-textured occluders over a 4-wide view of the same BVHs (quad records
   derived on upload: each visit tests the boxes two levels down), 0 (default) over the
   reference's 2-wide trees.  Results do not depend on any of them.  The defaults are the
   autotuner's choices on the flagship workload. */
typedef struct wgpt_wavefront_tuning {
  uint32_t trav_shape;
  uint32_t shade_block;
  uint32_t refill_closest;
  uint32_t refill_shadow;
  uint32_t shadow_wide;
} wgpt_wavefront_tuning;
int wgpt_set_wavefront_tuning(wgpt_ctx* ctx, const wgpt_wavefront_tuning* tuning);
int wgpt_get_wavefront_tuning(wgpt_ctx* ctx, wgpt_wavefront_tuning* tuning);

/* setScene(scene, true) + render(): one dispatch of gbuf_main (shader.wgsl:2510-2603) into the
   G-buffer and the debug quadrant image. */
int wgpt_render_gbuffer(wgpt_ctx* ctx, uint32_t sec_x, uint32_t sec_y, uint32_t sec_w, uint32_t sec_h);

/* Denoiser.execute (tracer.js:2583-2637): prepass, `passes` a-trous passes with the given step
   widths (the reference as run uses 2^(passes-1) for every pass, see denoiser quirk notes), and
   composite into the rgba8 output.  uniforms_48: wgpt_denoise_uniforms (width/height must match
   the context size; step_width and passes are taken from `steps`/`passes`). */
int wgpt_denoise(wgpt_ctx* ctx, const void* uniforms_48, const uint32_t* steps, uint32_t passes);

/* Arithmetic of the a-trous passes (no reference counterpart): WGPT_DENOISE_EXACT (default)
   evaluates every tap's four exponential edge stops and the normal stop with the pinned FP32
   built-ins in the reference's order, bit for bit like the CPU restatement; WGPT_DENOISE_FAST
   uses one hardware exponential of the summed stop arguments, the hardware power and fused
   multiply-adds, within 1e-5 relative of the exact result per pixel (the tolerance stated for
   the a-trous drop-in) but not bit-exact.  Applies to wgpt_denoise on this context. */
enum { WGPT_DENOISE_EXACT = 0, WGPT_DENOISE_FAST = 1 };
int wgpt_set_denoise_mode(wgpt_ctx* ctx, int mode);

/* renderPreview blit (tracer.js:2365-2389, scale.wgsl): bilinear resample of the output image
   (its top-left ratio_x/ratio_y part) into a dst_w x dst_h canvas image owned by the context. */
int wgpt_resample(wgpt_ctx* ctx, uint32_t dst_w, uint32_t dst_h, float ratio_x, float ratio_y);

/* Waits for queued work; returns WGPT_E_DEVICE if a kernel flagged an error. */
int wgpt_synchronize(wgpt_ctx* ctx);

/* Host watchdog (no reference counterpart): polls the queued work instead of blocking and
   returns WGPT_E_TIMEOUT after timeout_ms (the work keeps running; call again to keep waiting). */
int wgpt_synchronize_timeout(wgpt_ctx* ctx, uint32_t timeout_ms);

/* Readback / write-back of the context images (SaveRender, gui.js:1622; checkpoint/resume). */
int wgpt_read_accum(wgpt_ctx* ctx, float* dst_rgba32f);
int wgpt_write_accum(wgpt_ctx* ctx, const float* src_rgba32f);
int wgpt_read_output(wgpt_ctx* ctx, uint8_t* dst_rgba8);
int wgpt_read_gbuffer(wgpt_ctx* ctx, void* dst_48B_per_px);
int wgpt_write_gbuffer(wgpt_ctx* ctx, const void* src_48B_per_px);
int wgpt_read_denoised(wgpt_ctx* ctx, float* filtered_rgba32f, float* composited_rgba32f);
int wgpt_read_canvas(wgpt_ctx* ctx, uint8_t* dst_rgba8, uint32_t dst_w, uint32_t dst_h);

/* Batched views (no counterpart in the reference, which renders one canvas per device): many
   camera views of the uploaded scene, each with its own size, samples and images owned by the
   context, traced by one path pool in one graph launch.  wgpt_set_views allocates n view images
   (zeroed accumulation); wgpt_render_views adds spp[i] samples (sample_number first_frame[i] ..)
   to view i with the 112-byte params params_112n[i] (width/height = the view size; every view's
   sky fields equal, as they describe the one scene) and, when done_ms is not NULL, waits and
   stores per view the milliseconds from the start of the call's work to its last sample
   (-1 for a view without samples); npix * spp must stay below 2^32 per view.  Results equal
   wgpt_render of each view on its own. */
int wgpt_set_views(wgpt_ctx* ctx, uint32_t n, const uint32_t* widths, const uint32_t* heights);
int wgpt_render_views(wgpt_ctx* ctx, const void* params_112n, const uint32_t* first_frames, const uint32_t* spp,
                      float* done_ms);
int wgpt_read_view(wgpt_ctx* ctx, uint32_t view, float* accum_rgba32f, uint8_t* out_rgba8);
/* gbuf_main for every view (params as for wgpt_render_views; the G-buffers are allocated on first
   use), so the learned denoiser can finish each view (wgpt_kpcn_denoise_view). */
int wgpt_render_views_gbuffer(wgpt_ctx* ctx, const void* params_112n);

/* BF16 GEMM on the tensor cores (tcgen05, FP32 accumulation in tensor memory), the core of the
   learned denoiser's kernels (no counterpart in the reference): C[m x n] = A[m x k] * B[n x k]^T
   with row-major host matrices of BF16 bit patterns, k a multiple of 8.  For tests and tools. */
int wgpt_gemm_bf16(int device, const uint16_t* a, const uint16_t* b, float* c, int m, int n, int k);

/* Learned kernel-predicting denoiser (no counterpart in the reference, whose only denoiser is
   the a-trous filter, which stays the fallback).  A 5-level encoder-decoder (32/48/64/96/128
   channels, ~0.73 M parameters) over 10 features of the accumulation and G-buffer (log colour,
   albedo, normal, depth) predicts three 5x5 filters per pixel, applied to the noisy colour as
   a cascade at dilations 1, 2 and 4 (29 x 29 footprint).  BF16
   weights and activations, FP32 accumulation on the tensor cores, FP32 master weights trained
   by Adam on the relative L2 loss sum((f-t)^2/(t^2+0.01))/(3 pixels), each step's gradient
   clipped to 4x the running mean of past gradient norms (a step with a non-finite gradient is
   skipped; wgpt_kpcn_set_params resets the moments and the running mean).  Parameters are one flat
   FP32 array, per layer W[cout][taps][cin] then bias[cout] (layer table in kpcn.cu).
   Examples are (noisy rgba32f, 48-byte G-buffer, target rgba32f) images of one common size;
   training samples `batch` random crops of crop x crop pixels per step (losses: steps floats).
   wgpt_kpcn_loss_and_grads evaluates one whole image (for gradient checks).  wgpt_kpcn_denoise
   filters a context's accumulation with its G-buffer into its rgba8 image (tonemapped with
   `exposure`), ordered after the context's queued work; filtered (nullable, host) receives the
   linear result. */
typedef struct wgpt_kpcn wgpt_kpcn;
int wgpt_kpcn_create(int device, uint64_t seed, wgpt_kpcn** out);
int wgpt_kpcn_destroy(wgpt_kpcn* k);
const char* wgpt_kpcn_last_error(wgpt_kpcn* k);
int wgpt_kpcn_num_params(wgpt_kpcn* k, uint64_t* n);
int wgpt_kpcn_get_params(wgpt_kpcn* k, float* dst);
int wgpt_kpcn_set_params(wgpt_kpcn* k, const float* src);
int wgpt_kpcn_add_example(wgpt_kpcn* k, const float* noisy_rgba32f, const void* gbuf_48B, const float* target_rgba32f,
                          uint32_t w, uint32_t h);
int wgpt_kpcn_num_examples(wgpt_kpcn* k, uint32_t* n);
int wgpt_kpcn_train(wgpt_kpcn* k, uint32_t steps, uint32_t batch, uint32_t crop, float lr, uint64_t seed,
                    float* losses);
/* Data-parallel training in two halves around the caller's gradient all-reduce (no reference
   counterpart).  wgpt_kpcn_grads: forward and backward of `batch` crops drawn with `seed` from
   this denoiser's examples; writes the FP32 gradient (num_params floats) into dev_grads, DEVICE
   memory on the denoiser's device, and the batch loss to *loss (nullable); returns once both
   are written.  wgpt_kpcn_apply: one Adam step with the gradient dev_grads * scale (e.g. the
   sum over ranks with scale 1/ranks). */
int wgpt_kpcn_grads(wgpt_kpcn* k, uint32_t batch, uint32_t crop, uint64_t seed, float* loss, float* dev_grads);
int wgpt_kpcn_apply(wgpt_kpcn* k, const float* dev_grads, float scale, float lr);
int wgpt_kpcn_loss_and_grads(wgpt_kpcn* k, const float* noisy_rgba32f, const void* gbuf_48B,
                             const float* target_rgba32f, uint32_t w, uint32_t h, float* loss, float* grads,
                             float* out_rgba32f);
/* How the network's 3x3 convolutions run (same results up to FP32 summation order inside the
   tensor cores): WGPT_KPCN_CONV_PIPELINED (default) is a persistent warp-specialised kernel --
   TMA halo loads and bulk weight copies through a ring of shared-memory stages, one MMA warp,
   double-buffered tensor-memory accumulators drained by four epilogue warps;
   WGPT_KPCN_CONV_PER_TILE runs one CTA per 16 x 16 tile with all threads loading, then one
   thread issuing the MMAs. */
enum { WGPT_KPCN_CONV_PIPELINED = 0, WGPT_KPCN_CONV_PER_TILE = 1 };
int wgpt_kpcn_set_conv_mode(wgpt_kpcn* k, int mode);
int wgpt_kpcn_denoise(wgpt_kpcn* k, wgpt_ctx* ctx, float exposure, float* filtered_rgba32f);
int wgpt_kpcn_denoise_view(wgpt_kpcn* k, wgpt_ctx* ctx, uint32_t view, float exposure, float* filtered_rgba32f);

/* Closest hit of caller rays (trace_scene, shader.wgsl:754-774) for parity tests: rays are n x
   (origin, direction) floats; outputs object index, material index, global triangle index
   (-1 unless a mesh triangle), t, world normal (3 floats). Host pointers. */
int wgpt_trace_rays(wgpt_ctx* ctx, const float* rays, uint32_t n, int32_t* o_idx, int32_t* m_idx,
                    int32_t* prim, float* t, float* normal);

/* Work counters of the renders queued while counting is on, 16 x u64: 0 paths, 1 extension rays,
   2 shadow rays, 3 BVH nodes popped, 4 child AABB tests, 5 triangle tests, 6 TLAS objects
   visited, 7 shading events, 8 environment NEE samples, 9 CDF probes, 10 sky texel reads,
   11 hit-attribute evaluations, 12-15 reserved (zero). */
int wgpt_set_counting(wgpt_ctx* ctx, int on);
int wgpt_read_counters(wgpt_ctx* ctx, uint64_t* dst16);

/* The same counters split by stage (8 x 16 u64: 0 ray generation or the single kernel,
   1 closest hit, 2 surface shading, 3 shadow rays, 4 accumulation, 5 miss shading, 6-7 unused). */
int wgpt_read_stage_counters(wgpt_ctx* ctx, uint64_t* dst128);

/* CUDA-event timing of every stage launch queued while timing is on; wgpt_read_stage_times
   returns the summed milliseconds and launch counts of the 8 stages (as above) and restarts. */
int wgpt_set_stage_timing(wgpt_ctx* ctx, int on);
int wgpt_read_stage_times(wgpt_ctx* ctx, double* ms8, uint32_t* launches8);

/* The context's cudaStream_t (as void*) for callers that time or order work around it. */
void* wgpt_stream(wgpt_ctx* ctx);

/* Denoiser without any allocation (no counterpart in the reference).  For callers that cannot
   call cudaMalloc: code running while a stream is being captured into a CUDA graph (where the
   runtime refuses allocations), hosts that fix their GPU memory budget up front, and real-time
   loops that must not stall on the allocator.  It runs the same prepass / a-trous / composite
   kernels as wgpt_denoise, with the same results, but takes every input and output as a caller
   device pointer (color: W*H float4, gbuf: W*H 48-byte texels, out_rgba8: W*H*4 bytes,
   out_composited: W*H float4 or NULL) and keeps its intermediate images in one static device
   array of WGPT_NOALLOC_MAX_PIXELS * 80 bytes (10 MiB) that each GPU loading the library holds
   until the process exits.  uniforms_48 and steps are host memory.  Images larger than
   WGPT_NOALLOC_MAX_PIXELS return WGPT_E_TOO_LARGE before any work is queued.  The first call on
   a device looks up the array's device address (cudaGetSymbolAddress) with that device current:
   make that first call before capturing a stream.  The address is kept per device ordinal for
   the life of the process: after cudaDeviceReset the module is loaded again and the array may
   move, so a process that resets a device must not call this function on it again.  color, gbuf
   and out_composited must be 16-byte aligned and out_rgba8 4-byte aligned (WGPT_E_INVALID
   otherwise).  Work is queued on `stream` (a
   cudaStream_t, NULL for the legacy default stream) on the current device.  All calls share the
   one array: calls that overlap on the GPU (different streams, or different host threads)
   race and corrupt each other's intermediates; queue them on one stream. */
#define WGPT_NOALLOC_MAX_PIXELS 131072u
int wgpt_denoise_noalloc(const float* color, const void* gbuf, const void* uniforms_48, const uint32_t* steps,
                         uint32_t passes, uint8_t* out_rgba8, float* out_composited, void* stream);

/* Host-side builders of the scene buffers (tracer.js host math, native): */
/* ModelData.generateBVH (tracer.js:1025-1118): binned-SAH BLAS over n triangles given as
   n x 24 floats (v0 v1 v2 n0 n1 n2 as xyz, uv0 uv1 uv2 as xy).  Writes up to 2n-1 nodes and n
   triangles in flattened order; *n_nodes receives the node count. */
int wgpt_build_blas(const float* tris24, uint32_t n, wgpt_bvh_node* nodes_out, uint32_t* n_nodes,
                    wgpt_triangle* tris_out);
/* SceneBVHBuilder (tracer.js:1509-1619): median-split TLAS over n object AABBs (n x 6 floats,
   min xyz then max xyz).  Writes up to 2n-1 nodes; *n_nodes receives the count. */
int wgpt_build_tlas(const float* aabbs6, uint32_t n, wgpt_bvh_node* nodes_out, uint32_t* n_nodes);
/* HDRTexture.buildHDRCDF (tracer.js:135-204) over w x h rgba16f texels: writes (h+1) + h(w+1)
   floats and the total weight (sky_total_lum).  exposure is a JavaScript number (double). */
int wgpt_build_env_cdf(const uint16_t* rgba16f, uint32_t w, uint32_t h, double exposure, float* cdf_out,
                       double* total_weight);
/* Alias table over the texel weights buildHDRCDF uses (FP64): prob[i] (float) and alias[i] per
   texel, width * height entries each (no reference counterpart). */
int wgpt_build_env_alias(const uint16_t* rgba16f, uint32_t width, uint32_t height, double exposure, float* prob,
                         uint32_t* alias);
/* parseHdr (lib/parse-hdr.js:125-211) + HDRTexture.updateData (tracer.js:76-87): decodes a
   Radiance RLE RGBE file into w x h rgba16f texels (exposure applied, clamp 65519). Call with
   rgba16f == NULL to query w and h. */
int wgpt_decode_rgbe(const uint8_t* file, size_t bytes, double exposure, uint16_t* rgba16f, uint32_t* w,
                     uint32_t* h);

/* Model.parseOBJ + generateTriangles (tracer.js:949-1021): an OBJ text (v, vt, vn, f with
   1-based v/vt/vn indices, polygons fan-triangulated) to n_tris triangles of 24 floats
   (v0 v1 v2 n0 n1 n2 uv0 uv1 uv2), the input of wgpt_build_blas.  JavaScript number semantics:
   parseFloat/parseInt prefixes, face indices stored through an Int32Array (NaN -> 0), and NaN
   wherever the reference reads outside its vertex arrays (missing vt/vn, bad indices).  Call
   with tris24 = NULL to get the count, then with room for `capacity` >= n_tris triangles.
   positions (nullable) receives the vertex_positions array (n_positions floats, 3 per vertex)
   that Model.getBounds walks. */
int wgpt_parse_obj(const char* text, size_t bytes, float* tris24, uint32_t capacity, uint32_t* n_tris,
                   float* positions, uint32_t pos_capacity, uint32_t* n_positions);

/* ---------------------------------------------------------------------------------------
   Test and measurement support.  Not part of the renderer surface that tracer.js binds: the
   robustness tests and the benchmark call these. */

/* Self-test of the device-side bounded waits (no reference counterpart): a kernel waits on an
   mbarrier phase nothing completes, through the same wait the tensor-core kernels use, and must
   give up after `limit` polls (1..2^24); *status receives the device status word (4 = the wait
   timed out), *ms (nullable) the kernel's duration.  The context stays usable. */
int wgpt_selftest_wait(int device, uint32_t limit, uint32_t* status, float* ms);

/* Environment light samples of caller random pairs (known-answer tests of the CDF search; no
   reference counterpart): for each (u.x, u.y) of u2 (n pairs), the sky texel that sample_env_cdf
   (shader.wgsl:231-254) picks with the two binary_search_cdf calls (192-206) as (x, y) in
   texel_xy, and the sample's pdf.  Needs an uploaded scene with an importance-sampled sky and
   wgpt_set_params (its sky fields).  Host pointers; n <= 2^24. */
int wgpt_sample_env(wgpt_ctx* ctx, const float* u2, uint32_t n, uint32_t* texel_xy, float* pdf);

/* The random stream main draws for pixel `idx` at sample `sample_number` with `seed`
   (rand_pcg and its seeding, shader.wgsl:146-154, 2280-2282): draws 1..n after the discarded
   first one, computed on `device` (known-answer tests of the device's PCG; no reference
   counterpart).  n <= 2^20; host output. */
int wgpt_rng_stream(int device, uint32_t idx, uint32_t sample_number, uint32_t seed, uint32_t n, float* out);

/* L2 read bandwidth of `device` (measurement support, no reference counterpart): streams an
   L2-resident buffer of `bytes` (1 MiB .. 96 MiB, a multiple of 16) `reps` times (1..1000) with
   L2-only loads and writes the rate in GB/s.  Allocates and frees its buffer. */
int wgpt_probe_l2_read(int device, uint64_t bytes, uint32_t reps, double* gbps);

#ifdef __cplusplus
}
#endif

#endif /* WGPT_H */
