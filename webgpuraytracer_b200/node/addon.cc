// Node-API binding of libwgpt (include/wgpt.h) for tracer.js.
//
// tracer.js drives its shaders through WebGPU: Renderer.init requests a device
// (tracer.js:1733-1770), setScene creates and fills the bind-group buffers (tracer.js:1955-2102),
// updateObjects rewrites five of them (tracer.js:2132-2164), resize reallocates the images
// (tracer.js:2166-2205), updateUniforms writes the 112-byte uniform (tracer.js:2207-2240),
// render/renderSection dispatch `main` tile by tile (tracer.js:2242-2309), renderPreview blits
// through scale.wgsl (tracer.js:2334-2392) and Denoiser.execute runs the a-trous passes
// (tracer.js:2583-2637).  This addon replaces each of those device calls by one C-ABI call; the
// JavaScript packing code (packSceneData, buildHDRCDF, Camera.updateRays2) is kept as it is and
// its typed arrays are handed over unchanged.
//
// Conventions of every export:
//   * handles (renderer contexts, denoiser networks) are napi externals; destroy() frees them at
//     once, the garbage collector frees them otherwise;
//   * buffers are typed arrays (any element type where the ABI takes bytes, the named element
//     type where it takes floats or integers); sizes are checked against what the call reads or
//     writes before the call;
//   * a non-zero wgpt status throws an Error whose message is the library's message and whose
//     `code` is the status name (WGPT_E_LAYOUT, ...), except where a status is an answer
//     (updateObjects / updateScene return WGPT_E_REBUILD, synchronizeTimeout returns false);
//   * one context is used by one JavaScript thread at a time, as the C ABI requires; the two
//     async calls (synchronizeAsync, renderAsync) run on the libuv pool, so the caller awaits them
//     before the next call on the same context, as tracer.js awaits onSubmittedWorkDone;
//   * device pointers (the allocation-free denoiser, data-parallel training) are BigInt addresses
//     obtained from a CUDA binding of the caller's choice.
//
// Built by node-gyp with binding.gyp beside this file.

#include <node_api.h>

#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "wgpt.h"

namespace {

// ----------------------------------------------------------------------------------------------
// Errors

const char* status_name(int rc) {
  switch (rc) {
    case WGPT_OK: return "WGPT_OK";
    case WGPT_E_INVALID: return "WGPT_E_INVALID";
    case WGPT_E_LAYOUT: return "WGPT_E_LAYOUT";
    case WGPT_E_CUDA: return "WGPT_E_CUDA";
    case WGPT_E_NOMEM: return "WGPT_E_NOMEM";
    case WGPT_E_STATE: return "WGPT_E_STATE";
    case WGPT_E_UNSUPPORTED: return "WGPT_E_UNSUPPORTED";
    case WGPT_E_REBUILD: return "WGPT_E_REBUILD";
    case WGPT_E_DEVICE: return "WGPT_E_DEVICE";
    case WGPT_E_TOO_LARGE: return "WGPT_E_TOO_LARGE";
    case WGPT_E_TIMEOUT: return "WGPT_E_TIMEOUT";
    default: return "WGPT_E_UNKNOWN";
  }
}

// Thrown from argument checks; caught by the export wrapper and turned into a JS exception.
struct ArgError {
  std::string msg;
};

struct StatusError {
  int rc;
  std::string msg;
};

void throw_status(napi_env env, int rc, const std::string& what) {
  napi_value code, msg, err;
  napi_create_string_utf8(env, status_name(rc), NAPI_AUTO_LENGTH, &code);
  napi_create_string_utf8(env, what.c_str(), NAPI_AUTO_LENGTH, &msg);
  napi_create_error(env, code, msg, &err);
  napi_throw(env, err);
}

// The context's own message when it has one, else the call name.
std::string ctx_message(const wgpt_ctx* ctx, const char* call) {
  const char* m = ctx ? wgpt_last_error(ctx) : nullptr;
  return std::string(call) + ": " + (m && *m ? m : "failed");
}

void check(int rc, const wgpt_ctx* ctx, const char* call) {
  if (rc != WGPT_OK) throw StatusError{rc, ctx_message(ctx, call)};
}

void check_k(int rc, wgpt_kpcn* k, const char* call) {
  if (rc != WGPT_OK) {
    const char* m = k ? wgpt_kpcn_last_error(k) : nullptr;
    throw StatusError{rc, std::string(call) + ": " + (m && *m ? m : "failed")};
  }
}

// ----------------------------------------------------------------------------------------------
// Arguments

struct Args {
  napi_env env;
  size_t argc = 12;
  napi_value argv[12];
  Args(napi_env e, napi_callback_info info) : env(e) {
    napi_get_cb_info(env, info, &argc, argv, nullptr, nullptr);
  }
  napi_value at(size_t i) const {
    if (i >= argc) throw ArgError{"missing argument " + std::to_string(i)};
    return argv[i];
  }
  bool is_nullish(size_t i) const {
    if (i >= argc) return true;
    napi_valuetype t;
    napi_typeof(env, argv[i], &t);
    return t == napi_null || t == napi_undefined;
  }
  uint32_t u32(size_t i) const {
    uint32_t v;
    if (napi_get_value_uint32(env, at(i), &v) != napi_ok) throw ArgError{"argument " + std::to_string(i) + ": expected a number"};
    return v;
  }
  int32_t i32(size_t i) const {
    int32_t v;
    if (napi_get_value_int32(env, at(i), &v) != napi_ok) throw ArgError{"argument " + std::to_string(i) + ": expected a number"};
    return v;
  }
  double f64(size_t i) const {
    double v;
    if (napi_get_value_double(env, at(i), &v) != napi_ok) throw ArgError{"argument " + std::to_string(i) + ": expected a number"};
    return v;
  }
  bool boolean(size_t i) const {
    bool v = false;
    napi_valuetype t;
    napi_typeof(env, at(i), &t);
    if (t == napi_boolean) napi_get_value_bool(env, argv[i], &v);
    else v = u32(i) != 0;
    return v;
  }
  uint64_t u64(size_t i) const {   // a BigInt or a Number
    napi_valuetype t;
    napi_typeof(env, at(i), &t);
    if (t == napi_bigint) {
      uint64_t v;
      bool lossless;
      napi_get_value_bigint_uint64(env, argv[i], &v, &lossless);
      if (!lossless) throw ArgError{"argument " + std::to_string(i) + ": BigInt out of range"};
      return v;
    }
    return (uint64_t)f64(i);
  }
  void* device_ptr(size_t i) const { return is_nullish(i) ? nullptr : (void*)(uintptr_t)u64(i); }
  std::string str(size_t i) const {
    size_t n = 0;
    if (napi_get_value_string_utf8(env, at(i), nullptr, 0, &n) != napi_ok) throw ArgError{"argument " + std::to_string(i) + ": expected a string"};
    std::string s(n, '\0');
    napi_get_value_string_utf8(env, argv[i], &s[0], n + 1, &n);
    return s;
  }
};

struct View {   // a typed array's memory
  void* data = nullptr;
  size_t bytes = 0;
  size_t length = 0;
  napi_typedarray_type type = napi_uint8_array;
};

size_t elem_size(napi_typedarray_type t) {
  switch (t) {
    case napi_int8_array: case napi_uint8_array: case napi_uint8_clamped_array: return 1;
    case napi_int16_array: case napi_uint16_array: return 2;
    case napi_int32_array: case napi_uint32_array: case napi_float32_array: return 4;
    default: return 8;   // float64, bigint64, biguint64
  }
}

View typed(napi_env env, napi_value v, const char* what) {
  bool is = false;
  napi_is_typedarray(env, v, &is);
  if (!is) throw ArgError{std::string(what) + ": expected a typed array"};
  View out;
  napi_value ab;
  size_t off;
  napi_get_typedarray_info(env, v, &out.type, &out.length, &out.data, &ab, &off);
  out.bytes = out.length * elem_size(out.type);
  return out;
}

// A typed array of a given element type holding at least `min_elems` elements.
View typed_of(napi_env env, napi_value v, napi_typedarray_type want, size_t min_elems, const char* what) {
  View t = typed(env, v, what);
  bool ok = t.type == want || (want == napi_uint8_array && t.type == napi_uint8_clamped_array);
  if (!ok) throw ArgError{std::string(what) + ": wrong typed-array element type"};
  if (t.length < min_elems)
    throw ArgError{std::string(what) + ": needs " + std::to_string(min_elems) + " elements, got " + std::to_string(t.length)};
  return t;
}

// Any typed array of at least `min_bytes` bytes (byte-layout records).
View bytes_of(napi_env env, napi_value v, size_t min_bytes, const char* what) {
  View t = typed(env, v, what);
  if (t.bytes < min_bytes)
    throw ArgError{std::string(what) + ": needs " + std::to_string(min_bytes) + " bytes, got " + std::to_string(t.bytes)};
  return t;
}

napi_value make_u32(napi_env env, uint32_t v) { napi_value r; napi_create_uint32(env, v, &r); return r; }
napi_value make_f64(napi_env env, double v) { napi_value r; napi_create_double(env, v, &r); return r; }
napi_value make_bool(napi_env env, bool v) { napi_value r; napi_get_boolean(env, v, &r); return r; }
napi_value make_big(napi_env env, uint64_t v) { napi_value r; napi_create_bigint_uint64(env, v, &r); return r; }
napi_value undef(napi_env env) { napi_value r; napi_get_undefined(env, &r); return r; }
napi_value make_str(napi_env env, const char* s) { napi_value r; napi_create_string_utf8(env, s, NAPI_AUTO_LENGTH, &r); return r; }

// A new typed array of `n` elements; *data receives its memory.
napi_value new_typed(napi_env env, napi_typedarray_type t, size_t n, void** data) {
  napi_value ab, arr;
  napi_create_arraybuffer(env, n * elem_size(t), data, &ab);
  if (n) memset(*data, 0, n * elem_size(t));
  napi_create_typedarray(env, t, n, ab, 0, &arr);
  return arr;
}

void set(napi_env env, napi_value obj, const char* key, napi_value v) { napi_set_named_property(env, obj, key, v); }

napi_value get(napi_env env, napi_value obj, const char* key) {
  napi_value v;
  napi_get_named_property(env, obj, key, &v);
  return v;
}

bool present(napi_env env, napi_value v) {
  napi_valuetype t;
  napi_typeof(env, v, &t);
  return t != napi_null && t != napi_undefined;
}

// ----------------------------------------------------------------------------------------------
// Handles

struct CtxBox {
  wgpt_ctx* ctx = nullptr;
  uint32_t width = 0, height = 0;   // image size from resize(), for readback size checks
  bool gbuf = false;
  std::vector<uint32_t> view_w, view_h;
};

struct KpcnBox {
  wgpt_kpcn* k = nullptr;
};

void finalize_ctx(napi_env, void* data, void*) {
  auto* b = static_cast<CtxBox*>(data);
  if (b->ctx) wgpt_destroy(b->ctx);
  delete b;
}

void finalize_kpcn(napi_env, void* data, void*) {
  auto* b = static_cast<KpcnBox*>(data);
  if (b->k) wgpt_kpcn_destroy(b->k);
  delete b;
}

CtxBox* ctx_box(napi_env env, napi_value v) {
  void* p = nullptr;
  if (napi_get_value_external(env, v, &p) != napi_ok || !p) throw ArgError{"expected a renderer context"};
  auto* b = static_cast<CtxBox*>(p);
  if (!b->ctx) throw ArgError{"renderer context was destroyed"};
  return b;
}

KpcnBox* kpcn_box(napi_env env, napi_value v) {
  void* p = nullptr;
  if (napi_get_value_external(env, v, &p) != napi_ok || !p) throw ArgError{"expected a denoiser network"};
  auto* b = static_cast<KpcnBox*>(p);
  if (!b->k) throw ArgError{"denoiser network was destroyed"};
  return b;
}

// Runs an export body and maps C++ exceptions to JavaScript ones.
template <class F>
napi_value guard(napi_env env, F&& body) {
  try {
    return body();
  } catch (const StatusError& e) {
    throw_status(env, e.rc, e.msg);
  } catch (const ArgError& e) {
    napi_throw_type_error(env, "WGPT_E_INVALID", e.msg.c_str());
  } catch (const std::bad_alloc&) {
    throw_status(env, WGPT_E_NOMEM, "host allocation failed");
  }
  return nullptr;
}

#define EXPORT(name) napi_value name(napi_env env, napi_callback_info info)
#define BODY(...) return guard(env, [&]() -> napi_value { Args a(env, info); (void)a; __VA_ARGS__ });

// ----------------------------------------------------------------------------------------------
// Scene description: the object tracer.js builds from packSceneData(true) / buildHDRCDF.
//
//   { mat, object, tlas, mesh, bvh, triangle, plane, light, skyCDF,        typed arrays
//     sky16, skyW, skyH,                                                   Uint16Array + size
//     bounces, flags,                                                      override constants
//     tex, texW, texH, texLayers,                                          optional texture array
//     skyAlias }                                                           optional alias table
wgpt_scene_desc scene_desc(napi_env env, napi_value d, bool only_update_fields) {
  wgpt_scene_desc s{};
  auto buf = [&](const char* key) {
    napi_value v = get(env, d, key);
    if (!present(env, v)) return wgpt_buffer{nullptr, 0};
    View t = typed(env, v, key);
    return wgpt_buffer{t.data, t.bytes};
  };
  s.materials = buf("mat");
  s.objects = buf("object");
  s.tlas = buf("tlas");
  s.meshes = buf("mesh");
  s.planes = buf("plane");
  napi_value flags = get(env, d, "flags");
  if (present(env, flags)) napi_get_value_uint32(env, flags, &s.feature_flags);
  if (only_update_fields) return s;   // updateObjects reads nothing else
  s.bvh = buf("bvh");
  s.triangles = buf("triangle");
  s.lights = buf("light");
  s.sky_cdf = buf("skyCDF");
  napi_value sky = get(env, d, "sky16");
  if (!present(env, sky)) throw ArgError{"scene.sky16: required (the sky as rgba16f texels)"};
  View st = typed_of(env, sky, napi_uint16_array, 0, "scene.sky16");
  s.sky_rgba16f = static_cast<const uint16_t*>(st.data);
  napi_get_value_uint32(env, get(env, d, "skyW"), &s.sky_width);
  napi_get_value_uint32(env, get(env, d, "skyH"), &s.sky_height);
  if ((size_t)s.sky_width * s.sky_height * 4 > st.length) throw ArgError{"scene.sky16: smaller than skyW x skyH x 4"};
  napi_get_value_int32(env, get(env, d, "bounces"), &s.bounce_limit);
  napi_value tex = get(env, d, "tex");
  if (present(env, tex)) {
    View tt = bytes_of(env, tex, 0, "scene.tex");
    s.textures_rgba8 = static_cast<const uint8_t*>(tt.data);
    napi_get_value_uint32(env, get(env, d, "texW"), &s.tex_width);
    napi_get_value_uint32(env, get(env, d, "texH"), &s.tex_height);
    napi_get_value_uint32(env, get(env, d, "texLayers"), &s.tex_layers);
    if ((size_t)s.tex_width * s.tex_height * s.tex_layers * 4 > tt.bytes) throw ArgError{"scene.tex: smaller than texW x texH x texLayers x 4"};
  }
  napi_value alias = get(env, d, "skyAlias");
  if (present(env, alias)) {
    View at = bytes_of(env, alias, (size_t)s.sky_width * s.sky_height * 8, "scene.skyAlias");
    s.sky_alias = at.data;
  }
  return s;
}

// ----------------------------------------------------------------------------------------------
// Renderer (tracer.js:1719-2417)

// Renderer constructor + init (tracer.js:1720-1770): create(device) -> context
EXPORT(Create) {
  BODY(
    wgpt_ctx* ctx = nullptr;
    int rc = wgpt_create(a.is_nullish(0) ? 0 : a.i32(0), &ctx);
    if (rc != WGPT_OK) throw StatusError{rc, "wgpt_create: no usable CUDA device"};
    auto* b = new CtxBox();
    b->ctx = ctx;
    napi_value ext;
    napi_create_external(env, b, finalize_ctx, nullptr, &ext);
    return ext;
  )
}

EXPORT(Destroy) {
  BODY(
    void* p = nullptr;
    napi_get_value_external(env, a.at(0), &p);
    auto* b = static_cast<CtxBox*>(p);
    if (b && b->ctx) { wgpt_destroy(b->ctx); b->ctx = nullptr; }
    return undef(env);
  )
}

EXPORT(AbiVersion) { BODY(return make_u32(env, (uint32_t)wgpt_abi_version());) }

EXPORT(LastError) { BODY(return make_str(env, wgpt_last_error(ctx_box(env, a.at(0))->ctx));) }

// setScene buffers + pipeline constants (tracer.js:2015-2082): setScene(ctx, desc)
EXPORT(SetScene) {
  BODY(
    CtxBox* b = ctx_box(env, a.at(0));
    wgpt_scene_desc d = scene_desc(env, a.at(1), false);
    check(wgpt_upload_scene(b->ctx, &d), b->ctx, "setScene");
    return undef(env);
  )
}

// The upload checks alone: validateScene(desc) -> null, or {code, message}
EXPORT(ValidateScene) {
  BODY(
    wgpt_scene_desc d = scene_desc(env, a.at(0), false);
    char msg[512] = {0};
    int rc = wgpt_validate_scene(&d, msg, sizeof msg);
    if (rc == WGPT_OK) { napi_value n; napi_get_null(env, &n); return n; }
    napi_value o;
    napi_create_object(env, &o);
    set(env, o, "code", make_str(env, status_name(rc)));
    set(env, o, "message", make_str(env, msg));
    return o;
  )
}

// updateObjects fast path (tracer.js:2132-2164): updateObjects(ctx, {mat, object, tlas, mesh,
// plane, flags}) -> true when written in place, false when the caller must setScene again
// (WGPT_E_REBUILD, the reference's slow path)
EXPORT(UpdateObjects) {
  BODY(
    CtxBox* b = ctx_box(env, a.at(0));
    wgpt_scene_desc d = scene_desc(env, a.at(1), true);
    int rc = wgpt_update_objects(b->ctx, &d);
    if (rc == WGPT_E_REBUILD) return make_bool(env, false);
    check(rc, b->ctx, "updateObjects");
    return make_bool(env, true);
  )
}

// Every buffer rewritten in place: updateScene(ctx, desc) -> true, or false for WGPT_E_REBUILD
EXPORT(UpdateScene) {
  BODY(
    CtxBox* b = ctx_box(env, a.at(0));
    wgpt_scene_desc d = scene_desc(env, a.at(1), false);
    int rc = wgpt_update_scene(b->ctx, &d);
    if (rc == WGPT_E_REBUILD) return make_bool(env, false);
    check(rc, b->ctx, "updateScene");
    return make_bool(env, true);
  )
}

// resize (tracer.js:2166-2205): resize(ctx, width, height, isgbuf)
EXPORT(Resize) {
  BODY(
    CtxBox* b = ctx_box(env, a.at(0));
    uint32_t w = a.u32(1), h = a.u32(2);
    bool g = a.is_nullish(3) ? false : a.boolean(3);
    check(wgpt_resize(b->ctx, w, h, g ? 1 : 0), b->ctx, "resize");
    b->width = w; b->height = h; b->gbuf = g;
    return undef(env);
  )
}

// updateUniforms (tracer.js:2207-2240): setParams(ctx, uData) with the 28-float uniform block
EXPORT(SetParams) {
  BODY(
    CtxBox* b = ctx_box(env, a.at(0));
    View u = bytes_of(env, a.at(1), 112, "uniforms");
    check(wgpt_set_params(b->ctx, u.data), b->ctx, "setParams");
    return undef(env);
  )
}

// renderSection (tracer.js:2299-2309), `reps` frames at once: render(ctx, firstFrame, reps, x, y, w, h)
EXPORT(Render) {
  BODY(
    CtxBox* b = ctx_box(env, a.at(0));
    check(wgpt_render(b->ctx, a.u32(1), a.u32(2), a.u32(3), a.u32(4), a.u32(5), a.u32(6)), b->ctx, "render");
    return undef(env);
  )
}

// gbuf_main dispatch (setScene(scene, true) + render): renderGBuffer(ctx, x, y, w, h)
EXPORT(RenderGBuffer) {
  BODY(
    CtxBox* b = ctx_box(env, a.at(0));
    check(wgpt_render_gbuffer(b->ctx, a.u32(1), a.u32(2), a.u32(3), a.u32(4)), b->ctx, "renderGBuffer");
    return undef(env);
  )
}

EXPORT(SetRenderMode) {
  BODY(CtxBox* b = ctx_box(env, a.at(0)); check(wgpt_set_render_mode(b->ctx, a.i32(1)), b->ctx, "setRenderMode"); return undef(env);)
}

EXPORT(SetEnvSampling) {
  BODY(CtxBox* b = ctx_box(env, a.at(0)); check(wgpt_set_env_sampling(b->ctx, a.i32(1)), b->ctx, "setEnvSampling"); return undef(env);)
}

EXPORT(SetAccumF64) {
  BODY(CtxBox* b = ctx_box(env, a.at(0)); check(wgpt_set_accum_f64(b->ctx, a.boolean(1) ? 1 : 0), b->ctx, "setAccumF64"); return undef(env);)
}

// readAccumF64(ctx, Float64Array of width*height*8)
EXPORT(ReadAccumF64) {
  BODY(
    CtxBox* b = ctx_box(env, a.at(0));
    View d = typed_of(env, a.at(1), napi_float64_array, (size_t)b->width * b->height * 8, "accum64");
    check(wgpt_read_accum_f64(b->ctx, static_cast<double*>(d.data)), b->ctx, "readAccumF64");
    return undef(env);
  )
}

EXPORT(WriteAccumF64) {
  BODY(
    CtxBox* b = ctx_box(env, a.at(0));
    View d = typed_of(env, a.at(1), napi_float64_array, (size_t)b->width * b->height * 8, "accum64");
    check(wgpt_write_accum_f64(b->ctx, static_cast<const double*>(d.data)), b->ctx, "writeAccumF64");
    return undef(env);
  )
}

// setWavefrontConfig(ctx, poolPaths, unitsPerPass) (0 keeps a value)
EXPORT(SetWavefrontConfig) {
  BODY(
    CtxBox* b = ctx_box(env, a.at(0));
    check(wgpt_set_wavefront_config(b->ctx, a.u32(1), a.u64(2)), b->ctx, "setWavefrontConfig");
    return undef(env);
  )
}

// setWavefrontTuning(ctx, {travShape, shadeBlock, refillClosest, refillShadow, shadowWide})
EXPORT(SetWavefrontTuning) {
  BODY(
    CtxBox* b = ctx_box(env, a.at(0));
    wgpt_wavefront_tuning t{};
    wgpt_get_wavefront_tuning(b->ctx, &t);
    napi_value o = a.at(1);
    auto field = [&](const char* key, uint32_t* dst) {
      napi_value v = get(env, o, key);
      if (present(env, v) && napi_get_value_uint32(env, v, dst) != napi_ok) throw ArgError{std::string(key) + ": expected a number"};
    };
    field("travShape", &t.trav_shape);
    field("shadeBlock", &t.shade_block);
    field("refillClosest", &t.refill_closest);
    field("refillShadow", &t.refill_shadow);
    field("shadowWide", &t.shadow_wide);
    check(wgpt_set_wavefront_tuning(b->ctx, &t), b->ctx, "setWavefrontTuning");
    return undef(env);
  )
}

// getWavefrontTuning(ctx) -> {travShape, shadeBlock, refillClosest, refillShadow, shadowWide}
EXPORT(GetWavefrontTuning) {
  BODY(
    CtxBox* b = ctx_box(env, a.at(0));
    wgpt_wavefront_tuning t{};
    check(wgpt_get_wavefront_tuning(b->ctx, &t), b->ctx, "getWavefrontTuning");
    napi_value o;
    napi_create_object(env, &o);
    set(env, o, "travShape", make_u32(env, t.trav_shape));
    set(env, o, "shadeBlock", make_u32(env, t.shade_block));
    set(env, o, "refillClosest", make_u32(env, t.refill_closest));
    set(env, o, "refillShadow", make_u32(env, t.refill_shadow));
    set(env, o, "shadowWide", make_u32(env, t.shadow_wide));
    return o;
  )
}

// getWavefrontConfig(ctx) -> {poolPaths, unitsPerPass}
EXPORT(GetWavefrontConfig) {
  BODY(
    CtxBox* b = ctx_box(env, a.at(0));
    uint32_t pool = 0;
    uint64_t units = 0;
    check(wgpt_get_wavefront_config(b->ctx, &pool, &units), b->ctx, "getWavefrontConfig");
    napi_value o;
    napi_create_object(env, &o);
    set(env, o, "poolPaths", make_u32(env, pool));
    set(env, o, "unitsPerPass", make_f64(env, (double)units));
    return o;
  )
}

// Denoiser.execute (tracer.js:2583-2637): denoise(ctx, uBufData /*48 B*/, steps /*Uint32Array*/, passes)
EXPORT(Denoise) {
  BODY(
    CtxBox* b = ctx_box(env, a.at(0));
    View u = bytes_of(env, a.at(1), 48, "denoiser uniforms");
    uint32_t passes = a.u32(3);
    View s = typed_of(env, a.at(2), napi_uint32_array, passes, "steps");
    check(wgpt_denoise(b->ctx, u.data, static_cast<const uint32_t*>(s.data), passes), b->ctx, "denoise");
    return undef(env);
  )
}

// setDenoiseMode(ctx, DENOISE_EXACT | DENOISE_FAST): arithmetic of the a-trous passes
EXPORT(SetDenoiseMode) {
  BODY(CtxBox* b = ctx_box(env, a.at(0)); check(wgpt_set_denoise_mode(b->ctx, a.i32(1)), b->ctx, "setDenoiseMode"); return undef(env);)
}

// renderPreview blit (tracer.js:2365-2389): resample(ctx, dstW, dstH, ratioX, ratioY)
EXPORT(Resample) {
  BODY(
    CtxBox* b = ctx_box(env, a.at(0));
    check(wgpt_resample(b->ctx, a.u32(1), a.u32(2), (float)a.f64(3), (float)a.f64(4)), b->ctx, "resample");
    return undef(env);
  )
}

EXPORT(Synchronize) {
  BODY(CtxBox* b = ctx_box(env, a.at(0)); check(wgpt_synchronize(b->ctx), b->ctx, "synchronize"); return undef(env);)
}

// synchronizeTimeout(ctx, ms) -> true when the queued work finished, false while it still runs
EXPORT(SynchronizeTimeout) {
  BODY(
    CtxBox* b = ctx_box(env, a.at(0));
    int rc = wgpt_synchronize_timeout(b->ctx, a.u32(1));
    if (rc == WGPT_E_TIMEOUT) return make_bool(env, false);
    check(rc, b->ctx, "synchronizeTimeout");
    return make_bool(env, true);
  )
}

// ---- async: the equivalent of `await device.queue.onSubmittedWorkDone()` (tracer.js:2281)

struct AsyncJob {
  napi_async_work work = nullptr;
  napi_deferred deferred = nullptr;
  wgpt_ctx* ctx = nullptr;
  bool render = false;
  uint32_t args[6] = {0};
  int rc = WGPT_OK;
  std::string msg;
};

void async_execute(napi_env, void* data) {
  auto* j = static_cast<AsyncJob*>(data);
  if (j->render) j->rc = wgpt_render(j->ctx, j->args[0], j->args[1], j->args[2], j->args[3], j->args[4], j->args[5]);
  if (j->rc == WGPT_OK) j->rc = wgpt_synchronize(j->ctx);
  if (j->rc != WGPT_OK) j->msg = ctx_message(j->ctx, j->render ? "renderAsync" : "synchronizeAsync");
}

void async_complete(napi_env env, napi_status, void* data) {
  auto* j = static_cast<AsyncJob*>(data);
  if (j->rc == WGPT_OK) {
    napi_resolve_deferred(env, j->deferred, undef(env));
  } else {
    napi_value code, msg, err;
    napi_create_string_utf8(env, status_name(j->rc), NAPI_AUTO_LENGTH, &code);
    napi_create_string_utf8(env, j->msg.c_str(), NAPI_AUTO_LENGTH, &msg);
    napi_create_error(env, code, msg, &err);
    napi_reject_deferred(env, j->deferred, err);
  }
  napi_delete_async_work(env, j->work);
  delete j;
}

napi_value queue_async(napi_env env, AsyncJob* j, const char* name) {
  napi_value promise, res_name;
  napi_create_promise(env, &j->deferred, &promise);
  napi_create_string_utf8(env, name, NAPI_AUTO_LENGTH, &res_name);
  napi_create_async_work(env, nullptr, res_name, async_execute, async_complete, j, &j->work);
  napi_queue_async_work(env, j->work);
  return promise;
}

// synchronizeAsync(ctx) -> Promise, resolved once the context's queued work finished
EXPORT(SynchronizeAsync) {
  BODY(
    auto* j = new AsyncJob;
    j->ctx = ctx_box(env, a.at(0))->ctx;
    return queue_async(env, j, "wgpt.synchronizeAsync");
  )
}

// renderAsync(ctx, firstFrame, reps, x, y, w, h) -> Promise: one tile of Renderer.render with
// its submit + onSubmittedWorkDone (tracer.js:2262-2282), off the JavaScript thread
EXPORT(RenderAsync) {
  BODY(
    auto* j = new AsyncJob;
    j->ctx = ctx_box(env, a.at(0))->ctx;
    j->render = true;
    for (int i = 0; i < 6; ++i) j->args[i] = a.u32(1 + i);
    return queue_async(env, j, "wgpt.renderAsync");
  )
}

// ---- readback (SaveRender, gui.js:1622; canvas copies)

EXPORT(ReadAccum) {
  BODY(
    CtxBox* b = ctx_box(env, a.at(0));
    View d = typed_of(env, a.at(1), napi_float32_array, (size_t)b->width * b->height * 4, "accum");
    check(wgpt_read_accum(b->ctx, static_cast<float*>(d.data)), b->ctx, "readAccum");
    return undef(env);
  )
}

EXPORT(WriteAccum) {
  BODY(
    CtxBox* b = ctx_box(env, a.at(0));
    View d = typed_of(env, a.at(1), napi_float32_array, (size_t)b->width * b->height * 4, "accum");
    check(wgpt_write_accum(b->ctx, static_cast<const float*>(d.data)), b->ctx, "writeAccum");
    return undef(env);
  )
}

// readOutput(ctx, Uint8Array | Uint8ClampedArray of width*height*4), e.g. an ImageData's data
EXPORT(ReadOutput) {
  BODY(
    CtxBox* b = ctx_box(env, a.at(0));
    View d = typed_of(env, a.at(1), napi_uint8_array, (size_t)b->width * b->height * 4, "rgba8");
    check(wgpt_read_output(b->ctx, static_cast<uint8_t*>(d.data)), b->ctx, "readOutput");
    return undef(env);
  )
}

// readGBuffer(ctx, Float32Array of width*height*12): the 48-byte GBufferData records
EXPORT(ReadGBuffer) {
  BODY(
    CtxBox* b = ctx_box(env, a.at(0));
    View d = bytes_of(env, a.at(1), (size_t)b->width * b->height * 48, "gbuffer");
    check(wgpt_read_gbuffer(b->ctx, d.data), b->ctx, "readGBuffer");
    return undef(env);
  )
}

EXPORT(WriteGBuffer) {
  BODY(
    CtxBox* b = ctx_box(env, a.at(0));
    View d = bytes_of(env, a.at(1), (size_t)b->width * b->height * 48, "gbuffer");
    check(wgpt_write_gbuffer(b->ctx, d.data), b->ctx, "writeGBuffer");
    return undef(env);
  )
}

// readDenoised(ctx, filtered | null, composited | null): the last a-trous pass and the remodulated result
EXPORT(ReadDenoised) {
  BODY(
    CtxBox* b = ctx_box(env, a.at(0));
    size_t n = (size_t)b->width * b->height * 4;
    float* f = a.is_nullish(1) ? nullptr : static_cast<float*>(typed_of(env, a.at(1), napi_float32_array, n, "filtered").data);
    float* c = a.is_nullish(2) ? nullptr : static_cast<float*>(typed_of(env, a.at(2), napi_float32_array, n, "composited").data);
    check(wgpt_read_denoised(b->ctx, f, c), b->ctx, "readDenoised");
    return undef(env);
  )
}

// readCanvas(ctx, rgba8, dstW, dstH): the resample() result
EXPORT(ReadCanvas) {
  BODY(
    CtxBox* b = ctx_box(env, a.at(0));
    uint32_t w = a.u32(2), h = a.u32(3);
    View d = typed_of(env, a.at(1), napi_uint8_array, (size_t)w * h * 4, "canvas");
    check(wgpt_read_canvas(b->ctx, static_cast<uint8_t*>(d.data), w, h), b->ctx, "readCanvas");
    return undef(env);
  )
}

// ---- batched views

// setViews(ctx, widths Uint32Array, heights Uint32Array)
EXPORT(SetViews) {
  BODY(
    CtxBox* b = ctx_box(env, a.at(0));
    View w = typed_of(env, a.at(1), napi_uint32_array, 0, "widths");
    View h = typed_of(env, a.at(2), napi_uint32_array, w.length, "heights");
    const uint32_t* wp = static_cast<const uint32_t*>(w.data);
    const uint32_t* hp = static_cast<const uint32_t*>(h.data);
    check(wgpt_set_views(b->ctx, (uint32_t)w.length, wp, hp), b->ctx, "setViews");
    b->view_w.assign(wp, wp + w.length);
    b->view_h.assign(hp, hp + w.length);
    return undef(env);
  )
}

// renderViews(ctx, params /*n x 112 B*/, firstFrames Uint32Array, spp Uint32Array, doneMs Float32Array | null)
EXPORT(RenderViews) {
  BODY(
    CtxBox* b = ctx_box(env, a.at(0));
    size_t n = b->view_w.size();
    View p = bytes_of(env, a.at(1), n * 112, "params");
    View ff = typed_of(env, a.at(2), napi_uint32_array, n, "firstFrames");
    View sp = typed_of(env, a.at(3), napi_uint32_array, n, "spp");
    float* done = a.is_nullish(4) ? nullptr : static_cast<float*>(typed_of(env, a.at(4), napi_float32_array, n, "doneMs").data);
    check(wgpt_render_views(b->ctx, p.data, static_cast<const uint32_t*>(ff.data), static_cast<const uint32_t*>(sp.data), done),
          b->ctx, "renderViews");
    return undef(env);
  )
}

// renderViewsGBuffer(ctx, params /*n x 112 B*/)
EXPORT(RenderViewsGBuffer) {
  BODY(
    CtxBox* b = ctx_box(env, a.at(0));
    View p = bytes_of(env, a.at(1), b->view_w.size() * 112, "params");
    check(wgpt_render_views_gbuffer(b->ctx, p.data), b->ctx, "renderViewsGBuffer");
    return undef(env);
  )
}

// readView(ctx, view, accum Float32Array | null, rgba8 | null)
EXPORT(ReadView) {
  BODY(
    CtxBox* b = ctx_box(env, a.at(0));
    uint32_t v = a.u32(1);
    if (v >= b->view_w.size()) throw ArgError{"view index out of range"};
    size_t n = (size_t)b->view_w[v] * b->view_h[v] * 4;
    float* acc = a.is_nullish(2) ? nullptr : static_cast<float*>(typed_of(env, a.at(2), napi_float32_array, n, "accum").data);
    uint8_t* out = a.is_nullish(3) ? nullptr : static_cast<uint8_t*>(typed_of(env, a.at(3), napi_uint8_array, n, "rgba8").data);
    check(wgpt_read_view(b->ctx, v, acc, out), b->ctx, "readView");
    return undef(env);
  )
}

// ---- parity and measurement helpers

// traceRays(ctx, rays Float32Array n x 6) -> {objIdx, matIdx, prim, t, normal}
EXPORT(TraceRays) {
  BODY(
    CtxBox* b = ctx_box(env, a.at(0));
    View r = typed_of(env, a.at(1), napi_float32_array, 0, "rays");
    uint32_t n = (uint32_t)(r.length / 6);
    void *o, *m, *p, *t, *nn;
    napi_value ov = new_typed(env, napi_int32_array, n, &o), mv = new_typed(env, napi_int32_array, n, &m),
               pv = new_typed(env, napi_int32_array, n, &p), tv = new_typed(env, napi_float32_array, n, &t),
               nv = new_typed(env, napi_float32_array, (size_t)n * 3, &nn);
    check(wgpt_trace_rays(b->ctx, static_cast<const float*>(r.data), n, (int32_t*)o, (int32_t*)m, (int32_t*)p, (float*)t,
                          (float*)nn), b->ctx, "traceRays");
    napi_value res;
    napi_create_object(env, &res);
    set(env, res, "objIdx", ov); set(env, res, "matIdx", mv); set(env, res, "prim", pv);
    set(env, res, "t", tv); set(env, res, "normal", nv);
    return res;
  )
}

EXPORT(SetCounting) {
  BODY(CtxBox* b = ctx_box(env, a.at(0)); check(wgpt_set_counting(b->ctx, a.boolean(1) ? 1 : 0), b->ctx, "setCounting"); return undef(env);)
}

// readCounters(ctx) -> BigUint64Array(16)
EXPORT(ReadCounters) {
  BODY(
    CtxBox* b = ctx_box(env, a.at(0));
    void* d;
    napi_value arr = new_typed(env, napi_biguint64_array, 16, &d);
    check(wgpt_read_counters(b->ctx, static_cast<uint64_t*>(d)), b->ctx, "readCounters");
    return arr;
  )
}

// readStageCounters(ctx) -> BigUint64Array(128)
EXPORT(ReadStageCounters) {
  BODY(
    CtxBox* b = ctx_box(env, a.at(0));
    void* d;
    napi_value arr = new_typed(env, napi_biguint64_array, 128, &d);
    check(wgpt_read_stage_counters(b->ctx, static_cast<uint64_t*>(d)), b->ctx, "readStageCounters");
    return arr;
  )
}

EXPORT(SetStageTiming) {
  BODY(CtxBox* b = ctx_box(env, a.at(0)); check(wgpt_set_stage_timing(b->ctx, a.boolean(1) ? 1 : 0), b->ctx, "setStageTiming"); return undef(env);)
}

// readStageTimes(ctx) -> {ms Float64Array(8), launches Uint32Array(8)}
EXPORT(ReadStageTimes) {
  BODY(
    CtxBox* b = ctx_box(env, a.at(0));
    void *ms, *ln;
    napi_value msv = new_typed(env, napi_float64_array, 8, &ms), lnv = new_typed(env, napi_uint32_array, 8, &ln);
    check(wgpt_read_stage_times(b->ctx, static_cast<double*>(ms), static_cast<uint32_t*>(ln)), b->ctx, "readStageTimes");
    napi_value o;
    napi_create_object(env, &o);
    set(env, o, "ms", msv);
    set(env, o, "launches", lnv);
    return o;
  )
}

// stream(ctx) -> BigInt cudaStream_t, for callers that order their own CUDA work around renders
EXPORT(Stream) { BODY(return make_big(env, (uint64_t)(uintptr_t)wgpt_stream(ctx_box(env, a.at(0))->ctx));) }

// ---- allocation-free denoiser (device pointers as BigInt)

// denoiseNoalloc(color, gbuf, uniforms48, steps Uint32Array, passes, outRgba8, outComposited | null, stream | null)
EXPORT(DenoiseNoalloc) {
  BODY(
    View u = bytes_of(env, a.at(2), 48, "denoiser uniforms");
    uint32_t passes = a.u32(4);
    View s = typed_of(env, a.at(3), napi_uint32_array, passes, "steps");
    int rc = wgpt_denoise_noalloc(static_cast<const float*>(a.device_ptr(0)), a.device_ptr(1), u.data,
                                  static_cast<const uint32_t*>(s.data), passes, static_cast<uint8_t*>(a.device_ptr(5)),
                                  static_cast<float*>(a.device_ptr(6)), a.device_ptr(7));
    check(rc, nullptr, "denoiseNoalloc");
    return undef(env);
  )
}

// ----------------------------------------------------------------------------------------------
// Learned denoiser (no reference counterpart; Denoiser.execute stays the fallback)

// kpcnCreate(device, seed) -> network
EXPORT(KpcnCreate) {
  BODY(
    wgpt_kpcn* k = nullptr;
    int rc = wgpt_kpcn_create(a.i32(0), a.is_nullish(1) ? 1 : a.u64(1), &k);
    if (rc != WGPT_OK) throw StatusError{rc, "kpcnCreate: failed"};
    auto* b = new KpcnBox{k};
    napi_value ext;
    napi_create_external(env, b, finalize_kpcn, nullptr, &ext);
    return ext;
  )
}

EXPORT(KpcnDestroy) {
  BODY(
    void* p = nullptr;
    napi_get_value_external(env, a.at(0), &p);
    auto* b = static_cast<KpcnBox*>(p);
    if (b && b->k) { wgpt_kpcn_destroy(b->k); b->k = nullptr; }
    return undef(env);
  )
}

uint64_t kpcn_params(wgpt_kpcn* k) {
  uint64_t n = 0;
  check_k(wgpt_kpcn_num_params(k, &n), k, "kpcnNumParams");
  return n;
}

EXPORT(KpcnNumParams) { BODY(return make_f64(env, (double)kpcn_params(kpcn_box(env, a.at(0))->k));) }

// kpcnGetParams(k) -> Float32Array of every parameter (layer by layer: weights, then biases)
EXPORT(KpcnGetParams) {
  BODY(
    wgpt_kpcn* k = kpcn_box(env, a.at(0))->k;
    void* d;
    napi_value arr = new_typed(env, napi_float32_array, (size_t)kpcn_params(k), &d);
    check_k(wgpt_kpcn_get_params(k, static_cast<float*>(d)), k, "kpcnGetParams");
    return arr;
  )
}

EXPORT(KpcnSetParams) {
  BODY(
    wgpt_kpcn* k = kpcn_box(env, a.at(0))->k;
    View p = typed_of(env, a.at(1), napi_float32_array, (size_t)kpcn_params(k), "params");
    check_k(wgpt_kpcn_set_params(k, static_cast<const float*>(p.data)), k, "kpcnSetParams");
    return undef(env);
  )
}

// kpcnAddExample(k, noisy Float32Array w*h*4, gbuf (48 B/px), target Float32Array w*h*4, w, h)
EXPORT(KpcnAddExample) {
  BODY(
    wgpt_kpcn* k = kpcn_box(env, a.at(0))->k;
    uint32_t w = a.u32(4), h = a.u32(5);
    size_t n = (size_t)w * h;
    View noisy = typed_of(env, a.at(1), napi_float32_array, n * 4, "noisy");
    View gbuf = bytes_of(env, a.at(2), n * 48, "gbuffer");
    View target = typed_of(env, a.at(3), napi_float32_array, n * 4, "target");
    check_k(wgpt_kpcn_add_example(k, static_cast<const float*>(noisy.data), gbuf.data, static_cast<const float*>(target.data), w, h),
            k, "kpcnAddExample");
    return undef(env);
  )
}

EXPORT(KpcnNumExamples) {
  BODY(
    wgpt_kpcn* k = kpcn_box(env, a.at(0))->k;
    uint32_t n = 0;
    check_k(wgpt_kpcn_num_examples(k, &n), k, "kpcnNumExamples");
    return make_u32(env, n);
  )
}

// kpcnTrain(k, steps, batch, crop, lr, seed) -> Float32Array of per-step losses
EXPORT(KpcnTrain) {
  BODY(
    wgpt_kpcn* k = kpcn_box(env, a.at(0))->k;
    uint32_t steps = a.u32(1);
    void* d;
    napi_value arr = new_typed(env, napi_float32_array, steps, &d);
    check_k(wgpt_kpcn_train(k, steps, a.u32(2), a.u32(3), (float)a.f64(4), a.u64(5), static_cast<float*>(d)), k, "kpcnTrain");
    return arr;
  )
}

// kpcnGrads(k, batch, crop, seed, devGrads BigInt) -> loss; the gradient lands in device memory
EXPORT(KpcnGrads) {
  BODY(
    wgpt_kpcn* k = kpcn_box(env, a.at(0))->k;
    float loss = 0.f;
    check_k(wgpt_kpcn_grads(k, a.u32(1), a.u32(2), a.u64(3), &loss, static_cast<float*>(a.device_ptr(4))), k, "kpcnGrads");
    return make_f64(env, loss);
  )
}

// kpcnApply(k, devGrads BigInt, scale, lr): one Adam step with devGrads * scale
EXPORT(KpcnApply) {
  BODY(
    wgpt_kpcn* k = kpcn_box(env, a.at(0))->k;
    check_k(wgpt_kpcn_apply(k, static_cast<const float*>(a.device_ptr(1)), (float)a.f64(2), (float)a.f64(3)), k, "kpcnApply");
    return undef(env);
  )
}

// kpcnLossAndGrads(k, noisy, gbuf, target, w, h) -> {loss, grads Float32Array, out Float32Array}
EXPORT(KpcnLossAndGrads) {
  BODY(
    wgpt_kpcn* k = kpcn_box(env, a.at(0))->k;
    uint32_t w = a.u32(4), h = a.u32(5);
    size_t n = (size_t)w * h;
    View noisy = typed_of(env, a.at(1), napi_float32_array, n * 4, "noisy");
    View gbuf = bytes_of(env, a.at(2), n * 48, "gbuffer");
    View target = typed_of(env, a.at(3), napi_float32_array, n * 4, "target");
    void *g, *o;
    napi_value gv = new_typed(env, napi_float32_array, (size_t)kpcn_params(k), &g);
    napi_value ov = new_typed(env, napi_float32_array, n * 4, &o);
    float loss = 0.f;
    check_k(wgpt_kpcn_loss_and_grads(k, static_cast<const float*>(noisy.data), gbuf.data, static_cast<const float*>(target.data),
                                     w, h, &loss, static_cast<float*>(g), static_cast<float*>(o)), k, "kpcnLossAndGrads");
    napi_value res;
    napi_create_object(env, &res);
    set(env, res, "loss", make_f64(env, loss));
    set(env, res, "grads", gv);
    set(env, res, "out", ov);
    return res;
  )
}

// kpcnSetConvMode(k, KPCN_CONV_PIPELINED | KPCN_CONV_PER_TILE)
EXPORT(KpcnSetConvMode) {
  BODY(wgpt_kpcn* k = kpcn_box(env, a.at(0))->k; check_k(wgpt_kpcn_set_conv_mode(k, a.i32(1)), k, "kpcnSetConvMode"); return undef(env);)
}

// kpcnDenoise(k, ctx, exposure, filtered Float32Array | null): the context's accumulation and
// G-buffer into its rgba8 image (readOutput afterwards)
EXPORT(KpcnDenoise) {
  BODY(
    wgpt_kpcn* k = kpcn_box(env, a.at(0))->k;
    CtxBox* b = ctx_box(env, a.at(1));
    float* f = a.is_nullish(3) ? nullptr
                               : static_cast<float*>(typed_of(env, a.at(3), napi_float32_array, (size_t)b->width * b->height * 4, "filtered").data);
    check_k(wgpt_kpcn_denoise(k, b->ctx, (float)a.f64(2), f), k, "kpcnDenoise");
    return undef(env);
  )
}

// kpcnDenoiseView(k, ctx, view, exposure, filtered | null)
EXPORT(KpcnDenoiseView) {
  BODY(
    wgpt_kpcn* k = kpcn_box(env, a.at(0))->k;
    CtxBox* b = ctx_box(env, a.at(1));
    uint32_t v = a.u32(2);
    if (v >= b->view_w.size()) throw ArgError{"view index out of range"};
    float* f = a.is_nullish(4) ? nullptr
                               : static_cast<float*>(typed_of(env, a.at(4), napi_float32_array, (size_t)b->view_w[v] * b->view_h[v] * 4, "filtered").data);
    check_k(wgpt_kpcn_denoise_view(k, b->ctx, v, (float)a.f64(3), f), k, "kpcnDenoiseView");
    return undef(env);
  )
}

// gemmBf16(device, a Uint16Array m*k, b Uint16Array n*k, m, n, k) -> Float32Array m*n
EXPORT(GemmBf16) {
  BODY(
    int m = a.i32(3), n = a.i32(4), kk = a.i32(5);
    if (m <= 0 || n <= 0 || kk <= 0) throw ArgError{"gemmBf16: sizes must be positive"};
    View av = typed_of(env, a.at(1), napi_uint16_array, (size_t)m * kk, "a");
    View bv = typed_of(env, a.at(2), napi_uint16_array, (size_t)n * kk, "b");
    void* c;
    napi_value cv = new_typed(env, napi_float32_array, (size_t)m * n, &c);
    check(wgpt_gemm_bf16(a.i32(0), static_cast<const uint16_t*>(av.data), static_cast<const uint16_t*>(bv.data),
                         static_cast<float*>(c), m, n, kk), nullptr, "gemmBf16");
    return cv;
  )
}

// ----------------------------------------------------------------------------------------------
// Host builders (the tracer.js host math, native)

// ModelData.generateBVH (tracer.js:1025-1118): buildBlas(tris24 Float32Array) -> {bvh, triangle}
// as the byte arrays packSceneData concatenates (32-B nodes, 128-B triangles)
EXPORT(BuildBlas) {
  BODY(
    View t = typed_of(env, a.at(0), napi_float32_array, 0, "tris24");
    uint32_t n = (uint32_t)(t.length / 24);
    if (n == 0) throw ArgError{"buildBlas: no triangles"};
    std::vector<uint8_t> nodes((size_t)(2 * n - 1) * 32);
    void* tri;
    napi_value triv = new_typed(env, napi_uint8_array, (size_t)n * 128, &tri);
    uint32_t cnt = 0;
    check(wgpt_build_blas(static_cast<const float*>(t.data), n, (wgpt_bvh_node*)nodes.data(), &cnt, (wgpt_triangle*)tri),
          nullptr, "buildBlas");
    void* nd;
    napi_value ndv = new_typed(env, napi_uint8_array, (size_t)cnt * 32, &nd);
    memcpy(nd, nodes.data(), (size_t)cnt * 32);
    napi_value o;
    napi_create_object(env, &o);
    set(env, o, "bvh", ndv);
    set(env, o, "triangle", triv);
    return o;
  )
}

// SceneBVHBuilder (tracer.js:1509-1619): buildTlas(aabbs6 Float32Array) -> Uint8Array of 32-B nodes
EXPORT(BuildTlas) {
  BODY(
    View t = typed_of(env, a.at(0), napi_float32_array, 0, "aabbs6");
    uint32_t n = (uint32_t)(t.length / 6);
    if (n == 0) throw ArgError{"buildTlas: no objects"};
    std::vector<uint8_t> nodes((size_t)(2 * n - 1) * 32);
    uint32_t cnt = 0;
    check(wgpt_build_tlas(static_cast<const float*>(t.data), n, (wgpt_bvh_node*)nodes.data(), &cnt), nullptr, "buildTlas");
    void* nd;
    napi_value ndv = new_typed(env, napi_uint8_array, (size_t)cnt * 32, &nd);
    memcpy(nd, nodes.data(), (size_t)cnt * 32);
    return ndv;
  )
}

// HDRTexture.buildHDRCDF (tracer.js:135-204): buildEnvCdf(sky16, w, h, exposure) ->
// {skyCDF Float32Array, sky_cdf_index, totalWeight}
EXPORT(BuildEnvCdf) {
  BODY(
    uint32_t w = a.u32(1), h = a.u32(2);
    View s = typed_of(env, a.at(0), napi_uint16_array, (size_t)w * h * 4, "sky16");
    void* cdf;
    napi_value cv = new_typed(env, napi_float32_array, (size_t)(h + 1) + (size_t)h * (w + 1), &cdf);
    double total = 0.0;
    check(wgpt_build_env_cdf(static_cast<const uint16_t*>(s.data), w, h, a.f64(3), static_cast<float*>(cdf), &total), nullptr,
          "buildEnvCdf");
    napi_value o;
    napi_create_object(env, &o);
    set(env, o, "skyCDF", cv);
    set(env, o, "sky_cdf_index", make_u32(env, h + 1));
    set(env, o, "totalWeight", make_f64(env, total));
    return o;
  )
}

// buildEnvAlias(sky16, w, h, exposure) -> Uint8Array of {float prob; uint32 alias} per texel,
// ready for setScene's skyAlias
EXPORT(BuildEnvAlias) {
  BODY(
    uint32_t w = a.u32(1), h = a.u32(2);
    size_t n = (size_t)w * h;
    View s = typed_of(env, a.at(0), napi_uint16_array, n * 4, "sky16");
    std::vector<float> prob(n);
    std::vector<uint32_t> alias(n);
    check(wgpt_build_env_alias(static_cast<const uint16_t*>(s.data), w, h, a.f64(3), prob.data(), alias.data()), nullptr,
          "buildEnvAlias");
    void* d;
    napi_value out = new_typed(env, napi_uint8_array, n * 8, &d);
    uint8_t* p = static_cast<uint8_t*>(d);
    for (size_t i = 0; i < n; ++i) {
      memcpy(p + 8 * i, &prob[i], 4);
      memcpy(p + 8 * i + 4, &alias[i], 4);
    }
    return out;
  )
}

// parseHdr + HDRTexture.updateData (lib/parse-hdr.js:125-211, tracer.js:76-87):
// decodeRgbe(file Uint8Array, exposure) -> {data Uint16Array (rgba16f), width, height}
EXPORT(DecodeRgbe) {
  BODY(
    View f = bytes_of(env, a.at(0), 0, "file");
    double exposure = a.is_nullish(1) ? 1.0 : a.f64(1);
    uint32_t w = 0, h = 0;
    check(wgpt_decode_rgbe(static_cast<const uint8_t*>(f.data), f.bytes, exposure, nullptr, &w, &h), nullptr, "decodeRgbe");
    void* d;
    napi_value dv = new_typed(env, napi_uint16_array, (size_t)w * h * 4, &d);
    check(wgpt_decode_rgbe(static_cast<const uint8_t*>(f.data), f.bytes, exposure, static_cast<uint16_t*>(d), &w, &h), nullptr,
          "decodeRgbe");
    napi_value o;
    napi_create_object(env, &o);
    set(env, o, "data", dv);
    set(env, o, "width", make_u32(env, w));
    set(env, o, "height", make_u32(env, h));
    return o;
  )
}

// ModelData.parseOBJ (tracer.js:949-987): parseObj(text) -> {tris24 Float32Array, positions Float32Array}
EXPORT(ParseObj) {
  BODY(
    std::string text = a.str(0);
    uint32_t n_tris = 0, n_pos = 0;
    check(wgpt_parse_obj(text.data(), text.size(), nullptr, 0, &n_tris, nullptr, 0, &n_pos), nullptr, "parseObj");
    void *t, *p;
    napi_value tv = new_typed(env, napi_float32_array, (size_t)n_tris * 24, &t);
    napi_value pv = new_typed(env, napi_float32_array, n_pos, &p);
    check(wgpt_parse_obj(text.data(), text.size(), static_cast<float*>(t), n_tris, &n_tris, static_cast<float*>(p), n_pos, &n_pos),
          nullptr, "parseObj");
    napi_value o;
    napi_create_object(env, &o);
    set(env, o, "tris24", tv);
    set(env, o, "positions", pv);
    return o;
  )
}

// ----------------------------------------------------------------------------------------------
// Test and measurement support

// selftestWait(device, limit) -> {status, ms}
EXPORT(SelftestWait) {
  BODY(
    uint32_t status = 0;
    float ms = 0.f;
    check(wgpt_selftest_wait(a.i32(0), a.u32(1), &status, &ms), nullptr, "selftestWait");
    napi_value o;
    napi_create_object(env, &o);
    set(env, o, "status", make_u32(env, status));
    set(env, o, "ms", make_f64(env, ms));
    return o;
  )
}

// sampleEnv(ctx, u2 Float32Array n x 2) -> {texel Uint32Array n x 2, pdf Float32Array}
EXPORT(SampleEnv) {
  BODY(
    CtxBox* b = ctx_box(env, a.at(0));
    View u = typed_of(env, a.at(1), napi_float32_array, 0, "u2");
    uint32_t n = (uint32_t)(u.length / 2);
    void *t, *p;
    napi_value tv = new_typed(env, napi_uint32_array, (size_t)n * 2, &t);
    napi_value pv = new_typed(env, napi_float32_array, n, &p);
    check(wgpt_sample_env(b->ctx, static_cast<const float*>(u.data), n, static_cast<uint32_t*>(t), static_cast<float*>(p)),
          b->ctx, "sampleEnv");
    napi_value o;
    napi_create_object(env, &o);
    set(env, o, "texel", tv);
    set(env, o, "pdf", pv);
    return o;
  )
}

// rngStream(device, idx, sampleNumber, seed, n) -> Float32Array of main's random draws
EXPORT(RngStream) {
  BODY(
    uint32_t n = a.u32(4);
    void* d;
    napi_value dv = new_typed(env, napi_float32_array, n, &d);
    check(wgpt_rng_stream(a.i32(0), a.u32(1), a.u32(2), a.u32(3), n, static_cast<float*>(d)), nullptr, "rngStream");
    return dv;
  )
}

// probeL2Read(device, bytes, reps) -> GB/s
EXPORT(ProbeL2Read) {
  BODY(
    double gbps = 0.0;
    check(wgpt_probe_l2_read(a.i32(0), a.u64(1), a.u32(2), &gbps), nullptr, "probeL2Read");
    return make_f64(env, gbps);
  )
}

// ----------------------------------------------------------------------------------------------

napi_value Init(napi_env env, napi_value exports) {
#define FN(js, c) napi_property_descriptor{js, nullptr, c, nullptr, nullptr, nullptr, napi_default, nullptr}
  const napi_property_descriptor props[] = {
      FN("create", Create), FN("destroy", Destroy), FN("abiVersion", AbiVersion), FN("lastError", LastError),
      FN("setScene", SetScene), FN("validateScene", ValidateScene), FN("updateObjects", UpdateObjects),
      FN("updateScene", UpdateScene), FN("resize", Resize), FN("setParams", SetParams), FN("render", Render),
      FN("renderAsync", RenderAsync), FN("renderGBuffer", RenderGBuffer), FN("setRenderMode", SetRenderMode),
      FN("setEnvSampling", SetEnvSampling), FN("setAccumF64", SetAccumF64), FN("readAccumF64", ReadAccumF64),
      FN("writeAccumF64", WriteAccumF64), FN("setWavefrontConfig", SetWavefrontConfig),
      FN("getWavefrontConfig", GetWavefrontConfig), FN("setWavefrontTuning", SetWavefrontTuning),
      FN("getWavefrontTuning", GetWavefrontTuning), FN("denoise", Denoise), FN("setDenoiseMode", SetDenoiseMode), FN("resample", Resample),
      FN("synchronize", Synchronize), FN("synchronizeTimeout", SynchronizeTimeout),
      FN("synchronizeAsync", SynchronizeAsync), FN("readAccum", ReadAccum), FN("writeAccum", WriteAccum),
      FN("readOutput", ReadOutput), FN("readGBuffer", ReadGBuffer), FN("writeGBuffer", WriteGBuffer),
      FN("readDenoised", ReadDenoised), FN("readCanvas", ReadCanvas), FN("setViews", SetViews),
      FN("renderViews", RenderViews), FN("renderViewsGBuffer", RenderViewsGBuffer), FN("readView", ReadView),
      FN("traceRays", TraceRays), FN("setCounting", SetCounting), FN("readCounters", ReadCounters),
      FN("readStageCounters", ReadStageCounters), FN("setStageTiming", SetStageTiming),
      FN("readStageTimes", ReadStageTimes), FN("stream", Stream), FN("denoiseNoalloc", DenoiseNoalloc),
      FN("kpcnCreate", KpcnCreate), FN("kpcnDestroy", KpcnDestroy), FN("kpcnNumParams", KpcnNumParams),
      FN("kpcnGetParams", KpcnGetParams), FN("kpcnSetParams", KpcnSetParams), FN("kpcnAddExample", KpcnAddExample),
      FN("kpcnNumExamples", KpcnNumExamples), FN("kpcnTrain", KpcnTrain), FN("kpcnGrads", KpcnGrads),
      FN("kpcnApply", KpcnApply), FN("kpcnLossAndGrads", KpcnLossAndGrads), FN("kpcnDenoise", KpcnDenoise), FN("kpcnSetConvMode", KpcnSetConvMode),
      FN("kpcnDenoiseView", KpcnDenoiseView), FN("gemmBf16", GemmBf16), FN("buildBlas", BuildBlas),
      FN("buildTlas", BuildTlas), FN("buildEnvCdf", BuildEnvCdf), FN("buildEnvAlias", BuildEnvAlias),
      FN("decodeRgbe", DecodeRgbe), FN("parseObj", ParseObj), FN("selftestWait", SelftestWait),
      FN("probeL2Read", ProbeL2Read), FN("sampleEnv", SampleEnv), FN("rngStream", RngStream),
  };
#undef FN
  napi_define_properties(env, exports, sizeof props / sizeof props[0], props);
  // enum values tracer.js passes by name
  set(env, exports, "MODE_WAVEFRONT", make_u32(env, WGPT_MODE_WAVEFRONT));
  set(env, exports, "MODE_MEGAKERNEL", make_u32(env, WGPT_MODE_MEGAKERNEL));
  set(env, exports, "ENV_CDF", make_u32(env, WGPT_ENV_CDF));
  set(env, exports, "ENV_ALIAS", make_u32(env, WGPT_ENV_ALIAS));
  set(env, exports, "DENOISE_EXACT", make_u32(env, WGPT_DENOISE_EXACT));
  set(env, exports, "DENOISE_FAST", make_u32(env, WGPT_DENOISE_FAST));
  set(env, exports, "KPCN_CONV_PIPELINED", make_u32(env, WGPT_KPCN_CONV_PIPELINED));
  set(env, exports, "KPCN_CONV_PER_TILE", make_u32(env, WGPT_KPCN_CONV_PER_TILE));
  set(env, exports, "NOALLOC_MAX_PIXELS", make_u32(env, WGPT_NOALLOC_MAX_PIXELS));
  return exports;
}

}  // namespace

NAPI_MODULE(NODE_GYP_MODULE_NAME, Init)
