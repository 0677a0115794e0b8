// C ABI of the renderer (include/wgpt.h): context, scene upload with layout validation, image
// buffers, and the render / G-buffer / denoise / resample entry points.  Each call maps to one
// step of tracer.js's Renderer or Denoiser (cited per function in wgpt.h).
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>
#include <string>
#include <vector>
#include <set>
#include <utility>
#include <algorithm>
#include <chrono>
#include <thread>

#include "../../include/wgpt.h"
#include "wgpt_internal.h"

struct wgpt_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  // scene buffers: 0 materials, 1 objects, 2 tlas, 3 meshes, 4 bvh, 5 triangles, 6 planes,
  // 7 lights, 8 sky_cdf, 9 sky texels, 10 texture array, 11 sky alias table
  void* d_buf[12] = {nullptr};
  size_t cap[12] = {0};
  size_t bytes[12] = {0};
  bool has_alias = false;
  int env_mode = WGPT_ENV_CDF;
  wgpt::DeviceScene ds{};
  bool has_scene = false;
  // images
  uint32_t w = 0, h = 0;
  float* accum = nullptr;
  uint8_t* out = nullptr;
  float* gbuf = nullptr;
  // denoiser
  float* dn_a = nullptr;
  float* dn_b = nullptr;
  float* dn_guide = nullptr;
  float* dn_comp = nullptr;
  int dn_mode = WGPT_DENOISE_EXACT;
  const float* dn_final = nullptr;
  // preview canvas
  uint8_t* canvas = nullptr;
  uint32_t cw = 0, ch = 0;
  // params, status, counters
  wgpt_scene_params params{};
  bool has_params = false;
  uint32_t* d_status = nullptr;
  unsigned long long* d_counters = nullptr;
  bool counting = false;
  int mode = WGPT_MODE_WAVEFRONT;
  // derived child-pair node arrays (64 bytes per node) of the TLAS and the BLAS buffer
  void* d_pairs_tlas = nullptr;
  void* d_pairs_bvh = nullptr;
  uint32_t tlas_depth = 0, blas_depth = 0;   // deepest levels of the uploaded trees
  size_t pairs_cap[2] = {0, 0};
  wgpt::StageTimer* timer = nullptr;
  bool timing = false;
  wgpt::WfEngine* wf = nullptr;   // wavefront renderer: path pool, sample buffer, loop graph
  // batched views: size and images of each
  struct View { uint32_t w, h; float* accum; uint8_t* out; float* gbuf; };
  std::vector<View> views;
  double* acc64 = nullptr;        // optional FP64 Welford accumulation (8 doubles per pixel)
  // kept from the last full upload for the objects fast path: the (node, triangle) offset
  // pairs whose BLAS passed validation, and a host copy of the material buffer
  std::set<std::pair<uint32_t, uint32_t>> blas_checked;
  std::vector<wgpt_material> host_mats;
  std::vector<int32_t> light_objs;   // obj_idx of each resident light record
};

namespace {

int fail(wgpt_ctx* c, int code, const std::string& msg) {
  if (c) c->err = msg;
  return code;
}

int cuda_fail(wgpt_ctx* c, cudaError_t e, const char* what) {
  return fail(c, e == cudaErrorMemoryAllocation ? WGPT_E_NOMEM : WGPT_E_CUDA,
              std::string(what) + ": " + cudaGetErrorString(e));
}

#define CK(call, what)                                   \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) return cuda_fail(ctx, e_, what); \
  } while (0)

void dfree(void*& p) {
  if (p) cudaFree(p);
  p = nullptr;
}
template <typename T>
void dfree_t(T*& p) {
  if (p) cudaFree((void*)p);
  p = nullptr;
}

const uint32_t kStride[12] = {WGPT_STRIDE_MATERIAL, WGPT_STRIDE_OBJECT, WGPT_STRIDE_NODE, WGPT_STRIDE_MESH_READ,
                              WGPT_STRIDE_NODE, WGPT_STRIDE_TRIANGLE, WGPT_STRIDE_PLANE, WGPT_STRIDE_LIGHT, 4, 8, 4, 8};
const char* kName[12] = {"materials", "objects", "tlas", "meshes", "bvh", "triangles", "planes", "lights",
                         "sky_cdf", "sky", "textures", "sky_alias"};

struct HostScene {
  const wgpt_material* mats; uint32_t n_mats;
  const wgpt_object* objs; uint32_t n_objs;
  const wgpt_bvh_node* tlas; uint32_t n_tlas;
  const uint8_t* meshes; uint32_t n_meshes;
  const wgpt_bvh_node* bvh; uint32_t n_bvh;
  const wgpt_triangle* tris; uint32_t n_tris;
  const wgpt_plane* planes; uint32_t n_planes;
  const wgpt_light* lights; uint32_t n_lights;
  uint32_t tex_layers;
};

constexpr uint32_t kMaxDepth = 62;   // traversal stacks hold 64 entries (shader.wgsl:17)

// A BVH in the reference's DFS layout: left child = index + 1, right child = base + next
// (strictly after the left child), leaves reference [item_base + next, + count).  Returns an
// empty string when every reachable node and item is in range and the depth fits the stack.
std::string check_tree(const wgpt_bvh_node* nodes, uint32_t n_nodes, uint32_t root, uint32_t base,
                       uint32_t item_base, uint32_t n_items, const char* what) {
  if (root >= n_nodes) return std::string(what) + ": root node out of range";
  std::vector<std::pair<uint32_t, uint32_t>> st;
  st.push_back({root, 0u});
  char buf[256];
  while (!st.empty()) {
    auto [i, d] = st.back();
    st.pop_back();
    if (d > kMaxDepth) { snprintf(buf, sizeof buf, "%s: tree deeper than %u levels", what, kMaxDepth); return buf; }
    const wgpt_bvh_node& nd = nodes[i];
    if (nd.num_triangles > 0u) {
      uint64_t start = (uint64_t)item_base + nd.next;
      if (start + nd.num_triangles > n_items) {
        snprintf(buf, sizeof buf, "%s: leaf %u references items [%llu, %llu) beyond %u", what, i,
                 (unsigned long long)start, (unsigned long long)(start + nd.num_triangles), n_items);
        return buf;
      }
    } else {
      uint64_t l = (uint64_t)i + 1u, r = (uint64_t)base + nd.next;
      if (l >= n_nodes || r >= n_nodes || r <= i) {
        snprintf(buf, sizeof buf, "%s: inner node %u has children %llu/%llu outside (%u, %u)", what, i,
                 (unsigned long long)l, (unsigned long long)r, i, n_nodes);
        return buf;
      }
      st.push_back({(uint32_t)l, d + 1});
      st.push_back({(uint32_t)r, d + 1});
    }
  }
  return "";
}

std::string validate(const HostScene& s, uint32_t flags, std::set<std::pair<uint32_t, uint32_t>>& checked) {
  char buf[256];
  const uint32_t tlas_flags = WGPT_HAS_SPHERES | WGPT_HAS_CUBES | WGPT_HAS_CYLINDERS | WGPT_HAS_TORI | WGPT_HAS_MESHES;
  if (s.n_mats == 0) return "materials: at least one material record is required";
  for (uint32_t i = 0; i < s.n_mats; ++i) {
    const wgpt_material& m = s.mats[i];
    const int32_t idx[6] = {m.emissive_idx, m.albedo_idx, m.normal_idx, m.height_idx, m.roughness_idx, m.metallic_idx};
    for (int32_t t : idx)
      if (t >= 0 && (uint32_t)t >= s.tex_layers) {
        snprintf(buf, sizeof buf, "materials[%u]: texture index %d beyond the %u layers of the texture array", i, t,
                 s.tex_layers);
        return buf;
      }
  }
  auto mat_ok = [&](int32_t m) { return m >= -1 && m < (int32_t)s.n_mats; };
  auto blas_ok = [&](uint32_t node_offset, uint32_t tri_offset, const char* what) -> std::string {
    if (checked.count({node_offset, tri_offset})) return "";
    std::string e = check_tree(s.bvh, s.n_bvh, node_offset, node_offset, tri_offset, s.n_tris, what);
    if (e.empty()) checked.insert({node_offset, tri_offset});
    return e;
  };
  if (flags & tlas_flags) {
    if (s.n_tlas == 0) return "tlas: empty while object flags are set";
    std::string e = check_tree(s.tlas, s.n_tlas, 0, 0, 0, s.n_objs, "tlas");
    if (!e.empty()) return e;
    for (uint32_t i = 0; i < s.n_objs; ++i) {
      const wgpt_object& o = s.objs[i];
      if (!mat_ok(o.material_idx)) { snprintf(buf, sizeof buf, "objects[%u]: material %d out of range", i, o.material_idx); return buf; }
      if ((flags & WGPT_HAS_LIGHTS) && o.light_idx >= (int32_t)s.n_lights) {
        snprintf(buf, sizeof buf, "objects[%u]: light %d out of range", i, o.light_idx); return buf;
      }
      if (o.object_type == 0 && (flags & WGPT_HAS_MESHES)) {
        uint32_t no, to;
        memcpy(&no, &o.param0, 4); memcpy(&to, &o.param1, 4);
        e = blas_ok(no, to, "bvh");
        if (!e.empty()) { snprintf(buf, sizeof buf, "objects[%u]: ", i); return buf + e; }
        if (o.material_idx < 0) { snprintf(buf, sizeof buf, "objects[%u]: mesh without material", i); return buf; }
      }
    }
  }
  if (flags & WGPT_HAS_LIST_MESHES) {
    for (uint32_t i = 0; i < s.n_meshes; ++i) {
      wgpt_mesh_instance mi;
      memcpy(&mi, s.meshes + (size_t)i * WGPT_STRIDE_MESH_READ, sizeof mi);
      if (!mat_ok(mi.material_idx)) { snprintf(buf, sizeof buf, "meshes[%u] (80-byte read stride): material %d out of range", i, mi.material_idx); return buf; }
      std::string e = blas_ok(mi.node_offset, mi.tri_offset, "bvh");
      if (!e.empty()) { snprintf(buf, sizeof buf, "meshes[%u] (80-byte read stride): ", i); return buf + e; }
    }
  }
  if (flags & WGPT_HAS_PLANES) {
    for (uint32_t i = 0; i < s.n_planes; ++i)
      if (!mat_ok(s.planes[i].material_idx)) { snprintf(buf, sizeof buf, "planes[%u]: material out of range", i); return buf; }
  }
  if (flags & WGPT_HAS_LIGHTS) {
    for (uint32_t i = 0; i < s.n_lights; ++i) {
      int32_t oi = s.lights[i].obj_idx;
      if (oi >= (int32_t)s.n_objs) { snprintf(buf, sizeof buf, "lights[%u]: object %d out of range", i, oi); return buf; }
      if (oi >= 0 && s.objs[oi].material_idx < 0) { snprintf(buf, sizeof buf, "lights[%u]: object without material", i); return buf; }
    }
  }
  return "";
}

// Child-pair record of inner node i: both children's boxes; .w of each child's max is the
// absolute node index of an inner child or the reference's relative first item of a leaf.
void fill_pairs(const wgpt_bvh_node* nodes, uint32_t root, uint32_t base, float* pairs, std::vector<uint8_t>& done) {
  std::vector<uint32_t> st;
  st.push_back(root);
  while (!st.empty()) {
    uint32_t i = st.back();
    st.pop_back();
    const wgpt_bvh_node& nd = nodes[i];
    if (nd.num_triangles > 0u || done[i]) continue;
    done[i] = 1;
    uint32_t li = i + 1, ri = base + nd.next;
    const wgpt_bvh_node* ch[2] = {&nodes[li], &nodes[ri]};
    uint32_t abs_idx[2] = {li, ri};
    float* out = pairs + (size_t)i * 16;
    for (int c = 0; c < 2; ++c) {
      const wgpt_bvh_node& x = *ch[c];
      uint32_t w = x.num_triangles > 0u ? x.next : abs_idx[c];
      memcpy(out + c * 8 + 0, x.aabb_min, 12);
      memcpy(out + c * 8 + 3, &x.num_triangles, 4);
      memcpy(out + c * 8 + 4, x.aabb_max, 12);
      memcpy(out + c * 8 + 7, &w, 4);
      if (x.num_triangles == 0u) st.push_back(abs_idx[c]);
    }
  }
}

// Quad records for the any-hit (shadow) traversal over a 4-wide view of the same tree: for an
// inner node i, up to four entries -- each child that is a leaf, and both children of each child
// that is inner -- as (box min, count) (box max, item) float pairs, count 0xFFFFFFFF marking an
// empty entry, the items as in the pair records.  32 floats per node, indexed like the pairs by
// the reference node index; only nodes reached as quad roots are filled.  Boxes are copied bit
// for bit.
void fill_quads(const wgpt_bvh_node* nodes, uint32_t root, uint32_t base, float* quads, std::vector<uint8_t>& done) {
  std::vector<uint32_t> st;
  st.push_back(root);
  while (!st.empty()) {
    const uint32_t i = st.back();
    st.pop_back();
    const wgpt_bvh_node& nd = nodes[i];
    if (nd.num_triangles > 0u || done[i]) continue;
    done[i] = 1;
    float* out = quads + (size_t)i * 32;
    int k = 0;
    auto put = [&](uint32_t idx) {
      const wgpt_bvh_node& x = nodes[idx];
      const uint32_t w = x.num_triangles > 0u ? x.next : idx;
      memcpy(out + k * 8 + 0, x.aabb_min, 12);
      memcpy(out + k * 8 + 3, &x.num_triangles, 4);
      memcpy(out + k * 8 + 4, x.aabb_max, 12);
      memcpy(out + k * 8 + 7, &w, 4);
      if (x.num_triangles == 0u) st.push_back(idx);
      ++k;
    };
    const uint32_t ch[2] = {i + 1, base + nd.next};
    for (uint32_t c : ch) {
      if (nodes[c].num_triangles > 0u) {
        put(c);
      } else {
        put(c + 1);
        put(base + nodes[c].next);
      }
    }
    const uint32_t empty = 0xffffffffu;
    for (; k < 4; ++k) memcpy(out + k * 8 + 3, &empty, 4);
  }
}

// Levels below the root of the deepest leaf (trees validated on upload).
uint32_t tree_depth(const wgpt_bvh_node* nodes, uint32_t root, uint32_t base) {
  uint32_t best = 0;
  std::vector<std::pair<uint32_t, uint32_t>> st;
  st.push_back({root, 0u});
  while (!st.empty()) {
    auto [i, d] = st.back();
    st.pop_back();
    best = std::max(best, d);
    const wgpt_bvh_node& nd = nodes[i];
    if (nd.num_triangles == 0u) {
      st.push_back({i + 1, d + 1});
      st.push_back({base + nd.next, d + 1});
    }
  }
  return best;
}

// The 4-wide shadow walk keeps at most 3 pending entries per visited level pair of each tree, plus
// the instance's sentinel, a leaf remainder and the entry being expanded: it fits the 132-entry
// traversal stack for TLAS + BLAS depths up to about 80 (the two-wide walk's bound is 62 each).
bool wide_walk_fits(uint32_t tlas_depth, uint32_t blas_depth) {
  return 3u * ((tlas_depth + 1u) / 2u + (blas_depth + 1u) / 2u) + 4u <= 132u;
}

// The pair records (16 floats per node) followed by the quad records (32 floats per node).
int upload_pairs(wgpt_ctx* ctx, const HostScene& hs, uint32_t flags) {
  const uint32_t tlas_flags = WGPT_HAS_SPHERES | WGPT_HAS_CUBES | WGPT_HAS_CYLINDERS | WGPT_HAS_TORI | WGPT_HAS_MESHES;
  const size_t nt = std::max(1u, hs.n_tlas), nb = std::max(1u, hs.n_bvh);
  std::vector<float> pt(nt * 48, 0.0f), pb(nb * 48, 0.0f);
  if ((flags & tlas_flags) && hs.n_tlas) {
    std::vector<uint8_t> done(hs.n_tlas, 0);
    fill_pairs(hs.tlas, 0, 0, pt.data(), done);
    std::fill(done.begin(), done.end(), 0);
    fill_quads(hs.tlas, 0, 0, pt.data() + nt * 16, done);
    ctx->tlas_depth = tree_depth(hs.tlas, 0, 0);
  } else {
    ctx->tlas_depth = 0;
  }
  std::vector<uint8_t> done(std::max(1u, hs.n_bvh), 0);
  std::set<uint32_t> roots;
  if (flags & WGPT_HAS_MESHES)
    for (uint32_t i = 0; i < hs.n_objs; ++i)
      if (hs.objs[i].object_type == 0) { uint32_t no; memcpy(&no, &hs.objs[i].param0, 4); roots.insert(no); }
  if (flags & WGPT_HAS_LIST_MESHES)
    for (uint32_t i = 0; i < hs.n_meshes; ++i) {
      wgpt_mesh_instance mi;
      memcpy(&mi, hs.meshes + (size_t)i * WGPT_STRIDE_MESH_READ, sizeof mi);
      roots.insert(mi.node_offset);
    }
  for (uint32_t r : roots) fill_pairs(hs.bvh, r, r, pb.data(), done);
  std::fill(done.begin(), done.end(), 0);
  for (uint32_t r : roots) fill_quads(hs.bvh, r, r, pb.data() + nb * 16, done);
  ctx->blas_depth = 0;
  for (uint32_t r : roots) ctx->blas_depth = std::max(ctx->blas_depth, tree_depth(hs.bvh, r, r));
  void** dst[2] = {&ctx->d_pairs_tlas, &ctx->d_pairs_bvh};
  std::vector<float>* src[2] = {&pt, &pb};
  for (int k = 0; k < 2; ++k) {
    size_t bytes = src[k]->size() * sizeof(float);
    if (bytes > ctx->pairs_cap[k]) {
      dfree(*dst[k]);
      ctx->pairs_cap[k] = 0;
      CK(cudaMalloc(dst[k], bytes), "cudaMalloc node pairs");
      ctx->pairs_cap[k] = bytes;
    }
    CK(cudaMemcpy(*dst[k], src[k]->data(), bytes, cudaMemcpyHostToDevice), "upload node pairs");
  }
  return WGPT_OK;
}

int upload_buffers(wgpt_ctx* ctx, const wgpt_scene_desc* d, bool in_place_only) {
  const wgpt_buffer* src[9] = {&d->materials, &d->objects, &d->tlas, &d->meshes, &d->bvh,
                               &d->triangles, &d->planes, &d->lights, &d->sky_cdf};
  size_t sky_bytes = (size_t)d->sky_width * d->sky_height * 8;
  const size_t tex_bytes = d->textures_rgba8 ? (size_t)d->tex_width * d->tex_height * d->tex_layers * 4 : 0;
  const size_t alias_bytes = d->sky_alias ? (size_t)d->sky_width * d->sky_height * 8 : 0;
  for (int k = 0; k < 12; ++k) {
    const void* p = k < 9 ? src[k]->ptr : k == 9 ? (const void*)d->sky_rgba16f
                  : k == 10 ? (const void*)d->textures_rgba8 : d->sky_alias;
    size_t n = k < 9 ? src[k]->bytes : k == 9 ? sky_bytes : k == 10 ? tex_bytes : alias_bytes;
    if (n == 0 || p == nullptr) {
      // empty arrays are bound as one zeroed element (tracer.js:1789, makeBuf minimum sizes)
      n = kStride[k];
      p = nullptr;
    }
    if (in_place_only) {
      if (n > ctx->cap[k]) return fail(ctx, WGPT_E_REBUILD, std::string(kName[k]) + ": does not fit the existing buffer");
    } else if (n > ctx->cap[k]) {
      dfree(ctx->d_buf[k]);
      size_t alloc = (n + 255) & ~(size_t)255;
      CK(cudaMalloc(&ctx->d_buf[k], alloc), "cudaMalloc scene buffer");
      ctx->cap[k] = alloc;
    }
    if (p) {
      CK(cudaMemcpyAsync(ctx->d_buf[k], p, n, cudaMemcpyHostToDevice, ctx->stream), "upload scene buffer");
    } else {
      CK(cudaMemsetAsync(ctx->d_buf[k], 0, n, ctx->stream), "zero scene buffer");
    }
    ctx->bytes[k] = n;
  }
  // the sources are pageable host memory: the copies above have completed on return, but keep
  // the contract explicit for callers that free them right after.
  CK(cudaStreamSynchronize(ctx->stream), "scene upload");
  return WGPT_OK;
}

int check_desc(wgpt_ctx* ctx, const wgpt_scene_desc* d, HostScene& hs,
               std::set<std::pair<uint32_t, uint32_t>>* checked_out = nullptr) {
  if (!d) return fail(ctx, WGPT_E_INVALID, "scene descriptor is null");
  const wgpt_buffer* b[9] = {&d->materials, &d->objects, &d->tlas, &d->meshes, &d->bvh,
                             &d->triangles, &d->planes, &d->lights, &d->sky_cdf};
  for (int k = 0; k < 9; ++k) {
    if (b[k]->bytes && !b[k]->ptr) return fail(ctx, WGPT_E_INVALID, std::string(kName[k]) + ": null pointer with nonzero size");
    uint32_t stride = kStride[k];
    if (k != 3 && k != 8 && b[k]->bytes % stride != 0)
      return fail(ctx, WGPT_E_LAYOUT, std::string(kName[k]) + ": size is not a multiple of its record size");
  }
  if (d->bounce_limit < 0) return fail(ctx, WGPT_E_INVALID, "bounce_limit must be >= 0");
  if (d->feature_flags & ~0x7ffu) return fail(ctx, WGPT_E_INVALID, "unknown feature flag bits");
  if ((d->feature_flags & WGPT_HAS_SKYBOX) && (!d->sky_rgba16f || d->sky_width == 0 || d->sky_height == 0))
    return fail(ctx, WGPT_E_INVALID, "sky texture missing while HAS_SKYBOX is set");
  if (d->textures_rgba8 && (d->tex_width == 0 || d->tex_height == 0 || d->tex_layers == 0 ||
                            (uint64_t)d->tex_width * d->tex_height * d->tex_layers > (1ull << 30)))
    return fail(ctx, WGPT_E_INVALID, "texture array size must be nonzero and at most 2^30 texels");
  hs.tex_layers = d->textures_rgba8 ? d->tex_layers : 0u;
  if (d->sky_alias) {
    if (!d->sky_rgba16f || d->sky_width == 0 || d->sky_height == 0)
      return fail(ctx, WGPT_E_INVALID, "sky_alias given without a sky texture");
    const size_t na = (size_t)d->sky_width * d->sky_height;
    const uint32_t* a = (const uint32_t*)d->sky_alias;
    for (size_t i = 0; i < na; ++i) {
      float pr;
      memcpy(&pr, &a[2 * i], 4);
      if (!(pr >= 0.0f && pr <= 1.0f) || a[2 * i + 1] >= na)
        return fail(ctx, WGPT_E_LAYOUT, "sky_alias: entry " + std::to_string(i) + " has a probability outside [0, 1] or an alias out of range");
    }
  }
  auto cnt = [&](int k) { return (uint32_t)(b[k]->bytes / kStride[k]); };
  hs.mats = (const wgpt_material*)b[0]->ptr; hs.n_mats = cnt(0);
  hs.objs = (const wgpt_object*)b[1]->ptr; hs.n_objs = cnt(1);
  hs.tlas = (const wgpt_bvh_node*)b[2]->ptr; hs.n_tlas = cnt(2);
  hs.meshes = (const uint8_t*)b[3]->ptr; hs.n_meshes = cnt(3);
  hs.bvh = (const wgpt_bvh_node*)b[4]->ptr; hs.n_bvh = cnt(4);
  hs.tris = (const wgpt_triangle*)b[5]->ptr; hs.n_tris = cnt(5);
  hs.planes = (const wgpt_plane*)b[6]->ptr; hs.n_planes = cnt(6);
  hs.lights = (const wgpt_light*)b[7]->ptr; hs.n_lights = cnt(7);
  std::set<std::pair<uint32_t, uint32_t>> checked;
  std::string e = validate(hs, d->feature_flags, checked);
  if (!e.empty()) {
    if (e[0] == 'U') return fail(ctx, WGPT_E_UNSUPPORTED, e.substr(1));
    return fail(ctx, WGPT_E_LAYOUT, e);
  }
  if (checked_out) checked_out->swap(checked);
  return WGPT_OK;
}

// The wgpt::SCENE_* bits implied by a material buffer under the given feature flags.
uint32_t derived_flags(const wgpt_material* m, size_t n, uint32_t feature_flags) {
  uint32_t f = 0;
  const bool pom = (feature_flags & WGPT_HAS_HEIGHTMAPS) != 0u;
  for (size_t i = 0; i < n; ++i) {
    const bool height = pom && m[i].height_idx >= 0;
    if (m[i].emissive_idx >= 0 || m[i].albedo_idx >= 0 || m[i].normal_idx >= 0 || m[i].roughness_idx >= 0 ||
        m[i].metallic_idx >= 0 || height)
      f |= wgpt::SCENE_TEXTURED;
    if (m[i].albedo_idx >= 0) f |= wgpt::SCENE_ALPHA_SHADOWS;
    if (m[i].normal_idx >= 0 || height) f |= wgpt::SCENE_TANGENTS;
  }
  return f;
}

void fill_device_scene(wgpt_ctx* ctx, const wgpt_scene_desc* d) {
  auto cnt = [&](int k) { return (uint32_t)(ctx->bytes[k] / kStride[k]); };
  wgpt::DeviceScene& s = ctx->ds;
  s.mats = ctx->d_buf[0]; s.n_mats = cnt(0);
  s.objs = ctx->d_buf[1]; s.n_objs = cnt(1);
  s.tlas = ctx->d_buf[2]; s.n_tlas = cnt(2);
  s.meshes = ctx->d_buf[3]; s.n_meshes = d->meshes.bytes ? (uint32_t)(d->meshes.bytes / WGPT_STRIDE_MESH_READ) : 1u;
  s.bvh = ctx->d_buf[4]; s.n_bvh = cnt(4);
  s.tris = ctx->d_buf[5]; s.n_tris = cnt(5);
  s.planes = ctx->d_buf[6]; s.n_planes = cnt(6);
  s.lights = ctx->d_buf[7]; s.n_lights = cnt(7);
  s.cdf = ctx->d_buf[8]; s.n_cdf = cnt(8);
  s.sky = ctx->d_buf[9];
  s.sky_w = d->sky_rgba16f ? d->sky_width : 1u;
  s.sky_h = d->sky_rgba16f ? d->sky_height : 1u;
  s.tex = ctx->d_buf[10];
  s.tex_w = d->textures_rgba8 ? d->tex_width : 1u;
  s.tex_h = d->textures_rgba8 ? d->tex_height : 1u;
  s.tex_layers = d->textures_rgba8 ? d->tex_layers : 0u;
  s.alias = ctx->d_buf[11];
  ctx->has_alias = d->sky_alias != nullptr;
  s.bounce_limit = d->bounce_limit;
  const wgpt_material* m = (const wgpt_material*)d->materials.ptr;
  const size_t nm = d->materials.bytes / WGPT_STRIDE_MATERIAL;
  ctx->host_mats.assign(m, m + nm);
  s.flags = d->feature_flags | derived_flags(m, nm, d->feature_flags);
  if (ctx->has_alias && ctx->env_mode == WGPT_ENV_ALIAS) s.flags |= wgpt::SCENE_ENV_ALIAS;
  if (wide_walk_fits(ctx->tlas_depth, ctx->blas_depth)) s.flags |= wgpt::SCENE_WIDE_OK;
  const wgpt_light* lt = (const wgpt_light*)d->lights.ptr;
  ctx->light_objs.clear();
  for (size_t i = 0; i < d->lights.bytes / WGPT_STRIDE_LIGHT; ++i) ctx->light_objs.push_back(lt[i].obj_idx);
}

int check_section(wgpt_ctx* ctx, uint32_t sx, uint32_t sy, uint32_t sw, uint32_t sh) {
  if (ctx->w == 0) return fail(ctx, WGPT_E_STATE, "no image size: call wgpt_resize first");
  if (!ctx->has_params) return fail(ctx, WGPT_E_STATE, "no scene params: call wgpt_set_params first");
  // params.width/height may be smaller than the context (renderPreview renders a reduced image
  // into the canvas-sized buffers); the accumulation is indexed with params.width, the rgba8
  // image with the context width (the storage texture's row pitch).
  if (ctx->params.width == 0 || ctx->params.height == 0 || ctx->params.width > ctx->w || ctx->params.height > ctx->h)
    return fail(ctx, WGPT_E_INVALID, "params width/height must be nonzero and within the context size");
  if (sw == 0 || sh == 0 || (uint64_t)sx + sw > ctx->params.width || (uint64_t)sy + sh > ctx->params.height)
    return fail(ctx, WGPT_E_INVALID, "section outside the image");
  return WGPT_OK;
}

int check_env(wgpt_ctx* ctx, const wgpt_scene_params& p) {
  if ((ctx->ds.flags & WGPT_HAS_SKYBOX) && (ctx->ds.flags & WGPT_MIS_SKYBOX)) {
    if (p.sky_width == 0 || p.sky_height == 0) return fail(ctx, WGPT_E_INVALID, "params sky_width/sky_height are zero");
    uint64_t last = (uint64_t)p.sky_cdf_index + (uint64_t)(p.sky_height - 1) * (p.sky_width + 1) + p.sky_width - 1;
    if (p.sky_height > ctx->ds.n_cdf || last >= ctx->ds.n_cdf)
      return fail(ctx, WGPT_E_LAYOUT, "sky_cdf is smaller than the params' sky_width/sky_height/sky_cdf_index imply");
  }
  return WGPT_OK;
}

}  // namespace

bool wgpt::ctx_images(wgpt_ctx* ctx, int view, wgpt::CtxImages* out) {
  if (!ctx || !out) return false;
  out->device = ctx->device;
  out->stream = ctx->stream;
  if (view < 0) {
    if (ctx->w == 0 || !ctx->accum) return false;
    out->w = ctx->w;
    out->h = ctx->h;
    out->accum = ctx->accum;
    out->gbuf = ctx->gbuf;
    out->out = ctx->out;
    return true;
  }
  if ((size_t)view >= ctx->views.size()) return false;
  const auto& v = ctx->views[(size_t)view];
  out->w = v.w;
  out->h = v.h;
  out->accum = v.accum;
  out->gbuf = v.gbuf;
  out->out = v.out;
  return true;
}

extern "C" {

int wgpt_abi_version(void) { return WGPT_ABI_VERSION; }

int wgpt_create(int device, wgpt_ctx** out) {
  if (!out) return WGPT_E_INVALID;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return WGPT_E_CUDA;
  if (device < 0 || device >= n) return WGPT_E_INVALID;
  wgpt_ctx* ctx = new wgpt_ctx();
  ctx->device = device;
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc(&ctx->d_status, sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMemset(ctx->d_status, 0, sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMalloc(&ctx->d_counters, 128 * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMemset(ctx->d_counters, 0, 128 * sizeof(unsigned long long));
  if (e != cudaSuccess) {
    wgpt_destroy(ctx);
    return WGPT_E_CUDA;
  }
  *out = ctx;
  return WGPT_OK;
}

int wgpt_destroy(wgpt_ctx* ctx) {
  if (!ctx) return WGPT_E_INVALID;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  for (int k = 0; k < 12; ++k) dfree(ctx->d_buf[k]);
  dfree_t(ctx->accum); dfree_t(ctx->out); dfree_t(ctx->gbuf);
  dfree_t(ctx->dn_a); dfree_t(ctx->dn_b); dfree_t(ctx->dn_guide); dfree_t(ctx->dn_comp);
  dfree_t(ctx->canvas); dfree_t(ctx->d_status); dfree_t(ctx->d_counters); wgpt::wf_engine_destroy(ctx->wf);
  ctx->wf = nullptr;
  dfree_t(ctx->acc64);
  dfree(ctx->d_pairs_tlas); dfree(ctx->d_pairs_bvh);
  for (auto& v : ctx->views) { dfree_t(v.accum); dfree_t(v.out); dfree_t(v.gbuf); }
  if (ctx->timer) {
    if (ctx->timer->ready)
      for (int i = 0; i < wgpt::StageTimer::kMaxEvents; ++i) cudaEventDestroy(ctx->timer->ev[i]);
    delete ctx->timer;
  }
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return WGPT_OK;
}

const char* wgpt_last_error(const wgpt_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

void* wgpt_stream(wgpt_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int wgpt_validate_scene(const wgpt_scene_desc* desc, char* msg, size_t msg_len) {
  wgpt_ctx tmp;   // host-only: no device state is touched
  HostScene hs;
  int rc = check_desc(&tmp, desc, hs);
  if (msg && msg_len) {
    snprintf(msg, msg_len, "%s", tmp.err.c_str());
  }
  return rc;
}

int wgpt_upload_scene(wgpt_ctx* ctx, const wgpt_scene_desc* desc) {
  if (!ctx) return WGPT_E_INVALID;
  CK(wgpt::select_device(ctx->device), "cudaSetDevice");
  HostScene hs;
  std::set<std::pair<uint32_t, uint32_t>> checked;
  int rc = check_desc(ctx, desc, hs, &checked);
  if (rc) return rc;
  CK(cudaStreamSynchronize(ctx->stream), "drain before upload");
  rc = upload_buffers(ctx, desc, false);
  if (rc) return rc;
  rc = upload_pairs(ctx, hs, desc->feature_flags);
  if (rc) return rc;
  fill_device_scene(ctx, desc);
  ctx->blas_checked.swap(checked);
  ctx->has_scene = true;
  return WGPT_OK;
}

int wgpt_update_scene(wgpt_ctx* ctx, const wgpt_scene_desc* desc) {
  if (!ctx) return WGPT_E_INVALID;
  if (!ctx->has_scene) return fail(ctx, WGPT_E_STATE, "no scene uploaded");
  CK(wgpt::select_device(ctx->device), "cudaSetDevice");
  if (desc && (desc->feature_flags != (ctx->ds.flags & 0x7ffu) || desc->bounce_limit != ctx->ds.bounce_limit))
    return fail(ctx, WGPT_E_REBUILD, "pipeline constants changed: full upload required");
  HostScene hs;
  std::set<std::pair<uint32_t, uint32_t>> checked;
  int rc = check_desc(ctx, desc, hs, &checked);
  if (rc) return rc;
  CK(cudaStreamSynchronize(ctx->stream), "drain before update");
  rc = upload_buffers(ctx, desc, true);
  if (rc) return rc;
  rc = upload_pairs(ctx, hs, desc->feature_flags);
  if (rc) return rc;
  fill_device_scene(ctx, desc);
  ctx->blas_checked.swap(checked);
  return WGPT_OK;
}

// updateObjects fast path (tracer.js:2132-2164).  Only the five buffers the reference rewrites
// are read from the descriptor; each is written at offset 0 of the resident buffer, whose length
// (and so every arrayLength-bounded loop) stays what the upload set, like queue.writeBuffer into
// the existing GPU buffer.  The new records are validated against the resident scene: indices
// within the resident buffers, the TLAS self-contained, mesh instances only of BLAS offsets
// validated on upload.  Lights, BLAS, triangles, the sky and textures are not touched.
int wgpt_update_objects(wgpt_ctx* ctx, const wgpt_scene_desc* desc) {
  if (!ctx) return WGPT_E_INVALID;
  if (!desc) return fail(ctx, WGPT_E_INVALID, "scene descriptor is null");
  if (!ctx->has_scene) return fail(ctx, WGPT_E_STATE, "no scene uploaded");
  CK(wgpt::select_device(ctx->device), "cudaSetDevice");
  const uint32_t flags = desc->feature_flags;
  if (flags != (ctx->ds.flags & 0x7ffu)) return fail(ctx, WGPT_E_REBUILD, "pipeline constants changed: full upload required");
  const int ks[5] = {1, 2, 6, 3, 0};   // objects, tlas, planes, meshes, materials (tracer.js:2151-2155)
  const wgpt_buffer* b[5] = {&desc->objects, &desc->tlas, &desc->planes, &desc->meshes, &desc->materials};
  for (int j = 0; j < 5; ++j) {
    const int k = ks[j];
    if (b[j]->bytes && !b[j]->ptr) return fail(ctx, WGPT_E_INVALID, std::string(kName[k]) + ": null pointer with nonzero size");
    if (k != 3 && b[j]->bytes % kStride[k] != 0)
      return fail(ctx, WGPT_E_LAYOUT, std::string(kName[k]) + ": size is not a multiple of its record size");
    if (b[j]->bytes > ctx->bytes[k])
      return fail(ctx, WGPT_E_REBUILD, std::string(kName[k]) + ": does not fit the uploaded buffer");
  }
  const uint32_t n_mats = (uint32_t)(ctx->bytes[0] / WGPT_STRIDE_MATERIAL);
  const uint32_t n_objs = (uint32_t)(ctx->bytes[1] / WGPT_STRIDE_OBJECT);
  const uint32_t n_lights = (uint32_t)(ctx->bytes[7] / WGPT_STRIDE_LIGHT);
  const wgpt_material* mats = (const wgpt_material*)desc->materials.ptr;
  const wgpt_object* objs = (const wgpt_object*)desc->objects.ptr;
  const wgpt_bvh_node* tlas = (const wgpt_bvh_node*)desc->tlas.ptr;
  const wgpt_plane* planes = (const wgpt_plane*)desc->planes.ptr;
  const uint32_t nm = (uint32_t)(desc->materials.bytes / WGPT_STRIDE_MATERIAL);
  const uint32_t no = (uint32_t)(desc->objects.bytes / WGPT_STRIDE_OBJECT);
  const uint32_t nt = (uint32_t)(desc->tlas.bytes / WGPT_STRIDE_NODE);
  const uint32_t np = (uint32_t)(desc->planes.bytes / WGPT_STRIDE_PLANE);
  const uint32_t nl = (uint32_t)(desc->meshes.bytes / WGPT_STRIDE_MESH_READ);
  char buf[256];
  for (uint32_t i = 0; i < nm; ++i) {
    const int32_t idx[6] = {mats[i].emissive_idx, mats[i].albedo_idx, mats[i].normal_idx, mats[i].height_idx,
                            mats[i].roughness_idx, mats[i].metallic_idx};
    for (int32_t t : idx)
      if (t >= 0 && (uint32_t)t >= ctx->ds.tex_layers) {
        snprintf(buf, sizeof buf, "materials[%u]: texture index %d beyond the %u layers of the texture array", i, t,
                 ctx->ds.tex_layers);
        return fail(ctx, WGPT_E_LAYOUT, buf);
      }
  }
  auto mat_ok = [&](int32_t m) { return m >= -1 && m < (int32_t)n_mats; };
  const uint32_t tlas_flags = WGPT_HAS_SPHERES | WGPT_HAS_CUBES | WGPT_HAS_CYLINDERS | WGPT_HAS_TORI | WGPT_HAS_MESHES;
  if ((flags & tlas_flags) && nt > 0) {
    std::string e = check_tree(tlas, nt, 0, 0, 0, n_objs, "tlas");
    if (!e.empty()) return fail(ctx, WGPT_E_LAYOUT, e);
  }
  for (uint32_t i = 0; i < no; ++i) {
    const wgpt_object& o = objs[i];
    if (!mat_ok(o.material_idx)) { snprintf(buf, sizeof buf, "objects[%u]: material %d out of range", i, o.material_idx); return fail(ctx, WGPT_E_LAYOUT, buf); }
    if ((flags & WGPT_HAS_LIGHTS) && o.light_idx >= (int32_t)n_lights) {
      snprintf(buf, sizeof buf, "objects[%u]: light %d out of range", i, o.light_idx);
      return fail(ctx, WGPT_E_LAYOUT, buf);
    }
    if (o.object_type == 0 && (flags & WGPT_HAS_MESHES)) {
      uint32_t nof, tof;
      memcpy(&nof, &o.param0, 4); memcpy(&tof, &o.param1, 4);
      if (!ctx->blas_checked.count({nof, tof})) {
        snprintf(buf, sizeof buf, "objects[%u]: mesh instance of a BLAS that is not resident", i);
        return fail(ctx, WGPT_E_REBUILD, buf);
      }
      if (o.material_idx < 0) { snprintf(buf, sizeof buf, "objects[%u]: mesh without material", i); return fail(ctx, WGPT_E_LAYOUT, buf); }
    }
  }
  if (flags & WGPT_HAS_LIST_MESHES) {
    for (uint32_t i = 0; i < nl; ++i) {
      wgpt_mesh_instance mi;
      memcpy(&mi, (const uint8_t*)desc->meshes.ptr + (size_t)i * WGPT_STRIDE_MESH_READ, sizeof mi);
      if (!mat_ok(mi.material_idx)) {
        snprintf(buf, sizeof buf, "meshes[%u] (80-byte read stride): material %d out of range", i, mi.material_idx);
        return fail(ctx, WGPT_E_LAYOUT, buf);
      }
      if (!ctx->blas_checked.count({mi.node_offset, mi.tri_offset})) {
        snprintf(buf, sizeof buf, "meshes[%u] (80-byte read stride): BLAS not resident", i);
        return fail(ctx, WGPT_E_REBUILD, buf);
      }
    }
  }
  for (uint32_t i = 0; i < np; ++i)
    if (!mat_ok(planes[i].material_idx)) { snprintf(buf, sizeof buf, "planes[%u]: material out of range", i); return fail(ctx, WGPT_E_LAYOUT, buf); }
  // the resident light records keep their object indices: those objects need a material
  for (size_t i = 0; i < ctx->light_objs.size(); ++i) {
    const int32_t oi = ctx->light_objs[i];
    if (oi >= 0 && (uint32_t)oi < no && objs[oi].material_idx < 0) {
      snprintf(buf, sizeof buf, "lights[%zu]: object %d without material", i, oi);
      return fail(ctx, WGPT_E_LAYOUT, buf);
    }
  }
  // the writes (renders already queued read the old data first)
  CK(cudaStreamSynchronize(ctx->stream), "drain before update");
  for (int j = 0; j < 5; ++j)
    if (b[j]->bytes) CK(cudaMemcpyAsync(ctx->d_buf[ks[j]], b[j]->ptr, b[j]->bytes, cudaMemcpyHostToDevice, ctx->stream), "update buffer");
  if (nt > 0 && (flags & tlas_flags)) {
    std::vector<float> pt((size_t)nt * 16, 0.0f), qt((size_t)nt * 32, 0.0f);
    std::vector<uint8_t> done(nt, 0);
    fill_pairs(tlas, 0, 0, pt.data(), done);
    std::fill(done.begin(), done.end(), 0);
    fill_quads(tlas, 0, 0, qt.data(), done);
    CK(cudaMemcpyAsync(ctx->d_pairs_tlas, pt.data(), pt.size() * sizeof(float), cudaMemcpyHostToDevice, ctx->stream),
       "update node pairs");
    // the quad records follow the pair records of the uploaded node count (the buffer keeps it)
    float* quads = (float*)ctx->d_pairs_tlas + (size_t)std::max(1u, ctx->ds.n_tlas) * 16;
    CK(cudaMemcpyAsync(quads, qt.data(), qt.size() * sizeof(float), cudaMemcpyHostToDevice, ctx->stream),
       "update node quads");
    ctx->tlas_depth = tree_depth(tlas, 0, 0);
    if (wide_walk_fits(ctx->tlas_depth, ctx->blas_depth)) ctx->ds.flags |= wgpt::SCENE_WIDE_OK;
    else ctx->ds.flags &= ~wgpt::SCENE_WIDE_OK;
    CK(cudaStreamSynchronize(ctx->stream), "update");
  } else {
    CK(cudaStreamSynchronize(ctx->stream), "update");
  }
  if (nm) {
    std::copy(mats, mats + nm, ctx->host_mats.begin());
    ctx->ds.flags = flags | derived_flags(ctx->host_mats.data(), ctx->host_mats.size(), flags);
    if (ctx->has_alias && ctx->env_mode == WGPT_ENV_ALIAS) ctx->ds.flags |= wgpt::SCENE_ENV_ALIAS;
    if (wide_walk_fits(ctx->tlas_depth, ctx->blas_depth)) ctx->ds.flags |= wgpt::SCENE_WIDE_OK;
  }
  return WGPT_OK;
}

int wgpt_resize(wgpt_ctx* ctx, uint32_t width, uint32_t height, int want_gbuf) {
  if (!ctx) return WGPT_E_INVALID;
  if (width == 0 || height == 0 || (uint64_t)width * height > (1ull << 28)) return fail(ctx, WGPT_E_INVALID, "bad image size");
  CK(wgpt::select_device(ctx->device), "cudaSetDevice");
  CK(cudaStreamSynchronize(ctx->stream), "drain before resize");
  size_t npix = (size_t)width * height;
  bool same = width == ctx->w && height == ctx->h;
  const bool had_f64 = ctx->acc64 != nullptr;
  if (!same) {
    dfree_t(ctx->acc64);
    dfree_t(ctx->accum); dfree_t(ctx->out); dfree_t(ctx->gbuf);
    dfree_t(ctx->dn_a); dfree_t(ctx->dn_b); dfree_t(ctx->dn_guide); dfree_t(ctx->dn_comp);
    ctx->dn_final = nullptr;
    ctx->w = ctx->h = 0;
    CK(cudaMalloc(&ctx->accum, npix * 16), "cudaMalloc accum");
    CK(cudaMalloc(&ctx->out, npix * 4), "cudaMalloc output");
  }
  if (want_gbuf && !ctx->gbuf) CK(cudaMalloc(&ctx->gbuf, npix * 48), "cudaMalloc gbuffer");
  CK(cudaMemsetAsync(ctx->accum, 0, npix * 16, ctx->stream), "clear accum");
  CK(cudaMemsetAsync(ctx->out, 0, npix * 4, ctx->stream), "clear output");
  if (want_gbuf) CK(cudaMemsetAsync(ctx->gbuf, 0, npix * 48, ctx->stream), "clear gbuffer");
  if (had_f64 && !ctx->acc64) CK(cudaMalloc(&ctx->acc64, npix * 64), "cudaMalloc FP64 accumulation");
  if (ctx->acc64) CK(cudaMemsetAsync(ctx->acc64, 0, npix * 64, ctx->stream), "clear FP64 accumulation");
  ctx->w = width; ctx->h = height;
  CK(cudaStreamSynchronize(ctx->stream), "resize");
  return WGPT_OK;
}

int wgpt_set_params(wgpt_ctx* ctx, const void* p) {
  if (!ctx || !p) return WGPT_E_INVALID;
  memcpy(&ctx->params, p, sizeof(wgpt_scene_params));
  ctx->has_params = true;
  return WGPT_OK;
}

int wgpt_render(wgpt_ctx* ctx, uint32_t first_frame, uint32_t reps, uint32_t sx, uint32_t sy, uint32_t sw, uint32_t sh) {
  if (!ctx) return WGPT_E_INVALID;
  if (!ctx->has_scene) return fail(ctx, WGPT_E_STATE, "no scene uploaded");
  int rc = check_section(ctx, sx, sy, sw, sh);
  if (rc) return rc;
  rc = check_env(ctx, ctx->params);
  if (rc) return rc;
  if (reps == 0) return WGPT_OK;
  CK(wgpt::select_device(ctx->device), "cudaSetDevice");
  unsigned long long* cnt = ctx->counting ? ctx->d_counters : nullptr;
  wgpt::StageTimer* tm = ctx->timing ? ctx->timer : nullptr;
  if (ctx->mode == WGPT_MODE_MEGAKERNEL) {
    if (ctx->acc64) return fail(ctx, WGPT_E_UNSUPPORTED, "FP64 accumulation needs the wavefront mode");
    if (tm) tm->begin(0, ctx->stream);
    CK(wgpt::launch_render(ctx->ds, ctx->params, first_frame, reps, sx, sy, sw, sh, ctx->accum, ctx->out, ctx->w,
                           ctx->d_status, cnt, ctx->stream),
       "render launch");
    if (tm) tm->end(0, ctx->stream);
    return WGPT_OK;
  }
  if (!ctx->wf) ctx->wf = wgpt::wf_engine_create();
  wgpt::WfJobView v;
  v.q = ctx->params;
  v.sx = sx; v.sy = sy; v.sw = sw; v.sh = sh;
  v.first_frame = first_frame;
  v.spp = reps;
  v.accum = ctx->accum;
  v.out = ctx->out;
  v.out_pitch = ctx->w;
  v.acc64 = ctx->acc64;
  CK(wgpt::wf_render(ctx->wf, ctx->ds, ctx->d_pairs_tlas, ctx->d_pairs_bvh, &v, 1, ctx->d_status, cnt, ctx->stream,
                     tm),
     "wavefront render");
  return WGPT_OK;
}

int wgpt_render_gbuffer(wgpt_ctx* ctx, uint32_t sx, uint32_t sy, uint32_t sw, uint32_t sh) {
  if (!ctx) return WGPT_E_INVALID;
  if (!ctx->has_scene) return fail(ctx, WGPT_E_STATE, "no scene uploaded");
  int rc = check_section(ctx, sx, sy, sw, sh);
  if (rc) return rc;
  if (!ctx->gbuf) return fail(ctx, WGPT_E_STATE, "no G-buffer: resize with want_gbuf");
  CK(wgpt::select_device(ctx->device), "cudaSetDevice");
  CK(wgpt::launch_gbuffer(ctx->ds, ctx->params, sx, sy, sw, sh, ctx->gbuf, ctx->out, ctx->w, ctx->d_status,
                          ctx->stream),
     "gbuffer launch");
  return WGPT_OK;
}

int wgpt_denoise(wgpt_ctx* ctx, const void* uniforms, const uint32_t* steps, uint32_t passes) {
  if (!ctx || !uniforms || (passes && !steps)) return WGPT_E_INVALID;
  if (ctx->w == 0) return fail(ctx, WGPT_E_STATE, "no image size");
  if (!ctx->gbuf) return fail(ctx, WGPT_E_STATE, "no G-buffer: resize with want_gbuf and render it");
  wgpt_denoise_uniforms u;
  memcpy(&u, uniforms, sizeof u);
  if (u.width != ctx->w || u.height != ctx->h) return fail(ctx, WGPT_E_INVALID, "uniform width/height differ from the context size");
  if (passes > 64) return fail(ctx, WGPT_E_INVALID, "more than 64 passes");
  for (uint32_t i = 0; i < passes; ++i)
    if (steps[i] == 0 || steps[i] > (1u << 20)) return fail(ctx, WGPT_E_INVALID, "step width out of range");
  CK(wgpt::select_device(ctx->device), "cudaSetDevice");
  size_t npix = (size_t)ctx->w * ctx->h;
  if (!ctx->dn_a) {
    CK(cudaMalloc(&ctx->dn_a, npix * 16), "cudaMalloc denoise A");
    CK(cudaMalloc(&ctx->dn_b, npix * 16), "cudaMalloc denoise B");
    CK(cudaMalloc(&ctx->dn_guide, npix * 48), "cudaMalloc denoise guide");
    CK(cudaMalloc(&ctx->dn_comp, npix * 16), "cudaMalloc denoise composite");
  }
  CK(wgpt::launch_denoise(ctx->accum, ctx->gbuf, u, steps, passes, ctx->dn_a, ctx->dn_b, ctx->dn_guide, ctx->dn_comp,
                          ctx->out, &ctx->dn_final, ctx->stream, ctx->dn_mode == WGPT_DENOISE_FAST),
     "denoise launch");
  return WGPT_OK;
}

int wgpt_set_denoise_mode(wgpt_ctx* ctx, int mode) {
  if (!ctx) return WGPT_E_INVALID;
  if (mode != WGPT_DENOISE_EXACT && mode != WGPT_DENOISE_FAST) return fail(ctx, WGPT_E_INVALID, "unknown denoise mode");
  ctx->dn_mode = mode;
  return WGPT_OK;
}

int wgpt_resample(wgpt_ctx* ctx, uint32_t dst_w, uint32_t dst_h, float rx, float ry) {
  if (!ctx) return WGPT_E_INVALID;
  if (ctx->w == 0) return fail(ctx, WGPT_E_STATE, "no image size");
  if (dst_w == 0 || dst_h == 0 || (uint64_t)dst_w * dst_h > (1ull << 28)) return fail(ctx, WGPT_E_INVALID, "bad canvas size");
  CK(wgpt::select_device(ctx->device), "cudaSetDevice");
  if (dst_w != ctx->cw || dst_h != ctx->ch) {
    CK(cudaStreamSynchronize(ctx->stream), "drain before canvas resize");
    dfree_t(ctx->canvas);
    CK(cudaMalloc(&ctx->canvas, (size_t)dst_w * dst_h * 4), "cudaMalloc canvas");
    ctx->cw = dst_w; ctx->ch = dst_h;
  }
  CK(wgpt::launch_resample(ctx->out, ctx->w, ctx->h, ctx->canvas, dst_w, dst_h, rx, ry, ctx->stream), "resample launch");
  return WGPT_OK;
}

static int read_status(wgpt_ctx* ctx) {
  uint32_t st = 0;
  CK(cudaMemcpy(&st, ctx->d_status, sizeof st, cudaMemcpyDeviceToHost), "status readback");
  if (st) {
    CK(cudaMemset(ctx->d_status, 0, sizeof st), "status reset");
    if (st & 2u) return fail(ctx, WGPT_E_DEVICE, "the wavefront loop reached its iteration bound with paths left");
    return fail(ctx, WGPT_E_DEVICE, "a kernel overflowed its traversal stack");
  }
  return WGPT_OK;
}

int wgpt_synchronize(wgpt_ctx* ctx) {
  if (!ctx) return WGPT_E_INVALID;
  CK(wgpt::select_device(ctx->device), "cudaSetDevice");
  CK(cudaStreamSynchronize(ctx->stream), "stream synchronize");
  return read_status(ctx);
}

// Host watchdog: polls the context's stream instead of blocking on it, and gives up after
// timeout_ms with WGPT_E_TIMEOUT (the queued work keeps running; a later call can wait again).
int wgpt_synchronize_timeout(wgpt_ctx* ctx, uint32_t timeout_ms) {
  if (!ctx) return WGPT_E_INVALID;
  CK(wgpt::select_device(ctx->device), "cudaSetDevice");
  const auto t0 = std::chrono::steady_clock::now();
  while (true) {
    cudaError_t q = cudaStreamQuery(ctx->stream);
    if (q == cudaSuccess) break;
    if (q != cudaErrorNotReady) {
      ctx->err = std::string("stream query: ") + cudaGetErrorString(q);
      return WGPT_E_CUDA;
    }
    const auto ms = std::chrono::duration_cast<std::chrono::milliseconds>(std::chrono::steady_clock::now() - t0).count();
    if ((uint64_t)ms >= timeout_ms) {
      ctx->err = "the context's work did not finish within " + std::to_string(timeout_ms) + " ms";
      return WGPT_E_TIMEOUT;
    }
    std::this_thread::sleep_for(std::chrono::microseconds(100));
  }
  return read_status(ctx);
}

static int readback(wgpt_ctx* ctx, void* dst, const void* src, size_t n, const char* what) {
  if (!ctx || !dst) return WGPT_E_INVALID;
  if (!src) return fail(ctx, WGPT_E_STATE, std::string(what) + ": nothing to read");
  int rc = wgpt_synchronize(ctx);
  if (rc) return rc;
  CK(cudaMemcpy(dst, src, n, cudaMemcpyDeviceToHost), what);
  return WGPT_OK;
}

int wgpt_read_accum(wgpt_ctx* ctx, float* dst) {
  if (!ctx) return WGPT_E_INVALID;
  return readback(ctx, dst, ctx->accum, (size_t)ctx->w * ctx->h * 16, "read accum");
}
int wgpt_read_output(wgpt_ctx* ctx, uint8_t* dst) {
  if (!ctx) return WGPT_E_INVALID;
  return readback(ctx, dst, ctx->out, (size_t)ctx->w * ctx->h * 4, "read output");
}
int wgpt_read_gbuffer(wgpt_ctx* ctx, void* dst) {
  if (!ctx) return WGPT_E_INVALID;
  return readback(ctx, dst, ctx->gbuf, (size_t)ctx->w * ctx->h * 48, "read gbuffer");
}
int wgpt_read_denoised(wgpt_ctx* ctx, float* filtered, float* composited) {
  if (!ctx) return WGPT_E_INVALID;
  size_t n = (size_t)ctx->w * ctx->h * 16;
  int rc = WGPT_OK;
  if (filtered) rc = readback(ctx, filtered, ctx->dn_final, n, "read denoised");
  if (!rc && composited) rc = readback(ctx, composited, ctx->dn_final ? ctx->dn_comp : nullptr, n, "read composited");
  return rc;
}
int wgpt_read_canvas(wgpt_ctx* ctx, uint8_t* dst, uint32_t dst_w, uint32_t dst_h) {
  if (!ctx) return WGPT_E_INVALID;
  if (dst_w != ctx->cw || dst_h != ctx->ch) return fail(ctx, WGPT_E_INVALID, "canvas size mismatch");
  return readback(ctx, dst, ctx->canvas, (size_t)dst_w * dst_h * 4, "read canvas");
}

int wgpt_write_accum(wgpt_ctx* ctx, const float* src) {
  if (!ctx || !src) return WGPT_E_INVALID;
  if (!ctx->accum) return fail(ctx, WGPT_E_STATE, "no image size");
  CK(wgpt::select_device(ctx->device), "cudaSetDevice");
  CK(cudaStreamSynchronize(ctx->stream), "drain");
  CK(cudaMemcpy(ctx->accum, src, (size_t)ctx->w * ctx->h * 16, cudaMemcpyHostToDevice), "write accum");
  return WGPT_OK;
}
int wgpt_write_gbuffer(wgpt_ctx* ctx, const void* src) {
  if (!ctx || !src) return WGPT_E_INVALID;
  if (!ctx->gbuf) return fail(ctx, WGPT_E_STATE, "no G-buffer");
  CK(wgpt::select_device(ctx->device), "cudaSetDevice");
  CK(cudaStreamSynchronize(ctx->stream), "drain");
  CK(cudaMemcpy(ctx->gbuf, src, (size_t)ctx->w * ctx->h * 48, cudaMemcpyHostToDevice), "write gbuffer");
  return WGPT_OK;
}

int wgpt_trace_rays(wgpt_ctx* ctx, const float* rays, uint32_t n, int32_t* o_idx, int32_t* m_idx, int32_t* prim,
                    float* t, float* normal) {
  if (!ctx || !rays || !o_idx || !m_idx || !prim || !t || !normal) return WGPT_E_INVALID;
  if (!ctx->has_scene) return fail(ctx, WGPT_E_STATE, "no scene uploaded");
  if (n == 0) return WGPT_OK;
  CK(wgpt::select_device(ctx->device), "cudaSetDevice");
  void* d = nullptr;
  size_t per = 6 * 4 + 4 + 4 + 4 + 4 + 12;
  CK(cudaMalloc(&d, (size_t)n * per), "cudaMalloc rays");
  float* d_rays = (float*)d;
  int32_t* d_o = (int32_t*)(d_rays + (size_t)n * 6);
  int32_t* d_m = d_o + n;
  int32_t* d_p = d_m + n;
  float* d_t = (float*)(d_p + n);
  float* d_n = d_t + n;
  cudaError_t e = cudaMemcpyAsync(d_rays, rays, (size_t)n * 24, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) e = wgpt::launch_trace_rays(ctx->ds, d_rays, n, d_o, d_m, d_p, d_t, d_n, ctx->d_status, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e == cudaSuccess) e = cudaMemcpy(o_idx, d_o, (size_t)n * 4, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(m_idx, d_m, (size_t)n * 4, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(prim, d_p, (size_t)n * 4, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(t, d_t, (size_t)n * 4, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(normal, d_n, (size_t)n * 12, cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "trace rays");
  return wgpt_synchronize(ctx);
}

int wgpt_sample_env(wgpt_ctx* ctx, const float* u2, uint32_t n, uint32_t* texel_xy, float* pdf) {
  if (!ctx || !u2 || !texel_xy || !pdf) return WGPT_E_INVALID;
  if (!ctx->has_scene) return fail(ctx, WGPT_E_STATE, "no scene uploaded");
  if (!ctx->has_params) return fail(ctx, WGPT_E_STATE, "no scene params: call wgpt_set_params first");
  if (!(ctx->ds.flags & WGPT_HAS_SKYBOX) || !(ctx->ds.flags & WGPT_MIS_SKYBOX))
    return fail(ctx, WGPT_E_STATE, "the uploaded scene has no importance-sampled sky");
  int rc = check_env(ctx, ctx->params);
  if (rc) return rc;
  if (n == 0) return WGPT_OK;
  if (n > (1u << 24)) return fail(ctx, WGPT_E_INVALID, "at most 2^24 samples per call");
  CK(wgpt::select_device(ctx->device), "cudaSetDevice");
  void* d = nullptr;
  // per sample: u (2 floats), texel (2 uint32), pdf (1 float)
  CK(cudaMalloc(&d, (size_t)n * 20), "cudaMalloc env samples");
  float* d_u = (float*)d;
  uint32_t* d_t = (uint32_t*)(d_u + (size_t)n * 2);
  float* d_p = (float*)(d_t + (size_t)n * 2);
  cudaError_t e = cudaMemcpyAsync(d_u, u2, (size_t)n * 8, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) e = wgpt::launch_sample_env(ctx->ds, ctx->params, d_u, n, d_t, d_p, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e == cudaSuccess) e = cudaMemcpy(texel_xy, d_t, (size_t)n * 8, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(pdf, d_p, (size_t)n * 4, cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "sample env");
  return WGPT_OK;
}

int wgpt_rng_stream(int device, uint32_t idx, uint32_t sample_number, uint32_t seed, uint32_t n, float* out) {
  if (!out || n == 0 || n > (1u << 20)) return WGPT_E_INVALID;
  if (wgpt::select_device(device) != cudaSuccess) return WGPT_E_CUDA;
  float* d = nullptr;
  if (cudaMalloc(&d, (size_t)n * 4) != cudaSuccess) return WGPT_E_NOMEM;
  cudaError_t e = wgpt::launch_rng_stream(idx, sample_number, seed, n, d, 0);
  if (e == cudaSuccess) e = cudaMemcpy(out, d, (size_t)n * 4, cudaMemcpyDeviceToHost);
  cudaFree(d);
  return e == cudaSuccess ? WGPT_OK : WGPT_E_CUDA;
}

int wgpt_set_render_mode(wgpt_ctx* ctx, int mode) {
  if (!ctx) return WGPT_E_INVALID;
  if (mode != WGPT_MODE_WAVEFRONT && mode != WGPT_MODE_MEGAKERNEL) return fail(ctx, WGPT_E_INVALID, "unknown render mode");
  ctx->mode = mode;
  return WGPT_OK;
}

int wgpt_set_views(wgpt_ctx* ctx, uint32_t n, const uint32_t* widths, const uint32_t* heights) {
  if (!ctx || (n && (!widths || !heights))) return WGPT_E_INVALID;
  if (n > 4096) return fail(ctx, WGPT_E_INVALID, "more than 4096 views");
  for (uint32_t i = 0; i < n; ++i)
    if (widths[i] == 0 || heights[i] == 0 || widths[i] > 16384 || heights[i] > 16384)
      return fail(ctx, WGPT_E_INVALID, "view size must be 1..16384 per side");
  CK(wgpt::select_device(ctx->device), "cudaSetDevice");
  CK(cudaStreamSynchronize(ctx->stream), "drain before view allocation");
  for (auto& v : ctx->views) { dfree_t(v.accum); dfree_t(v.out); dfree_t(v.gbuf); }
  ctx->views.clear();
  for (uint32_t i = 0; i < n; ++i) {
    wgpt_ctx::View v{widths[i], heights[i], nullptr, nullptr, nullptr};
    size_t np = (size_t)v.w * v.h;
    ctx->views.push_back(v);
    CK(cudaMalloc(&ctx->views.back().accum, np * 16), "cudaMalloc view accumulation");
    CK(cudaMalloc(&ctx->views.back().out, np * 4), "cudaMalloc view image");
    CK(cudaMemsetAsync(ctx->views.back().accum, 0, np * 16, ctx->stream), "clear view accumulation");
    CK(cudaMemsetAsync(ctx->views.back().out, 0, np * 4, ctx->stream), "clear view image");
  }
  return WGPT_OK;
}

int wgpt_render_views(wgpt_ctx* ctx, const void* params_112n, const uint32_t* first_frames, const uint32_t* spp,
                      float* done_ms) {
  if (!ctx || !params_112n || !first_frames || !spp) return WGPT_E_INVALID;
  if (!ctx->has_scene) return fail(ctx, WGPT_E_STATE, "no scene uploaded");
  const uint32_t n = (uint32_t)ctx->views.size();
  if (n == 0) return fail(ctx, WGPT_E_STATE, "no views: call wgpt_set_views first");
  std::vector<wgpt::WfJobView> jv(n);
  wgpt_scene_params p0;
  memcpy(&p0, params_112n, sizeof p0);
  for (uint32_t i = 0; i < n; ++i) {
    wgpt_scene_params q;
    memcpy(&q, (const char*)params_112n + (size_t)i * sizeof q, sizeof q);
    const auto& v = ctx->views[i];
    char buf[160];
    if (q.width != v.w || q.height != v.h) {
      snprintf(buf, sizeof buf, "view %u: params %ux%u differ from the view size %ux%u", i, q.width, q.height, v.w, v.h);
      return fail(ctx, WGPT_E_INVALID, buf);
    }
    if (q.sky_width != p0.sky_width || q.sky_height != p0.sky_height || q.sky_cdf_index != p0.sky_cdf_index ||
        memcmp(&q.sky_total_lum, &p0.sky_total_lum, 4) != 0 || memcmp(&q.total_light_power, &p0.total_light_power, 4) != 0) {
      snprintf(buf, sizeof buf, "view %u: sky fields differ from view 0 (all views render one scene)", i);
      return fail(ctx, WGPT_E_INVALID, buf);
    }
    if ((uint64_t)v.w * v.h * spp[i] >= (1ull << 32)) {
      snprintf(buf, sizeof buf, "view %u: pixels x samples must stay below 2^32", i);
      return fail(ctx, WGPT_E_INVALID, buf);
    }
    int rc = check_env(ctx, q);
    if (rc) return rc;
    jv[i].q = q;
    jv[i].sx = 0; jv[i].sy = 0; jv[i].sw = v.w; jv[i].sh = v.h;
    jv[i].first_frame = first_frames[i];
    jv[i].spp = spp[i];
    jv[i].accum = v.accum;
    jv[i].out = v.out;
    jv[i].out_pitch = v.w;
  }
  CK(wgpt::select_device(ctx->device), "cudaSetDevice");
  if (!ctx->wf) ctx->wf = wgpt::wf_engine_create();
  unsigned long long* cnt = ctx->counting ? ctx->d_counters : nullptr;
  wgpt::StageTimer* tm = ctx->timing ? ctx->timer : nullptr;
  CK(wgpt::wf_render(ctx->wf, ctx->ds, ctx->d_pairs_tlas, ctx->d_pairs_bvh, jv.data(), n, ctx->d_status, cnt,
                     ctx->stream, tm, done_ms),
     "batched render");
  return WGPT_OK;
}

int wgpt_render_views_gbuffer(wgpt_ctx* ctx, const void* params_112n) {
  if (!ctx || !params_112n) return WGPT_E_INVALID;
  if (!ctx->has_scene) return fail(ctx, WGPT_E_STATE, "no scene uploaded");
  if (ctx->views.empty()) return fail(ctx, WGPT_E_STATE, "no views: call wgpt_set_views first");
  CK(wgpt::select_device(ctx->device), "cudaSetDevice");
  for (size_t i = 0; i < ctx->views.size(); ++i) {
    auto& v = ctx->views[i];
    wgpt_scene_params q;
    memcpy(&q, (const char*)params_112n + i * sizeof q, sizeof q);
    if (q.width != v.w || q.height != v.h) return fail(ctx, WGPT_E_INVALID, "view params size differs from the view");
    if (!v.gbuf) CK(cudaMalloc(&v.gbuf, (size_t)v.w * v.h * 48), "cudaMalloc view G-buffer");
    CK(wgpt::launch_gbuffer(ctx->ds, q, 0, 0, v.w, v.h, v.gbuf, v.out, v.w, ctx->d_status, ctx->stream),
       "view gbuffer launch");
  }
  return WGPT_OK;
}

int wgpt_read_view(wgpt_ctx* ctx, uint32_t view, float* accum, uint8_t* out) {
  if (!ctx) return WGPT_E_INVALID;
  if (view >= ctx->views.size()) return fail(ctx, WGPT_E_INVALID, "view index out of range");
  int rc = wgpt_synchronize(ctx);
  if (rc) return rc;
  const auto& v = ctx->views[view];
  size_t np = (size_t)v.w * v.h;
  if (accum) CK(cudaMemcpy(accum, v.accum, np * 16, cudaMemcpyDeviceToHost), "read view accumulation");
  if (out) CK(cudaMemcpy(out, v.out, np * 4, cudaMemcpyDeviceToHost), "read view image");
  return WGPT_OK;
}

int wgpt_set_env_sampling(wgpt_ctx* ctx, int mode) {
  if (!ctx || (mode != WGPT_ENV_CDF && mode != WGPT_ENV_ALIAS)) return WGPT_E_INVALID;
  if (mode == WGPT_ENV_ALIAS && !(ctx->has_scene && ctx->has_alias))
    return fail(ctx, WGPT_E_STATE, "no sky alias table uploaded (wgpt_scene_desc.sky_alias)");
  CK(wgpt::select_device(ctx->device), "cudaSetDevice");
  CK(cudaStreamSynchronize(ctx->stream), "drain");
  ctx->env_mode = mode;
  if (mode == WGPT_ENV_ALIAS) ctx->ds.flags |= wgpt::SCENE_ENV_ALIAS;
  else ctx->ds.flags &= ~(uint32_t)wgpt::SCENE_ENV_ALIAS;
  return WGPT_OK;
}

int wgpt_set_accum_f64(wgpt_ctx* ctx, int on) {
  if (!ctx) return WGPT_E_INVALID;
  if (ctx->w == 0) return fail(ctx, WGPT_E_STATE, "no image size: call wgpt_resize first");
  CK(wgpt::select_device(ctx->device), "cudaSetDevice");
  CK(cudaStreamSynchronize(ctx->stream), "drain");
  dfree_t(ctx->acc64);
  if (on) {
    size_t bytes = (size_t)ctx->w * ctx->h * 64;
    CK(cudaMalloc(&ctx->acc64, bytes), "cudaMalloc FP64 accumulation");
    CK(cudaMemsetAsync(ctx->acc64, 0, bytes, ctx->stream), "clear FP64 accumulation");
  }
  return WGPT_OK;
}

int wgpt_read_accum_f64(wgpt_ctx* ctx, double* dst) {
  if (!ctx) return WGPT_E_INVALID;
  return readback(ctx, dst, ctx->acc64, (size_t)ctx->w * ctx->h * 64, "read FP64 accumulation");
}

int wgpt_write_accum_f64(wgpt_ctx* ctx, const double* src) {
  if (!ctx || !src) return WGPT_E_INVALID;
  if (!ctx->acc64) return fail(ctx, WGPT_E_STATE, "FP64 accumulation is off");
  CK(wgpt::select_device(ctx->device), "cudaSetDevice");
  CK(cudaStreamSynchronize(ctx->stream), "drain");
  CK(cudaMemcpy(ctx->acc64, src, (size_t)ctx->w * ctx->h * 64, cudaMemcpyHostToDevice), "write FP64 accumulation");
  return WGPT_OK;
}

int wgpt_set_wavefront_config(wgpt_ctx* ctx, uint32_t pool_paths, uint64_t units_per_pass) {
  if (!ctx) return WGPT_E_INVALID;
  if (!ctx->wf) ctx->wf = wgpt::wf_engine_create();
  uint32_t cur_pool = 0;
  uint64_t cur_units = 0;
  wgpt::wf_engine_get(ctx->wf, &cur_pool, &cur_units);
  if (pool_paths == 0) pool_paths = cur_pool;
  if (units_per_pass == 0) units_per_pass = cur_units;
  if (wgpt::wf_engine_configure(ctx->wf, pool_paths, units_per_pass))
    return fail(ctx, WGPT_E_INVALID, "wavefront sizing out of range (pool 1024..2^26 paths, 2^16..2^30 units)");
  return WGPT_OK;
}

int wgpt_set_wavefront_tuning(wgpt_ctx* ctx, const wgpt_wavefront_tuning* t) {
  if (!ctx || !t) return WGPT_E_INVALID;
  if (!ctx->wf) ctx->wf = wgpt::wf_engine_create();
  CK(wgpt::select_device(ctx->device), "cudaSetDevice");
  CK(cudaStreamSynchronize(ctx->stream), "drain before retuning");
  if (wgpt::wf_engine_tune(ctx->wf, (int)t->trav_shape, (int)t->shade_block, t->refill_closest, t->refill_shadow,
                           (int)t->shadow_wide))
    return fail(ctx, WGPT_E_INVALID,
                "wavefront tuning out of range (shape 0..2, shading block 256 or 512, refill 1..32, shadow_wide 0 or 1)");
  return WGPT_OK;
}

int wgpt_get_wavefront_tuning(wgpt_ctx* ctx, wgpt_wavefront_tuning* t) {
  if (!ctx || !t) return WGPT_E_INVALID;
  if (!ctx->wf) ctx->wf = wgpt::wf_engine_create();
  int shape = 0, shade = 0, wide = 0;
  wgpt::wf_engine_tuning(ctx->wf, &shape, &shade, &t->refill_closest, &t->refill_shadow, &wide);
  t->trav_shape = (uint32_t)shape;
  t->shade_block = (uint32_t)shade;
  t->shadow_wide = (uint32_t)wide;
  return WGPT_OK;
}

int wgpt_get_wavefront_config(wgpt_ctx* ctx, uint32_t* pool_paths, uint64_t* units_per_pass) {
  if (!ctx || !pool_paths || !units_per_pass) return WGPT_E_INVALID;
  if (!ctx->wf) ctx->wf = wgpt::wf_engine_create();
  wgpt::wf_engine_get(ctx->wf, pool_paths, units_per_pass);
  return WGPT_OK;
}

int wgpt_set_counting(wgpt_ctx* ctx, int on) {
  if (!ctx) return WGPT_E_INVALID;
  CK(wgpt::select_device(ctx->device), "cudaSetDevice");
  if (on && !ctx->counting) CK(cudaMemsetAsync(ctx->d_counters, 0, 128 * sizeof(unsigned long long), ctx->stream), "reset counters");
  ctx->counting = on != 0;
  return WGPT_OK;
}

int wgpt_read_counters(wgpt_ctx* ctx, uint64_t* dst) {
  if (!ctx || !dst) return WGPT_E_INVALID;
  uint64_t all[128];
  int rc = readback(ctx, all, ctx->d_counters, sizeof all, "read counters");
  if (rc) return rc;
  for (int k = 0; k < 16; ++k) {
    dst[k] = 0;
    for (int st = 0; st < 8; ++st) dst[k] += all[16 * st + k];
  }
  return WGPT_OK;
}

int wgpt_read_stage_counters(wgpt_ctx* ctx, uint64_t* dst128) {
  if (!ctx) return WGPT_E_INVALID;
  return readback(ctx, dst128, ctx->d_counters, 128 * sizeof(unsigned long long), "read stage counters");
}

int wgpt_set_stage_timing(wgpt_ctx* ctx, int on) {
  if (!ctx) return WGPT_E_INVALID;
  CK(wgpt::select_device(ctx->device), "cudaSetDevice");
  if (on && !ctx->timer) {
    ctx->timer = new wgpt::StageTimer();
    for (int i = 0; i < wgpt::StageTimer::kMaxEvents; ++i) CK(cudaEventCreate(&ctx->timer->ev[i]), "cudaEventCreate");
    ctx->timer->ready = true;
  }
  if (ctx->timer) ctx->timer->used = 0;
  ctx->timing = on != 0;
  return WGPT_OK;
}

int wgpt_read_stage_times(wgpt_ctx* ctx, double* ms8, uint32_t* launches8) {
  if (!ctx || !ms8 || !launches8) return WGPT_E_INVALID;
  for (int k = 0; k < 8; ++k) { ms8[k] = 0; launches8[k] = 0; }
  if (!ctx->timer) return WGPT_OK;
  int rc = wgpt_synchronize(ctx);
  if (rc) return rc;
  for (int i = 0; i + 1 < ctx->timer->used; i += 2) {
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, ctx->timer->ev[i], ctx->timer->ev[i + 1]), "cudaEventElapsedTime");
    int stg = ctx->timer->stage_of[i / 2];
    ms8[stg] += ms;
    launches8[stg] += 1;
  }
  ctx->timer->used = 0;
  return WGPT_OK;
}

}  // extern "C"
