// Persistent two-level BVH traversal for the wavefront stages.
//
// Same tests, in the same order, as trace_tlas / trace_mesh / trace_tlas_shadow /
// trace_mesh_shadow of shader.wgsl (473-542, 694-752, 813-872, 1134-1184), restructured for SIMT
// efficiency:
//  * one loop over a single stack holds both levels: entering a mesh instance pushes an
//    end-of-instance marker under the instance's BLAS root, so a thread can be anywhere in either
//    level and the loop body stays the same for every lane;
//  * warps fetch rays from a shared queue cursor and refill a lane as soon as its ray is done,
//    so lanes do not idle behind the longest ray of their warp;
//  * inner nodes are read through a derived child-pair array: pair[i] holds both children's
//    boxes and what is needed to continue (absolute node index of an inner child, or the
//    reference's relative first-item index and count of a leaf) in one 64-byte record, instead
//    of three separate 32-byte node reads (the node itself, then each child).
// The pair arrays are built on upload from the reference's node buffers; node boxes are copied
// bit for bit, so every slab test sees the same operands.
#pragma once
#include "pt_device.cuh"

namespace pt {

struct DPairs {
  const float4* tlas;   // 4 x float4 per TLAS node
  const float4* bvh;    // 4 x float4 per BLAS node
  const float4* tlas4;  // quad records: 8 x float4 per TLAS node (4-wide any-hit traversal)
  const float4* bvh4;   // quad records: 8 x float4 per BLAS node
};

// Stack entries: .x = kind << 29 | item count, .y = node index or first item.
enum : uint32_t {
  K_TLAS_INNER = 0u,   // .y = TLAS node
  K_TLAS_LEAF = 1u,    // .y = first object, count = objects
  K_BLAS_INNER = 2u,   // .y = absolute BLAS node
  K_BLAS_LEAF = 3u,    // .y = first triangle relative to the instance's triangle offset
  K_SENTINEL = 4u,     // end of the current mesh instance
  K_TLAS_REST = 5u     // remaining objects of a multi-object TLAS leaf (not a node visit)
};
constexpr int TRAV_STACK = 132;   // TLAS depth + BLAS depth (each <= 62, checked on upload) + 2

__device__ __forceinline__ uint2 ent(uint32_t kind, uint32_t count, uint32_t val) {
  return make_uint2((kind << 29) | count, val);
}

struct TravCommon {
  Ray rw;
  v3 inv_w;
  Ray rl;
  v3 inv_l;
  uint32_t tri_offset;
  int32_t inst_mat;
  int32_t inst_oidx;
  int sp;
  uint2 stack[TRAV_STACK];

  __device__ __forceinline__ void push(uint2 e, uint32_t& err) {
    if (sp < TRAV_STACK) stack[sp++] = e; else err |= ERR_STACK;
  }
  // Children of a pair record, pushed in the reference's order (the nearer one last).
  __device__ __forceinline__ void push_children(float lt, float rt, float limit, float4 lmin, float4 lmax, float4 rmin,
                                                float4 rmax, bool blas, uint32_t& err) {
    uint32_t kin = blas ? K_BLAS_INNER : K_TLAS_INNER, klf = blas ? K_BLAS_LEAF : K_TLAS_LEAF;
    uint32_t ln = __float_as_uint(lmin.w), rn = __float_as_uint(rmin.w);
    uint2 le = ln > 0u ? ent(klf, ln, __float_as_uint(lmax.w)) : ent(kin, 0u, __float_as_uint(lmax.w));
    uint2 re = rn > 0u ? ent(klf, rn, __float_as_uint(rmax.w)) : ent(kin, 0u, __float_as_uint(rmax.w));
    bool push_l = lt >= 0.0f && lt < limit;
    bool push_r = rt >= 0.0f && rt < limit;
    if (lt < rt) {
      if (push_r) push(re, err);
      if (push_l) push(le, err);
    } else {
      if (push_l) push(le, err);
      if (push_r) push(re, err);
    }
  }
  // Root entry of a tree from the reference node record (lo, hi).
  __device__ __forceinline__ uint2 root_entry(float4 lo, float4 hi, uint32_t node, bool blas) {
    uint32_t n = __float_as_uint(lo.w);
    if (n > 0u) return ent(blas ? K_BLAS_LEAF : K_TLAS_LEAF, n, __float_as_uint(hi.w));
    return ent(blas ? K_BLAS_INNER : K_TLAS_INNER, 0u, node);
  }
};

__device__ __forceinline__ bool obj_enabled(const DScene& s, int32_t type) {
  return (type == 0 && HAS(s, WGPT_HAS_MESHES)) || (type == 1 && HAS(s, WGPT_HAS_SPHERES)) ||
         (type == 2 && HAS(s, WGPT_HAS_CUBES)) || (type == 3 && HAS(s, WGPT_HAS_CYLINDERS)) ||
         (type == 4 && HAS(s, WGPT_HAS_TORI));
}

// ------------------------------------------------------------------------ closest hit
struct ClosestTrav : TravCommon {
  HitRec hit;
};

// Planes and the TLAS root test (trace_scene, shader.wgsl:754-765; trace_tlas :695-703).
template <bool COUNT>
__device__ __forceinline__ void closest_init(const DScene& s, ClosestTrav& t, Counters<COUNT>& cn) {
  cn.add(C_RAYS_EXT);
  HitRec& hit = t.hit;
  hit.t = 1e10f; hit.m_idx = -1; hit.o_idx = -1; hit.kind = 0; hit.id = -1; hit.aux = -1; hit.bu = 0.0f; hit.bv = 0.0f;
  hit.tsrc = -1; hit.tsrc_t = 0.0f;
  t.sp = 0;
  if (HAS(s, WGPT_HAS_PLANES)) {
    for (uint32_t i = 0; i < s.n_planes; i++) {
      float4 a = ld4(s.planes + (size_t)i * 2);
      float4 b = ld4(s.planes + (size_t)i * 2 + 1);
      v3 pn = f3(a);
      float denom = dot(pn, t.rw.direction);
      float tt = -1.0f;
      if (absf(denom) > 1e-6f) {
        float x = (a.w - dot(pn, t.rw.origin)) / denom;
        if (x > 0.001f) tt = x;
      }
      if (tt > 0.001f && tt < hit.t) {
        hit.t = tt; hit.m_idx = __float_as_int(b.x); hit.kind = 1; hit.id = (int32_t)i;
        hit.tsrc = -2 - (int32_t)i; hit.tsrc_t = tt;
      }
    }
  }
  t.inv_w = 1.0f / t.rw.direction;
  if (HAS(s, WGPT_HAS_SPHERES | WGPT_HAS_CUBES | WGPT_HAS_CYLINDERS | WGPT_HAS_TORI | WGPT_HAS_MESHES)) {
    cn.add(C_CHILD_TESTS);
    float4 lo = ld4(s.tlas), hi = ld4(s.tlas + 1);
    float base_t = intersect_aabb(t.rw.origin, t.inv_w, lo, hi);
    if (!(base_t < 0.0f || base_t >= hit.t)) t.stack[t.sp++] = t.root_entry(lo, hi, 0u, false);
  }
}

// Enters mesh instance `i` (trace_mesh's set-up and root test, shader.wgsl:476-486).
template <bool COUNT>
__device__ __forceinline__ void enter_mesh(const DScene& s, TravCommon& t, const m4& inv, uint32_t node_offset,
                                           uint32_t tri_offset, int32_t mat, int32_t oidx, float limit,
                                           uint32_t& err, Counters<COUNT>& cn) {
  t.rl = to_local(inv, t.rw);
  t.inv_l = 1.0f / t.rl.direction;
  cn.add(C_CHILD_TESTS);
  float4 lo = ld4(s.bvh + (size_t)node_offset * 2), hi = ld4(s.bvh + (size_t)node_offset * 2 + 1);
  float base_t = intersect_aabb(t.rl.origin, t.inv_l, lo, hi);
  if (base_t < 0.0f || base_t >= limit) return;
  t.tri_offset = tri_offset;
  t.inst_mat = mat;
  t.inst_oidx = oidx;
  t.push(ent(K_SENTINEL, 0u, 0u), err);
  t.push(t.root_entry(lo, hi, node_offset, true), err);
}

// Pops and processes inner nodes until the stack top is something else, which is popped into
// `e` (true), or the stack runs empty (false).  No leaf is processed in between, so the pruning
// limit is the same as when entries are taken one at a time: the order of work is unchanged.
// Running inner nodes back to back keeps a warp's lanes on the node code together and then on
// the leaf code together, instead of splitting every step between the two.
template <bool COUNT>
__device__ __forceinline__ bool inner_run(const DPairs& P, TravCommon& t, float limit, uint32_t& err,
                                          Counters<COUNT>& cn, uint2& e) {
  while (t.sp > 0) {
    e = t.stack[--t.sp];
    const uint32_t kind = e.x >> 29;
    if (kind != K_BLAS_INNER && kind != K_TLAS_INNER) return true;
    cn.add(C_NODES);
    bool blas = kind == K_BLAS_INNER;
    const float4* pp = (blas ? P.bvh : P.tlas) + (size_t)e.y * 4;
    float4 a = ld4(pp), b = ld4(pp + 1), c = ld4(pp + 2), d = ld4(pp + 3);
    const Ray& r = blas ? t.rl : t.rw;
    v3 inv = blas ? t.inv_l : t.inv_w;
    cn.add(C_CHILD_TESTS, 2);
    float lt = intersect_aabb(r.origin, inv, a, b);
    float rt = intersect_aabb(r.origin, inv, c, d);
    t.push_children(lt, rt, limit, a, b, c, d, blas, err);
  }
  return false;
}

// The any-hit form of inner_run over the quad records: one visit tests the up to four boxes
// two levels down (the children that are leaves, and the children's children) and pushes the
// hits farthest first, so the nearest is taken next.  A box inside its parent's box is hit by a
// ray only if the parent is (the slab bounds are monotonic in the box), so exactly the leaves the
// two-wide walk reaches are reached; any-hit occlusion of opaque occluders does not depend on
// the order they are found in.  Used only where no occluder is alpha-textured (the transmittance
// product of those depends on the order) and no work is counted (the counters follow the
// reference's two-wide walk).
__device__ __forceinline__ bool inner_run_wide(const DPairs& P, TravCommon& t, float limit, uint32_t& err, uint2& e) {
  while (t.sp > 0) {
    e = t.stack[--t.sp];
    const uint32_t kind = e.x >> 29;
    if (kind != K_BLAS_INNER && kind != K_TLAS_INNER) return true;
    const bool blas = kind == K_BLAS_INNER;
    const float4* qp = (blas ? P.bvh4 : P.tlas4) + (size_t)e.y * 8;
    const Ray& r = blas ? t.rl : t.rw;
    const v3 inv = blas ? t.inv_l : t.inv_w;
    const uint32_t kin = blas ? K_BLAS_INNER : K_TLAS_INNER, klf = blas ? K_BLAS_LEAF : K_TLAS_LEAF;
    float tt[4];
    uint2 en[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const float4 lo = ld4(qp + 2 * c), hi = ld4(qp + 2 * c + 1);
      const uint32_t n = __float_as_uint(lo.w), item = __float_as_uint(hi.w);
      tt[c] = -1.0f;
      en[c] = n > 0u ? ent(klf, n, item) : ent(kin, 0u, item);
      if (n != 0xffffffffu) {
        const float x = intersect_aabb(r.origin, inv, lo, hi);
        if (x >= 0.0f && x < limit) tt[c] = x;
      }
    }
    // push the hits in decreasing distance (a fixed four-element selection)
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      int best = -1;
      float bt = -1.0f;
#pragma unroll
      for (int c = 0; c < 4; ++c)
        if (tt[c] >= 0.0f && tt[c] >= bt) { bt = tt[c]; best = c; }
      if (best < 0) break;
#pragma unroll
      for (int c = 0; c < 4; ++c)
        if (c == best) { t.push(en[c], err); tt[c] = -1.0f; }
    }
  }
  return false;
}

// A run of inner nodes and then one leaf (or instance end); returns true when the stack is
// empty (the ray is done).
template <bool COUNT>
__device__ __forceinline__ bool closest_step(const DScene& s, const DPairs& P, ClosestTrav& t, uint32_t& err,
                                             Counters<COUNT>& cn) {
  HitRec& hit = t.hit;
  uint2 e;
  if (!inner_run<COUNT>(P, t, hit.t, err, cn, e)) return true;
  uint32_t kind = e.x >> 29, cnt = e.x & 0x1fffffffu;
  if (kind == K_BLAS_LEAF) {
    // this leaf and any leaves directly under it on the stack (taken in stack order)
    while (true) {
      cn.add(C_NODES);
      uint32_t start = t.tri_offset + e.y;
      for (uint32_t i = start; i < start + cnt; i++) {
        const float4* tp = s.tris + (size_t)i * 8;
        float t_tri, u, v;
        cn.add(C_TRI_TESTS);
        if (intersect_triangle(t.rl, ld4(tp), ld4(tp + 1), ld4(tp + 2), &t_tri, &u, &v)) {
          if (t_tri >= 0.0f && t_tri < hit.t) {
            hit.t = t_tri; hit.m_idx = t.inst_mat; hit.o_idx = t.inst_oidx;
            hit.kind = 2; hit.id = (int32_t)i; hit.aux = -1; hit.bu = u; hit.bv = v;
          }
        }
      }
      if (t.sp == 0 || (t.stack[t.sp - 1].x >> 29) != K_BLAS_LEAF) break;
      e = t.stack[--t.sp];
      cnt = e.x & 0x1fffffffu;
    }
  } else if (kind == K_TLAS_LEAF || kind == K_TLAS_REST) {
    if (kind == K_TLAS_LEAF) cn.add(C_NODES);
    uint32_t end = e.y + cnt;
    for (uint32_t i = e.y; i < end; i++) {
      ObjHdr h = load_obj_hdr(s, i);
      cn.add(C_OBJ_VISITS);
      if (!obj_enabled(s, h.type)) continue;
      m4 inv = load_m4(s.objs + (size_t)i * 6);
      if (h.type == 0) {
        if (i + 1 < end) t.push(ent(K_TLAS_REST, end - (i + 1), i + 1), err);
        enter_mesh<COUNT>(s, t, inv, __float_as_uint(h.param0), __float_as_uint(h.param1), h.material_idx,
                          (int32_t)i, hit.t, err, cn);
        break;
      }
      float ta = 0.0f;
      if (analytic_t(inv, h, t.rw, &ta) && ta < hit.t) {
        hit.t = ta; hit.m_idx = h.material_idx; hit.o_idx = (int32_t)i; hit.kind = 3; hit.id = (int32_t)i;
        if (h.type <= 2) { hit.tsrc = (int32_t)i; hit.tsrc_t = ta; }
      }
    }
  }
  // K_SENTINEL: back at the TLAS level; the world ray is kept in t.rw
  return t.sp == 0;
}

// List meshes after the TLAS (trace_scene, shader.wgsl:767-771), nested form.
template <bool COUNT>
__device__ __forceinline__ void closest_finish(const DScene& s, ClosestTrav& t, uint32_t& err, Counters<COUNT>& cn) {
  if (HAS(s, WGPT_HAS_LIST_MESHES)) {
    for (uint32_t i = 0; i < s.n_meshes; i++) {
      const float4* mp = s.meshes + (size_t)i * 5;
      m4 inv = load_m4(mp);
      float4 e = ld4(mp + 4);
      trace_mesh<COUNT>(s, t.rw, inv, __float_as_uint(e.z), __float_as_uint(e.w), __float_as_int(e.x), -1, 4,
                        (int32_t)i, t.hit, err, cn);
    }
  }
}

// ------------------------------------------------------------------------ shadow (any hit)
struct ShadowTrav : TravCommon {
  float target_dist;
  int32_t target_idx;
  bool occluded;
  float trans;   // transmittance through the textured occluders crossed so far
};

// Planes first, then the TLAS from its root without a root test (shader.wgsl:1206-1218,
// 1134-1140).
template <bool COUNT, bool TEX>
__device__ __forceinline__ void shadow_init(const DScene& s, ShadowTrav& t, Counters<COUNT>& cn) {
  cn.add(C_RAYS_SHADOW);
  t.sp = 0;
  t.occluded = false;
  t.trans = 1.0f;
  if (HAS(s, WGPT_HAS_PLANES)) {
    for (uint32_t i = 0; i < s.n_planes; i++) {
      float4 a = ld4(s.planes + (size_t)i * 2);
      v3 pn = f3(a);
      float denom = dot(pn, t.rw.direction);
      if (absf(denom) > 1e-6f) {
        float x = (a.w - dot(pn, t.rw.origin)) / denom;
        if (x > 0.001f && x < t.target_dist && plane_blocks<TEX>(s, i, pn, t.rw, x, t.trans)) {
          t.occluded = true;
          return;
        }
      }
    }
  }
  t.inv_w = 1.0f / t.rw.direction;
  if (HAS(s, WGPT_HAS_SPHERES | WGPT_HAS_CUBES | WGPT_HAS_CYLINDERS | WGPT_HAS_TORI | WGPT_HAS_MESHES)) {
    float4 lo = ld4(s.tlas), hi = ld4(s.tlas + 1);
    t.stack[t.sp++] = t.root_entry(lo, hi, 0u, false);
  }
}

template <bool COUNT, bool TEX, bool WIDE = false>
__device__ __forceinline__ bool shadow_step(const DScene& s, const DPairs& P, ShadowTrav& t, uint32_t& err,
                                            Counters<COUNT>& cn) {
  if (t.occluded) return true;
  uint2 e;
  if (WIDE) {
    if (!inner_run_wide(P, t, t.target_dist, err, e)) return true;
  } else {
    if (!inner_run<COUNT>(P, t, t.target_dist, err, cn, e)) return true;
  }
  uint32_t kind = e.x >> 29, cnt = e.x & 0x1fffffffu;
  if (kind == K_BLAS_LEAF) {
    while (true) {
      cn.add(C_NODES);
      uint32_t start = t.tri_offset + e.y;
      for (uint32_t i = start; i < start + cnt; i++) {
        const float4* tp = s.tris + (size_t)i * 8;
        float t_tri, u, v;
        cn.add(C_TRI_TESTS);
        if (intersect_triangle(t.rl, ld4(tp), ld4(tp + 1), ld4(tp + 2), &t_tri, &u, &v)) {
          if (t_tri >= 0.0f && t_tri < t.target_dist && tri_blocks(s, occ_mat<TEX>(s, t.inst_mat), tp, u, v, t.trans)) {
            t.occluded = true;
            return true;
          }
        }
      }
      if (t.sp == 0 || (t.stack[t.sp - 1].x >> 29) != K_BLAS_LEAF) break;
      e = t.stack[--t.sp];
      cnt = e.x & 0x1fffffffu;
    }
  } else if (kind == K_TLAS_LEAF || kind == K_TLAS_REST) {
    if (kind == K_TLAS_LEAF) cn.add(C_NODES);
    uint32_t end = e.y + cnt;
    for (uint32_t i = e.y; i < end; i++) {
      if ((int32_t)i == t.target_idx) continue;
      ObjHdr h = load_obj_hdr(s, i);
      cn.add(C_OBJ_VISITS);
      if (!obj_enabled(s, h.type)) continue;
      m4 inv = load_m4(s.objs + (size_t)i * 6);
      if (h.type == 0) {
        if (i + 1 < end) t.push(ent(K_TLAS_REST, end - (i + 1), i + 1), err);
        enter_mesh<COUNT>(s, t, inv, __float_as_uint(h.param0), __float_as_uint(h.param1), h.material_idx,
                          (int32_t)i, t.target_dist, err, cn);
        break;
      }
      if (analytic_shadow<TEX>(s, inv, h, t.rw, t.target_dist, t.trans)) { t.occluded = true; return true; }
    }
  }
  return t.sp == 0;
}

template <bool COUNT, bool TEX>
__device__ __forceinline__ void shadow_finish(const DScene& s, ShadowTrav& t, uint32_t& err, Counters<COUNT>& cn) {
  if (t.occluded) return;
  if (HAS(s, WGPT_HAS_LIST_MESHES)) {
    for (uint32_t i = 0; i < s.n_meshes; i++) {
      const float4* mp = s.meshes + (size_t)i * 5;
      m4 inv = load_m4(mp);
      float4 e = ld4(mp + 4);
      if (mesh_shadow<COUNT, TEX>(s, t.rw, inv, __float_as_uint(e.z), __float_as_uint(e.w), __float_as_int(e.x),
                             t.target_dist, t.trans, err, cn)) {
        t.occluded = true;
        return;
      }
    }
  }
}

}  // namespace pt
