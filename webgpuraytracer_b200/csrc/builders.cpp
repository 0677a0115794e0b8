// Native versions of the host-side builders that produce the scene buffers (tracer.js runs these
// in JavaScript at scene load):
//   wgpt_build_blas    ModelData.generateBVH, binned SAH (tracer.js:1025-1118)
//   wgpt_build_tlas    SceneBVHBuilder, median split on the widest axis (tracer.js:1509-1619)
//   wgpt_build_env_cdf HDRTexture.buildHDRCDF (tracer.js:135-204)
//   wgpt_build_env_alias an alias table over the same weights (opt-in sampling mode)
//   wgpt_decode_rgbe   parseHdr (lib/parse-hdr.js:20-211) + HDRTexture.updateData (tracer.js:76-87)
// JavaScript numbers are IEEE doubles and Float32Array / Float16Array stores round to nearest
// even; the builders compute in double and round at the same stores, so their outputs are the
// bytes the reference would upload.
#include <stdint.h>
#include <stdio.h>
#include <string.h>
#include <math.h>
#include <cctype>
#include <cmath>
#include <cstdlib>
#include <algorithm>
#include <string>
#include <vector>

#include "../../include/wgpt.h"

namespace {

struct Tri {
  float v[3][3], n[3][3], uv[3][2];
  double c[3];        // centroid (tracer.js:1014-1018), double
  double lo[3], hi[3];
};

struct Box {
  double lo[3], hi[3];
  void reset() { for (int k = 0; k < 3; ++k) { lo[k] = INFINITY; hi[k] = -INFINITY; } }
  void add(const Tri& t) {
    for (int k = 0; k < 3; ++k) { lo[k] = std::min(lo[k], t.lo[k]); hi[k] = std::max(hi[k], t.hi[k]); }
  }
  double area() const {   // getArea, tracer.js:1041-1044
    double d0 = hi[0] - lo[0], d1 = hi[1] - lo[1], d2 = hi[2] - lo[2];
    return 2 * (d0 * d1 + d1 * d2 + d2 * d0);
  }
};

struct BNode { Box b; int left = -1, right = -1; std::vector<uint32_t> items; bool leaf = false; };

struct BlasBuilder {
  std::vector<Tri> tris;
  std::vector<BNode> tree;

  Box bounds(const std::vector<uint32_t>& idx) const {
    Box b; b.reset();
    for (uint32_t i : idx) b.add(tris[i]);
    return b;
  }

  // subdivide, tracer.js:1046-1087
  int subdivide(std::vector<uint32_t>&& idx) {
    int me = (int)tree.size();
    tree.emplace_back();
    Box b = bounds(idx);
    double root_area = b.area();
    double best_cost = (double)idx.size() * root_area;
    int best_axis = -1;
    double best_split = -1;
    const size_t n = idx.size();
    for (int axis = 0; axis < 3; ++axis) {
      double start = b.lo[axis], end = b.hi[axis];
      if (end - start < 1e-6) continue;
      int num_bins = (int)std::min<size_t>(n, 12);
      for (int i = 1; i < num_bins; ++i) {
        double split = start + ((double)i / (double)num_bins) * (end - start);
        Box bl, br; bl.reset(); br.reset();
        size_t nl = 0, nr = 0;
        for (uint32_t t : idx) {
          if (tris[t].c[axis] < split) { bl.add(tris[t]); ++nl; } else { br.add(tris[t]); ++nr; }
        }
        if (nl == 0 || nr == 0) continue;
        double cost = (double)nl * bl.area() + (double)nr * br.area();
        if (cost < best_cost) { best_cost = cost; best_axis = axis; best_split = split; }
      }
    }
    tree[me].b = b;
    if (best_axis == -1 || n <= 2) {
      tree[me].leaf = true;
      tree[me].items = std::move(idx);
      return me;
    }
    std::vector<uint32_t> l, r;
    l.reserve(n); r.reserve(n);
    for (uint32_t t : idx) (tris[t].c[best_axis] < best_split ? l : r).push_back(t);
    idx.clear(); idx.shrink_to_fit();
    int li = subdivide(std::move(l));
    int ri = subdivide(std::move(r));
    tree[me].left = li; tree[me].right = ri;
    return me;
  }
};

void put_node(wgpt_bvh_node* o, const Box& b, uint32_t num, uint32_t next) {
  for (int k = 0; k < 3; ++k) { o->aabb_min[k] = (float)b.lo[k]; o->aabb_max[k] = (float)b.hi[k]; }
  o->num_triangles = num;
  o->next = next;
}

// IEEE double -> binary16, round to nearest even (Float16Array store semantics).
uint16_t double_to_half(double x) {
  uint16_t sign = std::signbit(x) ? 0x8000u : 0u;
  double a = fabs(x);
  if (std::isnan(x)) return (uint16_t)(sign | 0x7e00u);
  if (a >= 65520.0) return (uint16_t)(sign | 0x7c00u);   // rounds to infinity
  if (a < 5.9604644775390625e-08 / 2) {                   // below half the smallest subnormal
    return sign;
  }
  int e;
  double m = frexp(a, &e);   // a = m * 2^e, m in [0.5, 1)
  int exp16 = e - 1 + 15;    // exponent of a in [1, 2) form, biased
  if (exp16 <= 0) {
    // subnormal: value = q * 2^-24
    double q = a / 5.9604644775390625e-08;
    double r = nearbyint(q);   // default rounding mode: ties to even
    return (uint16_t)(sign | (uint16_t)r);
  }
  double frac = (m * 2.0 - 1.0) * 1024.0;   // 10-bit mantissa, exact scaling
  double r = nearbyint(frac);
  uint32_t mant = (uint32_t)r;
  if (mant == 1024u) { mant = 0; exp16 += 1; }
  if (exp16 >= 31) return (uint16_t)(sign | 0x7c00u);
  return (uint16_t)(sign | (exp16 << 10) | mant);
}

double half_to_double(uint16_t h) {
  uint32_t e = (h >> 10) & 0x1fu, m = h & 0x3ffu;
  double v;
  if (e == 0) v = ldexp((double)m, -24);
  else if (e == 31) v = m ? NAN : INFINITY;
  else v = ldexp((double)(m | 0x400u), (int)e - 25);
  return (h & 0x8000u) ? -v : v;
}

}  // namespace

extern "C" {

int wgpt_build_blas(const float* tris24, uint32_t n, wgpt_bvh_node* nodes_out, uint32_t* n_nodes, wgpt_triangle* tris_out) {
  if (!tris24 || !nodes_out || !n_nodes || !tris_out || n == 0) return WGPT_E_INVALID;
  BlasBuilder b;
  b.tris.resize(n);
  for (uint32_t i = 0; i < n; ++i) {
    const float* s = tris24 + (size_t)i * 24;
    Tri& t = b.tris[i];
    for (int v = 0; v < 3; ++v) {
      for (int k = 0; k < 3; ++k) { t.v[v][k] = s[v * 3 + k]; t.n[v][k] = s[9 + v * 3 + k]; }
      for (int k = 0; k < 2; ++k) t.uv[v][k] = s[18 + v * 2 + k];
    }
    for (int k = 0; k < 3; ++k) {
      double a = t.v[0][k], bb = t.v[1][k], c = t.v[2][k];
      t.c[k] = (a + bb + c) / 3;
      t.lo[k] = std::min(std::min(std::min((double)INFINITY, a), bb), c);
      t.hi[k] = std::max(std::max(std::max(-(double)INFINITY, a), bb), c);
    }
  }
  std::vector<uint32_t> all(n);
  for (uint32_t i = 0; i < n; ++i) all[i] = i;
  b.tree.reserve(2 * (size_t)n);
  int root = b.subdivide(std::move(all));
  // flatten, tracer.js:1093-1115: DFS pre-order, left child first
  uint32_t count = 0, tri_count = 0;
  struct Frame { int node; int slot; };
  std::vector<Frame> stack;
  stack.push_back({root, -1});
  while (!stack.empty()) {
    Frame f = stack.back();
    stack.pop_back();
    uint32_t index = count++;
    if (f.slot >= 0) nodes_out[f.slot].next = index;   // the parent's 'next' = this right child
    const BNode& nd = b.tree[f.node];
    if (nd.leaf) {
      put_node(&nodes_out[index], nd.b, (uint32_t)nd.items.size(), tri_count);
      for (uint32_t t : nd.items) {
        const Tri& tr = b.tris[t];
        wgpt_triangle& o = tris_out[tri_count++];
        memset(&o, 0, sizeof o);
        memcpy(o.v0, tr.v[0], 12); memcpy(o.v1, tr.v[1], 12); memcpy(o.v2, tr.v[2], 12);
        memcpy(o.n0, tr.n[0], 12); memcpy(o.n1, tr.n[1], 12); memcpy(o.n2, tr.n[2], 12);
        memcpy(o.uv0, tr.uv[0], 8); memcpy(o.uv1, tr.uv[1], 8); memcpy(o.uv2, tr.uv[2], 8);
      }
    } else {
      put_node(&nodes_out[index], nd.b, 0u, 0u);
      stack.push_back({nd.right, (int)index});
      stack.push_back({nd.left, -1});
    }
  }
  *n_nodes = count;
  return WGPT_OK;
}

int wgpt_build_tlas(const float* aabbs6, uint32_t n, wgpt_bvh_node* nodes_out, uint32_t* n_nodes) {
  if (!n_nodes) return WGPT_E_INVALID;
  *n_nodes = 0;
  if (n == 0) return WGPT_OK;
  if (!aabbs6 || !nodes_out) return WGPT_E_INVALID;
  struct Item { uint32_t index; float lo[3], hi[3]; };
  std::vector<Item> items(n);
  for (uint32_t i = 0; i < n; ++i) {
    items[i].index = i;
    for (int k = 0; k < 3; ++k) { items[i].lo[k] = aabbs6[i * 6 + k]; items[i].hi[k] = aabbs6[i * 6 + 3 + k]; }
  }
  struct Node { float lo[3], hi[3]; uint32_t num, obj, next; };
  std::vector<Node> nodes;
  nodes.reserve(2 * (size_t)n);
  // recursiveBuild, tracer.js:1533-1579
  struct Rec {
    std::vector<Node>& nodes;
    void build(std::vector<Item> it, int depth) {
      size_t me = nodes.size();
      nodes.push_back(Node{});
      float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
      for (const Item& x : it)
        for (int k = 0; k < 3; ++k) {   // vec3.min / vec3.max (Math.min/max on float32 values)
          lo[k] = std::min(lo[k], x.lo[k]);
          hi[k] = std::max(hi[k], x.hi[k]);
        }
      for (int k = 0; k < 3; ++k) { nodes[me].lo[k] = lo[k]; nodes[me].hi[k] = hi[k]; }
      if (it.size() <= 1 || depth > 20) {
        nodes[me].num = (uint32_t)it.size();
        nodes[me].obj = it[0].index;
        return;
      }
      float size[3];
      for (int k = 0; k < 3; ++k) size[k] = hi[k] - lo[k];   // vec3.sub into a Float32Array
      int axis = 0;
      if (size[1] > size[0]) axis = 1;
      if (size[2] > size[axis]) axis = 2;
      std::stable_sort(it.begin(), it.end(), [axis](const Item& a, const Item& b) {
        double ca = ((double)a.lo[axis] + (double)a.hi[axis]) * 0.5;
        double cb = ((double)b.lo[axis] + (double)b.hi[axis]) * 0.5;
        return ca < cb;
      });
      size_t mid = it.size() / 2;
      build(std::vector<Item>(it.begin(), it.begin() + mid), depth + 1);
      nodes[me].next = (uint32_t)nodes.size();
      build(std::vector<Item>(it.begin() + mid, it.end()), depth + 1);
    }
  } rec{nodes};
  rec.build(items, 0);
  // flatten, tracer.js:1590-1618
  for (size_t i = 0; i < nodes.size(); ++i) {
    const Node& nd = nodes[i];
    wgpt_bvh_node& o = nodes_out[i];
    for (int k = 0; k < 3; ++k) { o.aabb_min[k] = nd.lo[k]; o.aabb_max[k] = nd.hi[k]; }
    o.num_triangles = nd.num;
    o.next = nd.num > 0 ? nd.obj : nd.next;
  }
  *n_nodes = (uint32_t)nodes.size();
  return WGPT_OK;
}

int wgpt_build_env_cdf(const uint16_t* data, uint32_t width, uint32_t height, double exposure_f, float* cdf,
                       double* total_weight) {
  if (!data || !cdf || width == 0 || height == 0) return WGPT_E_INVALID;
  const double exposure = exposure_f;
  const double threshold = 65536 - 16 - 1;   // tracer.js:30
  const size_t marg = (size_t)height + 1;
  float* margCDF = cdf;
  float* condCDF = cdf + marg;
  double total = 0;
  margCDF[0] = 0;
  for (uint32_t y = 0; y < height; ++y) {
    double row = 0;
    const double sin_theta = sin(M_PI * (y + 0.5) / height);
    float* rowp = condCDF + (size_t)y * (width + 1);
    rowp[0] = 0;
    for (uint32_t x = 0; x < width; ++x) {
      const uint16_t* t = data + ((size_t)y * width + x) * 4;
      double r = std::min(half_to_double(t[0]) * exposure, threshold);
      double g = std::min(half_to_double(t[1]) * exposure, threshold);
      double b = std::min(half_to_double(t[2]) * exposure, threshold);
      double lum = (0.2126 * r + 0.7152 * g + 0.0722 * b) * sin_theta;
      row += lum;
      rowp[x + 1] = (float)row;
    }
    if (row > 0) {
      for (uint32_t x = 1; x <= width; ++x) rowp[x] = (float)((double)rowp[x] / row);
    } else {
      for (uint32_t x = 1; x <= width; ++x) rowp[x] = (float)((double)x / width);
    }
    total += row;
    margCDF[y + 1] = (float)total;
  }
  if (total > 0) {
    for (uint32_t y = 1; y <= height; ++y) margCDF[y] = (float)((double)margCDF[y] / total);
  } else {
    for (uint32_t y = 1; y <= height; ++y) margCDF[y] = (float)((double)y / height);
  }
  if (total_weight) *total_weight = total;
  return WGPT_OK;
}

// Alias table (Walker / Vose) over the texels of the environment, from the same FP64 weights as
// buildHDRCDF (luminance of the clamped, exposed texel times the row's sin(theta)): texel i is
// drawn with probability w_i / sum(w) by picking a bin uniformly and keeping it with probability
// prob[i], else taking alias[i].  A zero total draws texels uniformly.
int wgpt_build_env_alias(const uint16_t* data, uint32_t width, uint32_t height, double exposure_f, float* prob,
                         uint32_t* alias) {
  if (!data || !prob || !alias || width == 0 || height == 0) return WGPT_E_INVALID;
  const double exposure = exposure_f;
  const double threshold = 65536 - 16 - 1;   // tracer.js:30
  const size_t n = (size_t)width * height;
  std::vector<double> w(n);
  double total = 0;
  for (uint32_t y = 0; y < height; ++y) {
    const double sin_theta = sin(M_PI * (y + 0.5) / height);
    for (uint32_t x = 0; x < width; ++x) {
      const uint16_t* t = data + ((size_t)y * width + x) * 4;
      double r = std::min(half_to_double(t[0]) * exposure, threshold);
      double g = std::min(half_to_double(t[1]) * exposure, threshold);
      double b = std::min(half_to_double(t[2]) * exposure, threshold);
      double lum = (0.2126 * r + 0.7152 * g + 0.0722 * b) * sin_theta;
      w[(size_t)y * width + x] = lum;
      total += lum;
    }
  }
  if (!(total > 0) || !std::isfinite(total)) {
    for (size_t i = 0; i < n; ++i) { prob[i] = 1.0f; alias[i] = (uint32_t)i; }
    return WGPT_OK;
  }
  std::vector<double> scaled(n);
  std::vector<uint32_t> small, large;
  small.reserve(n);
  large.reserve(n);
  for (size_t i = 0; i < n; ++i) {
    scaled[i] = std::max(w[i], 0.0) * (double)n / total;
    (scaled[i] < 1.0 ? small : large).push_back((uint32_t)i);
  }
  while (!small.empty() && !large.empty()) {
    const uint32_t sm = small.back(), lg = large.back();
    small.pop_back();
    large.pop_back();
    prob[sm] = (float)scaled[sm];
    alias[sm] = lg;
    scaled[lg] = (scaled[lg] + scaled[sm]) - 1.0;
    (scaled[lg] < 1.0 ? small : large).push_back(lg);
  }
  for (uint32_t i : large) { prob[i] = 1.0f; alias[i] = i; }
  for (uint32_t i : small) { prob[i] = 1.0f; alias[i] = i; }   // rounding leftovers
  return WGPT_OK;
}

int wgpt_decode_rgbe(const uint8_t* buf, size_t len, double exposure_f, uint16_t* out, uint32_t* w_out, uint32_t* h_out) {
  if (!buf || !w_out || !h_out) return WGPT_E_INVALID;
  size_t off = 0;
  auto read_line = [&]() {
    std::string s;
    while (off < len) {
      uint8_t b = buf[off];
      if (b == 10) { ++off; break; }
      s.push_back((char)b);
      ++off;
    }
    return s;
  };
  uint32_t width = 0, height = 0;
  bool rle = false;
  for (int i = 0; i < 20; ++i) {
    std::string line = read_line();
    if (line.find("#?RADIANCE") != std::string::npos) continue;
    if (line.find("FORMAT=32-bit_rle_rgbe") != std::string::npos) { rle = true; continue; }
    if (line.find("EXPOSURE=") != std::string::npos) continue;
    if (line.find('#') != std::string::npos) continue;
    size_t p = line.find("-Y ");
    if (p != std::string::npos) {
      unsigned hh = 0, ww = 0;
      if (sscanf(line.c_str() + p, "-Y %u +X %u", &hh, &ww) == 2) { height = hh; width = ww; break; }
    }
  }
  if (!rle) return WGPT_E_INVALID;   // "File is not run length encoded!"
  if (width == 0 || height == 0 || width > 32768 || height > 32768) return WGPT_E_INVALID;
  *w_out = width; *h_out = height;
  if (!out) return WGPT_OK;
  std::vector<uint8_t> data((size_t)width * height * 4);
  std::vector<uint8_t> scan((size_t)width * 4);
  size_t doff = 0;
  uint32_t lines = height;
  // readPixelsRawRLE, lib/parse-hdr.js:20-122
  while (lines > 0) {
    if (off + 4 > len) return WGPT_E_INVALID;
    uint8_t rgbe[4] = {buf[off], buf[off + 1], buf[off + 2], buf[off + 3]};
    off += 4;
    if (rgbe[0] != 2 || rgbe[1] != 2 || (rgbe[2] & 0x80) != 0) {
      // flat (non-RLE) pixels for the rest of the image
      memcpy(&data[doff], rgbe, 4);
      doff += 4;
      size_t need = ((size_t)width * lines - 1) * 4;
      if (off + need > len) return WGPT_E_INVALID;
      memcpy(&data[doff], buf + off, need);
      off += need;
      break;
    }
    if ((((uint32_t)rgbe[2] << 8) | rgbe[3]) != width) return WGPT_E_INVALID;
    size_t ptr = 0;
    for (int ch = 0; ch < 4; ++ch) {
      size_t end = (size_t)(ch + 1) * width;
      while (ptr < end) {
        if (off + 2 > len) return WGPT_E_INVALID;
        uint8_t b0 = buf[off], b1 = buf[off + 1];
        off += 2;
        if (b0 > 128) {
          size_t count = b0 - 128;
          if (count == 0 || count > end - ptr) return WGPT_E_INVALID;
          while (count-- > 0) scan[ptr++] = b1;
        } else {
          size_t count = b0;
          if (count == 0 || count > end - ptr) return WGPT_E_INVALID;
          scan[ptr++] = b1;
          if (--count > 0) {
            if (off + count > len) return WGPT_E_INVALID;
            memcpy(&scan[ptr], buf + off, count);
            ptr += count;
            off += count;
          }
        }
      }
    }
    for (uint32_t i = 0; i < width; ++i) {
      data[doff + 0] = scan[i];
      data[doff + 1] = scan[i + width];
      data[doff + 2] = scan[i + 2 * width];
      data[doff + 3] = scan[i + 3 * width];
      doff += 4;
    }
    --lines;
  }
  // float conversion (lib/parse-hdr.js:186-203) then updateData (tracer.js:76-87)
  const double exposure = exposure_f;
  const double threshold = 65536 - 16 - 1;
  for (size_t i = 0; i < (size_t)width * height; ++i) {
    const uint8_t* p = &data[i * 4];
    double f = ldexp(1.0, (int)p[3] - 128);
    for (int k = 0; k < 3; ++k) {
      float v = (float)(((double)p[k] / 255) * f);   // Float32Array store
      out[i * 4 + k] = double_to_half(std::min((double)v * exposure, threshold));
    }
    out[i * 4 + 3] = double_to_half(1.0);
  }
  return WGPT_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------- OBJ
// Model.parseOBJ + generateTriangles (tracer.js:949-1021): positions (v), texture coordinates
// (vt) and normals (vn) as JavaScript numbers, faces (f) as 1-based v/vt/vn index triples,
// polygons fan-triangulated from their first vertex.  Triangles come out as the 24 floats the
// BLAS builder takes (v0 v1 v2 n0 n1 n2 uv0 uv1 uv2), each value rounded to float32 the way the
// reference's Float32Array does.  Where the reference indexes outside its arrays (a missing vt or
// vn, an index out of range, a negative relative index, an unparsable number) it reads
// `undefined`, which a Float32Array stores as NaN; the same NaN is produced here.
namespace {

bool js_space(unsigned char c) { return c == ' ' || c == '\t' || c == '\r' || c == '\n' || c == '\v' || c == '\f'; }

// parseFloat: the longest prefix that is a decimal literal or "Infinity" (after leading white
// space and an optional sign); NaN when there is none.
double js_parse_float(const std::string& s) {
  size_t i = 0, n = s.size();
  while (i < n && js_space((unsigned char)s[i])) ++i;
  size_t start = i;
  if (i < n && (s[i] == '+' || s[i] == '-')) ++i;
  if (s.compare(i, 8, "Infinity") == 0) {
    return s[start] == '-' ? -HUGE_VAL : HUGE_VAL;
  }
  size_t digits = 0, j = i;
  while (j < n && isdigit((unsigned char)s[j])) { ++j; ++digits; }
  if (j < n && s[j] == '.') {
    ++j;
    while (j < n && isdigit((unsigned char)s[j])) { ++j; ++digits; }
  }
  if (digits == 0) return NAN;
  if (j < n && (s[j] == 'e' || s[j] == 'E')) {
    size_t k = j + 1;
    if (k < n && (s[k] == '+' || s[k] == '-')) ++k;
    size_t kd = k;
    while (k < n && isdigit((unsigned char)s[k])) ++k;
    if (k > kd) j = k;
  }
  return strtod(s.substr(start, j - start).c_str(), nullptr);
}

// parseInt without a radix: optional sign, "0x" selects hexadecimal, then the longest run of
// digits; NaN when there is none.
double js_parse_int(const std::string& s) {
  size_t i = 0, n = s.size();
  while (i < n && js_space((unsigned char)s[i])) ++i;
  double sign = 1.0;
  if (i < n && (s[i] == '+' || s[i] == '-')) { if (s[i] == '-') sign = -1.0; ++i; }
  int base = 10;
  if (i + 1 < n && s[i] == '0' && (s[i + 1] == 'x' || s[i + 1] == 'X')) { base = 16; i += 2; }
  double v = 0.0;
  size_t digits = 0;
  for (; i < n; ++i) {
    int d;
    char c = s[i];
    if (c >= '0' && c <= '9') d = c - '0';
    else if (base == 16 && c >= 'a' && c <= 'f') d = c - 'a' + 10;
    else if (base == 16 && c >= 'A' && c <= 'F') d = c - 'A' + 10;
    else break;
    v = v * base + d;
    ++digits;
  }
  return digits ? sign * v : NAN;
}

// array[index] of a JavaScript array of numbers: undefined (NaN once stored) unless the index is
// a non-negative integer inside the array.
float js_at(const std::vector<double>& a, double index) {
  if (!(index >= 0.0) || index != std::floor(index) || index >= (double)a.size()) return NAN;
  return (float)a[(size_t)index];
}

}  // namespace

extern "C" int wgpt_parse_obj(const char* text, size_t bytes, float* tris24, uint32_t capacity, uint32_t* n_tris,
                              float* positions, uint32_t pos_capacity, uint32_t* n_positions) {
  if ((!text && bytes) || !n_tris) return WGPT_E_INVALID;
  std::vector<double> P, U, N;
  std::vector<double> fp, fu, fn;   // per triangle corner: position, uv, normal index (0-based)
  size_t pos = 0;
  std::vector<std::string> parts;
  while (pos <= bytes) {
    size_t end = pos;
    while (end < bytes && text[end] != '\n') ++end;
    // line.trim().split(/\s+/)
    size_t a = pos, b = end;
    while (a < b && js_space((unsigned char)text[a])) ++a;
    while (b > a && js_space((unsigned char)text[b - 1])) --b;
    parts.clear();
    size_t k = a;
    while (true) {
      size_t t = k;
      while (t < b && !js_space((unsigned char)text[t])) ++t;
      parts.emplace_back(text + k, t - k);
      if (t >= b) break;
      k = t;
      while (k < b && js_space((unsigned char)text[k])) ++k;
    }
    const std::string& type = parts[0];
    auto part = [&](size_t i) -> std::string { return i < parts.size() ? parts[i] : std::string(); };
    if (type == "v") {
      P.push_back(js_parse_float(part(1))); P.push_back(js_parse_float(part(2))); P.push_back(js_parse_float(part(3)));
    } else if (type == "vt") {
      U.push_back(js_parse_float(part(1))); U.push_back(js_parse_float(part(2)));
    } else if (type == "vn") {
      N.push_back(js_parse_float(part(1))); N.push_back(js_parse_float(part(2))); N.push_back(js_parse_float(part(3)));
    } else if (type == "f") {
      struct Corner { double v, u, n; };
      std::vector<Corner> face;
      for (size_t i = 1; i < parts.size(); ++i) {
        std::vector<std::string> idx;
        size_t s0 = 0;
        const std::string& p = parts[i];
        while (true) {
          size_t sl = p.find('/', s0);
          idx.push_back(p.substr(s0, sl == std::string::npos ? std::string::npos : sl - s0));
          if (sl == std::string::npos) break;
          s0 = sl + 1;
        }
        Corner c;
        c.v = js_parse_int(idx[0]) - 1.0;
        c.u = idx.size() > 1 && !idx[1].empty() ? js_parse_int(idx[1]) - 1.0 : -1.0;
        c.n = idx.size() > 2 && !idx[2].empty() ? js_parse_int(idx[2]) - 1.0 : -1.0;
        face.push_back(c);
      }
      for (size_t i = 1; i + 1 < face.size(); ++i) {
        const Corner* cs[3] = {&face[0], &face[i], &face[i + 1]};
        for (const Corner* c : cs) { fp.push_back(c->v); fu.push_back(c->u); fn.push_back(c->n); }
      }
    }
    if (end >= bytes) break;
    pos = end + 1;
  }
  // Int32Array stores of the face indices: NaN becomes 0, values wrap to 32 bits
  auto i32 = [](double x) -> double {
    if (!std::isfinite(x)) return 0.0;
    double t = std::trunc(x);
    double m = std::fmod(t, 4294967296.0);
    if (m < 0) m += 4294967296.0;
    return m >= 2147483648.0 ? m - 4294967296.0 : m;
  };
  const size_t ntri = fp.size() / 3;
  *n_tris = (uint32_t)ntri;
  if (n_positions) *n_positions = (uint32_t)P.size();
  if (positions) {
    if (pos_capacity < P.size()) return WGPT_E_INVALID;
    for (size_t i = 0; i < P.size(); ++i) positions[i] = (float)P[i];
  }
  if (!tris24) return WGPT_OK;
  if (capacity < ntri) return WGPT_E_INVALID;
  for (size_t t = 0; t < ntri; ++t) {
    float* o = tris24 + t * 24;
    for (int c = 0; c < 3; ++c) {
      double ip = i32(fp[t * 3 + c]), in = i32(fn[t * 3 + c]), iu = i32(fu[t * 3 + c]);
      for (int d = 0; d < 3; ++d) o[c * 3 + d] = js_at(P, ip * 3 + d);
      for (int d = 0; d < 3; ++d) o[9 + c * 3 + d] = js_at(N, in * 3 + d);
      for (int d = 0; d < 2; ++d) o[18 + c * 2 + d] = js_at(U, iu * 2 + d);
    }
  }
  return WGPT_OK;
}
