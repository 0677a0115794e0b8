// Learned kernel-predicting denoiser: BF16 tensor-core GEMM entry point (this file grows into
// the network's forward/backward kernels).
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>
#include <string.h>

#include "../../include/wgpt.h"
#include "wgpt_internal.h"
#include "tc_gemm.cuh"
#include "conv_ws.cuh"

namespace kp {

// Row-major BF16 matrix (K contiguous), zero outside rows x k.
struct RowMajor {
  const uint16_t* p;
  int rows, k, ld;
  __device__ __forceinline__ uint4 chunk(int row, int k8) const {
    if (row >= rows || k8 * 8 >= k) return make_uint4(0u, 0u, 0u, 0u);
    return *reinterpret_cast<const uint4*>(p + (size_t)row * ld + k8 * 8);
  }
  template <int ROWS>
  __device__ __forceinline__ void fill(uint8_t* tile, int row0, int k0, int tid) const {
    tc::fill_chunks<ROWS>(*this, tile, row0, k0, tid);
  }
};

struct StoreF32 {
  float* c;
  int ldc, n;
  __device__ __forceinline__ void operator()(int row, int col0, const float (&v)[16]) const {
#pragma unroll
    for (int i = 0; i < 16; ++i)
      if (col0 + i < n) c[(size_t)row * ldc + col0 + i] = v[i];
  }
};

template <int BN, class LA, class LB, class EP>
cudaError_t launch_gemm(const LA& la, const LB& lb, const EP& ep, int M, int N, int K, uint32_t* err,
                        cudaStream_t st) {
  auto kern = tc::k_tc_gemm<BN, LA, LB, EP>;
  const int smem = tc::Smem<BN>::BYTES;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  const int kt_all = (K + tc::BK - 1) / tc::BK;
  dim3 grid((unsigned)((M + tc::BM - 1) / tc::BM), (unsigned)((N + BN - 1) / BN), 1u);
  kern<<<grid, tc::THREADS, smem, st>>>(la, lb, ep, M, N, K, kt_all, err);
  return cudaGetLastError();
}

}  // namespace kp

extern "C" int wgpt_gemm_bf16(int device, const uint16_t* a, const uint16_t* b, float* c, int m, int n, int k) {
  if (!a || !b || !c || m <= 0 || n <= 0 || k <= 0 || (k % 8) != 0) return WGPT_E_INVALID;
  if (wgpt::select_device(device) != cudaSuccess) return WGPT_E_CUDA;
  uint16_t *da = nullptr, *db = nullptr;
  float* dc = nullptr;
  uint32_t* derr = nullptr;
  size_t sa = (size_t)m * k * 2, sb = (size_t)n * k * 2, sc = (size_t)m * n * 4;
  int rc = WGPT_OK;
  cudaError_t e = cudaMalloc(&da, sa);
  if (e == cudaSuccess) e = cudaMalloc(&db, sb);
  if (e == cudaSuccess) e = cudaMalloc(&dc, sc);
  if (e == cudaSuccess) e = cudaMalloc(&derr, 4);
  if (e == cudaSuccess) e = cudaMemset(derr, 0, 4);
  if (e == cudaSuccess) e = cudaMemcpy(da, a, sa, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(db, b, sb, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    kp::RowMajor la{da, m, k, k}, lb{db, n, k, k};
    kp::StoreF32 ep{dc, n, n};
    if (n <= 32) e = kp::launch_gemm<32>(la, lb, ep, m, n, k, derr, 0);
    else if (n <= 64) e = kp::launch_gemm<64>(la, lb, ep, m, n, k, derr, 0);
    else if (n <= 128) e = kp::launch_gemm<128>(la, lb, ep, m, n, k, derr, 0);
    else e = kp::launch_gemm<256>(la, lb, ep, m, n, k, derr, 0);
  }
  uint32_t herr = 0;
  if (e == cudaSuccess) e = cudaMemcpy(c, dc, sc, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(&herr, derr, 4, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) rc = e == cudaErrorMemoryAllocation ? WGPT_E_NOMEM : WGPT_E_CUDA;
  else if (herr) rc = WGPT_E_DEVICE;
  cudaFree(da); cudaFree(db); cudaFree(dc); cudaFree(derr);
  return rc;
}

// ============================================================================================
// Kernel-predicting convolutional denoiser (KPCN).
//
// A 5-level encoder-decoder over 10 input features (log colour, albedo, normal, depth) predicts
// per pixel three 5x5 filters (softmax over 25 logits each) applied to the noisy linear colour
// as a cascade at dilations 1, 2 and 4.
// Activations are NHWC BF16 with channel counts padded to multiples of 16; every convolution
// (forward, data gradient, weight gradient) is one tensor-core GEMM whose loaders gather the
// implicit im2col operand straight from the NHWC tensors (2x nearest upsampling and the skip
// concatenation of the decoder are folded into the gather).  Weights are FP32 masters with BF16
// copies for the GEMMs, trained by Adam on a relative-L2 loss.
//
// Layer table (channels, resolution level):
//   E0a 10(16)->32 L0   E0 32->32 L0   E1 32->48 L1   E2 48->64 L2   E3 64->96 L3
//   E4a 96->128 L4      E4 128->128 L4
//   D3 [up E4 128, E3 96]->96 L3   D2 [up D3 96, E2 64]->64 L2   D1 [up D2 64, E1 48]->48 L1
//   D0 [up D1 48, E0 32]->32 L0    OUT 1x1 32->75(80) L0
// with 2x2 average pooling between encoder levels (E0->P1, E1->P2, E2->P3, E3->P4).
// ============================================================================================
#include <algorithm>
#include <cmath>
#include <vector>

namespace kp {

__device__ __forceinline__ uint16_t f2bf(float x) { return __bfloat16_as_ushort(__float2bfloat16_rn(x)); }
__device__ __forceinline__ float bf2f(uint16_t b) { return __uint_as_float((uint32_t)b << 16); }
__device__ __forceinline__ uint4 zero4() { return make_uint4(0u, 0u, 0u, 0u); }

// 8-channel vectors of a convolution's input: a coarse tensor read 2x-upsampled (nearest),
// channels [0, cu), concatenated with a tensor at the output resolution, channels [cu, cu+cs).
struct ConvSrc {
  const uint16_t* u;
  int cu, hc, wc;
  const uint16_t* s;
  int cs;
  int h, w;      // output resolution of one image
  int taps;      // 9 (3x3, padding 1) or 1
  int sign;      // +1: neighbour at p + offset (forward, weight gradient); -1: p - offset (data gradient)
  __device__ __forceinline__ uint4 vec(int p, int tap, int ci0) const {
    const int hw = h * w;
    const int b = p / hw;
    const int r = p - b * hw;
    int y = r / w, x = r - (r / w) * w;
    if (taps == 9) {
      y += sign * (tap / 3 - 1);
      x += sign * (tap % 3 - 1);
    }
    return vec_at(b, y, x, ci0);
  }
  // Address of the vector at (image b, row y, column x) of the output grid (null outside).
  __device__ __forceinline__ const uint16_t* ptr_at(int b, int y, int x, int ci0) const {
    if (y < 0 || y >= h || x < 0 || x >= w) return nullptr;
    if (ci0 < cu) return u + (((size_t)b * hc + (y >> 1)) * wc + (x >> 1)) * cu + ci0;
    return s + (((size_t)b * h + y) * w + x) * cs + (ci0 - cu);
  }
  // The vector at (image b, row y, column x) of the output grid (zero outside the image).
  __device__ __forceinline__ uint4 vec_at(int b, int y, int x, int ci0) const {
    if (y < 0 || y >= h || x < 0 || x >= w) return zero4();
    if (ci0 < cu) {
      size_t q = ((size_t)b * hc + (y >> 1)) * wc + (x >> 1);
      return *reinterpret_cast<const uint4*>(u + q * cu + ci0);
    }
    size_t q = ((size_t)b * h + y) * w + x;
    return *reinterpret_cast<const uint4*>(s + q * cs + (ci0 - cu));
  }
};

// A operand of a convolution: row = output pixel, k = tap * cin + ci.
struct ConvA {
  ConvSrc src;
  int P, cin;
  __device__ __forceinline__ uint4 chunk(int row, int k8) const {
    if (row >= P) return zero4();
    const int k = k8 * 8, tap = k / cin;
    if (tap >= src.taps) return zero4();
    return src.vec(row, tap, k - tap * cin);
  }
  template <int ROWS>
  __device__ __forceinline__ void fill(uint8_t* tile, int row0, int k0, int tid) const {
    tc::fill_chunks<ROWS>(*this, tile, row0, k0, tid);
  }
};

// Weight gradient, A operand: row = output channel co, k = pixel; dZ is NHWC [P][cout], so 8
// consecutive channels of one pixel are one 16-byte vector: the tile is stored MN-major.  Each
// group of 8 threads takes 8 consecutive pixels of one channel group (one 128-byte core matrix in
// shared memory); consecutive groups take the next channel group of the same pixels.
struct WgradA {
  static constexpr bool kMnMajor = true;
  const uint16_t* dz;
  int cout, P;
  template <int ROWS>
  __device__ __forceinline__ void fill(uint8_t* tile, int row0, int k0, int tid) const {
    const int G = ROWS / 8;
    for (int i = tid; i < G * tc::BK; i += tc::THREADS) {
      const int grp = i >> 3, g = grp % G, j = (grp / G) * 8 + (i & 7), p = k0 + j, co0 = row0 + g * 8;
      uint4 v = zero4();
      if (p < P && co0 < cout) v = *reinterpret_cast<const uint4*>(dz + (size_t)p * cout + co0);
      tc::put_mn8(tile, g * 8, j, v);
    }
  }
  static constexpr bool kAsync = true;
  template <int ROWS>
  __device__ __forceinline__ void fill_async(uint8_t* tile, int row0, int k0, int tid) const {
    const int G = ROWS / 8;
    const uint32_t base = tc::smem_u32(tile);
    for (int i = tid; i < G * tc::BK; i += tc::THREADS) {
      const int grp = i >> 3, g = grp % G, j = (grp / G) * 8 + (i & 7), p = k0 + j, co0 = row0 + g * 8;
      const bool in = p < P && co0 < cout;
      tc::cp_async_16(base + (uint32_t)(((g * (tc::BK / 8)) + (j >> 3)) * 128 + (j & 7) * 16),
                      in ? dz + (size_t)p * cout + co0 : dz, in ? 16u : 0u);
    }
  }
};

// Weight gradient, B operand: row n = tap * cin + ci, k = pixel; the input gathered at the tap
// (8 consecutive input channels of one pixel per vector; MN-major like WgradA).  With 128 rows
// and 128 threads, thread t always fills rows 8 * (t / 8) .. + 8 (one tap and channel group)
// at pixels k0 + (t % 8) + 8 * i, i = 0..7: the tap and the first pixel's position are divided
// out once, later pixels are stepped by 8.
struct WgradB {
  static constexpr bool kMnMajor = true;
  ConvSrc src;
  int cin, P, n_total;
  template <int ROWS>
  __device__ __forceinline__ void fill(uint8_t* tile, int row0, int k0, int tid) const {
    static_assert(ROWS == 128 && tc::THREADS == 128 && tc::BK == 64, "one channel group per thread");
    const int g = tid >> 3, n = row0 + g * 8;
    const bool n_ok = n < n_total;
    const int tap = n_ok ? n / cin : 0, ci0 = n - tap * cin;
    const int dy = src.taps == 9 ? src.sign * (tap / 3 - 1) : 0;
    const int dx = src.taps == 9 ? src.sign * (tap % 3 - 1) : 0;
    const int hw = src.h * src.w;
    int p = k0 + (tid & 7);
    int b = p / hw, r = p - b * hw, y = r / src.w, x = r - (r / src.w) * src.w;
#pragma unroll
    for (int it = 0; it < 8; ++it) {
      uint4 v = zero4();
      if (n_ok && p < P) v = src.vec_at(b, y + dy, x + dx, ci0);
      tc::put_mn8(tile, g * 8, it * 8 + (tid & 7), v);
      p += 8;
      x += 8;
      while (x >= src.w) {
        x -= src.w;
        if (++y == src.h) { y = 0; ++b; }
      }
    }
  }
  static constexpr bool kAsync = true;
  template <int ROWS>
  __device__ __forceinline__ void fill_async(uint8_t* tile, int row0, int k0, int tid) const {
    static_assert(ROWS == 128 && tc::THREADS == 128 && tc::BK == 64, "one channel group per thread");
    const int g = tid >> 3, n = row0 + g * 8;
    const bool n_ok = n < n_total;
    const int tap = n_ok ? n / cin : 0, ci0 = n - tap * cin;
    const int dy = src.taps == 9 ? src.sign * (tap / 3 - 1) : 0;
    const int dx = src.taps == 9 ? src.sign * (tap % 3 - 1) : 0;
    const int hw = src.h * src.w;
    int p = k0 + (tid & 7);
    int b = p / hw, r = p - b * hw, y = r / src.w, x = r - (r / src.w) * src.w;
    const uint32_t base = tc::smem_u32(tile) + (uint32_t)(g * (tc::BK / 8) * 128);
#pragma unroll
    for (int it = 0; it < 8; ++it) {
      const uint16_t* q = (n_ok && p < P) ? src.ptr_at(b, y + dy, x + dx, ci0) : nullptr;
      const int j = it * 8 + (tid & 7);
      tc::cp_async_16(base + (uint32_t)((j >> 3) * 128 + (j & 7) * 16), q ? q : (src.s ? src.s : src.u), q ? 16u : 0u);
      p += 8;
      x += 8;
      while (x >= src.w) {
        x -= src.w;
        if (++y == src.h) { y = 0; ++b; }
      }
    }
  }
};

// bias + optional ReLU, BF16 NHWC store of 16 channels.
struct EpiAct {
  uint16_t* y;
  const float* bias;
  int cstride, relu;
  __device__ __forceinline__ void operator()(int row, int col0, const float (&v)[16]) const {
    uint32_t w[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      float a = v[2 * i] + bias[col0 + 2 * i], b = v[2 * i + 1] + bias[col0 + 2 * i + 1];
      if (relu) { a = fmaxf(a, 0.0f); b = fmaxf(b, 0.0f); }
      w[i] = (uint32_t)f2bf(a) | ((uint32_t)f2bf(b) << 16);
    }
    uint4* dst = reinterpret_cast<uint4*>(y + (size_t)row * cstride + col0);
    dst[0] = make_uint4(w[0], w[1], w[2], w[3]);
    dst[1] = make_uint4(w[4], w[5], w[6], w[7]);
  }
};

// bias, FP32 store (filter logits).
struct EpiLogits {
  float* y;
  const float* bias;
  int cstride;
  __device__ __forceinline__ void operator()(int row, int col0, const float (&v)[16]) const {
    float4* dst = reinterpret_cast<float4*>(y + (size_t)row * cstride + col0);
#pragma unroll
    for (int i = 0; i < 4; ++i)
      dst[i] = make_float4(v[4 * i] + bias[col0 + 4 * i], v[4 * i + 1] + bias[col0 + 4 * i + 1],
                           v[4 * i + 2] + bias[col0 + 4 * i + 2], v[4 * i + 3] + bias[col0 + 4 * i + 3]);
  }
};

// BF16 store without bias (data gradients).
struct EpiStore {
  uint16_t* y;
  int cstride;
  __device__ __forceinline__ void operator()(int row, int col0, const float (&v)[16]) const {
    uint32_t w[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) w[i] = (uint32_t)f2bf(v[2 * i]) | ((uint32_t)f2bf(v[2 * i + 1]) << 16);
    uint4* dst = reinterpret_cast<uint4*>(y + (size_t)row * cstride + col0);
    dst[0] = make_uint4(w[0], w[1], w[2], w[3]);
    dst[1] = make_uint4(w[4], w[5], w[6], w[7]);
  }
};

// FP32 atomic accumulation (split-K weight gradients).
struct EpiAtomic {
  float* dw;
  int ld, ncols;
  __device__ __forceinline__ void operator()(int row, int col0, const float (&v)[16]) const {
#pragma unroll
    for (int i = 0; i < 16; ++i)
      if (col0 + i < ncols && v[i] != 0.0f) atomicAdd(dw + (size_t)row * ld + col0 + i, v[i]);
  }
};

// ---------------------------------------------------------------------------- 3x3 halo convolution
// A 3x3 convolution (padding 1) as 9 shifted GEMMs over one shared-memory halo tile: a CTA owns a
// 16 x 16 block of output pixels as two 128-pixel M tiles (8 wide x 16 tall each) and an NT-wide
// slice of the output channels.  Per 16 input channels it loads the 18 x 18 halo once (two 8-
// channel planes of 16-byte pixel vectors) and the weights of all 9 taps; tap (dy, dx) is then
// just a descriptor offset into the halo: 8 consecutive pixels of an output row are 8 consecutive
// 16-byte halo vectors (a core matrix), the next output row is 18 vectors further (SBO) and the
// next 8 channels one plane further (LBO).  Each input value is read from global memory about
// 1.3 times instead of 9 times.  Two accumulators (one per M tile) live in tensor memory.
constexpr int HALO_W = 18, HALO_P = HALO_W * HALO_W;

struct HaloSrc {
  const uint16_t* u;   // coarse tensor read 2x upsampled, channels [0, cu)
  int cu, hc, wc;
  const uint16_t* s;   // tensor at the output resolution, channels [cu, cu + cs)
  int cs;
  int h, w;
  __device__ __forceinline__ uint4 at(int b, int y, int x, int ci0) const {
    if (y < 0 || y >= h || x < 0 || x >= w) return zero4();
    if (ci0 < cu) return *reinterpret_cast<const uint4*>(u + (((size_t)b * hc + (y >> 1)) * wc + (x >> 1)) * cu + ci0);
    return *reinterpret_cast<const uint4*>(s + (((size_t)b * h + y) * w + x) * cs + (ci0 - cu));
  }
};

template <int NT>
struct HaloSmem {
  static constexpr int HALO = 2 * HALO_P * 16;   // 16 channels
  static constexpr int WTS = 9 * NT * 32;        // per tap: NT rows x 16 channels
  static constexpr int STAGE = HALO + WTS;
  static constexpr int BYTES = 2 * STAGE + 64;
};

// wb: [N][9][cin] BF16 weights (output channel, tap, input channel); grid (ceil(w/16),
// ceil(h/16), images * ceil(N/NT)); the epilogue gets (pixel index, first column, 16 values).
template <int NT, class EP>
__global__ void __launch_bounds__(tc::THREADS) k_conv3x3(HaloSrc src, const uint16_t* __restrict__ wb, int cin, int N,
                                                        EP ep, uint32_t* err) {
  extern __shared__ __align__(1024) uint8_t smem[];
  using S = HaloSmem<NT>;
  const int tid = threadIdx.x, warp = tid >> 5;
  const int ntiles = (N + NT - 1) / NT;
  const int b = blockIdx.z / ntiles, n0 = (blockIdx.z % ntiles) * NT;
  const int x0 = blockIdx.x * 16, y0 = blockIdx.y * 16;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + 2 * S::STAGE);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + 2 * S::STAGE + 16);
  volatile uint32_t* flag = reinterpret_cast<volatile uint32_t*>(smem + 2 * S::STAGE + 20);
  const uint32_t bar0 = tc::smem_u32(&bars[0]), bar1 = tc::smem_u32(&bars[1]);
  constexpr uint32_t NCOLS = tc::tmem_cols(2 * NT);
  if (warp == 0) tc::tmem_alloc(tc::smem_u32(tmem_slot), NCOLS);
  if (tid == 0) {
    tc::mbar_init(bar0, 1);
    tc::mbar_init(bar1, 1);
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const int KT = cin / 16;
  constexpr uint32_t IDESC = tc::idesc_bf16(NT);
  bool ok = true;
  int committed = 0;
  for (int kt = 0; kt < KT; ++kt) {
    const int st = kt & 1;
    uint8_t* halo = smem + st * S::STAGE;
    uint8_t* wts = halo + S::HALO;
    if (kt >= 2) {
      if (tid == 0) *flag = tc::mbar_wait(st ? bar1 : bar0, (uint32_t)((kt >> 1) - 1) & 1u) ? 1u : 0u;
      __syncthreads();
      if (*flag == 0u) { ok = false; break; }
    }
    const int ci = kt * 16;
    for (int i = tid; i < 2 * HALO_P; i += tc::THREADS) {
      const int c = i / HALO_P, q = i - c * HALO_P, hy = q / HALO_W, hx = q - hy * HALO_W;
      *reinterpret_cast<uint4*>(halo + i * 16) = src.at(b, y0 - 1 + hy, x0 - 1 + hx, ci + c * 8);
    }
    for (int i = tid; i < 9 * NT * 2; i += tc::THREADS) {
      const int c = i & 1, n = (i >> 1) % NT, t = (i >> 1) / NT, gn = n0 + n;
      uint4 v = zero4();
      if (gn < N) v = *reinterpret_cast<const uint4*>(wb + ((size_t)gn * 9 + t) * cin + ci + c * 8);
      *reinterpret_cast<uint4*>(wts + t * NT * 32 + ((n >> 3) * 2 + c) * 128 + (n & 7) * 16) = v;
    }
    tc::fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      tc::tc_fence_after();
      const uint32_t ha = tc::smem_u32(halo), wa = tc::smem_u32(wts);
#pragma unroll
      for (int t = 0; t < 9; ++t) {
        const int dy = t / 3, dx = t % 3;
        const uint64_t db = tc::smem_desc(wa + t * NT * 32, 128, 256);
#pragma unroll
        for (int m = 0; m < 2; ++m) {
          const uint64_t da = tc::smem_desc(ha + (dy * HALO_W + 8 * m + dx) * 16, HALO_P * 16, HALO_W * 16);
          tc::mma_bf16(tmem + (uint32_t)(m * NT), da, db, IDESC, (kt > 0 || t > 0) ? 1u : 0u);
        }
      }
      tc::mma_commit(st ? bar1 : bar0);
    }
    committed = kt + 1;
  }
  if (tid == 0) {
    const int last = committed - 1;
    *flag = committed == 0 || tc::mbar_wait((last & 1) ? bar1 : bar0, (uint32_t)(last >> 1) & 1u) ? 1u : 0u;
  }
  __syncthreads();
  ok = ok && *flag != 0u;
  if (!ok) {
    if (tid == 0) atomicOr(err, tc::ERR_TC_TIMEOUT);
  } else if (KT > 0) {
    tc::tc_fence_after();
    const int r = warp * 32 + (tid & 31), ty = r >> 3, tx = r & 7, y = y0 + ty;
#pragma unroll
    for (int m = 0; m < 2; ++m) {
      const int x = x0 + 8 * m + tx;
      for (int c0 = 0; c0 < NT; c0 += 16) {
        float v[16];
        tc::tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(m * NT + c0), v);
        if (y < src.h && x < src.w && n0 + c0 < N) ep((int)(((size_t)b * src.h + y) * src.w + x), n0 + c0, v);
      }
    }
  }
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 0) tc::tmem_free(tmem, NCOLS);
}

template <int NT, class EP>
cudaError_t conv3x3_nt(const HaloSrc& src, const uint16_t* wb, int cin, int N, int B, const EP& ep, uint32_t* err,
                       cudaStream_t st) {
  auto kern = k_conv3x3<NT, EP>;
  const int smem = HaloSmem<NT>::BYTES;
  static bool attr_set = false;
  if (!attr_set) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    attr_set = true;
  }
  const int ntiles = (N + NT - 1) / NT;
  dim3 grid((unsigned)((src.w + 15) / 16), (unsigned)((src.h + 15) / 16), (unsigned)(B * ntiles));
  kern<<<grid, tc::THREADS, smem, st>>>(src, wb, cin, N, ep, err);
  return cudaGetLastError();
}

// Output-channel slice width per launch: the whole N when it fits one MMA pair (two
// accumulators of N columns in 256 TMEM columns), else 128-wide slices.
static int sm_count();

template <class EP>
cudaError_t conv3x3(const HaloSrc& src, const uint16_t* wb, int cin, int N, int B, const EP& ep, uint32_t* err,
                    cudaStream_t st) {
  // small images (the coarse levels of training crops) have fewer 16 x 16 tiles than SMs: split
  // the output channels into 32-wide slices so that more CTAs share the work
  const int tiles = ((src.w + 15) / 16) * ((src.h + 15) / 16) * B;
  if (N > 32 && tiles * ((N + 127) / 128) < sm_count()) return conv3x3_nt<32>(src, wb, cin, N, B, ep, err, st);
  switch (N) {
    case 32: return conv3x3_nt<32>(src, wb, cin, N, B, ep, err, st);
    case 48: return conv3x3_nt<48>(src, wb, cin, N, B, ep, err, st);
    case 64: return conv3x3_nt<64>(src, wb, cin, N, B, ep, err, st);
    case 80: return conv3x3_nt<80>(src, wb, cin, N, B, ep, err, st);
    case 96: return conv3x3_nt<96>(src, wb, cin, N, B, ep, err, st);
    case 112: return conv3x3_nt<112>(src, wb, cin, N, B, ep, err, st);
    default: return conv3x3_nt<128>(src, wb, cin, N, B, ep, err, st);
  }
}

// Output-channel tile of the warp-specialised kernel for a convolution with N output channels
// (the whole N up to 128, else 128-wide tiles), shared by the weight packing and the launches.
__host__ __device__ inline int ws_nt(int N) {
  return N <= 32 ? 32 : N <= 48 ? 48 : N <= 64 ? 64 : N <= 80 ? 80 : N <= 96 ? 96 : N <= 112 ? 112 : 128;
}
inline size_t ws_packed_elems(int N, int K) {
  const int nt = ws_nt(N);
  return (size_t)((N + nt - 1) / nt) * (K / 16) * 9 * nt * 16;
}

static int sm_count() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
  }
  return n;
}

template <int NT, class EP>
cudaError_t conv3x3_ws_nt(const HaloSrc& src, const uint16_t* wpk, int cin, int N, int B, const EP& ep, uint32_t* err,
                          cudaStream_t st) {
  // images smaller than the 18 x 18 halo box go to the per-tile kernel (the callers' fallback)
  if (src.h < ws::HW || src.w < ws::HW) return cudaErrorNotSupported;
  CUtensorMap map;
  cudaError_t e = ws::make_halo_map(&map, src.s, src.cs, src.w, src.h, B);
  if (e != cudaSuccess) return cudaErrorNotSupported;
  auto kern = ws::k_conv3x3_ws<NT, EP>;
  // at most two CTAs per SM when each takes 256 tensor-memory columns: ask for enough shared
  // memory that a third cannot be resident (it would wait in tcgen05.alloc)
  constexpr int smem = (ws::acc_cols(NT) == 256 && ws::smem_bytes(NT) < 78 * 1024) ? 78 * 1024 : ws::smem_bytes(NT);
  static bool attr_set = false;
  if (!attr_set) {
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    attr_set = true;
  }
  ws::ConvGeom g;
  g.u = src.u; g.cu = src.cu; g.hc = src.hc; g.wc = src.wc; g.cs = src.cs;
  g.h = src.h; g.w = src.w; g.B = B; g.cin = cin; g.N = N;
  g.tiles_x = (src.w + 15) / 16; g.tiles_y = (src.h + 15) / 16; g.ntn = (N + NT - 1) / NT;
  g.n_tiles = g.tiles_x * g.tiles_y * B * g.ntn;
  const int per_sm = (ws::acc_cols(NT) <= 256 && 2 * smem <= 227 * 1024) ? 2 : 1;
  const int grid = std::min(g.n_tiles, sm_count() * per_sm);
  kern<<<grid, ws::THREADS, smem, st>>>(map, g, wpk, ep, err);
  return cudaGetLastError();
}

template <class EP>
cudaError_t conv3x3_ws(const HaloSrc& src, const uint16_t* wpk, int cin, int N, int B, const EP& ep, uint32_t* err,
                       cudaStream_t st) {
  switch (ws_nt(N)) {
    case 32: return conv3x3_ws_nt<32>(src, wpk, cin, N, B, ep, err, st);
    case 48: return conv3x3_ws_nt<48>(src, wpk, cin, N, B, ep, err, st);
    case 64: return conv3x3_ws_nt<64>(src, wpk, cin, N, B, ep, err, st);
    case 80: return conv3x3_ws_nt<80>(src, wpk, cin, N, B, ep, err, st);
    case 96: return conv3x3_ws_nt<96>(src, wpk, cin, N, B, ep, err, st);
    case 112: return conv3x3_ws_nt<112>(src, wpk, cin, N, B, ep, err, st);
    default: return conv3x3_ws_nt<128>(src, wpk, cin, N, B, ep, err, st);
  }
}

// Weights [N][9][K] (BF16) -> the warp-specialised kernel's blocks: per N tile and 16-channel
// chunk, 9 taps x NT rows x 16 channels in the shared-memory core-matrix layout (zeros for rows
// beyond N).
__global__ void k_pack_conv_w(const uint16_t* __restrict__ w, int N, int K, int NT, uint16_t* __restrict__ out) {
  const int KT = K / 16, ntn = (N + NT - 1) / NT;
  const size_t total = (size_t)ntn * KT * 9 * NT * 16;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    // i enumerates (nt, kt, t, n, c) with c fastest
    const int c = (int)(i % 16);
    size_t q = i / 16;
    const int n = (int)(q % NT); q /= NT;
    const int t = (int)(q % 9); q /= 9;
    const int kt = (int)(q % KT);
    const int nt = (int)(q / KT);
    const int gn = nt * NT + n;
    const uint16_t v = gn < N ? w[((size_t)gn * 9 + t) * K + kt * 16 + c] : (uint16_t)0;
    const size_t blk = ((size_t)nt * KT + kt) * 9 * NT * 16;   // elements
    const size_t off = (size_t)t * NT * 16 + (((n >> 3) * 2 + (c >> 3)) * 64) + (n & 7) * 8 + (c & 7);
    out[blk + off] = v;
  }
}

template <int BN, class LA, class LB, class EP>
cudaError_t gemm(const LA& la, const LB& lb, const EP& ep, int M, int N, int K, int splits, uint32_t* err,
                 cudaStream_t st) {
  auto kern = tc::k_tc_gemm<BN, LA, LB, EP>;
  const int smem = tc::Smem<BN>::BYTES;
  static bool attr_set = false;   // one instantiation per template: set its smem limit once
  if (!attr_set) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    attr_set = true;
  }
  const int kt_all = (K + tc::BK - 1) / tc::BK;
  const int kt_per = (kt_all + splits - 1) / splits;
  dim3 grid((unsigned)((M + tc::BM - 1) / tc::BM), (unsigned)((N + BN - 1) / BN), (unsigned)splits);
  kern<<<grid, tc::THREADS, smem, st>>>(la, lb, ep, M, N, K, kt_per, err);
  return cudaGetLastError();
}

// GEMMs whose N is an output-channel count (forward, data gradient): one N tile when N <= 128.
template <class LA, class LB, class EP>
cudaError_t gemm_n(const LA& la, const LB& lb, const EP& ep, int M, int N, int K, uint32_t* err, cudaStream_t st) {
  if (N <= 32) return gemm<32>(la, lb, ep, M, N, K, 1, err, st);
  if (N <= 64) return gemm<64>(la, lb, ep, M, N, K, 1, err, st);
  return gemm<128>(la, lb, ep, M, N, K, 1, err, st);
}

// ---------------------------------------------------------------------------- small kernels
struct Crop { int e, oy, ox, pad; };

// Batch gather: features (log1p colour, albedo, normal, depth/(depth+3); 16 channels, BF16),
// noisy colour and target of each crop pixel.  Dataset images are e x h_img x w_img.
// Input features of a pixel: log1p colour, albedo, normal, depth / (depth + 3), zero-padded to 16.
__global__ void k_gather(const float4* __restrict__ col, const float* __restrict__ gbuf, const float4* __restrict__ tgt,
                         int h_img, int w_img, const Crop* __restrict__ crops, int B, int h, int w,
                         uint16_t* __restrict__ x0, float4* __restrict__ col_out, float4* __restrict__ tgt_out) {
  const int P = B * h * w;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < P; p += gridDim.x * blockDim.x) {
    const int b = p / (h * w), r = p - b * h * w, y = r / w, x = r - (r / w) * w;
    const Crop c = crops[b];
    const size_t src = ((size_t)c.e * h_img + (c.oy + y)) * w_img + (c.ox + x);
    float4 cl = col[src];
    const float* g = gbuf + src * 12;
    float f[16];
    f[0] = log1pf(fmaxf(cl.x, 0.0f)); f[1] = log1pf(fmaxf(cl.y, 0.0f)); f[2] = log1pf(fmaxf(cl.z, 0.0f));
    f[3] = g[4]; f[4] = g[5]; f[5] = g[6];
    f[6] = g[0]; f[7] = g[1]; f[8] = g[2];
    float d = fmaxf(g[11], 0.0f);
    f[9] = d / (d + 3.0f);
#pragma unroll
    for (int i = 10; i < 16; ++i) f[i] = 0.0f;
    uint32_t wv[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) wv[i] = (uint32_t)f2bf(f[2 * i]) | ((uint32_t)f2bf(f[2 * i + 1]) << 16);
    uint4* dst = reinterpret_cast<uint4*>(x0 + (size_t)p * 16);
    dst[0] = make_uint4(wv[0], wv[1], wv[2], wv[3]);
    dst[1] = make_uint4(wv[4], wv[5], wv[6], wv[7]);
    col_out[p] = cl;
    if (tgt) tgt_out[p] = tgt[src];
  }
}

__device__ __forceinline__ void coarse_dims(int h, int w, int& hc, int& wc) { hc = (h + 1) >> 1; wc = (w + 1) >> 1; }

// 2x2 average pooling (children beyond an odd edge are left out of the mean).
__global__ void k_avgpool(const uint16_t* __restrict__ in, uint16_t* __restrict__ out, int B, int h, int w, int C) {
  int hc, wc;
  coarse_dims(h, w, hc, wc);
  const size_t n = (size_t)B * hc * wc * (C / 8);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int g = (int)(i % (C / 8));
    const size_t q = i / (C / 8);
    const int b = (int)(q / ((size_t)hc * wc)), r = (int)(q - (size_t)b * hc * wc), yc = r / wc, xc = r - (r / wc) * wc;
    float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    int cnt = 0;
    for (int dy = 0; dy < 2; ++dy)
      for (int dx = 0; dx < 2; ++dx) {
        int y = 2 * yc + dy, x = 2 * xc + dx;
        if (y >= h || x >= w) continue;
        ++cnt;
        uint4 v = *reinterpret_cast<const uint4*>(in + (((size_t)b * h + y) * w + x) * C + g * 8);
        const uint32_t ww[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int k = 0; k < 8; ++k) acc[k] += bf2f((uint16_t)(ww[k >> 1] >> ((k & 1) * 16)));
      }
    const float inv = 1.0f / (float)cnt;
    uint32_t o[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) o[k] = (uint32_t)f2bf(acc[2 * k] * inv) | ((uint32_t)f2bf(acc[2 * k + 1] * inv) << 16);
    *reinterpret_cast<uint4*>(out + q * C + g * 8) = make_uint4(o[0], o[1], o[2], o[3]);
  }
}

// The predicted filters: three 5x5 kernels per pixel (softmax over logits [25s, 25s + 25) of the
// 80-channel logit tensor) applied as a cascade at dilations 1, 2 and 4 -- f1 = K1 * colour,
// f2 = K2 (dilated 2) * f1, f3 = K3 (dilated 4) * f2 -- with clamp-to-edge neighbours, so the
// footprint grows to 29 x 29 pixels while every kernel stays 5 x 5.
constexpr int LOGITS = 80;

__device__ __forceinline__ void softmax25(const float* lg, float (&wk)[25]) {
  float mx = lg[0];
  for (int k = 1; k < 25; ++k) mx = fmaxf(mx, lg[k]);
  float sum = 0.0f;
  for (int k = 0; k < 25; ++k) { wk[k] = __expf(lg[k] - mx); sum += wk[k]; }
  const float inv = 1.0f / sum;
  for (int k = 0; k < 25; ++k) wk[k] *= inv;
}

__device__ __forceinline__ size_t tap_index(int b, int y, int x, int k, int d, int h, int w) {
  int yy = min(max(y + d * (k / 5 - 2), 0), h - 1), xx = min(max(x + d * (k % 5 - 2), 0), w - 1);
  return ((size_t)b * h + yy) * w + xx;
}

__global__ void k_filter_fwd(const float* __restrict__ logits, int stage, int d, const float4* __restrict__ in,
                             float4* __restrict__ out, int B, int h, int w) {
  const int P = B * h * w;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < P; p += gridDim.x * blockDim.x) {
    const int b = p / (h * w), r = p - b * h * w, y = r / w, x = r - (r / w) * w;
    float wk[25];
    softmax25(logits + (size_t)p * LOGITS + stage * 25, wk);
    float fx = 0.0f, fy = 0.0f, fz = 0.0f;
    for (int k = 0; k < 25; ++k) {
      float4 c = in[tap_index(b, y, x, k, d, h, w)];
      fx += wk[k] * c.x; fy += wk[k] * c.y; fz += wk[k] * c.z;
    }
    out[p] = make_float4(fx, fy, fz, 1.0f);
  }
}

// Relative L2 loss sum((f-t)^2 / (t^2 + 0.01)) / (3 P) and its gradient with respect to f.
__global__ void k_filter_loss(const float4* __restrict__ f, const float4* __restrict__ tgt, int P,
                              float4* __restrict__ g, float* __restrict__ loss) {
  const float norm = 1.0f / (3.0f * (float)P);
  float local = 0.0f;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < P; p += gridDim.x * blockDim.x) {
    float4 a = f[p], t = tgt[p];
    float ex = a.x - t.x, ey = a.y - t.y, ez = a.z - t.z;
    float dx = 1.0f / (t.x * t.x + 0.01f), dy = 1.0f / (t.y * t.y + 0.01f), dz = 1.0f / (t.z * t.z + 0.01f);
    local += ex * ex * dx + ey * ey * dy + ez * ez * dz;
    g[p] = make_float4(2.0f * ex * dx * norm, 2.0f * ey * dy * norm, 2.0f * ez * dz * norm, 0.0f);
  }
  for (int off = 16; off > 0; off >>= 1) local += __shfl_down_sync(0xffffffffu, local, off);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, local * norm);
}

// Backward of one filter stage at dilation D over a 32 x 8 pixel block: logit gradients of its
// 25 kernel weights (softmax Jacobian) and, when gin is given, the gradient of its input,
// scattered to the tap neighbours.  The block's input colours and a 2D-pixel apron (clamped to
// the image like tap_index) are staged in shared memory, and the input gradient is first summed
// in a shared-memory copy of the same window, so each window point costs one global atomic per
// channel instead of one per tap that reaches it (staged points that clamp onto the same pixel
// each add their own share).
template <int D>
__global__ void __launch_bounds__(256)
k_filter_bwd_tiled(const float* __restrict__ logits, int stage, const float4* __restrict__ in,
                   const float4* __restrict__ gout, uint16_t* __restrict__ dlogits, float* __restrict__ gin,
                   int B, int h, int w) {
  constexpr int BW = 32, BH = 8, SW = BW + 4 * D, SH = BH + 4 * D, NP = SW * SH;
  __shared__ float4 tile[NP];
  __shared__ float acc[3][NP];
  const int b = (int)blockIdx.z, x0 = (int)blockIdx.x * BW, y0 = (int)blockIdx.y * BH;
  const float4* src = in + (size_t)b * h * w;
  for (int i = threadIdx.x; i < NP; i += blockDim.x) {
    const int sy = i / SW, sx = i - (i / SW) * SW;
    const int yy = min(max(y0 - 2 * D + sy, 0), h - 1), xx = min(max(x0 - 2 * D + sx, 0), w - 1);
    tile[i] = src[(size_t)yy * w + xx];
    acc[0][i] = 0.0f; acc[1][i] = 0.0f; acc[2][i] = 0.0f;
  }
  __syncthreads();
  const int tx = (int)(threadIdx.x & 31), ty = (int)(threadIdx.x >> 5);
  const int x = x0 + tx, y = y0 + ty;
  if (x < w && y < h) {
    const size_t p = ((size_t)b * h + y) * w + x;
    float wk[25], G[25];
    softmax25(logits + p * LOGITS + stage * 25, wk);
    const float4 g = gout[p];
    float gw = 0.0f;
#pragma unroll
    for (int k = 0; k < 25; ++k) {
      const int q = (ty + 2 * D + D * (k / 5 - 2)) * SW + tx + 2 * D + D * (k % 5 - 2);
      const float4 c = tile[q];
      G[k] = g.x * c.x + g.y * c.y + g.z * c.z;
      gw += wk[k] * G[k];
      if (gin) {
        atomicAdd(&acc[0][q], wk[k] * g.x);
        atomicAdd(&acc[1][q], wk[k] * g.y);
        atomicAdd(&acc[2][q], wk[k] * g.z);
      }
    }
    uint16_t* dl = dlogits + p * LOGITS + stage * 25;
#pragma unroll
    for (int k = 0; k < 25; ++k) dl[k] = f2bf(wk[k] * (G[k] - gw));
    if (stage == 2)
      for (int k = 75; k < LOGITS; ++k) dlogits[p * LOGITS + k] = 0;
  }
  if (!gin) return;
  __syncthreads();
  for (int i = threadIdx.x; i < NP; i += blockDim.x) {
    const int sy = i / SW, sx = i - (i / SW) * SW;
    const int yy = min(max(y0 - 2 * D + sy, 0), h - 1), xx = min(max(x0 - 2 * D + sx, 0), w - 1);
    float* dst = gin + (((size_t)b * h + yy) * w + xx) * 4;
    if (acc[0][i] != 0.0f) atomicAdd(dst + 0, acc[0][i]);
    if (acc[1][i] != 0.0f) atomicAdd(dst + 1, acc[1][i]);
    if (acc[2][i] != 0.0f) atomicAdd(dst + 2, acc[2][i]);
  }
}

// d = (y > 0) ? d : 0 over n BF16 values (ReLU backward; in place).
__global__ void k_relu_mask(uint16_t* __restrict__ d, const uint16_t* __restrict__ y, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    if (!(bf2f(y[i]) > 0.0f)) d[i] = 0;
}

// Data gradient of a decoder convolution's input [up(coarse) cu | skip cs] at fine resolution:
// the coarse part sums its 2x2 children and is masked by the coarse activation's ReLU.
__global__ void k_split_up(const uint16_t* __restrict__ dx, int cu, int cs, int B, int h, int w,
                           const uint16_t* __restrict__ coarse_act, uint16_t* __restrict__ dcoarse) {
  int hc, wc;
  coarse_dims(h, w, hc, wc);
  const int cin = cu + cs;
  const size_t n = (size_t)B * hc * wc * cu;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int c = (int)(i % cu);
    const size_t q = i / cu;
    const int b = (int)(q / ((size_t)hc * wc)), r = (int)(q - (size_t)b * hc * wc), yc = r / wc, xc = r - (r / wc) * wc;
    float s = 0.0f;
    for (int dy = 0; dy < 2; ++dy)
      for (int dxx = 0; dxx < 2; ++dxx) {
        int y = 2 * yc + dy, x = 2 * xc + dxx;
        if (y < h && x < w) s += bf2f(dx[(((size_t)b * h + y) * w + x) * cin + c]);
      }
    dcoarse[i] = bf2f(coarse_act[i]) > 0.0f ? f2bf(s) : (uint16_t)0;
  }
}

// Gradient of an encoder activation E (fine): skip part from the decoder's concat gradient plus
// the pooled path's gradient spread over the 2x2 children, masked by E's ReLU.
__global__ void k_enc_grad(const uint16_t* __restrict__ dx_cat, int cat_stride, int cat_off,
                           const uint16_t* __restrict__ dpool, const uint16_t* __restrict__ e, int B, int h, int w,
                           int C, uint16_t* __restrict__ dz) {
  int hc, wc;
  coarse_dims(h, w, hc, wc);
  const size_t n = (size_t)B * h * w * C;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    const size_t p = i / C;
    const int b = (int)(p / ((size_t)h * w)), r = (int)(p - (size_t)b * h * w), y = r / w, x = r - (r / w) * w;
    float g = bf2f(dx_cat[p * cat_stride + cat_off + c]);
    if (dpool) {
      const int yc = y >> 1, xc = x >> 1;
      const int cnt = (min(2 * yc + 2, h) - 2 * yc) * (min(2 * xc + 2, w) - 2 * xc);
      g += bf2f(dpool[(((size_t)b * hc + yc) * wc + xc) * C + c]) / (float)cnt;
    }
    dz[i] = bf2f(e[i]) > 0.0f ? f2bf(g) : (uint16_t)0;
  }
}

// Bias gradient: column sums of dZ [P][C] (FP32 atomics per block).
__global__ void k_bias_grad(const uint16_t* __restrict__ dz, int P, int C, float* __restrict__ db) {
  extern __shared__ float acc[];
  for (int c = threadIdx.x; c < C; c += blockDim.x) acc[c] = 0.0f;
  __syncthreads();
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < (size_t)P * C; i += (size_t)gridDim.x * blockDim.x)
    atomicAdd(&acc[i % C], bf2f(dz[i]));
  __syncthreads();
  for (int c = threadIdx.x; c < C; c += blockDim.x)
    if (acc[c] != 0.0f) atomicAdd(&db[c], acc[c]);
}

// Adam (bias-corrected) over the flat FP32 parameters, with the gradient g * scale.
// Gradient clipping by global norm.  k_grad_sqnorm writes per-block partial sums of (g * scale)^2
// into clip[4 ..], k_clip_factor adds them in a fixed order (the same bits on every data-parallel
// rank that holds the same gradient) and sets the step's factor clip[2]: 1, or kClipRatio times
// the running mean of past step norms (clip[1]) over this norm when the norm is above that (a
// batch whose noisy input holds a firefly of the sun can carry a gradient thousands of times the
// usual one), or 0 for a non-finite norm (the step is skipped).  The first step sets the mean.
constexpr float kClipRatio = 4.0f;
constexpr int kNormBlocks = 296;

__global__ void __launch_bounds__(256) k_grad_sqnorm(const float* __restrict__ g, size_t n, float scale,
                                                     float* __restrict__ clip) {
  __shared__ float part[8];
  float s = 0.0f;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float v = g[i] * scale;
    s += v * v;
  }
  for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    float b = 0.0f;
    for (int w = 0; w < 8; ++w) b += part[w];
    clip[4 + blockIdx.x] = b;
  }
}

__global__ void k_clip_factor(float* __restrict__ clip) {
  if (threadIdx.x != 0) return;
  float sq = 0.0f;
  for (int b = 0; b < kNormBlocks; ++b) sq += clip[4 + b];
  const float norm = sqrtf(sq);
  if (!isfinite(norm)) {
    clip[2] = 0.0f;
    return;
  }
  const float mean = clip[1] > 0.0f ? clip[1] : norm;
  const float lim = kClipRatio * mean;
  clip[2] = norm > lim ? lim / norm : 1.0f;
  clip[1] = 0.98f * mean + 0.02f * fminf(norm, lim);
}

__global__ void k_adam(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       size_t n, float lr, float b1, float b2, float eps, float c1, float c2, float scale,
                       const float* __restrict__ clip) {
  const float f = clip[2];
  if (f == 0.0f) return;   // non-finite gradient: no step
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    float gi = g[i] * scale * f;
    float mi = b1 * m[i] + (1.0f - b1) * gi;
    float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

// BF16 copies of one layer's weights W[co][tap][ci]: as stored (forward) and transposed with the
// taps mirrored, Wt[ci][taps-1-tap][co], so the data gradient is the same 3x3 convolution of the
// output gradient with Wt.
__global__ void k_weights_bf16(const float* __restrict__ wf, int cout, int taps, int cin, uint16_t* __restrict__ wb,
                               uint16_t* __restrict__ wt) {
  const int n = cout * taps * cin;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int ci = i % cin, t = (i / cin) % taps, co = i / (cin * taps);
    uint16_t b = f2bf(wf[i]);
    wb[i] = b;
    wt[((size_t)ci * taps + (taps - 1 - t)) * cout + co] = b;
  }
}

// ---------------------------------------------------------------------------- inference tail
// Inference only.  The 1x1 output layer (32 -> 80 logits) runs on the tensor cores with the
// three stages' softmax and the first filter stage in its epilogue, so the 80 FP32 logits of a
// pixel never reach global memory: the epilogue writes the first stage's filtered colour and the
// normalised 5x5 kernels of stages 2 and 3 (50 floats a pixel).  Two filter kernels apply those,
// the last one also tonemapping into the rgba8 image.  Every value is computed with the training
// forward's arithmetic (the same bias add, softmax and tap order), so the images are identical to
// forward() followed by the tonemap.  The 50 kernel weights are stored as planes (weight k of
// pixel p at wk23[k * P + p]), so each store and each load of a warp covers 128 contiguous bytes.
constexpr int WK23 = 50;
static_assert(WK23 <= LOGITS, "the stored kernels live in the logits buffer (LOGITS floats a pixel)");

template <int N>
__device__ __forceinline__ void softmax_reg(const float (&lg)[80], int off, float (&wk)[N]) {
  float mx = lg[off];
#pragma unroll
  for (int k = 1; k < N; ++k) mx = fmaxf(mx, lg[off + k]);
  float sum = 0.0f;
#pragma unroll
  for (int k = 0; k < N; ++k) { wk[k] = __expf(lg[off + k] - mx); sum += wk[k]; }
  const float inv = 1.0f / sum;
#pragma unroll
  for (int k = 0; k < N; ++k) wk[k] *= inv;
}

// The output layer's bias as a kernel argument (read from the constant bank, no loads).
struct OutBias { float v[LOGITS]; };

// Persistent output-layer kernel: warps 0-3 are the epilogue (thread t owns tensor-memory lane t,
// pixel t of a 128-pixel tile), warp 4 loads each tile's D0 activations into one of two
// shared-memory stages and issues its two MMAs (K = 32) into the CTA's one accumulator as soon as
// the epilogue has read the previous tile out of it, so the next tile's loads and MMAs run while
// the epilogue computes.  Operand tiles use a compact K-major layout: 4 core matrices (32 K) per
// 8-row group, SBO 512 bytes.
namespace outk {
constexpr int THREADS = 160;
constexpr int A_BYTES = tc::BM * 32 * 2;     // 128 pixels x 32 channels
constexpr int B_BYTES = LOGITS * 32 * 2;     // 80 logits x 32 channels
constexpr int SMEM = 2 * A_BYTES + B_BYTES + 128;
constexpr int CTAS_PER_SM = 3;               // registers (136 a thread); 128 tensor-memory columns each
__device__ __forceinline__ void put4(uint8_t* tile, int r, int c, uint4 v) {
  *reinterpret_cast<uint4*>(tile + ((r >> 3) * 4 + c) * 128 + (r & 7) * 16) = v;
}
}  // namespace outk

// d0: [P][32] BF16, wb: [80][32] BF16.  Writes stage 1's filtered colour (f1) and the
// normalised kernels of stages 2 and 3 as 50 planes of P floats (wk23).
__global__ void __launch_bounds__(outk::THREADS, 3)
k_out_softmax(const uint16_t* __restrict__ d0, const uint16_t* __restrict__ wb, const OutBias bias,
              const float4* __restrict__ col, float4* __restrict__ f1, float* __restrict__ wk23, int B, int h,
              int w, uint32_t* err) {
  extern __shared__ __align__(1024) uint8_t smem[];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int P = B * h * w;
  const int n_tiles = (P + tc::BM - 1) / tc::BM;
  uint8_t* ta0 = smem;
  uint8_t* tb = smem + 2 * outk::A_BYTES;
  uint64_t* bars = reinterpret_cast<uint64_t*>(tb + outk::B_BYTES);
  // bars: 0 accumulator full, 1 accumulator read out, 2-3 A stage free
  const uint32_t bar_full = tc::smem_u32(&bars[0]), bar_tfree = tc::smem_u32(&bars[1]);
  auto bar_afree = [&](int st) { return tc::smem_u32(&bars[2 + st]); };
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(&bars[4]);
  volatile uint32_t* abort_flag = tmem_slot + 1;
  constexpr uint32_t NCOLS = tc::tmem_cols(LOGITS);
  if (warp == 0) tc::tmem_alloc(tc::smem_u32(tmem_slot), NCOLS);
  if (tid == 0) {
    tc::mbar_init(bar_full, 1);
    tc::mbar_init(bar_tfree, 128);
    tc::mbar_init(bar_afree(0), 1);
    tc::mbar_init(bar_afree(1), 1);
    *abort_flag = 0u;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // the weights, once: 80 rows x 4 chunks
  for (int i = tid; i < LOGITS * 4; i += outk::THREADS) {
    const int r = i % LOGITS, c = i / LOGITS;
    outk::put4(tb, r, c, *reinterpret_cast<const uint4*>(wb + (size_t)r * 32 + c * 8));
  }
  tc::fence_async_smem();
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  if (warp == 4) {
    // ---------------------------------------------------------------- loader + MMA issuer
    int last_j = -1;   // last tile whose MMAs were issued
    for (int j = 0, tile = blockIdx.x; tile < n_tiles; ++j, tile += gridDim.x) {
      const int st = j & 1;
      uint8_t* ta = ta0 + st * outk::A_BYTES;
      uint32_t go = 1u;
      if (lane == 0) {
        if (*abort_flag) go = 0u;
        // the MMAs that read this stage two tiles ago are done
        else if (j >= 2 && !tc::mbar_wait(bar_afree(st), (uint32_t)((j >> 1) - 1) & 1u)) go = 0u;
      }
      go = __shfl_sync(0xffffffffu, go, 0);
      if (!go) break;
      const int p0 = tile * tc::BM;
      for (int i = lane; i < tc::BM * 4; i += 32) {
        const int r = i % tc::BM, c = i / tc::BM, p = p0 + r;
        outk::put4(ta, r, c, p < P ? *reinterpret_cast<const uint4*>(d0 + (size_t)p * 32 + c * 8) : zero4());
      }
      tc::fence_async_smem();
      __syncwarp();
      if (lane == 0) {
        // the epilogue has read the previous tile out of the accumulator
        if (j >= 1 && !tc::mbar_wait(bar_tfree, (uint32_t)(j - 1) & 1u)) go = 0u;
        if (go) {
          tc::tc_fence_after();
          constexpr uint32_t IDESC = tc::idesc_bf16(LOGITS);
          const uint32_t a_addr = tc::smem_u32(ta), b_addr = tc::smem_u32(tb);
#pragma unroll
          for (int kk = 0; kk < 2; ++kk) {
            const uint64_t da = tc::smem_desc(a_addr + kk * 256, 128, 512);
            const uint64_t db = tc::smem_desc(b_addr + kk * 256, 128, 512);
            tc::mma_bf16(tmem, da, db, IDESC, kk > 0 ? 1u : 0u);
          }
          tc::mma_commit(bar_full);
          tc::mma_commit(bar_afree(st));
          last_j = j;
        } else {
          *abort_flag = 1u;
          atomicOr(err, tc::ERR_TC_TIMEOUT);
        }
      }
      go = __shfl_sync(0xffffffffu, go, 0);
      if (!go) break;
    }
    // the MMAs in flight finish before the tensor memory can be freed (the last commit covers all)
    if (lane == 0 && last_j >= 0) tc::mbar_wait(bar_afree(last_j & 1), (uint32_t)(last_j >> 1) & 1u);
  } else {
    // ---------------------------------------------------------------- epilogue
    for (int j = 0, tile = blockIdx.x; tile < n_tiles; ++j, tile += gridDim.x) {
      uint32_t go = 0u;
      if (lane == 0) {
        go = *abort_flag ? 0u : 1u;
        if (go && !tc::mbar_wait(bar_full, (uint32_t)j & 1u)) {
          go = 0u;
          *abort_flag = 1u;
          atomicOr(err, tc::ERR_TC_TIMEOUT);
        }
      }
      go = __shfl_sync(0xffffffffu, go, 0);
      if (!go) break;
      tc::tc_fence_after();
      float lg[80];
#pragma unroll
      for (int c0 = 0; c0 < 80; c0 += 16) {
        float v[16];
        tc::tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
#pragma unroll
        for (int i = 0; i < 16; ++i) lg[c0 + i] = v[i] + bias.v[c0 + i];
      }
      tc::tc_fence_before();
      ws::mbar_arrive(bar_tfree);
      const int p = tile * tc::BM + tid;
      if (p < P) {
        const int b = p / (h * w), r = p - b * h * w, y = r / w, x = r - (r / w) * w;
        float wk[25];
        softmax_reg<25>(lg, 0, wk);
        // the 5 clamped rows and columns of the taps (tap_index's clamping, computed once)
        const float4* img = col + (size_t)b * h * w;
        int rows[5], cols[5];
#pragma unroll
        for (int d = 0; d < 5; ++d) {
          rows[d] = min(max(y + d - 2, 0), h - 1) * w;
          cols[d] = min(max(x + d - 2, 0), w - 1);
        }
        float fx = 0.0f, fy = 0.0f, fz = 0.0f;
#pragma unroll
        for (int k = 0; k < 25; ++k) {
          float4 c = img[rows[k / 5] + cols[k % 5]];
          fx += wk[k] * c.x; fy += wk[k] * c.y; fz += wk[k] * c.z;
        }
        f1[p] = make_float4(fx, fy, fz, 1.0f);
        float* dst = wk23 + p;
        softmax_reg<25>(lg, 25, wk);
#pragma unroll
        for (int k = 0; k < 25; ++k, dst += P) __stcs(dst, wk[k]);
        softmax_reg<25>(lg, 50, wk);
#pragma unroll
        for (int k = 0; k < 25; ++k, dst += P) __stcs(dst, wk[k]);
      }
    }
  }
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 0) tc::tmem_free(tmem, NCOLS);
}

// A filter stage with stored normalised kernels (planes off..off+24 of wk23) at dilation D over
// a 32 x 8 pixel block: the block's colours and a 2D-pixel apron, clamped to the image like
// tap_index, are staged in shared memory once, and the weights are read as planes (128
// contiguous bytes a warp).  The taps are summed in tap_index order, so the result equals the
// direct gather's.  With rgba the result is also tonemapped into the rgba8 image with the
// accumulation pass's display transform (shader.wgsl:2487-2490).
template <int D>
__global__ void __launch_bounds__(256)
k_filter_stored(const float* __restrict__ wk23, int off, const float4* __restrict__ in, float4* __restrict__ out,
                uchar4* __restrict__ rgba, float exposure, int B, int h, int w) {
  constexpr int BW = 32, BH = 8, SW = BW + 4 * D, SH = BH + 4 * D;
  __shared__ float4 tile[SH * SW];
  const int b = (int)blockIdx.z, x0 = (int)blockIdx.x * BW, y0 = (int)blockIdx.y * BH;
  const float4* src = in + (size_t)b * h * w;
  for (int i = threadIdx.x; i < SH * SW; i += blockDim.x) {
    const int sy = i / SW, sx = i - (i / SW) * SW;
    const int yy = min(max(y0 - 2 * D + sy, 0), h - 1), xx = min(max(x0 - 2 * D + sx, 0), w - 1);
    tile[i] = src[(size_t)yy * w + xx];
  }
  __syncthreads();
  const int tx = (int)(threadIdx.x & 31), ty = (int)(threadIdx.x >> 5);
  const int x = x0 + tx, y = y0 + ty;
  if (x >= w || y >= h) return;
  const size_t P = (size_t)B * h * w;
  const size_t p = ((size_t)b * h + y) * w + x;
  const float* wk = wk23 + (size_t)off * P + p;
  float fx = 0.0f, fy = 0.0f, fz = 0.0f;
#pragma unroll
  for (int k = 0; k < 25; ++k) {
    const float wt = __ldcs(wk + (size_t)k * P);
    const float4 c = tile[(ty + 2 * D + D * (k / 5 - 2)) * SW + tx + 2 * D + D * (k % 5 - 2)];
    fx += wt * c.x; fy += wt * c.y; fz += wt * c.z;
  }
  const float4 v = make_float4(fx, fy, fz, 1.0f);
  out[p] = v;
  if (rgba) {
    float rr = v.x * exposure, gg = v.y * exposure, bb = v.z * exposure;
    rr = powf(rr / (rr + 0.3f), 0.4545f); gg = powf(gg / (gg + 0.3f), 0.4545f); bb = powf(bb / (bb + 0.3f), 0.4545f);
    auto u8 = [](float t) { return (unsigned char)floorf(fminf(fmaxf(t, 0.0f), 1.0f) * 255.0f + 0.5f); };
    rgba[p] = make_uchar4(u8(rr), u8(gg), u8(bb), 255);
  }
}

// ---------------------------------------------------------------------------- the network
struct Layer {
  const char* name;
  int cu, cs;        // input channels: upsampled coarse part, same-resolution part (padded)
  int cout;          // output channels (padded)
  int taps;          // 9 or 1
  int relu;
  int level;         // output resolution level
  int real_cin, real_cout;   // channels before padding (initialisation)
  size_t w_off, b_off;       // offsets into the flat parameters
  uint16_t* wb = nullptr;    // BF16 [cout][taps][cin]
  uint16_t* wt = nullptr;    // BF16 [cin][taps][cout]
  uint16_t* wpk = nullptr;   // wb in the warp-specialised convolution's blocks (3x3 layers)
  uint16_t* wtpk = nullptr;  // wt likewise (data gradient)
  int cin() const { return cu + cs; }
  size_t nw() const { return (size_t)cout * taps * cin(); }
};

enum { L_E0A, L_E0, L_E1, L_E2, L_E3, L_E4A, L_E4, L_D3, L_D2, L_D1, L_D0, L_OUT, NLAYERS };

struct Net {
  int device = 0;
  int conv_mode = 0;   // 3x3 convolutions: 0 warp-specialised TMA pipeline, 1 one CTA per tile
  cudaStream_t st = nullptr;
  Layer L[NLAYERS];
  size_t n_params = 0;
  float *w = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;   // FP32 parameters, gradients, Adam moments
  int adam_t = 0;
  uint32_t* err = nullptr;
  // activations / gradients for the current batch shape
  int B = 0, H = 0, W = 0;
  size_t cap[5] = {0, 0, 0, 0, 0};   // allocated pixels per level
  int hl[5], wl[5];
  uint16_t *x0 = nullptr, *e0a = nullptr, *e0 = nullptr, *p1 = nullptr, *e1 = nullptr, *p2 = nullptr, *e2 = nullptr,
           *p3 = nullptr, *e3 = nullptr, *p4 = nullptr, *e4a = nullptr, *e4 = nullptr, *d3 = nullptr, *d2 = nullptr,
           *d1 = nullptr, *d0 = nullptr;
  float* logits = nullptr;
  float4 *col = nullptr, *tgt = nullptr, *out = nullptr, *f1 = nullptr, *f2 = nullptr, *gf_a = nullptr,
         *gf_b = nullptr;
  uint16_t *dlog = nullptr, *dx = nullptr, *g_a = nullptr, *g_b = nullptr, *g_pool = nullptr, *g_skip = nullptr;
  std::vector<void*> bufs;
  float* loss = nullptr;
  OutBias out_bias;             // host copy of the output layer's bias for the inference tail
  bool out_bias_valid = false;  // cleared whenever the weights change
  float* clip = nullptr;   // gradient clipping: -, running mean of norms, step factor, -, block partial sums
  Crop* crops = nullptr;
  int crops_cap = 0;
  // dataset
  float4 *ds_col = nullptr, *ds_tgt = nullptr;
  float* ds_gbuf = nullptr;
  int ds_n = 0, ds_cap = 0, ds_h = 0, ds_w = 0;
};

static void set_layer(Layer& l, const char* name, int cu, int cs, int cout, int taps, int relu, int level, int rcin,
                      int rcout) {
  l.name = name; l.cu = cu; l.cs = cs; l.cout = cout; l.taps = taps; l.relu = relu; l.level = level;
  l.real_cin = rcin; l.real_cout = rcout;
}

static void define_layers(Net& n) {
  set_layer(n.L[L_E0A], "E0a", 0, 16, 32, 9, 1, 0, 10, 32);
  set_layer(n.L[L_E0], "E0", 0, 32, 32, 9, 1, 0, 32, 32);
  set_layer(n.L[L_E1], "E1", 0, 32, 48, 9, 1, 1, 32, 48);
  set_layer(n.L[L_E2], "E2", 0, 48, 64, 9, 1, 2, 48, 64);
  set_layer(n.L[L_E3], "E3", 0, 64, 96, 9, 1, 3, 64, 96);
  set_layer(n.L[L_E4A], "E4a", 0, 96, 128, 9, 1, 4, 96, 128);
  set_layer(n.L[L_E4], "E4", 0, 128, 128, 9, 1, 4, 128, 128);
  set_layer(n.L[L_D3], "D3", 128, 96, 96, 9, 1, 3, 224, 96);
  set_layer(n.L[L_D2], "D2", 96, 64, 64, 9, 1, 2, 160, 64);
  set_layer(n.L[L_D1], "D1", 64, 48, 48, 9, 1, 1, 112, 48);
  set_layer(n.L[L_D0], "D0", 48, 32, 32, 9, 1, 0, 80, 32);
  set_layer(n.L[L_OUT], "OUT", 0, 32, LOGITS, 1, 0, 0, 32, 75);
  size_t off = 0;
  for (int i = 0; i < NLAYERS; ++i) {
    n.L[i].w_off = off;
    off += n.L[i].nw();
    n.L[i].b_off = off;
    off += n.L[i].cout;
  }
  n.n_params = off;
}

static int grid1(size_t n) { return (int)std::min<size_t>((n + 255) / 256, 148 * 16); }

static cudaError_t refresh_bf16(Net& n) {
  n.out_bias_valid = false;
  for (int i = 0; i < NLAYERS; ++i) {
    Layer& l = n.L[i];
    k_weights_bf16<<<grid1(l.nw()), 256, 0, n.st>>>(n.w + l.w_off, l.cout, l.taps, l.cin(), l.wb, l.wt);
    if (l.taps == 9) {
      k_pack_conv_w<<<grid1(ws_packed_elems(l.cout, l.cin())), 256, 0, n.st>>>(l.wb, l.cout, l.cin(), ws_nt(l.cout), l.wpk);
      k_pack_conv_w<<<grid1(ws_packed_elems(l.cin(), l.cout)), 256, 0, n.st>>>(l.wt, l.cin(), l.cout, ws_nt(l.cin()), l.wtpk);
    }
  }
  return cudaGetLastError();
}

// Sets the batch shape; the buffers grow to the largest shape seen (per level) and are reused
// for smaller ones, so alternating image sizes (batched views) cost no allocation.
static cudaError_t ensure_batch(Net& n, int B, int H, int W) {
  if (n.B == B && n.H == H && n.W == W) return cudaSuccess;
  n.B = B; n.H = H; n.W = W;
  n.hl[0] = H; n.wl[0] = W;
  for (int l = 1; l < 5; ++l) { n.hl[l] = (n.hl[l - 1] + 1) / 2; n.wl[l] = (n.wl[l - 1] + 1) / 2; }
  bool fits = !n.bufs.empty();
  for (int l = 0; l < 5; ++l) fits = fits && (size_t)B * n.hl[l] * n.wl[l] <= n.cap[l];
  if (fits) return cudaSuccess;
  for (int l = 0; l < 5; ++l) n.cap[l] = std::max(n.cap[l], (size_t)B * n.hl[l] * n.wl[l]);
  cudaStreamSynchronize(n.st);
  for (void* p : n.bufs) cudaFree(p);
  n.bufs.clear();
  auto px = [&](int l) { return n.cap[l]; };
  cudaError_t e = cudaSuccess;
  auto alloc = [&](size_t bytes) -> void* {
    void* p = nullptr;
    if (e == cudaSuccess) e = cudaMalloc(&p, std::max<size_t>(bytes, 256));
    if (p) n.bufs.push_back(p);
    return p;
  };
  n.x0 = (uint16_t*)alloc(px(0) * 16 * 2);
  n.e0a = (uint16_t*)alloc(px(0) * 32 * 2);
  n.e0 = (uint16_t*)alloc(px(0) * 32 * 2);
  n.p1 = (uint16_t*)alloc(px(1) * 32 * 2);
  n.e1 = (uint16_t*)alloc(px(1) * 48 * 2);
  n.p2 = (uint16_t*)alloc(px(2) * 48 * 2);
  n.e2 = (uint16_t*)alloc(px(2) * 64 * 2);
  n.p3 = (uint16_t*)alloc(px(3) * 64 * 2);
  n.e3 = (uint16_t*)alloc(px(3) * 96 * 2);
  n.p4 = (uint16_t*)alloc(px(4) * 96 * 2);
  n.e4a = (uint16_t*)alloc(px(4) * 128 * 2);
  n.e4 = (uint16_t*)alloc(px(4) * 128 * 2);
  n.d3 = (uint16_t*)alloc(px(3) * 96 * 2);
  n.d2 = (uint16_t*)alloc(px(2) * 64 * 2);
  n.d1 = (uint16_t*)alloc(px(1) * 48 * 2);
  n.d0 = (uint16_t*)alloc(px(0) * 32 * 2);
  n.logits = (float*)alloc(px(0) * LOGITS * 4);
  n.col = (float4*)alloc(px(0) * 16);
  n.tgt = (float4*)alloc(px(0) * 16);
  n.out = (float4*)alloc(px(0) * 16);
  n.f1 = (float4*)alloc(px(0) * 16);
  n.f2 = (float4*)alloc(px(0) * 16);
  n.gf_a = (float4*)alloc(px(0) * 16);
  n.gf_b = (float4*)alloc(px(0) * 16);
  n.dlog = (uint16_t*)alloc(px(0) * LOGITS * 2);
  // the largest data gradient: a concat input (fine) of any level
  size_t dx_max = std::max({px(0) * 80, px(1) * 112, px(2) * 160, px(3) * 224, px(4) * 128});
  n.dx = (uint16_t*)alloc(dx_max * 2);
  size_t g_max = std::max({px(0) * 32, px(1) * 48, px(2) * 64, px(3) * 96, px(4) * 128});
  n.g_a = (uint16_t*)alloc(g_max * 2);
  n.g_b = (uint16_t*)alloc(g_max * 2);
  n.g_pool = (uint16_t*)alloc(g_max * 2);
  n.g_skip = (uint16_t*)alloc(dx_max * 2);
  return e;
}

// Convolution of layer l over its sources (coarse u read upsampled, s at the output level).
static cudaError_t conv_fwd(Net& n, const Layer& l, const uint16_t* u, const uint16_t* s, void* y, bool logits) {
  const int lv = l.level, h = n.hl[lv], w = n.wl[lv];
  const int P = n.B * h * w;
  ConvSrc src{u, l.cu, lv + 1 < 5 ? n.hl[lv + 1] : 1, lv + 1 < 5 ? n.wl[lv + 1] : 1, s, l.cs, h, w, l.taps, 1};
  if (l.taps == 9 && !logits) {
    HaloSrc hs{u, l.cu, src.hc, src.wc, s, l.cs, h, w};
    const EpiAct ep{(uint16_t*)y, n.w + l.b_off, l.cout, l.relu};
    if (n.conv_mode == 0) {
      cudaError_t e = conv3x3_ws(hs, l.wpk, l.cin(), l.cout, n.B, ep, n.err, n.st);
      if (e != cudaErrorNotSupported) return e;
    }
    return conv3x3(hs, l.wb, l.cin(), l.cout, n.B, ep, n.err, n.st);
  }
  ConvA a{src, P, l.cin()};
  RowMajor b{l.wb, l.cout, l.taps * l.cin(), l.taps * l.cin()};
  if (logits) return gemm_n(a, b, EpiLogits{(float*)y, n.w + l.b_off, l.cout}, P, l.cout, l.taps * l.cin(), n.err, n.st);
  return gemm_n(a, b, EpiAct{(uint16_t*)y, n.w + l.b_off, l.cout, l.relu}, P, l.cout, l.taps * l.cin(), n.err, n.st);
}

// Weight and bias gradients of layer l from dZ (its output gradient) and its sources; the data
// gradient of its (concatenated) input into n.dx when want_dx.
static cudaError_t conv_bwd(Net& n, const Layer& l, const uint16_t* dz, const uint16_t* u, const uint16_t* s,
                            bool want_dx) {
  const int lv = l.level, h = n.hl[lv], w = n.wl[lv];
  const int P = n.B * h * w, cin = l.cin(), K = l.taps * cin;
  ConvSrc src{u, l.cu, lv + 1 < 5 ? n.hl[lv + 1] : 1, lv + 1 < 5 ? n.wl[lv + 1] : 1, s, l.cs, h, w, l.taps, 1};
  // weight gradient: M = cout, N = taps * cin, K = pixels, split over pixel ranges
  const int kt_all = (P + tc::BK - 1) / tc::BK;
  const int n_tiles = (K + 127) / 128;
  // three CTAs per SM fit (64 KB of shared memory each): split the pixels so they all have work
  int splits = std::max(1, std::min(kt_all, (sm_count() * 3) / std::max(1, n_tiles)));
  cudaError_t e = gemm<128>(WgradA{dz, l.cout, P}, WgradB{src, cin, P, K}, EpiAtomic{n.g + l.w_off, K, K}, l.cout, K,
                            P, splits, n.err, n.st);
  if (e != cudaSuccess) return e;
  k_bias_grad<<<std::min(grid1((size_t)P * l.cout), 512), 256, l.cout * 4, n.st>>>(dz, P, l.cout, n.g + l.b_off);
  if (!want_dx) return cudaGetLastError();
  // data gradient: the 3x3 convolution of dZ with the tap-mirrored transposed weights
  if (l.taps == 9) {
    HaloSrc hs{nullptr, 0, 1, 1, dz, l.cout, h, w};
    if (n.conv_mode == 0) {
      cudaError_t e = conv3x3_ws(hs, l.wtpk, l.cout, cin, n.B, EpiStore{n.dx, cin}, n.err, n.st);
      if (e != cudaErrorNotSupported) return e;
    }
    return conv3x3(hs, l.wt, l.cout, cin, n.B, EpiStore{n.dx, cin}, n.err, n.st);
  }
  // (1x1: M = pixels, N = cin, K = cout)
  ConvSrc dsrc{nullptr, 0, 1, 1, dz, l.cout, h, w, l.taps, -1};
  ConvA a{dsrc, P, l.cout};
  RowMajor b{l.wt, cin, l.taps * l.cout, l.taps * l.cout};
  return gemm_n(a, b, EpiStore{n.dx, cin}, P, cin, l.taps * l.cout, n.err, n.st);
}

// The network on the batch in n.x0 / n.col; with infer_rgba (inference) the fused output tail
// also writes the tonemapped image there.
static cudaError_t forward(Net& n, uchar4* infer_rgba = nullptr, float exposure = 1.0f) {
  cudaError_t e;
  const int B = n.B;
  auto pool = [&](const uint16_t* in, uint16_t* outp, int lv, int C) {
    size_t cnt = (size_t)B * n.hl[lv + 1] * n.wl[lv + 1] * (C / 8);
    k_avgpool<<<grid1(cnt), 256, 0, n.st>>>(in, outp, B, n.hl[lv], n.wl[lv], C);
  };
  if ((e = conv_fwd(n, n.L[L_E0A], nullptr, n.x0, n.e0a, false))) return e;
  if ((e = conv_fwd(n, n.L[L_E0], nullptr, n.e0a, n.e0, false))) return e;
  pool(n.e0, n.p1, 0, 32);
  if ((e = conv_fwd(n, n.L[L_E1], nullptr, n.p1, n.e1, false))) return e;
  pool(n.e1, n.p2, 1, 48);
  if ((e = conv_fwd(n, n.L[L_E2], nullptr, n.p2, n.e2, false))) return e;
  pool(n.e2, n.p3, 2, 64);
  if ((e = conv_fwd(n, n.L[L_E3], nullptr, n.p3, n.e3, false))) return e;
  pool(n.e3, n.p4, 3, 96);
  if ((e = conv_fwd(n, n.L[L_E4A], nullptr, n.p4, n.e4a, false))) return e;
  if ((e = conv_fwd(n, n.L[L_E4], nullptr, n.e4a, n.e4, false))) return e;
  if ((e = conv_fwd(n, n.L[L_D3], n.e4, n.e3, n.d3, false))) return e;
  if ((e = conv_fwd(n, n.L[L_D2], n.d3, n.e2, n.d2, false))) return e;
  if ((e = conv_fwd(n, n.L[L_D1], n.d2, n.e1, n.d1, false))) return e;
  if ((e = conv_fwd(n, n.L[L_D0], n.d1, n.e0, n.d0, false))) return e;
  if (infer_rgba) {
    // inference: output layer, softmax and stage 1 fused; stages 2 and 3 read the stored kernels
    // (in the logits buffer, which inference does not otherwise use)
    const int P0 = B * n.H * n.W;
    const Layer& lo = n.L[L_OUT];
    if (!n.out_bias_valid) {
      // a host copy of the output bias, taken once after each weight change
      if ((e = cudaMemcpyAsync(n.out_bias.v, n.w + lo.b_off, sizeof n.out_bias.v, cudaMemcpyDeviceToHost, n.st)))
        return e;
      if ((e = cudaStreamSynchronize(n.st))) return e;
      n.out_bias_valid = true;
    }
    const int out_tiles = (P0 + tc::BM - 1) / tc::BM;
    k_out_softmax<<<std::min(out_tiles, sm_count() * outk::CTAS_PER_SM), outk::THREADS, outk::SMEM, n.st>>>(
        n.d0, lo.wb, n.out_bias, n.col, n.f1, n.logits, B, n.H, n.W, n.err);
    const dim3 fg((unsigned)((n.W + 31) / 32), (unsigned)((n.H + 7) / 8), (unsigned)B);
    k_filter_stored<2><<<fg, 256, 0, n.st>>>(n.logits, 0, n.f1, n.f2, nullptr, exposure, B, n.H, n.W);
    k_filter_stored<4><<<fg, 256, 0, n.st>>>(n.logits, 25, n.f2, n.out, infer_rgba, exposure, B, n.H, n.W);
    return cudaGetLastError();
  }
  if ((e = conv_fwd(n, n.L[L_OUT], nullptr, n.d0, n.logits, true))) return e;
  const int P0 = B * n.H * n.W;
  k_filter_fwd<<<grid1(P0), 256, 0, n.st>>>(n.logits, 0, 1, n.col, n.f1, B, n.H, n.W);
  k_filter_fwd<<<grid1(P0), 256, 0, n.st>>>(n.logits, 1, 2, n.f1, n.f2, B, n.H, n.W);
  k_filter_fwd<<<grid1(P0), 256, 0, n.st>>>(n.logits, 2, 4, n.f2, n.out, B, n.H, n.W);
  return cudaGetLastError();
}

// Loss and all parameter gradients (n.g, zeroed here) for the batch in n.x0 / n.col / n.tgt.
static cudaError_t backward(Net& n) {
  cudaError_t e;
  const int B = n.B;
  auto px = [&](int lv) { return (size_t)B * n.hl[lv] * n.wl[lv]; };
  if ((e = cudaMemsetAsync(n.g, 0, n.n_params * 4, n.st))) return e;
  if ((e = cudaMemsetAsync(n.loss, 0, 4, n.st))) return e;
  const int P0 = (int)px(0);
  k_filter_loss<<<grid1(px(0)), 256, 0, n.st>>>(n.out, n.tgt, P0, n.gf_a, n.loss);
  if ((e = cudaMemsetAsync(n.gf_b, 0, px(0) * 16, n.st))) return e;
  const dim3 fg((unsigned)((n.W + 31) / 32), (unsigned)((n.H + 7) / 8), (unsigned)B);
  k_filter_bwd_tiled<4><<<fg, 256, 0, n.st>>>(n.logits, 2, n.f2, n.gf_a, n.dlog, (float*)n.gf_b, B, n.H, n.W);
  if ((e = cudaMemsetAsync(n.gf_a, 0, px(0) * 16, n.st))) return e;
  k_filter_bwd_tiled<2><<<fg, 256, 0, n.st>>>(n.logits, 1, n.f1, n.gf_b, n.dlog, (float*)n.gf_a, B, n.H, n.W);
  k_filter_bwd_tiled<1><<<fg, 256, 0, n.st>>>(n.logits, 0, n.col, n.gf_a, n.dlog, nullptr, B, n.H, n.W);
  // OUT (1x1 over D0)
  if ((e = conv_bwd(n, n.L[L_OUT], n.dlog, nullptr, n.d0, true))) return e;
  uint16_t* gd0 = n.g_a;
  cudaMemcpyAsync(gd0, n.dx, px(0) * 32 * 2, cudaMemcpyDeviceToDevice, n.st);
  k_relu_mask<<<grid1(px(0) * 32), 256, 0, n.st>>>(gd0, n.d0, px(0) * 32);
  // decoder: dZ of D_l -> its gradients; input gradient split into the coarse part (masked by
  // the coarse activation) and the skip part (kept in g_skip for the encoder)
  struct Dec { int layer; const uint16_t* u; const uint16_t* s; int lv; int cu; int cs; };
  const Dec dec[4] = {{L_D0, n.d1, n.e0, 0, 48, 32}, {L_D1, n.d2, n.e1, 1, 64, 48}, {L_D2, n.d3, n.e2, 2, 96, 64},
                      {L_D3, n.e4, n.e3, 3, 128, 96}};
  // skip gradients of E0..E3 are needed after the decoder pass: keep them at offsets in g_skip
  size_t skip_off[4], off = 0;
  for (int i = 0; i < 4; ++i) { skip_off[i] = off; off += px(i) * dec[i].cs; }
  uint16_t* gz = gd0;
  uint16_t* gnext = n.g_b;
  for (int i = 0; i < 4; ++i) {
    const Dec& d = dec[i];
    if ((e = conv_bwd(n, n.L[d.layer], gz, d.u, d.s, true))) return e;
    size_t nc = (size_t)B * n.hl[d.lv + 1] * n.wl[d.lv + 1] * d.cu;
    k_split_up<<<grid1(nc), 256, 0, n.st>>>(n.dx, d.cu, d.cs, B, n.hl[d.lv], n.wl[d.lv], d.u, gnext);
    // skip part: copy channels [cu, cu+cs) of dx into g_skip (strided copy via 2D memcpy)
    cudaMemcpy2DAsync(n.g_skip + skip_off[d.lv], (size_t)d.cs * 2, n.dx + d.cu, (size_t)(d.cu + d.cs) * 2,
                      (size_t)d.cs * 2, px(d.lv), cudaMemcpyDeviceToDevice, n.st);
    std::swap(gz, gnext);
  }
  // gz = dZ of E4 (level 4, 128 channels)
  if ((e = conv_bwd(n, n.L[L_E4], gz, nullptr, n.e4a, true))) return e;
  uint16_t* ge4a = gnext;
  cudaMemcpyAsync(ge4a, n.dx, px(4) * 128 * 2, cudaMemcpyDeviceToDevice, n.st);
  k_relu_mask<<<grid1(px(4) * 128), 256, 0, n.st>>>(ge4a, n.e4a, px(4) * 128);
  if ((e = conv_bwd(n, n.L[L_E4A], ge4a, nullptr, n.p4, true))) return e;
  // encoder levels 3..0: dZ_E = mask(E) (skip + unpool(dP)), then the level's convolution
  struct Enc { int layer; const uint16_t* in; const uint16_t* e; int lv; int C; int cin; };
  const Enc enc[4] = {{L_E3, n.p3, n.e3, 3, 96, 64}, {L_E2, n.p2, n.e2, 2, 64, 48}, {L_E1, n.p1, n.e1, 1, 48, 32},
                      {L_E0, n.e0a, n.e0, 0, 32, 32}};
  for (int i = 0; i < 4; ++i) {
    const Enc& en = enc[i];
    // n.dx holds dP_{lv+1} (the data gradient of the next level's first convolution)
    cudaMemcpyAsync(n.g_pool, n.dx, px(en.lv + 1) * en.C * 2, cudaMemcpyDeviceToDevice, n.st);
    uint16_t* gz_e = n.g_a;
    k_enc_grad<<<grid1(px(en.lv) * en.C), 256, 0, n.st>>>(n.g_skip + skip_off[en.lv], en.C, 0, n.g_pool, en.e, B,
                                                          n.hl[en.lv], n.wl[en.lv], en.C, gz_e);
    if ((e = conv_bwd(n, n.L[en.layer], gz_e, nullptr, en.in, true))) return e;
  }
  // n.dx = gradient of E0a (level 0, 32 channels)
  uint16_t* ge0a = n.g_b;
  cudaMemcpyAsync(ge0a, n.dx, px(0) * 32 * 2, cudaMemcpyDeviceToDevice, n.st);
  k_relu_mask<<<grid1(px(0) * 32), 256, 0, n.st>>>(ge0a, n.e0a, px(0) * 32);
  if ((e = conv_bwd(n, n.L[L_E0A], ge0a, nullptr, n.x0, false))) return e;
  return cudaGetLastError();
}

}  // namespace kp

// ============================================================================================
// C ABI of the learned denoiser.
// ============================================================================================
#include <string>
#include "wgpt_internal.h"

struct wgpt_kpcn {
  kp::Net net;
  std::string err;
  float* d_losses = nullptr;
  int losses_cap = 0;
  kp::Crop* d_crops = nullptr;
  size_t crops_cap = 0;
  float4* d_img_col = nullptr;   // single-image staging (gradient check)
  float4* d_img_tgt = nullptr;
  float* d_img_gbuf = nullptr;
  size_t img_cap = 0;
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
};

namespace {

uint64_t splitmix(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
double uniform01(uint64_t& s) { return (double)(splitmix(s) >> 11) * (1.0 / 9007199254740992.0); }

int kfail(wgpt_kpcn* k, int code, const std::string& m) {
  if (k) k->err = m;
  return code;
}
int kcuda(wgpt_kpcn* k, cudaError_t e, const char* what) {
  return kfail(k, e == cudaErrorMemoryAllocation ? WGPT_E_NOMEM : WGPT_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}
#define KCK(call, what)                                   \
  do {                                                    \
    cudaError_t e_ = (call);                              \
    if (e_ != cudaSuccess) return kcuda(k, e_, what);     \
  } while (0)

int check_device_error(wgpt_kpcn* k) {
  uint32_t herr = 0;
  KCK(cudaMemcpyAsync(&herr, k->net.err, 4, cudaMemcpyDeviceToHost, k->net.st), "error readback");
  KCK(cudaStreamSynchronize(k->net.st), "synchronize");
  if (herr) {
    cudaMemsetAsync(k->net.err, 0, 4, k->net.st);
    return kfail(k, WGPT_E_DEVICE, "a tensor-core kernel timed out waiting for its MMAs");
  }
  return WGPT_OK;
}

// He-uniform initialisation over the real (unpadded) fan-in; padded weights stay zero.  The
// output layer starts small, so the first filters are close to a 5x5 box.
void init_params(kp::Net& n, uint64_t seed, std::vector<float>& w) {
  w.assign(n.n_params, 0.0f);
  uint64_t s = seed * 0x2545F4914F6CDD1Dull + 12345u;
  for (int i = 0; i < kp::NLAYERS; ++i) {
    const kp::Layer& l = n.L[i];
    const double a = std::sqrt(6.0 / (double)(l.taps * l.real_cin)) * (i == kp::L_OUT ? 0.1 : 1.0);
    for (int co = 0; co < l.cout; ++co)
      for (int t = 0; t < l.taps; ++t)
        for (int ci = 0; ci < l.cin(); ++ci) {
          float v = (float)((2.0 * uniform01(s) - 1.0) * a);
          bool real = co < l.real_cout && (i != kp::L_E0A || ci < l.real_cin);
          w[l.w_off + ((size_t)co * l.taps + t) * l.cin() + ci] = real ? v : 0.0f;
        }
  }
}

int stage_images(wgpt_kpcn* k, size_t npix) {
  if (k->img_cap >= npix) return WGPT_OK;
  cudaStreamSynchronize(k->net.st);
  cudaFree(k->d_img_col); cudaFree(k->d_img_tgt); cudaFree(k->d_img_gbuf);
  k->d_img_col = nullptr; k->d_img_tgt = nullptr; k->d_img_gbuf = nullptr; k->img_cap = 0;
  KCK(cudaMalloc(&k->d_img_col, npix * 16), "cudaMalloc image");
  KCK(cudaMalloc(&k->d_img_tgt, npix * 16), "cudaMalloc image");
  KCK(cudaMalloc(&k->d_img_gbuf, npix * 48), "cudaMalloc image");
  k->img_cap = npix;
  return WGPT_OK;
}

int ensure_crops(wgpt_kpcn* k, size_t n) {
  if (k->crops_cap >= n) return WGPT_OK;
  cudaStreamSynchronize(k->net.st);
  cudaFree(k->d_crops);
  k->d_crops = nullptr;
  k->crops_cap = 0;
  KCK(cudaMalloc(&k->d_crops, n * sizeof(kp::Crop)), "cudaMalloc crops");
  k->crops_cap = n;
  return WGPT_OK;
}

cudaError_t adam_step(kp::Net& n, float lr, const float* g = nullptr, float scale = 1.0f) {
  n.adam_t += 1;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.0f - (float)std::pow(0.9, n.adam_t), c2 = 1.0f - (float)std::pow(0.999, n.adam_t);
  kp::k_grad_sqnorm<<<kp::kNormBlocks, 256, 0, n.st>>>(g ? g : n.g, n.n_params, scale, n.clip);
  kp::k_clip_factor<<<1, 1, 0, n.st>>>(n.clip);
  kp::k_adam<<<kp::grid1(n.n_params), 256, 0, n.st>>>(n.w, g ? g : n.g, n.m, n.v, n.n_params, lr, b1, b2, 1e-8f, c1,
                                                      c2, scale, n.clip);
  return kp::refresh_bf16(n);
}

// Draws `count` crops of crop x crop pixels from the examples with the splitmix stream of `seed`
// and uploads them to k->d_crops.
int draw_crops(wgpt_kpcn* k, size_t count, uint32_t crop, uint64_t seed) {
  kp::Net& n = k->net;
  int rc = ensure_crops(k, count);
  if (rc) return rc;
  std::vector<kp::Crop> crops(count);
  uint64_t s = seed * 0x9E3779B97F4A7C15ull + 7u;
  for (auto& c : crops) {
    c.e = (int)(splitmix(s) % (uint64_t)n.ds_n);
    c.oy = (int)(splitmix(s) % (uint64_t)(n.ds_h - (int)crop + 1));
    c.ox = (int)(splitmix(s) % (uint64_t)(n.ds_w - (int)crop + 1));
    c.pad = 0;
  }
  KCK(cudaMemcpyAsync(k->d_crops, crops.data(), crops.size() * sizeof(kp::Crop), cudaMemcpyHostToDevice, n.st),
      "upload crops");
  KCK(cudaStreamSynchronize(n.st), "crops");
  return WGPT_OK;
}

}  // namespace

// Self-test of the tensor-core kernels' bounded waits: one thread waits on an mbarrier phase
// that nothing completes; the wait must give up after `limit` polls and report the timeout bit.
__global__ void k_selftest_wait(uint32_t limit, uint32_t* status) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    const uint32_t b = tc::smem_u32(&bar);
    tc::mbar_init(b, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    if (!tc::mbar_wait_n(b, 0u, limit)) atomicOr(status, tc::ERR_TC_TIMEOUT);
  }
}

extern "C" {

int wgpt_selftest_wait(int device, uint32_t limit, uint32_t* status, float* ms) {
  if (!status || limit == 0 || limit > (1u << 24)) return WGPT_E_INVALID;
  if (wgpt::select_device(device) != cudaSuccess) return WGPT_E_CUDA;
  uint32_t* d = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = WGPT_OK;
  if (cudaMalloc(&d, 4) != cudaSuccess) return WGPT_E_NOMEM;
  if (cudaMemset(d, 0, 4) != cudaSuccess || cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
    rc = WGPT_E_CUDA;
  } else {
    cudaEventRecord(e0);
    k_selftest_wait<<<1, 32>>>(limit, d);
    cudaEventRecord(e1);
    if (cudaEventSynchronize(e1) != cudaSuccess || cudaMemcpy(status, d, 4, cudaMemcpyDeviceToHost) != cudaSuccess)
      rc = WGPT_E_CUDA;
    else if (ms)
      cudaEventElapsedTime(ms, e0, e1);
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFree(d);
  return rc;
}

int wgpt_kpcn_create(int device, uint64_t seed, wgpt_kpcn** out) {
  if (!out) return WGPT_E_INVALID;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return WGPT_E_CUDA;
  if (device < 0 || device >= ndev) return WGPT_E_INVALID;
  if (wgpt::select_device(device) != cudaSuccess) return WGPT_E_CUDA;
  wgpt_kpcn* k = new wgpt_kpcn();
  kp::Net& n = k->net;
  n.device = device;
  kp::define_layers(n);
  cudaError_t e = cudaStreamCreateWithFlags(&n.st, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc(&n.w, n.n_params * 4);
  if (e == cudaSuccess) e = cudaMalloc(&n.g, n.n_params * 4);
  if (e == cudaSuccess) e = cudaMalloc(&n.m, n.n_params * 4);
  if (e == cudaSuccess) e = cudaMalloc(&n.v, n.n_params * 4);
  if (e == cudaSuccess) e = cudaMalloc(&n.err, 4);
  if (e == cudaSuccess) e = cudaMalloc(&n.loss, 4);
  if (e == cudaSuccess) e = cudaMalloc(&n.clip, (4 + kp::kNormBlocks) * 4);
  if (e == cudaSuccess) e = cudaMemset(n.clip, 0, (4 + kp::kNormBlocks) * 4);
  for (int i = 0; i < kp::NLAYERS && e == cudaSuccess; ++i) {
    e = cudaMalloc(&n.L[i].wb, n.L[i].nw() * 2);
    if (e == cudaSuccess) e = cudaMalloc(&n.L[i].wt, n.L[i].nw() * 2);
    if (e == cudaSuccess && n.L[i].taps == 9) {
      e = cudaMalloc(&n.L[i].wpk, kp::ws_packed_elems(n.L[i].cout, n.L[i].cin()) * 2);
      if (e == cudaSuccess) e = cudaMalloc(&n.L[i].wtpk, kp::ws_packed_elems(n.L[i].cin(), n.L[i].cout) * 2);
    }
  }
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&k->ev_in, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&k->ev_out, cudaEventDisableTiming);
  std::vector<float> w;
  if (e == cudaSuccess) {
    init_params(n, seed, w);
    e = cudaMemcpy(n.w, w.data(), n.n_params * 4, cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess) e = cudaMemset(n.m, 0, n.n_params * 4);
  if (e == cudaSuccess) e = cudaMemset(n.v, 0, n.n_params * 4);
  if (e == cudaSuccess) e = cudaMemset(n.err, 0, 4);
  if (e == cudaSuccess) e = kp::refresh_bf16(n);
  if (e == cudaSuccess) e = cudaStreamSynchronize(n.st);
  if (e != cudaSuccess) {
    wgpt_kpcn_destroy(k);
    return e == cudaErrorMemoryAllocation ? WGPT_E_NOMEM : WGPT_E_CUDA;
  }
  *out = k;
  return WGPT_OK;
}

int wgpt_kpcn_destroy(wgpt_kpcn* k) {
  if (!k) return WGPT_E_INVALID;
  kp::Net& n = k->net;
  wgpt::select_device(n.device);
  if (n.st) cudaStreamSynchronize(n.st);
  for (void* p : n.bufs) cudaFree(p);
  for (int i = 0; i < kp::NLAYERS; ++i) {
    cudaFree(n.L[i].wb); cudaFree(n.L[i].wt); cudaFree(n.L[i].wpk); cudaFree(n.L[i].wtpk);
  }
  cudaFree(n.w); cudaFree(n.g); cudaFree(n.m); cudaFree(n.v); cudaFree(n.err); cudaFree(n.loss); cudaFree(n.clip);
  cudaFree(n.ds_col); cudaFree(n.ds_tgt); cudaFree(n.ds_gbuf);
  cudaFree(k->d_losses); cudaFree(k->d_crops);
  cudaFree(k->d_img_col); cudaFree(k->d_img_tgt); cudaFree(k->d_img_gbuf);
  if (k->ev_in) cudaEventDestroy(k->ev_in);
  if (k->ev_out) cudaEventDestroy(k->ev_out);
  if (n.st) cudaStreamDestroy(n.st);
  delete k;
  return WGPT_OK;
}

const char* wgpt_kpcn_last_error(wgpt_kpcn* k) { return k ? k->err.c_str() : "null denoiser"; }

int wgpt_kpcn_set_conv_mode(wgpt_kpcn* k, int mode) {
  if (!k) return WGPT_E_INVALID;
  if (mode != WGPT_KPCN_CONV_PIPELINED && mode != WGPT_KPCN_CONV_PER_TILE) return kfail(k, WGPT_E_INVALID, "unknown conv mode");
  k->net.conv_mode = mode;
  return WGPT_OK;
}

int wgpt_kpcn_num_params(wgpt_kpcn* k, uint64_t* n) {
  if (!k || !n) return WGPT_E_INVALID;
  *n = k->net.n_params;
  return WGPT_OK;
}

int wgpt_kpcn_get_params(wgpt_kpcn* k, float* dst) {
  if (!k || !dst) return WGPT_E_INVALID;
  wgpt::select_device(k->net.device);
  KCK(cudaMemcpyAsync(dst, k->net.w, k->net.n_params * 4, cudaMemcpyDeviceToHost, k->net.st), "read params");
  KCK(cudaStreamSynchronize(k->net.st), "synchronize");
  return WGPT_OK;
}

int wgpt_kpcn_set_params(wgpt_kpcn* k, const float* src) {
  if (!k || !src) return WGPT_E_INVALID;
  kp::Net& n = k->net;
  wgpt::select_device(n.device);
  KCK(cudaMemcpyAsync(n.w, src, n.n_params * 4, cudaMemcpyHostToDevice, n.st), "write params");
  KCK(cudaMemsetAsync(n.m, 0, n.n_params * 4, n.st), "reset moments");
  KCK(cudaMemsetAsync(n.v, 0, n.n_params * 4, n.st), "reset moments");
  KCK(cudaMemsetAsync(n.clip, 0, 16, n.st), "reset clipping");   // the partial sums are rewritten each step
  n.adam_t = 0;
  KCK(kp::refresh_bf16(n), "bf16 weights");
  KCK(cudaStreamSynchronize(n.st), "synchronize");
  return WGPT_OK;
}

int wgpt_kpcn_add_example(wgpt_kpcn* k, const float* noisy, const void* gbuf, const float* target, uint32_t w,
                          uint32_t h) {
  if (!k || !noisy || !gbuf || !target || w < 16 || h < 16) return WGPT_E_INVALID;
  kp::Net& n = k->net;
  wgpt::select_device(n.device);
  if (n.ds_n > 0 && ((int)w != n.ds_w || (int)h != n.ds_h))
    return kfail(k, WGPT_E_INVALID, "every example must have the size of the first");
  const size_t npix = (size_t)w * h;
  if (n.ds_n == n.ds_cap) {
    int cap = std::max(8, n.ds_cap * 2);
    float4 *c = nullptr, *t = nullptr;
    float* g = nullptr;
    KCK(cudaMalloc(&c, npix * 16 * cap), "cudaMalloc dataset");
    KCK(cudaMalloc(&t, npix * 16 * cap), "cudaMalloc dataset");
    KCK(cudaMalloc(&g, npix * 48 * cap), "cudaMalloc dataset");
    if (n.ds_n) {
      KCK(cudaMemcpyAsync(c, n.ds_col, npix * 16 * n.ds_n, cudaMemcpyDeviceToDevice, n.st), "copy dataset");
      KCK(cudaMemcpyAsync(t, n.ds_tgt, npix * 16 * n.ds_n, cudaMemcpyDeviceToDevice, n.st), "copy dataset");
      KCK(cudaMemcpyAsync(g, n.ds_gbuf, npix * 48 * n.ds_n, cudaMemcpyDeviceToDevice, n.st), "copy dataset");
    }
    KCK(cudaStreamSynchronize(n.st), "synchronize");
    cudaFree(n.ds_col); cudaFree(n.ds_tgt); cudaFree(n.ds_gbuf);
    n.ds_col = c; n.ds_tgt = t; n.ds_gbuf = g;
    n.ds_cap = cap;
  }
  n.ds_w = (int)w;
  n.ds_h = (int)h;
  KCK(cudaMemcpyAsync(n.ds_col + npix * n.ds_n, noisy, npix * 16, cudaMemcpyHostToDevice, n.st), "upload example");
  KCK(cudaMemcpyAsync(n.ds_tgt + npix * n.ds_n, target, npix * 16, cudaMemcpyHostToDevice, n.st), "upload example");
  KCK(cudaMemcpyAsync(n.ds_gbuf + npix * 12 * n.ds_n, gbuf, npix * 48, cudaMemcpyHostToDevice, n.st), "upload example");
  KCK(cudaStreamSynchronize(n.st), "synchronize");
  n.ds_n += 1;
  return WGPT_OK;
}

int wgpt_kpcn_num_examples(wgpt_kpcn* k, uint32_t* n) {
  if (!k || !n) return WGPT_E_INVALID;
  *n = (uint32_t)k->net.ds_n;
  return WGPT_OK;
}

int wgpt_kpcn_train(wgpt_kpcn* k, uint32_t steps, uint32_t batch, uint32_t crop, float lr, uint64_t seed,
                    float* losses) {
  if (!k || batch == 0 || batch > 64 || crop < 16 || crop > 512 || (crop % 16) != 0 || !(lr > 0.0f))
    return WGPT_E_INVALID;
  kp::Net& n = k->net;
  if (n.ds_n == 0) return kfail(k, WGPT_E_STATE, "no training examples");
  if ((int)crop > n.ds_w || (int)crop > n.ds_h) return kfail(k, WGPT_E_INVALID, "crop larger than the examples");
  if (steps == 0) return WGPT_OK;
  wgpt::select_device(n.device);
  KCK(kp::ensure_batch(n, (int)batch, (int)crop, (int)crop), "batch buffers");
  if (k->losses_cap < (int)steps) {
    cudaFree(k->d_losses);
    k->d_losses = nullptr;
    KCK(cudaMalloc(&k->d_losses, steps * 4), "cudaMalloc losses");
    k->losses_cap = (int)steps;
  }
  int rc = draw_crops(k, (size_t)steps * batch, crop, seed);
  if (rc) return rc;
  const size_t P = (size_t)batch * crop * crop;
  for (uint32_t it = 0; it < steps; ++it) {
    kp::k_gather<<<kp::grid1(P), 256, 0, n.st>>>(n.ds_col, n.ds_gbuf, n.ds_tgt, n.ds_h, n.ds_w,
                                                 k->d_crops + (size_t)it * batch, (int)batch, (int)crop, (int)crop,
                                                 n.x0, n.col, n.tgt);
    KCK(kp::forward(n), "forward");
    KCK(kp::backward(n), "backward");
    KCK(cudaMemcpyAsync(k->d_losses + it, n.loss, 4, cudaMemcpyDeviceToDevice, n.st), "loss copy");
    KCK(adam_step(n, lr), "adam");
  }
  if (losses) KCK(cudaMemcpyAsync(losses, k->d_losses, steps * 4, cudaMemcpyDeviceToHost, n.st), "losses readback");
  return check_device_error(k);
}

int wgpt_kpcn_grads(wgpt_kpcn* k, uint32_t batch, uint32_t crop, uint64_t seed, float* loss, float* dev_grads) {
  if (!k || !dev_grads || batch == 0 || batch > 64 || crop < 16 || crop > 512 || (crop % 16) != 0)
    return WGPT_E_INVALID;
  kp::Net& n = k->net;
  if (n.ds_n == 0) return kfail(k, WGPT_E_STATE, "no training examples");
  if ((int)crop > n.ds_w || (int)crop > n.ds_h) return kfail(k, WGPT_E_INVALID, "crop larger than the examples");
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, dev_grads) != cudaSuccess || at.type != cudaMemoryTypeDevice ||
      at.device != n.device) {
    cudaGetLastError();
    return kfail(k, WGPT_E_INVALID, "dev_grads must be device memory on the denoiser's device");
  }
  wgpt::select_device(n.device);
  KCK(kp::ensure_batch(n, (int)batch, (int)crop, (int)crop), "batch buffers");
  int rc = draw_crops(k, batch, crop, seed);
  if (rc) return rc;
  const size_t P = (size_t)batch * crop * crop;
  kp::k_gather<<<kp::grid1(P), 256, 0, n.st>>>(n.ds_col, n.ds_gbuf, n.ds_tgt, n.ds_h, n.ds_w, k->d_crops, (int)batch,
                                               (int)crop, (int)crop, n.x0, n.col, n.tgt);
  KCK(kp::forward(n), "forward");
  KCK(kp::backward(n), "backward");
  KCK(cudaMemcpyAsync(dev_grads, n.g, n.n_params * 4, cudaMemcpyDeviceToDevice, n.st), "gradient copy");
  if (loss) KCK(cudaMemcpyAsync(loss, n.loss, 4, cudaMemcpyDeviceToHost, n.st), "loss readback");
  KCK(cudaStreamSynchronize(n.st), "synchronize");
  return check_device_error(k);
}

int wgpt_kpcn_apply(wgpt_kpcn* k, const float* dev_grads, float scale, float lr) {
  if (!k || !dev_grads || !(lr > 0.0f) || !(scale == scale)) return WGPT_E_INVALID;
  kp::Net& n = k->net;
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, dev_grads) != cudaSuccess || at.type != cudaMemoryTypeDevice ||
      at.device != n.device) {
    cudaGetLastError();
    return kfail(k, WGPT_E_INVALID, "dev_grads must be device memory on the denoiser's device");
  }
  wgpt::select_device(n.device);
  KCK(adam_step(n, lr, dev_grads, scale), "adam");
  KCK(cudaStreamSynchronize(n.st), "synchronize");
  return check_device_error(k);
}

int wgpt_kpcn_loss_and_grads(wgpt_kpcn* k, const float* noisy, const void* gbuf, const float* target, uint32_t w,
                             uint32_t h, float* loss, float* grads, float* out_rgba32f) {
  if (!k || !noisy || !gbuf || !target || w < 16 || h < 16 || w > 4096 || h > 4096) return WGPT_E_INVALID;
  kp::Net& n = k->net;
  wgpt::select_device(n.device);
  const size_t npix = (size_t)w * h;
  int rc = stage_images(k, npix);
  if (rc) return rc;
  rc = ensure_crops(k, 1);
  if (rc) return rc;
  KCK(kp::ensure_batch(n, 1, (int)h, (int)w), "batch buffers");
  kp::Crop c0{0, 0, 0, 0};
  KCK(cudaMemcpyAsync(k->d_crops, &c0, sizeof c0, cudaMemcpyHostToDevice, n.st), "upload crop");
  KCK(cudaMemcpyAsync(k->d_img_col, noisy, npix * 16, cudaMemcpyHostToDevice, n.st), "upload image");
  KCK(cudaMemcpyAsync(k->d_img_tgt, target, npix * 16, cudaMemcpyHostToDevice, n.st), "upload image");
  KCK(cudaMemcpyAsync(k->d_img_gbuf, gbuf, npix * 48, cudaMemcpyHostToDevice, n.st), "upload image");
  kp::k_gather<<<kp::grid1(npix), 256, 0, n.st>>>(k->d_img_col, k->d_img_gbuf, k->d_img_tgt, (int)h, (int)w,
                                                  k->d_crops, 1, (int)h, (int)w, n.x0, n.col, n.tgt);
  KCK(kp::forward(n), "forward");
  KCK(kp::backward(n), "backward");
  if (loss) KCK(cudaMemcpyAsync(loss, n.loss, 4, cudaMemcpyDeviceToHost, n.st), "loss readback");
  if (grads) KCK(cudaMemcpyAsync(grads, n.g, n.n_params * 4, cudaMemcpyDeviceToHost, n.st), "grads readback");
  if (out_rgba32f) KCK(cudaMemcpyAsync(out_rgba32f, n.out, npix * 16, cudaMemcpyDeviceToHost, n.st), "output readback");
  return check_device_error(k);
}

static int denoise_image(wgpt_kpcn* k, wgpt_ctx* ctx, int view, float exposure, float* filtered_rgba32f) {
  if (!k || !ctx) return WGPT_E_INVALID;
  kp::Net& n = k->net;
  wgpt::CtxImages im;
  if (!wgpt::ctx_images(ctx, view, &im)) return kfail(k, WGPT_E_STATE, "no such image (resize or set views first)");
  if (!im.gbuf) return kfail(k, WGPT_E_STATE, "context has no G-buffer: resize with want_gbuf and render it");
  if (im.device != n.device) return kfail(k, WGPT_E_INVALID, "context and denoiser are on different devices");
  wgpt::select_device(n.device);
  const size_t npix = (size_t)im.w * im.h;
  int rc = ensure_crops(k, 1);
  if (rc) return rc;
  KCK(kp::ensure_batch(n, 1, (int)im.h, (int)im.w), "batch buffers");
  kp::Crop c0{0, 0, 0, 0};
  KCK(cudaMemcpyAsync(k->d_crops, &c0, sizeof c0, cudaMemcpyHostToDevice, n.st), "upload crop");
  // the denoiser's stream waits for the context's queued work and the context's stream for the
  // denoiser's result
  KCK(cudaEventRecord(k->ev_in, im.stream), "event");
  KCK(cudaStreamWaitEvent(n.st, k->ev_in, 0), "event wait");
  kp::k_gather<<<kp::grid1(npix), 256, 0, n.st>>>((const float4*)im.accum, im.gbuf, nullptr, (int)im.h, (int)im.w,
                                                  k->d_crops, 1, (int)im.h, (int)im.w, n.x0, n.col, nullptr);
  KCK(kp::forward(n, (uchar4*)im.out, exposure), "forward");
  KCK(cudaGetLastError(), "denoise launch");
  KCK(cudaEventRecord(k->ev_out, n.st), "event");
  KCK(cudaStreamWaitEvent(im.stream, k->ev_out, 0), "event wait");
  if (filtered_rgba32f) {
    KCK(cudaMemcpyAsync(filtered_rgba32f, n.out, npix * 16, cudaMemcpyDeviceToHost, n.st), "filtered readback");
    return check_device_error(k);
  }
  return WGPT_OK;
}

int wgpt_kpcn_denoise(wgpt_kpcn* k, wgpt_ctx* ctx, float exposure, float* filtered_rgba32f) {
  return denoise_image(k, ctx, -1, exposure, filtered_rgba32f);
}

int wgpt_kpcn_denoise_view(wgpt_kpcn* k, wgpt_ctx* ctx, uint32_t view, float exposure, float* filtered_rgba32f) {
  return denoise_image(k, ctx, (int)view, exposure, filtered_rgba32f);
}

}  // extern "C"
