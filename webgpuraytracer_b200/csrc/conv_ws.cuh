// Warp-specialised 3x3 convolution on the tensor cores (tcgen05) with TMA halo loads.
//
// The same mathematics as k_conv3x3 (9 shifted GEMMs over a shared-memory halo per 16 input
// channels; tap (dy, dx) is a descriptor offset into the halo), organised as a persistent
// producer / MMA / epilogue pipeline:
//
//   warps 0-1  loaders: for every (tile, 16-channel chunk) fill one ring stage -- the two 8-channel
//              18 x 18 halo planes by TMA (cp.async.bulk.tensor, zero fill outside the image) when
//              the chunk comes from the tensor at the output resolution, by 16-byte loads when it
//              is the 2x-upsampled coarse tensor, and the chunk's 9-tap weights by one bulk copy
//              (cp.async.bulk) of a block pre-arranged in the shared-memory layout;
//   warp 2     MMA: one lane issues the 18 tcgen05.mma of a chunk (2 M tiles x 9 taps) into one of
//              two tensor-memory accumulators and commits the stage back to the loaders;
//   warps 3-6  epilogue: tcgen05.ld of the finished accumulator (warp w reads lanes
//              32*(w%4)..32*(w%4)+31, the tile rows), the layer's epilogue functor, then hands the
//              accumulator back, so a tile's stores overlap the next tile's MMAs.
//
// Stages are tracked by mbarriers: full (loaders -> MMA, 64 arrivals + TMA/bulk transaction
// bytes), empty (MMA -> loaders, tcgen05.commit), acc_full (MMA -> epilogue, commit) and
// acc_empty (epilogue -> MMA, 128 arrivals).  Every wait is bounded; on expiry the kernel records
// ERR_TC_TIMEOUT, stops issuing work, waits (bounded) for its own copies and MMAs in flight and
// frees its tensor memory before returning.
//
// The TMA tensor maps cover only this GPU's own activation buffers and no load uses cluster
// multicast.
#pragma once
#include <cuda.h>
#include <cudaTypedefs.h>
#include <stdint.h>
#include <cuda_runtime.h>

#include "tc_gemm.cuh"

namespace ws {

constexpr int HW = 18;                        // halo width / height
constexpr int PLANE_BYTES = HW * HW * 16;     // 8 channels x 18 x 18 pixels (5184 B, the TMA box)
constexpr int PLANE_STRIDE = 5248;            // padded to 128-byte alignment for the second plane
constexpr int HALO_BYTES = 2 * PLANE_STRIDE;
constexpr int LOADER_THREADS = 64;
constexpr int THREADS = 224;                  // 2 loader warps, 1 MMA warp, 4 epilogue warps

__host__ __device__ constexpr int wts_bytes(int nt) { return 9 * nt * 32; }
__host__ __device__ constexpr int stage_bytes(int nt) { return ((HALO_BYTES + wts_bytes(nt)) + 1023) / 1024 * 1024; }
// ring depth: 3 stages where two CTAs share an SM (up to 64 output channels: 256 tensor-memory
// columns each), 4 where one CTA holds all 512 columns
__host__ __device__ constexpr int stages_for(int nt) { return nt <= 64 ? 3 : 4; }
__host__ __device__ constexpr int smem_bytes(int nt) { return stages_for(nt) * stage_bytes(nt) + 2048; }
__host__ __device__ constexpr uint32_t acc_cols(int nt) {
  return 4 * nt <= 32 ? 32u : 4 * nt <= 64 ? 64u : 4 * nt <= 128 ? 128u : 4 * nt <= 256 ? 256u : 512u;
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
// Adds transaction bytes to the current phase without arriving.
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.expect_tx.relaxed.cta.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
using tc::cp_async_16;
using tc::cp_async_commit;
using tc::cp_async_wait;
__device__ __forceinline__ void tma_load_4d(uint32_t dst, const CUtensorMap* map, int c, int x, int y, int b,
                                            uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c), "r"(x), "r"(y), "r"(b), "r"(bar)
      : "memory");
}
__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(bar)
               : "memory");
}

// Geometry of one launch.  The source of a chunk of 16 input channels starting at ci is the
// coarse tensor u (read 2x upsampled, channels [0, cu)) or the tensor s at the output
// resolution (channels [cu, cu + cs), through the tensor map).
struct ConvGeom {
  const uint16_t* u;
  int cu, hc, wc;
  int cs;
  int h, w, B;
  int cin, N;            // input channels, output channels
  int tiles_x, tiles_y, ntn;
  int n_tiles;
};

// wpk: per N tile and chunk, the 9 taps' weights in the shared-memory core-matrix layout
// (t * NT * 32 + ((n / 8) * 2 + c / 8) * 128 + (n % 8) * 16 + (c % 8) * 2 bytes).
template <int NT, class EP>
__global__ void __launch_bounds__(THREADS, 1)
k_conv3x3_ws(const __grid_constant__ CUtensorMap tmap, ConvGeom g, const uint16_t* __restrict__ wpk, EP ep,
             uint32_t* err) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  constexpr int SB = stage_bytes(NT);
  constexpr int STAGES = stages_for(NT);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + STAGES * SB);
  // full[STAGES], empty[STAGES], acc_full[2], acc_empty[2], then the TMEM address and flags
  const uint32_t bar_base = tc::smem_u32(bars);
  auto full_bar = [&](int s) { return bar_base + 8u * (uint32_t)s; };
  auto empty_bar = [&](int s) { return bar_base + 8u * (uint32_t)(STAGES + s); };
  auto accf_bar = [&](int a) { return bar_base + 8u * (uint32_t)(2 * STAGES + a); };
  auto acce_bar = [&](int a) { return bar_base + 8u * (uint32_t)(2 * STAGES + 2 + a); };
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * STAGES + 4);
  volatile uint32_t* abort_flag = tmem_slot + 1;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  constexpr uint32_t NCOLS = acc_cols(NT);
  if (warp == 2) tc::tmem_alloc(tc::smem_u32(tmem_slot), NCOLS);
  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) {
      tc::mbar_init(full_bar(s), LOADER_THREADS);
      tc::mbar_init(empty_bar(s), 1);
    }
    for (int a = 0; a < 2; ++a) {
      tc::mbar_init(accf_bar(a), 1);
      tc::mbar_init(acce_bar(a), 128);
    }
    *abort_flag = 0u;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const int KT = g.cin / 16;
  const int KT_UP = g.cu / 16;   // the first KT_UP chunks come from the upsampled tensor

  auto fail = [&]() {
    *abort_flag = 1u;
    atomicOr(err, tc::ERR_TC_TIMEOUT);
  };

  if (warp < 2) {
    // ------------------------------------------------------------------ loaders
    int stage = 0;
    uint32_t phase = 0;
    int filled = 0;   // stages filled in total (to drain copies on abort)
    int pend = -1;    // stage whose 16-byte copies are in flight, not yet arrived on
    bool ok = true;
    for (int tile = blockIdx.x; tile < g.n_tiles && ok; tile += gridDim.x) {
      const int nt = tile % g.ntn, rest = tile / g.ntn;
      const int tx = rest % g.tiles_x, ty = (rest / g.tiles_x) % g.tiles_y, b = rest / (g.tiles_x * g.tiles_y);
      const int x0 = tx * 16, y0 = ty * 16;
      for (int kt = 0; kt < KT; ++kt) {
        if (*abort_flag) { ok = false; break; }
        // wait for the MMAs that read this stage last time round
        if (!tc::mbar_wait(empty_bar(stage), phase ^ 1u)) { fail(); ok = false; break; }
        uint8_t* st = smem + stage * SB;
        const uint32_t st_addr = tc::smem_u32(st);
        const uint16_t* wsrc = wpk + ((size_t)nt * KT + kt) * (wts_bytes(NT) / 2);
        if (kt >= KT_UP) {
          if (tid == 0) {
            mbar_arrive_tx(full_bar(stage), 2u * PLANE_BYTES + (uint32_t)wts_bytes(NT));
            const int c = (kt - KT_UP) * 16;
            tma_load_4d(st_addr, &tmap, c, x0 - 1, y0 - 1, b, full_bar(stage));
            tma_load_4d(st_addr + PLANE_STRIDE, &tmap, c + 8, x0 - 1, y0 - 1, b, full_bar(stage));
            bulk_load(st_addr + HALO_BYTES, wsrc, (uint32_t)wts_bytes(NT), full_bar(stage));
          } else {
            mbar_arrive(full_bar(stage));
          }
        } else {
          // upsampled coarse channels: one 16-byte asynchronous copy per halo position and
          // plane from its coarse pixel (zero outside the image); the stage is arrived on once
          // the copies have landed, after the next stage has been issued (below), so the copies
          // of consecutive stages overlap
          const int ci = kt * 16;
          for (int i = tid; i < 2 * HW * HW; i += LOADER_THREADS) {
            const int pl = i / (HW * HW), q = i - pl * (HW * HW), hy = q / HW, hx = q - hy * HW;
            const int y = y0 - 1 + hy, x = x0 - 1 + hx;
            const bool in = y >= 0 && y < g.h && x >= 0 && x < g.w;
            const uint16_t* src = in ? g.u + (((size_t)b * g.hc + (y >> 1)) * g.wc + (x >> 1)) * g.cu + ci + pl * 8 : g.u;
            cp_async_16(st_addr + (uint32_t)(pl * PLANE_STRIDE + q * 16), src, in ? 16u : 0u);
          }
          cp_async_commit();
          if (tid == 0) {
            mbar_expect_tx(full_bar(stage), (uint32_t)wts_bytes(NT));
            bulk_load(st_addr + HALO_BYTES, wsrc, (uint32_t)wts_bytes(NT), full_bar(stage));
          }
        }
        // the previous stage filled by 16-byte copies: once this thread's copies have landed,
        // make them visible to the tensor cores' proxy and arrive (stages older than the one
        // just issued cannot wait on anything this thread still holds, so this never deadlocks)
        if (pend >= 0) {
          if (kt < KT_UP) cp_async_wait<1>(); else cp_async_wait<0>();
          tc::fence_async_smem();
          mbar_arrive(full_bar(pend));
          pend = -1;
        }
        if (kt < KT_UP) pend = stage;
        ++filled;
        if (++stage == STAGES) { stage = 0; phase ^= 1u; }
      }
    }
    if (pend >= 0) {
      cp_async_wait<0>();
      tc::fence_async_smem();
      mbar_arrive(full_bar(pend));
    }
    if (!ok && tid == 0) {
      // drain: every stage filled so far must have landed before the CTA can leave
      const int n = filled < STAGES ? filled : STAGES;
      int s = stage;
      uint32_t ph = phase;
      for (int i = 0; i < n; ++i) {
        if (--s < 0) { s = STAGES - 1; ph ^= 1u; }
        tc::mbar_wait(full_bar(s), ph);
      }
    }
  } else if (warp == 2) {
    // ------------------------------------------------------------------ MMA issuer
    if (lane == 0) {
      constexpr uint32_t IDESC = tc::idesc_bf16(NT);
      int stage = 0;
      uint32_t phase = 0;
      int acc = 0;
      uint32_t acc_phase = 0;
      bool ok = true;
      bool issued = false;
      uint32_t last_commit_bar = 0, last_commit_parity = 0;
      for (int tile = blockIdx.x; tile < g.n_tiles && ok; tile += gridDim.x) {
        if (*abort_flag) { ok = false; break; }
        if (!tc::mbar_wait(acce_bar(acc), acc_phase ^ 1u)) { fail(); ok = false; break; }
        tc::tc_fence_after();
        const uint32_t d0 = tmem + (uint32_t)(acc * 2 * NT);
        for (int kt = 0; kt < KT; ++kt) {
          if (!tc::mbar_wait(full_bar(stage), phase)) { fail(); ok = false; break; }
          tc::tc_fence_after();
          const uint32_t ha = tc::smem_u32(smem + stage * SB), wa = ha + HALO_BYTES;
#pragma unroll
          for (int t = 0; t < 9; ++t) {
            const int dy = t / 3, dx = t % 3;
            const uint64_t db = tc::smem_desc(wa + t * NT * 32, 128, 256);
#pragma unroll
            for (int m = 0; m < 2; ++m) {
              const uint64_t da = tc::smem_desc(ha + (dy * HW + 8 * m + dx) * 16, PLANE_STRIDE, HW * 16);
              tc::mma_bf16(d0 + (uint32_t)(m * NT), da, db, IDESC, (kt > 0 || t > 0) ? 1u : 0u);
            }
          }
          tc::mma_commit(empty_bar(stage));
          last_commit_bar = empty_bar(stage);
          last_commit_parity = phase;
          issued = true;
          if (++stage == STAGES) { stage = 0; phase ^= 1u; }
        }
        if (!ok) break;
        tc::mma_commit(accf_bar(acc));
        if (++acc == 2) { acc = 0; acc_phase ^= 1u; }
      }
      // on abort, the MMAs in flight must finish before the tensor memory is freed
      if (!ok && issued) tc::mbar_wait(last_commit_bar, last_commit_parity);
    }
  } else {
    // ------------------------------------------------------------------ epilogue
    const int q = warp & 3;                       // TMEM lane quadrant of this warp
    const int r = q * 32 + lane;                  // tile row = pixel of an 8 x 16 M tile
    int acc = 0;
    uint32_t acc_phase = 0;
    for (int tile = blockIdx.x; tile < g.n_tiles; tile += gridDim.x) {
      // lane 0 decides for the warp, so the warp-wide tcgen05.ld below is never divergent
      uint32_t go = 0;
      if (lane == 0) {
        go = *abort_flag ? 0u : 1u;
        if (go && !tc::mbar_wait(accf_bar(acc), acc_phase)) { fail(); go = 0u; }
      }
      go = __shfl_sync(0xffffffffu, go, 0);
      if (!go) break;
      tc::tc_fence_after();
      const int nt = tile % g.ntn, rest = tile / g.ntn;
      const int tx = rest % g.tiles_x, ty = (rest / g.tiles_x) % g.tiles_y, b = rest / (g.tiles_x * g.tiles_y);
      const int n0 = nt * NT;
      const int y = ty * 16 + (r >> 3);
#pragma unroll
      for (int m = 0; m < 2; ++m) {
        const int x = tx * 16 + 8 * m + (r & 7);
#pragma unroll
        for (int c0 = 0; c0 < NT; c0 += 16) {
          float v[16];
          tc::tmem_ld16(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(acc * 2 * NT + m * NT + c0), v);
          if (y < g.h && x < g.w && n0 + c0 < g.N) ep((int)(((size_t)b * g.h + y) * g.w + x), n0 + c0, v);
        }
      }
      tc::tc_fence_before();
      mbar_arrive(acce_bar(acc));
      if (++acc == 2) { acc = 0; acc_phase ^= 1u; }
    }
  }
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 2) tc::tmem_free(tmem, NCOLS);
}

// Tensor map of an NHWC BF16 tensor [B][h][w][c] with an 8-channel x 18 x 18 box.
inline cudaError_t make_halo_map(CUtensorMap* map, const void* base, int c, int w, int h, int B) {
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  if (!encode) {
    cudaDriverEntryPointQueryResult q;
    void* fn = nullptr;
    cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
    if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn) return cudaErrorNotSupported;
    encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  }
  const cuuint64_t dims[4] = {(cuuint64_t)c, (cuuint64_t)w, (cuuint64_t)h, (cuuint64_t)B};
  const cuuint64_t strides[3] = {(cuuint64_t)c * 2, (cuuint64_t)w * c * 2, (cuuint64_t)h * w * c * 2};
  const cuuint32_t box[4] = {8, HW, HW, 1};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void*>(base), dims, strides, box, estr,
                      CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

}  // namespace ws
