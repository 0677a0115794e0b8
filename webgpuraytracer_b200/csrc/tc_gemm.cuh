// BF16 tensor-core GEMM core for sm_100a (tcgen05): D[M x N] = sum_k A[m][k] * B[n][k] with FP32
// accumulation in tensor memory.
//
// One CTA of 128 threads computes a 128 x BN tile.  Operand tiles of 128 (A) and BN (B) rows by
// 64 K-elements are gathered by the threads from global memory through loader functors (so a
// convolution's implicit im2col, a transpose or a plain row-major matrix all use the same core)
// and stored in shared memory in the no-swizzle K-major "core matrix" layout: 8 rows x 16 bytes
// per core matrix, core (row/8, k/8) at byte ((row/8) * 8 + k/8) * 128.  The elected thread
// issues four tcgen05.mma (K = 16 each) per tile and commits them to an mbarrier; two smem stages
// let the next tile's loads overlap the running MMAs.  The epilogue reads the accumulator with
// tcgen05.ld (warp w owns TMEM lanes 32w..32w+31 = tile rows) and hands 16 columns at a time to
// an epilogue functor.  Every mbarrier wait is bounded: on expiry the kernel records an error,
// waits (bounded) for its own MMAs and frees its tensor memory before returning.
#pragma once
#include <stdint.h>
#include <cuda_runtime.h>

namespace tc {

constexpr int BM = 128;          // tile rows (TMEM lanes)
constexpr int BK = 64;           // K elements per smem stage
constexpr int THREADS = 128;
constexpr uint32_t WAIT_LIMIT = 1u << 22;
enum : uint32_t { ERR_TC_TIMEOUT = 4u };

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor, no swizzle, K-major (tcgen05 "version 1" format):
// start address, leading byte offset (next core matrix along K), stride byte offset (next
// 8-row group), all in 16-byte units.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1u << 46;
  return d;
}

// Instruction descriptor of kind::f16 with BF16 A/B, FP32 D, both operands K-major, M = 128.
__host__ __device__ constexpr uint32_t idesc_bf16(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
      :
      : "r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

// Waits for the completion of the mbarrier phase with the given parity; false after `limit`
// polls.
__device__ __forceinline__ bool mbar_wait_n(uint32_t bar, uint32_t parity, uint32_t limit) {
  for (uint32_t i = 0; i < limit; ++i) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) { return mbar_wait_n(bar, parity, WAIT_LIMIT); }

__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_alloc(uint32_t dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst_smem), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 16 consecutive FP32 accumulator columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

template <int BN>
struct Smem {
  static constexpr int A_BYTES = BM * BK * 2;
  static constexpr int B_BYTES = BN * BK * 2;
  static constexpr int STAGE = A_BYTES + B_BYTES;
  static constexpr int BYTES = 2 * STAGE + 64;   // + two mbarriers and the TMEM address
};

__host__ __device__ constexpr uint32_t tmem_cols(int bn) {
  return bn <= 32 ? 32u : bn <= 64 ? 64u : bn <= 128 ? 128u : 256u;
}

// Stores one 16-byte chunk (8 K-elements) of tile row r, K-chunk c into the core-matrix layout.
__device__ __forceinline__ void put_chunk(uint8_t* tile, int r, int c, uint4 v) {
  *reinterpret_cast<uint4*>(tile + ((r >> 3) * (BK / 8) + c) * 128 + (r & 7) * 16) = v;
}
// Byte offset of element (r, k) of a tile in the core-matrix layout.
__device__ __forceinline__ int elem_off(int r, int k) { return ((r >> 3) * (BK / 8) + (k >> 3)) * 128 + (r & 7) * 16 + (k & 7) * 2; }

// MN-major tiles (operands whose 8 consecutive M or N elements of one K index are contiguous in
// memory, e.g. the NHWC activations of a weight gradient, where K runs over pixels): each core
// matrix holds 8 K indices x 16 bytes of 8 consecutive M (N) elements, at the same core
// positions as the K-major layout ((row/8) * (BK/8) + k/8) * 128, so the descriptors keep
// LBO = 128 B (next core along K) and SBO = 1024 B (next core along M/N, the no-swizzle
// MN-major canonical form) and the instruction descriptor's transpose bit selects the layout.
__device__ __forceinline__ void put_mn8(uint8_t* tile, int r0, int k, uint4 v) {
  *reinterpret_cast<uint4*>(tile + ((r0 >> 3) * (BK / 8) + (k >> 3)) * 128 + (k & 7) * 16) = v;
}
// 16-byte asynchronous global -> shared copy (cached in L1); src_bytes 0 writes zeros and reads
// nothing.
__device__ __forceinline__ void cp_async_16(uint32_t dst, const void* src, uint32_t src_bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// Loaders that store MN-major tiles declare `static constexpr bool kMnMajor = true`.
template <class L, class = void>
struct MnMajor { static constexpr bool value = false; };
template <class L>
struct MnMajor<L, decltype((void)L::kMnMajor)> { static constexpr bool value = L::kMnMajor; };
// Loaders whose tiles are plain 16-byte copies also provide `fill_async`, which issues them as
// cp.async (zero-filled where the operand has no element), and declare `kAsync = true`.
template <class L, class = void>
struct AsyncFill { static constexpr bool value = false; };
template <class L>
struct AsyncFill<L, decltype((void)L::kAsync)> { static constexpr bool value = L::kAsync; };

// Fills a ROWS x BK tile from a chunk loader: `uint4 chunk(int row, int k8) const` returns
// K-elements [8*k8, 8*k8 + 8) of operand row `row` as 8 BF16 values (zero outside the matrix).
// Consecutive threads take consecutive rows of one K-chunk: conflict-free 16-byte smem stores.
template <int ROWS, class L>
__device__ __forceinline__ void fill_chunks(const L& l, uint8_t* tile, int row0, int k0, int tid) {
  const int k8 = k0 >> 3;
  for (int i = tid; i < ROWS * (BK / 8); i += THREADS) {
    int r = i % ROWS, c = i / ROWS;
    put_chunk(tile, r, c, l.chunk(row0 + r, k8 + c));
  }
}

// Loader contract: `template <int ROWS> void fill(uint8_t* tile, int row0, int k0, int tid) const`
// writes rows [row0, row0 + ROWS) x K-elements [k0, k0 + BK) of the operand into a tile (all of
// it, zeros outside the matrix); the 128 threads of the CTA call it together.
// Split K: blockIdx.z takes K-tiles [z * kt_per, (z + 1) * kt_per).
template <int BN, class LA, class LB, class EP>
__global__ void __launch_bounds__(THREADS) k_tc_gemm(LA la, LB lb, EP ep, int M, int N, int K, int kt_per,
                                                     uint32_t* err) {
  extern __shared__ __align__(1024) uint8_t smem[];
  using S = Smem<BN>;
  const int tid = threadIdx.x, warp = tid >> 5;
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + 2 * S::STAGE);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + 2 * S::STAGE + 16);
  volatile uint32_t* flag = reinterpret_cast<volatile uint32_t*>(smem + 2 * S::STAGE + 20);
  const uint32_t bar0 = smem_u32(&bars[0]), bar1 = smem_u32(&bars[1]);
  constexpr uint32_t NCOLS = tmem_cols(BN);
  if (warp == 0) tmem_alloc(smem_u32(tmem_slot), NCOLS);
  if (tid == 0) {
    mbar_init(bar0, 1);
    mbar_init(bar1, 1);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const int KT_ALL = (K + BK - 1) / BK;
  const int kt_begin = blockIdx.z * kt_per;
  const int KT = max(0, min(KT_ALL - kt_begin, kt_per));   // k-tiles of this CTA
  constexpr uint32_t IDESC = idesc_bf16(BN) | (MnMajor<LA>::value ? 1u << 15 : 0u) | (MnMajor<LB>::value ? 1u << 16 : 0u);
  bool ok = true;
  int committed = 0;   // k-tiles whose MMAs were committed
  // With asynchronous loaders the copies of k-tile kt + 1 are issued before k-tile kt's MMAs, so
  // their latency overlaps the MMAs and the next iteration; otherwise each tile is filled in turn.
  constexpr bool ASYNC = AsyncFill<LA>::value && AsyncFill<LB>::value;
  if constexpr (ASYNC) {
    if (KT > 0) {
      la.template fill_async<BM>(smem, m0, kt_begin * BK, tid);
      lb.template fill_async<BN>(smem + S::A_BYTES, n0, kt_begin * BK, tid);
      cp_async_commit();
    }
  }
  for (int kt = 0; kt < KT; ++kt) {
    const int s = kt & 1;
    uint8_t* ta = smem + s * S::STAGE;
    uint8_t* tb = ta + S::A_BYTES;
    if constexpr (ASYNC) {
      if (kt + 1 < KT) {
        if (kt >= 1) {
          // the other stage was read by k-tile kt - 1's MMAs: done before it is overwritten
          if (tid == 0) *flag = mbar_wait(s ? bar0 : bar1, (uint32_t)((kt - 1) >> 1) & 1u) ? 1u : 0u;
          __syncthreads();
          if (*flag == 0u) { ok = false; break; }
        }
        uint8_t* na = smem + (s ^ 1) * S::STAGE;
        la.template fill_async<BM>(na, m0, (kt_begin + kt + 1) * BK, tid);
        lb.template fill_async<BN>(na + S::A_BYTES, n0, (kt_begin + kt + 1) * BK, tid);
        cp_async_commit();
        cp_async_wait<1>();   // this thread's copies of k-tile kt have landed
      } else {
        cp_async_wait<0>();
      }
    } else {
      if (kt >= 2) {
        // the MMAs that read this stage two tiles ago must be done before it is overwritten; one
        // thread waits and the block follows its verdict
        if (tid == 0) *flag = mbar_wait(s ? bar1 : bar0, (uint32_t)((kt >> 1) - 1) & 1u) ? 1u : 0u;
        __syncthreads();
        if (*flag == 0u) { ok = false; break; }
      }
      const int k0 = (kt_begin + kt) * BK;
      la.template fill<BM>(ta, m0, k0, tid);
      lb.template fill<BN>(tb, n0, k0, tid);
    }
    fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      const uint32_t a_addr = smem_u32(ta), b_addr = smem_u32(tb);
#pragma unroll
      for (int kk = 0; kk < BK / 16; ++kk) {
        uint64_t da = smem_desc(a_addr + kk * 256, 128, (BK / 8) * 128);
        uint64_t db = smem_desc(b_addr + kk * 256, 128, (BK / 8) * 128);
        mma_bf16(tmem, da, db, IDESC, (kt > 0 || kk > 0) ? 1u : 0u);
      }
      mma_commit(s ? bar1 : bar0);
    }
    committed = kt + 1;
  }
  if constexpr (ASYNC) cp_async_wait<0>();   // no copy outlives the loop (also after an abort)
  // all MMAs done: the last commit covers every earlier tcgen05 operation of the issuing thread
  // (after an expired wait this still waits, bounded, for the MMAs in flight before freeing)
  if (tid == 0) {
    const int last = committed - 1;
    *flag = committed == 0 || mbar_wait((last & 1) ? bar1 : bar0, (uint32_t)(last >> 1) & 1u) ? 1u : 0u;
  }
  __syncthreads();
  ok = ok && *flag != 0u;
  if (!ok) {
    if (tid == 0) atomicOr(err, ERR_TC_TIMEOUT);
  } else if (KT > 0) {
    tc_fence_after();
    const int row = m0 + warp * 32 + (tid & 31);
    for (int c0 = 0; c0 < BN; c0 += 16) {
      float v[16];
      tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
      if (row < M && n0 + c0 < N) ep(row, n0 + c0, v);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_free(tmem, NCOLS);
}

}  // namespace tc
