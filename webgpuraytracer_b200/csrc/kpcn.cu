// Learned kernel-predicting denoiser: BF16 tensor-core GEMM entry point (this file grows into
// the network's forward/backward kernels).
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>
#include <string.h>

#include "../../include/wgpt.h"
#include "tc_gemm.cuh"

namespace kp {

// Row-major BF16 matrix (K contiguous), zero outside rows x k.
struct RowMajor {
  const uint16_t* p;
  int rows, k, ld;
  __device__ __forceinline__ uint4 chunk(int row, int k8) const {
    if (row >= rows || k8 * 8 >= k) return make_uint4(0u, 0u, 0u, 0u);
    return *reinterpret_cast<const uint4*>(p + (size_t)row * ld + k8 * 8);
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
  dim3 grid((unsigned)((M + tc::BM - 1) / tc::BM), (unsigned)((N + BN - 1) / BN));
  kern<<<grid, tc::THREADS, smem, st>>>(la, lb, ep, M, N, K, err);
  return cudaGetLastError();
}

}  // namespace kp

extern "C" int wgpt_gemm_bf16(int device, const uint16_t* a, const uint16_t* b, float* c, int m, int n, int k) {
  if (!a || !b || !c || m <= 0 || n <= 0 || k <= 0 || (k % 8) != 0) return WGPT_E_INVALID;
  if (cudaSetDevice(device) != cudaSuccess) return WGPT_E_CUDA;
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
