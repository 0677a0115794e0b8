// L2 read-bandwidth probe: the denominator for reporting the traversal kernels against the
// on-chip bandwidth they actually draw on (their scene data is L2-resident), beside the HBM
// roofline.  Measurement support; the reference has no counterpart.
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/wgpt.h"

namespace {

// Streams the buffer `reps` times with L2-only loads (ld.global.cg: not cached in L1), so every
// load is served by L2 once the first pass has brought the buffer in.
__global__ void __launch_bounds__(512) k_l2_read(const float4* __restrict__ buf, size_t n4, uint32_t reps,
                                                 float* sink) {
  float acc = 0.0f;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (uint32_t r = 0; r < reps; ++r)
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += stride) {
      const float4 v = __ldcg(buf + i);
      acc += (v.x + v.y) + (v.z + v.w);
    }
  if (acc == 1234.5f) sink[0] = acc;   // keeps the loads live; the buffer is zero-filled
}

}  // namespace

extern "C" int wgpt_probe_l2_read(int device, uint64_t bytes, uint32_t reps, double* gbps) {
  if (!gbps || bytes < (1ull << 20) || bytes > (96ull << 20) || bytes % 16 != 0 || reps == 0 || reps > 1000)
    return WGPT_E_INVALID;
  if (cudaSetDevice(device) != cudaSuccess) return WGPT_E_CUDA;
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return WGPT_E_CUDA;
  float4* buf = nullptr;
  float* sink = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = WGPT_OK;
  float ms = 0.0f;
  const size_t n4 = bytes / 16;
  if (cudaMalloc(&buf, bytes) != cudaSuccess || cudaMalloc(&sink, sizeof(float)) != cudaSuccess) {
    rc = WGPT_E_NOMEM;
    goto done;
  }
  if (cudaMemset(buf, 0, bytes) != cudaSuccess || cudaEventCreate(&e0) != cudaSuccess ||
      cudaEventCreate(&e1) != cudaSuccess) {
    rc = WGPT_E_CUDA;
    goto done;
  }
  k_l2_read<<<sms * 4, 512>>>(buf, n4, 1u, sink);   // brings the buffer into L2
  cudaEventRecord(e0);
  k_l2_read<<<sms * 4, 512>>>(buf, n4, reps, sink);
  cudaEventRecord(e1);
  if (cudaEventSynchronize(e1) != cudaSuccess || cudaGetLastError() != cudaSuccess ||
      cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess || !(ms > 0.0f)) {
    rc = WGPT_E_CUDA;
    goto done;
  }
  *gbps = (double)bytes * reps / ((double)ms * 1e-3) / 1e9;
done:
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (buf) cudaFree(buf);
  if (sink) cudaFree(sink);
  return rc;
}
