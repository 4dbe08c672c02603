// Integer-ALU throughput probe: the roofline denominator for the search
// kernel, whose work is 32-bit integer add/sub/abs/compare (there is no
// tensor-core or floating-point content on this path). Every thread runs
// eight independent chains of dependent 32-bit adds, enough warps per SM to
// hide the pipeline latency; ops/s = threads * chains * iterations * 2 / t
// (each step is an add and an xor, both issued to the integer pipe).
#include <cuda_runtime.h>

#include "rme_internal.h"

namespace rme {
namespace {
__global__ void __launch_bounds__(512) int_probe_kernel(uint32_t seed, int iters, uint32_t* sink) {
  uint32_t a[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) a[k] = seed + threadIdx.x * 8 + k;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = (a[k] + 0x9E3779B9u) ^ (a[k] >> 3);
  }
  uint32_t x = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) x ^= a[k];
  if (x == 0x12345678u) sink[0] = x;  // keeps the chains live
}
}  // namespace
}  // namespace rme

extern "C" int rme_probe_int_peak(int32_t device, double* ops_per_s) {
  if (!ops_per_s) return RME_EINVAL;
  if (cudaSetDevice(device) != cudaSuccess) return RME_ECUDA;
  int nsm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
  uint32_t* sink = nullptr;
  if (cudaMalloc(&sink, 16) != cudaSuccess) return RME_ECUDA;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int threads = 512, blocks = nsm * 4, iters = 1 << 16;
  rme::int_probe_kernel<<<blocks, threads>>>(1u, 256, sink);  // warm-up
  cudaEventRecord(e0);
  rme::int_probe_kernel<<<blocks, threads>>>(2u, iters, sink);
  cudaEventRecord(e1);
  cudaError_t err = cudaEventSynchronize(e1);
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(sink);
  if (err != cudaSuccess || ms <= 0.0f) return RME_ECUDA;
  // per chain step: one add, one shift, one xor (three integer ops)
  *ops_per_s = (double)blocks * threads * 8.0 * iters * 3.0 / (ms * 1e-3);
  return 0;
}

// The failure path of the library's bounded waits, taken on purpose: a wait
// on a flag that nothing sets gives up after `polls` polls and reports it in
// the status word, and the device stays usable.
extern "C" int rme_probe_wait_timeout(int32_t device, uint32_t polls, uint32_t* status, double* seconds) {
  if (!status || polls == 0 || polls > (1u << 22)) return RME_EINVAL;
  if (cudaSetDevice(device) != cudaSuccess) return RME_ECUDA;
  int32_t* flag = nullptr;
  uint32_t* st = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = RME_ECUDA;
  if (cudaMalloc(&flag, 64) == cudaSuccess && cudaMemset(flag, 0, 64) == cudaSuccess) {
    st = reinterpret_cast<uint32_t*>(flag + 8);
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0);
    if (rme::launch_probe_wait(flag, polls, st, nullptr) == cudaSuccess && cudaEventRecord(e1) == cudaSuccess &&
        cudaMemcpy(status, st, sizeof(uint32_t), cudaMemcpyDeviceToHost) == cudaSuccess) {
      float ms = 0.0f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (seconds) *seconds = ms * 1e-3;
      rc = RME_OK;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  }
  if (flag) cudaFree(flag);
  return rc;
}
