// gs_probe.cu -- FP32 FMA throughput probe: the denominator of the raster
// kernels' roofline (the rasteriser is FP32-pipe bound; no tensor-core work
// exists on this path).  Every thread runs 8 independent FFMA chains so the
// pipe, not latency, limits the rate; the result is returned so the chains
// cannot be optimised away.
#include <cuda_runtime.h>

#include "../../include/splat_b200.h"
#include "gs_common.cuh"

namespace {

constexpr int CHAINS = 8;
constexpr int ITERS = 4096;

__global__ void __launch_bounds__(256) k_ffma(float* out, float a, float b) {
  float x[CHAINS];
#pragma unroll
  for (int k = 0; k < CHAINS; ++k) x[k] = (float)(threadIdx.x + k) * 1e-3f;
  for (int i = 0; i < ITERS; ++i) {
#pragma unroll
    for (int k = 0; k < CHAINS; ++k) x[k] = __fmaf_rn(x[k], a, b);
  }
  float s = 0.0f;
#pragma unroll
  for (int k = 0; k < CHAINS; ++k) s += x[k];
  if (s == 12345.678f) out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// every float in [lo, hi] (bit patterns): rcp_unit(x) against IEEE 1/x
__global__ void k_check_rcp(uint32_t lo, uint32_t hi, unsigned long long* bad, uint32_t* first) {
  for (uint32_t b = lo + blockIdx.x * blockDim.x + threadIdx.x; b <= hi; b += gridDim.x * blockDim.x) {
    const float x = __uint_as_float(b);
    if (__float_as_uint(gs::rcp_unit(x)) != __float_as_uint(__frcp_rn(x))) {
      atomicAdd(bad, 1ull);
      atomicMin(first, b);
    }
  }
}

}  // namespace

extern "C" GS_API int gs_debug_check_rcp(int32_t device, uint64_t* mismatches, uint32_t* firstBits) {
  if (!mismatches || !firstBits) return GS_E_INVALID;
  if (cudaSetDevice(device) != cudaSuccess) return GS_E_CUDA;
  unsigned long long* bad = nullptr;
  uint32_t* first = nullptr;
  if (cudaMalloc(&bad, 8) != cudaSuccess || cudaMalloc(&first, 4) != cudaSuccess) {
    cudaFree(bad);
    return GS_E_NOMEM;
  }
  cudaMemset(bad, 0, 8);
  cudaMemset(first, 0xFF, 4);
  k_check_rcp<<<1184, 256>>>(0x3C000000u, 0x3F800000u, bad, first);  // [2^-7, 1]
  unsigned long long nb = 0;
  uint32_t fb = 0;
  const bool ok = cudaMemcpy(&nb, bad, 8, cudaMemcpyDeviceToHost) == cudaSuccess &&
                  cudaMemcpy(&fb, first, 4, cudaMemcpyDeviceToHost) == cudaSuccess;
  cudaFree(bad);
  cudaFree(first);
  if (!ok) return GS_E_CUDA;
  *mismatches = nb;
  *firstBits = fb;
  return GS_OK;
}

extern "C" GS_API int gs_probe_fp32_peak(int32_t device, double* tflops) {
  if (!tflops) return GS_E_INVALID;
  if (cudaSetDevice(device) != cudaSuccess) return GS_E_CUDA;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const int blocks = sms * 8;
  float* out = nullptr;
  if (cudaMalloc(&out, (size_t)blocks * 256 * 4) != cudaSuccess) return GS_E_NOMEM;
  cudaStream_t s;
  cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  for (int w = 0; w < 3; ++w) k_ffma<<<blocks, 256, 0, s>>>(out, 0.999f, 1e-4f);
  const int reps = 20;
  cudaEventRecord(e0, s);
  for (int r = 0; r < reps; ++r) k_ffma<<<blocks, 256, 0, s>>>(out, 0.999f, 1e-4f);
  cudaEventRecord(e1, s);
  cudaError_t err = cudaEventSynchronize(e1);
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaStreamDestroy(s);
  cudaFree(out);
  if (err != cudaSuccess || ms <= 0.0f) return GS_E_CUDA;
  const double flops = 2.0 * CHAINS * ITERS * (double)blocks * 256.0 * reps;
  *tflops = flops / (ms * 1e-3) / 1e12;
  return GS_OK;
}
