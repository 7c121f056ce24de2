// gs_ingest.cu -- target ingestion on the device: the radial undistortion of
// the training frames (session.js:44-80, undistortFrames) and the RGBA8
// packing of GSTrainer.setup (trainer.js:115-139).
//
// The reference runs both as JavaScript loops over every pixel, in double
// precision for the resample (JavaScript numbers) with float32 stores.  Here
// one thread per pixel performs the same double-precision operations in the
// same order (no contraction: the library is built with -fmad=false, and
// IEEE division), so every resampled value is bit-identical to the
// JavaScript's; the packing is integer work on the float inputs.
#include <cmath>
#include <cuda_runtime.h>

#include "../../include/splat_b200.h"
#include "gs_common.cuh"
#include "gs_kernels.h"

namespace gs {
namespace {

// dst = undistorted copy of src (3 floats per pixel); pixels whose source
// falls outside the frame get the -1 sentinel in all three channels.
__global__ void __launch_bounds__(256) k_undistort(const float* __restrict__ src, float* __restrict__ dst,
                                                   uint32_t tw, uint32_t th, double f, double cx, double cy,
                                                   double k1, double k2) {
  const uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= (uint64_t)tw * th) return;
  const uint32_t y = (uint32_t)(p / tw), x = (uint32_t)(p - (uint64_t)y * tw);
  const double xp = ((double)x + 0.5 - cx) / f, yp = ((double)y + 0.5 - cy) / f;
  const double r2 = xp * xp + yp * yp;
  const double D = 1.0 + k1 * r2 + k2 * r2 * r2;
  const double rx = f * xp * D + cx - 0.5;
  const double ry = f * yp * D + cy - 0.5;
  float* o = dst + p * 3;
  if (rx < 0.0 || ry < 0.0 || rx > (double)tw - 1.001 || ry > (double)th - 1.001) {
    o[0] = -1.0f; o[1] = -1.0f; o[2] = -1.0f;
    return;
  }
  if (rx != rx || ry != ry) {  // NaN passes every test above; every weight is NaN then
    o[0] = o[1] = o[2] = __int_as_float(0x7FC00000);
    return;
  }
  // rx | 0 (ToInt32: truncation, rx in [0, tw - 1.001] here)
  const uint32_t x0 = (uint32_t)(int32_t)rx, y0 = (uint32_t)(int32_t)ry;
  const double fx = rx - (double)x0, fy = ry - (double)y0;
  const uint64_t i00 = ((uint64_t)y0 * tw + x0) * 3, i01 = i00 + 3;
  const uint64_t i10 = i00 + (uint64_t)tw * 3, i11 = i10 + 3;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const double v = (double)src[i00 + c] * (1.0 - fx) * (1.0 - fy) + (double)src[i01 + c] * fx * (1.0 - fy) +
                     (double)src[i10 + c] * (1.0 - fx) * fy + (double)src[i11 + c] * fx * fy;
    o[c] = __double2float_rn(v);
  }
}

// min(255, round(v * 255)) of one channel, the low byte kept
__device__ __forceinline__ uint32_t r255(float v) {
  double x = floor((double)v * 255.0 + 0.5);
  if (x > 255.0) x = 255.0;
  return (uint32_t)(int64_t)x & 0xFFu;
}

// RGBA8 of every pixel: alpha 255, or 0 (the whole word) where red < 0
__global__ void __launch_bounds__(256) k_pack_targets(const float* __restrict__ rgb, uint64_t np,
                                                      uint32_t* __restrict__ out) {
  const uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= np) return;
  const float r = rgb[p * 3];
  out[p] = r < 0.0f ? 0u : (255u << 24) | (r255(rgb[p * 3 + 2]) << 16) | (r255(rgb[p * 3 + 1]) << 8) | r255(r);
}

}  // namespace

int pack_targets_device(const float* rgbHost, uint64_t np, float* scratch, uint32_t* out, cudaStream_t s) {
  if (np == 0) return 0;
  if (cudaMemcpyAsync(scratch, rgbHost, np * 12, cudaMemcpyHostToDevice, s) != cudaSuccess) return -2;
  k_pack_targets<<<(unsigned)((np + 255) / 256), 256, 0, s>>>(scratch, np, out);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

}  // namespace gs

using namespace gs;

extern "C" int gs_undistort_frames(int32_t device, gs_frame* frames, uint32_t nframes, double k1, double k2,
                                   double fFeat, int32_t* resampled) {
  if (resampled) *resampled = 0;
  if (nframes && !frames) return GS_E_INVALID;
  // below ~0.01 the estimated distortion is noise: nothing is resampled
  if (std::fabs(k1) < 0.01 && std::fabs(k2) < 0.01) return GS_OK;
  uint64_t maxNp = 0;
  for (uint32_t i = 0; i < nframes; ++i) {
    if (!frames[i].rgb && frames[i].tw && frames[i].th) return GS_E_INVALID;
    const uint64_t np = (uint64_t)frames[i].tw * frames[i].th;
    if (np > maxNp) maxNp = np;
  }
  if (cudaSetDevice(device) != cudaSuccess) return GS_E_CUDA;
  float *dSrc = nullptr, *dDst = nullptr;
  cudaStream_t s = nullptr;
  int rc = GS_OK;
  if (maxNp && (cudaMalloc(&dSrc, maxNp * 12) != cudaSuccess || cudaMalloc(&dDst, maxNp * 12) != cudaSuccess))
    rc = GS_E_NOMEM;
  if (rc == GS_OK && cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) rc = GS_E_CUDA;
  for (uint32_t i = 0; i < nframes && rc == GS_OK; ++i) {
    const gs_frame& im = frames[i];
    const uint64_t np = (uint64_t)im.tw * im.th;
    if (np == 0) continue;
    const double f = fFeat * ((double)im.tw / im.fw);
    const double cx = (double)im.tw / 2.0, cy = (double)im.th / 2.0;
    if (cudaMemcpyAsync(dSrc, im.rgb, np * 12, cudaMemcpyHostToDevice, s) != cudaSuccess) { rc = GS_E_CUDA; break; }
    k_undistort<<<(unsigned)((np + 255) / 256), 256, 0, s>>>(dSrc, dDst, im.tw, im.th, f, cx, cy, k1, k2);
    if (cudaGetLastError() != cudaSuccess) { rc = GS_E_CUDA; break; }
    if (cudaMemcpyAsync(im.rgb, dDst, np * 12, cudaMemcpyDeviceToHost, s) != cudaSuccess) { rc = GS_E_CUDA; break; }
    if (cudaStreamSynchronize(s) != cudaSuccess) { rc = GS_E_CUDA; break; }
  }
  if (s) cudaStreamDestroy(s);
  cudaFree(dSrc);
  cudaFree(dDst);
  if (rc == GS_OK && resampled) *resampled = 1;
  return rc;
}
