// gs_export.cu -- PLY export of the trained Gaussians on the device: the
// opacity-compensation bake (ply.js:17-39, bakeOpacityCompensation) and the
// INRIA-layout record packing (ply.js:45-99, gaussiansToPly).
//
// The reference runs both as JavaScript loops in double precision (O(n x
// cameras) for the bake) and stores float32.  Here one thread per splat does
// the same double-precision arithmetic (the cameras staged in shared memory
// 256 at a time) and writes its record; the host adds the text header.
// Results round to float32 as Float32Array/DataView stores do; JavaScript's
// exp/log/hypot and CUDA's agree to a double ulp, so stored values agree to
// at most one float32 ulp (nearly always exactly).
#include <cuda_runtime.h>

#include "gs_common.cuh"

namespace gs {
namespace {

constexpr double PLY_SH_C0 = 0.28209479177387814;  // ply.js:9
constexpr int CAM_TILE = 256;

// One record: x y z nx ny nz f_dc[3] f_rest[3K] opacity scale[3] rot[4]
__global__ void __launch_bounds__(256) k_ply_records(const float* __restrict__ params, const float* __restrict__ sh,
                                                     uint32_t n, uint32_t K, int bake, double f,
                                                     const double* __restrict__ camPos, uint32_t ncams,
                                                     float* __restrict__ out) {
  __shared__ double s_cam[CAM_TILE * 3];
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = i < n;
  const float* P = params + (size_t)(valid ? i : 0) * STRIDE;
  const double px = P[0], py = P[1], pz = P[2];
  double z2min = __longlong_as_double(0x7FF0000000000000ll);  // +inf (no camera: z = inf, as in JS)
  if (bake) {
    for (uint32_t c0 = 0; c0 < ncams; c0 += CAM_TILE) {
      const uint32_t cn = ncams - c0 < (uint32_t)CAM_TILE ? ncams - c0 : (uint32_t)CAM_TILE;
      __syncthreads();
      for (uint32_t k = threadIdx.x; k < cn * 3; k += blockDim.x) s_cam[k] = camPos[(size_t)c0 * 3 + k];
      __syncthreads();
      for (uint32_t c = 0; c < cn; ++c) {
        const double dx = px - s_cam[c * 3], dy = py - s_cam[c * 3 + 1], dz = pz - s_cam[c * 3 + 2];
        const double d2 = dx * dx + dy * dy + dz * dz;
        if (d2 < z2min) z2min = d2;
      }
    }
  }
  if (!valid) return;
  const uint32_t stride = 17 + 3 * K;
  float* o = out + (size_t)i * stride;
  o[0] = P[0]; o[1] = P[1]; o[2] = P[2];
  o[3] = 0.0f; o[4] = 0.0f; o[5] = 0.0f;
  for (int c = 0; c < 3; ++c) {
    const double sg = 1.0 / (1.0 + exp(-(double)P[10 + c]));
    o[6 + c] = (float)((sg - 0.5) / PLY_SH_C0);
  }
  for (uint32_t k = 0; k < 3 * K; ++k) o[9 + k] = sh[(size_t)i * 3 * K + k];
  float* q = o + 9 + 3 * K;
  float logit = P[13];
  if (bake) {
    const double z = fmax(1e-3, sqrt(z2min));
    const double sMean = exp(((double)P[3] + (double)P[4] + (double)P[5]) / 3.0);
    const double s2d = f * sMean / z;
    const double comp = (s2d * s2d) / (s2d * s2d + 0.3);
    const double opa = comp / (1.0 + exp(-(double)P[13]));
    const double cl = fmin(1.0 - 1e-6, fmax(1e-6, opa));
    logit = (float)log(cl / (1.0 - cl));
  }
  q[0] = logit;
  q[1] = P[3]; q[2] = P[4]; q[3] = P[5];
  double qw = P[6], qx = P[7], qy = P[8], qz = P[9];
  const double ql = sqrt(qw * qw + qx * qx + qy * qy + qz * qz);
  if (ql < 1e-6) { qw = 1.0; qx = qy = qz = 0.0; }
  else { qw /= ql; qx /= ql; qy /= ql; qz /= ql; }
  q[4] = (float)qw; q[5] = (float)qx; q[6] = (float)qy; q[7] = (float)qz;
}

}  // namespace

int export_ply_records(const float* params, const float* sh, uint32_t n, uint32_t K, int bake, double f,
                       const double* camPosHost, uint32_t ncams, float* outHost, cudaStream_t s) {
  double* dCam = nullptr;
  float* dOut = nullptr;
  const size_t outBytes = (size_t)n * (17 + 3 * K) * 4;
  int rc = 0;
  if (bake && ncams && cudaMalloc(&dCam, (size_t)ncams * 3 * 8) != cudaSuccess) rc = -3;
  if (!rc && cudaMalloc(&dOut, outBytes > 0 ? outBytes : 4) != cudaSuccess) rc = -3;
  if (!rc && bake && ncams &&
      cudaMemcpyAsync(dCam, camPosHost, (size_t)ncams * 3 * 8, cudaMemcpyHostToDevice, s) != cudaSuccess)
    rc = -2;
  if (!rc && n) {
    k_ply_records<<<(n + 255) / 256, 256, 0, s>>>(params, sh, n, K, bake ? 1 : 0, f, dCam, ncams, dOut);
    if (cudaGetLastError() != cudaSuccess) rc = -2;
  }
  if (!rc && n && cudaMemcpyAsync(outHost, dOut, outBytes, cudaMemcpyDeviceToHost, s) != cudaSuccess) rc = -2;
  if (!rc && cudaStreamSynchronize(s) != cudaSuccess) rc = -2;
  cudaFree(dCam);
  cudaFree(dOut);
  return rc;
}

}  // namespace gs
