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
constexpr int PLY_THREADS = 128;
constexpr int PLY_MAX_STRIDE = 17 + 3 * MAX_K;  // floats per record at SH degree 3

// One record: x y z nx ny nz f_dc[3] f_rest[3K] opacity scale[3] rot[4].
// Each thread computes its splat's record into the block's shared-memory
// rows; the block then writes its records as one contiguous run, so the
// stores are coalesced (a record is 17 + 3K floats, not a power of two).
__global__ void __launch_bounds__(PLY_THREADS) k_ply_records(const float* __restrict__ params,
                                                             const float* __restrict__ sh, uint32_t n, uint32_t K,
                                                             int bake, double f,
                                                             const double* __restrict__ camPos, uint32_t ncams,
                                                             float* __restrict__ out) {
  __shared__ double s_cam[CAM_TILE * 3];
  __shared__ float s_rec[PLY_THREADS * PLY_MAX_STRIDE];
  const uint32_t i0 = blockIdx.x * PLY_THREADS;
  const uint32_t i = i0 + threadIdx.x;
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
  const uint32_t stride = 17 + 3 * K;
  if (valid) {
    float* o = s_rec + (size_t)threadIdx.x * stride;
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
  __syncthreads();
  const uint32_t cnt = n - i0 < (uint32_t)PLY_THREADS ? n - i0 : (uint32_t)PLY_THREADS;
  float* dst = out + (size_t)i0 * stride;
  for (uint32_t e = threadIdx.x; e < cnt * stride; e += PLY_THREADS) dst[e] = s_rec[e];
}
}  // namespace

// Records of n splats into outHost (host memory, any alignment); dCam and
// dOut are device scratch of ncams * 3 doubles and n * (17 + 3K) floats.
int export_ply_records(const float* params, const float* sh, uint32_t n, uint32_t K, int bake, double f,
                       const double* camPosHost, uint32_t ncams, double* dCam, float* dOut, void* outHost,
                       cudaStream_t s) {
  if (K > (uint32_t)MAX_K) return -1;
  const size_t outBytes = (size_t)n * (17 + 3 * K) * 4;
  if (bake && ncams &&
      cudaMemcpyAsync(dCam, camPosHost, (size_t)ncams * 3 * 8, cudaMemcpyHostToDevice, s) != cudaSuccess)
    return -2;
  if (n) {
    k_ply_records<<<(n + PLY_THREADS - 1) / PLY_THREADS, PLY_THREADS, 0, s>>>(params, sh, n, K, bake ? 1 : 0, f,
                                                                              dCam, ncams, dOut);
    if (cudaGetLastError() != cudaSuccess) return -2;
    if (cudaMemcpyAsync(outHost, dOut, outBytes, cudaMemcpyDeviceToHost, s) != cudaSuccess) return -2;
  }
  if (cudaStreamSynchronize(s) != cudaSuccess) return -2;
  return 0;
}
}  // namespace gs
