// gs_geom.cuh -- per-splat geometry shared by the project and chain kernels:
// computeGeom (shaders.js:164-225) and the real SH basis with its gradient
// (shaders.js:56-138).  Operation order follows the WGSL expressions left to
// right, unfused (the library is built with -fmad=false).
#pragma once
#include "gs_common.cuh"

namespace gs {

struct Geom {
  bool ok;
  float pc[3], q[4], r0[3], r1[3], r2[3], s[3], t0[3], t1[3];
  float va, vb, vc, s00, s01, s02, s11, s12, s22;
};

__device__ __forceinline__ float dot3(const float a[3], const float b[3]) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

// P: the 16 parameters of one splat (pos, logScale, quat w,x,y,z, logits, opacity)
__device__ __forceinline__ Geom computeGeom(const DevCam& c, const float* P) {
  Geom g;
  g.ok = false;
  const float p[3] = {P[0], P[1], P[2]};
  const float R0[3] = {c.R[0], c.R[1], c.R[2]};
  const float R1[3] = {c.R[3], c.R[4], c.R[5]};
  const float R2[3] = {c.R[6], c.R[7], c.R[8]};
  g.pc[0] = dot3(R0, p) + c.t[0];
  g.pc[1] = dot3(R1, p) + c.t[1];
  g.pc[2] = dot3(R2, p) + c.t[2];
  if (g.pc[2] < c.nearz) return g;

  float q[4] = {P[6], P[7], P[8], P[9]};
  const float ql = sqrtf(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
  if (ql < 1e-6f) { q[0] = 1.0f; q[1] = q[2] = q[3] = 0.0f; }
  else {
#pragma unroll
    for (int k = 0; k < 4; ++k) q[k] = q[k] / ql;
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) g.q[k] = q[k];
  const float qw = q[0], qx = q[1], qy = q[2], qz = q[3];
  g.r0[0] = 1.0f - 2.0f * (qy * qy + qz * qz);
  g.r0[1] = 2.0f * (qx * qy - qw * qz);
  g.r0[2] = 2.0f * (qx * qz + qw * qy);
  g.r1[0] = 2.0f * (qx * qy + qw * qz);
  g.r1[1] = 1.0f - 2.0f * (qx * qx + qz * qz);
  g.r1[2] = 2.0f * (qy * qz - qw * qx);
  g.r2[0] = 2.0f * (qx * qz - qw * qy);
  g.r2[1] = 2.0f * (qy * qz + qw * qx);
  g.r2[2] = 1.0f - 2.0f * (qx * qx + qy * qy);
#pragma unroll
  for (int k = 0; k < 3; ++k) g.s[k] = gexp(clampf(P[3 + k], -12.0f, 6.0f));

  float m0[3], m1[3], m2[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    m0[k] = g.r0[k] * g.s[k];
    m1[k] = g.r1[k] * g.s[k];
    m2[k] = g.r2[k] * g.s[k];
  }
  g.s00 = dot3(m0, m0); g.s01 = dot3(m0, m1); g.s02 = dot3(m0, m2);
  g.s11 = dot3(m1, m1); g.s12 = dot3(m1, m2); g.s22 = dot3(m2, m2);

  const float f = c.f;
  const float iz = 1.0f / g.pc[2];
  const float a0 = f * iz;
  const float b0 = (-f) * g.pc[0] * iz * iz;
  const float b1 = (-f) * g.pc[1] * iz * iz;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    g.t0[k] = a0 * R0[k] + b0 * R2[k];
    g.t1[k] = a0 * R1[k] + b1 * R2[k];
  }
  const float st0[3] = {g.s00 * g.t0[0] + g.s01 * g.t0[1] + g.s02 * g.t0[2],
                        g.s01 * g.t0[0] + g.s11 * g.t0[1] + g.s12 * g.t0[2],
                        g.s02 * g.t0[0] + g.s12 * g.t0[1] + g.s22 * g.t0[2]};
  const float st1[3] = {g.s00 * g.t1[0] + g.s01 * g.t1[1] + g.s02 * g.t1[2],
                        g.s01 * g.t1[0] + g.s11 * g.t1[1] + g.s12 * g.t1[2],
                        g.s02 * g.t1[0] + g.s12 * g.t1[1] + g.s22 * g.t1[2]};
  g.va = fmaxf(dot3(g.t0, st0), 0.0f);
  g.vb = dot3(g.t1, st0);
  g.vc = fmaxf(dot3(g.t1, st1), 0.0f);
  g.ok = true;
  return g;
}

// camPosWorld = -R^T t (shaders.js:121-126)
__device__ __forceinline__ void camPosWorld(const DevCam& c, float out[3]) {
#pragma unroll
  for (int j = 0; j < 3; ++j) out[j] = -(c.R[j] * c.t[0] + c.R[3 + j] * c.t[1] + c.R[6 + j] * c.t[2]);
}

// INRIA real SH constants (shaders.js:60-64)
#define GS_C1 0.4886025119029199f
#define GS_C2_0 1.0925484305920792f
#define GS_C2_1 -1.0925484305920792f
#define GS_C2_2 0.31539156525252005f
#define GS_C2_3 -1.0925484305920792f
#define GS_C2_4 0.5462742152960396f
#define GS_C3_0 -0.5900435899266435f
#define GS_C3_1 2.890611442640554f
#define GS_C3_2 -0.4570457994644658f
#define GS_C3_3 0.3731763325901154f
#define GS_C3_4 -0.4570457994644658f
#define GS_C3_5 1.445305721320277f
#define GS_C3_6 -0.5900435899266435f

template <int DEG>
__device__ __forceinline__ void shBasis(const float v[3], float Y[15]) {
  const float x = v[0], y = v[1], z = v[2];
  Y[0] = (-GS_C1) * y;
  Y[1] = GS_C1 * z;
  Y[2] = (-GS_C1) * x;
  if (DEG >= 2) {
    const float xx = x * x, yy = y * y, zz = z * z;
    Y[3] = GS_C2_0 * x * y;
    Y[4] = GS_C2_1 * y * z;
    Y[5] = GS_C2_2 * (2.0f * zz - xx - yy);
    Y[6] = GS_C2_3 * x * z;
    Y[7] = GS_C2_4 * (xx - yy);
    if (DEG >= 3) {
      Y[8] = GS_C3_0 * y * (3.0f * xx - yy);
      Y[9] = GS_C3_1 * x * y * z;
      Y[10] = GS_C3_2 * y * (4.0f * zz - xx - yy);
      Y[11] = GS_C3_3 * z * (2.0f * zz - 3.0f * xx - 3.0f * yy);
      Y[12] = GS_C3_4 * x * (4.0f * zz - xx - yy);
      Y[13] = GS_C3_5 * z * (xx - yy);
      Y[14] = GS_C3_6 * x * (xx - yy);
    }
  }
}

template <int DEG>
__device__ __forceinline__ void shBasisGrad(const float v[3], float D[15][3]) {
  const float x = v[0], y = v[1], z = v[2];
#define GS_SET(k, C, a, b, d) { D[k][0] = (C) * (a); D[k][1] = (C) * (b); D[k][2] = (C) * (d); }
  D[0][0] = 0.0f; D[0][1] = -GS_C1; D[0][2] = 0.0f;
  D[1][0] = 0.0f; D[1][1] = 0.0f; D[1][2] = GS_C1;
  D[2][0] = -GS_C1; D[2][1] = 0.0f; D[2][2] = 0.0f;
  if (DEG >= 2) {
    const float xx = x * x, yy = y * y, zz = z * z;
    GS_SET(3, GS_C2_0, y, x, 0.0f);
    GS_SET(4, GS_C2_1, 0.0f, z, y);
    GS_SET(5, GS_C2_2, -2.0f * x, -2.0f * y, 4.0f * z);
    GS_SET(6, GS_C2_3, z, 0.0f, x);
    GS_SET(7, GS_C2_4, 2.0f * x, -2.0f * y, 0.0f);
    if (DEG >= 3) {
      GS_SET(8, GS_C3_0, 6.0f * x * y, 3.0f * xx - 3.0f * yy, 0.0f);
      GS_SET(9, GS_C3_1, y * z, x * z, x * y);
      GS_SET(10, GS_C3_2, -2.0f * x * y, 4.0f * zz - xx - 3.0f * yy, 8.0f * y * z);
      GS_SET(11, GS_C3_3, -6.0f * x * z, -6.0f * y * z, 6.0f * zz - 3.0f * xx - 3.0f * yy);
      GS_SET(12, GS_C3_4, 4.0f * zz - 3.0f * xx - yy, -2.0f * x * y, 8.0f * x * z);
      GS_SET(13, GS_C3_5, 2.0f * x * z, -2.0f * y * z, xx - yy);
      GS_SET(14, GS_C3_6, 3.0f * xx - yy, -2.0f * x * y, 0.0f);
    }
  }
#undef GS_SET
}

// dY_k/dv for one coefficient k (the same expressions as shBasisGrad), so a
// loop over k need not hold the whole gradient table in registers.
template <int DEG>
__device__ __forceinline__ void shBasisGradK(int k, const float v[3], float d[3]) {
  const float x = v[0], y = v[1], z = v[2];
  const float xx = x * x, yy = y * y, zz = z * z;
  float C = 0.0f, a0 = 0.0f, a1 = 0.0f, a2 = 0.0f;
  switch (k) {
    case 0: d[0] = 0.0f; d[1] = -GS_C1; d[2] = 0.0f; return;
    case 1: d[0] = 0.0f; d[1] = 0.0f; d[2] = GS_C1; return;
    case 2: d[0] = -GS_C1; d[1] = 0.0f; d[2] = 0.0f; return;
    case 3: C = GS_C2_0; a0 = y; a1 = x; a2 = 0.0f; break;
    case 4: C = GS_C2_1; a0 = 0.0f; a1 = z; a2 = y; break;
    case 5: C = GS_C2_2; a0 = -2.0f * x; a1 = -2.0f * y; a2 = 4.0f * z; break;
    case 6: C = GS_C2_3; a0 = z; a1 = 0.0f; a2 = x; break;
    case 7: C = GS_C2_4; a0 = 2.0f * x; a1 = -2.0f * y; a2 = 0.0f; break;
    case 8: C = GS_C3_0; a0 = 6.0f * x * y; a1 = 3.0f * xx - 3.0f * yy; a2 = 0.0f; break;
    case 9: C = GS_C3_1; a0 = y * z; a1 = x * z; a2 = x * y; break;
    case 10: C = GS_C3_2; a0 = -2.0f * x * y; a1 = 4.0f * zz - xx - 3.0f * yy; a2 = 8.0f * y * z; break;
    case 11: C = GS_C3_3; a0 = -6.0f * x * z; a1 = -6.0f * y * z; a2 = 6.0f * zz - 3.0f * xx - 3.0f * yy; break;
    case 12: C = GS_C3_4; a0 = 4.0f * zz - 3.0f * xx - yy; a1 = -2.0f * x * y; a2 = 8.0f * x * z; break;
    case 13: C = GS_C3_5; a0 = 2.0f * x * z; a1 = -2.0f * y * z; a2 = xx - yy; break;
    default: C = GS_C3_6; a0 = 3.0f * xx - yy; a1 = -2.0f * x * y; a2 = 0.0f; break;
  }
  d[0] = C * a0; d[1] = C * a1; d[2] = C * a2;
}

}  // namespace gs
