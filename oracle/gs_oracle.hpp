// gs_oracle.hpp -- CPU restatement of splat.js's Gaussian-splat training step.
//
// TEST INFRASTRUCTURE ONLY.  This file is the parity oracle: tests, the
// smoke check and the CPU-baseline leg of bench.py call it as the checker.
// Nothing in the product (the CUDA library) includes, links or calls it.
//
// It restates, function by function, the WGSL kernels of the reference
// (src/gs/shaders.js) and the host logic of src/gs/trainer.js.  Every
// function cites the lines it follows.  The reference itself only runs
// under WebGPU (a graphics API), which is unavailable on this box, and it
// stores no golden vectors, so parity with the reference's own output is
// UNPINNED.  What pins this restatement is the reference's own check of its
// backward (src/gs/gradcheck.js): the same 160-splat rig and central finite
// differences of the FP64 loss (tests/test_oracle_pin.py).
//
// Two instantiations:
//   T = float   the FP32 path.  Its evaluation order is fixed exactly (see
//               "canonical FP32 arithmetic" below) and the CUDA kernels follow
//               the same order with the same fused multiply-adds, so the two
//               agree bit for bit.  WGSL leaves the precision of exp/log and
//               of division, and the contraction of a*b+c, to the
//               implementation; the choices made here are within WGSL's
//               stated accuracy bounds.
//   T = double  the FP64 host evaluation used for error statements and for
//               finite differences.  Gradients are accumulated in double with
//               no fixed-point quantisation.
//
// Build with -ffp-contract=off (the Makefile does): every fused
// multiply-add below is written out as std::fma.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace gso {

// ---------------------------------------------------------------------------
// Canonical scalar functions (shared numeric convention with the kernels).
// ---------------------------------------------------------------------------
inline uint32_t fbits(float x) { uint32_t u; std::memcpy(&u, &x, 4); return u; }
inline float bitsf(uint32_t u) { float x; std::memcpy(&x, &u, 4); return x; }

// exp(x) for |x| <= 87: Cody-Waite reduction x = k ln2 + r (ln2 split into a
// 16-bit head and a tail), e^r by its Taylor series to degree 7 (truncation
// error < 1e-8 relative on |r| <= ln2/2), scaled by 2^k built from the
// rounding constant's bits.  Within 2 ulp of exp; WGSL allows 3 + 2|x| ulp.
inline float exp_f(float x) {
  const float RND = 12582912.0f;  // 1.5 * 2^23: adding it rounds to an integer
  float t = std::fma(x, 1.44269504088896341f, RND);
  float k = t - RND;
  float r = std::fma(k, -0.693145751953125f, x);
  r = std::fma(k, -1.42860676533018700e-6f, r);
  float p = 1.98412698412698413e-4f;          // 1/7!
  p = std::fma(p, r, 1.38888888888888889e-3f);  // 1/6!
  p = std::fma(p, r, 8.33333333333333333e-3f);  // 1/5!
  p = std::fma(p, r, 4.16666666666666667e-2f);  // 1/4!
  p = std::fma(p, r, 1.66666666666666667e-1f);  // 1/3!
  p = std::fma(p, r, 0.5f);
  p = std::fma(p, r, 1.0f);
  p = std::fma(p, r, 1.0f);
  uint32_t sb = (fbits(t) << 23) + 0x3F800000u;  // bits of 2^k
  return p * bitsf(sb);
}

// log(x) for positive normal x: x = m 2^e with m in [sqrt(1/2), sqrt(2)),
// log m = 2 atanh(s), s = (m-1)/(m+1), |s| <= 0.1716, odd series to s^11.
inline float log_f(float x) {
  uint32_t b = fbits(x);
  int e = (int)((b >> 23) & 0xFFu) - 127;
  float m = bitsf((b & 0x7FFFFFu) | 0x3F800000u);
  if (m > 1.41421356f) { m = m * 0.5f; e += 1; }
  float s = (m - 1.0f) / (m + 1.0f);
  float s2 = s * s;
  float p = 9.09090909090909091e-2f;            // 1/11
  p = std::fma(p, s2, 1.11111111111111111e-1f);  // 1/9
  p = std::fma(p, s2, 1.42857142857142857e-1f);  // 1/7
  p = std::fma(p, s2, 2.00000000000000000e-1f);  // 1/5
  p = std::fma(p, s2, 3.33333333333333333e-1f);  // 1/3
  p = std::fma(p, s2, 1.0f);
  float lm = (s + s) * p;
  float fe = (float)e;
  return std::fma(fe, 0.693145751953125f, std::fma(fe, 1.42860676533018700e-6f, lm));
}

// sin(x) in double for |x| < 2^31 (only the PSNR dither uses it): quadrant
// reduction by pi/2 split into a 28-bit head (k * head is exact) and a tail,
// then the Taylor series of sin / cos on |r| <= pi/4 to degree 17 / 18.
// Plain double operations only, so host and device agree bit for bit.
inline double sin_d(double x) {
  const double PIO2_HI = 1.570796325802803;
  const double PIO2_LO = 9.920935796805404e-10;
  double k = std::nearbyint(x * 0.6366197723675814);
  double r = (x - k * PIO2_HI) - k * PIO2_LO;
  long q = ((long)k) & 3;
  double r2 = r * r;
  double s = 2.8114572543455206e-15;   // 1/17!
  s = s * r2 - 7.647163731819816e-13;  // 1/15!
  s = s * r2 + 1.6059043836821613e-10; // 1/13!
  s = s * r2 - 2.505210838544172e-08;  // 1/11!
  s = s * r2 + 2.7557319223985893e-06; // 1/9!
  s = s * r2 - 1.984126984126984e-04;  // 1/7!
  s = s * r2 + 8.333333333333333e-03;  // 1/5!
  s = s * r2 - 1.6666666666666666e-01; // 1/3!
  s = (s * r2) * r + r;
  double c = 1.5619206968586225e-16;   // 1/18!
  c = c * r2 - 4.779477332387385e-14;  // 1/16!
  c = c * r2 + 1.1470745597729725e-11; // 1/14!
  c = c * r2 - 2.08767569878681e-09;   // 1/12!
  c = c * r2 + 2.755731922398589e-07;  // 1/10!
  c = c * r2 - 2.48015873015873e-05;   // 1/8!
  c = c * r2 + 1.388888888888889e-03;  // 1/6!
  c = c * r2 - 4.1666666666666664e-02; // 1/4!
  c = c * r2 + 0.5;                    // 1/2!
  c = 1.0 - c * r2;
  if (q == 0) return s;
  if (q == 1) return c;
  if (q == 2) return -s;
  return -c;
}

// WGSL i32(f32) / u32(f32): truncate toward zero, saturate, NaN -> 0.
inline int32_t wgsl_i32(float x) {
  if (!(x == x)) return 0;
  if (x >= 2147483648.0f) return 2147483647;
  if (x <= -2147483648.0f) return (int32_t)0x80000000u;
  return (int32_t)x;
}
inline uint32_t wgsl_u32(float x) {
  if (!(x > 0.0f)) return 0u;
  if (x >= 4294967296.0f) return 0xFFFFFFFFu;
  return (uint32_t)x;
}
// i32(clamp(v * scale, -1e9, 1e9)): the render pass's fixed-point cast
// (shaders.js:529-541, 522-524).
inline int32_t fixq(float v, float scale) {
  float s = v * scale;
  s = std::fmin(std::fmax(s, -1.0e9f), 1.0e9f);
  return wgsl_i32(s);
}

template <class T> struct Math;
template <> struct Math<float> {
  static float exp(float x) { return exp_f(x); }
  static float log(float x) { return log_f(x); }
};
template <> struct Math<double> {
  static double exp(double x) { return std::exp(x); }
  static double log(double x) { return std::log(x); }
};
template <class T> inline T clampT(T x, T lo, T hi) { return std::fmin(std::fmax(x, lo), hi); }
template <class T> inline T sigm(T x) {  // 1 / (1 + exp(-clamp(x, -9, 9)))
  return T(1) / (T(1) + Math<T>::exp(-clampT(x, T(-9), T(9))));
}

// ---------------------------------------------------------------------------
// Options, camera and layout constants (shaders.js:14-54, trainer.js:20-49).
// ---------------------------------------------------------------------------
struct Opts {
  float eCut = 4.5f;        // DEFAULT_E_CUT (shaders.js:44)
  float aMin = 0.0039f;     // DEFAULT_A_MIN (shaders.js:45)
  float radClamp = 1.0f;    // RADCL (shaders.js:46-53)
  float anisoReg = 0.005f;  // AREG default (trainer.js:74)
  int shDeg = 2;            // trainer.js:32
  int tile = 16;            // TILE (shaders.js:32); 16 is the reference's value
  uint64_t entriesCap = 12000000ull;  // ENTCAP (shaders.js:34, trainer.js:48-49)
  int tileCull = 0;         // B200 library option (no reference counterpart): culled tile lists
};

// One view: the Cam uniform of shaders.js:140-152 as _camUniform fills it
// (trainer.js:357-372).  gain = exp(g) and the other host-side values are
// already rounded to f32, as Float32Array stores them.
struct Cam {
  float R[9];
  float t[3];
  float nearz;       // t.w = 0.05
  float f, cx, cy;   // proj.xyz
  float gain;        // proj.w = exp(g)
  int W, H;          // size.xy
  float bg[3];       // misc.xyz (black)
  uint32_t offset;   // misc.w bits: pixel offset of this view's target
  int train;         // misc2.x
  uint32_t camIdx;   // misc2.y
  uint32_t ncams;    // misc2.z
  float bias;        // misc2.w
  float activeSh;    // misc3.x
};

inline int tilesX(const Cam& c, int tile) { return (c.W + tile - 1) / tile; }
inline int tilesY(const Cam& c, int tile) { return (c.H + tile - 1) / tile; }
constexpr int STRIDE = 16;
constexpr float FIXED = 16384.0f;   // shaders.js:35
constexpr float FIXEDC = 16384.0f;  // shaders.js:39
constexpr float FIXCAM = 64.0f;     // shaders.js:158
constexpr uint32_t SHSORT = 2048;   // shaders.js:33

inline int shRestCoefs(int deg) { return deg > 0 ? (deg + 1) * (deg + 1) - 1 : 0; }  // shaders.js:65

// ---------------------------------------------------------------------------
// SH basis Y_k(v) and dY_k/dv (shaders.js:56-138), INRIA constants.
// ---------------------------------------------------------------------------
template <class T> struct SHC;
template <> struct SHC<float> {
  static constexpr float C1 = 0.4886025119029199f;
  static constexpr float C2[5] = {1.0925484305920792f, -1.0925484305920792f, 0.31539156525252005f,
                                  -1.0925484305920792f, 0.5462742152960396f};
  static constexpr float C3[7] = {-0.5900435899266435f, 2.890611442640554f, -0.4570457994644658f,
                                  0.3731763325901154f, -0.4570457994644658f, 1.445305721320277f,
                                  -0.5900435899266435f};
};
template <> struct SHC<double> {
  static constexpr double C1 = 0.4886025119029199;
  static constexpr double C2[5] = {1.0925484305920792, -1.0925484305920792, 0.31539156525252005,
                                   -1.0925484305920792, 0.5462742152960396};
  static constexpr double C3[7] = {-0.5900435899266435, 2.890611442640554, -0.4570457994644658,
                                   0.3731763325901154, -0.4570457994644658, 1.445305721320277,
                                   -0.5900435899266435};
};

template <class T>
inline void shBasis(int deg, const T v[3], T Y[15]) {
  using C = SHC<T>;
  const T x = v[0], y = v[1], z = v[2];
  Y[0] = (-C::C1) * y;
  Y[1] = C::C1 * z;
  Y[2] = (-C::C1) * x;
  if (deg >= 2) {
    const T xx = x * x, yy = y * y, zz = z * z;
    Y[3] = C::C2[0] * x * y;
    Y[4] = C::C2[1] * y * z;
    Y[5] = C::C2[2] * (T(2) * zz - xx - yy);
    Y[6] = C::C2[3] * x * z;
    Y[7] = C::C2[4] * (xx - yy);
    if (deg >= 3) {
      Y[8] = C::C3[0] * y * (T(3) * xx - yy);
      Y[9] = C::C3[1] * x * y * z;
      Y[10] = C::C3[2] * y * (T(4) * zz - xx - yy);
      Y[11] = C::C3[3] * z * (T(2) * zz - T(3) * xx - T(3) * yy);
      Y[12] = C::C3[4] * x * (T(4) * zz - xx - yy);
      Y[13] = C::C3[5] * z * (xx - yy);
      Y[14] = C::C3[6] * x * (xx - yy);
    }
  }
}

// D[k][0..2] = dY_k/dv (shaders.js:76-110)
template <class T>
inline void shBasisGrad(int deg, const T v[3], T D[15][3]) {
  using C = SHC<T>;
  const T x = v[0], y = v[1], z = v[2];
  auto set = [&](int k, T c, T a, T b, T d) { D[k][0] = c * a; D[k][1] = c * b; D[k][2] = c * d; };
  D[0][0] = T(0); D[0][1] = -C::C1; D[0][2] = T(0);
  D[1][0] = T(0); D[1][1] = T(0); D[1][2] = C::C1;
  D[2][0] = -C::C1; D[2][1] = T(0); D[2][2] = T(0);
  if (deg >= 2) {
    const T xx = x * x, yy = y * y, zz = z * z;
    set(3, C::C2[0], y, x, T(0));
    set(4, C::C2[1], T(0), z, y);
    set(5, C::C2[2], T(-2) * x, T(-2) * y, T(4) * z);
    set(6, C::C2[3], z, T(0), x);
    set(7, C::C2[4], T(2) * x, T(-2) * y, T(0));
    if (deg >= 3) {
      set(8, C::C3[0], T(6) * x * y, T(3) * xx - T(3) * yy, T(0));
      set(9, C::C3[1], y * z, x * z, x * y);
      set(10, C::C3[2], T(-2) * x * y, T(4) * zz - xx - T(3) * yy, T(8) * y * z);
      set(11, C::C3[3], T(-6) * x * z, T(-6) * y * z, T(6) * zz - T(3) * xx - T(3) * yy);
      set(12, C::C3[4], T(4) * zz - T(3) * xx - yy, T(-2) * x * y, T(8) * x * z);
      set(13, C::C3[5], T(2) * x * z, T(-2) * y * z, xx - yy);
      set(14, C::C3[6], T(3) * xx - yy, T(-2) * x * y, T(0));
    }
  }
}

// shActiveK (shaders.js:117-120)
inline int shActiveK(const Cam& c, int K) {
  uint32_t ad = wgsl_u32(c.activeSh + 0.5f);
  uint32_t k = (ad + 1u) * (ad + 1u) - 1u;
  return (int)std::min<uint32_t>(k, (uint32_t)K);
}

// camPosWorld = -R^T t (shaders.js:121-126)
template <class T>
inline void camPosWorld(const Cam& c, T out[3]) {
  for (int j = 0; j < 3; ++j)
    out[j] = -(T(c.R[j]) * T(c.t[0]) + T(c.R[3 + j]) * T(c.t[1]) + T(c.R[6 + j]) * T(c.t[2]));
}

template <class T> inline T dot3(const T a[3], const T b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

// ---------------------------------------------------------------------------
// computeGeom (shaders.js:164-225)
// ---------------------------------------------------------------------------
template <class T>
struct Geom {
  bool ok = false;
  T pc[3], q[4], r0[3], r1[3], r2[3], s[3], t0[3], t1[3];
  T va, vb, vc, s00, s01, s02, s11, s12, s22;
};

template <class T>
inline Geom<T> computeGeom(const Cam& c, const T* P) {
  Geom<T> g;
  const T p[3] = {P[0], P[1], P[2]};
  const T R0[3] = {T(c.R[0]), T(c.R[1]), T(c.R[2])};
  const T R1[3] = {T(c.R[3]), T(c.R[4]), T(c.R[5])};
  const T R2[3] = {T(c.R[6]), T(c.R[7]), T(c.R[8])};
  g.pc[0] = dot3(R0, p) + T(c.t[0]);
  g.pc[1] = dot3(R1, p) + T(c.t[1]);
  g.pc[2] = dot3(R2, p) + T(c.t[2]);
  if (g.pc[2] < T(c.nearz)) return g;

  T q[4] = {P[6], P[7], P[8], P[9]};
  T ql = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
  if (ql < T(1e-6)) { q[0] = T(1); q[1] = q[2] = q[3] = T(0); }
  else { for (int k = 0; k < 4; ++k) q[k] = q[k] / ql; }
  for (int k = 0; k < 4; ++k) g.q[k] = q[k];
  const T qw = q[0], qx = q[1], qy = q[2], qz = q[3];
  g.r0[0] = T(1) - T(2) * (qy * qy + qz * qz); g.r0[1] = T(2) * (qx * qy - qw * qz); g.r0[2] = T(2) * (qx * qz + qw * qy);
  g.r1[0] = T(2) * (qx * qy + qw * qz); g.r1[1] = T(1) - T(2) * (qx * qx + qz * qz); g.r1[2] = T(2) * (qy * qz - qw * qx);
  g.r2[0] = T(2) * (qx * qz - qw * qy); g.r2[1] = T(2) * (qy * qz + qw * qx); g.r2[2] = T(1) - T(2) * (qx * qx + qy * qy);

  for (int k = 0; k < 3; ++k) g.s[k] = Math<T>::exp(clampT(P[3 + k], T(-12), T(6)));

  T m0[3], m1[3], m2[3];
  for (int k = 0; k < 3; ++k) { m0[k] = g.r0[k] * g.s[k]; m1[k] = g.r1[k] * g.s[k]; m2[k] = g.r2[k] * g.s[k]; }
  g.s00 = dot3(m0, m0); g.s01 = dot3(m0, m1); g.s02 = dot3(m0, m2);
  g.s11 = dot3(m1, m1); g.s12 = dot3(m1, m2); g.s22 = dot3(m2, m2);

  const T f = T(c.f);
  const T iz = T(1) / g.pc[2];
  const T a0 = f * iz;
  const T b0 = (-f) * g.pc[0] * iz * iz;
  const T b1 = (-f) * g.pc[1] * iz * iz;
  for (int k = 0; k < 3; ++k) {
    g.t0[k] = a0 * R0[k] + b0 * R2[k];
    g.t1[k] = a0 * R1[k] + b1 * R2[k];
  }
  const T st0[3] = {g.s00 * g.t0[0] + g.s01 * g.t0[1] + g.s02 * g.t0[2],
                    g.s01 * g.t0[0] + g.s11 * g.t0[1] + g.s12 * g.t0[2],
                    g.s02 * g.t0[0] + g.s12 * g.t0[1] + g.s22 * g.t0[2]};
  const T st1[3] = {g.s00 * g.t1[0] + g.s01 * g.t1[1] + g.s02 * g.t1[2],
                    g.s01 * g.t1[0] + g.s11 * g.t1[1] + g.s12 * g.t1[2],
                    g.s02 * g.t1[0] + g.s12 * g.t1[1] + g.s22 * g.t1[2]};
  g.va = std::fmax(dot3(g.t0, st0), T(0));
  g.vb = dot3(g.t1, st0);
  g.vc = std::fmax(dot3(g.t1, st1), T(0));
  g.ok = true;
  return g;
}

// Tile bounds of a projected splat (shaders.js:303-308, 395-400).
struct TileRect { int x0, x1, y0, y1; };
template <class T>
inline TileRect tileRect(const Cam& c, int tile, T mx, T my, T rad) {
  const int tx = tilesX(c, tile), ty = tilesY(c, tile);
  const T TF = T(tile);
  auto cl = [](T v, int hi) { return (int)wgsl_u32((float)clampT(std::floor(v), T(0), T(hi))); };
  TileRect r;
  r.x0 = cl((mx - rad) / TF, tx - 1);
  r.x1 = cl((mx + rad) / TF, tx - 1);
  r.y0 = cl((my - rad) / TF, ty - 1);
  r.y1 = cl((my + rad) / TF, ty - 1);
  return r;
}

// ---------------------------------------------------------------------------
// Pass 1: project + SH colour + tile counts (shaders.js:228-315).
// proj layout (shaders.js:23-25): [mx,my,depth,cA,cB,cC,comp,opa,r,g,b,
// visible,va,vb,vc,rad].
// ---------------------------------------------------------------------------
template <class T>
inline void projectOne(const Opts& o, const Cam& c, const T* P, const T* shp, int K, T* pr) {
  pr[11] = T(0);
  Geom<T> g = computeGeom<T>(c, P);
  if (!g.ok) return;
  const T detV = std::fmax(g.va * g.vc - g.vb * g.vb, T(0));
  const T ad = g.va + T(0.3), cd = g.vc + T(0.3);
  const T detVd = ad * cd - g.vb * g.vb;
  if (detVd < T(1e-8)) return;
  const T comp = std::sqrt(std::fmax(detV / detVd, T(0)));
  const T opa = sigm(P[13]);
  if (opa * comp < T(o.aMin)) return;
  const T f = T(c.f);
  const T mx = f * g.pc[0] / g.pc[2] + T(c.cx);
  const T my = f * g.pc[1] / g.pc[2] + T(c.cy);
  const T mid = T(0.5) * (ad + cd);
  const T disc = std::sqrt(std::fmax(mid * mid - detVd, T(0)));
  const T eMax = std::fmin(T(o.eCut), Math<T>::log(std::fmax(opa * comp / T(o.aMin), T(1.0001))));
  const T rad = std::fmin(std::sqrt(T(2) * eMax) * std::sqrt(mid + disc), T(o.radClamp) * T(c.W));
  const T W = T(c.W), H = T(c.H);
  if (mx + rad < T(0) || my + rad < T(0) || mx - rad > W || my - rad > H) return;
  const T inv = T(1) / detVd;
  pr[0] = mx; pr[1] = my; pr[2] = g.pc[2];
  pr[3] = cd * inv; pr[4] = -g.vb * inv; pr[5] = ad * inv;
  pr[6] = comp; pr[7] = opa;
  T col[3] = {sigm(P[10]), sigm(P[11]), sigm(P[12])};
  if (K > 0) {
    T cp[3]; camPosWorld<T>(c, cp);
    T un[3] = {P[0] - cp[0], P[1] - cp[1], P[2] - cp[2]};
    T len = std::fmax(std::sqrt(dot3(un, un)), T(1e-9));
    T v[3] = {un[0] / len, un[1] / len, un[2] / len};
    T Y[15]; shBasis<T>(o.shDeg, v, Y);
    const int aK = shActiveK(c, K);
    for (int k = 0; k < aK; ++k) {
      col[0] = col[0] + shp[k] * Y[k];
      col[1] = col[1] + shp[K + k] * Y[k];
      col[2] = col[2] + shp[2 * K + k] * Y[k];
    }
    for (int j = 0; j < 3; ++j) col[j] = std::fmax(col[j], T(0));
  }
  pr[8] = col[0]; pr[9] = col[1]; pr[10] = col[2];
  pr[11] = T(1);
  pr[12] = g.va; pr[13] = g.vb; pr[14] = g.vc;
  pr[15] = rad;
}

// ---------------------------------------------------------------------------
// Passes 2-4: per-tile counts, budgeted scan, scatter, per-tile sort
// (shaders.js:303-313, 321-374, 378-413, 418-500).  The result is each tile's
// entry list in the reference's final order -- ascending (depth f32 bits,
// id) -- plus the budget drops (tiles whose padded segment would cross the
// entry budget are emptied and counted in stats[3]).
// ---------------------------------------------------------------------------
struct Bins {
  int numTiles = 0;
  std::vector<uint32_t> start;    // numTiles + 1, unpadded prefix of kept counts
  std::vector<uint32_t> ids;      // splat id per entry, tile-major
  std::vector<uint32_t> keys;     // depth f32 bits per entry
  std::vector<uint32_t> cnt;      // raw per-tile count (tileCnt after pass 1)
  std::vector<uint8_t> dropped;   // tile dropped by the entry budget
  uint32_t overflowTiles = 0;     // stats[3] increment
};

inline uint32_t paddedSize(uint32_t c) {  // shaders.js:330-333
  if (c <= SHSORT) return c;
  uint32_t p = 1; while (p < c) p <<= 1; return p;
}

template <class T>
struct Splat2D {  // per-splat values the raster reads (all from proj)
  T mx, my, cA, cB, cC, w, opa, r, g, b, cnorm;
};
template <class T>
inline Splat2D<T> splat2D(const T* pr) {
  Splat2D<T> s;
  s.mx = pr[0]; s.my = pr[1]; s.cA = pr[3]; s.cB = pr[4]; s.cC = pr[5];
  s.w = pr[7] * pr[6];  // proj[b+7] * proj[b+6] (shaders.js:569, 651)
  s.opa = pr[7]; s.r = pr[8]; s.g = pr[9]; s.b = pr[10];
  // cnorm = 1/(1 + lambda_max) of the dilated 2D covariance (shaders.js:674-678)
  const T cva = pr[12] + T(0.3), cvc = pr[14] + T(0.3);
  const T cmid = T(0.5) * (cva + cvc);
  const T lmax = cmid + std::sqrt(std::fmax(cmid * cmid - (cva * cvc - pr[13] * pr[13]), T(0)));
  s.cnorm = T(1) / (T(1) + lmax);
  return s;
}

// Tile cull of the B200 library (no reference counterpart).  Keeps a
// (splat, tile) entry only when some pixel centre of the tile can pass the
// rasteriser's test e <= eCut and w exp(-e) >= aMin; the library runs the
// same sequence (cullParams / bandInterval / tileLive), so both keep the same
// entries.  Culled entries contribute to no pixel.
//
// Per splat and view, completing the square in dx: a pixel (dx, dy) with
// exact exponent e <= t satisfies |dx - kA dy| <= sqrt(p - q dy^2), with
// kA = -B/(2 hA), p = t/hA, q = (4 hA hC - B^2)/(4 hA^2), and t =
// min(eCut, ln(w/aMin)) plus margins for the FP32 evaluation.  Computed in
// double; p rounded up, q down, kA to nearest.  p = +inf: keep everything.
inline float f32_up(double x) {
  float f = (float)x;
  if ((double)f < x) f = std::nextafter(f, INFINITY);
  return f;
}
inline float f32_down(double x) {
  float f = (float)x;
  if ((double)f > x) f = std::nextafter(f, -INFINITY);
  return f;
}
struct CullParams { float p, q, kA; };
inline CullParams cullParams(float mx, float my, float hA, float B, float hC, float w, float aMin, float eCut,
                             int x0, int x1, int y0, int y1, int tile) {
  CullParams c{INFINITY, 0.0f, 0.0f};
  const double A = hA, Bq = B, Cq = hC;
  const double det = 4.0 * A * Cq - Bq * Bq;
  if (A > 0.0 && Cq > 0.0 && det > 0.0) {
    const double dmx = mx, dmy = my, T = tile;
    const double ax = std::fmax(dmx - (double)x0 * T, (double)(x1 + 1) * T - dmx);
    const double ay = std::fmax(dmy - (double)y0 * T, (double)(y1 + 1) * T - dmy);
    const double smax = (A * ax) * ax + (std::fabs(Bq) * ax) * ay + (Cq * ay) * ay;
    const double eA = (double)log_f(w / aMin);
    const double tmax = std::fmin((double)eCut, eA + 1.0e-5) + 2.0e-6 * smax + 1.0e-6;
    c.p = f32_up(tmax / A);
    c.q = f32_down(det / (4.0 * A * A));
    c.kA = (float)(-Bq / (2.0 * A));
  }
  return c;
}
// dx interval of the reachable pixels of the band of rows dy in [Y0, Y1]
// (FP32, with slack for this evaluation); false: band unreachable.
inline bool bandInterval(const CullParams& c, float Y0, float Y1, float& xl, float& xr) {
  float d = Y0 > 0.0f ? Y0 : (Y1 < 0.0f ? -Y1 : 0.0f);
  d = std::fmax(d - (1.0e-3f + 1.0e-6f * d), 0.0f);
  const float rad2 = std::fma(-c.q, d * d, c.p) + 1.0e-5f * c.p;
  if (!(rad2 >= 0.0f)) return false;
  const float r = std::sqrt(rad2) * 1.00001f;
  const float c0 = c.kA * Y0, c1 = c.kA * Y1;
  const float cl = std::fmin(c0, c1), ch = std::fmax(c0, c1);
  const float sl = 4.0e-3f * (1.0f + std::fabs(c.kA)) + 1.0e-5f * (std::fabs(cl) + std::fabs(ch) + r);
  xl = (cl - r) - sl;
  xr = (ch + r) + sl;
  return true;
}
inline bool tileLive(const CullParams& c, float mx, float my, int tx, int ty, int tile, int W, int H) {
  if (!(c.p < 3.0e38f)) return true;
  const int xe = std::min(tx * tile + tile, W), ye = std::min(ty * tile + tile, H);
  float xl, xr;
  if (!bandInterval(c, ((float)(ty * tile) + 0.5f) - my, ((float)(ye - 1) + 0.5f) - my, xl, xr)) return false;
  const float X0 = ((float)(tx * tile) + 0.5f) - mx;
  const float X1 = ((float)(xe - 1) + 0.5f) - mx;
  return X1 >= xl && X0 <= xr;
}

template <class T>
inline Bins binTiles(const Opts& o, const Cam& c, const T* proj, uint32_t n) {
  Bins b;
  const int tx = tilesX(c, o.tile), ty = tilesY(c, o.tile);
  b.numTiles = tx * ty;
  b.cnt.assign(b.numTiles, 0);
  std::vector<std::vector<std::pair<uint32_t, uint32_t>>> lists(b.numTiles);
  for (uint32_t i = 0; i < n; ++i) {
    const T* pr = proj + (size_t)i * STRIDE;
    if (!(pr[11] > T(0))) continue;
    TileRect r = tileRect<T>(c, o.tile, pr[0], pr[1], pr[15]);
    const float depth = (float)pr[2];
    const bool test = o.tileCull && !(r.x0 == r.x1 && r.y0 == r.y1);
    CullParams cp{INFINITY, 0.0f, 0.0f};
    float cmx = 0.0f, cmy = 0.0f;
    if (test) {
      const Splat2D<T> s2 = splat2D<T>(pr);
      cmx = (float)s2.mx; cmy = (float)s2.my;
      cp = cullParams(cmx, cmy, (float)(T(0.5) * s2.cA), (float)s2.cB, (float)(T(0.5) * s2.cC), (float)s2.w, o.aMin,
                      o.eCut, r.x0, r.x1, r.y0, r.y1, o.tile);
    }
    for (int y = r.y0; y <= r.y1; ++y)
      for (int x = r.x0; x <= r.x1; ++x) {
        b.cnt[y * tx + x]++;  // the budget counts every rectangle tile
        if (test && !tileLive(cp, cmx, cmy, x, y, o.tile, c.W, c.H)) continue;
        lists[y * tx + x].push_back({fbits(depth), i});
      }
  }
  // budgeted scan (shaders.js:357-372): a tile is dropped when its padded
  // segment would end past ENTCAP; zero-count tiles never are.
  b.dropped.assign(b.numTiles, 0);
  uint64_t acc = 0;
  for (int t = 0; t < b.numTiles; ++t) {
    uint64_t p = paddedSize(b.cnt[t]);
    if (acc + p > o.entriesCap) { p = 0; b.overflowTiles++; b.dropped[t] = 1; }
    acc += p;
  }
  b.start.assign(b.numTiles + 1, 0);
  for (int t = 0; t < b.numTiles; ++t) {
    auto& L = lists[t];
    b.start[t + 1] = b.start[t];
    if (b.dropped[t]) continue;
    std::sort(L.begin(), L.end());  // ascending (key, id): shaders.js:454, 489
    for (auto& e : L) { b.keys.push_back(e.first); b.ids.push_back(e.second); }
    b.start[t + 1] += (uint32_t)L.size();
  }
  return b;
}

// ---------------------------------------------------------------------------
// Gradient / statistics accumulators for the render pass.
// ---------------------------------------------------------------------------
// FP32 path: the reference's fixed-point i32 accumulators (integer sums are
// order-independent, so the tile-parallel loop below is deterministic).
struct AccFixed {
  int32_t* gradP;     // n * 16, slots 0-9 used
  uint32_t* stats;    // [4]
  int32_t* gradCam;   // (ncams + 1) * 8
  void add(uint32_t id, int slot, float v) {
    int32_t q = fixq(v, FIXED);
    if (q) {
#pragma omp atomic
      gradP[(size_t)id * STRIDE + slot] += q;
    }
  }
  void stat(int k, uint32_t v) {
#pragma omp atomic
    stats[k] += v;
  }
  void cam(uint32_t idx, float v) {
    int32_t q = fixq(v, FIXCAM);
#pragma omp atomic
    gradCam[idx] += q;
  }
};
// FP64 path: unquantised double sums; loss kept as a double.  quantise
// truncates each per-pixel contribution to the fixed-point quantum as the
// reference does (i32(clamp(v * 16384, +-1e9)), shaders.js:529-541), in
// double: it separates the reference's quantisation error from FP32
// rounding when the FP32 path is compared with FP64.
struct AccF64 {
  double* gradP;      // n * 16
  double* lossSum;    // [0] sum of Charbonnier loss, [1] sum of squared error, [2] valid px
  double* gradCam;    // (ncams + 1) * 8
  bool quantise = false;
  void add(uint32_t id, int slot, double v) {
    if (quantise) v = std::trunc(std::fmin(std::fmax(v * (double)FIXED, -1.0e9), 1.0e9)) / (double)FIXED;
#pragma omp atomic
    gradP[(size_t)id * STRIDE + slot] += v;
  }
  void cam(uint32_t idx, double v) {
#pragma omp atomic
    gradCam[idx] += v;
  }
};

// Per-pixel outputs of the forward pass, kept for the backward.
struct PixelState {
  float T;        // final transmittance (FP32 path)
  uint32_t end;   // one past the last processed entry, relative to the tile start
};

// ---------------------------------------------------------------------------
// Render: forward composite, loss + stats, back-to-front backward
// (shaders.js:544-700).  Canonical FP32 arithmetic of the per-pair loop --
// the CUDA rasteriser evaluates exactly these operations:
//   dx = px - mx; dy = py - my
//   e  = max(fma(fma(cA/2, dx, cB*dy), dx, ((cC/2)*dy)*dy), 0)
//   G  = exp(-e); araw = w*G (w = opa*comp); alpha = min(0.99, araw)
//   fwd: ta = T*alpha; C = fma(ta, c, C); T = T*(1 - alpha)
//   bwd: inv = 1/(1 - alpha); Tb = Ta*inv; aT = alpha*Tb; gcv = gC*aT
//        galpha = fma(gCz, gz, fma(gCy, gy, gCx*gx)), g = fma(c, Tb, -(S*inv))
//        ga = galpha*araw; dmean = ga*fma(cA,dx,cB*dy), ga*fma(cB,dx,cC*dy)
//        gq = ga*(-0.5*cnorm); dconic = (gq*dx)*dx, ((gq*dx)*dy)*2, (gq*dy)*dy
//        dcomp = (galpha*opa)*G; dlogit = ga*(1-opa); S = fma(c, aT, S)
// (x*(1/y) stands in for WGSL's x/y, whose accuracy bound is 2.5 ulp.)
// ---------------------------------------------------------------------------
template <class T>
inline T pairExponent(const Splat2D<T>& s, T dx, T dy) {
  // e = 0.5 cA dx^2 + cB dx dy + 0.5 cC dy^2 evaluated as
  // fma(fma(cA/2, dx, cB*dy), dx, ((cC/2)*dy)*dy); halving is exact
  const T hA = T(0.5) * s.cA, hC = T(0.5) * s.cC;
  const T u = std::fma(hA, dx, s.cB * dy);
  return std::fmax(std::fma(u, dx, (hC * dy) * dy), T(0));
}

// Loss of one pixel (shaders.js:589-618).  Returns false for an invalid
// target pixel.  FP32 path.
struct PixelLoss { float gC[3]; float eg[3]; float sqerr16, lossv; };
inline float ditherOf(uint32_t pi) {  // fract(sin(f32(pi) * 12.9898) * 43758.5453)
  float a = (float)pi * 12.9898f;
  float s = (float)sin_d((double)a);
  float v = s * 43758.5453f;
  return v - std::floor(v);
}
inline bool targetRGB(uint32_t packed, float t[3]) {  // unpack4x8unorm (shaders.js:594-598)
  if ((packed >> 24) == 0u) return false;
  t[0] = (float)(packed & 0xFFu) / 255.0f;
  t[1] = (float)((packed >> 8) & 0xFFu) / 255.0f;
  t[2] = (float)((packed >> 16) & 0xFFu) / 255.0f;
  return true;
}
// DELTA*DELTA and 3*DELTA are WGSL const-expressions (abstract float) rounded once to f32.
constexpr float CHARB_D2 = (float)(0.03 * 0.03);
constexpr float CHARB_3D = (float)(3.0 * 0.03);

// Loss of one pixel (defined below for the FP32 and FP64 paths).
template <class T, class Acc>
inline bool lossPixel(const Cam& c, const uint32_t* targets, uint32_t pi, const T C[3], T gC[3], Acc& acc);

// Raster of one view.  variant 0 = recompute transmittance from the final T
// (the reference's division recursion); variant 1 = stored-state (the
// forward's T before each entry is kept and the backward reads it).
template <class T, class Acc>
void renderView(const Opts& o, const Cam& c, const T* proj, const Bins& b, const uint32_t* targets,
                float* outImg, PixelState* pxs, Acc acc, bool train, int variant, uint64_t* pairsOut,
                int tileStride = 1) {
  const int tile = o.tile;
  const int tx = tilesX(c, tile);
  const T E_CUT = T(o.eCut), A_MIN = T(o.aMin);
  uint64_t pairs = 0;
  if (tileStride < 1) tileStride = 1;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : pairs)
  for (int t = 0; t < b.numTiles; t += tileStride) {
    const uint32_t s0 = b.start[t], s1 = b.start[t + 1];
    const int ox = (t % tx) * tile, oy = (t / tx) * tile;
    std::vector<T> Tstore;
    for (int ly = 0; ly < tile; ++ly)
      for (int lx = 0; lx < tile; ++lx) {
        const int gx = ox + lx, gy = oy + ly;
        if (gx >= c.W || gy >= c.H) continue;
        const T px = T(gx) + T(0.5), py = T(gy) + T(0.5);
        // ---- forward (shaders.js:556-585) ----
        T Tr = T(1);
        T C[3] = {T(0), T(0), T(0)};
        uint32_t end = s0;
        if (variant == 1) Tstore.assign(s1 - s0, T(0));
        for (uint32_t k = s0; k < s1; ++k) {
          end = k + 1;
          const Splat2D<T> s = splat2D<T>(proj + (size_t)b.ids[k] * STRIDE);
          const T dx = px - s.mx, dy = py - s.my;
          const T e = pairExponent(s, dx, dy);
          if (e > E_CUT) continue;
          const T araw = s.w * Math<T>::exp(-e);
          const T alpha = std::fmin(T(0.99), araw);
          if (alpha < A_MIN) continue;
          if (variant == 1) Tstore[k - s0] = Tr;
          const T ta = Tr * alpha;
          C[0] = std::fma(ta, s.r, C[0]);
          C[1] = std::fma(ta, s.g, C[1]);
          C[2] = std::fma(ta, s.b, C[2]);
          Tr = Tr * (T(1) - alpha);
          if (Tr < T(1e-4)) break;
        }
        pairs += end - s0;
        const uint32_t pi = (uint32_t)(gy * c.W + gx);
        T Cf[3];
        for (int j = 0; j < 3; ++j) Cf[j] = C[j] + Tr * T(c.bg[j]);
        if (outImg) {
          outImg[pi * 4 + 0] = (float)Cf[0]; outImg[pi * 4 + 1] = (float)Cf[1];
          outImg[pi * 4 + 2] = (float)Cf[2]; outImg[pi * 4 + 3] = (float)(T(1) - Tr);
        }
        if (pxs) { pxs[pi].T = (float)Tr; pxs[pi].end = end - s0; }
        if (!train) continue;
        // ---- loss (shaders.js:589-618) ----
        T gC[3];
        if (!lossPixel<T>(c, targets, pi, Cf, gC, acc)) continue;
        // ---- backward (shaders.js:632-700) ----
        T S[3] = {T(c.bg[0]) * Tr, T(c.bg[1]) * Tr, T(c.bg[2]) * Tr};
        T Ta = Tr;
        for (uint32_t kk = end; kk > s0; --kk) {
          const uint32_t id = b.ids[kk - 1];
          const Splat2D<T> s = splat2D<T>(proj + (size_t)id * STRIDE);
          const T dx = px - s.mx, dy = py - s.my;
          const T e = pairExponent(s, dx, dy);
          if (e > E_CUT) continue;
          const T G = Math<T>::exp(-e);
          const T araw = s.w * G;
          const T alpha = std::fmin(T(0.99), araw);
          if (alpha < A_MIN) continue;
          const T inv = T(1) / (T(1) - alpha);
          const T Tb = (variant == 1) ? Tstore[kk - 1 - s0] : Ta * inv;
          const T aT = alpha * Tb;
          const T col[3] = {s.r, s.g, s.b};
          T gv[3];
          for (int j = 0; j < 3; ++j) gv[j] = std::fma(col[j], Tb, -(S[j] * inv));
          T galpha = std::fma(gC[2], gv[2], std::fma(gC[1], gv[1], gC[0] * gv[0]));
          if (araw > T(0.99)) galpha = T(0);
          const T ga = galpha * araw;
          acc.add(id, 0, ga * std::fma(s.cA, dx, s.cB * dy));
          acc.add(id, 1, ga * std::fma(s.cB, dx, s.cC * dy));
          const T gq = ga * (T(-0.5f) * s.cnorm);
          const T gqx = gq * dx;
          acc.add(id, 2, gqx * dx);
          acc.add(id, 3, (gqx * dy) * T(2));
          acc.add(id, 4, (gq * dy) * dy);
          acc.add(id, 5, (galpha * s.opa) * G);
          acc.add(id, 6, ga * (T(1) - s.opa));
          acc.add(id, 7, gC[0] * aT);
          acc.add(id, 8, gC[1] * aT);
          acc.add(id, 9, gC[2] * aT);
          for (int j = 0; j < 3; ++j) S[j] = std::fma(col[j], aT, S[j]);
          Ta = Tb;
        }
      }
  }
  if (pairsOut) *pairsOut += pairs;
}


template <>
inline bool lossPixel<float, AccFixed>(const Cam& c, const uint32_t* targets, uint32_t pi, const float C[3],
                                       float gC[3], AccFixed& acc) {
  float tc[3];
  if (!targetRGB(targets[(size_t)c.offset + pi], tc)) return false;
  acc.stat(2, 1u);
  const float gain = c.gain;
  float err[3], root[3], eg[3];
  for (int j = 0; j < 3; ++j) err[j] = (gain * C[j] + c.bias) - tc[j];
  const float dith = ditherOf(pi);
  acc.stat(0, wgsl_u32(dot3(err, err) * 16.0f + dith));
  for (int j = 0; j < 3; ++j) {
    root[j] = std::sqrt(err[j] * err[j] + CHARB_D2);
    eg[j] = err[j] / root[j];
    gC[j] = gain * eg[j];
  }
  const float lossv = (root[0] + root[1] + root[2]) - CHARB_3D;
  acc.stat(1, wgsl_u32(lossv * 32768.0f));
  const uint32_t ci8 = c.camIdx * 8u;
  acc.cam(ci8 + 6u, dot3(eg, C) * gain);
  acc.cam(ci8 + 7u, eg[0] + eg[1] + eg[2]);
  return true;
}

template <>
inline bool lossPixel<double, AccF64>(const Cam& c, const uint32_t* targets, uint32_t pi, const double C[3],
                                      double gC[3], AccF64& acc) {
  float tcf[3];
  if (!targetRGB(targets[(size_t)c.offset + pi], tcf)) return false;
  const double gain = c.gain, d2 = 0.03 * 0.03;
  double err[3], root[3], eg[3];
  for (int j = 0; j < 3; ++j) err[j] = (gain * C[j] + (double)c.bias) - (double)tcf[j];
  double lossv = 0;
  for (int j = 0; j < 3; ++j) {
    root[j] = std::sqrt(err[j] * err[j] + d2);
    eg[j] = err[j] / root[j];
    gC[j] = gain * eg[j];
    lossv += root[j];
  }
  lossv -= 3.0 * 0.03;
#pragma omp atomic
  acc.lossSum[0] += lossv;
#pragma omp atomic
  acc.lossSum[1] += dot3(err, err);
#pragma omp atomic
  acc.lossSum[2] += 1.0;
  const uint32_t ci8 = c.camIdx * 8u;
  acc.cam(ci8 + 6u, dot3(eg, C) * gain);
  acc.cam(ci8 + 7u, eg[0] + eg[1] + eg[2]);
  return true;
}

// ---------------------------------------------------------------------------
// Chain pass (shaders.js:704-949): screen-space grads -> parameter grads.
// gp[0..9] are the decoded screen-space grads (conic slots still carrying
// the render pass's 1/(1+lambda_max) normalisation).
// ---------------------------------------------------------------------------
template <class T, class CamAdd>
inline void chainOne(const Opts& o, const Cam& c, const T* P, const T* pr, const T* shp, int K, T gp[10],
                     T* gF, T* shG, CamAdd camAdd) {
  {  // undo the conic normalisation (shaders.js:735-744)
    const T cva = pr[12] + T(0.3), cvc = pr[14] + T(0.3);
    const T cmid = T(0.5) * (cva + cvc);
    const T lmax = cmid + std::sqrt(std::fmax(cmid * cmid - (cva * cvc - pr[13] * pr[13]), T(0)));
    const T cden = T(1) + lmax;
    gp[2] = gp[2] * cden; gp[3] = gp[3] * cden; gp[4] = gp[4] * cden;
  }
  for (int k = 0; k < STRIDE; ++k) gF[k] = T(0);
  for (int k = 0; k < 3 * K; ++k) shG[k] = T(0);
  if (!(pr[11] > T(0))) return;
  Geom<T> g = computeGeom<T>(c, P);
  if (!g.ok) return;
  const T f = T(c.f), z = g.pc[2], iz = T(1) / z;
  // conic -> dilated 2D covariance (shaders.js:758-777)
  const T ad = g.va + T(0.3), cd = g.vc + T(0.3);
  const T detVd = ad * cd - g.vb * g.vb;
  const T inv = T(1) / detVd;
  const T kA = cd * inv, kB = -g.vb * inv, kC = ad * inv;
  const T g11 = gp[2], g12 = T(0.5) * gp[3], g22 = gp[4];
  const T m100 = g11 * kA + g12 * kB, m101 = g11 * kB + g12 * kC;
  const T m110 = g12 * kA + g22 * kB, m111 = g12 * kB + g22 * kC;
  const T p00 = kA * m100 + kB * m110, p01 = kA * m101 + kB * m111;
  const T p10 = kB * m100 + kC * m110, p11 = kB * m101 + kC * m111;
  T gva = -p00, gvb = -(p01 + p10), gvc = -p11;
  // comp -> raw 2D covariance (shaders.js:779-788)
  const T detV = std::fmax(g.va * g.vc - g.vb * g.vb, T(0));
  const T comp = std::sqrt(std::fmax(detV / detVd, T(0)));
  if (comp > T(1e-4)) {
    const T gcomp = gp[5];
    const T denom = T(2) * comp * detVd;
    gva = gva + gcomp * (g.vc - comp * comp * cd) / denom;
    gvc = gvc + gcomp * (g.va - comp * comp * ad) / denom;
    gvb = gvb + gcomp * (T(2) * g.vb * (comp * comp - T(1))) / denom;
  }
  // V = T Sigma T^T backward (shaders.js:790-810)
  const T h11 = gva, h12 = T(0.5) * gvb, h22 = gvc;
  T u0[3], u1[3];
  for (int k = 0; k < 3; ++k) { u0[k] = h11 * g.t0[k] + h12 * g.t1[k]; u1[k] = h12 * g.t0[k] + h22 * g.t1[k]; }
  const T* t0 = g.t0; const T* t1 = g.t1;
  const T dS00 = t0[0] * u0[0] + t1[0] * u1[0];
  const T dS01 = T(0.5) * ((t0[0] * u0[1] + t1[0] * u1[1]) + (t0[1] * u0[0] + t1[1] * u1[0]));
  const T dS02 = T(0.5) * ((t0[0] * u0[2] + t1[0] * u1[2]) + (t0[2] * u0[0] + t1[2] * u1[0]));
  const T dS11 = t0[1] * u0[1] + t1[1] * u1[1];
  const T dS12 = T(0.5) * ((t0[1] * u0[2] + t1[1] * u1[2]) + (t0[2] * u0[1] + t1[2] * u1[1]));
  const T dS22 = t0[2] * u0[2] + t1[2] * u1[2];
  const T sT0[3] = {g.s00 * t0[0] + g.s01 * t0[1] + g.s02 * t0[2],
                    g.s01 * t0[0] + g.s11 * t0[1] + g.s12 * t0[2],
                    g.s02 * t0[0] + g.s12 * t0[1] + g.s22 * t0[2]};
  const T sT1[3] = {g.s00 * t1[0] + g.s01 * t1[1] + g.s02 * t1[2],
                    g.s01 * t1[0] + g.s11 * t1[1] + g.s12 * t1[2],
                    g.s02 * t1[0] + g.s12 * t1[1] + g.s22 * t1[2]};
  T dT0[3], dT1[3];
  for (int k = 0; k < 3; ++k) {
    dT0[k] = T(2) * (h11 * sT0[k] + h12 * sT1[k]);
    dT1[k] = T(2) * (h12 * sT0[k] + h22 * sT1[k]);
  }
  // T = J W: position through J (shaders.js:812-822)
  const T R0[3] = {T(c.R[0]), T(c.R[1]), T(c.R[2])};
  const T R1[3] = {T(c.R[3]), T(c.R[4]), T(c.R[5])};
  const T R2[3] = {T(c.R[6]), T(c.R[7]), T(c.R[8])};
  const T dJ00 = dot3(dT0, R0), dJ02 = dot3(dT0, R2), dJ11 = dot3(dT1, R1), dJ12 = dot3(dT1, R2);
  T dpc[3] = {T(0), T(0), T(0)};
  dpc[0] = dpc[0] + dJ02 * ((-f) * iz * iz);
  dpc[1] = dpc[1] + dJ12 * ((-f) * iz * iz);
  dpc[2] = dpc[2] + ((dJ00 + dJ11) * ((-f) * iz * iz) + dJ02 * (T(2) * f * g.pc[0] * iz * iz * iz) +
                     dJ12 * (T(2) * f * g.pc[1] * iz * iz * iz));
  // mean path (shaders.js:824-827)
  dpc[0] = dpc[0] + gp[0] * f * iz;
  dpc[1] = dpc[1] + gp[1] * f * iz;
  dpc[2] = dpc[2] + (-f) * (gp[0] * g.pc[0] + gp[1] * g.pc[1]) * iz * iz;
  // W^T dpc (shaders.js:830-832)
  gF[0] = R0[0] * dpc[0] + R1[0] * dpc[1] + R2[0] * dpc[2];
  gF[1] = R0[1] * dpc[0] + R1[1] * dpc[1] + R2[1] * dpc[2];
  gF[2] = R0[2] * dpc[0] + R1[2] * dpc[1] + R2[2] * dpc[2];
  // camera pose gradients (shaders.js:835-858)
  if (c.train) {
    const uint32_t ci = c.camIdx * 8u;
    camAdd(ci + 3u, dpc[0]); camAdd(ci + 4u, dpc[1]); camAdd(ci + 5u, dpc[2]);
    const T pt[3] = {g.pc[0] - T(c.t[0]), g.pc[1] - T(c.t[1]), g.pc[2] - T(c.t[2])};
    T dw[3] = {pt[1] * dpc[2] - pt[2] * dpc[1], pt[2] * dpc[0] - pt[0] * dpc[2], pt[0] * dpc[1] - pt[1] * dpc[0]};
    T dW0[3], dW1[3], dW2[3];
    for (int k = 0; k < 3; ++k) {
      dW0[k] = (f * iz) * dT0[k];
      dW1[k] = (f * iz) * dT1[k];
      dW2[k] = ((-f) * g.pc[0] * iz * iz) * dT0[k] + ((-f) * g.pc[1] * iz * iz) * dT1[k];
    }
    T acc3[3] = {T(0), T(0), T(0)};
    for (int k = 0; k < 3; ++k) {  // cross(wc_k, (dW0[k], dW1[k], dW2[k])), wc_k = column k of R
      const T wc[3] = {T(c.R[k]), T(c.R[3 + k]), T(c.R[6 + k])};
      const T v[3] = {dW0[k], dW1[k], dW2[k]};
      const T cr[3] = {wc[1] * v[2] - wc[2] * v[1], wc[2] * v[0] - wc[0] * v[2], wc[0] * v[1] - wc[1] * v[0]};
      if (k == 0) { acc3[0] = cr[0]; acc3[1] = cr[1]; acc3[2] = cr[2]; }
      else { acc3[0] = acc3[0] + cr[0]; acc3[1] = acc3[1] + cr[1]; acc3[2] = acc3[2] + cr[2]; }
    }
    for (int k = 0; k < 3; ++k) dw[k] = dw[k] + acc3[k];
    camAdd(ci, dw[0]); camAdd(ci + 1u, dw[1]); camAdd(ci + 2u, dw[2]);
    const T dlogf = gp[0] * f * g.pc[0] * iz + gp[1] * f * g.pc[1] * iz + (dJ00 + dJ11) * (f * iz) +
                    dJ02 * ((-f) * g.pc[0] * iz * iz) + dJ12 * ((-f) * g.pc[1] * iz * iz);
    camAdd(c.ncams * 8u, dlogf);
  }
  // Sigma = M M^T backward -> scales (shaders.js:860-884)
  T m0[3], m1[3], m2[3];
  for (int k = 0; k < 3; ++k) { m0[k] = g.r0[k] * g.s[k]; m1[k] = g.r1[k] * g.s[k]; m2[k] = g.r2[k] * g.s[k]; }
  T dM0[3], dM1[3], dM2[3];
  for (int k = 0; k < 3; ++k) {
    dM0[k] = T(2) * (dS00 * m0[k] + dS01 * m1[k] + dS02 * m2[k]);
    dM1[k] = T(2) * (dS01 * m0[k] + dS11 * m1[k] + dS12 * m2[k]);
    dM2[k] = T(2) * (dS02 * m0[k] + dS12 * m1[k] + dS22 * m2[k]);
  }
  T dsv[3];
  for (int k = 0; k < 3; ++k) dsv[k] = dM0[k] * g.r0[k] + dM1[k] * g.r1[k] + dM2[k] * g.r2[k];
  const T ls[3] = {clampT(P[3], T(-12), T(6)), clampT(P[4], T(-12), T(6)), clampT(P[5], T(-12), T(6))};
  const T mls = (ls[0] + ls[1] + ls[2]) / T(3);
  const T AREG = T(o.anisoReg);
  for (int k = 0; k < 3; ++k) gF[3 + k] = dsv[k] * g.s[k] + AREG * (ls[k] - mls);
  // quaternion backward (shaders.js:886-904)
  T dR0[3], dR1[3], dR2[3];
  for (int k = 0; k < 3; ++k) { dR0[k] = dM0[k] * g.s[k]; dR1[k] = dM1[k] * g.s[k]; dR2[k] = dM2[k] * g.s[k]; }
  const T qw = g.q[0], qx = g.q[1], qy = g.q[2], qz = g.q[3];
  const T gw = T(2) * (dR0[1] * (-qz) + dR0[2] * qy + dR1[0] * qz + dR1[2] * (-qx) + dR2[0] * (-qy) + dR2[1] * qx);
  const T gx = T(2) * (dR0[1] * qy + dR0[2] * qz + dR1[0] * qy + dR1[1] * (T(-2) * qx) + dR1[2] * (-qw) +
                       dR2[0] * qz + dR2[1] * qw + dR2[2] * (T(-2) * qx));
  const T gy = T(2) * (dR0[0] * (T(-2) * qy) + dR0[1] * qx + dR0[2] * qw + dR1[0] * qx + dR1[2] * qz +
                       dR2[0] * (-qw) + dR2[1] * qz + dR2[2] * (T(-2) * qy));
  const T gz = T(2) * (dR0[0] * (T(-2) * qz) + dR0[1] * (-qw) + dR0[2] * qx + dR1[0] * qw + dR1[1] * (T(-2) * qz) +
                       dR1[2] * qy + dR2[0] * qx + dR2[1] * qy);
  const T gq[4] = {gw, gx, gy, gz};
  const T qr[4] = {P[6], P[7], P[8], P[9]};
  const T ql = std::fmax(std::sqrt(qr[0] * qr[0] + qr[1] * qr[1] + qr[2] * qr[2] + qr[3] * qr[3]), T(1e-6));
  const T qd = g.q[0] * gq[0] + g.q[1] * gq[1] + g.q[2] * gq[2] + g.q[3] * gq[3];
  for (int k = 0; k < 4; ++k) gF[6 + k] = (gq[k] - g.q[k] * qd) / ql;
  // colour: DC sigmoid chain + SH bands (+ position via view dir) (shaders.js:906-947)
  const T sCol[3] = {sigm(P[10]), sigm(P[11]), sigm(P[12])};
  T dRGB[3] = {gp[7], gp[8], gp[9]};
  if (K > 0) {
    T cp[3]; camPosWorld<T>(c, cp);
    const T un[3] = {P[0] - cp[0], P[1] - cp[1], P[2] - cp[2]};
    const T ulen = std::fmax(std::sqrt(dot3(un, un)), T(1e-9));
    const T v[3] = {un[0] / ulen, un[1] / ulen, un[2] / ulen};
    T Y[15], D[15][3];
    shBasis<T>(o.shDeg, v, Y);
    shBasisGrad<T>(o.shDeg, v, D);
    const int aK = shActiveK(c, K);
    T col[3] = {sCol[0], sCol[1], sCol[2]};
    for (int k = 0; k < aK; ++k) {
      col[0] = col[0] + shp[k] * Y[k];
      col[1] = col[1] + shp[K + k] * Y[k];
      col[2] = col[2] + shp[2 * K + k] * Y[k];
    }
    for (int j = 0; j < 3; ++j) dRGB[j] = dRGB[j] * (col[j] > T(0) ? T(1) : T(0));
    T gv[3] = {T(0), T(0), T(0)};
    for (int k = 0; k < aK; ++k) {
      shG[k] = dRGB[0] * Y[k];
      shG[K + k] = dRGB[1] * Y[k];
      shG[2 * K + k] = dRGB[2] * Y[k];
      const T wk = dRGB[0] * shp[k] + dRGB[1] * shp[K + k] + dRGB[2] * shp[2 * K + k];
      for (int j = 0; j < 3; ++j) gv[j] = gv[j] + wk * D[k][j];
    }
    const T vg = dot3(v, gv);
    for (int j = 0; j < 3; ++j) gF[j] = gF[j] + (gv[j] - v[j] * vg) / ulen;
  }
  for (int j = 0; j < 3; ++j) gF[10 + j] = dRGB[j] * sCol[j] * (T(1) - sCol[j]);
  gF[13] = gp[6];
}

// ---------------------------------------------------------------------------
// Adam (shaders.js:984-1036) and SH-Adam (shaders.js:952-982).
// The bias corrections 1 - b^t are computed on the host in double and
// rounded to f32 (adamBiasCorrection); WGSL's pow is implementation-defined.
// ---------------------------------------------------------------------------
struct AdamHP {
  float lr[16];
  float b1 = 0.9f, b2 = 0.999f, eps = 1e-15f;
  float bc1, bc2;        // 1 - b1^t, 1 - b2^t
  float minLS, maxLS, maxLogit;
  float reg;             // opacity regularisation weight
  float shLr;
};
inline void adamBiasCorrection(double t, float& bc1, float& bc2) {
  bc1 = (float)(1.0 - std::pow((double)0.9f, t));
  bc2 = (float)(1.0 - std::pow((double)0.999f, t));
}

inline void adamParam(const AdamHP& h, int slot, float& p, float g, float& m, float& v) {
  const float lr = h.lr[slot];
  if (lr == 0.0f) return;
  if (!(std::fabs(g) < 1e18f)) g = 0.0f;
  if (slot == 13) {
    const float sg = sigm(p);
    g = g + h.reg * sg * (1.0f - sg);
  }
  m = h.b1 * m + (1.0f - h.b1) * g;
  v = h.b2 * v + (1.0f - h.b2) * g * g;
  const float mh = m / h.bc1, vh = v / h.bc2;
  float pn = p - lr * mh / (std::sqrt(vh) + h.eps);
  if (slot >= 3 && slot <= 5) pn = clampT(pn, h.minLS, h.maxLS);
  if (slot >= 10 && slot <= 13) pn = clampT(pn, -h.maxLogit, h.maxLogit);
  p = pn;
}
inline void adamSH(const AdamHP& h, float& p, float g, float& m, float& v) {
  if (!(std::fabs(g) < 1e18f)) g = 0.0f;
  m = h.b1 * m + (1.0f - h.b1) * g;
  v = h.b2 * v + (1.0f - h.b2) * g * g;
  const float mh = m / h.bc1, vh = v / h.bc2;
  p = p - h.shLr * mh / (std::sqrt(vh) + h.eps);
}

}  // namespace gso
