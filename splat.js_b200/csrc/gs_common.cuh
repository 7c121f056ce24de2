// gs_common.cuh -- device-side conventions shared by every kernel.
//
// Numerics.  The library is compiled with -fmad=false: no a*b+c is fused
// unless the source writes fmaf().  Division and square root are IEEE
// (-prec-div/-prec-sqrt default), denormals are kept (no -ftz).  exp, log and
// the dither's sin are computed by the canonical functions below (written
// from the mathematics, not from any library), so every FP32 value a kernel
// produces is reproducible bit for bit by a host restatement that performs
// the same operations.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace gs {

constexpr int STRIDE = 16;          // params / proj stride (shaders.js:14-25)
constexpr int GP_STRIDE = 12;       // screen-space gradient slots 0-9 (+2 pad) per splat
constexpr float FIXED = 16384.0f;   // shaders.js:35
constexpr float FIXEDC = 16384.0f;  // shaders.js:39
constexpr float FIXCAM = 64.0f;     // shaders.js:158
constexpr uint32_t SHSORT = 2048;   // shaders.js:33 (padding rule of the entry budget)
constexpr int MAX_K = 15;           // SH rest coefficients per channel at degree 3

// Device camera record: the Cam uniform of shaders.js:140-152 as
// _camUniform fills it (trainer.js:357-372), plus derived tile geometry.
constexpr int MAX_VIEWS = 16;  // most views one batched step can hold

struct DevCam {
  float R[9];
  float t[3];
  float nearz;
  float f, cx, cy, gain;
  float bg[3];
  float bias;
  float activeSh;
  int32_t W, H;
  int32_t tilesX, tilesY;
  uint32_t offset;     // pixel offset of this view's target image
  uint32_t camIdx;     // gradCam row
  uint32_t ncams;      // gradCam focal row index
  int32_t train;
  uint32_t tileBase;   // first global tile id of this view in a batch
  uint32_t pixBase;    // first pixel of this view in the batch's pixel buffers
};

// Copy n camera records to shared memory with every thread of the block
// taking 4-byte words, so the copy costs one load latency, not a chain of
// them in one thread (the caller's barrier publishes it).
static_assert(sizeof(DevCam) % 4 == 0, "camera records copy as words");
__device__ __forceinline__ void copy_cams(DevCam* dst, const DevCam* src, int n) {
  const uint32_t* s = reinterpret_cast<const uint32_t*>(src);
  uint32_t* d = reinterpret_cast<uint32_t*>(dst);
  const int words = n * (int)(sizeof(DevCam) / 4);
  for (int k = threadIdx.x; k < words; k += blockDim.x) d[k] = s[k];
}

// Per-(view, splat) record read by the rasteriser: 3 x float4 = 48 B.
//   r0 = (mx, my, cA/2, cB)  r1 = (cC/2, w = opa*comp, r, g)  r2 = (b, opa, -cnorm/2, 1 - opa)
struct __align__(16) RenderRec {
  float4 r0, r1, r2;
};

// ---- asynchronous staging (cp.async: global -> shared without registers) ----
// 16-byte copies bypassing L1 (each record is read once per block); a
// thread's copies complete, in commit order, at its wait_group.
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// ---- canonical scalar functions --------------------------------------------
// exp(x), |x| <= 87: Cody-Waite reduction x = k ln2 + r with ln2 split in a
// 16-bit head and a tail, e^r by its degree-7 Taylor series on
// |r| <= ln2/2, times 2^k assembled from the rounding constant's bits.
__device__ __forceinline__ float gexp(float x) {
  const float RND = 12582912.0f;  // 1.5 * 2^23
  float t = __fmaf_rn(x, 1.44269504088896341f, RND);
  float k = __fsub_rn(t, RND);
  float r = __fmaf_rn(k, -0.693145751953125f, x);
  r = __fmaf_rn(k, -1.42860676533018700e-6f, r);
  float p = 1.98412698412698413e-4f;
  p = __fmaf_rn(p, r, 1.38888888888888889e-3f);
  p = __fmaf_rn(p, r, 8.33333333333333333e-3f);
  p = __fmaf_rn(p, r, 4.16666666666666667e-2f);
  p = __fmaf_rn(p, r, 1.66666666666666667e-1f);
  p = __fmaf_rn(p, r, 0.5f);
  p = __fmaf_rn(p, r, 1.0f);
  p = __fmaf_rn(p, r, 1.0f);
  uint32_t sb = (__float_as_uint(t) << 23) + 0x3F800000u;
  return __fmul_rn(p, __uint_as_float(sb));
}

// 1/x rounded to nearest (equal to IEEE 1.0f / x) for x in [2^-7, 1]: the
// hardware's approximate reciprocal refined by two Newton-Raphson steps with
// fused multiply-adds (e = 1 - x y; y += e y), the last of which acts as
// Markstein's correction step.  The domain has no zeros, denormals or
// infinities, so no slow path is needed; gs_debug_check_rcp compares the
// result with IEEE division for every float in the domain.
__device__ __forceinline__ float rcp_unit(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  float e = __fmaf_rn(-x, y, 1.0f);
  y = __fmaf_rn(e, y, y);
  e = __fmaf_rn(-x, y, 1.0f);
  return __fmaf_rn(e, y, y);
}

// ---- packed forms (two pixels per thread) ----------------------------------
// sm_100 executes two FP32 operations per instruction (fma/mul/add.rn.f32x2),
// each element rounded exactly as the scalar instruction; a scalar operand is
// broadcast to both elements.  Each function below performs, element by
// element, the same operation sequence as its scalar counterpart above, so
// its results are bit-identical to two scalar calls.
__device__ __forceinline__ float2 bc2(float s) { return make_float2(s, s); }

__device__ __forceinline__ float2 gexp2(float2 x) {
  const float RND = 12582912.0f;
  const float2 t = __ffma2_rn(x, bc2(1.44269504088896341f), bc2(RND));
  const float2 k = __fadd2_rn(t, bc2(-RND));  // t - RND: subtraction is addition of the negation
  float2 r = __ffma2_rn(k, bc2(-0.693145751953125f), x);
  r = __ffma2_rn(k, bc2(-1.42860676533018700e-6f), r);
  float2 p = __ffma2_rn(bc2(1.98412698412698413e-4f), r, bc2(1.38888888888888889e-3f));
  p = __ffma2_rn(p, r, bc2(8.33333333333333333e-3f));
  p = __ffma2_rn(p, r, bc2(4.16666666666666667e-2f));
  p = __ffma2_rn(p, r, bc2(1.66666666666666667e-1f));
  p = __ffma2_rn(p, r, bc2(0.5f));
  p = __ffma2_rn(p, r, bc2(1.0f));
  p = __ffma2_rn(p, r, bc2(1.0f));
  const float2 sb = make_float2(__uint_as_float((__float_as_uint(t.x) << 23) + 0x3F800000u),
                                __uint_as_float((__float_as_uint(t.y) << 23) + 0x3F800000u));
  return __fmul2_rn(p, sb);
}

__device__ __forceinline__ float2 rcp_unit2(float2 x) {
  float2 y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y.x) : "f"(x.x));
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y.y) : "f"(x.y));
  const float2 nx = make_float2(-x.x, -x.y);
  float2 e = __ffma2_rn(nx, y, bc2(1.0f));
  y = __ffma2_rn(e, y, y);
  e = __ffma2_rn(nx, y, bc2(1.0f));
  return __ffma2_rn(e, y, y);
}

// log(x), x positive normal: x = m 2^e, m in [sqrt(1/2), sqrt(2)),
// log m = 2 atanh((m-1)/(m+1)) by its odd series to degree 11.
__device__ __forceinline__ float glog(float x) {
  uint32_t b = __float_as_uint(x);
  int e = (int)((b >> 23) & 0xFFu) - 127;
  float m = __uint_as_float((b & 0x7FFFFFu) | 0x3F800000u);
  if (m > 1.41421356f) { m = m * 0.5f; e += 1; }
  float s = __fdiv_rn(m - 1.0f, m + 1.0f);
  float s2 = s * s;
  float p = 9.09090909090909091e-2f;
  p = __fmaf_rn(p, s2, 1.11111111111111111e-1f);
  p = __fmaf_rn(p, s2, 1.42857142857142857e-1f);
  p = __fmaf_rn(p, s2, 2.00000000000000000e-1f);
  p = __fmaf_rn(p, s2, 3.33333333333333333e-1f);
  p = __fmaf_rn(p, s2, 1.0f);
  float lm = (s + s) * p;
  float fe = (float)e;
  return __fmaf_rn(fe, 0.693145751953125f, __fmaf_rn(fe, 1.42860676533018700e-6f, lm));
}

// Cull parameters of one splat in one view.  Completing the square in dx, a
// pixel (dx, dy) (offsets from the mean) with exact exponent
// e = hA dx^2 + B dx dy + hC dy^2 <= t satisfies
//   |dx - kA dy| <= sqrt(p - q dy^2),  kA = -B / (2 hA), p = t / hA,
//   q = (4 hA hC - B^2) / (4 hA^2).
// t is the largest exponent the rasteriser can accept, min(eCut, ln(w/aMin)),
// plus margins for its FP32 evaluation (2e-6 of the largest term over the
// splat's tile rectangle, which bounds a few ulp of every term) and for the
// canonical log (1e-5).  Computed in double; p is rounded up, q down and kA
// to nearest, so the bound stays conservative.  (p, q, kA) = (+inf, 0, 0)
// marks a degenerate conic: every pixel is kept.  The oracle repeats this
// sequence exactly.
__device__ __forceinline__ float4 cullParams(float mx, float my, float hA, float B, float hC, float w, float aMin,
                                             float eCut, uint32_t x0, uint32_t x1, uint32_t y0, uint32_t y1,
                                             int tile) {
  float4 cq = make_float4(__int_as_float(0x7F800000), 0.0f, 0.0f, 0.0f);
  const double A = (double)hA, Bq = (double)B, Cq = (double)hC;
  const double det = 4.0 * A * Cq - Bq * Bq;
  if (A > 0.0 && Cq > 0.0 && det > 0.0) {
    const double dmx = (double)mx, dmy = (double)my, T = (double)tile;
    const double ax = fmax(dmx - (double)x0 * T, (double)(x1 + 1) * T - dmx);
    const double ay = fmax(dmy - (double)y0 * T, (double)(y1 + 1) * T - dmy);
    const double smax = (A * ax) * ax + (fabs(Bq) * ax) * ay + (Cq * ay) * ay;
    const double eA = (double)glog(w / aMin);
    const double tmax = fmin((double)eCut, eA + 1.0e-5) + 2.0e-6 * smax + 1.0e-6;
    cq.x = __double2float_ru(tmax / A);
    cq.y = __double2float_rd(det / (4.0 * A * A));
    cq.z = __double2float_rn(-Bq / (2.0 * A));
  }
  return cq;
}

// The dx interval [xl, xr] that holds every reachable pixel of the band of
// pixel-centre rows with dy in [Y0, Y1]: |dx - kA dy| <= sqrt(p - q dmin^2),
// dmin the band's smallest |dy|.  Slack covers this FP32 evaluation (the
// rounding of Y0/Y1 and of the products).  false: the band is unreachable.
// p = +inf never gets here (callers keep everything).
__device__ __forceinline__ bool bandInterval(const float4 cq, float Y0, float Y1, float& xl, float& xr) {
  const float p = cq.x, q = cq.y, kA = cq.z;
  float d = Y0 > 0.0f ? Y0 : (Y1 < 0.0f ? -Y1 : 0.0f);
  d = fmaxf(d - (1.0e-3f + 1.0e-6f * d), 0.0f);
  const float rad2 = __fmaf_rn(-q, d * d, p) + 1.0e-5f * p;
  if (!(rad2 >= 0.0f)) return false;
  const float r = sqrtf(rad2) * 1.00001f;
  const float c0 = kA * Y0, c1 = kA * Y1;
  const float cl = fminf(c0, c1), ch = fmaxf(c0, c1);
  const float sl = 4.0e-3f * (1.0f + fabsf(kA)) + 1.0e-5f * (fabsf(cl) + fabsf(ch) + r);
  xl = (cl - r) - sl;
  xr = (ch + r) + sl;
  return true;
}

// bandInterval with the square root taken as rad2 * rsqrt(rad2) (a few ulp
// instead of correctly rounded), for the rasteriser's warp-block masks only:
// they need to be conservative, not reproducible, and the interval's 1e-5
// relative and 4e-3 px absolute slack exceed that error by two orders of
// magnitude.  The tile cull keeps bandInterval, which the oracle repeats.
__device__ __forceinline__ bool bandIntervalMask(const float4 cq, float Y0, float Y1, float& xl, float& xr) {
  const float p = cq.x, q = cq.y, kA = cq.z;
  float d = Y0 > 0.0f ? Y0 : (Y1 < 0.0f ? -Y1 : 0.0f);
  d = fmaxf(d - (1.0e-3f + 1.0e-6f * d), 0.0f);
  const float rad2 = __fmaf_rn(-q, d * d, p) + 1.0e-5f * p;
  if (!(rad2 >= 0.0f)) return false;
  const float r = (rad2 > 0.0f ? rad2 * rsqrtf(rad2) : 0.0f) * 1.00001f;
  const float c0 = kA * Y0, c1 = kA * Y1;
  const float cl = fminf(c0, c1), ch = fmaxf(c0, c1);
  const float sl = 4.0e-3f * (1.0f + fabsf(kA)) + 1.0e-5f * (fabsf(cl) + fabsf(ch) + r);
  xl = (cl - r) - sl;
  xr = (ch + r) + sl;
  return true;
}

// Tile cull: can any pixel centre of tile (tx, ty) (clipped to the W x H
// image) be reachable?  A (splat, tile) entry that fails cannot composite
// into any pixel of the tile, so dropping it changes no image, loss or
// gradient.  The oracle runs the same FP32 sequence, so both keep the same
// entries.
__device__ __forceinline__ bool tileLive(const float4 cq, float mx, float my, int tx, int ty, int tile, int W,
                                         int H) {
  if (!(cq.x < 3.0e38f)) return true;
  const int xe = tx * tile + tile < W ? tx * tile + tile : W;
  const int ye = ty * tile + tile < H ? ty * tile + tile : H;
  float xl, xr;
  if (!bandInterval(cq, ((float)(ty * tile) + 0.5f) - my, ((float)(ye - 1) + 0.5f) - my, xl, xr)) return false;
  const float X0 = ((float)(tx * tile) + 0.5f) - mx;
  const float X1 = ((float)(xe - 1) + 0.5f) - mx;
  return X1 >= xl && X0 <= xr;
}

// sin(x) in double, |x| < 2^31: quadrant reduction by pi/2 (28-bit head so
// k * head is exact, plus a tail), Taylor series of sin/cos on |r| <= pi/4.
__device__ __forceinline__ double gsin_d(double x) {
  const double PIO2_HI = 1.570796325802803;
  const double PIO2_LO = 9.920935796805404e-10;
  double k = rint(__dmul_rn(x, 0.6366197723675814));
  double r = __dsub_rn(__dsub_rn(x, __dmul_rn(k, PIO2_HI)), __dmul_rn(k, PIO2_LO));
  long long q = ((long long)k) & 3;
  double r2 = r * r;
  double s = 2.8114572543455206e-15;
  s = s * r2 - 7.647163731819816e-13;
  s = s * r2 + 1.6059043836821613e-10;
  s = s * r2 - 2.505210838544172e-08;
  s = s * r2 + 2.7557319223985893e-06;
  s = s * r2 - 1.984126984126984e-04;
  s = s * r2 + 8.333333333333333e-03;
  s = s * r2 - 1.6666666666666666e-01;
  s = (s * r2) * r + r;
  double c = 1.5619206968586225e-16;
  c = c * r2 - 4.779477332387385e-14;
  c = c * r2 + 1.1470745597729725e-11;
  c = c * r2 - 2.08767569878681e-09;
  c = c * r2 + 2.755731922398589e-07;
  c = c * r2 - 2.48015873015873e-05;
  c = c * r2 + 1.388888888888889e-03;
  c = c * r2 - 4.1666666666666664e-02;
  c = c * r2 + 0.5;
  c = 1.0 - c * r2;
  if (q == 0) return s;
  if (q == 1) return c;
  if (q == 2) return -s;
  return -c;
}

__device__ __forceinline__ float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }
// x / d (IEEE, div.rn.f32) with a zero numerator answered without dividing:
// +-0 / d = +-0 exactly for every d > 0, +inf included; other d divide as
// written.  Zero numerators are common in the per-splat passes (parameters
// whose gradient history is all zero, splats that composited nowhere), and
// the compiled division takes its out-of-line path for them: measured on the
// Adam pass, every division and square root branched out of line in about
// three warp-instances of four.  The division is written as a PTX
// instruction so that the guard's select stays on its operand (as a C
// expression the compiler may fold the select into the quotient and divide
// the zero after all).  The result is bit-identical to x / d.
__device__ __forceinline__ float div_nz(float x, float d) {
  const bool z = x == 0.0f && d > 0.0f;
  float q;
  asm("div.rn.f32 %0, %1, %2;" : "=f"(q) : "f"(z ? 1.0f : x), "f"(d));
  return z ? x : q;
}
// sqrt(x) (IEEE, sqrt.rn.f32) with zero answered without the root:
// sqrt(+-0) = +-0.
__device__ __forceinline__ float sqrt_nz(float x) {
  const bool z = x == 0.0f;
  float r;
  asm("sqrt.rn.f32 %0, %1;" : "=f"(r) : "f"(z ? 1.0f : x));
  return z ? x : r;
}
// 1 / (1 + exp(-clamp(x, -9, 9)))
__device__ __forceinline__ float sigm(float x) { return 1.0f / (1.0f + gexp(-clampf(x, -9.0f, 9.0f))); }
// i32(clamp(v * scale, -1e9, 1e9)) with WGSL's truncating cast (shaders.js:529-541)
__device__ __forceinline__ int32_t fixq(float v, float scale) {
  float s = v * scale;
  s = fminf(fmaxf(s, -1.0e9f), 1.0e9f);
  return __float2int_rz(s);
}
// u32(f32): truncate, saturate, NaN -> 0
__device__ __forceinline__ uint32_t u32sat(float x) { return __float2uint_rz(x); }

// fract(sin(f32(pi) * 12.9898) * 43758.5453): the PSNR dither (shaders.js:605)
__device__ __forceinline__ float dither(uint32_t pi) {
  float a = (float)pi * 12.9898f;
  float s = (float)gsin_d((double)a);
  float v = s * 43758.5453f;
  return v - floorf(v);
}

__device__ __forceinline__ int shActiveK(const DevCam& c, int K) {
  uint32_t ad = u32sat(c.activeSh + 0.5f);
  uint32_t k = (ad + 1u) * (ad + 1u) - 1u;
  return (int)min(k, (uint32_t)K);
}

// Status flags shared with the host (device status word, bit set).
enum StatusBits : uint32_t {
  ST_LOOKBACK_TIMEOUT = 1u << 0,  // a decoupled look-back spin reached its limit
  ST_ENTRY_OVERFLOW = 1u << 1,    // more (tile, splat) entries than the entry buffer holds
  ST_BAD_INPUT = 1u << 2,
};

}  // namespace gs
