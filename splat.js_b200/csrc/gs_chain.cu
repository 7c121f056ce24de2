// gs_chain.cu -- per-splat pass after the rasteriser: the chain rule from
// screen-space gradients to parameter gradients (shaders.js:704-949), fused
// with Adam (shaders.js:984-1036) and SH-Adam (shaders.js:952-982).
//
// Two passes.  Pass 1 (one thread per (view, splat)) decodes each visible
// splat's fixed-point screen-space gradients (clearing them for the next
// step) and chains them through that view's camera.  Pass 2 (one thread per
// splat) sums the views' parameter gradients in view order and runs Adam
// and SH-Adam once, with coalesced parameter and moment traffic.  The
// reference runs chain, Adam and SH-Adam as three dispatches with gradF /
// shGrad round-tripping through memory; here the summed gradients stay on
// chip unless the caller asks for them (gradient readout for checks).
// Operation order follows the WGSL.
#include "gs_geom.cuh"
#include "gs_kernels.h"

namespace gs {

struct CamGrad7 {
  float w[3], t[3], logf;
};

// chain for one visible splat in one view; gp = decoded screen-space grads
// shp: the splat's SH coefficients in global memory (read through the
// cache).  The SH coefficient gradients are dRGB[c] * Y[k] for k < aK: the
// gated dRGB, Y and aK are returned instead of the 3K products.
template <int DEG>
__device__ __forceinline__ void chainOne(const DevCam& c, const float* P, const Geom& g, float gp[10],
                                         const float* shp, float anisoReg, float gF[16], float dRGBo[3],
                                         float Yo[15], float vdo[3], int& aKo, CamGrad7& cg) {
  constexpr int K = DEG > 0 ? (DEG + 1) * (DEG + 1) - 1 : 0;
  const float f = c.f, z = g.pc[2], iz = 1.0f / z;
  // conic -> dilated 2D covariance (shaders.js:758-777)
  const float ad = g.va + 0.3f, cd = g.vc + 0.3f;
  const float detVd = ad * cd - g.vb * g.vb;
  const float inv = 1.0f / detVd;
  const float kA = cd * inv, kB = -g.vb * inv, kC = ad * inv;
  const float g11 = gp[2], g12 = 0.5f * gp[3], g22 = gp[4];
  const float m100 = g11 * kA + g12 * kB, m101 = g11 * kB + g12 * kC;
  const float m110 = g12 * kA + g22 * kB, m111 = g12 * kB + g22 * kC;
  const float p00 = kA * m100 + kB * m110, p01 = kA * m101 + kB * m111;
  const float p10 = kB * m100 + kC * m110, p11 = kB * m101 + kC * m111;
  float gva = -p00, gvb = -(p01 + p10), gvc = -p11;
  // comp -> raw 2D covariance (shaders.js:779-788)
  const float detV = fmaxf(g.va * g.vc - g.vb * g.vb, 0.0f);
  const float comp = sqrt_nz(fmaxf(div_nz(detV, detVd), 0.0f));
  if (comp > 1e-4f) {
    const float gcomp = gp[5];
    const float denom = 2.0f * comp * detVd;
    gva = gva + div_nz(gcomp * (g.vc - comp * comp * cd), denom);
    gvc = gvc + div_nz(gcomp * (g.va - comp * comp * ad), denom);
    gvb = gvb + div_nz(gcomp * (2.0f * g.vb * (comp * comp - 1.0f)), denom);
  }
  // V = T Sigma T^T backward (shaders.js:790-810)
  const float h11 = gva, h12 = 0.5f * gvb, h22 = gvc;
  float u0[3], u1[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    u0[k] = h11 * g.t0[k] + h12 * g.t1[k];
    u1[k] = h12 * g.t0[k] + h22 * g.t1[k];
  }
  const float* t0 = g.t0;
  const float* t1 = g.t1;
  const float dS00 = t0[0] * u0[0] + t1[0] * u1[0];
  const float dS01 = 0.5f * ((t0[0] * u0[1] + t1[0] * u1[1]) + (t0[1] * u0[0] + t1[1] * u1[0]));
  const float dS02 = 0.5f * ((t0[0] * u0[2] + t1[0] * u1[2]) + (t0[2] * u0[0] + t1[2] * u1[0]));
  const float dS11 = t0[1] * u0[1] + t1[1] * u1[1];
  const float dS12 = 0.5f * ((t0[1] * u0[2] + t1[1] * u1[2]) + (t0[2] * u0[1] + t1[2] * u1[1]));
  const float dS22 = t0[2] * u0[2] + t1[2] * u1[2];
  const float sT0[3] = {g.s00 * t0[0] + g.s01 * t0[1] + g.s02 * t0[2],
                        g.s01 * t0[0] + g.s11 * t0[1] + g.s12 * t0[2],
                        g.s02 * t0[0] + g.s12 * t0[1] + g.s22 * t0[2]};
  const float sT1[3] = {g.s00 * t1[0] + g.s01 * t1[1] + g.s02 * t1[2],
                        g.s01 * t1[0] + g.s11 * t1[1] + g.s12 * t1[2],
                        g.s02 * t1[0] + g.s12 * t1[1] + g.s22 * t1[2]};
  float dT0[3], dT1[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    dT0[k] = 2.0f * (h11 * sT0[k] + h12 * sT1[k]);
    dT1[k] = 2.0f * (h12 * sT0[k] + h22 * sT1[k]);
  }
  // T = J W: position through J (shaders.js:812-822)
  const float R0[3] = {c.R[0], c.R[1], c.R[2]};
  const float R1[3] = {c.R[3], c.R[4], c.R[5]};
  const float R2[3] = {c.R[6], c.R[7], c.R[8]};
  const float dJ00 = dot3(dT0, R0), dJ02 = dot3(dT0, R2), dJ11 = dot3(dT1, R1), dJ12 = dot3(dT1, R2);
  float dpc[3] = {0.0f, 0.0f, 0.0f};
  dpc[0] = dpc[0] + dJ02 * ((-f) * iz * iz);
  dpc[1] = dpc[1] + dJ12 * ((-f) * iz * iz);
  dpc[2] = dpc[2] + ((dJ00 + dJ11) * ((-f) * iz * iz) + dJ02 * (2.0f * f * g.pc[0] * iz * iz * iz) +
                     dJ12 * (2.0f * f * g.pc[1] * iz * iz * iz));
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
    cg.t[0] = dpc[0]; cg.t[1] = dpc[1]; cg.t[2] = dpc[2];
    const float pt[3] = {g.pc[0] - c.t[0], g.pc[1] - c.t[1], g.pc[2] - c.t[2]};
    float dw[3] = {pt[1] * dpc[2] - pt[2] * dpc[1], pt[2] * dpc[0] - pt[0] * dpc[2],
                   pt[0] * dpc[1] - pt[1] * dpc[0]};
    float dW0[3], dW1[3], dW2[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      dW0[k] = (f * iz) * dT0[k];
      dW1[k] = (f * iz) * dT1[k];
      dW2[k] = ((-f) * g.pc[0] * iz * iz) * dT0[k] + ((-f) * g.pc[1] * iz * iz) * dT1[k];
    }
    float acc3[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const float wc[3] = {c.R[k], c.R[3 + k], c.R[6 + k]};
      const float vv[3] = {dW0[k], dW1[k], dW2[k]};
      const float cr[3] = {wc[1] * vv[2] - wc[2] * vv[1], wc[2] * vv[0] - wc[0] * vv[2],
                           wc[0] * vv[1] - wc[1] * vv[0]};
      if (k == 0) { acc3[0] = cr[0]; acc3[1] = cr[1]; acc3[2] = cr[2]; }
      else { acc3[0] = acc3[0] + cr[0]; acc3[1] = acc3[1] + cr[1]; acc3[2] = acc3[2] + cr[2]; }
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) cg.w[k] = dw[k] + acc3[k];
    cg.logf = gp[0] * f * g.pc[0] * iz + gp[1] * f * g.pc[1] * iz + (dJ00 + dJ11) * (f * iz) +
              dJ02 * ((-f) * g.pc[0] * iz * iz) + dJ12 * ((-f) * g.pc[1] * iz * iz);
  }
  // Sigma = M M^T backward -> scales (shaders.js:860-884)
  float m0[3], m1[3], m2[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    m0[k] = g.r0[k] * g.s[k];
    m1[k] = g.r1[k] * g.s[k];
    m2[k] = g.r2[k] * g.s[k];
  }
  float dM0[3], dM1[3], dM2[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    dM0[k] = 2.0f * (dS00 * m0[k] + dS01 * m1[k] + dS02 * m2[k]);
    dM1[k] = 2.0f * (dS01 * m0[k] + dS11 * m1[k] + dS12 * m2[k]);
    dM2[k] = 2.0f * (dS02 * m0[k] + dS12 * m1[k] + dS22 * m2[k]);
  }
  float dsv[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) dsv[k] = dM0[k] * g.r0[k] + dM1[k] * g.r1[k] + dM2[k] * g.r2[k];
  const float ls[3] = {clampf(P[3], -12.0f, 6.0f), clampf(P[4], -12.0f, 6.0f), clampf(P[5], -12.0f, 6.0f)};
  const float mls = (ls[0] + ls[1] + ls[2]) / 3.0f;
#pragma unroll
  for (int k = 0; k < 3; ++k) gF[3 + k] = dsv[k] * g.s[k] + anisoReg * (ls[k] - mls);
  // quaternion backward (shaders.js:886-904)
  float dR0[3], dR1[3], dR2[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    dR0[k] = dM0[k] * g.s[k];
    dR1[k] = dM1[k] * g.s[k];
    dR2[k] = dM2[k] * g.s[k];
  }
  const float qw = g.q[0], qx = g.q[1], qy = g.q[2], qz = g.q[3];
  const float gw = 2.0f * (dR0[1] * (-qz) + dR0[2] * qy + dR1[0] * qz + dR1[2] * (-qx) + dR2[0] * (-qy) +
                           dR2[1] * qx);
  const float gx = 2.0f * (dR0[1] * qy + dR0[2] * qz + dR1[0] * qy + dR1[1] * (-2.0f * qx) + dR1[2] * (-qw) +
                           dR2[0] * qz + dR2[1] * qw + dR2[2] * (-2.0f * qx));
  const float gy = 2.0f * (dR0[0] * (-2.0f * qy) + dR0[1] * qx + dR0[2] * qw + dR1[0] * qx + dR1[2] * qz +
                           dR2[0] * (-qw) + dR2[1] * qz + dR2[2] * (-2.0f * qy));
  const float gz = 2.0f * (dR0[0] * (-2.0f * qz) + dR0[1] * (-qw) + dR0[2] * qx + dR1[0] * qw +
                           dR1[1] * (-2.0f * qz) + dR1[2] * qy + dR2[0] * qx + dR2[1] * qy);
  const float gq[4] = {gw, gx, gy, gz};
  const float ql = fmaxf(sqrtf(P[6] * P[6] + P[7] * P[7] + P[8] * P[8] + P[9] * P[9]), 1e-6f);
  const float qd = g.q[0] * gq[0] + g.q[1] * gq[1] + g.q[2] * gq[2] + g.q[3] * gq[3];
#pragma unroll
  for (int k = 0; k < 4; ++k) gF[6 + k] = div_nz(gq[k] - g.q[k] * qd, ql);
  // colour: DC sigmoid chain + SH bands (+ position via view dir) (shaders.js:906-947)
  const float sCol[3] = {sigm(P[10]), sigm(P[11]), sigm(P[12])};
  float dRGB[3] = {gp[7], gp[8], gp[9]};
  aKo = 0;
  if (K > 0) {
    float cp[3];
    camPosWorld(c, cp);
    const float un[3] = {P[0] - cp[0], P[1] - cp[1], P[2] - cp[2]};
    const float ulen = fmaxf(sqrtf(dot3(un, un)), 1e-9f);
    const float vd[3] = {un[0] / ulen, un[1] / ulen, un[2] / ulen};
    vdo[0] = vd[0]; vdo[1] = vd[1]; vdo[2] = vd[2];
    shBasis<DEG>(vd, Yo);
    const int aK = shActiveK(c, K);
    aKo = aK;
    float col[3] = {sCol[0], sCol[1], sCol[2]};
#pragma unroll
    for (int k = 0; k < K; ++k)
      if (k < aK) {
        col[0] = col[0] + __ldg(shp + k) * Yo[k];
        col[1] = col[1] + __ldg(shp + K + k) * Yo[k];
        col[2] = col[2] + __ldg(shp + 2 * K + k) * Yo[k];
      }
#pragma unroll
    for (int j = 0; j < 3; ++j) dRGB[j] = dRGB[j] * (col[j] > 0.0f ? 1.0f : 0.0f);
    float gv[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int k = 0; k < K; ++k)
      if (k < aK) {
        const float wk = dRGB[0] * __ldg(shp + k) + dRGB[1] * __ldg(shp + K + k) + dRGB[2] * __ldg(shp + 2 * K + k);
        float D[3];
        shBasisGradK<DEG>(k, vd, D);
#pragma unroll
        for (int j = 0; j < 3; ++j) gv[j] = gv[j] + wk * D[j];
      }
    const float vg = dot3(vd, gv);
#pragma unroll
    for (int j = 0; j < 3; ++j) gF[j] = gF[j] + div_nz(gv[j] - vd[j] * vg, ulen);
  }
#pragma unroll
  for (int j = 0; j < 3; ++j) gF[10 + j] = dRGB[j] * sCol[j] * (1.0f - sCol[j]);
  gF[13] = gp[6];
  dRGBo[0] = dRGB[0]; dRGBo[1] = dRGB[1]; dRGBo[2] = dRGB[2];
}

// Adam for one parameter slot (shaders.js:984-1036).  The slot's learning
// rate, clamp and regulariser are the same for every element a thread
// updates (a block's 128 threads cover the 16 slots eight times over), so
// they are resolved once per thread: AdamSlot holds them in registers and
// the per-element update is straight-line.  The opacity slot's regularised
// gradient (sanitised, plus reg * s * (1 - s) of the opacity before the
// update) is computed per splat beforehand and passed in as g.
struct AdamSlot {
  float lr, lo, hi;
  bool live, clamp, opa;
};
__device__ __forceinline__ AdamSlot adam_slot(const AdamHP& h, int slot) {
  AdamSlot r;
  r.lr = h.lr[slot];
  r.live = r.lr != 0.0f;
  const bool ls = slot >= 3 && slot <= 5, lg = slot >= 10 && slot <= 13;
  r.clamp = ls || lg;
  r.lo = ls ? h.minLS : -h.maxLogit;
  r.hi = ls ? h.maxLS : h.maxLogit;
  r.opa = slot == 13;
  return r;
}
struct AdamK {  // the step's Adam constants, read once per thread
  float b1, b2, ob1, ob2, bc1, bc2, eps, reg, shLr;
};
__device__ __forceinline__ AdamK adam_k(const AdamHP& h) {
  return AdamK{h.b1, h.b2, 1.0f - h.b1, 1.0f - h.b2, h.bc1, h.bc2, h.eps, h.reg, h.shLr};
}
// m, v and the parameter after one step; g already sanitised
__device__ __forceinline__ float adam_update(const AdamK& k, float lr, float p, float g, float& m, float& v) {
  m = k.b1 * m + k.ob1 * g;
  v = k.b2 * v + k.ob2 * g * g;
  const float mh = div_nz(m, k.bc1), vh = div_nz(v, k.bc2);
  return p - div_nz(lr * mh, sqrt_nz(vh) + k.eps);
}
// the sanitising of shaders.js:990 (non-finite or huge gradients count as 0)
__device__ __forceinline__ float adam_g(float g) { return fabsf(g) < 1e18f ? g : 0.0f; }

#ifndef GS_CHAIN_MIN_BLOCKS
#define GS_CHAIN_MIN_BLOCKS 4  // resident 128-thread blocks per SM the register allocation must allow (no spills)
#endif

// Visible-item lists: for each view, the indices of the splats whose
// rectangle survived projection, compacted with one atomic per block.  The
// order inside a list follows the blocks' atomics (roughly ascending), which
// pass 1 uses only for memory locality: each item's results go to its own
// slot and camera gradients are integer sums, so no result depends on it.
__global__ void __launch_bounds__(256) k_visible_list(ChainArgs a, uint32_t blocksPerView) {
  __shared__ uint32_t s_warp[8];
  __shared__ uint32_t s_base;
  const uint32_t v = blockIdx.x / blocksPerView;
  const uint32_t i = (blockIdx.x - v * blocksPerView) * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const bool vis = i < a.n && a.rect[(size_t)v * a.n + i].x != 0xFFFFFFFFu;
  const uint32_t b = __ballot_sync(0xFFFFFFFFu, vis);
  if (lane == 0) s_warp[wid] = (uint32_t)__popc(b);
  __syncthreads();
  if (threadIdx.x == 0) {  // one atomic per block
    uint32_t t = 0;
    for (int w = 0; w < 8; ++w) { const uint32_t c = s_warp[w]; s_warp[w] = t; t += c; }
    s_base = t ? atomicAdd(&a.visCount[v], t) : 0u;
  }
  __syncthreads();
  if (vis) a.visList[(size_t)v * a.n + s_base + s_warp[wid] + (uint32_t)__popc(b & ((1u << lane) - 1u))] = i;
}

// Pass 1: one thread per visible (view, splat) item of the lists above.
// Blocks are ordered list block major, view minor, so the views' items of
// similar splat indices run together and their parameters and SH
// coefficients are mostly read from DRAM once.  A visible splat's screen-space
// gradients are decoded (and cleared for the next step) and chained through
// the view's camera; the result -- the 14 parameter gradients, the gated
// colour gradient dRGB and the view direction (from which the SH basis Y is
// recomputed) -- goes to viewGrad[slot] for pass 2.  Camera gradients are
// summed per warp in fixed point (order-independent) with one atomic each.
template <int DEG>
__global__ void __launch_bounds__(128, GS_CHAIN_MIN_BLOCKS) k_chain_view(ChainArgs a) {
  constexpr int K = DEG > 0 ? (DEG + 1) * (DEG + 1) - 1 : 0;
  const uint32_t sb = blockIdx.x / (uint32_t)a.V;
  const int v = (int)(blockIdx.x - sb * (uint32_t)a.V);
  const uint32_t pos = sb * blockDim.x + threadIdx.x;
  const uint32_t cnt = a.visCount[v];
  if (sb * blockDim.x >= cnt) return;  // the whole block is past the list (uniform)
  const bool have = pos < cnt;
  const uint32_t i = have ? a.visList[(size_t)v * a.n + pos] : 0u;
  const int lane = threadIdx.x & 31;
  // the block's camera in shared memory (read once, not re-fetched from
  // global memory around every store); every thread issues its own loads
  // before the barrier that publishes it
  __shared__ DevCam s_cam;
  copy_cams(&s_cam, a.cams + v, 1);
  const size_t slot = (size_t)v * a.n + i;
  int4 q0 = make_int4(0, 0, 0, 0), q1 = q0, q2 = q0;
  float P[16];
  if (have) {
    const int4* G4 = reinterpret_cast<const int4*>(a.gradP + slot * GP_STRIDE);
    q0 = G4[0]; q1 = G4[1]; q2 = G4[2];
    const float4* P4 = reinterpret_cast<const float4*>(a.params + (size_t)i * STRIDE);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const float4 t = __ldg(P4 + k);
      P[4 * k] = t.x; P[4 * k + 1] = t.y; P[4 * k + 2] = t.z; P[4 * k + 3] = t.w;
    }
  }
  __syncthreads();
  const DevCam& c = s_cam;
  CamGrad7 cg = {{0.0f, 0.0f, 0.0f}, {0.0f, 0.0f, 0.0f}, 0.0f};
  if (have) {
    {
      int4* G4 = reinterpret_cast<int4*>(a.gradP + slot * GP_STRIDE);
      G4[0] = make_int4(0, 0, 0, 0);
      G4[1] = make_int4(0, 0, 0, 0);
      G4[2] = make_int4(0, 0, 0, 0);
      const int32_t qi[10] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w, q2.x, q2.y};
      float gp[10];
#pragma unroll
      for (int k = 0; k < 10; ++k) gp[k] = (float)qi[k] / ((k >= 2 && k <= 4) ? FIXEDC : FIXED);
      float gF[16];
#pragma unroll
      for (int k = 0; k < 16; ++k) gF[k] = 0.0f;
      float dRGB[3] = {0.0f, 0.0f, 0.0f}, vd[3] = {0.0f, 0.0f, 0.0f}, Y[15];
      int aK = 0;
      const Geom g = computeGeom(c, P);
      if (g.ok) {
        // undo the render pass's conic normalisation (shaders.js:735-744)
        const float cva = g.va + 0.3f, cvc = g.vc + 0.3f;
        const float cmid = 0.5f * (cva + cvc);
        const float lmax = cmid + sqrtf(fmaxf(cmid * cmid - (cva * cvc - g.vb * g.vb), 0.0f));
        const float cden = 1.0f + lmax;
        gp[2] = gp[2] * cden; gp[3] = gp[3] * cden; gp[4] = gp[4] * cden;
        const float* shp = K > 0 ? a.sh + (size_t)i * 3 * K : nullptr;
        chainOne<DEG>(c, P, g, gp, shp, a.anisoReg, gF, dRGB, Y, vd, aK, cg);
      }
      float4* o = reinterpret_cast<float4*>(a.viewGrad + slot * VIEWGRAD_STRIDE);
      o[0] = make_float4(gF[0], gF[1], gF[2], gF[3]);
      o[1] = make_float4(gF[4], gF[5], gF[6], gF[7]);
      o[2] = make_float4(gF[8], gF[9], gF[10], gF[11]);
      o[3] = make_float4(gF[12], gF[13], dRGB[0], dRGB[1]);
      o[4] = make_float4(dRGB[2], vd[0], vd[1], vd[2]);
    }
  }
  // camera gradients: warp sums of the fixed-point values, one atomic each
  if (c.train) {
    const float cv[7] = {cg.w[0], cg.w[1], cg.w[2], cg.t[0], cg.t[1], cg.t[2], cg.logf};
#pragma unroll
    for (int k = 0; k < 7; ++k) {
      const uint32_t r = __reduce_add_sync(0xFFFFFFFFu, (uint32_t)fixq(cv[k], FIXCAM));
      if (lane == 0 && r) {
        const uint32_t idx = k < 6 ? c.camIdx * 8u + (uint32_t)k : c.ncams * 8u;
        atomicAdd(&a.gradCam[idx], (int32_t)r);
      }
    }
  }
}

// Pass 2: one thread per splat sums its views' gradients in view order from
// zero (views where the splat was not visible add +0, which changes no sum,
// and are skipped), then the block updates its 128 splats with Adam and
// SH-Adam through shared memory, one float per thread per step, so every
// global access is coalesced.
template <int DEG>
__global__ void __launch_bounds__(128) k_chain_adam(ChainArgs a) {
  constexpr int K = DEG > 0 ? (DEG + 1) * (DEG + 1) - 1 : 0;
  constexpr int SHN = 3 * K;
  constexpr int GROW = 17;                 // padded rows: conflict-free column writes
  constexpr int SROW = SHN > 0 ? SHN + 1 : 1;
  constexpr uint32_t SHD = SHN > 0 ? SHN : 1;  // divisor (the SH loops are empty when SHN = 0)
  __shared__ float s_g[128 * GROW];
  __shared__ float s_sh[SHN > 0 ? 128 * SROW : 1];
  __shared__ float s_opa[128];
  const uint32_t i0 = blockIdx.x * blockDim.x;
  const uint32_t i = i0 + threadIdx.x;
  const int t = threadIdx.x;
  {
    float gFa[14];
    float shA[SHN > 0 ? SHN : 1];
#pragma unroll
    for (int k = 0; k < 14; ++k) gFa[k] = 0.0f;
#pragma unroll
    for (int k = 0; k < SHN; ++k) shA[k] = 0.0f;
    if (i < a.n) {
      for (int v = 0; v < a.V; ++v) {
        const size_t slot = (size_t)v * a.n + i;
        if (a.rect[slot].x == 0xFFFFFFFFu) continue;
        const float4* q = reinterpret_cast<const float4*>(a.viewGrad + slot * VIEWGRAD_STRIDE);
        const float4 q0 = q[0], q1 = q[1], q2 = q[2], q3 = q[3];
        const float gF[14] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w,
                              q2.x, q2.y, q2.z, q2.w, q3.x, q3.y};
#pragma unroll
        for (int k = 0; k < 14; ++k) gFa[k] = gFa[k] + gF[k];
        if (K > 0) {
          const float4 q4 = q[4];
          const float dRGB[3] = {q3.z, q3.w, q4.x};
          const float vd[3] = {q4.y, q4.z, q4.w};
          float Y[15];
          shBasis<DEG>(vd, Y);
          const int aK = shActiveK(a.cams[v], K);
#pragma unroll
          for (int ch = 0; ch < 3; ++ch)
#pragma unroll
            for (int k = 0; k < K; ++k)
              shA[ch * K + k] = shA[ch * K + k] + (k < aK ? dRGB[ch] * Y[k] : 0.0f);
        }
      }
    }
#pragma unroll
    for (int k = 0; k < 14; ++k) s_g[t * GROW + k] = gFa[k];
    s_g[t * GROW + 14] = 0.0f;
    s_g[t * GROW + 15] = 0.0f;
    if (a.doAdam && i < a.n) {  // the opacity slot's gradient as Adam sees it (shaders.js:990-995)
      const float sg = sigm(a.params[(size_t)i * STRIDE + 13]);
      s_opa[t] = adam_g(gFa[13]) + a.hp->reg * sg * (1.0f - sg);
    }
#pragma unroll
    for (int k = 0; k < SHN; ++k) s_sh[t * SROW + k] = shA[k];
  }
  __syncthreads();
  const uint32_t cnt = a.n - i0 < 128u ? a.n - i0 : 128u;  // splats of this block
  const uint32_t nP = cnt * STRIDE, nS = cnt * SHN;
  const size_t pBase = (size_t)i0 * STRIDE, sBase = (size_t)i0 * SHN;
  if (a.gradF) {
    for (uint32_t e = t; e < nP; e += 128) a.gradF[pBase + e] = s_g[(e / STRIDE) * GROW + e % STRIDE];
    for (uint32_t e = t; e < nS; e += 128) a.shGrad[sBase + e] = s_sh[(e / SHD) * SROW + e % SHD];
  }
  if (!a.doAdam) return;
  const AdamK k = adam_k(*a.hp);
  // U elements per thread in flight: loads first, then the updates.  At SH
  // degree 3 the summing phase above already sets the register count (96),
  // so six in flight cost no occupancy there (measured -10 % on the pass;
  // ptxas spills 4 bytes); at the lower degrees more than four would.
  constexpr uint32_t U = DEG == 3 ? 6 : 4;
  {
    float* __restrict__ Pp = a.params + pBase;
    float* __restrict__ Pm = a.m + pBase;
    float* __restrict__ Pv = a.v + pBase;
    const int slot = t % STRIDE;  // 128 is a multiple of the stride: one slot per thread
    const AdamSlot as = adam_slot(*a.hp, slot);
    if (as.live) {  // a zero learning rate leaves the slot as it is (shaders.js:986)
      for (uint32_t e0 = t; e0 < nP; e0 += 128 * U) {
        float p[U], m[U], vv[U];
#pragma unroll
        for (uint32_t u = 0; u < U; ++u) {
          const uint32_t e = e0 + 128 * u;
          if (e < nP) { p[u] = Pp[e]; m[u] = Pm[e]; vv[u] = Pv[e]; }
        }
#pragma unroll
        for (uint32_t u = 0; u < U; ++u) {
          const uint32_t e = e0 + 128 * u;
          if (e < nP) {
            const uint32_t row = e / STRIDE;
            const float g = as.opa ? s_opa[row] : adam_g(s_g[row * GROW + slot]);
            float pn = adam_update(k, as.lr, p[u], g, m[u], vv[u]);
            if (as.clamp) pn = clampf(pn, as.lo, as.hi);
            Pp[e] = pn; Pm[e] = m[u]; Pv[e] = vv[u];
          }
        }
      }
    }
  }
  if (SHN > 0) {
    float* __restrict__ Sw = a.sh + sBase;
    float* __restrict__ Sm = a.shM + sBase;
    float* __restrict__ Sv = a.shV + sBase;
    for (uint32_t e0 = t; e0 < nS; e0 += 128 * U) {
      float w[U], m[U], vv[U];
#pragma unroll
      for (uint32_t u = 0; u < U; ++u) {
        const uint32_t e = e0 + 128 * u;
        if (e < nS) { w[u] = Sw[e]; m[u] = Sm[e]; vv[u] = Sv[e]; }
      }
#pragma unroll
      for (uint32_t u = 0; u < U; ++u) {
        const uint32_t e = e0 + 128 * u;
        if (e < nS) {
          const float g = adam_g(s_sh[(e / SHD) * SROW + e % SHD]);
          const float wn = adam_update(k, k.shLr, w[u], g, m[u], vv[u]);
          Sm[e] = m[u];
          Sv[e] = vv[u];
          Sw[e] = wn;
        }
      }
    }
  }
}

void launch_chain_adam(const ChainArgs& a, int deg, cudaStream_t s) {
  const unsigned blocks = (a.n + 127) / 128;
  if (blocks == 0) return;
  const unsigned g1 = blocks * (unsigned)a.V;
  const unsigned bpv = (a.n + 255) / 256;
  k_visible_list<<<bpv * (unsigned)a.V, 256, 0, s>>>(a, bpv);
  switch (deg) {
    case 0: k_chain_view<0><<<g1, 128, 0, s>>>(a); k_chain_adam<0><<<blocks, 128, 0, s>>>(a); break;
    case 1: k_chain_view<1><<<g1, 128, 0, s>>>(a); k_chain_adam<1><<<blocks, 128, 0, s>>>(a); break;
    case 2: k_chain_view<2><<<g1, 128, 0, s>>>(a); k_chain_adam<2><<<blocks, 128, 0, s>>>(a); break;
    default: k_chain_view<3><<<g1, 128, 0, s>>>(a); k_chain_adam<3><<<blocks, 128, 0, s>>>(a); break;
  }
}

}  // namespace gs
