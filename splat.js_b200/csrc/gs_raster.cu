// gs_raster.cu -- the tiled rasteriser: forward composite, loss + stats and
// the back-to-front backward of the reference's render pass
// (shaders.js:544-700), over a shared (view, tile) work queue.
//
// One CTA works on one TILE x TILE tile at a time (TILE = 8, 16 or 32; one
// thread per pixel; each warp covers an 8x4 block of the tile).  Splat
// records of the tile's sorted entries are staged in shared memory BATCH at
// a time.  The fused train tile at TILE = 16 runs k_raster_px2 instead: two
// pixels per thread on sm_100's packed FP32 instructions, each warp covering
// an 8x8 block, with results identical to k_raster's.
//
// Forward: front-to-back compositing; the block leaves the tile when
// __syncthreads_count (a block-wide ballot) finds every pixel saturated.  In
// the fused train kernel each warp also records, per entry, whether any of
// its pixels composited it (a ballot bit in shared memory): on dense scenes
// only about a fifth of warp-entries composite anything.
// Backward: each warp walks only the entries its bits mark, back to front
// (without bits -- backward from saved state, or entries past the bit
// capacity -- a warp-uniform test against the splat's conservative radius,
// rad + 1 px, skips entries that cannot reach the warp's 8x4 pixels);
// each pixel recovers the transmittance in front of a splat from the final
// one (Tb = Ta / (1 - alpha)) -- or, in the stored-state variant, reads the
// value the forward saved.  The ten gradient contributions of each pixel are
// truncated to i32 fixed point (the reference's i32(clamp(v*16384, +-1e9)))
// and summed exactly: a warp REDUX per slot, a shared-memory add per
// (entry, slot) across the tile's warps, and one global atomic per (splat,
// slot, tile).  Integer sums commute, so results are bit-identical in any
// order -- the deterministic mode is the only mode.
//
// Control flow is warp-uniform (votes); per-lane work runs predicated, so
// no divergent branch needs a reconvergence scaffold in the hot loops.
// The per-pair arithmetic is the canonical FP32 sequence the CPU
// restatement performs.  The 2^14 fixed-point scale is folded into upstream
// factors (gC, hence galpha, which is accumulated from the scaled gC):
// scaling by a power of two is exact, so every truncated integer equals the
// one the unfolded sequence produces.  The
// +-1e9 clamp is skipped when a warp's scaled galpha is below 1e7: the
// conic normaliser bounds every slot by 80 |galpha * 2^14| (slots 7-9 by
// |gC * 2^14|), so the clamp cannot change a value then.
#include "gs_common.cuh"
#include "gs_kernels.h"

namespace gs {

constexpr int MASKW = 128;        // ballot-bit words per warp: entries 0..4095 of a tile
constexpr uint32_t FULL = 0xFFFFFFFFu;

// e = max(fma(fma(cA/2, dx, cB*dy), dx, ((cC/2)*dy)*dy), 0); r0 = (mx, my, cA/2, cB)
__device__ __forceinline__ float pairExponent(const float4& r0, float hC, float dx, float dy) {
  const float u = __fmaf_rn(r0.z, dx, r0.w * dy);
  return fmaxf(__fmaf_rn(u, dx, (hC * dy) * dy), 0.0f);
}

// trunc(clamp(x, -1e9, 1e9)) for an already scaled value
__device__ __forceinline__ int32_t fix_scaled(float x) { return __float2int_rz(fminf(fmaxf(x, -1.0e9f), 1.0e9f)); }


// Which of the tile's 8x4 warp blocks can the splat reach?  Bit w = warp w
// (block row w / (TILE/8), column w % (TILE/8)).  For each 4-row band, the
// splat's pixels lie within |dx - kA dy| <= sqrt(p - q dmin^2) (cull
// parameters (p, q, kA) from the projection; dmin = the band's smallest |dy|),
// an x interval checked against each block of the band.  Slack covers this
// FP32 evaluation, so a cleared bit means no pixel of the block can pass the
// rasteriser's cutoffs: skipping the entry there changes nothing.
template <int TILE>
__device__ __forceinline__ uint32_t warp_block_mask(const float4 cq, float mx, float my, int tx, int ty) {
  constexpr int NB = TILE / 4, WPR = TILE / 8;
  constexpr uint32_t ALL = NB * WPR >= 32 ? 0xFFFFFFFFu : (1u << (NB * WPR)) - 1u;
  if (!(cq.x < 3.0e38f)) return ALL;
  uint32_t m = 0;
#pragma unroll
  for (int b = 0; b < NB; ++b) {
    const float Y0 = ((float)(ty * TILE + 4 * b) + 0.5f) - my;
    float xl, xr;
    if (!bandInterval(cq, Y0, Y0 + 3.0f, xl, xr)) continue;
#pragma unroll
    for (int wb = 0; wb < WPR; ++wb) {
      const float bx0 = ((float)(tx * TILE + 8 * wb) + 0.5f) - mx;
      if (bx0 + 7.0f >= xl && bx0 <= xr) m |= 1u << (b * WPR + wb);
    }
  }
  return m;
}

#ifndef GS_RASTER16_MIN_BLOCKS
#define GS_RASTER16_MIN_BLOCKS 5  // resident 16x16-tile blocks per SM the register allocation must allow
#endif
// TILE x TILE pixels per CTA, one per thread; warps cover 8x4 blocks.
template <int TILE, int BATCH, bool FWD, bool BWD, bool STORED>
__global__ void __launch_bounds__(TILE * TILE, TILE == 16 ? GS_RASTER16_MIN_BLOCKS : TILE == 8 ? 16 : 1) k_raster(RasterArgs a) {
  constexpr int RT = TILE;
  constexpr int RTHREADS = TILE * TILE;
  constexpr int NW = RTHREADS / 32;  // warps
  constexpr int WPR = TILE / 8;      // 8-wide warp blocks per tile row
  constexpr bool MASKS = FWD && BWD;
  static_assert(BATCH % 32 == 0, "batches hold whole ballot words");
  __shared__ RenderRec s_rec[BATCH];
  __shared__ uint32_t s_id[BATCH];
  __shared__ int32_t s_acc[BWD ? BATCH * 10 : 1];
  __shared__ uint32_t s_mask[MASKS ? NW * MASKW : 1];
  __shared__ uint32_t s_live[FWD ? NW : 1][BATCH / 32];  // per warp: staged entries its block can reach
  __shared__ uint32_t s_item;
  __shared__ uint32_t s_redu[NW][5];
  __shared__ uint32_t s_endmax[NW];
  __shared__ __align__(16) int32_t s_stage[BWD ? NW : 1][12];  // per warp: the 10 sums of one entry

  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int lx = (wid % WPR) * 8 + (lane & 7);
  const int ly = (wid / WPR) * 4 + (lane >> 3);
  const float E_CUT = a.eCut, A_MIN = a.aMin;
  uint32_t* wmask = s_mask + (MASKS ? wid * MASKW : 0);

  if (BWD)
    for (int k = tid; k < BATCH * 10; k += RTHREADS) s_acc[k] = 0;

  for (uint32_t iter = 0;; ++iter) {
    // ---- next work item (a global tile of the batch) ----
    if (tid == 0) s_item = a.workCounter ? atomicAdd(a.workCounter, 1u) : (iter == 0 ? blockIdx.x : 0xFFFFFFFFu);
    __syncthreads();
    const uint32_t item = s_item;
    __syncthreads();
    if (item >= a.totalTiles) break;
    const uint32_t gt = a.workOrder ? a.workOrder[item] : item;
    int v = 0;
    while (v + 1 < a.V && a.cams[v + 1].tileBase <= gt) ++v;
    const DevCam& c = a.cams[v];
    const uint32_t t = gt - c.tileBase;
    const int tx = (int)(t % (uint32_t)c.tilesX), ty = (int)(t / (uint32_t)c.tilesX);
    const int x = tx * RT + lx, y = ty * RT + ly;
    const bool inside = x < c.W && y < c.H;
    const float px = (float)x + 0.5f, py = (float)y + 0.5f;
    const uint2 rg = a.ranges[gt];
    const uint32_t s = rg.x, e = rg.y;
    const size_t pix = (size_t)c.pixBase + (size_t)y * c.W + x;
    const RenderRec* recs = a.recs + (size_t)v * a.n;
    const float4* cullRecs = a.cullRecs + (size_t)v * a.n;

    float T = 1.0f;
    float C0 = 0.0f, C1 = 0.0f, C2 = 0.0f;
    uint32_t cnt = e - s;  // one past the last processed entry (relative)
    if (FWD) {
      bool done = !inside;
      if (MASKS) {
        for (int k = lane; k < MASKW; k += 32) wmask[k] = 0u;
        __syncwarp();
      }
      for (uint32_t base = s; base < e; base += BATCH) {
        if (__syncthreads_count(!done) == 0) break;
        const uint32_t nb = min((uint32_t)BATCH, e - base);
        // stage the batch; each staging thread also finds which warp blocks
        // its entry can reach, and a ballot per warp block transposes that
        // into one word per 32 entries
        for (uint32_t kb = 0; kb < (uint32_t)BATCH; kb += RTHREADS) {
          const uint32_t k = kb + tid;
          uint32_t m = 0;
          if (k < nb) {
            const uint32_t id = a.ids[base + k];
            s_id[k] = id;
            const RenderRec rec = recs[id];
            s_rec[k] = rec;
            m = warp_block_mask<TILE>(cullRecs[id], rec.r0.x, rec.r0.y, tx, ty);
          }
          const uint32_t word = (kb >> 5) + (uint32_t)wid;
#pragma unroll
          for (int w = 0; w < NW; ++w) {
            const uint32_t bw = __ballot_sync(FULL, (m >> w) & 1u);
            if (lane == 0 && word < (uint32_t)(BATCH / 32)) s_live[w][word] = bw;
          }
        }
        __syncthreads();
        if (!__all_sync(FULL, done)) {
          const uint32_t rbase = base - s;
          for (uint32_t jw = 0; jw < nb; jw += 32) {  // one ballot word per 32 entries
            uint32_t live = s_live[wid][jw >> 5];  // entries this warp's block can reach
            uint32_t bits = 0;
            while (live) {
              const uint32_t jj = (uint32_t)__ffs(live) - 1u;
              live &= live - 1u;
              const RenderRec& rr = s_rec[jw + jj];
              const float4 r0 = rr.r0;
              const float4 r1 = rr.r1;
              const float dx = px - r0.x, dy = py - r0.y;
              const float ee = pairExponent(r0, r1.x, dx, dy);
              const bool c1 = !done && ee <= E_CUT;
              // warp-uniform branch; the body runs predicated per lane (lanes
              // outside the cutoff see a clamped exponent and are masked off)
              if (__any_sync(FULL, c1)) {
                const float araw = r1.y * gexp(-fminf(ee, 80.0f));
                const float alpha = fminf(0.99f, araw);
                const bool c2 = c1 && alpha >= A_MIN;
                if (STORED && c2) a.tStore[(size_t)(base + jw + jj) * RTHREADS + tid] = T;
                const float ta = T * alpha;
                const float cb = rr.r2.x;
                if (c2) {
                  C0 = __fmaf_rn(ta, r1.z, C0);
                  C1 = __fmaf_rn(ta, r1.w, C1);
                  C2 = __fmaf_rn(ta, cb, C2);
                  T = T * (1.0f - alpha);
                  if (T < 1e-4f) { done = true; cnt = rbase + jw + jj + 1; }
                }
                if (MASKS) bits |= (__ballot_sync(FULL, c2) != 0u ? 1u : 0u) << jj;
              }
            }
            if (MASKS) {
              const uint32_t w = (rbase + jw) >> 5;
              if (lane == 0 && w < MASKW) wmask[w] = bits;
            }
            if (__all_sync(FULL, done)) break;
          }
        }
        __syncthreads();
      }
      C0 = C0 + T * c.bg[0];
      C1 = C1 + T * c.bg[1];
      C2 = C2 + T * c.bg[2];
      if (inside) {
        if (a.outImg) a.outImg[pix] = make_float4(C0, C1, C2, 1.0f - T);
        if (a.finalT) a.finalT[pix] = T;
        if (a.endIdx) a.endIdx[pix] = cnt;
      }
    } else if (inside) {
      const float4 o = a.outImg[pix];
      C0 = o.x; C1 = o.y; C2 = o.z;
      T = a.finalT[pix];
      cnt = a.endIdx[pix];
    }

    if (BWD) {
      // ---- loss (shaders.js:589-618) ----
      bool lossOk = false;
      float g16_0 = 0.0f, g16_1 = 0.0f, g16_2 = 0.0f;  // gC * 2^14
      uint32_t st0 = 0, st1 = 0, st2 = 0;
      int32_t cg6 = 0, cg7 = 0;
      if (inside) {
        const uint32_t pi = (uint32_t)(y * c.W + x);
        const uint32_t packed = a.targets[(size_t)c.offset + pi];
        if ((packed >> 24) != 0u) {
          lossOk = true;
          const float t0 = (float)(packed & 0xFFu) / 255.0f;
          const float t1 = (float)((packed >> 8) & 0xFFu) / 255.0f;
          const float t2 = (float)((packed >> 16) & 0xFFu) / 255.0f;
          st2 = 1u;
          const float gain = c.gain;
          const float er0 = (gain * C0 + c.bias) - t0;
          const float er1 = (gain * C1 + c.bias) - t1;
          const float er2 = (gain * C2 + c.bias) - t2;
          st0 = u32sat((er0 * er0 + er1 * er1 + er2 * er2) * 16.0f + dither(pi));
          const float D2 = 9.0000000000000003e-04f;  // f32(0.03 * 0.03), a WGSL const-expression
          const float rt0 = sqrtf(er0 * er0 + D2), rt1 = sqrtf(er1 * er1 + D2), rt2 = sqrtf(er2 * er2 + D2);
          const float eg0 = er0 / rt0, eg1 = er1 / rt1, eg2 = er2 / rt2;
          g16_0 = (gain * eg0) * FIXED; g16_1 = (gain * eg1) * FIXED; g16_2 = (gain * eg2) * FIXED;
          const float lossv = (rt0 + rt1 + rt2) - 8.9999999999999997e-02f;  // f32(3 * 0.03)
          st1 = u32sat(lossv * 32768.0f);
          cg6 = fixq((eg0 * C0 + eg1 * C1 + eg2 * C2) * gain, FIXCAM);
          cg7 = fixq(eg0 + eg1 + eg2, FIXCAM);
        }
      }
      // slots 7-9 stay within +-1e9 without clamping when |gC * 2^14| < 9e8
      const bool pixFast = fabsf(g16_0) < 9.0e8f && fabsf(g16_1) < 9.0e8f && fabsf(g16_2) < 9.0e8f;
      // block sums of the per-pixel stats (wrapping u32 / i32, as the
      // reference's atomics) and the largest end index of the tile
      const uint32_t myEnd = lossOk ? cnt : 0u;
      {
        const uint32_t r0 = __reduce_add_sync(FULL, st0);
        const uint32_t r1 = __reduce_add_sync(FULL, st1);
        const uint32_t r2 = __reduce_add_sync(FULL, st2);
        const uint32_t r3 = __reduce_add_sync(FULL, (uint32_t)cg6);
        const uint32_t r4 = __reduce_add_sync(FULL, (uint32_t)cg7);
        const uint32_t mx = __reduce_max_sync(FULL, myEnd);
        if (lane == 0) {
          s_redu[wid][0] = r0; s_redu[wid][1] = r1; s_redu[wid][2] = r2;
          s_redu[wid][3] = r3; s_redu[wid][4] = r4;
          s_endmax[wid] = mx;
        }
      }
      __syncthreads();
      if (tid < 5) {
        uint32_t sum = 0;
        for (int w = 0; w < NW; ++w) sum += s_redu[w][tid];
        if (sum) {
          if (tid < 3) atomicAdd(&a.stats[tid], sum);
          else atomicAdd(&a.gradCam[c.camIdx * 8u + 3u + (uint32_t)tid], (int32_t)sum);
        }
      }
      uint32_t endMax = 0;
#pragma unroll
      for (int w = 0; w < NW; ++w) endMax = max(endMax, s_endmax[w]);
      // ---- backward (shaders.js:632-700) ----
      float S0 = c.bg[0] * T, S1 = c.bg[1] * T, S2 = c.bg[2] * T;
      float Ta = T;
      int32_t* gradP = a.gradP + (size_t)v * a.n * GP_STRIDE;
      for (uint32_t hi = endMax; hi > 0;) {
        const uint32_t lo = hi > (uint32_t)BATCH ? hi - BATCH : 0u;
        const uint32_t nb = hi - lo;
        __syncthreads();
        for (uint32_t k = tid; k < nb; k += RTHREADS) {
          const uint32_t id = a.ids[s + lo + k];
          s_id[k] = id;
          s_rec[k] = recs[id];
        }
        __syncthreads();
        // this warp's entries in [lo, hi), back to front, one ballot word at a time
        for (int32_t w = (int32_t)((hi - 1) >> 5); w >= (int32_t)(lo >> 5); --w) {
          const uint32_t wb = (uint32_t)w << 5;
          const bool haveBits = MASKS && (uint32_t)w < (uint32_t)MASKW;
          uint32_t word = haveBits ? wmask[w] : FULL;
          if (wb + 32u > hi) word &= FULL >> (wb + 32u - hi);
          if (wb < lo) word &= FULL << (lo - wb);
          while (word) {
            const uint32_t bit = 31u - (uint32_t)__clz(word);
            word &= ~(1u << bit);
            const uint32_t j = wb + bit;
            const RenderRec& rr = s_rec[j - lo];
            const float4 r0 = rr.r0;
            const float4 r1 = rr.r1;
            const float4 r2 = rr.r2;
            // Straight-line body, predicated per lane: lanes that do not
            // composite this entry (past their end, outside a cutoff) compute
            // on a clamped exponent and have their contribution zeroed
            // through galpha and aT, and keep S and Ta.  Compositing lanes
            // perform exactly the canonical sequence.
            const float dx = px - r0.x, dy = py - r0.y;
            const float ee = pairExponent(r0, r1.x, dx, dy);
            const float G = gexp(-fminf(ee, 80.0f));
            const float araw = r1.y * G;
            const float alpha = fminf(0.99f, araw);
            const bool c2 = j < myEnd && ee <= E_CUT && alpha >= A_MIN;
            if (!__any_sync(FULL, c2)) continue;
            const float inv = rcp_unit(1.0f - alpha);  // 1 - alpha in [0.01, 1]: IEEE 1/x exactly
            const float Tb = STORED ? (c2 ? a.tStore[(size_t)(s + j) * RTHREADS + tid] : 0.0f) : Ta * inv;
            const float aT = c2 ? alpha * Tb : 0.0f;
            const float g0 = __fmaf_rn(r1.z, Tb, -(S0 * inv));
            const float g1 = __fmaf_rn(r1.w, Tb, -(S1 * inv));
            const float g2 = __fmaf_rn(r2.x, Tb, -(S2 * inv));
            // galpha * 2^14, accumulated from gC * 2^14
            const float gal16 = c2 && !(araw > 0.99f) ? __fmaf_rn(g16_2, g2, __fmaf_rn(g16_1, g1, g16_0 * g0)) : 0.0f;
            const float ga16 = gal16 * araw;
            const float cA = r0.z + r0.z, cC = r1.x + r1.x;  // exact doubling of the stored halves
            const float gq16 = ga16 * r2.z;  // r2.z = -cnorm / 2
            const float gqx16 = gq16 * dx;
            float xs[10];
            xs[0] = ga16 * __fmaf_rn(cA, dx, r0.w * dy);
            xs[1] = ga16 * __fmaf_rn(r0.w, dx, cC * dy);
            xs[2] = gqx16 * dx;
            xs[3] = (gqx16 * dy) * 2.0f;
            xs[4] = (gq16 * dy) * dy;
            xs[5] = (gal16 * r2.y) * G;
            xs[6] = ga16 * r2.w;  // r2.w = 1 - opacity
            xs[7] = g16_0 * aT;
            xs[8] = g16_1 * aT;
            xs[9] = g16_2 * aT;
            uint32_t rsum[10];
            if (__all_sync(FULL, fabsf(gal16) < 1.0e7f && pixFast)) {
#pragma unroll
              for (int k = 0; k < 10; ++k) rsum[k] = __reduce_add_sync(FULL, (uint32_t)__float2int_rz(xs[k]));
            } else {
#pragma unroll
              for (int k = 0; k < 10; ++k) rsum[k] = __reduce_add_sync(FULL, (uint32_t)fix_scaled(xs[k]));
            }
            if (c2) {
              S0 = __fmaf_rn(r1.z, aT, S0);
              S1 = __fmaf_rn(r1.w, aT, S1);
              S2 = __fmaf_rn(r2.x, aT, S2);
              Ta = Tb;
            }
            // lane 0 stages the 10 warp sums; lanes 0-9 add one each
            if (lane == 0) {
              int4* st = reinterpret_cast<int4*>(s_stage[wid]);
              st[0] = make_int4((int)rsum[0], (int)rsum[1], (int)rsum[2], (int)rsum[3]);
              st[1] = make_int4((int)rsum[4], (int)rsum[5], (int)rsum[6], (int)rsum[7]);
              reinterpret_cast<int2*>(s_stage[wid])[4] = make_int2((int)rsum[8], (int)rsum[9]);
            }
            __syncwarp();
            if (lane < 10) atomicAdd(&s_acc[(j - lo) * 10 + (uint32_t)lane], s_stage[wid][lane]);
            __syncwarp();
          }
        }
        __syncthreads();
        for (uint32_t k = tid; k < nb * 10; k += RTHREADS) {
          const int32_t val = s_acc[k];
          if (val) {
            const uint32_t jl = k / 10, slot = k - jl * 10;
            atomicAdd(&gradP[(size_t)s_id[jl] * GP_STRIDE + slot], val);
            s_acc[k] = 0;
          }
        }
        hi = lo;
      }
    }
    __syncthreads();
  }
}

// Which 8x8 warp blocks of a 16x16 tile can the splat reach?  Bit w = warp w
// (block row w / 2, column w % 2); the same band test as warp_block_mask on
// 8-row bands.
__device__ __forceinline__ uint32_t warp_block_mask8(const float4 cq, float mx, float my, int tx, int ty) {
  if (!(cq.x < 3.0e38f)) return 0xFu;
  uint32_t m = 0;
#pragma unroll
  for (int b = 0; b < 2; ++b) {
    const float Y0 = ((float)(ty * 16 + 8 * b) + 0.5f) - my;
    float xl, xr;
    if (!bandIntervalMask(cq, Y0, Y0 + 7.0f, xl, xr)) continue;
#pragma unroll
    for (int wb = 0; wb < 2; ++wb) {
      const float bx0 = ((float)(tx * 16 + 8 * wb) + 0.5f) - mx;
      if (bx0 + 7.0f >= xl && bx0 <= xr) m |= 1u << (b * 2 + wb);
    }
  }
  return m;
}

// e = max(fma(fma(cA/2, dx, cB*dy), dx, ((cC/2)*dy)*dy), 0) for two pixels
// that share dx; Bdy returns cB*dy.
__device__ __forceinline__ float2 pairExponent2(const float4& r0, float hC, float dx, float2 dy, float2& Bdy) {
  Bdy = __fmul2_rn(bc2(r0.w), dy);
  const float2 u = __ffma2_rn(bc2(r0.z), bc2(dx), Bdy);
  const float2 e = __ffma2_rn(u, bc2(dx), __fmul2_rn(__fmul2_rn(bc2(hC), dy), dy));
  return make_float2(fmaxf(e.x, 0.0f), fmaxf(e.y, 0.0f));
}

__device__ __forceinline__ void cp_async_rec(RenderRec* dst, const RenderRec* src) {
  cp_async16(&dst->r0, &src->r0);
  cp_async16(&dst->r1, &src->r1);
  cp_async16(&dst->r2, &src->r2);
}

#ifndef GS_RASTER_PX2_MIN_BLOCKS
#define GS_RASTER_PX2_MIN_BLOCKS 8  // resident 128-thread blocks per SM the register allocation must allow
#endif
// Fused train tile (forward + loss + backward) on a 16x16 tile with two
// pixels per thread: 128 threads, each warp covering an 8x8 block; lane l
// holds pixels (l % 8, l / 8) and (l % 8, l / 8 + 4) of its block, which
// share dx.  Every per-pixel operation runs on the pair with one packed
// instruction (or twice, for comparisons, selects and conversions) and
// performs the canonical sequence of k_raster on each pixel; the per-entry
// work (record loads, votes, the ten warp reductions and the shared-memory
// adds) is shared by 64 pixels instead of 32.  Results are bit-identical to
// k_raster<16, BATCH, true, true, false>: the same entries reach every pixel
// (an 8x8 block skips an entry only when neither of its 8x4 halves can use
// it), and integer sums do not depend on how pixels are grouped.
//
// Staging: each batch of BATCH entries is copied from global to shared
// memory with cp.async (16-byte copies, no register round trip); the entry
// ids of the next batch are loaded into registers while the current one is
// processed, so a batch's staging waits for one gather, not for the id load
// and then the gather.  Each thread copies its own entries (k = tid,
// tid + 128) and, in the forward, computes their warp-block masks from its
// own completed copies before the batch's barrier.  (Double-buffering the
// records as well -- the next batch copied while the current one is
// processed -- needs twice the record storage, which at 256 entries drops
// the block from 8 to 5 resident per SM; measured, it did not pay.)
template <int BATCH>
__global__ void __launch_bounds__(128, GS_RASTER_PX2_MIN_BLOCKS) k_raster_px2(RasterArgs a) {
  constexpr int NT = 128, NW = 4;
  constexpr int PER = BATCH >= NT ? BATCH / NT : 1;  // entries a thread stages per batch
  static_assert(BATCH % 32 == 0, "batches hold whole ballot words");
  static_assert(BATCH <= 2 * NT, "two staged entries per thread");
  __shared__ RenderRec s_rec[BATCH];
  // the forward's cull parameters and the backward's per-entry sums share storage
  constexpr int ACC_WORDS = BATCH * 10, CULL_WORDS = BATCH * 4;
  __shared__ __align__(16) int32_t s_accu[ACC_WORDS > CULL_WORDS ? ACC_WORDS : CULL_WORDS];
  int32_t* s_acc = s_accu;
  float4* s_cull = reinterpret_cast<float4*>(s_accu);
  __shared__ uint32_t s_id[BATCH];
  __shared__ uint32_t s_mask[NW * MASKW];
  __shared__ uint32_t s_live[NW][BATCH / 32];
  __shared__ uint32_t s_item;
  __shared__ uint32_t s_redu[NW][5];
  __shared__ uint32_t s_endmax[NW];
  __shared__ __align__(16) int32_t s_stage[NW][12];

  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int lx = (wid & 1) * 8 + (lane & 7);
  const int ly = (wid >> 1) * 8 + (lane >> 3);  // pixel a; pixel b is 4 rows below
  const float E_CUT = a.eCut, A_MIN = a.aMin;
  uint32_t* wmask = s_mask + wid * MASKW;

  for (uint32_t iter = 0;; ++iter) {
    if (tid == 0) s_item = a.workCounter ? atomicAdd(a.workCounter, 1u) : (iter == 0 ? blockIdx.x : 0xFFFFFFFFu);
    __syncthreads();
    const uint32_t item = s_item;
    __syncthreads();
    if (item >= a.totalTiles) break;
    const uint32_t gt = a.workOrder ? a.workOrder[item] : item;
    int v = 0;
    while (v + 1 < a.V && a.cams[v + 1].tileBase <= gt) ++v;
    const DevCam& c = a.cams[v];
    const uint32_t t = gt - c.tileBase;
    const int tx = (int)(t % (uint32_t)c.tilesX), ty = (int)(t / (uint32_t)c.tilesX);
    const int x = tx * 16 + lx, ya = ty * 16 + ly, yb = ya + 4;
    const bool inA = x < c.W && ya < c.H, inB = x < c.W && yb < c.H;
    const float px = (float)x + 0.5f;
    const float2 py = make_float2((float)ya + 0.5f, (float)yb + 0.5f);
    const uint2 rg = a.ranges[gt];
    const uint32_t s = rg.x, e = rg.y;
    const size_t pixA = (size_t)c.pixBase + (size_t)ya * c.W + x;
    const size_t pixB = pixA + (size_t)4 * c.W;
    const RenderRec* recs = a.recs + (size_t)v * a.n;
    const float4* cullRecs = a.cullRecs + (size_t)v * a.n;

    // ---- forward ----
    float2 T = bc2(1.0f);
    float2 C0 = bc2(0.0f), C1 = bc2(0.0f), C2 = bc2(0.0f);
    uint32_t cntA = e - s, cntB = e - s;
    bool doneA = !inA, doneB = !inB;
    for (int k = lane; k < MASKW; k += 32) wmask[k] = 0u;
    __syncwarp();
    // ids of entries [from, to) that this thread stages (k = tid, tid + 128)
    uint32_t pf[PER];
    auto load_ids = [&](uint32_t from, uint32_t to) {
#pragma unroll
      for (int u = 0; u < PER; ++u) {
        const uint32_t k = (uint32_t)(u * NT + tid);
        pf[u] = k < (uint32_t)BATCH && from + k < to ? a.ids[from + k] : 0u;
      }
    };
    load_ids(s, e);
    for (uint32_t base = s; base < e; base += BATCH) {
      // every warp has finished the previous batch: its buffers may be overwritten
      if (__syncthreads_count(!(doneA && doneB)) == 0) break;
      const uint32_t nb = min((uint32_t)BATCH, e - base);
#pragma unroll
      for (int u = 0; u < PER; ++u) {
        const uint32_t k = (uint32_t)(u * NT + tid);
        if (k < nb) {
          cp_async_rec(&s_rec[k], recs + pf[u]);
          cp_async16(&s_cull[k], cullRecs + pf[u]);
        }
      }
      cp_async_commit();
      load_ids(base + BATCH, e);  // the next batch's ids load while this one is processed
      cp_async_wait<0>();         // this thread's copies have landed
#pragma unroll
      for (int u = 0; u < (BATCH + NT - 1) / NT; ++u) {
        const uint32_t kb = (uint32_t)(u * NT);
        const uint32_t k = kb + tid;
        uint32_t m = 0;
        if (k < nb) m = warp_block_mask8(s_cull[k], s_rec[k].r0.x, s_rec[k].r0.y, tx, ty);
        const uint32_t word = (kb >> 5) + (uint32_t)wid;
#pragma unroll
        for (int w = 0; w < NW; ++w) {
          const uint32_t bw = __ballot_sync(FULL, (m >> w) & 1u);
          if (lane == 0 && word < (uint32_t)(BATCH / 32)) s_live[w][word] = bw;
        }
      }
      __syncthreads();
      if (!__all_sync(FULL, doneA && doneB)) {
        const uint32_t rbase = base - s;
        for (uint32_t jw = 0; jw < nb; jw += 32) {
          uint32_t live = s_live[wid][jw >> 5];
          uint32_t bits = 0;
          while (live) {
            const uint32_t jj = (uint32_t)__ffs(live) - 1u;
            live &= live - 1u;
            const RenderRec& rr = s_rec[jw + jj];
            const float4 r0 = rr.r0;
            const float4 r1 = rr.r1;
            const float dx = px - r0.x;
            const float2 dy = __fadd2_rn(py, bc2(-r0.y));
            float2 Bdy;
            const float2 ee = pairExponent2(r0, r1.x, dx, dy, Bdy);
            const bool c1a = !doneA && ee.x <= E_CUT, c1b = !doneB && ee.y <= E_CUT;
            if (__any_sync(FULL, c1a || c1b)) {
              const float2 G = gexp2(make_float2(-fminf(ee.x, 80.0f), -fminf(ee.y, 80.0f)));
              const float2 araw = __fmul2_rn(bc2(r1.y), G);
              const float2 alpha = make_float2(fminf(0.99f, araw.x), fminf(0.99f, araw.y));
              const bool c2a = c1a && alpha.x >= A_MIN, c2b = c1b && alpha.y >= A_MIN;
              // a pixel that does not composite sees alpha 0: C and T stay exactly as they are
              const float2 am = make_float2(c2a ? alpha.x : 0.0f, c2b ? alpha.y : 0.0f);
              const float2 ta = __fmul2_rn(T, am);
              C0 = __ffma2_rn(ta, bc2(r1.z), C0);
              C1 = __ffma2_rn(ta, bc2(r1.w), C1);
              C2 = __ffma2_rn(ta, bc2(rr.r2.x), C2);
              T = __fmul2_rn(T, __fadd2_rn(bc2(1.0f), make_float2(-am.x, -am.y)));
              if (c2a && T.x < 1e-4f) { doneA = true; cntA = rbase + jw + jj + 1; }
              if (c2b && T.y < 1e-4f) { doneB = true; cntB = rbase + jw + jj + 1; }
              bits |= (__ballot_sync(FULL, c2a || c2b) != 0u ? 1u : 0u) << jj;
            }
          }
          const uint32_t w = (rbase + jw) >> 5;
          if (lane == 0 && w < MASKW) wmask[w] = bits;
          if (__all_sync(FULL, doneA && doneB)) break;
        }
      }
    }
    C0 = __fadd2_rn(C0, __fmul2_rn(T, bc2(c.bg[0])));
    C1 = __fadd2_rn(C1, __fmul2_rn(T, bc2(c.bg[1])));
    C2 = __fadd2_rn(C2, __fmul2_rn(T, bc2(c.bg[2])));
    if (inA) {
      if (a.outImg) a.outImg[pixA] = make_float4(C0.x, C1.x, C2.x, 1.0f - T.x);
      if (a.finalT) a.finalT[pixA] = T.x;
      if (a.endIdx) a.endIdx[pixA] = cntA;
    }
    if (inB) {
      if (a.outImg) a.outImg[pixB] = make_float4(C0.y, C1.y, C2.y, 1.0f - T.y);
      if (a.finalT) a.finalT[pixB] = T.y;
      if (a.endIdx) a.endIdx[pixB] = cntB;
    }

    // ---- loss (shaders.js:589-618), per pixel ----
    float2 g16_0 = bc2(0.0f), g16_1 = bc2(0.0f), g16_2 = bc2(0.0f);
    uint32_t st0 = 0, st1 = 0, st2 = 0, cg6 = 0, cg7 = 0;
    uint32_t myEndA = 0, myEndB = 0;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const bool in = h ? inB : inA;
      if (!in) continue;
      const int yy = h ? yb : ya;
      const uint32_t pi = (uint32_t)(yy * c.W + x);
      const uint32_t packed = a.targets[(size_t)c.offset + pi];
      if ((packed >> 24) == 0u) continue;
      const float Cx = h ? C0.y : C0.x, Cy = h ? C1.y : C1.x, Cz = h ? C2.y : C2.x;
      const float t0 = (float)(packed & 0xFFu) / 255.0f;
      const float t1 = (float)((packed >> 8) & 0xFFu) / 255.0f;
      const float t2 = (float)((packed >> 16) & 0xFFu) / 255.0f;
      st2 += 1u;
      const float gain = c.gain;
      const float er0 = (gain * Cx + c.bias) - t0;
      const float er1 = (gain * Cy + c.bias) - t1;
      const float er2 = (gain * Cz + c.bias) - t2;
      st0 += u32sat((er0 * er0 + er1 * er1 + er2 * er2) * 16.0f + dither(pi));
      const float D2 = 9.0000000000000003e-04f;  // f32(0.03 * 0.03), a WGSL const-expression
      const float rt0 = sqrtf(er0 * er0 + D2), rt1 = sqrtf(er1 * er1 + D2), rt2 = sqrtf(er2 * er2 + D2);
      const float eg0 = er0 / rt0, eg1 = er1 / rt1, eg2 = er2 / rt2;
      const float q0 = gain * eg0, q1 = gain * eg1, q2 = gain * eg2;
      const float lossv = (rt0 + rt1 + rt2) - 8.9999999999999997e-02f;  // f32(3 * 0.03)
      st1 += u32sat(lossv * 32768.0f);
      cg6 += (uint32_t)fixq((eg0 * Cx + eg1 * Cy + eg2 * Cz) * gain, FIXCAM);
      cg7 += (uint32_t)fixq(eg0 + eg1 + eg2, FIXCAM);
      if (h) {
        g16_0.y = q0 * FIXED; g16_1.y = q1 * FIXED; g16_2.y = q2 * FIXED;
        myEndB = cntB;
      } else {
        g16_0.x = q0 * FIXED; g16_1.x = q1 * FIXED; g16_2.x = q2 * FIXED;
        myEndA = cntA;
      }
    }
    // slots 7-9 stay within +-1e9 without clamping when |gC * 2^14| < 9e8
    const bool pixFast = fabsf(g16_0.x) < 9.0e8f && fabsf(g16_1.x) < 9.0e8f && fabsf(g16_2.x) < 9.0e8f &&
                         fabsf(g16_0.y) < 9.0e8f && fabsf(g16_1.y) < 9.0e8f && fabsf(g16_2.y) < 9.0e8f;
    {
      const uint32_t r0 = __reduce_add_sync(FULL, st0);
      const uint32_t r1 = __reduce_add_sync(FULL, st1);
      const uint32_t r2 = __reduce_add_sync(FULL, st2);
      const uint32_t r3 = __reduce_add_sync(FULL, cg6);
      const uint32_t r4 = __reduce_add_sync(FULL, cg7);
      const uint32_t mx = __reduce_max_sync(FULL, max(myEndA, myEndB));
      if (lane == 0) {
        s_redu[wid][0] = r0; s_redu[wid][1] = r1; s_redu[wid][2] = r2;
        s_redu[wid][3] = r3; s_redu[wid][4] = r4;
        s_endmax[wid] = mx;
      }
    }
    __syncthreads();
    if (tid < 5) {
      uint32_t sum = 0;
      for (int w = 0; w < NW; ++w) sum += s_redu[w][tid];
      if (sum) {
        if (tid < 3) atomicAdd(&a.stats[tid], sum);
        else atomicAdd(&a.gradCam[c.camIdx * 8u + 3u + (uint32_t)tid], (int32_t)sum);
      }
    }
    uint32_t endMax = 0;
#pragma unroll
    for (int w = 0; w < NW; ++w) endMax = max(endMax, s_endmax[w]);
    // the forward's cull parameters shared storage with the per-entry sums:
    // every reader of them has passed the barrier above
    for (int k = tid; k < BATCH * 10; k += NT) s_acc[k] = 0;

    // ---- backward (shaders.js:632-700) ----
    float2 S0 = __fmul2_rn(bc2(c.bg[0]), T), S1 = __fmul2_rn(bc2(c.bg[1]), T), S2 = __fmul2_rn(bc2(c.bg[2]), T);
    float2 Ta = T;
    int32_t* gradP = a.gradP + (size_t)v * a.n * GP_STRIDE;
    // batches run back to front: [lo, hi) with hi = endMax, then hi = lo;
    // each batch's ids are loaded while the batch before it is processed
    auto lo_of = [](uint32_t hi) { return hi > (uint32_t)BATCH ? hi - (uint32_t)BATCH : 0u; };
    if (endMax > 0) load_ids(s + lo_of(endMax), s + endMax);
    for (uint32_t hi = endMax; hi > 0;) {
      const uint32_t lo = lo_of(hi);
      const uint32_t nb = hi - lo;
      __syncthreads();  // the previous batch's processing and flush are over
#pragma unroll
      for (int u = 0; u < PER; ++u) {
        const uint32_t k = (uint32_t)(u * NT + tid);
        if (k < nb) {
          s_id[k] = pf[u];
          cp_async_rec(&s_rec[k], recs + pf[u]);
        }
      }
      cp_async_commit();
      if (lo > 0) load_ids(s + lo_of(lo), s + lo);
      cp_async_wait<0>();
      __syncthreads();
      {
        const RenderRec* srec = s_rec;
        for (int32_t w = (int32_t)((hi - 1) >> 5); w >= (int32_t)(lo >> 5); --w) {
          const uint32_t wb = (uint32_t)w << 5;
          uint32_t word = (uint32_t)w < (uint32_t)MASKW ? wmask[w] : FULL;
          if (wb + 32u > hi) word &= FULL >> (wb + 32u - hi);
          if (wb < lo) word &= FULL << (lo - wb);
          while (word) {
            const uint32_t bit = 31u - (uint32_t)__clz(word);
            word &= ~(1u << bit);
            const uint32_t j = wb + bit;
            const RenderRec& rr = srec[j - lo];
            const float4 r0 = rr.r0;
            const float4 r1 = rr.r1;
            const float4 r2 = rr.r2;
            const float dx = px - r0.x;
            const float2 dy = __fadd2_rn(py, bc2(-r0.y));
            float2 Bdy;
            const float2 ee = pairExponent2(r0, r1.x, dx, dy, Bdy);
            const float2 G = gexp2(make_float2(-fminf(ee.x, 80.0f), -fminf(ee.y, 80.0f)));
            const float2 araw = __fmul2_rn(bc2(r1.y), G);
            const float2 alpha = make_float2(fminf(0.99f, araw.x), fminf(0.99f, araw.y));
            const bool c2a = j < myEndA && ee.x <= E_CUT && alpha.x >= A_MIN;
            const bool c2b = j < myEndB && ee.y <= E_CUT && alpha.y >= A_MIN;
            const uint32_t balA = __ballot_sync(FULL, c2a), balB = __ballot_sync(FULL, c2b);
            if ((balA | balB) == 0u) continue;
            const float2 inv = rcp_unit2(__fadd2_rn(bc2(1.0f), make_float2(-alpha.x, -alpha.y)));
            const float2 Tb = __fmul2_rn(Ta, inv);
            const float2 at = __fmul2_rn(alpha, Tb);
            const float2 aT = make_float2(c2a ? at.x : 0.0f, c2b ? at.y : 0.0f);
            const float2 g0 = __ffma2_rn(bc2(r1.z), Tb, __fmul2_rn(make_float2(-S0.x, -S0.y), inv));
            const float2 g1 = __ffma2_rn(bc2(r1.w), Tb, __fmul2_rn(make_float2(-S1.x, -S1.y), inv));
            const float2 g2 = __ffma2_rn(bc2(r2.x), Tb, __fmul2_rn(make_float2(-S2.x, -S2.y), inv));
            // galpha * 2^14, accumulated from gC * 2^14
            const float2 gal16r = __ffma2_rn(g16_2, g2, __ffma2_rn(g16_1, g1, __fmul2_rn(g16_0, g0)));
            const float2 gal16 = make_float2(c2a && !(araw.x > 0.99f) ? gal16r.x : 0.0f,
                                             c2b && !(araw.y > 0.99f) ? gal16r.y : 0.0f);
            const float2 ga16 = __fmul2_rn(gal16, araw);
            const float cA = r0.z + r0.z, cC = r1.x + r1.x;
            const float2 gq16 = __fmul2_rn(ga16, bc2(r2.z));
            const float2 gqx16 = __fmul2_rn(gq16, bc2(dx));
            float2 xs[10];
            xs[0] = __fmul2_rn(ga16, __ffma2_rn(bc2(cA), bc2(dx), Bdy));
            xs[1] = __fmul2_rn(ga16, __ffma2_rn(bc2(r0.w), bc2(dx), __fmul2_rn(bc2(cC), dy)));
            xs[2] = __fmul2_rn(gqx16, bc2(dx));
            xs[3] = __fmul2_rn(__fmul2_rn(gqx16, dy), bc2(2.0f));
            xs[4] = __fmul2_rn(__fmul2_rn(gq16, dy), dy);
            xs[5] = __fmul2_rn(__fmul2_rn(gal16, bc2(r2.y)), G);
            xs[6] = __fmul2_rn(ga16, bc2(r2.w));
            xs[7] = __fmul2_rn(g16_0, aT);
            xs[8] = __fmul2_rn(g16_1, aT);
            xs[9] = __fmul2_rn(g16_2, aT);
            uint32_t rsum[10];
            if (!__all_sync(FULL, fabsf(gal16.x) < 1.0e7f && fabsf(gal16.y) < 1.0e7f && pixFast)) {
#pragma unroll
              for (int k = 0; k < 10; ++k)
                xs[k] = make_float2(fminf(fmaxf(xs[k].x, -1.0e9f), 1.0e9f), fminf(fmaxf(xs[k].y, -1.0e9f), 1.0e9f));
            }
            // a half of the block with no compositing pixel has every value 0
            if (balA != 0u && balB != 0u) {
#pragma unroll
              for (int k = 0; k < 10; ++k)
                rsum[k] = __reduce_add_sync(FULL, (uint32_t)__float2int_rz(xs[k].x) + (uint32_t)__float2int_rz(xs[k].y));
            } else if (balA != 0u) {
#pragma unroll
              for (int k = 0; k < 10; ++k) rsum[k] = __reduce_add_sync(FULL, (uint32_t)__float2int_rz(xs[k].x));
            } else {
#pragma unroll
              for (int k = 0; k < 10; ++k) rsum[k] = __reduce_add_sync(FULL, (uint32_t)__float2int_rz(xs[k].y));
            }
            // a pixel that does not composite has aT = 0: S stays exactly as it is
            S0 = __ffma2_rn(bc2(r1.z), aT, S0);
            S1 = __ffma2_rn(bc2(r1.w), aT, S1);
            S2 = __ffma2_rn(bc2(r2.x), aT, S2);
            Ta = make_float2(c2a ? Tb.x : Ta.x, c2b ? Tb.y : Ta.y);
            if (lane == 0) {
              int4* st = reinterpret_cast<int4*>(s_stage[wid]);
              st[0] = make_int4((int)rsum[0], (int)rsum[1], (int)rsum[2], (int)rsum[3]);
              st[1] = make_int4((int)rsum[4], (int)rsum[5], (int)rsum[6], (int)rsum[7]);
              reinterpret_cast<int2*>(s_stage[wid])[4] = make_int2((int)rsum[8], (int)rsum[9]);
            }
            __syncwarp();
            if (lane < 10) atomicAdd(&s_acc[(j - lo) * 10 + (uint32_t)lane], s_stage[wid][lane]);
            __syncwarp();
          }
        }
        __syncthreads();
        for (uint32_t k = tid; k < nb * 10; k += NT) {
          const int32_t val = s_acc[k];
          if (val) {
            const uint32_t jl = k / 10, slot = k - jl * 10;
            atomicAdd(&gradP[(size_t)s_id[jl] * GP_STRIDE + slot], val);
            s_acc[k] = 0;
          }
        }
      }
      hi = lo;
    }
    __syncthreads();
  }
}

template <int TILE, int BATCH, bool FWD, bool BWD, bool STORED>
static void launch_one(const RasterArgs& a, unsigned grid, cudaStream_t s) {
  if constexpr (TILE == 16 && FWD && BWD && !STORED) k_raster_px2<BATCH><<<grid, 128, 0, s>>>(a);
  else k_raster<TILE, BATCH, FWD, BWD, STORED><<<grid, TILE * TILE, 0, s>>>(a);
}

template <int TILE, int BATCH>
static void launch_mode(const RasterArgs& a, int mode, bool stored, unsigned grid, cudaStream_t s) {
  // mode: 1 = forward, 2 = backward from saved state, 3 = fused train tile
  if (mode == 1) launch_one<TILE, BATCH, true, false, false>(a, grid, s);
  else if (mode == 2) {
    if (stored) launch_one<TILE, BATCH, false, true, true>(a, grid, s);
    else launch_one<TILE, BATCH, false, true, false>(a, grid, s);
  } else {
    if (stored) launch_one<TILE, BATCH, true, true, true>(a, grid, s);
    else launch_one<TILE, BATCH, true, true, false>(a, grid, s);
  }
}

template <int TILE>
static void launch_tile(const RasterArgs& a, int mode, bool stored, int batchDepth, unsigned grid, cudaStream_t s) {
  switch (batchDepth) {
    case 64: launch_mode<TILE, 64>(a, mode, stored, grid, s); break;
    case 128: launch_mode<TILE, 128>(a, mode, stored, grid, s); break;
    default: launch_mode<TILE, 256>(a, mode, stored, grid, s); break;
  }
}

void launch_raster(const RasterArgs& a, int mode, bool stored, int tile, int batchDepth, unsigned grid,
                   cudaStream_t s) {
  if (grid == 0) return;
  if (tile == 8) launch_tile<8>(a, mode, stored, batchDepth, grid, s);
  else if (tile == 32) launch_tile<32>(a, mode, stored, batchDepth, grid, s);
  else launch_tile<16>(a, mode, stored, batchDepth, grid, s);
}

// The kernel launch_one runs for (TILE, depth, forward-only or fused train
// tile, not stored) and its block size.
template <int TILE, int BATCH>
static const void* kernel_of_depth(bool fwdOnly, int& threads) {
  threads = TILE * TILE;
  if (fwdOnly) return (const void*)k_raster<TILE, BATCH, true, false, false>;
  if (TILE == 16) {
    threads = 128;
    return (const void*)k_raster_px2<BATCH>;
  }
  return (const void*)k_raster<TILE, BATCH, true, true, false>;
}

template <int TILE>
static const void* kernel_of(int batchDepth, int mode, int& threads) {
  const bool fwdOnly = mode == 1;
  switch (batchDepth) {
    case 64: return kernel_of_depth<TILE, 64>(fwdOnly, threads);
    case 128: return kernel_of_depth<TILE, 128>(fwdOnly, threads);
    default: return kernel_of_depth<TILE, 256>(fwdOnly, threads);
  }
}

int raster_blocks_per_sm(int tile, int batchDepth, int mode) {
  int threads = 0;
  const void* f = tile == 8 ? kernel_of<8>(batchDepth, mode, threads)
                            : tile == 32 ? kernel_of<32>(batchDepth, mode, threads)
                                         : kernel_of<16>(batchDepth, mode, threads);
  int perSm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, f, threads, 0);
  return perSm < 1 ? 1 : perSm;
}

// Work order for the persistent queue: global tiles by descending entry
// count (bucketed by log2), so the heaviest tiles start first.  Three small
// grid-wide kernels: bucket sizes, their exclusive scan, and the placement of
// every tile at its bucket's cursor.  The order inside a bucket follows the
// cursor atomics; no result depends on it (tiles write disjoint pixels and
// integer gradient sums), only the schedule does.
__device__ __forceinline__ uint32_t tile_bucket(const uint2* ranges, uint32_t t) {
  return (uint32_t)__clz(ranges[t].y - ranges[t].x);  // 32: empty, 0: longest
}

// one atomic per bucket per warp (whole warps step through the tiles; lanes
// past the end use bucket 64)
__global__ void __launch_bounds__(1024) k_work_count(const uint2* ranges, uint32_t totalTiles, uint32_t* counts) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = t < totalTiles;
  const uint32_t b = valid ? tile_bucket(ranges, t) : 64u;
  const uint32_t peers = __match_any_sync(0xFFFFFFFFu, b);
  if (valid && lane == (uint32_t)(__ffs(peers) - 1)) atomicAdd(&counts[b], (uint32_t)__popc(peers));
}

// cursors = exclusive scan of the 33 bucket sizes; the sizes are cleared for
// the next use
__global__ void k_work_scan(uint32_t* counts, uint32_t* cursors) {
  if (threadIdx.x == 0) {
    uint32_t acc = 0;
    for (int b = 0; b < 33; ++b) {
      cursors[b] = acc;
      acc += counts[b];
      counts[b] = 0u;
    }
  }
}

__global__ void __launch_bounds__(1024) k_work_place(const uint2* ranges, uint32_t totalTiles, uint32_t* cursors,
                                                     uint32_t* order) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = t < totalTiles;
  const uint32_t b = valid ? tile_bucket(ranges, t) : 64u;
  const uint32_t peers = __match_any_sync(0xFFFFFFFFu, b);
  const uint32_t lead = (uint32_t)(__ffs(peers) - 1);
  uint32_t base = 0;
  if (valid && lane == lead) base = atomicAdd(&cursors[b], (uint32_t)__popc(peers));
  base = __shfl_sync(0xFFFFFFFFu, base, lead);
  if (valid) order[base + (uint32_t)__popc(peers & ((1u << lane) - 1u))] = t;
}

// scratch: 66 words, the first 33 zero before the first call (each call
// leaves them zero)
void launch_work_order(const uint2* ranges, uint32_t totalTiles, uint32_t* order, uint32_t* scratch,
                       cudaStream_t s) {
  if (totalTiles == 0) return;
  const unsigned blocks = (totalTiles + 1023) / 1024;
  k_work_count<<<blocks, 1024, 0, s>>>(ranges, totalTiles, scratch);
  k_work_scan<<<1, 32, 0, s>>>(scratch, scratch + 33);
  k_work_place<<<blocks, 1024, 0, s>>>(ranges, totalTiles, scratch + 33, order);
}

}  // namespace gs
