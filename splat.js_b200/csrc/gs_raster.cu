// gs_raster.cu -- the tiled rasteriser: forward composite, loss + stats and
// the back-to-front backward of the reference's render pass
// (shaders.js:544-700), over a shared (view, tile) work queue.
//
// One CTA works on one 16x16 tile at a time (256 threads, one pixel each;
// warp w covers an 8x4 block of the tile so a splat's footprint tends to
// cover whole warps).  Splat records of the tile's sorted entries are staged
// in shared memory BATCH at a time.
//
// Forward: front-to-back compositing; the block leaves the tile as soon as
// __syncthreads_count (a block-wide ballot) finds every pixel saturated.
// Backward: each pixel walks its entries back to front from its own end
// index, recovering the transmittance in front of each splat from the final
// one (Tb = Ta / (1 - alpha)) -- or, in the stored-state variant, reading
// the value the forward saved.  Every pixel's ten gradient contributions are
// truncated to i32 fixed point (the reference's i32(clamp(v*16384, +-1e9)))
// and summed exactly: a warp REDUX per slot, a shared-memory add per
// (entry, slot) across the tile's warps, and one global atomic per (splat,
// slot, tile).  Integer sums commute, so the result is bit-identical in any
// order -- the deterministic mode is the only mode.
//
// The per-pair arithmetic is the canonical FP32 sequence (fused where
// written fmaf) that the CPU restatement performs too.
#include "gs_common.cuh"
#include "gs_kernels.h"

namespace gs {

constexpr int RT = 16;           // tile edge (pixels)
constexpr int RTHREADS = RT * RT;

struct PixelCtx {
  float px, py;
};

__device__ __forceinline__ float pairExponent(const float4& r0, float cC, float dx, float dy) {
  // e = max(fma(0.5, fma(cA*dx, dx, (cC*dy)*dy), (cB*dx)*dy), 0)
  const float q = __fmaf_rn(r0.z * dx, dx, (cC * dy) * dy);
  return fmaxf(__fmaf_rn(0.5f, q, (r0.w * dx) * dy), 0.0f);
}

template <int BATCH, bool FWD, bool BWD, bool STORED>
__global__ void __launch_bounds__(RTHREADS) k_raster(RasterArgs a) {
  __shared__ RenderRec s_rec[BATCH];
  __shared__ uint32_t s_id[BATCH];
  __shared__ int32_t s_acc[BWD ? BATCH * 10 : 1];
  __shared__ uint32_t s_item;
  __shared__ uint32_t s_redu[8][5];
  __shared__ uint32_t s_endmax[8];

  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int lx = ((wid & 1) << 3) | (lane & 7);
  const int ly = ((wid >> 1) << 2) | (lane >> 3);
  const float E_CUT = a.eCut, A_MIN = a.aMin;

  if (BWD)
    for (int k = tid; k < BATCH * 10; k += RTHREADS) s_acc[k] = 0;

  for (uint32_t iter = 0;; ++iter) {
    // ---- next work item (a global tile of the batch) ----
    if (a.workCounter) {
      if (tid == 0) s_item = atomicAdd(a.workCounter, 1u);
      __syncthreads();
    } else {
      if (tid == 0) s_item = iter == 0 ? blockIdx.x : 0xFFFFFFFFu;
      __syncthreads();
    }
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

    float T = 1.0f;
    float C0 = 0.0f, C1 = 0.0f, C2 = 0.0f;
    uint32_t cnt = 0;
    if (FWD) {
      bool done = !inside;
      for (uint32_t base = s; base < e; base += BATCH) {
        if (__syncthreads_count(!done) == 0) break;
        const uint32_t nb = min((uint32_t)BATCH, e - base);
        for (uint32_t k = tid; k < nb; k += RTHREADS) {
          const uint32_t id = a.ids[base + k];
          s_id[k] = id;
          s_rec[k] = recs[id];
        }
        __syncthreads();
        if (!done) {
          for (uint32_t j = 0; j < nb; ++j) {
            const float4 r0 = s_rec[j].r0;
            const float4 r1 = s_rec[j].r1;
            const float dx = px - r0.x, dy = py - r0.y;
            const float ee = pairExponent(r0, r1.x, dx, dy);
            cnt = base - s + j + 1;
            if (ee > E_CUT) continue;
            const float araw = r1.y * gexp(-ee);
            const float alpha = fminf(0.99f, araw);
            if (alpha < A_MIN) continue;
            if (STORED) a.tStore[(size_t)(base + j) * RTHREADS + tid] = T;
            const float ta = T * alpha;
            const float cb = s_rec[j].r2.x;
            C0 = __fmaf_rn(ta, r1.z, C0);
            C1 = __fmaf_rn(ta, r1.w, C1);
            C2 = __fmaf_rn(ta, cb, C2);
            T = T * (1.0f - alpha);
            if (T < 1e-4f) { done = true; break; }
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
      float gC0 = 0.0f, gC1 = 0.0f, gC2 = 0.0f;
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
          gC0 = gain * eg0; gC1 = gain * eg1; gC2 = gain * eg2;
          const float lossv = (rt0 + rt1 + rt2) - 8.9999999999999997e-02f;  // f32(3 * 0.03)
          st1 = u32sat(lossv * 32768.0f);
          cg6 = fixq((eg0 * C0 + eg1 * C1 + eg2 * C2) * gain, FIXCAM);
          cg7 = fixq(eg0 + eg1 + eg2, FIXCAM);
        }
      }
      // block sums of the per-pixel stats (wrapping u32 / i32, as the
      // reference's atomics) and the largest end index of the tile
      const uint32_t myEnd = lossOk ? cnt : 0u;
      {
        const uint32_t r0 = __reduce_add_sync(0xFFFFFFFFu, st0);
        const uint32_t r1 = __reduce_add_sync(0xFFFFFFFFu, st1);
        const uint32_t r2 = __reduce_add_sync(0xFFFFFFFFu, st2);
        const uint32_t r3 = __reduce_add_sync(0xFFFFFFFFu, (uint32_t)cg6);
        const uint32_t r4 = __reduce_add_sync(0xFFFFFFFFu, (uint32_t)cg7);
        const uint32_t mx = __reduce_max_sync(0xFFFFFFFFu, myEnd);
        if (lane == 0) {
          s_redu[wid][0] = r0; s_redu[wid][1] = r1; s_redu[wid][2] = r2;
          s_redu[wid][3] = r3; s_redu[wid][4] = r4;
          s_endmax[wid] = mx;
        }
      }
      __syncthreads();
      if (tid < 5) {
        uint32_t sum = 0;
        for (int w = 0; w < 8; ++w) sum += s_redu[w][tid];
        if (sum) {
          if (tid < 3) atomicAdd(&a.stats[tid], sum);
          else atomicAdd(&a.gradCam[c.camIdx * 8u + 3u + (uint32_t)tid], (int32_t)sum);
        }
      }
      uint32_t endMax = 0;
#pragma unroll
      for (int w = 0; w < 8; ++w) endMax = max(endMax, s_endmax[w]);
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
        for (uint32_t jj = nb; jj > 0; --jj) {
          const uint32_t j = lo + jj - 1;  // relative entry index
          int32_t q[10];
#pragma unroll
          for (int k = 0; k < 10; ++k) q[k] = 0;
          bool contrib = false;
          if (j < myEnd) {
            const float4 r0 = s_rec[jj - 1].r0;
            const float4 r1 = s_rec[jj - 1].r1;
            const float dx = px - r0.x, dy = py - r0.y;
            const float ee = pairExponent(r0, r1.x, dx, dy);
            if (ee <= E_CUT) {
              const float G = gexp(-ee);
              const float araw = r1.y * G;
              const float alpha = fminf(0.99f, araw);
              if (alpha >= A_MIN) {
                contrib = true;
                const float4 r2 = s_rec[jj - 1].r2;
                const float inv = __frcp_rn(1.0f - alpha);
                const float Tb = STORED ? a.tStore[(size_t)(s + j) * RTHREADS + tid] : Ta * inv;
                const float aT = alpha * Tb;
                const float g0 = __fmaf_rn(r1.z, Tb, -(S0 * inv));
                const float g1 = __fmaf_rn(r1.w, Tb, -(S1 * inv));
                const float g2 = __fmaf_rn(r2.x, Tb, -(S2 * inv));
                float galpha = __fmaf_rn(gC2, g2, __fmaf_rn(gC1, g1, gC0 * g0));
                if (araw > 0.99f) galpha = 0.0f;
                const float ga = galpha * araw;
                q[0] = fixq(ga * __fmaf_rn(r0.z, dx, r0.w * dy), FIXED);
                q[1] = fixq(ga * __fmaf_rn(r0.w, dx, r1.x * dy), FIXED);
                const float gq = ga * (-0.5f * r2.z);
                const float gqx = gq * dx;
                q[2] = fixq(gqx * dx, FIXEDC);
                q[3] = fixq((gqx * dy) * 2.0f, FIXEDC);
                q[4] = fixq((gq * dy) * dy, FIXEDC);
                q[5] = fixq((galpha * r2.y) * G, FIXED);
                q[6] = fixq(ga * (1.0f - r2.y), FIXED);
                q[7] = fixq(gC0 * aT, FIXED);
                q[8] = fixq(gC1 * aT, FIXED);
                q[9] = fixq(gC2 * aT, FIXED);
                S0 = __fmaf_rn(r1.z, aT, S0);
                S1 = __fmaf_rn(r1.w, aT, S1);
                S2 = __fmaf_rn(r2.x, aT, S2);
                Ta = Tb;
              }
            }
          }
          if (__any_sync(0xFFFFFFFFu, contrib)) {
            uint32_t r[10];
#pragma unroll
            for (int k = 0; k < 10; ++k) r[k] = __reduce_add_sync(0xFFFFFFFFu, (uint32_t)q[k]);
            uint32_t mine = r[0];
#pragma unroll
            for (int k = 1; k < 10; ++k) mine = lane == k ? r[k] : mine;
            if (lane < 10 && mine) atomicAdd(&s_acc[(jj - 1) * 10 + lane], (int32_t)mine);
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

template <int BATCH, bool FWD, bool BWD, bool STORED>
static void launch_one(const RasterArgs& a, unsigned grid, cudaStream_t s) {
  k_raster<BATCH, FWD, BWD, STORED><<<grid, RTHREADS, 0, s>>>(a);
}

template <int BATCH>
static void launch_batch(const RasterArgs& a, int mode, bool stored, unsigned grid, cudaStream_t s) {
  // mode: 1 = forward, 2 = backward from saved state, 3 = fused train tile
  if (mode == 1) {
    if (stored) launch_one<BATCH, true, false, true>(a, grid, s);
    else launch_one<BATCH, true, false, false>(a, grid, s);
  } else if (mode == 2) {
    if (stored) launch_one<BATCH, false, true, true>(a, grid, s);
    else launch_one<BATCH, false, true, false>(a, grid, s);
  } else {
    if (stored) launch_one<BATCH, true, true, true>(a, grid, s);
    else launch_one<BATCH, true, true, false>(a, grid, s);
  }
}

void launch_raster(const RasterArgs& a, int mode, bool stored, int batchDepth, unsigned grid, cudaStream_t s) {
  if (grid == 0) return;
  switch (batchDepth) {
    case 32: launch_batch<32>(a, mode, stored, grid, s); break;
    case 64: launch_batch<64>(a, mode, stored, grid, s); break;
    case 128: launch_batch<128>(a, mode, stored, grid, s); break;
    default: launch_batch<256>(a, mode, stored, grid, s); break;
  }
}

int raster_blocks_per_sm(int batchDepth, int mode) {
  int perSm = 0;
  const void* f;
  switch (batchDepth) {
    case 32: f = mode == 1 ? (const void*)k_raster<32, true, false, false> : (const void*)k_raster<32, true, true, false>; break;
    case 64: f = mode == 1 ? (const void*)k_raster<64, true, false, false> : (const void*)k_raster<64, true, true, false>; break;
    case 128: f = mode == 1 ? (const void*)k_raster<128, true, false, false> : (const void*)k_raster<128, true, true, false>; break;
    default: f = mode == 1 ? (const void*)k_raster<256, true, false, false> : (const void*)k_raster<256, true, true, false>; break;
  }
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, f, RTHREADS, 0);
  return perSm < 1 ? 1 : perSm;
}

// Work order for the persistent queue: global tiles by descending entry
// count (bucketed by log2), so the heaviest tiles start first.
__global__ void __launch_bounds__(1024) k_work_order(const uint2* ranges, uint32_t totalTiles, uint32_t* order) {
  __shared__ uint32_t s_hist[33];
  __shared__ uint32_t s_off[33];
  if (threadIdx.x < 33) s_hist[threadIdx.x] = 0;
  __syncthreads();
  for (uint32_t t = threadIdx.x; t < totalTiles; t += blockDim.x) {
    const uint32_t len = ranges[t].y - ranges[t].x;
    const uint32_t b = 32u - __clz(len);  // 0 for empty tiles
    atomicAdd(&s_hist[32 - b], 1u);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t acc = 0;
    for (int b = 0; b < 33; ++b) { s_off[b] = acc; acc += s_hist[b]; }
  }
  __syncthreads();
  for (uint32_t t = threadIdx.x; t < totalTiles; t += blockDim.x) {
    const uint32_t len = ranges[t].y - ranges[t].x;
    const uint32_t b = 32u - __clz(len);
    order[atomicAdd(&s_off[32 - b], 1u)] = t;
  }
}

void launch_work_order(const uint2* ranges, uint32_t totalTiles, uint32_t* order, cudaStream_t s) {
  k_work_order<<<1, 1024, 0, s>>>(ranges, totalTiles, order);
}

}  // namespace gs
