// gs_project.cu -- pass 1 of the training step: projection + SH colour
// (shaders.js:228-315), for every (view, splat) of a batch in one launch.
//
// Outputs per (view, splat):
//   RenderRec  the 48-byte record the rasteriser stages (mean, conic,
//              opacity*comp, colour, opacity, conic normaliser, depth);
//   rect       tile bounds packed as {x0 | y0<<16, x1 | y1<<16}, or
//              {0xFFFFFFFF, 0} when culled (the reference's visible flag);
// and four atomic adds into the view's tile "difference grid", whose 2D
// prefix sum is the reference's per-tile count tileCnt (shaders.js:303-313)
// at 4 atomics per splat instead of one per covered tile.
#include "gs_geom.cuh"
#include "gs_kernels.h"

namespace gs {

template <int DEG>
__global__ void __launch_bounds__(256) k_project(ProjectArgs a) {
  constexpr int K = DEG > 0 ? (DEG + 1) * (DEG + 1) - 1 : 0;
  const uint64_t gid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= (uint64_t)a.n * a.V) return;
  const uint32_t v = (uint32_t)(gid / a.n);
  const uint32_t i = (uint32_t)(gid - (uint64_t)v * a.n);
  const DevCam c = a.cams[v];
  const size_t slot = (size_t)v * a.n + i;
  a.rect[slot] = make_uint2(0xFFFFFFFFu, 0u);

  float P[16];
  const float4* P4 = reinterpret_cast<const float4*>(a.params + (size_t)i * STRIDE);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const float4 t = P4[k];
    P[4 * k] = t.x; P[4 * k + 1] = t.y; P[4 * k + 2] = t.z; P[4 * k + 3] = t.w;
  }
  const Geom g = computeGeom(c, P);
  if (!g.ok) return;
  const float detV = fmaxf(g.va * g.vc - g.vb * g.vb, 0.0f);
  const float ad = g.va + 0.3f, cd = g.vc + 0.3f;
  const float detVd = ad * cd - g.vb * g.vb;
  if (detVd < 1e-8f) return;
  const float comp = sqrtf(fmaxf(detV / detVd, 0.0f));
  const float opa = sigm(P[13]);
  if (opa * comp < a.aMin) return;
  const float f = c.f;
  const float mx = f * g.pc[0] / g.pc[2] + c.cx;
  const float my = f * g.pc[1] / g.pc[2] + c.cy;
  const float mid = 0.5f * (ad + cd);
  const float disc = sqrtf(fmaxf(mid * mid - detVd, 0.0f));
  const float eMax = fminf(a.eCut, glog(fmaxf(opa * comp / a.aMin, 1.0001f)));
  const float rad = fminf(sqrtf(2.0f * eMax) * sqrtf(mid + disc), a.radClamp * (float)c.W);
  const float W = (float)c.W, H = (float)c.H;
  if (mx + rad < 0.0f || my + rad < 0.0f || mx - rad > W || my - rad > H) return;
  const float inv = 1.0f / detVd;
  float col[3] = {sigm(P[10]), sigm(P[11]), sigm(P[12])};
  if (K > 0) {
    float cp[3];
    camPosWorld(c, cp);
    const float un[3] = {P[0] - cp[0], P[1] - cp[1], P[2] - cp[2]};
    const float len = fmaxf(sqrtf(dot3(un, un)), 1e-9f);
    const float vd[3] = {un[0] / len, un[1] / len, un[2] / len};
    float Y[15];
    shBasis<DEG>(vd, Y);
    const int aK = shActiveK(c, K);
    const float* shp = a.sh + (size_t)i * 3 * K;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      if (k < aK) {
        col[0] = col[0] + shp[k] * Y[k];
        col[1] = col[1] + shp[K + k] * Y[k];
        col[2] = col[2] + shp[2 * K + k] * Y[k];
      }
    }
#pragma unroll
    for (int j = 0; j < 3; ++j) col[j] = fmaxf(col[j], 0.0f);
  }
  // conic normaliser 1/(1 + lambda_max) (shaders.js:674-678); the same value
  // as 1/(1 + (mid + disc)) computed here from identical operands
  const float lmax = mid + disc;
  const float cnorm = 1.0f / (1.0f + lmax);

  // conservative cull radius for whole warps of pixels: beyond `rad` from the
  // mean no pixel passes both cutoffs (e >= d^2 / (2 lambda_max) > eMax),
  // unless the radius was clamped; one pixel of margin covers rounding
  const float cullR = rad >= a.radClamp * (float)c.W ? __int_as_float(0x7F800000) : rad + 1.0f;
  RenderRec r;
  // conic stored as (cA/2, cB, cC/2): halving is exact and saves the
  // rasteriser's per-pixel multiplies by 0.5
  r.r0 = make_float4(mx, my, 0.5f * (cd * inv), -g.vb * inv);
  r.r1 = make_float4(0.5f * (ad * inv), opa * comp, col[0], col[1]);
  r.r2 = make_float4(col[2], opa, cnorm, cullR);
  a.recs[slot] = r;
  a.depth[slot] = g.pc[2];

  // tile bounds (shaders.js:303-308)
  const int tx = c.tilesX, ty = c.tilesY;
  const float TF = (float)a.tile;
  const uint32_t x0 = u32sat(clampf(floorf((mx - rad) / TF), 0.0f, (float)(tx - 1)));
  const uint32_t x1 = u32sat(clampf(floorf((mx + rad) / TF), 0.0f, (float)(tx - 1)));
  const uint32_t y0 = u32sat(clampf(floorf((my - rad) / TF), 0.0f, (float)(ty - 1)));
  const uint32_t y1 = u32sat(clampf(floorf((my + rad) / TF), 0.0f, (float)(ty - 1)));
  a.rect[slot] = make_uint2(x0 | (y0 << 16), x1 | (y1 << 16));
  // rectangle add on the (tx+1) x (ty+1) difference grid
  int32_t* gd = a.diffGrid + a.gridBase[v];
  const int gw = tx + 1;
  atomicAdd(&gd[y0 * gw + x0], 1);
  atomicAdd(&gd[y0 * gw + x1 + 1], -1);
  atomicAdd(&gd[(y1 + 1) * gw + x0], -1);
  atomicAdd(&gd[(y1 + 1) * gw + x1 + 1], 1);
}

// One CTA per batch: per view, the 2D prefix sum of the difference grid gives
// the reference's tileCnt; then the budgeted scan of shaders.js:341-372 with
// its padding rule (segments above 2048 entries round up to a power of two)
// decides which tiles the entry budget drops (counted in stats[3]); the
// kept counts' exclusive scan over (view, tile) is each tile's range in the
// sorted entry list.  Views are processed in order so ranges are global.
__global__ void __launch_bounds__(1024) k_tile_ranges(TileRangeArgs a) {
  __shared__ uint32_t s_base;
  __shared__ uint32_t s_red[32];
  if (threadIdx.x == 0) s_base = 0;
  __syncthreads();
  for (int v = 0; v < a.V; ++v) {
    const DevCam c = a.cams[v];
    const int tx = c.tilesX, ty = c.tilesY, gw = tx + 1;
    int32_t* gd = a.diffGrid + a.gridBase[v];
    // rows: prefix along x
    for (int y = threadIdx.x; y < ty; y += blockDim.x) {
      int32_t acc = 0;
      for (int x = 0; x < tx; ++x) { acc += gd[y * gw + x]; gd[y * gw + x] = acc; }
    }
    __syncthreads();
    // columns: prefix along y -> per-tile count
    uint32_t* cnt = a.tileCnt + c.tileBase;
    for (int x = threadIdx.x; x < tx; x += blockDim.x) {
      int32_t acc = 0;
      for (int y = 0; y < ty; ++y) { acc += gd[y * gw + x]; cnt[y * tx + x] = (uint32_t)acc; }
    }
    __syncthreads();
    // budget: padded prefix; fast path when the whole view fits
    const int nt = tx * ty;
    uint64_t local = 0;
    for (int t = threadIdx.x; t < nt; t += blockDim.x) {
      const uint32_t cc = cnt[t];
      uint64_t p = cc;
      if (cc > SHSORT) { uint64_t q = 1; while (q < cc) q <<= 1; p = q; }
      local += p;
    }
    // block sum of the padded sizes (sums stay far below 2^32 per view in
    // practice; saturate anyway)
    uint32_t l32 = local > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)local;
    uint32_t wsum = __reduce_add_sync(0xFFFFFFFFu, l32);
    if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = wsum;
    __syncthreads();
    if (threadIdx.x == 0) {
      uint64_t tot = 0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += s_red[w];
      int drops = 0;
      uint8_t* dr = a.dropped + c.tileBase;
      if (tot > a.entriesCap) {
        // sequential budget rule (shaders.js:357-372)
        uint64_t acc = 0;
        for (int t = 0; t < nt; ++t) {
          const uint32_t cc = cnt[t];
          uint64_t p = cc;
          if (cc > SHSORT) { uint64_t q = 1; while (q < cc) q <<= 1; p = q; }
          if (acc + p > a.entriesCap) { dr[t] = 1; ++drops; }
          else { dr[t] = 0; acc += p; }
        }
      } else {
        for (int t = 0; t < nt; ++t) dr[t] = 0;
      }
      a.viewDrops[v] = (uint32_t)drops;
      if (drops) atomicAdd(&a.stats[3], (uint32_t)drops);
    }
    __syncthreads();
    // exclusive scan of kept counts in tile order -> ranges
    const uint8_t* dr = a.dropped + c.tileBase;
    const int per = (nt + blockDim.x - 1) / blockDim.x;
    const int t0 = threadIdx.x * per;
    uint32_t mine = 0;
    for (int t = t0; t < min(nt, t0 + per); ++t) mine += dr[t] ? 0u : cnt[t];
    // block exclusive scan of `mine`
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t inc = mine;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xFFFFFFFFu, inc, o);
      if (lane >= o) inc += y;
    }
    __syncthreads();
    if (lane == 31) s_red[wid] = inc;
    __syncthreads();
    if (wid == 0) {
      uint32_t w = (lane < (int)(blockDim.x >> 5)) ? s_red[lane] : 0u;
      uint32_t wi = w;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xFFFFFFFFu, wi, o);
        if (lane >= o) wi += y;
      }
      s_red[lane] = wi - w;  // exclusive prefix of warp sums
    }
    __syncthreads();
    uint32_t run = s_base + s_red[wid] + (inc - mine);
    uint2* rg = a.ranges + c.tileBase;
    for (int t = t0; t < min(nt, t0 + per); ++t) {
      const uint32_t k = dr[t] ? 0u : cnt[t];
      rg[t] = make_uint2(run, run + k);
      run += k;
    }
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) s_base = run;
    __syncthreads();
  }
  if (threadIdx.x == 0) a.totalEntries[0] = s_base;
}

// Entries each (view, splat) contributes: its bbox area, minus budget-dropped
// tiles when its view dropped any.
__global__ void __launch_bounds__(256) k_splat_counts(SplatCountArgs a) {
  const uint64_t gid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= (uint64_t)a.n * a.V) return;
  const uint32_t v = (uint32_t)(gid / a.n);
  const uint2 r = a.rect[gid];
  uint32_t cnt = 0;
  if (r.x != 0xFFFFFFFFu) {
    const uint32_t x0 = r.x & 0xFFFFu, y0 = r.x >> 16, x1 = r.y & 0xFFFFu, y1 = r.y >> 16;
    if (a.viewDrops[v] == 0) {
      cnt = (x1 - x0 + 1) * (y1 - y0 + 1);
    } else {
      const DevCam& c = a.cams[v];
      const uint8_t* dr = a.dropped + c.tileBase;
      for (uint32_t y = y0; y <= y1; ++y)
        for (uint32_t x = x0; x <= x1; ++x) cnt += dr[y * c.tilesX + x] ? 0u : 1u;
    }
  }
  a.counts[gid] = cnt;
}

// Key generation: entry (globalTile << 32 | depth f32 bits, splat id), written
// in (view, splat, tile row-major) order so a stable sort by key leaves equal
// keys in id order -- the reference's (key, id) tie-break (shaders.js:454).
__global__ void __launch_bounds__(256) k_keygen(KeygenArgs a) {
  const uint64_t gid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= (uint64_t)a.n * a.V) return;
  const uint2 r = a.rect[gid];
  if (r.x == 0xFFFFFFFFu) return;
  const uint32_t v = (uint32_t)(gid / a.n);
  const uint32_t i = (uint32_t)(gid - (uint64_t)v * a.n);
  const DevCam& c = a.cams[v];
  const uint32_t x0 = r.x & 0xFFFFu, y0 = r.x >> 16, x1 = r.y & 0xFFFFu, y1 = r.y >> 16;
  const uint32_t depthBits = __float_as_uint(a.depth[gid]);
  const uint8_t* dr = a.dropped + c.tileBase;
  const bool anyDrop = a.viewDrops[v] != 0;
  uint32_t o = a.offsets[gid];
  for (uint32_t y = y0; y <= y1; ++y)
    for (uint32_t x = x0; x <= x1; ++x) {
      const uint32_t t = y * c.tilesX + x;
      if (anyDrop && dr[t]) continue;
      if (o < a.capacity) {
        a.keys[o] = ((uint64_t)(c.tileBase + t) << 32) | depthBits;
        a.vals[o] = i;
      } else {
        atomicOr(a.status, ST_ENTRY_OVERFLOW);
      }
      ++o;
    }
}

void launch_project(const ProjectArgs& a, int deg, cudaStream_t s) {
  const uint64_t total = (uint64_t)a.n * a.V;
  const unsigned grid = (unsigned)((total + 255) / 256);
  if (grid == 0) return;
  switch (deg) {
    case 0: k_project<0><<<grid, 256, 0, s>>>(a); break;
    case 1: k_project<1><<<grid, 256, 0, s>>>(a); break;
    case 2: k_project<2><<<grid, 256, 0, s>>>(a); break;
    default: k_project<3><<<grid, 256, 0, s>>>(a); break;
  }
}
void launch_tile_ranges(const TileRangeArgs& a, cudaStream_t s) { k_tile_ranges<<<1, 1024, 0, s>>>(a); }
void launch_splat_counts(const SplatCountArgs& a, cudaStream_t s) {
  const uint64_t total = (uint64_t)a.n * a.V;
  const unsigned grid = (unsigned)((total + 255) / 256);
  if (grid) k_splat_counts<<<grid, 256, 0, s>>>(a);
}
void launch_keygen(const KeygenArgs& a, cudaStream_t s) {
  const uint64_t total = (uint64_t)a.n * a.V;
  const unsigned grid = (unsigned)((total + 255) / 256);
  if (grid) k_keygen<<<grid, 256, 0, s>>>(a);
}

}  // namespace gs
