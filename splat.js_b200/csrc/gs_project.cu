// gs_project.cu -- pass 1 of the training step: projection + SH colour
// (shaders.js:228-315) for every (view, splat) of a batch, and the binning
// that turns projected splats into sorted per-tile entry lists.
//
// Binning.  The reference counts tiles per splat, scans, scatters (key, id)
// pairs into per-tile segments with atomic cursors and bitonic-sorts each
// segment by (depth f32 bits, id) (shaders.js:303-500).  Here:
//   1. k_project writes, per (view, splat), the raster record, the tile
//      rectangle, cull parameters, four atomics into the view's tile
//      difference grid (its 2D prefix sum is the reference's per-tile
//      count), and a presort item: key = depth bits -- all ones when culled
//      -- and value slot = view * n + splat;
//   2. k_tile_counts (one block per view): tileCnt, the reference's entry
//      budget (drops), and view-local tile ranges; k_tile_ranges_finish
//      offsets them by the earlier views' totals;
//   3. the items are radix-sorted by depth bits (stable from slot order, so
//      equal depths keep id order; views stay interleaved);
//   4. k_expand (count pass) / scan / k_expand (key pass) expand the sorted
//      items into one entry per (splat, live tile) -- key = global tile id
//      (32 bits), value = splat id -- written in that order;
//   5. a stable radix sort on the global tile id (each id belongs to one
//      view) leaves every tile's entries in (depth bits, id) order: the
//      reference's per-tile order, with two passes over 8-byte entries
//      instead of six over 12-byte ones.
#include "gs_geom.cuh"
#include "gs_kernels.h"

namespace gs {

// One thread per splat, looping over the batch's views: parameters and SH
// coefficients are read once per step.
template <int DEG>
__global__ void __launch_bounds__(256, 4) k_project(ProjectArgs a) {  // 4 blocks/SM: 64 registers
  constexpr int K = DEG > 0 ? (DEG + 1) * (DEG + 1) - 1 : 0;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  // the batch's cameras in shared memory (read once per block); each thread
  // issues its parameter loads before the barrier that publishes them
  __shared__ DevCam s_cams[MAX_VIEWS];
  copy_cams(s_cams, a.cams, a.V);
  float P[16];
  if (i < a.n) {
    const float4* P4 = reinterpret_cast<const float4*>(a.params + (size_t)i * STRIDE);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const float4 t = P4[k];
      P[4 * k] = t.x; P[4 * k + 1] = t.y; P[4 * k + 2] = t.z; P[4 * k + 3] = t.w;
    }
  }
  __syncthreads();
  if (i >= a.n) return;
  const float* shp = K > 0 ? a.sh + (size_t)i * 3 * K : nullptr;
  const float sig0 = sigm(P[10]), sig1 = sigm(P[11]), sig2 = sigm(P[12]);
  const float opa = sigm(P[13]);

  for (int v = 0; v < a.V; ++v) {
    const DevCam& c = s_cams[v];
    const size_t slot = (size_t)v * a.n + i;
    a.rect[slot] = make_uint2(0xFFFFFFFFu, 0u);
    a.pkeys[slot] = 0xFFFFFFFFu;
    a.pvals[slot] = (uint32_t)slot;
    const Geom g = computeGeom(c, P);
    if (!g.ok) continue;
    const float detV = fmaxf(g.va * g.vc - g.vb * g.vb, 0.0f);
    const float ad = g.va + 0.3f, cd = g.vc + 0.3f;
    const float detVd = ad * cd - g.vb * g.vb;
    if (detVd < 1e-8f) continue;
    const float comp = sqrtf(fmaxf(detV / detVd, 0.0f));
    if (opa * comp < a.aMin) continue;
    const float f = c.f;
    const float mx = f * g.pc[0] / g.pc[2] + c.cx;
    const float my = f * g.pc[1] / g.pc[2] + c.cy;
    const float mid = 0.5f * (ad + cd);
    const float disc = sqrtf(fmaxf(mid * mid - detVd, 0.0f));
    const float eMax = fminf(a.eCut, glog(fmaxf(opa * comp / a.aMin, 1.0001f)));
    const float rad = fminf(sqrtf(2.0f * eMax) * sqrtf(mid + disc), a.radClamp * (float)c.W);
    const float W = (float)c.W, H = (float)c.H;
    if (mx + rad < 0.0f || my + rad < 0.0f || mx - rad > W || my - rad > H) continue;
    const float inv = 1.0f / detVd;
    float col[3] = {sig0, sig1, sig2};
    if (K > 0) {
      float cp[3];
      camPosWorld(c, cp);
      const float un[3] = {P[0] - cp[0], P[1] - cp[1], P[2] - cp[2]};
      const float len = fmaxf(sqrtf(dot3(un, un)), 1e-9f);
      const float vd[3] = {un[0] / len, un[1] / len, un[2] / len};
      float Y[15];
      shBasis<DEG>(vd, Y);
      const int aK = shActiveK(c, K);
#pragma unroll
      for (int k = 0; k < K; ++k) {
        if (k < aK) {
          col[0] = col[0] + __ldg(shp + k) * Y[k];
          col[1] = col[1] + __ldg(shp + K + k) * Y[k];
          col[2] = col[2] + __ldg(shp + 2 * K + k) * Y[k];
        }
      }
#pragma unroll
      for (int j = 0; j < 3; ++j) col[j] = fmaxf(col[j], 0.0f);
    }
    // conic normaliser 1/(1 + lambda_max) (shaders.js:674-678); the same value
    // as 1/(1 + (mid + disc)) computed here from identical operands
    const float lmax = mid + disc;
    const float cnorm = 1.0f / (1.0f + lmax);
    // the backward reads -cnorm/2 and 1 - opa (exact or identically rounded
    // forms of its own factors), stored here once per (view, splat)
    RenderRec r;
    // conic stored as (cA/2, cB, cC/2): halving is exact and saves the
    // rasteriser's per-pixel multiplies by 0.5
    r.r0 = make_float4(mx, my, 0.5f * (cd * inv), -g.vb * inv);
    r.r1 = make_float4(0.5f * (ad * inv), opa * comp, col[0], col[1]);
    r.r2 = make_float4(col[2], opa, -0.5f * cnorm, 1.0f - opa);
    a.recs[slot] = r;
    a.pkeys[slot] = __float_as_uint(g.pc[2]);  // positive: bit order = numeric order

    // tile bounds (shaders.js:303-308)
    const int tx = c.tilesX, ty = c.tilesY;
    const float TF = (float)a.tile;
    const uint32_t x0 = u32sat(clampf(floorf((mx - rad) / TF), 0.0f, (float)(tx - 1)));
    const uint32_t x1 = u32sat(clampf(floorf((mx + rad) / TF), 0.0f, (float)(tx - 1)));
    const uint32_t y0 = u32sat(clampf(floorf((my - rad) / TF), 0.0f, (float)(ty - 1)));
    const uint32_t y1 = u32sat(clampf(floorf((my + rad) / TF), 0.0f, (float)(ty - 1)));
    a.rect[slot] = make_uint2(x0 | (y0 << 16), x1 | (y1 << 16));
    // cull parameters: the tile cull and the rasteriser's warp-block masks
    const float4 cq = cullParams(mx, my, r.r0.z, r.r0.w, r.r1.x, r.r1.y, a.aMin, a.eCut, x0, x1, y0, y1, a.tile);
    a.cullRecs[slot] = cq;
    // what the expansion needs of this item, in one 32-byte record it
    // gathers with a single sector read
    a.itemSrc[2 * slot] = make_uint4(x0 | (y0 << 16), x1 | (y1 << 16), __float_as_uint(mx), __float_as_uint(my));
    a.itemSrc[2 * slot + 1] = make_uint4(__float_as_uint(cq.x), __float_as_uint(cq.y), __float_as_uint(cq.z),
                                         (uint32_t)slot);
    // rectangle add on the (tx+1) x (ty+1) difference grid
    int32_t* gd = a.diffGrid + (size_t)(i & (GRID_COPIES - 1u)) * a.gridCells + a.gridBase[v];
    const int gw = tx + 1;
    atomicAdd(&gd[y0 * gw + x0], 1);
    atomicAdd(&gd[y0 * gw + x1 + 1], -1);
    atomicAdd(&gd[(y1 + 1) * gw + x0], -1);
    atomicAdd(&gd[(y1 + 1) * gw + x1 + 1], 1);
  }
}

// One block (1024 threads) per view: the 2D prefix sum of the difference grid
// gives the reference's tileCnt; the budgeted scan of shaders.js:341-372 with
// its padding rule (segments above 2048 entries round up to a power of two)
// decides which tiles the entry budget drops (counted in stats[3]); the
// kept counts' exclusive scan gives view-local tile ranges.
__global__ void __launch_bounds__(1024) k_tile_counts(TileRangeArgs a) {
  __shared__ uint32_t s_red[33];
  const int v = blockIdx.x;
  const DevCam c = a.cams[v];
  const int tx = c.tilesX, ty = c.tilesY, gw = tx + 1;
  int32_t* gd = a.diffGrid + a.gridBase[v];
  // rows: prefix along x, one warp per row, 32 columns per step
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int y = wid; y < ty; y += nw) {
    int32_t carry = 0;
    for (int x0 = 0; x0 < tx; x0 += 32) {
      const int x = x0 + lane;
      int32_t v = 0;
      if (x < tx) {  // the copies' sum (order-free: integers)
#pragma unroll
        for (uint32_t k = 0; k < GRID_COPIES; ++k) v += gd[(size_t)k * a.gridCells + y * gw + x];
      }
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int32_t u = __shfl_up_sync(0xFFFFFFFFu, v, o);
        if (lane >= o) v += u;
      }
      v += carry;
      if (x < tx) gd[y * gw + x] = v;
      carry = __shfl_sync(0xFFFFFFFFu, v, 31);
    }
  }
  __syncthreads();
  // columns: prefix along y -> per-tile count, one warp per column
  uint32_t* cnt = a.tileCnt + c.tileBase;
  for (int x = wid; x < tx; x += nw) {
    int32_t carry = 0;
    for (int y0 = 0; y0 < ty; y0 += 32) {
      const int y = y0 + lane;
      int32_t v = y < ty ? gd[y * gw + x] : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int32_t u = __shfl_up_sync(0xFFFFFFFFu, v, o);
        if (lane >= o) v += u;
      }
      v += carry;
      if (y < ty) cnt[y * tx + x] = (uint32_t)v;
      carry = __shfl_sync(0xFFFFFFFFu, v, 31);
    }
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
  const uint32_t l32 = local > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)local;
  const uint32_t wsum = __reduce_add_sync(0xFFFFFFFFu, l32);
  if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = wsum;
  __syncthreads();
  uint8_t* dr = a.dropped + c.tileBase;
  if (threadIdx.x == 0) {
    uint64_t tot = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += s_red[w];
    int drops = 0;
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
    }
    s_red[32] = (uint32_t)drops;
    a.viewDrops[v] = (uint32_t)drops;
    if (drops) atomicAdd(&a.stats[3], (uint32_t)drops);
  }
  __syncthreads();
  const bool anyDrop = s_red[32] != 0;
  if (!anyDrop)
    for (int t = threadIdx.x; t < nt; t += blockDim.x) dr[t] = 0;
  __syncthreads();
  // exclusive scan of kept counts in tile order -> view-local ranges
  const int per = (nt + blockDim.x - 1) / blockDim.x;
  const int t0 = threadIdx.x * per;
  uint32_t mine = 0;
  for (int t = t0; t < min(nt, t0 + per); ++t) mine += dr[t] ? 0u : cnt[t];
  uint32_t inc = mine;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t yv = __shfl_up_sync(0xFFFFFFFFu, inc, o);
    if (lane >= o) inc += yv;
  }
  __syncthreads();
  if (lane == 31) s_red[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    const uint32_t w = (lane < (int)(blockDim.x >> 5)) ? s_red[lane] : 0u;
    uint32_t wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t yv = __shfl_up_sync(0xFFFFFFFFu, wi, o);
      if (lane >= o) wi += yv;
    }
    s_red[lane] = wi - w;
    if (lane == 31) a.viewTotal[v] = wi;
  }
  __syncthreads();
  uint32_t run = s_red[wid] + (inc - mine);
  uint2* rg = a.ranges + c.tileBase;
  for (int t = t0; t < min(nt, t0 + per); ++t) {
    const uint32_t k = dr[t] ? 0u : cnt[t];
    rg[t] = make_uint2(run, run + k);
    run += k;
  }
}

// Offsets every view's tile ranges by the entries of the views before it and
// writes the batch's entry total.
__global__ void k_tile_ranges_finish(TileRangeArgs a, uint32_t totalTiles) {
  const uint32_t gt = blockIdx.x * blockDim.x + threadIdx.x;
  if (gt == 0) {
    uint32_t tot = 0;
    for (int v = 0; v < a.V; ++v) tot += a.viewTotal[v];
    a.totalEntries[0] = tot;
  }
  if (gt >= totalTiles) return;
  int v = 0;
  while (v + 1 < a.V && a.cams[v + 1].tileBase <= gt) ++v;
  uint32_t base = 0;
  for (int u = 0; u < v; ++u) base += a.viewTotal[u];
  const uint2 r = a.ranges[gt];
  a.ranges[gt] = make_uint2(r.x + base, r.y + base);
}

// The live columns of one tile row of an item's rectangle.  tileLive(tx, ty)
// is X1(tx) >= xl && X0(tx) <= xr for the row's band interval [xl, xr], with
// X0 and X1 non-decreasing in tx, so the live tiles of a row form one run
// [ca, cb]; two binary searches on the same predicates find it, giving
// exactly the tiles tileLive() accepts.  Returns the run length (0: none).
__device__ __forceinline__ uint32_t row_run(const float4 cq, float mx, float my, uint32_t x0, uint32_t x1,
                                            uint32_t ty, int tile, int W, int H, uint32_t& ca) {
  ca = x0;
  if (!(cq.x < 3.0e38f)) return x1 - x0 + 1;
  const int ye = (int)ty * tile + tile < H ? (int)ty * tile + tile : H;
  float xl, xr;
  if (!bandInterval(cq, ((float)((int)ty * tile) + 0.5f) - my, ((float)(ye - 1) + 0.5f) - my, xl, xr)) return 0;
  // ca: first column with X1 >= xl
  uint32_t lo = x0, hi = x1 + 1;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    const int xe = (int)mid * tile + tile < W ? (int)mid * tile + tile : W;
    if (((float)(xe - 1) + 0.5f) - mx >= xl) hi = mid;
    else lo = mid + 1;
  }
  ca = lo;
  // cb + 1: first column after ca with X0 > xr
  hi = x1 + 1;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (((float)((int)mid * tile) + 0.5f) - mx <= xr) lo = mid + 1;
    else hi = mid;
  }
  return lo - ca;
}

// Entry expansion of the presorted items, in two passes over the same walk:
// KEYS = false counts each item's entries, KEYS = true writes them at the
// counts' exclusive scan -- key = global tile id, value = splat id, tiles of
// an item in row order.  An entry is a tile of the item's rectangle that the
// entry budget kept and, with culling on, that tileLive() accepts (a
// single-tile rectangle is kept untested).
//
// A warp walks the tile rows of its 32 items 32 rows at a time: each lane
// finds the item owning its row by a binary search over the items' row
// offsets (shuffles) and computes the row's run of live tiles.  The count
// pass sums the runs per item; the key pass ranks them (a segmented scan) and
// then fills the rows' outputs 32 entries at a time, each lane finding its
// row by a second binary search, so stores are coalesced.  Items of views
// that dropped tiles to the budget are walked by their own lane (rare).
template <bool KEYS>
__global__ void __launch_bounds__(256) k_expand(ExpandArgs a) {
  __shared__ uint32_t s_run[256];  // entries of each item so far
  const uint64_t items = (uint64_t)a.n * a.V;
  // culled items carry the all-ones key, which the presort drops: its output
  // holds the live items only
  const uint64_t live = *a.liveItems;
  const uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if ((uint64_t)blockIdx.x * blockDim.x >= live) {  // the whole block is culled items (uniform)
    if (!KEYS && p < items) a.counts[p] = 0u;
    return;
  }
  const int lane = threadIdx.x & 31;
  const int wbase = threadIdx.x & ~31;
  const uint32_t FULL = 0xFFFFFFFFu;
  const bool valid = p < live;
  uint32_t v = 0, i = 0, x0 = 0, x1 = 0, y0 = 0, rr = 0, out = 0;
  bool test = false;
  float mx = 0.0f, my = 0.0f;
  float4 cq = make_float4(__int_as_float(0x7F800000), 0.0f, 0.0f, 0.0f);
  s_run[threadIdx.x] = 0;
  if (valid) {
    // the item's rectangle, mean and cull parameters: gathered by slot in
    // the count pass (one 32-byte record the projection wrote) and written
    // in presort order, so the key pass reads them coalesced
    uint32_t slot;
    uint2 r;
    if (!KEYS) {
      slot = a.sortedSlots[p];
      const uint4 s0 = a.itemSrc[2 * slot], s1 = a.itemSrc[2 * slot + 1];
      r = make_uint2(s0.x, s0.y);
      if (r.x != 0xFFFFFFFFu && a.cull) {
        mx = __uint_as_float(s0.z); my = __uint_as_float(s0.w);
        cq = make_float4(__uint_as_float(s1.x), __uint_as_float(s1.y), __uint_as_float(s1.z), 0.0f);
      }
      a.itemRecs[2 * p] = make_uint4(r.x, r.y, __float_as_uint(mx), __float_as_uint(my));
      a.itemRecs[2 * p + 1] = make_uint4(__float_as_uint(cq.x), __float_as_uint(cq.y), __float_as_uint(cq.z), slot);
    } else {
      const uint4 e0 = a.itemRecs[2 * p], e1 = a.itemRecs[2 * p + 1];
      r = make_uint2(e0.x, e0.y);
      mx = __uint_as_float(e0.z); my = __uint_as_float(e0.w);
      cq = make_float4(__uint_as_float(e1.x), __uint_as_float(e1.y), __uint_as_float(e1.z), 0.0f);
      slot = e1.w;
      out = a.offsets[p];
    }
    if (r.x != 0xFFFFFFFFu) {
      v = slot / a.n;
      i = slot - v * a.n;
      x0 = r.x & 0xFFFFu; y0 = r.x >> 16;
      x1 = r.y & 0xFFFFu;
      const uint32_t y1 = r.y >> 16;
      test = a.cull && !(x0 == x1 && y0 == y1);
      if (a.viewDrops[v] == 0) {
        rr = y1 - y0 + 1;
      } else {
        const DevCam& c = a.cams[v];
        const uint8_t* dr = a.dropped + c.tileBase;
        uint32_t o = out, cnt = 0;
        for (uint32_t y = y0; y <= y1; ++y)
          for (uint32_t x = x0; x <= x1; ++x) {
            const uint32_t t = y * c.tilesX + x;
            if (dr[t]) continue;
            if (test && !tileLive(cq, mx, my, (int)x, (int)y, a.tile, c.W, c.H)) continue;
            if (KEYS) {
              if (o < a.capacity) { a.keys[o] = c.tileBase + t; a.vals[o] = i; }
              else atomicOr(a.status, ST_ENTRY_OVERFLOW);
              ++o;
            }
            ++cnt;
          }
        s_run[threadIdx.x] = cnt;
      }
    }
  }
  if (!test) cq = make_float4(__int_as_float(0x7F800000), 0.0f, 0.0f, 0.0f);  // untested: whole rows
  __syncwarp();
  // row offsets of the warp's items (inclusive scan of rr)
  uint32_t rEnd = rr;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(FULL, rEnd, o);
    if (lane >= o) rEnd += y;
  }
  const uint32_t rBase = rEnd - rr;
  const uint32_t R = __shfl_sync(FULL, rEnd, 31);
  for (uint32_t base = 0; base < R; base += 32) {
    const uint32_t u = base + (uint32_t)lane;
    const bool inRange = u < R;
    // owner: the last lane whose row offset is <= u
    int lo = 0;
#pragma unroll
    for (int step = 16; step >= 1; step >>= 1) {
      const uint32_t ob = __shfl_sync(FULL, rBase, (lo + step) & 31);
      if (lo + step < 32 && ob <= u) lo += step;
    }
    const uint32_t orb = __shfl_sync(FULL, rBase, lo);
    const uint32_t ox0 = __shfl_sync(FULL, x0, lo);
    const uint32_t ox1 = __shfl_sync(FULL, x1, lo);
    const uint32_t oy0 = __shfl_sync(FULL, y0, lo);
    const uint32_t ov = __shfl_sync(FULL, v, lo);
    const float omx = __shfl_sync(FULL, mx, lo);
    const float omy = __shfl_sync(FULL, my, lo);
    float4 ocq;
    ocq.x = __shfl_sync(FULL, cq.x, lo);
    ocq.y = __shfl_sync(FULL, cq.y, lo);
    ocq.z = __shfl_sync(FULL, cq.z, lo);
    ocq.w = 0.0f;
    uint32_t cnt = 0, ca = 0, ty = 0;
    if (inRange) {
      ty = oy0 + (u - orb);
      const DevCam& c = a.cams[ov];
      cnt = row_run(ocq, omx, omy, ox0, ox1, ty, a.tile, c.W, c.H, ca);
    }
    const uint32_t peers = __match_any_sync(FULL, inRange ? (uint32_t)lo : 32u);
    const int lead = __ffs(peers) - 1;
    const uint32_t prior = s_run[wbase + lo];
    // segmented scan of the run lengths over the rows of each item
    uint32_t inc = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(FULL, inc, o);
      if (lane >= o) inc += y;
    }
    const uint32_t before = __shfl_sync(FULL, inc, lead > 0 ? lead - 1 : 0);
    const uint32_t segIncl = inc - (lead > 0 ? before : 0u);  // rows of this item up to this lane
    if (KEYS) {
      // this row's entries start here; fill the chunk's outputs 32 at a time
      const uint32_t oout = __shfl_sync(FULL, out, lo);
      const uint32_t rowOut = oout + prior + segIncl - cnt;
      const uint32_t oi = __shfl_sync(FULL, i, lo);
      const uint32_t tileBase = a.cams[ov].tileBase, tilesX = (uint32_t)a.cams[ov].tilesX;
      const uint32_t rowKey = tileBase + ty * tilesX + ca;  // key of the run's first tile
      // the chunk's rows in output order: rowOut is non-decreasing over lanes with entries
      const uint32_t firstOut = __reduce_min_sync(FULL, cnt ? rowOut : 0xFFFFFFFFu);
      uint32_t lastEnd = __reduce_max_sync(FULL, cnt ? rowOut + cnt : 0u);
      // 32 rows hold at most 32 x 65535 tiles; anything larger is corrupt input
      if (lastEnd > firstOut && lastEnd - firstOut > 32u * 65535u) {
        if (lane == 0) atomicOr(a.status, ST_BAD_INPUT);
        lastEnd = firstOut;
      }
      for (uint32_t eb = firstOut; eb < lastEnd; eb += 32) {
        const uint32_t e = eb + (uint32_t)lane;
        // the last lane with entries whose rowOut <= e
        int w = -1;
        // non-decreasing over lanes: rows without entries keep their start
        const uint32_t key = inRange ? rowOut : 0xFFFFFFFFu;
        int l2 = 0;
#pragma unroll
        for (int step = 16; step >= 1; step >>= 1) {
          const uint32_t kb = __shfl_sync(FULL, key, (l2 + step) & 31);
          if (l2 + step < 32 && kb <= e) l2 += step;
        }
        const uint32_t k0 = __shfl_sync(FULL, key, l2);
        w = (k0 <= e) ? l2 : -1;
        const uint32_t wc = __shfl_sync(FULL, cnt, l2 & 31);
        const uint32_t wk = __shfl_sync(FULL, rowKey, l2 & 31);
        const uint32_t wi = __shfl_sync(FULL, oi, l2 & 31);
        if (w >= 0 && e < lastEnd && e - k0 < wc) {
          if (e < a.capacity) { a.keys[e] = wk + (e - k0); a.vals[e] = wi; }
          else atomicOr(a.status, ST_ENTRY_OVERFLOW);
        }
      }
    }
    uint32_t gsum = 0;
    if (inRange) gsum = __reduce_add_sync(peers, cnt);  // the lanes of one item call it together
    __syncwarp();
    if (inRange && lane == lead) s_run[wbase + lo] = prior + gsum;
    __syncwarp();
  }
  if (!KEYS && p < items) a.counts[p] = valid ? s_run[threadIdx.x] : 0u;
}

// Per-tile ranges from the sorted entry keys (culled lists): tile gt spans
// [lower_bound(gt), lower_bound(gt + 1)), so empty and dropped tiles get an
// empty range at their place in the order, as the budgeted scan gives them.
__device__ __forceinline__ uint32_t lower_bound_u32(const uint32_t* keys, uint32_t E, uint32_t x) {
  uint32_t lo = 0, hi = E;
  while (lo < hi) {
    const uint32_t mid = lo + ((hi - lo) >> 1);
    if (keys[mid] < x) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

__global__ void __launch_bounds__(256) k_ranges_from_keys(const uint32_t* keys, const uint32_t* nItems,
                                                          uint32_t totalTiles, uint2* ranges) {
  const uint32_t gt = blockIdx.x * blockDim.x + threadIdx.x;
  if (gt >= totalTiles) return;
  const uint32_t E = *nItems;
  ranges[gt] = make_uint2(lower_bound_u32(keys, E, gt), lower_bound_u32(keys, E, gt + 1));
}

void launch_project(const ProjectArgs& a, int deg, cudaStream_t s) {
  const unsigned grid = (a.n + 255) / 256;
  if (grid == 0) return;
  switch (deg) {
    case 0: k_project<0><<<grid, 256, 0, s>>>(a); break;
    case 1: k_project<1><<<grid, 256, 0, s>>>(a); break;
    case 2: k_project<2><<<grid, 256, 0, s>>>(a); break;
    default: k_project<3><<<grid, 256, 0, s>>>(a); break;
  }
}
void launch_tile_ranges(const TileRangeArgs& a, uint32_t totalTiles, cudaStream_t s) {
  k_tile_counts<<<a.V, 1024, 0, s>>>(a);
  k_tile_ranges_finish<<<(totalTiles + 255) / 256, 256, 0, s>>>(a, totalTiles);
}
void launch_expand(const ExpandArgs& a, bool keys, cudaStream_t s) {
  const uint64_t total = (uint64_t)a.n * a.V;
  const unsigned grid = (unsigned)((total + 255) / 256);
  if (!grid) return;
  if (keys) k_expand<true><<<grid, 256, 0, s>>>(a);
  else k_expand<false><<<grid, 256, 0, s>>>(a);
}
void launch_ranges_from_keys(const uint32_t* keys, const uint32_t* nItems, uint32_t totalTiles, uint2* ranges,
                             cudaStream_t s) {
  if (totalTiles) k_ranges_from_keys<<<(totalTiles + 255) / 256, 256, 0, s>>>(keys, nItems, totalTiles, ranges);
}

}  // namespace gs
