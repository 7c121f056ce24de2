// gs_kernels.h -- launch arguments of the training-step kernels (host and
// device share these plain structs; nothing here is part of the C ABI).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "gs_common.cuh"

namespace gs {

// The projection's rectangle adds go to one of GRID_COPIES copies of the
// difference grid (by splat index), summed when the counts are read: every
// splat of a tile adds to the same four corner cells, and spreading those
// atomics over copies shortens the queues on the busiest cells.  Integer
// sums: the counts do not depend on the split.
constexpr uint32_t GRID_COPIES = 4;

struct ProjectArgs {
  const float* params;     // n * 16
  const float* sh;         // n * 3K (channel-major) or null
  uint32_t n;
  int V;
  const DevCam* cams;      // V views
  float eCut, aMin, radClamp;
  int tile;
  RenderRec* recs;         // V * n
  uint32_t* pkeys;         // V * n presort keys: depth bits (all ones when culled)
  uint32_t* pvals;         // V * n presort values: slot = view * n + splat
  uint2* rect;             // V * n
  int32_t* diffGrid;       // GRID_COPIES copies of: per view (tilesX+1)*(tilesY+1), cleared before
  const uint32_t* gridBase;  // V offsets into a copy
  uint32_t gridCells;      // cells of one copy (all views)
  float4* cullRecs;        // V * n warp-block cull parameters (p, q, kA, 0)
  uint4* itemSrc;          // V * n * 2: per visible slot (rect, mean, cull parameters, slot) for the expansion
};

struct TileRangeArgs {
  int V;
  const DevCam* cams;
  int32_t* diffGrid;
  const uint32_t* gridBase;
  uint32_t gridCells;
  uint32_t* tileCnt;       // per global tile: the reference's tileCnt
  uint8_t* dropped;        // per global tile: dropped by the entry budget
  uint2* ranges;           // per global tile: [start, end) in the sorted entries
  uint32_t* viewDrops;     // per view: number of dropped tiles
  uint32_t* viewTotal;     // per view: kept entries
  uint32_t* stats;         // stats[3] += dropped tiles
  uint64_t entriesCap;     // per-view entry budget (ENTCAP)
  uint32_t* totalEntries;  // out: kept entries over the batch
};

// Entry expansion of the presorted (view, depth, id) items (k_expand).
struct ExpandArgs {
  uint32_t n;
  int V;
  const DevCam* cams;
  const uint32_t* sortedSlots;  // presorted (view, depth, id) order
  const uint4* itemSrc;         // V * n * 2 by slot: (rect, mean, cull parameters, slot) from the projection
  uint4* itemRecs;              // V * n * 2: the same per presorted item (mean and cull parameters only
                                // when cull != 0)
  const uint32_t* liveItems;    // presorted items kept (the culled ones left the presort)
  const uint8_t* dropped;
  const uint32_t* viewDrops;
  float eCut, aMin;
  int tile;
  int cull;                     // 1: keep only entries tileLive() accepts
  uint32_t* counts;             // count pass: V * n, in presorted order
  const uint32_t* offsets;      // key pass: V * n exclusive scan of counts
  uint32_t* keys;               // global tile id per entry
  uint32_t* vals;               // splat id per entry
  uint64_t capacity;
  uint32_t* status;
};

struct RadixHistArgs {
  const void* keys;        // uint32_t or uint64_t
  const uint32_t* nItems;
  uint32_t* hist;           // passes * 256
  int passes;
  uint32_t* epoch;
  uint32_t* nKept;          // non-null: all-ones keys are dropped (not counted); kept keys are counted here
};

#ifndef GS_SORT_ITEMS
#define GS_SORT_ITEMS 16  // keys per thread of a onesweep block (256 threads)
#endif
constexpr int SORT_BLOCK_ENTRIES = 256 * GS_SORT_ITEMS;  // entries one onesweep block ranks

struct OnesweepArgs {
  const void* keysIn;
  const uint32_t* valsIn;
  void* keysOut;            // null: do not write keys (last pass)
  uint32_t* valsOut;
  const uint32_t* nItems;
  const uint32_t* hist;
  uint32_t* tileCounter;    // per pass
  uint64_t* status;         // look-back words, one per (block, digit)
  uint32_t* statusWord;     // error bits
  const uint32_t* epoch;
  int pass;
  uint32_t spinLimit;       // look-back spins before the block gives up and flags a timeout
  int dropAllOnes;          // all-ones keys leave the sort (output compacted to the kept keys);
                            // selects the kernel instantiation that drops them
};

struct RadixSortArgs {
  void* keys[2];            // ping-pong key buffers of keyBytes-wide keys
  int keyBytes;             // 4 or 8
  uint32_t* vals[2];
  const uint32_t* nItems;
  uint32_t* hist;
  uint32_t* tileCounter;
  uint64_t* status;
  uint32_t* statusWord;
  uint32_t* epoch;
  int passes;
  bool keepKeys;
  unsigned histGrid, sweepGrid;
  uint32_t* nKept;          // non-null (32-bit keys): all-ones keys are dropped in the first pass and the
                            // kept count lands here (zero before the call); later passes sort only those
  uint32_t orPasses;        // 32-bit keys, bit p: pass p ranks its digits with the OR form (digits spread
                            // across a warp: tile ids, the low bytes of depths)
};

struct RasterArgs {
  const DevCam* cams;
  int V;
  uint32_t n;
  const RenderRec* recs;   // V * n
  const float4* cullRecs;  // V * n warp-block cull parameters
  const uint32_t* ids;     // sorted entry values (splat ids)
  const uint2* ranges;     // per global tile
  uint32_t totalTiles;
  const uint32_t* workOrder;  // null: item order
  uint32_t* workCounter;      // null: one item per block (blockIdx.x)
  float eCut, aMin;
  float4* outImg;          // per batch pixel (RGB, 1 - T)
  float* finalT;
  uint32_t* endIdx;
  const uint32_t* targets;
  int32_t* gradP;          // V * n * GP_STRIDE
  uint32_t* stats;
  int32_t* gradCam;
  float* tStore;           // stored-state variant: T before each entry, per pixel
};

struct AdamHP {
  float lr[16];
  float b1, b2, eps, bc1, bc2, minLS, maxLS, maxLogit, reg, shLr;
};

// floats per (view, splat) chain result: 14 parameter gradients, gated
// colour gradient (3), view direction (3)
constexpr int VIEWGRAD_STRIDE = 20;

struct ChainArgs {
  uint32_t n;
  int V;
  const DevCam* cams;
  float* params;
  float* sh;
  int32_t* gradP;
  const uint2* rect;
  float* viewGrad;         // V * n * VIEWGRAD_STRIDE: per-(view, splat) chain results
  uint32_t* visList;       // V * n: per view, indices of the visible splats
  uint32_t* visCount;      // V counters, cleared before the step
  float anisoReg;
  int32_t* gradCam;
  float* gradF;            // optional readout (n * 16)
  float* shGrad;           // optional readout (n * 3K)
  int doAdam;
  const AdamHP* hp;        // device-resident (updated every step)
  float* m;
  float* v;
  float* shM;
  float* shV;
};

// refine: one spawned splat of the plan the host draws (trainer.js:713-752)
struct RefineSpawn {
  uint32_t pos;    // position in the donor list, or in the sorted big-donor list when split
  uint32_t split;  // 1: split a big donor, 0: clone a donor
  double g[3];     // the three gauss() jitters of the position
};

struct RefineApplyArgs {
  const RefineSpawn* plan;
  uint32_t count;          // moved + grown
  uint32_t moved;          // the first `moved` spawns relocate dead splats
  uint32_t n;              // splat count before growth
  const uint32_t* deadList;
  const uint32_t* donorList;
  const uint32_t* bigSorted;   // donors by mean log-scale, descending (stable)
  const uint32_t* splitSeq;    // per splat: sequence number of its split, or ~0
  float* params;
  float* m;
  float* v;
  float* sh;
  float* shM;
  float* shV;
  int shr;                 // 3K
};

// launchers
void launch_project(const ProjectArgs& a, int deg, cudaStream_t s);
void launch_tile_ranges(const TileRangeArgs& a, uint32_t totalTiles, cudaStream_t s);
void launch_expand(const ExpandArgs& a, bool keys, cudaStream_t s);
void launch_ranges_from_keys(const uint32_t* keys, const uint32_t* nItems, uint32_t totalTiles, uint2* ranges,
                             cudaStream_t s);
uint32_t scan_partials_needed(uint64_t N);
void launch_exclusive_scan(const uint32_t* in, uint64_t N, uint32_t* out, uint32_t* partials, uint32_t* total,
                           cudaStream_t s);
int onesweep_grid(int device);
// RGBA8 packing of one camera's float RGB target (host memory) into out,
// staged through scratch (3 floats per pixel) on stream s.
int pack_targets_device(const float* rgbHost, uint64_t np, float* scratch, uint32_t* out, cudaStream_t s);
int export_ply_records(const float* params, const float* sh, uint32_t n, uint32_t K, int bake, double f,
                       const double* camPosHost, uint32_t ncams, double* dCam, float* dOut, void* outHost,
                       cudaStream_t s);
int debug_lookback_timeout(int device, uint32_t spinLimit, uint32_t* statusOut, double* msOut);
void launch_radix_sort(const RadixSortArgs& a, cudaStream_t s);
void launch_raster(const RasterArgs& a, int mode, bool stored, int tile, int batchDepth, unsigned grid,
                   cudaStream_t s);
int raster_blocks_per_sm(int tile, int batchDepth, int mode);
void launch_work_order(const uint2* ranges, uint32_t totalTiles, uint32_t* order, uint32_t* scratch,
                       cudaStream_t s);
void launch_chain_adam(const ChainArgs& a, int deg, cudaStream_t s);
void launch_refine_classify(const float* params, uint32_t n, uint32_t* deadFlag, uint32_t* donorFlag,
                            cudaStream_t s);
void launch_refine_compact(const float* params, uint32_t n, const uint32_t* deadFlag, const uint32_t* deadOff,
                           const uint32_t* donorFlag, const uint32_t* donorOff, uint32_t* deadList,
                           uint32_t* donorList, uint64_t* donorKeys, uint32_t* donorVals, cudaStream_t s);
void launch_refine_apply(const RefineApplyArgs& a, uint32_t* splitSeq, cudaStream_t s);
void launch_donor_opacity(const float* params, const uint32_t* donorList, uint32_t nDonors, float* out,
                          cudaStream_t s);
void launch_max_u32(const uint32_t* x, uint32_t count, uint32_t* out, cudaStream_t s);

}  // namespace gs
