// gs_sort.cu -- global sorted binning: exclusive scan of per-splat entry
// counts, and a onesweep LSD radix sort (8-bit digits, decoupled look-back)
// of the (globalTile << 32 | depth bits, splat id) entries.
//
// The reference bins with atomic per-tile cursors and sorts each tile segment
// with a bitonic network (shaders.js:378-500); its final order is, per tile,
// ascending (depth f32 bits, id).  Here every entry is keyed by
// (tile, depth) and written in splat order, so one stable sort over all
// entries leaves each tile's ids in exactly that order.
//
// Onesweep: one histogram kernel reads every key once and counts all digit
// positions; each digit pass then ranks a block of entries in shared memory
// (warp ballots give each key its rank among equal digits), publishes the
// block's per-digit counts, and obtains the count of every earlier block by
// decoupled look-back before scattering.  Blocks are claimed in order through
// an atomic counter by a grid that is entirely resident, so every block it
// waits on is already running.  Each spin has an iteration limit; on expiry
// the kernel sets ST_LOOKBACK_TIMEOUT in the status word and carries on.
//
// Look-back status words are 64-bit: [63:32] epoch tag, [31:30] flag,
// [29:0] count.  The tag changes every pass of every sort (the histogram
// kernel advances a device epoch), so words left by earlier sorts read as
// "not published" and the status array never needs clearing.
#include <cuda/atomic>

#include "gs_common.cuh"
#include "gs_kernels.h"

namespace gs {

// ---------------------------------------------------------------------------
// Exclusive scan of u32 counts (3 phases: block sums, scan of block sums,
// block rescans).  Block = 1024 threads x 4 items.
// ---------------------------------------------------------------------------
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_BLOCK = 1024 * SCAN_ITEMS;

__device__ __forceinline__ uint32_t block_exclusive_scan_1024(uint32_t x, uint32_t* s_warp, uint32_t* total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  uint32_t inc = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xFFFFFFFFu, inc, o);
    if (lane >= o) inc += y;
  }
  if (lane == 31) s_warp[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    uint32_t w = s_warp[lane];
    uint32_t wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xFFFFFFFFu, wi, o);
      if (lane >= o) wi += y;
    }
    s_warp[lane] = wi - w;
    if (lane == 31) s_warp[32] = wi;
  }
  __syncthreads();
  const uint32_t r = s_warp[wid] + inc - x;
  if (total) *total = s_warp[32];
  __syncthreads();
  return r;
}

__global__ void __launch_bounds__(1024) k_scan_reduce(const uint32_t* in, uint64_t N, uint32_t* partials) {
  __shared__ uint32_t s_warp[33];
  const uint64_t base = (uint64_t)blockIdx.x * SCAN_BLOCK + (uint64_t)threadIdx.x * SCAN_ITEMS;
  uint32_t s = 0;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k)
    if (base + k < N) s += in[base + k];
  uint32_t tot;
  block_exclusive_scan_1024(s, s_warp, &tot);
  if (threadIdx.x == 0) partials[blockIdx.x] = tot;
}

// single block: exclusive scan of the block sums, total to *total
__global__ void __launch_bounds__(1024) k_scan_partials(uint32_t* partials, uint32_t nb, uint32_t* total) {
  __shared__ uint32_t s_warp[33];
  __shared__ uint32_t s_carry;
  if (threadIdx.x == 0) s_carry = 0;
  __syncthreads();
  for (uint32_t base = 0; base < nb; base += 1024 * SCAN_ITEMS) {
    const uint32_t i0 = base + threadIdx.x * SCAN_ITEMS;
    uint32_t v[SCAN_ITEMS];
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) { v[k] = (i0 + k < nb) ? partials[i0 + k] : 0u; s += v[k]; }
    uint32_t tot;
    uint32_t ex = block_exclusive_scan_1024(s, s_warp, &tot) + s_carry;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
      if (i0 + k < nb) partials[i0 + k] = ex;
      ex += v[k];
    }
    __syncthreads();
    if (threadIdx.x == 0) s_carry += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = s_carry;
}

__global__ void __launch_bounds__(1024) k_scan_down(const uint32_t* in, uint64_t N, const uint32_t* partials,
                                                    uint32_t* out) {
  __shared__ uint32_t s_warp[33];
  const uint64_t base = (uint64_t)blockIdx.x * SCAN_BLOCK + (uint64_t)threadIdx.x * SCAN_ITEMS;
  uint32_t v[SCAN_ITEMS];
  uint32_t s = 0;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k) { v[k] = (base + k < N) ? in[base + k] : 0u; s += v[k]; }
  uint32_t ex = block_exclusive_scan_1024(s, s_warp, nullptr) + partials[blockIdx.x];
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    if (base + k < N) out[base + k] = ex;
    ex += v[k];
  }
}

uint32_t scan_partials_needed(uint64_t N) { return (uint32_t)((N + SCAN_BLOCK - 1) / SCAN_BLOCK); }

void launch_exclusive_scan(const uint32_t* in, uint64_t N, uint32_t* out, uint32_t* partials, uint32_t* total,
                           cudaStream_t s) {
  const uint32_t nb = scan_partials_needed(N);
  if (nb == 0) { cudaMemsetAsync(total, 0, 4, s); return; }
  k_scan_reduce<<<nb, 1024, 0, s>>>(in, N, partials);
  k_scan_partials<<<1, 1024, 0, s>>>(partials, nb, total);
  k_scan_down<<<nb, 1024, 0, s>>>(in, N, partials, out);
}

// ---------------------------------------------------------------------------
// Onesweep radix sort.
// ---------------------------------------------------------------------------
constexpr int RS_THREADS = 256;
constexpr int RS_WARPS = RS_THREADS / 32;
constexpr int RS_ITEMS = GS_SORT_ITEMS;
constexpr int RS_TILE = RS_THREADS * RS_ITEMS;  // entries per block
static_assert(RS_TILE == SORT_BLOCK_ENTRIES, "look-back buffers are sized by SORT_BLOCK_ENTRIES");
constexpr int RS_MAX_PASSES = 8;
constexpr uint32_t FLAG_AGG = 1u, FLAG_INC = 2u;
constexpr uint32_t LOOKBACK_SPIN_LIMIT = 1u << 22;

// Histogram of every digit position: one read of all keys (DROP: all-ones
// keys are not counted; the kept ones are counted into nKept).
template <typename KT, bool DROP>
__global__ void __launch_bounds__(256) k_radix_hist(RadixHistArgs a) {
  __shared__ uint32_t h[RS_MAX_PASSES][256];
  for (int i = threadIdx.x; i < RS_MAX_PASSES * 256; i += blockDim.x) (&h[0][0])[i] = 0;
  __syncthreads();
  const uint32_t N = *a.nItems;
  const KT* keys = static_cast<const KT*>(a.keys);
  // four keys per thread in flight, then their digits counted
  const uint32_t stride = gridDim.x * blockDim.x;
  const KT ALL = ~KT(0);
  uint32_t kept = 0;
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  for (; i + 3 * stride < N; i += 4 * stride) {
    const KT k0 = keys[i], k1 = keys[i + stride], k2 = keys[i + 2 * stride], k3 = keys[i + 3 * stride];
    const bool u0 = !DROP || k0 != ALL, u1 = !DROP || k1 != ALL, u2 = !DROP || k2 != ALL, u3 = !DROP || k3 != ALL;
    kept += (uint32_t)u0 + (uint32_t)u1 + (uint32_t)u2 + (uint32_t)u3;
    for (int p = 0; p < a.passes; ++p) {
      const int sh = 8 * p;
      if (u0) atomicAdd(&h[p][(k0 >> sh) & 0xFF], 1u);
      if (u1) atomicAdd(&h[p][(k1 >> sh) & 0xFF], 1u);
      if (u2) atomicAdd(&h[p][(k2 >> sh) & 0xFF], 1u);
      if (u3) atomicAdd(&h[p][(k3 >> sh) & 0xFF], 1u);
    }
  }
  for (; i < N; i += stride) {
    const KT k = keys[i];
    if (DROP && k == ALL) continue;
    ++kept;
    for (int p = 0; p < a.passes; ++p) atomicAdd(&h[p][(k >> (8 * p)) & 0xFF], 1u);
  }
  if (DROP) {
    const uint32_t wk = __reduce_add_sync(0xFFFFFFFFu, kept);
    if ((threadIdx.x & 31) == 0 && wk) atomicAdd(a.nKept, wk);
  }
  __syncthreads();
  for (int p = 0; p < a.passes; ++p)
    for (int d = threadIdx.x; d < 256; d += blockDim.x)
      if (h[p][d]) atomicAdd(&a.hist[p * 256 + d], h[p][d]);
  if (blockIdx.x == 0 && threadIdx.x == 0) a.epoch[0] = a.epoch[0] + 1u;
}

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Digit ranking inside a warp (stable: items in order, lanes in order).
// Ballot form: eight votes on the digit's bits intersect to the lanes that
// share it.  OR form (ORM): every lane sets its bit in a shared-memory word
// of its digit and reads the word back, so one shared atomic and two loads
// replace the eight votes and their bit tests; lanes with equal digits hit
// the same word, so it pays where a warp's digits are spread (tile ids) and
// not where most of them are equal (the top bytes of depths).
template <typename KT, bool DROP = false, bool ORM = false>
#ifndef GS_SORT_MIN_BLOCKS
#define GS_SORT_MIN_BLOCKS 3  // resident blocks per SM the register allocation must allow
#endif
__global__ void __launch_bounds__(RS_THREADS, GS_SORT_MIN_BLOCKS) k_onesweep(OnesweepArgs a) {
  extern __shared__ __align__(16) unsigned char rs_dyn[];
  KT* s_keys = reinterpret_cast<KT*>(rs_dyn);                                    // RS_TILE keys
  uint32_t* s_vals = reinterpret_cast<uint32_t*>(rs_dyn + RS_TILE * sizeof(KT));  // RS_TILE values
  const KT* keysIn = static_cast<const KT*>(a.keysIn);
  KT* keysOut = static_cast<KT*>(a.keysOut);
  __shared__ uint32_t s_whist[RS_WARPS][256];
  __shared__ uint32_t s_count[256];     // this block's count per digit
  __shared__ uint32_t s_run[256];       // the same, kept for the look-back
  __shared__ uint32_t s_local[256];     // exclusive prefix of s_count over digits
  __shared__ uint32_t s_gbase[256];     // global start of this block's run per digit
  __shared__ uint32_t s_dbase[256];     // exclusive scan of the pass histogram
  __shared__ uint32_t s_warp[33];
  __shared__ uint32_t s_tile;
  __shared__ uint32_t s_match[ORM ? RS_WARPS : 1][256];  // OR form: per warp, lanes holding each digit

  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const uint32_t N = *a.nItems;
  const uint32_t numTiles = (N + RS_TILE - 1) / RS_TILE;
  const uint32_t tag = a.epoch[0] * RS_MAX_PASSES + (uint32_t)a.pass + 1u;
  const int shift = 8 * a.pass;

  if (ORM) {  // the words return to zero after every item, so once per launch
#pragma unroll
    for (int w = 0; w < RS_WARPS; ++w) s_match[ORM ? w : 0][tid] = 0u;
  }
  // global digit bases: exclusive scan of this pass's histogram (256 threads)
  {
    const uint32_t hv = a.hist[a.pass * 256 + tid];
    uint32_t inc = hv;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xFFFFFFFFu, inc, o);
      if (lane >= o) inc += y;
    }
    if (lane == 31) s_warp[wid] = inc;
    __syncthreads();
    if (wid == 0) {
      uint32_t w = lane < RS_WARPS ? s_warp[lane] : 0u, wi = w;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xFFFFFFFFu, wi, o);
        if (lane >= o) wi += y;
      }
      if (lane < RS_WARPS) s_warp[lane] = wi - w;
    }
    __syncthreads();
    s_dbase[tid] = s_warp[wid] + inc - hv;
    __syncthreads();
  }

  for (;;) {
    if (tid == 0) s_tile = atomicAdd(a.tileCounter + a.pass, 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    if (tile >= numTiles) break;
    const uint32_t base = tile * RS_TILE;

    // load: warp w holds entries [base + w*512, +512), item j at lane l
    KT key[RS_ITEMS];
    uint32_t val[RS_ITEMS];
    uint32_t dig[RS_ITEMS];
#pragma unroll
    for (int j = 0; j < RS_ITEMS; ++j) {
      const uint32_t idx = base + wid * (32 * RS_ITEMS) + j * 32 + lane;
      if (idx < N) {
        key[j] = keysIn[idx];
        val[j] = a.valsIn[idx];
        dig[j] = DROP && key[j] == ~KT(0) ? 0x100u : (uint32_t)(key[j] >> shift) & 0xFFu;
      } else {
        key[j] = 0; val[j] = 0; dig[j] = 0x100u;
      }
    }
#pragma unroll
    for (int k = 0; k < 256 / 32; ++k) s_whist[wid][lane + 32 * k] = 0;
    __syncwarp();

    // rank within the warp, items in order, lanes in order
    uint32_t rank[RS_ITEMS];
    const uint32_t ltm = lanemask_lt();
    if (ORM) {
      uint32_t* wm = s_match[ORM ? wid : 0];
#pragma unroll
      for (int j = 0; j < RS_ITEMS; ++j) {
        const bool valid = dig[j] < 0x100u;
        if (valid) atomicOr(&wm[dig[j]], 1u << lane);
        __syncwarp();
        uint32_t peers = 0, pre = 0;
        if (valid) { peers = wm[dig[j]]; pre = s_whist[wid][dig[j]]; }
        __syncwarp();
        if (valid) {
          const uint32_t below = __popc(peers & ltm);
          rank[j] = pre + below;
          if (below == 0) {  // the digit's first lane advances its count and clears the word
            s_whist[wid][dig[j]] = pre + __popc(peers);
            wm[dig[j]] = 0u;
          }
        } else {
          rank[j] = 0;
        }
        __syncwarp();
      }
    } else {
#pragma unroll
      for (int j = 0; j < RS_ITEMS; ++j) {
        const bool valid = dig[j] < 0x100u;
        uint32_t peers = __ballot_sync(0xFFFFFFFFu, valid);
#pragma unroll
        for (int b = 0; b < 8; ++b) {
          const uint32_t bal = __ballot_sync(0xFFFFFFFFu, (dig[j] >> b) & 1u);
          peers &= ((dig[j] >> b) & 1u) ? bal : ~bal;
        }
        uint32_t pre = 0;
        if (valid) pre = s_whist[wid][dig[j]];
        __syncwarp();
        if (valid) {
          const uint32_t below = __popc(peers & ltm);
          rank[j] = pre + below;
          if (below == 0) s_whist[wid][dig[j]] = pre + __popc(peers);
        } else {
          rank[j] = 0;
        }
        __syncwarp();
      }
    }
    __syncthreads();

    // per digit: exclusive scan across warps, block count
    {
      const int d = tid;
      uint32_t run = 0;
#pragma unroll
      for (int w = 0; w < RS_WARPS; ++w) {
        const uint32_t c = s_whist[w][d];
        s_whist[w][d] = run;
        run += c;
      }
      s_count[d] = run;

      // publish this block's count (the whole prefix for block 0) at once, so
      // the blocks behind it can proceed while it stages its entries
      cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> my(
          *reinterpret_cast<unsigned long long*>(a.status + (size_t)tile * 256 + d));
      my.store(((unsigned long long)tag << 32) |
                   ((unsigned long long)(tile == 0 ? FLAG_INC : FLAG_AGG) << 30) | run,
               cuda::memory_order_relaxed);
      s_run[d] = run;
    }
    // exclusive scan of s_count over digits -> s_local
    {
      const uint32_t cv = s_count[tid];
      uint32_t inc = cv;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xFFFFFFFFu, inc, o);
        if (lane >= o) inc += y;
      }
      __syncthreads();
      if (lane == 31) s_warp[wid] = inc;
      __syncthreads();
      if (wid == 0) {
        uint32_t w = lane < RS_WARPS ? s_warp[lane] : 0u, wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          uint32_t y = __shfl_up_sync(0xFFFFFFFFu, wi, o);
          if (lane >= o) wi += y;
        }
        if (lane < RS_WARPS) s_warp[lane] = wi - w;
      }
      __syncthreads();
      s_local[tid] = s_warp[wid] + inc - cv;
    }
    __syncthreads();

    // stage in shared memory in sorted order
#pragma unroll
    for (int j = 0; j < RS_ITEMS; ++j) {
      if (dig[j] < 0x100u) {
        const uint32_t pos = s_local[dig[j]] + s_whist[wid][dig[j]] + rank[j];
        s_keys[pos] = key[j];
        s_vals[pos] = val[j];
      }
    }
    __syncthreads();
    // decoupled look-back for digit d (the staged entries wait in shared
    // memory, so no per-entry registers are held while it spins)
    {
      const int d = tid;
      const uint32_t run = s_run[d];
      cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> my(
          *reinterpret_cast<unsigned long long*>(a.status + (size_t)tile * 256 + d));
      uint32_t excl = 0;
      if (tile != 0) {
        // LB predecessors' words are loaded at once and summed nearest first
        // up to the first inclusive one; a word not yet published ends the
        // round there, and the next round starts from it
        constexpr int LB = 4;
        int64_t t = (int64_t)tile - 1;
        uint32_t spins = 0;
        while (t >= 0) {
          unsigned long long w[LB];
#pragma unroll
          for (int k = 0; k < LB; ++k) {
            w[k] = 0ull;
            if (t - k >= 0) {
              cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> pr(
                  *reinterpret_cast<unsigned long long*>(a.status + (size_t)(t - k) * 256 + d));
              w[k] = pr.load(cuda::memory_order_relaxed);
            }
          }
          int used = 0, state = 0;  // state: 0 keep going, 1 inclusive word found, 2 a word not ready
#pragma unroll
          for (int k = 0; k < LB; ++k) {
            if (state == 0 && t - k >= 0) {
              const uint32_t stag = (uint32_t)(w[k] >> 32);
              const uint32_t flag = (uint32_t)(w[k] >> 30) & 3u;
              if (stag != tag || flag == 0) {
                state = 2;
              } else {
                excl += (uint32_t)(w[k] & 0x3FFFFFFFull);
                ++used;
                if (flag == FLAG_INC) state = 1;
              }
            }
          }
          if (state == 1) break;
          t -= used;
          if (state == 2) {
            if (++spins > a.spinLimit) { atomicOr(a.statusWord, ST_LOOKBACK_TIMEOUT); break; }
            __nanosleep(32);
          }
        }
        my.store(((unsigned long long)tag << 32) | ((unsigned long long)FLAG_INC << 30) | (excl + run),
                 cuda::memory_order_relaxed);
      }
      s_gbase[d] = s_dbase[d] + excl;
    }
    __syncthreads();
    // the block's entries (DROP: the kept ones), staged first to last
    const uint32_t cnt = DROP ? s_local[255] + s_run[255] : min((uint32_t)RS_TILE, N - base);
    // scatter, every round unrolled so the shared-memory reads of all rounds
    // are in flight together
#pragma unroll
    for (int r = 0; r < RS_ITEMS; ++r) {
      const uint32_t i = (uint32_t)tid + (uint32_t)r * RS_THREADS;
      if (i < cnt) {
        const KT k = s_keys[i];
        const uint32_t d = (uint32_t)(k >> shift) & 0xFFu;
        const uint32_t g = s_gbase[d] + (i - s_local[d]);
        if (keysOut) keysOut[g] = k;
        a.valsOut[g] = s_vals[i];
      }
    }
    __syncthreads();
  }
}

template <typename KT>
constexpr size_t rs_dyn_smem() { return (size_t)RS_TILE * (sizeof(KT) + 4); }

int onesweep_grid(int device) {
  int sms = 0, per32 = 0, per64 = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  cudaFuncSetAttribute(k_onesweep<uint32_t>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)rs_dyn_smem<uint32_t>());
  cudaFuncSetAttribute(k_onesweep<uint32_t, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)rs_dyn_smem<uint32_t>());
  cudaFuncSetAttribute(k_onesweep<uint64_t>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)rs_dyn_smem<uint64_t>());
  cudaFuncSetAttribute(k_onesweep<uint32_t, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)rs_dyn_smem<uint32_t>());
  cudaFuncSetAttribute(k_onesweep<uint32_t, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)rs_dyn_smem<uint32_t>());
  int perOr = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per32, k_onesweep<uint32_t>, RS_THREADS, rs_dyn_smem<uint32_t>());
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per64, k_onesweep<uint64_t>, RS_THREADS, rs_dyn_smem<uint64_t>());
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perOr, k_onesweep<uint32_t, false, true>, RS_THREADS,
                                                rs_dyn_smem<uint32_t>());
  int perSm = per32 < per64 ? per32 : per64;  // one grid size that is fully resident for every form
  if (perOr < perSm) perSm = perOr;
  if (perSm < 1) perSm = 1;
  return sms * perSm;
}

// Sorts N = *nItems entries (N known only on the device) with keys of
// keyBytes (4 or 8) on key bits [0, 8*passes).  Result lands in
// (keys,vals)[passes & 1] of the ping-pong pair.  hist must hold passes*256
// u32, tileCounter passes u32; the caller clears both before the call.
template <typename KT>
static void radix_sort_t(const RadixSortArgs& a, cudaStream_t s) {
  RadixHistArgs h;
  h.keys = a.keys[0];
  h.nItems = a.nItems;
  h.hist = a.hist;
  h.passes = a.passes;
  h.epoch = a.epoch;
  const bool drop = a.nKept != nullptr && sizeof(KT) == 4;
  h.nKept = drop ? a.nKept : nullptr;
  if (drop) k_radix_hist<KT, true><<<a.histGrid, 256, 0, s>>>(h);
  else k_radix_hist<KT, false><<<a.histGrid, 256, 0, s>>>(h);
  for (int p = 0; p < a.passes; ++p) {
    OnesweepArgs o;
    o.keysIn = a.keys[p & 1];
    o.valsIn = a.vals[p & 1];
    o.keysOut = (p == a.passes - 1 && !a.keepKeys) ? nullptr : a.keys[(p + 1) & 1];
    o.valsOut = a.vals[(p + 1) & 1];
    // the first pass reads every key and drops the all-ones ones; the later
    // passes sort only the kept keys
    o.nItems = drop && p > 0 ? a.nKept : a.nItems;
    o.dropAllOnes = drop && p == 0 ? 1 : 0;
    o.hist = a.hist;
    o.tileCounter = a.tileCounter;
    o.status = a.status;
    o.statusWord = a.statusWord;
    o.epoch = a.epoch;
    o.pass = p;
    o.spinLimit = LOOKBACK_SPIN_LIMIT;
    const bool orForm = sizeof(KT) == 4 && ((a.orPasses >> p) & 1u);
    if (o.dropAllOnes && orForm)
      k_onesweep<uint32_t, true, true><<<a.sweepGrid, RS_THREADS, rs_dyn_smem<uint32_t>(), s>>>(o);
    else if (o.dropAllOnes) k_onesweep<KT, true><<<a.sweepGrid, RS_THREADS, rs_dyn_smem<KT>(), s>>>(o);
    else if (orForm)
      k_onesweep<uint32_t, false, true><<<a.sweepGrid, RS_THREADS, rs_dyn_smem<uint32_t>(), s>>>(o);
    else k_onesweep<KT><<<a.sweepGrid, RS_THREADS, rs_dyn_smem<KT>(), s>>>(o);
  }
}

void launch_radix_sort(const RadixSortArgs& a, cudaStream_t s) {
  if (a.keyBytes == 4) radix_sort_t<uint32_t>(a, s);
  else radix_sort_t<uint64_t>(a, s);
}

// ---------------------------------------------------------------------------
// Failure-detection check: a look-back that can never complete.
// One onesweep pass over 3 blocks of keys with the block counter starting at
// 1, so block 0 is never processed and its status word is never published.
// Blocks 1 and 2 wait on it, give up after `spinLimit` spins, flag
// ST_LOOKBACK_TIMEOUT and finish (their scatter positions use a partial
// prefix, which is smaller than the true one, so every store stays inside
// the buffers).  Nothing hangs; the context stays usable.
// ---------------------------------------------------------------------------
int debug_lookback_timeout(int device, uint32_t spinLimit, uint32_t* statusOut, double* msOut) {
  if (cudaSetDevice(device) != cudaSuccess) return -2;
  const uint32_t n = 3u * RS_TILE;
  uint32_t *keys = nullptr, *vals = nullptr, *outVals = nullptr, *small = nullptr;
  uint64_t* status = nullptr;
  int rc = 0;
  cudaStream_t s = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (cudaMalloc(&keys, n * 4) != cudaSuccess || cudaMalloc(&vals, n * 4) != cudaSuccess ||
      cudaMalloc(&outVals, n * 4) != cudaSuccess || cudaMalloc(&small, 4096 * 4) != cudaSuccess ||
      cudaMalloc(&status, (size_t)8 * 256 * 8) != cudaSuccess || cudaStreamCreate(&s) != cudaSuccess ||
      cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
    rc = -3;
  } else {
    // small: [0, 2048) histograms, [2048, 2056) block counters, 2056 status word, 2057 epoch, 2058 count
    cudaMemsetAsync(keys, 0, n * 4, s);
    cudaMemsetAsync(vals, 0, n * 4, s);
    cudaMemsetAsync(small, 0, 4096 * 4, s);
    cudaMemsetAsync(status, 0, (size_t)8 * 256 * 8, s);
    const uint32_t one = 1u;
    cudaMemcpyAsync(small + 2048, &one, 4, cudaMemcpyHostToDevice, s);  // block 0 is never claimed
    cudaMemcpyAsync(small + 2058, &n, 4, cudaMemcpyHostToDevice, s);
    RadixHistArgs h;
    h.keys = keys; h.nItems = small + 2058; h.hist = small; h.passes = 1; h.epoch = small + 2057;
    h.nKept = nullptr;
    k_radix_hist<uint32_t, false><<<4, 256, 0, s>>>(h);
    OnesweepArgs o;
    o.keysIn = keys; o.valsIn = vals; o.keysOut = nullptr; o.valsOut = outVals;
    o.nItems = small + 2058; o.hist = small; o.tileCounter = small + 2048; o.status = status;
    o.statusWord = small + 2056; o.epoch = small + 2057; o.pass = 0; o.spinLimit = spinLimit;
    o.dropAllOnes = 0;
    cudaFuncSetAttribute(k_onesweep<uint32_t>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)rs_dyn_smem<uint32_t>());
    cudaEventRecord(e0, s);
    k_onesweep<uint32_t><<<3, RS_THREADS, rs_dyn_smem<uint32_t>(), s>>>(o);
    cudaEventRecord(e1, s);
    uint32_t st = 0;
    cudaMemcpyAsync(&st, small + 2056, 4, cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess || cudaGetLastError() != cudaSuccess) rc = -2;
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (statusOut) *statusOut = st;
    if (msOut) *msOut = ms;
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (s) cudaStreamDestroy(s);
  cudaFree(keys); cudaFree(vals); cudaFree(outVals); cudaFree(small); cudaFree(status);
  return rc;
}

}  // namespace gs
