// gs_static_sort.cu -- an allocation-free variant of the tile-entry sort.
//
// The trainer sorts its (tile id, splat id) entries with the onesweep radix
// sort of gs_sort.cu, whose scratch (the second ping-pong buffer, the digit
// histograms, the block counters and the look-back status words) lives in
// buffers the trainer allocates at set-up.  This entry point runs the same
// kernels with all of that scratch in file-scope __device__ arrays sized for
// at most GS_STATIC_SORT_MAX entries, so a call allocates no device or host
// memory.  It serves callers that cannot call cudaMalloc: code whose device
// memory is owned by another runtime's pool, and code on a path where an
// allocation (which may synchronise the device) is not allowed.  Every GPU
// that loads the library holds the arrays (about 8.5 MB) until exit.  In host
// code the arrays' names are host-side stand-ins, never device addresses:
// only the addresses cudaGetSymbolAddress returns are passed to kernels.
//
// Set-up: the first call on a device computes the launch grids (device
// attributes and kernel occupancy) once.  Every call resolves the arrays'
// addresses again with cudaGetSymbolAddress, with the caller's device
// current, so a context that was torn down and made again (which reloads the
// module and may move the arrays) never sees a stale address.  The arrays
// start zeroed whenever the module loads (static storage), which is the state
// the epoch-tagged look-back words need; each call clears only the per-sort
// histograms, block counters and status word.  The scratch is shared by
// every caller, so two calls whose work overlaps in time (different streams
// or host threads) race.
#include <cuda_runtime.h>

#include <mutex>

#include "gs_common.cuh"
#include "gs_kernels.h"
#include "../../include/splat_b200.h"

namespace gs {
namespace {

constexpr uint32_t SS_MAX = GS_STATIC_SORT_MAX;
constexpr uint32_t SS_BLOCK = SORT_BLOCK_ENTRIES;          // entries per onesweep block
constexpr uint32_t SS_STATUS = (SS_MAX / SS_BLOCK + 2) * 256;  // look-back words (block x digit)
constexpr uint32_t SS_HIST = 8 * 256;                      // digit histograms of up to 8 passes
// small words: [0, 2048) histograms, [2048, 2056) block counters,
// 2056 status word, 2057 epoch, 2058 entry count
constexpr uint32_t SS_SMALL = SS_HIST + 8 + 3;
constexpr int SS_MAX_DEVICES = 64;

__device__ __align__(256) uint32_t g_ssKeys[SS_MAX];
__device__ __align__(256) uint32_t g_ssVals[SS_MAX];
__device__ __align__(256) unsigned long long g_ssStatus[SS_STATUS];
__device__ __align__(256) uint32_t g_ssSmall[SS_SMALL];

struct StaticGrids {
  bool ready = false;
  unsigned histGrid = 0, sweepGrid = 0;
};
StaticGrids g_grids[SS_MAX_DEVICES];
std::mutex g_setupMutex;

struct StaticScratch {
  uint32_t* keys = nullptr;
  uint32_t* vals = nullptr;
  uint64_t* status = nullptr;
  uint32_t* small = nullptr;
  unsigned histGrid = 0, sweepGrid = 0;
};

__global__ void k_ss_set_count(uint32_t* word, uint32_t n) { *word = n; }

// The scratch addresses on the current device (looked up on every call) and
// the launch grids (computed once per device).
int static_scratch(int device, StaticScratch* sc) {
  if (device < 0 || device >= SS_MAX_DEVICES) return GS_E_INVALID;
  void* p = nullptr;
  if (cudaGetSymbolAddress(&p, g_ssKeys) != cudaSuccess) return GS_E_CUDA;
  sc->keys = static_cast<uint32_t*>(p);
  if (cudaGetSymbolAddress(&p, g_ssVals) != cudaSuccess) return GS_E_CUDA;
  sc->vals = static_cast<uint32_t*>(p);
  if (cudaGetSymbolAddress(&p, g_ssStatus) != cudaSuccess) return GS_E_CUDA;
  sc->status = static_cast<uint64_t*>(p);
  if (cudaGetSymbolAddress(&p, g_ssSmall) != cudaSuccess) return GS_E_CUDA;
  sc->small = static_cast<uint32_t*>(p);
  std::lock_guard<std::mutex> lock(g_setupMutex);
  StaticGrids& g = g_grids[device];
  if (!g.ready) {
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return GS_E_CUDA;
    g.histGrid = (unsigned)(sms * 4);
    g.sweepGrid = (unsigned)onesweep_grid(device);
    if (g.sweepGrid == 0) return GS_E_CUDA;
    g.ready = true;
  }
  sc->histGrid = g.histGrid;
  sc->sweepGrid = g.sweepGrid;
  return GS_OK;
}

}  // namespace
}  // namespace gs

using namespace gs;

extern "C" int gs_sort_entries_static(uint32_t* keys, uint32_t* vals, uint32_t n, uint32_t keyBits, void* stream) {
  if (n > GS_STATIC_SORT_MAX) return GS_E_LIMIT;
  if (keyBits < 1 || keyBits > 32) return GS_E_INVALID;
  if (n == 0) return GS_OK;
  if (!keys || !vals) return GS_E_INVALID;
  // an error an earlier call on this thread left pending is reported, and
  // left pending, rather than taken for a failure of this call's launches
  if (cudaPeekAtLastError() != cudaSuccess) return GS_E_CUDA;
  int device = -1;
  if (cudaGetDevice(&device) != cudaSuccess) return GS_E_CUDA;
  StaticScratch scr;
  const int rc = static_scratch(device, &scr);
  if (rc != GS_OK) return rc;
  StaticScratch* sc = &scr;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  uint32_t* statusWord = sc->small + SS_HIST + 8;
  uint32_t* epoch = sc->small + SS_HIST + 9;
  uint32_t* count = sc->small + SS_HIST + 10;
  // per sort: histograms, block counters and the status word start at zero
  if (cudaMemsetAsync(sc->small, 0, (SS_HIST + 8 + 1) * 4, s) != cudaSuccess) return GS_E_CUDA;
  k_ss_set_count<<<1, 1, 0, s>>>(count, n);
  RadixSortArgs a{};
  a.keys[0] = keys; a.keys[1] = sc->keys;
  a.vals[0] = vals; a.vals[1] = sc->vals;
  a.keyBytes = 4;
  a.nItems = count;
  a.hist = sc->small;
  a.tileCounter = sc->small + SS_HIST;
  a.status = sc->status;
  a.statusWord = statusWord;
  a.epoch = epoch;
  a.passes = (int)((keyBits + 7) / 8);
  a.keepKeys = true;
  a.histGrid = sc->histGrid;
  a.sweepGrid = sc->sweepGrid;
  launch_radix_sort(a, s);
  if (a.passes & 1) {  // the result is in the scratch half of the ping-pong pair
    if (cudaMemcpyAsync(keys, sc->keys, (size_t)n * 4, cudaMemcpyDeviceToDevice, s) != cudaSuccess) return GS_E_CUDA;
    if (cudaMemcpyAsync(vals, sc->vals, (size_t)n * 4, cudaMemcpyDeviceToDevice, s) != cudaSuccess) return GS_E_CUDA;
  }
  if (cudaGetLastError() != cudaSuccess) return GS_E_CUDA;
  uint32_t st = 0;
  if (cudaMemcpyAsync(&st, statusWord, 4, cudaMemcpyDeviceToHost, s) != cudaSuccess) return GS_E_CUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return GS_E_CUDA;
  return st ? GS_E_DEVICE : GS_OK;
}
