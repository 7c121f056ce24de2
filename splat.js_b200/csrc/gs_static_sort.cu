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
// Set-up: the first call on a device resolves the arrays' addresses with
// cudaGetSymbolAddress (with that device current) and clears the look-back
// status words once; later calls on that device only clear the per-sort
// histograms and counters.  The scratch is shared by every caller, so two
// calls whose work overlaps in time (different streams or host threads) race.
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

struct StaticScratch {
  bool ready = false;
  uint32_t* keys = nullptr;
  uint32_t* vals = nullptr;
  uint64_t* status = nullptr;
  uint32_t* small = nullptr;
  unsigned histGrid = 0, sweepGrid = 0;
};
StaticScratch g_scratch[SS_MAX_DEVICES];
std::mutex g_setupMutex;

__global__ void k_ss_set_count(uint32_t* word, uint32_t n) { *word = n; }

// Resolves the scratch of the current device (once per device).
int static_scratch(int device, StaticScratch** out) {
  if (device < 0 || device >= SS_MAX_DEVICES) return GS_E_INVALID;
  std::lock_guard<std::mutex> lock(g_setupMutex);
  StaticScratch& sc = g_scratch[device];
  if (!sc.ready) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_ssKeys) != cudaSuccess) return GS_E_CUDA;
    sc.keys = static_cast<uint32_t*>(p);
    if (cudaGetSymbolAddress(&p, g_ssVals) != cudaSuccess) return GS_E_CUDA;
    sc.vals = static_cast<uint32_t*>(p);
    if (cudaGetSymbolAddress(&p, g_ssStatus) != cudaSuccess) return GS_E_CUDA;
    sc.status = static_cast<uint64_t*>(p);
    if (cudaGetSymbolAddress(&p, g_ssSmall) != cudaSuccess) return GS_E_CUDA;
    sc.small = static_cast<uint32_t*>(p);
    // status words and the epoch start at zero; synchronous, before first use
    if (cudaMemset(sc.status, 0, sizeof(g_ssStatus)) != cudaSuccess) return GS_E_CUDA;
    if (cudaMemset(sc.small, 0, sizeof(g_ssSmall)) != cudaSuccess) return GS_E_CUDA;
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return GS_E_CUDA;
    sc.histGrid = (unsigned)(sms * 4);
    sc.sweepGrid = (unsigned)onesweep_grid(device);
    if (cudaDeviceSynchronize() != cudaSuccess) return GS_E_CUDA;
    sc.ready = true;
  }
  *out = &sc;
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
  int device = -1;
  if (cudaGetDevice(&device) != cudaSuccess) return GS_E_CUDA;
  StaticScratch* sc = nullptr;
  const int rc = static_scratch(device, &sc);
  if (rc != GS_OK) return rc;
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
