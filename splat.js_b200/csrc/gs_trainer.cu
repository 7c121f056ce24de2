// gs_trainer.cu -- host runtime of libsplat_b200.so: the C ABI declared in
// include/splat_b200.h, over the kernels of gs_project / gs_sort / gs_raster
// / gs_chain.
//
// It restates GSTrainer's host logic (src/gs/trainer.js): setup's buffer
// sizing and RGBA8 target packing (:100-355), the camera record (:357-372),
// stepOnce's schedules (:398-429), readLoss (:615-631), readGaussians
// (:797-817), renderView (:634-655), _evalPass (:542-574).  The step itself
// is one stream of kernels, optionally replayed from a CUDA graph captured
// once per step shape (number of views, their resolutions, splat count).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/splat_b200.h"
#include "gs_kernels.h"

using namespace gs;

namespace {

constexpr int MAXB = MAX_VIEWS;  // hard upper bound of views per batch
constexpr int RING = 8;      // pinned step-parameter slots

struct StepParams {
  AdamHP hp;
  uint32_t gridBase[MAXB];
  uint32_t itemCount;        // V * n presort items of this step
  DevCam cams[MAXB];
};

thread_local std::string g_createError;

struct Shape {
  int V;
  int w[MAXB], h[MAXB];
  uint32_t n;
  int mode;       // 1 forward, 3 train
  int chain;      // 0 none, 1 chain (+ Adam when adam)
  int adam;
  int grads;      // write gradF/shGrad readout
  int variant;
  int tile;       // raster tile edge
  int depth;      // splat-batch depth
  int cull;       // tile lists culled by the ellipse/tile test
  bool operator<(const Shape& o) const { return std::memcmp(this, &o, sizeof(Shape)) < 0; }
};

}  // namespace

struct gs_trainer {
  gs_options o{};
  std::string err;
  int device = 0;
  cudaStream_t stream = nullptr;
  int sms = 148;
  bool ready = false;

  // ---- host state (GSTrainer fields) ----
  uint32_t n = 0, cap = 0, K = 0, ncams = 0, iter = 0, horizon = 60000, growLimit = 0;
  uint64_t pixelsSeen = 0, entriesCap = 12000000ull, overflowTiles = 0;
  uint64_t rngState[2] = {0x2BD3AB5E4C1D2B3Bull, 0x9C3F7A1E0D5B6C47ull};  // built-in refine generator
  double sceneRadius = 1.0;
  double basePosLr = 0.0;
  float lrs[16] = {};
  float minLS = 0, maxLS = 0;
  std::vector<gs_camera> cams;
  std::vector<uint32_t> camOffset;
  std::vector<float> camActiveSh;
  uint32_t maxTiles = 0, maxPix = 0, maxGrid = 0;
  uint64_t totalPix = 0;

  // ---- device buffers ----
  float *params = nullptr, *m = nullptr, *v = nullptr, *sh = nullptr, *shM = nullptr, *shV = nullptr;
  RenderRec* recs = nullptr;
  uint2* rect = nullptr;
  uint32_t *counts = nullptr, *offsets = nullptr;
  float4* cullRecs = nullptr;
  uint4* itemRecs = nullptr;
  float* viewGrad = nullptr;
  uint32_t* visList = nullptr;
  uint4* itemSrc = nullptr;
  int32_t* gradP = nullptr;
  int32_t* diffGrid = nullptr;
  uint32_t* tileCnt = nullptr;
  uint8_t* dropped = nullptr;
  uint2* ranges = nullptr;
  uint32_t* viewDrops = nullptr;
  uint32_t* workOrder = nullptr;
  uint32_t* keys[2] = {nullptr, nullptr};     // entries: global tile id
  uint32_t* vals[2] = {nullptr, nullptr};     // entries: splat id
  uint64_t* pkeys[2] = {nullptr, nullptr};    // presort keys (u32 depth bits); refine's u64 donor keys
  uint32_t* pvals[2] = {nullptr, nullptr};    // presort items: slot = view * n + splat
  uint32_t* viewTotal = nullptr;
  uint64_t capacity = 0;
  uint32_t* small = nullptr;  // [0,2048) hist | [2048,2056) tileCounter | 2056 workCounter | 2057 totalEntries | 2058 scanTotal | 2059 epoch | 2060 status
  uint64_t* lbStatus = nullptr;
  // PLY export scratch, grown on demand and kept: camera positions, records
  double* plyCam = nullptr;
  size_t plyCamCap = 0;
  float* plyOut = nullptr;
  size_t plyOutCap = 0;
  uint32_t* scanPartials = nullptr;
  float4* outImg = nullptr;
  float* finalT = nullptr;
  uint32_t* endIdx = nullptr;
  uint32_t* targets = nullptr;
  uint32_t* stats = nullptr;
  int32_t* gradCam = nullptr;
  float* gradFOut = nullptr;
  float* shGradOut = nullptr;
  float* tStore = nullptr;
  size_t tStoreCap = 0;
  StepParams* dParams = nullptr;
  StepParams* hRing = nullptr;
  cudaEvent_t ringEv[RING] = {};
  int ringPos = 0;
  std::vector<void*> allocs;

  // ---- last raster (for introspection) ----
  int lastV = 0;
  DevCam lastCams[MAXB];
  int lastPasses = 0;
  uint32_t lastLaunches = 0;
  uint32_t lastTotalTiles = 0;

  // ---- refine scratch (allocated at the first refine) ----
  struct {
    uint32_t *deadFlag = nullptr, *donorFlag = nullptr, *deadOff = nullptr, *donorOff = nullptr;
    uint32_t *deadList = nullptr, *donorList = nullptr, *splitSeq = nullptr, *partials = nullptr;
    uint32_t* counts = nullptr;
    RefineSpawn* plan = nullptr;
  } rf;
  bool camIdxZero = false;   // after growth every training view uses gradCam row 0 (trainer.js:768)

  std::map<Shape, cudaGraphExec_t> graphs;
  int histGrid = 0, sweepGrid = 0;
  int tile = 16;                 // current raster tile edge (8, 16 or 32)
  int rasterPerSm[3][3][2] = {};  // occupancy per (tile, batch depth, forward-only / train)

  // ---- measurement ----
  cudaStream_t ownStream = nullptr;
  bool profiling = false;
  std::vector<cudaEvent_t> evPool;       // recorded events awaiting read, 2 per timed phase
  std::vector<int> evPhase;
  double profMs[4] = {0, 0, 0, 0};
  uint32_t profN[4] = {0, 0, 0, 0};
};

#define GS_CK(call)                                                                   \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess) {                                                          \
      h->err = std::string(#call) + ": " + cudaGetErrorString(e_);                    \
      return GS_E_CUDA;                                                               \
    }                                                                                 \
  } while (0)

static int fail(gs_trainer* h, int code, const std::string& msg) {
  h->err = msg;
  return code;
}

// refine()'s default rng (the reference defaults to Math.random, a native
// generator): xorshift128+ (S. Vigna, "Further scramblings of Marsaglia's
// xorshift generators", J. Comput. Appl. Math. 315, 2017; shifts 23, 18, 5),
// 53 high bits of each output as a double in [0, 1).  The state lives in the
// handle, starts from the same two words for every handle and continues
// across refine calls, so a run is reproducible; the draws cost nanoseconds
// instead of a call into the caller's language per draw.
static double builtin_rng(void* ctx) {
  uint64_t* st = static_cast<gs_trainer*>(ctx)->rngState;
  uint64_t s1 = st[0];
  const uint64_t s0 = st[1];
  const uint64_t out = s0 + s1;
  st[0] = s0;
  s1 ^= s1 << 23;
  st[1] = s1 ^ s0 ^ (s1 >> 18) ^ (s0 >> 5);
  return (double)(out >> 11) * 0x1.0p-53;
}

template <class T>
static int dalloc(gs_trainer* h, T** p, size_t count) {
  const size_t bytes = std::max<size_t>(count * sizeof(T), 16);
  void* q = nullptr;
  cudaError_t e = cudaMalloc(&q, bytes);
  if (e != cudaSuccess) {
    h->err = "cudaMalloc(" + std::to_string(bytes) + " bytes): " + cudaGetErrorString(e);
    return GS_E_NOMEM;
  }
  h->allocs.push_back(q);
  *p = static_cast<T*>(q);
  return GS_OK;
}

static void free_all(gs_trainer* h) {
  for (auto& kv : h->graphs) cudaGraphExecDestroy(kv.second);
  h->graphs.clear();
  for (void* p : h->allocs) cudaFree(p);
  h->allocs.clear();
  if (h->hRing) { cudaFreeHost(h->hRing); h->hRing = nullptr; }
  if (h->tStore) { cudaFree(h->tStore); h->tStore = nullptr; h->tStoreCap = 0; }
  if (h->plyCam) { cudaFree(h->plyCam); h->plyCam = nullptr; h->plyCamCap = 0; }
  if (h->plyOut) { cudaFree(h->plyOut); h->plyOut = nullptr; h->plyOutCap = 0; }
  h->rf = {};
  h->ready = false;
}

static inline uint32_t ceil_div(uint32_t a, uint32_t b) { return (a + b - 1) / b; }

// _camUniform (trainer.js:357-372): the view record kernels read.
static DevCam make_cam(const gs_trainer* h, const gs_camera& c, int train, uint32_t offset, uint32_t camIdx,
                       float activeSh) {
  DevCam d{};
  for (int k = 0; k < 9; ++k) d.R[k] = c.R[k];
  for (int k = 0; k < 3; ++k) { d.t[k] = c.t[k]; d.bg[k] = 0.0f; }
  d.nearz = 0.05f;
  d.f = c.f; d.cx = c.cx; d.cy = c.cy;
  d.gain = (float)std::exp(c.g);
  d.bias = (float)c.b;
  d.activeSh = activeSh;
  d.W = c.w; d.H = c.h;
  d.tilesX = (int)ceil_div((uint32_t)c.w, (uint32_t)h->tile);
  d.tilesY = (int)ceil_div((uint32_t)c.h, (uint32_t)h->tile);
  d.offset = offset;
  d.camIdx = camIdx;
  d.ncams = h->ncams;
  d.train = train;
  return d;
}

extern "C" {

int gs_abi_version(void) { return GS_ABI_VERSION; }

int gs_default_options(gs_options* o) {
  if (!o) return GS_E_INVALID;
  std::memset(o, 0, sizeof(*o));
  o->eCut = 4.5f;
  o->aMin = 0.0039f;
  o->radClamp = 1.0f;
  o->anisoReg = 0.005f;
  o->shDeg = 2;
  o->tileGrad = 1;
  o->entriesCap = 0;
  o->maxSplats = 0;
  o->capMult = 4.0;
  o->maxIters = 60000;
  o->minScale = 1e-4;
  o->opacityReg = 0.01f;
  o->shLr = 1.25e-4f;
  o->growRate = 0.15;
  o->growUntil = -1.0;
  o->tile = 16;
  o->batchDepth = 64;
  o->maxBatch = 8;
  o->backwardVariant = 0;
  o->persistent = 1;
  o->useGraphs = 1;
  o->device = 0;
  o->tileCull = 1;
  o->donorSampling = 0;
  return GS_OK;
}

const char* gs_last_error(const gs_trainer* h) { return h ? h->err.c_str() : g_createError.c_str(); }

int gs_create(const gs_options* opts, gs_trainer** out) {
  if (!out) return GS_E_INVALID;
  *out = nullptr;
  gs_options o;
  if (opts) o = *opts; else gs_default_options(&o);
  if (o.shDeg < 0 || o.shDeg > 3) { g_createError = "shDeg must be 0..3"; return GS_E_INVALID; }
  // exp(-e) is evaluated for e <= eCut; the canonical exp is defined on |x| <= 87
  if (!(o.eCut > 0.0f && o.eCut <= 80.0f)) { g_createError = "eCut must be in (0, 80]"; return GS_E_INVALID; }
  if (o.tile != 8 && o.tile != 16 && o.tile != 32) { g_createError = "tile must be 8, 16 or 32"; return GS_E_INVALID; }
  if (o.tileCull != 0 && o.tileCull != 1) { g_createError = "tileCull must be 0 or 1"; return GS_E_INVALID; }
  if (o.donorSampling != 0 && o.donorSampling != 1) {
    g_createError = "donorSampling must be 0 or 1";
    return GS_E_INVALID;
  }
  if (o.batchDepth != 64 && o.batchDepth != 128 && o.batchDepth != 256) {
    g_createError = "batchDepth must be 64, 128 or 256";
    return GS_E_INVALID;
  }
  if (o.maxBatch < 1 || o.maxBatch > MAXB) { g_createError = "maxBatch must be 1..16"; return GS_E_INVALID; }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    g_createError = "no CUDA device";
    return GS_E_CUDA;
  }
  if (o.device < 0 || o.device >= ndev) { g_createError = "device ordinal out of range"; return GS_E_INVALID; }
  gs_trainer* h = new gs_trainer();
  h->o = o;
  h->device = o.device;
  cudaSetDevice(h->device);
  cudaDeviceGetAttribute(&h->sms, cudaDevAttrMultiProcessorCount, h->device);
  if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
    g_createError = "cudaStreamCreate failed";
    delete h;
    return GS_E_CUDA;
  }
  for (int k = 0; k < RING; ++k) cudaEventCreateWithFlags(&h->ringEv[k], cudaEventDisableTiming);
  h->K = o.shDeg > 0 ? (uint32_t)((o.shDeg + 1) * (o.shDeg + 1) - 1) : 0u;
  h->horizon = o.maxIters ? o.maxIters : 60000u;
  h->histGrid = h->sms * 4;
  h->sweepGrid = onesweep_grid(h->device);
  h->tile = o.tile;
  for (int ti = 0; ti < 3; ++ti)
    for (int di = 0; di < 3; ++di)
      for (int m = 0; m < 2; ++m)
        h->rasterPerSm[ti][di][m] = raster_blocks_per_sm(8 << ti, 64 << di, m == 0 ? 1 : 3);
  *out = h;
  return GS_OK;
}

void gs_destroy(gs_trainer* h) {
  if (!h) return;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  free_all(h);
  for (int k = 0; k < RING; ++k)
    if (h->ringEv[k]) cudaEventDestroy(h->ringEv[k]);
  cudaStream_t own = h->ownStream ? h->ownStream : h->stream;
  if (own) cudaStreamDestroy(own);
  delete h;
}

int gs_setup(gs_trainer* h, const float* params, uint32_t n, const float* sh, const gs_camera* cams,
             uint32_t ncams, const gs_image* images, uint32_t nimages, uint32_t maxViewW, uint32_t maxViewH,
             double sceneRadius) {
  if (!h) return GS_E_INVALID;
  if (!params || n == 0 || !cams || ncams == 0 || !images) return fail(h, GS_E_INVALID, "setup: empty input");
  cudaSetDevice(h->device);
  cudaStreamSynchronize(h->stream);
  free_all(h);
  const gs_options& o = h->o;
  h->n = n;
  // cap (trainer.js:105-107)
  const uint64_t want = std::max<uint64_t>((uint64_t)std::floor((double)n * (o.capMult > 0 ? o.capMult : 4.0)), n);
  const uint64_t lim = o.maxSplats ? o.maxSplats : 600000u;
  h->cap = (uint32_t)std::min<uint64_t>(want, lim);
  if (h->cap < n)
    return fail(h, GS_E_LIMIT, "setup: " + std::to_string(n) + " splats exceed the buffer cap " +
                                   std::to_string(h->cap) + " (raise maxSplats)");
  // entry budget (trainer.js:48-49)
  h->entriesCap = o.entriesCap ? o.entriesCap
                               : (o.maxSplats ? std::max<uint64_t>(12000000ull, (uint64_t)o.maxSplats * 24ull)
                                              : 12000000ull);
  h->ncams = ncams;
  h->cams.assign(cams, cams + ncams);
  h->camOffset.resize(ncams);
  h->camActiveSh.assign(ncams, (float)o.shDeg);
  // targets (trainer.js:115-139): per-camera RGBA8 at pixel offsets
  uint64_t total = 0;
  for (uint32_t c = 0; c < ncams; ++c) {
    if (cams[c].imgIdx < 0 || (uint32_t)cams[c].imgIdx >= nimages)
      return fail(h, GS_E_INVALID, "setup: camera imgIdx out of range");
    const gs_image& im = images[cams[c].imgIdx];
    h->cams[c].w = (int32_t)im.tw;
    h->cams[c].h = (int32_t)im.th;
    h->camOffset[c] = (uint32_t)total;
    total += (uint64_t)im.tw * im.th;
  }
  if (total > 0xFFFFFFFFull) return fail(h, GS_E_LIMIT, "setup: training targets exceed 2^32 pixels");
  h->totalPix = total;
  uint64_t maxImgPix = 0;
  for (uint32_t c = 0; c < ncams; ++c) {
    const gs_image& im = images[cams[c].imgIdx];
    if (!im.rgb && im.tw && im.th) return fail(h, GS_E_INVALID, "setup: image without pixels");
    maxImgPix = std::max<uint64_t>(maxImgPix, (uint64_t)im.tw * im.th);
  }
  // view limits
  h->maxPix = maxViewW * maxViewH;
  // tile-indexed buffers are sized for the smallest tile (8) so the tile
  // size can change after setup (gs_autotune)
  h->maxTiles = ceil_div(maxViewW, 8) * ceil_div(maxViewH, 8);
  h->maxGrid = (ceil_div(maxViewW, 8) + 1) * (ceil_div(maxViewH, 8) + 1);
  for (uint32_t c = 0; c < ncams; ++c) {
    const uint32_t w = (uint32_t)h->cams[c].w, hh = (uint32_t)h->cams[c].h;
    h->maxPix = std::max(h->maxPix, w * hh);
    h->maxTiles = std::max(h->maxTiles, ceil_div(w, 8) * ceil_div(hh, 8));
    h->maxGrid = std::max(h->maxGrid, (ceil_div(w, 8) + 1) * (ceil_div(hh, 8) + 1));
  }
  const uint32_t B = (uint32_t)o.maxBatch;
  const size_t cap = h->cap, shn = (size_t)h->cap * 3 * h->K;
  h->capacity = std::min<uint64_t>((uint64_t)B * h->entriesCap, 0xFFFFFFF0ull);
  int rc;
#define GS_AL(ptr, cnt) if ((rc = dalloc(h, &(ptr), (cnt))) != GS_OK) { free_all(h); return rc; }
  GS_AL(h->params, cap * 16);
  GS_AL(h->m, cap * 16);
  GS_AL(h->v, cap * 16);
  GS_AL(h->sh, std::max<size_t>(shn, 1));
  GS_AL(h->shM, std::max<size_t>(shn, 1));
  GS_AL(h->shV, std::max<size_t>(shn, 1));
  GS_AL(h->recs, (size_t)B * cap);
  GS_AL(h->pkeys[0], (size_t)B * cap);
  GS_AL(h->pkeys[1], (size_t)B * cap);
  GS_AL(h->pvals[0], (size_t)B * cap);
  GS_AL(h->pvals[1], (size_t)B * cap);
  GS_AL(h->viewTotal, (size_t)MAXB);
  GS_AL(h->rect, (size_t)B * cap);
  GS_AL(h->counts, (size_t)B * cap);
  GS_AL(h->offsets, (size_t)B * cap);
  GS_AL(h->cullRecs, (size_t)B * cap);
  GS_AL(h->itemRecs, (size_t)B * cap * 2);
  GS_AL(h->itemSrc, (size_t)B * cap * 2);
  GS_AL(h->viewGrad, (size_t)B * cap * VIEWGRAD_STRIDE);
  GS_AL(h->visList, (size_t)B * cap);
  GS_AL(h->gradP, (size_t)B * cap * GP_STRIDE);
  // (tx+1)(ty+1) = tiles + tx + ty + 1 <= 3 * maxTiles + 1 for any view of at most maxTiles tiles
  GS_AL(h->diffGrid, (size_t)B * (3 * (size_t)h->maxTiles + 1) * GRID_COPIES);
  GS_AL(h->tileCnt, (size_t)B * h->maxTiles);
  GS_AL(h->dropped, (size_t)B * h->maxTiles);
  GS_AL(h->ranges, (size_t)B * h->maxTiles);
  GS_AL(h->viewDrops, (size_t)MAXB);
  GS_AL(h->workOrder, (size_t)B * h->maxTiles);
  GS_AL(h->keys[0], h->capacity);
  GS_AL(h->keys[1], h->capacity);
  GS_AL(h->vals[0], h->capacity);
  GS_AL(h->vals[1], h->capacity);
  GS_AL(h->small, (size_t)4096);
  GS_AL(h->lbStatus, (size_t)(std::max<uint64_t>(h->capacity, (uint64_t)B * cap) / SORT_BLOCK_ENTRIES + 2) * 256);
  GS_AL(h->scanPartials, (size_t)scan_partials_needed((uint64_t)B * cap) + 1);
  GS_AL(h->outImg, (size_t)B * h->maxPix);
  GS_AL(h->finalT, (size_t)B * h->maxPix);
  GS_AL(h->endIdx, (size_t)B * h->maxPix);
  GS_AL(h->targets, std::max<uint64_t>(total, 4));
  GS_AL(h->stats, (size_t)4);
  GS_AL(h->gradCam, (size_t)(ncams + 1) * 8);
  GS_AL(h->gradFOut, cap * 16);
  GS_AL(h->shGradOut, std::max<size_t>(shn, 1));
  GS_AL(h->dParams, (size_t)1);
#undef GS_AL
  if (cudaMallocHost(&h->hRing, sizeof(StepParams) * RING) != cudaSuccess) {
    free_all(h);
    return fail(h, GS_E_NOMEM, "cudaMallocHost(step parameters) failed");
  }
  std::memset(h->hRing, 0, sizeof(StepParams) * RING);
  cudaStream_t s = h->stream;
  GS_CK(cudaMemcpyAsync(h->params, params, (size_t)n * 64, cudaMemcpyHostToDevice, s));
  GS_CK(cudaMemsetAsync(h->m, 0, cap * 64, s));
  GS_CK(cudaMemsetAsync(h->v, 0, cap * 64, s));
  if (shn) {
    GS_CK(cudaMemsetAsync(h->sh, 0, shn * 4, s));
    if (sh) GS_CK(cudaMemcpyAsync(h->sh, sh, (size_t)n * 3 * h->K * 4, cudaMemcpyHostToDevice, s));
    GS_CK(cudaMemsetAsync(h->shM, 0, shn * 4, s));
    GS_CK(cudaMemsetAsync(h->shV, 0, shn * 4, s));
  }
  GS_CK(cudaMemsetAsync(h->gradP, 0, (size_t)B * cap * GP_STRIDE * 4, s));
  GS_CK(cudaMemsetAsync(h->small, 0, 4096 * 4, s));
  GS_CK(cudaMemsetAsync(h->lbStatus, 0, (size_t)(std::max<uint64_t>(h->capacity, (uint64_t)B * cap) / SORT_BLOCK_ENTRIES + 2) * 256 * 8, s));
  // targets packed on the device, one camera at a time through a scratch
  // buffer of the largest image
  {
    float* scratch = nullptr;
    if (maxImgPix && cudaMalloc(&scratch, maxImgPix * 12) != cudaSuccess) {
      free_all(h);
      return fail(h, GS_E_NOMEM, "setup: target staging buffer");
    }
    GS_CK(cudaMemsetAsync(h->targets, 0, std::max<uint64_t>(total, 4) * 4, s));
    int prc = 0;
    for (uint32_t c = 0; c < ncams && prc == 0; ++c) {
      const gs_image& im = images[cams[c].imgIdx];
      prc = pack_targets_device(im.rgb, (uint64_t)im.tw * im.th, scratch, h->targets + h->camOffset[c], s);
    }
    const cudaError_t se = cudaStreamSynchronize(s);
    cudaFree(scratch);
    if (prc != 0 || se != cudaSuccess) return fail(h, GS_E_CUDA, "setup: target packing");
  }
  GS_CK(cudaMemsetAsync(h->stats, 0, 16, s));
  GS_CK(cudaMemsetAsync(h->gradCam, 0, (size_t)(ncams + 1) * 32, s));
  GS_CK(cudaStreamSynchronize(s));
  // Adam hyper-parameters (trainer.js:315-342)
  h->sceneRadius = sceneRadius;
  const double r = sceneRadius;
  h->basePosLr = 3e-4 * r;
  const float lr[16] = {(float)h->basePosLr, (float)h->basePosLr, (float)h->basePosLr, 5e-3f, 5e-3f, 5e-3f,
                        1e-3f, 1e-3f, 1e-3f, 1e-3f, 1.5e-2f, 1.5e-2f, 1.5e-2f, 2.5e-2f, 0.0f, 0.0f};
  std::memcpy(h->lrs, lr, sizeof(lr));
  h->minLS = (float)std::log(r * (o.minScale > 0 ? o.minScale : 1e-4));
  h->maxLS = (float)std::log(r * 0.05);
  h->iter = 0;
  h->pixelsSeen = 0;
  h->overflowTiles = 0;
  h->lastV = 0;
  h->camIdxZero = false;
  h->rf = {};
  h->ready = true;
  return GS_OK;
}

int gs_get_state(const gs_trainer* h, gs_state* out) {
  if (!h || !out) return GS_E_INVALID;
  out->iter = h->iter;
  out->n = h->n;
  out->cap = h->cap;
  out->shDeg = (uint32_t)h->o.shDeg;
  out->shK = h->K;
  out->stride = 16;
  out->ncams = h->ncams;
  out->maxTiles = h->maxTiles;
  out->pixelsSeen = h->pixelsSeen;
  out->entriesCap = h->entriesCap;
  out->horizon = h->horizon;
  uint32_t le = 0;
  if (h->ready) cudaMemcpy(&le, h->small + 2057, 4, cudaMemcpyDeviceToHost);
  out->lastEntries = le;
  out->stepUploadBytes = (uint32_t)sizeof(StepParams);
  out->lastLaunches = h->lastLaunches;
  return GS_OK;
}

int gs_set_iter(gs_trainer* h, uint32_t iter) {
  if (!h) return GS_E_INVALID;
  h->iter = iter;
  return GS_OK;
}
int gs_set_horizon(gs_trainer* h, uint32_t horizon) {
  if (!h || horizon == 0) return GS_E_INVALID;
  h->horizon = horizon;
  return GS_OK;
}
int gs_set_grow_limit(gs_trainer* h, uint32_t growLimit) {
  if (!h) return GS_E_INVALID;
  h->growLimit = growLimit;
  return GS_OK;
}
int gs_set_camera(gs_trainer* h, uint32_t ci, const gs_camera* cam) {
  if (!h || !cam || ci >= h->ncams) return GS_E_INVALID;
  const int32_t w = h->cams[ci].w, hh = h->cams[ci].h, im = h->cams[ci].imgIdx;
  h->cams[ci] = *cam;
  h->cams[ci].w = w; h->cams[ci].h = hh; h->cams[ci].imgIdx = im;  // training resolution stays the image's
  h->camIdxZero = false;  // _applyCamGrads rebuilds every camUniform with its index (trainer.js:533)
  h->camActiveSh[ci] = (float)h->o.shDeg;  // ... and with every SH band active (_camUniform, trainer.js:367)
  return GS_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// The step pipeline.
// ---------------------------------------------------------------------------
static int bits_for(uint32_t x) {  // bits needed to hold values 0..x
  int b = 1;
  while (b < 32 && (x >> b) != 0) ++b;
  return b;
}

// Fills a ring slot with the views' records and the Adam parameters and
// queues its upload.  Returns the slot used.
static int upload_params(gs_trainer* h, const DevCam* views, int V, const AdamHP& hp) {
  const int k = h->ringPos;
  h->ringPos = (h->ringPos + 1) % RING;
  cudaEventSynchronize(h->ringEv[k]);
  StepParams& P = h->hRing[k];
  P.hp = hp;
  P.itemCount = (uint32_t)((uint64_t)V * h->n);
  uint32_t tb = 0, pb = 0, gb = 0;
  for (int v = 0; v < V; ++v) {
    P.cams[v] = views[v];
    P.cams[v].tileBase = tb;
    P.cams[v].pixBase = pb;
    P.gridBase[v] = gb;
    tb += (uint32_t)(views[v].tilesX * views[v].tilesY);
    pb += (uint32_t)(views[v].W * views[v].H);
    gb += (uint32_t)((views[v].tilesX + 1) * (views[v].tilesY + 1));
  }
  cudaMemcpyAsync(h->dParams, &P, sizeof(StepParams), cudaMemcpyHostToDevice, h->stream);
  cudaEventRecord(h->ringEv[k], h->stream);
  for (int v = 0; v < V; ++v) h->lastCams[v] = P.cams[v];
  h->lastV = V;
  return k;
}

// Enqueues project -> bin -> sort -> raster [-> chain/Adam] for the views
// whose records were uploaded last.  All sizes the device decides (entry
// counts) are read on the device, so the sequence can be captured.
static int enqueue_body(gs_trainer* h, const Shape& sh) {
  cudaStream_t s = h->stream;
  const int V = sh.V;
  uint32_t totalTiles = 0, gridCells = 0;
  for (int v = 0; v < V; ++v) {
    const uint32_t tx = ceil_div((uint32_t)sh.w[v], (uint32_t)sh.tile), ty = ceil_div((uint32_t)sh.h[v], (uint32_t)sh.tile);
    totalTiles += tx * ty;
    gridCells += (tx + 1) * (ty + 1);
  }
  h->lastTotalTiles = totalTiles;
  const DevCam* dcams = h->dParams->cams;
  uint32_t* hist = h->small;
  uint32_t* tileCounter = h->small + 2048;
  uint32_t* workCounter = h->small + 2056;
  uint32_t* totalEntries = h->small + 2057;
  uint32_t* scanTotal = h->small + 2058;
  uint32_t* epoch = h->small + 2059;
  uint32_t* statusWord = h->small + 2060;

  cudaEvent_t ph[5] = {};
  if (h->profiling) {
    for (int k = 0; k < 5; ++k) cudaEventCreate(&ph[k]);
    cudaEventRecord(ph[0], s);
  }
  cudaMemsetAsync(h->diffGrid, 0, (size_t)gridCells * GRID_COPIES * 4, s);
  cudaMemsetAsync(h->small, 0, 2057 * 4, s);  // hist, tile counters, work counter
  cudaMemsetAsync(h->small + 2062, 0, MAXB * 4, s);  // visible-item counters of the chain
  const uint64_t items = (uint64_t)sh.n * V;

  ProjectArgs pa{};
  pa.params = h->params;
  pa.sh = h->K ? h->sh : nullptr;
  pa.n = sh.n;
  pa.V = V;
  pa.cams = dcams;
  pa.eCut = h->o.eCut;
  pa.aMin = h->o.aMin;
  pa.radClamp = h->o.radClamp;
  pa.tile = sh.tile;
  pa.recs = h->recs;
  pa.pkeys = reinterpret_cast<uint32_t*>(h->pkeys[0]);
  pa.pvals = h->pvals[0];
  pa.rect = h->rect;
  pa.diffGrid = h->diffGrid;
  pa.gridCells = gridCells;
  pa.gridBase = h->dParams->gridBase;
  pa.cullRecs = h->cullRecs;
  pa.itemSrc = h->itemSrc;
  launch_project(pa, h->o.shDeg, s);

  TileRangeArgs ta{};
  ta.V = V;
  ta.cams = dcams;
  ta.diffGrid = h->diffGrid;
  ta.gridCells = gridCells;
  ta.gridBase = h->dParams->gridBase;
  ta.tileCnt = h->tileCnt;
  ta.dropped = h->dropped;
  ta.ranges = h->ranges;
  ta.viewDrops = h->viewDrops;
  ta.viewTotal = h->viewTotal;
  ta.stats = h->stats;
  ta.entriesCap = h->entriesCap;
  ta.totalEntries = totalEntries;
  launch_tile_ranges(ta, totalTiles, s);

  // presort of the (view, splat) items by depth: 4 byte digits of the depth
  // bits, stable from slot order, so equal depths stay in splat order.  Views
  // stay interleaved: the tile sort groups entries by global tile id (which
  // belongs to one view) and keeps this order inside every tile.
  uint32_t* nItems = h->small + 2061;
  cudaMemcpyAsync(nItems, &h->dParams->itemCount, 4, cudaMemcpyDeviceToDevice, s);
  RadixSortArgs pr{};
  pr.keys[0] = h->pkeys[0]; pr.keys[1] = h->pkeys[1];
  pr.vals[0] = h->pvals[0]; pr.vals[1] = h->pvals[1];
  pr.keyBytes = 4;
  pr.nItems = nItems;
  pr.hist = hist;
  pr.tileCounter = tileCounter;
  pr.status = h->lbStatus;
  pr.statusWord = statusWord;
  pr.epoch = epoch;
  pr.passes = 4;
  pr.keepKeys = false;
  pr.orPasses = 0x7u;  // depth bytes 0-2 spread across a warp; the top byte (sign, exponent) is shared
  pr.histGrid = (unsigned)h->histGrid;
  pr.sweepGrid = (unsigned)h->sweepGrid;
  // culled items (all-ones keys) leave the presort: only the visible ones
  // are sorted, and their count sizes the expansion
  uint32_t* liveItems = h->small + 2150;
  pr.nKept = liveItems;
  cudaMemsetAsync(liveItems, 0, 4, s);
  if (h->profiling) cudaEventRecord(ph[1], s);
  launch_radix_sort(pr, s);
  const uint32_t* sortedSlots = h->pvals[pr.passes & 1];

  const bool cull = sh.cull != 0;
  ExpandArgs ea{};
  ea.n = sh.n;
  ea.V = V;
  ea.cams = dcams;
  ea.sortedSlots = sortedSlots;
  ea.itemSrc = h->itemSrc;
  ea.itemRecs = h->itemRecs;
  ea.liveItems = liveItems;
  ea.dropped = h->dropped;
  ea.viewDrops = h->viewDrops;
  ea.eCut = h->o.eCut;
  ea.aMin = h->o.aMin;
  ea.tile = sh.tile;
  ea.cull = cull ? 1 : 0;
  ea.counts = h->counts;
  ea.offsets = h->offsets;
  ea.keys = h->keys[0];
  ea.vals = h->vals[0];
  ea.capacity = h->capacity;
  ea.status = statusWord;
  launch_expand(ea, false, s);
  launch_exclusive_scan(h->counts, items, h->offsets, h->scanPartials, scanTotal, s);
  launch_expand(ea, true, s);
  // culled lists: the entry total is the counts' sum, not the budgeted tile sum
  if (cull) cudaMemcpyAsync(totalEntries, scanTotal, 4, cudaMemcpyDeviceToDevice, s);

  // stable sort of the entries by global tile id
  cudaMemsetAsync(h->small, 0, 2056 * 4, s);  // histograms and block counters of the second sort
  const int passes = (bits_for(totalTiles ? totalTiles - 1 : 0) + 7) / 8;
  RadixSortArgs ra{};
  ra.keys[0] = h->keys[0]; ra.keys[1] = h->keys[1];
  ra.vals[0] = h->vals[0]; ra.vals[1] = h->vals[1];
  ra.keyBytes = 4;
  ra.nItems = totalEntries;
  ra.hist = hist;
  ra.tileCounter = tileCounter;
  ra.status = h->lbStatus;
  ra.statusWord = statusWord;
  ra.epoch = epoch;
  ra.passes = passes;
  ra.keepKeys = cull;  // culled lists take their tile ranges from the sorted keys
  ra.orPasses = 0xFFu;  // tile ids: every byte spread across a warp
  ra.histGrid = (unsigned)h->histGrid;
  ra.sweepGrid = (unsigned)h->sweepGrid;
  launch_radix_sort(ra, s);
  h->lastPasses = passes;
  if (cull) launch_ranges_from_keys(h->keys[passes & 1], totalEntries, totalTiles, h->ranges, s);
  // kernels: project, tile counts + finish, presort (histogram + passes),
  // entry counts, 3 scan kernels, entry keys, tile sort (histogram +
  // passes), [ranges from keys], [work order: 3], raster, [visible lists, chain per view, sum + Adam]
  h->lastLaunches = 3u + 1u + (uint32_t)pr.passes + 1u + 3u + 1u + 1u + (uint32_t)passes + (cull ? 1u : 0u) +
                    (h->o.persistent ? 3u : 0u) + 1u + (sh.chain ? 3u : 0u);
  const uint32_t* sortedIds = h->vals[passes & 1];

  const bool persistent = h->o.persistent != 0;
  if (persistent) launch_work_order(h->ranges, totalTiles, h->workOrder, h->small + 2080, s);  // [2080, 2146)
  if (h->profiling) cudaEventRecord(ph[2], s);
  RasterArgs rr{};
  rr.cams = dcams;
  rr.V = V;
  rr.n = sh.n;
  rr.recs = h->recs;
  rr.cullRecs = h->cullRecs;
  rr.ids = sortedIds;
  rr.ranges = h->ranges;
  rr.totalTiles = totalTiles;
  rr.workOrder = persistent ? h->workOrder : nullptr;
  rr.workCounter = persistent ? workCounter : nullptr;
  rr.eCut = h->o.eCut;
  rr.aMin = h->o.aMin;
  rr.outImg = h->outImg;
  rr.finalT = h->finalT;
  rr.endIdx = h->endIdx;
  rr.targets = h->targets;
  rr.gradP = h->gradP;
  rr.stats = h->stats;
  rr.gradCam = h->gradCam;
  rr.tStore = h->tStore;
  unsigned grid = totalTiles;
  if (persistent) {
    const int ti = sh.tile == 8 ? 0 : sh.tile == 16 ? 1 : 2;
    const int di = sh.depth == 64 ? 0 : sh.depth == 128 ? 1 : 2;
    const unsigned full = (unsigned)(h->sms * h->rasterPerSm[ti][di][sh.mode == 1 ? 0 : 1]);
    grid = std::min(grid, full);
  }
  launch_raster(rr, sh.mode, sh.variant == 1, sh.tile, sh.depth, grid, s);
  if (h->profiling) cudaEventRecord(ph[3], s);

  if (sh.chain) {
    ChainArgs c{};
    c.n = sh.n;
    c.V = V;
    c.cams = dcams;
    c.params = h->params;
    c.sh = h->K ? h->sh : nullptr;
    c.gradP = h->gradP;
    c.rect = h->rect;
    c.viewGrad = h->viewGrad;
    c.visList = h->visList;
    c.visCount = h->small + 2062;
    c.anisoReg = h->o.anisoReg;
    c.gradCam = h->gradCam;
    c.gradF = sh.grads ? h->gradFOut : nullptr;
    c.shGrad = sh.grads ? h->shGradOut : nullptr;
    c.doAdam = sh.adam;
    c.hp = &h->dParams->hp;
    c.m = h->m;
    c.v = h->v;
    c.shM = h->shM;
    c.shV = h->shV;
    launch_chain_adam(c, h->o.shDeg, s);
  }
  if (h->profiling) {
    cudaEventRecord(ph[4], s);
    for (int k = 0; k < 4; ++k) {
      if (k == 3 && !sh.chain) continue;
      h->evPool.push_back(ph[k]);
      h->evPool.push_back(ph[k + 1]);
      h->evPhase.push_back(k);
    }
    h->evPool.push_back(nullptr);  // marks the end of this launch's events (owner of ph[])
    h->evPhase.push_back(-1);
    h->evPool.push_back(ph[0]); h->evPool.push_back(ph[1]); h->evPool.push_back(ph[2]);
    h->evPool.push_back(ph[3]); h->evPool.push_back(ph[4]);
  }
  return GS_OK;
}

// Sizes the stored-state buffer (T before every entry, per pixel of its
// tile) for the coming pass: runs the binning once to learn the entry count.
static int ensure_tstore(gs_trainer* h, const Shape& sh) {
  Shape probe = sh;
  probe.mode = 1;
  probe.chain = 0;
  probe.variant = 0;
  int rc = enqueue_body(h, probe);
  if (rc) return rc;
  uint32_t E = 0;
  GS_CK(cudaMemcpyAsync(&E, h->small + 2057, 4, cudaMemcpyDeviceToHost, h->stream));
  GS_CK(cudaStreamSynchronize(h->stream));
  const size_t need = (size_t)E * sh.tile * sh.tile + 1;  // T per (entry, pixel of its tile)
  if (need > h->tStoreCap) {
    if (h->tStore) cudaFree(h->tStore);
    h->tStore = nullptr;
    h->tStoreCap = 0;
    void* q = nullptr;
    if (cudaMalloc(&q, need * 4) != cudaSuccess)
      return fail(h, GS_E_NOMEM, "stored-state variant: cannot allocate " + std::to_string(need * 4) + " bytes");
    h->tStore = (float*)q;
    h->tStoreCap = need;
    for (auto& kv : h->graphs) cudaGraphExecDestroy(kv.second);
    h->graphs.clear();
  }
  return GS_OK;
}

static int run_shape(gs_trainer* h, const Shape& sh) {
  if (sh.variant == 1) {
    int rc = ensure_tstore(h, sh);
    if (rc) return rc;
  }
  if (!h->o.useGraphs || sh.variant == 1 || h->profiling) return enqueue_body(h, sh);
  auto it = h->graphs.find(sh);
  if (it == h->graphs.end()) {
    cudaGraph_t g = nullptr;
    GS_CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    int rc = enqueue_body(h, sh);
    cudaError_t e = cudaStreamEndCapture(h->stream, &g);
    if (rc) { if (g) cudaGraphDestroy(g); return rc; }
    if (e != cudaSuccess) return fail(h, GS_E_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    cudaGraphExec_t ex = nullptr;
    e = cudaGraphInstantiate(&ex, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(h, GS_E_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
    it = h->graphs.emplace(sh, ex).first;
  }
  GS_CK(cudaGraphLaunch(it->second, h->stream));
  return GS_OK;
}

static AdamHP make_hp(gs_trainer* h) {
  AdamHP hp{};
  std::memcpy(hp.lr, h->lrs, sizeof(hp.lr));
  // exponential position-lr decay (trainer.js:422)
  const double posLr = h->basePosLr * std::pow(0.01, std::min(1.0, (double)h->iter / (0.75 * h->horizon)));
  hp.lr[0] = hp.lr[1] = hp.lr[2] = (float)posLr;
  hp.b1 = 0.9f; hp.b2 = 0.999f; hp.eps = 1e-15f;
  const double t = (double)h->iter;
  hp.bc1 = (float)(1.0 - std::pow((double)0.9f, t));
  hp.bc2 = (float)(1.0 - std::pow((double)0.999f, t));
  hp.minLS = h->minLS;
  hp.maxLS = h->maxLS;
  hp.maxLogit = 8.0f;
  hp.reg = h->o.opacityReg;
  hp.shLr = h->o.shLr;
  return hp;
}

static int check_views(gs_trainer* h, const uint32_t* ci, uint32_t nv) {
  if (!h->ready) return fail(h, GS_E_INVALID, "setup() first");
  if (!ci || nv == 0) return fail(h, GS_E_INVALID, "no views");
  if (nv > (uint32_t)h->o.maxBatch)
    return fail(h, GS_E_LIMIT, "batch of " + std::to_string(nv) + " views exceeds maxBatch " +
                                   std::to_string(h->o.maxBatch));
  for (uint32_t k = 0; k < nv; ++k)
    if (ci[k] >= h->ncams) return fail(h, GS_E_INVALID, "camera index out of range");
  return GS_OK;
}

static Shape make_shape(gs_trainer* h, const DevCam* views, int V, int mode, int chain, int adam, int grads) {
  Shape sh;
  std::memset(&sh, 0, sizeof(sh));
  sh.V = V;
  for (int v = 0; v < V; ++v) { sh.w[v] = views[v].W; sh.h[v] = views[v].H; }
  sh.n = h->n;
  sh.mode = mode;
  sh.chain = chain;
  sh.adam = adam;
  sh.grads = grads;
  sh.variant = h->o.backwardVariant;
  sh.tile = h->tile;
  sh.depth = h->o.batchDepth;
  sh.cull = h->o.tileCull;
  return sh;
}

extern "C" {

int gs_step_batch(gs_trainer* h, const uint32_t* ci, uint32_t nv) {
  if (!h) return GS_E_INVALID;
  int rc = check_views(h, ci, nv);
  if (rc) return rc;
  cudaSetDevice(h->device);
  DevCam views[MAXB];
  for (uint32_t k = 0; k < nv; ++k) {
    const uint32_t c = ci[k];
    // SH band ramp, one degree per 1000 iterations (trainer.js:409-412)
    if (h->K) h->camActiveSh[c] = (float)std::min<uint32_t>((uint32_t)h->o.shDeg, h->iter / 1000u);
    views[k] = make_cam(h, h->cams[c], 1, h->camOffset[c], h->camIdxZero ? 0u : c, h->camActiveSh[c]);
  }
  h->iter++;
  for (uint32_t k = 0; k < nv; ++k) h->pixelsSeen += (uint64_t)views[k].W * views[k].H;
  const AdamHP hp = make_hp(h);
  upload_params(h, views, (int)nv, hp);
  return run_shape(h, make_shape(h, views, (int)nv, 3, 1, 1, 0));
}

int gs_step(gs_trainer* h, uint32_t ci) { return gs_step_batch(h, &ci, 1); }

static int check_status(gs_trainer* h) {
  uint32_t st = 0;
  GS_CK(cudaMemcpyAsync(&st, h->small + 2060, 4, cudaMemcpyDeviceToHost, h->stream));
  GS_CK(cudaStreamSynchronize(h->stream));
  if (st) {
    cudaMemsetAsync(h->small + 2060, 0, 4, h->stream);
    std::string m = "device status:";
    if (st & ST_LOOKBACK_TIMEOUT) m += " sort look-back wait exceeded its limit;";
    if (st & ST_ENTRY_OVERFLOW) m += " entry buffer overflow;";
    if (st & ST_BAD_INPUT) m += " inconsistent entry expansion;";
    return fail(h, GS_E_DEVICE, m);
  }
  return GS_OK;
}

int gs_sync(gs_trainer* h) {
  if (!h) return GS_E_INVALID;
  cudaSetDevice(h->device);
  GS_CK(cudaStreamSynchronize(h->stream));
  GS_CK(cudaGetLastError());
  return h->ready ? check_status(h) : GS_OK;
}

int gs_read_stats(gs_trainer* h, uint32_t out[4]) {
  if (!h || !out) return GS_E_INVALID;
  if (!h->ready) return fail(h, GS_E_INVALID, "setup() first");
  cudaSetDevice(h->device);
  GS_CK(cudaMemcpyAsync(out, h->stats, 16, cudaMemcpyDeviceToHost, h->stream));
  GS_CK(cudaMemsetAsync(h->stats, 0, 16, h->stream));
  GS_CK(cudaStreamSynchronize(h->stream));
  h->overflowTiles += out[3];
  h->pixelsSeen = 0;
  return check_status(h);
}

int gs_read_stats_async(gs_trainer* h, uint32_t* out) {
  if (!h || !out) return GS_E_INVALID;
  if (!h->ready) return fail(h, GS_E_INVALID, "setup() first");
  cudaSetDevice(h->device);
  GS_CK(cudaMemcpyAsync(out, h->stats, 16, cudaMemcpyDeviceToHost, h->stream));
  GS_CK(cudaMemsetAsync(h->stats, 0, 16, h->stream));
  h->pixelsSeen = 0;
  return GS_OK;
}

int gs_export_ply(gs_trainer* h, int32_t bake, double f, const double* camPositions, uint32_t ncams, uint8_t* out,
                  uint64_t cap, uint64_t* size) {
  if (!h || !size) return GS_E_INVALID;
  if (!h->ready) return fail(h, GS_E_INVALID, "setup() first");
  if (bake && ncams && !camPositions) return fail(h, GS_E_INVALID, "camPositions is NULL");
  // header of gaussiansToPly (ply.js:51-69)
  std::string hdr = "ply\nformat binary_little_endian 1.0\nelement vertex " + std::to_string(h->n) + "\n";
  const char* head[] = {"x", "y", "z", "nx", "ny", "nz", "f_dc_0", "f_dc_1", "f_dc_2"};
  for (const char* p : head) hdr += std::string("property float ") + p + "\n";
  for (uint32_t k = 0; k < 3 * h->K; ++k) hdr += "property float f_rest_" + std::to_string(k) + "\n";
  const char* tail[] = {"opacity", "scale_0", "scale_1", "scale_2", "rot_0", "rot_1", "rot_2", "rot_3"};
  for (const char* p : tail) hdr += std::string("property float ") + p + "\n";
  hdr += "end_header\n";
  const uint64_t body = (uint64_t)h->n * (17 + 3 * h->K) * 4;
  *size = hdr.size() + body;
  if (!out) return GS_OK;
  if (cap < *size) return fail(h, GS_E_LIMIT, "output buffer smaller than the PLY");
  cudaSetDevice(h->device);
  std::memcpy(out, hdr.data(), hdr.size());
  const size_t camBytes = bake && ncams ? (size_t)ncams * 3 * 8 : 8;
  if (camBytes > h->plyCamCap) {
    if (h->plyCam) cudaFree(h->plyCam);
    h->plyCam = nullptr; h->plyCamCap = 0;
    if (cudaMalloc(&h->plyCam, camBytes) != cudaSuccess) return fail(h, GS_E_NOMEM, "PLY export buffers");
    h->plyCamCap = camBytes;
  }
  const size_t recBytes = body > 0 ? (size_t)body : 4;
  if (recBytes > h->plyOutCap) {
    if (h->plyOut) cudaFree(h->plyOut);
    h->plyOut = nullptr; h->plyOutCap = 0;
    if (cudaMalloc(&h->plyOut, recBytes) != cudaSuccess) return fail(h, GS_E_NOMEM, "PLY export buffers");
    h->plyOutCap = recBytes;
  }
  // the records go from the device straight into the caller's buffer after the header
  const int rc = export_ply_records(h->params, h->K ? h->sh : nullptr, h->n, h->K, bake, f, camPositions, ncams,
                                    h->plyCam, h->plyOut, out + hdr.size(), h->stream);
  if (rc) return fail(h, GS_E_CUDA, "PLY export kernel");
  return GS_OK;
}

int gs_read_gaussians(gs_trainer* h, float* params, float* sh, uint32_t* n) {
  if (!h) return GS_E_INVALID;
  if (!h->ready) return fail(h, GS_E_INVALID, "setup() first");
  cudaSetDevice(h->device);
  if (params) GS_CK(cudaMemcpyAsync(params, h->params, (size_t)h->n * 64, cudaMemcpyDeviceToHost, h->stream));
  if (sh && h->K)
    GS_CK(cudaMemcpyAsync(sh, h->sh, (size_t)h->n * 3 * h->K * 4, cudaMemcpyDeviceToHost, h->stream));
  if (n) *n = h->n;
  GS_CK(cudaStreamSynchronize(h->stream));
  return check_status(h);
}

int gs_write_gaussians(gs_trainer* h, const float* params, const float* sh, uint32_t n) {
  if (!h) return GS_E_INVALID;
  if (!h->ready) return fail(h, GS_E_INVALID, "setup() first");
  if (n > h->n) return fail(h, GS_E_INVALID, "write_gaussians: n exceeds the splat count");
  cudaSetDevice(h->device);
  if (params) GS_CK(cudaMemcpyAsync(h->params, params, (size_t)n * 64, cudaMemcpyHostToDevice, h->stream));
  if (sh && h->K)
    GS_CK(cudaMemcpyAsync(h->sh, sh, (size_t)n * 3 * h->K * 4, cudaMemcpyHostToDevice, h->stream));
  GS_CK(cudaStreamSynchronize(h->stream));
  return GS_OK;
}

int gs_reset_moments(gs_trainer* h) {
  if (!h) return GS_E_INVALID;
  if (!h->ready) return fail(h, GS_E_INVALID, "setup() first");
  cudaSetDevice(h->device);
  const size_t pb = (size_t)h->cap * 64, sb = (size_t)h->cap * 3 * h->K * 4;
  GS_CK(cudaMemsetAsync(h->m, 0, pb, h->stream));
  GS_CK(cudaMemsetAsync(h->v, 0, pb, h->stream));
  if (sb) {
    GS_CK(cudaMemsetAsync(h->shM, 0, sb, h->stream));
    GS_CK(cudaMemsetAsync(h->shV, 0, sb, h->stream));
  }
  GS_CK(cudaStreamSynchronize(h->stream));
  return GS_OK;
}

int gs_read_moments(gs_trainer* h, float* m, float* v, float* shM, float* shV) {
  if (!h) return GS_E_INVALID;
  if (!h->ready) return fail(h, GS_E_INVALID, "setup() first");
  cudaSetDevice(h->device);
  const size_t pb = (size_t)h->n * 64, sb = (size_t)h->n * 3 * h->K * 4;
  if (m) GS_CK(cudaMemcpyAsync(m, h->m, pb, cudaMemcpyDeviceToHost, h->stream));
  if (v) GS_CK(cudaMemcpyAsync(v, h->v, pb, cudaMemcpyDeviceToHost, h->stream));
  if (shM && sb) GS_CK(cudaMemcpyAsync(shM, h->shM, sb, cudaMemcpyDeviceToHost, h->stream));
  if (shV && sb) GS_CK(cudaMemcpyAsync(shV, h->shV, sb, cudaMemcpyDeviceToHost, h->stream));
  GS_CK(cudaStreamSynchronize(h->stream));
  return GS_OK;
}

int gs_render(gs_trainer* h, const gs_camera* cam, int32_t trainMode, uint32_t offset, float* outRGBA) {
  if (!h || !cam) return GS_E_INVALID;
  if (!h->ready) return fail(h, GS_E_INVALID, "setup() first");
  if ((uint64_t)cam->w * cam->h > h->maxPix || cam->w <= 0 || cam->h <= 0)
    return fail(h, GS_E_LIMIT, "renderView: view larger than setup's maxViewW x maxViewH");
  if (ceil_div((uint32_t)cam->w, (uint32_t)h->tile) * ceil_div((uint32_t)cam->h, (uint32_t)h->tile) > h->maxTiles)
    return fail(h, GS_E_LIMIT, "renderView: view has more tiles than setup's maximum");
  if (trainMode && (uint64_t)offset + (uint64_t)cam->w * cam->h > h->totalPix)
    return fail(h, GS_E_LIMIT, "renderView: trainMode target offset + view size exceeds the training targets");
  cudaSetDevice(h->device);
  // _camUniform(camParams, trainMode, offset): camIdx 0, active degree = shDeg
  const DevCam view = make_cam(h, *cam, trainMode ? 1 : 0, offset, 0u, (float)h->o.shDeg);
  upload_params(h, &view, 1, make_hp(h));
  int rc = run_shape(h, make_shape(h, &view, 1, trainMode ? 3 : 1, 0, 0, 0));
  if (rc) return rc;
  if (outRGBA)
    GS_CK(cudaMemcpyAsync(outRGBA, h->outImg, (size_t)cam->w * cam->h * 16, cudaMemcpyDeviceToHost, h->stream));
  GS_CK(cudaStreamSynchronize(h->stream));
  return check_status(h);
}

int gs_eval_pass(gs_trainer* h, uint32_t ci, const gs_camera* cam, uint32_t stats[4], int32_t* camGrad) {
  if (!h) return GS_E_INVALID;
  int rc = check_views(h, &ci, 1);
  if (rc) return rc;
  cudaSetDevice(h->device);
  const bool over = cam != nullptr;
  gs_camera c = over ? *cam : h->cams[ci];
  c.w = h->cams[ci].w; c.h = h->cams[ci].h;
  // With an override the reference builds a fresh uniform (trainer.js:547):
  // gradient row ci and every SH band active.  Without one it reuses
  // camUniforms[ci] as the last step or rebuild left it: the ramped SH degree
  // of that camera's last step, and gradient row 0 after growth rebuilt the
  // uniforms without their index (trainer.js:768).
  const uint32_t row = (!over && h->camIdxZero) ? 0u : ci;
  const float act = over ? (float)h->o.shDeg : h->camActiveSh[ci];
  const DevCam view = make_cam(h, c, 1, h->camOffset[ci], row, act);
  GS_CK(cudaMemsetAsync(h->stats, 0, 16, h->stream));
  upload_params(h, &view, 1, make_hp(h));
  rc = run_shape(h, make_shape(h, &view, 1, 3, 1, 0, 0));
  if (rc) return rc;
  uint32_t st[4];
  GS_CK(cudaMemcpyAsync(st, h->stats, 16, cudaMemcpyDeviceToHost, h->stream));
  if (camGrad)
    GS_CK(cudaMemcpyAsync(camGrad, h->gradCam, (size_t)(h->ncams + 1) * 32, cudaMemcpyDeviceToHost, h->stream));
  GS_CK(cudaMemsetAsync(h->gradCam, 0, (size_t)(h->ncams + 1) * 32, h->stream));
  GS_CK(cudaMemsetAsync(h->stats, 0, 16, h->stream));
  GS_CK(cudaStreamSynchronize(h->stream));
  if (stats) std::memcpy(stats, st, 16);
  h->pixelsSeen = 0;
  return check_status(h);
}

int gs_grad_pass(gs_trainer* h, uint32_t ci, float* gradF, float* shGrad, uint32_t stats[4]) {
  if (!h) return GS_E_INVALID;
  int rc = check_views(h, &ci, 1);
  if (rc) return rc;
  cudaSetDevice(h->device);
  const DevCam view = make_cam(h, h->cams[ci], 1, h->camOffset[ci], ci, h->camActiveSh[ci]);
  GS_CK(cudaMemsetAsync(h->stats, 0, 16, h->stream));
  upload_params(h, &view, 1, make_hp(h));
  rc = run_shape(h, make_shape(h, &view, 1, 3, 1, 0, 1));
  if (rc) return rc;
  if (gradF) GS_CK(cudaMemcpyAsync(gradF, h->gradFOut, (size_t)h->n * 64, cudaMemcpyDeviceToHost, h->stream));
  if (shGrad && h->K)
    GS_CK(cudaMemcpyAsync(shGrad, h->shGradOut, (size_t)h->n * 3 * h->K * 4, cudaMemcpyDeviceToHost, h->stream));
  if (stats) GS_CK(cudaMemcpyAsync(stats, h->stats, 16, cudaMemcpyDeviceToHost, h->stream));
  GS_CK(cudaStreamSynchronize(h->stream));
  return check_status(h);
}

int gs_read_cam_grads(gs_trainer* h, int32_t* out, int32_t reset) {
  if (!h || !out) return GS_E_INVALID;
  if (!h->ready) return fail(h, GS_E_INVALID, "setup() first");
  cudaSetDevice(h->device);
  GS_CK(cudaMemcpyAsync(out, h->gradCam, (size_t)(h->ncams + 1) * 32, cudaMemcpyDeviceToHost, h->stream));
  if (reset) GS_CK(cudaMemsetAsync(h->gradCam, 0, (size_t)(h->ncams + 1) * 32, h->stream));
  GS_CK(cudaStreamSynchronize(h->stream));
  return GS_OK;
}

int gs_raster_pass(gs_trainer* h, const uint32_t* ci, uint32_t nv, int32_t mode) {
  if (!h) return GS_E_INVALID;
  int rc = check_views(h, ci, nv);
  if (rc) return rc;
  if (mode != 1 && mode != 3) return fail(h, GS_E_INVALID, "raster_pass: mode must be 1 or 3");
  cudaSetDevice(h->device);
  DevCam views[MAXB];
  for (uint32_t k = 0; k < nv; ++k)
    views[k] = make_cam(h, h->cams[ci[k]], mode == 3 ? 1 : 0, h->camOffset[ci[k]], ci[k], h->camActiveSh[ci[k]]);
  upload_params(h, views, (int)nv, make_hp(h));
  rc = run_shape(h, make_shape(h, views, (int)nv, mode, 0, 0, 0));
  if (rc) return rc;
  return gs_sync(h);
}

int gs_debug_records(gs_trainer* h, uint32_t view, float* rec12, uint32_t* rect2) {
  if (!h || view >= (uint32_t)h->lastV) return GS_E_INVALID;
  cudaSetDevice(h->device);
  if (rec12)
    GS_CK(cudaMemcpyAsync(rec12, h->recs + (size_t)view * h->n, (size_t)h->n * sizeof(RenderRec),
                          cudaMemcpyDeviceToHost, h->stream));
  if (rect2)
    GS_CK(cudaMemcpyAsync(rect2, h->rect + (size_t)view * h->n, (size_t)h->n * 8, cudaMemcpyDeviceToHost,
                          h->stream));
  GS_CK(cudaStreamSynchronize(h->stream));
  return GS_OK;
}

int gs_debug_binning(gs_trainer* h, uint32_t view, uint32_t* tileCnt, uint32_t* rangesOut, uint32_t* ids,
                     uint64_t cap, uint64_t* nEntries) {
  if (!h || view >= (uint32_t)h->lastV) return GS_E_INVALID;
  cudaSetDevice(h->device);
  const DevCam& c = h->lastCams[view];
  const size_t nt = (size_t)c.tilesX * c.tilesY;
  uint32_t E = 0;
  GS_CK(cudaMemcpyAsync(&E, h->small + 2057, 4, cudaMemcpyDeviceToHost, h->stream));
  if (tileCnt)
    GS_CK(cudaMemcpyAsync(tileCnt, h->tileCnt + c.tileBase, nt * 4, cudaMemcpyDeviceToHost, h->stream));
  if (rangesOut)
    GS_CK(cudaMemcpyAsync(rangesOut, h->ranges + c.tileBase, nt * 8, cudaMemcpyDeviceToHost, h->stream));
  GS_CK(cudaStreamSynchronize(h->stream));
  if (nEntries) *nEntries = E;
  if (ids) {
    const uint64_t k = std::min<uint64_t>(cap, E);
    GS_CK(cudaMemcpyAsync(ids, h->vals[h->lastPasses & 1], k * 4, cudaMemcpyDeviceToHost, h->stream));
    GS_CK(cudaStreamSynchronize(h->stream));
  }
  return GS_OK;
}

int gs_debug_targets(gs_trainer* h, uint32_t* out, uint64_t count) {
  if (!h || !h->ready || !out || count > h->totalPix) return GS_E_INVALID;
  cudaSetDevice(h->device);
  if (count) GS_CK(cudaMemcpyAsync(out, h->targets, count * 4, cudaMemcpyDeviceToHost, h->stream));
  GS_CK(cudaStreamSynchronize(h->stream));
  return GS_OK;
}

int gs_debug_pixels(gs_trainer* h, uint32_t view, float* rgba, float* finalT, uint32_t* endIdx) {
  if (!h || view >= (uint32_t)h->lastV) return GS_E_INVALID;
  cudaSetDevice(h->device);
  const DevCam& c = h->lastCams[view];
  const size_t np = (size_t)c.W * c.H;
  if (rgba) GS_CK(cudaMemcpyAsync(rgba, h->outImg + c.pixBase, np * 16, cudaMemcpyDeviceToHost, h->stream));
  if (finalT) GS_CK(cudaMemcpyAsync(finalT, h->finalT + c.pixBase, np * 4, cudaMemcpyDeviceToHost, h->stream));
  if (endIdx) GS_CK(cudaMemcpyAsync(endIdx, h->endIdx + c.pixBase, np * 4, cudaMemcpyDeviceToHost, h->stream));
  GS_CK(cudaStreamSynchronize(h->stream));
  return GS_OK;
}

int gs_debug_gradp(gs_trainer* h, uint32_t view, int32_t* gradP10, int32_t clear) {
  if (!h || view >= (uint32_t)h->lastV) return GS_E_INVALID;
  cudaSetDevice(h->device);
  std::vector<int32_t> tmp((size_t)h->n * GP_STRIDE);
  int32_t* src = h->gradP + (size_t)view * h->n * GP_STRIDE;
  GS_CK(cudaMemcpyAsync(tmp.data(), src, tmp.size() * 4, cudaMemcpyDeviceToHost, h->stream));
  if (clear) GS_CK(cudaMemsetAsync(src, 0, tmp.size() * 4, h->stream));
  GS_CK(cudaStreamSynchronize(h->stream));
  if (gradP10)
    for (size_t i = 0; i < h->n; ++i)
      for (int k = 0; k < 10; ++k) gradP10[i * 10 + k] = tmp[i * GP_STRIDE + k];
  return GS_OK;
}

// Autotuner: times the training pass (raster + chain, parameters untouched)
// on views ci[0..nviews) for every tile edge {8, 16, 32} x splat-batch depth
// {64, 128, 256} and keeps the fastest.  Loss statistics and camera
// gradients accumulated meanwhile are restored.
int gs_autotune(gs_trainer* h, const uint32_t* ci, uint32_t nv, int32_t reps, int32_t* bestTile, int32_t* bestDepth,
                float* msOut) {
  if (!h) return GS_E_INVALID;
  int rc = check_views(h, ci, nv);
  if (rc) return rc;
  if (reps < 1) reps = 1;
  cudaSetDevice(h->device);
  cudaStream_t s = h->stream;
  uint32_t st[4];
  std::vector<int32_t> cg((size_t)(h->ncams + 1) * 8);
  GS_CK(cudaMemcpyAsync(st, h->stats, 16, cudaMemcpyDeviceToHost, s));
  GS_CK(cudaMemcpyAsync(cg.data(), h->gradCam, cg.size() * 4, cudaMemcpyDeviceToHost, s));
  GS_CK(cudaStreamSynchronize(s));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int tiles[3] = {8, 16, 32}, depths[3] = {64, 128, 256};
  float best = 3.0e38f;
  int bt = h->tile, bd = h->o.batchDepth;
  for (int ti = 0; ti < 3 && rc == GS_OK; ++ti)
    for (int di = 0; di < 3 && rc == GS_OK; ++di) {
      h->tile = tiles[ti];
      h->o.batchDepth = depths[di];
      DevCam views[MAXB];
      for (uint32_t k = 0; k < nv; ++k)
        views[k] = make_cam(h, h->cams[ci[k]], 1, h->camOffset[ci[k]], ci[k], h->camActiveSh[ci[k]]);
      upload_params(h, views, (int)nv, make_hp(h));
      const Shape sh = make_shape(h, views, (int)nv, 3, 1, 0, 0);
      rc = run_shape(h, sh);  // warm-up (and graph capture)
      if (rc) break;
      cudaEventRecord(e0, s);
      for (int r = 0; r < reps && rc == GS_OK; ++r) rc = run_shape(h, sh);
      cudaEventRecord(e1, s);
      cudaEventSynchronize(e1);
      float ms = 0.0f;
      cudaEventElapsedTime(&ms, e0, e1);
      ms /= (float)reps;
      if (msOut) msOut[ti * 3 + di] = ms;
      if (ms < best) { best = ms; bt = tiles[ti]; bd = depths[di]; }
    }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  h->tile = bt;
  h->o.batchDepth = bd;
  cudaMemcpyAsync(h->stats, st, 16, cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(h->gradCam, cg.data(), cg.size() * 4, cudaMemcpyHostToDevice, s);
  GS_CK(cudaStreamSynchronize(s));
  if (rc) return rc;
  if (bestTile) *bestTile = bt;
  if (bestDepth) *bestDepth = bd;
  return check_status(h);
}

int gs_set_raster_config(gs_trainer* h, int32_t tile, int32_t batchDepth) {
  if (!h) return GS_E_INVALID;
  if (tile != 8 && tile != 16 && tile != 32) return fail(h, GS_E_INVALID, "tile must be 8, 16 or 32");
  if (batchDepth != 64 && batchDepth != 128 && batchDepth != 256)
    return fail(h, GS_E_INVALID, "batchDepth must be 64, 128 or 256");
  h->tile = tile;
  h->o.batchDepth = batchDepth;
  return GS_OK;
}

int gs_debug_lookback_timeout(int32_t device, uint32_t spinLimit, uint32_t* statusOut, double* msOut) {
  if (spinLimit == 0 || spinLimit > (1u << 22)) return GS_E_INVALID;
  const int rc = debug_lookback_timeout(device, spinLimit, statusOut, msOut);
  return rc == 0 ? GS_OK : rc == -3 ? GS_E_NOMEM : GS_E_CUDA;
}

int gs_set_tile_cull(gs_trainer* h, int32_t enable) {
  if (!h) return GS_E_INVALID;
  if (enable != 0 && enable != 1) return fail(h, GS_E_INVALID, "tileCull must be 0 or 1");
  h->o.tileCull = enable;
  return GS_OK;
}

int gs_set_stream(gs_trainer* h, void* stream) {
  if (!h) return GS_E_INVALID;
  cudaSetDevice(h->device);
  GS_CK(cudaStreamSynchronize(h->stream));
  if (!h->ownStream) h->ownStream = h->stream;
  h->stream = stream ? (cudaStream_t)stream : h->ownStream;
  return GS_OK;
}

int gs_profile(gs_trainer* h, int32_t enable) {
  if (!h) return GS_E_INVALID;
  h->profiling = enable != 0;
  return GS_OK;
}

int gs_profile_read(gs_trainer* h, double ms[4], uint32_t launches[4]) {
  if (!h || !ms || !launches) return GS_E_INVALID;
  cudaSetDevice(h->device);
  GS_CK(cudaStreamSynchronize(h->stream));
  // evPool holds, per launch: (start, end) pairs for its phases, a null
  // separator, then the 5 owned events to destroy.
  size_t i = 0, p = 0;
  while (i < h->evPool.size()) {
    if (h->evPhase[p] >= 0) {
      float t = 0.0f;
      cudaEventElapsedTime(&t, h->evPool[i], h->evPool[i + 1]);
      h->profMs[h->evPhase[p]] += t;
      h->profN[h->evPhase[p]] += 1;
      i += 2;
      ++p;
    } else {
      for (int k = 1; k <= 5; ++k) cudaEventDestroy(h->evPool[i + k]);
      i += 6;
      ++p;
    }
  }
  h->evPool.clear();
  h->evPhase.clear();
  for (int k = 0; k < 4; ++k) { ms[k] = h->profMs[k]; launches[k] = h->profN[k]; h->profMs[k] = 0; h->profN[k] = 0; }
  return GS_OK;
}

// refine(rng) (trainer.js:666-794).  Classification, compaction, the donor
// order and every parameter write run on the device; the host reads three
// counts and makes the rng() draws in the reference's order (the draws
// decide which donor each spawn copies, so they are inherently sequential).
int gs_refine(gs_trainer* h, gs_rng_fn rng, void* ctx, gs_refine_result* out) {
  if (!h || !out) return GS_E_INVALID;
  if (!rng) { rng = builtin_rng; ctx = h; }
  if (!h->ready) return fail(h, GS_E_INVALID, "setup() first");
  cudaSetDevice(h->device);
  cudaStream_t s = h->stream;
  const uint32_t n = h->n, cap = h->cap;
  if (!h->rf.deadFlag) {
    int rc;
#define GS_AL(ptr, cnt) if ((rc = dalloc(h, &(ptr), (cnt))) != GS_OK) return rc;
    GS_AL(h->rf.deadFlag, cap);
    GS_AL(h->rf.donorFlag, cap);
    GS_AL(h->rf.deadOff, cap);
    GS_AL(h->rf.donorOff, cap);
    GS_AL(h->rf.deadList, cap);
    GS_AL(h->rf.donorList, cap);
    GS_AL(h->rf.splitSeq, cap);
    GS_AL(h->rf.plan, cap);
    GS_AL(h->rf.partials, (size_t)scan_partials_needed(cap) + 1);
    GS_AL(h->rf.counts, (size_t)4);
#undef GS_AL
  }
  launch_refine_classify(h->params, n, h->rf.deadFlag, h->rf.donorFlag, s);
  launch_exclusive_scan(h->rf.deadFlag, n, h->rf.deadOff, h->rf.partials, h->rf.counts + 0, s);
  launch_exclusive_scan(h->rf.donorFlag, n, h->rf.donorOff, h->rf.partials, h->rf.counts + 1, s);
  launch_refine_compact(h->params, n, h->rf.deadFlag, h->rf.deadOff, h->rf.donorFlag, h->rf.donorOff,
                        h->rf.deadList, h->rf.donorList, h->pkeys[0], h->pvals[0], s);
  uint32_t cnt[2] = {0, 0};
  GS_CK(cudaMemcpyAsync(cnt, h->rf.counts, 8, cudaMemcpyDeviceToHost, s));
  GS_CK(cudaStreamSynchronize(s));
  const uint32_t nDead = cnt[0], nDonors = cnt[1];
  std::memset(out, 0, sizeof(*out));
  out->n = n;
  if (nDonors < 16) { out->early = 1; return GS_OK; }  // trainer.js:695
  // stable sort of the donors by mean log-scale, descending (8 byte digits)
  GS_CK(cudaMemsetAsync(h->small, 0, 2057 * 4, s));
  RadixSortArgs ra{};
  ra.keys[0] = h->pkeys[0]; ra.keys[1] = h->pkeys[1];
  ra.vals[0] = h->pvals[0]; ra.vals[1] = h->pvals[1];
  ra.keyBytes = 8;
  ra.nItems = h->rf.counts + 1;
  ra.hist = h->small;
  ra.tileCounter = h->small + 2048;
  ra.status = h->lbStatus;
  ra.statusWord = h->small + 2060;
  ra.epoch = h->small + 2059;
  ra.passes = 8;
  ra.keepKeys = false;
  ra.histGrid = (unsigned)h->histGrid;
  ra.sweepGrid = (unsigned)h->sweepGrid;
  launch_radix_sort(ra, s);
  const uint32_t* bigSorted = h->pvals[0];  // 8 passes: result back in buffer 0
  // opacity-weighted donor sampling: cumulative sigmoid(opacity) over the
  // donor list (index order), in double; a clone pick is the first donor
  // whose cumulative weight exceeds rng() * total
  std::vector<double> cdf;
  if (h->o.donorSampling == 1) {
    std::vector<float> logit(nDonors);
    float* dLogit = reinterpret_cast<float*>(h->rf.splitSeq);  // free until the plan is applied
    launch_donor_opacity(h->params, h->rf.donorList, nDonors, dLogit, s);
    GS_CK(cudaMemcpyAsync(logit.data(), dLogit, (size_t)nDonors * 4, cudaMemcpyDeviceToHost, s));
    GS_CK(cudaStreamSynchronize(s));
    cdf.resize(nDonors);
    double acc = 0.0;
    for (uint32_t k = 0; k < nDonors; ++k) {
      acc += 1.0 / (1.0 + std::exp(-(double)logit[k]));
      cdf[k] = acc;
    }
  }
  // the host plan: rng() draws in the reference's order
  const uint32_t moveCap = (uint32_t)std::ceil((double)n * 0.05);
  const uint32_t moved = std::min(nDead, moveCap);
  const uint32_t L = std::min<uint32_t>(nDonors, std::max<uint32_t>(16u, nDonors >> 2));
  const uint32_t limit = std::min(cap, h->growLimit ? h->growLimit : cap);
  const double growUntil = h->o.growUntil >= 0.0 ? h->o.growUntil : 0.75 * h->horizon;
  uint32_t grown = 0;
  if ((double)h->iter < growUntil) {
    const double want = std::ceil((double)n * h->o.growRate);
    grown = (uint32_t)std::max(0.0, std::min(want, (double)limit - (double)n));
  }
  std::vector<uint32_t> big(L);
  for (uint32_t k = 0; k < L; ++k) big[k] = k;
  std::vector<RefineSpawn> plan((size_t)moved + grown);
  auto gauss = [&]() {
    const double u = std::max(1e-9, rng(ctx)), w = rng(ctx);
    return std::sqrt(-2.0 * std::log(u)) * std::cos(2.0 * M_PI * w);
  };
  for (size_t q = 0; q < plan.size(); ++q) {
    const bool allowSplit = q >= moved;
    bool doSplit = false;
    if (allowSplit && big.size() > 16) doSplit = rng(ctx) < 0.7;
    RefineSpawn& sp = plan[q];
    if (doSplit) {
      const size_t di = (size_t)(int32_t)(rng(ctx) * (double)big.size());
      sp.pos = big[di];
      big[di] = big.back();
      big.pop_back();
      sp.split = 1;
    } else {
      const double u = rng(ctx);
      if (cdf.empty()) {
        sp.pos = (uint32_t)(int32_t)(u * (double)nDonors);
      } else {
        const size_t k = (size_t)(std::upper_bound(cdf.begin(), cdf.end(), u * cdf.back()) - cdf.begin());
        sp.pos = (uint32_t)std::min<size_t>(k, nDonors - 1);
      }
      sp.split = 0;
    }
    for (int k = 0; k < 3; ++k) sp.g[k] = gauss();
  }
  if (!plan.empty()) {
    GS_CK(cudaMemcpyAsync(h->rf.plan, plan.data(), plan.size() * sizeof(RefineSpawn), cudaMemcpyHostToDevice, s));
    GS_CK(cudaMemsetAsync(h->rf.splitSeq, 0xFF, (size_t)cap * 4, s));
    RefineApplyArgs a{};
    a.plan = h->rf.plan;
    a.count = (uint32_t)plan.size();
    a.moved = moved;
    a.n = n;
    a.deadList = h->rf.deadList;
    a.donorList = h->rf.donorList;
    a.bigSorted = bigSorted;
    a.splitSeq = h->rf.splitSeq;
    a.params = h->params;
    a.m = h->m;
    a.v = h->v;
    a.sh = h->sh;
    a.shM = h->shM;
    a.shV = h->shV;
    a.shr = (int)(3 * h->K);
    launch_refine_apply(a, h->rf.splitSeq, s);
  }
  if (grown > 0) {
    h->n = n + grown;
    // camUniforms are rebuilt without a camera index and at the full SH
    // degree after growth (trainer.js:768)
    h->camIdxZero = true;
    for (auto& a : h->camActiveSh) a = (float)h->o.shDeg;
  }
  // tile-pressure telemetry over the most recent raster's tiles (trainer.js:779-790)
  launch_max_u32(h->tileCnt, h->lastTotalTiles, h->rf.counts + 2, s);
  uint32_t maxTile = 0;
  GS_CK(cudaMemcpyAsync(&maxTile, h->rf.counts + 2, 4, cudaMemcpyDeviceToHost, s));
  GS_CK(cudaStreamSynchronize(s));
  int rc = check_status(h);
  if (rc) return rc;
  out->moved = moved;
  out->grown = grown;
  out->n = h->n;
  out->maxTile = maxTile;
  out->overflow = (uint32_t)h->overflowTiles;
  out->early = 0;
  return GS_OK;
}

}  // extern "C"
