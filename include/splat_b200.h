/* splat_b200.h -- C ABI of libsplat_b200.so, the B200-native training step
 * behind splat.js's createTrainer API (src/index.js:56-58).
 *
 * One handle = one trainer = one CUDA stream on one device.  Handles are not
 * re-entrant: JavaScript drives one from a single thread, as the reference's
 * GSTrainer is driven (src/session.js:447-546).  Inputs are copied at call
 * time (like GPUQueue.writeBuffer); outputs go to caller-owned host buffers;
 * device memory belongs to the handle.  Every function returns 0 on success
 * or a negative GS_E* code; gs_last_error() then describes the failure.
 * Step functions only enqueue work (like stepOnce's queue.submit); functions
 * that return data synchronise the handle's stream.
 *
 * Parameter layout (src/gs/shaders.js:14-22): 16 f32 per splat
 *   [0-2 pos, 3-5 logScale, 6-9 quat (w,x,y,z, raw), 10-12 colour logits,
 *    13 opacity logit, 14-15 pad];
 * SH: 3*K f32 per splat, channel-major (K red, K green, K blue),
 *   K = (shDeg+1)^2 - 1.
 */
#ifndef SPLAT_B200_H
#define SPLAT_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GS_ABI_VERSION 2  /* 2: gs_options.donorSampling */

#if defined(__GNUC__)
#define GS_API __attribute__((visibility("default")))
#else
#define GS_API
#endif

#define GS_OK 0
#define GS_E_INVALID (-1)  /* bad argument or call order (the reference throws Error) */
#define GS_E_CUDA (-2)     /* CUDA runtime failure */
#define GS_E_NOMEM (-3)    /* device allocation failed */
#define GS_E_DEVICE (-4)   /* device status word reported a fault (look-back timeout, entry overflow) */
#define GS_E_LIMIT (-5)    /* a documented size limit was exceeded */

typedef struct gs_trainer gs_trainer;

/* GSTrainer constructor options (src/gs/trainer.js:18-49, 105-107, 300-341). */
typedef struct gs_options {
  float eCut;          /* opts.eCut: exponent cutoff, default 4.5 (shaders.js:44) */
  float aMin;          /* opts.aMin: minimum alpha, default 0.0039 (shaders.js:45) */
  float radClamp;      /* opts.radClamp: bin radius clamp, fraction of width, default 1 (shaders.js:46-53) */
  float anisoReg;      /* opts.anisoReg, default 0.005 (trainer.js:74) */
  int32_t shDeg;       /* opts.shDeg, default 2 (trainer.js:32) */
  int32_t tileGrad;    /* opts.tileGrad (trainer.js:26): accepted; gradients are identical either way */
  uint64_t entriesCap; /* opts.entriesCap; 0 = reference default (trainer.js:48-49) */
  uint32_t maxSplats;  /* opts.maxSplats; 0 = unset (cap limit 600000, trainer.js:105-107) */
  uint32_t maxIters;   /* opts.maxIters: schedule horizon, default 60000 (trainer.js:319) */
  /* options the reference uses in double arithmetic on the host */
  double capMult;      /* opts.capMult, default 4 (trainer.js:106) */
  double minScale;     /* opts.minScale, default 1e-4 (trainer.js:338) */
  double growRate;     /* opts.growRate, default 0.15 (trainer.js:763) */
  double growUntil;    /* opts.growUntil; negative = 0.75 * horizon (trainer.js:762) */
  float opacityReg;    /* opts.opacityReg, default 0.01 (trainer.js:341) */
  float shLr;          /* opts.shLr, default 1.25e-4 (trainer.js:302) */
  /* B200 options (no reference counterpart) */
  int32_t tile;            /* raster tile edge in pixels: 8, 16 (the reference's TILE) or 32 */
  int32_t batchDepth;      /* splat records staged per shared-memory batch: 64, 128 or 256 */
  int32_t maxBatch;        /* most views one gs_step_batch may take (buffers are sized for it) */
  int32_t backwardVariant; /* 0: recompute transmittance from the final T (reference); 1: stored-state */
  int32_t persistent;      /* 1: raster over a persistent (view, tile) work queue, heaviest tiles first */
  int32_t useGraphs;       /* 1: capture each step shape in a CUDA graph and replay it */
  int32_t device;          /* CUDA device ordinal */
  int32_t tileCull;        /* 1: tile lists keep only entries whose splat can reach a pixel of the tile
                              (exact ellipse/tile test); images and gradients are identical either way */
  int32_t donorSampling;   /* refine's clone donors: 0 uniform over the donors (the reference,
                              trainer.js:722); 1 opacity-weighted (probability proportional to
                              sigmoid(opacity logit)), one rng() draw per pick either way */
} gs_options;

/* One camera of setup's cams[] (trainer.js:95-99) with the exposure state
 * (g = log gain, b = bias) that _camUniform reads (trainer.js:357). */
typedef struct gs_camera {
  float R[9];     /* world-to-camera rotation, row-major */
  float t[3];
  float f, cx, cy;
  int32_t w, h;   /* training resolution */
  int32_t imgIdx; /* index into setup's images[] */
  double g, b;    /* log exposure gain and bias (JavaScript numbers) */
} gs_camera;

/* One training image of setup's images[] (trainer.js:98): tw*th RGB f32,
 * r < 0 marks an invalid pixel (trainer.js:133). */
typedef struct gs_image {
  uint32_t tw, th;
  const float* rgb;
} gs_image;

/* Trainer fields the reference's callers read (session.js:284-305, 349,
 * 484-485; app.js:830, 933, 1100, 1157). */
typedef struct gs_state {
  uint32_t iter, n, cap, shDeg, shK, stride, ncams, maxTiles;
  uint64_t pixelsSeen;
  uint64_t entriesCap;
  uint32_t horizon;
  uint32_t lastEntries;   /* kept (tile, splat) entries of the most recent raster */
  uint32_t stepUploadBytes; /* host->device bytes one step copies (view records + Adam parameters) */
  uint32_t lastLaunches;  /* kernels the most recent step enqueued (graph nodes that are kernels) */
} gs_state;

/* refine() result (trainer.js:695, 793). early = the donors<16 return. */
typedef struct gs_refine_result {
  uint32_t moved, grown, n, maxTile;
  uint32_t overflow;
  int32_t early;
} gs_refine_result;

/* rng() of refine(rng) (trainer.js:666): a double in [0, 1). */
typedef double (*gs_rng_fn)(void* ctx);

/* Defaults of the GSTrainer constructor (trainer.js:18-49). */
GS_API int gs_default_options(gs_options* out);
/* GSTrainer.create / constructor (trainer.js:13-36). */
GS_API int gs_create(const gs_options* opts, gs_trainer** out);
GS_API void gs_destroy(gs_trainer* h);
/* Description of the last failure of h (or of gs_create when h is NULL). */
GS_API const char* gs_last_error(const gs_trainer* h);
GS_API int gs_abi_version(void);

/* GSTrainer.setup(gaussians, cams, images, maxViewW, maxViewH, sceneRadius)
 * (trainer.js:100-355).  sh may be NULL (zero-initialised as WebGPU buffers
 * are). */
GS_API int gs_setup(gs_trainer* h, const float* params, uint32_t n, const float* sh, const gs_camera* cams,
             uint32_t ncams, const gs_image* images, uint32_t nimages, uint32_t maxViewW, uint32_t maxViewH,
             double sceneRadius);
GS_API int gs_get_state(const gs_trainer* h, gs_state* out);
/* trainer.iter / trainer.horizon / trainer.growLimit writes (session.js:348-349, app.js). */
GS_API int gs_set_iter(gs_trainer* h, uint32_t iter);
GS_API int gs_set_horizon(gs_trainer* h, uint32_t horizon);
GS_API int gs_set_grow_limit(gs_trainer* h, uint32_t growLimit);
/* Replace camera ci (pose / exposure updates of _applyCamGrads, trainer.js:512-533). */
GS_API int gs_set_camera(gs_trainer* h, uint32_t ci, const gs_camera* cam);

/* stepOnce (trainer.js:398-458) on camera ci; the caller keeps the rand()
 * camera pick and the holdout skip (trainer.js:400-406). */
GS_API int gs_step(gs_trainer* h, uint32_t ci);
/* One optimiser step over several views (uneven resolutions allowed): every
 * view is projected, binned, rendered and backpropagated in one pass over a
 * shared (view, tile) queue; the per-view parameter gradients are summed in
 * view order and Adam runs once.  iter advances by one. */
GS_API int gs_step_batch(gs_trainer* h, const uint32_t* ci, uint32_t nviews);

/* readLoss (trainer.js:615-631): copies and resets stats[4] = {SSE*16,
 * Charbonnier*32768, valid px, dropped tiles}; resets pixelsSeen. */
GS_API int gs_read_stats(gs_trainer* h, uint32_t stats[4]);
/* readLoss as the reference uses it, a Promise (trainer.js:615-631): enqueues
 * the copy of stats[4] into `stats` (pinned host memory, else the copy is
 * synchronous) and the reset, and returns at once; the values are valid after
 * gs_sync.  Status bits and dropped-tile totals are checked at that sync by
 * the caller (gs_sync reports device faults). */
GS_API int gs_read_stats_async(gs_trainer* h, uint32_t* stats);
/* readGaussians (trainer.js:797-817): params n*16, sh n*3K (either may be NULL). */
/* PLY export: bakeOpacityCompensation (ply.js:17-39; bake = 0 skips it, f the
 * focal length, camPositions ncams xyz JavaScript numbers) followed by
 * gaussiansToPly (ply.js:45-99) of the current Gaussians (with SH when
 * shDeg > 0), computed on the device in double precision as the JavaScript
 * does.  Writes the binary PLY (text header + n records) to out; out = NULL
 * only reports the size in *size; cap < size gives GS_E_LIMIT. */
GS_API int gs_export_ply(gs_trainer* h, int32_t bake, double f, const double* camPositions, uint32_t ncams,
                         uint8_t* out, uint64_t cap, uint64_t* size);
GS_API int gs_read_gaussians(gs_trainer* h, float* params, float* sh, uint32_t* n);
/* Overwrite the first n splats' parameters / SH (the parameter pokes of
 * gradcheck.js:320-323; either pointer may be NULL). */
GS_API int gs_write_gaussians(gs_trainer* h, const float* params, const float* sh, uint32_t n);
/* No reference counterpart: zeroes the Adam and SH-Adam moments of every
 * slot, as setup() does (trainer.js:100-355), so a model written with
 * gs_write_gaussians trains from the same optimiser state as a fresh setup. */
GS_API int gs_reset_moments(gs_trainer* h);
/* Adam moments (for refine parity checks): m, v n*16; shM, shV n*3K. */
GS_API int gs_read_moments(gs_trainer* h, float* m, float* v, float* shM, float* shV);

/* renderView(camParams, ctx, trainMode, offset) (trainer.js:634-655) into a
 * host buffer of cam->w * cam->h * 4 f32 (RGB, alpha = 1 - T) instead of a
 * canvas.  trainMode 1 also accumulates loss statistics and gradients, as
 * the reference's render pass does. */
GS_API int gs_render(gs_trainer* h, const gs_camera* cam, int32_t trainMode, uint32_t offset, float* outRGBA);
/* _evalPass(ci, override) (trainer.js:542-574): one training-path pass
 * without Adam on camera ci (or on cam when not NULL), stats reset before;
 * returns stats[4] and the (ncams+1)*8 camera gradients (drained). */
GS_API int gs_eval_pass(gs_trainer* h, uint32_t ci, const gs_camera* cam, uint32_t stats[4], int32_t* camGrad);
/* gradcheck's runPass (gradcheck.js:273-284): raster + chain, no Adam;
 * returns gradF n*16 and shGrad n*3K (either may be NULL) and stats[4]. */
GS_API int gs_grad_pass(gs_trainer* h, uint32_t ci, float* gradF, float* shGrad, uint32_t stats[4]);
/* Camera-gradient accumulator (ncams+1)*8 i32 (trainer.js:173); reset drains it. */
GS_API int gs_read_cam_grads(gs_trainer* h, int32_t* out, int32_t reset);

/* refine(rng) (trainer.js:666-794): dead/donor classification, donor order
 * and the parameter writes run on the device; only rng() draws are made on
 * the host, in the reference's order.  gs_options.donorSampling = 1 picks
 * clone donors by opacity weight from the same draws.  rng = NULL (the
 * reference's default, Math.random) draws from the handle's own generator,
 * xorshift128+ with a fixed starting state that continues across calls
 * (ctx unused): reproducible, and no call per draw into the caller. */
GS_API int gs_refine(gs_trainer* h, gs_rng_fn rng, void* ctx, gs_refine_result* out);
/* device.queue.onSubmittedWorkDone() (session.js:520, 542): waits for the stream. */
GS_API int gs_sync(gs_trainer* h);

/* ---- measurement hooks (no reference counterpart) ----
 * Run the handle's work on the caller's CUDA stream (a cudaStream_t; NULL
 * restores the handle's own stream), so CUDA events the caller records on
 * that stream bracket the step. */
GS_API int gs_set_stream(gs_trainer* h, void* stream);
/* Per-phase CUDA-event timing: while enabled, steps run without graph replay
 * and each phase (0 projection + tile counts, 1 presort + entry expansion + tile
 * sort + work order, 2 raster, 3 chain + Adam) is
 * bracketed by events on the launching stream.  gs_profile_read returns the
 * summed milliseconds and the number of timed launches per phase, then
 * clears them. */
GS_API int gs_profile(gs_trainer* h, int32_t enable);
GS_API int gs_profile_read(gs_trainer* h, double ms[4], uint32_t launches[4]);
/* FP32 FMA throughput of device `device` in TFLOP/s (an FFMA-chain kernel),
 * the peak the raster kernels' roofline is quoted against. */
GS_API int gs_probe_fp32_peak(int32_t device, double* tflops);
/* Check of the rasteriser's reciprocal of 1 - alpha (no reference
 * counterpart): compares it with IEEE 1/x for every float x in [2^-7, 1];
 * *mismatches must be 0 (*firstBits: the first failing x's bits). */
GS_API int gs_debug_check_rcp(int32_t device, uint64_t* mismatches, uint32_t* firstBits);

/* ---- target ingestion ----
 * A training frame for gs_undistort_frames: tw x th pixels, 3 floats each
 * (rgb, modified in place), fw = the width the camera model's focal length
 * fFeat refers to (the frame's feature-extraction width). */
typedef struct gs_frame {
  uint32_t tw, th;
  double fw;
  float* rgb;
} gs_frame;
/* undistortFrames(frames, recon) (session.js:44-80): resamples every frame
 * in place through the radial model D = 1 + k1 r^2 + k2 r^4 (bilinear, in
 * double precision, float32 results identical to the JavaScript's); a pixel
 * whose source falls outside the frame becomes -1 in all three channels,
 * which setup packs as an invalid target.  |k1| and |k2| both below 0.01
 * change nothing (*resampled = 0), as in the reference.  Runs on `device`;
 * allocates and frees its own scratch. */
GS_API int gs_undistort_frames(int32_t device, gs_frame* frames, uint32_t nframes, double k1, double k2,
                               double fFeat, int32_t* resampled);
/* The packed RGBA8 targets gs_setup built (trainer.js:115-139), pixels
 * [0, count) in camera-offset order (no reference counterpart: parity
 * introspection). */
GS_API int gs_debug_targets(gs_trainer* h, uint32_t* out, uint64_t count);

/* ---- allocation-free entry sort (no counterpart in the reference) ----
 * For callers that cannot call cudaMalloc: code whose device memory is owned
 * by another runtime's pool (a host application or binding that forbids
 * foreign allocations), and code on a path where an allocation -- which may
 * synchronise the device -- is not allowed.
 * Stable LSD radix sort of n (key, value) pairs held in device memory, in
 * place, by key: the sort that orders the trainer's (tile id, splat id)
 * entries, run with its scratch in statically sized device arrays instead
 * of buffers the trainer allocates, so the call allocates nothing.  Keys
 * must be below 2^keyBits: the sort runs ceil(keyBits / 8) passes over
 * 8-bit digits, so key bits from keyBits up to the next multiple of 8 would
 * also order the output.  Every GPU that loads the library holds that
 * scratch (about 8.5 MB) until the process exits.  n above
 * GS_STATIC_SORT_MAX returns GS_E_LIMIT.
 * keys/vals: device pointers on the current device; stream may be NULL.
 * The first call on a device sets up the launch grids (device attributes
 * and kernel occupancy), so make it before any stream capture; every call
 * looks the scratch's device addresses up again.  Each call copies the
 * device status word to the host and synchronises `stream` before it
 * returns, so it returns after the sort has finished (GS_E_DEVICE on a
 * look-back timeout).  A CUDA error that an earlier call on the thread left
 * pending is returned as GS_E_CUDA before any work, and stays pending.
 * The scratch is shared: calls that overlap in time race. */
#define GS_STATIC_SORT_MAX (1u << 20)
GS_API int gs_sort_entries_static(uint32_t* keys, uint32_t* vals, uint32_t n, uint32_t keyBits, void* stream);

/* ---- raster configuration (no reference counterpart; results do not depend
 * on it: images and gradients are identical for every tile size and depth,
 * only the per-tile entry lists follow the tile size) ----
 * gs_autotune times the training pass on views ci[0..nviews) for each tile
 * edge {8, 16, 32} x splat-batch depth {64, 128, 256}, keeps the fastest
 * and reports it; msOut (9 floats, tile-major) may be NULL. */
GS_API int gs_autotune(gs_trainer* h, const uint32_t* ci, uint32_t nviews, int32_t reps, int32_t* bestTile,
                       int32_t* bestDepth, float* msOut);
GS_API int gs_set_raster_config(gs_trainer* h, int32_t tile, int32_t batchDepth);
/* Switch the tile cull (gs_options.tileCull) for later steps: 0 gives the
 * reference's full rectangle lists (used to count the reference's pixel-entry
 * pairs); results are identical either way. */
GS_API int gs_set_tile_cull(gs_trainer* h, int32_t enable);

/* ---- introspection of the most recent raster (parity checks) ----
 * gs_raster_pass runs project -> bin -> raster (no chain, no Adam) on views
 * ci[0..nviews); mode 1 = forward only, 3 = forward + loss + backward. */
GS_API int gs_raster_pass(gs_trainer* h, const uint32_t* ci, uint32_t nviews, int32_t mode);
/* Per-splat raster record of view slot `view`: rec n*12 f32
 * (mx, my, cA/2, cB, cC/2, opa*comp, r, g, b, opa, -1/(2(1+lambda_max)), 1 - opa),
 * rect n*2 u32 (x0 | y0<<16, x1 | y1<<16; 0xFFFFFFFF = culled). */
GS_API int gs_debug_records(gs_trainer* h, uint32_t view, float* rec12, uint32_t* rect2);
/* Binning of view slot `view`: tileCnt[tiles], ranges[2*tiles] (global entry
 * indices), and the batch's sorted splat ids (up to cap; *nEntries = total). */
GS_API int gs_debug_binning(gs_trainer* h, uint32_t view, uint32_t* tileCnt, uint32_t* ranges, uint32_t* ids,
                     uint64_t cap, uint64_t* nEntries);
/* Pixels of view slot `view`: rgba w*h*4, finalT w*h, end w*h (relative). */
GS_API int gs_debug_pixels(gs_trainer* h, uint32_t view, float* rgba, float* finalT, uint32_t* endIdx);
/* Fixed-point screen-space gradients of view slot `view`: n*10 i32
 * (shaders.js:26-28 slots 0-9); clear = 1 zeroes them afterwards. */
/* Failure-detection check (no reference counterpart): runs one radix-sort
 * pass whose decoupled look-back can never complete (its first block is
 * never processed), so the waiting blocks give up after spinLimit spins
 * (1 .. 2^22) and set the look-back-timeout bit (1) of the status word,
 * returned in *statusOut with the kernel's time in ms.  Nothing hangs and the
 * device stays usable; the trainer reports the same bit as GS_E_DEVICE. */
GS_API int gs_debug_lookback_timeout(int32_t device, uint32_t spinLimit, uint32_t* statusOut, double* msOut);
GS_API int gs_debug_gradp(gs_trainer* h, uint32_t view, int32_t* gradP10, int32_t clear);

#ifdef __cplusplus
}
#endif
#endif /* SPLAT_B200_H */
