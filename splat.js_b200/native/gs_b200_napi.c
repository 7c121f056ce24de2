/* gs_b200_napi.c -- Node-API addon: splat.js's JavaScript calls the B200
 * training step in libsplat_b200.so (C ABI, include/splat_b200.h) through
 * these functions; js/trainer_b200.js wraps them in a class with the surface
 * of the reference's GSTrainer (src/gs/trainer.js).
 *
 * Threading.  JavaScript runs on one thread; the reads the reference returns
 * as Promises (readLoss, readGaussians, onSubmittedWorkDone) run their
 * synchronising library call on a libuv worker (napi async work) and resolve
 * on the JavaScript thread.  A trainer handle is not re-entrant, so every
 * library call on it, from either thread, holds the handle's mutex: a step
 * issued while a read waits for the stream blocks until the read returns.
 * refine(rng) runs on the JavaScript thread: the library calls rng() from the
 * thread that called gs_refine (src/gs/trainer.js:666 draws Math.random-style
 * numbers in order), so the callback calls the JavaScript function directly.
 *
 * Errors: a negative status throws (or rejects with) Error(gs_last_error),
 * as the reference throws on setup-time limits (trainer.js:122-126). */
#include <node_api.h>
#include <pthread.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "splat_b200.h"

typedef struct {
  gs_trainer* h;
  pthread_mutex_t mu;
} Handle;

/* ---- small helpers ---------------------------------------------------- */
#define NAPI_OK(env, call)                                   \
  do {                                                       \
    if ((call) != napi_ok) {                                 \
      napi_throw_error((env), NULL, "gs_b200: " #call);      \
      return NULL;                                           \
    }                                                        \
  } while (0)

static napi_value js_undefined(napi_env env) {
  napi_value u;
  napi_get_undefined(env, &u);
  return u;
}

static napi_value throw_gs(napi_env env, const Handle* H, int rc) {
  char msg[512];
  snprintf(msg, sizeof msg, "splat_b200 error %d: %s", rc, gs_last_error(H ? H->h : NULL));
  napi_throw_error(env, NULL, msg);
  return NULL;
}

static Handle* arg_handle(napi_env env, napi_value v) {
  void* p = NULL;
  if (napi_get_value_external(env, v, &p) != napi_ok || !p) {
    napi_throw_error(env, NULL, "gs_b200: expected a trainer handle");
    return NULL;
  }
  return (Handle*)p;
}

static int get_num(napi_env env, napi_value obj, const char* name, double* out) {
  bool has = false;
  napi_value v;
  napi_valuetype t;
  if (napi_has_named_property(env, obj, name, &has) != napi_ok || !has) return 0;
  if (napi_get_named_property(env, obj, name, &v) != napi_ok) return 0;
  if (napi_typeof(env, v, &t) != napi_ok || (t != napi_number && t != napi_boolean)) return 0;
  if (t == napi_boolean) {
    bool b = false;
    napi_get_value_bool(env, v, &b);
    *out = b ? 1.0 : 0.0;
    return 1;
  }
  return napi_get_value_double(env, v, out) == napi_ok;
}

static int get_vec(napi_env env, napi_value obj, const char* name, double* out, uint32_t count) {
  napi_value arr, e;
  if (napi_get_named_property(env, obj, name, &arr) != napi_ok) return 0;
  for (uint32_t k = 0; k < count; ++k) {
    if (napi_get_element(env, arr, k, &e) != napi_ok) return 0;
    if (napi_get_value_double(env, e, &out[k]) != napi_ok) return 0;
  }
  return 1;
}

/* typed-array data of the expected type (NULL for null/undefined) */
static void* typed(napi_env env, napi_value v, napi_typedarray_type want, size_t* len, int* bad) {
  napi_valuetype t;
  *bad = 0;
  if (len) *len = 0;
  if (napi_typeof(env, v, &t) != napi_ok) { *bad = 1; return NULL; }
  if (t == napi_null || t == napi_undefined) return NULL;
  napi_typedarray_type tt;
  size_t n = 0, off = 0;
  void* data = NULL;
  napi_value ab;
  if (napi_get_typedarray_info(env, v, &tt, &n, &data, &ab, &off) != napi_ok || tt != want) {
    *bad = 1;
    return NULL;
  }
  if (len) *len = n;
  return data;
}

/* one camera record {R[9], t[3], f, cx, cy, w, h, imgIdx, g, b} (trainer.js:95-99, :357) */
static int read_camera(napi_env env, napi_value obj, gs_camera* c) {
  double R[9], t[3], x;
  memset(c, 0, sizeof *c);
  if (!get_vec(env, obj, "R", R, 9) || !get_vec(env, obj, "t", t, 3)) return 0;
  for (int k = 0; k < 9; ++k) c->R[k] = (float)R[k];
  for (int k = 0; k < 3; ++k) c->t[k] = (float)t[k];
  if (!get_num(env, obj, "f", &x)) return 0;
  c->f = (float)x;
  if (!get_num(env, obj, "cx", &x)) return 0;
  c->cx = (float)x;
  if (!get_num(env, obj, "cy", &x)) return 0;
  c->cy = (float)x;
  if (get_num(env, obj, "w", &x)) c->w = (int32_t)x;
  if (get_num(env, obj, "h", &x)) c->h = (int32_t)x;
  if (get_num(env, obj, "imgIdx", &x)) c->imgIdx = (int32_t)x;
  if (get_num(env, obj, "g", &x)) c->g = x;
  if (get_num(env, obj, "b", &x)) c->b = x;
  return 1;
}

static napi_value make_u32(napi_env env, uint32_t v) {
  napi_value r;
  napi_create_uint32(env, v, &r);
  return r;
}

static napi_value make_f64(napi_env env, double v) {
  napi_value r;
  napi_create_double(env, v, &r);
  return r;
}

static napi_value new_typed(napi_env env, napi_typedarray_type type, size_t count, size_t elem, void** data) {
  napi_value ab, arr;
  if (napi_create_arraybuffer(env, count * elem, data, &ab) != napi_ok) return NULL;
  if (napi_create_typedarray(env, type, count, ab, 0, &arr) != napi_ok) return NULL;
  return arr;
}

static void finalize_handle(napi_env env, void* data, void* hint) {
  (void)env;
  (void)hint;
  Handle* H = (Handle*)data;
  gs_destroy(H->h);
  pthread_mutex_destroy(&H->mu);
  free(H);
}

/* ---- construction and setup ------------------------------------------ */
/* create(opts): GSTrainer constructor options (trainer.js:18-49) */
static napi_value Create(napi_env env, napi_callback_info info) {
  size_t argc = 1;
  napi_value argv[1];
  NAPI_OK(env, napi_get_cb_info(env, info, &argc, argv, NULL, NULL));
  gs_options o;
  gs_default_options(&o);
  if (argc >= 1) {
    napi_valuetype t;
    napi_typeof(env, argv[0], &t);
    if (t == napi_object) {
      double x;
      napi_value js = argv[0];
#define OPT_F(name) if (get_num(env, js, #name, &x)) o.name = (float)x;
#define OPT_I(name) if (get_num(env, js, #name, &x)) o.name = (int32_t)x;
#define OPT_U(name) if (get_num(env, js, #name, &x)) o.name = (uint32_t)x;
#define OPT_D(name) if (get_num(env, js, #name, &x)) o.name = x;
      OPT_F(eCut) OPT_F(aMin) OPT_F(radClamp) OPT_F(anisoReg) OPT_I(shDeg) OPT_I(tileGrad)
      OPT_U(maxSplats) OPT_U(maxIters) OPT_D(capMult) OPT_D(minScale) OPT_D(growRate) OPT_D(growUntil)
      OPT_F(opacityReg) OPT_F(shLr) OPT_I(tile) OPT_I(batchDepth) OPT_I(maxBatch) OPT_I(backwardVariant)
      OPT_I(persistent) OPT_I(useGraphs) OPT_I(device) OPT_I(tileCull) OPT_I(donorSampling)
      if (get_num(env, js, "entriesCap", &x)) o.entriesCap = (uint64_t)x;
#undef OPT_F
#undef OPT_I
#undef OPT_U
#undef OPT_D
    }
  }
  Handle* H = (Handle*)calloc(1, sizeof(Handle));
  if (!H) return throw_gs(env, NULL, GS_E_NOMEM);
  int rc = gs_create(&o, &H->h);
  if (rc != GS_OK) {
    free(H);
    return throw_gs(env, NULL, rc);
  }
  pthread_mutex_init(&H->mu, NULL);
  napi_value ext;
  NAPI_OK(env, napi_create_external(env, H, finalize_handle, NULL, &ext));
  return ext;
}

/* setup(h, data Float32Array(n*16), n, sh Float32Array|null, cams[], images[], maxViewW, maxViewH,
 *       sceneRadius) (trainer.js:100-355); images[k] = {tw, th, rgb Float32Array(3*tw*th)} */
static napi_value Setup(napi_env env, napi_callback_info info) {
  size_t argc = 9;
  napi_value argv[9];
  NAPI_OK(env, napi_get_cb_info(env, info, &argc, argv, NULL, NULL));
  if (argc < 9) { napi_throw_error(env, NULL, "setup: 9 arguments"); return NULL; }
  Handle* H = arg_handle(env, argv[0]);
  if (!H) return NULL;
  int bad = 0, bad2 = 0;
  size_t np = 0, ns = 0;
  const float* params = (const float*)typed(env, argv[1], napi_float32_array, &np, &bad);
  uint32_t n = 0;
  NAPI_OK(env, napi_get_value_uint32(env, argv[2], &n));
  const float* sh = (const float*)typed(env, argv[3], napi_float32_array, &ns, &bad2);
  if (bad || bad2 || !params || np < (size_t)n * 16) {
    napi_throw_error(env, NULL, "setup: data must be a Float32Array of n*16, sh a Float32Array or null");
    return NULL;
  }
  uint32_t ncams = 0, nimg = 0;
  NAPI_OK(env, napi_get_array_length(env, argv[4], &ncams));
  NAPI_OK(env, napi_get_array_length(env, argv[5], &nimg));
  gs_camera* cams = (gs_camera*)calloc(ncams ? ncams : 1, sizeof(gs_camera));
  gs_image* imgs = (gs_image*)calloc(nimg ? nimg : 1, sizeof(gs_image));
  int okc = cams && imgs;
  for (uint32_t k = 0; okc && k < ncams; ++k) {
    napi_value c;
    okc = napi_get_element(env, argv[4], k, &c) == napi_ok && read_camera(env, c, &cams[k]);
  }
  for (uint32_t k = 0; okc && k < nimg; ++k) {
    napi_value im, rgb;
    double tw = 0, th = 0;
    size_t len = 0;
    okc = napi_get_element(env, argv[5], k, &im) == napi_ok && get_num(env, im, "tw", &tw) &&
          get_num(env, im, "th", &th) && napi_get_named_property(env, im, "rgb", &rgb) == napi_ok;
    if (okc) {
      imgs[k].tw = (uint32_t)tw;
      imgs[k].th = (uint32_t)th;
      imgs[k].rgb = (const float*)typed(env, rgb, napi_float32_array, &len, &bad);
      okc = !bad && imgs[k].rgb && len >= (size_t)imgs[k].tw * imgs[k].th * 3;
    }
  }
  uint32_t maxW = 0, maxH = 0;
  double radius = 0;
  okc = okc && napi_get_value_uint32(env, argv[6], &maxW) == napi_ok &&
        napi_get_value_uint32(env, argv[7], &maxH) == napi_ok &&
        napi_get_value_double(env, argv[8], &radius) == napi_ok;
  if (!okc) {
    free(cams);
    free(imgs);
    napi_throw_error(env, NULL, "setup: malformed cameras or images");
    return NULL;
  }
  pthread_mutex_lock(&H->mu);
  const int rc = gs_setup(H->h, params, n, sh, cams, ncams, imgs, nimg, maxW, maxH, radius);
  pthread_mutex_unlock(&H->mu);
  free(cams);
  free(imgs);
  if (rc != GS_OK) return throw_gs(env, H, rc);
  return js_undefined(env);
}

/* ---- fields ----------------------------------------------------------- */
/* state(h): the fields callers read (session.js:284-305, app.js) */
static napi_value State(napi_env env, napi_callback_info info) {
  size_t argc = 1;
  napi_value argv[1], o;
  NAPI_OK(env, napi_get_cb_info(env, info, &argc, argv, NULL, NULL));
  Handle* H = arg_handle(env, argv[0]);
  if (!H) return NULL;
  gs_state s;
  pthread_mutex_lock(&H->mu);
  const int rc = gs_get_state(H->h, &s);
  pthread_mutex_unlock(&H->mu);
  if (rc != GS_OK) return throw_gs(env, H, rc);
  NAPI_OK(env, napi_create_object(env, &o));
  napi_set_named_property(env, o, "iter", make_u32(env, s.iter));
  napi_set_named_property(env, o, "n", make_u32(env, s.n));
  napi_set_named_property(env, o, "cap", make_u32(env, s.cap));
  napi_set_named_property(env, o, "shDeg", make_u32(env, s.shDeg));
  napi_set_named_property(env, o, "shK", make_u32(env, s.shK));
  napi_set_named_property(env, o, "stride", make_u32(env, s.stride));
  napi_set_named_property(env, o, "ncams", make_u32(env, s.ncams));
  napi_set_named_property(env, o, "maxTiles", make_u32(env, s.maxTiles));
  napi_set_named_property(env, o, "pixelsSeen", make_f64(env, (double)s.pixelsSeen));
  napi_set_named_property(env, o, "entriesCap", make_f64(env, (double)s.entriesCap));
  napi_set_named_property(env, o, "horizon", make_u32(env, s.horizon));
  return o;
}

/* setIter / setHorizon / setGrowLimit(h, value) */
static napi_value set_u32(napi_env env, napi_callback_info info, int (*fn)(gs_trainer*, uint32_t)) {
  size_t argc = 2;
  napi_value argv[2];
  NAPI_OK(env, napi_get_cb_info(env, info, &argc, argv, NULL, NULL));
  Handle* H = arg_handle(env, argv[0]);
  if (!H) return NULL;
  uint32_t v = 0;
  NAPI_OK(env, napi_get_value_uint32(env, argv[1], &v));
  pthread_mutex_lock(&H->mu);
  const int rc = fn(H->h, v);
  pthread_mutex_unlock(&H->mu);
  return rc == GS_OK ? js_undefined(env) : throw_gs(env, H, rc);
}
static napi_value SetIter(napi_env env, napi_callback_info info) { return set_u32(env, info, gs_set_iter); }
static napi_value SetHorizon(napi_env env, napi_callback_info info) { return set_u32(env, info, gs_set_horizon); }
/* resetMoments(h): Adam moments back to setup()'s zeros (no reference counterpart) */
static napi_value ResetMoments(napi_env env, napi_callback_info info) {
  size_t argc = 1;
  napi_value argv[1];
  NAPI_OK(env, napi_get_cb_info(env, info, &argc, argv, NULL, NULL));
  Handle* H = arg_handle(env, argv[0]);
  if (!H) return NULL;
  pthread_mutex_lock(&H->mu);
  const int rc = gs_reset_moments(H->h);
  pthread_mutex_unlock(&H->mu);
  return rc == GS_OK ? js_undefined(env) : throw_gs(env, H, rc);
}
static napi_value SetGrowLimit(napi_env env, napi_callback_info info) {
  return set_u32(env, info, gs_set_grow_limit);
}

/* setCamera(h, ci, cam): the camUniforms rewrite of _applyCamGrads (trainer.js:512-533) */
static napi_value SetCamera(napi_env env, napi_callback_info info) {
  size_t argc = 3;
  napi_value argv[3];
  NAPI_OK(env, napi_get_cb_info(env, info, &argc, argv, NULL, NULL));
  Handle* H = arg_handle(env, argv[0]);
  if (!H) return NULL;
  uint32_t ci = 0;
  gs_camera c;
  NAPI_OK(env, napi_get_value_uint32(env, argv[1], &ci));
  if (!read_camera(env, argv[2], &c)) { napi_throw_error(env, NULL, "setCamera: malformed camera"); return NULL; }
  pthread_mutex_lock(&H->mu);
  const int rc = gs_set_camera(H->h, ci, &c);
  pthread_mutex_unlock(&H->mu);
  return rc == GS_OK ? js_undefined(env) : throw_gs(env, H, rc);
}

/* ---- training ----------------------------------------------------------- */
/* step(h, ci): stepOnce after the rand() camera pick made in JavaScript (trainer.js:398-471) */
static napi_value Step(napi_env env, napi_callback_info info) {
  size_t argc = 2;
  napi_value argv[2];
  NAPI_OK(env, napi_get_cb_info(env, info, &argc, argv, NULL, NULL));
  Handle* H = arg_handle(env, argv[0]);
  if (!H) return NULL;
  uint32_t ci = 0;
  NAPI_OK(env, napi_get_value_uint32(env, argv[1], &ci));
  pthread_mutex_lock(&H->mu);
  const int rc = gs_step(H->h, ci);
  pthread_mutex_unlock(&H->mu);
  return rc == GS_OK ? js_undefined(env) : throw_gs(env, H, rc);
}

/* stepBatch(h, Uint32Array of camera indices): one optimiser step over several views */
static napi_value StepBatch(napi_env env, napi_callback_info info) {
  size_t argc = 2;
  napi_value argv[2];
  NAPI_OK(env, napi_get_cb_info(env, info, &argc, argv, NULL, NULL));
  Handle* H = arg_handle(env, argv[0]);
  if (!H) return NULL;
  int bad = 0;
  size_t nv = 0;
  const uint32_t* ci = (const uint32_t*)typed(env, argv[1], napi_uint32_array, &nv, &bad);
  if (bad || !ci) { napi_throw_error(env, NULL, "stepBatch: cameras must be a Uint32Array"); return NULL; }
  pthread_mutex_lock(&H->mu);
  const int rc = gs_step_batch(H->h, ci, (uint32_t)nv);
  pthread_mutex_unlock(&H->mu);
  return rc == GS_OK ? js_undefined(env) : throw_gs(env, H, rc);
}

/* ---- Promise-returning reads (libuv worker) ------------------------------ */
enum { W_STATS, W_SYNC, W_GAUSSIANS };
typedef struct {
  Handle* H;
  int kind, rc;
  napi_deferred deferred;
  napi_async_work work;
  napi_ref keep[3];      /* handle and output arrays, alive until resolution */
  uint32_t stats[4];
  float* params;
  float* sh;
  uint32_t n, shK;
  char err[512];
} Work;

static void work_execute(napi_env env, void* data) {
  (void)env;
  Work* w = (Work*)data;
  pthread_mutex_lock(&w->H->mu);
  if (w->kind == W_STATS) w->rc = gs_read_stats(w->H->h, w->stats);
  else if (w->kind == W_SYNC) w->rc = gs_sync(w->H->h);
  else w->rc = gs_read_gaussians(w->H->h, w->params, w->sh, &w->n);
  if (w->rc != GS_OK) snprintf(w->err, sizeof w->err, "splat_b200 error %d: %s", w->rc, gs_last_error(w->H->h));
  pthread_mutex_unlock(&w->H->mu);
}

static void work_complete(napi_env env, napi_status status, void* data) {
  Work* w = (Work*)data;
  napi_value result = NULL;
  if (status != napi_ok || w->rc != GS_OK) {
    napi_value msg, err;
    napi_create_string_utf8(env, w->rc != GS_OK ? w->err : "gs_b200: async work cancelled", (size_t)-1, &msg);
    napi_create_error(env, NULL, msg, &err);
    napi_reject_deferred(env, w->deferred, err);
  } else {
    if (w->kind == W_STATS) {
      uint32_t* d = NULL;
      result = new_typed(env, napi_uint32_array, 4, 4, (void**)&d);
      if (result && d) memcpy(d, w->stats, sizeof w->stats);
    } else if (w->kind == W_SYNC) {
      result = js_undefined(env);
    } else {
      napi_value data, sh;
      napi_create_object(env, &result);
      napi_get_reference_value(env, w->keep[1], &data);
      napi_set_named_property(env, result, "data", data);
      napi_set_named_property(env, result, "n", make_u32(env, w->n));
      if (w->keep[2]) {
        napi_get_reference_value(env, w->keep[2], &sh);
      } else {
        napi_get_null(env, &sh);
      }
      napi_set_named_property(env, result, "sh", sh);
      napi_set_named_property(env, result, "shK", make_u32(env, w->shK));
    }
    napi_resolve_deferred(env, w->deferred, result ? result : js_undefined(env));
  }
  for (int k = 0; k < 3; ++k)
    if (w->keep[k]) napi_delete_reference(env, w->keep[k]);
  napi_delete_async_work(env, w->work);
  free(w);
}

static napi_value queue_work(napi_env env, napi_value handleArg, Work* w, const char* name) {
  napi_value promise, resource;
  NAPI_OK(env, napi_create_reference(env, handleArg, 1, &w->keep[0]));
  NAPI_OK(env, napi_create_promise(env, &w->deferred, &promise));
  NAPI_OK(env, napi_create_string_utf8(env, name, (size_t)-1, &resource));
  NAPI_OK(env, napi_create_async_work(env, NULL, resource, work_execute, work_complete, w, &w->work));
  NAPI_OK(env, napi_queue_async_work(env, w->work));
  return promise;
}

/* readStats(h) -> Promise<Uint32Array(4)>: readLoss's copy of the stats
 * (trainer.js:615-631); the library resets them and pixelsSeen */
static napi_value ReadStats(napi_env env, napi_callback_info info) {
  size_t argc = 1;
  napi_value argv[1];
  NAPI_OK(env, napi_get_cb_info(env, info, &argc, argv, NULL, NULL));
  Handle* H = arg_handle(env, argv[0]);
  if (!H) return NULL;
  Work* w = (Work*)calloc(1, sizeof(Work));
  if (!w) return throw_gs(env, H, GS_E_NOMEM);
  w->H = H;
  w->kind = W_STATS;
  return queue_work(env, argv[0], w, "gs_b200.readStats");
}

/* sync(h) -> Promise: device.queue.onSubmittedWorkDone() (session.js:520, 542) */
static napi_value Sync(napi_env env, napi_callback_info info) {
  size_t argc = 1;
  napi_value argv[1];
  NAPI_OK(env, napi_get_cb_info(env, info, &argc, argv, NULL, NULL));
  Handle* H = arg_handle(env, argv[0]);
  if (!H) return NULL;
  Work* w = (Work*)calloc(1, sizeof(Work));
  if (!w) return throw_gs(env, H, GS_E_NOMEM);
  w->H = H;
  w->kind = W_SYNC;
  return queue_work(env, argv[0], w, "gs_b200.sync");
}

/* readGaussians(h) -> Promise<{data, n, sh, shK}> (trainer.js:797-817): the
 * layout gaussiansToPly(data, n, sh, shK) reads (ply.js:45-99) */
static napi_value ReadGaussians(napi_env env, napi_callback_info info) {
  size_t argc = 1;
  napi_value argv[1];
  NAPI_OK(env, napi_get_cb_info(env, info, &argc, argv, NULL, NULL));
  Handle* H = arg_handle(env, argv[0]);
  if (!H) return NULL;
  gs_state s;
  pthread_mutex_lock(&H->mu);
  const int rc = gs_get_state(H->h, &s);
  pthread_mutex_unlock(&H->mu);
  if (rc != GS_OK) return throw_gs(env, H, rc);
  Work* w = (Work*)calloc(1, sizeof(Work));
  if (!w) return throw_gs(env, H, GS_E_NOMEM);
  w->H = H;
  w->kind = W_GAUSSIANS;
  w->shK = s.shK;
  napi_value data = new_typed(env, napi_float32_array, (size_t)s.n * 16, 4, (void**)&w->params);
  if (!data) { free(w); return throw_gs(env, H, GS_E_NOMEM); }
  NAPI_OK(env, napi_create_reference(env, data, 1, &w->keep[1]));
  if (s.shK) {
    napi_value sh = new_typed(env, napi_float32_array, (size_t)s.n * 3 * s.shK, 4, (void**)&w->sh);
    if (!sh) { napi_delete_reference(env, w->keep[1]); free(w); return throw_gs(env, H, GS_E_NOMEM); }
    NAPI_OK(env, napi_create_reference(env, sh, 1, &w->keep[2]));
  }
  return queue_work(env, argv[0], w, "gs_b200.readGaussians");
}

/* ---- views and evaluation ------------------------------------------------- */
/* renderView(h, cam, trainMode, offset, out Float32Array(w*h*4)|null) (trainer.js:634-655) */
static napi_value RenderView(napi_env env, napi_callback_info info) {
  size_t argc = 5;
  napi_value argv[5];
  NAPI_OK(env, napi_get_cb_info(env, info, &argc, argv, NULL, NULL));
  if (argc < 4) { napi_throw_error(env, NULL, "renderView: (h, cam, trainMode, offset[, out])"); return NULL; }
  Handle* H = arg_handle(env, argv[0]);
  if (!H) return NULL;
  gs_camera c;
  if (!read_camera(env, argv[1], &c)) { napi_throw_error(env, NULL, "renderView: malformed camera"); return NULL; }
  int32_t mode = 0;
  uint32_t offset = 0;
  NAPI_OK(env, napi_get_value_int32(env, argv[2], &mode));
  NAPI_OK(env, napi_get_value_uint32(env, argv[3], &offset));
  const size_t need = (size_t)c.w * (size_t)c.h * 4;
  float* out = NULL;
  napi_value arr = NULL;
  int bad = 0;
  size_t len = 0;
  if (argc >= 5) out = (float*)typed(env, argv[4], napi_float32_array, &len, &bad);
  if (bad || (out && len < need)) { napi_throw_error(env, NULL, "renderView: out too small"); return NULL; }
  if (out) arr = argv[4];
  else if (!(arr = new_typed(env, napi_float32_array, need, 4, (void**)&out))) return throw_gs(env, H, GS_E_NOMEM);
  pthread_mutex_lock(&H->mu);
  const int rc = gs_render(H->h, &c, mode, offset, out);
  pthread_mutex_unlock(&H->mu);
  return rc == GS_OK ? arr : throw_gs(env, H, rc);
}

/* evalPass(h, ci, cam|null) -> {stats, camGrad}: _evalPass (trainer.js:542-574) */
static napi_value EvalPass(napi_env env, napi_callback_info info) {
  size_t argc = 3;
  napi_value argv[3];
  NAPI_OK(env, napi_get_cb_info(env, info, &argc, argv, NULL, NULL));
  Handle* H = arg_handle(env, argv[0]);
  if (!H) return NULL;
  uint32_t ci = 0;
  NAPI_OK(env, napi_get_value_uint32(env, argv[1], &ci));
  gs_camera c;
  const gs_camera* cp = NULL;
  napi_valuetype t = napi_undefined;
  if (argc >= 3) napi_typeof(env, argv[2], &t);
  if (t == napi_object) {
    if (!read_camera(env, argv[2], &c)) { napi_throw_error(env, NULL, "evalPass: malformed camera"); return NULL; }
    cp = &c;
  }
  gs_state s;
  pthread_mutex_lock(&H->mu);
  int rc = gs_get_state(H->h, &s);
  pthread_mutex_unlock(&H->mu);
  if (rc != GS_OK) return throw_gs(env, H, rc);
  uint32_t* st = NULL;
  int32_t* cg = NULL;
  napi_value sa = new_typed(env, napi_uint32_array, 4, 4, (void**)&st);
  napi_value ca = new_typed(env, napi_int32_array, (size_t)(s.ncams + 1) * 8, 4, (void**)&cg);
  if (!sa || !ca) return throw_gs(env, H, GS_E_NOMEM);
  pthread_mutex_lock(&H->mu);
  rc = gs_eval_pass(H->h, ci, cp, st, cg);
  pthread_mutex_unlock(&H->mu);
  if (rc != GS_OK) return throw_gs(env, H, rc);
  napi_value o;
  NAPI_OK(env, napi_create_object(env, &o));
  napi_set_named_property(env, o, "stats", sa);
  napi_set_named_property(env, o, "camGrad", ca);
  return o;
}

/* readCamGrads(h, reset) -> Int32Array((ncams+1)*8): the drain of _applyCamGrads (trainer.js:476-491) */
static napi_value ReadCamGrads(napi_env env, napi_callback_info info) {
  size_t argc = 2;
  napi_value argv[2];
  NAPI_OK(env, napi_get_cb_info(env, info, &argc, argv, NULL, NULL));
  Handle* H = arg_handle(env, argv[0]);
  if (!H) return NULL;
  bool reset = false;
  if (argc >= 2) napi_get_value_bool(env, argv[1], &reset);
  gs_state s;
  pthread_mutex_lock(&H->mu);
  int rc = gs_get_state(H->h, &s);
  pthread_mutex_unlock(&H->mu);
  if (rc != GS_OK) return throw_gs(env, H, rc);
  int32_t* cg = NULL;
  napi_value ca = new_typed(env, napi_int32_array, (size_t)(s.ncams + 1) * 8, 4, (void**)&cg);
  if (!ca) return throw_gs(env, H, GS_E_NOMEM);
  pthread_mutex_lock(&H->mu);
  rc = gs_read_cam_grads(H->h, cg, reset ? 1 : 0);
  pthread_mutex_unlock(&H->mu);
  return rc == GS_OK ? ca : throw_gs(env, H, rc);
}

/* ---- refine(rng) on the JavaScript thread -------------------------------- */
typedef struct {
  napi_env env;
  napi_value fn;
  int failed;
} RngCtx;

/* gs_rng_fn: one rng() call of the JavaScript function; a throw or a
 * non-number ends the draws with 0 and is reported after gs_refine returns */
static double call_rng(void* ctx) {
  RngCtx* r = (RngCtx*)ctx;
  if (r->failed) return 0.0;
  napi_value undef, res;
  double x = 0.0;
  napi_get_undefined(r->env, &undef);
  if (napi_call_function(r->env, undef, r->fn, 0, NULL, &res) != napi_ok ||
      napi_get_value_double(r->env, res, &x) != napi_ok) {
    r->failed = 1;
    return 0.0;
  }
  return x;
}

/* refine(h, rng) -> {moved, grown, n, maxTile, overflow} or {moved: 0, grown: 0, n}
 * (the donors < 16 early return, trainer.js:695); rng undefined or null: the
 * library's own generator draws, with no call into JavaScript per draw */
static napi_value Refine(napi_env env, napi_callback_info info) {
  size_t argc = 2;
  napi_value argv[2];
  NAPI_OK(env, napi_get_cb_info(env, info, &argc, argv, NULL, NULL));
  Handle* H = arg_handle(env, argv[0]);
  if (!H) return NULL;
  napi_valuetype t = napi_undefined;
  if (argc > 1) NAPI_OK(env, napi_typeof(env, argv[1], &t));
  const bool own = t == napi_undefined || t == napi_null;  // the library's generator (no JS call per draw)
  if (!own && t != napi_function) {
    napi_throw_error(env, NULL, "refine: rng must be a function or undefined");
    return NULL;
  }
  RngCtx ctx = {env, own ? NULL : argv[1], 0};
  gs_refine_result r;
  pthread_mutex_lock(&H->mu);
  const int rc = own ? gs_refine(H->h, NULL, NULL, &r) : gs_refine(H->h, call_rng, &ctx, &r);
  pthread_mutex_unlock(&H->mu);
  bool pending = false;
  napi_is_exception_pending(env, &pending);
  if (pending) return NULL;
  if (ctx.failed) { napi_throw_error(env, NULL, "refine: rng() did not return a number"); return NULL; }
  if (rc != GS_OK) return throw_gs(env, H, rc);
  napi_value o;
  NAPI_OK(env, napi_create_object(env, &o));
  napi_set_named_property(env, o, "moved", make_u32(env, r.early ? 0u : r.moved));
  napi_set_named_property(env, o, "grown", make_u32(env, r.early ? 0u : r.grown));
  napi_set_named_property(env, o, "n", make_u32(env, r.n));
  if (!r.early) {
    napi_set_named_property(env, o, "maxTile", make_u32(env, r.maxTile));
    napi_set_named_property(env, o, "overflow", make_u32(env, r.overflow));
  }
  return o;
}

/* exportPly(h, bake, f, camPositions Float64Array(3*ncams)) -> Uint8Array:
 * bakeOpacityCompensation + gaussiansToPly (ply.js:17-99) on the device */
static napi_value ExportPly(napi_env env, napi_callback_info info) {
  size_t argc = 4;
  napi_value argv[4];
  NAPI_OK(env, napi_get_cb_info(env, info, &argc, argv, NULL, NULL));
  Handle* H = arg_handle(env, argv[0]);
  if (!H) return NULL;
  bool bake = false;
  double f = 0.0;
  NAPI_OK(env, napi_get_value_bool(env, argv[1], &bake));
  NAPI_OK(env, napi_get_value_double(env, argv[2], &f));
  int bad = 0;
  size_t nc = 0;
  const double* cp = (const double*)typed(env, argv[3], napi_float64_array, &nc, &bad);
  if (bad) { napi_throw_error(env, NULL, "exportPly: camera positions must be a Float64Array"); return NULL; }
  uint64_t size = 0;
  pthread_mutex_lock(&H->mu);
  int rc = gs_export_ply(H->h, bake ? 1 : 0, f, cp, (uint32_t)(nc / 3), NULL, 0, &size);
  pthread_mutex_unlock(&H->mu);
  if (rc != GS_OK) return throw_gs(env, H, rc);
  uint8_t* out = NULL;
  napi_value arr = new_typed(env, napi_uint8_array, (size_t)size, 1, (void**)&out);
  if (!arr) return throw_gs(env, H, GS_E_NOMEM);
  pthread_mutex_lock(&H->mu);
  rc = gs_export_ply(H->h, bake ? 1 : 0, f, cp, (uint32_t)(nc / 3), out, size, &size);
  pthread_mutex_unlock(&H->mu);
  return rc == GS_OK ? arr : throw_gs(env, H, rc);
}

static napi_value AbiVersion(napi_env env, napi_callback_info info) {
  (void)info;
  return make_u32(env, (uint32_t)gs_abi_version());
}

/* ---- module ------------------------------------------------------------- */
NAPI_MODULE_INIT() {
  static const struct {
    const char* name;
    napi_callback fn;
  } fns[] = {
      {"create", Create},         {"setup", Setup},
      {"state", State},           {"setIter", SetIter},
      {"setHorizon", SetHorizon}, {"setGrowLimit", SetGrowLimit},
      {"setCamera", SetCamera},   {"step", Step},
      {"stepBatch", StepBatch},   {"readStats", ReadStats},
      {"sync", Sync},             {"readGaussians", ReadGaussians},
      {"renderView", RenderView}, {"evalPass", EvalPass},
      {"readCamGrads", ReadCamGrads}, {"refine", Refine},
      {"exportPly", ExportPly},   {"abiVersion", AbiVersion},
      {"resetMoments", ResetMoments},
  };
  for (size_t k = 0; k < sizeof fns / sizeof fns[0]; ++k) {
    napi_value f;
    if (napi_create_function(env, fns[k].name, (size_t)-1, fns[k].fn, NULL, &f) != napi_ok) return NULL;
    if (napi_set_named_property(env, exports, fns[k].name, f) != napi_ok) return NULL;
  }
  return exports;
}
