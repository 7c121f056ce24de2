// oracle_capi.cpp -- C entry points over gs_oracle.hpp for ctypes.
//
// TEST INFRASTRUCTURE ONLY (the parity checker and the CPU baseline); the
// product never links it.  Layouts follow the reference: params stride 16
// (shaders.js:14-16), SH channel-major 3K per splat (shaders.js:17-22),
// proj stride 16 (shaders.js:23-25), gradP stride 16 i32 (shaders.js:26-28).
#include <algorithm>
#include <cstdio>
#include <memory>

#include <omp.h>

#include "gs_oracle.hpp"

using namespace gso;

extern "C" {

// Host threads the parallel loops use (the CPU baseline is timed at one
// thread and at all of them); returns the count now in effect.
int oracle_set_threads(int n) {
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
}

// Plain-C mirrors of gso::Opts / gso::Cam (field order is the ABI).
struct OOpts {
  float eCut, aMin, radClamp, anisoReg;
  int32_t shDeg, tile;
  uint64_t entriesCap;
  int32_t tileCull;
};
struct OCam {
  float R[9];
  float t[3];
  float f, cx, cy;
  int32_t w, h;
  float gain, bias;
  uint32_t offset, camIdx, ncams;
  float activeSh;
  int32_t train;
};
struct OAdam {
  float lr[16];
  float b1, b2, eps, bc1, bc2, minLS, maxLS, maxLogit, reg, shLr;
};

static Opts toOpts(const OOpts* o) {
  Opts r;
  r.eCut = o->eCut; r.aMin = o->aMin; r.radClamp = o->radClamp; r.anisoReg = o->anisoReg;
  r.shDeg = o->shDeg; r.tile = o->tile; r.entriesCap = o->entriesCap; r.tileCull = o->tileCull;
  return r;
}
static Cam toCam(const OCam* c) {
  Cam r;
  for (int k = 0; k < 9; ++k) r.R[k] = c->R[k];
  for (int k = 0; k < 3; ++k) { r.t[k] = c->t[k]; r.bg[k] = 0.0f; }
  r.nearz = 0.05f;
  r.f = c->f; r.cx = c->cx; r.cy = c->cy; r.gain = c->gain;
  r.W = c->w; r.H = c->h;
  r.offset = c->offset; r.train = c->train; r.camIdx = c->camIdx; r.ncams = c->ncams;
  r.bias = c->bias; r.activeSh = c->activeSh;
  return r;
}
static AdamHP toAdam(const OAdam* a) {
  AdamHP h;
  for (int k = 0; k < 16; ++k) h.lr[k] = a->lr[k];
  h.b1 = a->b1; h.b2 = a->b2; h.eps = a->eps; h.bc1 = a->bc1; h.bc2 = a->bc2;
  h.minLS = a->minLS; h.maxLS = a->maxLS; h.maxLogit = a->maxLogit; h.reg = a->reg; h.shLr = a->shLr;
  return h;
}

int oracle_abi_version() { return 1; }

void oracle_adam_bias(double t, float* bc1, float* bc2) { adamBiasCorrection(t, *bc1, *bc2); }
float oracle_exp_f32(float x) { return exp_f(x); }
float oracle_log_f32(float x) { return log_f(x); }
double oracle_sin_f64(double x) { return sin_d(x); }
float oracle_dither(uint32_t pi) { return ditherOf(pi); }

// ---- pass 1: project (shaders.js:228-315) ----
void oracle_project_f32(const OOpts* oo, const OCam* oc, const float* params, const float* sh, uint32_t n,
                        float* proj) {
  const Opts o = toOpts(oo);
  const Cam c = toCam(oc);
  const int K = shRestCoefs(o.shDeg);
#pragma omp parallel for schedule(static)
  for (long i = 0; i < (long)n; ++i)
    projectOne<float>(o, c, params + (size_t)i * STRIDE, sh ? sh + (size_t)i * 3 * K : nullptr, K,
                      proj + (size_t)i * STRIDE);
}
void oracle_project_f64(const OOpts* oo, const OCam* oc, const double* params, const double* sh, uint32_t n,
                        double* proj) {
  const Opts o = toOpts(oo);
  const Cam c = toCam(oc);
  const int K = shRestCoefs(o.shDeg);
#pragma omp parallel for schedule(static)
  for (long i = 0; i < (long)n; ++i)
    projectOne<double>(o, c, params + (size_t)i * STRIDE, sh ? sh + (size_t)i * 3 * K : nullptr, K,
                       proj + (size_t)i * STRIDE);
}

// Per-splat values the rasteriser reads, derived from proj exactly as the
// render pass does (w = opa*comp, -cnorm/2 with cnorm = 1/(1+lambda_max),
// 1 - opa), in the CUDA library's record layout, plus tile
// bounds packed {x0 | y0<<16, x1 | y1<<16} ({~0, 0} when culled).
void oracle_records_f32(const OOpts* oo, const OCam* oc, const float* proj, uint32_t n, float* rec12,
                        uint32_t* rect2) {
  const Opts o = toOpts(oo);
  const Cam c = toCam(oc);
  for (uint32_t i = 0; i < n; ++i) {
    const float* pr = proj + (size_t)i * STRIDE;
    float* r = rec12 + (size_t)i * 12;
    if (!(pr[11] > 0.0f)) {
      for (int k = 0; k < 12; ++k) r[k] = 0.0f;
      rect2[2 * i] = 0xFFFFFFFFu; rect2[2 * i + 1] = 0u;
      continue;
    }
    const Splat2D<float> s = splat2D<float>(pr);
    const float v[12] = {s.mx, s.my, 0.5f * s.cA, s.cB, 0.5f * s.cC, s.w, s.r, s.g, s.b, s.opa, -0.5f * s.cnorm,
                         1.0f - s.opa};
    for (int k = 0; k < 12; ++k) r[k] = v[k];
    const TileRect t = tileRect<float>(c, o.tile, pr[0], pr[1], pr[15]);
    rect2[2 * i] = (uint32_t)t.x0 | ((uint32_t)t.y0 << 16);
    rect2[2 * i + 1] = (uint32_t)t.x1 | ((uint32_t)t.y1 << 16);
  }
}

// ---- passes 2-4: binning (shaders.js:303-500) ----
// Writes start[numTiles+1], ids/keys (up to cap entries), per-tile raw
// counts and drop flags.  Returns the number of kept entries.
uint64_t oracle_bin_f32(const OOpts* oo, const OCam* oc, const float* proj, uint32_t n, uint32_t* start,
                        uint32_t* ids, uint32_t* keys, uint64_t cap, uint32_t* cnt, uint8_t* dropped,
                        uint32_t* overflowTiles) {
  const Opts o = toOpts(oo);
  const Cam c = toCam(oc);
  Bins b = binTiles<float>(o, c, proj, n);
  std::copy(b.start.begin(), b.start.end(), start);
  const size_t E = std::min<size_t>(b.ids.size(), cap);
  std::copy(b.ids.begin(), b.ids.begin() + E, ids);
  std::copy(b.keys.begin(), b.keys.begin() + E, keys);
  if (cnt) std::copy(b.cnt.begin(), b.cnt.end(), cnt);
  if (dropped) std::copy(b.dropped.begin(), b.dropped.end(), dropped);
  if (overflowTiles) *overflowTiles = b.overflowTiles;
  return b.ids.size();
}

static Bins binsFromArrays(const Opts& o, const Cam& c, const uint32_t* start, const uint32_t* ids) {
  Bins b;
  b.numTiles = tilesX(c, o.tile) * tilesY(c, o.tile);
  b.start.assign(start, start + b.numTiles + 1);
  b.ids.assign(ids, ids + b.start[b.numTiles]);
  return b;
}

// ---- render (shaders.js:544-700) on a given binning ----
void oracle_render_f32(const OOpts* oo, const OCam* oc, const float* proj, const uint32_t* start,
                       const uint32_t* ids, const uint32_t* targets, float* outImg, float* finalT,
                       uint32_t* endIdx, int32_t* gradP, uint32_t* stats, int32_t* gradCam, uint64_t* pairs,
                       int train, int variant) {
  const Opts o = toOpts(oo);
  const Cam c = toCam(oc);
  Bins b = binsFromArrays(o, c, start, ids);
  std::vector<PixelState> px((size_t)c.W * c.H);
  AccFixed acc{gradP, stats, gradCam};
  renderView<float, AccFixed>(o, c, proj, b, targets, outImg, px.data(), acc, train != 0, variant, pairs);
  for (size_t p = 0; p < px.size(); ++p) {
    if (finalT) finalT[p] = px[p].T;
    if (endIdx) endIdx[p] = px[p].end;
  }
}

// Render of every tileStride-th tile only (a bounded sample of a view for
// the CPU baseline's timing; tile work is independent per tile).
void oracle_render_sample_f32(const OOpts* oo, const OCam* oc, const float* proj, const uint32_t* start,
                              const uint32_t* ids, const uint32_t* targets, int32_t* gradP, uint32_t* stats,
                              int32_t* gradCam, uint64_t* pairs, int train, int tileStride) {
  const Opts o = toOpts(oo);
  const Cam c = toCam(oc);
  Bins b = binsFromArrays(o, c, start, ids);
  std::vector<PixelState> px((size_t)c.W * c.H);
  AccFixed acc{gradP, stats, gradCam};
  renderView<float, AccFixed>(o, c, proj, b, targets, nullptr, px.data(), acc, train != 0, 0, pairs, tileStride);
}

// ---- chain (shaders.js:704-949): consumes and zeroes gradP ----
void oracle_chain_f32(const OOpts* oo, const OCam* oc, const float* params, const float* proj, const float* sh,
                      uint32_t n, int32_t* gradP, float* gradF, float* shGrad, int32_t* gradCam) {
  const Opts o = toOpts(oo);
  const Cam c = toCam(oc);
  const int K = shRestCoefs(o.shDeg);
#pragma omp parallel for schedule(static)
  for (long i = 0; i < (long)n; ++i) {
    float gp[10];
    int32_t* G = gradP + (size_t)i * STRIDE;
    for (int k = 0; k < 10; ++k) {
      const float scale = (k >= 2 && k <= 4) ? FIXEDC : FIXED;
      gp[k] = (float)G[k] / scale;
      G[k] = 0;
    }
    float shDummy[1];
    auto camAdd = [&](uint32_t idx, float v) {
      int32_t q = fixq(v, FIXCAM);
#pragma omp atomic
      gradCam[idx] += q;
    };
    chainOne<float>(o, c, params + (size_t)i * STRIDE, proj + (size_t)i * STRIDE,
                    K ? sh + (size_t)i * 3 * K : nullptr, K, gp, gradF + (size_t)i * STRIDE,
                    K ? shGrad + (size_t)i * 3 * K : shDummy, camAdd);
  }
}

// ---- Adam + SH-Adam (shaders.js:952-1036) over n splats ----
void oracle_adam_f32(const OAdam* oa, uint32_t n, int K, float* params, const float* gradF, float* m, float* v,
                     float* sh, const float* shGrad, float* shM, float* shV) {
  const AdamHP h = toAdam(oa);
#pragma omp parallel for schedule(static)
  for (long i = 0; i < (long)n; ++i) {
    for (int s = 0; s < STRIDE; ++s) {
      const size_t j = (size_t)i * STRIDE + s;
      adamParam(h, s, params[j], gradF[j], m[j], v[j]);
    }
    for (int k = 0; k < 3 * K; ++k) {
      const size_t j = (size_t)i * 3 * K + k;
      adamSH(h, sh[j], shGrad[j], shM[j], shV[j]);
    }
  }
}

// ---- a whole step over V views: per view project -> bin -> render ->
// chain, gradients summed over views in view order, then (optionally) Adam.
// With V = 1 this is stepOnce (trainer.js:398-458).  gradF/shGrad receive
// the summed gradients when non-null.  Returns 0, or 1 if any view's entry
// count exceeded entriesCap (the kept entries are still processed).
int oracle_step_f32(const OOpts* oo, const OCam* cams, int V, const OAdam* oa, uint32_t n, float* params,
                    float* sh, const uint32_t* targets, float* m, float* v, float* shM, float* shV,
                    uint32_t* stats, int32_t* gradCam, float* gradF, float* shGrad, int doAdam, int variant,
                    uint64_t* pairs, float* outImg0) {
  const Opts o = toOpts(oo);
  const int K = shRestCoefs(o.shDeg);
  std::vector<float> gF((size_t)n * STRIDE, 0.0f), sG((size_t)n * 3 * K, 0.0f);
  std::vector<float> proj((size_t)n * STRIDE), gFv((size_t)n * STRIDE), sGv((size_t)n * 3 * K);
  std::vector<int32_t> gP((size_t)n * STRIDE, 0);
  for (int vi = 0; vi < V; ++vi) {
    const Cam c = toCam(&cams[vi]);
    oracle_project_f32(oo, &cams[vi], params, K ? sh : nullptr, n, proj.data());
    Bins b = binTiles<float>(o, c, proj.data(), n);
    if (stats) stats[3] += b.overflowTiles;
    std::vector<PixelState> px((size_t)c.W * c.H);
    std::vector<float> img;
    if (vi == 0 && outImg0) img.assign((size_t)c.W * c.H * 4, 0.0f);
    AccFixed acc{gP.data(), stats, gradCam};
    renderView<float, AccFixed>(o, c, proj.data(), b, targets, img.empty() ? nullptr : img.data(), px.data(), acc,
                                true, variant, pairs);
    if (!img.empty()) std::copy(img.begin(), img.end(), outImg0);
    oracle_chain_f32(oo, &cams[vi], params, proj.data(), K ? sh : nullptr, n, gP.data(), gFv.data(),
                     K ? sGv.data() : nullptr, gradCam);
    for (size_t j = 0; j < gF.size(); ++j) gF[j] = gF[j] + gFv[j];
    for (size_t j = 0; j < sG.size(); ++j) sG[j] = sG[j] + sGv[j];
  }
  if (gradF) std::copy(gF.begin(), gF.end(), gradF);
  if (shGrad && K) std::copy(sG.begin(), sG.end(), shGrad);
  if (doAdam) oracle_adam_f32(oa, n, K, params, gF.data(), m, v, sh, sG.data(), shM, shV);
  return 0;
}

// ---- FP64 host evaluation: loss (Charbonnier sum, squared error, valid
// px) and unquantised gradients of one view.  gradF/shGrad may be null
// (loss only, for finite differences). ----
void oracle_eval_f64(const OOpts* oo, const OCam* oc, const double* params, const double* sh, uint32_t n,
                     const uint32_t* targets, double* loss3, double* gradF, double* shGrad, float* outImg,
                     int quantise) {
  const Opts o = toOpts(oo);
  const Cam c = toCam(oc);
  const int K = shRestCoefs(o.shDeg);
  std::vector<double> proj((size_t)n * STRIDE);
  oracle_project_f64(oo, oc, params, sh, n, proj.data());
  Bins b = binTiles<double>(o, c, proj.data(), n);
  std::vector<double> gP((size_t)n * STRIDE, 0.0), gCam((size_t)(c.ncams + 1) * 8, 0.0);
  loss3[0] = loss3[1] = loss3[2] = 0.0;
  AccF64 acc{gP.data(), loss3, gCam.data(), quantise != 0};
  renderView<double, AccF64>(o, c, proj.data(), b, targets, outImg, nullptr, acc, true, 0, nullptr);
  if (!gradF) return;
#pragma omp parallel for schedule(static)
  for (long i = 0; i < (long)n; ++i) {
    double gp[10];
    for (int k = 0; k < 10; ++k) gp[k] = gP[(size_t)i * STRIDE + k];
    double shDummy[1];
    auto camAdd = [](uint32_t, double) {};
    chainOne<double>(o, c, params + (size_t)i * STRIDE, proj.data() + (size_t)i * STRIDE,
                     K ? sh + (size_t)i * 3 * K : nullptr, K, gp, gradF + (size_t)i * STRIDE,
                     (K && shGrad) ? shGrad + (size_t)i * 3 * K : shDummy, camAdd);
  }
}

// ---- FP64 central differences local to one splat's tiles ----
// gradcheck.js:307-329 differentiates the whole-image loss.  A splat's
// parameters change only the pixels of the tiles whose lists hold it, so in
// L(+h) - L(-h) the loss over every other tile cancels exactly; summing the
// union of the splat's tiles at p, p + h and p - h gives the same central
// difference at a cost that does not grow with the image.  The perturbed
// splat leaves each list and re-enters it where binTiles would place it
// (rectangle, tile cull, ascending (depth bits, id)).  out: nids rows of
// 14 parameter slots then 3K SH coefficients, column k differenced with step
// hcol[k]; a splat whose union exceeds maxTiles gets NaN rows.  Returns -1
// when the entry budget drops a tile.
namespace {
struct LocalTiles {
  const Opts& o;
  const Cam& c;
  const double* proj;
  const Bins& b;
  const uint32_t* targets;
  // loss over `tiles` with splat s at projection prS (prS[11] <= 0: culled)
  double loss(const std::vector<int>& tiles, uint32_t s, const double* prS, std::vector<uint32_t>& list) const {
    const int tile = o.tile, tx = tilesX(c, tile);
    const bool vis = prS[11] > 0.0;
    TileRect r{0, -1, 0, -1};
    bool test = false;
    CullParams cp{INFINITY, 0.0f, 0.0f};
    float cmx = 0.0f, cmy = 0.0f;
    if (vis) {
      r = tileRect<double>(c, tile, prS[0], prS[1], prS[15]);
      test = o.tileCull && !(r.x0 == r.x1 && r.y0 == r.y1);
      if (test) {
        const Splat2D<double> s2 = splat2D<double>(prS);
        cmx = (float)s2.mx; cmy = (float)s2.my;
        cp = cullParams(cmx, cmy, (float)(0.5 * s2.cA), (float)s2.cB, (float)(0.5 * s2.cC), (float)s2.w, o.aMin,
                        o.eCut, r.x0, r.x1, r.y0, r.y1, tile);
      }
    }
    const uint32_t key = fbits((float)prS[2]);
    double lossSum[3] = {0.0, 0.0, 0.0};
    std::vector<double> camDummy((size_t)(c.ncams + 1) * 8, 0.0);
    AccF64 acc{nullptr, lossSum, camDummy.data(), false};
    for (int t : tiles) {
      const int x = t % tx, y = t / tx;
      const bool member = vis && x >= r.x0 && x <= r.x1 && y >= r.y0 && y <= r.y1 &&
                          (!test || tileLive(cp, cmx, cmy, x, y, tile, c.W, c.H));
      list.clear();
      bool placed = !member;
      for (uint32_t k = b.start[t]; k < b.start[t + 1]; ++k) {
        const uint32_t id = b.ids[k];
        if (id == s) continue;
        if (!placed && (key < b.keys[k] || (key == b.keys[k] && s < id))) { list.push_back(s); placed = true; }
        list.push_back(id);
      }
      if (!placed) list.push_back(s);
      const int ox = x * tile, oy = y * tile;
      for (int ly = 0; ly < tile; ++ly)
        for (int lx = 0; lx < tile; ++lx) {
          const int gx = ox + lx, gy = oy + ly;
          if (gx >= c.W || gy >= c.H) continue;
          const double px = gx + 0.5, py = gy + 0.5;
          double Tr = 1.0, C[3] = {0.0, 0.0, 0.0};
          for (uint32_t id : list) {  // the forward of renderView, in double
            const Splat2D<double> sp = splat2D<double>(id == s ? prS : proj + (size_t)id * STRIDE);
            const double dx = px - sp.mx, dy = py - sp.my;
            const double e = pairExponent(sp, dx, dy);
            if (e > (double)o.eCut) continue;
            const double alpha = std::fmin(0.99, sp.w * Math<double>::exp(-e));
            if (alpha < (double)o.aMin) continue;
            const double ta = Tr * alpha;
            C[0] = std::fma(ta, sp.r, C[0]);
            C[1] = std::fma(ta, sp.g, C[1]);
            C[2] = std::fma(ta, sp.b, C[2]);
            Tr = Tr * (1.0 - alpha);
            if (Tr < 1e-4) break;
          }
          double Cf[3], gC[3];
          for (int j = 0; j < 3; ++j) Cf[j] = C[j] + Tr * (double)c.bg[j];
          lossPixel<double>(c, targets, (uint32_t)(gy * c.W + gx), Cf, gC, acc);
        }
    }
    return lossSum[0];
  }
};
}  // namespace

int oracle_fd_local_f64(const OOpts* oo, const OCam* oc, const double* params, const double* sh, uint32_t n,
                        const uint32_t* targets, const uint32_t* ids, uint32_t nids, const double* hcol,
                        uint32_t maxTiles, double* out) {
  const Opts o = toOpts(oo);
  const Cam c = toCam(oc);
  const int K = shRestCoefs(o.shDeg);
  const int np = 14 + 3 * K;
  std::vector<double> proj((size_t)n * STRIDE);
  oracle_project_f64(oo, oc, params, sh, n, proj.data());
  const Bins b = binTiles<double>(o, c, proj.data(), n);
  if (b.overflowTiles) return -1;
  const LocalTiles lt{o, c, proj.data(), b, targets};
  const int tx = tilesX(c, o.tile);
#pragma omp parallel for schedule(dynamic, 1)
  for (long q = 0; q < (long)nids; ++q) {
    const uint32_t s = ids[q];
    double P[STRIDE], prp[STRIDE], prm[STRIDE];
    std::vector<double> S((size_t)std::max(1, 3 * K), 0.0);
    std::memcpy(P, params + (size_t)s * STRIDE, sizeof(P));
    if (K) std::memcpy(S.data(), sh + (size_t)s * 3 * K, sizeof(double) * 3 * K);
    std::vector<int> tiles;
    std::vector<uint32_t> list;
    auto addRect = [&](const double* pr) {
      if (!(pr[11] > 0.0)) return;
      const TileRect r = tileRect<double>(c, o.tile, pr[0], pr[1], pr[15]);
      for (int y = r.y0; y <= r.y1; ++y)
        for (int x = r.x0; x <= r.x1; ++x) tiles.push_back(y * tx + x);
    };
    for (int k = 0; k < np; ++k) {
      double* v = k < 14 ? &P[k] : &S[(size_t)(k - 14)];
      const double v0 = *v, h = hcol[k];
      *v = v0 + h;
      projectOne<double>(o, c, P, K ? S.data() : nullptr, K, prp);
      *v = v0 - h;
      projectOne<double>(o, c, P, K ? S.data() : nullptr, K, prm);
      *v = v0;
      tiles.clear();
      addRect(proj.data() + (size_t)s * STRIDE);
      addRect(prp);
      addRect(prm);
      std::sort(tiles.begin(), tiles.end());
      tiles.erase(std::unique(tiles.begin(), tiles.end()), tiles.end());
      double& o_ = out[(size_t)q * np + k];
      if (tiles.size() > maxTiles) { o_ = NAN; continue; }
      o_ = (lt.loss(tiles, s, prp, list) - lt.loss(tiles, s, prm, list)) / (2.0 * h);
    }
  }
  return 0;
}

// ---- refine: MCMC-lite relocation + growth (trainer.js:666-794) ----
// params/m/v are cap*16 f32, sh/shM/shV cap*3K f32.  rng() returns doubles
// in [0,1) in the order the reference draws them.  JS arithmetic is double;
// Float32Array stores round to f32, which the casts below reproduce.
// donorSampling 1 (no reference counterpart): a clone's donor is the first
// whose cumulative sigmoid(opacity) over the donor list exceeds rng() * total,
// the same single draw the uniform pick makes.
typedef double (*oracle_rng_fn)(void*);
struct ORefineOut { uint32_t moved, grown, n; int32_t early; };

void oracle_refine(uint32_t n, uint32_t cap, uint32_t growLimit, double iter, double growUntil, double growRate,
                   int K, float* params, float* m, float* v, float* sh, float* shM, float* shV, oracle_rng_fn rng,
                   void* ctx, ORefineOut* out, int donorSampling) {
  auto sig = [](double x) { return 1.0 / (1.0 + std::exp(-x)); };
  std::vector<uint32_t> dead, donors;
  for (uint32_t i = 0; i < n; ++i) {
    const double o = sig((double)params[(size_t)i * 16 + 13]);
    if (o < 0.02) dead.push_back(i);
    else if (o > 0.4) donors.push_back(i);
  }
  out->moved = out->grown = 0; out->n = n; out->early = 0;
  if (donors.size() < 16) { out->early = 1; return; }
  const size_t moveCap = (size_t)std::ceil((double)n * 0.05);
  if (dead.size() > moveCap) dead.resize(moveCap);
  auto mls = [&](uint32_t i) {
    const float* p = params + (size_t)i * 16;
    return ((double)p[3] + (double)p[4] + (double)p[5]) / 3.0;
  };
  std::vector<double> cdf;
  if (donorSampling == 1) {
    double acc = 0.0;
    for (uint32_t i : donors) {
      acc += sig((double)params[(size_t)i * 16 + 13]);
      cdf.push_back(acc);
    }
  }
  std::vector<uint32_t> big(donors);
  std::stable_sort(big.begin(), big.end(), [&](uint32_t a, uint32_t b) { return mls(b) - mls(a) < 0; });
  big.resize(std::min(big.size(), std::max<size_t>(16, donors.size() >> 2)));
  const int shr = 3 * K;
  auto gauss = [&]() {
    const double u = std::max(1e-9, rng(ctx)), w = rng(ctx);
    return std::sqrt(-2.0 * std::log(u)) * std::cos(2.0 * M_PI * w);
  };
  auto spawnAt = [&](size_t bi, bool allowSplit) {
    bool doSplit = false;
    if (allowSplit && big.size() > 16) doSplit = rng(ctx) < 0.7;
    uint32_t don;
    if (doSplit) {
      const size_t di = (size_t)(int32_t)(rng(ctx) * (double)big.size());
      don = big[di];
      big[di] = big.back();
      big.pop_back();
    } else if (cdf.empty()) {
      don = donors[(size_t)(int32_t)(rng(ctx) * (double)donors.size())];
    } else {
      const double target = rng(ctx) * cdf.back();
      size_t k = 0;
      while (k + 1 < cdf.size() && !(cdf[k] > target)) ++k;
      don = donors[k];
    }
    const size_t bd = (size_t)don * 16;
    const double s = std::exp(mls(don));
    for (int k = 0; k < 3; ++k) {
      const double base = (double)params[bd + k];
      params[bi + k] = (float)(base + gauss() * s * 0.7);
    }
    for (int k = 3; k <= 12; ++k) params[bi + k] = params[bd + k];
    if (doSplit) {
      const double shrink = std::log(1.0 / 1.6);
      for (int k = 3; k <= 5; ++k) {
        params[bi + k] = (float)((double)params[bi + k] + shrink);
        params[bd + k] = (float)((double)params[bd + k] + shrink);
      }
      params[bi + 13] = params[bd + 13];
      for (int k = 0; k < 16; ++k) { m[bd + k] = 0.0f; v[bd + k] = 0.0f; }
    } else {
      for (int k = 3; k <= 5; ++k) params[bi + k] = (float)((double)params[bi + k] + std::log(0.85));
      params[bi + 13] = (float)std::log(0.25 / 0.75);
    }
    params[bi + 14] = 0.0f; params[bi + 15] = 0.0f;
    for (int k = 0; k < 16; ++k) { m[bi + k] = 0.0f; v[bi + k] = 0.0f; }
    if (shr) {
      const size_t so = (bi / 16) * shr, sd = (size_t)don * shr;
      for (int k = 0; k < shr; ++k) {
        sh[so + k] = sh[sd + k];
        shM[so + k] = 0.0f; shV[so + k] = 0.0f;
        if (doSplit) { shM[sd + k] = 0.0f; shV[sd + k] = 0.0f; }
      }
    }
  };
  for (uint32_t i : dead) spawnAt((size_t)i * 16, false);
  const uint32_t limit = std::min(cap, growLimit ? growLimit : cap);
  uint32_t grown = 0;
  if (iter < growUntil) {
    const double want = std::ceil((double)n * growRate);
    const double room = (double)limit - (double)n;
    grown = (uint32_t)std::max(0.0, std::min(want, room));
  }
  for (uint32_t k = 0; k < grown; ++k) spawnAt((size_t)(n + k) * 16, true);
  out->moved = (uint32_t)dead.size();
  out->grown = grown;
  out->n = n + grown;
}

}  // extern "C"
