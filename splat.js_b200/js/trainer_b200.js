// trainer_b200.js -- the GSTrainer class of splat.js (src/gs/trainer.js) over
// the B200 library, for Node: createTrainer(opts) / GSTrainer.create(opts)
// (src/index.js:56-58, trainer.js:13-16) return this class when the addon
// (native/gs_b200_napi.c, built by native/binding.gyp) loads.
//
// Kept on the JavaScript side, as in the reference: the rand() camera pick of
// stepOnce with the holdout / excluded skip (trainer.js:400-406), the
// camera-pose Adam of _applyCamGrads (trainer.js:476-537) and the test-time
// pose refinement of evalCamPsnrRefined (trainer.js:584-612).  Everything
// else runs in libsplat_b200.so.  Buffers keep the reference's layouts
// (params stride 16 f32; SH channel-major 3K f32 per splat), so
// readGaussians() feeds gaussiansToPly unchanged.
import { createRequire } from 'node:module';

const require = createRequire(import.meta.url);
const addon = require('../native/build/Release/gs_b200.node');

const STRIDE = 16;

// src/sfm/geometry.js:150-160 and :108-114
function rodrigues(w) {
  const th = Math.hypot(w[0], w[1], w[2]);
  if (th < 1e-12) return [1, 0, 0, 0, 1, 0, 0, 0, 1];
  const k = [w[0] / th, w[1] / th, w[2] / th];
  const c = Math.cos(th), s = Math.sin(th), v = 1 - c;
  return [c + k[0] * k[0] * v, k[0] * k[1] * v - k[2] * s, k[0] * k[2] * v + k[1] * s,
    k[1] * k[0] * v + k[2] * s, c + k[1] * k[1] * v, k[1] * k[2] * v - k[0] * s,
    k[2] * k[0] * v - k[1] * s, k[2] * k[1] * v + k[0] * s, c + k[2] * k[2] * v];
}
function m3mul(A, B) {
  const r = new Array(9);
  for (let i = 0; i < 3; i++) {
    for (let j = 0; j < 3; j++) r[i * 3 + j] = A[i * 3] * B[j] + A[i * 3 + 1] * B[3 + j] + A[i * 3 + 2] * B[6 + j];
  }
  return r;
}

export class GSTrainer {
  static async create(opts = {}) { return new GSTrainer(opts); }

  constructor(opts = {}) {
    this.opts = opts;
    this.h = addon.create(opts);
    const st = addon.state(this.h);
    this.shDeg = st.shDeg;
    this.shK = st.shK;
    this.stride = STRIDE;
    this.tileGrad = opts.tileGrad ?? true;
    this.holdout = -1;
    this.excluded = new Set();
    this.lastCam = 0;
    this.lastRefine = 0;
    this.growLimit = 0;
    this.entryOverflowTiles = 0;
    this.rand = () => Math.random();
    this.camMeta = [];
    // device.queue.onSubmittedWorkDone() (session.js:520, 542)
    this.device = { queue: { onSubmittedWorkDone: () => addon.sync(this.h) } };
  }

  // ---- fields the reference's callers read and write ----
  get iter() { return addon.state(this.h).iter; }
  set iter(v) { addon.setIter(this.h, v); }
  get n() { return addon.state(this.h).n; }
  get cap() { return addon.state(this.h).cap; }
  get horizon() { return addon.state(this.h).horizon; }
  set horizon(v) { addon.setHorizon(this.h, v); }
  get pixelsSeen() { return addon.state(this.h).pixelsSeen; }

  // setup(gaussians, cams, images, maxViewW, maxViewH, sceneRadius) (trainer.js:100-355)
  setup(gaussians, cams, images, maxViewW, maxViewH, sceneRadius) {
    addon.setup(this.h, gaussians.data, gaussians.n, gaussians.sh ?? null, cams, images, maxViewW, maxViewH,
      sceneRadius);
    let total = 0;
    this.camMeta = cams.map((c) => {
      const im = images[c.imgIdx];
      const m = { ...c, R: Array.from(c.R), t: Array.from(c.t), w: im.tw, h: im.th, offset: total, f0: c.f };
      total += im.tw * im.th;
      return m;
    });
    this.sceneRadius = sceneRadius;
    this.holdout = -1;
    this.logfScale = 0;
    this.camStep = 0;
    this.camM = new Float64Array((cams.length + 1) * 8);
    this.camV = new Float64Array((cams.length + 1) * 8);
    this.lastRefine = 0;
  }

  // stepOnce (trainer.js:398-471): camera pick here, the step in the library
  stepOnce() {
    let ci = (this.rand() * this.camMeta.length) | 0;
    for (let tries = 0; tries < 16; tries++) {
      const bad = ci === this.holdout || (this.excluded && this.excluded.has(ci));
      if (!bad) break;
      ci = (ci + 1) % this.camMeta.length;
    }
    this.lastCam = ci;
    addon.step(this.h, ci);
    const it = this.iter;
    if ((this.opts.camOpt ?? false) && it > 1500 && it % 25 === 0) this._applyCamGrads();
  }

  // several views per optimiser step (no reference counterpart)
  stepBatch(cams) {
    addon.stepBatch(this.h, Uint32Array.from(cams));
    this.lastCam = cams[cams.length - 1];
  }

  // readLoss (trainer.js:615-631): mean squared error per pixel-channel, or null
  async readLoss() {
    const px = this.pixelsSeen;
    const s = await addon.readStats(this.h);
    this.entryOverflowTiles += s[3];
    if (!px || !s[2]) return null;
    return s[0] / 16 / (s[2] * 3);
  }

  // readGaussians (trainer.js:797-817): {data, n, sh, shK}
  async readGaussians() { return addon.readGaussians(this.h); }

  // no reference counterpart: the Adam moments back to setup()'s zeros, so a
  // model written back trains on from a fresh optimiser state
  resetMoments() { addon.resetMoments(this.h); }

  // renderView(camParams, target, trainMode, offset) (trainer.js:634-655): a
  // headless RGBA Float32Array replaces the canvas
  renderView(camParams, target = null, trainMode = 0, offset = 0) {
    return addon.renderView(this.h, camParams, trainMode, offset,
      target instanceof Float32Array ? target : null);
  }

  renderTrainCam(ci, target = null) {
    const m = this.camMeta[ci];
    return this.renderView(m, target, 0, m.offset);
  }

  // refine(rng) (trainer.js:666-794); rng must not call back into this trainer.
  // Without an rng the library's own generator draws (the reference's default
  // is Math.random): no call into JavaScript per draw.
  async refine(rng) {
    addon.setGrowLimit(this.h, this.growLimit || 0);
    return addon.refine(this.h, rng);
  }

  // ---- evaluation (trainer.js:542-612) ----
  _evalPass(ci, override) {
    const cam = override ? { ...this.camMeta[ci], ...override } : null;
    const { stats, camGrad } = addon.evalPass(this.h, ci, cam);
    const validPx = Math.max(1, stats[2]);
    const mse = stats[0] / 16 / (validPx * 3);
    return { psnr: mse > 0 ? -10 * Math.log10(mse) : Infinity, camGrad };
  }

  async evalCamPsnr(ci) { return this._evalPass(ci).psnr; }

  async evalCamPsnrRefined(ci, steps = 200) {
    const meta = this.camMeta[ci];
    let R = Array.from(meta.R);
    let t = meta.t.slice();
    let g = 0, b = 0;
    const doExp = this.opts.expComp ?? false;
    const m = new Float64Array(8), v = new Float64Array(8);
    const b1 = 0.9, b2 = 0.99, eps = 1e-15;
    const rotLr = 3e-4, trnLr = 3e-4 * this.sceneRadius, expLr = 5e-3;
    for (let s = 1; s <= steps; s++) {
      const { camGrad } = this._evalPass(ci, { R, t, g, b });
      const upd = new Float64Array(8);
      for (let k = 0; k < 8; k++) {
        const grad = camGrad[ci * 8 + k] / 64;
        m[k] = b1 * m[k] + (1 - b1) * grad;
        v[k] = b2 * v[k] + (1 - b2) * grad * grad;
        const mh = m[k] / (1 - Math.pow(b1, s));
        const vh = v[k] / (1 - Math.pow(b2, s));
        upd[k] = (k < 3 ? rotLr : (k < 6 ? trnLr : expLr)) * mh / (Math.sqrt(vh) + eps);
      }
      R = m3mul(rodrigues([-upd[0], -upd[1], -upd[2]]), R);
      t = [t[0] - upd[3], t[1] - upd[4], t[2] - upd[5]];
      if (doExp) {
        g = Math.max(-0.1, Math.min(0.1, g - upd[6]));
        b = Math.max(-0.05, Math.min(0.05, b - upd[7]));
      }
    }
    return this._evalPass(ci, { R, t, g, b }).psnr;
  }

  // _applyCamGrads (trainer.js:476-537): one Adam step on every camera pose + the shared focal
  _applyCamGrads() {
    const g = addon.readCamGrads(this.h, true);
    this.camStep++;
    const t = this.camStep;
    const decay = Math.pow(0.02, Math.min(1, this.iter / (0.75 * this.horizon)));
    const rotLr = 2e-4 * decay, trnLr = 2e-4 * this.sceneRadius * decay, focLr = 1e-4 * decay;
    const b1 = 0.9, b2 = 0.99, eps = 1e-15;
    const step = (row, slot, lr) => {
      const j = row * 8 + slot;
      const grad = g[j] / 64;
      this.camM[j] = b1 * this.camM[j] + (1 - b1) * grad;
      this.camV[j] = b2 * this.camV[j] + (1 - b2) * grad * grad;
      const mh = this.camM[j] / (1 - Math.pow(b1, t));
      const vh = this.camV[j] / (1 - Math.pow(b2, t));
      return lr * mh / (Math.sqrt(vh) + eps);
    };
    const expLr = 5e-3;
    const doExp = this.opts.expComp ?? false;
    for (let r = 1; r < this.camMeta.length; r++) {
      if (r === this.holdout) continue;
      const meta = this.camMeta[r];
      const dw = [-step(r, 0, rotLr), -step(r, 1, rotLr), -step(r, 2, rotLr)];
      meta.R = m3mul(rodrigues(dw), meta.R);
      meta.t = [meta.t[0] - step(r, 3, trnLr), meta.t[1] - step(r, 4, trnLr), meta.t[2] - step(r, 5, trnLr)];
      if (doExp) {
        meta.g = Math.max(-0.1, Math.min(0.1, (meta.g || 0) - step(r, 6, expLr)));
        meta.b = Math.max(-0.05, Math.min(0.05, (meta.b || 0) - step(r, 7, expLr)));
      }
    }
    const nr = this.camMeta.length;
    this.logfScale = Math.max(-0.3, Math.min(0.3, this.logfScale - step(nr, 0, focLr)));
    this.camMeta.forEach((m, i) => {
      m.f = m.f0 * Math.exp(this.logfScale);
      addon.setCamera(this.h, i, m);
    });
  }

  // PLY bytes (bakeOpacityCompensation + gaussiansToPly, ply.js:17-99) computed on the device
  exportPly(bake = false, f = 0, camPositions = new Float64Array(0)) {
    return addon.exportPly(this.h, bake, f, Float64Array.from(camPositions));
  }
}

export default GSTrainer;
