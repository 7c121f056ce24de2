"""GSTrainer: the host-side mirror of splat.js's trainer (src/gs/trainer.js)
over the C ABI of libsplat_b200.so.

Method names, arguments and error behaviour follow the reference so a caller
of ``GSTrainer`` (src/session.js, src/gs/gradcheck.js) finds the same surface:
``create / setup / stepOnce / renderView / renderTrainCam / readLoss /
refine / readGaussians / evalCamPsnr / evalCamPsnrRefined``, plus
``stepBatch`` (several views per optimiser step).  The reference's methods
that return Promises return plain values here.  The camera pick of stepOnce
(``rand``, holdout and excluded cameras) stays on the host, as in the
reference; everything else runs in the CUDA library.
"""
from __future__ import annotations

import ctypes as C
import math
import random

import numpy as np

from . import native as N

STRIDE = 16


def rodrigues(w):
    """Axis-angle -> rotation (src/sfm/geometry.js:150-160)."""
    th = math.sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2])
    if th < 1e-12:
        return [1.0, 0, 0, 0, 1.0, 0, 0, 0, 1.0]
    k = [w[0] / th, w[1] / th, w[2] / th]
    c, s = math.cos(th), math.sin(th)
    v = 1 - c
    return [c + k[0] * k[0] * v, k[0] * k[1] * v - k[2] * s, k[0] * k[2] * v + k[1] * s,
            k[1] * k[0] * v + k[2] * s, c + k[1] * k[1] * v, k[1] * k[2] * v - k[0] * s,
            k[2] * k[0] * v - k[1] * s, k[2] * k[1] * v + k[0] * s, c + k[2] * k[2] * v]


def m3mul(A, B):
    """3x3 row-major product (src/sfm/geometry.js:108-114)."""
    return [A[i * 3] * B[j] + A[i * 3 + 1] * B[3 + j] + A[i * 3 + 2] * B[6 + j] for i in range(3) for j in range(3)]


def _cam_struct(c, imgIdx=0):
    s = N.GsCamera()
    s.R[:] = [float(x) for x in c["R"]]
    s.t[:] = [float(x) for x in c["t"]]
    s.f, s.cx, s.cy = float(c["f"]), float(c["cx"]), float(c["cy"])
    s.w, s.h = int(c["w"]), int(c["h"])
    s.imgIdx = int(c.get("imgIdx", imgIdx))
    s.g, s.b = float(c.get("g", 0.0) or 0.0), float(c.get("b", 0.0) or 0.0)
    return s


# option names of the reference (trainer.js:18-49) -> gs_options fields
_OPT_FIELDS = [name for name, _ in N.GsOptions._fields_]


class _Queue:
    """device.queue stand-in: onSubmittedWorkDone() waits for the stream."""

    def __init__(self, trainer):
        self._t = trainer

    def onSubmittedWorkDone(self):
        N.check(N.lib().gs_sync(self._t._h), self._t._h)


class _Device:
    def __init__(self, trainer):
        self.queue = _Queue(trainer)


class GSTrainer:
    """createTrainer(opts) / GSTrainer.create(opts) (src/index.js:56-58, trainer.js:13-16)."""

    @staticmethod
    def create(opts=None):
        return GSTrainer(opts or {})

    def __init__(self, opts=None):
        self.opts = dict(opts or {})
        L = N.lib()
        o = N.GsOptions()
        N.check(L.gs_default_options(C.byref(o)))
        for k in _OPT_FIELDS:
            if self.opts.get(k) is not None:
                val = self.opts[k]
                setattr(o, k, int(val) if isinstance(getattr(o, k), int) else float(val))
        if self.opts.get("tileGrad") is not None:
            o.tileGrad = 1 if self.opts["tileGrad"] else 0
        h = C.c_void_p()
        N.check(L.gs_create(C.byref(o), C.byref(h)), None)
        self._h = h
        self._o = o
        self.tileGrad = bool(o.tileGrad)
        self.shDeg = int(o.shDeg)
        self.shK = (self.shDeg + 1) ** 2 - 1 if self.shDeg > 0 else 0
        self.stride = STRIDE
        self.iter_ = 0
        self.holdout = -1
        self.excluded = set()
        self.lastCam = 0
        self.lastRefine = 0
        self.growLimit = 0
        self.entryOverflowTiles = 0
        self.rand = random.random
        self.device = _Device(self)
        self.camMeta = []

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            N.lib().gs_destroy(h)
            self._h = None

    # ---- fields (trainer.js state the callers read/write) ----
    def _state(self):
        s = N.GsState()
        N.check(N.lib().gs_get_state(self._h, C.byref(s)), self._h)
        return s

    @property
    def iter(self):
        return self._state().iter

    @iter.setter
    def iter(self, v):
        N.check(N.lib().gs_set_iter(self._h, int(v)), self._h)

    @property
    def n(self):
        return self._state().n

    @property
    def cap(self):
        return self._state().cap

    @property
    def pixelsSeen(self):
        return self._state().pixelsSeen

    @property
    def horizon(self):
        return self._state().horizon

    @horizon.setter
    def horizon(self, v):
        N.check(N.lib().gs_set_horizon(self._h, int(v)), self._h)

    @property
    def maxTiles(self):
        return self._state().maxTiles

    # ---- setup (trainer.js:100-355) ----
    def setup(self, gaussians, cams, images, maxViewW, maxViewH, sceneRadius):
        data = np.ascontiguousarray(gaussians["data"], np.float32)
        n = int(gaussians["n"])
        if data.size < n * STRIDE:
            raise ValueError("gaussians.data holds fewer than n*16 floats")
        sh = gaussians.get("sh")
        sh = None if sh is None else np.ascontiguousarray(sh, np.float32)
        self._rgbs = [np.ascontiguousarray(im["rgb"], np.float32) for im in images]
        imgs = (N.GsImage * len(images))()
        for k, im in enumerate(images):
            imgs[k].tw, imgs[k].th = int(im["tw"]), int(im["th"])
            imgs[k].rgb = N.ptr(self._rgbs[k])
        cs = (N.GsCamera * len(cams))(*[_cam_struct(c) for c in cams])
        N.check(N.lib().gs_setup(self._h, N.ptr(data), n, N.ptr(sh), cs, len(cams), imgs, len(images),
                                 int(maxViewW), int(maxViewH), float(sceneRadius)), self._h)
        total = 0
        self.camMeta = []
        for i, c in enumerate(cams):
            im = images[c["imgIdx"]]
            m = dict(c)
            m.update(w=int(im["tw"]), h=int(im["th"]), offset=total, f0=c["f"])
            total += int(im["tw"]) * int(im["th"])
            self.camMeta.append(m)
        self.cams = cams
        self.sceneRadius = sceneRadius
        self.holdout = -1
        self.logfScale = 0.0
        self.camStep = 0
        self.camM = np.zeros((len(cams) + 1) * 8)
        self.camV = np.zeros((len(cams) + 1) * 8)
        self.lastRefine = 0
        r = sceneRadius
        self.hBySlot = [r * 2e-3, r * 2e-3, r * 2e-3, 0.02, 0.02, 0.02, 0.02, 0.02, 0.02, 0.02, 0.05, 0.05, 0.05,
                        0.05, 0, 0]
        self.slotNames = ['pos.x', 'pos.y', 'pos.z', 'logSx', 'logSy', 'logSz', 'q.w', 'q.x', 'q.y', 'q.z', 'c.r',
                          'c.g', 'c.b', 'opa', 'pad', 'pad']

    # ---- training (trainer.js:398-471) ----
    def _pick(self):
        nc = len(self.camMeta)
        ci = int(self.rand() * nc)
        for _ in range(16):
            bad = ci == self.holdout or ci in self.excluded
            if not bad:
                break
            ci = (ci + 1) % nc
        return ci

    def stepOnce(self):
        ci = self._pick()
        self.lastCam = ci
        N.check(N.lib().gs_step(self._h, ci), self._h)
        it = self.iter
        if self.opts.get("camOpt", False) and it > 1500 and it % 25 == 0:
            self._applyCamGrads()

    def stepBatch(self, cams=None, nviews=None):
        """One optimiser step over several views (camera indices, or
        `nviews` picks made like stepOnce's)."""
        if cams is None:
            cams = [self._pick() for _ in range(int(nviews or 1))]
        arr = (C.c_uint32 * len(cams))(*[int(c) for c in cams])
        N.check(N.lib().gs_step_batch(self._h, arr, len(cams)), self._h)
        self.lastCam = int(cams[-1])

    # ---- readouts ----
    def readLoss(self):
        """trainer.js:615-631: mean squared error per pixel-channel, or None."""
        px = self.pixelsSeen
        st = (C.c_uint32 * 4)()
        N.check(N.lib().gs_read_stats(self._h, st), self._h)  # also resets pixelsSeen
        self.entryOverflowTiles += st[3]
        if px == 0 or st[2] == 0:
            return None
        return st[0] / 16 / (st[2] * 3)

    def readGaussians(self):
        n = self.n
        data = np.zeros(n * STRIDE, np.float32)
        sh = np.zeros(n * 3 * self.shK, np.float32) if self.shK else None
        nn = C.c_uint32()
        N.check(N.lib().gs_read_gaussians(self._h, N.ptr(data), N.ptr(sh), C.byref(nn)), self._h)
        return {"data": data, "n": int(nn.value), "sh": sh, "shK": self.shK}

    def writeGaussians(self, data=None, sh=None, n=None):
        n = self.n if n is None else int(n)
        d = None if data is None else np.ascontiguousarray(data, np.float32)
        s = None if sh is None else np.ascontiguousarray(sh, np.float32)
        N.check(N.lib().gs_write_gaussians(self._h, N.ptr(d), N.ptr(s), n), self._h)

    def resetMoments(self):
        """Zero the Adam and SH-Adam moments, as setup() does (no reference
        counterpart): with writeGaussians, restarts training from a model."""
        N.check(N.lib().gs_reset_moments(self._h), self._h)

    def readMoments(self):
        n, k3 = self.n, 3 * self.shK
        m = np.zeros(n * STRIDE, np.float32)
        v = np.zeros(n * STRIDE, np.float32)
        shM = np.zeros(max(1, n * k3), np.float32)
        shV = np.zeros(max(1, n * k3), np.float32)
        N.check(N.lib().gs_read_moments(self._h, N.ptr(m), N.ptr(v), N.ptr(shM), N.ptr(shV)), self._h)
        return m, v, shM[:n * k3], shV[:n * k3]

    # ---- views (trainer.js:634-660) ----
    def renderView(self, camParams, target=None, trainMode=0, offset=0):
        """Render into an (h, w, 4) float32 array (RGB, alpha = 1 - T); when
        `target` is a numpy array of that size it is filled in place."""
        c = _cam_struct(camParams)
        out = target if isinstance(target, np.ndarray) else np.zeros((c.h, c.w, 4), np.float32)
        N.check(N.lib().gs_render(self._h, C.byref(c), int(trainMode), int(offset), N.ptr(out)), self._h)
        return out

    def renderTrainCam(self, ci, target=None):
        meta = self.camMeta[ci]
        return self.renderView(meta, target, 0, meta["offset"])

    # ---- evaluation (trainer.js:542-612) ----
    def _evalPass(self, ci, override=None):
        nr = len(self.camMeta) + 1
        st = (C.c_uint32 * 4)()
        cg = np.zeros(nr * 8, np.int32)
        cam = None
        if override:
            meta = dict(self.camMeta[ci])
            meta.update(override)
            cam = C.byref(_cam_struct(meta))
        N.check(N.lib().gs_eval_pass(self._h, int(ci), cam, st, N.ptr(cg, C.c_int32)), self._h)
        v = st[0]
        valid = max(1, st[2])
        mse = v / 16 / (valid * 3)
        return {"psnr": -10 * math.log10(mse) if mse > 0 else math.inf, "camGrad": cg}

    def evalCamPsnr(self, ci):
        return self._evalPass(ci)["psnr"]

    def evalCamPsnrRefined(self, ci, steps=200):
        meta = self.camMeta[ci]
        R = list(meta["R"])
        t = list(meta["t"])
        g = b = 0.0
        doExp = self.opts.get("expComp", False)
        m = [0.0] * 8
        v = [0.0] * 8
        b1, b2, eps = 0.9, 0.99, 1e-15
        rotLr, trnLr, expLr = 3e-4, 3e-4 * self.sceneRadius, 5e-3
        for s in range(1, steps + 1):
            cg = self._evalPass(ci, {"R": R, "t": t, "g": g, "b": b})["camGrad"]
            upd = [0.0] * 8
            for k in range(8):
                grad = cg[ci * 8 + k] / 64
                m[k] = b1 * m[k] + (1 - b1) * grad
                v[k] = b2 * v[k] + (1 - b2) * grad * grad
                mh = m[k] / (1 - b1 ** s)
                vh = v[k] / (1 - b2 ** s)
                upd[k] = (rotLr if k < 3 else (trnLr if k < 6 else expLr)) * mh / (math.sqrt(vh) + eps)
            R = m3mul(rodrigues([-upd[0], -upd[1], -upd[2]]), R)
            t = [t[0] - upd[3], t[1] - upd[4], t[2] - upd[5]]
            if doExp:
                g = max(-0.1, min(0.1, g - upd[6]))
                b = max(-0.05, min(0.05, b - upd[7]))
        return self._evalPass(ci, {"R": R, "t": t, "g": g, "b": b})["psnr"]

    def _applyCamGrads(self):
        """trainer.js:476-537: one Adam step on every camera pose + shared focal."""
        rows = len(self.camMeta) + 1
        g = np.zeros(rows * 8, np.int32)
        N.check(N.lib().gs_read_cam_grads(self._h, N.ptr(g, C.c_int32), 1), self._h)
        self.camStep += 1
        t = self.camStep
        it = self.iter
        decay = 0.02 ** min(1, it / (0.75 * self.horizon))
        rotLr, trnLr, focLr = 2e-4 * decay, 2e-4 * self.sceneRadius * decay, 1e-4 * decay
        b1, b2, eps = 0.9, 0.99, 1e-15

        def step(row, slot, lr):
            j = row * 8 + slot
            grad = g[j] / 64
            self.camM[j] = b1 * self.camM[j] + (1 - b1) * grad
            self.camV[j] = b2 * self.camV[j] + (1 - b2) * grad * grad
            mh = self.camM[j] / (1 - b1 ** t)
            vh = self.camV[j] / (1 - b2 ** t)
            return lr * mh / (math.sqrt(vh) + eps)
        expLr = 5e-3
        doExp = self.opts.get("expComp", False)
        for r in range(1, len(self.camMeta)):
            if r == self.holdout:
                continue
            meta = self.camMeta[r]
            dw = [-step(r, 0, rotLr), -step(r, 1, rotLr), -step(r, 2, rotLr)]
            meta["R"] = m3mul(rodrigues(dw), meta["R"])
            meta["t"] = [meta["t"][0] - step(r, 3, trnLr), meta["t"][1] - step(r, 4, trnLr),
                         meta["t"][2] - step(r, 5, trnLr)]
            if doExp:
                meta["g"] = max(-0.1, min(0.1, (meta.get("g") or 0) - step(r, 6, expLr)))
                meta["b"] = max(-0.05, min(0.05, (meta.get("b") or 0) - step(r, 7, expLr)))
        nr = len(self.camMeta)
        self.logfScale = max(-0.3, min(0.3, self.logfScale - step(nr, 0, focLr)))
        for i, m in enumerate(self.camMeta):
            m["f"] = m["f0"] * math.exp(self.logfScale)
            N.check(N.lib().gs_set_camera(self._h, i, C.byref(_cam_struct(m))), self._h)

    # ---- refinement (trainer.js:666-794) ----
    def refine(self, rng=None):
        """refine(rng) (trainer.js:666-794).  rng: a callable returning floats
        in [0, 1), drawn in the reference's order; None draws from the
        library's own generator (the reference's default is Math.random), with
        no Python call per draw."""
        cb = N.RNG_FN(lambda _ctx: float(rng())) if rng is not None else N.RNG_FN()  # NULL: own generator
        out = N.GsRefineResult()
        gl = int(self.growLimit or 0)
        N.check(N.lib().gs_set_grow_limit(self._h, gl), self._h)
        N.check(N.lib().gs_refine(self._h, cb, None, C.byref(out)), self._h)
        if out.early:
            return {"moved": 0, "grown": 0, "n": int(out.n)}
        return {"moved": int(out.moved), "grown": int(out.grown), "n": int(out.n), "maxTile": int(out.maxTile),
                "overflow": int(out.overflow)}

    # ---- raster configuration ----
    def autotune(self, cams=None, reps=3):
        """Pick tile size {8,16,32} x splat-batch depth {64,128,256} by timing
        the training pass on `cams` (default: the first few cameras).
        Returns (tile, depth, {(tile, depth): ms})."""
        if cams is None:
            cams = list(range(min(len(self.camMeta), int(self._o.maxBatch))))
        arr = (C.c_uint32 * len(cams))(*[int(c) for c in cams])
        bt, bd = C.c_int32(), C.c_int32()
        ms = (C.c_float * 9)()
        N.check(N.lib().gs_autotune(self._h, arr, len(cams), int(reps), C.byref(bt), C.byref(bd), ms), self._h)
        table = {(8 << i, 64 << j): ms[i * 3 + j] for i in range(3) for j in range(3)}
        return bt.value, bd.value, table

    def setRasterConfig(self, tile, depth):
        N.check(N.lib().gs_set_raster_config(self._h, int(tile), int(depth)), self._h)

    # ---- gradient check support (gradcheck.js:266-356) ----
    def gradPass(self, ci=0):
        """encodeRaster + chain without Adam; returns (gradF, shGrad, stats)."""
        n = self.n
        gF = np.zeros(n * STRIDE, np.float32)
        sG = np.zeros(max(1, n * 3 * self.shK), np.float32)
        st = np.zeros(4, np.uint32)
        N.check(N.lib().gs_grad_pass(self._h, int(ci), N.ptr(gF), N.ptr(sG), N.ptr(st, C.c_uint32)), self._h)
        return gF, sG[:n * 3 * self.shK], st
