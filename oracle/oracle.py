"""ctypes wrapper over oracle/liboracle.so.

TEST INFRASTRUCTURE ONLY: the parity checker and the CPU baseline.  Only
tests/, ``__graft_entry__.smoke()`` and the CPU legs of ``bench.py`` import
this module; the product (the CUDA library and its host mirror) never does.

Array layouts follow the reference (src/gs/shaders.js:14-28): params stride
16 f32, SH channel-major 3K f32 per splat, proj stride 16 f32, gradP stride 16
i32.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")


class OOpts(C.Structure):
    _fields_ = [("eCut", C.c_float), ("aMin", C.c_float), ("radClamp", C.c_float), ("anisoReg", C.c_float),
                ("shDeg", C.c_int32), ("tile", C.c_int32), ("entriesCap", C.c_uint64), ("tileCull", C.c_int32)]


class OCam(C.Structure):
    _fields_ = [("R", C.c_float * 9), ("t", C.c_float * 3), ("f", C.c_float), ("cx", C.c_float), ("cy", C.c_float),
                ("w", C.c_int32), ("h", C.c_int32), ("gain", C.c_float), ("bias", C.c_float),
                ("offset", C.c_uint32), ("camIdx", C.c_uint32), ("ncams", C.c_uint32), ("activeSh", C.c_float),
                ("train", C.c_int32)]


class OAdam(C.Structure):
    _fields_ = [("lr", C.c_float * 16), ("b1", C.c_float), ("b2", C.c_float), ("eps", C.c_float),
                ("bc1", C.c_float), ("bc2", C.c_float), ("minLS", C.c_float), ("maxLS", C.c_float),
                ("maxLogit", C.c_float), ("reg", C.c_float), ("shLr", C.c_float)]


class ORefineOut(C.Structure):
    _fields_ = [("moved", C.c_uint32), ("grown", C.c_uint32), ("n", C.c_uint32), ("early", C.c_int32)]


RNG_FN = C.CFUNCTYPE(C.c_double, C.c_void_p)


def build() -> None:
    """Compile liboracle.so with the committed Makefile (no-op when current)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        L = C.CDLL(_LIB)
        P = C.POINTER
        f32p, f64p, u32p, i32p, u64p, u8p = (P(C.c_float), P(C.c_double), P(C.c_uint32), P(C.c_int32),
                                             P(C.c_uint64), P(C.c_uint8))
        L.oracle_set_threads.restype = C.c_int
        L.oracle_set_threads.argtypes = [C.c_int]
        L.oracle_exp_f32.restype = C.c_float
        L.oracle_exp_f32.argtypes = [C.c_float]
        L.oracle_log_f32.restype = C.c_float
        L.oracle_log_f32.argtypes = [C.c_float]
        L.oracle_sin_f64.restype = C.c_double
        L.oracle_sin_f64.argtypes = [C.c_double]
        L.oracle_dither.restype = C.c_float
        L.oracle_dither.argtypes = [C.c_uint32]
        L.oracle_adam_bias.argtypes = [C.c_double, f32p, f32p]
        L.oracle_project_f32.argtypes = [P(OOpts), P(OCam), f32p, f32p, C.c_uint32, f32p]
        L.oracle_project_f64.argtypes = [P(OOpts), P(OCam), f64p, f64p, C.c_uint32, f64p]
        L.oracle_records_f32.argtypes = [P(OOpts), P(OCam), f32p, C.c_uint32, f32p, u32p]
        L.oracle_bin_f32.restype = C.c_uint64
        L.oracle_bin_f32.argtypes = [P(OOpts), P(OCam), f32p, C.c_uint32, u32p, u32p, u32p, C.c_uint64, u32p,
                                     u8p, u32p]
        L.oracle_render_f32.argtypes = [P(OOpts), P(OCam), f32p, u32p, u32p, u32p, f32p, f32p, u32p, i32p, u32p,
                                        i32p, u64p, C.c_int, C.c_int]
        L.oracle_render_sample_f32.argtypes = [P(OOpts), P(OCam), f32p, u32p, u32p, u32p, i32p, u32p, i32p, u64p,
                                               C.c_int, C.c_int]
        L.oracle_chain_f32.argtypes = [P(OOpts), P(OCam), f32p, f32p, f32p, C.c_uint32, i32p, f32p, f32p, i32p]
        L.oracle_adam_f32.argtypes = [P(OAdam), C.c_uint32, C.c_int, f32p, f32p, f32p, f32p, f32p, f32p, f32p,
                                      f32p]
        L.oracle_step_f32.restype = C.c_int
        L.oracle_step_f32.argtypes = [P(OOpts), P(OCam), C.c_int, P(OAdam), C.c_uint32, f32p, f32p, u32p, f32p,
                                      f32p, f32p, f32p, u32p, i32p, f32p, f32p, C.c_int, C.c_int, u64p, f32p]
        L.oracle_eval_f64.argtypes = [P(OOpts), P(OCam), f64p, f64p, C.c_uint32, u32p, f64p, f64p, f64p, f32p,
                                      C.c_int]
        L.oracle_fd_local_f64.argtypes = [P(OOpts), P(OCam), f64p, f64p, C.c_uint32, u32p, u32p, C.c_uint32,
                                          f64p, C.c_uint32, f64p]
        L.oracle_fd_local_f64.restype = C.c_int
        L.oracle_refine.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, C.c_double, C.c_double, C.c_double,
                                    C.c_int, f32p, f32p, f32p, f32p, f32p, f32p, RNG_FN, C.c_void_p,
                                    P(ORefineOut), C.c_int]
        _lib = L
    return _lib


def set_threads(n: int = 0) -> int:
    """Host threads of the oracle's parallel loops (n <= 0 keeps the current
    setting); returns the count in effect."""
    return int(lib().oracle_set_threads(int(n)))


def _p(a, ct):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(ct))


def opts(eCut=4.5, aMin=0.0039, radClamp=1.0, anisoReg=0.005, shDeg=2, tile=16, entriesCap=12_000_000, tileCull=0):
    """tileCull=1 mirrors the B200 library's culled tile lists (its default);
    0 keeps the reference's full rectangle lists."""
    return OOpts(eCut, aMin, radClamp, anisoReg, shDeg, tile, entriesCap, tileCull)


def cam(R, t, f, cx, cy, w, h, gain=1.0, bias=0.0, offset=0, camIdx=0, ncams=1, activeSh=2.0, train=1):
    c = OCam()
    c.R[:] = [float(x) for x in R]
    c.t[:] = [float(x) for x in t]
    c.f, c.cx, c.cy, c.w, c.h = f, cx, cy, int(w), int(h)
    c.gain, c.bias, c.offset, c.camIdx, c.ncams = gain, bias, int(offset), int(camIdx), int(ncams)
    c.activeSh, c.train = activeSh, int(train)
    return c


def adam_hp(lr16, t, minLS, maxLS, maxLogit=8.0, reg=0.01, shLr=1.25e-4):
    h = OAdam()
    h.lr[:] = [float(x) for x in lr16]
    h.b1, h.b2, h.eps = 0.9, 0.999, 1e-15
    bc1, bc2 = C.c_float(), C.c_float()
    lib().oracle_adam_bias(float(t), C.byref(bc1), C.byref(bc2))
    h.bc1, h.bc2 = bc1.value, bc2.value
    h.minLS, h.maxLS, h.maxLogit, h.reg, h.shLr = minLS, maxLS, maxLogit, reg, shLr
    return h


def sh_rest(deg: int) -> int:
    return (deg + 1) * (deg + 1) - 1 if deg > 0 else 0


def project(o, c, params, sh, n):
    proj = np.zeros(n * 16, np.float32)
    lib().oracle_project_f32(C.byref(o), C.byref(c), _p(params, C.c_float), _p(sh, C.c_float), n,
                             _p(proj, C.c_float))
    return proj


def records(o, c, proj, n):
    rec = np.zeros(n * 12, np.float32)
    rect = np.zeros(n * 2, np.uint32)
    lib().oracle_records_f32(C.byref(o), C.byref(c), _p(proj, C.c_float), n, _p(rec, C.c_float),
                             _p(rect, C.c_uint32))
    return rec, rect


def bin_tiles(o, c, proj, n, cap=None):
    tx = (c.w + o.tile - 1) // o.tile
    ty = (c.h + o.tile - 1) // o.tile
    nt = tx * ty
    if cap is None:
        cap = max(1, int(n) * ((c.w // o.tile + 2) * (c.h // o.tile + 2)))
        cap = min(cap, 200_000_000)
    start = np.zeros(nt + 1, np.uint32)
    ids = np.zeros(cap, np.uint32)
    keys = np.zeros(cap, np.uint32)
    cnt = np.zeros(nt, np.uint32)
    dropped = np.zeros(nt, np.uint8)
    ov = C.c_uint32()
    E = lib().oracle_bin_f32(C.byref(o), C.byref(c), _p(proj, C.c_float), n, _p(start, C.c_uint32),
                             _p(ids, C.c_uint32), _p(keys, C.c_uint32), cap, _p(cnt, C.c_uint32),
                             _p(dropped, C.c_uint8), C.byref(ov))
    assert E <= cap, "entry buffer too small"
    return dict(start=start, ids=ids[:E].copy(), keys=keys[:E].copy(), cnt=cnt, dropped=dropped,
                overflow=ov.value, numTiles=nt)


def render(o, c, proj, bins, targets, n, train=True, variant=0, ncams=1):
    W, H = c.w, c.h
    out = np.zeros(W * H * 4, np.float32)
    finalT = np.zeros(W * H, np.float32)
    end = np.zeros(W * H, np.uint32)
    gradP = np.zeros(n * 16, np.int32)
    stats = np.zeros(4, np.uint32)
    gradCam = np.zeros((ncams + 1) * 8, np.int32)
    pairs = C.c_uint64(0)
    lib().oracle_render_f32(C.byref(o), C.byref(c), _p(proj, C.c_float), _p(bins["start"], C.c_uint32),
                            _p(bins["ids"], C.c_uint32), _p(targets, C.c_uint32), _p(out, C.c_float),
                            _p(finalT, C.c_float), _p(end, C.c_uint32), _p(gradP, C.c_int32),
                            _p(stats, C.c_uint32), _p(gradCam, C.c_int32), C.byref(pairs), int(train),
                            int(variant))
    return dict(img=out, finalT=finalT, end=end, gradP=gradP, stats=stats, gradCam=gradCam, pairs=pairs.value)


def chain(o, c, params, proj, sh, n, gradP, gradCam):
    K = sh_rest(o.shDeg)
    gradF = np.zeros(n * 16, np.float32)
    shGrad = np.zeros(max(1, n * 3 * K), np.float32)
    lib().oracle_chain_f32(C.byref(o), C.byref(c), _p(params, C.c_float), _p(proj, C.c_float),
                           _p(sh, C.c_float), n, _p(gradP, C.c_int32), _p(gradF, C.c_float),
                           _p(shGrad, C.c_float), _p(gradCam, C.c_int32))
    return gradF, shGrad[: n * 3 * K]


def step(o, cams, hp, params, sh, targets, m, v, shM, shV, n, stats=None, gradCam=None, do_adam=True,
         variant=0, want_image=False):
    """One (batched) training step in place on params/sh/m/v/shM/shV.

    Returns the summed gradients, the pair count and the first view's image."""
    K = sh_rest(o.shDeg)
    V = len(cams)
    arr = (OCam * V)(*cams)
    if stats is None:
        stats = np.zeros(4, np.uint32)
    if gradCam is None:
        gradCam = np.zeros((max(c.ncams for c in cams) + 1) * 8, np.int32)
    gradF = np.zeros(n * 16, np.float32)
    shGrad = np.zeros(max(1, n * 3 * K), np.float32)
    pairs = C.c_uint64(0)
    img = np.zeros(cams[0].w * cams[0].h * 4, np.float32) if want_image else None
    lib().oracle_step_f32(C.byref(o), arr, V, C.byref(hp), n, _p(params, C.c_float), _p(sh, C.c_float),
                          _p(targets, C.c_uint32), _p(m, C.c_float), _p(v, C.c_float), _p(shM, C.c_float),
                          _p(shV, C.c_float), _p(stats, C.c_uint32), _p(gradCam, C.c_int32),
                          _p(gradF, C.c_float), _p(shGrad, C.c_float), int(do_adam), int(variant),
                          C.byref(pairs), _p(img, C.c_float))
    return dict(gradF=gradF, shGrad=shGrad[: n * 3 * K], pairs=pairs.value, stats=stats, gradCam=gradCam,
                img=img)


def eval_f64(o, c, params64, sh64, n, targets, grads=True, want_image=False, quantise=False):
    """FP64 host evaluation: (loss, sqerr, validPx), gradF, shGrad.  Unquantised
    unless `quantise`, which truncates each per-pixel gradient contribution to
    the reference's 1/16384 fixed-point quantum (in double)."""
    K = sh_rest(o.shDeg)
    loss3 = np.zeros(3, np.float64)
    gF = np.zeros(n * 16, np.float64) if grads else None
    sG = np.zeros(max(1, n * 3 * K), np.float64) if grads else None
    img = np.zeros(c.w * c.h * 4, np.float32) if want_image else None
    lib().oracle_eval_f64(C.byref(o), C.byref(c), _p(params64, C.c_double), _p(sh64, C.c_double), n,
                          _p(targets, C.c_uint32), _p(loss3, C.c_double), _p(gF, C.c_double),
                          _p(sG, C.c_double), _p(img, C.c_float), int(quantise))
    return loss3, gF, (sG[: n * 3 * K] if grads else None), img


def fd_local(o, c, params64, sh64, n, targets, ids, h=1e-4, max_tiles=1 << 20):
    """FP64 central differences of the loss for every parameter slot (0-13)
    and SH coefficient of the splats `ids`, over the tiles each perturbed
    splat can touch (equal to the whole-image difference).  `h` is one step
    or one per column.  Returns an (len(ids), 14 + 3K) array; rows of splats
    whose tiles exceed max_tiles are NaN."""
    K = sh_rest(o.shDeg)
    hcol = np.ascontiguousarray(np.broadcast_to(np.asarray(h, np.float64), (14 + 3 * K,)))
    ids = np.ascontiguousarray(ids, np.uint32)
    out = np.zeros((len(ids), 14 + 3 * K), np.float64)
    sh_arg = sh64 if K else np.zeros(1, np.float64)
    rc = lib().oracle_fd_local_f64(C.byref(o), C.byref(c), _p(params64, C.c_double), _p(sh_arg, C.c_double), n,
                                   _p(targets, C.c_uint32), _p(ids, C.c_uint32), len(ids), _p(hcol, C.c_double),
                                   int(max_tiles),
                                   _p(out, C.c_double))
    if rc != 0:
        raise RuntimeError("fd_local: the entry budget dropped a tile")
    return out


def refine(n, cap, params, m, v, sh, shM, shV, K, rng, iter_, growUntil, growRate=0.15, growLimit=0,
           donorSampling=0):
    """MCMC-lite refine (trainer.js:666-794) in place; rng() -> float in [0,1).
    donorSampling 1 picks clone donors by opacity weight (no reference
    counterpart; the reference samples uniformly, trainer.js:722)."""
    cb = RNG_FN(lambda _ctx: float(rng()))
    out = ORefineOut()
    dummy = np.zeros(1, np.float32)
    lib().oracle_refine(n, cap, growLimit, float(iter_), float(growUntil), float(growRate), K,
                        _p(params, C.c_float), _p(m, C.c_float), _p(v, C.c_float),
                        _p(sh if K else dummy, C.c_float), _p(shM if K else dummy, C.c_float),
                        _p(shV if K else dummy, C.c_float), cb, None, C.byref(out), int(donorSampling))
    return dict(moved=out.moved, grown=out.grown, n=out.n, early=bool(out.early))


def render_sample(o, c, proj, bins, targets, n, tile_stride, train=True, ncams=1):
    """Raster of every `tile_stride`-th tile (CPU-baseline sampling); returns the pair count."""
    gradP = np.zeros(n * 16, np.int32)
    stats = np.zeros(4, np.uint32)
    gradCam = np.zeros((ncams + 1) * 8, np.int32)
    pairs = C.c_uint64(0)
    lib().oracle_render_sample_f32(C.byref(o), C.byref(c), _p(proj, C.c_float), _p(bins["start"], C.c_uint32),
                                   _p(bins["ids"], C.c_uint32), _p(targets, C.c_uint32), _p(gradP, C.c_int32),
                                   _p(stats, C.c_uint32), _p(gradCam, C.c_int32), C.byref(pairs), int(train),
                                   int(tile_stride))
    return pairs.value, gradP


def adam(hp, n, K, params, gradF, m, v, sh, shGrad, shM, shV):
    lib().oracle_adam_f32(C.byref(hp), n, K, _p(params, C.c_float), _p(gradF, C.c_float), _p(m, C.c_float),
                          _p(v, C.c_float), _p(sh, C.c_float), _p(shGrad, C.c_float), _p(shM, C.c_float),
                          _p(shV, C.c_float))


def ply_export(params, n, sh=None, shK=0, bake=False, f=0.0, cam_positions=()):
    """ply.js:17-99 restated in numpy (double precision, float32 stores):
    bakeOpacityCompensation (when bake) followed by gaussiansToPly.  Returns
    the PLY bytes."""
    P = np.asarray(params, np.float32).reshape(-1, 16)[:n].astype(np.float64)
    K = shK if sh is not None else 0
    logit = P[:, 13].copy()
    if bake:
        cams = np.asarray(cam_positions, np.float64).reshape(-1, 3)
        z2min = np.full(n, np.inf)
        for c in cams:                                    # ply.js:22-29
            d2 = (P[:, 0] - c[0]) * (P[:, 0] - c[0]) + (P[:, 1] - c[1]) * (P[:, 1] - c[1]) \
                + (P[:, 2] - c[2]) * (P[:, 2] - c[2])
            z2min = np.minimum(z2min, d2)
        z = np.maximum(1e-3, np.sqrt(z2min))
        s_mean = np.exp((P[:, 3] + P[:, 4] + P[:, 5]) / 3)
        s2d = f * s_mean / z
        comp = (s2d * s2d) / (s2d * s2d + 0.3)
        opa = comp / (1 + np.exp(-P[:, 13]))
        cl = np.minimum(1 - 1e-6, np.maximum(1e-6, opa))
        logit = np.log(cl / (1 - cl)).astype(np.float32).astype(np.float64)
    props = ['x', 'y', 'z', 'nx', 'ny', 'nz', 'f_dc_0', 'f_dc_1', 'f_dc_2'] + \
        [f'f_rest_{k}' for k in range(3 * K)] + \
        ['opacity', 'scale_0', 'scale_1', 'scale_2', 'rot_0', 'rot_1', 'rot_2', 'rot_3']
    header = 'ply\nformat binary_little_endian 1.0\n' + f'element vertex {n}\n' + \
        '\n'.join(f'property float {p}' for p in props) + '\nend_header\n'
    rec = np.zeros((n, len(props)), np.float32)
    rec[:, 0:3] = P[:, 0:3]
    sig = 1 / (1 + np.exp(-P[:, 10:13]))
    rec[:, 6:9] = (sig - 0.5) / 0.28209479177387814
    if K:
        rec[:, 9:9 + 3 * K] = np.asarray(sh, np.float32).reshape(-1, 3 * K)[:n]
    q0 = 9 + 3 * K
    rec[:, q0] = logit
    rec[:, q0 + 1:q0 + 4] = P[:, 3:6]
    q = P[:, 6:10].copy()
    ql = np.sqrt((q * q).sum(1))
    small = ql < 1e-6
    q[~small] = q[~small] / ql[~small, None]
    q[small] = [1.0, 0.0, 0.0, 0.0]
    rec[:, q0 + 4:q0 + 8] = q
    return header.encode() + rec.astype('<f4').tobytes()


def undistort_frames(frames, recon):
    """session.js:44-80 (undistortFrames) restated in numpy float64 with the
    JavaScript's operation order and float32 stores; returns (resampled,
    list of new rgb arrays).  Out-of-frame pixels get -1 in every channel."""
    k1, k2 = float(recon["k1"]), float(recon["k2"])
    if abs(k1) < 0.01 and abs(k2) < 0.01:
        return False, [np.asarray(im["rgb"], np.float32) for im in frames]
    out = []
    for im in frames:
        tw, th = int(im["tw"]), int(im["th"])
        f = float(recon["fFeat"]) * (tw / float(im["fw"]))        # session.js:50
        cx, cy = tw / 2, th / 2
        src = np.asarray(im["rgb"], np.float32).reshape(th, tw, 3).astype(np.float64)
        x = np.arange(tw, dtype=np.float64)[None, :]
        y = np.arange(th, dtype=np.float64)[:, None]
        xp = (x + 0.5 - cx) / f                                   # :55-59, left to right
        yp = (y + 0.5 - cy) / f
        r2 = xp * xp + yp * yp
        D = 1 + k1 * r2 + k2 * r2 * r2
        rx = f * xp * D + cx - 0.5
        ry = f * yp * D + cy - 0.5
        rx, ry = np.broadcast_to(rx, (th, tw)), np.broadcast_to(ry, (th, tw))
        outside = (rx < 0) | (ry < 0) | (rx > tw - 1.001) | (ry > th - 1.001)   # :61
        rxi = np.where(outside, 0.0, rx)
        ryi = np.where(outside, 0.0, ry)
        x0 = rxi.astype(np.int64)                                 # rx | 0
        y0 = ryi.astype(np.int64)
        fx, fy = rxi - x0, ryi - y0
        x1, y1 = np.minimum(x0 + 1, tw - 1), np.minimum(y0 + 1, th - 1)
        s00, s01 = src[y0, x0], src[y0, x1]
        s10, s11 = src[y1, x0], src[y1, x1]
        fx3, fy3 = fx[..., None], fy[..., None]
        v = s00 * (1 - fx3) * (1 - fy3) + s01 * fx3 * (1 - fy3) + s10 * (1 - fx3) * fy3 + s11 * fx3 * fy3   # :71-74
        dst = v.astype(np.float32)
        dst[outside] = -1.0
        out.append(dst.reshape(-1))
    return True, out


def pack_rgba8(rgb):
    """GSTrainer.setup's target packing for one image (trainer.js:127-136):
    alpha 255 with min(255, round(255 v)) per channel (low byte), or the
    whole word 0 where red < 0."""
    a = np.asarray(rgb, np.float32).reshape(-1, 3)

    def r255(v):
        x = np.floor(v.astype(np.float64) * 255.0 + 0.5)
        return (np.minimum(x, 255.0).astype(np.int64) & 0xFF).astype(np.uint32)

    packed = (np.uint32(255) << np.uint32(24)) | (r255(a[:, 2]) << np.uint32(16)) | \
        (r255(a[:, 1]) << np.uint32(8)) | r255(a[:, 0])
    return np.where(a[:, 0] < 0, np.uint32(0), packed).astype(np.uint32)
