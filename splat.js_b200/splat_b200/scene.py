"""Host-side inputs of the training step: target packing, cameras, scenes.

* ``pack_targets`` restates GSTrainer.setup's RGBA8 packing
  (src/gs/trainer.js:115-139).
* ``look_at_pose`` restates src/synthetic.js:276-292 (world y points down).
* ``uniform_scene`` / ``surface_scene`` are the seeded synthetic scenes the
  benchmark uses in place of captured data (numpy ``default_rng(seed)``).
"""
from __future__ import annotations

import math

import numpy as np

STRIDE = 16
SH_C0 = 0.28209479177387814  # src/io/ply.js:9


def sh_rest_coefs(deg: int) -> int:
    """K = (deg+1)^2 - 1 rest coefficients per channel (shaders.js:65)."""
    return (deg + 1) * (deg + 1) - 1 if deg > 0 else 0


def js_round255(v: np.ndarray) -> np.ndarray:
    """Math.min(255, Math.round(v * 255)) on f32 inputs promoted to double."""
    x = np.floor(v.astype(np.float64) * 255.0 + 0.5)
    return np.minimum(255, x).astype(np.int64)


def pack_targets(images, cams):
    """Pack every camera's target image as RGBA8 (alpha 0 = invalid pixel).

    images: list of dicts {tw, th, rgb (float32, 3*tw*th; r < 0 marks an
    invalid pixel)}; cams: list of dicts with ``imgIdx``.  Returns (packed
    uint32 array, per-camera metadata with w/h/offset in pixels)."""
    total = 0
    metas = []
    for c in cams:
        im = images[c["imgIdx"]]
        meta = dict(c)
        meta.update(w=int(im["tw"]), h=int(im["th"]), offset=total)
        total += int(im["tw"]) * int(im["th"])
        metas.append(meta)
    out = np.zeros(max(total, 4), np.uint32)
    for meta in metas:
        rgb = np.asarray(images[meta["imgIdx"]]["rgb"], np.float32).reshape(-1, 3)
        npx = meta["w"] * meta["h"]
        rgb = rgb[:npx]
        r, g, b = js_round255(rgb[:, 0]), js_round255(rgb[:, 1]), js_round255(rgb[:, 2])
        packed = (255 << 24) | ((b & 0xFF) << 16) | ((g & 0xFF) << 8) | (r & 0xFF)
        packed = np.where(rgb[:, 0] < 0, 0, packed)
        out[meta["offset"]:meta["offset"] + npx] = packed.astype(np.uint32)
    return out, metas


def look_at_pose(eye, center):
    """World-to-camera (R row-major, t) looking from eye at center, y down."""
    eye = np.asarray(eye, np.float64)
    center = np.asarray(center, np.float64)
    up = np.array([0.0, -1.0, 0.0])

    def norm(a):
        return a / math.sqrt(float(a @ a))
    zc = norm(center - eye)
    xc = norm(np.cross(zc, up))
    yc = np.cross(zc, xc)
    R = np.array([xc, yc, zc])
    t = -(R @ eye)
    return R.reshape(-1).tolist(), t.tolist()


def ring_cameras(count, radius, height, W, H, f=None, phase=0.0):
    """Cameras on a ring of `radius` at world height `height` (y up is -y),
    aimed at the origin.  f defaults to 1.171875 W (a 46.2 deg horizontal
    field of view, the same as f=300 at W=256)."""
    if f is None:
        f = 1.171875 * W
    cams = []
    for i in range(count):
        a = phase + 2.0 * math.pi * i / count
        eye = [radius * math.cos(a), -height, radius * math.sin(a)]
        R, t = look_at_pose(eye, [0.0, 0.0, 0.0])
        cams.append(dict(R=R, t=t, f=float(f), cx=W / 2.0, cy=H / 2.0, w=int(W), h=int(H)))
    return cams


def _unit_quats(rng, n):
    q = rng.normal(0.0, 1.0, (n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    return q


def _colour_logits(rng, n):
    """SH DC ~ N(0, 0.3) mapped to the trainer's colour logit: the trainer's
    DC colour is sigmoid(logit) = 0.5 + C0 f_dc (ply.js:77-79 inverts it)."""
    fdc = rng.normal(0.0, 0.3, (n, 3))
    c = np.clip(0.5 + SH_C0 * fdc, 1e-4, 1 - 1e-4)
    return np.log(c / (1 - c))


def _assemble(pos, log_scale, quat, logits, opa_logit):
    n = pos.shape[0]
    P = np.zeros((n, STRIDE), np.float32)
    P[:, 0:3] = pos
    P[:, 3:6] = log_scale
    P[:, 6:10] = quat
    P[:, 10:13] = logits
    P[:, 13] = opa_logit
    return P.reshape(-1)


def uniform_scene(n, seed=0, sh_deg=2):
    """20k-style scene: means U[-1,1]^3, log-scales N(-4, 0.5), random unit
    quaternions, opacity logits N(0,1), SH DC N(0,0.3), rest N(0,0.05)."""
    rng = np.random.default_rng(seed)
    pos = rng.uniform(-1.0, 1.0, (n, 3))
    ls = rng.normal(-4.0, 0.5, (n, 3))
    q = _unit_quats(rng, n)
    logits = _colour_logits(rng, n)
    op = rng.normal(0.0, 1.0, n)
    K = sh_rest_coefs(sh_deg)
    sh = rng.normal(0.0, 0.05, n * 3 * K).astype(np.float32)
    return _assemble(pos, ls, q, logits, op), sh


def surface_scene(n, seed=0, sh_deg=2, log_scale=(-5.0, 0.7), fine_frac=0.0, fine_log_scale=(-7.0, 0.5)):
    """Surface scene: 60% on the planes x=0, y=0, z=0 (20% each, U[-2,2]^2),
    30% on the unit sphere, 10% on a radius-20 shell.  A `fine_frac` share
    of splats takes log-scales from `fine_log_scale` (dense fine detail)."""
    rng = np.random.default_rng(seed)
    n_pl = int(round(0.6 * n))
    n_sp = int(round(0.3 * n))
    n_sh = n - n_pl - n_sp
    pos = np.zeros((n, 3))
    per = [n_pl // 3, n_pl // 3, n_pl - 2 * (n_pl // 3)]
    o = 0
    for axis, cnt in enumerate(per):
        uv = rng.uniform(-2.0, 2.0, (cnt, 2))
        other = [a for a in range(3) if a != axis]
        pos[o:o + cnt, other[0]] = uv[:, 0]
        pos[o:o + cnt, other[1]] = uv[:, 1]
        pos[o:o + cnt, axis] = 0.0
        o += cnt
    d = rng.normal(0.0, 1.0, (n_sp, 3))
    pos[o:o + n_sp] = d / np.linalg.norm(d, axis=1, keepdims=True)
    o += n_sp
    d = rng.normal(0.0, 1.0, (n_sh, 3))
    pos[o:o + n_sh] = 20.0 * d / np.linalg.norm(d, axis=1, keepdims=True)
    perm = rng.permutation(n)
    pos = pos[perm]
    ls = rng.normal(log_scale[0], log_scale[1], (n, 3))
    if fine_frac > 0:
        nf = int(round(fine_frac * n))
        idx = rng.choice(n, nf, replace=False)
        ls[idx] = rng.normal(fine_log_scale[0], fine_log_scale[1], (nf, 3))
    q = _unit_quats(rng, n)
    logits = _colour_logits(rng, n)
    op = rng.normal(0.0, 1.0, n)
    K = sh_rest_coefs(sh_deg)
    sh = rng.normal(0.0, 0.05, n * 3 * K).astype(np.float32)
    return _assemble(pos, ls, q, logits, op), sh


def perturb(params, sh, sigma=0.02, seed=1):
    """Copy of the scene with N(0, sigma) added to every parameter (pads kept 0)."""
    rng = np.random.default_rng(seed)
    P = params.reshape(-1, STRIDE).astype(np.float64).copy()
    P[:, :14] += rng.normal(0.0, sigma, (P.shape[0], 14))
    S = sh.astype(np.float64) + rng.normal(0.0, sigma, sh.shape)
    return P.astype(np.float32).reshape(-1), S.astype(np.float32)


def uniform_target(W, H, seed=0):
    """A uniform-random RGB image in [0,1] (float32, 3*W*H)."""
    rng = np.random.default_rng(seed)
    return rng.uniform(0.0, 1.0, W * H * 3).astype(np.float32)
