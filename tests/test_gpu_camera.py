"""Camera gradients and the eval passes on the B200 against the CPU oracle,
through the C ABI.

Every training pass of the reference accumulates per-camera gradients into
(ncams + 1) x 8 i32 rows: exposure gain and bias from the render pass's
per-pixel sums (shaders.js:522-524, 614-616), pose and the shared focal
length from the chain pass (shaders.js:835-858).  _applyCamGrads
(trainer.js:476-537) drains them for the camera-pose Adam; the eval passes
(_evalPass, evalCamPsnr, evalCamPsnrRefined: trainer.js:542-612) read the
stats and the drained rows of one extra training-path pass.  Integer sums
commute, so every row is compared bit for bit.
"""
import ctypes as C
import math

import numpy as np
import pytest

import rigs
from oracle import oracle as O
from splat_b200 import native as N
from splat_b200 import scene
from test_gpu_parity import assert_bits, config0, make, oracle_adam, oracle_cam, oracle_opts, rig_setup
from test_host_logic import js_m3mul, js_psnr, js_rodrigues

pytestmark = pytest.mark.gpu


def read_cam_grads(t, reset=False):
    rows = len(t.camMeta) + 1
    g = np.zeros(rows * 8, np.int32)
    N.check(N.lib().gs_read_cam_grads(t._h, N.ptr(g, C.c_int32), 1 if reset else 0), t._h)
    return g


def zero_state(n, K):
    return (np.zeros(n * 16, np.float32), np.zeros(n * 16, np.float32), np.zeros(max(1, n * 3 * K), np.float32),
            np.zeros(max(1, n * 3 * K), np.float32))


def test_rig_camera_gradients_with_exposure():
    """The gradient-check rig with a non-unit exposure (log gain 0.08, bias
    -0.02): one pass, rows 0 (pose + exposure) and 1 (focal)."""
    params, sh, cams, rgbs, opts, n = rig_setup()
    cams[0].update(g=0.08, b=-0.02)
    t, targets, metas = make(params, sh, cams, rgbs, opts)
    t.gradPass(0)
    got = read_cam_grads(t)
    o = oracle_opts(opts)
    K = O.sh_rest(opts["shDeg"])
    gc = np.zeros(16, np.int32)
    m, v, sm, sv = zero_state(n, K)
    O.step(o, [oracle_cam(metas[0], 0, 1, opts["shDeg"])], O.adam_hp([0] * 16, 1, -10, 0), params.copy(),
           sh.copy(), targets, m, v, sm, sv, n, gradCam=gc, do_adam=False)
    assert np.count_nonzero(gc[:8]) >= 6 and gc[8] != 0, gc  # pose, exposure and focal rows move
    assert_bits(got, gc, "camera gradient rows (rig)")


def test_config0_camera_gradients_accumulate_over_steps():
    """Config 0 with exposure (log gain -0.05, bias 0.03): three optimiser
    steps; the rows accumulate across steps until drained, as the reference's
    buffer does between two _applyCamGrads."""
    params, sh, cams, rgbs = config0()
    cams[0].update(g=-0.05, b=0.03)
    n, K = len(params) // 16, 8
    t, targets, metas = make(params, sh, cams, rgbs, dict(shDeg=2), radius=1.0)
    t.iter = 2000
    o = oracle_opts(dict(shDeg=2))
    p, s = params.copy(), sh.copy()
    m, v, sm, sv = zero_state(n, K)
    gc = np.zeros(16, np.int32)
    for k in range(3):
        t.stepBatch([0])
        O.step(o, [oracle_cam(metas[0], 0, 1, 2)], oracle_adam(t, 2001 + k, 1.0), p, s, targets, m, v, sm, sv, n,
               gradCam=gc)
        assert_bits(read_cam_grads(t), gc, f"camera gradient rows after step {k + 1}")
    assert_bits(read_cam_grads(t, reset=True), gc, "rows read with reset")
    assert not read_cam_grads(t).any()


def ring_scene(n=6000, ncams=4, W=160, H=96, seed=3):
    params, sh = scene.surface_scene(n, seed=seed, sh_deg=2, log_scale=(-3.5, 0.5))
    cams = scene.ring_cameras(ncams, 4.0, 0.5, W, H, phase=0.3)
    for k, c in enumerate(cams):
        c.update(g=0.02 * (k - 1), b=0.01 * (2 - k))
    rgbs = [scene.uniform_target(W, H, seed=20 + k) for k in range(ncams)]
    return params, sh, cams, rgbs


def test_plain_steps_camera_rows_follow_the_picked_camera():
    """Plain stepOnce steps with the reference's rand() camera pick over four
    cameras with different exposures: each step adds to its own camera's row
    and to the shared focal row."""
    params, sh, cams, rgbs = ring_scene()
    n, K = len(params) // 16, 8
    t, targets, metas = make(params, sh, cams, rgbs, dict(shDeg=2), radius=2.0)
    t.iter = 2000
    t.rand = rigs.lcg(5)
    o = oracle_opts(dict(shDeg=2))
    p, s = params.copy(), sh.copy()
    m, v, sm, sv = zero_state(n, K)
    gc = np.zeros(5 * 8, np.int32)
    seen = set()
    for k in range(6):
        t.stepOnce()
        ci = t.lastCam
        seen.add(ci)
        O.step(o, [oracle_cam(metas[ci], ci, 4, 2)], oracle_adam(t, 2001 + k, 2.0), p, s, targets, m, v, sm, sv, n,
               gradCam=gc)
        assert_bits(read_cam_grads(t), gc, f"camera gradient rows after plain step {k + 1} (camera {ci})")
    assert len(seen) >= 2
    for ci in range(4):
        assert gc[ci * 8:ci * 8 + 8].any() == (ci in seen)


def test_batched_uneven_step_camera_rows():
    """One batched step over three views of uneven resolution: one row per
    view (camIdx of each view) plus the focal row, bit-exact."""
    n = 6000
    params, sh = scene.surface_scene(n, seed=3, sh_deg=2, log_scale=(-3.5, 0.5))
    res = [(160, 96), (96, 64), (200, 120)]
    cams = [scene.ring_cameras(3, 4.0, 0.5, w, h, phase=0.3)[k] for k, (w, h) in enumerate(res)]
    for k, c in enumerate(cams):
        c.update(g=0.03 * k, b=-0.01 * k)
    rgbs = [scene.uniform_target(w, h, seed=10 + k) for k, (w, h) in enumerate(res)]
    t, targets, metas = make(params, sh, cams, rgbs, dict(shDeg=2, maxBatch=4), radius=2.0)
    t.iter = 2000
    o = oracle_opts(dict(shDeg=2))
    K = 8
    m, vv, sm, sv = zero_state(n, K)
    p, s = params.copy(), sh.copy()
    gc = np.zeros(4 * 8, np.int32)
    t.stepBatch([0, 1, 2])
    O.step(o, [oracle_cam(metas[v], v, 3, 2) for v in range(3)], oracle_adam(t, 2001, 2.0), p, s, targets, m, vv,
           sm, sv, n, gradCam=gc)
    for v in range(3):
        assert gc[v * 8:v * 8 + 8].any()
    assert_bits(read_cam_grads(t), gc, "camera gradient rows of an uneven batched step")


def eval_oracle(o, meta, ci, ncams, activeSh, params, sh, targets, n, gc, row=None, override=None):
    """One eval pass of the oracle: stats reset before, no Adam, camera
    gradients added to gc."""
    mm = dict(meta)
    if override:
        mm.update(override)
    c = oracle_cam(mm, ci if row is None else row, ncams, activeSh)
    stats = np.zeros(4, np.uint32)
    m, v, sm, sv = zero_state(n, O.sh_rest(o.shDeg))
    O.step(o, [c], O.adam_hp([0] * 16, 1, -10, 0), params.copy(), sh.copy(), targets, m, v, sm, sv, n, stats=stats,
           gradCam=gc, do_adam=False)
    return stats


def test_eval_pass_stats_and_drained_rows():
    """_evalPass without and with a pose override, after two training steps
    at iteration 500 (SH degree ramped to 0 for the stepped camera):
    - without an override the camera's uniform is reused as the step left it
      (SH degree 0), and the drained rows hold the steps' sums plus the eval
      pass's own;
    - an override builds a fresh uniform (every SH band, row ci);
    - PSNR from the pass's stats; the rows are zero afterwards."""
    params, sh, cams, rgbs = ring_scene()
    n, K = len(params) // 16, 8
    t, targets, metas = make(params, sh, cams, rgbs, dict(shDeg=2), radius=2.0)
    t.iter = 500
    o = oracle_opts(dict(shDeg=2))
    p, s = params.copy(), sh.copy()
    m, v, sm, sv = zero_state(n, K)
    gc = np.zeros(5 * 8, np.int32)
    for k, ci in enumerate([2, 1]):
        t.stepBatch([ci])
        O.step(o, [oracle_cam(metas[ci], ci, 4, 0)], oracle_adam(t, 501 + k, 2.0), p, s, targets, m, v, sm, sv, n,
               gradCam=gc)
    ev = t._evalPass(2)
    want = eval_oracle(o, metas[2], 2, 4, 0, p, s, targets, n, gc)
    assert_bits(ev["camGrad"], gc, "drained rows: two steps + the eval pass")
    assert ev["psnr"] == js_psnr(want)
    assert not read_cam_grads(t).any()
    # a pose / exposure override (rows drained above, so only this pass)
    R = js_m3mul(js_rodrigues([0.01, -0.02, 0.005]), list(metas[3]["R"]))
    tt = [metas[3]["t"][0] + 0.03, metas[3]["t"][1] - 0.01, metas[3]["t"][2]]
    ov = dict(R=R, t=tt, g=0.04, b=-0.02)
    ev = t._evalPass(3, ov)
    gc2 = np.zeros(5 * 8, np.int32)
    want = eval_oracle(o, metas[3], 3, 4, 2, p, s, targets, n, gc2, override=ov)
    assert_bits(ev["camGrad"], gc2, "rows of an override eval pass")
    assert gc2[3 * 8:3 * 8 + 8].any()
    assert ev["psnr"] == js_psnr(want)
    assert t.evalCamPsnr(1) == js_psnr(eval_oracle(o, metas[1], 1, 4, 0, p, s, targets, n,
                                                   np.zeros(40, np.int32)))
    assert t.pixelsSeen == 0


@pytest.mark.parametrize("expComp", [False, True])
def test_eval_refined_pose_matches_oracle(expComp):
    """evalCamPsnrRefined: test-time Adam on one camera's pose (and
    exposure with expComp) over four eval passes, each pass's rows feeding
    the next pose; the final PSNR and every pass's rows equal a transcription
    of the JavaScript loop (trainer.js:584-612) run over oracle passes."""
    params, sh, cams, rgbs = ring_scene(seed=8)
    n = len(params) // 16
    opts = dict(shDeg=2, expComp=expComp)
    t, targets, metas = make(params, sh, cams, rgbs, opts, radius=2.0)
    t.iter = 2000
    o = oracle_opts(dict(shDeg=2))
    ci, steps, radius = 1, 4, 2.0
    got = t.evalCamPsnrRefined(ci, steps)
    meta = metas[ci]
    R, tt, g, b = list(meta["R"]), list(meta["t"]), 0.0, 0.0
    mo, vo = [0.0] * 8, [0.0] * 8
    b1, b2, eps = 0.9, 0.99, 1e-15
    rotLr, trnLr, expLr = 3e-4, 3e-4 * radius, 5e-3
    for st in range(1, steps + 1):
        cg = np.zeros(5 * 8, np.int32)
        eval_oracle(o, meta, ci, 4, 2, params, sh, targets, n, cg, override=dict(R=R, t=tt, g=g, b=b))
        upd = [0.0] * 8
        for k in range(8):
            grad = int(cg[ci * 8 + k]) / 64
            mo[k] = b1 * mo[k] + (1 - b1) * grad
            vo[k] = b2 * vo[k] + (1 - b2) * grad * grad
            mh = mo[k] / (1 - math.pow(b1, st))
            vh = vo[k] / (1 - math.pow(b2, st))
            upd[k] = (rotLr if k < 3 else (trnLr if k < 6 else expLr)) * mh / (math.sqrt(vh) + eps)
        R = js_m3mul(js_rodrigues([-upd[0], -upd[1], -upd[2]]), R)
        tt = [tt[0] - upd[3], tt[1] - upd[4], tt[2] - upd[5]]
        if expComp:
            g = max(-0.1, min(0.1, g - upd[6]))
            b = max(-0.05, min(0.05, b - upd[7]))
    stats = eval_oracle(o, meta, ci, 4, 2, params, sh, targets, n, np.zeros(40, np.int32),
                        override=dict(R=R, t=tt, g=g, b=b))
    assert got == js_psnr(stats)
    assert (g != 0.0) == expComp
    base = t.evalCamPsnr(ci)
    assert math.isfinite(base) and math.isfinite(got)


def test_eval_after_growth_uses_row_zero():
    """After refine() grows the model the reference rebuilds the camera
    uniforms without their index (trainer.js:768): an eval pass without an
    override then sums its pose and exposure gradients into row 0."""
    n = 4000
    params, sh = scene.uniform_scene(n, seed=7, sh_deg=2)
    P = params.reshape(-1, 16)
    P[:, 13] = np.random.default_rng(9).normal(-1.0, 3.0, n)
    params = P.reshape(-1)
    cams = scene.ring_cameras(3, 3.0, 0.3, 128, 96)
    rgbs = [scene.uniform_target(128, 96, seed=40 + k) for k in range(3)]
    t, targets, metas = make(params, sh, cams, rgbs, dict(shDeg=2, maxSplats=8000), radius=1.0)
    t.iter = 2000
    t.stepBatch([2])
    read_cam_grads(t, reset=True)
    r = t.refine(rigs.lcg(4))
    assert r["grown"] > 0
    g = t.readGaussians()
    n2 = g["n"]
    ev = t._evalPass(2)
    gc = np.zeros(4 * 8, np.int32)
    o = oracle_opts(dict(shDeg=2))
    want = eval_oracle(o, metas[2], 2, 3, 2, g["data"], g["sh"], targets, n2, gc, row=0)
    assert gc[0:8].any() and not gc[16:24].any()
    assert_bits(ev["camGrad"], gc, "eval rows after growth (row 0)")
    assert ev["psnr"] == js_psnr(want)
