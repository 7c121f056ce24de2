"""Host logic of the GSTrainer mirror, without a device.

A fake library stands in for libsplat_b200.so, so these run on the CPU.
They cover the parts the reference keeps on the host: the rand() camera
pick with the holdout/excluded skip (trainer.js:400-406), the camera-pose
Adam of _applyCamGrads (trainer.js:476-537) with its every-25-iterations
trigger (trainer.js:467-469), readLoss (trainer.js:615-631), and the eval
passes' PSNR and test-time pose refinement (trainer.js:542-612).  Each is
checked against a statement-for-statement transcription of the
JavaScript."""
import copy
import math

import numpy as np
import pytest

import rigs
from splat_b200 import native as N
from splat_b200 import trainer as T


class FakeLib:
    """The entry points the host logic calls, recording what it sends."""

    def __init__(self, iter_=0, horizon=60000, stats=(0, 0, 0, 0), pixels=0, cam_grads=None):
        self.iter, self.horizon, self.stats, self.pixels = iter_, horizon, list(stats), pixels
        self.cam_grads = cam_grads
        self.cameras = {}
        self.steps = []

    def gs_get_state(self, h, ref):
        s = ref._obj
        s.iter, s.horizon, s.pixelsSeen = self.iter, self.horizon, self.pixels
        return 0

    def gs_step(self, h, ci):
        self.steps.append(ci)
        self.iter += 1
        return 0

    def gs_read_cam_grads(self, h, p, reset):
        for k, v in enumerate(self.cam_grads):
            p[k] = int(v)
        return 0

    def gs_set_camera(self, h, i, ref):
        s = ref._obj
        self.cameras[i] = dict(R=list(s.R), t=list(s.t), f=s.f, g=s.g, b=s.b)
        return 0

    def gs_read_stats(self, h, st):
        for k in range(4):
            st[k] = self.stats[k]
        self.pixels = 0
        return 0

    def gs_last_error(self, h):
        return b"fake"


def bare_trainer(fake, monkeypatch, ncams=5, opts=None, radius=2.0):
    monkeypatch.setattr(N, "lib", lambda: fake)
    t = T.GSTrainer.__new__(T.GSTrainer)
    t._h = None
    t.opts = dict(opts or {})
    t.holdout, t.excluded, t.lastCam = -1, set(), 0
    t.entryOverflowTiles = 0
    t.rand = rigs.lcg(3)
    rng = np.random.default_rng(1)
    t.camMeta = []
    for i in range(ncams):
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        w, x, y, z = q
        R = [1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y),
             2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x),
             2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]
        t.camMeta.append(dict(R=R, t=list(rng.normal(size=3)), f=300.0 + i, f0=300.0 + i, cx=64.0, cy=48.0,
                              w=128, h=96, imgIdx=i, offset=i * 128 * 96, g=0.0, b=0.0))
    t.sceneRadius = radius
    t.logfScale = 0.0
    t.camStep = 0
    t.camM = np.zeros((ncams + 1) * 8)
    t.camV = np.zeros((ncams + 1) * 8)
    return t


def js_pick(rand, n, holdout, excluded):
    """trainer.js:400-406."""
    ci = int(rand() * n) | 0
    for _ in range(16):
        bad = ci == holdout or ci in excluded
        if not bad:
            break
        ci = (ci + 1) % n
    return ci


def test_pick_skips_the_holdout_and_excluded_cameras(monkeypatch):
    fake = FakeLib()
    t = bare_trainer(fake, monkeypatch, ncams=6)
    t.holdout, t.excluded = 2, {3, 5}
    ref = rigs.lcg(3)
    want = [js_pick(ref, 6, 2, {3, 5}) for _ in range(200)]
    for _ in range(200):
        t.stepOnce()
    assert fake.steps == want
    assert not set(want) & {2, 3, 5} and set(want) == {0, 1, 4}
    assert t.lastCam == want[-1]


def test_pick_gives_up_after_sixteen_tries(monkeypatch):
    """With every camera excluded the reference stops after 16 tries."""
    fake = FakeLib()
    t = bare_trainer(fake, monkeypatch, ncams=4)
    t.excluded = {0, 1, 2, 3}
    ref = rigs.lcg(3)
    want = [js_pick(ref, 4, -1, {0, 1, 2, 3}) for _ in range(20)]
    for _ in range(20):
        t.stepOnce()
    assert fake.steps == want


def js_rodrigues(w):
    th = math.sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2])
    if th < 1e-12:
        return [1, 0, 0, 0, 1, 0, 0, 0, 1]
    k = [w[0] / th, w[1] / th, w[2] / th]
    c, s = math.cos(th), math.sin(th)
    v = 1 - c
    return [c + k[0] * k[0] * v, k[0] * k[1] * v - k[2] * s, k[0] * k[2] * v + k[1] * s,
            k[1] * k[0] * v + k[2] * s, c + k[1] * k[1] * v, k[1] * k[2] * v - k[0] * s,
            k[2] * k[0] * v - k[1] * s, k[2] * k[1] * v + k[0] * s, c + k[2] * k[2] * v]


def js_m3mul(A, B):
    return [sum(A[i * 3 + k] * B[k * 3 + j] for k in range(3)) for i in range(3) for j in range(3)]


def js_apply_cam_grads(st, g, it, horizon, radius, holdout, expComp):
    """trainer.js:476-537 on a plain state dict (camMeta, camM, camV, camStep, logfScale)."""
    st["camStep"] += 1
    t = st["camStep"]
    decay = math.pow(0.02, min(1, it / (0.75 * horizon)))
    rotLr, trnLr, focLr = 2e-4 * decay, 2e-4 * radius * decay, 1e-4 * decay
    b1, b2, eps = 0.9, 0.99, 1e-15

    def step(row, slot, lr):
        j = row * 8 + slot
        grad = g[j] / 64
        st["camM"][j] = b1 * st["camM"][j] + (1 - b1) * grad
        st["camV"][j] = b2 * st["camV"][j] + (1 - b2) * grad * grad
        mh = st["camM"][j] / (1 - math.pow(b1, t))
        vh = st["camV"][j] / (1 - math.pow(b2, t))
        return lr * mh / (math.sqrt(vh) + eps)
    expLr = 5e-3
    metas = st["camMeta"]
    for r in range(1, len(metas)):
        if r == holdout:
            continue
        meta = metas[r]
        dw = [-step(r, 0, rotLr), -step(r, 1, rotLr), -step(r, 2, rotLr)]
        meta["R"] = js_m3mul(js_rodrigues(dw), meta["R"])
        meta["t"] = [meta["t"][0] - step(r, 3, trnLr), meta["t"][1] - step(r, 4, trnLr),
                     meta["t"][2] - step(r, 5, trnLr)]
        if expComp:
            meta["g"] = max(-0.1, min(0.1, (meta["g"] or 0) - step(r, 6, expLr)))
            meta["b"] = max(-0.05, min(0.05, (meta["b"] or 0) - step(r, 7, expLr)))
    nr = len(metas)
    st["logfScale"] = max(-0.3, min(0.3, st["logfScale"] - step(nr, 0, focLr)))
    for m in metas:
        m["f"] = m["f0"] * math.exp(st["logfScale"])


@pytest.mark.parametrize("expComp", [False, True])
def test_camera_gradients_follow_the_reference(monkeypatch, expComp):
    """camOpt: every 25th iteration past 1500 the pose/exposure/focal Adam
    step runs; camera 0 stays pinned and the holdout is skipped; every camera
    record is re-sent with the new focal."""
    ncams = 5
    rng = np.random.default_rng(7)
    grads = rng.integers(-4000, 4000, (ncams + 1) * 8)
    fake = FakeLib(iter_=1523, cam_grads=grads)
    t = bare_trainer(fake, monkeypatch, ncams=ncams, opts=dict(camOpt=True, expComp=expComp))
    t.holdout = 3
    start = copy.deepcopy(t.camMeta)
    st = dict(camMeta=copy.deepcopy(t.camMeta), camM=np.zeros((ncams + 1) * 8), camV=np.zeros((ncams + 1) * 8),
              camStep=0, logfScale=0.0)
    applied = []
    for _ in range(60):           # iterations 1524 .. 1583: applies at 1525, 1550, 1575
        t.stepOnce()
        if fake.iter > 1500 and fake.iter % 25 == 0:
            js_apply_cam_grads(st, grads, fake.iter, 60000, 2.0, 3, expComp)
            applied.append(fake.iter)
    assert applied == [1525, 1550, 1575] and t.camStep == 3
    for i, (m, w) in enumerate(zip(t.camMeta, st["camMeta"])):
        for key in ("R", "t", "f", "g", "b"):
            assert np.array_equal(np.asarray(m[key], np.float64), np.asarray(w[key], np.float64)), (i, key)
        sent = fake.cameras[i]
        assert sent["f"] == np.float32(w["f"])
        assert np.array_equal(np.asarray(sent["R"], np.float32), np.asarray(w["R"], np.float32))
    assert t.logfScale == st["logfScale"] != 0.0
    assert t.camMeta[0]["R"] == st["camMeta"][0]["R"]            # camera 0 pinned
    moved = [not np.array_equal(m["t"], m0["t"]) for m, m0 in zip(t.camMeta, start)]
    assert moved == [False, True, True, False, True]             # 0 pinned, 3 the holdout
    assert (t.camMeta[1]["g"] != 0.0) == expComp


def test_camera_gradients_wait_for_camopt(monkeypatch):
    fake = FakeLib(iter_=1549, cam_grads=np.ones(6 * 8))
    t = bare_trainer(fake, monkeypatch, ncams=5)
    t.stepOnce()
    assert fake.iter == 1550 and t.camStep == 0 and not fake.cameras


def test_read_loss_follows_the_reference(monkeypatch):
    """v / 16 / (validPx * 3), None when no pixel was seen or none was valid;
    stats[3] (budget-dropped tiles) accumulates into entryOverflowTiles."""
    fake = FakeLib(stats=(123456, 99, 2000, 2), pixels=4096)
    t = bare_trainer(fake, monkeypatch)
    assert t.readLoss() == 123456 / 16 / (2000 * 3)
    assert t.entryOverflowTiles == 2
    assert t.readLoss() is None                  # pixelsSeen was reset by the read
    assert t.entryOverflowTiles == 4
    fake.pixels = 10
    fake.stats = [5, 0, 0, 0]
    assert t.readLoss() is None                  # no valid pixel


def pose_response(R, t, g, b, nr, ci):
    """A smooth stand-in for the device: stats and camera gradients as
    functions of the pose the pass renders (float32 R and t, as the camera
    record carries them)."""
    R = np.asarray(R, np.float32).astype(np.float64)
    t = np.asarray(t, np.float32).astype(np.float64)
    cg = np.zeros(nr * 8, np.int64)
    for k in range(8):
        cg[ci * 8 + k] = int(round(3000 * math.sin(1.3 * k + R[k % 9] + 2 * t[k % 3] + 3 * g + 5 * b)))
    v = int(4e6 * (1.5 + math.sin(R.sum() + t.sum() + g - b)))
    return [v, 0, 5000, 0], cg


class EvalLib(FakeLib):
    def __init__(self, metas):
        super().__init__()
        self.metas = metas
        self.seen = []

    def gs_eval_pass(self, h, ci, cam, st, cgp):
        if cam is None:
            m = self.metas[ci]
            R, t, g, b = m["R"], m["t"], m["g"], m["b"]
        else:
            s = cam._obj
            R, t, g, b = list(s.R), list(s.t), s.g, s.b
        self.seen.append((list(np.float32(R)), list(np.float32(t)), g, b))
        stats, cg = pose_response(R, t, g, b, len(self.metas) + 1, ci)
        for k in range(4):
            st[k] = stats[k]
        for k, x in enumerate(cg):
            cgp[k] = int(x)
        return 0


def js_psnr(stats):
    """_evalPass (trainer.js:564-572)."""
    mse = stats[0] / 16 / (max(1, stats[2]) * 3)
    return -10 * math.log10(mse) if mse > 0 else math.inf


def js_eval_refined(meta, ci, nr, steps, radius, expComp):
    """evalCamPsnrRefined (trainer.js:584-612) against pose_response."""
    R, t, g, b = list(meta["R"]), list(meta["t"]), 0.0, 0.0
    m, v = [0.0] * 8, [0.0] * 8
    b1, b2, eps = 0.9, 0.99, 1e-15
    rotLr, trnLr, expLr = 3e-4, 3e-4 * radius, 5e-3
    for s in range(1, steps + 1):
        _, cg = pose_response(R, t, g, b, nr, ci)
        upd = [0.0] * 8
        for k in range(8):
            grad = cg[ci * 8 + k] / 64
            m[k] = b1 * m[k] + (1 - b1) * grad
            v[k] = b2 * v[k] + (1 - b2) * grad * grad
            mh = m[k] / (1 - math.pow(b1, s))
            vh = v[k] / (1 - math.pow(b2, s))
            upd[k] = (rotLr if k < 3 else (trnLr if k < 6 else expLr)) * mh / (math.sqrt(vh) + eps)
        R = js_m3mul(js_rodrigues([-upd[0], -upd[1], -upd[2]]), R)
        t = [t[0] - upd[3], t[1] - upd[4], t[2] - upd[5]]
        if expComp:
            g = max(-0.1, min(0.1, g - upd[6]))
            b = max(-0.05, min(0.05, b - upd[7]))
    stats, _ = pose_response(R, t, g, b, nr, ci)
    return js_psnr(stats), (R, t, g, b)


def test_eval_psnr_follows_the_reference(monkeypatch):
    t = bare_trainer(FakeLib(), monkeypatch, ncams=4)
    lib = EvalLib(t.camMeta)
    monkeypatch.setattr(N, "lib", lambda: lib)
    for ci in range(4):
        stats, _ = pose_response(t.camMeta[ci]["R"], t.camMeta[ci]["t"], 0.0, 0.0, 5, ci)
        assert t.evalCamPsnr(ci) == js_psnr(stats)
    assert js_psnr([0, 0, 0, 0]) == math.inf
    def no_valid_pixel(h, ci, cam, st, cg):
        for k, x in enumerate([96, 0, 0, 0]):
            st[k] = x
        return 0
    lib.gs_eval_pass = no_valid_pixel
    assert t.evalCamPsnr(1) == -10 * math.log10(96 / 16 / 3)     # validPx 0 counts as 1


@pytest.mark.parametrize("expComp", [False, True])
def test_eval_refined_pose_follows_the_reference(monkeypatch, expComp):
    """Test-time pose refinement of one camera: the Adam loop over the
    pass's camera gradients, then the PSNR at the refined pose."""
    t = bare_trainer(FakeLib(), monkeypatch, ncams=4, opts=dict(expComp=expComp), radius=1.7)
    lib = EvalLib(t.camMeta)
    monkeypatch.setattr(N, "lib", lambda: lib)
    ci, steps = 2, 30
    got = t.evalCamPsnrRefined(ci, steps)
    want, (R, tt, g, b) = js_eval_refined(t.camMeta[ci], ci, 5, steps, 1.7, expComp)
    assert len(lib.seen) == steps + 1
    assert got == want
    last = lib.seen[-1]
    assert last[0] == list(np.float32(R)) and last[1] == list(np.float32(tt))
    assert (last[2], last[3]) == (g, b) and ((g, b) != (0.0, 0.0)) == expComp


def so3_log(R):
    """Rotation -> axis-angle (restated for the round trip below)."""
    c = max(-1.0, min(1.0, (R[0] + R[4] + R[8] - 1) / 2))
    th = math.acos(c)
    if th < 1e-12:
        return [0.0, 0.0, 0.0]
    k = th / (2 * math.sin(th))
    return [k * (R[7] - R[5]), k * (R[2] - R[6]), k * (R[3] - R[1])]


def test_rodrigues_properties_of_the_reference_tests():
    """tests/unit/test_geometry.mjs:41-49 for the mirror's rodrigues: the
    log-map round trip within 1e-10 and det R = 1 within 1e-12; plus
    orthonormality and the identity below 1e-12 rad."""
    w = [0.3, -0.7, 0.2]
    R = T.rodrigues(w)
    assert max(abs(a - b) for a, b in zip(w, so3_log(R))) < 1e-10
    M = np.asarray(R, np.float64).reshape(3, 3)
    assert abs(np.linalg.det(M) - 1) < 1e-12
    assert np.abs(M @ M.T - np.eye(3)).max() < 1e-12
    assert T.rodrigues([1e-13, 0.0, 0.0]) == [1.0, 0, 0, 0, 1.0, 0, 0, 0, 1.0]
    assert np.allclose(np.asarray(T.m3mul(R, T.rodrigues([-0.3, 0.7, -0.2]))).reshape(3, 3), np.eye(3), atol=1e-12)
