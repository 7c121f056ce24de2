"""Target ingestion: undistortFrames (src/session.js:44-80) and the RGBA8
target packing of GSTrainer.setup (src/gs/trainer.js:115-139).

CPU: the numpy oracle against a line-by-line transcription of the
JavaScript loops (Python floats are IEEE doubles, as JavaScript numbers).
GPU: gs_undistort_frames and the device packing against the oracle, bit for
bit."""
import math
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path[:0] = [ROOT, os.path.join(ROOT, "splat.js_b200")]

from oracle import oracle as O  # noqa: E402


def js_undistort(frames, recon):
    """session.js:44-80, statement for statement."""
    k1, k2 = recon["k1"], recon["k2"]
    if abs(k1) < 0.01 and abs(k2) < 0.01:
        return False, [np.asarray(im["rgb"], np.float32) for im in frames]
    out = []
    for im in frames:
        f = recon["fFeat"] * (im["tw"] / im["fw"])
        cx, cy = im["tw"] / 2, im["th"] / 2
        src = [float(v) for v in np.asarray(im["rgb"], np.float32)]
        dst = np.zeros(len(src), np.float32)
        for y in range(im["th"]):
            for x in range(im["tw"]):
                xp, yp = (x + 0.5 - cx) / f, (y + 0.5 - cy) / f
                r2 = xp * xp + yp * yp
                D = 1 + k1 * r2 + k2 * r2 * r2
                rx = f * xp * D + cx - 0.5
                ry = f * yp * D + cy - 0.5
                o = (y * im["tw"] + x) * 3
                if rx < 0 or ry < 0 or rx > im["tw"] - 1.001 or ry > im["th"] - 1.001:
                    dst[o] = dst[o + 1] = dst[o + 2] = -1
                    continue
                x0, y0 = int(rx), int(ry)
                fx, fy = rx - x0, ry - y0
                i00 = (y0 * im["tw"] + x0) * 3
                i01 = i00 + 3
                i10 = i00 + im["tw"] * 3
                i11 = i10 + 3
                for c in range(3):
                    dst[o + c] = np.float32(src[i00 + c] * (1 - fx) * (1 - fy) + src[i01 + c] * fx * (1 - fy) +
                                            src[i10 + c] * (1 - fx) * fy + src[i11 + c] * fx * fy)
        out.append(dst)
    return True, out


def js_pack(rgb):
    """trainer.js:127-136 for one image (min(255, Math.round(255 v)), low byte)."""
    a = np.asarray(rgb, np.float32).reshape(-1, 3)
    out = np.zeros(len(a), np.uint32)

    def r255(v):
        return min(255, math.floor(float(v) * 255 + 0.5)) & 0xFF

    for p, (r, g, b) in enumerate(a):
        out[p] = 0 if r < 0 else (255 << 24) | (r255(b) << 16) | (r255(g) << 8) | r255(r)
    return out


def frames(seed=0, sizes=((13, 9, 17.0), (24, 16, 24.0), (7, 11, 5.5))):
    rng = np.random.default_rng(seed)
    return [dict(tw=w, th=h, fw=fw, rgb=rng.random(3 * w * h, dtype=np.float32)) for w, h, fw in sizes]


RECONS = [dict(k1=0.2, k2=-0.05, fFeat=14.0), dict(k1=-0.3, k2=0.0, fFeat=20.0), dict(k1=0.0, k2=0.04, fFeat=9.0)]


@pytest.mark.parametrize("recon", RECONS)
def test_undistort_oracle_matches_the_javascript_loop(recon):
    fr = frames()
    did, want = js_undistort(fr, recon)
    got_did, got = O.undistort_frames(fr, recon)
    assert did and got_did
    for a, b in zip(got, want):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    if recon["k1"] > 0:  # pincushion: corners sample outside the frame (the sentinel path)
        assert any((w == -1).any() for w in want)


def test_undistort_below_the_noise_floor_is_a_no_op():
    fr = frames()
    did, got = O.undistort_frames(fr, dict(k1=0.009, k2=-0.009, fFeat=10.0))
    assert not did
    for a, im in zip(got, fr):
        assert np.array_equal(a, im["rgb"])


def test_pack_oracle_matches_the_javascript_loop():
    rng = np.random.default_rng(3)
    rgb = rng.random(3 * 500, dtype=np.float32)
    rgb[::7] = -1.0                                   # invalid sentinels (red channel)
    rgb[1::11] = np.float32(0.5 / 255)                # rounding boundary
    rgb[2::13] = np.float32(1.2)                      # above 1: capped at 255
    assert np.array_equal(O.pack_rgba8(rgb), js_pack(rgb))


@pytest.mark.gpu
@pytest.mark.parametrize("recon", RECONS)
def test_gpu_undistort_is_bitexact(recon):
    from splat_b200.session import undistort_frames
    fr = frames(seed=1, sizes=((13, 9, 17.0), (64, 48, 80.0), (7, 11, 5.5), (1, 1, 1.0)))
    _, want = O.undistort_frames(fr, recon)
    assert undistort_frames(fr, recon)
    for im, w in zip(fr, want):
        assert np.array_equal(im["rgb"].view(np.uint32), w.view(np.uint32))


@pytest.mark.gpu
def test_gpu_undistort_below_the_noise_floor_changes_nothing():
    from splat_b200.session import undistort_frames
    fr = frames(seed=2)
    before = [im["rgb"].copy() for im in fr]
    assert not undistort_frames(fr, dict(k1=0.0, k2=0.005, fFeat=10.0))
    for im, b in zip(fr, before):
        assert np.array_equal(im["rgb"], b)


@pytest.mark.gpu
def test_gpu_target_packing_is_bitexact():
    import ctypes as C

    from splat_b200 import native as N, scene
    from splat_b200.session import undistort_frames
    from splat_b200.trainer import GSTrainer
    params, sh = scene.uniform_scene(200, seed=0, sh_deg=1)
    fr = frames(seed=4, sizes=((40, 24, 40.0), (17, 33, 20.0)))
    undistort_frames(fr, dict(k1=0.25, k2=0.0, fFeat=36.0))      # adds -1 sentinels
    fr[0]["rgb"][5::9] = np.float32(0.5 / 255)
    fr[1]["rgb"][4::10] = np.float32(1.5)
    R, t = scene.look_at_pose([0.0, 0.0, -3.0], [0.0, 0.0, 0.0])
    cams = [dict(R=R, t=t, f=30.0, cx=20.0, cy=12.0, w=40, h=24, imgIdx=0),
            dict(R=R, t=t, f=30.0, cx=8.5, cy=16.5, w=17, h=33, imgIdx=1),
            dict(R=R, t=t, f=30.0, cx=20.0, cy=12.0, w=40, h=24, imgIdx=0)]
    images = [dict(tw=im["tw"], th=im["th"], rgb=im["rgb"]) for im in fr]
    tr = GSTrainer.create(dict(shDeg=1))
    tr.setup(dict(data=params, n=200, sh=sh), cams, images, 40, 33, 1.0)
    total = sum(im["tw"] * im["th"] for im in (images[0], images[1], images[0]))
    got = np.zeros(total, np.uint32)
    N.check(N.lib().gs_debug_targets(tr._h, got.ctypes.data_as(C.POINTER(C.c_uint32)), total), tr._h)
    want = np.concatenate([O.pack_rgba8(images[c["imgIdx"]]["rgb"]) for c in cams])
    assert np.array_equal(got, want)
    assert (want == 0).any() and (want != 0).any()
