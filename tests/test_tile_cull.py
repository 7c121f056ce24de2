"""Tile culling (the library's default tile lists) against the reference's
full rectangle lists, on the CPU oracle.

With culling, a (splat, tile) entry is kept only when the exact minimum of
the splat's exponent over the tile's pixel centres, plus FP32 error margins,
passes the rasteriser's cutoffs.  A culled entry must contribute to no pixel,
so images, final transmittance, loss statistics and every gradient have to be
bit-identical to rendering with the full lists, and each culled list has to be
an ordered subsequence of the full one."""
import numpy as np
import pytest

from oracle import oracle as O
import rigs
from splat_b200 import scene


def anisotropic_scene(n, seed, W=256, H=256):
    """Needle- and disc-like splats at every orientation, some tiny."""
    rng = np.random.default_rng(seed)
    P = np.zeros((n, 16), np.float32)
    P[:, 0] = rng.uniform(-1.2, 1.2, n)
    P[:, 1] = rng.uniform(-1.2, 1.2, n)
    P[:, 2] = rng.uniform(-0.8, 0.8, n)
    big = rng.uniform(-2.5, -0.3, n)
    small = rng.uniform(-7.0, -3.5, n)
    mid = np.where(rng.random(n) < 0.5, small, rng.uniform(-3.0, -1.0, n))
    ls = np.stack([big, small, mid], 1)
    for k in range(n):
        rng.shuffle(ls[k])
    P[:, 3:6] = ls
    q = rng.normal(size=(n, 4))
    P[:, 6:10] = q / np.linalg.norm(q, axis=1, keepdims=True)
    P[:, 10:13] = rng.normal(0, 1.5, (n, 3))
    P[:, 13] = rng.uniform(-3.0, 5.0, n)
    R, t = scene.look_at_pose([0.0, 0.0, -3.0], [0.0, 0.0, 0.0])
    cam = dict(R=R, t=t, f=300.0, cx=W / 2, cy=H / 2, w=W, h=H)
    return P.reshape(-1), cam


def render_both(o_kw, params, sh, cam, rgb, n, sh_deg):
    targets, _ = scene.pack_targets([dict(tw=cam["w"], th=cam["h"], rgb=rgb)], [dict(imgIdx=0)])
    c = O.cam(cam["R"], cam["t"], cam["f"], cam["cx"], cam["cy"], cam["w"], cam["h"], activeSh=float(sh_deg))
    out = {}
    for cull in (0, 1):
        o = O.opts(shDeg=sh_deg, tileCull=cull, **o_kw)
        proj = O.project(o, c, params, sh, n)
        bins = O.bin_tiles(o, c, proj, n)
        r = O.render(o, c, proj, bins, targets, n, train=True)
        out[cull] = (bins, r)
    return out


def check_identical(out):
    (b0, r0), (b1, r1) = out[0], out[1]
    for k in ("img", "finalT", "gradP", "stats", "gradCam"):
        assert np.array_equal(r0[k].view(np.uint32), r1[k].view(np.uint32)), k
    np.testing.assert_array_equal(b0["cnt"], b1["cnt"])  # the budget still counts rectangles
    nt = b0["numTiles"]
    for t in range(nt):
        full = b0["ids"][b0["start"][t]:b0["start"][t + 1]]
        kept = b1["ids"][b1["start"][t]:b1["start"][t + 1]]
        # ordered subsequence: walk the full list
        j = 0
        for x in kept:
            while j < full.size and full[j] != x:
                j += 1
            assert j < full.size, f"tile {t}: culled list is not a subsequence"
            j += 1
    return b0["ids"].size, b1["ids"].size


def test_cull_is_exact_on_the_gradcheck_rig():
    n = 160
    params = rigs.gradcheck_params(n)
    sh, _ = rigs.gradcheck_sh(n, O.sh_rest(3))
    cam = dict(R=[1, 0, 0, 0, 1, 0, 0, 0, 1], t=[0, 0, 0], f=60.0, cx=32.0, cy=32.0, w=64, h=64)
    full, kept = check_identical(render_both(rigs.STRICT, params, sh, cam, rigs.gradcheck_rgb(), n, 3))
    assert kept <= full


@pytest.mark.parametrize("seed", [0, 1])
def test_cull_is_exact_on_a_uniform_scene(seed):
    params, sh = scene.uniform_scene(6000, seed=seed, sh_deg=2)
    R, t = scene.look_at_pose([0.0, 0.0, -3.0], [0.0, 0.0, 0.0])
    cam = dict(R=R, t=t, f=300.0, cx=128.0, cy=128.0, w=256, h=256)
    full, kept = check_identical(render_both({}, params, sh, cam, scene.uniform_target(256, 256, seed=seed),
                                             6000, 2))
    assert kept < full


@pytest.mark.parametrize("seed,tile", [(3, 16), (4, 8), (5, 32)])
def test_cull_is_exact_on_needles_and_discs(seed, tile):
    n = 4000
    params, cam = anisotropic_scene(n, seed)
    sh = np.zeros(n * 3 * O.sh_rest(2), np.float32)
    out = render_both(dict(tile=tile), params, sh, cam, scene.uniform_target(256, 256, seed=seed), n, 2)
    full, kept = check_identical(out)
    assert kept < 0.8 * full, (kept, full)
