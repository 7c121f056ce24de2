"""Seeded random configurations against the oracle (B200 required).

The fixed parity tests hold most options apart; each case here draws them
together: SH degree 0-3 and the iteration (so some bands may still be off),
tile size 8/16/32, splat-batch depth 64/128/256, tile cull on or off, 1 to
16 views of independent sizes that are not multiples of the tile, a scene
with fine and coarse splats, a few huge ones, and a few placed between each
of two cameras and its near plane or behind it.  Every view's records,
per-tile lists, pixels and fixed-point gradients are compared, then one
batched step's parameters, SH and Adam moments -- all bit for bit."""
import numpy as np
import pytest

from oracle import oracle as O
from splat_b200 import scene
from test_gpu_parity import assert_bits, check_view_against_oracle, gpu_raster, make, oracle_adam, oracle_cam, \
    oracle_opts

pytestmark = pytest.mark.gpu


def random_case(seed):
    rng = np.random.default_rng(1000 + seed)
    deg = int(rng.integers(0, 4))
    tile = (8, 16, 32)[seed % 3]           # every (tile, depth, cull) combination appears
    depth = (64, 128, 256)[(seed // 3) % 3]
    cull = (seed // 9) % 2 if seed < 18 else seed % 2
    V = int(rng.integers(1, 17))
    n = int(rng.integers(500, 5000))
    params, sh = scene.surface_scene(n, seed=1000 + seed, sh_deg=deg,
                                     log_scale=(float(rng.uniform(-5.0, -2.5)), float(rng.uniform(0.3, 1.0))),
                                     fine_frac=float(rng.uniform(0.0, 0.3)))
    ring = float(rng.uniform(3.0, 5.0))
    phase = float(rng.uniform(0.0, 6.28))
    cams = []
    for k in range(V):
        w, h = int(rng.integers(40, 260)), int(rng.integers(30, 200))
        cams.append(scene.ring_cameras(V, ring, 0.5, w, h, phase=phase)[k])
    P = params.reshape(-1, 16)
    k = max(2, n // 100)
    idx = rng.choice(n, 3 * k, replace=False)
    P[idx[:k], 3:6] = rng.uniform(-1.2, -0.2, (k, 3))  # huge splats
    # splats just in front of and behind two of the cameras
    for j, c in enumerate(cams[:2]):
        R = np.asarray(c["R"], np.float64).reshape(3, 3)
        eye = -R.T @ np.asarray(c["t"], np.float64)
        fwd = R[2]
        sel = idx[k + j * k: k + (j + 1) * k]
        d = rng.uniform(-0.5, 0.5, sel.size)
        P[sel, 0:3] = eye + np.outer(d, fwd) + rng.normal(0, 0.05, (sel.size, 3))
    rgbs = [scene.uniform_target(c["w"], c["h"], seed=2000 + seed * 20 + v) for v, c in enumerate(cams)]
    opts = dict(shDeg=deg, tile=tile, batchDepth=depth, tileCull=cull, maxBatch=V)
    it0 = int(rng.integers(0, 3500))
    return P.reshape(-1), sh, cams, rgbs, opts, V, n, deg, it0


@pytest.mark.parametrize("seed", range(24))
def test_random_configuration_bitexact(seed):
    params, sh, cams, rgbs, opts, V, n, deg, it0 = random_case(seed)
    K = (deg + 1) ** 2 - 1
    t, targets, metas = make(params, sh, cams, rgbs, opts, radius=2.0)
    t.iter = it0
    o = oracle_opts(opts)
    # a raster pass before any step sees every SH band, as setup() leaves the
    # cameras (trainer.js:367); the step then applies the band ramp
    # (one degree per 1000 iterations, trainer.js:409-412)
    gpu_raster(t, list(range(V)), 3)
    for v in range(V):
        check_view_against_oracle(t, o, oracle_cam(metas[v], v, V, deg), params, sh, targets, n, view=v)
    act = min(deg, it0 // 1000)
    p, s = params.copy(), sh.copy()
    m = np.zeros(n * 16, np.float32)
    vv = np.zeros(n * 16, np.float32)
    sm = np.zeros(n * 3 * K, np.float32)
    sv = np.zeros(n * 3 * K, np.float32)
    t.stepBatch(list(range(V)))
    O.step(o, [oracle_cam(metas[v], v, V, act) for v in range(V)], oracle_adam(t, it0 + 1, 2.0), p, s, targets,
           m, vv, sm, sv, n)
    g = t.readGaussians()
    tag = f"seed {seed}: SH {deg}, tile {opts['tile']}, depth {opts['batchDepth']}, cull {opts['tileCull']}, {V} views"
    assert_bits(g["data"], p, f"params after a step ({tag})")
    gm, gv, gsm, gsv = t.readMoments()
    assert_bits(gm, m, f"Adam m ({tag})")
    assert_bits(gv, vv, f"Adam v ({tag})")
    if K:
        assert_bits(g["sh"], s, f"SH after a step ({tag})")
        assert_bits(gsm, sm, f"SH-Adam m ({tag})")
        assert_bits(gsv, sv, f"SH-Adam v ({tag})")
