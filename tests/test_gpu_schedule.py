"""Config 4's training pattern over several refine cycles, bit for bit
against the oracle (B200 required).

Config 4 trains 2M splats at SH degree 3 (a fifth of them fine) on four
1080p views per step, with MCMC relocation and growth (refine,
trainer.js:666-794) every 100 steps.  Here the same pattern runs at a
reduced size so the oracle keeps up: 30k splats, four 320x180 ring views,
refine every 4 steps for three cycles (relocation every cycle, growth into
the headroom), and every parameter, Adam moment and SH coefficient is
compared after each cycle, with the caller's rng and with the library's own
generator (refine() without an rng).  The schedule at full size is measured by
``python -m splat_b200.schedule``."""
import numpy as np
import pytest

import rigs
from oracle import oracle as O
from splat_b200 import scene
from test_gpu_parity import assert_bits, make, oracle_adam, oracle_cam, oracle_opts

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("donorSampling,rng", [(0, "caller"), (1, "caller"), (1, "own")])
def test_refine_cycles_bitexact(donorSampling, rng):
    """rng "caller": a seeded LCG passed to refine() (one call per draw);
    "own": refine() without an rng draws from the library's generator, which
    the oracle replays from its restatement."""
    n, cap, K, W, H = 30_000, 42_000, 15, 320, 180
    params, sh = scene.surface_scene(n, seed=14, sh_deg=3, log_scale=(-3.5, 0.6), fine_frac=0.2)
    P0 = params.reshape(-1, 16)
    P0[:, 13] = np.random.default_rng(3).normal(-0.5, 2.5, n)  # dead splats and donors both present
    params = P0.reshape(-1)
    ring = scene.ring_cameras(8, 4.0, 0.5, W, H)
    cams = [ring[k] for k in (0, 2, 4, 6)]
    rgbs = [scene.uniform_target(W, H, seed=60 + k) for k in range(4)]
    opts = dict(shDeg=3, maxSplats=cap, entriesCap=24 * cap, donorSampling=donorSampling)
    t, targets, metas = make(params, sh, cams, rgbs, opts, radius=4.0)
    assert t.cap == cap
    t.iter = 3000
    o = oracle_opts(opts)
    ocams = [oracle_cam(metas[v], v, 4, 3) for v in range(4)]
    P = np.zeros(cap * 16, np.float32)
    P[:n * 16] = params
    S = np.zeros(cap * 3 * K, np.float32)
    S[:n * 3 * K] = sh
    M, V = np.zeros(cap * 16, np.float32), np.zeros(cap * 16, np.float32)
    SM, SV = np.zeros(cap * 3 * K, np.float32), np.zeros(cap * 3 * K, np.float32)
    nn, it = n, 3000
    if rng == "caller":
        rng_gpu, rng_cpu = rigs.lcg(77 + donorSampling), rigs.lcg(77 + donorSampling)
    else:
        rng_gpu, rng_cpu = None, rigs.xorshift128p()
    moved = grown = 0
    for cycle in range(3):
        for _ in range(4):
            t.stepBatch([0, 1, 2, 3])
            it += 1
            O.step(o, ocams, oracle_adam(t, it, 4.0), P, S, targets, M, V, SM, SV, nn)
        r_gpu = t.refine(rng_gpu)
        r_cpu = O.refine(nn, cap, P, M, V, S, SM, SV, K, rng_cpu, it, 0.75 * 60000, donorSampling=donorSampling)
        assert (r_gpu["moved"], r_gpu["grown"], r_gpu["n"]) == (r_cpu["moved"], r_cpu["grown"], r_cpu["n"])
        moved += r_gpu["moved"]
        grown += r_gpu["grown"]
        nn = r_gpu["n"]
        g = t.readGaussians()
        m, v, sm, sv = t.readMoments()
        assert g["n"] == nn
        assert_bits(g["data"], P[:nn * 16], f"params after cycle {cycle + 1}")
        assert_bits(g["sh"], S[:nn * 3 * K], f"SH after cycle {cycle + 1}")
        assert_bits(m, M[:nn * 16], f"m after cycle {cycle + 1}")
        assert_bits(v, V[:nn * 16], f"v after cycle {cycle + 1}")
        assert_bits(sm, SM[:nn * 3 * K], f"SH m after cycle {cycle + 1}")
        assert_bits(sv, SV[:nn * 3 * K], f"SH v after cycle {cycle + 1}")
    assert moved > 0 and grown > 0 and nn <= cap
