"""refine()'s edge cases against the oracle (B200 required).

trainer.js:666-794: fewer than 16 donors returns early with nothing moved;
with no dead splats only growth spawns; growth stops at the grow limit, at
the buffer's capacity, and after growUntil (0.75 of the horizon by default).
Each case runs one step (so moments are live), then refine with the same
rng draws on the device and in the oracle, and compares the counts and
every parameter, SH coefficient and moment bit for bit."""
import numpy as np
import pytest

from oracle import oracle as O
import rigs
from splat_b200 import scene
from test_gpu_parity import assert_bits, make

pytestmark = pytest.mark.gpu

CASES = ["few_donors", "no_dead", "grow_limit", "past_grow_until", "at_cap"]


@pytest.mark.parametrize("case", CASES)
def test_refine_edge_case_bitexact(case):
    n = 3000
    params, sh = scene.uniform_scene(n, seed=40 + CASES.index(case), sh_deg=2)
    P = params.reshape(-1, 16)
    rng = np.random.default_rng(50 + CASES.index(case))
    if case == "few_donors":
        P[:, 13] = -6.0
        P[rng.choice(n, 10, replace=False), 13] = 3.0      # 10 donors (< 16)
    elif case == "no_dead":
        P[:, 13] = rng.normal(2.0, 0.5, n)                 # nothing below sigmoid 0.02
    else:
        P[:, 13] = rng.normal(-1.0, 3.0, n)                # dead splats and donors
    params = P.reshape(-1)
    cap = n if case == "at_cap" else 2 * n
    R, tt = scene.look_at_pose([0.0, 0.0, -3.0], [0.0, 0.0, 0.0])
    cams = [dict(R=R, t=tt, f=150.0, cx=64.0, cy=64.0, w=128, h=128)]
    t, _, _ = make(params, sh, cams, [scene.uniform_target(128, 128, seed=3)], dict(shDeg=2, maxSplats=cap),
                   radius=1.0)
    t.iter = 50000 if case == "past_grow_until" else 2000
    growLimit = n + 137 if case == "grow_limit" else 0
    t.growLimit = growLimit
    t.stepBatch([0])
    g = t.readGaussians()
    m, v, sm, sv = t.readMoments()
    assert t.cap == cap
    K = 8
    op = np.zeros(cap * 16, np.float32); op[:n * 16] = g["data"]
    om = np.zeros(cap * 16, np.float32); om[:n * 16] = m
    ov = np.zeros(cap * 16, np.float32); ov[:n * 16] = v
    osh = np.zeros(cap * 3 * K, np.float32); osh[:n * 3 * K] = g["sh"]
    osm = np.zeros(cap * 3 * K, np.float32); osm[:n * 3 * K] = sm
    osv = np.zeros(cap * 3 * K, np.float32); osv[:n * 3 * K] = sv
    r_cpu = O.refine(n, cap, op, om, ov, osh, osm, osv, K, rigs.lcg(77), t.iter, 0.75 * 60000,
                     growLimit=growLimit)
    r_gpu = t.refine(rigs.lcg(77))
    assert (r_gpu["moved"], r_gpu["grown"], r_gpu["n"]) == (r_cpu["moved"], r_cpu["grown"], r_cpu["n"])
    if case == "few_donors":
        assert r_cpu["early"] and r_gpu["moved"] == 0 and r_gpu["n"] == n
    elif case == "no_dead":
        assert r_gpu["moved"] == 0 and r_gpu["grown"] > 0
    elif case == "grow_limit":
        assert r_gpu["grown"] == 137 and r_gpu["moved"] > 0
    else:                                                   # past growUntil, at capacity: relocation only
        assert r_gpu["grown"] == 0 and r_gpu["moved"] > 0
    n2 = r_gpu["n"]
    g2 = t.readGaussians()
    m2, v2, sm2, sv2 = t.readMoments()
    assert_bits(g2["data"], op[:n2 * 16], f"params after refine ({case})")
    assert_bits(g2["sh"], osh[:n2 * 3 * K], f"SH after refine ({case})")
    assert_bits(m2, om[:n2 * 16], f"m after refine ({case})")
    assert_bits(v2, ov[:n2 * 16], f"v after refine ({case})")
    assert_bits(sm2, osm[:n2 * 3 * K], f"SH m after refine ({case})")
    assert_bits(sv2, osv[:n2 * 3 * K], f"SH v after refine ({case})")
