"""Donor sampling of refine (trainer.js:713-722).

The reference clones a donor drawn uniformly from the donor list
(`donors[(rng() * donors.length) | 0]`).  donorSampling = 1 is the
opacity-weighted option: the same single rng() draw picks the first donor
whose cumulative sigmoid(opacity) exceeds rng() * total.  These CPU tests
check the oracle's picks draw by draw against numpy; the GPU refine is
compared with the oracle bit for bit in test_gpu_parity.py."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path[:0] = [ROOT, os.path.join(ROOT, "splat.js_b200")]

from oracle import oracle as O  # noqa: E402
import rigs  # noqa: E402

N_SPLATS, CAP = 4000, 8000
LOW, HIGH = 0.0, 6.0          # donor opacity logits: sigmoid 0.5 and 0.9975


def population():
    """400 dead splats (sigmoid 0.0025), 32 donors each with its own colour
    logit (slot 10 names the donor a clone copied), the rest in between."""
    P = np.zeros((CAP, 16), np.float32)
    P[:N_SPLATS, 3:6] = -4.0
    P[:N_SPLATS, 6] = 1.0
    P[:N_SPLATS, 13] = -1.0                       # sigmoid 0.27: neither dead nor donor
    dead = np.arange(0, 4000, 10)
    P[dead, 13] = -6.0
    donors = np.arange(7, 7 + 32 * 20, 20)
    assert not np.intersect1d(donors, dead).size
    P[donors, 13] = np.where(np.arange(32) % 2 == 0, LOW, HIGH)
    P[donors, 10] = np.arange(32, dtype=np.float32) + 1.0
    return P, dead, donors


def run(donorSampling, seed=11):
    P, dead, donors = population()
    draws = []
    base = rigs.lcg(seed)

    def rng():
        draws.append(base())
        return draws[-1]
    z = np.zeros(CAP * 16, np.float32)
    params = P.reshape(-1).copy()
    out = O.refine(N_SPLATS, CAP, params, z.copy(), z.copy(), z[:1].copy(), z[:1].copy(), z[:1].copy(), 0, rng,
                   50000, 0.0, donorSampling=donorSampling)   # iter past growUntil: relocation only
    return out, params.reshape(-1, 16), dead, donors, draws


@pytest.mark.parametrize("donorSampling", [0, 1])
def test_each_pick_follows_its_draw(donorSampling):
    out, p, dead, donors, draws = run(donorSampling)
    moved = out["moved"]
    assert moved == 200 and out["grown"] == 0 and not out["early"]
    assert len(draws) == 7 * moved               # per relocation: the pick, then three gauss() pairs
    picks = np.asarray(draws[0::7])
    sig = 1.0 / (1.0 + np.exp(-p[donors, 13].astype(np.float64)))
    if donorSampling:
        cdf = np.cumsum(sig)
        want = np.minimum(np.searchsorted(cdf, picks * cdf[-1], side="right"), len(donors) - 1)
    else:
        want = (picks * len(donors)).astype(np.int64)
    got = p[dead[:moved], 10].astype(np.int64) - 1
    assert np.array_equal(got, want)


def test_weighted_sampling_prefers_opaque_donors():
    frac = {}
    for mode in (0, 1):
        out, p, dead, donors, _ = run(mode, seed=5)
        got = p[dead[:out["moved"]], 10].astype(np.int64) - 1
        frac[mode] = float(np.mean(got % 2 == 1))     # odd donors carry the HIGH opacity
    w_hi = 1.0 / (1.0 + np.exp(-HIGH))
    expect = w_hi / (w_hi + 0.5)
    assert abs(frac[0] - 0.5) < 0.12
    assert abs(frac[1] - expect) < 0.12 and frac[1] > frac[0]
