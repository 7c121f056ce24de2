"""Test inputs: the reference's gradient-check rig and seeded synthetic scenes.

The gradcheck rig restates src/gs/gradcheck.js:93-131 (LCG s = s*1664525 +
1013904223, 160 splats, one 64x64 camera with f=60 and a procedural sin/cos
target) and :192-202 (SH coefficients from seed 424242).
"""
from __future__ import annotations

import math

import numpy as np


def lcg(seed: int):
    """gradcheck.js:98-99: rnd() = (s = s*1664525 + 1013904223 mod 2^32) / 2^32."""
    s = [seed & 0xFFFFFFFF]

    def rnd():
        s[0] = (s[0] * 1664525 + 1013904223) & 0xFFFFFFFF
        return s[0] / 4294967296.0
    return rnd


def xorshift128p(s0: int = 0x2BD3AB5E4C1D2B3B, s1: int = 0x9C3F7A1E0D5B6C47):
    """The library's own refine() generator, restated: xorshift128+ (Vigna
    2017, shifts 23, 18, 5) from the handle's fixed starting state, the 53
    high bits of each output as a double in [0, 1)."""
    M = (1 << 64) - 1
    st = [s0, s1]

    def rnd():
        a, b = st
        out = (a + b) & M
        st[0] = b
        a = (a ^ (a << 23)) & M
        st[1] = a ^ b ^ (a >> 18) ^ (b >> 5)
        return (out >> 11) * 2.0 ** -53
    return rnd


def gradcheck_params(n=160):
    rnd = lcg(123456789)
    data = np.zeros(n * 16, np.float32)
    for i in range(n):
        b = i * 16
        data[b] = (rnd() - 0.5) * 2.4
        data[b + 1] = (rnd() - 0.5) * 2.4
        data[b + 2] = 2 + rnd() * 2
        data[b + 3] = math.log(0.04 + rnd() * 0.1)
        data[b + 4] = math.log(0.04 + rnd() * 0.1)
        data[b + 5] = math.log(0.04 + rnd() * 0.1)
        data[b + 6] = rnd() * 2 - 1
        data[b + 7] = rnd() * 2 - 1
        data[b + 8] = rnd() * 2 - 1
        data[b + 9] = rnd() * 2 - 1
        data[b + 10] = (rnd() - 0.5) * 4
        data[b + 11] = (rnd() - 0.5) * 4
        data[b + 12] = (rnd() - 0.5) * 4
        data[b + 13] = math.log(0.4 / 0.6) + rnd() * 2 - 1
    return data


def gradcheck_rgb(W=64, H=64):
    rgb = np.zeros(W * H * 3, np.float32)
    for y in range(H):
        for x in range(W):
            i = (y * W + x) * 3
            rgb[i] = 0.5 + 0.4 * math.sin(x * 0.31) * math.cos(y * 0.17)
            rgb[i + 1] = 0.5 + 0.4 * math.sin(x * 0.11 + 1) * math.cos(y * 0.23 + 2)
            rgb[i + 2] = 0.5 + 0.4 * math.sin((x + y) * 0.19)
    return rgb


def gradcheck_sh(n, K):
    """gradcheck.js:198-201: sh = (rnd() - 0.5) * 0.5 from seed 424242."""
    rnd = lcg(424242)
    total = n * 3 * K
    return np.array([(rnd() - 0.5) * 0.5 for _ in range(total)], np.float32), rnd


# hBySlot (trainer.js:347-350) with scene radius r
def h_by_slot(r):
    return [r * 2e-3, r * 2e-3, r * 2e-3, 0.02, 0.02, 0.02, 0.02, 0.02, 0.02, 0.02, 0.05, 0.05, 0.05, 0.05, 0, 0]


SLOT_NAMES = ['pos.x', 'pos.y', 'pos.z', 'logSx', 'logSy', 'logSz', 'q.w', 'q.x', 'q.y', 'q.z', 'c.r', 'c.g',
              'c.b', 'opa', 'pad', 'pad']

# the strict cutoffs of the gradient-check rig (gradcheck.js:95, :144-146)
STRICT = dict(eCut=9.0, aMin=1e-4, radClamp=10.0, anisoReg=0.0)
