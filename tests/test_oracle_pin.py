"""Pins the CPU oracle before anything is compared against it.

The reference keeps no golden vectors for the trainer; its own check of the
backward is src/gs/gradcheck.js (central finite differences on a 160-splat
64x64 rig with strict cutoffs, per-slot median relative error < 0.05).  These
tests run that protocol against the oracle: its FP32 gradients (fixed-point
accumulation, as the reference computes them) and its FP64 gradients against
FP64 central differences of the loss.  The canonical exp/log/sin are checked
against libm.
"""
import math
import struct

import numpy as np
import pytest

from oracle import oracle as O
import rigs
from splat_b200 import scene


def ulp_diff(a, b):
    ia = struct.unpack('i', struct.pack('f', a))[0]
    ib = struct.unpack('i', struct.pack('f', b))[0]
    return abs(ia - ib)


def test_canonical_exp_log_sin_accuracy():
    L = O.lib()
    worst = 0
    for x in np.linspace(-20.0, 20.0, 20001, dtype=np.float32):
        ref = np.float32(math.exp(float(x)))
        worst = max(worst, ulp_diff(L.oracle_exp_f32(float(x)), float(ref)))
    assert worst <= 2, worst
    worst = 0
    for x in np.geomspace(1.0001, 1e4, 5001).astype(np.float32):
        ref = np.float32(math.log(float(x)))
        got = L.oracle_log_f32(float(x))
        worst = max(worst, ulp_diff(got, float(ref)))
    assert worst <= 2, worst
    for x in np.linspace(0, 3e7, 1001):
        x = float(np.float32(x))
        assert abs(L.oracle_sin_f64(x) - math.sin(x)) < 1e-12


def rig(sh_deg=2, with_sh=False):
    n = 160
    params = rigs.gradcheck_params(n)
    K = O.sh_rest(sh_deg)
    if with_sh:
        sh, _ = rigs.gradcheck_sh(n, K)
    else:
        sh = np.zeros(n * 3 * K, np.float32)
    rgb = rigs.gradcheck_rgb()
    targets, metas = scene.pack_targets([dict(tw=64, th=64, rgb=rgb)], [dict(imgIdx=0)])
    o = O.opts(shDeg=sh_deg, **rigs.STRICT)
    c = O.cam([1, 0, 0, 0, 1, 0, 0, 0, 1], [0, 0, 0], 60.0, 32.0, 32.0, 64, 64, activeSh=float(sh_deg))
    return o, c, params, sh, targets, n


def fp32_grads(o, c, params, sh, targets, n):
    K = O.sh_rest(o.shDeg)
    z = np.zeros(n * 16, np.float32)
    zs = np.zeros(max(1, n * 3 * K), np.float32)
    hp = O.adam_hp([0] * 16, 1, -10, 0)
    r = O.step(o, [c], hp, params.copy(), sh.copy(), targets, z.copy(), z.copy(), zs.copy(), zs.copy(), n,
               do_adam=False)
    return r["gradF"], r["shGrad"]


def fd_check(o, c, params, sh, targets, n, grad, samples=80, seed=7, use_fixed_h=None):
    """gradcheck.js:307-329 sampling; FD of the FP64 Charbonnier loss."""
    p64 = params.astype(np.float64)
    s64 = sh.astype(np.float64)
    hb = rigs.h_by_slot(1.5)
    rnd = rigs.lcg(seed)
    res = {}
    attempts = 0
    got = 0
    while got < samples and attempts < samples * 8:
        attempts += 1
        j = int(rnd() * n * 16)
        slot = j % 16
        if hb[slot] == 0:
            continue
        if abs(grad[j]) < 0.03 and rnd() < 0.9:
            continue
        h = use_fixed_h or hb[slot]
        orig = p64[j]
        p64[j] = orig + h
        lp = O.eval_f64(o, c, p64, s64, n, targets, grads=False)[0][0]
        p64[j] = orig - h
        lm = O.eval_f64(o, c, p64, s64, n, targets, grads=False)[0][0]
        p64[j] = orig
        fd = (lp - lm) / (2 * h)
        a = float(grad[j])
        den = max(abs(a), abs(fd))
        rel = 0.0 if den < 1e-3 else abs(a - fd) / den
        res.setdefault(rigs.SLOT_NAMES[slot], []).append(rel)
        got += 1
    return {k: float(np.median(v)) for k, v in res.items()}, got


@pytest.mark.parametrize("sh_deg,with_sh", [(2, False), (3, True)])
def test_gradcheck_rig_fp32_vs_fd(sh_deg, with_sh):
    """gradCheckSmall / gradCheckSH protocol: per-slot median relErr < 0.05."""
    o, c, params, sh, targets, n = rig(sh_deg, with_sh)
    gF, sG = fp32_grads(o, c, params, sh, targets, n)
    med, got = fd_check(o, c, params, sh, targets, n, gF)
    assert got >= 60, got
    worst = max(med.values())
    assert worst < 0.05, med


def test_gradcheck_rig_fp64_analytic_vs_fd_tight():
    """FP64 analytic gradients against FP64 central differences, h = 1e-4."""
    o, c, params, sh, targets, n = rig(3, True)
    loss, gF, sG, _ = O.eval_f64(o, c, params.astype(np.float64), sh.astype(np.float64), n, targets)
    med, got = fd_check(o, c, params, sh, targets, n, gF, use_fixed_h=1e-4)
    assert max(med.values()) < 2e-3, med
    # SH coefficients (gradcheck.js:233-251), h = 1e-4
    s64 = sh.astype(np.float64)
    p64 = params.astype(np.float64)
    rnd = rigs.lcg(99)
    errs = []
    for _ in range(40):
        j = int(rnd() * len(s64))
        orig = s64[j]
        s64[j] = orig + 1e-4
        lp = O.eval_f64(o, c, p64, s64, n, targets, grads=False)[0][0]
        s64[j] = orig - 1e-4
        lm = O.eval_f64(o, c, p64, s64, n, targets, grads=False)[0][0]
        s64[j] = orig
        fd = (lp - lm) / 2e-4
        den = max(abs(sG[j]), abs(fd))
        errs.append(0.0 if den < 1e-3 else abs(sG[j] - fd) / den)
    assert np.median(errs) < 2e-3


def test_fp32_gradients_track_fp64():
    """FP32 (fixed-point) gradients against the FP64 host evaluation."""
    o, c, params, sh, targets, n = rig(3, True)
    gF, sG = fp32_grads(o, c, params, sh, targets, n)
    _, g64, s64, _ = O.eval_f64(o, c, params.astype(np.float64), sh.astype(np.float64), n, targets)
    m = np.zeros(16, bool)
    m[:14] = True
    a = gF.reshape(-1, 16)[:, m]
    b = g64.reshape(-1, 16)[:, m]
    # the reference truncates every pixel's contribution to 1/16384 before
    # summing (shaders.js:529-541), so FP32 sits ~1e-3 (norm-wise) from FP64
    rel = np.linalg.norm(a - b) / np.linalg.norm(b)
    assert rel < 5e-3, rel
    rel_sh = np.linalg.norm(sG - s64) / np.linalg.norm(s64)
    assert rel_sh < 5e-3, rel_sh


def test_fp32_gradients_track_quantised_fp64():
    """With the reference's per-pixel truncation applied in double as well,
    the FP64 evaluation leaves only FP32 rounding between the two paths: the
    ~1e-3 gap above is the fixed-point quantisation, not FP32 arithmetic."""
    o, c, params, sh, targets, n = rig(3, True)
    gF, sG = fp32_grads(o, c, params, sh, targets, n)
    a = gF.reshape(-1, 16)[:, :14]
    rel = {}
    for q in (False, True):
        _, g64, s64, _ = O.eval_f64(o, c, params.astype(np.float64), sh.astype(np.float64), n, targets, quantise=q)
        b = g64.reshape(-1, 16)[:, :14]
        rel[q] = (np.linalg.norm(a - b) / np.linalg.norm(b), np.linalg.norm(sG - s64) / np.linalg.norm(s64))
    assert rel[True][0] < 1e-4 and rel[True][1] < 1e-4, rel
    assert rel[True][0] < rel[False][0] / 20 and rel[True][1] < rel[False][1] / 20, rel


@pytest.mark.parametrize("cull", [0, 1])
def test_local_central_differences_equal_whole_image_ones(cull):
    """fd_local (the loss over the tiles a perturbed splat can touch) equals
    the whole-image central difference: the other tiles cancel."""
    o, c, params, sh, targets, n = rig(3, True)
    o.tileCull = cull
    p64, s64 = params.astype(np.float64), sh.astype(np.float64)
    K = O.sh_rest(3)
    ids = [3, 41, 77, 150]
    h = 1e-4
    fd = O.fd_local(o, c, p64, s64, n, targets, ids, h=h)
    rnd = rigs.lcg(5)
    checked = 0
    for r, s in enumerate(ids):
        for k in [0, 1, 2, 3, 5, 6, 8, 10, 12, 13] + [14 + int(rnd() * 3 * K) for _ in range(3)]:
            arr, j = (p64, s * 16 + k) if k < 14 else (s64, s * 3 * K + k - 14)
            orig = arr[j]
            arr[j] = orig + h
            lp = O.eval_f64(o, c, p64, s64, n, targets, grads=False)[0][0]
            arr[j] = orig - h
            lm = O.eval_f64(o, c, p64, s64, n, targets, grads=False)[0][0]
            arr[j] = orig
            whole = (lp - lm) / (2 * h)
            # the whole-image loss (~4e3) is summed in a thread-dependent
            # order: ~1e-12 per sum, ~1e-8 in the difference quotient
            assert abs(fd[r, k] - whole) <= 1e-6, (s, k, fd[r, k], whole)
            checked += 1
    assert checked == 4 * 13
    assert np.isfinite(fd).all() and (np.abs(fd) > 0).sum() > fd.size // 2
