"""Regenerate the oracle's regression fixtures for the gradcheck rig.

The reference stores no outputs for its trainer (it runs only under
WebGPU), so these fixtures are the oracle's own results, not the
reference's: they pin the oracle's arithmetic against later edits.  The
rig is gradcheck.js's (160 splats, 64x64, LCG seed 123456789, SH seed
424242, strict cutoffs) at SH degree 3.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "splat.js_b200"), os.path.dirname(HERE)]

from oracle import oracle as O  # noqa: E402
import rigs  # noqa: E402
from splat_b200 import scene  # noqa: E402

OUT = os.path.join(HERE, "rig_sh3.npz")


def rig_outputs():
    """FP32 gradients, stats and image of one training pass on the rig, and
    the parameters after one Adam step."""
    n, deg = 160, 3
    K = O.sh_rest(deg)
    params = rigs.gradcheck_params(n)
    sh, _ = rigs.gradcheck_sh(n, K)
    targets, _ = scene.pack_targets([dict(tw=64, th=64, rgb=rigs.gradcheck_rgb())], [dict(imgIdx=0)])
    o = O.opts(shDeg=deg, **rigs.STRICT)
    c = O.cam([1, 0, 0, 0, 1, 0, 0, 0, 1], [0, 0, 0], 60.0, 32.0, 32.0, 64, 64, activeSh=float(deg))
    z, zs = np.zeros(n * 16, np.float32), np.zeros(n * 3 * K, np.float32)
    stats = np.zeros(4, np.uint32)
    r = O.step(o, [c], O.adam_hp([0] * 16, 1, -10, 0), params.copy(), sh.copy(), targets, z.copy(), z.copy(),
               zs.copy(), zs.copy(), n, stats=stats, do_adam=False, want_image=True)
    lr = [float(np.float32(x)) for x in [3e-4] * 3 + [5e-3] * 3 + [1e-3] * 4 + [1.5e-2] * 3 + [2.5e-2, 0, 0]]
    hp = O.adam_hp(lr, 1, float(np.float32(np.log(1.5e-4))), float(np.float32(np.log(0.075))))
    p, s = params.copy(), sh.copy()
    O.step(o, [c], hp, p, s, targets, z.copy(), z.copy(), zs.copy(), zs.copy(), n)
    return dict(gradF=r["gradF"], shGrad=r["shGrad"], stats=stats, image=r["img"], params_after=p, sh_after=s)


if __name__ == "__main__":
    np.savez_compressed(OUT, **rig_outputs())
    print("wrote", OUT, os.path.getsize(OUT), "bytes")
