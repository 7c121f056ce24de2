"""Config 4's training schedule on one GPU, end to end through the public
API: batched steps with MCMC relocation / growth (refine, trainer.js:666-794)
every `--refine-every` steps.

    python -m splat_b200.schedule            # 2M splats, SH 3, 20% fine, 4 x 1080p, 2000 steps

Defaults are config 4: 2,000,000 splats of the seeded surface scene at SH
degree 3 with a fifth of them fine (log-scale N(-7, 0.5)), four 1920x1080
ring views per step (cameras spread over a 24-camera ring, rotating every
step), 2000 steps starting at iteration 3000 (every SH band active), refine
every 100 steps with opacity-weighted clone donors, the library's own
reproducible generator as rng() (--rng lcg: a seeded LCG called from Python
per draw, as a caller-supplied rng is) and 10%
splat headroom (maxSplats = 1.1 n, so growth runs until the headroom is
used and relocation every time).  Targets are the scene rendered from a
perturbed copy.  Prints one JSON line: wall time of the whole schedule
(steps + refines, host work included), steps/s and views/s with refine,
refine count / time / moved / grown, a per-phase CUDA-event profile of five
steps at the end, and the SM clocks sampled over the run.

--profile-window warms up, then runs one refine and one step between
cudaProfilerStart/Stop (for an ncu launch list of both) and prints no
schedule line.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import time

import numpy as np

from . import native as N
from . import scene
from .clocks import ClockSampler
from .trainer import GSTrainer


def lcg(seed: int):
    """rng() for refine: a 32-bit LCG (s = 1664525 s + 1013904223) / 2^32."""
    st = [seed & 0xFFFFFFFF]

    def rnd():
        st[0] = (st[0] * 1664525 + 1013904223) & 0xFFFFFFFF
        return st[0] / 4294967296.0
    return rnd


def parse(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--splats", type=int, default=2_000_000)
    ap.add_argument("--sh-degree", type=int, default=3, choices=[0, 1, 2, 3])
    ap.add_argument("--fine-frac", type=float, default=0.2)
    ap.add_argument("--views", type=int, default=4)
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--cams", type=int, default=24)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--refine-every", type=int, default=100)
    ap.add_argument("--headroom", type=float, default=0.1, help="maxSplats = (1 + headroom) * splats")
    ap.add_argument("--donor-sampling", type=int, default=1, choices=[0, 1])
    ap.add_argument("--batch-depth", type=int, default=256, choices=[64, 128, 256])
    ap.add_argument("--seed", type=int, default=4)
    ap.add_argument("--rng", choices=["own", "lcg"], default="own",
                    help="refine's rng(): the library's own generator (the reference's default is Math.random), "
                         "or a seeded LCG in Python called once per draw")
    ap.add_argument("--profile-window", action="store_true")
    return ap.parse_args(argv)


def main(argv=None):
    a = parse(argv)
    n, V, W, H = a.splats, a.views, a.width, a.height
    cap = int(round(n * (1.0 + a.headroom)))
    params, sh = scene.surface_scene(n, seed=a.seed, sh_deg=a.sh_degree, log_scale=(-5.0, 0.7),
                                     fine_frac=a.fine_frac)
    cams = scene.ring_cameras(a.cams, 4.0, 0.5, W, H)
    for k, c in enumerate(cams):
        c["imgIdx"] = k
    pp, ps = scene.perturb(params, sh, 0.02, seed=a.seed + 1)
    blank = [dict(tw=W, th=H, rgb=np.zeros(W * H * 3, np.float32)) for _ in cams]
    opts = dict(shDeg=a.sh_degree, maxSplats=cap, maxBatch=V, batchDepth=a.batch_depth, entriesCap=24 * cap,
                donorSampling=a.donor_sampling)
    t = GSTrainer.create(opts)
    t.setup(dict(data=pp, n=n, sh=ps), cams, blank, W, H, 4.0)
    images = [dict(tw=W, th=H, rgb=np.ascontiguousarray(np.clip(t.renderView(c)[..., :3], 0, 1).reshape(-1)))
              for c in cams]
    t.setup(dict(data=params, n=n, sh=sh), cams, images, W, H, 4.0)
    del images, blank
    t.iter = 3000
    L, h = N.lib(), t._h
    stride = max(1, a.cams // V)

    def batch(k):
        return [(k + j * stride) % a.cams for j in range(V)]

    rng = lcg(a.seed) if a.rng == "lcg" else None
    if a.profile_window:
        import torch
        for k in range(3):
            t.stepBatch(batch(k))
        t.refine(rng)
        t.stepBatch(batch(3))
        N.check(L.gs_sync(h), h)
        torch.cuda.profiler.start()
        r = t.refine(rng)
        t.stepBatch(batch(4))
        N.check(L.gs_sync(h), h)
        torch.cuda.profiler.stop()
        print(json.dumps({"profile_window": "one refine + one batched step", "refine": r, "n": t.n}))
        return 0

    for k in range(3):                        # warm-up: graph capture of the step shape
        t.stepBatch(batch(k))
    N.check(L.gs_sync(h), h)
    refines, moved, grown, refine_s = 0, 0, 0, 0.0
    with ClockSampler(int(t._o.device)) as clk:
        t0 = time.perf_counter()
        for k in range(a.steps):
            t.stepBatch(batch(k))
            if (k + 1) % a.refine_every == 0:
                r0 = time.perf_counter()
                r = t.refine(rng)                 # synchronises: waits for the steps before it
                refine_s += time.perf_counter() - r0
                refines += 1
                moved += r.get("moved", 0)
                grown += r.get("grown", 0)
        N.check(L.gs_sync(h), h)
        wall = time.perf_counter() - t0
    clocks = clk.summary()
    N.check(L.gs_profile(h, 1), h)
    for k in range(5):
        t.stepBatch(batch(k))
    ms, cnt = (C.c_double * 4)(), (C.c_uint32 * 4)()
    N.check(L.gs_profile_read(h, ms, cnt), h)
    N.check(L.gs_profile(h, 0), h)
    ph = [ms[i] / max(1, cnt[i]) for i in range(4)]
    print(json.dumps(dict(
        workload=dict(splats=n, max_splats=cap, sh_degree=a.sh_degree, fine_frac=a.fine_frac, views_per_step=V,
                      resolution=f"{W}x{H}", steps=a.steps, refine_every=a.refine_every,
                      donor_sampling="opacity-weighted" if a.donor_sampling else "uniform (reference)",
                      iteration_start=3000, rng="library generator" if a.rng == "own" else "Python LCG per draw"),
        wall_s=wall, steps_per_s=a.steps / wall, views_per_s=a.steps * V / wall,
        refines=refines, refine_s=refine_s, refine_ms_each=refine_s / max(1, refines) * 1e3,
        moved=moved, grown=grown, final_splats=t.n,
        phases_ms_per_step=dict(zip(["project_bin", "sort", "raster", "chain_adam"], ph)),
        clocks=clocks)))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
