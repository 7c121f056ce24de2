"""Phase times and roofline fractions of the batched training step on a
synthetic surface scene (one GPU).

    python -m splat_b200.phases --splats 2000000 --sh-degree 3 --fine-frac 0.2 --views 4

Sets up the seeded surface scene (targets rendered from a perturbed copy),
runs warm-up steps, times `--steps` graph-replayed batched steps, then the
per-phase CUDA-event profile (graphs off) and the raster's pixel-entry pair
count P on the reference's full rectangle lists.  Prints one JSON line:
step time, views/s, phase times, and per phase the achieved rate against
the measured peaks (FP32 FFMA for the raster, HBM copy bandwidth for the
rest).  Work units per splat and view: projection 64 + 12K read, 64 + 4
written; chain 232 + 24K; Adam 28 bytes per learnable scalar (14 + 3K per
splat); sort 172 bytes per reference (tile, splat) entry; raster 96 flop
per pair.

--profile-window sets the workload up, warms up three steps, then runs ONE
batched step between cudaProfilerStart/Stop (for ncu --profile-from-start
off) and prints no phase line.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import time

import numpy as np

from . import native as N
from . import scene
from .trainer import GSTrainer

FLOP_PER_PAIR = 96


def parse(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--splats", type=int, default=1_000_000)
    ap.add_argument("--sh-degree", type=int, default=2, choices=[0, 1, 2, 3])
    ap.add_argument("--fine-frac", type=float, default=0.0, help="share of splats at log-scale N(-7, 0.5)")
    ap.add_argument("--views", type=int, default=8, help="views per batched step")
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--cams", type=int, default=24)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--batch-depth", type=int, default=256, choices=[64, 128, 256])
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--hbm-gbs", type=float, default=None,
                    help="HBM copy bandwidth, GB/s (default: MEASURED_PEAKS.json's hbm_gbs at the repository root)")
    ap.add_argument("--profile-window", action="store_true")
    return ap.parse_args(argv)


def measured_hbm_gbs(default: float = 6542.1) -> tuple[float, str]:
    """The measured HBM copy bandwidth of MEASURED_PEAKS.json (repository
    root) when the file is present, else the default (a copy-bandwidth
    measurement on a B200 of the same pool)."""
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", "..", "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "MEASURED_PEAKS.json"
    except (OSError, KeyError, ValueError):
        return default, "default"


def main(argv=None):
    a = parse(argv)
    if a.hbm_gbs is None:
        a.hbm_gbs, hbm_source = measured_hbm_gbs()
    else:
        hbm_source = "--hbm-gbs"
    n, V, W, H = a.splats, a.views, a.width, a.height
    K = scene.sh_rest_coefs(a.sh_degree)
    params, sh = scene.surface_scene(n, seed=a.seed, sh_deg=a.sh_degree, log_scale=(-5.0, 0.7),
                                     fine_frac=a.fine_frac)
    cams = scene.ring_cameras(a.cams, 4.0, 0.5, W, H)
    for k, c in enumerate(cams):
        c["imgIdx"] = k
    pp, ps = scene.perturb(params, sh, 0.02, seed=a.seed + 1)
    blank = [dict(tw=W, th=H, rgb=np.zeros(W * H * 3, np.float32)) for _ in cams]
    t = GSTrainer.create(dict(shDeg=a.sh_degree, maxSplats=n, maxBatch=V, batchDepth=a.batch_depth,
                              entriesCap=24 * n))
    t.setup(dict(data=pp, n=n, sh=ps), cams, blank, W, H, 4.0)
    images = [dict(tw=W, th=H, rgb=np.ascontiguousarray(np.clip(t.renderView(c)[..., :3], 0, 1).reshape(-1)))
              for c in cams]
    t.setup(dict(data=params, n=n, sh=sh), cams, images, W, H, 4.0)
    del images, blank
    t.iter = 1000 * a.sh_degree          # every SH band active
    L, h = N.lib(), t._h
    stride = max(1, a.cams // V)

    def batch(k):
        return [(V * k + j * stride) % a.cams for j in range(V)]
    for k in range(3):
        t.stepBatch(batch(k))
    N.check(L.gs_sync(h), h)
    if a.profile_window:
        import torch
        torch.cuda.profiler.start()
        t.stepBatch(batch(3))
        N.check(L.gs_sync(h), h)
        torch.cuda.profiler.stop()
        print(json.dumps({"profile_window": "one batched step", "views": batch(3), "splats": n,
                          "sh_degree": a.sh_degree}))
        return
    t0 = time.perf_counter()
    for k in range(a.steps):
        t.stepBatch(batch(3 + k))
    N.check(L.gs_sync(h), h)
    step_ms = (time.perf_counter() - t0) / a.steps * 1e3
    N.check(L.gs_profile(h, 1), h)
    for k in range(5):
        t.stepBatch(batch(k))
    ms, cnt = (C.c_double * 4)(), (C.c_uint32 * 4)()
    N.check(L.gs_profile_read(h, ms, cnt), h)
    N.check(L.gs_profile(h, 0), h)
    ph = [ms[i] / max(1, cnt[i]) for i in range(4)]
    # pairs and reference entries of one batch on full rectangle lists (tile cull off)
    N.check(L.gs_set_tile_cull(h, 0), h)
    cs = batch(0)
    N.check(L.gs_raster_pass(h, (C.c_uint32 * V)(*cs), V, 3), h)
    tiles = ((W + 15) // 16) * ((H + 15) // 16)
    P = E = 0
    for v in range(V):
        end = np.zeros(W * H, np.uint32)
        N.check(L.gs_debug_pixels(h, v, None, None, N.ptr(end, C.c_uint32)), h)
        P += int(end.astype(np.uint64).sum())
        tc, nE = np.zeros(tiles, np.uint32), C.c_uint64()
        N.check(L.gs_debug_binning(h, v, N.ptr(tc, C.c_uint32), None, None, 0, C.byref(nE)), h)
        E += int(tc.astype(np.uint64).sum())
        N.check(L.gs_debug_gradp(h, v, None, 1), h)
    N.check(L.gs_set_tile_cull(h, 1), h)
    peak = C.c_double()
    N.check(L.gs_probe_fp32_peak(int(t._o.device), C.byref(peak)), None)
    rate = {
        "raster_tflops": P * FLOP_PER_PAIR / (ph[2] * 1e-3) / 1e12,
        "project_gbs": (128 + 12 * K + 4) * n * V / (ph[0] * 1e-3) / 1e9,
        "sort_gbs_equiv": 172 * E / (ph[1] * 1e-3) / 1e9,
        "chain_adam_gbs": ((232 + 24 * K) * n * V + 28 * (14 + 3 * K) * n) / (ph[3] * 1e-3) / 1e9,
    }
    frac = {"raster": rate["raster_tflops"] / peak.value, "project": rate["project_gbs"] / a.hbm_gbs,
            "sort": rate["sort_gbs_equiv"] / a.hbm_gbs, "chain_adam": rate["chain_adam_gbs"] / a.hbm_gbs}
    print(json.dumps(dict(workload=dict(splats=n, sh_degree=a.sh_degree, fine_frac=a.fine_frac, views=V,
                                        resolution=f"{W}x{H}"),
                          step_ms=step_ms, views_per_s=V / step_ms * 1e3,
                          phases_ms=dict(zip(["project_bin", "sort", "raster", "chain_adam"], ph)),
                          pairs=P, reference_entries=E, fp32_peak_tflops=peak.value,
                          hbm_gbs=a.hbm_gbs, hbm_source=hbm_source, rates=rate,
                          roofline_frac=frac)))


if __name__ == "__main__":
    main()
