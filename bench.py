"""Training-step benchmark: train views/s at 1M splats, 1920x1080, SH degree 2.

Workload (the metric's configuration): a seeded 1,000,000-splat surface
scene (60% on three planes, 30% on a unit sphere, 10% on a radius-20 shell;
log-scales N(-5, 0.7)), SH degree 2 with all bands active (iteration counter
started at 2000), 24 ring cameras at 1920x1080 (f = 1.171875 W), targets
rendered from a perturbed copy of the scene (N(0, 0.02) on every
parameter).  A step is one optimiser step: the batched step renders and
backpropagates 8 views in one graph-captured launch sequence; the plain
step is the reference's stepOnce (one view).  `value` is the batched
step's views/s (device-resident inputs); the plain step's views/s is
reported beside it.  The working set (params, Adam moments, SH, entries)
is several GB, larger than the 126 MB L2, so no flush is needed.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

--impl reference times the CPU restatement of the reference's step (the
oracle, all host threads): each step one whole view of the workload
(cameras 0-7 in turn), plus one step on a single thread.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (ROOT, os.path.join(ROOT, "splat.js_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

from splat_b200.clocks import ClockSampler  # noqa: E402

METRIC = "train views/s @1M splats 1080p, batched vs plain step, 1 B200, grads within 1e-4"
FLOP_PER_PAIR = 26 + 70   # raster forward + backward per evaluated pixel-entry pair (FFMA = 2)
# DRAM bytes (read + write) of one raster launch over an 8-view batch at the
# default workload: one ncu capture of a 2-view launch of the same scene
# (two 1080p ring views; 311.98 MB read + 95.85 MB written), scaled by the
# view count (not measured live)
RASTER_DRAM_BYTES_8VIEW = (311.978240e6 + 95.846656e6) * 4


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--splats", type=int, default=1_000_000)
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--cams", type=int, default=24)
    ap.add_argument("--batch-depth", type=int, default=64)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--side-paths", action="store_true",
                    help="measure the paths either side of the training step instead (the eval pass, PLY export "
                         "with the opacity bake, frame undistortion), each through the C ABI beside the CPU "
                         "restatement on the same inputs; prints one JSON line")
    ap.add_argument("--profile-window", action="store_true",
                    help="set up the workload, warm up, then run ONE batched step (tile 16, depth 256) between "
                         "cudaProfilerStart/Stop for ncu --profile-from-start off; prints no bench line")
    return ap.parse_args()


def workload(args):
    from splat_b200 import scene
    params, sh = scene.surface_scene(args.splats, seed=args.seed, sh_deg=2, log_scale=(-5.0, 0.7))
    cams = scene.ring_cameras(args.cams, 4.0, 0.5, args.width, args.height)
    for k, c in enumerate(cams):
        c["imgIdx"] = k
    return params, sh, cams


def config_dict(args, extra=None):
    d = {"workload": f"{args.splats // 1000}k-splat surface scene, SH deg 2, {args.width}x{args.height}, "
                     f"batch of {args.batch} views per step",
         "splats": args.splats, "resolution": f"{args.width}x{args.height}", "views_per_batched_step": args.batch,
         "cameras": args.cams, "sh_degree": 2, "tile": 16, "l2": "working set > L2 (no flush needed)",
         "iteration_start": 2000}
    if extra:
        d.update(extra)
    return d


# ---------------------------------------------------------------------------
# CPU side (oracle): baseline sample and the --impl reference arm
# ---------------------------------------------------------------------------
CPU_CAMS = 8  # the CPU arm trains cameras 0..7 in turn: the views of the GPU arm's first batch


def cpu_adam_hp(iter_after, radius, horizon=60000):
    """The trainer's Adam uniforms after `iter_after` increments
    (trainer.js:319-342, 417-424): position lr 3e-4 r decayed to 1% at 75% of
    the horizon, scale 5e-3, rotation 1e-3, colour 1.5e-2, opacity 2.5e-2;
    log-scale clamps [log(1e-4 r), log(0.05 r)]."""
    from oracle import oracle as O
    pos = 3e-4 * radius * math.pow(0.01, min(1.0, iter_after / (0.75 * horizon)))
    lr = [pos, pos, pos, 5e-3, 5e-3, 5e-3, 1e-3, 1e-3, 1e-3, 1e-3, 1.5e-2, 1.5e-2, 1.5e-2, 2.5e-2, 0, 0]
    lr = [float(np.float32(x)) for x in lr]
    return O.adam_hp(lr, iter_after, float(np.float32(math.log(radius * 1e-4))),
                     float(np.float32(math.log(radius * 0.05))))


def cpu_setup(args, params, sh, cams, ncams):
    """Inputs of the CPU arm: targets of cameras 0..ncams-1 rendered forward
    by the oracle from the same perturbed copy the GPU arm renders its targets
    from, packed RGBA8 as setup does (trainer.js:115-139)."""
    from oracle import oracle as O
    from splat_b200 import scene
    n = len(params) // 16
    pp, ps = scene.perturb(params, sh, 0.02, seed=args.seed + 1)
    o = O.opts(shDeg=2, entriesCap=max(12_000_000, n * 24))
    sizes = [c["w"] * c["h"] for c in cams[:ncams]]
    offsets = [int(x) for x in np.concatenate([[0], np.cumsum(sizes)[:-1]])]
    targets = np.zeros(sum(sizes), np.uint32)
    for ci in range(ncams):
        c = cams[ci]
        oc = O.cam(c["R"], c["t"], c["f"], c["cx"], c["cy"], c["w"], c["h"], activeSh=2.0, train=0)
        proj = O.project(o, oc, pp, ps, n)
        bins = O.bin_tiles(o, oc, proj, n, cap=max(1, n * 40))
        img = O.render(o, oc, proj, bins, targets, n, train=False)["img"].reshape(-1, 4)
        q = np.minimum(255, np.floor(np.clip(img[:, :3], 0, 1).astype(np.float64) * 255 + 0.5)).astype(np.uint32)
        targets[offsets[ci]:offsets[ci] + sizes[ci]] = (255 << 24) | (q[:, 2] << 16) | (q[:, 1] << 8) | q[:, 0]
    ocams = [O.cam(c["R"], c["t"], c["f"], c["cx"], c["cy"], c["w"], c["h"], offset=offsets[ci], camIdx=ci,
                   ncams=len(cams), activeSh=2.0) for ci, c in enumerate(cams[:ncams])]
    return o, ocams, targets


class CpuTrainer:
    """The oracle's plain training step (project, bin, per-tile sort, raster
    forward + loss + backward, chain, Adam + SH-Adam) over whole views, on
    its own copy of the model, starting at iteration 2000 like the GPU arm."""

    def __init__(self, o, ocams, targets, params, sh, radius=4.0):
        self.o, self.ocams, self.targets, self.radius = o, ocams, targets, radius
        self.p, self.s = params.copy(), sh.copy()
        self.m, self.v = np.zeros_like(self.p), np.zeros_like(self.p)
        self.sm, self.sv = np.zeros_like(self.s), np.zeros_like(self.s)
        self.iter = 2000

    def step(self, ci):
        """One optimiser step on camera ci; returns its wall time in seconds."""
        from oracle import oracle as O
        self.iter += 1
        hp = cpu_adam_hp(self.iter, self.radius)
        t0 = time.perf_counter()
        O.step(self.o, [self.ocams[ci]], hp, self.p, self.s, self.targets, self.m, self.v, self.sm, self.sv,
               len(self.p) // 16)
        return time.perf_counter() - t0


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle import oracle as O
    O.build()
    params, sh, cams = workload(args)
    ncams = min(CPU_CAMS, len(cams))
    o, ocams, targets = cpu_setup(args, params, sh, cams, ncams)
    cores = O.set_threads(0)
    tr = CpuTrainer(o, ocams, targets, params, sh)
    times = []
    for k in range(args.warmup + args.steps):
        dt = tr.step(k % ncams)
        if k >= args.warmup:
            times.append(dt)
    sec = sum(times) / max(1, len(times))
    v = 1.0 / sec
    # one more whole-view step on a single host thread, beside the all-core figure
    O.set_threads(1)
    one = tr.step((args.warmup + args.steps) % ncams)
    O.set_threads(cores)
    sample = (f"each step: one whole {args.width}x{args.height} view (cameras 0-{ncams - 1} in turn), the "
              f"oracle's plain training step over all {args.splats} splats; {cores} threads")
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "views/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded surface scene)",
            "config": config_dict(args, {"parallelism": "host threads", "views_per_step": 1,
                                         "cameras_trained": f"0-{ncams - 1} in turn"}),
            "cpu_baseline": {"value": v, "unit": "views/s", "cores": cores, "kind": "port", "sample": sample},
            "single_thread": {"value": 1.0 / one, "unit": "views/s", "cores": 1, "ms_per_view": one * 1e3},
            "nproc": os.cpu_count(),
            "e2e": {"value": v, "unit": "views/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# Rank plumbing (one process per GPU; replicas, no data-path collective)
# ---------------------------------------------------------------------------
def init_ranks(backend="nccl", timeout_s=300):
    """(rank, world, local rank, torch.distributed or None) from the launcher's
    environment; a process group only when WORLD_SIZE > 1."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return rank, world, local, dist


def max_over_ranks(ms, dist, device):
    """The slowest rank's time: every rank returns the same value."""
    if not dist:
        return ms
    import torch
    tt = torch.tensor([float(ms)], device=device, dtype=torch.float64)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    return float(tt.item())


def job_rate(units_per_step, steps, world, ms):
    """Whole-job throughput: units every rank processed / the slowest rank's time."""
    return units_per_step * steps * world / (ms / 1e3)


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def run_ours(args):
    import torch
    rank, world, local, dist = init_ranks("nccl")
    torch.cuda.set_device(local)

    from splat_b200 import native as N
    from splat_b200 import scene
    from splat_b200.trainer import GSTrainer

    params, sh, cams = workload(args)
    n = args.splats
    B = args.batch
    # config-3 style uneven batch, appended as cameras 24..31
    uneven_res = [(640, 360), (960, 540), (1280, 720), (1280, 720), (1600, 900), (1920, 1080), (1920, 1080),
                  (1920, 1080)]
    extra = []
    for k, (w, h) in enumerate(uneven_res):
        cc = scene.ring_cameras(len(uneven_res), 4.0, 0.5, w, h, phase=0.13)[k]
        cc["imgIdx"] = len(cams) + k
        extra.append(cc)
    allcams = cams + extra
    opts = dict(shDeg=2, maxSplats=n, maxBatch=max(B, len(uneven_res)), batchDepth=args.batch_depth,
                device=local, persistent=1, useGraphs=1)
    # targets: render the perturbed scene with the same library, then train the clean one
    pp, ps = scene.perturb(params, sh, 0.02, seed=args.seed + 1)
    blank = [dict(tw=c["w"], th=c["h"], rgb=np.zeros(c["w"] * c["h"] * 3, np.float32)) for c in allcams]
    t = GSTrainer.create(opts)
    t.setup(dict(data=pp, n=n, sh=ps), allcams, blank, args.width, args.height, 4.0)
    images = []
    for c in allcams:
        img = t.renderView(c)
        images.append(dict(tw=c["w"], th=c["h"], rgb=np.ascontiguousarray(np.clip(img[..., :3], 0, 1).reshape(-1))))
    t.setup(dict(data=params, n=n, sh=sh), allcams, images, args.width, args.height, 4.0)
    del images
    if args.profile_window:
        t.iter = 2000
        t.setRasterConfig(16, 256)
        cs = list(range(B))
        for _ in range(3):
            t.stepBatch(cs)
        N.check(N.lib().gs_sync(t._h), t._h)
        torch.cuda.profiler.start()
        t.stepBatch(cs)
        N.check(N.lib().gs_sync(t._h), t._h)
        torch.cuda.profiler.stop()
        print(json.dumps({"profile_window": "one batched step", "views": cs, "entries": t._state().lastEntries}))
        return 0
    stream = torch.cuda.Stream(device=local)
    N.check(N.lib().gs_set_stream(t._h, C.c_void_p(stream.cuda_stream)), t._h)
    L = N.lib()
    h = t._h

    def batch_cams(k):
        return [(k * B + j) % len(cams) for j in range(B)]

    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()

    def timed(fn, steps, views_per_step):
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for k in range(steps):
            fn(k)
        e1.record(stream)
        # wait in the library (ctypes drops the GIL), so the clock sampler's
        # thread keeps sampling while the device works
        N.check(L.gs_sync(h), h)
        barrier()
        ms = max_over_ranks(e0.elapsed_time(e1), dist, f"cuda:{local}")
        return ms, job_rate(views_per_step, steps, world, ms)

    arrs = {}

    def step_batched(k):
        cs = batch_cams(k)
        key = tuple(cs)
        if key not in arrs:
            arrs[key] = (C.c_uint32 * len(cs))(*cs)
        N.check(L.gs_step_batch(h, arrs[key], len(cs)), h)

    def step_plain(k):
        N.check(L.gs_step(h, k % len(cams)), h)

    uneven_idx = (C.c_uint32 * len(extra))(*range(len(cams), len(allcams)))

    def step_uneven(k):
        N.check(L.gs_step_batch(h, uneven_idx, len(extra)), h)

    p_host = np.ascontiguousarray(params, np.float32)
    s_host = np.ascontiguousarray(sh, np.float32)

    def restore():
        # every timed segment starts from the same trainer state: the
        # generator's parameters and SH, zero Adam moments (as setup leaves
        # them) and iteration 2000 (the steps train the model, and the
        # splats' footprints, hence the work, drift as they do)
        N.check(L.gs_write_gaussians(h, p_host.ctypes.data_as(C.POINTER(C.c_float)),
                                     s_host.ctypes.data_as(C.POINTER(C.c_float)), n), h)
        N.check(L.gs_reset_moments(h), h)
        t.iter = 2000

    restore()
    # ---- autotuner: tile size x splat-batch depth on the first batch ----
    tune_tile, tune_depth, tune_table = t.autotune(batch_cams(0), reps=2)
    # ---- plain per-view step (the reference's stepOnce) ----
    restore()
    for k in range(args.warmup):
        step_plain(k)
    plain_ms, plain_vps = timed(step_plain, args.steps, 1)
    # ---- batched step (headline) ----
    restore()
    for k in range(args.warmup):
        step_batched(k)
    with ClockSampler(local) as clk:
        batch_ms, batch_vps = timed(step_batched, args.steps, B)
    clocks = clk.summary()
    st_b = N.GsState()
    L.gs_get_state(h, C.byref(st_b))
    batch_launches = int(st_b.lastLaunches)  # kernels one batched step enqueues
    # ---- uneven-resolution batch (config 3) ----
    restore()
    for k in range(args.warmup):
        step_uneven(k)
    uneven_ms, uneven_vps = timed(step_uneven, args.steps, len(extra))
    # ---- end to end through the public API: per step the camera/Adam records
    # go host->device from pinned memory and the loss statistics come back to
    # pinned host memory (readLoss, a Promise in the reference: the copy is
    # enqueued each step and complete when the timed region's sync returns);
    # the blocking variant (one host sync per step) is reported beside it ----
    st = (C.c_uint32 * 4)()
    st_pinned = torch.zeros((max(args.steps, args.warmup), 4), dtype=torch.int32, pin_memory=True)

    def step_e2e(k):
        step_batched(k)
        N.check(L.gs_read_stats_async(h, C.c_void_p(st_pinned[k].data_ptr())), h)

    def step_e2e_sync(k):
        step_batched(k)
        N.check(L.gs_read_stats(h, st), h)
    restore()
    for k in range(args.warmup):
        step_e2e(k)
    e2e_ms, e2e_vps = timed(step_e2e, args.steps, B)
    N.check(L.gs_sync(h), h)
    restore()
    for k in range(args.warmup):
        step_e2e_sync(k)
    e2e_sync_ms, e2e_sync_vps = timed(step_e2e_sync, args.steps, B)
    # ---- per-phase profile of the batched step (CUDA events on the stream) ----
    prof_steps = min(args.steps, 5)
    restore()
    N.check(L.gs_profile(h, 1), h)
    for k in range(prof_steps):
        step_batched(k)
    ms4 = (C.c_double * 4)()
    cnt4 = (C.c_uint32 * 4)()
    N.check(L.gs_profile_read(h, ms4, cnt4), h)
    N.check(L.gs_profile(h, 0), h)
    phase = {nm: ms4[i] / max(1, cnt4[i]) for i, nm in enumerate(["project_bin", "sort", "raster", "chain_adam"])}
    # pixel-entry pairs of one batch (the raster roofline's work unit): the sum
    # of per-pixel end indices.  The algorithmic count P is taken on the
    # reference's full rectangle tile lists (tile cull off); the culled lists
    # the step actually walks give the executed count beside it.
    def count_pairs(cull):
        N.check(L.gs_set_tile_cull(h, cull), h)
        restore()
        total = 0
        for k in range(prof_steps):
            cs = batch_cams(k)
            arr = (C.c_uint32 * len(cs))(*cs)
            N.check(L.gs_raster_pass(h, arr, len(cs), 3), h)
            for v, ci in enumerate(cs):
                w, hh = allcams[ci]["w"], allcams[ci]["h"]
                end = np.zeros(w * hh, np.uint32)
                N.check(L.gs_debug_pixels(h, v, None, None, N.ptr(end, C.c_uint32)), h)
                total += int(end.astype(np.uint64).sum())
                N.check(L.gs_debug_gradp(h, v, None, 1), h)   # leave no gradients behind
        return total / prof_steps
    pairs_exec = count_pairs(1)
    pairs_per_launch = count_pairs(0)
    N.check(L.gs_set_tile_cull(h, 1), h)
    peak = C.c_double()
    N.check(L.gs_probe_fp32_peak(local, C.byref(peak)), None)
    raster_ms = phase["raster"]
    achieved = pairs_per_launch * FLOP_PER_PAIR / (raster_ms * 1e-3) / 1e12
    state = N.GsState()
    L.gs_get_state(h, C.byref(state))

    line = None
    if rank == 0:
        cpu = None
        if not args.no_cpu_baseline and world == 1:
            cpu = cpu_baseline_line(args, params, sh, cams)
        h2d = int(state.stepUploadBytes)  # view records + Adam parameters, from pinned memory
        line = {"metric": METRIC, "value": batch_vps, "unit": "views/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": batch_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic: seeded surface scene, targets rendered from a perturbed copy",
                "config": config_dict(args, {"parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                                             "graphs": True, "tile": tune_tile, "batch_depth": tune_depth}),
                "autotune_ms_per_pass": {f"{k[0]}x{k[1]}": round(v, 3) for k, v in tune_table.items()},
                "plain_step": {"views_per_s": plain_vps, "ms_per_step": plain_ms / args.steps},
                "batched_vs_plain": batch_vps / plain_vps,
                "uneven_batch": {"views": [f"{w}x{hh}" for w, hh in uneven_res], "views_per_s": uneven_vps,
                                 "ms_per_step": uneven_ms / args.steps},
                "e2e": {"value": e2e_vps, "unit": "views/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": 16,
                        "read": "gs_read_stats_async into pinned memory each step (readLoss as a Promise)"},
                "e2e_blocking_read": {"value": e2e_sync_vps, "unit": "views/s",
                                      "read": "gs_read_stats each step (one host sync per step)"},
                "gpu_launches": None,
                "phases_ms_per_step": phase,
                "steps_per_s": args.steps / (batch_ms * 1e-3),
                "pairs_per_step": pairs_per_launch,
                "pairs_executed_per_step": pairs_exec,
                # splat-pixel evaluations/s: the reference's pixel-entry pairs P of a step over its time
                "splat_pixel_evals_per_s": pairs_per_launch / (batch_ms * 1e-3 / args.steps)
                if pairs_per_launch else None,
                "roofline": {"bound": "fp32", "kernel": "raster (fused forward + loss + backward)",
                             "bound_note": "FP32 CUDA-core (issue) bound: no tensor-core or HBM bound applies; "
                                           "the peak is this GPU's measured FFMA throughput",
                             "achieved": achieved, "peak": peak.value, "unit": "TFLOP/s",
                             "frac": achieved / peak.value if peak.value else None,
                             "traffic": RASTER_DRAM_BYTES_8VIEW if (B == 8 and n == 1_000_000 and args.width == 1920)
                             else None,
                             "traffic_source": "one ncu capture of the raster over a 2-view step of this scene "
                                               "(two 1080p ring views), scaled to 8 views",
                             "peak_source": "gs_probe_fp32_peak FFMA kernel on this GPU (measured)",
                             "work": f"{FLOP_PER_PAIR} flop per pixel-entry pair P of the reference's tile lists "
                                     "(pairs up to each pixel's termination index); the step walks culled lists "
                                     "with pairs_executed_per_step of them"},
                "clocks": clocks,
                "cpu_baseline": cpu}
        line["gpu_launches"] = batch_launches * args.steps
        line["gpu_launches_per_step"] = batch_launches
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def cpu_baseline_line(args, params, sh, cams):
    """The oracle's plain step on one whole view of camera 0, all host
    threads: one untimed step, then one timed."""
    try:
        from oracle import oracle as O
        O.build()
        o, ocams, targets = cpu_setup(args, params, sh, cams, 1)
        cores = O.set_threads(0)
        tr = CpuTrainer(o, ocams, targets, params, sh)
        tr.step(0)
        sec = tr.step(0)
        return {"value": 1.0 / sec, "unit": "views/s", "cores": cores, "kind": "port",
                "sample": f"one whole {args.width}x{args.height} view of camera 0 (the oracle's plain training "
                          f"step over all splats, after one untimed step): {sec:.2f} s"}
    except Exception as e:  # the baseline is reported, never required
        return {"value": None, "unit": "views/s", "cores": os.cpu_count() or 1, "kind": "port",
                "sample": f"failed: {e}"}


def run_side_paths(args):
    """The steps either side of the training path, on the headline scene: the
    eval pass (_evalPass, trainer.js:542-574: a training-path pass without
    Adam on one view, stats and camera gradients back), the PLY export with
    the opacity bake over the 24 ring cameras (ply.js:17-99) and the frame
    undistortion (undistortFrames, session.js:44-80) of eight 1080p frames.
    Each is timed end to end through the C ABI (host buffers in and out, the
    call returns when its results are in host memory), beside the oracle's
    CPU restatement of the same step on the same inputs, all host threads."""
    import torch
    from oracle import oracle as O
    from splat_b200 import native as N
    from splat_b200 import scene
    from splat_b200.session import cam_position, undistort_frames
    from splat_b200.trainer import GSTrainer
    O.build()
    torch.cuda.set_device(0)
    params, sh, cams = workload(args)
    n = args.splats
    opts = dict(shDeg=2, maxSplats=n, maxBatch=1, batchDepth=256, device=0, persistent=1, useGraphs=1)
    pp, ps = scene.perturb(params, sh, 0.02, seed=args.seed + 1)
    blank = [dict(tw=c["w"], th=c["h"], rgb=np.zeros(c["w"] * c["h"] * 3, np.float32)) for c in cams]
    t = GSTrainer.create(opts)
    t.setup(dict(data=pp, n=n, sh=ps), cams, blank, args.width, args.height, 4.0)
    images = [dict(tw=c["w"], th=c["h"], rgb=np.ascontiguousarray(np.clip(t.renderView(c)[..., :3], 0, 1)
                                                                  .reshape(-1))) for c in cams]
    t.setup(dict(data=params, n=n, sh=sh), cams, images, args.width, args.height, 4.0)
    del images, blank
    t.iter = 2000
    L, h = N.lib(), t._h
    cores = O.set_threads(0)
    out = {"workload": f"{n}-splat surface scene, SH 2, {args.width}x{args.height}", "cpu_threads": cores}

    def wall(fn, reps):
        fn()
        t0 = time.perf_counter()
        for _ in range(reps):
            fn()
        return (time.perf_counter() - t0) / reps

    # eval pass on camera 0
    st = (C.c_uint32 * 4)()
    cg = (C.c_int32 * ((len(cams) + 1) * 8))()
    gpu_eval = wall(lambda: N.check(L.gs_eval_pass(h, 0, None, st, cg), h), 10)
    o, ocams, targets = cpu_setup(args, params, sh, cams, 1)
    p, s_ = params.copy(), sh.copy()
    m, v = np.zeros_like(p), np.zeros_like(p)
    sm, sv = np.zeros_like(s_), np.zeros_like(s_)
    cpu_eval = wall(lambda: O.step(o, [ocams[0]], cpu_adam_hp(2001, 4.0), p, s_, targets, m, v, sm, sv, n,
                                   do_adam=False), 1)
    out["eval_pass"] = {"gpu_ms": gpu_eval * 1e3, "cpu_ms": cpu_eval * 1e3, "speedup": cpu_eval / gpu_eval,
                        "what": "one 1080p view: project, bin, sort, raster forward + loss + backward, chain; "
                                "stats and camera gradients read back"}
    # PLY export with the opacity bake over the 24 ring cameras
    campos = np.ascontiguousarray([cam_position(c) for c in cams], np.float64)
    size = C.c_uint64()
    N.check(L.gs_export_ply(h, 1, float(cams[0]["f"]), campos.ctypes.data_as(C.POINTER(C.c_double)),
                            len(cams), None, 0, C.byref(size)), h)
    buf = np.empty(size.value, np.uint8)
    gpu_ply = wall(lambda: N.check(L.gs_export_ply(h, 1, float(cams[0]["f"]),
                                                   campos.ctypes.data_as(C.POINTER(C.c_double)), len(cams),
                                                   C.c_void_p(buf.ctypes.data), size.value, C.byref(size)), h), 5)
    g = t.readGaussians()
    cpu_ply = wall(lambda: O.ply_export(g["data"], g["n"], g["sh"], g["shK"], bake=True, f=float(cams[0]["f"]),
                                        cam_positions=campos), 1)
    out["ply_export"] = {"gpu_ms": gpu_ply * 1e3, "cpu_ms": cpu_ply * 1e3, "speedup": cpu_ply / gpu_ply,
                         "bytes": int(size.value), "cameras": len(cams),
                         "what": "bakeOpacityCompensation over the 24 cameras + gaussiansToPly, PLY bytes in "
                                 "host memory (CPU: the numpy restatement of ply.js)"}
    # undistortion of eight 1080p frames
    rng = np.random.default_rng(args.seed + 7)
    frames = [dict(tw=args.width, th=args.height, fw=float(args.width),
                   rgb=rng.random(args.width * args.height * 3, dtype=np.float32)) for _ in range(8)]
    recon = dict(k1=0.05, k2=-0.01, fFeat=1.17 * args.width)
    gpu_und = wall(lambda: undistort_frames([dict(f) for f in frames], recon), 3)
    cpu_und = wall(lambda: O.undistort_frames([dict(f) for f in frames], recon), 1)
    out["undistort"] = {"gpu_ms": gpu_und * 1e3, "cpu_ms": cpu_und * 1e3, "speedup": cpu_und / gpu_und,
                        "frames": len(frames), "bytes_each_way": len(frames) * args.width * args.height * 12,
                        "what": "undistortFrames of 8 RGB float32 frames, k1 0.05, k2 -0.01, frames copied in "
                                "and out (CPU: the numpy restatement of session.js)"}
    out["clock"] = "host wall time around each call (the calls return with their results in host memory)"
    print(json.dumps({"side_paths": out}), flush=True)
    return 0


def main():
    args = parse()
    if args.side_paths:
        return run_side_paths(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
