#!/usr/bin/env python
"""Benchmark: the full frame-to-depth pipeline on one 728x544 pair with 128
disparities and 8 paths (Rectification -> Disparity -> SpeckleFilter -> Depth
-> PointCloud(decimation 4)), pairs/s.

A step is one pair through the pipeline. `value` times the device pipeline on
inputs already in HBM (per-step CUDA events on the launching stream, L2
flushed between steps outside the events); `e2e` times the same pipeline
through the public API (CudaSegment.send_request / await_) from host frames,
host<->device copies included, up to depth() pairs in flight. Multi-GPU runs
are independent replicas (pairs do not shard: SGM paths cross the whole
image), timed as the max over ranks.

Beside the headline, rank 0 of a one-GPU run also reports `batched` (64
rectified pairs of mixed sizes and disparity ranges in one persistent,
graph-captured launch, against the single-pair matcher on the same pairs),
`large_range` (8 pairs of 1920x1080 at 256 disparities), `coarse_to_fine`
(Stage.Disparity's coarse-to-fine search at 728x544, band 16, beside the full
search), `config0` (the 364x272, 64-disparity matcher, beside the CPU port)
and `serving` (32 camera streams with Poisson arrivals at 30 pairs/s
each: p50/p99 latency).

`--impl reference` times the reference's CPU formulation of the same pipeline
(the oracle's C port of the reference's Rust matcher and stages) on all host
threads, one pair per thread per step.
"""
import argparse
import collections
import ctypes
import gc
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "pairs/s at 728x544x128 d, 8 paths (full frame-to-depth pipeline)"
WIDTH, HEIGHT, DISPARITIES, PATHS = 728, 544, 128, 8
DECIMATION = 4
KERNELS_PER_STEP = 6  # rectify, census+costs, paths, select, check+median, despeckle+depth+cloud
PATHS_EVERY = 4  # timed steps between those whose path kernel is bracketed by events
# At most this many pairs on the device at once in the serving run, oldest
# arrival first (None: up to every stream's request slots; caps of 4, 8 and 16
# kept p99 at 30 pairs/s/stream the same and lowered the saturation rate).
SERVING_CAP = None
# DRAM bytes (read + write) of one path-aggregation launch on this workload, from
# an ncu capture of this command (dram__bytes_read.sum + dram__bytes_write.sum).
PATHS_TRAFFIC_BYTES = 114_332_416 + 350_151_936


# The workload's config, the same on both arms.
CONFIG = {"workload": "full pipeline 728x544 frames -> 728x544, D128, 8 paths, despeckle, depth, "
                      "cloud (decimation 4)",
          "width": WIDTH, "height": HEIGHT, "disparities": DISPARITIES, "paths": PATHS,
          "decimation": DECIMATION, "pairs_per_step": 1}
E2E_MIN_SECONDS = 1.0  # the end-to-end loop runs at least this long (and at least --steps pairs)


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=200)
    p.add_argument("--warmup", type=int, default=10)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--inputs", type=int, default=8, help="distinct pairs cycled through")
    p.add_argument("--no-batch", action="store_true", help="skip the batched workload")
    p.add_argument("--no-serving", action="store_true", help="skip the serving workload")
    p.add_argument("--no-large", action="store_true", help="skip the large-range workload")
    p.add_argument("--aggregate", default="volumes", choices=["volumes", "sums"],
                   help="the device pipeline's aggregation: 8 path volumes summed by selection "
                        "(the default), or every direction adding into one u16 volume")
    p.add_argument("--path-tiles", type=int, default=1, choices=[0, 1, 2],
                   help="path scans take their costs by bulk tensor copies: 0 never, 2 always, "
                        "1 for large pairs (the library's default)")
    p.add_argument("--no-coarse-to-fine", action="store_true",
                   help="skip the coarse-to-fine workload")
    return p.parse_args()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            m = json.load(f)
        return float(m["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ---------------------------------------------------------------- inputs
def make_inputs(count, seed):
    from nx_stereo_b200 import scene

    rig = scene.rig(WIDTH, HEIGHT)
    frames = []
    for i in range(count):
        left, right = scene.rectified_pair(WIDTH, HEIGHT, seed=seed * 1000 + i, rectangles=6,
                                           min_disparity=4, max_disparity=120)
        frames.append(scene.raw_frames(left, right, rig))
    return rig, frames


# ---------------------------------------------------------------- clocks
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_id):
        self.samples = []
        self.proc = None
        self.device_id = device_id

    def start(self):
        cmd = ["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
               "-lms", "200"]
        if self.device_id is not None:
            cmd += ["-i", str(self.device_id)]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                                         text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append((time.monotonic(), [f.strip() for f in line.split(",")]))

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self, t0, t1):
        rows = [s for t, s in self.samples if t0 - 0.25 <= t <= t1 + 0.25] or \
            [s for _, s in self.samples]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}

        def num(v):
            try:
                return float(v)
            except ValueError:
                return None

        sm = [num(r[1]) for r in rows if num(r[1]) is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": num(rows[0][2]), "reasons": reasons, "samples": len(rows),
                "power_w_max": max((num(r[3]) or 0.0) for r in rows)}


# ---------------------------------------------------------------- our arm
class DevicePipeline:
    """The pipeline's kernels on device buffers, one C-ABI call per stage; CUDA
    events bracket the path-aggregation kernel (the dominant one). The
    rectification maps are the stream's state, made once for its cameras and
    kept on the device, as a segment keeps them."""

    def __init__(self, native, torch, ctx, rig, stream, aggregate="volumes"):
        from nx_stereo_b200 import scene

        self.native, self.torch, self.ctx, self.stream = native, torch, ctx, stream
        self.sums = aggregate == "sums"
        cams = scene.cameras(rig)
        self.cameras = [native.make_camera(cams[s]["k"], cams[s]["d"], cams[s]["inverse_pr"])
                        for s in ("left", "right")]
        self.focal, self.baseline = rig["focal_length_px"], rig["baseline_m"]
        self.cx, self.cy = rig["principal_point"]
        px, vol = WIDTH * HEIGHT, WIDTH * HEIGHT * DISPARITIES
        dev = torch.device("cuda")
        u8, f32 = torch.uint8, torch.float32
        self.images = torch.empty((2, HEIGHT, WIDTH), dtype=u8, device=dev)
        self.costs = torch.empty(vol, dtype=u8, device=dev)
        self.volumes = torch.empty(PATHS * vol, dtype=u8, device=dev)
        self.selected = torch.empty(px, dtype=f32, device=dev)
        self.keys = torch.empty(px, dtype=torch.int32, device=dev)
        self.checked = torch.empty(px, dtype=f32, device=dev)
        self.disparity = torch.empty(px, dtype=f32, device=dev)
        self.speckled = torch.empty(px, dtype=f32, device=dev)
        self.depth_mm = torch.empty(px, dtype=torch.int16, device=dev)
        self.depth_m = torch.empty(px, dtype=f32, device=dev)
        self.grid = torch.empty((HEIGHT // DECIMATION) * (WIDTH // DECIMATION) * 3, dtype=f32,
                                device=dev)
        self.kept = torch.empty(1, dtype=torch.int32, device=dev)
        # The costs and path volumes in the order the matcher itself keeps them.
        self.span = int(native.load().nxs_matcher_span(DISPARITIES))
        self.maps = torch.empty((2, HEIGHT, WIDTH, 2), dtype=f32, device=dev)
        native.call("nxs_rectify_maps_device", ctypes.byref(self.cameras[0]),
                    ctypes.byref(self.cameras[1]), WIDTH, HEIGHT, WIDTH, HEIGHT,
                    self.maps.data_ptr(), stream)

    STAGES = ["rectify", "census_costs", "paths", "select", "check_median",
              "despeckle_depth_cloud"]

    def step(self, frames, marks=None):
        """One pair; `marks` (len(STAGES) + 1 CUDA events or None) bracket the
        stages. An event between two kernels also ends the overlap of the
        second's launch with the first's tail (programmatic dependent launch),
        so the timed steps record only the step's ends and the path stage."""
        s, call = self.stream, self.native.call

        def mark(i):
            if marks is not None and marks[i] is not None:
                marks[i].record()

        mark(0)
        call("nxs_rectify_pair_mapped_device", frames[0].data_ptr(), frames[1].data_ptr(), WIDTH,
             HEIGHT, self.maps.data_ptr(), WIDTH, HEIGHT, self.images[0].data_ptr(),
             self.images[1].data_ptr(), s)
        mark(1)
        call("nxs_census_costs_device_ordered", self.images[0].data_ptr(),
             self.images[1].data_ptr(), WIDTH, HEIGHT, DISPARITIES, self.span,
             self.costs.data_ptr(), s)
        mark(2)
        if self.sums:  # every direction adds into one u16 volume (in the volumes' room)
            call("nxs_path_sums_device", self.costs.data_ptr(), WIDTH, HEIGHT, DISPARITIES, PATHS,
                 8, 64, self.volumes.data_ptr(), s)
            mark(3)
            call("nxs_select_path_sums_device", self.volumes.data_ptr(), WIDTH, HEIGHT,
                 DISPARITIES, 1.0526315789473684, self.selected.data_ptr(), self.keys.data_ptr(),
                 s)
        else:
            call("nxs_paths_device_ordered", self.costs.data_ptr(), WIDTH, HEIGHT, DISPARITIES,
                 PATHS, 8, 64, self.span, self.volumes.data_ptr(), s)
            mark(3)
            call("nxs_select_paths_device_ordered", self.volumes.data_ptr(), WIDTH, HEIGHT,
                 DISPARITIES, PATHS, 1.0526315789473684, self.span, self.selected.data_ptr(),
                 self.keys.data_ptr(), s)
        mark(4)
        call("nxs_check_median_device", self.selected.data_ptr(), self.keys.data_ptr(), WIDTH,
             HEIGHT, 1, self.disparity.data_ptr(), s)
        mark(5)
        call("nxs_despeckle_depth_cloud_device", self.disparity.data_ptr(), WIDTH, HEIGHT, 12.0,
             1.0, 3, self.focal, self.baseline, DECIMATION, self.cx, self.cy, 0.05, 20.0,
             self.speckled.data_ptr(), self.depth_mm.data_ptr(), self.depth_m.data_ptr(),
             self.grid.data_ptr(), self.kept.data_ptr(), s)
        mark(6)


def run_ours(args, rank, world, local_rank):
    import torch

    from nx_stereo_b200 import native, replicas, segment, stage

    torch.cuda.set_device(local_rank)
    native.load().nxs_set_path_tiles(args.path_tiles)
    ctx = native.Context(local_rank)
    rig, frames = make_inputs(args.inputs, seed=replicas.seed(rank, 0))
    stream_obj = torch.cuda.Stream()

    with torch.cuda.stream(stream_obj):
        s = stream_obj.cuda_stream
        pipe = DevicePipeline(native, torch, ctx, rig, s, args.aggregate)
        d_frames = [(torch.from_numpy(l).cuda(), torch.from_numpy(r).cuda()) for l, r in frames]
        flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
        for i in range(args.warmup):
            pipe.step(d_frames[i % len(d_frames)])
        torch.cuda.synchronize()
        replicas.barrier()
        sampler = ClockSampler(local_rank if os.environ.get("CUDA_VISIBLE_DEVICES") is None else None)
        sampler.start()
        time.sleep(0.3)
        n_marks = len(DevicePipeline.STAGES) + 1
        paths_at = DevicePipeline.STAGES.index("paths")
        # Every step records its ends; every PATHS_EVERY-th also brackets the path
        # kernel (each event between kernels costs ~2.5 us a step).
        ends, with_paths = (0, n_marks - 1), (0, paths_at, paths_at + 1, n_marks - 1)

        def events(which):
            return [[torch.cuda.Event(enable_timing=True) if k in which(i) else None
                     for k in range(n_marks)] for i in range(args.steps)]

        marks = events(lambda i: with_paths if i % PATHS_EVERY == 0 else ends)
        torch.cuda.synchronize()
        t0 = time.monotonic()
        for i in range(args.steps):
            flush.fill_(i & 0xFF)  # evict L2 between timed steps, outside the events
            pipe.step(d_frames[i % len(d_frames)], marks[i])
        torch.cuda.synchronize()
        t1 = time.monotonic()
        step_ms = [m[0].elapsed_time(m[-1]) for m in marks]
        paths_ms = [m[paths_at].elapsed_time(m[paths_at + 1]) for m in marks
                    if m[paths_at] is not None]
        # Each stage's time from a second, untimed run with an event at every stage.
        stage_marks = events(lambda i: range(n_marks))
        for i in range(args.steps):
            flush.fill_(i & 0xFF)
            pipe.step(d_frames[i % len(d_frames)], stage_marks[i])
        torch.cuda.synchronize()
        stage_ms = {name: statistics.mean(m[k].elapsed_time(m[k + 1]) for m in stage_marks)
                    for k, name in enumerate(DevicePipeline.STAGES)}
    total_s = replicas.max_over_ranks(sum(step_ms) / 1000.0, device="cuda")
    value = replicas.whole_job_rate(args.steps, world, total_s)

    # e2e: the public API, host frames in, outputs back to the host.
    geometry = segment.standard_geometry(WIDTH, HEIGHT, the_rig=rig)
    status, members = segment.members(
        [stage.Rectification, (stage.Disparity, {"num_disparities": DISPARITIES}),
         stage.SpeckleFilter, stage.Depth, (stage.PointCloud, {"decimation": DECIMATION})],
        geometry)
    assert status == "ok", members
    status, seg = segment.CudaSegment.build(members, geometry, {"device": local_rank})
    assert status == "ok", seg
    mod = segment.CudaSegment
    entries = [{"left_frame": l, "right_frame": r} for l, r in frames]
    h2d = sum(a.nbytes for a in entries[0].values())
    d2h = None

    inflight = collections.deque()
    sent = 0

    def take_reply():
        nonlocal d2h
        reply = mod.await_(inflight.popleft(), seg, 60000)
        assert reply[0] == "ok", reply
        d2h = sum(v.nbytes for v in reply[1].values())

    def e2e_send(count):
        """Sends `count` pairs, awaiting the oldest whenever depth are in flight."""
        nonlocal sent
        for _ in range(count):
            status, req = mod.send_request(entries[sent % len(entries)], seg)
            assert status == "ok", req
            sent += 1
            inflight.append(req)
            if len(inflight) >= mod.depth():
                take_reply()

    e2e_send(max(args.warmup, mod.depth()))
    while inflight:
        take_reply()
    torch.cuda.synchronize()
    replicas.barrier()
    # The cyclic collector paused for the timed loop, as the serving loop does:
    # a collection of the replies' objects stalls the host for milliseconds.
    # The loop sends --steps pairs at a time, keeping depth pairs in flight from
    # one round to the next, until it has run E2E_MIN_SECONDS; then it takes the
    # last replies. Every rank runs the same number of rounds (the first rank's).
    collecting = gc.isenabled()
    gc.disable()
    try:
        e0 = time.perf_counter()
        c0 = time.thread_time()  # the calling thread's CPU time: the API's host cost
        e2e_pairs = 0
        while True:
            e2e_send(args.steps)
            e2e_pairs += args.steps
            more = time.perf_counter() - e0 < E2E_MIN_SECONDS
            if not replicas.agree(more, device="cuda"):
                break
        while inflight:
            take_reply()
        e_elapsed = time.perf_counter() - e0
        host_cpu_s = time.thread_time() - c0
        e1 = time.monotonic()
    finally:
        if collecting:
            gc.enable()
    e_s = replicas.max_over_ranks(e_elapsed, device="cuda")
    sampler.stop()
    # Device-timed steps are short (milliseconds), so the clock record spans
    # them, the stage-time run and the end-to-end loop: all under load.
    clocks = sampler.summary(t0, e1)
    seg.release()

    peak, peak_kind = peaks()
    px, vol = WIDTH * HEIGHT, WIDTH * HEIGHT * DISPARITIES
    paths_bytes = vol + PATHS * vol  # u8 costs read once, 8 u8 path volumes written
    paths_avg_s = statistics.mean(paths_ms) / 1000.0
    achieved = paths_bytes / paths_avg_s / 1e9
    b_alg = 8 * vol + 6 * px  # per pair: u16 cost + aggregate written and read, images, disparity
    line = {
        "metric": METRIC, "value": round(value, 2), "unit": "pairs/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(statistics.mean(step_ms), 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8/u16",
        "data": "synthetic (seeded piecewise-planar scenes, raw frames from a synthetic rig)",
        "config": dict(CONFIG, parallelism=f"replicas x{world}",
                       l2="flushed between steps (256 MiB write outside the step events); "
                          "per-step working set 460 MB > 126 MB L2"),
        "mdisp_s": round(value * px * DISPARITIES / 1e6, 1),
        "gpu_launches": KERNELS_PER_STEP * args.steps,
        "roofline": {"bound": "hbm", "kernel": "paths_kernel (8-path aggregation)",
                     "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "peak_kind": peak_kind,
                     "algorithmic_bytes_per_launch": paths_bytes,
                     "avg_launch_ms": round(paths_avg_s * 1000, 4),
                     "traffic": PATHS_TRAFFIC_BYTES,
                     "limiter": "dependent latency of the longest scan lines' steps and "
                                "instruction issue with ~8 warps a SM (ncu: issue 57%, integer "
                                "ALU pipe 61%, FMA pipe 12%, HBM 45%)"},
        "stages_ms": {k: round(v, 4) for k, v in stage_ms.items()},
        "stages_ms_from": "a second run of the same steps with an event between every stage",
        "pipeline_roofline": {"b_alg_per_pair": b_alg,
                              "achieved_gbs": round(b_alg * value / world / 1e9, 1),
                              "frac": round(b_alg * value / world / 1e9 / peak, 4)},
        "e2e": {"value": round(replicas.whole_job_rate(e2e_pairs, world, e_s), 2),
                "unit": "pairs/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "pairs": e2e_pairs, "seconds": round(e_s, 3),
                "host_cpu_us_per_pair": round(1e6 * host_cpu_s / e2e_pairs, 1),
                "api": "CudaSegment.send_request/await_ (C ABI nxs_run_async), depth "
                       f"{mod.depth()}, cyclic garbage collector paused while timed"},
        "clocks": clocks,
        "aggregate": args.aggregate,
        "path_tiles": args.path_tiles,
    }
    return line


# ---------------------------------------------------------------- other workloads
def _time_events(torch, stream, fn, repeats):
    """Median ms of fn() on `stream`, by CUDA events."""
    times = []
    with torch.cuda.stream(stream):
        for _ in range(repeats):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            b.synchronize()
            times.append(a.elapsed_time(b))
    return statistics.median(times)


def _plain_and_batched(torch, ctx, shapes, pairs, tuner_search=None, repeats=5):
    """Times the batched launch (autotuned) and the single-pair matcher one pair
    after another on the same device-resident pairs; checks every output."""
    from nx_stereo_b200 import batch

    stream = torch.cuda.Stream()
    handle = stream.cuda_stream
    plan = batch.BatchPlan(ctx, shapes)
    for i, (left, right) in enumerate(pairs):
        plan.set_inputs(i, left, right)
    host_outputs = plan.run()  # host buffers in, one launch, host buffers out
    tuner = batch.Autotuner(repeats=3, sweeps=1, search=tuner_search)
    tuning, _ = tuner.tune(plan, use_cache=False)
    with torch.cuda.stream(stream):
        for _ in range(2):
            plan.launch(stream=handle)
    batched_ms = _time_events(torch, stream, lambda: plan.launch(stream=handle), repeats)
    plan.check()
    t0 = time.perf_counter()
    for _ in range(3):
        plan.run(copy=False)
    e2e_s = (time.perf_counter() - t0) / 3
    plain_e2e_s, pipelined_exact = _plain_pipelined(shapes, pairs, host_outputs)
    devs = [(torch.from_numpy(l).cuda(), torch.from_numpy(r).cuda()) for l, r in pairs]
    outs = [torch.empty((h, w), dtype=torch.float32, device="cuda") for w, h, _ in shapes]

    def plain():
        for (w, h, settings), (dl, dr), out in zip(shapes, devs, outs):
            ctx.sgm_device(dl.data_ptr(), dr.data_ptr(), w, h, out.data_ptr(), stream=handle,
                           **settings)

    with torch.cuda.stream(stream):
        plain()
    plain_ms = _time_events(torch, stream, plain, max(2, repeats // 2))
    torch.cuda.synchronize()
    exact = sum(int(np.array_equal(o.cpu().numpy().view(np.uint32), h.view(np.uint32)))
                for o, h in zip(outs, host_outputs))
    stats = plan.stats()
    disparities = plan.disparities()
    b_alg = sum(8 * w * h * s["disparities"] + 6 * w * h for w, h, s in shapes)
    plan.close()
    n = len(shapes)
    return {"pairs": n, "batched_ms": round(batched_ms, 3),
            "pairs_per_s": round(n / batched_ms * 1e3, 1),
            "mdisp_s": round(disparities / batched_ms / 1e3, 1),
            "plain_ms": round(plain_ms, 3), "plain_pairs_per_s": round(n / plain_ms * 1e3, 1),
            "batched_over_plain": round(plain_ms / batched_ms, 3),
            "e2e_pairs_per_s": round(n / e2e_s, 1),
            "plain_e2e_pairs_per_s": round(n / plain_e2e_s, 1),
            "batched_over_plain_e2e": round(plain_e2e_s / e2e_s, 3),
            "plain_e2e_api": "the pipelined per-pair API: a CudaSegment (Stage.Disparity) per "
                             "distinct shape, pinned staging, pairs sent in order with up to "
                             f"{PIPELINE_DEPTH} at the device (C ABI nxs_run_async)",
            "plain_e2e_exact_pairs": pipelined_exact,
            "e2e_api": "BatchPlan.run (C ABI nxs_batch_run: one graph, host in and out)",
            "h2d_bytes": stats["input_bytes"], "d2h_bytes": stats["output_bytes"],
            "bit_exact_pairs": exact, "tuning": tuning, "queue_items": stats["items"],
            "device_gb": round(stats["device_bytes"] / 1e9, 2),
            "b_alg_gbs": round(b_alg / batched_ms / 1e6, 1), "gpu_launches_per_batch": 1}


PIPELINE_DEPTH = 4


def _plain_pipelined(shapes, pairs, batch_outputs, depth=PIPELINE_DEPTH):
    """The single-pair form end to end through the public per-pair API: a
    CudaSegment with Stage.Disparity alone for each distinct shape (pinned
    staging, two compute lanes), the pairs sent in order with up to `depth`
    at the device. Returns (seconds, pairs equal to the batch's outputs
    after Stage.Disparity's mask)."""
    from nx_stereo_b200 import segment, stage

    mod = segment.CudaSegment
    segments = {}

    def segment_of(w, h, settings):
        key = (w, h, settings["disparities"], settings.get("paths", 8))
        if key not in segments:
            geometry = segment.standard_geometry(w, h)
            status, members = segment.members(
                [(stage.Disparity, {"num_disparities": key[2], "paths": key[3]})], geometry)
            assert status == "ok", members
            status, segments[key] = mod.build(members, geometry)
            assert status == "ok", segments[key]
        return segments[key]

    def loop():
        inflight, outputs = [], []

        def reply():
            request, seg = inflight.pop(0)
            answer = mod.await_(request, seg, 60000)
            assert answer[0] == "ok", answer
            outputs.append(np.array(answer[1]["disparity"]))

        for (w, h, settings), (left, right) in zip(shapes, pairs):
            seg = segment_of(w, h, settings)
            status, request = mod.send_request({"left": left, "right": right}, seg)
            assert status == "ok", request
            inflight.append((request, seg))
            if len(inflight) >= depth:
                reply()
        while inflight:
            reply()
        return outputs

    loop()  # configures every segment (device memory, pinned staging)
    collecting = gc.isenabled()
    gc.disable()
    try:
        times = []  # the median of 5 passes: one pass is ~30 ms of host-bound calls
        for _ in range(5):
            t0 = time.perf_counter()
            outputs = loop()
            times.append(time.perf_counter() - t0)
        seconds = statistics.median(times)
    finally:
        if collecting:
            gc.enable()
    exact = sum(int(np.array_equal(o.view(np.uint32),
                                   np.where(b > 0, b, np.float32(-1.0)).astype(np.float32)
                                   .view(np.uint32)))
                for o, b in zip(outputs, batch_outputs))
    for seg in segments.values():
        seg.release()
    return seconds, exact


def bench_batched(torch, ctx):
    """64 rectified pairs of seeded sizes {320x240 .. 1280x720} x D {64, 96,
    128, 192}, 8 paths, in one persistent graph-captured launch."""
    from nx_stereo_b200 import batch, scene

    shapes = batch.sample_shapes(64, seed=2024)
    pairs = [scene.rectified_pair(w, h, seed=7000 + i, max_disparity=min(56, s["disparities"] - 8))
             for i, (w, h, s) in enumerate(shapes)]
    out = _plain_and_batched(torch, ctx, shapes, pairs)
    out["workload"] = ("64 pairs, sizes drawn from 320x240, 480x270, 640x480, 728x544, 1280x720, "
                       "disparities from 64, 96, 128, 192 (seed 2024), 8 paths")
    return out


def bench_large(torch, ctx):
    """8 pairs of 1920x1080 at 256 disparities, 12 rectangles at 8-240, sigma 3."""
    from nx_stereo_b200 import scene

    shapes = [(1920, 1080, {"disparities": 256})] * 8
    pairs = [scene.rectified_pair(1920, 1080, seed=900 + i, rectangles=12, min_disparity=8,
                                  max_disparity=240, sigma=3.0) for i in range(8)]
    out = _plain_and_batched(torch, ctx, shapes, pairs, repeats=3,
                             tuner_search={"engine": (0, 1), "streams": (1, 2, 8),
                                           "order": (0, 1), "group_pairs": (1, 2)})
    out["workload"] = "8 pairs 1920x1080, 256 disparities, 8 paths"
    out.update(_large_overlap(torch, ctx, shapes, pairs))
    return out


def _large_overlap(torch, ctx, shapes, pairs):
    """The large-range batch with each pair's kernels as a chain on 1, 2 or 4
    streams of one graph (with 2, pair k + 1's census and costs run beside
    pair k's path aggregation) and as the persistent launch, each timed by
    CUDA events; and one pair's stages, each bracketed by events."""
    from nx_stereo_b200 import batch, native

    stream = torch.cuda.Stream()
    handle = stream.cuda_stream
    plan = batch.BatchPlan(ctx, shapes, {"engine": 1, "streams": 1})
    for i, (left, right) in enumerate(pairs):
        plan.set_inputs(i, left, right)
    want = plan.run()
    streams_ms = {}
    for count in (1, 2, 4):
        plan.retune(engine=1, streams=count)
        with torch.cuda.stream(stream):
            plan.launch(stream=handle)
        streams_ms[str(count)] = round(
            _time_events(torch, stream, lambda: plan.launch(stream=handle), 3), 3)
    plan.retune(engine=0)
    with torch.cuda.stream(stream):
        plan.launch(stream=handle)
    persistent_ms = round(_time_events(torch, stream, lambda: plan.launch(stream=handle), 3), 3)
    got = plan.run()
    exact = sum(int(np.array_equal(a.view(np.uint32), b.view(np.uint32))) for a, b in zip(got, want))
    plan.close()
    # One pair's stages on device buffers, in the order the matcher runs them.
    w, h, d = 1920, 1080, 256
    span = int(native.load().nxs_matcher_span(d))
    dl, dr = (torch.from_numpy(a).cuda() for a in pairs[0])
    costs = torch.empty(w * h * d, dtype=torch.uint8, device="cuda")
    volumes = torch.empty(8 * w * h * d, dtype=torch.uint8, device="cuda")
    selected = torch.empty(w * h, dtype=torch.float32, device="cuda")
    keys = torch.empty(w * h, dtype=torch.int32, device="cuda")
    out = torch.empty(w * h, dtype=torch.float32, device="cuda")
    steps = {
        "census_costs": lambda: native.call("nxs_census_costs_device_ordered", dl.data_ptr(),
                                            dr.data_ptr(), w, h, d, span, costs.data_ptr(),
                                            handle),
        "paths": lambda: native.call("nxs_paths_device_ordered", costs.data_ptr(), w, h, d, 8, 8,
                                     64, span, volumes.data_ptr(), handle),
        "select": lambda: native.call("nxs_select_paths_device_ordered", volumes.data_ptr(), w, h,
                                      d, 8, 1.0526315789473684, span, selected.data_ptr(),
                                      keys.data_ptr(), handle),
        "check_median": lambda: native.call("nxs_check_median_device", selected.data_ptr(),
                                            keys.data_ptr(), w, h, 0, out.data_ptr(), handle),
    }
    stage_ms = {}
    for name, fn in steps.items():
        with torch.cuda.stream(stream):
            fn()
        stage_ms[name] = round(_time_events(torch, stream, fn, 3), 3)
    del costs, volumes
    return {"streams_engine_ms": streams_ms, "persistent_ms": persistent_ms,
            "overlap_exact_pairs": exact, "pair_stages_ms": stage_ms,
            "overlap_note": "streams_engine_ms: each pair's kernels chained on one of k streams "
                            "of one CUDA graph, so with k >= 2 the next pair's census and "
                            "costs run beside the current pair's path aggregation"}


def bench_coarse_to_fine(torch, ctx, pairs=64):
    """Stage.Disparity's coarse-to-fine search at 728x544 (band 16, margin 4,
    8 paths, the reference's fast setting): CUDA-event ms a pair on device
    buffers, beside the full search of the same rectified pairs; both checked
    against the oracle on the first pair."""
    from nx_stereo_b200 import scene
    from oracle import oracle

    w, h = WIDTH, HEIGHT
    inputs = [scene.rectified_pair(w, h, seed=3000 + i, rectangles=6, max_disparity=120)
              for i in range(8)]
    devs = [(torch.from_numpy(l).cuda(), torch.from_numpy(r).cuda()) for l, r in inputs]
    out = torch.empty((h, w), dtype=torch.float32, device="cuda")
    stream = torch.cuda.Stream()
    handle = stream.cuda_stream
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    settings = {"band": 16, "margin": 4, "paths": PATHS}

    def c2f(i):
        dl, dr = devs[i % len(devs)]
        ctx.sgm_coarse_to_fine_device(dl.data_ptr(), dr.data_ptr(), w, h, out.data_ptr(),
                                      stream=handle, **settings)

    def full(i):
        dl, dr = devs[i % len(devs)]
        ctx.sgm_device(dl.data_ptr(), dr.data_ptr(), w, h, out.data_ptr(), stream=handle,
                       disparities=DISPARITIES, paths=PATHS)

    results = {}
    for name, fn in (("coarse_to_fine", c2f), ("full", full)):
        marks = []
        with torch.cuda.stream(stream):
            for i in range(3):
                fn(i)
            for i in range(pairs):
                flush.fill_(i & 0xFF)
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record(stream)
                fn(i)
                b.record(stream)
                marks.append((a, b))
        torch.cuda.synchronize()
        results[name] = statistics.mean(a.elapsed_time(b) for a, b in marks)
    left, right = inputs[0]
    c2f(0)
    torch.cuda.synchronize()
    want = oracle.sgm_coarse_to_fine(left, right, PATHS, PATHS, 16, 4)
    exact = bool(np.array_equal(out.cpu().numpy().view(np.uint32), want.view(np.uint32)))
    return {"workload": "728x544 rectified pairs, coarse to fine: sgm/3 at 364x272 D64 8 paths, "
                        "then sgm_band/4 D128 band 16 margin 4 8 paths (+ check, median)",
            "pairs": pairs, "ms_per_pair": round(results["coarse_to_fine"], 4),
            "pairs_per_s": round(1000.0 / results["coarse_to_fine"], 1),
            "full_search_ms_per_pair": round(results["full"], 4),
            "over_full_search": round(results["full"] / results["coarse_to_fine"], 3),
            "bit_exact_first_pair": exact,
            "timing": "CUDA events around each pair on device buffers, L2 flushed between "
                      "pairs outside the events"}


def bench_config0(torch, ctx, pairs=200):
    """The plain single-pair matcher on the 364x272, 64-disparity, 8-path pair
    (NxStereo.sgm/3: census, costs, paths, selection, check, median), device
    buffers, CUDA events around each pair with L2 flushed between pairs; beside
    it the C port of the reference's Rust matcher on every host thread."""
    from nx_stereo_b200 import scene
    from oracle import oracle

    w, h, d = 364, 272, 64
    inputs = [scene.rectified_pair(w, h, seed=400 + i, rectangles=6, max_disparity=56)
              for i in range(8)]
    devs = [(torch.from_numpy(l).cuda(), torch.from_numpy(r).cuda()) for l, r in inputs]
    out = torch.empty((h, w), dtype=torch.float32, device="cuda")
    stream = torch.cuda.Stream()
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    marks = []
    with torch.cuda.stream(stream):
        for i in range(pairs + 3):
            dl, dr = devs[i % len(devs)]
            flush.fill_(i & 0xFF)
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            ctx.sgm_device(dl.data_ptr(), dr.data_ptr(), w, h, out.data_ptr(),
                           stream=stream.cuda_stream, disparities=d, paths=PATHS)
            b.record(stream)
            if i >= 3:
                marks.append((a, b))
    torch.cuda.synchronize()
    ms = statistics.mean(a.elapsed_time(b) for a, b in marks)
    exact = bool(np.array_equal(out.cpu().numpy().view(np.uint32),
                                oracle.sgm(*inputs[(pairs + 2) % len(inputs)], d, PATHS)
                                .view(np.uint32)))
    threads = host_threads()
    lefts = np.stack([inputs[i % len(inputs)][0] for i in range(threads)])
    rights = np.stack([inputs[i % len(inputs)][1] for i in range(threads)])
    t = time.perf_counter()
    oracle.fast_sgm_batch(lefts, rights, d, PATHS, threads=threads)
    cpu = threads / (time.perf_counter() - t)
    return {"workload": "364x272 rectified pairs, D64, 8 paths, sgm/3 (check and median)",
            "pairs": pairs, "ms_per_pair": round(ms, 4), "pairs_per_s": round(1000.0 / ms, 1),
            "bit_exact_last_pair": exact,
            "cpu_port_pairs_per_s": round(cpu, 2), "cpu_threads": threads,
            "timing": "CUDA events around each pair on device buffers, L2 flushed between "
                      "pairs outside the events"}


def bench_serving(seconds=3.0, max_in_flight=SERVING_CAP):
    """32 camera streams (728x544 and 1280x720 alternating), Poisson arrivals
    at 30 pairs/s each, Rectification -> Disparity(128) -> SpeckleFilter ->
    TemporalFilter -> Depth -> Quality; then every stream back to back."""
    from nx_stereo_b200 import serving

    specs = serving.synthetic_streams(32, frames=8, seed=0)
    server = serving.Server(reserve_bytes=2 << 30, max_in_flight=max_in_flight)
    ids = [server.open(g) for g, _ in specs]
    frames_of = [fr for _, fr in specs]
    admitted = sum(server.admitted(i) for i in ids)
    serving.warm(server, ids, frames_of)
    arrivals = serving.poisson_arrivals(32, 30.0, seconds, seed=1)
    st = serving.run_load(server, ids, frames_of, arrivals)
    server.max_in_flight = 0
    burst = serving.run_load(server, ids, frames_of, [(0.0, s) for s in range(32) for _ in range(8)])
    used = server.used
    # The plain form on the same pipeline and frames: one stream at a time
    # (one of each size), its pairs pipelined through its segment as the
    # headline's end-to-end run sends them.
    plain_pairs = 64
    t0 = time.monotonic_ns()
    for index in (0, 1):
        for k in range(plain_pairs // 2):
            server.submit(ids[index], frames_of[index][k % len(frames_of[index])])
        while server.in_flight():
            server.poll(wait=True)
    plain_s = (time.monotonic_ns() - t0) / 1e9
    for sid in ids:
        server.close(sid)
    return {"workload": "32 streams (16 at 728x544, 16 at 1280x720), Poisson 30 pairs/s each, "
                        "Rect -> Disparity(128, 8 paths) -> Speckle -> Temporal -> Depth -> Quality",
            "offered_pairs_per_s": 32 * 30, "pairs": st["pairs"],
            "max_in_flight_cap": max_in_flight,
            "pairs_per_s": round(st["pairs_per_s"], 1), "p50_ms": round(st["p50_ms"], 3),
            "p99_ms": round(st["p99_ms"], 3), "max_in_flight": st["max_in_flight"],
            "streams_admitted": admitted, "device_gb_admitted": round(used / 1e9, 2),
            "saturation_pairs_per_s": round(burst["pairs_per_s"], 1),
            "plain_pairs_per_s": round(plain_pairs / plain_s, 1),
            "served_over_plain": round(burst["pairs_per_s"] / (plain_pairs / plain_s), 3),
            "latency": "arrival to device completion (CLOCK_MONOTONIC), percentile index "
                       "ceil(n p) - 1"}


def cpu_sample(rig, frames, threads, pairs):
    from nx_stereo_b200 import scene
    from oracle import oracle

    cams = scene.cameras(rig)
    cl = oracle.make_camera(cams["left"]["k"], cams["left"]["d"], cams["left"]["inverse_pr"])
    cr = oracle.make_camera(cams["right"]["k"], cams["right"]["d"], cams["right"]["inverse_pr"])
    lefts = np.stack([frames[i % len(frames)][0] for i in range(pairs)])
    rights = np.stack([frames[i % len(frames)][1] for i in range(pairs)])
    t = time.perf_counter()
    oracle.fast_pipeline_batch(lefts, rights, cl, cr, (HEIGHT, WIDTH), DISPARITIES, PATHS,
                               focal_length_px=rig["focal_length_px"],
                               baseline_m=rig["baseline_m"], decimation=DECIMATION,
                               principal_point=rig["principal_point"], threads=threads)
    return pairs / (time.perf_counter() - t)


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def run_reference(args):
    threads = host_threads()
    rig, frames = make_inputs(min(args.inputs, 4), seed=1)
    values = []
    for i in range(args.warmup + args.steps):
        v = cpu_sample(rig, frames, threads, threads)
        if i >= args.warmup:
            values.append(v)
    value = statistics.mean(values)
    sample = f"{threads} pairs per step (one per thread), {args.steps} steps"
    return {"metric": METRIC, "value": round(value, 3), "unit": "pairs/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1000 * threads / value, 2),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8/u16",
            "data": "synthetic", "impl": "reference",
            "config": dict(CONFIG, parallelism=f"{threads} host threads"),
            "cpu_baseline": {"value": round(value, 3), "unit": "pairs/s", "cores": threads,
                             "kind": "port", "sample": sample},
            "e2e": {"value": round(value, 3), "unit": "pairs/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


def section(name, run):
    """One of the bench's sections inside an NVTX range of its name, so that a
    profiler can take its launches alone (ncu --nvtx --nvtx-include name/)."""
    import torch

    torch.cuda.nvtx.range_push(name)
    try:
        return run()
    finally:
        torch.cuda.nvtx.range_pop()


def main():
    from nx_stereo_b200 import replicas

    args = parse()
    rank, world, local_rank = replicas.ranks()
    if args.impl == "reference":
        if rank != 0:
            return 0
        print(json.dumps(run_reference(args)))
        return 0
    if world > 1:
        import torch

        torch.cuda.set_device(local_rank)
        replicas.init("nccl", device=torch.device("cuda", local_rank))
    line = run_ours(args, rank, world, local_rank)
    if rank == 0 and world == 1:
        import torch

        from nx_stereo_b200 import native

        ctx = native.Context(local_rank)
        if not args.no_batch:
            line["batched"] = section("batched", lambda: bench_batched(torch, ctx))
        if not args.no_large:
            line["large_range"] = section("large_range", lambda: bench_large(torch, ctx))
        if not args.no_coarse_to_fine:
            line["coarse_to_fine"] = section("coarse_to_fine", lambda: bench_coarse_to_fine(torch, ctx))
        if not args.no_cpu_baseline:
            line["config0"] = section("config0", lambda: bench_config0(torch, ctx))
        ctx.close()
        if not args.no_serving:
            line["serving"] = section("serving", lambda: bench_serving())
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = host_threads()
        rig, frames = make_inputs(4, seed=1)
        value = cpu_sample(rig, frames, threads, threads)
        line["cpu_baseline"] = {"value": round(value, 3), "unit": "pairs/s", "cores": threads,
                                "kind": "port",
                                "sample": f"{threads} pairs, one per host thread (C port of the "
                                          "reference's Rust pipeline)"}
    if world > 1:
        import torch.distributed as td

        replicas.barrier()
        td.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))
    return 0


if __name__ == "__main__":
    sys.exit(main())
