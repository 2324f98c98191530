"""Batched matching: many rectified pairs of uneven size and disparity range
matched in one persistent, graph-captured launch (nxs_batch_* in
include/nx_stereo_b200.h), and the autotuner that picks the launch's shapes.

Each pair is matched exactly as NxStereo.sgm/3 matches it alone
(lib/nx_stereo.ex:64-74): the batch changes the schedule, never the integer
arithmetic, so every output is bit-identical to the single-pair call.

    plan = BatchPlan(context, [(640, 480, {"disparities": 128}), ...])
    plan.set_inputs(0, left, right)
    disparities = plan.run()          # host in, one launch, host out
    Autotuner().tune(plan)            # picks blocks, tile and queue shapes
"""
import ctypes
import hashlib
import json
import os

import numpy as np

from . import native

PHASES = ("census", "costs", "paths", "select", "check", "median")
TUNING_FIELDS = ("blocks_per_sm", "cost_rows", "select_passes", "group_pairs", "quantum_us",
                 "order", "path_words", "engine", "streams", "wait_limit_us")


def default_tuning():
    t = native.BatchTuning()
    native.load().nxs_batch_default_tuning(ctypes.byref(t))
    return {name: getattr(t, name) for name in TUNING_FIELDS}


def _tuning_struct(tuning):
    merged = default_tuning()
    if tuning:
        unknown = set(tuning) - set(TUNING_FIELDS)
        if unknown:
            raise ValueError(f"unknown tuning fields {sorted(unknown)}")
        merged.update(tuning)
    return native.BatchTuning(int(merged["blocks_per_sm"]), int(merged["cost_rows"]),
                              int(merged["select_passes"]), int(merged["group_pairs"]),
                              float(merged["quantum_us"]), int(merged["order"]),
                              int(merged["path_words"]), int(merged["engine"]),
                              int(merged["streams"]), int(merged["wait_limit_us"]))


def _pairs_struct(shapes):
    arr = (native.BatchPair * len(shapes))()
    for i, shape in enumerate(shapes):
        width, height, settings = _shape(shape)
        arr[i] = native.BatchPair(width, height, native.sgm_params(**settings))
    return arr


def _shape(shape):
    if isinstance(shape, dict):
        settings = dict(shape)
        return int(settings.pop("width")), int(settings.pop("height")), settings
    width, height = shape[0], shape[1]
    settings = dict(shape[2]) if len(shape) > 2 else {}
    return int(width), int(height), settings


def queue(shapes, tuning=None):
    """The work queue a plan of these pairs would run, computed on the host:
    (items, runs, total) with items[i, k] the items of phase k of pair i and
    runs[r] = (first position, pair, phase, first item of the phase)."""
    lib = native.load()
    pairs = _pairs_struct(shapes)
    t = _tuning_struct(tuning)
    n_runs = ctypes.c_uint32()
    buf = native._errbuf()
    native._check(lib.nxs_batch_queue(len(shapes), pairs, ctypes.byref(t), None, None, 0,
                                      ctypes.byref(n_runs), buf, 1024), buf)
    items = np.zeros((len(shapes), len(PHASES)), np.uint32)
    runs = np.zeros((n_runs.value, 4), np.uint32)
    native._check(lib.nxs_batch_queue(
        len(shapes), pairs, ctypes.byref(t),
        items.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
        runs.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), n_runs.value,
        ctypes.byref(n_runs), buf, 1024), buf)
    return items, runs, int(items.sum())


class _View:
    """An array interface over the plan's pinned memory that keeps the plan alive."""

    def __init__(self, plan, address, shape, dtype):
        self._plan = plan
        self.__array_interface__ = {"data": (address, False), "shape": shape,
                                    "typestr": np.dtype(dtype).str, "version": 3}


class _DeviceView:
    """__cuda_array_interface__ over device memory the plan owns."""

    def __init__(self, plan, address, shape, typestr):
        self._plan = plan
        self.__cuda_array_interface__ = {"data": (address, False), "shape": shape,
                                         "typestr": typestr, "version": 2, "strides": None}


class BatchPlan:
    """A planned batch: buffers for every pair, the work queue and two CUDA
    graphs (device-resident, and host in / host out)."""

    def __init__(self, context, shapes, tuning=None):
        self.context = context
        self.shapes = [_shape(s) for s in shapes]
        self._pairs = _pairs_struct(shapes)
        t = _tuning_struct(tuning)
        handle = ctypes.c_void_p()
        buf = native._errbuf()
        native._check(native.load().nxs_batch_create(context.handle, len(shapes), self._pairs,
                                                     ctypes.byref(t), ctypes.byref(handle),
                                                     buf, 1024), buf)
        self._handle = handle
        self._tuning = {name: getattr(t, name) for name in TUNING_FIELDS}

    def __len__(self):
        return len(self.shapes)

    @property
    def tuning(self):
        return dict(self._tuning)

    def _buffers(self, i, device_side):
        left, right, disparity = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        status = native.load().nxs_batch_buffers(self._handle, i, 1 if device_side else 0,
                                                 ctypes.byref(left), ctypes.byref(right),
                                                 ctypes.byref(disparity))
        native._check(status, None)
        return left.value, right.value, disparity.value

    def host_views(self, i):
        """(left, right, disparity) arrays over pair i's pinned host buffers."""
        width, height, _ = self.shapes[i]
        left, right, disparity = self._buffers(i, False)
        return (np.asarray(_View(self, left, (height, width), np.uint8)),
                np.asarray(_View(self, right, (height, width), np.uint8)),
                np.asarray(_View(self, disparity, (height, width), np.float32)))

    def device_buffers(self, i):
        """Device addresses of pair i's left, right and disparity."""
        return self._buffers(i, True)

    def device_views(self, i):
        """(left, right, disparity) torch tensors over pair i's device buffers
        (no copy; valid while the plan lives)."""
        import torch

        width, height, _ = self.shapes[i]
        views = []
        for address, typestr in zip(self._buffers(i, True), ("|u1", "|u1", "<f4")):
            views.append(torch.as_tensor(_DeviceView(self, address, (height, width), typestr),
                                         device=f"cuda:{self.context.device}"))
        return tuple(views)

    def set_inputs(self, i, left, right):
        l, r, _ = self.host_views(i)
        l[...] = left
        r[...] = right

    def run(self, copy=True):
        """Copies every pair in, matches the batch, copies the disparities out."""
        buf = native._errbuf()
        native._check(native.load().nxs_batch_run(self._handle, buf, 1024), buf)
        outputs = [self.host_views(i)[2] for i in range(len(self))]
        return [o.copy() for o in outputs] if copy else outputs

    def launch(self, host_buffers=False, stream=None):
        """Enqueues one run without waiting (stream: a cudaStream_t address)."""
        buf = native._errbuf()
        native._check(native.load().nxs_batch_launch(self._handle, 1 if host_buffers else 0,
                                                     stream, buf, 1024), buf)

    def check(self):
        buf = native._errbuf()
        native._check(native.load().nxs_batch_check(self._handle, buf, 1024), buf)

    def retune(self, **tuning):
        merged = self.tuning
        merged.update(tuning)
        t = _tuning_struct(merged)
        buf = native._errbuf()
        native._check(native.load().nxs_batch_retune(self._handle, ctypes.byref(t), buf, 1024),
                      buf)
        self._tuning = {name: getattr(t, name) for name in TUNING_FIELDS}

    def clocks(self):
        """SM cycles summed over blocks in the last launch: {phase: working},
        {"wait " + phase: waiting for the phase before}, {"take": taking items}."""
        cycles = (ctypes.c_uint64 * 16)()
        native._check(native.load().nxs_batch_clocks(self._handle, cycles), None)
        names = PHASES + tuple("wait " + p for p in PHASES) + ("take",)
        return dict(zip(names, list(cycles)))

    def stats(self):
        s = native.BatchStats()
        native._check(native.load().nxs_batch_info(self._handle, ctypes.byref(s)), None)
        return {name: getattr(s, name) for name, _ in native.BatchStats._fields_}

    def disparities(self):
        """Σ width x height x disparities over the pairs (the Mdisp/s numerator)."""
        return sum(w * h * s.get("disparities", 64) for w, h, s in self.shapes)

    def close(self):
        if getattr(self, "_handle", None):
            native.load().nxs_batch_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# The autotuner's search space: one coordinate at a time from the current
# best, for `sweeps` sweeps.
SEARCH = {
    "engine": (0, 1),
    "streams": (4, 8, 16, 32),
    "path_words": (8, 16),
    "order": (0, 1),
    "group_pairs": (2, 4, 8, 16),
    "blocks_per_sm": (6, 8),
    "select_passes": (4, 8, 16),
    "cost_rows": (1, 2, 4),
    "quantum_us": (1.0, 2.0, 4.0),
}


class Autotuner:
    """Times a plan's launch under candidate shapes (CUDA events on the
    launching stream, median of `repeats` after a warm-up) and keeps the
    fastest; results are cached by the batch's composition and device."""

    def __init__(self, cache_path=None, repeats=3, sweeps=2, search=None):
        self.cache_path = cache_path
        self.repeats = repeats
        self.sweeps = sweeps
        self.search = dict(search or SEARCH)
        self.trials = []  # (tuning, ms) in the order they were timed

    @staticmethod
    def key(plan):
        import torch

        shapes = sorted((w, h, int(s.get("disparities", 64)), int(s.get("paths", 8)))
                        for w, h, s in plan.shapes)
        name = torch.cuda.get_device_name(plan.context.device)
        digest = hashlib.sha256(json.dumps([name, shapes]).encode()).hexdigest()[:16]
        return f"{name}:{len(shapes)}:{digest}"

    def _load(self):
        if self.cache_path and os.path.exists(self.cache_path):
            with open(self.cache_path) as f:
                return json.load(f)
        return {}

    def _store(self, key, tuning, ms):
        if not self.cache_path:
            return
        cache = self._load()
        cache[key] = {"tuning": tuning, "ms": ms}
        os.makedirs(os.path.dirname(os.path.abspath(self.cache_path)), exist_ok=True)
        with open(self.cache_path, "w") as f:
            json.dump(cache, f, indent=1, sort_keys=True)

    def time(self, plan, tuning):
        import torch

        plan.retune(**tuning)
        stream = torch.cuda.Stream(device=plan.context.device)
        handle = stream.cuda_stream
        with torch.cuda.stream(stream):
            plan.launch(stream=handle)
            times = []
            for _ in range(self.repeats):
                start = torch.cuda.Event(enable_timing=True)
                end = torch.cuda.Event(enable_timing=True)
                start.record(stream)
                plan.launch(stream=handle)
                end.record(stream)
                end.synchronize()
                times.append(start.elapsed_time(end))
        plan.check()
        ms = float(np.median(times))
        self.trials.append((dict(plan.tuning), ms))
        return ms

    def tune(self, plan, use_cache=True):
        """Leaves the plan on the fastest shapes found; returns (tuning, ms)."""
        key = self.key(plan)
        if use_cache:
            hit = self._load().get(key)
            if hit:
                plan.retune(**hit["tuning"])
                return plan.tuning, hit["ms"]
        best = plan.tuning
        best_ms = self.time(plan, best)
        for _ in range(self.sweeps):
            improved = False
            for name, values in self.search.items():
                candidates = [dict(best, **{name: value}) for value in values
                              if value != best[name]]
                if name == "engine":  # the stream engine, with every stream count searched
                    candidates = [dict(c, streams=n) for c in candidates
                                  for n in (self.search.get("streams") or (c["streams"],))
                                  if c["engine"] == 1] + [c for c in candidates
                                                           if c["engine"] != 1]
                for candidate in candidates:
                    try:
                        ms = self.time(plan, candidate)
                    except native.NativeError:  # a combination the plan refuses
                        plan.retune(**best)
                        continue
                    if ms < best_ms * 0.995:
                        best, best_ms, improved = dict(plan.tuning), ms, True
            if not improved:
                break
        plan.retune(**best)
        self._store(key, best, best_ms)
        return plan.tuning, best_ms


def sample_shapes(count, seed, sizes=((320, 240), (480, 270), (640, 480), (728, 544),
                                      (1280, 720)),
                  disparities=(64, 96, 128, 192), paths=8):
    """Seeded random pair shapes drawn from `sizes` x `disparities`."""
    rng = np.random.default_rng(seed)
    shapes = []
    for _ in range(count):
        w, h = sizes[int(rng.integers(len(sizes)))]
        d = int(disparities[int(rng.integers(len(disparities)))])
        shapes.append((w, h, {"disparities": d, "paths": paths}))
    return shapes


def main(argv=None):
    """python -m nx_stereo_b200.batch [--pairs N] [--size WxH] [--disparities D]
    [--runs R]: matches N synthetic pairs of one shape as one batch R times
    (host buffers in and out) and prints the plan's statistics."""
    import argparse

    from . import scene

    p = argparse.ArgumentParser(description=main.__doc__)
    p.add_argument("--pairs", type=int, default=4)
    p.add_argument("--size", default="728x544")
    p.add_argument("--disparities", type=int, default=128)
    p.add_argument("--runs", type=int, default=2)
    args = p.parse_args(argv)
    width, height = (int(v) for v in args.size.split("x"))
    context = native.Context(0)
    shapes = [(width, height, {"disparities": args.disparities})] * args.pairs
    plan = BatchPlan(context, shapes)
    for i in range(args.pairs):
        plan.set_inputs(i, *scene.rectified_pair(width, height, seed=50 + i,
                                                 max_disparity=min(56, args.disparities - 8)))
    for _ in range(args.runs):
        plan.run(copy=False)
    print(plan.stats())
    plan.close()
    context.close()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
