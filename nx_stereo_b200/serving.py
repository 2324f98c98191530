"""Serving many camera streams on one GPU.

A request loop admits stereo pairs from many camera streams as they arrive
and keeps every admitted stream's work on the device at once: each stream is a
CudaSegment (Rectification -> Disparity -> SpeckleFilter -> TemporalFilter ->
Depth -> Quality by default) whose carried state (the temporal filter's and
the quality stage's previous disparity, the rectification maps' cameras)
stays on the device, with its own upload, compute and download streams and
CudaSegment.DEPTH request slots. A pair that arrives while others are on the
GPU is sent as soon as its stream has a free slot, so pairs of different
streams overlap on the device; a stream's pairs stay in order (its carried
state depends on it, lib/nx_stereo/native_segment.ex:164-171).

Admission is sized by device memory: a stream is opened only while the
device memory its segment needs (the cost and path volumes of its matcher,
its slots' buffers) fits in the free HBM measured when the server started,
less a reserve; a stream that does not fit waits until another closes.

Latency is measured per pair from its arrival to the device finishing it
(CLOCK_MONOTONIC on both sides), and reported as p50 and p99 with the
percentile rule of the reference's stream benchmark, index ceil(n p) - 1
(test/bench/stream.exs:223).
"""
import collections
import gc
import heapq
import math
import time

import numpy as np

from . import segment as segment_module
from . import stage as stage_module

SERVING_PIPELINE = [stage_module.Rectification, (stage_module.Disparity, {"num_disparities": 128}),
                    stage_module.SpeckleFilter, stage_module.TemporalFilter, stage_module.Depth,
                    stage_module.Quality]


def percentile(values, p):
    """The p-th quantile (0 < p <= 1) by the rule index = ceil(n p) - 1."""
    ordered = sorted(values)
    if not ordered:
        return float("nan")
    return ordered[max(0, math.ceil(len(ordered) * p) - 1)]


def stream_bytes(geometry, stages, depth):
    """Device bytes a stream's segment holds: for each compute lane its
    matcher's volumes (costs, path volumes, per-pixel maps), its depth map and,
    with a Rectification member, its rectification maps; `depth` slots of
    frames, images and per-pixel outputs; the carried state. A segment has two
    compute lanes unless a stage carrying state keeps it on one (no split
    matcher: a carrying stage before the Disparity member, or no full search)."""
    from . import native

    w, h = geometry["width"], geometry["height"]
    fw, fh = geometry.get("frame_width", w), geometry.get("frame_height", h)
    d = 64
    modules = [entry[0] if isinstance(entry, tuple) else entry for entry in stages]
    full_search, carries, carries_before = False, False, False
    for entry, module in zip(stages, modules):
        settings = entry[1] if isinstance(entry, tuple) else {}
        if module is stage_module.Disparity:
            d = int(settings.get("num_disparities", 64))
            full_search = settings.get("search", "full") != "coarse_to_fine"
            carries_before = carries
        if module in (stage_module.TemporalFilter, stage_module.Quality):
            carries = True
    lanes = 1 if carries and (carries_before or not full_search) else 2
    px = w * h
    scratch = int(native.load().nxs_sgm_scratch_bytes(w, h, d))
    maps = 16 * px if stage_module.Rectification in modules else 0
    slot = 2 * fw * fh + 2 * px + 4 * (4 * px) + 2 * px
    carried = 4 * (4 * px)
    return lanes * (scratch + 4 * px + maps) + depth * slot + carried


Completed = collections.namedtuple("Completed", "stream seq arrival_ns done_ns outputs")


class _Device:
    """The device side of the server: CudaSegments on one GPU."""

    def __init__(self, device=0):
        self.device = device
        self.depth = segment_module.CudaSegment.DEPTH

    def memory(self):
        return segment_module.context(self.device).memory()

    def open(self, geometry, stages):
        status, members = segment_module.members(stages, geometry)
        if status != "ok":
            raise ValueError(f"the stream's stages: {members}")
        status, seg = segment_module.CudaSegment.build(members, geometry, {"device": self.device})
        if status != "ok":
            raise ValueError(f"the stream's stages: {seg}")
        return seg

    def send(self, seg, entries):
        status, request = segment_module.CudaSegment.send_request(entries, seg)
        if status != "ok":
            raise ValueError(f"the pair's entries: {request}")
        return request

    def done(self, request):
        return segment_module._done(request)

    def finish(self, seg, request):
        """(outputs, done_ns) of a finished request."""
        reply = segment_module.CudaSegment.await_(request, seg, 0)
        if reply[0] != "ok":
            raise RuntimeError(f"a pair failed: {reply}")
        return reply[1], request.done_ns()

    def close(self, seg):
        seg.release()


class _Stream:
    def __init__(self, sid, geometry, stages, need):
        self.id = sid
        self.geometry = geometry
        self.stages = stages
        self.need = need
        self.segment = None
        self.waiting = collections.deque()  # (seq, entries, arrival_ns) not yet sent
        self.in_flight = collections.deque()  # (seq, request, arrival_ns), in order
        self.sent = 0


class Server:
    """Admits pairs of many streams as they arrive; see the module."""

    def __init__(self, device=0, reserve_bytes=2 << 30, backend=None, max_in_flight=None):
        """max_in_flight: at most this many pairs on the device at once, the
        oldest arrivals first (None: every stream's slots)."""
        self.backend = backend or _Device(device)
        self.cap = max_in_flight
        self.ready = collections.deque()  # stream ids of waiting pairs, in arrival order
        self._in_flight = 0
        free, _ = self.backend.memory()
        self.budget = max(0, free - reserve_bytes)
        self.used = 0
        self.streams = {}
        self.pending = collections.deque()  # streams waiting for memory, in order
        self._next_id = 0
        self.max_in_flight = 0

    # -- streams
    def open(self, geometry, stages=None):
        """A new stream; it starts once its memory fits (admitted(id))."""
        stages = stages or SERVING_PIPELINE
        sid = self._next_id
        self._next_id += 1
        stream = _Stream(sid, geometry, stages, stream_bytes(geometry, stages,
                                                             self.backend.depth))
        self.streams[sid] = stream
        self.pending.append(stream)
        self._admit()
        return sid

    def admitted(self, sid):
        return self.streams[sid].segment is not None

    def close(self, sid):
        """Ends a stream after its pairs finish; its memory goes to waiting streams."""
        stream = self.streams[sid]
        results = []
        while stream.in_flight or stream.waiting:
            results += self.poll(wait=True)
        if stream.segment is not None:
            self.backend.close(stream.segment)
            self.used -= stream.need
        elif stream in self.pending:
            self.pending.remove(stream)
        del self.streams[sid]
        self._admit()
        return results

    def _admit(self):
        while self.pending and self.used + self.pending[0].need <= self.budget:
            stream = self.pending.popleft()
            stream.segment = self.backend.open(stream.geometry, stream.stages)
            self.used += stream.need
        self._pump()

    # -- pairs
    def submit(self, sid, entries, arrival_ns=None):
        """Queues a pair of stream `sid`; it goes to the device as soon as the
        stream is admitted and has a free slot. Returns its sequence number."""
        stream = self.streams[sid]
        seq = stream.sent + len(stream.waiting) + len(stream.in_flight)
        arrival = time.monotonic_ns() if arrival_ns is None else arrival_ns
        stream.waiting.append((seq, entries, arrival))
        self.ready.append(sid)
        self._pump()
        return seq

    def _pump(self):
        """Sends waiting pairs, oldest arrival first, while the cap allows and
        their streams are admitted and have a free slot."""
        if not self.ready:
            return
        skipped = collections.deque()
        while self.ready and (self.cap is None or self._in_flight < self.cap):
            sid = self.ready.popleft()
            stream = self.streams.get(sid)
            if stream is None:
                continue
            if stream.segment is None or len(stream.in_flight) >= self.backend.depth:
                skipped.append(sid)  # its stream is busy: later arrivals may go first
                continue
            seq, entries, arrival = stream.waiting.popleft()
            request = self.backend.send(stream.segment, entries)
            stream.in_flight.append((seq, request, arrival))
            self._in_flight += 1
        skipped.extend(self.ready)
        self.ready = skipped
        self.max_in_flight = max(self.max_in_flight, self._in_flight)

    def in_flight(self):
        return self._in_flight

    def poll(self, wait=False):
        """The pairs finished since the last poll, oldest first per stream."""
        done = []
        while True:
            for stream in list(self.streams.values()):
                while stream.in_flight and self.backend.done(stream.in_flight[0][1]):
                    seq, request, arrival = stream.in_flight.popleft()
                    outputs, done_ns = self.backend.finish(stream.segment, request)
                    done.append(Completed(stream.id, seq, arrival, done_ns, outputs))
                    stream.sent += 1
                    self._in_flight -= 1
            self._pump()
            if done or not wait or not self.in_flight():
                return done
            time.sleep(50e-6)


# ---------------------------------------------------------------- the load
def synthetic_streams(count, sizes=((728, 544), (1280, 720)), frames=8, seed=0, drift=2.0):
    """`count` streams, stream i at sizes[i % len(sizes)] (fixed per stream):
    the rig of scene.rig over a piecewise-planar scene whose rectangles drift
    up to `drift` px a frame, as raw frame pairs. Streams of a size share the
    same `frames` frames, each starting at its own frame."""
    from . import scene

    by_size = {}
    for w, h in sizes:
        rig = scene.rig(w, h)
        pairs = []
        for f in range(frames):
            left, right = scene.rectified_pair(w, h, seed=seed + w, frame=f, drift=drift)
            lf, rf = scene.raw_frames(left, right, rig)
            pairs.append({"left_frame": lf, "right_frame": rf})
        by_size[(w, h)] = (segment_module.standard_geometry(w, h, the_rig=rig), pairs)
    streams = []
    for i in range(count):
        geometry, pairs = by_size[sizes[i % len(sizes)]]
        start = i // len(sizes)
        streams.append((geometry, [pairs[(start + k) % frames] for k in range(frames)]))
    return streams


def poisson_arrivals(count, rate_hz, duration_s, seed=0):
    """[(t_seconds, stream)] of `count` Poisson streams at `rate_hz` each."""
    rng = np.random.default_rng(seed)
    events = []
    for stream in range(count):
        t = rng.exponential(1.0 / rate_hz)
        while t < duration_s:
            events.append((t, stream))
            t += rng.exponential(1.0 / rate_hz)
    events.sort()
    return events


def run_load(server, stream_ids, frames_of, arrivals, lead_s=0.02):
    """Submits each arrival (t, stream index) at its time and collects every
    result. Returns {latencies_ms, pairs, seconds, pairs_per_s, p50_ms, p99_ms,
    max_in_flight}. frames_of[stream index] cycles through that stream's pairs.
    The interpreter's cyclic garbage collector is paused while the loop runs
    (after one collection), so that none of its passes stalls the loop."""
    gc_was_enabled = gc.isenabled()
    gc.collect()
    gc.disable()
    try:
        return _run_load(server, stream_ids, frames_of, arrivals, lead_s)
    finally:
        if gc_was_enabled:
            gc.enable()


def _run_load(server, stream_ids, frames_of, arrivals, lead_s):
    counters = collections.Counter()
    pending = list(arrivals)
    heapq.heapify(pending)
    t0 = time.monotonic_ns() + int(lead_s * 1e9)
    latencies, first, last = [], None, None
    total = len(pending)
    got = 0
    while got < total:
        now = time.monotonic_ns()
        busy = False
        while pending and t0 + int(pending[0][0] * 1e9) <= now:
            t, index = heapq.heappop(pending)
            frames = frames_of[index]
            entries = frames[counters[index] % len(frames)]
            counters[index] += 1
            arrival = t0 + int(t * 1e9)
            first = arrival if first is None else min(first, arrival)
            server.submit(stream_ids[index], entries, arrival_ns=arrival)
            busy = True
        for c in server.poll():
            latencies.append((c.done_ns - c.arrival_ns) / 1e6)
            last = c.done_ns if last is None else max(last, c.done_ns)
            got += 1
            busy = True
        if not busy:
            time.sleep(50e-6)
    seconds = (last - first) / 1e9 if got else float("nan")
    return {"latencies_ms": latencies, "pairs": got, "seconds": seconds,
            "pairs_per_s": got / seconds if got else 0.0,
            "p50_ms": percentile(latencies, 0.50), "p99_ms": percentile(latencies, 0.99),
            "max_in_flight": server.max_in_flight}


def warm(server, stream_ids, frames_of):
    """DEPTH pairs through every stream before timing: each segment is
    configured and each of its request slots has its pinned buffers."""
    for sid, frames in zip(stream_ids, frames_of):
        for k in range(server.backend.depth):
            server.submit(sid, frames[k % len(frames)])
    while server.in_flight():
        server.poll(wait=True)
    server.max_in_flight = 0
