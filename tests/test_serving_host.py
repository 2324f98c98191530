"""The serving loop's host logic with a stand-in device (no GPU): admission
by device memory (streams wait while their segment does not fit and start as
others close), each stream's pairs in order with at most DEPTH on the device,
pairs of different streams in flight together, the percentile rule of the
reference's stream benchmark, and Poisson arrivals at the offered rate."""
import time

import pytest

from nx_stereo_b200 import serving


class FakeDevice:
    """Requests finish `delay_s` after they are sent; memory as given."""

    depth = 2

    def __init__(self, free, delay_s=0.002):
        self.free = free
        self.delay_s = delay_s
        self.opened, self.closed, self.sent = [], [], []

    def memory(self):
        return self.free, self.free

    def open(self, geometry, stages):
        seg = {"geometry": geometry, "n": len(self.opened)}
        self.opened.append(seg)
        return seg

    def send(self, seg, entries):
        request = {"seg": seg, "entries": entries, "at": time.monotonic_ns()}
        self.sent.append(request)
        return request

    def done(self, request):
        return time.monotonic_ns() >= request["at"] + int(self.delay_s * 1e9)

    def finish(self, seg, request):
        return {"frame": request["entries"]["frame"]}, request["at"] + int(self.delay_s * 1e9)

    def close(self, seg):
        self.closed.append(seg)


GEOMETRY = {"width": 728, "height": 544}


def test_percentile_rule():
    values = list(range(1, 101))
    assert serving.percentile(values, 0.5) == 50
    assert serving.percentile(values, 0.99) == 99
    assert serving.percentile([7.0], 0.99) == 7.0
    assert serving.percentile([3, 1, 2], 0.5) == 2  # ceil(1.5) - 1 = 1 -> sorted[1]


def test_streams_wait_for_memory_and_start_as_others_close():
    need = serving.stream_bytes(GEOMETRY, serving.SERVING_PIPELINE, FakeDevice.depth)
    device = FakeDevice(free=2 * need + need // 2)
    server = serving.Server(reserve_bytes=0, backend=device)
    ids = [server.open(GEOMETRY) for _ in range(3)]
    assert [server.admitted(i) for i in ids] == [True, True, False]
    server.submit(ids[2], {"frame": 0})  # waits with its stream
    assert len(device.sent) == 0
    server.close(ids[0])
    assert server.admitted(ids[2])
    assert len(device.sent) == 1 and device.sent[0]["entries"] == {"frame": 0}
    while server.in_flight():
        server.poll(wait=True)


def test_each_stream_in_order_with_at_most_depth_in_flight():
    device = FakeDevice(free=1 << 40)
    server = serving.Server(reserve_bytes=0, backend=device)
    a, b = server.open(GEOMETRY), server.open(GEOMETRY)
    for k in range(5):
        server.submit(a, {"frame": k})
        server.submit(b, {"frame": 100 + k})
    assert server.in_flight() == 2 * FakeDevice.depth  # both streams at once
    done = []
    while len(done) < 10:
        done += server.poll(wait=True)
    for sid, base in ((a, 0), (b, 100)):
        mine = [c for c in done if c.stream == sid]
        assert [c.seq for c in mine] == list(range(5))
        assert [c.outputs["frame"] for c in mine] == [base + k for k in range(5)]
        assert all(c.done_ns >= c.arrival_ns for c in mine)
    assert server.max_in_flight == 4


def test_poisson_arrivals_at_the_offered_rate():
    events = serving.poisson_arrivals(32, 30.0, 10.0, seed=1)
    assert events == sorted(events)
    assert abs(len(events) - 32 * 30 * 10) < 4 * (32 * 30 * 10) ** 0.5
    assert {s for _, s in events} == set(range(32))


def test_a_load_run_completes_every_pair():
    device = FakeDevice(free=1 << 40, delay_s=0.001)
    server = serving.Server(reserve_bytes=0, backend=device)
    ids = [server.open(GEOMETRY) for _ in range(4)]
    frames = [[{"frame": k} for k in range(3)] for _ in ids]
    arrivals = serving.poisson_arrivals(4, 200.0, 0.2, seed=2)
    stats = serving.run_load(server, ids, frames, arrivals)
    assert stats["pairs"] == len(arrivals)
    assert 1.0 <= stats["p50_ms"] <= stats["p99_ms"] < 200.0
    assert stats["pairs_per_s"] > 0


def test_closing_waits_for_the_streams_pairs():
    device = FakeDevice(free=1 << 40)
    server = serving.Server(reserve_bytes=0, backend=device)
    a = server.open(GEOMETRY)
    for k in range(3):
        server.submit(a, {"frame": k})
    results = server.close(a)
    assert [c.seq for c in results] == [0, 1, 2]
    assert device.closed and not server.in_flight()


def test_a_cap_on_pairs_in_flight_sends_the_oldest_arrivals_first():
    device = FakeDevice(free=1 << 40)
    server = serving.Server(reserve_bytes=0, backend=device, max_in_flight=3)
    a, b, c = (server.open(GEOMETRY) for _ in range(3))
    order = [(a, 0), (b, 1), (a, 2), (c, 3), (b, 4), (c, 5)]
    for k, (sid, frame) in enumerate(order):
        server.submit(sid, {"frame": frame}, arrival_ns=k)
    assert server.in_flight() == 3
    assert [r["entries"]["frame"] for r in device.sent] == [0, 1, 2]
    done = []
    while len(done) < 6:
        done += server.poll(wait=True)
        assert server.in_flight() <= 3
    assert [r["entries"]["frame"] for r in device.sent] == [0, 1, 2, 3, 4, 5]
    assert server.max_in_flight == 3


def test_stream_bytes_count_each_compute_lane():
    """A segment holds a matcher scratch, a depth map and, with a Rectification
    member, rectification maps for each compute lane: two lanes unless a stage
    carrying state keeps it on one (a carrying stage before the Disparity member,
    or the coarse-to-fine search with one after it)."""
    from nx_stereo_b200 import native, stage

    g = {"width": 728, "height": 544}
    px = 728 * 544
    lane = int(native.load().nxs_sgm_scratch_bytes(728, 544, 128)) + 4 * px
    full = (stage.Disparity, {"num_disparities": 128})
    c2f = (stage.Disparity, {"num_disparities": 128, "search": "coarse_to_fine"})
    base = serving.stream_bytes(g, [full], 4)
    # stateless: two lanes; the state after a full search: still two (the split matcher)
    assert serving.stream_bytes(g, [full, stage.Depth], 4) == base
    assert serving.stream_bytes(g, [full, stage.TemporalFilter], 4) == base
    # the state before the matcher, or after a coarse-to-fine search: one lane
    assert serving.stream_bytes(g, [stage.TemporalFilter, full], 4) == base - lane
    assert serving.stream_bytes(g, [c2f, stage.Quality], 4) == base - lane
    assert serving.stream_bytes(g, [c2f], 4) == base
    # the rectification maps: 2 sides x (x, y) f32 a pixel, each lane
    assert serving.stream_bytes(g, [stage.Rectification, full], 4) == base + 2 * 16 * px
