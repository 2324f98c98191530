"""A segment's failure paths, made on the host (no device): a fake of the
library's context and requests stands in for the C ABI, so a reply can be
held back, a run can fail, a device error can surface while waiting, and a
configuration can be refused. CudaSegment must answer as the reference's
Matcher does (test/nx_stereo/matcher_test.exs:85-131 and
lib/nx_stereo/matcher.ex:107-146): a request with no reply within its
timeout gives "timeout" and the caller may wait again; a failed run fails
that request only ("error", reason) and the next pair goes through; a
refused configuration stops the segment ("stop", reason).
"""
import numpy as np
import pytest

from nx_stereo_b200 import native, segment, stage


class FakeRequest:
    """A request whose reply arrives after `ready_after` waits, or fails."""

    def __init__(self, outputs, ready_after=0, fail=None):
        self._outputs = outputs
        self._ready_after = ready_after
        self._fail = fail
        self.freed = False
        self.waits = []

    def poll(self):
        return self._ready_after <= 0

    def wait(self, timeout_ms=-1):
        self.waits.append(timeout_ms)
        if self._fail:
            raise native.NativeError(native.CUDA_ERROR, self._fail)
        if self._ready_after > 0:
            self._ready_after -= 1
            return False
        return True

    def outputs(self, copy=True):
        return dict(self._outputs)

    def times_us(self):
        return [1] * 5

    def free(self):
        self.freed = True


class FakeContext:
    """Records what the segment asks of the library and answers as told."""

    def __init__(self):
        self.configured = []
        self.runs = 0
        self.refuse_configuration = None
        self.fail_next_run = None
        self.next_request = None

    def configure(self, segment_id, geometry, members):
        if self.refuse_configuration:
            raise native.NativeError(native.BAD_ARGUMENT, self.refuse_configuration)
        self.configured.append((segment_id, geometry, [kind for kind, _ in members]))

    def run_async(self, segment_id, params, entries, done=None, tag=0):
        self.runs += 1
        if self.fail_next_run:
            reason, self.fail_next_run = self.fail_next_run, None
            raise native.NativeError(native.BAD_ARGUMENT, reason)
        request, self.next_request = self.next_request, None
        if request is None:
            h, w = entries["left"].shape
            request = FakeRequest({"disparity": np.full((h, w), 3.5, np.float32)})
        return request

    def release(self, segment_id):
        pass


@pytest.fixture
def fake(monkeypatch):
    ctx = FakeContext()
    monkeypatch.setattr(segment, "context", lambda device=0: ctx)
    return ctx


def _segment(w=64, h=48):
    geometry = segment.standard_geometry(w, h)
    status, members = segment.members([(stage.Disparity, {"num_disparities": 64})], geometry)
    assert status == "ok", members
    status, built = segment.CudaSegment.build(members, geometry)
    assert status == "ok", built
    return built


def _entries(w=64, h=48):
    return {"left": np.zeros((h, w), np.uint8), "right": np.zeros((h, w), np.uint8)}


def test_a_reply_that_is_late_times_out_and_can_be_waited_for_again(fake):
    seg = _segment()
    fake.next_request = FakeRequest({"disparity": np.zeros((48, 64), np.float32)}, ready_after=2)
    status, request = segment.CudaSegment.send_request(_entries(), seg)
    assert status == "ok"
    assert segment.CudaSegment.await_(request, seg, 50) == "timeout"
    assert segment.CudaSegment.await_(request, seg, 50) == "timeout"
    reply = segment.CudaSegment.await_(request, seg, 50)
    assert reply[0] == "ok" and set(reply[1]) == {"disparity"}
    assert request.waits == [50, 50, 50]
    # segment.run passes the timeout through and gives "timeout" too.
    fake.next_request = FakeRequest({"disparity": np.zeros((48, 64), np.float32)}, ready_after=1)
    assert segment.run(segment.CudaSegment, _entries(), seg, 10) == "timeout"


def test_response_recognises_only_its_own_finished_request(fake):
    seg = _segment()
    late = FakeRequest({"disparity": np.zeros((48, 64), np.float32)}, ready_after=1)
    fake.next_request = late
    _, request = segment.CudaSegment.send_request(_entries(), seg)
    assert segment.CudaSegment.response(object(), request, seg) == ("no_reply",)
    assert segment.CudaSegment.response(request, request, seg) == ("no_reply",)
    late._ready_after = 0
    assert segment.CudaSegment.response(request, request, seg)[0] == "ok"


def test_a_failed_run_fails_that_pair_only(fake):
    seg = _segment()
    fake.fail_next_run = "the device has no room for this pair"
    status, request = segment.CudaSegment.send_request(_entries(), seg)
    assert status == "ok"
    assert segment.CudaSegment.await_(request, seg, 100) == \
        ("error", "the device has no room for this pair")
    reply = segment.run(segment.CudaSegment, _entries(), seg, 100)
    assert reply[0] == "ok" and (reply[1]["disparity"] == 3.5).all()
    assert fake.runs == 2 and len(fake.configured) == 1


def test_a_device_error_while_waiting_fails_the_pair_and_frees_its_request(fake):
    seg = _segment()
    broken = FakeRequest({}, fail="an illegal memory access was encountered")
    fake.next_request = broken
    _, request = segment.CudaSegment.send_request(_entries(), seg)
    assert segment.CudaSegment.await_(request, seg, -1) == \
        ("error", "an illegal memory access was encountered")
    assert broken.freed


def test_a_refused_configuration_stops_the_segment_and_is_tried_again(fake):
    seg = _segment()
    fake.refuse_configuration = "width 64 is below the smallest the kernels take"
    _, request = segment.CudaSegment.send_request(_entries(), seg)
    assert segment.CudaSegment.await_(request, seg, 100) == \
        ("stop", "width 64 is below the smallest the kernels take")
    assert fake.runs == 0
    # Not configured, so the next pair configures again (and now succeeds).
    fake.refuse_configuration = None
    assert segment.run(segment.CudaSegment, _entries(), seg, 100)[0] == "ok"
    assert len(fake.configured) == 1


def test_entries_that_do_not_fit_are_refused_before_the_device(fake):
    seg = _segment()
    assert segment.CudaSegment.send_request({"left": np.zeros((48, 64), np.uint8)}, seg) == \
        ("error", ("missing_entry", "right"))
    wrong = {"left": np.zeros((47, 64), np.uint8), "right": np.zeros((48, 64), np.uint8)}
    assert segment.CudaSegment.send_request(wrong, seg) == \
        ("error", ("frame_size", "left", (47, 64), (48, 64)))
    assert fake.runs == 0 and fake.configured == []


def test_a_reload_configures_again_on_the_next_pair(fake):
    seg = _segment()
    assert segment.run(segment.CudaSegment, _entries(), seg, 100)[0] == "ok"
    assert segment.run(segment.CudaSegment, _entries(), seg, 100)[0] == "ok"
    assert len(fake.configured) == 1
    segment.CudaSegment.reload(seg, seg.members, seg.geometry)
    assert segment.run(segment.CudaSegment, _entries(), seg, 100)[0] == "ok"
    assert len(fake.configured) == 2
