"""The NIF on the GPU, under the fake Erlang runtime: a segment configured
from NativeSegment's record, pairs run and replied to by message in order
with the outputs record, each equal to CudaSegment's; a run past its timeout
fails with :timeout and so does the run behind it; a refused configuration;
and the owner's exit releasing its segment."""
import numpy as np
import pytest

from nx_stereo_b200 import segment, stage
from tests import port_client as pc
from tests.erts_stub import harness

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def nif():
    return harness.Nif()


def test_runs_reply_in_order_with_cuda_segments_outputs(nif):
    from nx_stereo_b200 import scene

    ok = nif.call("open", nif.lib.fake_int(0))
    text = nif.text(ok)
    assert text.startswith("{:ok, #Resource")
    ctx = _second(nif, ok)
    w, h = 364, 272
    geometry = segment.standard_geometry(w, h)
    status, members = segment.members(
        [(stage.Disparity, {"num_disparities": 64}), stage.SpeckleFilter, stage.Depth], geometry)
    status, seg = segment.CudaSegment.build(members, geometry)
    record = pc.configure_record(21, geometry, segment._configuration(seg))
    assert nif.text(nif.call("configure", ctx, nif.binary(record))) == ":ok"
    pairs = [scene.rectified_pair(w, h, seed=300 + k) for k in range(3)]
    for k, (left, right) in enumerate(pairs):
        run = pc.run_record(21, seg.inputs, [("left", left), ("right", right)])
        assert nif.text(nif.call("run", ctx, nif.binary(run), nif.lib.fake_pid(9),
                                 nif.lib.fake_ref(100 + k), nif.lib.fake_int(30000))) == ":ok"
    for k, (left, right) in enumerate(pairs):
        message = nif.message()
        prefix = f"#PID<9> {{#Ref<{100 + k}>, {{:ok, "
        assert message.startswith(prefix), message[:80]
        _, got = pc.decode_outputs(harness.hex_binary(message[len(prefix):-2]))
        status, want, seg = segment.run(segment.CudaSegment, {"left": left, "right": right}, seg,
                                        60000)
        for key in got:
            assert got[key].tobytes() == np.asarray(want[key]).astype(got[key].dtype).tobytes()
    # A run past its timeout fails, and so does the one sent behind it. A
    # large pair (ref 199, milliseconds of device work, a long timeout) holds
    # the waiter while the late run (ref 200: as much work, a 1 ms timeout)
    # and a small run behind it (ref 201) are sent: the device cannot finish
    # ref 200 within 1 ms of its sending, so it is late however soon the
    # waiter looks, and ref 201 is waiting behind it then.
    big_geometry = segment.standard_geometry(4096, 2160)
    status, big_members = segment.members([(stage.Disparity, {"num_disparities": 128})],
                                          big_geometry)
    status, big = segment.CudaSegment.build(big_members, big_geometry)
    record = pc.configure_record(23, big_geometry, segment._configuration(big))
    assert nif.text(nif.call("configure", ctx, nif.binary(record))) == ":ok"
    big_left, big_right = scene.rectified_pair(4096, 2160, seed=7)
    big_run = pc.run_record(23, big.inputs, [("left", big_left), ("right", big_right)])
    left, right = pairs[0]
    run = pc.run_record(21, seg.inputs, [("left", left), ("right", right)])
    for ref, record, timeout in ((199, big_run, 30000), (200, big_run, 1), (201, run, 30000)):
        assert nif.text(nif.call("run", ctx, nif.binary(record), nif.lib.fake_pid(9),
                                 nif.lib.fake_ref(ref), nif.lib.fake_int(timeout))) == ":ok"
    assert nif.message().startswith("#PID<9> {#Ref<199>, {:ok, ")
    assert nif.message() == "#PID<9> {#Ref<200>, {:error, :timeout}}"
    assert nif.message() == "#PID<9> {#Ref<201>, {:error, :timeout}}"
    nif.call("release", ctx, nif.lib.fake_int(23))
    big.release()
    # the owner's exit releases the segment
    assert nif.text(nif.call("watch", ctx, nif.lib.fake_pid(9), nif.lib.fake_int(21))) == ":ok"
    nif.lib.fake_process_down(9)
    refused = nif.text(nif.call("run", ctx, nif.binary(run), nif.lib.fake_pid(9),
                                nif.lib.fake_ref(300), nif.lib.fake_int(1000)))
    assert refused == "{:error, <<" + b"segment 21 is not configured".hex() + ">>}"
    bad = pc.configure_record(22, geometry, [("median_filter", {"kernel_size": 5.0})])
    reply = nif.text(nif.call("configure", ctx, nif.binary(bad)))
    assert reply.startswith("{:error, {:configuration_refused, <<")
    seg.release()


def _second(nif, tuple_term):
    """The second element of a 2-tuple term of the fake runtime."""
    import ctypes

    fn = getattr(nif.lib, "fake_tuple_item", None)
    if fn is None:
        raise RuntimeError("fake_tuple_item missing")
    fn.restype, fn.argtypes = ctypes.c_size_t, [ctypes.c_size_t, ctypes.c_int]
    return fn(tuple_term, 1)
