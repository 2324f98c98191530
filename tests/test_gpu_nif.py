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
    # a run past its timeout fails, and so does the one behind it
    left, right = pairs[0]
    run = pc.run_record(21, seg.inputs, [("left", left), ("right", right)])
    for k, timeout in enumerate((0, 30000)):
        nif.call("run", ctx, nif.binary(run), nif.lib.fake_pid(9), nif.lib.fake_ref(200 + k),
                 nif.lib.fake_int(timeout))
    assert nif.message() == "#PID<9> {#Ref<200>, {:error, :timeout}}"
    assert nif.message() == "#PID<9> {#Ref<201>, {:error, :timeout}}"
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
