"""The serving loop on the GPU: a stream's results are bit-identical alone and
in a mix of streams of two resolutions whose pairs overlap on the device (as
the reference's stream benchmark checks serial against overlapped runs,
test/bench/stream.exs:139-151), and a short Poisson load of 8 streams
completes every pair with its latency measured."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def streams():
    from nx_stereo_b200 import serving

    return serving.synthetic_streams(3, frames=4, seed=5)


def _results(server, completed):
    out = {}
    for c in completed:
        out[(c.stream, c.seq)] = {k: np.array(v) for k, v in c.outputs.items()
                                  if isinstance(v, np.ndarray)}
    return out


def test_a_stream_alone_and_in_the_mix(streams):
    from nx_stereo_b200 import serving

    geometry, frames = streams[0]
    alone = serving.Server(reserve_bytes=1 << 30)
    sid = alone.open(geometry)
    for f in frames:
        alone.submit(sid, f)
    alone_results = _results(alone, alone.close(sid))
    assert len(alone_results) == 4

    mixed = serving.Server(reserve_bytes=1 << 30)
    ids = [mixed.open(g) for g, _ in streams]
    for k in range(4):
        for sid_, (_, fr) in zip(ids, streams):
            mixed.submit(sid_, fr[k])
    assert mixed.in_flight() > 4  # pairs of several streams on the device together
    done = []
    while mixed.in_flight():
        done += mixed.poll(wait=True)
    mixed_results = _results(mixed, done)
    for k in range(4):
        a, m = alone_results[(sid, k)], mixed_results[(ids[0], k)]
        assert a.keys() == m.keys() and "disparity" in a
        for name in a:
            assert np.array_equal(a[name].view(np.uint8), m[name].view(np.uint8)), (k, name)
    # the third stream has the first one's size but its own frames
    assert not np.array_equal(mixed_results[(ids[2], 0)]["disparity"],
                              mixed_results[(ids[0], 0)]["disparity"])
    for sid_ in ids:
        mixed.close(sid_)


def test_a_short_poisson_load(streams):
    from nx_stereo_b200 import serving

    server = serving.Server(reserve_bytes=1 << 30)
    specs = [streams[i % 2] for i in range(8)]
    ids = [server.open(g) for g, _ in specs]
    frames_of = [fr for _, fr in specs]
    serving.warm(server, ids, frames_of)
    arrivals = serving.poisson_arrivals(8, 30.0, 0.5, seed=3)
    stats = serving.run_load(server, ids, frames_of, arrivals)
    assert stats["pairs"] == len(arrivals)
    assert 0 < stats["p50_ms"] <= stats["p99_ms"] < 1000
    for sid in ids:
        server.close(sid)
