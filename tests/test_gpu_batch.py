"""The batched launch on the GPU: every pair of a mixed batch (sizes and
disparity ranges drawn as the batched workload draws them, 3 and 8 paths,
several penalties, the stage mask on and off) comes out bit-identical to the
single-pair matcher, which the oracle pins; runs repeat exactly, the queue
never times out, re-tuning changes nothing in the results, the device-side
launch agrees with the host-buffer run, the engine that runs each pair's
single-pair kernels on forked streams gives the same results, and the
autotuner leaves a valid, equally exact plan."""
import numpy as np
import pytest

from tests import gpu_util as g

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from nx_stereo_b200 import native

    c = native.Context(0)
    yield c
    c.close()


def _inputs(shapes, seed):
    from nx_stereo_b200 import scene

    pairs = []
    for i, (w, h, s) in enumerate(shapes):
        d = s.get("disparities", 64)
        pairs.append(scene.rectified_pair(w, h, seed=seed + i, rectangles=6,
                                          max_disparity=min(56, d - 8)))
    return pairs


def _plan(ctx, shapes, pairs, tuning=None):
    from nx_stereo_b200 import batch

    plan = batch.BatchPlan(ctx, shapes, tuning)
    for i, (left, right) in enumerate(pairs):
        plan.set_inputs(i, left, right)
    return plan


MIXED = [
    (97, 31, {"disparities": 64, "paths": 3}),
    (64, 48, {"disparities": 64, "p1": 0, "p2": 1, "uniqueness": 1.0}),
    (320, 240, {"disparities": 96}),
    (480, 270, {"disparities": 192, "stage_mask": True}),
    (131, 77, {"disparities": 128, "paths": 3, "p1": 78, "p2": 79, "uniqueness": 2.5}),
    (640, 480, {"disparities": 128, "p1": 4, "p2": 40, "uniqueness": 1.2}),
    (728, 544, {"disparities": 128, "stage_mask": True}),
    (200, 100, {"disparities": 256}),
]


def test_a_mixed_batch_matches_single_pair_runs_bit_for_bit(ctx, oracle):
    pairs = _inputs(MIXED, 100)
    plan = _plan(ctx, MIXED, pairs)
    outputs = plan.run()
    for (w, h, s), (left, right), got in zip(MIXED, pairs, outputs):
        assert got.shape == (h, w)
        want = ctx.sgm(left, right, **s)
        assert g.same_bits(got, want), (w, h, s)
    # the small ones against the oracle directly
    for i in (0, 1, 4):
        (w, h, s), (left, right) = MIXED[i], pairs[i]
        want = oracle.sgm(left, right, s.get("disparities", 64), s.get("paths", 8),
                          s.get("p1", 8), s.get("p2", 64), s.get("uniqueness", 1.0526315789473684))
        assert g.same_bits(outputs[i], want)
    plan.close()


def test_the_batched_workload_64_pairs(ctx):
    from nx_stereo_b200 import batch

    shapes = batch.sample_shapes(64, seed=2024)
    pairs = _inputs(shapes, 7000)
    plan = _plan(ctx, shapes, pairs)
    first = plan.run()
    for (w, h, s), (left, right), got in zip(shapes, pairs, first):
        assert g.same_bits(got, ctx.sgm(left, right, **s)), (w, h, s)
    second = plan.run()  # the graph replays over the same buffers
    assert all(g.same_bits(a, b) for a, b in zip(first, second))
    assert sum((o > 0).mean() for o in first) / len(first) > 0.5
    plan.close()


def test_retuning_changes_nothing_but_speed(ctx):
    shapes = MIXED[2:6]
    pairs = _inputs(shapes, 300)
    plan = _plan(ctx, shapes, pairs)
    want = plan.run()
    for tuning in ({"blocks_per_sm": 4, "cost_rows": 1, "select_passes": 1, "quantum_us": 1.0,
                    "group_pairs": 1},
                   {"blocks_per_sm": 6, "cost_rows": 4, "select_passes": 16, "group_pairs": 3,
                    "quantum_us": 8.0},
                   {"order": 1},
                   {"engine": 1, "streams": 4},
                   {"engine": 1, "streams": 1}):
        plan.retune(**tuning)
        assert all(plan.tuning[k] == v for k, v in tuning.items())
        got = plan.run()
        assert all(g.same_bits(a, b) for a, b in zip(got, want))
    plan.close()


def test_device_launch_matches_the_host_run(ctx):
    torch = g.torch()
    shapes = MIXED[:4]
    pairs = _inputs(shapes, 400)
    plan = _plan(ctx, shapes, pairs)
    want = plan.run()
    # Fill the device inputs from torch tensors, clear the device outputs and
    # launch on torch's stream, without the host copies.
    for i, (left, right) in enumerate(pairs):
        dl, dr, dd = plan.device_views(i)
        dl.copy_(g.dev(left))
        dr.copy_(g.dev(right))
        dd.fill_(7.0)
        plan.set_inputs(i, np.zeros_like(left), np.zeros_like(right))  # host side unused
    plan.launch(host_buffers=False, stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    plan.check()
    for i in range(len(shapes)):
        assert g.same_bits(plan.device_views(i)[2].cpu().numpy(), want[i])
    plan.close()


def test_the_autotuner_leaves_an_exact_plan(ctx, tmp_path):
    from nx_stereo_b200 import batch

    shapes = MIXED[2:6]
    pairs = _inputs(shapes, 500)
    plan = _plan(ctx, shapes, pairs)
    want = plan.run()
    tuner = batch.Autotuner(cache_path=str(tmp_path / "tuning.json"), repeats=2, sweeps=1,
                            search={"blocks_per_sm": (4, 8), "cost_rows": (1, 2),
                                    "quantum_us": (2.0, 4.0)})
    tuning, ms = tuner.tune(plan)
    assert ms > 0 and len(tuner.trials) >= 4
    assert all(g.same_bits(a, b) for a, b in zip(plan.run(), want))
    # the cache answers the same batch without timing again
    again = batch.Autotuner(cache_path=str(tmp_path / "tuning.json"))
    assert again.tune(plan)[0] == tuning and not again.trials
    plan.close()


def test_a_batch_too_big_for_the_device_is_refused(ctx):
    from nx_stereo_b200 import batch, native

    with pytest.raises(native.NativeError, match="GB of device memory"):
        batch.BatchPlan(ctx, [(4096, 4096, {"disparities": 256})] * 16)


def test_the_streams_engine_on_the_mixed_batch(ctx):
    pairs = _inputs(MIXED, 600)
    plan = _plan(ctx, MIXED, pairs, {"engine": 1, "streams": 3})
    for (w, h, s), (left, right), got in zip(MIXED, pairs, plan.run()):
        assert g.same_bits(got, ctx.sgm(left, right, **s)), (w, h, s)
    plan.close()


def test_a_dependency_no_launch_meets_times_out_at_the_plans_limit(ctx):
    """The persistent launch's waits are bounded: with one selection planned
    to wait for a path item that does not exist, the launch ends after the
    plan's 1 ms limit (not the 2 s default) with NXS_TIMEOUT, and a fresh
    plan of the same batch meets every dependency again, results unchanged."""
    import time

    from nx_stereo_b200 import native

    shapes = [(97, 31, {"disparities": 64}), (64, 48, {"disparities": 64, "paths": 3})]
    plan = _plan(ctx, shapes, _inputs(shapes, 300), {"engine": 0, "wait_limit_us": 1000})
    want = plan.run()
    plan.check()
    buf = native._errbuf()
    native._check(native.load().nxs_batch_hold_phase(plan._handle, 1, 3, buf, 1024), buf)
    started = time.monotonic()
    with pytest.raises(native.NativeError) as raised:
        plan.run()
    assert raised.value.status == native.TIMEOUT
    assert "0.001000 s" in raised.value.message
    assert time.monotonic() - started < 1.0
    with pytest.raises(native.NativeError):
        plan.check()
    plan.retune()
    got = plan.run()
    plan.check()
    for a, b in zip(got, want):
        assert g.same_bits(a, b)
    plan.close()
