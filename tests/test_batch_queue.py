"""The batched launch's work queue, computed on the host (no GPU): every item
of every phase of every pair is queued exactly once, and every item of phase
k of a pair comes after every item of phase k - 1 of that pair. Blocks take
items in queue order and an item waits only for the phase before it, so this
ordering is what keeps the persistent launch from deadlocking."""
import numpy as np
import pytest

from nx_stereo_b200 import batch, native

SHAPES = batch.sample_shapes(64, seed=2024)


def _check_queue(shapes, tuning=None):
    items, runs, total = batch.queue(shapes, tuning)
    assert items.shape == (len(shapes), 6)
    assert (items > 0).all()
    starts = runs[:, 0].astype(np.int64)
    assert starts[0] == 0 and (np.diff(starts) > 0).all() and starts[-1] < total
    ends = np.append(starts[1:], total)
    covered = {}
    first_at, last_at = {}, {}
    for (start, pair, phase, first), end in zip(runs, ends):
        key = (int(pair), int(phase))
        count = int(end - start)
        covered.setdefault(key, []).append((int(first), int(first) + count))
        first_at[key] = min(first_at.get(key, start), start)
        last_at[key] = max(last_at.get(key, end - 1), end - 1)
    for pair in range(len(shapes)):
        for phase in range(6):
            spans = sorted(covered[(pair, phase)])
            assert spans[0][0] == 0 and spans[-1][1] == items[pair, phase]
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))  # no gap, no repeat
            if phase:
                assert last_at[(pair, phase - 1)] < first_at[(pair, phase)]
    return items, runs, total


def test_the_queue_covers_every_item_once_in_dependency_order():
    items, runs, total = _check_queue(SHAPES)
    assert total == items.sum()
    # Phases of different pairs interleave: somewhere a run of paths sits
    # between runs of selection or costs of other pairs.
    phases = runs[:, 2]
    assert len(set(zip(phases[:-1], phases[1:]))) > 6


@pytest.mark.parametrize("tuning", [
    {"group_pairs": 1, "quantum_us": 1.0},
    {"group_pairs": 3, "cost_rows": 4, "select_passes": 16, "quantum_us": 8.0},
    {"group_pairs": 64, "blocks_per_sm": 4, "cost_rows": 1, "select_passes": 1},
    {"order": 1},
])
def test_every_tuning_keeps_the_order(tuning):
    _check_queue(SHAPES[:16], tuning)


def test_item_counts_follow_the_shapes():
    shapes = [(728, 544, {"disparities": 128}), (97, 31, {"disparities": 64, "paths": 3})]
    items, _, _ = batch.queue(shapes, {"cost_rows": 2, "select_passes": 8})
    # census: 128 x 4 tiles of both images
    assert items[0, 0] == 2 * 6 * 136 and items[1, 0] == 2 * 1 * 8
    # costs: 64-pixel blocks of 2 rows
    assert items[0, 1] == 12 * 272 and items[1, 1] == 2 * 16
    # selection: 128 / lanes pixels a pass, 8 passes an item (8 lanes at 128 d)
    assert items[0, 3] == -(-728 * 544 // 128)
    # check and median: 1024 pixels an item
    assert items[0, 4] == items[0, 5] == -(-728 * 544 // 1024)
    # paths: 4 warps an item. At 128 d a warp follows 4 lines: 2 x 136 warps
    # of rows, 2 x 182 of columns, 4 x 318 of diagonals (1271 lines each).
    assert items[0, 2] == (2 * 136 + 2 * 182 + 4 * 318) // 4
    # At 64 d a warp follows 8 lines; 3 paths are two row directions (4 warps
    # each) and one column direction (13 warps), no diagonals.
    assert items[1, 2] == -(-(4 + 4 + 13) // 4)


def test_a_single_pair_queue():
    _check_queue([(64, 48, {"disparities": 64})])


@pytest.mark.parametrize("shape,tuning,reason", [
    ((64, 6, {}), None, "higher than 6"),
    ((64, 48, {"disparities": 80}), None, "disparities"),
    ((64, 48, {"paths": 4}), None, "paths"),
    ((64, 48, {}), {"blocks_per_sm": 0}, "tuning"),
    ((64, 48, {}), {"quantum_us": 0.0}, "tuning"),
    ((64, 48, {}), {"group_pairs": 0}, "tuning"),
])
def test_refusals(shape, tuning, reason):
    with pytest.raises(native.NativeError, match=reason):
        batch.queue([shape], tuning)


class _FakePlan:
    """A plan whose launch time is a given function of its shapes (no GPU)."""

    def __init__(self, tuning, cost):
        self._tuning, self.cost = dict(tuning), cost
        self.shapes = []

    @property
    def tuning(self):
        return dict(self._tuning)

    def retune(self, **tuning):
        self._tuning.update(tuning)


def test_autotuner_tries_the_stream_engine_with_each_stream_count():
    # The stream engine is fastest only with one stream: a search one coordinate
    # at a time from (engine 0, streams 8) reaches it only if the engine's trial
    # covers every stream count.
    def cost(t):
        if t["engine"] == 1:
            return {1: 10.0, 2: 11.0, 8: 13.0}[t["streams"]]
        return 12.0 - (0.5 if t["order"] == 1 else 0.0)

    start = {"engine": 0, "streams": 8, "order": 0}
    plan = _FakePlan(start, cost)
    tuner = batch.Autotuner(search={"engine": (0, 1), "streams": (1, 2, 8), "order": (0, 1)})
    tuner.key = lambda p: "a fake plan"  # (the real key names the device)
    tuner.time = lambda p, t: (p.retune(**t), tuner.trials.append((p.tuning, p.cost(p.tuning))),
                               p.cost(p.tuning))[-1]
    tuning, ms = tuner.tune(plan, use_cache=False)
    assert (tuning["engine"], tuning["streams"], ms) == (1, 1, 10.0)
    tried = {(t["engine"], t["streams"]) for t, _ in tuner.trials}
    assert {(1, 1), (1, 2), (1, 8)} <= tried


def test_the_wait_limit_is_a_checked_plan_setting():
    from nx_stereo_b200 import batch, native

    shapes = [(64, 48, {"disparities": 64})]
    assert batch.default_tuning()["wait_limit_us"] == 0
    batch.queue(shapes, {"wait_limit_us": 1000})
    with pytest.raises(native.NativeError) as raised:
        batch.queue(shapes, {"wait_limit_us": 60_000_001})
    assert raised.value.status == native.BAD_ARGUMENT
    assert "wait_limit_us" in raised.value.message
