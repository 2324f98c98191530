"""The oracle's frozen regression fixtures (tests/golden/sgm_fixtures.npz,
made by tests/golden/make_golden.py from the oracle on the reference's test
images; the reference's own outputs are checked in test_reference_pin.py and
test_gpu_reference.py): the oracle still reproduces them (CPU), and the CUDA
path equals them bit for bit (GPU)."""
import hashlib
import os

import numpy as np
import pytest

from tests import gpu_util as g
from tests.golden import make_golden

FIXTURES = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "sgm_fixtures.npz")


@pytest.fixture(scope="module")
def golden():
    with np.load(FIXTURES) as data:
        return {k: data[k] for k in data.files}


def test_the_oracle_reproduces_the_fixtures(golden):
    fresh = make_golden.fixtures()
    assert sorted(fresh) == sorted(golden)
    for key, value in fresh.items():
        assert np.array_equal(value, golden[key]), key


def _cases():
    for kind, w, h, seed in make_golden.CASES:
        for d, p in make_golden.SETTINGS:
            yield kind, w, h, seed, d, p


@pytest.mark.gpu
def test_the_cuda_matcher_equals_the_fixtures(golden):
    from nx_stereo_b200 import native

    ctx = native.Context(0)
    for kind, w, h, seed, d, p in _cases():
        left, right = make_golden.pair(kind, w, h, seed)
        got = ctx.sgm(left, right, disparities=d, paths=p)
        assert np.array_equal(got.view(np.uint32), golden[f"sgm_{kind}_{w}x{h}_d{d}_p{p}"])
    left, right = make_golden.oracle.scene(80, 40, 3)
    for p1, p2, u in make_golden.PENALTIES:
        for paths in (3, 8):
            got = ctx.sgm(left, right, disparities=64, paths=paths, p1=p1, p2=p2, uniqueness=u)
            assert np.array_equal(got.view(np.uint32),
                                  golden[f"sgm_penalties_{p1}_{p2}_{u}_p{paths}"])
    ctx.close()


@pytest.mark.gpu
def test_the_cuda_steps_equal_the_fixtures(golden):
    from nx_stereo_b200 import native

    left, right = make_golden.oracle.scene(64, 48, 7)
    ctx = native.Context(0)
    torch = g.torch()
    d_l, d_r = g.dev(left), g.dev(right)
    codes = g.empty((2, 48, 64), torch.int64)
    native.call("nxs_census_device", g.ptr(d_l), 64, 48, codes[0].data_ptr(), g.stream())
    native.call("nxs_census_device", g.ptr(d_r), 64, 48, codes[1].data_ptr(), g.stream())
    assert np.array_equal(g.host(codes[0]).view(np.uint64), golden["census_scene_64x48_left"])
    costs = g.empty((48, 64, 64), torch.uint8)
    native.call("nxs_costs_device", codes[0].data_ptr(), codes[1].data_ptr(), 64, 48, 64,
                g.ptr(costs), g.stream())
    digest = hashlib.sha256(g.host(costs).tobytes()).hexdigest()
    assert digest == str(golden["costs_scene_64x48_d64_sha256"])
    sums = g.empty((48, 64, 64), torch.int16)
    native.call("nxs_aggregate_device", ctx.handle, g.ptr(costs), 64, 48, 64, 8, 8, 64,
                g.ptr(sums), g.stream())
    digest = hashlib.sha256(g.host(sums).view(np.uint16).tobytes()).hexdigest()
    assert digest == str(golden["sums_scene_64x48_d64_p8_sha256"])
    ctx.close()
