"""Generates tests/golden/sgm_fixtures.npz: the oracle's own outputs, frozen.

These are regression fixtures of the oracle, not outputs of the reference:
the reference's own outputs are tests/golden/reference_sgm.npz (made by
make_reference_fixtures.py from the reference's shader sources). Inputs are
the reference's test images (the xorshift `scene` and `noise` generators of
native/stereo_match/src/lib.rs:447-508) at the sizes its differential tests
use (lib.rs:535-593); freezing the oracle's outputs on them checks the CUDA
path against committed data as well as against the live oracle, and shows
any later change of the oracle.

    python tests/golden/make_golden.py
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle  # noqa: E402

CASES = [("scene", 64, 48, 7), ("scene", 97, 31, 7), ("noise", 64, 48, 1), ("noise", 97, 31, 1)]
SETTINGS = [(64, 3), (64, 8), (128, 3), (128, 8)]
PENALTIES = [(0, 1, 1.0), (4, 40, 1.2), (78, 79, 2.5), (10, 79, 1.0526316)]


def pair(kind, w, h, seed):
    if kind == "scene":
        return oracle.scene(w, h, seed)
    return oracle.noise(w, h, seed), oracle.noise(w, h, seed + 1)


def digest(array):
    return hashlib.sha256(np.ascontiguousarray(array).tobytes()).hexdigest()


def fixtures():
    out = {}
    for kind, w, h, seed in CASES:
        left, right = pair(kind, w, h, seed)
        for d, p in SETTINGS:
            key = f"sgm_{kind}_{w}x{h}_d{d}_p{p}"
            out[key] = oracle.sgm(left, right, d, p).view(np.uint32)
    left, right = oracle.scene(80, 40, 3)
    for p1, p2, u in PENALTIES:
        for paths in (3, 8):
            out[f"sgm_penalties_{p1}_{p2}_{u}_p{paths}"] = \
                oracle.sgm(left, right, 64, paths, p1, p2, u).view(np.uint32)
    left, right = oracle.scene(64, 48, 7)
    lc, rc = oracle.census(left), oracle.census(right)
    out["census_scene_64x48_left"] = lc
    costs = oracle.costs(lc, rc, 64)
    out["costs_scene_64x48_d64_sha256"] = np.array(digest(costs.astype(np.uint8)))
    sums = oracle.aggregate(costs, 8, 8, 64)
    out["sums_scene_64x48_d64_p8_sha256"] = np.array(digest(sums.astype(np.uint16)))
    return out


if __name__ == "__main__":
    path = os.path.join(HERE, "sgm_fixtures.npz")
    np.savez_compressed(path, **fixtures())
    print(path, os.path.getsize(path), "bytes")
