"""Generates tests/golden/reference_sgm.npz: the reference's own outputs.

NxStereo.sgm/3 on a GPU is the reference's shader pipeline
(lib/nx_stereo/vulkan.ex:262-333 over shaders/census_pair.comp,
cost_first.comp, cost_scan.comp, cost_line.comp, select.comp,
consistency_projected.comp and filter.comp), which the reference's own
tests hold to its Nx definition (test/nx_stereo/full_range_test.exs:7-36:
the same sign and within 1e-4). oracle/build_ref.py compiles those shader
sources, unchanged but for their GLSL declarations, as C++ on the CPU, and
this script runs them (oracle/reference_shaders.py) on:

  - the 364x272 pair at 64 disparities, 8 paths, default penalties (the
    plain single-pair workload the reference runs on its CPU paths), with
    the selection's keys and pre-check disparity as well;
  - the 728x544 pair at 128 disparities with 8 paths (the matcher of the
    frame-to-depth workload) and 3 paths at 364x272;
  - the shapes and penalties of full_range_test.exs (19x101 and 90x70
    uniform-noise textures, 128 disparities, 3 and 8 paths, penalties 0/1,
    8/64 and 78/79) and of its known-shift case (a 24x160 crop of a 24x256
    texture shifted by 96 columns);
  - edge shapes: the smallest accepted image (9x7), the widest (4096x7),
    and 64 disparities at ragged sizes.

Inputs are seeded (numpy's PCG64 for the noise textures, the bench's own
scene generator for the scenes) and stored in the file with the outputs.
tests/golden/reference_stages.npz holds the stages around the matcher the
same way (stage_fixtures below).
Needs the reference checkout (to build oracle/_ref); the tests only read the
committed file.

    python tests/golden/make_reference_fixtures.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from nx_stereo_b200 import scene  # noqa: E402
from oracle import reference_shaders  # noqa: E402

UNIQUENESS = 1.0526315789473684


def _noise(shape, seed):
    return np.random.default_rng(seed).integers(0, 256, shape, dtype=np.uint8)


def cases():
    """(name, left, right, disparities, paths, p1, p2, keep_selection)."""
    out = []
    left, right = scene.rectified_pair(364, 272, seed=11)
    out.append(("scene_364x272_d64_p8", left, right, 64, 8, 8, 64, True))
    out.append(("scene_364x272_d128_p3", left, right, 128, 3, 8, 64, False))
    left, right = scene.rectified_pair(728, 544, seed=11, rectangles=6, max_disparity=120)
    out.append(("scene_728x544_d128_p8", left, right, 128, 8, 8, 64, False))
    for h, w in ((19, 101), (90, 70)):
        left, right = _noise((h, w), 53), _noise((h, w), 92)
        for paths in (3, 8):
            for p1, p2 in ((0, 1), (8, 64), (78, 79)):
                out.append((f"noise_{w}x{h}_d128_p{paths}_{p1}_{p2}", left, right, 128, paths, p1,
                            p2, False))
    texture = _noise((24, 256), 14)
    left, right = texture[:, :160].copy(), texture[:, 96:256].copy()
    for paths in (3, 8):
        out.append((f"shift96_160x24_d128_p{paths}", left, right, 128, paths, 8, 64, False))
    for w, h, d in ((9, 7, 64), (4096, 7, 64), (33, 17, 64), (130, 45, 128)):
        left, right = scene.rectified_pair(w, h, seed=w + h, rectangles=2, max_disparity=min(56, w))
        for paths in (3, 8):
            out.append((f"scene_{w}x{h}_d{d}_p{paths}", left, right, d, paths, 8, 64, False))
    return out


def fixtures():
    data = {}
    for name, left, right, d, paths, p1, p2, keep in cases():
        out, selected, keys = reference_shaders.sgm(left, right, d, paths, p1, p2, UNIQUENESS,
                                                    with_selection=True)
        data[name + "/left"] = left
        data[name + "/right"] = right
        data[name + "/settings"] = np.array([d, paths, p1, p2], np.int32)
        data[name + "/disparity"] = out
        if keep:
            data[name + "/selected"] = selected
            data[name + "/keys"] = keys
    return data


def stage_fixtures():
    """The stages around the matcher as the reference's shaders compute them
    (lib/nx_stereo/kernels.ex over shaders/rectify.comp, despeckle.comp,
    temporal_filter.comp, depth.comp, point_cloud_rows.comp,
    disparity_rows.comp and column_sums.comp), at 364x272 on the frame-to-
    depth rig: rectification of both raw frames; then, on the reference's own
    disparity of the rectified pair (with Stage.Disparity's mask), despeckle,
    a temporal step against a perturbed previous map, depth, the point cloud
    and the quality sums."""
    from nx_stereo_b200 import segment

    w, h = 364, 272
    geometry = segment.standard_geometry(w, h)
    left, right = scene.rectified_pair(w, h, seed=3, rectangles=6, max_disparity=56)
    frames = scene.raw_frames(left, right, scene.rig(w, h))
    data = {"left_frame": frames[0], "right_frame": frames[1]}
    images = []
    for side, frame in zip(("left", "right"), frames):
        c = geometry[side + "_camera"]
        data[side + "_camera"] = np.concatenate(
            [np.ravel(c["k"]), np.ravel(c["d"]), np.ravel(c["inverse_pr"])]).astype(np.float32)
        images.append(reference_shaders.rectify(frame, c["k"], c["d"], c["inverse_pr"], (h, w)))
        data[side + "_image"] = images[-1]
    d = reference_shaders.sgm(images[0], images[1], 64, 8, 8, 64, UNIQUENESS)
    d = np.where(d > 0, d, np.float32(-1.0)).astype(np.float32)
    data["disparity"] = d
    data["despeckled"] = reference_shaders.despeckle(d, 12.0, 1.0)
    rng = np.random.default_rng(17)
    previous = np.where(rng.random(d.shape) < 0.9,
                        d + rng.normal(0, 1.5, d.shape).astype(np.float32), -1).astype(np.float32)
    missed = rng.integers(0, 4, d.shape).astype(np.float32)
    data["previous"], data["missed"] = previous, missed
    data["filtered"], data["missed_out"] = reference_shaders.temporal(data["despeckled"], previous,
                                                                      missed, 0.4, 2.0, 2.0)
    f, baseline = geometry["focal_length_px"], geometry["baseline_m"]
    data["depth_mm"], data["depth_m"] = reference_shaders.depth(data["filtered"], f, baseline)
    cx, cy = geometry["principal_point"]
    data["cloud_grid"], kept = reference_shaders.point_cloud(data["depth_m"], 4, f, cx, cy, 0.05,
                                                             20.0)
    data["cloud_kept"] = np.array(kept, np.int32)
    data["quality_sums"] = reference_shaders.quality(data["filtered"], previous)
    data["geometry"] = np.array([f, baseline, cx, cy], np.float32)
    return data


if __name__ == "__main__":
    path = os.path.join(HERE, "reference_sgm.npz")
    np.savez_compressed(path, **fixtures())
    print(path, os.path.getsize(path), "bytes")
    path = os.path.join(HERE, "reference_stages.npz")
    np.savez_compressed(path, **stage_fixtures())
    print(path, os.path.getsize(path), "bytes")
