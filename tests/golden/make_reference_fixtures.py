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
tests/golden/reference_stages.npz holds the stages around the matcher and
tests/golden/reference_band.npz the coarse-to-fine search the same way
(stage_fixtures and band_fixtures below).
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


def band_fixtures():
    """The coarse-to-fine search as the reference's shaders compute it
    (lib/nx_stereo/vulkan.ex:111-255 over shrink.comp, band_base.comp,
    census_dense_pair.comp, band_cost.comp, band_transpose.comp,
    band_scan.comp, band_scan_lanes.comp, band_scan_aggregate.comp and
    band_select.comp):

      - sgm_band/4 at band_bounds_test.exs's shape (19x101 noise textures
        and a random base in -1..128 - band) for every band and path count,
        at uniqueness 1.0 as that test sets it;
      - sgm_band/4 at wide_band_test.exs's shape and bases (18x98; base 0 or
        128 - band by a phase of the pixel) for bands 32 and 64 at its
        penalty limits 0/1, 0/79 and 78/79;
      - the dense census windows (plain and blended) in the fine pass;
      - sgm_coarse_to_fine/3 on 258x128 unrelated noise halves (the shape of
        coarse_to_fine_test.exs, 3 coarse paths), on a 364x272 scene and on
        the 728x544 scene of the frame-to-depth workload (band 16, 8 paths,
        the reference's fast setting), with their band bases."""
    data = {}
    rng = np.random.default_rng(77)
    for band in (8, 16, 32, 64):
        for paths in (3, 8):
            left = rng.integers(0, 256, (19, 101)).astype(np.uint8)
            right = rng.integers(0, 256, (19, 101)).astype(np.uint8)
            base = rng.integers(-1, 129 - band, (19, 101)).astype(np.int32)
            name = f"bounds_b{band}_p{paths}"
            data.update({name + "/left": left, name + "/right": right, name + "/base": base,
                         name + "/settings": np.array([band, paths, 8, 64, 0], np.int32),
                         name + "/uniqueness": np.float32(1.0),
                         name + "/disparity": reference_shaders.sgm_band(
                             left, right, base, 128, paths, band, "sparse_9x7", 8, 64, 1.0)})
    left = rng.integers(0, 256, (18, 98)).astype(np.uint8)
    right = rng.integers(0, 256, (18, 98)).astype(np.uint8)
    phase = np.arange(98)[None, :] + 2 * np.arange(18)[:, None]
    for band in (32, 64):
        base = np.where(phase % 3 == 0, 0, 128 - band).astype(np.int32)
        for paths in (3, 8):
            for p1, p2 in ((0, 1), (0, 79), (78, 79)):
                name = f"wide_b{band}_p{paths}_{p1}_{p2}"
                data.update({name + "/left": left, name + "/right": right, name + "/base": base,
                             name + "/settings": np.array([band, paths, p1, p2, 0], np.int32),
                             name + "/uniqueness": np.float32(UNIQUENESS),
                             name + "/disparity": reference_shaders.sgm_band(
                                 left, right, base, 128, paths, band, "sparse_9x7", p1, p2,
                                 UNIQUENESS)})
    texture = rng.integers(0, 256, (128, 516)).astype(np.uint8)
    halves = (texture[:, :258].copy(), texture[:, 258:].copy())
    scene364 = scene.rectified_pair(364, 272, seed=21, rectangles=6, max_disparity=120)
    scene728 = scene.rectified_pair(728, 544, seed=11, rectangles=6, max_disparity=120)
    runs = [("c2f_noise_258x128_b16_p8_cp3", halves, 16, 8, 3, "sparse_9x7"),
            ("c2f_scene_364x272_b16_p8", scene364, 16, 8, 8, "sparse_9x7"),
            ("c2f_scene_364x272_b32_p3", scene364, 32, 3, 3, "sparse_9x7"),
            ("c2f_scene_364x272_b16_p8_dense", scene364, 16, 8, 8, "dense_9x5"),
            ("c2f_scene_364x272_b8_p8_blend", scene364, 8, 8, 8, "dense_9x5_blend"),
            ("c2f_scene_728x544_b16_p8", scene728, 16, 8, 8, "sparse_9x7")]
    windows = {"sparse_9x7": 0, "dense_9x5": 1, "dense_9x5_blend": 2}
    for name, (left, right), band, paths, coarse_paths, census in runs:
        out, base = reference_shaders.sgm_coarse_to_fine(left, right, paths, coarse_paths, band, 4,
                                                         census, with_base=True)
        data.update({name + "/left": left, name + "/right": right, name + "/base": base,
                     name + "/settings": np.array([band, paths, 8, 64, windows[census],
                                                   coarse_paths, 4], np.int32),
                     name + "/uniqueness": np.float32(UNIQUENESS), name + "/disparity": out})
    return data


if __name__ == "__main__":
    path = os.path.join(HERE, "reference_sgm.npz")
    np.savez_compressed(path, **fixtures())
    print(path, os.path.getsize(path), "bytes")
    path = os.path.join(HERE, "reference_stages.npz")
    np.savez_compressed(path, **stage_fixtures())
    print(path, os.path.getsize(path), "bytes")
    path = os.path.join(HERE, "reference_band.npz")
    np.savez_compressed(path, **band_fixtures())
    print(path, os.path.getsize(path), "bytes")
