"""Host-side logic without a GPU: the C ABI library loads and exports what the
header declares, the settings checker refuses what the reference refuses, and
the Segment helpers and CudaSegment encode entries, configuration and params
as the reference's (test/nx_stereo/segment_test.exs,
native_segment_test.exs, native/stereo_match/src/lib.rs:646-686)."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from nx_stereo_b200 import native, segment, stage

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "nx_stereo_b200.h")


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^[A-Za-z0-9_ ]+\*?\s*\*?(nxs_\w+)\(", text, re.M)))


def test_the_library_exports_every_declared_function():
    names = declared_functions()
    assert len(names) >= 30
    lib = ctypes.CDLL(native.library_path())
    for name in names:
        assert hasattr(lib, name), name
    exported = subprocess.run(["nm", "-D", "--defined-only", native.library_path()],
                              capture_output=True, text=True).stdout
    for name in names:
        assert re.search(rf"\bT {name}\b", exported), name


def test_the_binding_declares_every_function_but_the_static_scratch_one():
    assert set(declared_functions()) - set(native.SIGNATURES) == {"nxs_sgm_device_static"}


def test_the_library_loads_without_a_gpu_and_reports_its_version():
    assert native.load().nxs_version().startswith(b"nx_stereo_b200")


def test_sgm_check_refuses_what_nx_stereo_refuses():
    # lib.rs:646-686, extended to the disparity counts 96, 192 and 256.
    assert native.check_sgm(64, 48, disparities=64, paths=3) is None
    for d in (96, 128, 192, 256):
        assert native.check_sgm(64, 48, disparities=d) is None
    refusals = [((8, 48), {}), ((64, 6), {}), ((4097, 48), {}), ((64, 48), dict(disparities=80)),
                ((64, 48), dict(paths=4)), ((64, 48), dict(p1=64, p2=64)),
                ((64, 48), dict(p1=8, p2=80)), ((64, 48), dict(uniqueness=0.9)),
                ((64, 48), dict(uniqueness=float("nan")))]
    for (w, h), settings in refusals:
        error = native.check_sgm(w, h, **settings)
        assert error is not None and error.status == native.BAD_ARGUMENT, (w, h, settings)
    assert "wider than 8" in native.check_sgm(8, 48).message
    assert "p1 < p2" in native.check_sgm(64, 48, p1=64, p2=64).message


def test_device_path_entries_refuse_disparities_their_kernels_do_not_cover():
    # The path kernels hold 8 to 32 disparities a lane in 2 to 32 lanes a scan
    # line: 64 to 256 disparities in steps of 32. The refusal comes before any
    # device work, so fake non-null pointers never reach a kernel.
    for d in (0, 32, 48, 80, 288):
        calls = [("nxs_paths_device", (1, 8, 8, d, 8, 8, 64, 1, None)),
                 ("nxs_paths_device_ordered", (1, 8, 8, d, 8, 8, 64, 16, 1, None)),
                 ("nxs_aggregate_device", (1, 1, 8, 8, d, 8, 8, 64, 1, None))]
        for name, args in calls:
            with pytest.raises(native.NativeError) as refused:
                native.call(name, *args)
            assert refused.value.status == native.BAD_ARGUMENT, (name, d)


# ---------------------------------------------------------------- stage settings
GEOMETRY = {"width": 4, "height": 2, "frame_width": 6, "frame_height": 3,
            "focal_length_px": 100.0, "baseline_m": 0.1, "principal_point": (2.0, 1.0)}


def test_disparity_settings_and_refusals():
    status, state = stage.Disparity.init({}, GEOMETRY)
    assert status == "ok"
    assert (state["p1"], state["p2"], state["num_disparities"], state["paths"]) == (8, 64, 64, 8)
    assert state["uniqueness"] == 1.0526315789473684
    assert stage.Disparity.init({"p1": 8, "p2": 8}, GEOMETRY) == \
        ("error", "p2 must be above p1 (8), got 8")
    assert stage.Disparity.init({"p2": 80}, GEOMETRY)[1] == "p2 must be from 1 to 79, got 80"
    assert stage.Disparity.init({"num_disparities": 80}, GEOMETRY)[1].startswith(
        "num_disparities must be one of")
    assert stage.Disparity.init({"paths": 4}, GEOMETRY)[1] == "paths must be one of [3, 8], got 4"
    assert stage.Disparity.init({"uniqueness": 0.5}, GEOMETRY)[0] == "error"
    assert stage.Disparity.init({"scale": 2}, GEOMETRY) == ("error", "unknown settings ['scale']")
    assert stage.Disparity.params(state, GEOMETRY) == {"p1": 8, "p2": 64,
                                                       "uniqueness": 1.0526315789473684}
    assert stage.Disparity.native_settings(state) == [("num_disparities", 64), ("paths", 8)]


def test_other_stages_settings():
    assert stage.SpeckleFilter.init({"min_support": 49}, GEOMETRY)[0] == "error"
    assert stage.SpeckleFilter.init({"min_support": 48}, GEOMETRY)[0] == "ok"
    assert stage.SpeckleFilter.native_constants() == {"radius": 3}
    assert stage.TemporalFilter.init({"alpha": 0.01}, GEOMETRY)[0] == "error"
    assert stage.TemporalFilter.native_constants() == {"max_missed": 255.0}
    assert stage.PointCloud.init({"decimation": 3}, GEOMETRY) == \
        ("error", "decimation must fit working size 4x2, got 3")
    assert stage.PointCloud.init({"decimation": 2}, GEOMETRY)[0] == "ok"
    assert stage.Rectification.init({}, dict(GEOMETRY, frame_width=3))[1].startswith(
        "rectification only shrinks")
    assert stage.Depth.init({"scale": 2}, GEOMETRY) == ("error", "unknown settings ['scale']")


# ---------------------------------------------------------------- segment helpers
def members_of(modules):
    return [{"module": m, "name": m.__name__, "state": None} for m in modules]


def test_entry_specs_at_frame_and_working_sizes():
    # segment_test.exs:32-46
    assert segment.entry_specs(members_of([stage.Rectification]), GEOMETRY) == \
        ("ok", [("left_frame", ((3, 6), np.uint8)), ("right_frame", ((3, 6), np.uint8))])
    assert segment.entry_specs(members_of([stage.SpeckleFilter]), GEOMETRY) == \
        ("ok", [("disparity", ((2, 4), np.float32))])
    assert segment.entry_specs(members_of([stage.Disparity, stage.SpeckleFilter]), GEOMETRY) == \
        ("ok", [("left", ((2, 4), np.uint8)), ("right", ((2, 4), np.uint8))])


def test_the_stages_in_depth_order_read_nothing_but_the_frames():
    # segment_test.exs:58-76
    stages = [stage.Rectification, stage.Disparity, stage.SpeckleFilter, stage.TemporalFilter,
              stage.Depth, stage.PointCloud, stage.Quality]
    assert segment.entry_fields(members_of(stages)) == ["left_frame", "right_frame"]


def test_cannot_take_as_an_entry_a_tensor_no_stage_before_it_fills():
    assert segment.entry_specs(members_of([stage.PointCloud]), GEOMETRY) == \
        ("error", "no stage before it provides :depth_m, and a segment cannot take it as an entry")


def test_entry_tensors_of_their_spec_or_why_not():
    # segment_test.exs:84-103
    _, specs = segment.entry_specs(members_of([stage.Rectification, stage.SpeckleFilter]),
                                   GEOMETRY)
    frame = np.full((3, 6), 7, np.uint8)
    entries = {"left_frame": frame, "right_frame": frame,
               "disparity": np.full((2, 4), 1.5, np.float64)}
    status, tensors = segment.entry_tensors(entries, specs)
    assert status == "ok"
    assert [name for name, _ in tensors] == ["left_frame", "right_frame", "disparity"]
    assert tensors[2][1].dtype == np.float32 and tensors[0][1] is not None
    _, specs = segment.entry_specs(members_of([stage.SpeckleFilter]), GEOMETRY)
    assert segment.entry_tensors({"disparity": np.zeros((3, 4), np.float32)}, specs) == \
        ("error", ("frame_size", "disparity", (3, 4), (2, 4)))
    assert segment.entry_tensors({"disparity": None}, specs) == \
        ("error", ("not_a_tensor", "disparity", None))
    assert segment.entry_tensors({}, specs) == ("error", ("missing_entry", "disparity"))


def test_run_returns_the_entries_but_the_frames_with_the_outputs():
    class Echo:
        @staticmethod
        def send_request(entries, seg):
            return ("ok", dict(entries))

        @staticmethod
        def await_(request, seg, timeout):
            return ("ok", {"echoed": request}, seg, 0)

        @staticmethod
        def collect(outputs, seg, timeout):
            return ("ok", outputs)

    status, outputs, _ = segment.run(Echo, {"left_frame": 1, "disparity": 2}, "segment", None)
    assert status == "ok" and sorted(outputs) == ["disparity", "echoed"]


def test_members_initialise_or_say_which_refuses():
    status, members = segment.members([stage.Depth, (stage.SpeckleFilter, {"min_support": 4})],
                                      GEOMETRY)
    assert status == "ok" and members[1]["state"]["min_support"] == 4
    assert segment.members([(stage.Depth, {"scale": 2})], GEOMETRY) == \
        ("error", "Depth: unknown settings ['scale']")


# ---------------------------------------------------------------- CudaSegment host side
def built(stages, geometry):
    status, members = segment.members(stages, geometry)
    assert status == "ok", members
    status, seg = segment.CudaSegment.build(members, geometry)
    assert status == "ok", seg
    return seg


def test_configuration_is_each_kind_with_its_settings_and_constants():
    # native_segment_test.exs:62-76
    geometry = segment.standard_geometry(16, 12)
    seg = built([stage.Rectification, (stage.Disparity, {"num_disparities": 128}),
                 stage.SpeckleFilter, stage.TemporalFilter, stage.Depth,
                 (stage.PointCloud, {"decimation": 2}), stage.Quality], geometry)
    assert segment._configuration(seg) == [
        ("rectification", {}), ("disparity", {"num_disparities": 128.0, "paths": 8.0}),
        ("speckle_filter", {"radius": 3.0}), ("temporal_filter", {"max_missed": 255.0}),
        ("depth", {}), ("point_cloud", {"decimation": 2.0, "max_depth_m": 20.0,
                                        "min_depth_m": 0.05}), ("quality", {})]
    assert [sorted(i) for i in seg.inputs] == [
        ["left.d", "left.inverse_pr", "left.k", "right.d", "right.inverse_pr", "right.k"],
        ["p1", "p2", "uniqueness"], ["max_diff", "min_support"], ["alpha", "delta", "hold"],
        ["baseline_m", "focal_length_px"], ["cx", "cy", "focal_length_px"], []]
    assert seg.inputs[1]["uniqueness"].dtype == np.float32
    assert seg.inputs[0]["left.inverse_pr"].shape == (9,)
    seg.release()


def test_a_new_member_state_changes_its_params_not_its_settings():
    geometry = segment.standard_geometry(16, 12)
    seg = built([stage.SpeckleFilter], geometry)
    _, state = stage.SpeckleFilter.init({"min_support": 5}, geometry)
    segment.CudaSegment.put_member_state(seg, 0, state)
    assert float(seg.inputs[0]["min_support"][0]) == 5.0
    assert segment._configuration(seg) == [("speckle_filter", {"radius": 3.0})]
    version = seg.version
    segment.CudaSegment.reload(seg, seg.members, geometry)
    assert seg.version == version + 1
    seg.release()


def test_accepts_native_kinds_only_and_refuses_unknown_build_options():
    # native_segment_test.exs:182-237
    assert segment.CudaSegment.accepts(stage.Disparity, {"matcher": None}, "native")
    assert not segment.CudaSegment.accepts(stage.Disparity, {"matcher": "nx"}, "native")
    assert not segment.CudaSegment.accepts(stage.Disparity, {"matcher": None}, "nx")

    class NxOnly(stage.Stage):
        @staticmethod
        def requires():
            return ["disparity"]

        @staticmethod
        def provides():
            return ["disparity"]

    assert not segment.CudaSegment.accepts(NxOnly, None, "native")
    geometry = segment.standard_geometry(16, 12)
    status, members = segment.members([stage.Depth], geometry)
    assert segment.CudaSegment.build(members, geometry, {"threads": 2}) == \
        ("error", "unknown build options ['threads']")
    assert segment.CudaSegment.compute(None)["runs_on"] == "gpu"
    assert segment.CudaSegment.depth() >= 2


def test_camera_mirrors_rectify_camera():
    from nx_stereo_b200 import rectify

    k = [100.0, 0.0, 32.0, 0.0, 100.0, 24.0, 0.0, 0.0, 1.0]
    identity = [1.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 1.0]
    cam = rectify.camera(k, [0.02], identity, [90.0, 0, 30.0, 0, 0, 90.0, 22.0, 0, 0, 0, 1.0, 0])
    assert cam["d"].tolist() == [np.float32(0.02), 0, 0, 0, 0]
    assert np.allclose(cam["inverse_pr"], np.linalg.inv([[90, 0, 30], [0, 90, 22], [0, 0, 1]]),
                       rtol=1e-6)
    with pytest.raises(ValueError):
        rectify.camera(k, [0.1, 0, 0, 0, 0, 0.2], identity, [0] * 12)
    moved = rectify.move_rows(cam, 2.0)
    assert moved["inverse_pr"][1, 2] == np.float32(cam["inverse_pr"][1, 2] +
                                                   np.float32(2.0) * cam["inverse_pr"][1, 1])


def test_band_check_refuses_what_the_coarse_to_fine_search_refuses():
    # sgm_band/4 (lib/nx_stereo.ex:300-304) and sgm_coarse_to_fine/3 (173-183)
    assert native.check_band(64, 48) == (True, "")
    assert native.check_band(65, 48, coarse_to_fine=False, disparities=64) == (True, "")
    refusals = [((65, 48), {}, "even height and width"),
                ((64, 48), dict(disparities=64), "must be 128"),
                ((64, 48), dict(band=12), ":band must be 8, 16, 32 or 64"),
                ((64, 48), dict(census="dense_9x5", coarse_paths=4), "coarse_paths"),
                ((64, 48), dict(margin=128), "margin"),
                ((16, 48), {}, "wider than 8"),  # the half-size pair is 8 wide
                ((64, 12), {}, "higher than 6")]
    for (w, h), settings, why in refusals:
        ok, message = native.check_band(w, h, **settings)
        assert not ok and why in message, (w, h, settings, message)
    ok, message = native.check_band(64, 48, coarse_to_fine=False, band=12)
    assert not ok and ":band" in message
    p = native.band_params()
    p.census = 3
    buf = native._errbuf()
    assert native.load().nxs_band_check(ctypes.byref(p), 64, 48, 1, buf, 1024) == \
        native.BAD_ARGUMENT
    assert native.band_scratch_bytes(728, 544, 16) > native.band_scratch_bytes(728, 544, 16, False)


def test_coarse_to_fine_settings_and_refusals():
    # stage/disparity.ex:72-108, 120-128, 165-166, 196-219
    geometry = {**GEOMETRY, "width": 64, "height": 48}
    status, state = stage.Disparity.init({"search": "coarse_to_fine", "num_disparities": 128},
                                         geometry)
    assert status == "ok"
    assert (state["band"], state["margin"], state["coarse_paths"], state["fine_census"]) == \
        (16, 4, 8, "sparse_9x7")
    assert stage.Disparity.compute(state) == "nx"  # computed in Nx unless pinned
    assert not segment.CudaSegment.accepts(stage.Disparity, state, "native")
    status, native_state = stage.Disparity.init(
        {"search": "coarse_to_fine", "num_disparities": 128, "matcher": "native", "band": 32,
         "coarse_paths": 3, "fine_census": "dense_9x5_blend"}, geometry)
    assert status == "ok" and stage.Disparity.compute(native_state) == "native"
    assert segment.CudaSegment.accepts(stage.Disparity, native_state, "native")
    assert stage.Disparity.native_settings(native_state) == [
        ("num_disparities", 128), ("paths", 8), ("coarse_to_fine", 1), ("band", 32),
        ("margin", 4), ("coarse_paths", 3), ("fine_census", 2)]
    refusals = [({"search": "coarse_to_fine"}, geometry, "searches 128 disparities, got 64"),
                ({"search": "coarse_to_fine", "num_disparities": 128}, {**geometry, "width": 63},
                 "even width and height, got 63x48"),
                ({"search": "coarse_to_fine", "num_disparities": 128, "band": 8, "margin": 8},
                 geometry, "margin must be below band (8), got 8"),
                ({"fine_census": "dense_9x5"}, geometry, "fine_census requires coarse_to_fine"),
                ({"search": "coarse_to_fine", "num_disparities": 128, "band": 12}, geometry,
                 "band must be one of")]
    for given, g, why in refusals:
        status, message = stage.Disparity.init(given, g)
        assert status == "error" and why in message, (given, message)


def test_rectify_map_entries_refuse_bad_arguments():
    # The maps are 8-byte (x, y) f32 pairs; sizes as the pair rectification's.
    cam = native.make_camera([873.0, 0.0, 4.0, 0.0, 873.0, 4.0, 0.0, 0.0, 1.0],
                             [0.0] * 5, [1.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 1.0])
    lib = native.load()
    ref = ctypes.byref(cam)
    for maps, size, frame in [(0, (8, 8), (8, 8)), (4, (8, 8), (8, 8)),
                              (4096, (0, 8), (8, 8)), (4096, (8, 8), (7, 8))]:
        (w, h), (fw, fh) = size, frame
        assert lib.nxs_rectify_maps_device(ref, ref, fw, fh, w, h, maps, None) == \
            native.BAD_ARGUMENT, (maps, size, frame)
        assert lib.nxs_rectify_pair_mapped_device(4096, 4096, fw, fh, maps, w, h, 4096, 4096,
                                                  None) == native.BAD_ARGUMENT
    assert lib.nxs_rectify_maps_device(None, ref, 8, 8, 8, 8, 4096, None) == native.BAD_ARGUMENT


def test_tuning_knobs_refuse_out_of_range_and_read_back():
    # Library-wide tuning knobs: none changes a result, each refuses a value it
    # does not know and leaves the setting as it was.
    lib = native.load()
    before = lib.nxs_lean_select()
    try:
        assert lib.nxs_set_lean_select(17) == native.BAD_ARGUMENT
        assert lib.nxs_lean_select() == before
        for value in (0, 1, 16, 8):
            assert lib.nxs_set_lean_select(value) == native.OK
            assert lib.nxs_lean_select() == value
    finally:
        lib.nxs_set_lean_select(before)
    assert lib.nxs_set_split_lanes(2) == native.BAD_ARGUMENT
    tiles = lib.nxs_path_tiles()
    try:
        for mode in (0, 1, 2):
            assert lib.nxs_set_path_tiles(mode) == native.OK
            assert lib.nxs_path_tiles() == mode
    finally:
        lib.nxs_set_path_tiles(tiles)
