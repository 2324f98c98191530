"""Rectification through kept maps: the frame positions a pair's rectified
pixels sample (nxs_rectify_maps_device), then the pair sampled through them
(nxs_rectify_pair_mapped_device), give the bytes of the one-launch pair
rectification; a segment keeps the maps on the device and remakes them when a
request's cameras change, so every request is rectified through its own cameras
(lib/nx_stereo/rectify.ex:133-207, stage/rectification.ex:48-58)."""
import ctypes

import numpy as np
import pytest

from tests import gpu_util as g

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def native():
    from nx_stereo_b200 import native as n

    n.load()
    return n


@pytest.mark.parametrize("size,frame", [((728, 544), (800, 600)), ((97, 31), (120, 40)),
                                        ((364, 272), (364, 272))])
def test_maps_then_mapped_equal_the_pair_kernel(native, size, frame):
    from nx_stereo_b200 import scene

    torch = g.torch()
    (w, h), (fw, fh) = size, frame
    rig = scene.rig(w, h, k1=-0.07, yaw_degrees=0.7)
    cams = scene.cameras(rig)
    cameras = [native.make_camera(cams[s]["k"], cams[s]["d"], cams[s]["inverse_pr"])
               for s in ("left", "right")]
    left, right = scene.rectified_pair(w, h, seed=11)
    lf, rf = scene.raw_frames(left, right, rig, frame_size=(fh, fw))
    d_lf, d_rf = g.dev(lf), g.dev(rf)
    want = [g.empty((h, w), torch.uint8) for _ in range(2)]
    got = [g.empty((h, w), torch.uint8) for _ in range(2)]
    maps = g.empty((2, h, w, 2), torch.float32)
    native.call("nxs_rectify_pair_device", g.ptr(d_lf), g.ptr(d_rf), fw, fh,
                ctypes.byref(cameras[0]), ctypes.byref(cameras[1]), w, h, g.ptr(want[0]),
                g.ptr(want[1]), g.stream())
    native.call("nxs_rectify_maps_device", ctypes.byref(cameras[0]), ctypes.byref(cameras[1]),
                fw, fh, w, h, g.ptr(maps), g.stream())
    native.call("nxs_rectify_pair_mapped_device", g.ptr(d_lf), g.ptr(d_rf), fw, fh, g.ptr(maps),
                w, h, g.ptr(got[0]), g.ptr(got[1]), g.stream())
    for a, b in zip(want, got):
        assert (g.host(a) == g.host(b)).all()


def test_segment_maps_follow_each_requests_cameras(oracle):
    """One configured segment; requests whose cameras switch between two rigs,
    all sent before any is awaited: each pair is rectified through its own
    cameras, as the oracle rectifies it."""
    from nx_stereo_b200 import scene, segment, stage

    w, h = 364, 272
    rigs = [scene.rig(w, h), scene.rig(w, h, focal=850.0, k1=-0.08, yaw_degrees=0.8)]
    geometries = [segment.standard_geometry(w, h, the_rig=r) for r in rigs]
    status, members = segment.members([stage.Rectification], geometries[0])
    assert status == "ok", members
    status, seg = segment.CudaSegment.build(members, geometries[0])
    assert status == "ok", seg
    inputs = [segment._inputs(members, geom) for geom in geometries]
    left, right = scene.rectified_pair(w, h, seed=21)
    frames = [scene.raw_frames(left, right, r) for r in rigs]
    order = [0, 0, 1, 0, 1, 1, 0, 1, 1, 0]
    sent = []
    for which in order:
        seg.inputs = inputs[which]  # the params of this request, same configuration
        status, request = segment.CudaSegment.send_request(
            {"left_frame": frames[which][0], "right_frame": frames[which][1]}, seg)
        assert status == "ok"
        sent.append(request)
    for which, request in zip(order, sent):
        reply = segment.CudaSegment.await_(request, seg, 60000)
        assert reply[0] == "ok", reply
        cams = (geometries[which]["left_camera"], geometries[which]["right_camera"])
        for name, frame, c in zip(("left", "right"), frames[which], cams):
            want = oracle.rectify(frame, oracle.make_camera(c["k"], c["d"], c["inverse_pr"]),
                                  (h, w))
            assert np.array_equal(np.asarray(reply[1][name]), want), (which, name)
    seg.release()
