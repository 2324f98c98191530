"""nxs_port, the stereo_match Port served by this library, without a GPU: it
frames and parses records as the reference's Port does and refuses what it
refuses (native/stereo_match/src/protocol.rs tests, main.rs), logs first, and
says why it cannot configure without a CUDA device."""
import os
import subprocess

import numpy as np
import pytest

from nx_stereo_b200 import build
from tests import port_client as pc


@pytest.fixture
def port():
    build.build()
    p = pc.Port(build.PORT)
    yield p
    p.close()


def test_refuses_short_long_or_unknown_requests(port):
    # protocol.rs:233-244
    port.send(bytes([2, 1, 0]))
    assert port.receive() == b"\x09the request ends 2 bytes early"
    port.send(bytes([3, 1, 0, 0, 0, 9]))
    assert port.receive() == b"\x091 bytes follow the request"
    port.send(bytes([9, 1, 0, 0, 0]))
    assert port.receive() == b"\x09unknown request kind 9"
    # a release is not replied to: the next reply is the next request's
    port.send(pc.release_record(1))
    port.send(bytes([7, 0, 0, 0, 0]))
    assert port.receive() == b"\x09unknown request kind 7"
    assert port.logs and port.logs[0][0] == 0 and "nx_stereo_b200" in port.logs[0][1]


def test_a_tensor_of_an_unknown_type_or_short_elements_is_refused(port):
    record = bytearray(pc.run_record(5, [], [("left", np.zeros((1, 2), "u1"))]))
    record[-10 - 2] = 7  # the entry's type code
    port.send(bytes(record))
    assert port.receive() == b"\x09unknown tensor type 7"
    port.send(pc.run_record(5, [], [("left", np.zeros((1, 2), "u1"))])[:-1])
    assert port.receive() == b"\x09the request ends 1 bytes early"


@pytest.mark.skipif(os.environ.get("CUDA_VISIBLE_DEVICES") is None and
                    os.path.exists("/dev/nvidia0"), reason="a GPU is present")
def test_without_a_device_every_configure_is_refused_with_why(port):
    geometry = {"width": 64, "height": 48, "frame_width": 64, "frame_height": 48}
    port.send(pc.configure_record(7, geometry, [("depth", {})]))
    reply = port.receive()
    assert reply[:1] == b"\x09" and b"no CUDA device" in reply


def test_argument_refusals():
    build.build()
    for args in (["--threads", "0"], ["--bogus"]):
        r = subprocess.run([build.PORT, *args], stdin=subprocess.DEVNULL, capture_output=True)
        assert r.returncode == 2
