"""A client of the stereo_match Port protocol (native/stereo_match/src/protocol.rs),
for testing nxs_port: records encoded as NxStereo.NativeSegment encodes them
(lib/nx_stereo/native_segment.ex:256-344) and framed as NxStereo.Matcher's
{:packet, 4} Port frames them, replies decoded as NativeSegment decodes them
(native_segment.ex:346-393)."""
import struct
import subprocess

import numpy as np

TYPE_CODES = {np.dtype(np.uint8): 0, np.dtype(np.uint16): 1, np.dtype(np.float32): 2,
              np.dtype(np.int32): 3}
TYPES = {v: k for k, v in TYPE_CODES.items()}


def name(text):
    b = text.encode()
    return bytes([len(b)]) + b


def configure_record(segment_id, geometry, members):
    """members: [(kind, {setting: value})] (native_segment.ex:256-273)."""
    out = bytes([1]) + struct.pack("<IHHHHB", segment_id, geometry["width"], geometry["height"],
                                   geometry["frame_width"], geometry["frame_height"], len(members))
    for kind, settings in members:
        out += name(kind) + bytes([len(settings)])
        for key, value in settings.items():
            out += name(key) + struct.pack("<d", float(value))
    return out


def run_record(segment_id, inputs, entries):
    """inputs: one {name: f32 values} per member, written sorted by name
    (native_segment.ex:292-309); entries: [(field, 2-D array)] (331-344)."""
    out = bytes([2]) + struct.pack("<I", segment_id) + bytes([len(inputs)])
    for member in inputs:
        out += bytes([len(member)])
        for key in sorted(member):
            values = np.ascontiguousarray(np.atleast_1d(member[key]), "<f4")
            out += name(key) + struct.pack("<H", values.size) + values.tobytes()
    out += bytes([len(entries)])
    for field, tensor in entries:
        tensor = np.ascontiguousarray(tensor)
        h, w = tensor.shape
        out += name(field) + bytes([TYPE_CODES[tensor.dtype], 2]) + struct.pack("<II", h, w)
        out += tensor.tobytes()
    return out


def release_record(segment_id):
    return bytes([3]) + struct.pack("<I", segment_id)


def decode_outputs(record):
    """(times_us, {name: array}) of a tag-8 reply."""
    assert record[0] == 8, record[:64]
    at = 1
    count = record[at]
    at += 1
    times = list(struct.unpack_from(f"<{count}I", record, at))
    at += 4 * count
    n = record[at]
    at += 1
    outputs = {}
    for _ in range(n):
        length = record[at]
        key = record[at + 1:at + 1 + length].decode()
        at += 1 + length
        dtype, rank = TYPES[record[at]], record[at + 1]
        at += 2
        shape = struct.unpack_from(f"<{rank}I", record, at)
        at += 4 * rank
        size = int(np.prod(shape, dtype=np.int64)) * dtype.itemsize
        outputs[key] = np.frombuffer(record, dtype, int(np.prod(shape)), at).reshape(shape).copy()
        at += size
    assert at == len(record)
    return times, outputs


class Port:
    """nxs_port as a child process, as NxStereo.Matcher opens stereo_match."""

    def __init__(self, path, *args):
        self.proc = subprocess.Popen([path, *args], stdin=subprocess.PIPE, stdout=subprocess.PIPE)

    def send(self, record):
        self.proc.stdin.write(struct.pack(">I", len(record)) + record)
        self.proc.stdin.flush()

    def receive(self):
        """The next record that is not a log record; log records are kept."""
        while True:
            head = self.proc.stdout.read(4)
            if len(head) < 4:
                return None
            record = self.proc.stdout.read(struct.unpack(">I", head)[0])
            if record[:1] != b"\x02":
                return record
            self.logs.append((record[1], record[2:].decode()))

    logs = []

    def close(self):
        self.proc.stdin.close()
        code = self.proc.wait(timeout=60)
        self.proc.stdout.close()
        return code
