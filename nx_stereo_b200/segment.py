"""The NxStereo.Segment behaviour (lib/nx_stereo/segment.ex) and CudaSegment,
the drop-in for NativeSegment (lib/nx_stereo/native_segment.ex) that computes
its stages with this library's kernels through the C ABI.

A pair goes through a segment in three steps, as in the reference:
`send_request` hands its entries to the device without waiting,
`await_`/`response` recognise its reply, and `collect` returns what it
brought back; `run` does all three. Up to `depth()` pairs may be at the
device at once, and their replies complete in the order sent: a segment
whose stages carry state from pair to pair computes them one after another,
one whose stages carry nothing computes neighbouring pairs at once on two
streams. A reply ("error", reason) fails
that pair only; ("stop", reason) says the device refuses the segment itself.
"""
import itertools
import threading
import time
import weakref

import numpy as np

from . import native
from . import stage as stage_module

FRAMES = ["left_frame", "right_frame"]
IMAGES = ["left", "right"]
MAPS = ["disparity"]


# ---------------------------------------------------------------- segment.ex helpers
def members(stages, geometry):
    """Each stage (a class, or (class, settings)) initialised for `geometry`
    (segment.ex:168-186); or the first refusal, prefixed with its name."""
    result = []
    for entry in stages:
        module, given = (entry, {}) if isinstance(entry, type) else entry
        status, state = module.init(given, geometry)
        if status != "ok":
            return ("error", f"{module.__name__}: {state}")
        result.append({"module": module, "name": module.__name__, "state": state})
    return ("ok", result)


def entry_fields(members_):
    """The tensors members read that no member before the reader provides (segment.ex:188-201)."""
    entry, provided = [], set()
    for member in members_:
        for field in member["module"].requires():
            if field not in provided and field not in entry:
                entry.append(field)
        provided |= set(member["module"].provides())
    return entry


def entry_spec(field, geometry):
    if field in FRAMES:
        return ((geometry["frame_height"], geometry["frame_width"]), np.uint8)
    if field in IMAGES:
        return ((geometry["height"], geometry["width"]), np.uint8)
    if field in MAPS:
        return ((geometry["height"], geometry["width"]), np.float32)
    return None


def entry_specs(members_, geometry):
    """Each entry field with its shape and type (segment.ex:203-250)."""
    specs = []
    for field in entry_fields(members_):
        spec = entry_spec(field, geometry)
        if spec is None:
            return ("error", f"no stage before it provides :{field}, and a segment cannot take "
                             "it as an entry")
        specs.append((field, spec))
    return ("ok", specs)


def entry_tensors(entries, specs):
    """The entries the specs name, each of its shape, cast to its type; or why not
    (segment.ex:255-304): ("frame_size", field, shape, expected), ("missing_entry",
    field) or ("not_a_tensor", field, value)."""
    entries = dict(entries)
    tensors = []
    for field, (expected, dtype) in specs:
        if field not in entries:
            return ("error", ("missing_entry", field))
        value = entries[field]
        if not isinstance(value, np.ndarray):
            return ("error", ("not_a_tensor", field, value))
        if tuple(value.shape) != tuple(expected):
            return ("error", ("frame_size", field, tuple(value.shape), tuple(expected)))
        tensors.append((field, np.ascontiguousarray(value.astype(dtype, copy=False))))
    return ("ok", tensors)


def run(module, entries, segment, timeout):
    """segment.ex:154-166: the outputs merged over the entries other than the frames."""
    sent = module.send_request(entries, segment)
    if sent[0] != "ok":
        return ("refused", sent[1])
    reply = module.await_(sent[1], segment, timeout)
    if reply == "timeout" or reply[0] != "ok":
        return reply
    _, outputs, segment, _done_ns = reply
    collected = module.collect(outputs, segment, timeout)
    if collected == "timeout" or collected[0] != "ok":
        return collected
    merged = {k: v for k, v in dict(entries).items() if k not in FRAMES}
    merged.update(collected[1])
    return ("ok", merged, segment)


def flatten(params, prefix=""):
    """native_segment.ex:311-322: nested maps become "prefix.key", sorted by name."""
    flat = []
    for key, value in params.items():
        if isinstance(value, dict):
            flat += flatten(value, f"{prefix}{key}.")
        else:
            flat.append((f"{prefix}{key}", np.atleast_1d(np.asarray(value, np.float32)).ravel()))
    return sorted(flat)


# ---------------------------------------------------------------- CudaSegment
_context_lock = threading.Lock()
_contexts = {}
_ids = itertools.count(1)


def context(device=0):
    """The process's context on `device`, opened once."""
    with _context_lock:
        if device not in _contexts:
            _contexts[device] = native.Context(device)
        return _contexts[device]


class CudaSegment:
    """A list of stages computed on a B200 by this library's kernels, run on
    each pair as one request: the counterpart of NativeSegment with the same
    stages, settings, params and outputs (native_segment.ex:1-43).

    Building does not reach the device: the segment is configured on its first
    pair. A configuration the library refuses answers that pair with
    ("stop", reason). The outputs are numpy arrays by name; depth_m stays on
    the device. Dropping the segment releases it on the device, as the Port
    releases a segment when its owner exits (matcher.ex:148-160).
    """

    DEPTH = 4

    def __init__(self, device, members_, specs, geometry):
        self.device = device
        self.id = next(_ids) & 0xFFFFFFFF
        self.version = 0
        self.configured_version = None
        self.members = members_
        self.specs = specs
        self.geometry = geometry
        self.inputs = _inputs(members_, geometry)
        self._prepared = None  # (inputs, their PreparedParams)
        self._times = []
        self._timed = None  # the last reply's request, until its member times are read
        self._finalizer = weakref.finalize(self, _release, device, self.id)

    # -- the behaviour's callbacks, as functions of the class (module-like)
    @staticmethod
    def compute(segment):
        return {"runs_on": "gpu", "implementation": "cuda", "backend": "nx_stereo_b200"}

    @staticmethod
    def depth():
        """Pairs that may be at the device at once."""
        return CudaSegment.DEPTH

    @staticmethod
    def accepts(module, state, compute):
        """native_segment.ex:83-91: a native kind, and settings that do not ask for Nx."""
        return compute == "native" and _refusal({"module": module, "state": state}) is None

    @staticmethod
    def build(members_, geometry, opts=None):
        opts = dict(opts or {})
        unknown = [k for k in opts if k != "device"]
        if unknown:
            return ("error", f"unknown build options {unknown}")
        for member in members_:
            why = _refusal(member)
            if why:
                return ("error", why)
        status, specs = entry_specs(members_, geometry)
        if status != "ok":
            return (status, specs)
        return ("ok", CudaSegment(opts.get("device", 0), members_, specs, geometry))

    @staticmethod
    def reload(segment, members_, geometry):
        """Re-initialised for a new geometry of the same size: configured again on
        the next pair, carrying nothing over."""
        segment.members = members_
        segment.geometry = geometry
        segment.inputs = _inputs(members_, geometry)
        segment.version += 1
        return segment

    @staticmethod
    def put_member_state(segment, index, state):
        segment.members[index] = dict(segment.members[index], state=state)
        segment.inputs = _inputs(segment.members, segment.geometry)
        return segment

    @staticmethod
    def merge_carry(current, replied):
        """The device keeps what the stages carry: `current`."""
        return current

    @staticmethod
    def send_request(entries, segment):
        status, tensors = entry_tensors(entries, segment.specs)
        if status != "ok":
            return (status, tensors)
        ctx = context(segment.device)
        if segment.configured_version != segment.version:
            try:
                ctx.configure(segment.id, _geometry(segment.geometry), _configuration(segment))
            except native.NativeError as error:
                return ("ok", _Refused(error.message))
            segment.configured_version = segment.version
        # The params are marshalled again only when they change (reload and
        # put_member_state give the segment a new inputs list).
        prepared = segment._prepared
        if prepared is None or prepared[0] is not segment.inputs:
            prepared = segment._prepared = (segment.inputs, native.PreparedParams(segment.inputs))
        try:
            request = ctx.run_async(segment.id, prepared[1], dict(tensors))
        except native.NativeError as error:
            return ("ok", _Failed(error.message))
        return ("ok", request)

    @staticmethod
    def response(message, request, segment):
        """The reply when `message` is `request` done; ("no_reply",) otherwise."""
        if message is not request:
            return ("no_reply",)
        return CudaSegment.await_(request, segment, 0) if _done(request) else ("no_reply",)

    @staticmethod
    def await_(request, segment, timeout):
        if isinstance(request, _Refused):
            return ("stop", request.reason)
        if isinstance(request, _Failed):
            return ("error", request.reason)
        try:
            if not request.wait(-1 if timeout is None else int(timeout)):
                return "timeout"
            # Views of the request's pinned memory: the request lives as long as they do.
            outputs = request.outputs(copy=False)
            # The member times are read from the device's events only when asked
            # for (member_times): reading them costs host time on every pair.
            segment._timed = request
        except native.NativeError as error:
            request.free()
            return ("error", error.message)
        if "cloud_points" in outputs:
            outputs["cloud_points"] = outputs["cloud_points"].reshape(())
        return ("ok", outputs, segment, time.monotonic_ns())

    @staticmethod
    def collect(outputs, segment, timeout):
        """The reply brought the outputs back: nothing to download."""
        return ("ok", outputs)

    @property
    def times_us(self):
        """Each member's device time (us) for the last pair replied to."""
        if self._timed is not None:
            self._times, self._timed = self._timed.times_us(), None
        return self._times

    @staticmethod
    def member_times(segment):
        return [(m["name"], t * 1000) for m, t in zip(segment.members, segment.times_us)]

    def release(self):
        self._finalizer()


class _Refused:
    def __init__(self, reason):
        self.reason = reason


class _Failed:
    def __init__(self, reason):
        self.reason = reason


def _done(request):
    try:
        return request.poll()
    except native.NativeError:
        return True


def _release(device, segment_id):
    with _context_lock:
        ctx = _contexts.get(device)
    if ctx is not None and ctx.handle:
        try:
            ctx.release(segment_id)
        except Exception:
            pass


def _refusal(member):
    module = member["module"]
    kind = getattr(module, "native_kind", None)
    if kind is None:
        return f"{module.__name__} has no native implementation"
    if module.compute(member["state"]) == "nx":
        return f"{module.__name__} is computed in Nx, as its settings ask"
    return None


def _geometry(g):
    return (g["width"], g["height"], g["frame_width"], g["frame_height"])


def _setting_float(value):
    return float(value)


def _configuration(segment):
    """Each member's kind and its build settings and native constants (native_segment.ex:256-290)."""
    config = []
    for member in segment.members:
        module = member["module"]
        settings = {k: _setting_float(v) for k, v in module.native_settings(member["state"])}
        settings.update({k: _setting_float(v) for k, v in sorted(module.native_constants().items())})
        config.append((module.native_kind(), settings))
    return config


def _inputs(members_, geometry):
    """Each member's params as f32 values by flattened name (native_segment.ex:292-309)."""
    return [dict(flatten(m["module"].params(m["state"], geometry))) for m in members_]


def standard_geometry(width, height, frame_width=None, frame_height=None, the_rig=None):
    """A geometry map with the keys the stages read, from a rig built by
    `scene.rig` (cameras through `rectify.camera`)."""
    from . import scene

    # The calibration at the working size, as Stage.Rectification takes it.
    the_rig = the_rig or scene.rig(width, height)
    cams = scene.cameras(the_rig)
    return {"width": width, "height": height, "frame_width": frame_width or width,
            "frame_height": frame_height or height,
            "focal_length_px": the_rig["focal_length_px"], "baseline_m": the_rig["baseline_m"],
            "principal_point": the_rig["principal_point"], "left_camera": cams["left"],
            "right_camera": cams["right"]}


PIPELINE = [stage_module.Rectification, (stage_module.Disparity, {"num_disparities": 128}),
            stage_module.SpeckleFilter, stage_module.Depth, stage_module.PointCloud]
