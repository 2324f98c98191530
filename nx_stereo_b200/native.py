"""ctypes binding of the C ABI in include/nx_stereo_b200.h.

The library (nx_stereo_b200/libnxs_b200.so) is the only compute path: there is
no CPU fallback, and loading fails loudly when it is missing or cannot open a
CUDA device.
"""
import ctypes
import struct
import threading
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBRARY = os.path.join(HERE, "libnxs_b200.so")

# nxs_status
OK, PENDING, REFUSED, BAD_RUN, CUDA_ERROR, TIMEOUT, BAD_ARGUMENT, NO_SEGMENT = range(8)
STATUS_NAMES = ["ok", "pending", "refused", "bad_run", "cuda_error", "timeout", "bad_argument",
                "no_segment"]
# element types (tensor.rs:25-30)
U8, U16, F32, S32 = 0, 1, 2, 3
DTYPES = {U8: np.uint8, U16: np.uint16, F32: np.float32, S32: np.int32}
TYPE_CODES = {np.dtype(np.uint8): U8, np.dtype(np.uint16): U16, np.dtype(np.float32): F32,
              np.dtype(np.int32): S32}


class NativeError(RuntimeError):
    """A status other than OK from the library, with its message."""

    def __init__(self, status, message):
        super().__init__(f"{STATUS_NAMES[status] if 0 <= status < 8 else status}: {message}")
        self.status = status
        self.message = message


class Setting(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char_p), ("value", ctypes.c_double)]


class Member(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_char_p), ("n_settings", ctypes.c_uint32),
                ("settings", ctypes.POINTER(Setting))]


class Geometry(ctypes.Structure):
    _fields_ = [("width", ctypes.c_uint32), ("height", ctypes.c_uint32),
                ("frame_width", ctypes.c_uint32), ("frame_height", ctypes.c_uint32)]


class Param(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char_p), ("count", ctypes.c_uint32),
                ("values", ctypes.POINTER(ctypes.c_float))]


class MemberParams(ctypes.Structure):
    _fields_ = [("n_params", ctypes.c_uint32), ("params", ctypes.POINTER(Param))]


class Tensor(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char_p), ("type", ctypes.c_uint32), ("rank", ctypes.c_uint32),
                ("dims", ctypes.c_uint32 * 4), ("data", ctypes.c_void_p),
                ("bytes", ctypes.c_uint64)]


class SgmParams(ctypes.Structure):
    _fields_ = [("disparities", ctypes.c_uint32), ("paths", ctypes.c_uint32),
                ("p1", ctypes.c_uint32), ("p2", ctypes.c_uint32),
                ("uniqueness", ctypes.c_float), ("stage_mask", ctypes.c_uint32)]


class BandParams(ctypes.Structure):
    _fields_ = [("sgm", SgmParams), ("band", ctypes.c_uint32), ("margin", ctypes.c_uint32),
                ("coarse_paths", ctypes.c_uint32), ("census", ctypes.c_uint32)]


CENSUS_WINDOWS = {"sparse_9x7": 0, "dense_9x5": 1, "dense_9x5_blend": 2}


class Camera(ctypes.Structure):
    _fields_ = [("k", ctypes.c_float * 9), ("d", ctypes.c_float * 5),
                ("inverse_pr", ctypes.c_float * 9)]


class BatchPair(ctypes.Structure):
    _fields_ = [("width", ctypes.c_uint32), ("height", ctypes.c_uint32), ("params", SgmParams)]


class BatchTuning(ctypes.Structure):
    _fields_ = [("blocks_per_sm", ctypes.c_int32), ("cost_rows", ctypes.c_int32),
                ("select_passes", ctypes.c_int32), ("group_pairs", ctypes.c_int32),
                ("quantum_us", ctypes.c_float), ("order", ctypes.c_int32),
                ("path_words", ctypes.c_int32), ("engine", ctypes.c_int32),
                ("streams", ctypes.c_int32), ("wait_limit_us", ctypes.c_uint32)]


class BatchStats(ctypes.Structure):
    _fields_ = [("pairs", ctypes.c_uint32), ("items", ctypes.c_uint32), ("runs", ctypes.c_uint32),
                ("blocks", ctypes.c_uint32), ("shared_bytes", ctypes.c_uint64),
                ("device_bytes", ctypes.c_uint64), ("input_bytes", ctypes.c_uint64),
                ("output_bytes", ctypes.c_uint64)]


DONE_FN = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_uint64)

_P = ctypes.c_void_p
_u32, _u64, _f, _i = ctypes.c_uint32, ctypes.c_uint64, ctypes.c_float, ctypes.c_int
_err = [ctypes.c_char_p, ctypes.c_size_t]

# Every symbol the header declares, with its signature.
SIGNATURES = {
    "nxs_create": (_i, [_i, ctypes.POINTER(_P)] + _err),
    "nxs_destroy": (None, [_P]),
    "nxs_version": (ctypes.c_char_p, []),
    "nxs_configure": (_i, [_P, _u32, ctypes.POINTER(Geometry), _u32, ctypes.POINTER(Member)] + _err),
    "nxs_run_async": (_i, [_P, _u32, _u32, ctypes.POINTER(MemberParams), _u32,
                           ctypes.POINTER(Tensor), DONE_FN, _P, _u64, ctypes.POINTER(_P)] + _err),
    "nxs_request_poll": (_i, [_P] + _err),
    "nxs_request_wait": (_i, [_P, ctypes.c_int64] + _err),
    "nxs_request_outputs": (_i, [_P, ctypes.POINTER(_u32), ctypes.POINTER(ctypes.POINTER(Tensor))]),
    "nxs_request_times": (_i, [_P, ctypes.POINTER(_u32), ctypes.POINTER(ctypes.POINTER(_u32))]),
    "nxs_request_free": (None, [_P]),
    "nxs_request_done_ns": (_u64, [_P]),
    "nxs_device_memory": (_i, [_P, ctypes.POINTER(_u64), ctypes.POINTER(_u64)]),
    "nxs_release": (_i, [_P, _u32]),
    "nxs_sgm_check": (_i, [ctypes.POINTER(SgmParams), _u32, _u32] + _err),
    "nxs_sgm": (_i, [_P, _P, _P, _u32, _u32, ctypes.POINTER(SgmParams), _P] + _err),
    "nxs_sgm_device": (_i, [_P, _P, _P, _u32, _u32, ctypes.POINTER(SgmParams), _P, _P] + _err),
    "nxs_sgm_scratch_bytes": (_u64, [_u32, _u32, _u32]),
    "nxs_set_path_words": (_i, [_u32, _u32]),
    "nxs_path_words": (_u32, [_u32]),
    "nxs_set_path_sums": (_i, [_u32]),
    "nxs_path_sums": (_u32, [_u32, _u32, _u32]),
    "nxs_set_path_tiles": (_i, [_u32]),
    "nxs_set_split_lanes": (_i, [_u32]),
    "nxs_set_lean_select": (_i, [_u32]),
    "nxs_lean_select": (_u32, []),
    "nxs_path_tiles": (_u32, []),
    "nxs_path_wait_failures": (_u32, []),
    "nxs_band_check": (_i, [ctypes.POINTER(BandParams), _u32, _u32, ctypes.c_int32] + _err),
    "nxs_band_scratch_bytes": (_u64, [_u32, _u32, _u32, ctypes.c_int32]),
    "nxs_sgm_band_device": (_i, [_P, _P, _P, _P, _u32, _u32, ctypes.POINTER(BandParams), _P, _P]
                            + _err),
    "nxs_sgm_coarse_to_fine_device": (_i, [_P, _P, _P, _u32, _u32, ctypes.POINTER(BandParams),
                                           _P, _P, _P] + _err),
    "nxs_sgm_coarse_to_fine": (_i, [_P, _P, _P, _u32, _u32, ctypes.POINTER(BandParams), _P]
                               + _err),
    "nxs_census_device": (_i, [_P, _u32, _u32, _P, _P]),
    "nxs_census_pair_device": (_i, [_P, _P, _u32, _u32, _P, _P, _P]),
    "nxs_check_median_device": (_i, [_P, _P, _u32, _u32, _u32, _P, _P]),
    "nxs_costs_device": (_i, [_P, _P, _u32, _u32, _u32, _P, _P]),
    "nxs_aggregate_device": (_i, [_P, _P, _u32, _u32, _u32, _u32, _u32, _u32, _P, _P]),
    "nxs_paths_device": (_i, [_P, _u32, _u32, _u32, _u32, _u32, _u32, _P, _P]),
    "nxs_select_paths_device": (_i, [_P, _u32, _u32, _u32, _u32, _f, _P, _P, _P]),
    "nxs_select_device": (_i, [_P, _u32, _u32, _u32, _f, _P, _P, _P]),
    "nxs_matcher_span": (_u32, [_u32]),
    "nxs_costs_device_ordered": (_i, [_P, _P, _u32, _u32, _u32, _u32, _P, _P]),
    "nxs_census_costs_device_ordered": (_i, [_P, _P, _u32, _u32, _u32, _u32, _P, _P]),
    "nxs_paths_device_ordered": (_i, [_P, _u32, _u32, _u32, _u32, _u32, _u32, _u32, _P, _P]),
    "nxs_select_paths_device_ordered": (_i, [_P, _u32, _u32, _u32, _u32, _f, _u32, _P, _P, _P]),
    "nxs_path_sums_device": (_i, [_P, _u32, _u32, _u32, _u32, _u32, _u32, _P, _P]),
    "nxs_select_path_sums_device": (_i, [_P, _u32, _u32, _u32, _f, _P, _P, _P]),
    "nxs_consistency_device": (_i, [_P, _P, _u32, _u32, _P, _P]),
    "nxs_median3_device": (_i, [_P, _u32, _u32, _u32, _P, _P]),
    "nxs_rectify_device": (_i, [_P, _u32, _u32, ctypes.POINTER(Camera), _u32, _u32, _P, _P]),
    "nxs_rectify_pair_device": (_i, [_P, _P, _u32, _u32, ctypes.POINTER(Camera),
                                     ctypes.POINTER(Camera), _u32, _u32, _P, _P, _P]),
    "nxs_rectify_maps_device": (_i, [ctypes.POINTER(Camera), ctypes.POINTER(Camera), _u32, _u32,
                                     _u32, _u32, _P, _P]),
    "nxs_rectify_pair_mapped_device": (_i, [_P, _P, _u32, _u32, _P, _u32, _u32, _P, _P, _P]),
    "nxs_despeckle_device": (_i, [_P, _u32, _u32, _f, _f, _u32, _P, _P]),
    "nxs_temporal_device": (_i, [_P, _P, _P, _u64, _f, _f, _f, _f, _P]),
    "nxs_depth_device": (_i, [_P, _u64, _f, _f, _P, _P, _P]),
    "nxs_cloud_device": (_i, [_P, _u32, _u32, _u32, _f, _f, _f, _f, _f, _P, _P, _P]),
    "nxs_despeckle_depth_cloud_device": (_i, [_P, _u32, _u32, _f, _f, _u32, _f, _f, _u32, _f,
                                              _f, _f, _f, _P, _P, _P, _P, _P, _P]),
    "nxs_quality_device": (_i, [_P, _P, _u32, _u32, _P, _P]),
    "nxs_batch_default_tuning": (None, [ctypes.POINTER(BatchTuning)]),
    "nxs_batch_create": (_i, [_P, _u32, ctypes.POINTER(BatchPair), ctypes.POINTER(BatchTuning),
                              ctypes.POINTER(_P)] + _err),
    "nxs_batch_buffers": (_i, [_P, _u32, ctypes.c_int32, ctypes.POINTER(_P), ctypes.POINTER(_P),
                               ctypes.POINTER(_P)]),
    "nxs_batch_retune": (_i, [_P, ctypes.POINTER(BatchTuning)] + _err),
    "nxs_batch_run": (_i, [_P] + _err),
    "nxs_batch_launch": (_i, [_P, ctypes.c_int32, _P] + _err),
    "nxs_batch_check": (_i, [_P] + _err),
    "nxs_batch_hold_phase": (_i, [_P, _u32, _u32] + _err),
    "nxs_batch_info": (_i, [_P, ctypes.POINTER(BatchStats)]),
    "nxs_batch_clocks": (_i, [_P, ctypes.POINTER(_u64)]),
    "nxs_batch_queue": (_i, [_u32, ctypes.POINTER(BatchPair), ctypes.POINTER(BatchTuning),
                             ctypes.POINTER(_u32), ctypes.POINTER(_u32), _u32,
                             ctypes.POINTER(_u32)] + _err),
    "nxs_batch_destroy": (None, [_P]),
}

_lib = None


def library_path():
    return LIBRARY


def load():
    """The loaded library; raises when the built library is missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIBRARY):
            raise ImportError(
                f"{LIBRARY} is missing: build it with `python -m nx_stereo_b200.build` "
                "(there is no CPU fallback)")
        lib = ctypes.CDLL(LIBRARY)
        for name, (restype, argtypes) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = restype
            fn.argtypes = argtypes
        _lib = lib
    return _lib


def _check(status, buf):
    if status != OK:
        raise NativeError(status, buf.value.decode("utf-8", "replace") if buf is not None else "")


_local = threading.local()


def _errbuf():
    """This thread's error-text buffer (each call reads it before the next)."""
    buf = getattr(_local, "errbuf", None)
    if buf is None:
        buf = _local.errbuf = ctypes.create_string_buffer(1024)
    buf[0] = b"\0"
    return buf


def sgm_params(disparities=64, paths=8, p1=8, p2=64, uniqueness=1.0526315789473684,
               stage_mask=False):
    return SgmParams(disparities, paths, p1, p2, uniqueness, 1 if stage_mask else 0)


def band_params(disparities=128, paths=8, p1=8, p2=64, uniqueness=1.0526315789473684,
                stage_mask=False, band=16, margin=4, coarse_paths=None, census="sparse_9x7"):
    return BandParams(sgm_params(disparities, paths, p1, p2, uniqueness, stage_mask), band,
                      margin, coarse_paths or paths, CENSUS_WINDOWS[census])


def check_band(width, height, coarse_to_fine=True, **settings):
    """(True, "") or (False, why) for sgm_coarse_to_fine/3 (or sgm_band/4)."""
    p = band_params(**settings)
    buf = _errbuf()
    status = load().nxs_band_check(ctypes.byref(p), width, height, 1 if coarse_to_fine else 0,
                                   buf, 1024)
    return (status == OK, buf.value.decode() if status != OK else "")


def check_sgm(width, height, **settings):
    """NxStereo.sgm/3's refusal of these settings, as a NativeError, or None."""
    buf = _errbuf()
    status = load().nxs_sgm_check(ctypes.byref(sgm_params(**settings)), width, height, buf, 1024)
    return None if status == OK else NativeError(status, buf.value.decode())


def make_camera(k, d, inverse_pr):
    cam = Camera()
    cam.k[:] = [float(v) for v in np.asarray(k, np.float32).ravel()]
    cam.d[:] = [float(v) for v in np.asarray(d, np.float32).ravel()]
    cam.inverse_pr[:] = [float(v) for v in np.asarray(inverse_pr, np.float32).ravel()]
    return cam


# nxs_tensor as laid out in memory: name, type, rank, dims[4], data, bytes.
_TENSOR = struct.Struct("<QII4IQQ")
assert _TENSOR.size == ctypes.sizeof(Tensor)
_LAYOUTS = {}  # output descriptors without their addresses -> (name, dtype, shape, bytes)


class _PinnedView:
    """An array interface over a request's pinned output block; holding the
    request keeps the block from being recycled."""

    def __init__(self, request, address, shape, dtype):
        self._request = request
        self.__array_interface__ = {"data": (address, False), "shape": shape,
                                    "typestr": dtype.str, "version": 3}


class PreparedParams:
    """A segment's per-member live params marshalled once for nxs_run_async
    (a list of {name: float or sequence}, one per member, names sorted): a
    segment whose params do not change between pairs reuses it."""

    def __init__(self, params):
        self.count = len(params)
        self._keep = []
        self.members = (MemberParams * max(self.count, 1))()
        for i, member in enumerate(params):
            ps = (Param * max(len(member), 1))()
            for j, (name, value) in enumerate(sorted(member.items())):
                values = np.ascontiguousarray(np.atleast_1d(np.asarray(value, np.float32)))
                b = name.encode()
                self._keep += [b, values]
                ps[j] = Param(b, values.size, values.ctypes.data_as(ctypes.POINTER(ctypes.c_float)))
            self._keep.append(ps)
            self.members[i] = MemberParams(len(member), ps)


class Request:
    """A pair sent through a segment: wait for it, then read its outputs."""

    def __init__(self, handle, keep):
        self._handle = handle
        self._keep = keep  # the callback object must outlive the request

    def poll(self):
        buf = _errbuf()
        status = load().nxs_request_poll(self._handle, buf, 1024)
        if status == PENDING:
            return False
        _check(status, buf)
        return True

    def wait(self, timeout_ms=-1):
        buf = _errbuf()
        status = load().nxs_request_wait(self._handle, int(timeout_ms), buf, 1024)
        if status == TIMEOUT:
            return False
        _check(status, buf)
        return True

    def outputs(self, copy=True):
        """{name: numpy array}. With copy=False the arrays view the request's
        pinned host memory and keep the request alive until they are dropped."""
        n = ctypes.c_uint32()
        tensors = ctypes.POINTER(Tensor)()
        _check(load().nxs_request_outputs(self._handle, ctypes.byref(n), ctypes.byref(tensors)),
               None)
        if n.value == 0:
            return {}
        # The descriptors in one read; their names, types and shapes are the
        # segment's, so their layout is worked out once and kept.
        raw = ctypes.string_at(ctypes.addressof(tensors.contents), n.value * _TENSOR.size)
        fields = list(_TENSOR.iter_unpack(raw))
        key = tuple(f[:7] + f[8:] for f in fields)
        layout = _LAYOUTS.get(key)
        if layout is None:
            if len(_LAYOUTS) >= 256:
                _LAYOUTS.clear()
            layout = [(ctypes.string_at(f[0]).decode(), np.dtype(DTYPES[f[1]]), tuple(f[3:3 + f[2]]),
                       f[8]) for f in fields]
            _LAYOUTS[key] = layout
        # One view spanning the outputs (one pinned block when they are packed),
        # each output a slice of it.
        datas = [f[7] for f in fields]
        low = min(datas)
        high = max(d + entry[3] for d, entry in zip(datas, layout))
        block = np.asarray(_PinnedView(self, low, (high - low,), np.dtype(np.uint8)))
        result = {}
        for d, (name, dtype, shape, nbytes) in zip(datas, layout):
            view = block[d - low:d - low + nbytes].view(dtype).reshape(shape)
            result[name] = view.copy() if copy else view
        return result

    def done_ns(self):
        """time.monotonic_ns() of the device finishing the request; 0 while pending."""
        return int(load().nxs_request_done_ns(self._handle)) if self._handle else 0

    def times_us(self):
        n = ctypes.c_uint32()
        times = ctypes.POINTER(ctypes.c_uint32)()
        _check(load().nxs_request_times(self._handle, ctypes.byref(n), ctypes.byref(times)), None)
        return [times[i] for i in range(n.value)]

    def free(self):
        if self._handle:
            load().nxs_request_free(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Context:
    """A device context: the segment protocol and the direct entry points."""

    def __init__(self, device=0):
        lib = load()
        handle = ctypes.c_void_p()
        buf = _errbuf()
        _check(lib.nxs_create(device, ctypes.byref(handle), buf, 1024), buf)
        self._handle = handle
        self.device = device

    @property
    def handle(self):
        return self._handle

    def memory(self):
        """(free, total) bytes of the context's device."""
        free, total = ctypes.c_uint64(), ctypes.c_uint64()
        status = load().nxs_device_memory(self._handle, ctypes.byref(free), ctypes.byref(total))
        if status != OK:
            raise NativeError(status, "device memory")
        return free.value, total.value

    def close(self):
        if self._handle:
            load().nxs_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- the segment protocol
    def configure(self, segment, geometry, members):
        """members: [(kind, {setting: value})]; geometry: (w, h, frame_w, frame_h)."""
        keep = []
        arr = (Member * max(len(members), 1))()
        for i, (kind, settings) in enumerate(members):
            s = (Setting * max(len(settings), 1))()
            for j, (name, value) in enumerate(sorted(settings.items())):
                b = name.encode()
                keep.append(b)
                s[j] = Setting(b, float(value))
            kb = kind.encode()
            keep += [kb, s]
            arr[i] = Member(kb, len(settings), s)
        g = Geometry(*geometry)
        buf = _errbuf()
        _check(load().nxs_configure(self._handle, segment, ctypes.byref(g), len(members), arr,
                                    buf, 1024), buf)

    def run_async(self, segment, params, entries, done=None, tag=0):
        """params: per member {name: float or sequence}, or those already
        marshalled once by PreparedParams; entries: {name: ndarray}."""
        if not isinstance(params, PreparedParams):
            params = PreparedParams(params)
        mps, keep = params.members, [params]
        arrays = [np.ascontiguousarray(a) for a in entries.values()]
        # The descriptors of entries of these names, types and shapes are made
        # once a thread and reused with the new addresses (the call copies the
        # entries before it returns).
        key = tuple((name, a.dtype.str, a.shape) for name, a in zip(entries, arrays))
        cache = getattr(_local, "entries", None)
        if cache is None:
            cache = _local.entries = {}
        ts = cache.get(key)
        if ts is None:
            if len(cache) >= 64:  # shapes come and go: keep the cache small
                cache.clear()
            ts = (Tensor * max(len(arrays), 1))()
            names = [name.encode() for name in entries]
            for i, (b, a) in enumerate(zip(names, arrays)):
                dims = (ctypes.c_uint32 * 4)(*(list(a.shape) + [0] * (4 - a.ndim)))
                ts[i] = Tensor(b, TYPE_CODES[a.dtype], a.ndim, dims, 0, a.nbytes)
            ts._names = names  # the descriptors point at these bytes
            cache[key] = ts
        for i, a in enumerate(arrays):
            ts[i].data = a.ctypes.data
        keep.append(arrays)
        callback = DONE_FN(done) if done else DONE_FN()
        handle = ctypes.c_void_p()
        buf = _errbuf()
        status = load().nxs_run_async(self._handle, segment, params.count, mps, len(entries), ts,
                                      callback, None, tag, ctypes.byref(handle), buf, 1024)
        _check(status, buf)
        return Request(handle, callback)

    def release(self, segment):
        status = load().nxs_release(self._handle, segment)
        if status not in (OK, NO_SEGMENT):
            raise NativeError(status, "release")

    # ---- direct entry points
    def sgm(self, left, right, **settings):
        """NxStereo.sgm/3 of a host u8 pair; returns f32 disparity (-1 unmatched)."""
        left = np.ascontiguousarray(left, np.uint8)
        right = np.ascontiguousarray(right, np.uint8)
        h, w = left.shape
        out = np.empty((h, w), np.float32)
        p = sgm_params(**settings)
        buf = _errbuf()
        _check(load().nxs_sgm(self._handle, left.ctypes.data, right.ctypes.data, w, h,
                              ctypes.byref(p), out.ctypes.data, buf, 1024), buf)
        return out

    def sgm_coarse_to_fine(self, left, right, **settings):
        """NxStereo.sgm_coarse_to_fine/3 on a host pair (band_params' settings)."""
        left = np.ascontiguousarray(left, np.uint8)
        right = np.ascontiguousarray(right, np.uint8)
        h, w = left.shape
        out = np.empty((h, w), np.float32)
        p = band_params(**settings)
        buf = _errbuf()
        _check(load().nxs_sgm_coarse_to_fine(self._handle, left.ctypes.data, right.ctypes.data,
                                             w, h, ctypes.byref(p), out.ctypes.data, buf, 1024),
               buf)
        return out

    def sgm_coarse_to_fine_device(self, d_left, d_right, width, height, d_out, d_base=None,
                                  stream=0, **settings):
        p = band_params(**settings)
        buf = _errbuf()
        _check(load().nxs_sgm_coarse_to_fine_device(self._handle, d_left, d_right, width, height,
                                                    ctypes.byref(p), d_out, d_base, stream, buf,
                                                    1024), buf)

    def sgm_band_device(self, d_left, d_right, d_base, width, height, d_out, stream=0,
                        **settings):
        p = band_params(**settings)
        buf = _errbuf()
        _check(load().nxs_sgm_band_device(self._handle, d_left, d_right, d_base, width, height,
                                          ctypes.byref(p), d_out, stream, buf, 1024), buf)

    def sgm_device(self, d_left, d_right, width, height, d_out, stream=0, **settings):
        p = sgm_params(**settings)
        buf = _errbuf()
        _check(load().nxs_sgm_device(self._handle, d_left, d_right, width, height,
                                     ctypes.byref(p), d_out, stream, buf, 1024), buf)


def band_scratch_bytes(width, height, band, coarse_to_fine=True):
    return int(load().nxs_band_scratch_bytes(width, height, band, 1 if coarse_to_fine else 0))


def scratch_bytes(width, height, disparities):
    return int(load().nxs_sgm_scratch_bytes(width, height, disparities))


def call(name, *args):
    """Calls a device entry point by name, raising on a status other than OK."""
    status = getattr(load(), name)(*args)
    if status != OK:
        raise NativeError(status, name)
