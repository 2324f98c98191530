"""The NxStereo.Stage behaviour for the stages this library computes, with the
reference's settings checker (lib/nx_stereo/stage.ex).

A stage is a class with the reference's callbacks as static methods:
`settings()`, `requires()`, `provides()`, `init(settings, geometry)`,
`params(state, geometry)`, `carry(state, geometry)`, `compute(state)`,
`native_kind()`, `native_settings(state)` and `native_constants()`. Results
follow the reference's tagged tuples: ("ok", value) or ("error", message).

Settings, defaults, ranges and refusals are the reference's
(stage/disparity.ex:35-114, stage/rectification.ex:28-45,
stage/speckle_filter.ex:13-47, stage/temporal_filter.ex:25-59,
stage/depth.ex:19-22, stage/point_cloud.ex:58-121, stage/quality.ex:12-24).
Beyond the reference, Disparity also takes num_disparities of 96, 192 and 256,
and its coarse-to-fine search may be pinned to the native matcher.
"""
import numpy as np

MAX_PENALTY = 79
DEFAULT_UNIQUENESS = 1.0526315789473684


def _typed(kind, value):
    if kind == "integer":
        return isinstance(value, (int, np.integer)) and not isinstance(value, bool)
    if kind == "float":
        return isinstance(value, (int, float, np.integer, np.floating)) and not isinstance(value, bool)
    if kind == "boolean":
        return isinstance(value, bool)
    if kind == "string":
        return isinstance(value, str)
    if kind == "atom":
        return value is None or isinstance(value, str)
    return False


def _accepts(setting, value):
    if "values" in setting:
        return value in setting["values"]
    if "range" in setting:
        lo, hi = setting["range"]
        if not (_typed(setting["type"], value) and lo <= value <= hi):
            return False
        if "step" in setting:
            return round((value - lo) * 1_000_000) % round(setting["step"] * 1_000_000) == 0
        return True
    return _typed(setting["type"], value)


def _accepted(setting):
    if "values" in setting:
        return f"one of {setting['values']}"
    if "range" in setting:
        return f"from {setting['range'][0]} to {setting['range'][1]}"
    return f"of type {setting['type']}"


def settings(given, defaults):
    """`given` over `defaults` (a list of (key, default)); an unknown key is an error
    (stage.ex:133-143)."""
    given = dict(given or {})
    names = [k for k, _ in defaults]
    unknown = [k for k in given if k not in names]
    if unknown:
        return ("error", f"unknown settings {unknown}")
    values = dict(defaults)
    values.update(given)
    return ("ok", values)


def init_settings(module, given):
    """stage.ex:153-212: the declared defaults, each value checked, then the order."""
    declared = module.settings()
    status, values = settings(given, [(k, s["default"]) for k, s in declared])
    if status != "ok":
        return (status, values)
    for key, setting in declared:
        value = values[key]
        if value is None and setting["default"] is None:
            continue
        if not _accepts(setting, value):
            return ("error", f"{key} must be {_accepted(setting)}, got {value!r}")
    for key, setting in declared:
        other = setting.get("greater_than")
        if other and values[key] <= values[other]:
            return ("error", f"{key} must be above {other} ({values[other]}), got {values[key]}")
    return ("ok", values)


def size(geometry):
    return (geometry["height"], geometry["width"])


class Stage:
    @staticmethod
    def settings():
        return []

    @staticmethod
    def params(state, geometry):
        return {}

    @staticmethod
    def carry(state, geometry):
        return {}

    @staticmethod
    def compute(state):
        return None

    @staticmethod
    def native_settings(state):
        return []

    @staticmethod
    def native_constants():
        return {}

    @staticmethod
    def device_only():
        return []


class Rectification(Stage):
    """Rectifies :left_frame and :right_frame into :left and :right."""

    @staticmethod
    def requires():
        return ["left_frame", "right_frame"]

    @staticmethod
    def provides():
        return ["left", "right"]

    @staticmethod
    def settings():
        return [("right_row_offset", {"default": 0.0, "type": "float", "range": (-8, 8),
                                      "live": True})]

    @staticmethod
    def init(given, geometry):
        if geometry["frame_width"] < geometry["width"] or geometry["frame_height"] < geometry["height"]:
            return ("error", f"rectification only shrinks: {geometry['frame_width']}x"
                             f"{geometry['frame_height']} frames are smaller than the "
                             f"{geometry['width']}x{geometry['height']} working size")
        status, state = init_settings(Rectification, given)
        if status != "ok":
            return (status, state)
        state["size"] = size(geometry)
        return ("ok", state)

    @staticmethod
    def params(state, geometry):
        from . import rectify

        return {"left": geometry["left_camera"],
                "right": rectify.move_rows(geometry["right_camera"], state["right_row_offset"])}

    @staticmethod
    def native_kind():
        return "rectification"


class Disparity(Stage):
    """Matches :left and :right into :disparity, unmatched pixels at -1.0."""

    @staticmethod
    def settings():
        return [
            ("p1", {"default": 8, "type": "integer", "range": (0, MAX_PENALTY - 1), "live": True}),
            ("p2", {"default": 64, "type": "integer", "range": (1, MAX_PENALTY),
                    "greater_than": "p1", "live": True}),
            ("uniqueness", {"default": DEFAULT_UNIQUENESS, "type": "float", "range": (1, 3),
                            "live": True}),
            ("num_disparities", {"default": 64, "type": "integer",
                                 "values": [64, 96, 128, 192, 256]}),
            ("paths", {"default": 8, "type": "integer", "values": [3, 8]}),
            ("search", {"default": "full", "type": "string",
                        "values": ["full", "coarse_to_fine"]}),
            ("coarse_paths", {"when": {"search": "coarse_to_fine"}, "default": None,
                              "type": "integer", "values": [3, 8]}),
            ("band", {"when": {"search": "coarse_to_fine"}, "default": 16, "type": "integer",
                      "values": [8, 16, 32, 64]}),
            ("margin", {"when": {"search": "coarse_to_fine"}, "default": 4, "type": "integer",
                        "range": (0, 63)}),
            ("fine_census", {"when": {"search": "coarse_to_fine"}, "default": "sparse_9x7",
                             "type": "atom",
                             "values": ["sparse_9x7", "dense_9x5", "dense_9x5_blend"]}),
            ("matcher", {"default": None, "type": "atom", "values": [None, "nx", "native"]}),
        ]

    @staticmethod
    def requires():
        return ["left", "right"]

    @staticmethod
    def provides():
        return ["disparity"]

    @staticmethod
    def init(given, geometry):
        """stage/disparity.ex:120-128 and its checks (196-219). Beyond the
        reference, the coarse-to-fine search may be pinned to the native
        matcher (matcher "native"): this library computes it."""
        status, state = init_settings(Disparity, given)
        if status != "ok":
            return (status, state)
        if state["coarse_paths"] is None:
            state["coarse_paths"] = state["paths"]
        if state["search"] == "coarse_to_fine":
            if state["num_disparities"] != 128:
                return ("error", "coarse_to_fine searches 128 disparities, got "
                                 f"{state['num_disparities']}")
            width, height = geometry["width"], geometry["height"]
            if width % 2 or height % 2:
                return ("error", f"coarse_to_fine needs an even width and height, got "
                                 f"{width}x{height}")
            if state["margin"] >= state["band"]:
                return ("error", f"margin must be below band ({state['band']}), got "
                                 f"{state['margin']}")
        elif state["fine_census"] != "sparse_9x7":
            return ("error", "fine_census requires coarse_to_fine search")
        return ("ok", state)

    @staticmethod
    def params(state, geometry):
        return {k: state[k] for k in ("p1", "p2", "uniqueness")}

    @staticmethod
    def compute(state):
        """stage/disparity.ex:165-166: coarse_to_fine is computed in Nx unless pinned."""
        if state.get("search") == "coarse_to_fine":
            return state.get("matcher") or "nx"
        return state.get("matcher")

    @staticmethod
    def native_kind():
        return "disparity"

    @staticmethod
    def native_settings(state):
        """The member's build settings (stage/disparity.ex:171); the
        coarse-to-fine search adds its own, the census window as its index."""
        out = [("num_disparities", state["num_disparities"]), ("paths", state["paths"])]
        if state["search"] == "coarse_to_fine":
            windows = ["sparse_9x7", "dense_9x5", "dense_9x5_blend"]
            out += [("coarse_to_fine", 1), ("band", state["band"]), ("margin", state["margin"]),
                    ("coarse_paths", state["coarse_paths"]),
                    ("fine_census", windows.index(state["fine_census"]))]
        return out


class SpeckleFilter(Stage):
    """Drops speckles from :disparity: 7x7 support of at least min_support."""

    RADIUS = 3

    @staticmethod
    def settings():
        neighbours = (2 * SpeckleFilter.RADIUS + 1) ** 2 - 1
        return [("min_support", {"default": 12, "type": "integer", "range": (0, neighbours),
                                 "live": True}),
                ("max_diff", {"default": 1.0, "type": "float", "range": (0, 8), "live": True})]

    @staticmethod
    def requires():
        return ["disparity"]

    @staticmethod
    def provides():
        return ["disparity"]

    @staticmethod
    def init(given, geometry):
        return init_settings(SpeckleFilter, given)

    @staticmethod
    def params(state, geometry):
        return {k: state[k] for k in ("min_support", "max_diff")}

    @staticmethod
    def native_kind():
        return "speckle_filter"

    @staticmethod
    def native_constants():
        return {"radius": SpeckleFilter.RADIUS}


class TemporalFilter(Stage):
    """Smooths :disparity over successive pairs, carrying previous and missed."""

    MAX_MISSED = 255

    @staticmethod
    def settings():
        return [("alpha", {"default": 0.4, "type": "float", "range": (0.05, 1), "live": True}),
                ("delta", {"default": 2.0, "type": "float", "range": (0, 8), "live": True}),
                ("hold", {"default": 2, "type": "integer", "range": (0, 10), "live": True})]

    @staticmethod
    def requires():
        return ["disparity"]

    @staticmethod
    def provides():
        return ["disparity"]

    @staticmethod
    def init(given, geometry):
        status, state = init_settings(TemporalFilter, given)
        if status == "ok":
            state["size"] = size(geometry)
        return (status, state)

    @staticmethod
    def params(state, geometry):
        return {k: state[k] for k in ("alpha", "delta", "hold")}

    @staticmethod
    def carry(state, geometry):
        return {"previous": np.full(state["size"], -1.0, np.float32),
                "missed": np.zeros(state["size"], np.float32)}

    @staticmethod
    def native_kind():
        return "temporal_filter"

    @staticmethod
    def native_constants():
        return {"max_missed": float(TemporalFilter.MAX_MISSED)}


class Depth(Stage):
    """:depth_mm (u16) and :depth_m (f32, left on the device) from :disparity."""

    @staticmethod
    def requires():
        return ["disparity"]

    @staticmethod
    def provides():
        return ["depth_mm", "depth_m"]

    @staticmethod
    def device_only():
        return ["depth_m"]

    @staticmethod
    def init(given, geometry):
        status, value = settings(given, [])
        return ("ok", None) if status == "ok" else (status, value)

    @staticmethod
    def params(state, geometry):
        return {"focal_length_px": geometry["focal_length_px"],
                "baseline_m": geometry["baseline_m"]}

    @staticmethod
    def native_kind():
        return "depth"


class PointCloud(Stage):
    """:cloud_grid and :cloud_points from :depth_m, NaN outside 5 cm to 20 m."""

    MIN_DEPTH_M = 0.05
    MAX_DEPTH_M = 20.0

    @staticmethod
    def settings():
        return [("decimation", {"default": 4, "type": "integer", "range": (1, 16), "step": 1})]

    @staticmethod
    def requires():
        return ["depth_m"]

    @staticmethod
    def provides():
        return ["cloud_grid", "cloud_points"]

    @staticmethod
    def init(given, geometry):
        status, state = init_settings(PointCloud, given)
        if status != "ok":
            return (status, state)
        if state["decimation"] > geometry["height"] or state["decimation"] > geometry["width"]:
            return ("error", f"decimation must fit working size {geometry['width']}x"
                             f"{geometry['height']}, got {state['decimation']}")
        return ("ok", state)

    @staticmethod
    def params(state, geometry):
        cx, cy = geometry["principal_point"]
        return {"focal_length_px": geometry["focal_length_px"], "cx": cx, "cy": cy}

    @staticmethod
    def native_kind():
        return "point_cloud"

    @staticmethod
    def native_settings(state):
        return [("decimation", state["decimation"])]

    @staticmethod
    def native_constants():
        return {"min_depth_m": PointCloud.MIN_DEPTH_M, "max_depth_m": PointCloud.MAX_DEPTH_M}


class Quality(Stage):
    """:quality_sums of :disparity, carrying the previous disparity."""

    @staticmethod
    def requires():
        return ["disparity"]

    @staticmethod
    def provides():
        return ["quality_sums"]

    @staticmethod
    def init(given, geometry):
        status, value = settings(given, [])
        return ("ok", {"size": size(geometry)}) if status == "ok" else (status, value)

    @staticmethod
    def carry(state, geometry):
        return {"previous": np.full(state["size"], -1.0, np.float32)}

    @staticmethod
    def native_kind():
        return "quality"


def disparity_stats(sums, pixels):
    """NxStereo.Diagnostics.disparity_stats/2 (lib/nx_stereo/diagnostics.ex:273-298)."""
    matched, total, squares, both, change = [float(v) for v in sums]
    mean = total / max(matched, 1)
    variance = max(squares / max(matched, 1) - mean * mean, 0.0)
    return {"matched": matched / pixels, "mean_px": mean, "spread_px": variance ** 0.5,
            "jitter_px": change / max(both, 1)}
