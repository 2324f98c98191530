"""Seeded synthetic stereo inputs with the shapes and statistics of the
benchmark workloads (no dataset is used).

rectified_pair: the left image is uniform u8 noise, 3x3 box-blurred, with a
few linear gradient patches; the right image is the left one warped by a
piecewise-planar disparity field (a slanted background plane plus random
axis-aligned rectangles, each its own plane), nearer surfaces winning, holes
(occlusions) filled with fresh noise; Gaussian noise is added to both and the
result clipped to u8.

rig / raw_frames: a synthetic calibrated rig (fx = fy, principal point at the
centre, radial k1, k2, the right camera rotated about y with a baseline along
x) and the raw camera frames that rectify to a given rectified pair.
"""
import math

import numpy as np

from . import rectify


def _box3(image):
    padded = np.pad(image, 1, mode="edge")
    h, w = image.shape
    acc = np.zeros((h, w), np.float32)
    for dy in range(3):
        for dx in range(3):
            acc += padded[dy:dy + h, dx:dx + w]
    return acc / 9.0


def rectified_pair(width, height, seed=0, rectangles=6, min_disparity=4, max_disparity=56,
                   background=(10, 20), sigma=2.0, return_disparity=False, frame=0, drift=0.0):
    """A seeded pair (see the module's description). With drift > 0 the
    rectangles move: each gets a speed of up to `drift` px per frame in a
    random direction and lies where it has moved to at `frame`."""
    rng = np.random.default_rng(seed)
    left = _box3(rng.integers(0, 256, (height, width)).astype(np.float32))
    yy, xx = np.mgrid[0:height, 0:width].astype(np.float32)
    for _ in range(3):  # gradient patches
        x0, y0 = int(rng.integers(0, width // 2)), int(rng.integers(0, height // 2))
        x1 = min(width, x0 + int(rng.integers(width // 8, width // 3 + 1)))
        y1 = min(height, y0 + int(rng.integers(height // 8, height // 3 + 1)))
        gx, gy = rng.uniform(-2, 2, size=2)
        patch = 128 + gx * (xx[y0:y1, x0:x1] - x0) + gy * (yy[y0:y1, x0:x1] - y0)
        left[y0:y1, x0:x1] = 0.5 * left[y0:y1, x0:x1] + 0.5 * patch
    # Disparity field in the left view: a slanted background, then rectangles.
    b0, b1 = background
    a = rng.uniform(b0, b1)
    slope_x, slope_y = rng.uniform(-(b1 - b0) / 2, (b1 - b0) / 2, size=2)
    disparity = np.clip(a + slope_x * xx / width + slope_y * yy / height, b0, b1)
    for _ in range(rectangles):
        rw = int(rng.integers(width // 10, width // 3 + 1))
        rh = int(rng.integers(height // 10, height // 3 + 1))
        x0, y0 = int(rng.integers(0, width - rw)), int(rng.integers(0, height - rh))
        d0 = rng.uniform(min_disparity, max_disparity)
        sx, sy = rng.uniform(-4, 4, size=2)
        if drift > 0:
            speed, heading = rng.uniform(0, drift), rng.uniform(0, 2 * math.pi)
            x0 = int(np.clip(x0 + round(speed * math.cos(heading) * frame), 0, width - rw))
            y0 = int(np.clip(y0 + round(speed * math.sin(heading) * frame), 0, height - rh))
        plane = d0 + sx * (xx[y0:y0 + rh, x0:x0 + rw] - x0) / rw \
            + sy * (yy[y0:y0 + rh, x0:x0 + rw] - y0) / rh
        region = disparity[y0:y0 + rh, x0:x0 + rw]
        disparity[y0:y0 + rh, x0:x0 + rw] = np.maximum(
            region, np.clip(plane, min_disparity, max_disparity))
    # Forward warp: left pixel x lands at x - d in the right view; nearer wins.
    right = np.full((height, width), np.nan, np.float32)
    target = np.rint(xx - disparity).astype(np.int64)
    for y in range(height):
        order = np.argsort(disparity[y], kind="stable")  # far first, near last
        tx = target[y, order]
        keep = (tx >= 0) & (tx < width)
        right[y, tx[keep]] = left[y, order[keep]]
    holes = np.isnan(right)
    right[holes] = rng.integers(0, 256, int(holes.sum())).astype(np.float32)
    left = left + rng.normal(0, sigma, left.shape)
    right = right + rng.normal(0, sigma, right.shape)
    out = (np.clip(np.rint(left), 0, 255).astype(np.uint8),
           np.clip(np.rint(right), 0, 255).astype(np.uint8))
    return out + (disparity,) if return_disparity else out


def _rot_y(degrees):
    t = math.radians(degrees)
    return np.array([[math.cos(t), 0, math.sin(t)], [0, 1, 0], [-math.sin(t), 0, math.cos(t)]])


def rig(width, height, focal=873.0, k1=-0.05, k2=0.01, yaw_degrees=0.5, baseline_m=0.2):
    """A calibrated pair: per side the K, D, R, P lists camera/4 takes, plus
    the rectified focal length, baseline and principal point."""
    cx, cy = width / 2.0, height / 2.0
    k = [focal, 0.0, cx, 0.0, focal, cy, 0.0, 0.0, 1.0]
    d = [k1, k2, 0.0, 0.0, 0.0]
    # Each camera rotated half the relative yaw back into a common frame.
    r_left = _rot_y(yaw_degrees / 2.0)
    r_right = _rot_y(-yaw_degrees / 2.0)
    p_left = [focal, 0.0, cx, 0.0, 0.0, focal, cy, 0.0, 0.0, 0.0, 1.0, 0.0]
    p_right = [focal, 0.0, cx, -focal * baseline_m, 0.0, focal, cy, 0.0, 0.0, 0.0, 1.0, 0.0]
    return {
        "left": {"k": k, "d": d, "r": r_left.ravel().tolist(), "p": p_left},
        "right": {"k": k, "d": d, "r": r_right.ravel().tolist(), "p": p_right},
        "focal_length_px": focal, "baseline_m": baseline_m, "principal_point": (cx, cy),
    }


def cameras(the_rig):
    return {side: rectify.camera(**{key: the_rig[side][key] for key in ("k", "d", "r", "p")})
            for side in ("left", "right")}


def _bilinear(image, x, y):
    h, w = image.shape
    x0, y0 = np.floor(x).astype(np.int64), np.floor(y).astype(np.int64)
    fx, fy = x - x0, y - y0

    def at(yy, xx):
        return image[np.clip(yy, 0, h - 1), np.clip(xx, 0, w - 1)].astype(np.float64)

    top = (1 - fx) * at(y0, x0) + fx * at(y0, x0 + 1)
    bottom = (1 - fx) * at(y0 + 1, x0) + fx * at(y0 + 1, x0 + 1)
    return (1 - fy) * top + fy * bottom


_maps = {}


def _raw_map(side, frame_size):
    """Where each raw pixel of `side` lands in the rectified image (cached)."""
    key = (tuple(side["k"]), tuple(side["d"]), tuple(side["r"]), tuple(side["p"]),
           tuple(frame_size))
    if key in _maps:
        return _maps[key]
    fh, fw = frame_size
    k = np.array(side["k"]).reshape(3, 3)
    k1, k2 = side["d"][0], side["d"][1]
    r = np.array(side["r"]).reshape(3, 3)
    p3 = np.array(side["p"]).reshape(3, 4)[:, :3]
    v, u = np.mgrid[0:fh, 0:fw].astype(np.float64)
    xd, yd = (u - k[0, 2]) / k[0, 0], (v - k[1, 2]) / k[1, 1]
    x, y = xd.copy(), yd.copy()
    for _ in range(8):  # undistort by fixed-point iteration
        r2 = x * x + y * y
        radial = 1 + k1 * r2 + k2 * r2 * r2
        x, y = xd / radial, yd / radial
    ray = np.stack([x, y, np.ones_like(x)], axis=-1) @ r.T
    pix = ray @ p3.T
    _maps[key] = (pix[..., 0] / pix[..., 2], pix[..., 1] / pix[..., 2])
    return _maps[key]


def raw_frame(rectified, side, frame_size):
    """The raw frame whose rectification through `side` is `rectified`."""
    mx, my = _raw_map(side, frame_size)
    return np.clip(np.rint(_bilinear(rectified, mx, my)), 0, 255).astype(np.uint8)


def raw_frames(left, right, the_rig, frame_size=None):
    frame_size = frame_size or left.shape
    return (raw_frame(left, the_rig["left"], frame_size),
            raw_frame(right, the_rig["right"], frame_size))
