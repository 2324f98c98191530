"""Host-side camera models for Stage.Rectification, as NxStereo builds them.

`camera(k, d, r, p)` mirrors NxStereo.Rectify.camera/4
(lib/nx_stereo/rectify.ex:28-50, 209-232): the inverse of the rectified
camera matrix (the left 3x3 of P) times the rectifying rotation R is computed
in f64 with the same cofactor inversion, then every value is cast to f32.
`move_rows` mirrors Stage.Rectification's right_row_offset
(lib/nx_stereo/stage/rectification.ex:84-89), in f32.
`params` flattens a camera to the run request's "<side>.k", "<side>.d" and
"<side>.inverse_pr" inputs (lib/nx_stereo/native_segment.ex:311-322).
"""
import numpy as np


def _multiply_3x3(a, b):
    return [sum(a[i * 3 + n] * b[n * 3 + j] for n in range(3)) for i in range(3) for j in range(3)]


def _invert_3x3(m):
    a, b, c, d, e, f, g, h, i = m
    cofactors = [e * i - f * h, c * h - b * i, b * f - c * e,
                 f * g - d * i, a * i - c * g, c * d - a * f,
                 d * h - e * g, b * g - a * h, a * e - b * d]
    determinant = a * cofactors[0] + b * cofactors[3] + c * cofactors[6]
    return [v / determinant for v in cofactors]


def camera(k, d, r, p):
    """{k, d, inverse_pr} as f32 arrays from row-major lists (k, r: 9; p: 12)."""
    k, r, p = [float(v) for v in k], [float(v) for v in r], [float(v) for v in p]
    if len(k) != 9 or len(r) != 9 or len(p) != 12:
        raise ValueError("camera/4 takes k and r with 9 values and p with 12")
    p3 = [p[i] for i in (0, 1, 2, 4, 5, 6, 8, 9, 10)]
    coefficients = (list(d) + [0.0] * 5)
    if any(v != 0 for v in coefficients[5:]):
        raise ValueError(f"rectify/2 models plumb_bob distortion (5 coefficients), got {list(d)}")
    return {
        "k": np.array(k, np.float32).reshape(3, 3),
        "d": np.array(coefficients[:5], np.float32),
        "inverse_pr": np.array(_invert_3x3(_multiply_3x3(p3, r)), np.float32).reshape(3, 3),
    }


def move_rows(cam, rows):
    """The camera sampling row v + rows: inverse_pr[:, 2] += rows * inverse_pr[:, 1] in f32."""
    inverse = cam["inverse_pr"].astype(np.float32).copy()
    inverse[:, 2] = inverse[:, 2] + np.float32(rows) * inverse[:, 1]
    return dict(cam, inverse_pr=inverse)


def params(side, cam):
    return {f"{side}.k": cam["k"].ravel(), f"{side}.d": cam["d"].ravel(),
            f"{side}.inverse_pr": cam["inverse_pr"].ravel()}
