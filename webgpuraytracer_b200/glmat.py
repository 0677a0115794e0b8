"""The gl-matrix 3.4.4 operations tracer.js uses, with JavaScript's numeric semantics.

gl-matrix computes in IEEE doubles (JavaScript numbers) and stores every result element into a
Float32Array.  Each function below does the same: arithmetic on Python floats (doubles) read
from float32 inputs, one rounding to float32 per stored element.  Formulas follow the vendored
library (lib/gl-matrix-min.js) function by function.
"""
from __future__ import annotations

import math

import numpy as np

F32 = np.float32


def f32(x) -> np.ndarray:
    return np.asarray(x, dtype=np.float64).astype(np.float32)


def vec3(x=0.0, y=0.0, z=0.0) -> np.ndarray:
    return np.array([x, y, z], dtype=np.float32)


def _d(a) -> list[float]:
    return [float(v) for v in a]


def quat_identity() -> np.ndarray:
    return np.array([0, 0, 0, 1], dtype=np.float32)


def quat_set_axis_angle(axis, rad: float) -> np.ndarray:
    """quat.setAxisAngle"""
    rad = rad * 0.5
    s = math.sin(rad)
    ax = _d(axis)
    return f32([s * ax[0], s * ax[1], s * ax[2], math.cos(rad)])


def vec3_normalize(a) -> np.ndarray:
    """vec3.normalize"""
    x, y, z = _d(a)
    ln = x * x + y * y + z * z
    if ln > 0:
        ln = 1 / math.sqrt(ln)
    return f32([x * ln, y * ln, z * ln])


def vec3_cross(a, b) -> np.ndarray:
    ax, ay, az = _d(a)
    bx, by, bz = _d(b)
    return f32([ay * bz - az * by, az * bx - ax * bz, ax * by - ay * bx])


def vec3_dot(a, b) -> float:
    a = _d(a)
    b = _d(b)
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]


def vec3_length(a) -> float:
    x, y, z = _d(a)
    return math.hypot(x, y, z)


def quat_normalize(q) -> np.ndarray:
    x, y, z, w = _d(q)
    ln = x * x + y * y + z * z + w * w
    if ln > 0:
        ln = 1 / math.sqrt(ln)
    return f32([x * ln, y * ln, z * ln, w * ln])


def quat_rotation_to(a, b) -> np.ndarray:
    """quat.rotationTo: the rotation taking unit vector a onto unit vector b."""
    d = vec3_dot(a, b)
    if d < -0.999999:
        tmp = vec3_cross([1, 0, 0], a)
        if vec3_length(tmp) < 0.000001:
            tmp = vec3_cross([0, 1, 0], a)
        tmp = vec3_normalize(tmp)
        return quat_set_axis_angle(tmp, math.pi)
    if d > 0.999999:
        return quat_identity()
    tmp = vec3_cross(a, b)
    q = f32([float(tmp[0]), float(tmp[1]), float(tmp[2]), 1 + d])
    return quat_normalize(q)


def vec3_transform_quat(a, q) -> np.ndarray:
    """vec3.transformQuat (3.4.4 form: t = 2 cross(q.xyz, v); v + w t + cross(q.xyz, t))."""
    qx, qy, qz, qw = _d(q)
    x, y, z = _d(a)
    h = qy * z - qz * y
    m = qz * x - qx * z
    f = qx * y - qy * x
    h += h
    m += m
    f += f
    return f32([x + qw * h + qy * f - qz * m, y + qw * m + qz * h - qx * f, z + qw * f + qx * m - qy * h])


def mat4_from_rts(q, v, s) -> np.ndarray:
    """mat4.fromRotationTranslationScale (column-major, 16 floats)."""
    x, y, z, w = _d(q)
    x2, y2, z2 = x + x, y + y, z + z
    xx, xy, xz = x * x2, x * y2, x * z2
    yy, yz, zz = y * y2, y * z2, z * z2
    wx, wy, wz = w * x2, w * y2, w * z2
    sx, sy, sz = _d(s)
    v = _d(v)
    return f32([
        (1 - (yy + zz)) * sx, (xy + wz) * sx, (xz - wy) * sx, 0,
        (xy - wz) * sy, (1 - (xx + zz)) * sy, (yz + wx) * sy, 0,
        (xz + wy) * sz, (yz - wx) * sz, (1 - (xx + yy)) * sz, 0,
        v[0], v[1], v[2], 1,
    ])


def mat4_invert(m) -> np.ndarray | None:
    """mat4.invert"""
    a00, a01, a02, a03, a10, a11, a12, a13, a20, a21, a22, a23, a30, a31, a32, a33 = _d(m)
    b00 = a00 * a11 - a01 * a10
    b01 = a00 * a12 - a02 * a10
    b02 = a00 * a13 - a03 * a10
    b03 = a01 * a12 - a02 * a11
    b04 = a01 * a13 - a03 * a11
    b05 = a02 * a13 - a03 * a12
    b06 = a20 * a31 - a21 * a30
    b07 = a20 * a32 - a22 * a30
    b08 = a20 * a33 - a23 * a30
    b09 = a21 * a32 - a22 * a31
    b10 = a21 * a33 - a23 * a31
    b11 = a22 * a33 - a23 * a32
    det = b00 * b11 - b01 * b10 + b02 * b09 + b03 * b08 - b04 * b07 + b05 * b06
    if not det:
        return None
    det = 1.0 / det
    return f32([
        (a11 * b11 - a12 * b10 + a13 * b09) * det,
        (a02 * b10 - a01 * b11 - a03 * b09) * det,
        (a31 * b05 - a32 * b04 + a33 * b03) * det,
        (a22 * b04 - a21 * b05 - a23 * b03) * det,
        (a12 * b08 - a10 * b11 - a13 * b07) * det,
        (a00 * b11 - a02 * b08 + a03 * b07) * det,
        (a32 * b02 - a30 * b05 - a33 * b01) * det,
        (a20 * b05 - a22 * b02 + a23 * b01) * det,
        (a10 * b10 - a11 * b08 + a13 * b06) * det,
        (a01 * b08 - a00 * b10 - a03 * b06) * det,
        (a30 * b04 - a31 * b02 + a33 * b00) * det,
        (a21 * b02 - a20 * b04 - a23 * b00) * det,
        (a11 * b07 - a10 * b09 - a12 * b06) * det,
        (a00 * b09 - a01 * b07 + a02 * b06) * det,
        (a31 * b01 - a30 * b03 - a32 * b00) * det,
        (a20 * b03 - a21 * b01 + a22 * b00) * det,
    ])


def vec3_transform_mat4(a, m) -> np.ndarray:
    """vec3.transformMat4"""
    x, y, z = _d(a)
    m = _d(m)
    w = m[3] * x + m[7] * y + m[11] * z + m[15]
    w = w or 1.0
    return f32([
        (m[0] * x + m[4] * y + m[8] * z + m[12]) / w,
        (m[1] * x + m[5] * y + m[9] * z + m[13]) / w,
        (m[2] * x + m[6] * y + m[10] * z + m[14]) / w,
    ])


def vec3_min(a, b) -> np.ndarray:
    a, b = _d(a), _d(b)
    return f32([min(a[0], b[0]), min(a[1], b[1]), min(a[2], b[2])])


def vec3_max(a, b) -> np.ndarray:
    a, b = _d(a), _d(b)
    return f32([max(a[0], b[0]), max(a[1], b[1]), max(a[2], b[2])])
