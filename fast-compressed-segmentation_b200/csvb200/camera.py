"""Camera and orbit helpers for the ray marcher (host side, double precision as the reference's JS).

Restates web/scripts/camera.js:61-77 (getUniformData: forward/right/up basis
with the world-up switch near the poles, tan(fov/2)) and
web/scripts/orbitController.js:100-123 (yaw/pitch/radius orbit about a
target).  Results are packed into the 16-float layout csv_camera uses.
"""
from __future__ import annotations

import math

import numpy as np

SLOT_DTYPE = np.dtype([("offset", "<u8"), ("lod", "<u4"), ("flags", "<u4")])  # csv_brick_slot
SLOT_EMPTY = 0x1
SLOT_MISSING = 0x2


def _norm(v):
    n = math.hypot(v[0], v[1], v[2]) or 1.0
    return (v[0] / n, v[1] / n, v[2] / n)


def _cross(a, b):
    return (a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0])


def camera_uniform(position, direction, fov: float) -> np.ndarray:
    """camera.js:61-77 -> float32[16]: position, tanHalfFov, forward, 0, right, 0, up, 0."""
    f = _norm(direction)
    world_up = (1.0, 0.0, 0.0) if abs(f[1]) > 0.999 else (0.0, 1.0, 0.0)
    r = _norm(_cross(f, world_up))
    u = _norm(_cross(r, f))
    return np.array([*position, math.tan(fov * 0.5), *f, 0.0, *r, 0.0, *u, 0.0], dtype=np.float32)


def orbit(target, radius: float, yaw: float, pitch: float):
    """orbitController.js:100-123: camera position on the orbit and its view direction (towards the target)."""
    cp, sp, cy, sy = math.cos(pitch), math.sin(pitch), math.cos(yaw), math.sin(yaw)
    pos = (target[0] + radius * cp * sy, target[1] + radius * sp, target[2] + radius * cp * cy)
    d = _norm((target[0] - pos[0], target[1] - pos[1], target[2] - pos[2]))
    return pos, d


def focal_length(screen_px: float, fov: float) -> float:
    """camera.js:115: (screenWidth / 2) / tan(fov / 2); the viewer passes min(width, height) (renderLoop.js:374)."""
    return (screen_px / 2.0) / math.tan(fov / 2.0)


def camera_struct(cam16: np.ndarray):
    """ctypes csv_camera from the 16-float layout."""
    import ctypes as C

    class CsvCamera(C.Structure):
        _fields_ = [("v", C.c_float * 16)]

    c = CsvCamera()
    for i in range(16):
        c.v[i] = float(cam16[i])
    return c
