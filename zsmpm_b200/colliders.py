"""Analytic colliders: Collider<AnalyticLevelSet<shape, f32, 3>> (geometry/Collider.h,
geometry/AnalyticLevelSet.h), placed by scale s, rotation R (row-major) and translation t, with
their rates dsdt, omega and dt/dt.  Build them with plane / cuboid / sphere / cylinder and hand a
list to Scene.set_colliders; the grid update applies them after the scene's walls, in order.
"""
from __future__ import annotations

import numpy as np

from . import _abi

TYPES = {"sticky": _abi.WALL_STICKY, "slip": _abi.WALL_SLIP, "separate": _abi.WALL_SEPARATE}


def _make(shape, a, b, kind, axis=0, s=1.0, dsdt=0.0, R=None, omega=(0, 0, 0), t=(0, 0, 0),
          dtdt=(0, 0, 0)) -> _abi.Collider:
    c = _abi.Collider()
    c.shape = shape
    c.type = TYPES[kind] if isinstance(kind, str) else int(kind)
    c.axis = axis
    c.a[:] = [float(v) for v in a]
    c.b[:] = [float(v) for v in b]
    c.s = s
    c.dsdt = dsdt
    c.R[:] = [float(v) for v in np.asarray(np.eye(3) if R is None else R, np.float64).reshape(9)]
    c.omega[:] = [float(v) for v in omega]
    c.t[:] = [float(v) for v in t]
    c.dtdt[:] = [float(v) for v in dtdt]
    return c


def plane(origin, normal, kind="sticky", **motion) -> _abi.Collider:
    """AnalyticLevelSet<Plane>: signed distance normal . (X - origin); the normal is used as given."""
    return _make(_abi.SHAPE_PLANE, origin, normal, kind, **motion)


def cuboid(lo, hi, kind="sticky", **motion) -> _abi.Collider:
    return _make(_abi.SHAPE_CUBOID, lo, hi, kind, **motion)


def sphere(center, radius, kind="sticky", **motion) -> _abi.Collider:
    return _make(_abi.SHAPE_SPHERE, center, (radius, 0.0, 0.0), kind, **motion)


def cylinder(bottom, radius, length, axis, kind="sticky", **motion) -> _abi.Collider:
    return _make(_abi.SHAPE_CYLINDER, bottom, (radius, length, 0.0), kind, axis=axis, **motion)


def rotation(axis, angle) -> np.ndarray:
    """Row-major rotation matrix about a unit axis (Rodrigues)."""
    k = np.asarray(axis, np.float64)
    k = k / np.linalg.norm(k)
    K = np.array([[0, -k[2], k[1]], [k[2], 0, -k[0]], [-k[1], k[0], 0]])
    return np.eye(3) + np.sin(angle) * K + (1 - np.cos(angle)) * (K @ K)


def array(colliders) -> "_abi.Collider * n":
    arr = (_abi.Collider * max(len(colliders), 1))()
    for i, c in enumerate(colliders):
        arr[i] = c
    return arr
