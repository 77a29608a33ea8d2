"""Boundaries of the grid update.

Analytic colliders: Collider<AnalyticLevelSet<shape, f32, 3>> (geometry/Collider.h,
geometry/AnalyticLevelSet.h), placed by scale s, rotation R (row-major) and translation t, with
their rates dsdt, omega and dt/dt.  Build them with plane / cuboid / sphere / cylinder and hand a
list to Scene.set_colliders; the grid update applies them after the scene's walls, in order.

Sparse level sets: LevelSetBoundary<SparseLevelSet<3>> (geometry/SparseLevelSet.hpp), a signed
distance on 8^3 blocks sampled trilinearly; build one with LevelSet.from_function and add it with
Scene.add_levelset (applied after the colliders).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

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


@dataclass
class LevelSet:
    """A SparseLevelSet<3> boundary: block origins (multiples of 8) in index space, 512 distances
    per block (cell x*64 + y*8 + z), the background value outside the blocks, and the
    world-to-index transform X = ((x - t) rinv) sinv (row vectors, row-major 3x3)."""
    keys: np.ndarray
    sdf: np.ndarray
    kind: str = "sticky"
    background: float = 1.0
    sinv: np.ndarray = field(default_factory=lambda: np.eye(3, dtype=np.float32))
    rinv: np.ndarray = field(default_factory=lambda: np.eye(3, dtype=np.float32))
    t: np.ndarray = field(default_factory=lambda: np.zeros(3, np.float32))

    @classmethod
    def from_function(cls, phi, lo, hi, h: float, kind: str = "sticky", rinv=None, t=(0.0, 0.0, 0.0),
                      background: float = 1.0) -> "LevelSet":
        """Samples phi (world positions [n, 3] -> distances) on every block whose index-space
        box meets the world box [lo, hi], voxel size h, rotation rinv (world->index, applied
        before the scale) and translation t."""
        rinv = np.eye(3) if rinv is None else np.asarray(rinv, np.float64)
        t = np.asarray(t, np.float64)
        corners = np.array([[a, b, c] for a in (lo[0], hi[0]) for b in (lo[1], hi[1]) for c in (lo[2], hi[2])],
                           np.float64)
        X = ((corners - t) @ rinv) / h
        blo = (np.floor(X.min(0)).astype(np.int64) // 8) - 1
        bhi = (np.floor(X.max(0)).astype(np.int64) // 8) + 1
        axes = [np.arange(blo[d], bhi[d] + 1) for d in range(3)]
        keys = np.stack(np.meshgrid(*axes, indexing="ij"), -1).reshape(-1, 3) * 8
        cell = np.arange(512)
        loc = np.stack([cell >> 6, (cell >> 3) & 7, cell & 7], 1)
        nodes = (keys[:, None, :] + loc[None]).reshape(-1, 3).astype(np.float64)
        world = (nodes * h) @ rinv.T + t
        sdf = np.asarray(phi(world), np.float64).reshape(len(keys), 512)
        return cls(keys=keys.astype(np.int32), sdf=sdf.astype(np.float32), kind=kind, background=background,
                   sinv=(np.eye(3) / h).astype(np.float32), rinv=rinv.astype(np.float32),
                   t=t.astype(np.float32))

    def desc(self) -> _abi.LevelSetDesc:
        """The zsmpm_levelset_desc; the arrays stay owned by this object."""
        self._keys = np.ascontiguousarray(self.keys, np.int32)
        self._sdf = np.ascontiguousarray(self.sdf, np.float32)
        d = _abi.LevelSetDesc()
        d.nblocks = len(self._keys)
        d.type = TYPES[self.kind] if isinstance(self.kind, str) else int(self.kind)
        d.keys = self._keys.ctypes.data_as(C.c_void_p)
        d.sdf = self._sdf.ctypes.data_as(C.c_void_p)
        d.background = float(self.background)
        d.sinv[:] = [float(v) for v in np.asarray(self.sinv, np.float32).reshape(9)]
        d.rinv[:] = [float(v) for v in np.asarray(self.rinv, np.float32).reshape(9)]
        d.t[:] = [float(v) for v in np.asarray(self.t, np.float32).reshape(3)]
        return d
