"""Seeded synthetic MPM scenes: jittered sub-lattice particles in boxes and spheres.

Every particle sits at a sub-lattice point of its cell plus a uniform jitter of +-0.25 dx
per axis drawn from a counter-based generator (splitmix64 of seed and particle index),
so a scene is a pure function of its description.  8 particles per cell use the 2x2x2
points (0.25|0.75)^3, 4 use the tetrahedral points (0.25,0.25,0.25), (0.75,0.75,0.25),
(0.75,0.25,0.75), (0.25,0.75,0.75), 1 uses the cell centre.  Mass m = rho * dx^3 / ppc,
F = I, C = 0, plastic state 0 (logJp) or 1 (Jp).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import _abi

M64 = np.uint64(0xFFFFFFFFFFFFFFFF)

SUBPOINTS = {
    1: np.array([[0.5, 0.5, 0.5]]),
    4: np.array([[0.25, 0.25, 0.25], [0.75, 0.75, 0.25], [0.75, 0.25, 0.75], [0.25, 0.75, 0.75]]),
    8: np.array([[a, b, c] for a in (0.25, 0.75) for b in (0.25, 0.75) for c in (0.25, 0.75)]),
}


def splitmix64(x: np.ndarray) -> np.ndarray:
    with np.errstate(over="ignore"):
        z = (x + np.uint64(0x9E3779B97F4A7C15)) & M64
        z = ((z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & M64
        z = ((z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & M64
        return z ^ (z >> np.uint64(31))


def uniform01(seed: int, index: np.ndarray) -> np.ndarray:
    """u in [0, 1) with 24 random bits, from (seed, index)."""
    with np.errstate(over="ignore"):
        h = splitmix64(index.astype(np.uint64) * np.uint64(0x9E3779B97F4A7C15) ^ np.uint64(seed))
    return (h >> np.uint64(40)).astype(np.float64) * (1.0 / (1 << 24))


@dataclass
class Shape:
    kind: str                      # "box" or "sphere"
    lo: tuple = (0.0, 0.0, 0.0)    # box corner / sphere centre
    hi: tuple = (0.0, 0.0, 0.0)    # box corner / (radius, -, -)
    velocity: tuple = (0.0, 0.0, 0.0)


@dataclass
class MaterialSpec:
    model: int = _abi.FIXED_COROTATED
    E: float = 1e4
    nu: float = 0.3
    rho: float = 1000.0
    friction_deg: float = 30.0
    cohesion: float = 0.0
    beta: float = 1.0
    volume_correction: int = 1
    hardening: float = 10.0
    theta_c: float = 2.5e-2
    theta_s: float = 7.5e-3
    plasticity_mode: int = _abi.PLASTICITY_COMMITTED


@dataclass
class SceneSpec:
    name: str
    dx: float
    ppc: int
    shapes: list
    material: MaterialSpec
    dt: float
    substeps: int
    gravity: tuple = (0.0, -9.8, 0.0)
    wall_type: int = _abi.WALL_STICKY
    wall_cells: int = 3
    seed: int = 1234

    @property
    def volume(self) -> float:
        return self.dx ** 3 / self.ppc


@dataclass
class Particles:
    """Particle arrays in the reference's zs::Particles<f32,3> layout."""
    m: np.ndarray
    x: np.ndarray
    v: np.ndarray
    C: np.ndarray
    F: np.ndarray
    plastic: np.ndarray

    @property
    def n(self) -> int:
        return len(self.m)

    def copy(self) -> "Particles":
        return Particles(*(a.copy() for a in (self.m, self.x, self.v, self.C, self.F, self.plastic)))

    def subset(self, idx) -> "Particles":
        return Particles(*(a[idx].copy() for a in (self.m, self.x, self.v, self.C, self.F, self.plastic)))


def _shape_points(shape: Shape, dx: float, ppc: int) -> np.ndarray:
    """Unjittered sub-lattice points inside the shape, as (cell, subpoint) float64 coords in
    cell units, cell-major (x slowest, z fastest) with subpoints fastest."""
    sub = SUBPOINTS[ppc]
    if shape.kind == "box":
        lo = np.array(shape.lo) / dx
        hi = np.array(shape.hi) / dx
    elif shape.kind == "sphere":
        c = np.array(shape.lo) / dx
        r = shape.hi[0] / dx
        lo, hi = c - r, c + r
    else:
        raise ValueError(shape.kind)
    i0 = np.floor(lo).astype(np.int64) - 1
    i1 = np.ceil(hi).astype(np.int64) + 1
    axes = [np.arange(i0[d], i1[d], dtype=np.int64) for d in range(3)]
    cells = np.stack(np.meshgrid(*axes, indexing="ij"), -1).reshape(-1, 1, 3)
    pts = (cells + sub[None]).reshape(-1, 3)
    if shape.kind == "box":
        keep = np.all((pts >= lo - 1e-9) & (pts < hi - 1e-9), axis=1)
    else:
        keep = np.sum((pts - c) ** 2, axis=1) < r * r
    return pts[keep]


def generate(spec: SceneSpec) -> Particles:
    xs, vs = [], []
    for s in spec.shapes:
        p = _shape_points(s, spec.dx, spec.ppc)
        xs.append(p)
        vs.append(np.broadcast_to(np.array(s.velocity, np.float64), p.shape))
    pts = np.concatenate(xs) if xs else np.zeros((0, 3))
    vel = np.concatenate(vs) if vs else np.zeros((0, 3))
    n = len(pts)
    idx = np.arange(n, dtype=np.uint64)
    jit = np.stack([uniform01(spec.seed, idx * np.uint64(3) + np.uint64(a)) for a in range(3)], 1)
    x = ((pts + (jit - 0.5) * 0.5) * spec.dx).astype(np.float32)
    m = np.full(n, spec.material.rho * spec.volume, np.float32)
    F = np.tile(np.eye(3, dtype=np.float32).reshape(1, 9), (n, 1))
    C = np.zeros((n, 9), np.float32)
    pl = np.full(n, 1.0 if spec.material.model == _abi.SNOW else 0.0, np.float32)
    return Particles(m=m, x=np.ascontiguousarray(x), v=vel.astype(np.float32).copy(), C=C, F=F,
                     plastic=pl)


def count_particles(spec: SceneSpec) -> int:
    return sum(len(_shape_points(s, spec.dx, spec.ppc)) for s in spec.shapes)


# ------------------------------------------------------------------ the benchmark scenes
def config1(scale: float = 1.0) -> SceneSpec:
    """Fixed-corotated cube [0.4,0.6]^3, dx=1/128, 8 ppc, sticky walls, 100 substeps."""
    return SceneSpec(
        name="fc_cube_dx128", dx=1 / 128 / scale, ppc=8,
        shapes=[Shape("box", (0.4, 0.4, 0.4), (0.6, 0.6, 0.6))],
        material=MaterialSpec(model=_abi.FIXED_COROTATED, E=1e4, nu=0.3, rho=1000.0),
        dt=1e-4, substeps=100, wall_type=_abi.WALL_STICKY, wall_cells=3)


def config2(dx: float = 1 / 256) -> SceneSpec:
    """Drucker-Prager sand, two boxes, the second moving at (-1,0,0) m/s, slip walls."""
    return SceneSpec(
        name="dp_two_boxes_dx256", dx=dx, ppc=8,
        shapes=[Shape("box", (0.1, 0.1, 0.1), (0.45, 0.6, 0.9)),
                Shape("box", (0.55, 0.1, 0.1), (0.9, 0.4, 0.9), velocity=(-1.0, 0.0, 0.0))],
        material=MaterialSpec(model=_abi.DRUCKER_PRAGER, E=3.5e5, nu=0.3, rho=2200.0,
                              friction_deg=30.0, cohesion=0.0),
        dt=5e-5, substeps=200, wall_type=_abi.WALL_SLIP, wall_cells=3)


def config5(dx: float = 1 / 512) -> SceneSpec:
    """Snow sphere (r=0.2, v=(0,-3,0)) above a slab, fixed corotated + Stomakhin snow."""
    return SceneSpec(
        name="snow_sphere_slab", dx=dx, ppc=4,
        shapes=[Shape("box", (0.05, 0.05, 0.05), (0.95, 0.2, 0.95)),
                Shape("sphere", (0.5, 0.45, 0.5), (0.2, 0.0, 0.0), velocity=(0.0, -3.0, 0.0))],
        material=MaterialSpec(model=_abi.SNOW, E=1.4e5, nu=0.2, rho=400.0, hardening=10.0,
                              theta_c=2.5e-2, theta_s=7.5e-3),
        dt=2e-5, substeps=100, wall_type=_abi.WALL_STICKY, wall_cells=3)


def config5_16m() -> SceneSpec:
    """The snow scene with dx chosen so that it holds about 16.0 M particles."""
    return config5(dx=1 / 295)


def small_scene(model: int = _abi.FIXED_COROTATED, n_side: float = 0.06, dx: float = 1 / 128,
                velocity=(0.3, -0.2, 0.1), mode: int = _abi.PLASTICITY_COMMITTED,
                wall_type: int = _abi.WALL_STICKY, center=(0.5, 0.5, 0.5), ppc: int = 8,
                seed: int = 7) -> SceneSpec:
    """A small box for parity tests (a few thousand particles)."""
    lo = tuple(c - n_side / 2 for c in center)
    hi = tuple(c + n_side / 2 for c in center)
    mat = MaterialSpec(model=model, plasticity_mode=mode)
    if model == _abi.DRUCKER_PRAGER:
        mat.E, mat.nu, mat.rho = 3.5e5, 0.3, 2200.0
    elif model == _abi.SNOW:
        mat.E, mat.nu, mat.rho = 1.4e5, 0.2, 400.0
    return SceneSpec(name="small", dx=dx, ppc=ppc, shapes=[Shape("box", lo, hi, velocity)],
                     material=mat, dt=1e-4, substeps=10, wall_type=wall_type, seed=seed)
