"""Batched scenes: many independent MPM systems advanced by one launch per stage.

A `Batch` is a `Scene` whose particles come from several scenes that share dx, dt, gravity and
walls but each have their own material.  The library keeps particle positions in scene
coordinates and offsets each scene's block keys into its own slot of the shared key space, so
one activation / binning / P2G / grid update / G2P pass (and one CUDA graph) covers all of
them.  Downloads return the particles of all scenes concatenated; `download_scenes` splits them.

`config4` builds the 256-scene workload: per-scene particle counts log-uniform in
[4,000, 200,000], boxes whose aspect ratio is drawn from extents in [0.1, 0.5] and whose size
is set by the count (8 particles per cell at dx = 1/128), random placement inside the walls and
a random initial velocity, half fixed corotated (E log-uniform in [1e3, 1e5]) and half
Drucker-Prager sand (friction 25-40 degrees).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import Scene, _abi, material_struct, scene_desc
from .scenes import MaterialSpec, Particles, SceneSpec, Shape, generate, uniform01


def _concat(parts: list[Particles]) -> Particles:
    return Particles(*(np.ascontiguousarray(np.concatenate([getattr(p, k) for p in parts]))
                       for k in ("m", "x", "v", "C", "F", "plastic")))


class Batch(Scene):
    """Several scenes in one zsmpm_scene handle (zsmpm_batch_create)."""

    def __init__(self, specs: list[SceneSpec], particles: list[Particles] | None = None, device: int = 0,
                 table_expected: int = 0, max_particles: int = 0):
        first = specs[0]
        for sp in specs[1:]:
            if (sp.dx, sp.dt, tuple(sp.gravity), sp.wall_type, sp.wall_cells) != \
                    (first.dx, first.dt, tuple(first.gravity), first.wall_type, first.wall_cells):
                raise ValueError("batched scenes share dx, dt, gravity and walls")
        self.spec = first
        self.specs = list(specs)
        self._lib = _abi.lib()
        self._h = C.c_void_p()
        desc = scene_desc(first, max_particles=max_particles, device=device, table_expected=table_expected)
        mats = (_abi.Material * len(specs))(*[material_struct(sp.material, sp.volume) for sp in specs])
        _abi.check(self._lib.zsmpm_batch_create(C.byref(desc), mats, len(specs), C.byref(self._h)),
                   "batch_create")
        self.n = 0
        self.counts: list[int] = []
        if particles is not None:
            self.upload(particles)

    def upload(self, parts, stream: int = 0) -> None:  # type: ignore[override]
        """Upload a list of Particles, one per scene."""
        if len(parts) != len(self.specs):
            raise ValueError("one Particles per scene")
        allp = _concat(parts)
        counts = (C.c_int64 * len(parts))(*[p.n for p in parts])
        arrs = _abi.ParticleArrays(**{k: getattr(allp, k).ctypes.data_as(C.c_void_p)
                                      for k in ("m", "x", "v", "C", "F", "plastic")})
        _abi.check(self._lib.zsmpm_batch_upload(self._h, C.byref(arrs), counts, 0, C.c_void_p(stream)),
                   "batch_upload")
        self._keep = allp
        self.n = allp.n
        self.counts = [p.n for p in parts]

    def download_scenes(self, stream: int = 0) -> list[Particles]:
        allp = self.download(stream)
        out, start = [], 0
        for c in self.counts:
            out.append(allp.subset(slice(start, start + c)))
            start += c
        return out

    def num_scenes(self) -> int:
        n = C.c_int32()
        _abi.check(self._lib.zsmpm_batch_num_scenes(self._h, C.byref(n)), "batch_num_scenes")
        return n.value


def config4(n_scenes: int = 256, seed: int = 4, dx: float = 1 / 128, ppc: int = 8,
            n_min: int = 4000, n_max: int = 200000) -> list[SceneSpec]:
    """The batched workload (see the module docstring); a pure function of its arguments."""
    idx = np.arange(n_scenes * 16, dtype=np.uint64)
    u = uniform01(seed, idx).reshape(n_scenes, 16)
    margin = 4 * dx  # walls at 3 dx
    specs = []
    for k in range(n_scenes):
        r = u[k]
        target = math.exp(math.log(n_min) + (math.log(n_max) - math.log(n_min)) * r[0])
        ext = 0.1 + 0.4 * r[1:4]
        vol = target * dx ** 3 / ppc
        ext = ext * (vol / float(np.prod(ext))) ** (1.0 / 3.0)
        ext = np.minimum(ext, 1.0 - 2 * margin - 1e-3)
        lo = margin + (1.0 - 2 * margin - ext) * r[4:7]
        hi = lo + ext
        vel = tuple(float(v) for v in (2.0 * r[7:10] - 1.0))
        if r[10] < 0.5:
            E = math.exp(math.log(1e3) + (math.log(1e5) - math.log(1e3)) * r[11])
            mat = MaterialSpec(model=_abi.FIXED_COROTATED, E=E, nu=0.3, rho=1000.0)
        else:
            mat = MaterialSpec(model=_abi.DRUCKER_PRAGER, E=3.5e5, nu=0.3, rho=2200.0,
                               friction_deg=25.0 + 15.0 * float(r[12]), cohesion=0.0)
        specs.append(SceneSpec(name=f"batch{k}", dx=dx, ppc=ppc,
                               shapes=[Shape("box", tuple(lo), tuple(hi), vel)], material=mat,
                               dt=1e-4, substeps=50, wall_type=_abi.WALL_STICKY, wall_cells=3,
                               seed=seed * 100003 + k))
    return specs


def generate_all(specs: list[SceneSpec]) -> list[Particles]:
    return [generate(sp) for sp in specs]
