"""zsmpm_b200: B200-native explicit MLS/APIC MPM substep (sm_100a CUDA behind a C ABI).

Host-side mirror of the reference's MPM operator surface.  A `Scene` owns one MPM system on
one GPU; its stage methods are the kernels that replace the reference operators launched by
a zs execution policy:

    Scene.activate_blocks()  CleanSparsity + ComputeSparsity + EnlargeSparsity
    Scene.bin_particles()    SpatiallyCount + exclusive_scan + SpatiallyDistribute
    Scene.p2g()              CleanGridBlocks + P2GTransfer
    Scene.grid_update()      ComputeGridBlockVelocity + ApplyBoundaryConditionOnGridBlocks
    Scene.g2p()              G2PTransfer (+ constitutive update)
    Scene.substep()/run(n)   all of the above; run() replays a CUDA graph

Errors surface as `ZsmpmError` carrying the library's zsmpm_status, as the reference
reports launch failures through checkCuKernelLaunchError.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from ._abi import (BLOCK_ORDER_SORTED, DRUCKER_PRAGER, FIXED_COROTATED, PLASTICITY_COMMITTED,
                   PLASTICITY_REFERENCE, SNOW, WALL_NONE, WALL_SEPARATE, WALL_SLIP, WALL_STICKY,
                   ZsmpmError)
from .scenes import MaterialSpec, Particles, SceneSpec, Shape, generate

__all__ = ["Scene", "ZsmpmError", "SceneSpec", "MaterialSpec", "Shape", "Particles", "generate",
           "device_count", "FIXED_COROTATED", "DRUCKER_PRAGER", "SNOW", "PLASTICITY_COMMITTED",
           "PLASTICITY_REFERENCE", "WALL_STICKY", "WALL_SLIP", "WALL_SEPARATE", "WALL_NONE"]


def bht_build_host(keys: np.ndarray, expected: int = 0) -> dict:
    """The bht<i32,3,int,16> layout of keys [n][3] inserted in order (host only)."""
    keys = np.ascontiguousarray(keys, dtype=np.int32).reshape(-1, 3)
    lib = _abi.lib()
    size = C.c_int32()
    hashers = (C.c_uint32 * 6)()
    lib.zsmpm_bht_build_host(_ptr(keys), len(keys), expected, None, None, None, 0, C.byref(size), hashers)
    n = size.value
    tk = np.empty((n, 4), np.int32)
    ti = np.empty(n, np.int32)
    ts = np.empty(n, np.int32)
    _abi.check(lib.zsmpm_bht_build_host(_ptr(keys), len(keys), expected, _ptr(tk), _ptr(ti), _ptr(ts), n,
                                        C.byref(size), hashers), "bht_build_host")
    return {"table_size": n, "hash": np.array(list(hashers), np.uint32), "keys": tk, "indices": ti,
            "status": ts}


def bht_build_device(keys: np.ndarray, expected: int = 0) -> dict:
    """The same layout built on the device (zsmpm_bht_build_device); returns host copies."""
    import torch
    keys = np.ascontiguousarray(keys, dtype=np.int32).reshape(-1, 3)
    lib = _abi.lib()
    size = C.c_int32()
    hashers = (C.c_uint32 * 6)()
    lib.zsmpm_bht_build_host(_ptr(keys), len(keys), expected, None, None, None, 0, C.byref(size), hashers)
    n = size.value
    dk = torch.from_numpy(keys.copy()).cuda() if len(keys) else torch.zeros((1, 3), dtype=torch.int32).cuda()
    tk = torch.empty((max(n, 1), 4), dtype=torch.int32, device="cuda")
    ti = torch.empty(max(n, 1), dtype=torch.int32, device="cuda")
    ts = torch.empty(max(n, 1), dtype=torch.int32, device="cuda")
    _abi.check(lib.zsmpm_bht_build_device(C.c_void_p(dk.data_ptr()), len(keys), expected, C.c_void_p(tk.data_ptr()),
                                          C.c_void_p(ti.data_ptr()), C.c_void_p(ts.data_ptr()), n, C.byref(size),
                                          hashers, None), "bht_build_device")
    return {"table_size": n, "hash": np.array(list(hashers), np.uint32), "keys": tk[:n].cpu().numpy(),
            "indices": ti[:n].cpu().numpy(), "status": ts[:n].cpu().numpy()}


def device_count() -> int:
    return int(_abi.lib().zsmpm_device_count())


def _ptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.c_void_p)


def material_struct(spec: MaterialSpec, volume: float) -> _abi.Material:
    return _abi.Material(model=spec.model, plasticity_mode=spec.plasticity_mode, E=spec.E,
                         nu=spec.nu, rho=spec.rho, volume=volume, friction_deg=spec.friction_deg,
                         cohesion=spec.cohesion, beta=spec.beta,
                         volume_correction=spec.volume_correction, hardening=spec.hardening,
                         theta_c=spec.theta_c, theta_s=spec.theta_s)


def scene_desc(spec: SceneSpec, max_particles: int = 0, device: int = 0,
               table_expected: int = 0) -> _abi.SceneDesc:
    d = _abi.SceneDesc()
    d.dx = spec.dx
    d.dt = spec.dt
    for k in range(3):
        d.gravity[k] = spec.gravity[k]
    d.wall_type = spec.wall_type
    d.wall_cells = spec.wall_cells
    d.material = material_struct(spec.material, spec.volume)
    d.max_particles = max_particles
    d.table_expected = table_expected
    d.block_order = BLOCK_ORDER_SORTED
    d.device = device
    d.threads_per_cta = 0
    return d


class Scene:
    """One MPM system on one GPU (wraps a zsmpm_scene handle)."""

    def __init__(self, spec: SceneSpec, particles: Particles | None = None, device: int = 0,
                 table_expected: int = 0, max_particles: int = 0, transfer: str = "apic"):
        self.spec = spec
        self.device = device
        self._lib = _abi.lib()
        self._h = C.c_void_p()
        desc = scene_desc(spec, max_particles=max_particles, device=device,
                          table_expected=table_expected)
        _abi.check(self._lib.zsmpm_scene_create(C.byref(desc), C.byref(self._h)), "scene_create")
        self.n = 0
        if transfer != "apic":
            self.set_transfer(transfer)
        if particles is not None:
            self.upload(particles)

    # ---- lifetime
    def close(self) -> None:
        if self._h:
            self._lib.zsmpm_scene_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    # ---- particles
    def upload(self, p: Particles, stream: int = 0) -> None:
        arrs = _abi.ParticleArrays(m=_ptr(p.m), x=_ptr(p.x), v=_ptr(p.v), C=_ptr(p.C),
                                   F=_ptr(p.F), plastic=_ptr(p.plastic))
        _abi.check(self._lib.zsmpm_scene_upload(self._h, C.byref(arrs), p.n, 0, C.c_void_p(stream)),
                   "scene_upload")
        self.n = p.n

    def upload_device(self, ptrs: dict, n: int, stream: int = 0) -> None:
        """Upload from device pointers (ints), e.g. torch tensors' data_ptr()."""
        arrs = _abi.ParticleArrays(**{k: C.c_void_p(ptrs.get(k) or 0) or None for k in
                                      ("m", "x", "v", "C", "F", "plastic")})
        _abi.check(self._lib.zsmpm_scene_upload(self._h, C.byref(arrs), n, 1, C.c_void_p(stream)),
                   "scene_upload")
        self.n = n

    def download(self, stream: int = 0) -> Particles:
        n = self.n
        out = Particles(m=np.empty(n, np.float32), x=np.empty((n, 3), np.float32),
                        v=np.empty((n, 3), np.float32), C=np.empty((n, 9), np.float32),
                        F=np.empty((n, 9), np.float32), plastic=np.empty(n, np.float32))
        arrs = _abi.ParticleArrays(m=_ptr(out.m), x=_ptr(out.x), v=_ptr(out.v), C=_ptr(out.C),
                                   F=_ptr(out.F), plastic=_ptr(out.plastic))
        _abi.check(self._lib.zsmpm_scene_download(self._h, C.byref(arrs), 0, C.c_void_p(stream)),
                   "scene_download")
        return out

    def download_device(self, ptrs: dict, stream: int = 0) -> None:
        arrs = _abi.ParticleArrays(**{k: C.c_void_p(ptrs.get(k) or 0) or None for k in
                                      ("m", "x", "v", "C", "F", "plastic")})
        _abi.check(self._lib.zsmpm_scene_download(self._h, C.byref(arrs), 1, C.c_void_p(stream)),
                   "scene_download")

    # ---- colliders
    def set_colliders(self, colliders, stream: int = 0) -> None:
        """Analytic colliders (zsmpm_b200.colliders) applied after the walls, in list order."""
        from . import colliders as col
        arr = col.array(list(colliders))
        _abi.check(self._lib.zsmpm_scene_set_colliders(self._h, arr, len(colliders), C.c_void_p(stream)),
                   "scene_set_colliders")

    def add_levelset(self, levelset, stream: int = 0) -> None:
        """A sparse level-set boundary (zsmpm_b200.colliders.LevelSet), applied after the colliders."""
        d = levelset.desc()
        _abi.check(self._lib.zsmpm_scene_add_levelset(self._h, C.byref(d), C.c_void_p(stream)),
                   "scene_add_levelset")

    def clear_levelsets(self) -> None:
        _abi.check(self._lib.zsmpm_scene_clear_levelsets(self._h), "scene_clear_levelsets")

    # ---- stages
    def activate_blocks(self, stream: int = 0):
        _abi.check(self._lib.zsmpm_activate_blocks(self._h, C.c_void_p(stream)), "activate_blocks")

    def bin_particles(self, stream: int = 0):
        _abi.check(self._lib.zsmpm_bin_particles(self._h, C.c_void_p(stream)), "bin_particles")

    def p2g(self, stream: int = 0):
        _abi.check(self._lib.zsmpm_p2g(self._h, C.c_void_p(stream)), "p2g")

    def grid_update(self, stream: int = 0):
        _abi.check(self._lib.zsmpm_grid_update(self._h, C.c_void_p(stream)), "grid_update")

    def g2p(self, stream: int = 0):
        _abi.check(self._lib.zsmpm_g2p(self._h, C.c_void_p(stream)), "g2p")

    TRANSFERS = {"apic": 0, "cell": 1}
    P2C2G_PARTS = {"all": 0, "momentum": 1, "force": 2}

    def set_transfer(self, transfer: str, stream: int = 0):
        """"apic" (P2GTransfer / G2PTransfer) or "cell" (P2C2GTransfer / G2C2PTransfer, fixed
        corotated; the C attribute then holds the pair's B matrix), see zsmpm_scene_set_transfer."""
        _abi.check(self._lib.zsmpm_scene_set_transfer(self._h, self.TRANSFERS[transfer], C.c_void_p(stream)),
                   "scene_set_transfer")

    def p2c2g(self, part: str = "all", stream: int = 0):
        _abi.check(self._lib.zsmpm_p2c2g(self._h, self.P2C2G_PARTS[part], C.c_void_p(stream)), "p2c2g")

    def g2c2p(self, stream: int = 0):
        _abi.check(self._lib.zsmpm_g2c2p(self._h, C.c_void_p(stream)), "g2c2p")

    def substep(self, stream: int = 0):
        _abi.check(self._lib.zsmpm_substep(self._h, C.c_void_p(stream)), "substep")

    def run(self, nsteps: int, stream: int = 0):
        """nsteps substeps from the scene's CUDA graph of four; run(0) only captures that graph
        for the current buffer parity (to keep the capture out of a timed region)."""
        _abi.check(self._lib.zsmpm_run(self._h, nsteps, C.c_void_p(stream)), "run")

    def status(self) -> None:
        _abi.check(self._lib.zsmpm_scene_status(self._h), "device status")

    # ---- views
    def num_blocks(self) -> int:
        nb = C.c_int32()
        _abi.check(self._lib.zsmpm_num_blocks(self._h, C.byref(nb)), "num_blocks")
        return nb.value

    def binning_info(self) -> int:
        """-1 when the last binning counted every particle, else the number of particles that
        the incremental binning moved into other cells (see zsmpm_binning_info)."""
        m = C.c_int32()
        _abi.check(self._lib.zsmpm_binning_info(self._h, C.byref(m)), "binning_info")
        return m.value

    def download_grid(self):
        nb = self.num_blocks()
        keys = np.empty((max(nb, 1), 3), np.int32)
        grid = np.empty((max(nb, 1), 4, 512), np.float32)
        out_nb = C.c_int32()
        _abi.check(self._lib.zsmpm_download_grid(self._h, _ptr(keys), _ptr(grid), nb, C.byref(out_nb)),
                   "download_grid")
        return keys[:nb], grid[:nb]

    def download_binning(self):
        nb = self.num_blocks()
        order = np.empty(self.n, np.int32)
        bstart = np.empty(nb + 1, np.int32)
        _abi.check(self._lib.zsmpm_download_binning(self._h, _ptr(order), _ptr(bstart), nb),
                   "download_binning")
        return order, bstart

    def bht_view(self) -> _abi.BhtView:
        """The active blocks as the reference's bht<i32,3,int,16> (device pointers)."""
        v = _abi.BhtView()
        _abi.check(self._lib.zsmpm_get_bht_view(self._h, C.byref(v)), "bht_view")
        return v

    def table_view(self) -> _abi.TableView:
        tv = _abi.TableView()
        _abi.check(self._lib.zsmpm_get_table_view(self._h, C.byref(tv)), "table_view")
        return tv

    def grid_view(self) -> _abi.GridView:
        gv = _abi.GridView()
        _abi.check(self._lib.zsmpm_get_grid_view(self._h, C.byref(gv)), "grid_view")
        return gv

    def set_stage_timing(self, on: bool) -> None:
        _abi.check(self._lib.zsmpm_set_stage_timing(self._h, int(on)), "stage_timing")

    def stage_times(self) -> list[float]:
        ms = (C.c_float * 5)()
        _abi.check(self._lib.zsmpm_stage_times(self._h, ms, 5), "stage_times")
        return list(ms)

    def kernels_per_substep(self) -> int:
        return int(self._lib.zsmpm_kernels_per_substep(self._h))

    # ---- launch shapes
    def autotune(self, trials: int = 2, stream: int = 0) -> dict:
        """Times G2P and P2G launch shapes on the uploaded particles (advancing the simulation by
        the substeps it times) and keeps the fastest; returns the choice."""
        t = _abi.Tuning()
        _abi.check(self._lib.zsmpm_autotune(self._h, trials, C.byref(t), C.c_void_p(stream)), "autotune")
        return {"g2p_threads": t.g2p_threads, "g2p_ctas_per_sm": t.g2p_ctas_per_sm,
                "p2g_ctas_per_sm": t.p2g_ctas_per_sm, "p2g_ranks": t.p2g_ranks, "g2p_ms": t.g2p_ms,
                "p2g_ms": t.p2g_ms}

    def set_tuning(self, g2p_threads: int = 0, g2p_ctas_per_sm: int = 0, p2g_ctas_per_sm: int = 0,
                   p2g_ranks: int = 0) -> None:
        t = _abi.Tuning(g2p_threads=g2p_threads, g2p_ctas_per_sm=g2p_ctas_per_sm, p2g_ctas_per_sm=p2g_ctas_per_sm,
                        p2g_ranks=p2g_ranks)
        _abi.check(self._lib.zsmpm_set_tuning(self._h, C.byref(t)), "set_tuning")
