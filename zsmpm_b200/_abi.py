"""ctypes mirror of include/zsmpm.h (the C ABI of libzsmpm.so).

The library is loaded from zsmpm_b200/lib/libzsmpm.so, built in-tree by zsmpm_b200/build.py.
There is no fallback: if the library is missing, importing the bindings raises.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libzsmpm.so"

# zsmpm_status
OK, ERR_TABLE_FULL, ERR_CAPACITY, ERR_INVALID_ARG, ERR_CUDA, ERR_TIMEOUT, ERR_OUT_OF_DOMAIN, \
    ERR_NO_DEVICE, ERR_NOT_READY = range(9)
STATUS_NAMES = {OK: "OK", ERR_TABLE_FULL: "TABLE_FULL", ERR_CAPACITY: "CAPACITY",
                ERR_INVALID_ARG: "INVALID_ARG", ERR_CUDA: "CUDA", ERR_TIMEOUT: "TIMEOUT",
                ERR_OUT_OF_DOMAIN: "OUT_OF_DOMAIN", ERR_NO_DEVICE: "NO_DEVICE",
                ERR_NOT_READY: "NOT_READY"}

FIXED_COROTATED, DRUCKER_PRAGER, SNOW = 0, 1, 2
PLASTICITY_COMMITTED, PLASTICITY_REFERENCE = 0, 1
WALL_STICKY, WALL_SLIP, WALL_SEPARATE, WALL_NONE = 0, 1, 2, 3
BLOCK_ORDER_SORTED, BLOCK_ORDER_INSERTION = 0, 1


class Material(C.Structure):
    _fields_ = [("model", C.c_int32), ("plasticity_mode", C.c_int32),
                ("E", C.c_float), ("nu", C.c_float), ("rho", C.c_float), ("volume", C.c_float),
                ("friction_deg", C.c_float), ("cohesion", C.c_float), ("beta", C.c_float),
                ("volume_correction", C.c_int32),
                ("hardening", C.c_float), ("theta_c", C.c_float), ("theta_s", C.c_float)]


class SceneDesc(C.Structure):
    _fields_ = [("dx", C.c_float), ("dt", C.c_float), ("gravity", C.c_float * 3),
                ("wall_type", C.c_int32), ("wall_cells", C.c_int32), ("material", Material),
                ("max_particles", C.c_int64), ("table_expected", C.c_int32),
                ("block_order", C.c_int32), ("device", C.c_int32), ("threads_per_cta", C.c_int32)]


class ParticleArrays(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("m", "x", "v", "C", "F", "plastic")]


class TileVectorView(C.Structure):
    _fields_ = [("base", C.c_void_p), ("num_channels", C.c_int32), ("lane_width", C.c_int32),
                ("off_m", C.c_int32), ("off_x", C.c_int32), ("off_v", C.c_int32),
                ("off_C", C.c_int32), ("off_F", C.c_int32), ("off_plastic", C.c_int32)]


class TableView(C.Structure):
    _fields_ = [("keys", C.c_void_p), ("indices", C.c_void_p), ("status", C.c_void_p),
                ("active_keys", C.c_void_p), ("cnt", C.c_void_p), ("table_size", C.c_int32)]


class GridView(C.Structure):
    _fields_ = [("base", C.c_void_p), ("num_channels", C.c_int32), ("num_blocks", C.c_int32),
                ("keys", C.c_void_p)]


class BhtView(C.Structure):
    _fields_ = [("keys", C.c_void_p), ("indices", C.c_void_p), ("status", C.c_void_p),
                ("active_keys", C.c_void_p), ("cnt", C.c_void_p), ("success", C.c_void_p),
                ("table_size", C.c_int32), ("hashers", C.c_uint32 * 6)]


class Tuning(C.Structure):
    _fields_ = [("g2p_threads", C.c_int32), ("g2p_ctas_per_sm", C.c_int32), ("p2g_ctas_per_sm", C.c_int32),
                ("g2p_ms", C.c_float), ("p2g_ms", C.c_float), ("p2g_ranks", C.c_int32)]


MLP_PARAMS = 9158  # 6 -> 64 -> 64 -> 64 -> 6


class ClosureState(C.Structure):
    _fields_ = [("model", C.c_int32), ("params", C.c_float * MLP_PARAMS),
                ("in_mean", C.c_float * 6), ("in_inv_std", C.c_float * 6),
                ("in_min", C.c_float * 6), ("in_max", C.c_float * 6), ("out_scale", C.c_float * 6)]


class ClosureAudit(C.Structure):
    _fields_ = [("audited", C.c_int64), ("mean_rel_error", C.c_double),
                ("max_rel_error", C.c_double), ("agg_rel_error", C.c_double),
                ("fallbacks", C.c_int64), ("network_updates", C.c_int64), ("updates", C.c_int64)]


class Collider(C.Structure):
    """zsmpm_collider: Collider<AnalyticLevelSet<shape, f32, 3>> (geometry/Collider.h)."""
    _fields_ = [("shape", C.c_int32), ("type", C.c_int32), ("axis", C.c_int32), ("reserved", C.c_int32),
                ("a", C.c_float * 3), ("b", C.c_float * 3), ("s", C.c_float), ("dsdt", C.c_float),
                ("R", C.c_float * 9), ("omega", C.c_float * 3), ("t", C.c_float * 3), ("dtdt", C.c_float * 3)]


class LevelSetDesc(C.Structure):
    """zsmpm_levelset_desc: LevelSetBoundary<SparseLevelSet<3>> data (host pointers)."""
    _fields_ = [("nblocks", C.c_int32), ("type", C.c_int32), ("keys", C.c_void_p), ("sdf", C.c_void_p),
                ("background", C.c_float), ("sinv", C.c_float * 9), ("rinv", C.c_float * 9), ("t", C.c_float * 3)]


SHAPE_PLANE, SHAPE_CUBOID, SHAPE_SPHERE, SHAPE_CYLINDER = 0, 1, 2, 3
MAX_COLLIDERS = 16


class CgOptions(C.Structure):
    _fields_ = [("max_iters", C.c_int32), ("tol", C.c_float), ("rel_tol", C.c_float)]


_P = C.c_void_p
_S = C.c_int  # zsmpm_status

# name -> (restype, argtypes); every symbol include/zsmpm.h declares
SIGNATURES = {
    "zsmpm_last_error_string": (C.c_char_p, []),
    "zsmpm_version": (C.c_char_p, []),
    "zsmpm_device_count": (C.c_int, []),
    "zsmpm_scene_create": (_S, [C.POINTER(SceneDesc), C.POINTER(_P)]),
    "zsmpm_scene_destroy": (_S, [_P]),
    "zsmpm_scene_upload": (_S, [_P, C.POINTER(ParticleArrays), C.c_int64, C.c_int32, _P]),
    "zsmpm_scene_upload_tilevector": (_S, [_P, C.POINTER(TileVectorView), C.c_int64, _P]),
    "zsmpm_scene_download": (_S, [_P, C.POINTER(ParticleArrays), C.c_int32, _P]),
    "zsmpm_scene_download_tilevector": (_S, [_P, C.POINTER(TileVectorView), _P]),
    "zsmpm_scene_num_particles": (C.c_int64, [_P]),
    "zsmpm_scene_status": (_S, [_P]),
    "zsmpm_activate_blocks": (_S, [_P, _P]),
    "zsmpm_bin_particles": (_S, [_P, _P]),
    "zsmpm_p2g": (_S, [_P, _P]),
    "zsmpm_grid_update": (_S, [_P, _P]),
    "zsmpm_g2p": (_S, [_P, _P]),
    "zsmpm_scene_set_transfer": (_S, [_P, C.c_int32, _P]),
    "zsmpm_p2c2g": (_S, [_P, C.c_int32, _P]),
    "zsmpm_g2c2p": (_S, [_P, _P]),
    "zsmpm_download_table": (_S, [_P, _P, _P, _P, _P, C.c_int32, _P, C.c_int32, _P]),
    "zsmpm_substep": (_S, [_P, _P]),
    "zsmpm_run": (_S, [_P, C.c_int32, _P]),
    "zsmpm_get_table_view": (_S, [_P, C.POINTER(TableView)]),
    "zsmpm_get_grid_view": (_S, [_P, C.POINTER(GridView)]),
    "zsmpm_num_blocks": (_S, [_P, C.POINTER(C.c_int32)]),
    "zsmpm_binning_info": (_S, [_P, C.POINTER(C.c_int32)]),
    "zsmpm_download_grid": (_S, [_P, _P, _P, C.c_int32, C.POINTER(C.c_int32)]),
    "zsmpm_download_binning": (_S, [_P, _P, _P, C.c_int32]),
    "zsmpm_set_stage_timing": (_S, [_P, C.c_int32]),
    "zsmpm_stage_times": (_S, [_P, C.POINTER(C.c_float), C.c_int32]),
    "zsmpm_kernels_per_substep": (C.c_int32, [_P]),
    "zsmpm_svd3": (_S, [_P, _P, _P, _P, C.c_int64, _P]),
    "zsmpm_constitutive": (_S, [C.POINTER(Material), _P, _P, _P, C.c_int64, _P]),
    "zsmpm_scene_set_colliders": (_S, [_P, _P, C.c_int32, _P]),
    "zsmpm_scene_add_levelset": (_S, [_P, C.POINTER(LevelSetDesc), _P]),
    "zsmpm_scene_clear_levelsets": (_S, [_P]),
    "zsmpm_g2p2g": (_S, [_P, _P, _P, C.c_int64, C.c_float, _P]),
    "zsmpm_implicit_multiply": (_S, [_P, _P, _P, C.c_int64, C.c_float, _P]),
    "zsmpm_implicit_project": (_S, [_P, _P, C.c_int64, _P]),
    "zsmpm_implicit_precondition": (_S, [_P, _P, _P, C.c_int64, _P]),
    "zsmpm_implicit_cg": (_S, [_P, _P, _P, C.c_int64, C.c_float, C.POINTER(CgOptions), C.POINTER(C.c_int32), _P]),
    "zsmpm_get_bht_view": (_S, [_P, C.POINTER(BhtView)]),
    "zsmpm_bht_build_host": (_S, [_P, C.c_int32, C.c_int32, _P, _P, _P, C.c_int32, C.POINTER(C.c_int32), _P]),
    "zsmpm_bht_build_device": (_S, [_P, C.c_int32, C.c_int32, _P, _P, _P, C.c_int32, C.POINTER(C.c_int32), _P, _P]),
    "zsmpm_batch_create": (_S, [C.POINTER(SceneDesc), C.POINTER(Material), C.c_int32, C.POINTER(_P)]),
    "zsmpm_batch_upload": (_S, [_P, C.POINTER(ParticleArrays), _P, C.c_int32, _P]),
    "zsmpm_batch_num_scenes": (_S, [_P, C.POINTER(C.c_int32)]),
    "zsmpm_autotune": (_S, [_P, C.c_int32, C.POINTER(Tuning), _P]),
    "zsmpm_set_tuning": (_S, [_P, C.POINTER(Tuning)]),
    "zsmpm_closure_create": (_S, [C.POINTER(Material), C.c_int32, C.POINTER(_P)]),
    "zsmpm_closure_destroy": (_S, [_P]),
    "zsmpm_closure_build_dataset": (_S, [_P, C.c_int64, C.c_uint64, _P, C.c_int64, _P]),
    "zsmpm_closure_train": (_S, [_P, C.c_int32, C.c_int32, C.c_float, C.c_uint64, _P, _P]),
    "zsmpm_closure_loss_grad": (_S, [_P, _P, _P, C.c_int64, _P, _P, _P]),
    "zsmpm_closure_infer": (_S, [_P, _P, _P, C.c_int64, C.c_int32, _P]),
    "zsmpm_closure_targets": (_S, [_P, _P, _P, C.c_int64, _P]),
    "zsmpm_closure_status": (_S, [_P]),
    "zsmpm_closure_get_state": (_S, [_P, C.POINTER(ClosureState)]),
    "zsmpm_closure_set_state": (_S, [_P, C.POINTER(ClosureState)]),
    "zsmpm_scene_set_closure": (_S, [_P, _P, C.c_int32]),
    "zsmpm_closure_dataset_size": (_S, [_P, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "zsmpm_scene_closure_audit": (_S, [_P, C.POINTER(ClosureAudit), C.c_int32]),
    "zsmpm_scene_set_state_log": (_S, [_P, _P, C.c_int64, C.c_int32]),
    "zsmpm_scene_state_log_count": (_S, [_P, C.POINTER(C.c_int64)]),
    "zsmpm_write_partio": (_S, [C.c_char_p, _P, C.c_int64, C.c_char_p]),
    "zsmpm_write_partio_with_stress": (_S, [C.c_char_p, _P, _P, C.c_int64]),
    "zsmpm_write_partio_with_grid": (_S, [C.c_char_p, _P, _P, C.c_int64]),
    "zsmpm_scene_write_partio": (_S, [_P, C.c_char_p]),
    "zsmpm_activate_blocks_noalloc": (_S, [_P, C.c_int64, C.c_float, _P, C.c_int32, _P, _P]),
}

_lib = None


def lib() -> C.CDLL:
    """The loaded libzsmpm.so; raises when it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: run `python zsmpm_b200/build.py` "
                               "(the CUDA path has no fallback)")
        handle = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


class ZsmpmError(RuntimeError):
    def __init__(self, status: int, where: str):
        msg = lib().zsmpm_last_error_string().decode(errors="replace")
        super().__init__(f"{where}: {STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def check(status: int, where: str) -> None:
    if status != OK:
        raise ZsmpmError(status, where)
