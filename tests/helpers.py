"""Shared comparison helpers for the parity tests."""
from __future__ import annotations

import numpy as np


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    """||a - b|| / ||b|| in float64."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (den if den > 0 else 1.0))


def rel_l2_disp(x: np.ndarray, xref: np.ndarray, x0: np.ndarray) -> float:
    """Relative error of the displacement x - x0 against xref - x0."""
    return rel_l2(np.asarray(x, np.float64) - x0, np.asarray(xref, np.float64) - x0)


def grid_by_key(keys: np.ndarray, grid: np.ndarray) -> dict:
    return {tuple(int(c) for c in k): grid[i] for i, k in enumerate(keys)}


def grid_mass_momentum(keys, grid):
    """Total grid mass and momentum sum_i m_i v_i from (m, vx, vy, vz) blocks."""
    g = np.asarray(grid, np.float64)
    m = g[:, 0]
    return m.sum(), np.array([(m * g[:, 1 + d]).sum() for d in range(3)])


def aligned_grids(keys_a, grid_a, keys_b, grid_b):
    """Stacks the blocks present in both grids, ordered by key."""
    da, db = grid_by_key(keys_a, grid_a), grid_by_key(keys_b, grid_b)
    common = sorted(set(da) & set(db))
    return (np.stack([da[k] for k in common]), np.stack([db[k] for k in common]), set(da) ^ set(db))


def d2h(ptr: int, shape, dtype) -> np.ndarray:
    """Copies a device array of the library into host memory (cudaMemcpy, device->host)."""
    import ctypes
    out = np.empty(shape, dtype)
    rt = ctypes.CDLL("libcudart.so.12")
    rt.cudaMemcpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
    assert rt.cudaMemcpy(out.ctypes.data, ptr, out.nbytes, 2) == 0
    return out
