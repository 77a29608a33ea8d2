"""Test infrastructure: ctypes front end of the C restatement oracle (oracle/_build/liboracle.so).

The restatement follows the reference's files line by line (see oracle/oracle.h); its FP32
build is pinned bit-exactly to the compiled reference by tests/test_oracle_pin.py.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from dataclasses import dataclass
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"

FC, DP, SNOW = 0, 1, 2
MODE_COMMITTED, MODE_REFERENCE = 0, 1


class OracleParams(C.Structure):
    _fields_ = [("model", C.c_int), ("mode", C.c_int), ("wall_type", C.c_int), ("wall_cells", C.c_int),
                ("table_expected", C.c_int), ("volume_correction", C.c_int),
                ("dx", C.c_double), ("dt", C.c_double), ("gx", C.c_double), ("gy", C.c_double),
                ("gz", C.c_double), ("E", C.c_double), ("nu", C.c_double), ("volume", C.c_double),
                ("friction_deg", C.c_double), ("cohesion", C.c_double), ("beta", C.c_double),
                ("hardening", C.c_double), ("theta_c", C.c_double), ("theta_s", C.c_double),
                ("ncolliders", C.c_int), ("colliders", C.c_void_p),
                ("nlevelsets", C.c_int), ("levelsets", C.c_void_p)]


_lib = None


def build() -> None:
    subprocess.run(["bash", str(HERE / "build_oracle.sh")], check=True, capture_output=True)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        _lib = C.CDLL(str(LIB))
        P = C.c_void_p
        _lib.oracle_run_f32.argtypes = [C.POINTER(OracleParams), C.c_int] + [P] * 6 + [C.c_int, C.c_int, P, P, P]
        _lib.oracle_run_f64.argtypes = _lib.oracle_run_f32.argtypes
        _lib.oracle_svd_f32.argtypes = [P] * 4
        _lib.oracle_svd_f64.argtypes = [P] * 4
        _lib.oracle_stress_f32.argtypes = [C.POINTER(OracleParams), P, P, P]
        _lib.oracle_stress_f64.argtypes = [C.POINTER(OracleParams), P, P, P]
        _lib.oracle_activate.argtypes = [C.c_int, P, C.c_float, C.c_int, C.c_int, P, P, P, P, P]
        _lib.oracle_hash_slot.argtypes = [C.c_int32] * 4
        _lib.oracle_hash_slot.restype = C.c_int32
        _lib.oracle_bin_order.argtypes = [C.c_int, C.c_int, P, P, P, P]
        _lib.oracle_g2p2g_f32.argtypes = [C.POINTER(OracleParams), C.c_int, P, P, P, C.c_int, P, P, P]
        _lib.oracle_g2p2g_f64.argtypes = _lib.oracle_g2p2g_f32.argtypes
        _lib.oracle_run_cell_f32.argtypes = [C.POINTER(OracleParams), C.c_int] + [P] * 5 + [C.c_int, C.c_int, P, P, P]
        _lib.oracle_run_cell_f64.argtypes = _lib.oracle_run_cell_f32.argtypes
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def params_from_spec(spec, mode=None, table_expected=0) -> OracleParams:
    m = spec.material
    n_est = max(int(table_expected), 0)
    return OracleParams(model=m.model, mode=m.plasticity_mode if mode is None else mode,
                        wall_type=spec.wall_type, wall_cells=spec.wall_cells,
                        table_expected=n_est, volume_correction=m.volume_correction,
                        dx=spec.dx, dt=spec.dt, gx=spec.gravity[0], gy=spec.gravity[1],
                        gz=spec.gravity[2], E=m.E, nu=m.nu, volume=spec.volume,
                        friction_deg=m.friction_deg, cohesion=m.cohesion, beta=m.beta,
                        hardening=m.hardening, theta_c=m.theta_c, theta_s=m.theta_s)


def _abi_levelset_desc():
    """oracle_levelset has the layout of zsmpm_levelset_desc with the pointers first."""
    class OracleLevelSet(C.Structure):
        _fields_ = [("nblocks", C.c_int), ("type", C.c_int), ("background", C.c_float),
                    ("sinv", C.c_float * 9), ("rinv", C.c_float * 9), ("t", C.c_float * 3),
                    ("keys", C.c_void_p), ("sdf", C.c_void_p)]

        def __init__(self, d=None):
            super().__init__()
            if d is not None:
                self.nblocks, self.type, self.background = d.nblocks, d.type, d.background
                self.sinv[:], self.rinv[:], self.t[:] = d.sinv[:], d.rinv[:], d.t[:]
                self.keys, self.sdf = d.keys, d.sdf
    return OracleLevelSet


@dataclass
class RunResult:
    x: np.ndarray
    v: np.ndarray
    C: np.ndarray
    F: np.ndarray
    plastic: np.ndarray
    keys: np.ndarray
    grid: np.ndarray  # [nb, 4, 512] = (m, vx, vy, vz) after the walls


def run(spec, particles, nsteps: int, precision: str = "f32", mode=None, table_expected=None,
        cap_blocks: int = 1 << 16, colliders=(), levelsets=()) -> RunResult:
    """Runs the restated substep nsteps times on a copy of `particles`; `colliders` are
    zsmpm_collider records and `levelsets` LevelSet objects (zsmpm_b200.colliders), applied
    after the walls."""
    dt = np.float32 if precision == "f32" else np.float64
    n = particles.n
    if table_expected is None:
        table_expected = max(n // 512, 64)
    prm = params_from_spec(spec, mode=mode, table_expected=table_expected)
    cols = (C.c_char * (120 * max(len(colliders), 1)))()
    for i, c in enumerate(colliders):
        C.memmove(C.addressof(cols) + 120 * i, C.addressof(c), 120)
    prm.ncolliders = len(colliders)
    prm.colliders = C.addressof(cols)
    ls_cls = _abi_levelset_desc()
    descs = (ls_cls * max(len(levelsets), 1))()
    for i, L in enumerate(levelsets):
        descs[i] = ls_cls(L.desc())
    prm.nlevelsets = len(levelsets)
    prm.levelsets = C.addressof(descs)
    m = particles.m.astype(dt)
    x = particles.x.astype(dt).copy()
    v = particles.v.astype(dt).copy()
    Cm = particles.C.astype(dt).copy()
    F = particles.F.astype(dt).copy()
    pl = particles.plastic.astype(dt).copy()
    nb = C.c_int()
    keys = np.zeros((cap_blocks, 3), np.int32)
    grid = np.zeros((cap_blocks, 4, 512), dt)
    fn = lib().oracle_run_f32 if precision == "f32" else lib().oracle_run_f64
    st = fn(C.byref(prm), n, _p(m), _p(x), _p(v), _p(Cm), _p(F), _p(pl), nsteps, cap_blocks,
            C.byref(nb), _p(keys), _p(grid))
    if st != 0:
        raise RuntimeError(f"oracle_run failed with status {st}")
    return RunResult(x=x, v=v, C=Cm, F=F, plastic=pl, keys=keys[:nb.value].copy(),
                     grid=grid[:nb.value].copy())


def run_cell(spec, particles, nsteps: int, precision: str = "f32", table_expected=None,
             cap_blocks: int = 1 << 16) -> RunResult:
    """The substep with the cell-centric transfers (P2C2GTransfer / G2C2PTransfer, fixed
    corotated), restated, nsteps times on a copy of `particles`; C carries the B attribute."""
    dt = np.float32 if precision == "f32" else np.float64
    n = particles.n
    if table_expected is None:
        table_expected = max(n // 512, 64)
    prm = params_from_spec(spec, table_expected=table_expected)
    m = particles.m.astype(dt)
    x = particles.x.astype(dt).copy()
    v = particles.v.astype(dt).copy()
    Cm = particles.C.astype(dt).copy()
    F = particles.F.astype(dt).copy()
    nb = C.c_int()
    keys = np.zeros((cap_blocks, 3), np.int32)
    grid = np.zeros((cap_blocks, 4, 512), dt)
    fn = lib().oracle_run_cell_f32 if precision == "f32" else lib().oracle_run_cell_f64
    st = fn(C.byref(prm), n, _p(m), _p(x), _p(v), _p(Cm), _p(F), nsteps, cap_blocks, C.byref(nb), _p(keys),
            _p(grid))
    if st != 0:
        raise RuntimeError(f"oracle_run_cell failed with status {st}")
    return RunResult(x=x, v=v, C=Cm, F=F, plastic=particles.plastic.astype(dt).copy(),
                     keys=keys[:nb.value].copy(), grid=grid[:nb.value].copy())


def svd(A: np.ndarray, precision: str = "f32"):
    dt = np.float32 if precision == "f32" else np.float64
    A = np.ascontiguousarray(A.reshape(-1, 9), dtype=dt)
    U = np.zeros_like(A)
    V = np.zeros_like(A)
    S = np.zeros((len(A), 3), dt)
    fn = lib().oracle_svd_f32 if precision == "f32" else lib().oracle_svd_f64
    for i in range(len(A)):
        fn(_p(A[i]), _p(U[i]), _p(S[i]), _p(V[i]))
    return U, S, V


def stress(spec, F: np.ndarray, plastic: np.ndarray, precision: str = "f32", mode=None):
    """Constitutive update of a batch: returns (tau, F_projected, plastic_new)."""
    dt = np.float32 if precision == "f32" else np.float64
    prm = params_from_spec(spec, mode=mode)
    F = np.ascontiguousarray(F.reshape(-1, 9), dtype=dt).copy()
    pl = np.ascontiguousarray(plastic, dtype=dt).copy()
    tau = np.zeros_like(F)
    fn = lib().oracle_stress_f32 if precision == "f32" else lib().oracle_stress_f64
    for i in range(len(F)):
        fn(C.byref(prm), _p(F[i]), _p(pl[i:i + 1]), _p(tau[i]))
    return tau, F, pl


def activate(x: np.ndarray, dx: float, table_expected: int, cap: int = 1 << 16):
    x = np.ascontiguousarray(x, dtype=np.float32)
    nb, npb, ts = C.c_int(), C.c_int(), C.c_int()
    keys = np.zeros((cap, 3), np.int32)
    slots = np.zeros(cap, np.int32)
    st = lib().oracle_activate(len(x), _p(x), dx, table_expected, cap, C.byref(nb), C.byref(npb),
                               _p(keys), _p(slots), C.byref(ts))
    if st != 0:
        raise RuntimeError(f"oracle_activate failed with status {st}")
    return keys[:nb.value].copy(), slots[:nb.value].copy(), npb.value, ts.value


def hash_slot(k, table_size: int) -> int:
    return int(lib().oracle_hash_slot(int(k[0]), int(k[1]), int(k[2]), table_size))


def bin_order(block: np.ndarray, cell: np.ndarray, nblocks: int):
    block = np.ascontiguousarray(block, dtype=np.int32)
    cell = np.ascontiguousarray(cell, dtype=np.int32)
    order = np.zeros(len(block), np.int32)
    bstart = np.zeros(nblocks + 1, np.int32)
    lib().oracle_bin_order(len(block), nblocks, _p(block), _p(cell), _p(order), _p(bstart))
    return order, bstart


def g2p2g(spec, x, F, plastic, keys, vin, dt: float | None = None, precision: str = "f32"):
    """G2P2GTransfer restated: forces [nb*512*3] for the velocity field vin (same layout) over
    the canonical blocks `keys`."""
    t = np.float32 if precision == "f32" else np.float64
    prm = params_from_spec(spec, table_expected=max(len(keys), 64))
    if dt is not None:
        prm.dt = dt
    x = np.ascontiguousarray(x, t)
    F = np.ascontiguousarray(F, t)
    pl = np.ascontiguousarray(plastic, t)
    keys = np.ascontiguousarray(keys, np.int32)
    vin = np.ascontiguousarray(vin, t).reshape(-1)
    fout = np.zeros_like(vin)
    fn = lib().oracle_g2p2g_f32 if precision == "f32" else lib().oracle_g2p2g_f64
    st = fn(C.byref(prm), len(x), _p(x), _p(F), _p(pl), len(keys), _p(keys), _p(vin), _p(fout))
    if st != 0:
        raise RuntimeError(f"oracle_g2p2g failed with status {st}")
    return fout
