"""Test infrastructure: runs the reference's own MPM path (oracle/_ref/zsref_cli, compiled from
the zpc sources by oracle/build_ref.sh) in a subprocess, exchanging raw little-endian files.

The reference's host runtime is run in its own process.  Loaded into a Python process, it
intermittently blocked on a futex before its first operator launch.  The cause is in the
reference: zs::MemoryBackendRegistry is allocated with `new` and its zs::Mutex member has no
initializer, so the first lock waits forever when the heap word under it is nonzero
(oracle/ref_shims/zeroed_new.hpp, which the CLI now links, gives it zeroed memory).  Every call
has a timeout and is retried once.
"""
from __future__ import annotations

import os
import struct
import subprocess
import tempfile
from dataclasses import dataclass
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
CLI = HERE / "_ref" / "zsref_cli"

POLICY_SEQ, POLICY_OMP = 0, 1


def available() -> bool:
    return CLI.exists()


def _run(request: bytes, timeout: float) -> bytes:
    if not CLI.exists():
        raise FileNotFoundError(f"{CLI} not built (oracle/build_ref.sh needs the reference sources)")
    last = None
    for _attempt in range(2):
        with tempfile.TemporaryDirectory() as td:
            req = os.path.join(td, "req.bin")
            rep = os.path.join(td, "rep.bin")
            with open(req, "wb") as f:
                f.write(request)
            try:
                r = subprocess.run([str(CLI), req, rep], capture_output=True, timeout=timeout)
            except subprocess.TimeoutExpired as e:
                last = e
                continue
            if r.returncode != 0:
                raise RuntimeError(f"zsref_cli failed: {r.stderr.decode(errors='replace')}")
            with open(rep, "rb") as f:
                return f.read()
    raise RuntimeError(f"zsref_cli timed out twice: {last}")


def _params_bytes(spec, policy: int, threads: int, order: int, table_expected: int) -> bytes:
    m = spec.material
    ints = [m.model, policy, threads, order, spec.wall_type, spec.wall_cells, table_expected,
            m.volume_correction]
    floats = [spec.dx, spec.dt, *spec.gravity, m.E, m.nu, spec.volume, m.friction_deg, m.cohesion,
              m.beta]
    return struct.pack("<8i11f", *ints, *floats)


@dataclass
class RefResult:
    status: int
    seconds: float
    x: np.ndarray
    v: np.ndarray
    C: np.ndarray
    F: np.ndarray
    logJp: np.ndarray
    keys: np.ndarray
    grid: np.ndarray


def run(spec, particles, nsteps: int, policy: int = POLICY_SEQ, threads: int = 0, order: int = 1,
        table_expected: int | None = None, cap_blocks: int = 1 << 15,
        timeout: float = 600.0, colliders=(), levelsets=(), cell: bool = False) -> RefResult:
    """`colliders`: zsmpm_collider records (ctypes), applied after the walls by the reference's
    own Collider<AnalyticLevelSet<...>> launches; `levelsets`: LevelSet objects
    (zsmpm_b200.colliders), applied after them as LevelSetBoundary<SparseLevelSet<3>>.
    `cell`: the substep transfers with P2C2GTransfer / G2C2PTransfer instead of P2G / G2P
    (fixed corotated; C carries the pair's B attribute)."""
    n = particles.n
    if table_expected is None:
        table_expected = max(n // 512, 64)
    if cell and (colliders or levelsets):
        raise ValueError("the cell-centric run takes the walls only")
    cmd = 10 if cell else (9 if levelsets else (8 if colliders else 1))
    req = struct.pack("<i", cmd) + _params_bytes(spec, policy, threads, order, table_expected)
    req += struct.pack("<3i", n, nsteps, cap_blocks)
    for a in (particles.m, particles.x, particles.v, particles.C, particles.F, particles.plastic):
        req += np.ascontiguousarray(a, dtype="<f4").tobytes()
    if cmd in (8, 9):
        req += struct.pack("<i", len(colliders)) + b"".join(bytes(c) for c in colliders)
    if cmd == 9:
        from zsmpm_b200.colliders import TYPES
        req += struct.pack("<i", len(levelsets))
        for L in levelsets:
            keys = np.ascontiguousarray(L.keys, dtype="<i4").reshape(-1, 3)
            kind = TYPES[L.kind] if isinstance(L.kind, str) else int(L.kind)
            req += struct.pack("<iif", len(keys), kind, float(L.background))
            for m in (L.sinv, L.rinv, L.t):
                req += np.ascontiguousarray(m, dtype="<f4").reshape(-1).tobytes()
            req += keys.tobytes() + np.ascontiguousarray(L.sdf, dtype="<f4").reshape(-1).tobytes()
    rep = _run(req, timeout)
    status, nb = struct.unpack_from("<2i", rep, 0)
    secs = struct.unpack_from("<d", rep, 8)[0]
    off = 16
    out = []
    for cnt, shape in ((3 * n, (n, 3)), (3 * n, (n, 3)), (9 * n, (n, 9)), (9 * n, (n, 9)), (n, (n,))):
        out.append(np.frombuffer(rep, "<f4", cnt, off).reshape(shape).copy())
        off += 4 * cnt
    keys = np.zeros((0, 3), np.int32)
    grid = np.zeros((0, 4, 512), np.float32)
    if status == 0 and cap_blocks:
        keys = np.frombuffer(rep, "<i4", 3 * nb, off).reshape(nb, 3).copy()
        off += 12 * nb
        grid = np.frombuffer(rep, "<f4", nb * 2048, off).reshape(nb, 4, 512).copy()
    return RefResult(status, secs, *out, keys, grid)


def activate(x: np.ndarray, dx: float, table_expected: int, cap: int = 1 << 16, timeout: float = 120.0):
    x = np.ascontiguousarray(x, dtype="<f4")
    req = struct.pack("<iifii", 2, len(x), dx, table_expected, cap) + x.tobytes()
    rep = _run(req, timeout)
    st, nb, npb, ts = struct.unpack_from("<4i", rep, 0)
    if st != 0:
        raise RuntimeError(f"zsref activate failed: {st}")
    keys = np.frombuffer(rep, "<i4", 3 * nb, 16).reshape(nb, 3).copy()
    slots = np.frombuffer(rep, "<i4", nb, 16 + 12 * nb).copy()
    return keys, slots, npb, ts


def bht(keys: np.ndarray, expected: int, cap_slots: int = 1 << 20, timeout: float = 120.0) -> dict:
    """The reference's bht<i32,3,int,16> (container/Bht.hpp) after its host insert of `keys` in
    order: table size, hasher parameters, and per slot key, index and status."""
    keys = np.ascontiguousarray(keys, dtype="<i4").reshape(-1, 3)
    req = struct.pack("<iiii", 5, len(keys), expected, cap_slots) + keys.tobytes()
    rep = _run(req, timeout)
    st, ts = struct.unpack_from("<2i", rep, 0)
    hash6 = np.frombuffer(rep, "<u4", 6, 8).copy()
    cnt = struct.unpack_from("<i", rep, 32)[0]
    if st != 0:
        raise RuntimeError(f"zsref bht failed: {st}")
    off = 36
    tkeys = np.frombuffer(rep, "<i4", 3 * ts, off).reshape(ts, 3).copy()
    off += 12 * ts
    idx = np.frombuffer(rep, "<i4", ts, off).copy()
    off += 4 * ts
    status = np.frombuffer(rep, "<i4", ts, off).copy()
    return {"table_size": ts, "hash": hash6, "cnt": cnt, "keys": tkeys, "indices": idx, "status": status}


def stress(spec, F: np.ndarray, logJp: np.ndarray, timeout: float = 120.0):
    """Reference compute_stress_* on a batch: returns (PF, F_projected, logJp_new)."""
    m = spec.material
    F = np.ascontiguousarray(F.reshape(-1, 9), dtype="<f4")
    cnt = len(F)
    req = struct.pack("<iii6fi", 3, cnt, m.model, spec.volume, m.E, m.nu, m.friction_deg, m.cohesion,
                      m.beta, m.volume_correction)
    req += F.tobytes() + np.ascontiguousarray(logJp, dtype="<f4").tobytes()
    rep = _run(req, timeout)
    PF = np.frombuffer(rep, "<f4", 9 * cnt, 0).reshape(cnt, 9).copy()
    Fo = np.frombuffer(rep, "<f4", 9 * cnt, 36 * cnt).reshape(cnt, 9).copy()
    lj = np.frombuffer(rep, "<f4", cnt, 72 * cnt).copy()
    return PF, Fo, lj


def svd(A: np.ndarray, timeout: float = 120.0):
    A = np.ascontiguousarray(A.reshape(-1, 9), dtype="<f4")
    cnt = len(A)
    rep = _run(struct.pack("<ii", 4, cnt) + A.tobytes(), timeout)
    U = np.frombuffer(rep, "<f4", 9 * cnt, 0).reshape(cnt, 9).copy()
    S = np.frombuffer(rep, "<f4", 3 * cnt, 36 * cnt).reshape(cnt, 3).copy()
    V = np.frombuffer(rep, "<f4", 9 * cnt, 48 * cnt).reshape(cnt, 9).copy()
    return U, S, V


def g2p2g(spec, x, F, logJp, keys, vin, dt: float | None = None, policy: int = POLICY_SEQ,
          threads: int = 0, timeout: float = 600.0):
    """The reference's G2P2GTransfer (simulation/transfer/G2P2G.hpp) on the given state and
    velocity field vin ([nb*512*3], node-major over the canonical blocks `keys`): returns
    (forces, seconds)."""
    import copy
    keys = np.ascontiguousarray(keys, dtype="<i4").reshape(-1, 3)
    nb = len(keys)
    n = len(x)
    sp = spec
    if dt is not None:
        sp = copy.copy(spec)
        sp.dt = dt
    req = struct.pack("<i", 6) + _params_bytes(sp, policy, threads, 1, max(n // 512, 64))
    req += struct.pack("<2i", n, nb)
    for a in (x, F, logJp):
        req += np.ascontiguousarray(a, dtype="<f4").tobytes()
    req += keys.tobytes() + np.ascontiguousarray(vin, dtype="<f4").reshape(-1).tobytes()
    rep = _run(req, timeout)
    st = struct.unpack_from("<i", rep, 0)[0]
    secs = struct.unpack_from("<d", rep, 4)[0]
    if st != 0:
        raise RuntimeError(f"zsref g2p2g failed: {st}")
    return np.frombuffer(rep, "<f4", 1536 * nb, 12).copy(), secs


IMPLICIT_MULTIPLY, IMPLICIT_PROJECT, IMPLICIT_PRECONDITION, IMPLICIT_CG = 0, 1, 2, 3


def implicit(spec, particles, keys, a, b=None, op: int = IMPLICIT_MULTIPLY, dt: float | None = None,
             max_iters: int = 1000, tol: float = 1e-6, rel_tol: float = 0.5, timeout: float = 600.0):
    """The reference's implicit system (simulation/mpm/ImplicitMPM.hpp) and its
    ConjugateGradient (math/linear/ConjugateGradient.hpp) on a particle state, after its
    activation and a P2GTransfer for the grid mass.  Returns (out, mass [nb, 512], iters, seconds)."""
    import copy
    keys = np.ascontiguousarray(keys, dtype="<i4").reshape(-1, 3)
    nb = len(keys)
    n = particles.n
    sp = spec
    if dt is not None:
        sp = copy.copy(spec)
        sp.dt = dt
    if b is None:
        b = np.zeros(1536 * nb, np.float32)
    req = struct.pack("<i", 7) + _params_bytes(sp, POLICY_SEQ, 0, 1, max(n // 512, 64))
    req += struct.pack("<4i2f", op, n, nb, max_iters, tol, rel_tol)
    for arr in (particles.m, particles.x, particles.v, particles.C, particles.F, particles.plastic):
        req += np.ascontiguousarray(arr, dtype="<f4").tobytes()
    req += keys.tobytes()
    req += np.ascontiguousarray(a, dtype="<f4").reshape(-1).tobytes()
    req += np.ascontiguousarray(b, dtype="<f4").reshape(-1).tobytes()
    rep = _run(req, timeout)
    st, iters = struct.unpack_from("<2i", rep, 0)
    secs = struct.unpack_from("<d", rep, 8)[0]
    if st != 0:
        raise RuntimeError(f"zsref implicit failed: {st}")
    out = np.frombuffer(rep, "<f4", 1536 * nb, 16).copy()
    mass = np.frombuffer(rep, "<f4", 512 * nb, 16 + 4 * 1536 * nb).reshape(nb, 512).copy()
    return out, mass, iters, secs
