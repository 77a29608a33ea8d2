"""Generates the golden fixtures in tests/golden/ by running the REFERENCE's own MPM path
(oracle/_ref/zsref_cli, compiled from the zpc sources by oracle/build_ref.sh).

The reference ships no MPM tests or golden data, so these fixtures are outputs of the
reference itself on seeded synthetic inputs:
  ref_substep_fc.npz / ref_substep_dp.npz   5 substeps, sequential policy, canonical block
                                            order: inputs, particle outputs, active keys, grid
  ref_svd.npz                               math::svd_3d on 256 matrices
  ref_stress.npz                            compute_stress_fixedcorotated / _sand on 256 F
  ref_activation.npz                        ComputeSparsity + EnlargeSparsity keys and slots
  ref_colliders_fc.npz / ref_colliders_dp.npz 5 substeps with four moving analytic colliders
                                            (Collider<AnalyticLevelSet<...>>) after slip walls
  ref_levelsets_fc.npz                      5 substeps with two sparse level-set boundaries
                                            (LevelSetBoundary<SparseLevelSet<3>>), one rotated
                                            and translated
  ref_implicit_fc.npz / ref_implicit_dp.npz G2P2GTransfer, ImplicitMPMSystem's multiply /
                                            project / precondition and ConjugateGradient::solve
                                            on a small state with a smooth grid velocity field
  ref_cell_fc.npz                           5 substeps with the cell-centric transfers
                                            (P2C2GTransfer / G2C2PTransfer, fixed corotated)
                                            from a state with random B and F
Run:  python tests/golden/make_golden.py [name ...]   (no names: every fixture; a name such as
      "cell" makes only the fixtures whose file name contains it)
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))

from oracle import reference  # noqa: E402
from zsmpm_b200 import scenes  # noqa: E402


def random_F(rng, n, spread):
    q = rng.normal(size=(2, n, 4))
    q /= np.linalg.norm(q, axis=2, keepdims=True)

    def rot(q):
        w, x, y, z = q.T
        return np.stack([1 - 2 * (y * y + z * z), 2 * (x * y + w * z), 2 * (x * z - w * y),
                         2 * (x * y - w * z), 1 - 2 * (x * x + z * z), 2 * (y * z + w * x),
                         2 * (x * z + w * y), 2 * (y * z - w * x), 1 - 2 * (x * x + y * y)], 1).reshape(-1, 3, 3)
    s = np.exp(rng.uniform(-spread, spread, size=(n, 3)))
    A = rot(q[0]) @ (s[:, :, None] * np.eye(3)) @ rot(q[1])
    return np.ascontiguousarray(A.transpose(0, 2, 1).reshape(n, 9)).astype(np.float32)


def main(only=()) -> None:
    if not reference.available():
        raise SystemExit("oracle/_ref/zsref_cli is missing: run oracle/build_ref.sh first")
    if only:
        if any("cell" in o for o in only):
            make_cell(HERE / "ref_cell_fc.npz")
        return
    for model, name in ((0, "fc"), (1, "dp")):
        spec = scenes.small_scene(model=model, mode=1, velocity=(0.4, -0.3, 0.2))
        p = scenes.generate(spec)
        r = reference.run(spec, p, 5, policy=reference.POLICY_SEQ)
        assert r.status == 0
        np.savez_compressed(HERE / f"ref_substep_{name}.npz", m=p.m, x0=p.x, v0=p.v, C0=p.C, F0=p.F,
                            plastic0=p.plastic, x=r.x, v=r.v, C=r.C, F=r.F, logJp=r.logJp,
                            keys=r.keys, grid=r.grid, steps=5, model=model)
    rng = np.random.default_rng(42)
    A = np.concatenate([random_F(rng, 192, 0.5), random_F(rng, 64, 0.02)])
    U, S, V = reference.svd(A)
    np.savez_compressed(HERE / "ref_svd.npz", A=A, U=U, S=S, V=V)
    spec_dp = scenes.small_scene(model=1, mode=1)
    F = random_F(rng, 256, 0.2)
    lj = rng.uniform(-0.05, 0.05, 256).astype(np.float32)
    PF_dp, F_dp, lj_dp = reference.stress(spec_dp, F, lj)
    spec_fc = scenes.small_scene(model=0)
    PF_fc, _, _ = reference.stress(spec_fc, F, np.zeros(256, np.float32))
    np.savez_compressed(HERE / "ref_stress.npz", F=F, logJp=lj, PF_fc=PF_fc, PF_dp=PF_dp, F_dp=F_dp,
                        logJp_dp=lj_dp)
    spec = scenes.small_scene(model=0, n_side=0.25, velocity=(0, 0, 0), ppc=1, seed=3)
    p = scenes.generate(spec)
    keys, slots, npb, ts = reference.activate(p.x, spec.dx, 64)
    np.savez_compressed(HERE / "ref_activation.npz", x=p.x, dx=spec.dx, expected=64, keys=keys,
                        slots=slots, nparblocks=npb, table_size=ts)
    for model, name in ((0, "fc"), (1, "dp")):
        make_implicit(model, HERE / f"ref_implicit_{name}.npz")
        make_colliders(model, HERE / f"ref_colliders_{name}.npz")
    make_levelsets(0, HERE / "ref_levelsets_fc.npz")
    make_cell(HERE / "ref_cell_fc.npz")
    print("wrote", sorted(f.name for f in HERE.glob("*.npz")))


def velocity_field(keys: np.ndarray, dx: float) -> np.ndarray:
    """A smooth grid velocity field over the nodes of `keys`, node-major [nb*512*3]."""
    cell = np.arange(512)
    loc = np.stack([cell >> 6, (cell >> 3) & 7, cell & 7], 1)
    pos = (keys[:, None, :].astype(np.int64) * 8 + loc[None]) * dx
    v = np.stack([np.sin(7 * pos[..., 1]) + 0.3, np.cos(5 * pos[..., 2]) - 0.2,
                  np.sin(3 * pos[..., 0] + pos[..., 1])], -1)
    return v.astype(np.float32).reshape(-1)


def implicit_state(model: int, seed: int = 5):
    """A small deformed state for the implicit-system fixtures: random F, and logJp for sand."""
    spec = scenes.small_scene(model=model, mode=1, n_side=0.04)
    p = scenes.generate(spec)
    rng = np.random.default_rng(seed)
    p.F = random_F(rng, p.n, 0.15)
    p.plastic = (rng.uniform(-0.05, 0.05, p.n) if model else np.zeros(p.n)).astype(np.float32)
    return spec, p


def make_implicit(model: int, path: Path, dt: float = 1e-3, cg_iters: int = 20) -> None:
    spec, p = implicit_state(model)
    keys, _slots, _npb, _ts = reference.activate(p.x, spec.dx, max(p.n // 512, 64))
    keys = keys[np.lexsort((keys[:, 2], keys[:, 1], keys[:, 0]))]
    v = velocity_field(keys, spec.dx)
    f, _ = reference.g2p2g(spec, p.x, p.F, p.plastic, keys, v, dt=dt)
    mult, mass, _, _ = reference.implicit(spec, p, keys, v, op=reference.IMPLICIT_MULTIPLY, dt=dt)
    proj, _, _, _ = reference.implicit(spec, p, keys, v, op=reference.IMPLICIT_PROJECT, dt=dt)
    b = (np.repeat(mass.reshape(-1), 3) * v).astype(np.float32)
    prec_base = np.full_like(v, 7.0)
    prec, _, _, _ = reference.implicit(spec, p, keys, v, prec_base, op=reference.IMPLICIT_PRECONDITION, dt=dt)
    x0 = np.zeros_like(v)
    cg_x, _, iters, _ = reference.implicit(spec, p, keys, x0, b, op=reference.IMPLICIT_CG, dt=dt,
                                           max_iters=cg_iters)
    np.savez_compressed(path, model=model, dt=dt, m=p.m, x=p.x, v=p.v, C=p.C, F=p.F, plastic=p.plastic,
                        keys=keys, vel=v, f=f, mult=mult, mass=mass, proj=proj, prec_base=prec_base, prec=prec,
                        b=b, cg_x=cg_x, cg_iters=iters, cg_max_iters=cg_iters)




def collider_set():
    """One moving collider of each shape and every collision type, placed in the small scene's
    path: a translating sphere (slip), a rotating, growing box (separate), a sticky cylinder
    and a separating plane."""
    from zsmpm_b200 import colliders as col
    R = col.rotation((1, 1, 0), 0.3)
    return [col.sphere((0.52, 0.46, 0.5), 0.03, "slip", t=(0.0, 0.0, 0.001), dtdt=(0.0, 0.5, 0.0)),
            col.cuboid((-0.02, -0.01, -0.02), (0.02, 0.01, 0.02), "separate", R=R, t=(0.47, 0.52, 0.5),
                       omega=(0, 0, 3.0), s=1.2, dsdt=0.1),
            col.cylinder((0.5, 0.45, 0.53), 0.01, 0.05, 1, "sticky", dtdt=(0.1, 0, 0)),
            col.plane((0.5, 0.475, 0.5), (0.0, 1.0, 0.0), "separate")]


def collider_scene(model: int):
    return scenes.small_scene(model=model, mode=1, velocity=(0.4, -0.6, 0.2), wall_type=1)


def make_colliders(model: int, path: Path, steps: int = 5) -> None:
    spec = collider_scene(model)
    p = scenes.generate(spec)
    cols = collider_set()
    r = reference.run(spec, p, steps, policy=reference.POLICY_SEQ, colliders=cols)
    assert r.status == 0
    raw = np.frombuffer(b"".join(bytes(c) for c in cols), np.uint8)
    np.savez_compressed(path, m=p.m, x0=p.x, v0=p.v, C0=p.C, F0=p.F, plastic0=p.plastic, colliders=raw,
                        x=r.x, v=r.v, C=r.C, F=r.F, logJp=r.logJp, keys=r.keys, grid=r.grid, steps=steps,
                        model=model)


def levelset_set(spec):
    """A sphere of radius 0.025 (slip, voxel size dx) and a thin box rotated 0.4 rad about z and
    shifted by 0.01 in x (separate), sampled as sparse level sets in the small scene's path."""
    from zsmpm_b200 import colliders as col
    ball = col.LevelSet.from_function(lambda x: np.linalg.norm(x - np.array([0.51, 0.465, 0.5]), axis=1) - 0.025,
                                      (0.48, 0.435, 0.47), (0.54, 0.495, 0.53), spec.dx, "slip")

    def box(x):
        q = np.abs(x - np.array([0.5, 0.53, 0.5])) - np.array([0.03, 0.006, 0.03])
        return np.linalg.norm(np.maximum(q, 0), axis=1) + np.minimum(q.max(1), 0)

    slab = col.LevelSet.from_function(box, (0.46, 0.52, 0.46), (0.54, 0.54, 0.54), spec.dx, "separate",
                                      rinv=col.rotation((0, 0, 1), 0.4), t=(0.01, 0.0, 0.0))
    return [ball, slab]


def make_levelsets(model: int, path: Path, steps: int = 5) -> None:
    spec = collider_scene(model)
    p = scenes.generate(spec)
    ls = levelset_set(spec)
    r = reference.run(spec, p, steps, policy=reference.POLICY_SEQ, levelsets=ls)
    assert r.status == 0
    extra = {}
    for i, L in enumerate(ls):
        extra.update({f"ls{i}_keys": L.keys, f"ls{i}_sdf": L.sdf, f"ls{i}_sinv": L.sinv, f"ls{i}_rinv": L.rinv,
                      f"ls{i}_t": L.t, f"ls{i}_kind": L.kind, f"ls{i}_background": L.background})
    np.savez_compressed(path, m=p.m, x0=p.x, v0=p.v, C0=p.C, F0=p.F, plastic0=p.plastic, x=r.x, v=r.v, C=r.C,
                        F=r.F, logJp=r.logJp, keys=r.keys, grid=r.grid, steps=steps, model=model, nls=len(ls),
                        **extra)


def cell_state(seed: int = 9):
    """The small fixed-corotated scene moving at (0.4, -0.3, 0.2) with a random B (the
    cell-centric pair's affine attribute) of size 1e-3 dx and a random F near the identity."""
    spec = scenes.small_scene(model=0, mode=0, velocity=(0.4, -0.3, 0.2))
    p = scenes.generate(spec)
    rng = np.random.default_rng(seed)
    p.C = (rng.normal(size=(p.n, 9)) * 1e-3 * spec.dx).astype(np.float32)
    p.F = random_F(rng, p.n, 0.02)
    return spec, p


def make_cell(path: Path, steps: int = 5) -> None:
    spec, p = cell_state()
    r = reference.run(spec, p, steps, policy=reference.POLICY_SEQ, cell=True)
    assert r.status == 0
    np.savez_compressed(path, m=p.m, x0=p.x, v0=p.v, C0=p.C, F0=p.F, x=r.x, v=r.v, C=r.C, F=r.F, keys=r.keys,
                        grid=r.grid, steps=steps)


if __name__ == "__main__":
    main(tuple(sys.argv[1:]))
