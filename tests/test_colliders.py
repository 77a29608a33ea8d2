"""Analytic colliders: Collider<AnalyticLevelSet<shape, f32, 3>> (geometry/Collider.h,
geometry/AnalyticLevelSet.h) applied after the walls in the grid update
(ApplyBoundaryConditionOnGridBlocks, simulation/grid/GridOp.hpp:113-158).

CPU: the restated oracle against the reference's own substeps with four moving colliders
(tests/golden/ref_colliders_*.npz, made by tests/golden/make_golden.py).  GPU: the CUDA path
through the C ABI against the same fixtures and against the oracle with colliders that move
between graph replays."""
import ctypes as C
import sys
from pathlib import Path

import numpy as np
import pytest

from helpers import aligned_grids, grid_mass_momentum, rel_l2

GOLDEN = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(GOLDEN))
MODELS = ("fc", "dp")


def _fixture(name):
    from zsmpm_b200 import _abi
    from zsmpm_b200.scenes import Particles
    g = np.load(GOLDEN / f"ref_colliders_{name}.npz")
    raw = g["colliders"].tobytes()
    size = C.sizeof(_abi.Collider)
    cols = [_abi.Collider.from_buffer_copy(raw[i:i + size]) for i in range(0, len(raw), size)]
    p = Particles(m=g["m"], x=g["x0"], v=g["v0"], C=g["C0"], F=g["F0"], plastic=g["plastic0"])
    return g, p, cols


def _spec(model):
    from make_golden import collider_scene
    return collider_scene(model)


def test_collider_record_layout():
    from zsmpm_b200 import _abi
    assert C.sizeof(_abi.Collider) == 120
    assert _abi.Collider.R.offset == 48 and _abi.Collider.dtdt.offset == 108


@pytest.mark.parametrize("name", MODELS)
def test_restated_colliders_bit_exact_with_reference(name):
    from oracle import restated
    g, p, cols = _fixture(name)
    assert len(cols) == 4
    spec = _spec(int(g["model"]))
    o = restated.run(spec, p, int(g["steps"]), mode=1, colliders=cols)
    for k in ("x", "v", "C", "F"):
        assert np.array_equal(getattr(o, k), g[k]), k
    assert np.array_equal(o.plastic, g["logJp"])
    assert np.array_equal(o.keys, g["keys"]) and np.array_equal(o.grid, g["grid"])
    # the colliders act: without them the velocities differ
    free = restated.run(spec, p, int(g["steps"]), mode=1)
    assert np.abs(free.v - g["v"]).max() > 0.1


def _run(zs, spec, p, plan):
    """plan: list of (colliders, nsteps); colliders are set before each group of substeps."""
    with zs.Scene(spec, p) as sc:
        for cols, n in plan:
            sc.set_colliders(cols)
            sc.run(n)
        sc.status()
        out = sc.download()
        keys, grid = sc.download_grid()
    return out, keys, grid


@pytest.mark.gpu
@pytest.mark.parametrize("name", MODELS)
def test_colliders_match_reference(zs, gpu, name):
    """Relative L2 against the reference's sequential path: the FP32 rounding of the level-set
    tests near a surface is the only source beyond that of the substep."""
    g, p, cols = _fixture(name)
    spec = _spec(int(g["model"]))
    out, keys, grid = _run(zs, spec, p, [(cols, int(g["steps"]))])
    err = {k: rel_l2(getattr(out, k), g[k]) for k in ("x", "v")}
    print(f"\ncolliders {name}: x {err['x']:.2e} v {err['v']:.2e}")
    assert err["x"] < 1e-6
    assert err["v"] < 1e-4
    ga, gb, diff = aligned_grids(keys, grid, g["keys"], g["grid"])
    assert not diff
    mg, pg = grid_mass_momentum(keys, grid)
    mb, pb = grid_mass_momentum(g["keys"], g["grid"])
    assert abs(mg - mb) / mb < 1e-6
    assert np.linalg.norm(pg - pb) / np.linalg.norm(pb) < 1e-4


@pytest.mark.gpu
def test_moving_colliders_between_graph_replays(zs, gpu):
    """A sphere that moves between replays of the two-substep graph: the device reads the
    colliders when the grid update runs, so each replay sees the latest placement."""
    from oracle import restated
    from zsmpm_b200 import colliders as col
    from zsmpm_b200.scenes import Particles
    g, p, _ = _fixture("fc")
    spec = _spec(0)
    plan = [([col.sphere((0.5, 0.47 + 0.004 * k, 0.5), 0.025, "slip", dtdt=(0.0, 0.4, 0.0))], 2) for k in range(4)]
    out, _, _ = _run(zs, spec, p, plan)
    q = p.copy()
    for cols, n in plan:
        r = restated.run(spec, q, n, mode=1, colliders=cols)
        q = Particles(m=q.m, x=r.x, v=r.v, C=r.C, F=r.F, plastic=r.plastic)
    assert rel_l2(out.x, q.x) < 1e-6
    assert rel_l2(out.v, q.v) < 1e-4
    fixed, _, _ = _run(zs, spec, p, [(plan[0][0], 8)])
    assert np.abs(fixed.v - out.v).max() > 1e-3  # the motion mattered


@pytest.mark.gpu
def test_set_colliders_rejects_bad_input(zs, gpu):
    from zsmpm_b200 import colliders as col
    g, p, cols = _fixture("fc")
    spec = _spec(0)
    with zs.Scene(spec, p) as sc:
        bad = col.sphere((0.5, 0.5, 0.5), 0.1)
        bad.shape = 9
        with pytest.raises(zs._abi.ZsmpmError):
            sc.set_colliders([bad])
        zero = col.sphere((0.5, 0.5, 0.5), 0.1, s=0.0)
        with pytest.raises(zs._abi.ZsmpmError):
            sc.set_colliders([zero])
        with pytest.raises(zs._abi.ZsmpmError):
            sc.set_colliders([col.sphere((0.5, 0.5, 0.5), 0.1)] * 17)
        sc.set_colliders(cols)
        sc.set_colliders([])
        sc.run(2)
        sc.status()


# ------------------------------------------------------------------ sparse level sets
def _levelset_fixture():
    from zsmpm_b200.colliders import LevelSet
    from zsmpm_b200.scenes import Particles
    g = np.load(GOLDEN / "ref_levelsets_fc.npz")
    ls = [LevelSet(keys=g[f"ls{i}_keys"], sdf=g[f"ls{i}_sdf"], kind=str(g[f"ls{i}_kind"]),
                   background=float(g[f"ls{i}_background"]), sinv=g[f"ls{i}_sinv"], rinv=g[f"ls{i}_rinv"],
                   t=g[f"ls{i}_t"]) for i in range(int(g["nls"]))]
    p = Particles(m=g["m"], x=g["x0"], v=g["v0"], C=g["C0"], F=g["F0"], plastic=g["plastic0"])
    return g, p, ls


def test_restated_levelsets_bit_exact_with_reference():
    """LevelSetBoundary<SparseLevelSet<3>> through the reference's own bht, grid storage and
    SparseLevelSetView sampling, against the restated trilinear sampler."""
    from oracle import restated
    g, p, ls = _levelset_fixture()
    spec = _spec(0)
    o = restated.run(spec, p, int(g["steps"]), mode=1, levelsets=ls)
    for k in ("x", "v", "C", "F"):
        assert np.array_equal(getattr(o, k), g[k]), k
    assert np.array_equal(o.grid, g["grid"])
    free = restated.run(spec, p, int(g["steps"]), mode=1)
    assert np.abs(free.v - g["v"]).max() > 0.1


@pytest.mark.gpu
def test_levelsets_match_reference(zs, gpu):
    g, p, ls = _levelset_fixture()
    spec = _spec(0)
    with zs.Scene(spec, p) as sc:
        for L in ls:
            sc.add_levelset(L)
        sc.run(int(g["steps"]))
        sc.status()
        out = sc.download()
        keys, grid = sc.download_grid()
    ex, ev = rel_l2(out.x, g["x"]), rel_l2(out.v, g["v"])
    print(f"\nlevel sets: x {ex:.2e} v {ev:.2e}")
    assert ex < 1e-6
    assert ev < 1e-4
    mg, pg = grid_mass_momentum(keys, grid)
    mb, pb = grid_mass_momentum(g["keys"], g["grid"])
    assert abs(mg - mb) / mb < 1e-6
    assert np.linalg.norm(pg - pb) / np.linalg.norm(pb) < 1e-4


@pytest.mark.gpu
def test_levelsets_add_clear_and_reject(zs, gpu):
    from zsmpm_b200.colliders import LevelSet
    g, p, ls = _levelset_fixture()
    spec = _spec(0)
    with zs.Scene(spec, p) as sc:
        bad = LevelSet(keys=ls[0].keys + 1, sdf=ls[0].sdf)
        with pytest.raises(zs._abi.ZsmpmError):
            sc.add_levelset(bad)  # keys must be block origins
        dup = LevelSet(keys=np.concatenate([ls[0].keys[:2], ls[0].keys[:1]]), sdf=ls[0].sdf[:3])
        with pytest.raises(zs._abi.ZsmpmError):
            sc.add_levelset(dup)
        for _ in range(4):
            sc.add_levelset(ls[0])
        with pytest.raises(zs._abi.ZsmpmError):
            sc.add_levelset(ls[0])  # at most four
        sc.clear_levelsets()
        sc.run(2)
        sc.status()
        cleared = sc.download()
    with zs.Scene(spec, p) as sc:
        sc.run(2)
        plain = sc.download()
    # float atomics make two runs differ in the last bits; a level set left behind would not
    assert rel_l2(cleared.v, plain.v) < 1e-6
