"""The cell-centric transfer pair P2C2GTransfer / G2C2PTransfer (simulation/transfer/P2C2G.hpp,
G2C2P.hpp; fixed corotated) on the GPU, through the C ABI: against the compiled reference's
sequential run (the golden fixture tests/golden/ref_cell_fc.npz), against the FP64 restatement,
and by the properties that hold at any size."""
import dataclasses
from pathlib import Path

import numpy as np
import pytest

from helpers import aligned_grids, rel_l2

GOLDEN = Path(__file__).resolve().parent / "golden"


def _fixture():
    from zsmpm_b200 import scenes
    z = np.load(GOLDEN / "ref_cell_fc.npz")
    spec = scenes.small_scene(model=0, mode=0, velocity=(0.4, -0.3, 0.2))
    n = len(z["m"])
    p = scenes.Particles(m=z["m"], x=z["x0"], v=z["v0"], C=z["C0"], F=z["F0"], plastic=np.zeros(n, np.float32))
    return spec, p, z


def _stages(sc, steps):
    for _ in range(steps):
        sc.activate_blocks()
        sc.bin_particles()
        sc.p2c2g()
        sc.grid_update()
        sc.g2c2p()


@pytest.mark.gpu
def test_cell_substeps_match_reference(zs, gpu):
    """5 substeps from a state with random B and F: x and v as close to the compiled reference
    as FP32 rounding allows; B and F - I closer to the FP64 restatement than the reference is
    (the reference forms B from absolute positions; the device from cell-relative ones)."""
    from oracle import restated
    spec, p, z = _fixture()
    steps = int(z["steps"])
    o64 = restated.run_cell(spec, p, steps, "f64")
    with zs.Scene(spec, p, transfer="cell") as sc:
        _stages(sc, steps)
        sc.status()
        g = sc.download()
        keys, grid = sc.download_grid()
    err = {"x_disp": rel_l2(g.x - p.x, z["x"] - p.x), "v": rel_l2(g.v, z["v"]),
           "C_f64": rel_l2(g.C, o64.C), "C_ref_f64": rel_l2(z["C"], o64.C),
           "F_f64": rel_l2(g.F - p.F, o64.F - p.F), "F_ref_f64": rel_l2(z["F"] - p.F, o64.F - p.F),
           "x_f64": rel_l2(g.x - p.x, o64.x - p.x), "x_ref_f64": rel_l2(z["x"] - p.x, o64.x - p.x),
           "v_f64": rel_l2(g.v, o64.v), "v_ref_f64": rel_l2(z["v"], o64.v)}
    print("\ncell pair, 5 substeps, relative L2: " + ", ".join(f"{k} {v:.2e}" for k, v in err.items()))
    assert err["v"] < 1e-5
    assert err["x_disp"] < 1e-3
    assert err["v_f64"] <= max(2 * err["v_ref_f64"], 1e-6)
    assert err["x_f64"] <= max(2 * err["x_ref_f64"], 1e-6)
    assert err["C_f64"] < 1e-3 and err["C_f64"] < err["C_ref_f64"]
    # F - I changes by dt B Dinv F per substep; its error is FP32 rounding of F (~1e-7) against
    # that change
    assert err["F_f64"] < 2e-3 and err["F_f64"] < err["F_ref_f64"]
    assert np.array_equal(keys, z["keys"])
    ga, gb, missing = aligned_grids(keys, grid, z["keys"], z["grid"])
    assert not missing
    assert rel_l2(ga[:, 0], gb[:, 0]) < 1e-6
    assert rel_l2(ga[:, 1:], gb[:, 1:]) < 1e-5


@pytest.mark.gpu
def test_cell_graph_run_matches_stages(zs, gpu):
    spec, p, _ = _fixture()
    with zs.Scene(spec, p, transfer="cell") as a, zs.Scene(spec, p, transfer="cell") as b:
        a.run(6)
        a.status()
        _stages(b, 6)
        b.status()
        ra, rb = a.download(), b.download()
    # the float atomics of P2C2G sum in another order in each run: v agrees to rounding, and B,
    # a small difference of nearly equal node velocities (the box moves rigidly), to 3e-4
    assert rel_l2(ra.x, rb.x) < 1e-7
    assert rel_l2(ra.v, rb.v) < 1e-6
    assert rel_l2(ra.C, rb.C) < 3e-4
    assert rel_l2(ra.F - p.F, rb.F - p.F) < 3e-4


@pytest.mark.gpu
def test_p2c2g_parts_add_up(zs, gpu):
    """P2C2GTransferMomentum + P2C2GTransferForce = P2C2GTransfer node by node; the force part
    leaves the mass channel untouched."""
    spec, p, _ = _fixture()
    grids = {}
    with zs.Scene(spec, p, transfer="cell") as sc:
        for part in ("momentum", "force", "all"):
            sc.activate_blocks()
            sc.bin_particles()
            sc.p2c2g(part)
            sc.status()
            grids[part] = sc.download_grid()
    km, gm = grids["momentum"]
    kf, gf = grids["force"]
    ka, ga = grids["all"]
    assert np.array_equal(km, ka) and np.array_equal(kf, ka)
    assert np.all(gf[:, 0] == 0)
    assert np.array_equal(gm[:, 0], ga[:, 0]) or rel_l2(gm[:, 0], ga[:, 0]) < 1e-7
    assert rel_l2(gm[:, 1:] + gf[:, 1:], ga[:, 1:]) < 1e-6
    # the force part is a real contribution here (the fixture's F is deformed)
    assert np.abs(gf[:, 1:]).max() > 1e-3 * np.abs(ga[:, 1:]).max()


@pytest.mark.gpu
def test_cell_p2c2g_conserves_mass_and_momentum_at_full_size(zs, gpu):
    """The two-box geometry of the benchmark at dx = 1/256 (30,089,900 particles) in fixed
    corotated with a random B and F: the node weights of a particle sum to one and its affine
    weights sum_i W_i (x_i - x_p) to zero, so the grid holds sum m and sum m v whatever B and F."""
    from zsmpm_b200 import scenes
    spec = scenes.config2()
    spec = dataclasses.replace(spec, material=scenes.MaterialSpec(model=0, E=1e4, nu=0.3, rho=1000.0),
                        wall_type=3, gravity=(0.0, 0.0, 0.0))
    p = scenes.generate(spec)
    assert p.n == 30_089_900
    rng = np.random.default_rng(4)
    p.C = (rng.standard_normal((p.n, 9), np.float32) * np.float32(0.05 * spec.dx)).astype(np.float32)
    p.F = (np.eye(3, dtype=np.float32).reshape(1, 9) +
           rng.standard_normal((p.n, 9), np.float32) * np.float32(1e-2)).astype(np.float32)
    with zs.Scene(spec, p, transfer="cell") as sc:
        sc.activate_blocks()
        sc.bin_particles()
        sc.p2c2g()
        sc.status()
        _keys, grid = sc.download_grid()
    g = grid.astype(np.float64)
    m_tot = float(p.m.astype(np.float64).sum())
    mom = (p.m[:, None].astype(np.float64) * p.v).sum(0)
    assert abs(g[:, 0].sum() / m_tot - 1) < 1e-6
    scale = float(np.abs(p.m[:, None].astype(np.float64) * p.v).sum(0).max())
    for d in range(3):
        assert abs(g[:, 1 + d].sum() - mom[d]) < 1e-5 * scale


@pytest.mark.gpu
def test_cell_transfer_refusals(zs, gpu):
    from zsmpm_b200 import closure as cl
    from zsmpm_b200 import scenes
    dp = scenes.small_scene(model=1)
    with zs.Scene(dp, scenes.generate(dp)) as sc:
        with pytest.raises(zs.ZsmpmError) as e:
            sc.set_transfer("cell")
        assert e.value.status == zs._abi.ERR_INVALID_ARG
    fc = scenes.small_scene(model=0)
    with zs.Scene(fc, scenes.generate(fc)) as sc:
        sc.activate_blocks()
        sc.bin_particles()
        with pytest.raises(zs.ZsmpmError) as e:
            sc.p2c2g()
        assert e.value.status == zs._abi.ERR_INVALID_ARG
        with pytest.raises(zs.ZsmpmError):
            sc.g2c2p()
        sc.set_transfer("cell")
        assert zs._abi.lib().zsmpm_p2c2g(sc.handle, 7, None) == zs._abi.ERR_INVALID_ARG  # not a part
    sp = scenes.small_scene(model=1)
    c = cl.Closure(sp.material, sp.volume)
    try:
        c.build_dataset(20_000, seed=1)
        with zs.Scene(fc, scenes.generate(fc), transfer="cell") as sc:
            with pytest.raises(zs.ZsmpmError) as e:
                cl.attach(sc, c)
            assert e.value.status == zs._abi.ERR_INVALID_ARG
    finally:
        c.close()
