"""The benchmark workload at full size (the two-box sand scene at dx = 1/256, 30,089,900
particles), checked through size-independent properties:

- the active block keys are sorted, unique, and exactly the particles' blocks with their
  +{0,1}^3 neighbours;
- the binned order is sorted by (block, cell, upload index), and the block starts count it;
- P2G and the grid update conserve mass and momentum (walls off);
- a run of substeps stays finite, keeps the particles inside the walls and reports no device
  error.
"""
import numpy as np
import pytest

from helpers import grid_mass_momentum

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sand():
    from zsmpm_b200 import scenes
    spec = scenes.config2()
    p = scenes.generate(spec)
    assert p.n == 30_089_900
    return spec, p


def _blocks_and_cells(x, dx):
    inv = np.float32(1.0) / np.float32(dx)
    c = np.floor(x * inv + np.float32(0.5)).astype(np.int64) - 2
    b = np.floor_divide(c, 8)
    lc = c - 8 * b
    return b, (lc[:, 0] << 6) | (lc[:, 1] << 3) | lc[:, 2]


def _key_code(k):
    k = np.asarray(k, np.int64) + (1 << 20)
    return (k[:, 0] << 42) | (k[:, 1] << 21) | k[:, 2]


def test_activation_and_binning_at_full_size(zs, gpu, sand):
    spec, p = sand
    with zs.Scene(spec, p) as sc:
        sc.activate_blocks()
        sc.bin_particles()
        sc.status()
        keys, _ = sc.download_grid()
        order, bstart = sc.download_binning()
    b, cell = _blocks_and_cells(p.x, spec.dx)
    pb = np.unique(_key_code(b))
    enlarged = np.unique(np.concatenate([_key_code(np.stack([(pb >> 42) - (1 << 20) + a, ((pb >> 21) & ((1 << 21) - 1)) - (1 << 20) + bb,
                                                             (pb & ((1 << 21) - 1)) - (1 << 20) + cc], 1))
                                         for a in (0, 1) for bb in (0, 1) for cc in (0, 1)]))
    got = _key_code(keys)
    assert np.all(np.diff(got) > 0)  # ascending (bx, by, bz), unique
    assert np.array_equal(got, enlarged)
    # binned order: (block rank, cell, upload index) non-decreasing along the slots
    rank = np.searchsorted(got, _key_code(b))
    assert np.array_equal(np.sort(order), np.arange(p.n))
    r, c = rank[order], cell[order]
    code = (r.astype(np.int64) << 41) | (c.astype(np.int64) << 32) | order.astype(np.int64)
    assert np.all(np.diff(code) > 0)
    assert bstart[0] == 0 and bstart[-1] == p.n
    assert np.array_equal(np.diff(bstart), np.bincount(rank, minlength=len(got)))


def test_substep_conserves_mass_and_momentum_at_full_size(zs, gpu, sand):
    """P2G and the grid update with the walls off: sum_i m_i = sum_p m_p and
    sum_i m_i v_i = sum_p m_p v_p + M g dt."""
    import dataclasses
    spec, p = sand
    free = dataclasses.replace(spec, wall_type=zs.WALL_NONE)
    with zs.Scene(free, p) as sc:
        sc.substep()
        sc.status()
        keys, grid = sc.download_grid()
    M, P = grid_mass_momentum(keys, grid)
    M0 = p.m.astype(np.float64).sum()
    P0 = (p.m[:, None].astype(np.float64) * p.v).sum(0) + M0 * np.array(free.gravity) * free.dt
    assert abs(M - M0) / M0 < 1e-6
    assert np.linalg.norm(P - P0) / np.linalg.norm(P0) < 1e-5


def test_run_stays_finite_and_inside_at_full_size(zs, gpu, sand):
    spec, p = sand
    with zs.Scene(spec, p) as sc:
        sc.run(20)
        sc.status()
        out = sc.download()
        # the graph's binnings merge the movers of each G2P; a full binning of the same
        # activation gives the same order
        sc.activate_blocks()
        sc.bin_particles()
        merged = sc.binning_info()
        order_inc, bstart_inc = sc.download_binning()
        sc.bin_particles()
        order_full, bstart_full = sc.download_binning()
    assert 0 < merged < p.n // 10
    assert np.array_equal(bstart_inc, bstart_full)
    assert np.array_equal(order_inc, order_full)
    assert np.all(np.isfinite(out.x)) and np.all(np.isfinite(out.v)) and np.all(np.isfinite(out.F))
    lo, hi = 2 * spec.dx, 1 - 2 * spec.dx  # slip walls 3 cells in
    assert out.x.min() > lo and out.x.max() < hi
    assert np.array_equal(out.m, p.m)
    # the second box moves at -1 m/s in x: after 20 substeps of 5e-5 s, about 1e-3
    moved = out.x[:, 0] - p.x[:, 0]
    second = p.v[:, 0] < -0.5
    assert abs(np.median(moved[second]) + 20 * spec.dt) < 2e-4
