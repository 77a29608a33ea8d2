"""The incremental binning against the full one, through the C ABI.

After a G2P whose particles all stayed within their block's 3x3x3 neighbourhood, the next
binning keeps the previous order of the particles that stayed in their cell and merges the
ones that left (zsmpm_binning_info reports how many).  A second zsmpm_bin_particles after the
same activation counts every particle again (the full path: SparsityOp.hpp:115-196 restated
as count / scan / scatter / sort by upload index).  The two orders must be equal slot for slot,
and equal to the oracle's stable (block, cell, upload index) order of the same positions.
"""
import numpy as np
import pytest

from test_gpu_parity import deforming

pytestmark = pytest.mark.gpu


def _order_from_positions(x, keys, dx):
    from oracle import restated
    inv = np.float32(1.0) / np.float32(dx)
    c = np.floor(x * inv + np.float32(0.5)).astype(np.int64) - 2
    b = np.floor_divide(c, 8)
    lookup = {tuple(k): i for i, k in enumerate(keys.tolist())}
    blk = np.array([lookup[tuple(k)] for k in b.tolist()], np.int32)
    lc = c - 8 * b
    cell = ((lc[:, 0] << 6) | (lc[:, 1] << 3) | lc[:, 2]).astype(np.int32)
    return restated.bin_order(blk, cell, len(keys))


@pytest.mark.parametrize("model", [0, 1])
def test_incremental_binning_equals_full_binning(zs, gpu, model):
    from zsmpm_b200 import scenes
    spec = scenes.small_scene(model=model, mode=0, n_side=0.1, velocity=(0.6, -0.9, 0.4))
    p = deforming(scenes.generate(spec), omega=(3.0, 0.0, 8.0), squeeze=5.0)
    merged_total = 0
    with zs.Scene(spec, p) as sc:
        for step in range(6):
            sc.activate_blocks()
            sc.bin_particles()
            info = sc.binning_info()
            order_inc, bstart_inc = sc.download_binning()
            sc.bin_particles()  # the same activation again: a full binning
            assert sc.binning_info() == -1
            order_full, bstart_full = sc.download_binning()
            if step == 0:
                assert info == -1  # after the upload every particle is counted
            else:
                assert info >= 0  # the movers of the last G2P merged into its order
                merged_total += info
            assert np.array_equal(bstart_inc, bstart_full)
            assert np.array_equal(order_inc, order_full)
            keys, _ = sc.download_grid()
            st = sc.download()
            o_order, o_bstart = _order_from_positions(st.x, keys, spec.dx)
            assert np.array_equal(order_inc, o_order)
            assert np.array_equal(bstart_inc, o_bstart)
            sc.p2g()
            sc.grid_update()
            sc.g2p()
        sc.status()
    assert merged_total > 0  # particles did cross cells, so the merge was exercised


def test_graph_substeps_take_the_incremental_path(zs, gpu):
    """zsmpm_run's graph: after the first substep every binning is incremental, and the run
    matches the same substeps with a full binning each time.  The order is the same, but the
    float atomics of P2G add in an order that changes from run to run, so the comparison is
    to FP32 rounding, as between two runs of the same path."""
    from helpers import rel_l2
    from zsmpm_b200 import scenes
    spec = scenes.small_scene(model=1, mode=0, n_side=0.1, velocity=(0.6, -0.9, 0.4))
    p = deforming(scenes.generate(spec), omega=(3.0, 0.0, 8.0), squeeze=5.0)
    with zs.Scene(spec, p) as sc:
        sc.run(8)
        sc.status()
        sc.activate_blocks()
        sc.bin_particles()
        assert sc.binning_info() >= 0
        a = sc.download()
    with zs.Scene(spec, p) as sc:
        for _ in range(8):
            sc.activate_blocks()
            sc.bin_particles()
            sc.bin_particles()  # full
            sc.p2g()
            sc.grid_update()
            sc.g2p()
        sc.status()
        b = sc.download()
    assert rel_l2(a.x, b.x) < 1e-6
    assert rel_l2(a.v, b.v) < 1e-5
    assert rel_l2(a.F, b.F) < 1e-5
    assert np.max(np.abs(a.plastic - b.plastic)) < 1e-5
