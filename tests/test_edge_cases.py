"""Edge cases of the substep through the C ABI, against the restated oracle:

- an upload of zero particles is refused, and a scene without particles refuses to step;
- ragged particle counts (1, 31, 33 and 1,000 particles: partial warps and CTAs), with the
  keys and the binning order bit-exact and the state as close to the FP64 restatement as the
  FP32 restatement is (within 2x);
- a box straddling the origin, so that block keys and cells are negative (the floor division
  of ComputeSparsity, SparsityOp.hpp:75-77);
- hash collisions: with more blocks than home slots can hold apart, keys take the stride-127
  probe of HashTable::insert (HashTable.hpp:356-456), and every key is still found on it.
"""
import numpy as np
import pytest

from helpers import d2h, rel_l2

pytestmark = pytest.mark.gpu


def _random_particles(n, lo, hi, seed, velocity_scale=0.5):
    from zsmpm_b200.scenes import Particles
    rng = np.random.default_rng(seed)
    x = rng.uniform(lo, hi, size=(n, 3)).astype(np.float32)
    v = rng.uniform(-velocity_scale, velocity_scale, size=(n, 3)).astype(np.float32)
    m = np.full(n, 1e-3, np.float32) * rng.uniform(0.5, 1.5, size=n).astype(np.float32)
    F = np.tile(np.eye(3, dtype=np.float32).reshape(9), (n, 1))
    F += rng.uniform(-0.01, 0.01, size=(n, 9)).astype(np.float32)
    C = rng.uniform(-0.5, 0.5, size=(n, 9)).astype(np.float32)
    return Particles(m=m, x=x, v=v, C=C, F=F, plastic=np.zeros(n, np.float32))


def _gpu(zs, spec, p, steps):
    with zs.Scene(spec, p) as sc:
        sc.run(steps)
        sc.status()
        out = sc.download()
        keys, grid = sc.download_grid()
    return out, keys


def _binning(zs, spec, p):
    with zs.Scene(spec, p) as sc:
        sc.activate_blocks()
        sc.bin_particles()
        sc.status()
        keys, _ = sc.download_grid()
        order, bstart = sc.download_binning()
    return keys, order, bstart


def _oracle_binning(p, dx, keys):
    from oracle import restated
    inv = np.float32(1.0) / np.float32(dx)
    c = np.floor(p.x * inv + np.float32(0.5)).astype(np.int64) - 2
    b = np.floor_divide(c, 8)
    lookup = {tuple(k): i for i, k in enumerate(keys.tolist())}
    blk = np.array([lookup[tuple(k)] for k in b.tolist()], np.int32)
    lc = c - 8 * b
    cell = ((lc[:, 0] << 6) | (lc[:, 1] << 3) | lc[:, 2]).astype(np.int32)
    return restated.bin_order(blk, cell, len(keys))


def _check_state(zs, spec, p, steps):
    """Keys bit-exact; displacement, v and F within 2x of the FP32 restatement's own distance to
    the FP64 restatement (random placements leave grid nodes of tiny mass, where v = p/m
    amplifies rounding), and within 1e-4 of the FP32 restatement."""
    from oracle import restated
    g, gk = _gpu(zs, spec, p, steps)
    o32 = restated.run(spec, p, steps, "f32", mode=0)
    o64 = restated.run(spec, p, steps, "f64", mode=0)
    assert np.array_equal(gk, o32.keys[np.lexsort((o32.keys[:, 2], o32.keys[:, 1], o32.keys[:, 0]))])
    pairs = {"x": (g.x - p.x, o32.x - p.x, o64.x - p.x), "v": (g.v, o32.v, o64.v), "F": (g.F, o32.F, o64.F)}
    for k, (a, b, c) in pairs.items():
        assert rel_l2(a, c) <= max(2 * rel_l2(b, c), 1e-6), k
        assert rel_l2(a, b) < 1e-4, k


def test_zero_particles_refused(zs, gpu):
    from zsmpm_b200 import scenes
    spec = scenes.small_scene(model=0)
    empty = _random_particles(0, 0.45, 0.55, 1)
    with zs.Scene(spec) as sc:
        with pytest.raises(zs.ZsmpmError) as e:
            sc.upload(empty)
        assert e.value.status == zs._abi.ERR_INVALID_ARG
        with pytest.raises(zs.ZsmpmError) as e:
            sc.substep()
        assert e.value.status == zs._abi.ERR_NOT_READY
        # the scene stays usable
        sc.upload(_random_particles(64, 0.45, 0.55, 2))
        sc.run(2)
        sc.status()


@pytest.mark.parametrize("n", [1, 31, 33, 1000])
@pytest.mark.parametrize("model", [0, 1])
def test_ragged_counts_match_oracle(zs, gpu, n, model):
    from zsmpm_b200 import scenes
    spec = scenes.small_scene(model=model, mode=0)
    p = _random_particles(n, 0.44, 0.56, 10 + n)
    keys, order, bstart = _binning(zs, spec, p)
    o_order, o_bstart = _oracle_binning(p, spec.dx, keys)
    assert np.array_equal(order, o_order) and np.array_equal(bstart, o_bstart)
    _check_state(zs, spec, p, 3)


def test_negative_keys_match_oracle(zs, gpu):
    """A box around (0, 0.02, -0.03) without walls: cells and blocks below zero."""
    from zsmpm_b200 import scenes
    spec = scenes.small_scene(model=1, mode=0, center=(0.0, 0.02, -0.03), wall_type=zs.WALL_NONE,
                              velocity=(0.4, -0.6, 0.2))
    p = scenes.generate(spec)
    keys, order, bstart = _binning(zs, spec, p)
    assert (keys < 0).any(axis=0).all()  # negative coordinates on every axis
    o_order, o_bstart = _oracle_binning(p, spec.dx, keys)
    assert np.array_equal(order, o_order) and np.array_equal(bstart, o_bstart)
    _check_state(zs, spec, p, 5)


def test_hash_collisions_take_the_probe(zs, gpu):
    """1,000 particles spread over [0.3, 0.7]^3 make about 500 blocks in the reference's
    next_2pow(64) * 16 = 1,024 slots: many keys share a home slot.  Where a colliding key lands
    depends on the order of the inserts, so the check is the probe invariant a query relies on:
    every slot before a key on its probe sequence is occupied."""
    from oracle import restated
    from zsmpm_b200 import scenes
    spec = scenes.small_scene(model=0)
    p = _random_particles(1000, 0.3, 0.7, 99)
    with zs.Scene(spec, p) as sc:
        sc.activate_blocks()
        sc.status()
        nb = sc.num_blocks()
        keys, _ = sc.download_grid()
        tv = sc.table_view()
        T = tv.table_size
        kh = d2h(tv.keys, (T, 3), np.int32)
        ih = d2h(tv.indices, T, np.int32)
    okeys, _, _, ts = restated.activate(p.x, spec.dx, max(p.n // 512, 64))
    assert T == ts == 1024
    assert np.array_equal(keys, okeys[np.lexsort((okeys[:, 2], okeys[:, 1], okeys[:, 0]))])
    occupied = np.nonzero(ih >= 0)[0]
    assert len(occupied) == nb > 300
    homes = np.array([restated.hash_slot(kh[slot], T) for slot in occupied])
    assert len(np.unique(homes)) < len(homes)  # collisions
    inv127 = pow(127, -1, T)
    probed = 0
    for slot, home in zip(occupied.tolist(), homes.tolist()):
        k = ((slot - home) * inv127) % T
        probed += k > 0
        for j in range(k):
            assert ih[(home + 127 * j) % T] >= 0
        # the table index is the key's rank in ascending (bx, by, bz) order
        assert tuple(keys[ih[slot]]) == tuple(kh[slot])
    assert probed > 10


def _activation_keys_after(zs, spec, p, steps):
    """Runs `steps` substeps, then one activation; returns its keys and the particles' positions."""
    with zs.Scene(spec, p) as sc:
        sc.run(steps)
        x = sc.download().x
        sc.activate_blocks()
        sc.status()
        keys, _ = sc.download_grid()
    return keys, x


def _oracle_keys(x, dx):
    from oracle import restated
    okeys, _, _, _ = restated.activate(x, dx, max(len(x) // 512, 64))
    return okeys[np.lexsort((okeys[:, 2], okeys[:, 1], okeys[:, 0]))]


def test_activation_from_moved_blocks_matches_oracle(zs, gpu):
    """After a G2P the activation inserts the blocks recorded per block of the last binning
    (k_insert_moved_blocks); the keys equal those of the particles' stored positions."""
    from zsmpm_b200 import scenes
    spec = scenes.small_scene(model=1, mode=0, n_side=0.2, velocity=(3.0, -2.0, 1.5))
    p = scenes.generate(spec)
    for steps in (1, 7):
        keys, x = _activation_keys_after(zs, spec, p, steps)
        assert np.array_equal(keys, _oracle_keys(x, spec.dx)), steps


def test_activation_after_a_far_move_matches_oracle(zs, gpu):
    """A particle that crosses more than one block in a substep (|v| dt > 8 dx) sends the next
    activation back to the particle pass."""
    from zsmpm_b200 import scenes
    spec = scenes.small_scene(model=0, mode=0)
    p = scenes.generate(spec)
    lone = _random_particles(1, 0.30, 0.30, 5, velocity_scale=0.0)
    lone.x[:] = (0.2, 0.5, 0.5)
    lone.v[:] = (1500.0, 0.0, 0.0)  # 0.15 per substep at dt = 1e-4: 19 cells
    from zsmpm_b200.scenes import Particles
    both = Particles(*(np.concatenate([a, b]) for a, b in zip(
        (p.m, p.x, p.v, p.C, p.F, p.plastic), (lone.m, lone.x, lone.v, lone.C, lone.F, lone.plastic))))
    keys, x = _activation_keys_after(zs, spec, both, 1)
    assert x[-1, 0] > 0.3  # it crossed blocks
    assert np.array_equal(keys, _oracle_keys(x, spec.dx))


def test_position_that_becomes_nan_is_reported_after_moved_blocks(zs, gpu):
    """A NaN velocity turns positions NaN in the first G2P; that G2P cannot record their blocks,
    so the next activation reads every particle and reports them out of domain."""
    from zsmpm_b200 import scenes
    spec = scenes.small_scene(model=0)
    p = scenes.generate(spec)
    p.v[7] = np.nan
    with zs.Scene(spec, p) as sc:
        sc.substep()
        sc.status()  # the upload's positions are finite
        sc.substep()
        with pytest.raises(zs.ZsmpmError) as e:
            sc.status()
        assert e.value.status == zs._abi.ERR_OUT_OF_DOMAIN


def test_run_zero_captures_without_stepping(zs, gpu):
    """zsmpm_run with nsteps = 0 captures the substep graph and leaves the state as it was; the
    graph of four substeps plus a direct one (run(5)) then gives the state of five single
    substeps, up to the order of P2G's float sums."""
    from zsmpm_b200 import scenes
    spec = scenes.small_scene(model=1)
    p = zs.generate(spec)
    with zs.Scene(spec, p) as a, zs.Scene(spec, p) as b:
        before = a.download()
        a.run(0)
        a.status()
        same = a.download()
        for k in ("x", "v", "C", "F", "plastic"):
            assert np.array_equal(getattr(before, k), getattr(same, k)), k
        a.run(5)
        a.status()
        for _ in range(5):
            b.substep()
        b.status()
        ga, gb = a.download(), b.download()
    assert rel_l2(ga.x - p.x, gb.x - p.x) < 1e-5
    assert rel_l2(ga.v, gb.v) < 1e-5
    assert rel_l2(ga.F, gb.F) < 1e-5
