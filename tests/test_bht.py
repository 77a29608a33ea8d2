"""The bht<i32,3,int,16> layout (container/Bht.hpp) of block keys: the library's host builder
against the reference's own host insert (oracle/_ref/zsref_cli), slot for slot; on the GPU the
device builder against both (including tables dense enough that keys move to their second and
third buckets), and the scene's bht view against the library's block indices."""
import numpy as np
import pytest

SENT = 0x3F3F3F3F


def _ref():
    from oracle import reference
    if not reference.available():
        pytest.skip("the compiled reference (oracle/_ref) is not built")
    return reference


def _scene_keys(spec):
    """Sorted active keys of a scene, from the reference's own activation."""
    from zsmpm_b200 import scenes
    ref = _ref()
    p = scenes.generate(spec)
    keys, _, _, _ = ref.activate(p.x, spec.dx, max(p.n // 512, 64))
    order = np.lexsort((keys[:, 2], keys[:, 1], keys[:, 0]))
    return keys[order]


def _compare(ours, theirs, nkeys):
    assert ours["table_size"] == theirs["table_size"]
    assert np.array_equal(ours["hash"], theirs["hash"])
    assert np.array_equal(ours["keys"][:, :3], theirs["keys"])
    occupied = theirs["keys"][:, 0] != SENT
    assert occupied.sum() == nkeys == theirs["cnt"]
    # the reference leaves the index of an empty slot uninitialised; compare occupied slots
    assert np.array_equal(ours["indices"][occupied], theirs["indices"][occupied])
    assert np.all(ours["indices"][~occupied] == -1)
    assert np.array_equal(ours["status"], theirs["status"])
    assert np.all(ours["keys"][:, 3] == SENT)


@pytest.mark.parametrize("expected_factor", [1.0, 0.7])
def test_host_layout_bit_exact_with_reference(zs, expected_factor):
    from zsmpm_b200 import scenes
    keys = _scene_keys(scenes.small_scene(model=1, n_side=0.3))
    ref = _ref()
    expected = max(int(len(keys) * expected_factor), 16)
    theirs = ref.bht(keys, expected)
    ours = zs.bht_build_host(keys, expected)
    _compare(ours, theirs, len(keys))
    # at the denser load some keys do not fit their first bucket and go to hf1 / hf2
    if expected_factor < 1:
        tk = ours["keys"][:, :3]
        slot = {tuple(k): i for i, k in enumerate(tk.tolist()) if k[0] != SENT}
        buckets = ours["table_size"] // 16

        def h(k, a, b):
            r = None
            for c in k:
                v = ((a ^ (c & 0xFFFFFFFF)) + b) & 0xFFFFFFFF
                v %= 4294967291
                r = v if r is None else r ^ ((v + 0x9E3779B9 + (r << 6) + (r >> 2)) & 0xFFFFFFFF)
                r &= 0xFFFFFFFF
            return r
        a0, b0 = int(ours["hash"][0]), int(ours["hash"][1])
        moved = sum(1 for k, i in slot.items() if i // 16 != h(k, a0, b0) % buckets)
        assert moved > 0


def test_host_layout_edge_cases(zs):
    ref = _ref()
    for keys in (np.zeros((0, 3), np.int32), np.array([[0, 0, 0]], np.int32),
                 np.array([[-1, -2, -3], [1048575, -1048576, 7]], np.int32)):
        theirs = ref.bht(keys, 16)
        ours = zs.bht_build_host(keys, 16)
        _compare(ours, theirs, len(keys))


@pytest.mark.gpu
def test_scene_bht_view_indexes_blocks(zs, gpu):
    from helpers import d2h
    from zsmpm_b200 import scenes
    spec = scenes.small_scene(model=1, n_side=0.2)
    with zs.Scene(spec, scenes.generate(spec)) as sc:
        sc.activate_blocks()
        keys, _ = sc.download_grid()
        v = sc.bht_view()
        n = v.table_size
        tk = d2h(v.keys, (n, 4), np.int32)
        ti = d2h(v.indices, n, np.int32)
        ak = d2h(v.active_keys, (len(keys), 3), np.int32)
        cnt = d2h(v.cnt, 1, np.int32)
        ok = d2h(v.success, 1, np.int32)
    host = zs.bht_build_host(keys, max(len(keys), 16))
    assert n == host["table_size"]
    assert np.array_equal(tk, host["keys"]) and np.array_equal(ti, host["indices"])
    assert np.array_equal(ak, keys) and cnt[0] == len(keys) and ok[0] == 1
    # every active block is found at its own index
    occupied = tk[:, 0] != SENT
    found = {tuple(k): i for k, i in zip(tk[occupied, :3].tolist(), ti[occupied].tolist())}
    assert [found[tuple(k)] for k in keys.tolist()] == list(range(len(keys)))


@pytest.mark.gpu
@pytest.mark.parametrize("expected_factor", [1.0, 0.7, 0.55])
def test_device_build_bit_exact_with_reference(zs, gpu, reference_cli, expected_factor):
    from zsmpm_b200 import scenes
    keys = _scene_keys(scenes.small_scene(model=1, n_side=0.3))
    expected = max(int(len(keys) * expected_factor), 16)
    theirs = reference_cli.bht(keys, expected)
    ours = zs.bht_build_device(keys, expected)
    _compare(ours, theirs, len(keys))
    host = zs.bht_build_host(keys, expected)
    for k in ("keys", "indices", "status"):
        assert np.array_equal(ours[k], host[k])


@pytest.mark.gpu
def test_device_build_edge_cases(zs, gpu, reference_cli):
    for keys in (np.zeros((0, 3), np.int32), np.array([[0, 0, 0]], np.int32),
                 np.array([[-1, -2, -3], [1048575, -1048576, 7]], np.int32)):
        theirs = reference_cli.bht(keys, 16)
        ours = zs.bht_build_device(keys, 16)
        _compare(ours, theirs, len(keys))


@pytest.mark.gpu
def test_device_build_many_keys(zs, gpu):
    """A large random key set at the densest table the sizing rule allows (n just below a power
    of two, about 7.9 keys per 16-slot bucket): the device table equals the in-order host one."""
    rng = np.random.default_rng(5)
    n = 60000
    keys = np.unique(rng.integers(-5000, 5000, size=(2 * n, 3)).astype(np.int32), axis=0)[:n]
    keys = keys[rng.permutation(len(keys))]
    ours = zs.bht_build_device(keys, len(keys))
    host = zs.bht_build_host(keys, len(keys))
    for k in ("keys", "indices", "status"):
        assert np.array_equal(ours[k], host[k])
